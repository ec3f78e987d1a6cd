// ADC tables: query-independent (pre_compute1) and per-query (pre_compute2).
//
// The exact form reproduces the reference's float arithmetic: every dot
// product is a sequential loop in which each multiply and each add rounds on
// its own (__fmul_rn / __fadd_rn, so nothing is contracted into an FMA), in
// the reference's order.  Entries are therefore bit-identical to
// PQQuery::pre_compute1 / pre_compute2 (query.h:91-184) with BLAS sdot taken
// as the sequential loop.
#include "scg_internal.cuh"

namespace scg {

namespace {

__device__ __forceinline__ float seq_dot(const float *x, const float *y, int n) {
    float d = 0.0f;
    for (int k = 0; k < n; k++) d = __fadd_rn(d, __fmul_rn(x[k], y[k]));
    return d;
}

// norm_c (query.h:105-114) and norm_r (query.h:116-125): one thread per centroid.
__global__ void k_norms(const float *__restrict__ C, int rows, int len, float *__restrict__ out) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= rows) return;
    const float *c = C + (size_t)i * len;
    float d = 0.0f;
    for (int k = 0; k < len; k++) {
        float t = c[k];
        d = __fadd_rn(d, __fmul_rn(t, t));
    }
    out[i] = d;
}

// dot_cr[((i*kc + j)*(mp/mc) + i1)*kp + j1] = 2 * <cq[i][j] chunk i1, pq[i*(mp/mc)+i1][j1]>
// (query.h:127-147): one thread per entry.
__global__ void k_dot_cr(const float *__restrict__ cq, const float *__restrict__ pq, int mc, int kc,
                         int mp, int kp, int bsc, int bsp, float *__restrict__ dot_cr) {
    size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    size_t total = (size_t)kc * kp * mp;
    if (e >= total) return;
    int per = mp / mc;
    int j1 = (int)(e % kp);
    size_t t = e / kp;
    int i1 = (int)(t % per);
    t /= per;
    int j = (int)(t % kc);
    int i = (int)(t / kc);
    const float *c = cq + ((size_t)i * kc + j) * bsc + (size_t)i1 * bsp;
    const float *r = pq + (((size_t)i * per + i1) * kp + j1) * bsp;
    dot_cr[e] = __fmul_rn(2.0f, seq_dot(c, r, bsp));
}

constexpr int QT = 16;    // queries per block
constexpr int ET = 128;   // table entries per block (one per thread)
constexpr int KCH = 32;   // dimensions staged per step

// Per-query tables (query.h:154-184, intended sequencing):
//   dqc[q][i*kc + j] = (norm_c[i*kc+j] - d) - d,  d = sum_t q[i*bsc+t] * cq[i][j][t]
//   dqr[q][k*kp + j] = (norm_r[k*kp+j] - d) - d,  d = sum_t q[k*bsp+t] * pq[k][j][t]
// Blocks cover (segment tile, query tile); a segment is one coarse part or one
// PQ subspace.  Each thread owns one table entry and keeps QT sequential
// accumulators; dimensions are staged through shared memory in chunks.
__global__ void __launch_bounds__(ET) k_tables_exact(TablesArgs a, int ctiles, int ptiles) {
    __shared__ float qs[QT][KCH];
    __shared__ float cs[KCH][ET + 1];
    int tile = blockIdx.x;
    int seg, e0, seglen, len, qoff;
    const float *cent;
    const float *norm;
    float *out;
    int outstride, outoff;
    if (tile < a.mc * ctiles) {
        seg = tile / ctiles;
        e0 = (tile % ctiles) * ET;
        seglen = a.kc;
        len = a.dim / a.mc;
        qoff = seg * len;
        cent = a.cq + (size_t)seg * a.kc * len;
        norm = a.norm_c + (size_t)seg * a.kc;
        out = a.dqc;
        outstride = a.mc * a.kc;
        outoff = seg * a.kc;
    } else {
        tile -= a.mc * ctiles;
        seg = tile / ptiles;
        e0 = (tile % ptiles) * ET;
        seglen = a.kp;
        len = a.dim / a.mp;
        qoff = seg * len;
        cent = a.pq + (size_t)seg * a.kp * len;
        norm = a.norm_r + (size_t)seg * a.kp;
        out = a.dqr;
        outstride = a.mp * a.kp;
        outoff = seg * a.kp;
    }
    int q0 = blockIdx.y * QT;
    int t = threadIdx.x;
    int e = e0 + t;
    float acc[QT];
#pragma unroll
    for (int i = 0; i < QT; i++) acc[i] = 0.0f;
    for (int k0 = 0; k0 < len; k0 += KCH) {
        int kn = min(KCH, len - k0);
        for (int i = t; i < QT * KCH; i += ET) {
            int qq = i / KCH, kk = i % KCH;
            int q = q0 + qq;
            qs[qq][kk] = (q < a.nq && kk < kn) ? a.Q[(size_t)q * a.dim + qoff + k0 + kk] : 0.0f;
        }
        for (int i = t; i < ET * KCH; i += ET) {
            int ee = i / KCH, kk = i % KCH;
            int eg = e0 + ee;
            cs[kk][ee] = (eg < seglen && kk < kn) ? cent[(size_t)eg * len + k0 + kk] : 0.0f;
        }
        __syncthreads();
        for (int kk = 0; kk < kn; kk++) {
            float c = cs[kk][t];
#pragma unroll
            for (int i = 0; i < QT; i++) acc[i] = __fadd_rn(acc[i], __fmul_rn(qs[i][kk], c));
        }
        __syncthreads();
    }
    if (e < seglen) {
        // the fast form keeps ||r||^2 in the per-vector term: its LUT is -2<q,r>
        const bool lut_only = a.lut_only && out == a.dqr;
        float nv = lut_only ? 0.0f : norm[e];
#pragma unroll
        for (int i = 0; i < QT; i++) {
            int q = q0 + i;
            if (q < a.nq) out[(size_t)q * outstride + outoff + e] = __fsub_rn(__fsub_rn(nv, acc[i]), acc[i]);
        }
    }
}

// Query norms: per coarse part (multi_query.h:102-112) and the total the
// ADC uses (q_sum: the sum of the part norms for IMI, the sequential sum over
// all dimensions for IVFADC / SC, query.h:223-228, sc_query.h:91-96).
__global__ void k_query_norms(const float *__restrict__ Q, int nq, int dim, int mc,
                              float *__restrict__ qn, float *__restrict__ qsum) {
    int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= nq) return;
    const float *x = Q + (size_t)q * dim;
    int bsc = dim / mc;
    float n[2] = {0.0f, 0.0f};
    for (int i = 0; i < mc && i < 2; i++) {
        float d = 0.0f;
        for (int j = 0; j < bsc; j++) {
            float t = x[i * bsc + j];
            d = __fadd_rn(d, __fmul_rn(t, t));
        }
        n[i] = d;
    }
    qn[2 * q] = n[0];
    qn[2 * q + 1] = n[1];
    qsum[q] = (mc == 2) ? __fadd_rn(__fadd_rn(0.0f, n[0]), n[1]) : n[0];
}

// The same norms with the rows staged in shared memory: a block copies qb
// query rows with coalesced loads (row stride dim + 1 words, so threads
// summing neighbouring rows read different banks), then thread (row, part)
// adds its part in the order above.  One thread per query reading its own
// row straight from global memory touched a different 512-byte row per lane
// and left most SMs idle at 10,000 queries.
constexpr int QN_THREADS = 256;
constexpr int QN_MAX_ROWS = 64;
constexpr int QN_SMEM_WORDS = 12288;  // 48 KB: no opt-in needed

__global__ void __launch_bounds__(QN_THREADS) k_query_norms_staged(const float *__restrict__ Q, int nq, int dim,
                                                                   int mc, int qb, float *__restrict__ qn,
                                                                   float *__restrict__ qsum) {
    extern __shared__ float rows[];
    __shared__ float part_sum[QN_MAX_ROWS][2];
    const int q0 = blockIdx.x * qb;
    const int nr = min(qb, nq - q0);
    const int ld = dim + 1;
    const float *src = Q + (size_t)q0 * dim;
    for (int i = threadIdx.x; i < nr * dim; i += QN_THREADS) {
        const int r = i / dim;
        rows[r * ld + (i - r * dim)] = __ldg(src + i);
    }
    __syncthreads();
    const int parts = mc < 2 ? 1 : 2;
    const int bsc = dim / mc;
    const int t = threadIdx.x;
    if (t < nr * parts) {
        const int r = t / parts, i = t - r * parts;
        const float *x = rows + r * ld + i * bsc;
        float d = 0.0f;
        for (int j = 0; j < bsc; j++) d = __fadd_rn(d, __fmul_rn(x[j], x[j]));
        part_sum[r][i] = d;
    }
    __syncthreads();
    if (t < nr) {
        const float n0 = part_sum[t][0], n1 = parts == 2 ? part_sum[t][1] : 0.0f;
        const int q = q0 + t;
        qn[2 * q] = n0;
        qn[2 * q + 1] = n1;
        qsum[q] = (mc == 2) ? __fadd_rn(__fadd_rn(0.0f, n0), n1) : n0;
    }
}

// Per-vector term of the fast ADC form, in CSR order:
//   vterm[p] = sum_k ( ||r_k(c_k)||^2 + 2<c_part(k), r_k(c_k)> )
// so that ||q - c - r||^2 = q_sum + dqc(cell) + vterm + sum_k (-2<q_k, r_k>).
__global__ void k_vterm(int mode, int kc, int mp, int kp, int mc, uint64_t ncells, int64_t N,
                        const uint32_t *__restrict__ off, const uint8_t *__restrict__ codes,
                        const float *__restrict__ norm_r, const float *__restrict__ dot_cr,
                        float *__restrict__ vterm) {
    int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= N) return;
    // cell of CSR position p: last c with off[c] <= p
    uint64_t lo = 0, hi = ncells - 1;
    while (lo < hi) {
        uint64_t mid = (lo + hi + 1) >> 1;
        if ((int64_t)off[mid] <= p) lo = mid;
        else hi = mid - 1;
    }
    uint32_t cell = (uint32_t)lo;
    int bs = kp * mp / mc;
    const float *r1, *r2;
    if (mode == SCG_IMI) {
        uint32_t h3 = cell / (uint32_t)kc, h4 = cell - h3 * (uint32_t)kc;
        r1 = dot_cr + (size_t)h3 * bs;
        r2 = dot_cr + (size_t)(h4 + kc - 1) * bs;
    } else {
        // the residual's centroid: the cell's first nearest one (second candidate)
        uint32_t h3 = (mode == SCG_SC2) ? cell / (uint32_t)kc : (mode == SCG_SC3 ? cell / ((uint32_t)kc * kc) : cell);
        r1 = dot_cr + (size_t)h3 * bs;
        r2 = r1;
    }
    const uint8_t *c = codes + (size_t)p * mp;
    int half = (mode == SCG_IMI) ? (mp >> 1) : mp;
    float v = 0.0f;
    for (int k = 0; k < mp; k++) {
        int bc = k * kp + c[k];
        v += norm_r[bc] + (k < half ? r1 : r2)[bc];
    }
    vterm[p] = v;
}

}  // namespace

void launch_vterm(int mode, int kc, int mp, int kp, int mc, uint64_t ncells, int64_t N, const uint32_t *off,
                  const uint8_t *codes, const float *norm_r, const float *dot_cr, float *vterm, cudaStream_t s) {
    if (N <= 0) return;
    k_vterm<<<(unsigned)((N + 255) / 256), 256, 0, s>>>(mode, kc, mp, kp, mc, ncells, N, off, codes, norm_r, dot_cr,
                                                          vterm);
}

void launch_norms(const float *C, int rows, int len, float *out, cudaStream_t s) {
    if (rows <= 0) return;
    k_norms<<<(rows + 255) / 256, 256, 0, s>>>(C, rows, len, out);
}

void launch_precompute1(int dim, int mc, int kc, int mp, int kp, const float *cq, const float *pq,
                        float *norm_c, float *norm_r, float *dot_cr, cudaStream_t s) {
    int bsc = dim / mc, bsp = dim / mp;
    k_norms<<<(mc * kc + 255) / 256, 256, 0, s>>>(cq, mc * kc, bsc, norm_c);
    k_norms<<<(mp * kp + 255) / 256, 256, 0, s>>>(pq, mp * kp, bsp, norm_r);
    size_t total = (size_t)kc * kp * mp;
    k_dot_cr<<<(unsigned)((total + 255) / 256), 256, 0, s>>>(cq, pq, mc, kc, mp, kp, bsc, bsp, dot_cr);
}

void launch_tables_exact(const TablesArgs &a, cudaStream_t s) {
    if (a.nq <= 0) return;
    int ctiles = (a.kc + ET - 1) / ET, ptiles = (a.kp + ET - 1) / ET;
    dim3 grid(a.mc * ctiles + a.mp * ptiles, (a.nq + QT - 1) / QT);
    k_tables_exact<<<grid, ET, 0, s>>>(a, ctiles, ptiles);
    launch_query_norms(a, s);
}

void launch_query_norms(const TablesArgs &a, cudaStream_t s) {
    if (a.nq <= 0 || !a.qn) return;
    const int qb = std::min(QN_MAX_ROWS, QN_SMEM_WORDS / (a.dim + 1));
    if (qb >= 1) {
        const size_t smem = sizeof(float) * (size_t)qb * (a.dim + 1);
        k_query_norms_staged<<<(a.nq + qb - 1) / qb, QN_THREADS, smem, s>>>(a.Q, a.nq, a.dim, a.mc, qb, a.qn,
                                                                           a.qsum);
    } else {
        k_query_norms<<<(a.nq + 127) / 128, 128, 0, s>>>(a.Q, a.nq, a.dim, a.mc, a.qn, a.qsum);
    }
}

}  // namespace scg
