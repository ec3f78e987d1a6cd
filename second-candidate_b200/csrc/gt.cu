// Exact nearest neighbour of each query among the base rows (ground truth for
// recall@R, Evaluation::calc_recall, evaluation.h:58-92).
//
// The base is taken a chunk of rows at a time.  For every (query, chunk) the
// tcgen05 split-BF16 tile kernel (tables_tc.cu) gives t(x) = ||x||^2 - 2<q,
// x> for all rows x of the chunk; as in the encoder (encode_tc.cu), the
// exact squared distance minus ||q||^2 is within 2^-12 (||q||^2 + ||x||^2) of
// t(x), so a row more than 2^-10 (||q||^2 + max ||x||^2) above the chunk's
// minimum cannot be the chunk's nearest.  One warp per query scores the rows
// inside that margin exactly (float differences, squared and summed in
// double, as distance_l2_square) and folds the chunk's best into the query's
// running best; equal distances keep the lowest row id.
#include "scg_internal.cuh"

namespace scg {

namespace {

constexpr int NT_GT = 256;

__device__ __forceinline__ double exact_sq(const float *__restrict__ q, const float *__restrict__ x, int dim) {
    double d = 0.0;
    for (int t = 0; t < dim; t++) {
        const double tmp = (double)__fsub_rn(q[t], __ldg(x + t));
        d = __dadd_rn(d, __dmul_rn(tmp, tmp));
    }
    return d;
}

__global__ void __launch_bounds__(NT_GT) k_nn_fold(const float *__restrict__ Q, int nq, int dim,
                                                   const float *__restrict__ X, int64_t r0, int rows,
                                                   const float *__restrict__ tab, const float *__restrict__ xmax,
                                                   double *__restrict__ best_d, long long *__restrict__ best_i) {
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const int q = blockIdx.x * (NT_GT / 32) + (threadIdx.x >> 5);
    if (q >= nq) return;  // whole warps leave together
    const float *qv = Q + (size_t)q * dim;
    const float *t = tab + (size_t)q * rows;
    float qn = 0.0f;
    for (int i = lane; i < dim; i += 32) qn = fmaf(qv[i], qv[i], qn);
    float tmin = __int_as_float(0x7f800000);
    for (int c = lane; c < rows; c += 32) tmin = fminf(tmin, t[c]);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        qn += __shfl_xor_sync(FULL, qn, o);
        tmin = fminf(tmin, __shfl_xor_sync(FULL, tmin, o));
    }
    const float lim = tmin + 0x1p-10f * (qn + xmax[0]) + 1e-30f;
    double bd = 1.7976931348623157e308;
    long long bi = -1;
    for (int c = lane; c < rows; c += 32) {
        if (t[c] <= lim) {
            const double d = exact_sq(qv, X + (size_t)c * dim, dim);
            if (d < bd) {  // a lane's rows come in increasing order: first minimum
                bd = d;
                bi = r0 + c;
            }
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const double od = __shfl_xor_sync(FULL, bd, o);
        const long long oi = __shfl_xor_sync(FULL, bi, o);
        if (oi >= 0 && (bi < 0 || od < bd || (od == bd && oi < bi))) {
            bd = od;
            bi = oi;
        }
    }
    if (lane == 0 && bi >= 0) {
        const double cur = best_d[q];
        const long long ci = best_i[q];
        if (ci < 0 || bd < cur || (bd == cur && bi < ci)) {
            best_d[q] = bd;
            best_i[q] = bi;
        }
    }
}

__global__ void k_nn_init(int nq, double *best_d, long long *best_i) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q < nq) {
        best_d[q] = 1.7976931348623157e308;
        best_i[q] = -1;
    }
}

__global__ void k_nn_out(int nq, const double *best_d, const long long *best_i, int *ids, float *dists) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q < nq) {
        ids[q] = (int)best_i[q];
        if (dists) dists[q] = (float)best_d[q];
    }
}

}  // namespace

size_t exact_nn_work_bytes(int nq, int64_t chunk) {
    return 16ull * nq + 4ull * chunk + 4ull * chunk * nq + 6 * 256;
}

int exact_nn(const float *X, int64_t n, const float *Q, int nq, int dim, int *ids, float *dists, unsigned char *work,
             int64_t chunk, int *status, cudaStream_t s) {
    unsigned char *cur = work;
    auto take = [&](size_t bytes) {
        unsigned char *p = cur;
        cur += (bytes + 255) & ~(size_t)255;
        return p;
    };
    double *bd = (double *)take(8ull * nq);
    long long *bi = (long long *)take(8ull * nq);
    float *norms = (float *)take(4ull * chunk);
    float *xmax = (float *)take(4);
    float *tab = (float *)take(4ull * chunk * nq);
    k_nn_init<<<(nq + 255) / 256, 256, 0, s>>>(nq, bd, bi);
    for (int64_t r0 = 0; r0 < n; r0 += chunk) {
        const int rows = (int)std::min<int64_t>(chunk, n - r0);
        const float *xc = X + (size_t)r0 * dim;
        launch_norms(xc, rows, dim, norms, s);
        launch_segmax(norms, 1, rows, xmax, s);
        TablesArgs ta;
        memset(&ta, 0, sizeof(ta));
        ta.dim = dim; ta.mc = 1; ta.kc = rows; ta.mp = 1; ta.kp = 1; ta.nq = nq;
        ta.Q = Q;
        ta.cq = xc; ta.pq = xc;
        ta.norm_c = norms; ta.norm_r = norms;
        ta.dqc = tab; ta.dqr = tab;
        ta.status = status;
        ta.segs = 1;
        launch_tables_tc(ta, 3, 1, s);
        k_nn_fold<<<(nq + NT_GT / 32 - 1) / (NT_GT / 32), NT_GT, 0, s>>>(Q, nq, dim, xc, r0, rows, tab, xmax, bd, bi);
    }
    k_nn_out<<<(nq + 255) / 256, 256, 0, s>>>(nq, bd, bi, ids, dists);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, "exact nearest neighbour kernels");
    return SCG_OK;
}

}  // namespace scg
