// Encoder on the tensor cores, with the reference's codes.
//
// Encoder::encode<T> (encoder.h:69-192) takes, per coarse part and then per
// PQ subspace of the residual, the first centroid of minimum
// distance_l2_square (float differences, squared and summed in double; a
// strict '>' keeps the first minimum).  Here the distances are ranked first
// by a tensor-core table t(c) = ||c||^2 - 2<x, c> (the tcgen05 split-BF16
// tile kernel of tables_tc.cu, over a chunk of rows), whose error against
// the exact distance minus ||x||^2 is below 2^-12 (||x||^2 + ||c||^2): the
// split products are within 3 * 2^-16 of 2 sum |x_t c_t| <= ||x||^2 +
// ||c||^2, and the reference's own float differences and double sums add
// less than 2^-22 of the distance.  Any centroid whose t(c) is more than
// twice that bound above the row's minimum cannot be the exact argmin, so
// `k_pick` scores every centroid within the margin
// 2^-10 (||x||^2 + max ||c||^2) of the minimum with the reference's
// arithmetic and keeps the first exact minimum -- usually one or two
// centroids.  The codes are therefore the reference's, bit for bit.  The
// second-candidate encoder (SCEncoder::encode<T>) runs the same way: its nc
// nearest coarse centroids come from the candidates within the margin of the
// nc-th smallest table value, and its float-rounded comparisons are kept.
#include <type_traits>

#include "scg_internal.cuh"

namespace scg {

namespace {

constexpr int PK_THREADS = 256;  // 8 warps, one (row, segment) each

__device__ __forceinline__ double exact_l2(const float *__restrict__ x, const float *__restrict__ c, int len) {
    double d = 0.0;
    for (int t = 0; t < len; t++) {
        const double tmp = (double)__fsub_rn(x[t], __ldg(c + t));
        d = __dadd_rn(d, __dmul_rn(tmp, tmp));
    }
    return d;
}

// (key, id) lexicographic order of the candidate lists below.
template <class K>
__device__ __forceinline__ bool key_less(K ka, int ia, K kb, int ib) {
    return ka < kb || (ka == kb && ia < ib);
}

// NB = 1: the first minimum (Encoder::encode<T>: double distances, strict
// '>', encoder.h:143-160).  NB = 2, 3 with FC: the NB smallest float-rounded
// distances, equal ones by centroid id (SCEncoder::encode<T>,
// sc_encoder.h:255-290, whose insertion keeps the earlier centroid first);
// NB = 1 with FC: the first minimum of the float-rounded distances (its PQ
// step, sc_encoder.h:300-320).  The NB smallest keys by (key, id) of all
// centroids whose table value is within the margin of the NB-th smallest
// table value are the reference's: a centroid further from it is beaten by
// NB others by more than the table's error bound plus the float rounding.
// Lists start at (largest key, id 0) and take a centroid only below the
// current last key, so missing entries stay id 0 as in the reference.
template <int NB, bool FC>
__global__ void __launch_bounds__(PK_THREADS) k_pick(PickArgs a) {
    using K = typename std::conditional<FC, float, double>::type;
    const K KMAX = FC ? (K)__int_as_float(0x7f7fffff) : (K)1.7976931348623157e308;  // as sc_encoder.h / encoder.h:143
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const int64_t item = (int64_t)blockIdx.x * (PK_THREADS / 32) + (threadIdx.x >> 5);
    if (item >= a.n * a.nseg) return;  // whole warps leave together
    const int64_t row = item / a.nseg;
    const int j = (int)(item - row * a.nseg);
    const float *x = a.X + (size_t)row * a.dim + (size_t)j * a.len;
    const float *t = a.tab + (size_t)row * a.nseg * a.kseg + (size_t)j * a.kseg;
    const float *C = a.C + (size_t)j * a.kseg * a.len;
    // ||x_seg||^2 (for the margin only) and the NB-th smallest table value
    float xn = 0.0f;
    for (int i = lane; i < a.len; i += 32) xn = fmaf(x[i], x[i], xn);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) xn += __shfl_xor_sync(FULL, xn, o);
    float tl[NB];
#pragma unroll
    for (int i = 0; i < NB; i++) tl[i] = __int_as_float(0x7f800000);
    for (int c = lane; c < a.kseg; c += 32) {
        float v = t[c];
#pragma unroll
        for (int i = 0; i < NB; i++) {
            const float lo = fminf(tl[i], v), hi = fmaxf(tl[i], v);
            tl[i] = lo;
            v = hi;
        }
    }
    float tnb = __int_as_float(0x7f800000);
    {
        // NB rounds of a warp minimum over the lanes' list heads
        int head = 0;
#pragma unroll
        for (int r = 0; r < NB; r++) {
            float h = __int_as_float(0x7f800000);
#pragma unroll
            for (int i = 0; i < NB; i++)
                if (i == head) h = tl[i];
            float m = h;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) m = fminf(m, __shfl_xor_sync(FULL, m, o));
            tnb = m;
            const unsigned own = __ballot_sync(FULL, h == m);
            if (lane == __ffs(own) - 1) head++;
        }
    }
    const float margin = 0x1p-10f * (xn + a.segmax[j]) + 1e-30f;
    const float lim = tnb + margin;
    // exact re-check of the candidates: this lane's NB smallest (key, id)
    K bk[NB];
    int bi[NB];
#pragma unroll
    for (int i = 0; i < NB; i++) {
        bk[i] = KMAX;
        bi[i] = 0;
    }
    bool any = false;
    for (int c = lane; c < a.kseg; c += 32) {
        if (t[c] <= lim) {
            const double d = exact_l2(x, C + (size_t)c * a.len, a.len);
            K k = FC ? (K)(float)d : (K)d;
            any = true;
            if (k < bk[NB - 1]) {
                // candidates come in increasing c, so an equal key goes
                // behind; from the insertion point on every entry moves down
                int ci = c;
                bool moved = false;
#pragma unroll
                for (int i = 0; i < NB; i++) {
                    if (moved || k < bk[i]) {
                        const K tk = bk[i];
                        const int ti = bi[i];
                        bk[i] = k;
                        bi[i] = ci;
                        k = tk;
                        ci = ti;
                        moved = true;
                    }
                }
            }
        }
    }
    // the warp's NB smallest (key, id): NB rounds of a warp minimum of heads
    int out[NB];
    {
        int head = 0;
#pragma unroll
        for (int r = 0; r < NB; r++) {
            K hk = KMAX;
            int hi = 0x7fffffff;
#pragma unroll
            for (int i = 0; i < NB; i++)
                if (i == head) {
                    hk = bk[i];
                    hi = bk[i] < KMAX ? bi[i] : 0x7fffffff;
                }
            K mk = hk;
            int mi = hi;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                const K ok = __shfl_xor_sync(FULL, mk, o);
                const int oi = __shfl_xor_sync(FULL, mi, o);
                if (key_less(ok, oi, mk, mi)) {
                    mk = ok;
                    mi = oi;
                }
            }
            const unsigned own = __ballot_sync(FULL, hk == mk && hi == mi && mi != 0x7fffffff);
            if (own && lane == __ffs(own) - 1) head++;
            out[r] = mi;  // 0x7fffffff: fewer than r + 1 centroids below the largest key
        }
    }
    if (!__any_sync(FULL, any) || out[0] >= a.kseg) {
        // no candidate (a NaN in the row): the reference keeps centroid 0
#pragma unroll
        for (int r = 0; r < NB; r++) out[r] = 0;
        if (lane == 0 && a.status) atomicOr(a.status, ST_BAD_ARG);
    }
#pragma unroll
    for (int r = 0; r < NB; r++) out[r] = out[r] >= a.kseg ? 0 : out[r];  // unfilled entries keep id 0
    if (lane == 0) {
#pragma unroll
        for (int r = 0; r < NB; r++) {
            if (a.cid) a.cid[((size_t)row * a.nseg + j) * NB + r] = (uint16_t)out[r];
        }
        if (a.code) a.code[(size_t)row * a.nseg + j] = (uint8_t)out[0];
    }
    if (a.resid) {
        const float *cc = C + (size_t)out[0] * a.len;
        float *r = a.resid + (size_t)row * a.dim + (size_t)j * a.len;
        for (int i = lane; i < a.len; i += 32) r[i] = __fsub_rn(x[i], cc[i]);
    }
}

__global__ void k_segmax(const float *__restrict__ norms, int nseg, int kseg, float *__restrict__ out) {
    __shared__ float red[32];
    const int j = blockIdx.x;
    float m = 0.0f;
    for (int c = threadIdx.x; c < kseg; c += blockDim.x) m = fmaxf(m, norms[(size_t)j * kseg + c]);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x == 0) {
        float r = 0.0f;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) r = fmaxf(r, red[w]);
        out[j] = r;
    }
}

}  // namespace

void launch_pick(const PickArgs &a, cudaStream_t s) {
    const int64_t items = a.n * a.nseg;
    if (items <= 0) return;
    const unsigned grid = (unsigned)((items + PK_THREADS / 32 - 1) / (PK_THREADS / 32));
    if (!a.fcmp) k_pick<1, false><<<grid, PK_THREADS, 0, s>>>(a);
    else if (a.nbest == 3) k_pick<3, true><<<grid, PK_THREADS, 0, s>>>(a);
    else if (a.nbest == 2) k_pick<2, true><<<grid, PK_THREADS, 0, s>>>(a);
    else k_pick<1, true><<<grid, PK_THREADS, 0, s>>>(a);
}

void launch_segmax(const float *norms, int nseg, int kseg, float *out, cudaStream_t s) {
    if (nseg <= 0) return;
    k_segmax<<<nseg, 256, 0, s>>>(norms, nseg, kseg, out);
}

}  // namespace scg
