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
// centroids.  The codes are therefore the reference's, bit for bit.
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

__global__ void __launch_bounds__(PK_THREADS) k_pick(PickArgs a) {
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const int64_t item = (int64_t)blockIdx.x * (PK_THREADS / 32) + (threadIdx.x >> 5);
    if (item >= a.n * a.nseg) return;  // whole warps leave together
    const int64_t row = item / a.nseg;
    const int j = (int)(item - row * a.nseg);
    const float *x = a.X + (size_t)row * a.dim + (size_t)j * a.len;
    const float *t = a.tab + (size_t)row * a.nseg * a.kseg + (size_t)j * a.kseg;
    const float *C = a.C + (size_t)j * a.kseg * a.len;
    // ||x_seg||^2 (for the margin only) and the table minimum
    float xn = 0.0f;
    for (int i = lane; i < a.len; i += 32) xn = fmaf(x[i], x[i], xn);
    float tmin = __int_as_float(0x7f800000);
    for (int c = lane; c < a.kseg; c += 32) tmin = fminf(tmin, t[c]);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        xn += __shfl_xor_sync(FULL, xn, o);
        tmin = fminf(tmin, __shfl_xor_sync(FULL, tmin, o));
    }
    const float margin = 0x1p-10f * (xn + a.segmax[j]) + 1e-30f;
    const float lim = tmin + margin;
    // exact re-check of the candidates; first minimum in centroid order
    double best = 1.7976931348623157e308;  // DBL_MAX, as encoder.h:143
    int bi = 0x7fffffff;
    bool any = false;
    for (int c = lane; c < a.kseg; c += 32) {
        if (t[c] <= lim) {
            const double d = exact_l2(x, C + (size_t)c * a.len, a.len);
            if (d < best || (d == best && c < bi)) {
                best = d;
                bi = c;
            }
            any = true;
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const double ob = __shfl_xor_sync(FULL, best, o);
        const int oi = __shfl_xor_sync(FULL, bi, o);
        if (ob < best || (ob == best && oi < bi)) {
            best = ob;
            bi = oi;
        }
    }
    if (!__any_sync(FULL, any) || bi >= a.kseg) {
        // no candidate (a NaN in the row): the reference keeps centroid 0
        bi = 0;
        if (lane == 0 && a.status) atomicOr(a.status, ST_BAD_ARG);
    }
    if (lane == 0) {
        if (a.cid) a.cid[(size_t)row * a.nseg + j] = (uint16_t)bi;
        if (a.code) a.code[(size_t)row * a.nseg + j] = (uint8_t)bi;
    }
    if (a.resid) {
        const float *cc = C + (size_t)bi * a.len;
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
    const int64_t grid = (items + PK_THREADS / 32 - 1) / (PK_THREADS / 32);
    k_pick<<<(unsigned)grid, PK_THREADS, 0, s>>>(a);
}

void launch_segmax(const float *norms, int nseg, int kseg, float *out, cudaStream_t s) {
    if (nseg <= 0) return;
    k_segmax<<<nseg, 256, 0, s>>>(norms, nseg, kseg, out);
}

}  // namespace scg
