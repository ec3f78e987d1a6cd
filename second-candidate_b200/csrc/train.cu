// Codebook training on the GPU: k-means++ seeding and Lloyd iterations for
// several segments at once (the coarse parts of an IMI, or the PQ
// subspaces of the residuals).
//
// The reference trains with PQQuantizer::create_sub_quantizers /
// calc_residual_vector (quantizer.h:235-272, 456-510) around greg_kmeans
// (k-means.h:671-912), whose Lloyd loop stops after one pass with shifted
// centroids; this trainer runs the algorithm as published: k-means++ seeding
// (each new centre drawn with probability proportional to the squared
// distance to the nearest centre so far) and `iters` Lloyd steps.
//   - seeding stays on the device: per step one kernel folds the newest
//     centre into the per-row minimum distances and sums them per block, and
//     one block per segment draws the next centre from those sums (a counter
//     hash of (seed, segment, step) gives the uniform draw);
//   - assignment uses the tcgen05 distance tables of tables_tc.cu
//     (||c||^2 - 2<x, c>, split BF16) and a warp argmin per (row, segment);
//   - the update sums members in FP64 (atomics) and divides in FP64; an empty
//     cluster keeps its centre.
#include "scg_internal.cuh"

namespace scg {

namespace {

constexpr int KT = 256;  // threads per block of the row-parallel kernels

__device__ __forceinline__ uint64_t mix64(uint64_t x) {
    // splitmix64 finaliser
    x += 0x9e3779b97f4a7c15ull;
    x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ull;
    x = (x ^ (x >> 27)) * 0x94d049bb133111ebull;
    return x ^ (x >> 31);
}

__device__ __forceinline__ double uniform01(uint64_t seed, int seg, int step) {
    const uint64_t h = mix64(seed ^ mix64(((uint64_t)seg << 32) | (uint32_t)step));
    return (double)(h >> 11) * (1.0 / 9007199254740992.0);  // [0, 1)
}

// Folds centre `step` of every segment into the rows' nearest squared
// distance d2[seg][row] and writes per-block sums bsum[seg][block].
__global__ void __launch_bounds__(KT) k_pp_update(const float *__restrict__ X, int64_t n, int dim, int len,
                                                  const float *__restrict__ C, int k, int step,
                                                  float *__restrict__ d2, double *__restrict__ bsum, int nblk) {
    __shared__ double red[KT / 32];
    const int seg = blockIdx.y;
    const int64_t i = (int64_t)blockIdx.x * KT + threadIdx.x;
    double v = 0.0;
    if (i < n) {
        const float *x = X + (size_t)i * dim + (size_t)seg * len;
        const float *c = C + ((size_t)seg * k + step) * len;
        float d = 0.0f;
        for (int t = 0; t < len; t++) {
            const float u = x[t] - c[t];
            d = fmaf(u, u, d);
        }
        float *p = d2 + (size_t)seg * n + i;
        const float m = step == 0 ? d : fminf(*p, d);
        *p = m;
        v = m;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int w = 0; w < KT / 32; w++) s += red[w];
        bsum[(size_t)seg * nblk + blockIdx.x] = s;
    }
}

// One block per segment: draws centre `step` (step 0: uniform over rows;
// later: proportional to d2) and copies that row's slice into C.
__global__ void __launch_bounds__(KT) k_pp_pick(const float *__restrict__ X, int64_t n, int dim, int len,
                                                float *__restrict__ C, int k, int step, const float *__restrict__ d2,
                                                const double *__restrict__ bsum, int nblk, uint64_t seed) {
    __shared__ int64_t s_row;
    __shared__ double s_acc;
    __shared__ int s_blk;
    const int seg = blockIdx.x;
    const double u = uniform01(seed, seg, step);
    if (threadIdx.x == 0) {
        int64_t row = 0;
        if (step == 0) {
            row = (int64_t)(u * (double)n);
        } else {
            double tot = 0.0;
            for (int b = 0; b < nblk; b++) tot += bsum[(size_t)seg * nblk + b];
            double target = u * tot, acc = 0.0;
            int blk = nblk - 1;
            for (int b = 0; b < nblk; b++) {
                const double s = bsum[(size_t)seg * nblk + b];
                if (acc + s > target) {
                    blk = b;
                    break;
                }
                acc += s;
            }
            s_blk = blk;
            s_acc = target - acc;
            row = -1;
        }
        s_row = row;
    }
    __syncthreads();
    if (s_row < 0) {
        // inside the chosen block: the first row whose running d2 passes the draw
        if (threadIdx.x == 0) {
            const int blk = s_blk;
            double acc = 0.0;
            int64_t pick = -1, last = -1;
            for (int t = 0; t < KT; t++) {
                const int64_t i = (int64_t)blk * KT + t;
                if (i >= n) break;
                const double v = d2[(size_t)seg * n + i];
                if (v > 0.0) last = i;
                acc += v;
                if (acc > s_acc && v > 0.0) {
                    pick = i;
                    break;
                }
            }
            if (pick < 0) pick = last >= 0 ? last : (int64_t)blk * KT;
            s_row = pick < n ? pick : n - 1;
        }
        __syncthreads();
    }
    const int64_t row = s_row;
    for (int t = threadIdx.x; t < len; t += KT)
        C[((size_t)seg * k + step) * len + t] = X[(size_t)row * dim + (size_t)seg * len + t];
}

// Assignment: warp per (row, segment) of a chunk of n rows starting at row
// r0, first minimum of the distance table; asg is [nseg][stride].
__global__ void __launch_bounds__(KT) k_assign(const float *__restrict__ tab, int64_t n, int nseg, int k,
                                               int *__restrict__ asg, int64_t stride, int64_t r0) {
    const int lane = threadIdx.x & 31;
    const int64_t item = (int64_t)blockIdx.x * (KT / 32) + (threadIdx.x >> 5);
    if (item >= n * nseg) return;
    const int64_t row = item / nseg;
    const int seg = (int)(item - row * nseg);
    const float *t = tab + (size_t)row * nseg * k + (size_t)seg * k;
    float best = __int_as_float(0x7f800000);
    int bi = 0x7fffffff;
    for (int c = lane; c < k; c += 32) {
        const float v = t[c];
        if (v < best) {
            best = v;
            bi = c;
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const float ob = __shfl_xor_sync(0xffffffffu, best, o);
        const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
        if (ob < best || (ob == best && oi < bi)) {
            best = ob;
            bi = oi;
        }
    }
    if (lane == 0) asg[(size_t)seg * stride + r0 + row] = bi < k ? bi : 0;
}

// FP64 member sums and counts.
__global__ void __launch_bounds__(KT) k_accumulate(const float *__restrict__ X, int64_t n, int dim, int len, int k,
                                                   const int *__restrict__ asg, double *__restrict__ sums,
                                                   unsigned long long *__restrict__ cnt) {
    const int seg = blockIdx.y;
    const int64_t i = (int64_t)blockIdx.x * KT + threadIdx.x;
    if (i >= n) return;
    const int c = asg[(size_t)seg * n + i];
    const float *x = X + (size_t)i * dim + (size_t)seg * len;
    double *s = sums + ((size_t)seg * k + c) * len;
    for (int t = 0; t < len; t++) atomicAdd(s + t, (double)x[t]);
    atomicAdd(cnt + (size_t)seg * k + c, 1ull);
}

__global__ void k_update(float *__restrict__ C, int nseg, int k, int len, const double *__restrict__ sums,
                         const unsigned long long *__restrict__ cnt) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (int64_t)nseg * k * len) return;
    const int64_t c = e / len;
    if (cnt[c] > 0) C[e] = (float)(sums[e] / (double)cnt[c]);
}

// r = x - C[asg] per segment (float, as the encoder's residual).
__global__ void __launch_bounds__(KT) k_residual(const float *__restrict__ X, int64_t n, int dim, int len, int k,
                                                 const float *__restrict__ C, const int *__restrict__ asg,
                                                 float *__restrict__ R) {
    const int seg = blockIdx.y;
    const int64_t i = (int64_t)blockIdx.x * KT + threadIdx.x;
    if (i >= n) return;
    const int c = asg[(size_t)seg * n + i];
    const float *x = X + (size_t)i * dim + (size_t)seg * len;
    const float *cc = C + ((size_t)seg * k + c) * len;
    float *r = R + (size_t)i * dim + (size_t)seg * len;
    for (int t = 0; t < len; t++) r[t] = __fsub_rn(x[t], cc[t]);
}

}  // namespace

// Work buffers of kmeans_segments, sized by the caller.
size_t kmeans_work_bytes(int64_t n, int nseg, int k, int len, int64_t chunk) {
    const int64_t nblk = (n + KT - 1) / KT;
    return 4ull * nseg * n                  // d2
           + 8ull * nseg * nblk             // block sums
           + 4ull * nseg * n                // assignments
           + 8ull * nseg * k * len          // FP64 sums
           + 8ull * nseg * k                // counts
           + 4ull * nseg * k                // norms
           + 4ull * chunk * nseg * k        // distance tables of one row chunk
           + 6 * 256;
}

// k-means over nseg segments of X (n rows, row stride dim, segment j = dims
// [j len, (j+1) len)); C receives [nseg][k][len].  asg_out (may be null)
// receives the final assignment [nseg][n].  status: ST_* bits of the
// tensor-core kernels.
int kmeans_segments(const float *X, int64_t n, int dim, int nseg, int k, int iters, uint64_t seed, float *C,
                    unsigned char *work, int64_t chunk, int *status, int *asg_out, cudaStream_t s) {
    const int len = dim / nseg;
    const int64_t nblk = (n + KT - 1) / KT;
    unsigned char *cur = work;
    auto take = [&](size_t bytes) {
        unsigned char *p = cur;
        cur += (bytes + 255) & ~(size_t)255;
        return p;
    };
    float *d2 = (float *)take(4ull * nseg * n);
    double *bsum = (double *)take(8ull * nseg * nblk);
    int *asg = (int *)take(4ull * nseg * n);
    double *sums = (double *)take(8ull * nseg * k * len);
    unsigned long long *cnt = (unsigned long long *)take(8ull * nseg * k);
    float *norms = (float *)take(4ull * nseg * k);
    float *tab = (float *)take(4ull * chunk * nseg * k);
    // k-means++ seeding
    const dim3 rows_grid((unsigned)nblk, (unsigned)nseg);
    for (int step = 0; step < k; step++) {
        if (step > 0) k_pp_update<<<rows_grid, KT, 0, s>>>(X, n, dim, len, C, k, step - 1, d2, bsum, (int)nblk);
        k_pp_pick<<<nseg, KT, 0, s>>>(X, n, dim, len, C, k, step, d2, bsum, (int)nblk, seed);
    }
    // Lloyd
    for (int it = 0; it <= iters; it++) {
        launch_norms(C, nseg * k, len, norms, s);
        for (int64_t r0 = 0; r0 < n; r0 += chunk) {
            const int nr = (int)std::min<int64_t>(chunk, n - r0);
            TablesArgs ta;
            memset(&ta, 0, sizeof(ta));
            ta.dim = dim; ta.mc = nseg; ta.kc = k; ta.mp = 1; ta.kp = 1; ta.nq = nr;
            ta.Q = X + (size_t)r0 * dim;
            ta.cq = C; ta.pq = C;
            ta.norm_c = norms; ta.norm_r = norms;
            ta.dqc = tab; ta.dqr = tab;
            ta.status = status;
            ta.segs = 1;
            launch_tables_tc(ta, 3, 1, s);
            const int64_t items = (int64_t)nr * nseg;
            k_assign<<<(unsigned)((items + KT / 32 - 1) / (KT / 32)), KT, 0, s>>>(tab, nr, nseg, k, asg, n, r0);
        }
        if (it == iters) break;  // the last pass only assigns
        cudaMemsetAsync(sums, 0, 8ull * nseg * k * len, s);
        cudaMemsetAsync(cnt, 0, 8ull * nseg * k, s);
        k_accumulate<<<rows_grid, KT, 0, s>>>(X, n, dim, len, k, asg, sums, cnt);
        const int64_t tot = (int64_t)nseg * k * len;
        k_update<<<(unsigned)((tot + 255) / 256), 256, 0, s>>>(C, nseg, k, len, sums, cnt);
    }
    if (asg_out) cudaMemcpyAsync(asg_out, asg, 4ull * nseg * n, cudaMemcpyDeviceToDevice, s);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, "k-means kernels");
    return SCG_OK;
}

void launch_residual(const float *X, int64_t n, int dim, int nseg, int k, const float *C, const int *asg, float *R,
                     cudaStream_t s) {
    const int64_t nblk = (n + KT - 1) / KT;
    k_residual<<<dim3((unsigned)nblk, (unsigned)nseg), KT, 0, s>>>(X, n, dim, dim / nseg, k, C, asg, R);
}

}  // namespace scg
