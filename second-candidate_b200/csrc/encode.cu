// Encoders: nearest coarse centroid(s), residual, nearest PQ centroid per
// subspace -- with the reference's arithmetic so that codes are identical.
//
// Encoder::encode<T> (encoder.h:69-192): every distance is
// distance_l2_square<float> (utilities.h:195-207): the difference of two
// floats, squared and summed in double; the argmin keeps the first minimum
// (strict '>').  SCEncoder::encode<T> (sc_encoder.h:205-332) rounds the coarse
// distances to float and takes the nc smallest (equal distances by centroid
// id), residual to the nearest; its PQ argmin compares float-rounded
// distances.  Multiplies and adds round separately (__dmul_rn / __dadd_rn).
//
// One thread encodes one row.  Rows of a block are staged in shared memory
// one coarse part at a time; centroids stream through shared memory in
// chunks and are read by all threads of a warp at once (broadcast).
#include "scg_internal.cuh"

namespace scg {

namespace {

constexpr int ECH = 8192;   // floats of centroid data staged per chunk
// rows per block (one per thread): 64, or 16 when the staged rows of a wide
// vector (D up to ~1,400) would not fit shared memory at 64

__device__ __forceinline__ double l2sq(const float *x, int xstride, const float *c, int len) {
    double dis = 0.0;
    for (int t = 0; t < len; t++) {
        double tmp = (double)__fsub_rn(x[t * xstride], c[t]);
        dis = __dadd_rn(dis, __dmul_rn(tmp, tmp));
    }
    return dis;
}

// Stages rows [r0, r0+ERT) x dims [d0, d0+len) into xs laid out [dim][ERT]
// (thread t reads column t: conflict-free).
template <int ERT>
__device__ void stage_rows(const float *X, int64_t n, int dim, int64_t r0, int d0, int len, float *xs) {
    for (int i = threadIdx.x; i < ERT * len; i += ERT) {
        int r = i / len, t = i % len;
        int64_t row = r0 + r;
        xs[t * ERT + r] = row < n ? X[(size_t)row * dim + d0 + t] : 0.0f;
    }
}

// Finds the nearest of `kcount` centroids of length `len` (rows of C) for
// this thread's staged vector; first minimum in double.  nbest >= 1 keeps the
// nbest smallest float-rounded distances instead (SC coarse step).
template <int NB, int ERT>
__device__ void nearest(const float *C, int kcount, int len, const float *xs, float *cs, bool float_cmp,
                        int *best_idx) {
    double bd = 1.7976931348623157e308;  // DBL_MAX, as encoder.h:143
    float bf[NB];
    int bi[NB];
#pragma unroll
    for (int i = 0; i < NB; i++) {
        bf[i] = __int_as_float(0x7f7fffff);
        bi[i] = 0;
    }
    int per = ECH / len;
    if (per < 1) per = 1;
    for (int k0 = 0; k0 < kcount; k0 += per) {
        int kn = min(per, kcount - k0);
        __syncthreads();
        for (int i = threadIdx.x; i < kn * len; i += ERT) cs[i] = C[(size_t)k0 * len + i];
        __syncthreads();
        for (int kk = 0; kk < kn; kk++) {
            double dt = l2sq(xs + threadIdx.x, ERT, cs + kk * len, len);
            int k = k0 + kk;
            if (NB == 1 && !float_cmp) {
                if (bd > dt) {
                    bd = dt;
                    bi[0] = k;
                }
            } else if (NB == 1) {
                float f = (float)dt;
                if (bf[0] > f) {
                    bf[0] = f;
                    bi[0] = k;
                }
            } else {
                float f = (float)dt;
                if (f < bf[NB - 1]) {
                    int j = NB - 1;
                    while (j > 0 && bf[j - 1] > f) {
                        bf[j] = bf[j - 1];
                        bi[j] = bi[j - 1];
                        j--;
                    }
                    bf[j] = f;
                    bi[j] = k;
                }
            }
        }
    }
#pragma unroll
    for (int i = 0; i < NB; i++) best_idx[i] = bi[i];
}

template <int NC, int ERT>
__global__ void __launch_bounds__(ERT) k_encode(EncodeArgs a) {
    extern __shared__ __align__(16) float esm[];
    const int mcp = NC ? 1 : a.mc;
    const int bsc = a.dim / mcp, bsp = a.dim / a.mp;
    float *cs = esm;                       // ECH
    float *xs = cs + ECH;                  // [bsc][ERT] staged part
    float *rs = xs + (size_t)bsc * ERT;    // [dim][ERT] residual
    const int64_t r0 = (int64_t)blockIdx.x * ERT;
    const int64_t row = r0 + threadIdx.x;
    const bool live = row < a.n;
    for (int j = 0; j < mcp; j++) {
        __syncthreads();
        stage_rows<ERT>(a.X, a.n, a.dim, r0, j * bsc, bsc, xs);
        __syncthreads();
        int idx[NC ? NC : 1];
        const float *C = a.cq + (size_t)j * a.kc * bsc;
        if (NC) nearest<NC ? NC : 1, ERT>(C, a.kc, bsc, xs, cs, true, idx);
        else nearest<1, ERT>(C, a.kc, bsc, xs, cs, false, idx);
        const float *c0 = C + (size_t)idx[0] * bsc;
        for (int t = 0; t < bsc; t++) rs[(j * bsc + t) * ERT + threadIdx.x] = __fsub_rn(xs[t * ERT + threadIdx.x], c0[t]);
        if (live) {
            if (NC) {
                for (int i = 0; i < NC; i++) a.cid[(size_t)row * NC + i] = (uint16_t)idx[i];
            } else {
                a.cid[(size_t)row * a.mc + j] = (uint16_t)idx[0];
            }
        }
    }
    for (int j = 0; j < a.mp; j++) {
        int idx[1];
        nearest<1, ERT>(a.pq + (size_t)j * a.kp * bsp, a.kp, bsp, rs + (size_t)j * bsp * ERT, cs, NC != 0, idx);
        if (live) a.codes[(size_t)row * a.mp + j] = (uint8_t)idx[0];
    }
}

size_t encode_smem(int dim, int mcp, int ert) {
    return sizeof(float) * ((size_t)ECH + (size_t)(dim / mcp) * ert + (size_t)dim * ert);
}

constexpr size_t SMEM_MAX = 227 * 1024;

template <int NC, int ERT>
void launch_k(const EncodeArgs &a, size_t smem, cudaStream_t s) {
    cudaFuncSetAttribute(k_encode<NC, ERT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k_encode<NC, ERT><<<(unsigned)((a.n + ERT - 1) / ERT), ERT, smem, s>>>(a);
}

template <int ERT>
void launch_nc(const EncodeArgs &a, size_t smem, cudaStream_t s) {
    if (a.nc == 0) launch_k<0, ERT>(a, smem, s);
    else if (a.nc == 2) launch_k<2, ERT>(a, smem, s);
    else launch_k<3, ERT>(a, smem, s);
}

}  // namespace

size_t encode_smem_bytes(int dim, int mcp) {
    const size_t s64 = encode_smem(dim, mcp, 64);
    return s64 <= SMEM_MAX ? s64 : encode_smem(dim, mcp, 16);
}

void launch_encode(const EncodeArgs &a, cudaStream_t s) {
    if (a.n <= 0) return;
    const int mcp = a.nc ? 1 : a.mc;
    const size_t s64 = encode_smem(a.dim, mcp, 64);
    if (s64 <= SMEM_MAX) launch_nc<64>(a, s64, s);
    else launch_nc<16>(a, encode_smem(a.dim, mcp, 16), s);
}

}  // namespace scg
