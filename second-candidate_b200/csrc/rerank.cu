// Shortlist re-rank by exact distance.
//
// The reference's real_dist branch (query.h:307-312, multi_query.h:255-259,
// sc_query.h:232-236) scores a candidate by distance_l2_square against the
// raw vector (lib/simple-cluster/include/utilities.h:217-230): each
// difference is a float subtraction, squared and summed in double in
// dimension order, and the result is stored as float.  Here the ADC search
// first keeps a shortlist of L candidates per query; this kernel gives each
// of them that exact distance (one thread per candidate, the reference's
// order, so the value is bit-identical) and keeps the R smallest in
// (distance, id) order with one bitonic sort of the shortlist in shared
// memory.  Raw vectors are float32 or uint8 (uint8 data give the same
// differences as their float copies, at a quarter of the gather bytes).
#include "exact_dist.cuh"

namespace scg {

namespace {

constexpr int RR_THREADS = 256;

template <typename T>
__global__ void __launch_bounds__(RR_THREADS) k_rerank(const float *__restrict__ Q, int dim,
                                                       const T *__restrict__ raw, int64_t N,
                                                       const int *__restrict__ sl_ids, int L, int Lp, int R,
                                                       int *__restrict__ out_ids, float *__restrict__ out_d,
                                                       int *__restrict__ status) {
    extern __shared__ __align__(16) unsigned char rsm[];
    uint64_t *keys = (uint64_t *)rsm;                 // [Lp]
    float *qs = (float *)(rsm + (((size_t)Lp * 8 + 15) & ~(size_t)15));  // [dim], 16-byte aligned
    const int q = blockIdx.x;
    for (int t = threadIdx.x; t < dim; t += RR_THREADS) qs[t] = Q[(size_t)q * dim + t];
    // whole rows as 16-byte loads when every row starts 16-byte aligned
    const bool vec = ((reinterpret_cast<uintptr_t>(raw) & 15) == 0) && ((dim * sizeof(T)) % 16 == 0);
    __syncthreads();
    for (int i = threadIdx.x; i < Lp; i += RR_THREADS) {
        uint64_t key = ~0ull;
        if (i < L) {
            const int id = sl_ids[(size_t)q * L + i];
            if (id >= 0 && id < N) {
                const float d = vec ? exact_dist_vec(qs, raw + (size_t)id * dim, dim)
                                    : exact_dist(qs, raw + (size_t)id * dim, dim);
                key = ((uint64_t)f2o(d) << 32) | (uint32_t)id;
            } else if (id >= N) {
                atomicOr(status, ST_BAD_ARG);
            }
        }
        keys[i] = key;
    }
    __syncthreads();
    // bitonic sort of Lp keys, ascending
    for (int k = 2; k <= Lp; k <<= 1) {
        for (int j = k >> 1; j > 0; j >>= 1) {
            for (int i = threadIdx.x; i < Lp; i += RR_THREADS) {
                const int p = i ^ j;
                if (p > i) {
                    const uint64_t a = keys[i], b = keys[p];
                    const bool up = (i & k) == 0;
                    if ((a > b) == up) {
                        keys[i] = b;
                        keys[p] = a;
                    }
                }
            }
            __syncthreads();
        }
    }
    for (int i = threadIdx.x; i < R; i += RR_THREADS) {
        const uint64_t key = i < Lp ? keys[i] : ~0ull;
        const bool none = key == ~0ull;
        out_ids[(size_t)q * R + i] = none ? -1 : (int)(uint32_t)key;
        out_d[(size_t)q * R + i] = none ? __int_as_float(0x7f800000) : o2f((uint32_t)(key >> 32));
    }
}

}  // namespace

size_t rerank_smem_bytes(int L, int dim) {
    int Lp = 1;
    while (Lp < L) Lp <<= 1;
    return (((size_t)Lp * 8 + 15) & ~(size_t)15) + (size_t)dim * 4;
}

int launch_rerank(const float *Q, int nq, int dim, const void *raw, int raw_u8, int64_t N, const int *sl_ids, int L,
                  int R, int *out_ids, float *out_d, int *status, cudaStream_t s) {
    if (nq <= 0) return 0;
    int Lp = 1;
    while (Lp < L) Lp <<= 1;
    const size_t smem = rerank_smem_bytes(L, dim);
    if (raw_u8) {
        cudaFuncSetAttribute(k_rerank<uint8_t>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        k_rerank<uint8_t><<<nq, RR_THREADS, smem, s>>>(Q, dim, (const uint8_t *)raw, N, sl_ids, L, Lp, R, out_ids,
                                                      out_d, status);
    } else {
        cudaFuncSetAttribute(k_rerank<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        k_rerank<float><<<nq, RR_THREADS, smem, s>>>(Q, dim, (const float *)raw, N, sl_ids, L, Lp, R, out_ids,
                                                    out_d, status);
    }
    return 0;
}

}  // namespace scg
