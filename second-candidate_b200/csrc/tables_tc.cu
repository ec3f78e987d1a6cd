// Per-query tables on the tensor cores (tcgen05, kind::f16).
//
// pre_compute2 (query.h:154-184) is, over a batch, one small GEMM per
// segment (a coarse part or a PQ subspace): dot[q][e] = <Q_seg[q], C_seg[e]>,
// M = queries, N = centroids of the segment, K = the segment's dimensions.
// Each CTA computes one 128 x 256 tile (128 queries = the 128 TMEM lanes,
// 256 centroids = 256 fp32 TMEM columns):
//   - 128 threads load fp32 queries and centroids, round them to 16-bit
//     operands and store them in shared memory in the canonical K-major
//     no-swizzle layout: 8-row x 16-byte core matrices, element (row r, k)
//     at byte ((k / 8) * ROWS + r) * 16 + (k % 8) * 2;
//   - one thread issues tcgen05.mma (M = 128, N = 256, K = 16 per
//     instruction) accumulating in TMEM, and commits to an mbarrier;
//   - the four warps read their 32 lanes back with tcgen05.ld and write
//     (norm - dot) - dot, or -2 dot for the fast form's LUT.
// Split form: NSPLIT = 3 takes BF16 operands to near-FP32 accuracy: each
// value x = hi + lo with hi = bf16(x), lo = bf16(x - hi) (|x - hi - lo| <=
// 2^-16 |x|), and the product is hi_a hi_b + hi_a lo_b + lo_a hi_b, within
// 3 * 2^-16 |a b| (exact for the second operand's error alone when a is an
// integer below 256, as uint8 data are).  NSPLIT = 1 is one BF16 or FP16
// product (2^-7 or 2^-10 of |a b|).
//
// Every wait on the mbarrier is bounded: on expiry the CTA records
// ST_TC_TIMEOUT in the status word, skips its epilogue, frees its TMEM and
// returns.
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include "scg_internal.cuh"

namespace scg {

namespace {

constexpr int TM = 128;            // queries per tile (TMEM lanes)
constexpr int TN = 256;            // entries per tile (TMEM columns)
constexpr int TK = 64;             // K elements staged per chunk
constexpr int TC_THREADS = 256;  // 8 warps: warp w reads TMEM lanes 32 (w % 4).., columns half w / 4
constexpr int A_BYTES = TM * TK * 2;
constexpr int B_BYTES = TN * TK * 2;
constexpr int OFF_A0 = 0;
constexpr int OFF_A1 = OFF_A0 + A_BYTES;
constexpr int OFF_B0 = OFF_A1 + A_BYTES;
constexpr int OFF_B1 = OFF_B0 + B_BYTES;
constexpr int OFF_NORM = OFF_B1 + B_BYTES;  // the tile's TN centroid norms (fp32)
constexpr int OFF_BAR = OFF_NORM + TN * 4;
// 97 KB + control words: at most two CTAs per SM, so two 256-column TMEM
// allocations never exceed the SM's 512 columns.
constexpr int TC_SMEM = OFF_BAR + 64;
constexpr long long WAIT_CYCLES = 1ll << 30;  // ~0.5 s at the boost clock

__device__ __forceinline__ uint32_t smem_addr(const void *p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

// Shared-memory matrix descriptor: start address, leading-dimension byte
// offset (between the two 8-element K halves of an MMA), stride byte offset
// (between 8-row groups), descriptor version 1, no swizzle.
__device__ __forceinline__ uint64_t mat_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    uint64_t d = (uint64_t)((addr >> 4) & 0x3FFFu);
    d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1 << 46;
    return d;
}

// Instruction descriptor of kind::f16: FP32 accumulator, A and B of the same
// 16-bit type (fmt 0 = f16, 1 = bf16), both K-major, N = TN, M = TM.
__host__ __device__ constexpr uint32_t instr_desc(uint32_t fmt) {
    return (1u << 4) | (fmt << 7) | (fmt << 10) | ((uint32_t)(TN >> 3) << 17) | ((uint32_t)(TM >> 4) << 24);
}

__device__ __forceinline__ void mma_issue(uint32_t tmem, uint64_t da, uint64_t db, uint32_t idesc, uint32_t accum) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem),
        "l"(da), "l"(db), "r"(idesc), "r"(accum)
        : "memory");
}

__device__ __forceinline__ void mma_commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
                 : "memory");
}

// Waits for the mbarrier phase of the given parity; false after WAIT_CYCLES.
__device__ __forceinline__ bool bar_wait(uint32_t bar, uint32_t parity) {
    const long long t0 = clock64();
    for (;;) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done)
            : "r"(bar), "r"(parity)
            : "memory");
        if (done) return true;
        if (clock64() - t0 > WAIT_CYCLES) return false;
    }
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// 16 consecutive fp32 columns of this thread's TMEM lane.
__device__ __forceinline__ void tmem_load16(uint32_t taddr, float (&v)[16]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
        "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; i++) v[i] = __uint_as_float(r[i]);
}

// Rounds 8 floats to 16-bit operands: hi always, lo = x - hi when split.
template <int FMT, bool SPLIT>
__device__ __forceinline__ void pack8(const float (&x)[8], uint4 &hi, uint4 &lo) {
    uint32_t h[4], l[4];
#pragma unroll
    for (int j = 0; j < 4; j++) {
        if (FMT == 1) {
            __nv_bfloat16 a = __float2bfloat16_rn(x[2 * j]), b = __float2bfloat16_rn(x[2 * j + 1]);
            h[j] = (uint32_t)__bfloat16_as_ushort(a) | ((uint32_t)__bfloat16_as_ushort(b) << 16);
            if (SPLIT) {
                __nv_bfloat16 c = __float2bfloat16_rn(x[2 * j] - __bfloat162float(a));
                __nv_bfloat16 d = __float2bfloat16_rn(x[2 * j + 1] - __bfloat162float(b));
                l[j] = (uint32_t)__bfloat16_as_ushort(c) | ((uint32_t)__bfloat16_as_ushort(d) << 16);
            }
        } else {
            __half a = __float2half_rn(x[2 * j]), b = __float2half_rn(x[2 * j + 1]);
            h[j] = (uint32_t)__half_as_ushort(a) | ((uint32_t)__half_as_ushort(b) << 16);
            if (SPLIT) {
                __half c = __float2half_rn(x[2 * j] - __half2float(a));
                __half d = __float2half_rn(x[2 * j + 1] - __half2float(b));
                l[j] = (uint32_t)__half_as_ushort(c) | ((uint32_t)__half_as_ushort(d) << 16);
            }
        }
    }
    hi = make_uint4(h[0], h[1], h[2], h[3]);
    if (SPLIT) lo = make_uint4(l[0], l[1], l[2], l[3]);
}

// Stages rows [0, rows) x K groups [0, ngroups) of one operand: row r is
// src + r * ld (valid when r < nrows), elements k0 .. k0 + 8 * ngroups of it
// (valid when < len).  A thread loads SB groups before it converts and
// stores any of them, so a batch costs one global-load round trip instead of
// one per group (the stores to shared memory would otherwise keep the next
// group's loads from being issued early).
constexpr int SB = 8;

template <int FMT, bool SPLIT>
__device__ __forceinline__ void stage(const float *__restrict__ src, int nrows, size_t ld, int len, int k0, int rows,
                                      int ngroups, unsigned char *hi, unsigned char *lo) {
    // whole groups of 8 load as two float4 when every row starts 16-byte aligned
    const bool vec = ((reinterpret_cast<uintptr_t>(src) & 15) == 0) && (ld % 4 == 0);
    const int total = rows * ngroups;
    for (int u0 = threadIdx.x; u0 < total; u0 += SB * TC_THREADS) {
        float x[SB][8];
#pragma unroll
        for (int b = 0; b < SB; b++) {
            const int u = u0 + b * TC_THREADS;
            const int r = u % rows, g = u / rows;
            const int kb = k0 + g * 8;
            const bool row_ok = u < total && r < nrows;
            const float *p = src + (size_t)r * ld + kb;
            if (vec && row_ok && kb + 8 <= len) {
                const float4 v0 = __ldg(reinterpret_cast<const float4 *>(p));
                const float4 v1 = __ldg(reinterpret_cast<const float4 *>(p) + 1);
                x[b][0] = v0.x; x[b][1] = v0.y; x[b][2] = v0.z; x[b][3] = v0.w;
                x[b][4] = v1.x; x[b][5] = v1.y; x[b][6] = v1.z; x[b][7] = v1.w;
            } else {
#pragma unroll
                for (int j = 0; j < 8; j++) x[b][j] = (row_ok && kb + j < len) ? __ldg(p + j) : 0.0f;
            }
        }
#pragma unroll
        for (int b = 0; b < SB; b++) {
            const int u = u0 + b * TC_THREADS;
            if (u < total) {
                const int r = u % rows, g = u / rows;
                uint4 h, l;
                pack8<FMT, SPLIT>(x[b], h, l);
                const size_t off = ((size_t)g * rows + r) * 16;
                *(uint4 *)(hi + off) = h;
                if (SPLIT) *(uint4 *)(lo + off) = l;
            }
        }
    }
}

template <int NSPLIT, int FMT>
__global__ void __launch_bounds__(TC_THREADS, 1) k_tables_tc(TablesArgs a, int ctiles, int ptiles, int tile0) {
    extern __shared__ __align__(1024) unsigned char tsm[];
    constexpr bool SPLIT = NSPLIT == 3;
    unsigned char *A0 = tsm + OFF_A0, *A1 = tsm + OFF_A1, *B0 = tsm + OFF_B0, *B1 = tsm + OFF_B1;
    uint64_t *bar = (uint64_t *)(tsm + OFF_BAR);
    uint32_t *tslot = (uint32_t *)(tsm + OFF_BAR + 8);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

    int tile = blockIdx.x + tile0;
    int e0, seglen, len, qoff, outstride, outoff;
    const float *cent, *norm;
    float *out;
    bool lut_only;
    if (tile < a.mc * ctiles) {
        const int seg = tile / ctiles;
        e0 = (tile % ctiles) * TN;
        seglen = a.kc;
        len = a.dim / a.mc;
        qoff = seg * len;
        cent = a.cq + (size_t)seg * a.kc * len;
        norm = a.norm_c + (size_t)seg * a.kc;
        out = a.dqc;
        outstride = a.mc * a.kc;
        outoff = seg * a.kc;
        lut_only = false;
    } else {
        tile -= a.mc * ctiles;
        const int seg = tile / ptiles;
        e0 = (tile % ptiles) * TN;
        seglen = a.kp;
        len = a.dim / a.mp;
        qoff = seg * len;
        cent = a.pq + (size_t)seg * a.kp * len;
        norm = a.norm_r + (size_t)seg * a.kp;
        out = a.dqr;
        outstride = a.mp * a.kp;
        outoff = seg * a.kp;
        lut_only = a.lut_only != 0;
    }
    const int q0 = blockIdx.y * TM;
    const int kpad = (len + 15) & ~15;

    const uint32_t bar_a = smem_addr(bar);
    if (threadIdx.x == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar_a) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(tslot)),
                     "r"(TN)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    // the tile's centroid norms for the epilogue (0 for the fast form's LUT
    // and past the segment's end), read once here instead of per lane there
    float *snorm = (float *)(tsm + OFF_NORM);
    for (int t = threadIdx.x; t < TN; t += TC_THREADS)
        snorm[t] = (lut_only || e0 + t >= seglen) ? 0.0f : __ldg(norm + e0 + t);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tslot;

    constexpr uint32_t IDESC = instr_desc(FMT);
    const float *qsrc = a.Q + (size_t)q0 * a.dim + qoff;
    const float *csrc = cent + (size_t)e0 * len;
    const int qrows = min(TM, a.nq - q0), crows = min(TN, seglen - e0);
    uint32_t parity = 0;
    bool failed = false;
    for (int k0 = 0; k0 < kpad; k0 += TK) {
        const int kn = min(TK, kpad - k0);  // a multiple of 16
        const int ng = kn / 8;
        stage<FMT, SPLIT>(qsrc, qrows, (size_t)a.dim, len, k0, TM, ng, A0, A1);
        stage<FMT, SPLIT>(csrc, crows, (size_t)len, len, k0, TN, ng, B0, B1);
        // make the generic-proxy stores visible to the tensor cores
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        if (threadIdx.x == 0) {
            tc_fence_after();
            const uint32_t a0 = smem_addr(A0), a1 = smem_addr(A1), b0 = smem_addr(B0), b1 = smem_addr(B1);
            for (int s = 0; s < kn / 16; s++) {
                const uint32_t ao = (uint32_t)(s * 2 * TM * 16), bo = (uint32_t)(s * 2 * TN * 16);
                const uint64_t da0 = mat_desc(a0 + ao, TM * 16, 128), db0 = mat_desc(b0 + bo, TN * 16, 128);
                mma_issue(tmem, da0, db0, IDESC, (k0 > 0 || s > 0) ? 1u : 0u);
                if (SPLIT) {
                    const uint64_t da1 = mat_desc(a1 + ao, TM * 16, 128), db1 = mat_desc(b1 + bo, TN * 16, 128);
                    mma_issue(tmem, da0, db1, IDESC, 1u);
                    mma_issue(tmem, da1, db0, IDESC, 1u);
                }
            }
            mma_commit(bar_a);
        }
        const bool ok = bar_wait(bar_a, parity);
        parity ^= 1u;
        failed = __syncthreads_or(!ok) != 0;
        tc_fence_after();
        if (failed) break;
    }

    if (!failed) {
        // warp w: TMEM lanes (queries) 32 (w % 4) .. + 31 (the lanes a warp
        // may read), columns [TN / 2 (w / 4), TN / 2 (w / 4 + 1))
        const int wq = warp & 3, half = warp >> 2;
        const int q = q0 + wq * 32 + lane;
        const uint32_t lane_base = tmem + ((uint32_t)(wq * 32) << 16);
        const bool vec = (outstride % 4) == 0 && (outoff % 4) == 0;
        for (int c = half * (TN / 2); c < (half + 1) * (TN / 2) && e0 + c < seglen; c += 16) {
            float v[16];
            tmem_load16(lane_base + (uint32_t)c, v);
            if (q < a.nq) {
                float *dst = out + (size_t)q * outstride + outoff + e0 + c;
                float r[16];
#pragma unroll
                for (int j = 0; j < 16; j++) r[j] = __fsub_rn(__fsub_rn(snorm[c + j], v[j]), v[j]);
                if (vec && e0 + c + 16 <= seglen) {
#pragma unroll
                    for (int j = 0; j < 16; j += 4) *(float4 *)(dst + j) = make_float4(r[j], r[j + 1], r[j + 2], r[j + 3]);
                } else {
                    for (int j = 0; j < 16 && e0 + c + j < seglen; j++) dst[j] = r[j];
                }
            }
        }
    } else {
        if (threadIdx.x == 0 && a.status) atomicOr(a.status, ST_TC_TIMEOUT);
        // give MMAs still in flight one more bounded wait before freeing TMEM
        bar_wait(bar_a, parity ^ 1u);
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TN) : "memory");
    }
}

template <int NSPLIT, int FMT>
void launch_tc(const TablesArgs &a, dim3 grid, int ctiles, int ptiles, int tile0, cudaStream_t s) {
    cudaFuncSetAttribute(k_tables_tc<NSPLIT, FMT>, cudaFuncAttributeMaxDynamicSharedMemorySize, TC_SMEM);
    k_tables_tc<NSPLIT, FMT><<<grid, TC_THREADS, TC_SMEM, s>>>(a, ctiles, ptiles, tile0);
}

}  // namespace

void launch_tables_tc(const TablesArgs &a, int nsplit, int fmt, cudaStream_t s) {
    if (a.nq <= 0) return;
    const int ctiles = (a.kc + TN - 1) / TN, ptiles = (a.kp + TN - 1) / TN;
    const bool coarse = a.segs != 2, pq = a.segs != 1;
    const int tile0 = coarse ? 0 : a.mc * ctiles;
    const int ntiles = (coarse ? a.mc * ctiles : 0) + (pq ? a.mp * ptiles : 0);
    dim3 grid(ntiles, (a.nq + TM - 1) / TM);
    if (nsplit == 3) {
        if (fmt == 1) launch_tc<3, 1>(a, grid, ctiles, ptiles, tile0, s);
        else launch_tc<3, 0>(a, grid, ctiles, ptiles, tile0, s);
    } else {
        if (fmt == 1) launch_tc<1, 1>(a, grid, ctiles, ptiles, tile0, s);
        else launch_tc<1, 0>(a, grid, ctiles, ptiles, tile0, s);
    }
    launch_query_norms(a, s);
}

}  // namespace scg
