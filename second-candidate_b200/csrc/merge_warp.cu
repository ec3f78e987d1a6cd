// Top-R of a query's scan survivors with one warp per query: the last step
// of the split search (query.h:321-324, multi_query.h:269-272,
// sc_query.h:250-252: nth_element_id + sort_id over the candidates), after
// the scan-only kernel kept the candidates at or below its threshold.
//
// The scan kernel hands over up to SURV_CAP survivors per query as (ordered
// distance << 32 | CSR position) words.  Here a bisection over the distance
// words finds the R-th smallest (stopping early at a value with exactly R
// words at or below it); every survivor at or below it -- the R best and
// every entry tied with the R-th -- gets its id, and one sort of
// (distance, id) keys gives the R best in order, equal distances by id.  A
// query the scan kernel merged itself has surv_n = -1 and is skipped.
#include "scg_internal.cuh"

namespace scg {

namespace {

constexpr int MW_WARPS = 4;
constexpr int MKPL = SURV_CAP / 32;  // survivors per lane

__device__ __forceinline__ uint64_t shfl_xor64m(uint64_t v, int m) {
    const uint32_t lo = __shfl_xor_sync(0xffffffffu, (uint32_t)v, m);
    const uint32_t hi = __shfl_xor_sync(0xffffffffu, (uint32_t)(v >> 32), m);
    return ((uint64_t)hi << 32) | lo;
}

// Ascending bitonic sort of 32 * P keys held striped (element r * 32 + lane).
template <int P>
__device__ __forceinline__ void msort(uint64_t *buf, int lane) {
    uint64_t v[P];
#pragma unroll
    for (int r = 0; r < P; r++) v[r] = buf[r * 32 + lane];
    constexpr int n = 32 * P;
#pragma unroll
    for (int k = 2; k <= n; k <<= 1) {
#pragma unroll
        for (int j = k >> 1; j > 0; j >>= 1) {
            if (j >= 32) {
                const int rj = j >> 5;
#pragma unroll
                for (int r = 0; r < P; r++) {
                    const int pr = r ^ rj;
                    if (pr > r) {
                        const bool asc = ((r * 32) & k) == 0;
                        const uint64_t x = v[r], y = v[pr];
                        if ((x > y) == asc) {
                            v[r] = y;
                            v[pr] = x;
                        }
                    }
                }
            } else {
                const bool lower = (lane & j) == 0;
#pragma unroll
                for (int r = 0; r < P; r++) {
                    const bool asc = ((r * 32 + lane) & k) == 0;
                    const uint64_t o = shfl_xor64m(v[r], j);
                    const uint64_t mn = v[r] < o ? v[r] : o, mx = v[r] < o ? o : v[r];
                    v[r] = (lower == asc) ? mn : mx;
                }
            }
        }
    }
#pragma unroll
    for (int r = 0; r < P; r++) buf[r * 32 + lane] = v[r];
}

// Longer key sets (many ties at the R-th distance): the same network in the
// warp's shared buffer.
__device__ __noinline__ void msort_smem(uint64_t *buf, int n, int lane) {
    for (int k = 2; k <= n; k <<= 1) {
        for (int j = k >> 1; j > 0; j >>= 1) {
            for (int i = lane; i < n; i += 32) {
                const int ixj = i ^ j;
                if (ixj > i) {
                    const uint64_t x = buf[i], y = buf[ixj];
                    if ((x > y) == ((i & k) == 0)) {
                        buf[i] = y;
                        buf[ixj] = x;
                    }
                }
            }
            __syncwarp();
        }
    }
}

__global__ void __launch_bounds__(MW_WARPS * 32) k_merge_warp(const uint64_t *__restrict__ surv,
                                                              const int *__restrict__ surv_n, int cap,
                                                              const int *__restrict__ pid, int nq, int R,
                                                              int *__restrict__ out_ids, float *__restrict__ out_d) {
    __shared__ uint64_t buf[MW_WARPS][SURV_CAP];
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    uint64_t *b = buf[wid];
    const int nwarps = gridDim.x * MW_WARPS;
    for (int q = blockIdx.x * MW_WARPS + wid; q < nq; q += nwarps) {
        const int n = surv_n[q];
        if (n < 0) continue;  // merged by the scan kernel
        const uint64_t *src = surv + (size_t)q * cap;
        // the distance words, MKPL per lane (element j * 32 + lane)
        uint32_t dw[MKPL];
#pragma unroll
        for (int j = 0; j < MKPL; j++) {
            const int i = j * 32 + lane;
            dw[j] = i < n ? (uint32_t)(__ldg(src + i) >> 32) : 0xffffffffu;
        }
        // v: keep the words <= v -- every word when n <= R, else the R-th
        // smallest or a word with exactly R words at or below it
        uint32_t v = 0xffffffffu;
        if (n > R) {
            uint32_t lo = 0xffffffffu, hi = 0;
#pragma unroll
            for (int j = 0; j < MKPL; j++)
                if (j * 32 + lane < n) {
                    lo = min(lo, dw[j]);
                    hi = max(hi, dw[j]);
                }
            lo = __reduce_min_sync(FULL, lo);
            hi = __reduce_max_sync(FULL, hi);
            while (lo < hi) {
                const uint32_t mid = lo + ((hi - lo) >> 1);
                uint32_t c = 0;
#pragma unroll
                for (int j = 0; j < MKPL; j++) c += dw[j] <= mid ? 1u : 0u;
                c = __reduce_add_sync(FULL, c);
                if (c == (uint32_t)R) {
                    lo = hi = mid;
                    break;
                }
                if (c > (uint32_t)R) hi = mid;
                else lo = mid + 1;
            }
            v = lo;
        }
        // the kept survivors as (distance, id) keys, compacted in order
        int m = 0;
#pragma unroll
        for (int j = 0; j < MKPL; j++) {
            if (j * 32 >= n) break;  // warp-uniform
            const int i = j * 32 + lane;
            const bool in = i < n && dw[j] <= v;
            const unsigned bal = __ballot_sync(FULL, in);
            if (in) {
                const uint32_t pos = (uint32_t)__ldg(src + i);
                b[m + __popc(bal & ((1u << lane) - 1u))] = ((uint64_t)dw[j] << 32) | (uint32_t)__ldg(pid + pos);
            }
            m += __popc(bal);
        }
        int m2 = 32;
        while (m2 < m) m2 <<= 1;
        for (int i = m + lane; i < m2; i += 32) b[i] = ~0ull;
        __syncwarp();
        switch (m2) {
            case 32: msort<1>(b, lane); break;
            case 64: msort<2>(b, lane); break;
            case 128: msort<4>(b, lane); break;
            case 256: msort<8>(b, lane); break;
            default: msort_smem(b, m2, lane); break;
        }
        __syncwarp();
        const int keep = m < R ? m : R;
        for (int j = lane; j < R; j += 32) {
            const size_t o = (size_t)q * R + j;
            if (j < keep) {
                const uint64_t e = b[j];
                out_ids[o] = (int)(uint32_t)e;
                out_d[o] = o2f((uint32_t)(e >> 32));
            } else {
                out_ids[o] = -1;
                out_d[o] = __int_as_float(0x7f800000);
            }
        }
        __syncwarp();
    }
}

}  // namespace

void merge_warp_launch(const uint64_t *surv, const int *surv_n, int cap, const int *pid, int nq, int R,
                       int *out_ids, float *out_d, int nsm, cudaStream_t s) {
    if (nq <= 0) return;
    const int want = (nq + MW_WARPS - 1) / MW_WARPS;
    const int grid = want < nsm * 8 ? want : nsm * 8;
    k_merge_warp<<<grid, MW_WARPS * 32, 0, s>>>(surv, surv_n, cap, pid, nq, R, out_ids, out_d);
}

}  // namespace scg
