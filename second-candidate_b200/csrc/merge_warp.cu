// Top-R of a query's scan survivors with one warp per query: the last step
// of the split search (query.h:321-324, multi_query.h:269-272,
// sc_query.h:250-252: nth_element_id + sort_id over the candidates), after
// the scan-only kernel kept the candidates at or below its threshold.
//
// The scan kernel hands over up to SURV_CAP survivors per query as (ordered
// distance << 32 | CSR position) words.  Here a bisection over the distance
// words finds the R-th smallest (stopping early at a value with exactly R
// words at or below it); every survivor at or below it -- the R best and
// every entry tied with the R-th -- is kept, and one sort gives the R best in
// order, equal distances by id.  The sort key is 32 bits, ((distance -
// smallest) << 10 | survivor index), when the kept distances span fewer than
// 2^22 ordered-float steps and at most 256 are kept; if two kept distances
// are then equal (the order of a tie must be by id, not by survivor index)
// or the key does not fit, (distance << 32 | id) keys are sorted instead.  A
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

__device__ __forceinline__ uint32_t shfl_xor_key(uint32_t v, int m) { return __shfl_xor_sync(0xffffffffu, v, m); }
__device__ __forceinline__ uint64_t shfl_xor_key(uint64_t v, int m) { return shfl_xor64m(v, m); }

// Ascending bitonic sort of 32 * P keys held striped (element r * 32 + lane).
template <int P, class K>
__device__ __forceinline__ void msort(K *buf, int lane) {
    K v[P];
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
                        const K x = v[r], y = v[pr];
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
                    const K o = shfl_xor_key(v[r], j);
                    const K mn = v[r] < o ? v[r] : o, mx = v[r] < o ? o : v[r];
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

// The kept survivors (distance word <= v) as (distance << 32 | id) keys,
// sorted into b[0, m); returns m.
__device__ __noinline__ int sort_wide(const uint64_t *__restrict__ src, int n, uint32_t v,
                                      const int *__restrict__ pid, uint64_t *b, int lane) {
    const unsigned FULL = 0xffffffffu;
    int m = 0;
    for (int j = 0; j * 32 < n; j++) {  // warp-uniform
        const int i = j * 32 + lane;
        const uint64_t e = i < n ? __ldg(src + i) : ~0ull;
        const bool in = i < n && (uint32_t)(e >> 32) <= v;
        const unsigned bal = __ballot_sync(FULL, in);
        if (in) b[m + __popc(bal & ((1u << lane) - 1u))] = (e & 0xffffffff00000000ull) | (uint32_t)__ldg(pid + (uint32_t)e);
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
    return m;
}

__global__ void __launch_bounds__(MW_WARPS * 32) k_merge_warp(const uint64_t *__restrict__ surv,
                                                              const int *__restrict__ surv_n, int cap,
                                                              const int *__restrict__ pid, int nq, int R,
                                                              int *__restrict__ out_ids, float *__restrict__ out_d) {
    __shared__ uint64_t buf[MW_WARPS][SURV_CAP];
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    uint64_t *b = buf[wid];
    uint32_t *b32 = reinterpret_cast<uint32_t *>(b);
    const int nwarps = gridDim.x * MW_WARPS;
    for (int q = blockIdx.x * MW_WARPS + wid; q < nq; q += nwarps) {
        const int n = surv_n[q];
        if (n < 0) continue;  // merged by the scan kernel
        const uint64_t *src = surv + (size_t)q * cap;
        // the distance words of the nj occupied rows (element j * 32 + lane)
        const int nj = (n + 31) >> 5;
        uint32_t dw[MKPL];
        uint32_t lo = 0xffffffffu, hi = 0;
#pragma unroll
        for (int j = 0; j < MKPL; j++) {
            const int i = j * 32 + lane;
            dw[j] = 0xffffffffu;
            if (j < nj && i < n) {
                dw[j] = (uint32_t)(__ldg(src + i) >> 32);
                lo = min(lo, dw[j]);
                hi = max(hi, dw[j]);
            }
        }
        lo = __reduce_min_sync(FULL, lo);
        hi = __reduce_max_sync(FULL, hi);
        const uint32_t dmin = lo;
        // v: keep the words <= v -- every word when n <= R, else the R-th
        // smallest or a word with exactly R words at or below it
        uint32_t v = hi;
        if (n > R) {
            while (lo < hi) {
                const uint32_t mid = lo + ((hi - lo) >> 1);
                uint32_t c = 0;
#pragma unroll
                for (int j = 0; j < MKPL; j++) {
                    if (j >= nj) break;  // warp-uniform
                    c += dw[j] <= mid ? 1u : 0u;
                }
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
        // narrow keys: ((distance - dmin) << 10 | survivor index)
        bool wide = n > 0 && (v - dmin >= (1u << 22) || n > SURV_CAP);
        int m = 0;
        if (!wide && n > 0) {
#pragma unroll
            for (int j = 0; j < MKPL; j++) {
                if (j >= nj) break;  // warp-uniform
                const int i = j * 32 + lane;
                const bool in = i < n && dw[j] <= v;
                const unsigned bal = __ballot_sync(FULL, in);
                const int at = m + __popc(bal & ((1u << lane) - 1u));
                if (in && at < 256) b32[at] = ((dw[j] - dmin) << 10) | (uint32_t)i;
                m += __popc(bal);
            }
            if (m > 256) {
                wide = true;
            } else {
                int m2 = 32;
                while (m2 < m) m2 <<= 1;
                for (int i = m + lane; i < m2; i += 32) b32[i] = 0xffffffffu;
                __syncwarp();
                switch (m2) {
                    case 32: msort<1>(b32, lane); break;
                    case 64: msort<2>(b32, lane); break;
                    case 128: msort<4>(b32, lane); break;
                    default: msort<8>(b32, lane); break;
                }
                __syncwarp();
                // equal kept distances must be ordered by id
                bool tie = false;
                for (int e = lane; e + 1 < m; e += 32) tie |= (b32[e] >> 10) == (b32[e + 1] >> 10);
                wide = __any_sync(FULL, tie);
                __syncwarp();
            }
        }
        if (wide) m = sort_wide(src, n, v, pid, b, lane);
        const int keep = min(m, R);
        for (int j = lane; j < R; j += 32) {
            const size_t o = (size_t)q * R + j;
            int id = -1;
            float d = __int_as_float(0x7f800000);
            if (j < keep && wide) {
                const uint64_t e = b[j];
                id = (int)(uint32_t)e;
                d = o2f((uint32_t)(e >> 32));
            } else if (j < keep) {
                const uint32_t k = b32[j];
                const uint32_t pos = (uint32_t)__ldg(src + (k & 1023u));
                id = __ldg(pid + pos);
                d = o2f((k >> 10) + dmin);
            }
            out_ids[o] = id;
            out_d[o] = d;
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
