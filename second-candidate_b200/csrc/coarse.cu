// Coarse ranking of a whole batch ahead of the fused search.
//
// The reference sorts each coarse list of a query completely
// (nth_element_id + sort_id with M = kc, multi_query.h:114-128,
// sc_query.h:98-106, query.h:230-234), but the multi-sequence walk only
// reaches a prefix.  For kc <= 1024 one warp handles one list (longer lists,
// up to 8192, one block: k_coarse_prefix_block): the keys
// (ordered float of q_part + diff_qc, << 32 | centroid id, so equal keys go
// by id) sit 32 per lane at most; a binary search over the high words finds
// vm, the M-th smallest (M from the query's candidate target and the cell
// density seen so far, prefix_density), every key with high word <= vm is
// compacted through shared memory and sorted by a register bitonic network
// (register swaps for
// partner distances >= 32, warp shuffles below).  Per list the kernel writes
// the sorted prefix, its length and the smallest high word after it; the
// fused kernel then treats the prefix exactly as its own radix-selected
// prefix (and still sorts everything itself if the walk leaves the prefix).
#include "scg_internal.cuh"

namespace scg {

namespace {

constexpr int CS_THREADS = 128;  // 4 warps, one list each

// Candidates per cell for the prefix length rule: a quarter of what the
// selection kernel has seen on this index so far (cells near queries are
// denser than the average, but a query in a sparser region reaches further:
// the quarter doubles the prefix), else N / cells.  A prefix too short for a
// query only costs that query a complete sort inside the selection kernel.
__device__ __forceinline__ double prefix_density(const CoarseArgs &a) {
    if (a.dens_acc) {
        const unsigned long long cells = __ldcg(a.dens_acc + 1);
        if (cells > 0) {
            const double d = 0.25 * (double)__ldcg(a.dens_acc) / (double)cells;
            return d < a.avg_density ? a.avg_density : d;
        }
    }
    return a.avg_density;
}
constexpr int CS_CAP = 1024;     // keys per list

__device__ __forceinline__ uint64_t shfl_xor64(uint64_t v, int m) {
    const uint32_t lo = __shfl_xor_sync(0xffffffffu, (uint32_t)v, m);
    const uint32_t hi = __shfl_xor_sync(0xffffffffu, (uint32_t)(v >> 32), m);
    return ((uint64_t)hi << 32) | lo;
}

// Ascending bitonic sort of 32 * P keys held striped (element r * 32 + lane).
template <int P>
__device__ __forceinline__ void warp_sort(uint64_t (&v)[P], int lane) {
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
                    const uint64_t o = shfl_xor64(v[r], j);
                    const uint64_t mn = v[r] < o ? v[r] : o, mx = v[r] < o ? o : v[r];
                    v[r] = (lower == asc) ? mn : mx;
                }
            }
        }
    }
}

// Sorts buf[0, 32 * P) (padding already ~0) and writes it to dst.
template <int P>
__device__ __forceinline__ void sort_out(const uint64_t *buf, uint64_t *dst, int lane) {
    uint64_t v[P];
#pragma unroll
    for (int r = 0; r < P; r++) v[r] = buf[r * 32 + lane];
    warp_sort<P>(v, lane);
#pragma unroll
    for (int r = 0; r < P; r++) dst[r * 32 + lane] = v[r];
}

// The sorts of 128 and 256 keys out of line: each prefix length runs one
// of them, and the kernel body stays small in the instruction cache.
template <int P>
__device__ __noinline__ void sort_out_far(const uint64_t *buf, uint64_t *dst, int lane) {
    sort_out<P>(buf, dst, lane);
}

// Longer prefixes (512 or 1024 keys, rare): a bitonic sort in the warp's
// shared buffer with few registers, then the copy to dst.
__device__ __noinline__ void sort_out_smem(uint64_t *buf, uint64_t *dst, int n, int lane) {
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
    for (int i = lane; i < n; i += 32) dst[i] = buf[i];
}

template <int P>
__global__ void __launch_bounds__(CS_THREADS) k_coarse_prefix(CoarseArgs a) {
    __shared__ uint64_t buf[CS_THREADS / 32][CS_CAP];
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int list = blockIdx.x * (CS_THREADS / 32) + wid;
    const int nlists = a.imi ? 2 : 1;
    if (list >= a.nq * nlists) return;  // whole warps leave together
    const int q = list / nlists, part = list - q * nlists;
    const float base = a.imi ? a.qn[2 * q + part] : a.qsum[q];
    const float *row = a.dqc + (size_t)q * a.mc * a.kc + (size_t)part * a.kc;
    // the high words (ordered keys) only: the centroid id of element
    // r * 32 + lane is its position; positions past kc hold 0xffffffff,
    // above every key (the ordered form of any float is below it)
    uint32_t v[P];
#pragma unroll
    for (int r = 0; r < P; r++) {
        const int i = r * 32 + lane;
        v[r] = i < a.kc ? f2o(__fadd_rn(base, row[i])) : 0xffffffffu;
    }
    // prefix length rule of the fused kernel
    const int T = a.Tq ? a.Tq[q] : a.T;
    const double dens = prefix_density(a);
    const double c0 = (T > 0 ? (double)T : 1.0) / (dens > 1e-9 ? dens : 1e-9);
    int M = 1;
    while (M < 4 * (int)sqrt(c0) + 1) M <<= 1;
    if (M < 128) M = 128;
    if (a.fixed_prefix > 0) M = a.fixed_prefix;  // the autotuner's choice
    if (M > a.max_prefix) M = a.max_prefix;
    uint32_t vm = 0xfffffffeu;  // every key
    if (M < a.kc) {
        // vm: a high word with exactly M keys at or below it if one exists
        // (the bisection stops there), else the M-th smallest (ties)
        uint32_t lo = 0xffffffffu, hi = 0;
#pragma unroll
        for (int r = 0; r < P; r++) {
            if (r * 32 + lane < a.kc) {
                lo = v[r] < lo ? v[r] : lo;
                hi = v[r] > hi ? v[r] : hi;
            }
        }
        lo = __reduce_min_sync(FULL, lo);
        hi = __reduce_max_sync(FULL, hi);
        while (lo < hi) {
            const uint32_t mid = lo + ((hi - lo) >> 1);
            int cnt = 0;
#pragma unroll
            for (int r = 0; r < P; r++) cnt += v[r] <= mid ? 1 : 0;
            cnt = __reduce_add_sync(FULL, cnt);
            if (cnt == M) {
                lo = hi = mid;
                break;
            }
            if (cnt > M) hi = mid;
            else lo = mid + 1;
        }
        vm = lo;
    }
    // compact the keys with high word <= vm; the smallest high word above vm
    uint64_t *b = buf[wid];
    int c = 0;
    uint32_t nxt = 0xffffffffu;
#pragma unroll
    for (int r = 0; r < P; r++) {
        const bool in = v[r] <= vm;
        if (!in && v[r] < nxt) nxt = v[r];
        const unsigned m = __ballot_sync(FULL, in);
        if (in) b[c + __popc(m & ((1u << lane) - 1))] = ((uint64_t)v[r] << 32) | (uint32_t)(r * 32 + lane);
        c += __popc(m);
    }
    nxt = __reduce_min_sync(FULL, nxt);
    int c2 = 32;
    while (c2 < c) c2 <<= 1;
    for (int i = c + lane; i < c2; i += 32) b[i] = ~0ull;
    __syncwarp();
    uint64_t *dst = a.out + (size_t)list * a.width;
    switch (c2) {
        case 32: sort_out<1>(b, dst, lane); break;
        case 64: sort_out<2>(b, dst, lane); break;
        case 128: sort_out_far<4>(b, dst, lane); break;
        case 256: sort_out_far<8>(b, dst, lane); break;
        default: sort_out_smem(b, dst, c2, lane); break;
    }
    if (lane == 0) {
        a.meta[2 * list] = (uint32_t)c;
        a.meta[2 * list + 1] = nxt;
    }
}

// Lists longer than 1024 (kc up to 8192): one block of 256 threads per list,
// P keys per thread, striped (element i = r * 256 + tid); the same
// prefix rule by a block-wide radix select (4 x 8 bits); keys at or below vm are
// gathered in shared memory (unordered, then sorted by warp 0).  A prefix
// longer than 1024 keys (many ties) is left to the selection kernel
// (length 0 in the metadata).
template <int P>
__global__ void __launch_bounds__(256) k_coarse_prefix_block(CoarseArgs a) {
    constexpr int NTB = 256;
    __shared__ uint64_t buf[CS_CAP];
    __shared__ uint32_t hist[NTB];
    __shared__ int s_cnt[NTB / 32];
    __shared__ uint32_t s_min[NTB / 32];
    __shared__ int s_c, s_acc;
    __shared__ uint32_t s_bin;
    const unsigned FULL = 0xffffffffu;
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    const int list = blockIdx.x;
    const int nlists = a.imi ? 2 : 1;
    const int q = list / nlists, part = list - q * nlists;
    const float base = a.imi ? a.qn[2 * q + part] : a.qsum[q];
    const float *row = a.dqc + (size_t)q * a.mc * a.kc + (size_t)part * a.kc;
    uint64_t v[P];
#pragma unroll
    for (int r = 0; r < P; r++) {
        const int i = r * NTB + tid;
        v[r] = i < a.kc ? (((uint64_t)f2o(__fadd_rn(base, row[i])) << 32) | (uint32_t)i) : ~0ull;
    }
    const int T = a.Tq ? a.Tq[q] : a.T;
    const double dens = prefix_density(a);
    const double c0 = (T > 0 ? (double)T : 1.0) / (dens > 1e-9 ? dens : 1e-9);
    int M = 1;
    while (M < 4 * (int)sqrt(c0) + 1) M <<= 1;
    if (M < 128) M = 128;
    if (a.fixed_prefix > 0) M = a.fixed_prefix;  // the autotuner's choice
    if (M > a.max_prefix) M = a.max_prefix;
    auto block_count = [&](uint32_t lim) {
        int cnt = 0;
#pragma unroll
        for (int r = 0; r < P; r++) cnt += (uint32_t)(v[r] >> 32) <= lim;
        cnt = __reduce_add_sync(FULL, cnt);
        __syncthreads();
        if (lane == 0) s_cnt[wid] = cnt;
        __syncthreads();
        int t = 0;
        for (int w = 0; w < NTB / 32; w++) t += s_cnt[w];
        return t;
    };
    uint32_t vm = 0xffffffffu;
    if (M < a.kc) {
        // vm = the M-th smallest high word: radix select, 4 passes of 8 bits
        // (one histogram bin per thread)
        uint32_t prefix = 0;
        int need = M;
        for (int shift = 24; shift >= 0; shift -= 8) {
            hist[tid] = 0;
            __syncthreads();
#pragma unroll
            for (int r = 0; r < P; r++) {
                const uint32_t hw = (uint32_t)(v[r] >> 32);
                if (v[r] != ~0ull && (shift == 24 || (hw >> (shift + 8)) == (prefix >> (shift + 8))))
                    atomicAdd(&hist[(hw >> shift) & 255u], 1u);
            }
            __syncthreads();
            // exclusive scan of the 256 bins (thread = bin)
            const uint32_t cnt = hist[tid];
            uint32_t x = cnt;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t y = __shfl_up_sync(FULL, x, o);
                if (lane >= o) x += y;
            }
            if (lane == 31) s_cnt[wid] = (int)x;
            __syncthreads();
            uint32_t wpre = 0;
            for (int w = 0; w < wid; w++) wpre += (uint32_t)s_cnt[w];
            const uint32_t ex = wpre + x - cnt;
            if (ex < (uint32_t)need && ex + cnt >= (uint32_t)need) {
                s_bin = (uint32_t)tid;
                s_acc = (int)ex;
            }
            __syncthreads();
            prefix |= s_bin << shift;
            need -= s_acc;
            __syncthreads();
        }
        vm = prefix;
    }
    // prefix length and the smallest high word above vm
    uint32_t nxt = 0xffffffffu;
#pragma unroll
    for (int r = 0; r < P; r++) {
        const uint32_t hw = (uint32_t)(v[r] >> 32);
        if (v[r] != ~0ull && hw > vm && hw < nxt) nxt = hw;
    }
    nxt = __reduce_min_sync(FULL, nxt);
    if (lane == 0) s_min[wid] = nxt;
    if (tid == 0) s_c = 0;
    __syncthreads();
    for (int w = 0; w < NTB / 32; w++) nxt = min(nxt, s_min[w]);
    const int c = block_count(vm);
    uint64_t *dst = a.out + (size_t)list * a.width;
    if (c > CS_CAP) {
        if (tid == 0) {
            a.meta[2 * list] = 0u;  // the selection kernel ranks this list itself
            a.meta[2 * list + 1] = 0xffffffffu;
        }
        return;
    }
#pragma unroll
    for (int r = 0; r < P; r++) {
        if (v[r] != ~0ull && (uint32_t)(v[r] >> 32) <= vm) buf[atomicAdd(&s_c, 1)] = v[r];
    }
    __syncthreads();
    int c2 = 32;
    while (c2 < c) c2 <<= 1;
    for (int i = c + tid; i < c2; i += NTB) buf[i] = ~0ull;
    __syncthreads();
    if (wid == 0) {
        switch (c2) {
            case 32: sort_out<1>(buf, dst, lane); break;
            case 64: sort_out<2>(buf, dst, lane); break;
            case 128: sort_out<4>(buf, dst, lane); break;
            case 256: sort_out<8>(buf, dst, lane); break;
            case 512: sort_out<16>(buf, dst, lane); break;
            default: sort_out<32>(buf, dst, lane); break;
        }
        if (lane == 0) {
            a.meta[2 * list] = (uint32_t)c;
            a.meta[2 * list + 1] = nxt;
        }
    }
}

template <int P>
void launch_p(const CoarseArgs &a, cudaStream_t s) {
    const int lists = a.nq * (a.imi ? 2 : 1);
    const int grid = (lists + CS_THREADS / 32 - 1) / (CS_THREADS / 32);
    k_coarse_prefix<P><<<grid, CS_THREADS, 0, s>>>(a);
}

}  // namespace

int coarse_sort_width(int kc) {
    int p = 32;
    while (p < kc) p <<= 1;
    if (p <= CS_CAP) return p;
    return kc <= 8192 ? CS_CAP : 0;  // long lists keep a prefix of at most CS_CAP keys
}

void launch_coarse_prefix(const CoarseArgs &a, cudaStream_t s) {
    if (a.nq <= 0) return;
    switch (coarse_sort_width(a.kc)) {
        case 32: launch_p<1>(a, s); break;
        case 64: launch_p<2>(a, s); break;
        case 128: launch_p<4>(a, s); break;
        case 256: launch_p<8>(a, s); break;
        case 512: launch_p<16>(a, s); break;
        case 1024:
            if (a.kc <= 1024) {
                launch_p<32>(a, s);
            } else {
                const int lists = a.nq * (a.imi ? 2 : 1);
                if (a.kc <= 2048) k_coarse_prefix_block<8><<<lists, 256, 0, s>>>(a);
                else if (a.kc <= 4096) k_coarse_prefix_block<16><<<lists, 256, 0, s>>>(a);
                else k_coarse_prefix_block<32><<<lists, 256, 0, s>>>(a);
            }
            break;
        default: break;
    }
}

}  // namespace scg
