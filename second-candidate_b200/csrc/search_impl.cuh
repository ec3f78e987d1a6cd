// Fused batched search (the kernel template; search_u2/u4/u8.cu instantiate it): per query, coarse ranking -> multi-sequence cell
// selection -> ADC scan with a fused top-R.  One CTA works on one query at a
// time and takes the next query from a global counter, so queries with
// uneven posting-list totals balance across the persistent grid.
//
// Coarse ranking.  The reference sorts each coarse list completely
// (nth_element_id + sort_id with M = kc, multi_query.h:125-128).  Only a
// prefix of each sorted list is ever reached, so a radix select finds the
// prefix of the M smallest keys (ties included) and sorts only it.  If the
// cell selection below then reaches a key at or beyond the smallest key a
// cell outside the prefix grid can have, the lists are sorted completely and
// the selection is repeated -- the result is the same as with full sorts.
//
// Cell selection.  The reference walks the grid of rank pairs (h1, h2) of the
// two sorted lists with a binary heap (multi_query.h:133-205,
// sc_query.h:112-186) and stops after the first cell at which the candidate
// total reaches T (or the cell cap w).  The visited set is therefore a
// prefix of the cells sorted by key(h1,h2) = A[h1] + B[h2].  Here the prefix
// is found without a serial heap:
//   1. rounds of "all cells with key <= tau": tau is bisected so that the
//      staircase {key <= tau} holds about a target number of cells (one
//      binary search per row, all rows in parallel); the new cells of the
//      round are enumerated, their lengths read from the CSR offsets and
//      kept as records (key, rank pair, length) in a per-CTA scratch slot;
//   2. once the totals reach T (or w), the exact cut key is found by a radix
//      select over the last round's records, weighted by length (or by
//      cell count for the w rule);
//   3. cells tied at the cut key are taken in (rank1, rank2) order until the
//      rule fires -- the order an exact priority queue yields.
// The ADC scan then scores the first WARMN candidates into shared memory;
// their R-th smallest distance bounds the final R-th distance, so a
// barrier-free warp-centric scan of the rest (warps claim chunks of
// candidates, keep their own window of visited cells, and add the table
// entries in the reference's order) keeps only candidates at or below that
// bound, and one radix-select merge over them gives the R best.
#pragma once

#include <type_traits>

#include "exact_dist.cuh"

namespace scg {

namespace {

constexpr int NT = 256;
constexpr int NWARP = NT / 32;
constexpr int HBITS = 11;
constexpr int HBINS = 1 << HBITS;
constexpr int TIECAP = 64;
constexpr int RBINS = 256;      // bins of the 8-bit radix selects of the scan phase (one per thread)
constexpr int RMAX = 1024;      // largest R
#ifndef SCG_WARMN
#define SCG_WARMN 4096
#endif
constexpr int WARMN = SCG_WARMN;  // candidates scored before the threshold is set
// The threshold is within 2^SCG_WARM_SBITS ordered-float steps above the R-th
// warm-up distance (2^(SCG_WARM_SBITS - 23) relative).  15 (0.4%) leaves
// one radix pass where 8 took two, for a few more survivors.
#ifndef SCG_WARM_SBITS
#define SCG_WARM_SBITS 15
#endif
constexpr int WWIN = 32;        // per-warp window of visited cells
constexpr int MERGE_KPT = 16;   // survivors per thread of the final merge's register bisection
// Candidates per lane per claimed chunk (U, a template parameter of the
// scan: 2, 4 or 8); a warp claims 32 * U candidates at a time.
constexpr int SBCAP = 2048;     // sorted coarse prefix capacity
// Kernel variants (template parameter VAR): the ADC scan in any form, the
// scan-only kernel of the fast form with kp == 256 (its own chunking and
// LUT), and the exact-distance scan over raw rows (rerank = -1).
constexpr int V_ADC = 0, V_FAST256 = 1, V_EXACT = 2;
constexpr int MAX_ROUNDS = 64;

struct CellWin {
    uint32_t pre;    // candidates before this cell (flat index)
    uint32_t start;  // CSR start
    float d0;        // per-cell constant of the ADC sum
    uint32_t h34;    // h3 | h4 << 16
};

__host__ __device__ __forceinline__ int next_pow2(int x) {
    int p = 1;
    while (p < x) p <<= 1;
    return p;
}
__host__ __device__ __forceinline__ size_t align16(size_t x) { return (x + 15) & ~(size_t)15; }

// Shared memory.  The LUT lives for the whole query; the selection phase
// (coarse lists, staircase rows, histograms) and the scan phase (cell
// windows, warm-up scores, top-R buffers) share the rest.  Inside the scan
// phase the top-R buffers alias the warm-up scores, which are dead once the
// threshold and the survivor buffer are set.  The selection-only kernel
// (part 1) has no LUT and no scan phase, the scan-only kernel (part 2) no
// selection phase.
struct Smem {
    float *lut;
    // selection phase
    uint64_t *LA, *LB;
    uint16_t *rowc, *rowp;
    uint32_t *rowpre;
    uint32_t *hist;   // HBINS
    uint64_t *ties;   // TIECAP
    uint64_t *sb;     // SBCAP (aliases hist/ties)
    // scan phase (aliases the selection phase)
    CellWin *wwin;    // [NWARP][WWIN]
    uint64_t *warm;   // [WARMN]
    uint64_t *top, *tmp;  // [RMAX] each, inside warm
    uint32_t *hist2;
    uint64_t *ties2;
};

// Bytes of the rotated LUT of the fast form (kp == 256, mp in {8, 16, 32}):
// 256 code rows x 32 banks of words, 32/mp copies of the [mp][256] table.
constexpr int ROT_LUT_BYTES = 256 * 32 * 4;

// The scan form that uses the rotated, bank-private LUT.
__host__ __device__ inline bool rot_form(int precision, int mp, int kp) {
    return precision == SCG_FAST && kp == 256 && (mp == 8 || mp == 16 || mp == 32);
}

// qdim > 0: the exact-distance scan (every candidate scored against its raw
// row), whose query of qdim floats takes the LUT's place.
__host__ __device__ inline size_t carve(int mode, int kc, int mp, int kp, int part, int rot, int qdim, Smem *s,
                                        unsigned char *base) {
    const int kcP = next_pow2(kc);
    size_t off = 0;
    if (s) s->lut = (float *)(base + off);
    if (part != 1)
        off += qdim > 0 ? align16((size_t)qdim * 4) : (rot ? (size_t)ROT_LUT_BYTES : align16((size_t)mp * kp * 4));
    const size_t phase0 = off;
    size_t end1 = phase0, end2 = phase0;
    if (part != 2) {
        // selection phase
        if (s) s->LA = (uint64_t *)(base + off);
        off += (size_t)kcP * 8;
        if (s) s->LB = (mode == SCG_IMI) ? (uint64_t *)(base + off) : s->LA;
        off += (mode == SCG_IMI) ? (size_t)kcP * 8 : 0;
        if (s) s->rowc = (uint16_t *)(base + off);
        off += align16((size_t)kc * 2);
        if (s) s->rowp = (uint16_t *)(base + off);
        off += align16((size_t)kc * 2);
        if (s) s->rowpre = (uint32_t *)(base + off);
        off += align16((size_t)(kc + 1) * 4);
        if (s) {
            s->hist = (uint32_t *)(base + off);
            s->ties = (uint64_t *)(base + off + (size_t)HBINS * 4);
            s->sb = (uint64_t *)(base + off);
        }
        size_t trav = (size_t)HBINS * 4 + (size_t)TIECAP * 8;
        size_t sbb = (size_t)SBCAP * 8;
        off += trav > sbb ? trav : sbb;
        end1 = off;
    }
    if (part != 1) {
        // scan phase (aliases the selection phase)
        off = phase0;
        // the radix-select bins and the tie buffer of the threshold and the
        // final merge alias the per-warp cell windows: both run between
        // scans, when no window is live
        if (s) {
            s->wwin = (CellWin *)(base + off);
            s->hist2 = (uint32_t *)(base + off);
            s->ties2 = (uint64_t *)(base + off + (size_t)RBINS * 4);
        }
        off += (size_t)NWARP * WWIN * sizeof(CellWin);
        if (s) {
            s->warm = (uint64_t *)(base + off);
            s->top = s->warm;
            s->tmp = s->warm + RMAX;
        }
        off += (size_t)WARMN * 8;
        end2 = off;
    }
    return end1 > end2 ? end1 : end2;
}

static_assert(2 * RMAX <= WARMN, "top-R buffers live inside the warm-up scores");
static_assert(2 * RMAX + 2 * NT <= WARMN, "the final merge's filtered survivors live inside the warm-up scores");
static_assert(RBINS * 4 + TIECAP * 8 <= NWARP * WWIN * sizeof(CellWin), "select bins alias the cell windows");
static_assert((1 << 10) * 4 <= NWARP * WWIN * sizeof(CellWin), "threshold bins alias the cell windows");
static_assert(WARMN % 32 == 0, "scan chunks start at multiples of 32 (the rotated LUT relies on it)");

// ---------------------------------------------------------------------------
// Block-wide helpers (NT threads, all threads must call)

__device__ __forceinline__ uint64_t warp_sum64(uint64_t v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Sums three values over the block.
__device__ void block_sum3(uint64_t &a, uint64_t &b, uint64_t &c, uint64_t *red) {
    int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    a = warp_sum64(a);
    b = warp_sum64(b);
    c = warp_sum64(c);
    __syncthreads();
    if (lane == 0) {
        red[wid] = a;
        red[NWARP + wid] = b;
        red[2 * NWARP + wid] = c;
    }
    __syncthreads();
    uint64_t x = 0, y = 0, z = 0;
    for (int i = 0; i < NWARP; i++) {
        x += red[i];
        y += red[NWARP + i];
        z += red[2 * NWARP + i];
    }
    a = x;
    b = y;
    c = z;
    __syncthreads();
}

__device__ uint64_t block_sum(uint64_t v, uint64_t *red) {
    uint64_t b = 0, c = 0;
    block_sum3(v, b, c, red);
    return v;
}

// Minimum and maximum of one u64 per thread over the block.
__device__ void block_minmax(uint64_t &mn, uint64_t &mx, uint64_t *red) {
    int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        uint64_t a = __shfl_xor_sync(0xffffffffu, mn, o);
        uint64_t b = __shfl_xor_sync(0xffffffffu, mx, o);
        mn = a < mn ? a : mn;
        mx = b > mx ? b : mx;
    }
    __syncthreads();
    if (lane == 0) {
        red[wid] = mn;
        red[NWARP + wid] = mx;
    }
    __syncthreads();
    mn = ~0ull;
    mx = 0;
    for (int i = 0; i < NWARP; i++) {
        mn = red[i] < mn ? red[i] : mn;
        mx = red[NWARP + i] > mx ? red[NWARP + i] : mx;
    }
    __syncthreads();
}

// Exclusive scan of one u64 per thread; returns the exclusive prefix and the
// block total.
__device__ uint64_t block_exscan(uint64_t v, uint64_t *red, uint64_t &total) {
    int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    uint64_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint64_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    __syncthreads();
    if (lane == 31) red[wid] = x;
    __syncthreads();
    uint64_t wpre = 0, tot = 0;
    for (int i = 0; i < NWARP; i++) {
        uint64_t r = red[i];
        if (i < wid) wpre += r;
        tot += r;
    }
    total = tot;
    __syncthreads();
    return wpre + x - v;
}

// Ascending bitonic sort of n (a power of two) u64 keys in shared memory.
// n <= NT (one key per thread) and n == 2 NT (two): keys in registers;
// partners closer than 32 are exchanged by warp shuffles, partners NT apart
// inside the thread, the rest through shared memory (two barriers per such
// stage instead of one per stage).
__device__ void bitonic_sort64(uint64_t *key, int n) {
    if (n <= NT) {
        const int t = threadIdx.x;
        uint64_t v = t < n ? key[t] : ~0ull;
        for (int k = 2; k <= n; k <<= 1) {
            for (int j = k >> 1; j > 0; j >>= 1) {
                uint64_t p;
                if (j >= 32) {
                    if (t < n) key[t] = v;
                    __syncthreads();
                    p = t < n ? key[t ^ j] : ~0ull;
                    __syncthreads();
                } else {
                    p = __shfl_xor_sync(0xffffffffu, v, j);
                }
                // the lower index of a pair keeps the minimum in ascending runs
                const bool keep_min = ((t & j) == 0) == ((t & k) == 0);
                v = keep_min ? (v < p ? v : p) : (v > p ? v : p);
            }
        }
        if (t < n) key[t] = v;
        __syncthreads();
        return;
    }
    if (n == 2 * NT) {
        // two keys per thread (indices t and t + NT): partners NT apart are
        // in the same thread, closer than 32 in the same warp
        const int t = threadIdx.x;
        uint64_t v0 = key[t], v1 = key[t + NT];
        for (int k = 2; k <= n; k <<= 1) {
            for (int j = k >> 1; j > 0; j >>= 1) {
                if (j == NT) {
                    // index t < t + NT: ascending iff (t & k) == 0 (k = 2 NT: always)
                    const uint64_t lo = v0 < v1 ? v0 : v1, hi = v0 < v1 ? v1 : v0;
                    v0 = lo;
                    v1 = hi;
                    continue;
                }
                uint64_t p0, p1;
                if (j >= 32) {
                    key[t] = v0;
                    key[t + NT] = v1;
                    __syncthreads();
                    p0 = key[t ^ j];
                    p1 = key[(t + NT) ^ j];
                    __syncthreads();
                } else {
                    p0 = __shfl_xor_sync(0xffffffffu, v0, j);
                    p1 = __shfl_xor_sync(0xffffffffu, v1, j);
                }
                const bool lower = (t & j) == 0;
                const bool min0 = lower == ((t & k) == 0), min1 = lower == (((t + NT) & k) == 0);
                v0 = min0 ? (v0 < p0 ? v0 : p0) : (v0 > p0 ? v0 : p0);
                v1 = min1 ? (v1 < p1 ? v1 : p1) : (v1 > p1 ? v1 : p1);
            }
        }
        key[t] = v0;
        key[t + NT] = v1;
        __syncthreads();
        return;
    }
    for (int k = 2; k <= n; k <<= 1) {
        for (int j = k >> 1; j > 0; j >>= 1) {
            for (int i = threadIdx.x; i < n; i += NT) {
                int ixj = i ^ j;
                if (ixj > i) {
                    uint64_t x = key[i], y = key[ixj];
                    bool up = (i & k) == 0;
                    if ((x > y) == up) {
                        key[i] = y;
                        key[ixj] = x;
                    }
                }
            }
            __syncthreads();
        }
    }
}

struct QState {
    int err;
    uint32_t s_bin;
    uint64_t s_acc;
    uint32_t kappa;
    uint32_t rank_cut;
    int take_all;
    int nties;
    uint64_t sumv, nv, nev;
    int nvis;
    int kA, kB;
    uint32_t nextA, nextB;  // smallest key outside the sorted prefix (ordered)
    // scan
    int ncur, npend;
    uint64_t thr;
    uint32_t next_flat;  // next unclaimed candidate of the scan (shared claims)
    int top_sorted;      // top[0..ncur) is already in (distance, id) order
    int handed;          // the survivors went to the merge kernel (no outputs here)
    double dens_est;     // candidates per cell seen by this CTA's last query
    uint32_t tau_gap;    // first-round tau - lowest key of that query (0: none)
    int tau_T;           // and its candidate target
    uint32_t pool_off, pool_cap;  // the query's visited-list region (selection kernel)
};

// The prefix of a coarse list: the smallest keys of L[0..n) (u64: ordered
// key << 32 | centroid id) up to and including every key equal to the m-th
// smallest, sorted ascending into L[0..c).  Returns c, or -1 when the prefix
// would exceed SBCAP (the caller then sorts the whole list).  st.nextA/B
// receives the smallest ordered key left outside.
__device__ int select_prefix(uint64_t *L, int n, int m, uint64_t *sb, uint32_t *hist, uint64_t *red,
                             QState &st, uint32_t *next_out) {
    const int tid = threadIdx.x;
    // radix select (4 x 8 bits) of the m-th smallest high word
    uint32_t prefix = 0;
    uint64_t need = (uint64_t)m;
    for (int shift = 24; shift >= 0; shift -= 8) {
        hist[tid] = 0;  // NT == 256 bins
        __syncthreads();
        for (int i = tid; i < n; i += NT) {
            uint32_t v = (uint32_t)(L[i] >> 32);
            if (shift == 24 || (v >> (shift + 8)) == (prefix >> (shift + 8))) atomicAdd(&hist[(v >> shift) & 255u], 1u);
        }
        __syncthreads();
        uint64_t cnt = hist[tid], tot;
        uint64_t ex = block_exscan(cnt, red, tot);
        if (ex < need && ex + cnt >= need) {
            st.s_bin = (uint32_t)tid;
            st.s_acc = ex;
        }
        __syncthreads();
        prefix |= st.s_bin << shift;
        need -= st.s_acc;
        __syncthreads();
    }
    const uint32_t vm = prefix;
    // compact every key with high word <= vm; smallest high word above vm
    uint64_t mine = 0, mn = ~0ull, mx = 0;
    for (int i = tid; i < n; i += NT) {
        uint32_t v = (uint32_t)(L[i] >> 32);
        if (v <= vm) mine++;
        else if (v < mn) mn = v;
    }
    block_minmax(mn, mx, red);
    uint64_t c;
    uint64_t pos = block_exscan(mine, red, c);
    if (c > (uint64_t)SBCAP) return -1;
    for (int i = tid; i < n; i += NT) {
        uint64_t k = L[i];
        if ((uint32_t)(k >> 32) <= vm) sb[pos++] = k;
    }
    int c2 = next_pow2((int)c);
    for (int i = (int)c + tid; i < c2; i += NT) sb[i] = ~0ull;
    __syncthreads();
    bitonic_sort64(sb, c2);
    for (int i = tid; i < (int)c; i += NT) L[i] = sb[i];
    if (tid == 0) *next_out = mn == ~0ull ? 0xffffffffu : (uint32_t)mn;
    __syncthreads();
    return (int)c;
}

// ---------------------------------------------------------------------------

struct Lists {
    const uint64_t *LA, *LB;
    int kA, kB;  // sorted prefix lengths
    int kc;      // codebook size (cell ids)
    bool ivf;
    __device__ __forceinline__ float a(int h) const { return o2f((uint32_t)(LA[h] >> 32)); }
    __device__ __forceinline__ float b(int h) const { return ivf ? 0.0f : o2f((uint32_t)(LB[h] >> 32)); }
    __device__ __forceinline__ uint32_t ta(int h) const { return (uint32_t)LA[h]; }
    __device__ __forceinline__ uint32_t tb(int h) const { return (uint32_t)LB[h]; }
    // number of h2 in [0, kB) with f2o(a + B[h2]) <= tau
    __device__ __forceinline__ int row_count(float av, uint32_t tau) const {
        if (f2o(__fadd_rn(av, b(0))) > tau) return 0;
        int lo = 1, hi = kB;  // answer in [1, kB]
        while (lo < hi) {
            int mid = (lo + hi + 1) >> 1;
            if (f2o(__fadd_rn(av, b(mid - 1))) <= tau) lo = mid;
            else hi = mid - 1;
        }
        return lo;
    }
};

__device__ uint64_t staircase_count(const Lists &L, uint32_t tau, uint64_t *red) {
    uint64_t c = 0;
    for (int h = threadIdx.x; h < L.kA; h += NT) {
        float av = L.a(h);
        if (f2o(__fadd_rn(av, L.b(0))) > tau) continue;
        c += (uint64_t)L.row_count(av, tau);
    }
    return block_sum(c, red);
}

// Three-list staircase of the second candidate with three nearest
// centroids (sc_query.h:265-405): rank triples (h1, h2, h3) of one sorted
// coarse list with key (A[h1] + A[h2]) + A[h3] (float adds in the reference's
// order, sc_query.h:355-390).  With L.LB == L.LA, L.row_count(base, tau) is
// the number of h3 with base + A[h3] <= tau.  The number of triples with key
// <= tau (rows (h1, h2) in parallel over h1):
__device__ uint64_t staircase3_count(const Lists &L, uint32_t tau, uint64_t *red) {
    uint64_t c = 0;
    const float a0 = L.a(0);
    for (int h1 = threadIdx.x; h1 < L.kA; h1 += NT) {
        const float a1 = L.a(h1);
        for (int h2 = 0; h2 < L.kA; h2++) {
            const float base = __fadd_rn(a1, L.a(h2));
            if (f2o(__fadd_rn(base, a0)) > tau) break;
            c += (uint64_t)L.row_count(base, tau);
        }
    }
    return block_sum(c, red);
}

// Rank triple packing of the three-list walk (kc <= 1024): lexicographic
// order of (h1, h2, h3) is the order of the packed word.
__device__ __forceinline__ uint32_t rank3(int h1, int h2, int h3) {
    return ((uint32_t)h1 << 20) | ((uint32_t)h2 << 10) | (uint32_t)h3;
}
// Cell of a rank triple: t[h1] kc^2 + t[h2] kc + t[h3] (sc_query.h:335).
__device__ __forceinline__ uint32_t cell_of3(const Lists &L, uint32_t rank) {
    const uint32_t kc = (uint32_t)L.kc;
    return (L.ta((int)(rank >> 20)) * kc + L.ta((int)((rank >> 10) & 1023u))) * kc + L.ta((int)(rank & 1023u));
}

// Radix select over the last round's records [r0, r1): the smallest key x
// with base + sum_{key <= x} weight >= need.  weight: 0 = length, 1 = one per
// cell, 2 = one per non-empty cell.
__device__ uint32_t radix_cut(const uint32_t *rk, const uint32_t *rc, int r0, int r1, uint32_t lo,
                              uint32_t hi, uint64_t base, uint64_t need, int weight, uint32_t *hist,
                              uint64_t *red, QState &st) {
    uint32_t range = hi - lo;
    int nbits = range ? 32 - __clz(range) : 0;
    uint32_t prefix = 0;
    uint64_t acc = base;
    int shift = nbits;
    while (shift > 0) {
        int db = shift < HBITS ? shift : HBITS;
        shift -= db;
        int nb = 1 << db;
        for (int i = threadIdx.x; i < nb; i += NT) hist[i] = 0;
        __syncthreads();
        int hs = shift + db;
        for (int r = r0 + threadIdx.x; r < r1; r += NT) {
            uint32_t rel = rk[r] - lo;
            if (hs < 32 && (rel >> hs) != (prefix >> hs)) continue;
            uint32_t dg = (rel >> shift) & (nb - 1);
            uint32_t c = rc[r];
            uint32_t wt = weight == 0 ? c : (weight == 1 ? 1u : (c > 0 ? 1u : 0u));
            if (wt) atomicAdd(&hist[dg], wt);
        }
        __syncthreads();
        // first bin at which acc + inclusive prefix >= need
        int per = (nb + NT - 1) / NT;
        int b0 = threadIdx.x * per;
        uint64_t mine = 0;
        for (int i = 0; i < per; i++)
            if (b0 + i < nb) mine += hist[b0 + i];
        uint64_t tot;
        uint64_t ex = block_exscan(mine, red, tot);
        uint64_t run = acc + ex;
        for (int i = 0; i < per; i++) {
            int bb = b0 + i;
            if (bb >= nb) break;
            uint64_t nxt = run + hist[bb];
            if (run < need && nxt >= need) {
                st.s_bin = (uint32_t)bb;
                st.s_acc = run;
            }
            run = nxt;
        }
        __syncthreads();
        prefix |= st.s_bin << shift;
        acc = st.s_acc;
        __syncthreads();
    }
    return lo + prefix;
}

__device__ __forceinline__ uint32_t cell_of(const Lists &L, uint32_t rank) {
    int h1 = rank >> 16, h2 = rank & 0xffff;
    return L.ivf ? L.ta(h1) : L.ta(h1) * (uint32_t)L.kc + L.tb(h2);
}

// The mp code bytes of one candidate.  MPC > 0: mp == MPC, loaded with
// 16/8/4-byte vector loads (rows are MPC-byte aligned); MPC == 0: any mp,
// byte loads on demand.
template <int MPC>
struct CodeWords {
    uint32_t w[(MPC + 3) / 4];
    __device__ __forceinline__ void load(const uint8_t *codes, uint32_t pos, int) { load_at(codes + (size_t)pos * MPC); }
    __device__ __forceinline__ void load_at(const uint8_t *p) {
        if constexpr (MPC % 16 == 0) {
#pragma unroll
            for (int i = 0; i < MPC / 16; i++) {
                uint4 v = __ldg((const uint4 *)p + i);
                w[4 * i] = v.x; w[4 * i + 1] = v.y; w[4 * i + 2] = v.z; w[4 * i + 3] = v.w;
            }
        } else if constexpr (MPC % 8 == 0) {
#pragma unroll
            for (int i = 0; i < MPC / 8; i++) {
                uint2 v = __ldg((const uint2 *)p + i);
                w[2 * i] = v.x; w[2 * i + 1] = v.y;
            }
        } else {
#pragma unroll
            for (int i = 0; i < MPC / 4; i++) w[i] = __ldg((const uint32_t *)p + i);
        }
    }
    __device__ __forceinline__ void load_smem(const unsigned char *p, int) {
        if constexpr (MPC % 16 == 0) {
#pragma unroll
            for (int i = 0; i < MPC / 16; i++) {
                uint4 v = ((const uint4 *)p)[i];
                w[4 * i] = v.x; w[4 * i + 1] = v.y; w[4 * i + 2] = v.z; w[4 * i + 3] = v.w;
            }
        } else if constexpr (MPC % 8 == 0) {
#pragma unroll
            for (int i = 0; i < MPC / 8; i++) {
                uint2 v = ((const uint2 *)p)[i];
                w[2 * i] = v.x; w[2 * i + 1] = v.y;
            }
        } else {
#pragma unroll
            for (int i = 0; i < MPC / 4; i++) w[i] = ((const uint32_t *)p)[i];
        }
    }
    __device__ __forceinline__ int n(int) const { return MPC; }
    __device__ __forceinline__ uint32_t code(int k) const { return (w[k >> 2] >> ((k & 3) * 8)) & 0xffu; }
};

template <>
struct CodeWords<0> {
    const uint8_t *p;
    __device__ __forceinline__ void load(const uint8_t *codes, uint32_t pos, int mp) { p = codes + (size_t)pos * mp; }
    __device__ __forceinline__ void load_smem(const unsigned char *q, int) { p = q; }
    __device__ __forceinline__ int n(int mp) const { return mp; }
    __device__ __forceinline__ uint32_t code(int k) const { return p[k]; }
};

// Optional per-phase cycle counters (thread 0 of each CTA), accumulated
// into a.phase_cycles[phase] when that pointer is set.
#define PHASE_MARK(i)                                                                                 \
    do {                                                                                              \
        if (a.phase_cycles && tid == 0) {                                                             \
            long long _t = clock64();                                                                 \
            atomicAdd((unsigned long long *)&a.phase_cycles[(i)], (unsigned long long)(_t - t_prev)); \
            t_prev = _t;                                                                              \
        }                                                                                             \
    } while (0)
#define COUNT(i, v)                                                                                \
    do {                                                                                           \
        if (a.phase_cycles && tid == 0)                                                            \
            atomicAdd((unsigned long long *)&a.phase_cycles[(i)], (unsigned long long)(v));        \
    } while (0)

constexpr int RK_BATCH = 8;  // words per thread in flight in the radix passes of radix_kth_word

// The k-th smallest (1-based) of n 32-bit words word(i): a radix select of
// 4 x 8 bits over RBINS = NT bins (one per thread).  Returns the word;
// `need` becomes how many entries equal to it complete the k smallest.  With
// npass < 4 only the top 8 npass bits are selected (the low bits are 0).
template <class Word>
__device__ uint32_t radix_kth_word(Word word, int n, uint64_t k, uint32_t *hist, uint64_t *red, QState &st,
                                   uint64_t &need, int npass = 4) {
    static_assert(RBINS == NT, "one bin per thread");
    const int tid = threadIdx.x;
    uint32_t prefix = 0;
    need = k;
#pragma unroll 1
    for (int sh = 24; sh >= 32 - 8 * npass; sh -= 8) {
        hist[tid] = 0;
        __syncthreads();
        // RK_BATCH words loaded before their histogram adds: the words may
        // live in global memory, and one load per add waits out a round trip
        for (int i0 = tid; i0 < n; i0 += RK_BATCH * NT) {
            uint32_t vb[RK_BATCH];
#pragma unroll
            for (int j = 0; j < RK_BATCH; j++) vb[j] = i0 + j * NT < n ? word(i0 + j * NT) : 0u;
#pragma unroll
            for (int j = 0; j < RK_BATCH; j++) {
                const uint32_t v = vb[j];
                if (i0 + j * NT < n && (sh == 24 || (v >> (sh + 8)) == (prefix >> (sh + 8))))
                    atomicAdd(&hist[(v >> sh) & 255u], 1u);
            }
        }
        __syncthreads();
        const uint64_t cnt = hist[tid];
        uint64_t tot;
        const uint64_t ex = block_exscan(cnt, red, tot);
        if (ex < need && ex + cnt >= need) {
            st.s_bin = (uint32_t)tid;
            st.s_acc = ex;
        }
        __syncthreads();
        prefix |= st.s_bin << sh;
        need -= st.s_acc;
        __syncthreads();
    }
    return prefix;
}

// An upper bound b of the k-th smallest (1-based, 1 <= k <= n) of the n
// 32-bit words word(i), n <= NT * KPT, less than 2^sbits above it: at least
// k words are <= b.  The words sit in registers (KPT per thread); radix
// passes of up to KBITS bits over the range [min, max] of the words (one
// histogram of 2^KBITS bins in `hist` per pass) narrow the k-th smallest to
// a bin of at most 2^sbits words, whose upper end is returned.  With ordered
// float words and sbits = 8 the bound is within 2^-15 relative of the k-th
// distance; on distances two or three passes suffice.
constexpr int KBITS = 10;
template <int KPT, class Word>
__device__ uint32_t block_kth_bound(Word word, int n, int k, int sbits, uint32_t *hist, uint64_t *red, QState &st) {
    __shared__ uint32_t s_red[2 * NWARP];
    const unsigned FULL = 0xffffffffu;
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    uint32_t v[KPT];
    uint32_t mn = 0xffffffffu, mx = 0u;
#pragma unroll
    for (int j = 0; j < KPT; j++) {
        const int i = tid + j * NT;
        v[j] = i < n ? word(i) : 0u;
        if (i < n) {
            mn = min(mn, v[j]);
            mx = max(mx, v[j]);
        }
    }
    mn = __reduce_min_sync(FULL, mn);
    mx = __reduce_max_sync(FULL, mx);
    __syncthreads();  // the previous call's readers of s_red are done
    if (lane == 0) {
        s_red[wid] = mn;
        s_red[NWARP + wid] = mx;
    }
    __syncthreads();
#pragma unroll
    for (int w2 = 0; w2 < NWARP; w2++) {
        mn = min(mn, s_red[w2]);
        mx = max(mx, s_red[NWARP + w2]);
    }
    const uint32_t range = mx - mn;
    int shift = range ? 32 - __clz(range) : 0;  // unresolved low bits of (word - min)
    uint32_t prefix = 0;                        // resolved high bits of (word - min)
    uint32_t need = (uint32_t)k;
    while (shift > sbits) {
        const int db = shift < KBITS ? shift : KBITS, hs = shift;
        shift -= db;
        const uint32_t nbins = 1u << db;
        for (uint32_t b = (uint32_t)tid; b < nbins; b += NT) hist[b] = 0u;
        __syncthreads();
#pragma unroll
        for (int j = 0; j < KPT; j++) {
            const uint32_t rel = v[j] - mn;
            const bool in = tid + j * NT < n && (hs >= 32 || (rel >> hs) == (prefix >> hs));
            if (in) atomicAdd(&hist[(rel >> shift) & (nbins - 1u)], 1u);
        }
        __syncthreads();
        // the bin holding the need-th word: bins split evenly over the threads
        constexpr int PB = (1 << KBITS) / NT;
        const uint32_t b0 = (uint32_t)tid * PB;
        uint32_t c[PB], mine = 0;
#pragma unroll
        for (int i = 0; i < PB; i++) {
            c[i] = b0 + i < nbins ? hist[b0 + i] : 0u;
            mine += c[i];
        }
        uint64_t tot;
        uint32_t run = (uint32_t)block_exscan(mine, red, tot);
#pragma unroll
        for (int i = 0; i < PB; i++) {
            if (run < need && run + c[i] >= need) {
                st.s_bin = b0 + (uint32_t)i;
                st.s_acc = run;
            }
            run += c[i];
        }
        __syncthreads();
        prefix |= st.s_bin << shift;
        need -= (uint32_t)st.s_acc;
        __syncthreads();
    }
    const uint64_t b = (uint64_t)mn + prefix + ((1ull << shift) - 1ull);
    return b < (uint64_t)mx ? (uint32_t)b : mx;
}

// The R smallest (distance, id) keys of nb pending entries by one bitonic
// sort in top[] (room for WARMN keys, nb <= WARMN), in order; pid != null
// turns the entries' CSR positions into ids first.
__device__ void sort_merge(uint64_t *top, const uint64_t *pend, int nb, int R, const int *pid, QState &st) {
    const int tid = threadIdx.x;
    const int n2 = next_pow2(nb > 1 ? nb : 1);
    for (int i = tid; i < n2; i += NT) {
        uint64_t e = ~0ull;
        if (i < nb) {
            e = pend[i];
            if (pid) e = (e & 0xffffffff00000000ull) | (uint32_t)__ldg(pid + (uint32_t)e);
        }
        top[i] = e;
    }
    __syncthreads();
    if (n2 > 1) bitonic_sort64(top, n2);
    if (tid == 0) {
        st.ncur = nb < R ? nb : R;
        st.npend = 0;
        st.thr = nb < R ? ~0ull : top[R - 1];
        st.top_sorted = 1;
    }
    __syncthreads();
}

// Keeps the R smallest of top[0..ncur) and the pending entries.  Pending
// entries hold (distance, CSR position); the kept ones and those tied at the
// R-th distance become (distance, id) here.  A radix select
// over the distance words finds the R-th smallest distance v; every entry
// below v is kept and the entries equal to v are taken in id order.  The top
// list stays unsorted (the output step sorts it); st.thr becomes the R-th
// smallest (distance, id) once R entries exist.  More than TIECAP entries
// equal to v: the pending buffer is merged again by one sort (sort_merge)
// when it fits, else ST_TIE_OVERFLOW is raised.
__device__ void merge_topk(uint64_t *top, uint64_t *pend, uint64_t *tmp, uint32_t *hist, uint64_t *ties, int R,
                           const int *pid, uint64_t *red, QState &st, int *status) {
    const int tid = threadIdx.x;
    const int na = st.ncur, nb = st.npend;
    // (distance, id) of entry i: top entries carry ids already, pending ones
    // carry CSR positions until they are kept (the id loads of the entries
    // the merge drops are never issued)
    auto as_id = [&](uint64_t e) -> uint64_t {
        return pid ? (e & 0xffffffff00000000ull) | (uint32_t)__ldg(pid + (uint32_t)e) : e;
    };
    const int n = na + nb;
    if (n <= R) {
        for (int i = tid; i < nb; i += NT) top[na + i] = as_id(pend[i]);
        __syncthreads();
        if (tid == 0) {
            st.ncur = n;
            st.npend = 0;
            st.thr = ~0ull;
        }
        __syncthreads();
        return;
    }
    if (na == 0 && nb <= NT) {
        // few survivors: one register sort of (distance, id) keys gives the R
        // best in order
        sort_merge(top, pend, nb, R, pid, st);
        return;
    }
    if (na == 0 && nb <= NT * MERGE_KPT) {
        // an upper bound b of the R-th distance (within 2^-15) keeps every
        // entry of the R best and few others; those are sorted as above
        auto word = [&](int i) { return (uint32_t)(pend[i] >> 32); };
        const uint32_t b = nb <= 2 * NT ? block_kth_bound<2>(word, nb, R, 8, hist, red, st)
                                        : block_kth_bound<MERGE_KPT>(word, nb, R, 8, hist, red, st);
        uint64_t mine = 0;
        for (int i = tid; i < nb; i += NT) mine += (uint32_t)(pend[i] >> 32) <= b;
        uint64_t total;
        uint64_t pos = block_exscan(mine, red, total);
        if (total <= (uint64_t)(2 * NT)) {
            uint64_t *fil = tmp + RMAX;  // past the top and tmp lists, inside the warm-up scores
            for (int i = tid; i < nb; i += NT) {
                const uint64_t e = pend[i];
                if ((uint32_t)(e >> 32) <= b) fil[pos++] = e;
            }
            __syncthreads();
            sort_merge(top, fil, (int)total, R, pid, st);
            return;
        }
        // many entries within 2^-15 of the R-th distance: the radix select below
    }
    // radix select of the R-th smallest distance word
    uint64_t need;
    const uint32_t prefix = radix_kth_word(
        [&](int i) { return (uint32_t)((i < na ? top[i] : pend[i - na]) >> 32); }, n, (uint64_t)R, hist, red, st,
        need);
    const uint32_t v = prefix;
    // keep everything below v; gather the entries equal to v
    uint64_t mine = 0;
    for (int i0 = tid; i0 < n; i0 += RK_BATCH * NT) {
        uint32_t hb[RK_BATCH];
#pragma unroll
        for (int j = 0; j < RK_BATCH; j++) {
            const int i = i0 + j * NT;
            hb[j] = i < n ? (uint32_t)((i < na ? top[i] : pend[i - na]) >> 32) : 0xffffffffu;
        }
#pragma unroll
        for (int j = 0; j < RK_BATCH; j++) mine += hb[j] < v;
    }
    uint64_t total;
    uint64_t pos = block_exscan(mine, red, total);
    if (tid == 0) st.nties = 0;
    __syncthreads();
    // the same entries in the same order per thread as the count above, so
    // that pos runs through this thread's range of the exclusive scan
    for (int i0 = tid; i0 < n; i0 += RK_BATCH * NT) {
        uint64_t eb[RK_BATCH];
#pragma unroll
        for (int j = 0; j < RK_BATCH; j++) {
            const int i = i0 + j * NT;
            eb[j] = i < n ? (i < na ? top[i] : pend[i - na]) : ~0ull;
        }
#pragma unroll
        for (int j = 0; j < RK_BATCH; j++) {
            const int i = i0 + j * NT;
            if (i >= n) continue;
            const uint64_t e = eb[j];
            const uint32_t hv = (uint32_t)(e >> 32);
            if (hv < v) tmp[pos++] = i < na ? e : as_id(e);
            else if (hv == v) {
                int slot = atomicAdd(&st.nties, 1);
                if (slot < TIECAP) ties[slot] = i < na ? e : as_id(e);
            }
        }
    }
    __syncthreads();
    const bool resort = st.nties > TIECAP && na == 0 && nb <= WARMN;
    if (resort) {
        // the tie buffer kept only some of the entries equal to v
        __syncthreads();
        sort_merge(top, pend, nb, R, pid, st);
        return;
    }
    if (tid == 0) {
        // `need` entries equal to v complete the R: the smallest ids
        int nt = st.nties < TIECAP ? st.nties : TIECAP;
        for (int i = 1; i < nt; i++) {
            uint64_t x = ties[i];
            int j = i - 1;
            while (j >= 0 && ties[j] > x) {
                ties[j + 1] = ties[j];
                j--;
            }
            ties[j + 1] = x;
        }
        int take = (int)need;
        if (st.nties > TIECAP) {
            // more equal distances at the R-th place than the tie buffer holds
            atomicOr(status, ST_TIE_OVERFLOW);
            if (take > nt) take = nt;
        }
        for (int i = 0; i < take; i++) tmp[total + i] = ties[i];
        st.ncur = (int)total + take;
        st.npend = 0;
        st.thr = take > 0 ? ties[take - 1] : ~0ull;
    }
    __syncthreads();
    for (int i = tid; i < st.ncur; i += NT) top[i] = tmp[i];
    __syncthreads();
}

// Everything the candidate scan needs about one query.
struct ScanCtx {
    const uint32_t *vis_cell, *vis_pre;
    int nvis;
    uint32_t Svis;
    int kc, mp, kp, bsI;
    uint32_t cdiv;  // second candidate: cell / cdiv is the residual's centroid (kc, or kc^2 with three)
    bool imi, sc, fast, rot;
    float qs;
    const float *dqc;
    // exact-distance scan (raw_dim > 0): the query in shared memory, raw rows
    // by id (uint8 or float; raw_vec: rows read 16 bytes at a time)
    int raw_dim;
    bool raw_u8, raw_vec;
    const float *qv;
    // survivor slots below scap go to sq (the query's hand-off to the merge
    // kernel), the others to the pending buffer
    uint64_t *sq;
    uint32_t scap;
};

// The MPC / 4 code words of one candidate with word i moved to i ^ xw (log
// steps of selects on a lane-constant xw): word (s ^ x) / 4 of the code is
// then word s / 4 of the result.
template <int MPC>
__device__ __forceinline__ void permute_words(const uint32_t *w, uint32_t *r, uint32_t xw) {
    constexpr int n = MPC / 4;
#pragma unroll
    for (int i = 0; i < n; i++) r[i] = w[i];
#pragma unroll
    for (int b = 1; b < n; b <<= 1) {
        const bool on = (xw & (uint32_t)b) != 0;
        uint32_t x[n];
#pragma unroll
        for (int i = 0; i < n; i++) x[i] = r[i ^ b];
#pragma unroll
        for (int i = 0; i < n; i++) r[i] = on ? x[i] : r[i];
    }
}

// The fast form's table sum of one candidate: a tree over the n entries
// (pairs (k, k + 1), then (k, k + 2), ...), its two halves summed side by
// side with packed two-wide adds (add.rn.f32x2: each element an ordinary
// round-to-nearest add, so the float is the one of scalar adds in the same
// tree), then one add of the halves.
template <int N>
__device__ __forceinline__ float tree_sum(float (&v)[N]) {
    if constexpr (N < 4) {
#pragma unroll
        for (int s2 = 1; s2 < N; s2 <<= 1)
#pragma unroll
            for (int k = 0; k + s2 < N; k += 2 * s2) v[k] = __fadd_rn(v[k], v[k + s2]);
        return v[0];
    } else {
        constexpr int H = N / 2;
        uint64_t p[H];
#pragma unroll
        for (int j = 0; j < H; j++) asm("mov.b64 %0, {%1, %2};" : "=l"(p[j]) : "f"(v[j]), "f"(v[j + H]));
#pragma unroll
        for (int s2 = 1; s2 < H; s2 <<= 1)
#pragma unroll
            for (int k = 0; k + s2 < H; k += 2 * s2) asm("add.rn.f32x2 %0, %0, %1;" : "+l"(p[k]) : "l"(p[k + s2]));
        float lo, hi;
        asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(p[0]));
        return __fadd_rn(lo, hi);
    }
}

// One float of shared memory at a 32-bit shared-window address.
__device__ __forceinline__ float lds_f32(uint32_t addr) {
    float v;
    asm volatile("ld.shared.f32 %0, [%1];" : "=f"(v) : "r"(addr));
    return v;
}

// Sum of the LUT entries of one candidate's code words `w` on the
// bank-private LUT (see scan_chunks): word permutation by xl / 4, then per
// step s the byte select, the lane's bank of table s ^ xl and one LDS; the
// entries summed as a tree over s (the same float as the tree over k).
template <int MPC>
__device__ __forceinline__ float rot_lut_sum(const uint32_t *w, const uint32_t *roff, const uint32_t *bsel, uint32_t xl,
                                             uint32_t lut_s, int lane) {
    uint32_t pw[MPC / 4];
    permute_words<MPC>(w, pw, xl >> 2);
    float v[MPC];
#pragma unroll
    for (int s2 = 0; s2 < MPC; s2++) {
        // code byte s2 ^ x: word (s2 ^ x) / 4 = pw[s2 / 4]
        const uint32_t cb = __byte_perm(pw[s2 >> 2], 0u, bsel[s2 & 3]);
        uint32_t ro;
        if constexpr (MPC <= 16) ro = roff[s2];
        else ro = lut_s + (((uint32_t)lane - xl + ((uint32_t)s2 ^ xl)) << 2);
        v[s2] = lds_f32(ro + (cb << 7));
    }
    return tree_sum<MPC>(v);
}

// Warp-centric ADC scan of the candidates [first, limit), cut into chunks of
// 32 * U candidates.  FK (the fast form with kp == 256): every warp takes an
// equal, contiguous run of chunks, so it walks its visited cells in order.
// Otherwise warps claim chunks from a shared counter (st.next_flat, set to
// `first` by the caller), which keeps the warps of a CTA on neighbouring
// cells: the exact forms gather dot_cr rows per cell, and neighbouring cells
// share rows in L1.  A warp keeps a window of WWIN visited cells; when the
// scan leaves it at its end the next WWIN cells are loaded, otherwise a
// binary search over the visited-cell prefix finds the cell that holds the
// chunk.  U candidates per lane are loaded at once and the table entries are
// added in the reference's order (exact forms) or as a tree (fast form).
//
// The fast form with kp == 256 and mp in {8, 16, 32} (ScanCtx::rot) reads a
// bank-private LUT: bank b holds table b mod mp (32 / mp copies), and at
// step s lane l reads table k = s ^ x, x = l mod mp, from bank
// (l - x) + k, so the 32 lookups of a warp hit 32 different banks (no
// conflicts).  The lane permutes its code's words by x / 4 first, so that a
// byte select with a lane-constant selector gives code byte k.  Summed as a
// tree over s, step pairs (s, s ^ 1), (s, s ^ 2), ... hold exactly the table
// pairs of the tree over k, so with commutative adds the sum is the same
// float for every lane -- identical codes in one cell give identical
// distances, and all kernels agree.
//
// The exact-distance variant (VAR == V_EXACT, rerank = -1) scores each
// candidate by the distance_l2_square of its raw row instead.
//
// WARM == true stores every candidate's (distance, position) at warm[flat];
// otherwise candidates with a distance word <= tau are appended to out[]
// (global, capacity cap) through warp-aggregated atomics on st.npend.
template <int MPC, bool WARM, int U, int VAR, bool ROTOK>
__device__ __forceinline__ void scan_chunks(const SearchArgs &a, const Smem &S, QState &st, const ScanCtx &c,
                                            uint32_t first, uint32_t limit, uint32_t tau, uint64_t *warm,
                                            uint64_t *out, uint32_t cap) {
    const unsigned FULL = 0xffffffffu;
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    CellWin *W = S.wwin + wid * WWIN;
    const uint32_t lut_s = (uint32_t)__cvta_generic_to_shared(S.lut);
    constexpr bool FK = VAR == V_FAST256;
    constexpr bool KP256 = FK && MPC > 0;
    // ROTOK: the kernel can meet the bank-private LUT (the fused kernel and
    // the fast form's scan-only kernel; the general scan-only kernel never)
    constexpr bool ROTC = ROTOK && (MPC == 8 || MPC == 16 || MPC == 32);
    constexpr bool rawm = VAR == V_EXACT;
    const bool fast = FK || c.fast;
    const bool rot = ROTC && (FK || c.rot);
    // bank-private LUT: this lane's shared address of step s (mp <= 16: kept
    // in registers; mp == 32: computed per lookup) and the byte selectors of
    // code byte (4 j) ^ x within a permuted word
    const uint32_t xl = (uint32_t)lane & (ROTC ? MPC - 1 : 0);
    constexpr int NROFF = (ROTC && MPC <= 16) ? MPC : 1;
    uint32_t roff[NROFF], bsel[4];
    if constexpr (ROTC && MPC <= 16) {
#pragma unroll
        for (int s2 = 0; s2 < MPC; s2++)
            roff[s2] = lut_s + (((uint32_t)lane - xl + ((uint32_t)s2 ^ xl)) << 2);
    }
#pragma unroll
    for (int j = 0; j < 4; j++) bsel[j] = 0x4440u | ((uint32_t)j ^ (xl & 3u));
    uint32_t whi = 0;
    int wcn = 0, wci = -1;
    // this lane's window index: candidates only move forward within a window,
    // so the cell lookup resumes where the last one stopped; the current cell
    // is cached in registers ([r_pre, r_next) of the flat candidate index)
    int ci_l = 0;
    uint32_t r_pre = 0, r_next = 0, r_start = 0, r_h34 = 0;
    float r_d0 = 0.0f;
    constexpr uint32_t WCH = 32u * U;
    // FK: this warp's run of chunks
    const uint64_t nch = limit > first ? ((uint64_t)(limit - first) + WCH - 1) / WCH : 0;
    const uint64_t per = (nch + NWARP - 1) / NWARP;
    const uint64_t lo64 = (uint64_t)first + (uint64_t)wid * per * WCH;
    const uint32_t hi = FK ? (uint32_t)min(lo64 + per * WCH, (uint64_t)limit) : limit;
    uint32_t next = (uint32_t)min(lo64, (uint64_t)limit);
    for (;;) {
        uint32_t base;
        if constexpr (FK) {
            base = next;
            next += WCH;
        } else {
            base = 0;
            if (lane == 0) base = atomicAdd(&st.next_flat, WCH);
            base = __shfl_sync(FULL, base, 0);
        }
        if (base >= hi) break;
        const uint32_t end = min(base + WCH, hi);
        uint32_t f = base;
        while (f < end) {
            if (f >= whi) {
                // window of visited cells from the one holding f (f only
                // grows): the next WWIN cells when f is the old window's end
                int ci = 0;
                if (wci >= 0 && f == whi) {
                    ci = wci + wcn;
                } else {
                    if (lane == 0) {
                        int lo2 = 0, hi2 = c.nvis - 1;
                        while (lo2 < hi2) {
                            int mid = (lo2 + hi2 + 1) >> 1;
                            if (c.vis_pre[mid] <= f) lo2 = mid;
                            else hi2 = mid - 1;
                        }
                        ci = lo2;
                    }
                    ci = __shfl_sync(FULL, ci, 0);
                }
                __syncwarp();  // the previous window's readers are done
                const int cc = ci + lane;
                if (cc < c.nvis) {
                    uint32_t cell = c.vis_cell[cc];
                    CellWin cw;
                    cw.pre = c.vis_pre[cc];
                    cw.start = a.off[cell];
                    uint32_t h3, h4;
                    if (c.imi) {
                        h3 = cell / (uint32_t)c.kc;
                        h4 = cell - h3 * (uint32_t)c.kc;
                        cw.d0 = __fadd_rn(__fadd_rn(c.qs, c.dqc[h3]), c.dqc[c.kc + h4]);
                    } else if (c.sc) {
                        h3 = cell / c.cdiv;
                        h4 = 0;
                        cw.d0 = __fadd_rn(c.qs, c.dqc[h3]);
                    } else {
                        h3 = cell;
                        h4 = 0;
                        cw.d0 = __fadd_rn(c.qs, c.dqc[h3]);
                    }
                    cw.h34 = h3 | (h4 << 16);
                    W[lane] = cw;
                }
                wci = ci;
                wcn = min(WWIN, c.nvis - ci);
                __syncwarp();
                whi = (ci + wcn < c.nvis) ? c.vis_pre[ci + wcn] : c.Svis;
                ci_l = 0;
                r_next = 0;  // the cached cell belongs to the old window
            }
            const uint32_t e2 = min(end, whi);
            // loads of U candidates per lane, issued together
            uint32_t pos[U], h34[U];
            float dd[U], vt[U];
            CodeWords<MPC> cwd[U];
            int ci = ci_l;
#pragma unroll
            for (int u = 0; u < U; u++) {
                const uint32_t ff = f + lane + 32u * u;
                pos[u] = 0xffffffffu;
                if (ff < e2) {
                    if (ff >= r_next || ff < r_pre) {
                        while (ci + 1 < wcn && W[ci + 1].pre <= ff) ci++;
                        const CellWin cw = W[ci];
                        r_pre = cw.pre;
                        r_start = cw.start;
                        r_d0 = cw.d0;
                        r_h34 = cw.h34;
                        r_next = (ci + 1 < wcn) ? W[ci + 1].pre : whi;
                    }
                    pos[u] = r_start + (ff - r_pre);
                    dd[u] = r_d0;
                    h34[u] = r_h34;
                    if (!rawm) {
                        cwd[u].load(a.codes, pos[u], c.mp);
                        if (fast) vt[u] = __ldg(a.vterm + pos[u]);
                    }
                }
            }
            ci_l = ci;
#pragma unroll
            for (int u = 0; u < U; u++) {
                bool pass = false;
                uint32_t du = 0;
                if (pos[u] != 0xffffffffu) {
                    float d = dd[u];
                    const uint32_t h3 = h34[u] & 0xffffu, h4 = h34[u] >> 16;
                    if (rawm) {
                        // the real_dist branch (query.h:307-312,
                        // multi_query.h:255-259, sc_query.h:232-236): the
                        // exact distance of the candidate's raw row
                        const int id = __ldg(a.pid + pos[u]);
                        d = c.raw_u8 ? exact_dist_row(c.qv, (const uint8_t *)a.raw + (size_t)id * c.raw_dim, c.raw_dim,
                                                      c.raw_vec)
                                     : exact_dist_row(c.qv, (const float *)a.raw + (size_t)id * c.raw_dim, c.raw_dim,
                                                      c.raw_vec);
                    } else if (fast) {
                        // d0 + per-vector term + sum_k LUT[k][c_k], the LUT
                        // entries summed as a tree (independent adds)
                        d = __fadd_rn(d, vt[u]);
                        bool done = false;
                        if constexpr (ROTC) {
                            if (rot) {
                                d = __fadd_rn(d, rot_lut_sum<MPC>(cwd[u].w, roff, bsel, xl, lut_s, lane));
                                done = true;
                            }
                        }
                        if (!done) {
                            if constexpr (MPC > 0) {
                                float v[MPC];
                                if constexpr (KP256) {
#pragma unroll
                                    for (int k = 0; k < MPC; k++)
                                        v[k] = lds_f32(lut_s + (cwd[u].code(k) << 2) + (uint32_t)k * 1024u);
                                } else {
#pragma unroll
                                    for (int k = 0; k < MPC; k++) v[k] = S.lut[k * c.kp + cwd[u].code(k)];
                                }
                                d = __fadd_rn(d, tree_sum<MPC>(v));
                            } else {
                                for (int k = 0; k < cwd[u].n(c.mp); k++)
                                    d = __fadd_rn(d, S.lut[k * c.kp + cwd[u].code(k)]);
                            }
                        }
                    } else if (c.imi) {
                        // multi_query.h:237-254: two adds per subspace
                        const int half = c.mp >> 1;
                        const float *r1 = a.dot_cr + (size_t)h3 * c.bsI;
                        const float *r2 = a.dot_cr + (size_t)(h4 + c.kc - 1) * c.bsI;
                        for (int k = 0; k < cwd[u].n(c.mp); k++) {
                            int bc = k * c.kp + cwd[u].code(k);
                            d = __fadd_rn(d, S.lut[bc]);
                            d = __fadd_rn(d, __ldg((k < half ? r1 : r2) + bc));
                        }
                    } else {
                        // query.h:295-306, sc_query.h:222-229: pair sum per subspace
                        const float *r1 = a.dot_cr + (size_t)h3 * c.bsI;
                        for (int k = 0; k < cwd[u].n(c.mp); k++) {
                            int bc = k * c.kp + cwd[u].code(k);
                            d = __fadd_rn(d, __fadd_rn(S.lut[bc], __ldg(r1 + bc)));
                        }
                    }
                    du = f2o(d);
                    if (WARM) warm[f + lane + 32u * u] = ((uint64_t)du << 32) | pos[u];
                    else pass = du <= tau;
                }
                if (!WARM) {
                    const unsigned m = __ballot_sync(FULL, pass);
                    if (m) {
                        uint32_t slot0 = 0;
                        if (lane == __ffs(m) - 1) slot0 = atomicAdd((unsigned *)&st.npend, (unsigned)__popc(m));
                        slot0 = __shfl_sync(FULL, slot0, __ffs(m) - 1);
                        const uint32_t slot = slot0 + __popc(m & ((1u << lane) - 1));
                        if (pass && slot < cap) (slot < c.scap ? c.sq : out)[slot] = ((uint64_t)du << 32) | pos[u];
                    }
                }
            }
            f = e2;
        }
    }
}

// The fast form's scan-only kernel with kp == 256 and mp in {8, 16, 32}: each
// warp takes an equal, contiguous run of the candidates [first, limit) and
// walks it cell by cell, so the cell is the same for the whole warp.  Each
// cell's candidates go in chunks of 32 * U (lane l takes the chunk's
// candidates l, l + 32, ...): a full chunk loads from one base at immediate
// offsets; the cell's last, partial chunk clamps positions to the cell and
// masks its distances.  Distances are d0 + per-vector term + the
// bank-private LUT sum (rot_lut_sum), the same floats as in scan_chunks.
// Cells come from the warp's window of WWIN visited cells in shared memory.
// WARM == true stores every candidate's (distance, position) at
// warm[flat]; otherwise candidates with a distance at or below tau are
// appended to out[] through warp-aggregated atomics on st.npend.
template <int MPC, bool WARM, int U>
__device__ __forceinline__ void scan_cells(const SearchArgs &a, const Smem &S, QState &st, const ScanCtx &c,
                                           uint32_t first, uint32_t limit, uint32_t tau, uint64_t *warm,
                                           uint64_t *out, uint32_t cap) {
    static_assert(MPC == 8 || MPC == 16 || MPC == 32, "bank-private LUT widths");
    const unsigned FULL = 0xffffffffu;
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    CellWin *W = S.wwin + wid * WWIN;
    const uint32_t lut_s = (uint32_t)__cvta_generic_to_shared(S.lut);
    const uint32_t xl = (uint32_t)lane & (MPC - 1);
    constexpr int NROFF = MPC <= 16 ? MPC : 1;
    uint32_t roff[NROFF], bsel[4];
    if constexpr (MPC <= 16) {
#pragma unroll
        for (int s2 = 0; s2 < MPC; s2++) roff[s2] = lut_s + (((uint32_t)lane - xl + ((uint32_t)s2 ^ xl)) << 2);
    }
#pragma unroll
    for (int j = 0; j < 4; j++) bsel[j] = 0x4440u | ((uint32_t)j ^ (xl & 3u));
    const float tauf = tau == 0xffffffffu ? __int_as_float(0x7f800000) : o2f(tau);
    constexpr uint32_t WCH = 32u * U;
    // this warp's run
    const uint64_t nch = limit > first ? ((uint64_t)(limit - first) + WCH - 1) / WCH : 0;
    const uint64_t per = (nch + NWARP - 1) / NWARP;
    const uint64_t lo64 = (uint64_t)first + (uint64_t)wid * per * WCH;
    const uint32_t hi = (uint32_t)min(lo64 + per * WCH, (uint64_t)limit);
    uint32_t f = (uint32_t)min(lo64, (uint64_t)limit);
    if (f >= hi) return;
    // the visited cell holding f
    int ci = 0;
    if (lane == 0) {
        int lo2 = 0, hi2 = c.nvis - 1;
        while (lo2 < hi2) {
            const int mid = (lo2 + hi2 + 1) >> 1;
            if (c.vis_pre[mid] <= f) lo2 = mid;
            else hi2 = mid - 1;
        }
        ci = lo2;
    }
    ci = __shfl_sync(FULL, ci, 0);
    int wci = 0, wcn = 0;
    uint32_t whi = 0;
    while (f < hi) {
        if (ci >= wci + wcn) {
            // the next window of visited cells, from ci
            __syncwarp();  // the previous window's readers are done
            const int cc = ci + lane;
            if (cc < c.nvis) {
                const uint32_t cell = c.vis_cell[cc];
                CellWin cw;
                cw.pre = c.vis_pre[cc];
                cw.start = a.off[cell];
                if (c.imi) {
                    const uint32_t h3 = cell / (uint32_t)c.kc, h4 = cell - h3 * (uint32_t)c.kc;
                    cw.d0 = __fadd_rn(__fadd_rn(c.qs, c.dqc[h3]), c.dqc[c.kc + h4]);
                } else {
                    cw.d0 = __fadd_rn(c.qs, c.dqc[c.sc ? cell / c.cdiv : cell]);
                }
                cw.h34 = 0;
                W[lane] = cw;
            }
            wci = ci;
            wcn = min(WWIN, c.nvis - ci);
            __syncwarp();
            whi = (ci + wcn < c.nvis) ? c.vis_pre[ci + wcn] : c.Svis;
        }
        const CellWin cw = W[ci - wci];
        const uint32_t cnext = (ci + 1 < wci + wcn) ? W[ci - wci + 1].pre : whi;
        const uint32_t cend = min(cnext, hi);
        const float d0 = cw.d0;
        // one chunk of 32 * U candidates from g; FULLC: all inside the cell
        auto chunk = [&](uint32_t g, auto fullc) {
            constexpr bool FULLC = decltype(fullc)::value;
            const uint32_t ff0 = g + lane;
            const uint32_t p0 = cw.start + (ff0 - cw.pre);
            CodeWords<MPC> cwd[U];
            float dist[U];
            if constexpr (FULLC) {
                const uint8_t *cp = a.codes + (size_t)p0 * MPC;
                const float *vp = a.vterm + p0;
#pragma unroll
                for (int u = 0; u < U; u++) {
                    cwd[u].load_at(cp + (size_t)u * 32u * MPC);
                    dist[u] = __ldg(vp + 32u * u);
                }
            } else {
                // the cell's last chunk: positions clamped to the cell
                const uint32_t plast = cw.start + (cend - 1u - cw.pre);
#pragma unroll
                for (int u = 0; u < U; u++) {
                    const uint32_t pu = min(p0 + 32u * u, plast);
                    cwd[u].load(a.codes, pu, MPC);
                    dist[u] = __ldg(a.vterm + pu);
                }
            }
            uint32_t pm = 0;  // bit u: this lane's u-th candidate is at or below tau
#pragma unroll
            for (int u = 0; u < U; u++) {
                const bool act = FULLC || ff0 + 32u * u < cend;
                dist[u] = __fadd_rn(__fadd_rn(d0, dist[u]), rot_lut_sum<MPC>(cwd[u].w, roff, bsel, xl, lut_s, lane));
                if constexpr (WARM) {
                    if (act) warm[ff0 + 32u * u] = ((uint64_t)f2o(dist[u]) << 32) | (p0 + 32u * u);
                } else {
                    pm |= (act && dist[u] <= tauf ? 1u : 0u) << u;
                }
            }
            if constexpr (!WARM) {
                if (__any_sync(FULL, pm != 0u)) {
                    // the chunk's survivors: one atomic for the warp, slots
                    // in (u, lane) order
                    unsigned m[U];
                    uint32_t tot = 0;
#pragma unroll
                    for (int u = 0; u < U; u++) {
                        m[u] = __ballot_sync(FULL, (pm >> u) & 1u);
                        tot += (uint32_t)__popc(m[u]);
                    }
                    uint32_t base = 0;
                    if (lane == 0) base = atomicAdd((unsigned *)&st.npend, tot);
                    base = __shfl_sync(FULL, base, 0);
                    const uint32_t lt = (1u << lane) - 1u;
#pragma unroll
                    for (int u = 0; u < U; u++) {
                        const uint32_t slot = base + (uint32_t)__popc(m[u] & lt);
                        if (((pm >> u) & 1u) && slot < cap)
                            (slot < c.scap ? c.sq : out)[slot] = ((uint64_t)f2o(dist[u]) << 32) | (p0 + 32u * u);
                        base += (uint32_t)__popc(m[u]);
                    }
                }
            }
        };
        uint32_t g = f;
        for (; g + WCH <= cend; g += WCH) chunk(g, std::true_type{});
        if (g < cend) chunk(g, std::false_type{});
        f = cend;
        ci++;
    }
}

// Resident CTAs per SM the register allocation is sized for.
#ifndef SCG_SEARCH_MIN_BLOCKS
#define SCG_SEARCH_MIN_BLOCKS 2
#endif
// ... of the selection-only kernel (part 1) and of the scan-only kernel (part 2).
#ifndef SCG_SELECT_MIN_BLOCKS
#define SCG_SELECT_MIN_BLOCKS 5
#endif
#ifndef SCG_SCAN_MIN_BLOCKS
#define SCG_SCAN_MIN_BLOCKS 4
#endif
// ... of the fast form's scan-only kernel (its 32 KB rotated LUT leaves room
// for fewer CTAs, each with more registers)
#ifndef SCG_SCAN_FK_MIN_BLOCKS
#define SCG_SCAN_FK_MIN_BLOCKS 3
#endif

// PART 0: selection and scan fused; 1: selection only, publishing each
// query's visited cells (a.qmeta, a.pool_*); 2: scan only, from them.  FK:
// the scan-only kernel of the fast form with kp == 256 (scan_chunks).
template <int MPC, int U, int PART, int VAR = V_ADC>
__global__ void __launch_bounds__(NT, PART == 2   ? (VAR == V_FAST256 ? SCG_SCAN_FK_MIN_BLOCKS : SCG_SCAN_MIN_BLOCKS)
                                      : PART == 1 ? SCG_SELECT_MIN_BLOCKS
                                                  : SCG_SEARCH_MIN_BLOCKS) k_search(SearchArgs a) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ uint64_t red[3 * NWARP];
    __shared__ QState st;
    __shared__ int s_q;
    Smem S;
    carve(a.mode, a.kc, a.mp, a.kp, PART, a.rot, a.raw_dim, &S, smem);
    const int tid = threadIdx.x;
    const int kc = a.kc, mp = a.mp, kp = a.kp;
    const int kcP = next_pow2(kc);
    const bool imi = a.mode == SCG_IMI, sc = a.mode == SCG_SC2, ivf = a.mode == SCG_IVFADC;
    // the three-list walk (fused kernel only): like sc for the w rule, the
    // cell-0 rule and the residual's centroid
    const bool sc3 = a.mode == SCG_SC3, scx = sc || sc3;
    const bool fast = a.precision == SCG_FAST;
    const int kBfull = ivf ? 1 : kc;
    const int cap = a.cap_rec;
    uint32_t *rec_key = a.rec_key + (size_t)blockIdx.x * cap;
    uint32_t *rec_rank = a.rec_rank + (size_t)blockIdx.x * cap;
    uint32_t *rec_cnt = a.rec_cnt + (size_t)blockIdx.x * cap;
    uint32_t *vis_cell = a.vis_cell ? a.vis_cell + (size_t)blockIdx.x * (cap + 1) : nullptr;
    uint32_t *vis_pre = a.vis_pre ? a.vis_pre + (size_t)blockIdx.x * (cap + 1) : nullptr;
    uint32_t *hist = S.hist;
    uint64_t *ties = S.ties;
    uint64_t *sb = S.sb;  // sorted coarse prefix scratch
    const int bsI = kp * mp / a.mc;  // dot_cr block of one coarse centroid
    const double avg_density = (double)a.N / (double)(a.ncells ? a.ncells : 1);

    if (tid == 0) {
        st.dens_est = 0.0;
        st.tau_gap = 0u;
        st.tau_T = 0;
    }
    for (;;) {
        if (tid == 0) {
            // a query list (the queries the warp-wide selection deferred):
            // qlist[0] entries follow it; else the whole batch
            const int i = atomicAdd(a.qcounter, 1);
            s_q = a.qlist ? (i < a.qlist[0] ? a.qlist[1 + i] : a.nq) : i;
        }
        __syncthreads();
        const int q = s_q;
        if (q >= a.nq) break;
        long long t_prev = clock64();
        const int T = a.Tq ? a.Tq[q] : a.T;
        const int w = a.w;
        const int R = a.R;
        const float *dqc = a.dqc + (size_t)q * a.mc * kc;
        const float qn0 = a.qn[2 * q], qn1 = a.qn[2 * q + 1], qs = a.qsum[q];
        if constexpr (PART != 1) {
            const float *src = a.dqr + (size_t)q * mp * kp;
            if (VAR == V_EXACT) {
                // the exact-distance scan keeps the query instead of a LUT
                for (int i = tid; i < a.raw_dim; i += NT) S.lut[i] = a.Q[(size_t)q * a.raw_dim + i];
            } else if (a.rot) {
                // bank-private LUT: word c * 32 + b holds table (b mod mp) at
                // code c, so bank b serves table b mod mp (32 / mp copies)
                if constexpr (MPC == 8 || MPC == 16 || MPC == 32) {
                    // every entry loaded once (entry e = tid + NT j: table
                    // e mod MPC, code e / MPC), all loads in flight together,
                    // then its copies stored; copy r goes to bank k + MPC r',
                    // r' = (r + code) mod (32 / MPC), so that the 32 stores of
                    // a warp hit 32 different banks
                    constexpr int NC = 32 / MPC;
                    float vals[MPC];
#pragma unroll
                    for (int j = 0; j < MPC; j++) {
                        const int e = tid + NT * j;
                        vals[j] = __ldg(src + (size_t)(e & (MPC - 1)) * 256 + (e / MPC));
                    }
#pragma unroll
                    for (int j = 0; j < MPC; j++) {
                        const int e = tid + NT * j;
                        const int k = e & (MPC - 1), cc = e / MPC;
#pragma unroll
                        for (int r = 0; r < NC; r++) S.lut[cc * 32 + k + MPC * ((r + cc) & (NC - 1))] = vals[j];
                    }
                } else {
#pragma unroll 8
                    for (int wd = tid; wd < ROT_LUT_BYTES / 4; wd += NT)
                        S.lut[wd] = __ldg(src + (size_t)(wd & (mp - 1)) * 256 + (wd >> 5));
                }
            } else {
                for (int i = tid; i < mp * kp; i += NT) S.lut[i] = src[i];
            }
        }

        bool nothing_q = false;  // the query visits nothing (T <= 0 or w <= 0)
        int nvis = 0;
        bool qerr2 = false;
        uint32_t Svis = 0;
        const uint32_t *vcell = vis_cell, *vpre = vis_pre;
        if constexpr (PART == 2) {
            // the selection kernel's result for this query
            const QMeta m = a.qmeta[q];
            nvis = m.nvis;
            Svis = m.svis;
            qerr2 = m.err != 0;
            vcell = a.pool_cell + m.off;
            vpre = a.pool_pre + m.off;
            if (tid == 0) st.err = qerr2 ? 1 : 0;
            __syncthreads();
            PHASE_MARK(12);  // LUT (or query) staging
        } else {
            // PART 1 compacts straight into the query's pool region (set
            // after the cut, when the list's length is known)
            uint32_t *vis_cell_w = (uint32_t *)vcell, *vis_pre_w = (uint32_t *)vpre;
            // entries a visited list holds (the last is the closing prefix)
            uint64_t vcap = (uint64_t)cap;

        // IMI and SC test the rules before each pop (multi_query.h:151,
        // sc_query.h:130); IVFADC pops first and tests after
        // (query.h:249-259), so T <= 0 still visits one cell there.
        const bool nothing = (w <= 0) || (!ivf && T <= 0);
        uint64_t needT = (uint64_t)(T > 0 ? T : 0);
        uint64_t needW = (uint64_t)(w > 0 ? w : 0);
        if (ivf && T <= 0) {
            needT = ~0ull;
            needW = 1;
        }
        const double c0 = (T > 0 ? (double)T : 1.0) / (avg_density > 1e-9 ? avg_density : 1e-9);
        int M = next_pow2(4 * (int)sqrt(c0) + 1);
        if (M < 128) M = 128;
        if (M > SBCAP / 2) M = SBCAP / 2;

        uint64_t Ssum = 0, Ncell = 0, NEc = 0;  // totals over enumerated cells
        uint64_t S0 = 0, N0 = 0, NE0 = 0;       // totals before the last round
        int nrec = 0, r0 = 0;
        bool trig = false;
        Lists L;
        for (int attempt = 0; attempt < 2; attempt++) {
            const bool full = attempt == 1 || M >= kc;
            bool done_a = false, done_b = !imi;
            const uint32_t *meta = a.slist ? a.smeta + (size_t)q * (imi ? 2 : 1) * 2 : nullptr;
            if (a.slist && attempt == 0 && meta[0] > 0 && (!imi || meta[2] > 0)) {
                // prefixes sorted ahead by k_coarse_prefix (same prefix rule;
                // length 0 = left to this kernel)
                const int nl = imi ? 2 : 1;
                const uint64_t *src = a.slist + (size_t)q * nl * a.slist_w;
                const int ca = (int)meta[0], cb = imi ? (int)meta[2] : 0;
                for (int h = tid; h < ca; h += NT) S.LA[h] = src[h];
                for (int h = tid; h < cb; h += NT) S.LB[h] = src[a.slist_w + h];
                if (tid == 0) {
                    st.err = 0;
                    st.kA = ca;
                    st.kB = imi ? cb : kBfull;
                    st.nextA = meta[1];
                    st.nextB = imi ? meta[3] : 0xffffffffu;
                }
                done_a = done_b = true;
                __syncthreads();
            } else {
                // (1) coarse lists (sort_id/nth_element_id with M = kc;
                //     multi_query.h:114-128, sc_query.h:98-106, query.h:230-234):
                //     ordered key << 32 | centroid id; equal keys by id.
                for (int h = tid; h < kcP; h += NT) {
                    if (h < kc) {
                        float ka = __fadd_rn(imi ? qn0 : qs, dqc[h]);
                        S.LA[h] = ((uint64_t)f2o(ka) << 32) | (uint32_t)h;
                        if (imi) {
                            float kb = __fadd_rn(qn1, dqc[kc + h]);
                            S.LB[h] = ((uint64_t)f2o(kb) << 32) | (uint32_t)h;
                        }
                    } else {
                        S.LA[h] = ~0ull;
                        if (imi) S.LB[h] = ~0ull;
                    }
                }
                if (tid == 0) {
                    st.err = 0;
                    st.kA = kc;
                    st.kB = kBfull;
                    st.nextA = 0xffffffffu;
                    st.nextB = 0xffffffffu;
                }
                __syncthreads();
                if (!full) {
                    int ca = select_prefix(S.LA, kc, M, sb, hist, red, st, &st.nextA);
                    if (ca > 0) {
                        done_a = true;
                        if (tid == 0) st.kA = ca;
                    }
                    if (imi) {
                        int cb = select_prefix(S.LB, kc, M, sb, hist, red, st, &st.nextB);
                        if (cb > 0) {
                            done_b = true;
                            if (tid == 0) st.kB = cb;
                        }
                    }
                    __syncthreads();
                    if (!done_a || !done_b) {
                        // a prefix beyond SBCAP: sort everything instead
                        done_a = done_b = false;
                        for (int h = tid; h < kcP; h += NT) {
                            if (h < kc) {
                                S.LA[h] = ((uint64_t)f2o(__fadd_rn(imi ? qn0 : qs, dqc[h])) << 32) | (uint32_t)h;
                                if (imi) S.LB[h] = ((uint64_t)f2o(__fadd_rn(qn1, dqc[kc + h])) << 32) | (uint32_t)h;
                            }
                        }
                        if (tid == 0) {
                            st.kA = kc;
                            st.kB = kBfull;
                            st.nextA = st.nextB = 0xffffffffu;
                        }
                        __syncthreads();
                    }
                }
            }
            if (!done_a) bitonic_sort64(S.LA, kcP);
            if (imi && !done_b) bitonic_sort64(S.LB, kcP);
            __syncthreads();
            // ranks 0..lim-1 of each sorted list take part: the rank limit M
            // of search_multi2 / search_mr_ivf / search_mr_ivf3 confines the
            // walk to the top-M grid (kc: the whole grid; IVFADC has none)
            const int lim = (!ivf && a.rank_limit > 0 && a.rank_limit < kc) ? a.rank_limit : kc;
            const int kB0 = scx ? st.kA : st.kB;
            L.LA = S.LA;
            L.LB = S.LB;
            L.kA = min(st.kA, lim);
            L.kB = ivf ? kB0 : min(kB0, lim);
            L.kc = kc;
            L.ivf = ivf;
            // smallest keys left outside the prefixes, within the rank limit
            const uint32_t nextA = st.kA >= lim ? 0xffffffffu : st.nextA;
            const uint32_t nextB = (ivf || kB0 >= lim) ? 0xffffffffu : (sc ? st.nextA : st.nextB);
            // every cell outside the prefix grid has a key >= bound
            uint32_t bound = 0xffffffffu;
            if (sc3) {
                if (nextA != 0xffffffffu) {
                    const float nx = o2f(nextA), a0 = L.a(0);
                    bound = min(f2o(__fadd_rn(__fadd_rn(nx, a0), a0)), f2o(__fadd_rn(__fadd_rn(a0, a0), nx)));
                }
            } else {
                if (nextA != 0xffffffffu) bound = min(bound, f2o(__fadd_rn(o2f(nextA), L.b(0))));
                if (nextB != 0xffffffffu) bound = min(bound, f2o(__fadd_rn(L.a(0), o2f(nextB))));
            }
            const bool whole = L.kA == lim && (ivf || L.kB == lim);
            PHASE_MARK(0);  // lists

            // (2) rounds of staircase enumeration over the prefix grid
            for (int h = tid; h < L.kA; h += NT) S.rowp[h] = (sc && h == 0) ? 1 : 0;
            Ssum = Ncell = NEc = 0;
            S0 = N0 = NE0 = 0;
            nrec = 0;
            r0 = 0;
            trig = false;
            const uint64_t grid_cells = (uint64_t)L.kA * L.kB * (sc3 ? (uint64_t)L.kA : 1ull);
            const uint64_t total_cells = grid_cells - (sc ? 1 : 0);
            uint32_t tau_prev = 0, tau_old = 0;  // tau_old: the last enumerated round's tau
            const uint32_t lo_key = sc3 ? f2o(__fadd_rn(__fadd_rn(L.a(0), L.a(0)), L.a(0)))
                                        : f2o(__fadd_rn(L.a(0), L.b(0)));
            const uint32_t hi_key =
                sc3 ? f2o(__fadd_rn(__fadd_rn(L.a(L.kA - 1), L.a(L.kA - 1)), L.a(L.kA - 1)))
                    : f2o(__fadd_rn(L.a(L.kA - 1), L.b(L.kB - 1)));
            // first round: an eighth of the cells the density of this CTA's
            // previous query (else the index average) predicts; the visited
            // set does not depend on the round sizes
            const double dloc = st.dens_est > 1e-9 ? st.dens_est : (avg_density > 1e-9 ? avg_density : 1e-9);
            uint64_t target = (uint64_t)((T > 0 ? (double)T : 1.0) / dloc / 8.0);
            if (target < 64) target = 64;
            if (target > 1024) target = 1024;
            if (sc) target += 1;
            __syncthreads();
            int round = 0;
            if (!nothing) {
                for (; round < MAX_ROUNDS; round++) {
                    if (target > grid_cells) target = grid_cells;
                    if (!scx && needW < target) {
                        // the w rule caps popped cells: never enumerate past w
                        uint64_t tw = needW;
                        if (tw < Ncell + 1) tw = Ncell + 1;
                        if (tw < target) target = tw;
                    }
                    // bisection for tau: smallest key with staircase count >= target
                    uint32_t lo = round == 0 ? lo_key : tau_prev + 1, hi = hi_key;
                    uint64_t thi = target + target / 4 + 32;
                    COUNT(8, 1);
                    if (lo > hi) lo = hi;
                    int it = 0;
                    // a previous query with a target within 25% of this one
                    const int tp = st.tau_T;
                    const uint32_t gap0 = (4ll * (tp > T ? tp - T : T - tp) <= (long long)tp) ? st.tau_gap : 0u;
                    if (round == 0 && gap0 != 0u && lo < hi) {
                        // first probe where this CTA's previous query ended
                        const uint32_t mid = (hi - lo > gap0) ? lo + gap0 : hi - 1;
                        uint64_t c = sc3 ? staircase3_count(L, mid, red) : staircase_count(L, mid, red);
                        COUNT(9, 1);
                        if (c >= target) hi = mid;
                        else lo = mid + 1;
                        if (c >= target && c <= thi) lo = hi;
                        it++;
                    }
                    while (lo < hi && it < 40) {
                        uint32_t mid = lo + ((hi - lo) >> 1);
                        uint64_t c = sc3 ? staircase3_count(L, mid, red) : staircase_count(L, mid, red);
                        COUNT(9, 1);
                        if (c >= target) {
                            hi = mid;
                            if (c <= thi) break;
                        } else {
                            lo = mid + 1;
                        }
                        it++;
                    }
                    const uint32_t tau = hi;
                    PHASE_MARK(14);  // the round's bisection for tau
                    tau_prev = tau;  // the next round's bisection starts above tau
                    if (round == 0 && tid == 0) {
                        st.tau_gap = tau - lo_key;
                        st.tau_T = T;
                    }
                    uint64_t ls = 0, lne = 0, dummy = 0;
                    int nnew = 0;
                    if (sc3) {
                        // the triples with tau_prev < key <= tau (round 0: key <=
                        // tau): per row (h1, h2) the h3 between the two counts;
                        // a counting pass, then the records
                        const float a0 = L.a(0);
                        auto rows = [&](auto &&emit) {
                            for (int h1 = tid; h1 < L.kA; h1 += NT) {
                                const float a1 = L.a(h1);
                                for (int h2 = 0; h2 < L.kA; h2++) {
                                    const float base = __fadd_rn(a1, L.a(h2));
                                    if (f2o(__fadd_rn(base, a0)) > tau) break;
                                    const int c1 = L.row_count(base, tau);
                                    const int c0 = round == 0 ? 0 : min(c1, L.row_count(base, tau_old));
                                    if (c1 > c0) emit(h1, h2, base, c0, c1);
                                }
                            }
                        };
                        uint64_t mine = 0;
                        rows([&](int, int, float, int c0, int c1) { mine += (uint64_t)(c1 - c0); });
                        uint64_t tot_new;
                        uint64_t pos = block_exscan(mine, red, tot_new);
                        if ((uint64_t)nrec + tot_new > (uint64_t)cap) {
                            if (tid == 0) {
                                st.err = 1;
                                atomicOr(a.status, ST_CELL_BUDGET);
                            }
                            __syncthreads();
                            break;
                        }
                        rows([&](int h1, int h2, float base, int c0, int c1) {
                            for (int h3 = c0; h3 < c1; h3++) {
                                const uint32_t rank = rank3(h1, h2, h3);
                                const uint32_t cell = cell_of3(L, rank);
                                uint32_t c = a.off[cell + 1] - a.off[cell];
                                if (cell == 0) c = 0;  // sc_query.h:336-339
                                const size_t r = (size_t)nrec + pos++;
                                rec_key[r] = f2o(__fadd_rn(base, L.a(h3)));
                                rec_rank[r] = rank;
                                rec_cnt[r] = c;
                                ls += c;
                                lne += (c > 0);
                            }
                        });
                        nnew = (int)tot_new;
                        COUNT(10, nnew);
                    } else {
                    // row counts at tau and the new cells per row
                    uint32_t mycnt = 0;
                    const int per = (L.kA + NT - 1) / NT;
                    const int hb = tid * per;
                    for (int i = 0; i < per; i++) {
                        int h = hb + i;
                        if (h >= L.kA) break;
                        int c = L.row_count(L.a(h), tau);
                        int p0 = S.rowp[h];
                        if (c < p0) c = p0;
                        S.rowc[h] = (uint16_t)c;
                        mycnt += (uint32_t)(c - p0);
                    }
                    uint64_t tot_new;
                    uint64_t ex = block_exscan(mycnt, red, tot_new);
                    {
                        uint32_t run = (uint32_t)ex;
                        for (int i = 0; i < per; i++) {
                            int h = hb + i;
                            if (h >= L.kA) break;
                            S.rowpre[h] = run;
                            run += (uint32_t)(S.rowc[h] - S.rowp[h]);
                        }
                    }
                    if ((uint64_t)nrec + tot_new > (uint64_t)cap) {
                        if (tid == 0) {
                            st.err = 1;
                            atomicOr(a.status, ST_CELL_BUDGET);
                        }
                        __syncthreads();
                        break;
                    }
                    __syncthreads();
                    nnew = (int)tot_new;
                    COUNT(10, nnew);
                    int h1 = 0;
                    for (int idx = tid; idx < nnew; idx += NT) {
                        // row of idx: last h with rowpre[h] <= idx (rows only grow)
                        int lo2 = h1, hi2 = L.kA - 1;
                        while (lo2 < hi2) {
                            int mid = (lo2 + hi2 + 1) >> 1;
                            if (S.rowpre[mid] <= (uint32_t)idx) lo2 = mid;
                            else hi2 = mid - 1;
                        }
                        h1 = lo2;
                        int h2 = S.rowp[h1] + (idx - (int)S.rowpre[h1]);
                        float key = __fadd_rn(L.a(h1), L.b(h2));
                        uint32_t rank = ((uint32_t)h1 << 16) | (uint32_t)h2;
                        uint32_t cell = cell_of(L, rank);
                        uint32_t c = a.off[cell + 1] - a.off[cell];
                        if (sc && cell == 0) c = 0;  // sc_query.h:138-140
                        rec_key[nrec + idx] = f2o(key);
                        rec_rank[nrec + idx] = rank;
                        rec_cnt[nrec + idx] = c;
                        ls += c;
                        lne += (c > 0);
                    }
                    }
                    block_sum3(ls, lne, dummy, red);  // also orders the record loop's rowp reads before the update
                    if (!sc3)
                        for (int h = tid; h < L.kA; h += NT) S.rowp[h] = S.rowc[h];
                    S0 = Ssum;
                    N0 = Ncell;
                    NE0 = NEc;
                    r0 = nrec;
                    nrec += nnew;
                    Ssum += ls;
                    Ncell += (uint64_t)nnew;
                    NEc += lne;
                    tau_old = tau;
                    __syncthreads();
                    uint64_t wcnt = scx ? NEc : Ncell;
                    trig = (Ssum >= needT) || (wcnt >= needW);
                    PHASE_MARK(1);  // the round's enumeration
                    if (trig || Ncell >= total_cells || tau >= hi_key) break;
                    // next target from the density seen so far
                    double dens = Ncell ? (double)Ssum / (double)Ncell : avg_density;
                    if (dens < 1e-6) dens = avg_density > 1e-6 ? avg_density : 1e-6;
                    double need_cells = (double)(needT - Ssum) / dens;
                    uint64_t grow = (uint64_t)(need_cells * 1.25) + 64;
                    uint64_t minimum = Ncell / 4 + 64;
                    target = Ncell + (sc ? 1 : 0) + (grow > minimum ? grow : minimum);
                }
                if (round >= MAX_ROUNDS && tid == 0) {
                    st.err = 1;
                    atomicOr(a.status, ST_ITER_CAP);
                }
            }
            if (tid == 0 && Ncell > 0 && Ssum > 0) {
                st.dens_est = (double)Ssum / (double)Ncell;
                if (a.dens_acc) {
                    atomicAdd(&a.dens_acc[0], (unsigned long long)Ssum);
                    atomicAdd(&a.dens_acc[1], (unsigned long long)Ncell);
                }
            }
            __syncthreads();
            const bool qerr = st.err != 0;
            PHASE_MARK(1);  // staircase rounds

            // (3) the cut within the last round
            bool cut_done = false;
            const int nr = nrec - r0;
            if (!nothing && !qerr && trig && nr > 0 && nr <= 2 * NT && (!sc3 || L.kA <= NT)) {
                // few records: sort them by (key, rank) and scan the running
                // totals.  The enumeration wrote a round's records in rank
                // order, so (key << 32 | index) sorts them by (key, rank).
                uint64_t *sk = reinterpret_cast<uint64_t *>(hist);  // 2 NT keys inside the bins
                const int n2 = next_pow2(nr);
                for (int i = tid; i < n2; i += NT)
                    sk[i] = i < nr ? ((uint64_t)rec_key[r0 + i] << 32) | (uint32_t)i : ~0ull;
                if (tid == 0) st.s_bin = 0xffffffffu;
                __syncthreads();
                bitonic_sort64(sk, n2);
                // thread t: sorted positions 2t and 2t + 1; candidates in
                // bits 0..39 of the scan, non-empty cells in bits 40..63
                uint64_t cT[2] = {0, 0}, cN[2] = {0, 0};
#pragma unroll
                for (int j = 0; j < 2; j++) {
                    const int pz = 2 * tid + j;
                    if (pz < nr) {
                        const uint32_t c = rec_cnt[r0 + (uint32_t)sk[pz]];
                        cT[j] = c;
                        cN[j] = c > 0 ? 1u : 0u;
                    }
                }
                const uint64_t M40 = (1ull << 40) - 1;
                uint64_t tot;
                const uint64_t ex = block_exscan((cT[0] + cT[1]) | ((cN[0] + cN[1]) << 40), red, tot);
                uint64_t accT = S0 + (ex & M40), accN = NE0 + (ex >> 40);
#pragma unroll
                for (int j = 0; j < 2; j++) {
                    const int pz = 2 * tid + j;
                    if (pz < nr) {
                        const uint64_t nT = accT + cT[j], nN = accN + cN[j];
                        // the w rule counts non-empty cells (SC) or every cell
                        const uint64_t wb = scx ? accN : N0 + (uint64_t)pz, wa = scx ? nN : N0 + (uint64_t)pz + 1;
                        const bool before = accT >= needT || wb >= needW, after = nT >= needT || wa >= needW;
                        if (after && !before) {
                            // the first record at which a rule fires: the cut
                            const uint32_t idx = (uint32_t)sk[pz];
                            st.kappa = (uint32_t)(sk[pz] >> 32);
                            st.rank_cut = rec_rank[r0 + idx];
                            st.take_all = 0;
                            st.sumv = nT;
                            st.nv = N0 + (uint64_t)pz + 1;
                            st.nev = nN;
                            st.s_bin = (uint32_t)pz;
                        }
                        accT = nT;
                        accN = nN;
                    }
                }
                __syncthreads();
                cut_done = st.s_bin != 0xffffffffu;
                __syncthreads();
            }
            if (cut_done) {
            } else if (!nothing && !qerr && trig) {
                uint64_t mn = 0xffffffffull, mx = 0;
                for (int r = r0 + tid; r < nrec; r += NT) {
                    uint64_t k = rec_key[r];
                    mn = k < mn ? k : mn;
                    mx = k > mx ? k : mx;
                }
                block_minmax(mn, mx, red);
                uint32_t klo = (uint32_t)mn, khi = (uint32_t)mx;
                uint32_t kap = 0xffffffffu;
                if (Ssum >= needT)
                    kap = radix_cut(rec_key, rec_cnt, r0, nrec, klo, khi, S0, needT, 0, hist, red, st);
                uint64_t wcnt = scx ? NEc : Ncell;
                if (wcnt >= needW) {
                    uint32_t kw = radix_cut(rec_key, rec_cnt, r0, nrec, klo, khi, scx ? NE0 : N0, needW, scx ? 2 : 1,
                                            hist, red, st);
                    if (kw < kap) kap = kw;
                }
                // totals strictly below kappa, and the ties at kappa
                uint64_t ls = 0, ln = 0, lne = 0;
                if (tid == 0) st.nties = 0;
                __syncthreads();
                for (int r = r0 + tid; r < nrec; r += NT) {
                    uint32_t k = rec_key[r];
                    if (k < kap) {
                        uint32_t c = rec_cnt[r];
                        ls += c;
                        ln += 1;
                        lne += (c > 0);
                    } else if (k == kap) {
                        int slot = atomicAdd(&st.nties, 1);
                        if (slot < TIECAP) ties[slot] = ((uint64_t)rec_rank[r] << 32) | rec_cnt[r];
                    }
                }
                block_sum3(ls, ln, lne, red);
                if (tid == 0) {
                    uint64_t s = S0 + ls, n = N0 + ln, ne = NE0 + lne;
                    int nt = st.nties;
                    if (nt > TIECAP) {
                        st.err = 1;
                        atomicOr(a.status, ST_TIE_OVERFLOW);
                        nt = TIECAP;
                    }
                    // ties in rank order (an exact priority queue's order)
                    for (int i = 1; i < nt; i++) {
                        uint64_t v = ties[i];
                        int j = i - 1;
                        while (j >= 0 && ties[j] > v) {
                            ties[j + 1] = ties[j];
                            j--;
                        }
                        ties[j + 1] = v;
                    }
                    uint32_t rc_ = 0;
                    for (int i = 0; i < nt; i++) {
                        uint32_t c = (uint32_t)ties[i];
                        s += c;
                        n += 1;
                        ne += (c > 0);
                        rc_ = (uint32_t)(ties[i] >> 32);
                        if (s >= needT || (scx ? ne : n) >= needW) break;
                    }
                    st.kappa = kap;
                    st.rank_cut = rc_;
                    st.take_all = 0;
                    st.sumv = s;
                    st.nv = n;
                    st.nev = ne;
                }
                __syncthreads();
            } else if (tid == 0) {
                st.kappa = 0xffffffffu;
                st.rank_cut = 0xffffffffu;
                st.take_all = 1;
                st.sumv = nothing ? 0 : Ssum;
                st.nv = nothing ? 0 : Ncell;
                st.nev = nothing ? 0 : NEc;
            }
            __syncthreads();
            PHASE_MARK(2);  // cut
            // the prefix grid holds every cell with a key <= the cut
            const bool valid = nothing || st.err || (trig ? st.kappa < bound : whole);
            if (valid) break;
            COUNT(11, 1);
            __syncthreads();
        }
        if constexpr (PART == 1) {
            // the query's region of the pool: its own stride-sized slot, or a
            // range of the shared overflow area for a longer list
            if (tid == 0) {
                const uint32_t need = (!nothing && !st.err) ? (uint32_t)st.nev + 1u : 1u;
                uint32_t off = (uint32_t)q * a.pool_stride, capv = a.pool_stride;
                if (need > a.pool_stride) {
                    const uint32_t o = atomicAdd(a.pool_over, need);
                    if ((uint64_t)o + need <= (uint64_t)a.pool_over_cap) {
                        off = (uint32_t)a.nq * a.pool_stride + o;
                        capv = need;
                    } else {
                        st.err = 1;
                        atomicOr(a.status, ST_POOL);
                    }
                }
                st.pool_off = off;
                st.pool_cap = capv;
            }
            __syncthreads();
            vcell = a.pool_cell + st.pool_off;
            vpre = a.pool_pre + st.pool_off;
            vis_cell_w = (uint32_t *)vcell;
            vis_pre_w = (uint32_t *)vpre;
            vcap = (uint64_t)st.pool_cap - 1;
        }

        // (4) visited non-empty cells -> (cell, prefix) list
        if (!nothing && !st.err) {
            const uint32_t kap = st.kappa, rcut = st.rank_cut;
            const bool all = st.take_all != 0;
            uint64_t pos = 0, runc = 0;
            for (int base = 0; base < nrec; base += NT) {
                int r = base + tid;
                bool f = false;
                uint32_t c = 0, rank = 0;
                if (r < nrec) {
                    c = rec_cnt[r];
                    rank = rec_rank[r];
                    uint32_t k = rec_key[r];
                    bool inc = all || r < r0 || k < kap || (k == kap && rank <= rcut);
                    f = inc && c > 0;
                }
                uint64_t v = f ? ((1ull << 40) | c) : 0ull;
                uint64_t tot;
                uint64_t ex = block_exscan(v, red, tot);
                if (f) {
                    uint64_t p = pos + (ex >> 40);
                    if (p < vcap) {
                        vis_cell_w[p] = sc3 ? cell_of3(L, rank) : cell_of(L, rank);
                        vis_pre_w[p] = (uint32_t)(runc + (ex & 0xffffffffffull));
                    }
                }
                pos += tot >> 40;
                runc += tot & 0xffffffffffull;
            }
            nvis = (int)pos;
            if (tid == 0) {
                if (pos <= vcap) {
                    vis_pre_w[nvis] = (uint32_t)runc;
                } else {
                    // more visited cells than the list holds: an error, never a truncation
                    st.err = 1;
                    atomicOr(a.status, ST_CELL_BUDGET);
                }
                st.sumv = runc;  // the candidates of the visited cells
            }
        }
        if (tid == 0) st.nvis = nvis;
        __syncthreads();
        nvis = st.nvis;
        qerr2 = st.err != 0;
        Svis = (nvis > 0) ? (uint32_t)st.sumv : 0u;
        nothing_q = nothing;
        PHASE_MARK(3);  // compaction
            if constexpr (PART == 1) {
                if (tid == 0) {
                    QMeta m;
                    m.off = st.pool_off;
                    m.nvis = qerr2 ? 0 : nvis;
                    m.svis = Svis;
                    m.err = qerr2 ? 1 : 0;
                    a.qmeta[q] = m;
                    a.out_sum[q] = qerr2 ? -1 : (int)(nothing ? 0 : st.sumv);
                    if (a.out_nvis) a.out_nvis[q] = nvis;
                    if (a.out_empty) a.out_empty[q] = qerr2 ? 0 : (int)(st.nv - st.nev);
                }
                __syncthreads();
                continue;
            }
        }

        // (5) ADC scan with the fused top-R.  The first WARMN candidates are
        // scored into shared memory; their R-th smallest distance bounds the
        // final R-th distance from above, so the rest of the scan keeps only
        // candidates at or below it, appended to a per-CTA buffer; one merge
        // over that buffer (merge_topk) gives the R best.  The scan-only
        // kernel with a hand-off buffer (a.surv) writes the first surv_cap
        // survivors of query q to surv[q] instead and, when they all fit,
        // leaves the merge to k_merge_warp (surv_n[q] = their count).
        uint64_t *top = S.top, *tmpk = S.tmp;
        uint64_t *pend_g = a.pend + (size_t)blockIdx.x * a.pcap;
        if (tid == 0) {
            st.ncur = 0;
            st.npend = 0;
            st.next_flat = 0;
            st.top_sorted = 0;
            st.handed = 0;
        }
        __syncthreads();
        if (!qerr2 && nvis > 0) {
            ScanCtx c;
            c.vis_cell = vcell;
            c.vis_pre = vpre;
            c.nvis = nvis;
            c.Svis = Svis;
            c.kc = kc;
            c.mp = mp;
            c.kp = kp;
            c.bsI = bsI;
            c.imi = imi;
            c.sc = scx;
            c.cdiv = sc3 ? (uint32_t)kc * (uint32_t)kc : (uint32_t)kc;
            c.fast = fast;
            c.rot = a.rot != 0;
            c.raw_dim = a.raw_dim;
            c.raw_u8 = a.raw_u8 != 0;
            c.raw_vec = a.raw_dim > 0 && ((reinterpret_cast<uintptr_t>(a.raw) & 15) == 0) &&
                        (((size_t)a.raw_dim * (a.raw_u8 ? 1 : 4)) % 16 == 0);
            c.qv = S.lut;
            c.qs = qs;
            c.dqc = dqc;
            const bool hand = PART == 2 && a.surv != nullptr;
            c.sq = hand ? a.surv + (size_t)q * a.surv_cap : nullptr;
            c.scap = hand ? (uint32_t)a.surv_cap : 0u;
            const uint32_t K = Svis < (uint32_t)WARMN ? Svis : (uint32_t)WARMN;
            constexpr bool ROTOK = PART == 0 || VAR == V_FAST256;
            constexpr bool CELLS = VAR == V_FAST256 && (MPC == 8 || MPC == 16 || MPC == 32);
            if constexpr (CELLS) scan_cells<(CELLS ? MPC : 8), true, U>(a, S, st, c, 0u, K, 0u, S.warm, nullptr, 0u);
            else scan_chunks<MPC, true, U, VAR, ROTOK>(a, S, st, c, 0u, K, 0u, S.warm, nullptr, 0u);
            __syncthreads();
            uint32_t tau = 0xffffffffu;
            // an upper bound of the R-th warm-up distance (within
            // 2^(SCG_WARM_SBITS - 23) of it, relative)
            if (K > (uint32_t)R) {
                const uint64_t *wk = S.warm;
                tau = block_kth_bound<WARMN / NT>([&](int i) { return (uint32_t)(wk[i] >> 32); }, (int)K, R, SCG_WARM_SBITS,
                                                  S.hist2, red, st);
            }
            // the warm entries at or below tau open the pending buffer
            {
                uint64_t mine = 0;
                for (int i = tid; i < (int)K; i += NT) mine += ((uint32_t)(S.warm[i] >> 32) <= tau);
                uint64_t tot;
                uint64_t p = block_exscan(mine, red, tot);
                for (int i = tid; i < (int)K; i += NT) {
                    uint64_t e = S.warm[i];
                    if ((uint32_t)(e >> 32) <= tau) {
                        (p < c.scap ? c.sq : pend_g)[p] = e;
                        p++;
                    }
                }
                if (tid == 0) {
                    st.npend = (int)tot;
                    st.next_flat = K;
                }
                __syncthreads();
            }
            PHASE_MARK(13);  // warm-up scores and the threshold
            if constexpr (CELLS) scan_cells<(CELLS ? MPC : 8), false, U>(a, S, st, c, K, Svis, tau, nullptr, pend_g, a.pcap);
            else scan_chunks<MPC, false, U, VAR, ROTOK>(a, S, st, c, K, Svis, tau, nullptr, pend_g, a.pcap);
            __syncthreads();
            PHASE_MARK(4);  // scan
            if ((uint32_t)st.npend > a.pcap) {
                if (tid == 0) {
                    st.err = 1;
                    atomicOr(a.status, ST_CELL_BUDGET);
                }
                __syncthreads();
            } else if (c.scap && (uint32_t)st.npend <= c.scap) {
                // every survivor is in the query's hand-off slots: the merge
                // kernel finishes the query
                COUNT(6, st.npend);
                if (tid == 0) {
                    a.surv_n[q] = st.npend;
                    st.handed = 1;
                }
            } else if (st.npend > 0) {
                COUNT(6, st.npend);
                // the first slots went to the hand-off buffer
                for (uint32_t i = (uint32_t)tid; i < c.scap; i += NT) pend_g[i] = c.sq[i];
                if (c.scap) __syncthreads();
                merge_topk(top, pend_g, tmpk, S.hist2, S.ties2, R, a.pid, red, st, a.status);
            }
        }
        __syncthreads();
        PHASE_MARK(5);  // final merge
        if (st.handed) continue;  // uniform: read after the barrier
        if (PART == 2 && a.surv && tid == 0) a.surv_n[q] = -1;  // outputs written here
        // (6) outputs: the R best sorted by (distance, id) (a shortlist for
        // the exact re-rank in any order: the re-rank sorts it itself)
        {
            const bool qerr3 = st.err != 0;
            int keep = (qerr3 || nvis == 0) ? 0 : st.ncur;
            if (keep > 1 && !st.top_sorted && !a.shortlist) {
                const int k2 = next_pow2(keep);
                for (int i = keep + tid; i < k2; i += NT) top[i] = ~0ull;
                __syncthreads();
                bitonic_sort64(top, k2);
            }
            for (int j = tid; j < R; j += NT) {
                size_t o = (size_t)q * R + j;
                if (j < keep) {
                    uint64_t e = top[j];
                    a.out_ids[o] = (int)(uint32_t)e;
                    a.out_d[o] = o2f((uint32_t)(e >> 32));
                } else {
                    a.out_ids[o] = -1;
                    a.out_d[o] = __int_as_float(0x7f800000);
                }
            }
            if (tid == 0) {
                if constexpr (PART == 0) {
                    a.out_sum[q] = qerr3 ? -1 : (int)(nothing_q ? 0 : st.sumv);
                    if (a.out_nvis) a.out_nvis[q] = nvis;
                    if (a.out_empty) a.out_empty[q] = qerr3 ? 0 : (int)(st.nv - st.nev);
                } else if (qerr3 && !qerr2) {
                    // the selection kernel wrote the facts; a scan failure voids them
                    a.out_sum[q] = -1;
                    if (a.out_empty) a.out_empty[q] = 0;
                }
            }
        }
        __syncthreads();
    }
}


// Dynamic shared memory already granted to a kernel variant, per device
// (the attribute is set once, not on every launch).
template <int MPC, int U, int PART, int VAR>
int grant_smem(size_t smem) {
    static int granted[64] = {0};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64 || granted[dev] < (int)smem) {
        cudaError_t e =
            cudaFuncSetAttribute(k_search<MPC, U, PART, VAR>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return cuda_fail(e, "cudaFuncSetAttribute(k_search)");
        if (dev >= 0 && dev < 64) granted[dev] = (int)smem;
    }
    return SCG_OK;
}

template <int MPC, int U, int PART, int VAR = V_ADC>
int occupancy(size_t smem) {
    if (grant_smem<MPC, U, PART, VAR>(smem)) return 0;
    int nb = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_search<MPC, U, PART, VAR>, NT, smem);
    return nb;
}

// var: the kernel variant the launch will pick (V_FAST256 only for the
// scan-only kernel with a fixed code width; V_EXACT is one variant for every
// code width).
template <int MPC, int U, int PART>
int occupancy_var(size_t smem, int var) {
    if (var == V_EXACT) return occupancy<0, U, PART, V_EXACT>(smem);
    if constexpr (PART == 2 && MPC > 0) {
        if (var == V_FAST256) return occupancy<MPC, U, PART, V_FAST256>(smem);
    }
    return occupancy<MPC, U, PART, V_ADC>(smem);
}

template <int U, int PART>
int occupancy_mp(int mp, size_t smem, int var = V_ADC) {
    switch (mp) {
        case 4: return occupancy_var<4, U, PART>(smem, var);
        case 8: return occupancy_var<8, U, PART>(smem, var);
        case 16: return occupancy_var<16, U, PART>(smem, var);
        case 32: return occupancy_var<32, U, PART>(smem, var);
        default: return occupancy_var<0, U, PART>(smem, var);
    }
}

template <int MPC, int U, int PART, int VAR = V_ADC>
int launch(const SearchArgs &a, int grid, size_t smem, cudaStream_t s) {
    int rc = grant_smem<MPC, U, PART, VAR>(smem);
    if (rc) return rc;
    k_search<MPC, U, PART, VAR><<<grid, NT, smem, s>>>(a);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, "k_search launch");
    return SCG_OK;
}

// The variant of a launch: the exact-distance scan (one variant for every
// code width), the fast form's scan-only kernel with kp == 256, or the
// general ADC kernel.
template <int MPC, int U, int PART>
int launch_var(const SearchArgs &a, int grid, size_t smem, cudaStream_t s) {
    if (a.raw_dim > 0) return launch<0, U, PART, V_EXACT>(a, grid, smem, s);
    if constexpr (PART == 2 && MPC > 0) {
        if (a.precision == SCG_FAST && a.kp == 256) return launch<MPC, U, PART, V_FAST256>(a, grid, smem, s);
    }
    return launch<MPC, U, PART, V_ADC>(a, grid, smem, s);
}

template <int U, int PART>
int launch_mp(const SearchArgs &a, int grid, size_t smem, cudaStream_t s) {
    switch (a.mp) {
        case 4: return launch_var<4, U, PART>(a, grid, smem, s);
        case 8: return launch_var<8, U, PART>(a, grid, smem, s);
        case 16: return launch_var<16, U, PART>(a, grid, smem, s);
        case 32: return launch_var<32, U, PART>(a, grid, smem, s);
        default: return launch_var<0, U, PART>(a, grid, smem, s);
    }
}

}  // namespace

}  // namespace scg
