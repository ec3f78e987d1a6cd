// Cell selection with one warp per query: part 1 of the split search for
// IVFADC, the inverted multi-index and the two-centroid second candidate,
// when the coarse prefixes were sorted ahead (k_coarse_prefix).
//
// It runs the block-wide selection's algorithm (search_impl.cuh: staircase
// rounds over the sorted prefixes, the exact cut in (key, rank) order, the
// compaction of the visited non-empty cells) on one warp per query, with
// warp reductions and warp scans instead of block barriers: the selection
// work of one query is small (a prefix of ~128 ranks per list, ~100
// enumerated cells), and spread over 256 threads it was bound by the
// barriers' and the idle threads' instructions.  The rounds enumerate the
// cells of a prefix grid in rank order, so (key << 32 | record index) sorts
// the last round by (key, rank), the exact priority order; the visited list
// is identical as a set to the block-wide kernel's and reaches the scan with
// the last round in key order.
//
// A query that does not fit the warp's buffers -- a prefix longer than KW,
// more than RW enumerated cells, more than WMAX_ROUNDS rounds, a cut at or
// past the smallest key outside the sorted prefixes, an exhausted prefix grid
// that is not the whole grid, or no sorted prefix -- is appended to a
// deferred list, which the block-wide kernel then serves from scratch.
#include "search_impl.cuh"

namespace scg {

namespace {

constexpr int WS_WARPS = 4;     // warps (queries in flight) per CTA
constexpr int KW = 256;         // longest prefix a warp holds
constexpr int RW = 256;         // enumerated cells a warp holds
constexpr int WMAX_ROUNDS = 8;  // rounds before the query is deferred

struct WarpSmem {
    uint64_t la[KW];  // sorted prefix of list A (then the last round's sorted records)
    uint64_t lb[KW];  // sorted prefix of list B (IMI)
    uint32_t rkey[RW], rcell[RW], rcnt[RW];  // enumerated cells in rank order
    uint16_t rowp[KW];  // per row of A: columns already enumerated
    uint16_t rowq[KW];  // per row of A: first record of the round's new cells
    uint16_t rows0[KW];  // per row of A: first new column of the round
};

__device__ __forceinline__ uint64_t shfl64(uint64_t v, int src) {
    const uint32_t lo = __shfl_sync(0xffffffffu, (uint32_t)v, src);
    const uint32_t hi = __shfl_sync(0xffffffffu, (uint32_t)(v >> 32), src);
    return ((uint64_t)hi << 32) | lo;
}

__device__ __forceinline__ uint64_t shfl_xor64(uint64_t v, int m) {
    const uint32_t lo = __shfl_xor_sync(0xffffffffu, (uint32_t)v, m);
    const uint32_t hi = __shfl_xor_sync(0xffffffffu, (uint32_t)(v >> 32), m);
    return ((uint64_t)hi << 32) | lo;
}

// Exclusive prefix of v over the lanes (lane order); `total` the warp sum.
__device__ __forceinline__ uint64_t warp_exscan64(uint64_t v, int lane, uint64_t &total) {
    uint64_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t lo = __shfl_up_sync(0xffffffffu, (uint32_t)x, o);
        const uint32_t hi = __shfl_up_sync(0xffffffffu, (uint32_t)(x >> 32), o);
        if (lane >= o) x += ((uint64_t)hi << 32) | lo;
    }
    total = shfl64(x, 31);
    return x - v;
}

// Ascending bitonic sort of 32 * P keys held striped (element r * 32 + lane
// in v[r]): partners 32 or more apart inside the lane, closer ones by
// shuffles.
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

// The same network on 32-bit keys.
template <int P>
__device__ __forceinline__ void warp_sort32(uint32_t (&v)[P], int lane) {
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
                        const uint32_t x = v[r], y = v[pr];
                        v[r] = asc ? min(x, y) : max(x, y);
                        v[pr] = asc ? max(x, y) : min(x, y);
                    }
                }
            } else {
                const bool lower = (lane & j) == 0;
#pragma unroll
                for (int r = 0; r < P; r++) {
                    const bool asc = ((r * 32 + lane) & k) == 0;
                    const uint32_t o = __shfl_xor_sync(0xffffffffu, v[r], j);
                    v[r] = (lower == asc) ? min(v[r], o) : max(v[r], o);
                }
            }
        }
    }
}

template <int P>
__device__ __forceinline__ void sort_buf32(uint32_t *buf, int lane) {
    uint32_t v[P];
#pragma unroll
    for (int r = 0; r < P; r++) v[r] = buf[r * 32 + lane];
    warp_sort32<P>(v, lane);
#pragma unroll
    for (int r = 0; r < P; r++) buf[r * 32 + lane] = v[r];
}

// Sorts the n2 (a power of two, 32..RW) keys of buf in place.
template <int P>
__device__ __forceinline__ void sort_buf(uint64_t *buf, int lane) {
    uint64_t v[P];
#pragma unroll
    for (int r = 0; r < P; r++) v[r] = buf[r * 32 + lane];
    warp_sort<P>(v, lane);
#pragma unroll
    for (int r = 0; r < P; r++) buf[r * 32 + lane] = v[r];
}

__global__ void __launch_bounds__(WS_WARPS * 32, 6) k_select_warp(SearchArgs a, int *defer) {
    __shared__ WarpSmem sm[WS_WARPS];
    const unsigned FULL = 0xffffffffu;
    const uint32_t INF = 0xffffffffu;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    WarpSmem &W = sm[wid];
    const int kc = a.kc;
    const bool imi = a.mode == SCG_IMI, sc = a.mode == SCG_SC2, ivf = a.mode == SCG_IVFADC;
    const int nl = imi ? 2 : 1;
    const double avg_density = (double)a.N / (double)(a.ncells ? a.ncells : 1);
    const uint32_t lt = (1u << lane) - 1u;
    // per warp, carried from query to query (heuristics only): candidates
    // per cell of the last query, its first round's tau above the lowest key
    // and its target
    double dens_est = 0.0;
    uint32_t tau_gap = 0;
    int tau_T = 0;
    for (;;) {
        int q = 0;
        if (lane == 0) q = atomicAdd(a.qcounter, 1);
        q = __shfl_sync(FULL, q, 0);
        if (q >= a.nq) break;
        const long long t0 = clock64();
        long long tp = t0;
        // optional phase cycles (lane 0): [0] prefixes, [14] bisections,
        // [1] enumeration, [2] cut, [3] compaction
        auto mark = [&](int i) {
            if (a.phase_cycles && lane == 0) {
                const long long t = clock64();
                atomicAdd((unsigned long long *)&a.phase_cycles[i], (unsigned long long)(t - tp));
                tp = t;
            }
        };
        const int T = a.Tq ? a.Tq[q] : a.T;
        const int w = a.w;
        // IMI and SC test the rules before each pop (multi_query.h:151,
        // sc_query.h:130); IVFADC pops first and tests after
        // (query.h:249-259), so T <= 0 still visits one cell there.
        const bool nothing = (w <= 0) || (!ivf && T <= 0);
        uint64_t needT = (uint64_t)(T > 0 ? T : 0), needW = (uint64_t)(w > 0 ? w : 0);
        if (ivf && T <= 0) {
            needT = ~0ull;
            needW = 1;
        }
        auto finish = [&](uint32_t off, int nvis, uint32_t svis, int err, uint64_t sumv, uint64_t nempty) {
            if (lane == 0) {
                QMeta m;
                m.off = off;
                m.nvis = err ? 0 : nvis;
                m.svis = svis;
                m.err = err;
                a.qmeta[q] = m;
                a.out_sum[q] = err ? -1 : (int)sumv;
                if (a.out_nvis) a.out_nvis[q] = err ? 0 : nvis;
                if (a.out_empty) a.out_empty[q] = err ? 0 : (int)nempty;
                if (a.phase_cycles) atomicAdd((unsigned long long *)&a.phase_cycles[15], (unsigned long long)(clock64() - t0));
            }
        };
        auto defer_q = [&]() {
            if (lane == 0) {
                const int i = atomicAdd(defer, 1);
                defer[1 + i] = q;
                if (a.phase_cycles) atomicAdd((unsigned long long *)&a.phase_cycles[7], 1ull);
            }
        };
        if (nothing) {
            finish((uint32_t)q * a.pool_stride, 0, 0u, 0, 0, 0);
            continue;
        }
        // the sorted prefixes and the rank limit (M of search_multi2 /
        // search_mr_ivf): ranks 0..lim-1 of each list take part
        const uint32_t *meta = a.smeta + (size_t)q * nl * 2;
        const int ca = (int)meta[0], cbl = imi ? (int)meta[2] : ca;
        const int lim = (!ivf && a.rank_limit > 0 && a.rank_limit < kc) ? a.rank_limit : kc;
        const int kA = min(ca, lim), kB = ivf ? 1 : min(cbl, lim);
        if (ca <= 0 || cbl <= 0 || kA > KW || kB > KW) {
            defer_q();
            continue;
        }
        const uint64_t *src = a.slist + (size_t)q * nl * a.slist_w;
        for (int h = lane; h < kA; h += 32) W.la[h] = src[h];
        if (imi)
            for (int h = lane; h < kB; h += 32) W.lb[h] = src[a.slist_w + h];
        for (int h = lane; h < kA; h += 32) W.rowp[h] = (sc && h == 0) ? 1 : 0;  // cell (0, 0) is preset traversed
        __syncwarp();
        Lists L;
        L.LA = W.la;
        L.LB = imi ? W.lb : W.la;
        L.kA = kA;
        L.kB = kB;
        L.kc = kc;
        L.ivf = ivf;
        // every cell outside the prefix grid (within the rank limit) has a
        // key >= bound
        const uint32_t nextA = ca >= lim ? INF : meta[1];
        const uint32_t nextB = (ivf || cbl >= lim) ? INF : (imi ? meta[3] : meta[1]);
        uint32_t bound = INF;
        if (nextA != INF) bound = min(bound, f2o(__fadd_rn(o2f(nextA), L.b(0))));
        if (nextB != INF) bound = min(bound, f2o(__fadd_rn(L.a(0), o2f(nextB))));
        const bool whole = kA == lim && (ivf || kB == lim);

        mark(0);
        // (2) rounds of staircase enumeration over the prefix grid; lane l
        // owns the rows [l * rpl, l * rpl + rpl) of list A
        const int rpl = (kA + 31) / 32;
        const int hb = lane * rpl;
        const uint64_t grid_cells = (uint64_t)kA * kB, total_cells = grid_cells - (sc ? 1 : 0);
        const uint32_t lo_key = f2o(__fadd_rn(L.a(0), L.b(0)));
        const uint32_t hi_key = f2o(__fadd_rn(L.a(kA - 1), L.b(kB - 1)));
        // staircase count at tau, each row's count searched only between its
        // counts at the bisection's current ends (rlo, rhi): cc[i] gets the
        // lane's row counts
        int rlo[KW / 32], rhi[KW / 32];
        auto count_at = [&](uint32_t tau, int (&cc)[KW / 32]) -> uint64_t {
            uint32_t c = 0;
#pragma unroll 8
            for (int i = 0; i < KW / 32; i++) {
                cc[i] = 0;
                const int h = hb + i;
                if (i < rpl && h < kA) {
                    const float av = L.a(h);
                    int lo2 = rlo[i], hi2 = rhi[i];  // the count lies in [lo2, hi2]
                    while (lo2 < hi2) {
                        const int mid = (lo2 + hi2 + 1) >> 1;
                        if (f2o(__fadd_rn(av, L.b(mid - 1))) <= tau) lo2 = mid;
                        else hi2 = mid - 1;
                    }
                    cc[i] = lo2;
                    c += (uint32_t)lo2;
                }
            }
            return (uint64_t)__reduce_add_sync(FULL, c);
        };
        const double dloc = dens_est > 1e-9 ? dens_est : (avg_density > 1e-9 ? avg_density : 1e-9);
        uint64_t target = (uint64_t)((T > 0 ? (double)T : 1.0) / dloc / 8.0);
        if (target < 64) target = 64;
        if (target > RW / 2) target = RW / 2;
        if (sc) target += 1;
        uint64_t Ssum = 0, Ncell = 0, NEc = 0, S0 = 0, N0 = 0, NE0 = 0;
        int nrec = 0, r0 = 0;
        bool trig = false, defer = false;
        uint32_t tau_prev = 0;
        int round = 0;
        for (; round < WMAX_ROUNDS; round++) {
            if (target > grid_cells) target = grid_cells;
            if (!sc && needW < target) {
                // the w rule caps popped cells: never enumerate past w
                uint64_t tw = needW;
                if (tw < Ncell + 1) tw = Ncell + 1;
                if (tw < target) target = tw;
            }
            // bisection for tau: smallest key with staircase count >= target
            // (a count within 25% above the target ends it early)
            uint32_t lo = round == 0 ? lo_key : tau_prev + 1, hi = hi_key;
            const uint64_t thi = target + target / 4 + 32;
            if (lo > hi) lo = hi;
            // row counts at the ends: at tau_prev (the enumerated columns;
            // row 0 of SC starts at 1, below every key >= lo_key) and at
            // hi_key (every column: the last row's last key is the largest)
#pragma unroll 8
            for (int i = 0; i < KW / 32; i++) {
                const int h = hb + i;
                rlo[i] = (i < rpl && h < kA) ? (int)W.rowp[h] : 0;
                rhi[i] = kB;
            }
            int cc[KW / 32];
            auto take = [&](uint64_t c, uint32_t mid) {
                // the probe's counts become the bracket's new end
                if (c >= target) {
                    hi = mid;
#pragma unroll 8
                    for (int i = 0; i < KW / 32; i++) rhi[i] = cc[i];
                } else {
                    lo = mid + 1;
#pragma unroll 8
                    for (int i = 0; i < KW / 32; i++) rlo[i] = cc[i];
                }
            };
            int it = 0;
            const int tp = tau_T;
            const uint32_t gap0 = (4ll * (tp > T ? tp - T : T - tp) <= (long long)tp) ? tau_gap : 0u;
            if (round == 0 && gap0 != 0u && lo < hi) {
                // first probe where this warp's previous query ended
                const uint32_t mid = (hi - lo > gap0) ? lo + gap0 : hi - 1;
                const uint64_t c = count_at(mid, cc);
                take(c, mid);
                if (c >= target && c <= thi) lo = hi;
                it++;
            }
            while (lo < hi && it < 40) {
                const uint32_t mid = lo + ((hi - lo) >> 1);
                const uint64_t c = count_at(mid, cc);
                take(c, mid);
                if (c >= target && c <= thi) break;
                it++;
            }
            const uint32_t tau = hi;
            mark(14);
            tau_prev = tau;
            if (round == 0) {
                tau_gap = tau - lo_key;
                tau_T = T;
            }
            // the new cells per row (tau_prev < key <= tau), in rank order
            int cn[KW / 32];
            uint32_t mine = 0;
#pragma unroll 8
            for (int i = 0; i < KW / 32; i++) {
                cn[i] = 0;
                const int h = hb + i;
                if (i < rpl && h < kA) {
                    // the row's count at tau = hi: the bracket's upper end
                    const int p0 = W.rowp[h];
                    cn[i] = rhi[i] < p0 ? p0 : rhi[i];
                    mine += (uint32_t)(cn[i] - p0);
                }
            }
            uint64_t tot_new;
            const uint32_t base = (uint32_t)warp_exscan64(mine, lane, tot_new);
            // the block-wide kernel holds more cells, and reports a
            // query beyond the cell budget as an error
            if ((uint64_t)nrec + tot_new > (uint64_t)min(RW, a.cap_rec)) {
                defer = true;
                break;
            }
            {
                // each row's first record and first new column, then the
                // records spread evenly over the lanes: record r is in the
                // last row whose first record is <= r
                uint32_t pos = (uint32_t)nrec + base;
#pragma unroll 8
                for (int i = 0; i < KW / 32; i++) {
                    const int h = hb + i;
                    if (i >= rpl || h >= kA) continue;
                    W.rowq[h] = (uint16_t)pos;
                    W.rows0[h] = W.rowp[h];
                    pos += (uint32_t)(cn[i] - W.rowp[h]);
                    W.rowp[h] = (uint16_t)cn[i];
                }
            }
            __syncwarp();
            // the new records with their cells' lengths
            uint64_t ls = 0;
            uint32_t lne = 0;
            const int n1 = nrec + (int)tot_new;
            for (int r = nrec + lane; r < n1; r += 32) {
                int lo2 = 0, hi2 = kA - 1;
                while (lo2 < hi2) {
                    const int mid = (lo2 + hi2 + 1) >> 1;
                    if (W.rowq[mid] <= (uint32_t)r) lo2 = mid;
                    else hi2 = mid - 1;
                }
                const int h = lo2, h2 = W.rows0[h] + (r - (int)W.rowq[h]);
                const uint32_t rank = ((uint32_t)h << 16) | (uint32_t)h2;
                const uint32_t cell = cell_of(L, rank);
                W.rkey[r] = f2o(__fadd_rn(L.a(h), L.b(h2)));
                W.rcell[r] = cell;
                uint32_t c = __ldg(a.off + cell + 1) - __ldg(a.off + cell);
                if (sc && cell == 0) c = 0;  // sc_query.h:138-140
                W.rcnt[r] = c;
                ls += c;
                lne += c > 0 ? 1u : 0u;
            }
            ls = warp_sum64(ls);
            lne = __reduce_add_sync(FULL, lne);
            __syncwarp();
            S0 = Ssum;
            N0 = Ncell;
            NE0 = NEc;
            r0 = nrec;
            nrec = n1;
            Ssum += ls;
            Ncell += tot_new;
            NEc += lne;
            const uint64_t wcnt = sc ? NEc : Ncell;
            trig = (Ssum >= needT) || (wcnt >= needW);
            if (trig || Ncell >= total_cells || tau >= hi_key) break;
            // next target from the density seen so far
            double dens = Ncell ? (double)Ssum / (double)Ncell : avg_density;
            if (dens < 1e-6) dens = avg_density > 1e-6 ? avg_density : 1e-6;
            const double need_cells = (double)(needT - Ssum) / dens;
            const uint64_t grow = (uint64_t)(need_cells * 1.25) + 64;
            const uint64_t minimum = Ncell / 4 + 64;
            target = Ncell + (sc ? 1 : 0) + (grow > minimum ? grow : minimum);
        }
        if (round >= WMAX_ROUNDS) defer = true;
        if (Ncell > 0 && Ssum > 0) dens_est = (double)Ssum / (double)Ncell;
        if (defer) {
            defer_q();
            continue;
        }
        if (Ncell > 0 && Ssum > 0 && lane == 0 && a.dens_acc) {
            atomicAdd(&a.dens_acc[0], (unsigned long long)Ssum);
            atomicAdd(&a.dens_acc[1], (unsigned long long)Ncell);
        }

        mark(1);
        // (3) the cut: the last round's records sorted by (key, rank) -- the
        // rank order of the enumeration, so (key << 32 | index) -- and the
        // first record at which the T rule (candidates) or the w rule (cells,
        // or non-empty cells for SC) fires.  The records before it, and it,
        // are visited.  No rule firing: every enumerated cell is visited.
        int pcut = -1;  // the cut's position in the sorted last round
        uint64_t nv = Ncell, nev = NEc;
        uint64_t *sb = W.la;  // the prefixes are no longer needed
        const int nr = nrec - r0;
        if (trig) {
            int n2 = 32;
            while (n2 < nr) n2 <<= 1;
            uint32_t kmin = INF, kmax = 0;
            for (int i = lane; i < nr; i += 32) {
                kmin = min(kmin, W.rkey[r0 + i]);
                kmax = max(kmax, W.rkey[r0 + i]);
            }
            kmin = __reduce_min_sync(FULL, kmin);
            kmax = __reduce_max_sync(FULL, kmax);
            if (kmax - kmin < (1u << 24) - 1u) {
                // keys within 2^24 of the smallest: (key - min) << 8 | index
                // sorts as 32 bits (list B's buffer is free by now), then
                // expands to the 64-bit (key, index) words
                uint32_t *s32 = reinterpret_cast<uint32_t *>(W.lb);
                for (int i = lane; i < n2; i += 32)
                    s32[i] = i < nr ? ((W.rkey[r0 + i] - kmin) << 8) | (uint32_t)i : INF;
                __syncwarp();
                switch (n2) {
                    case 32: sort_buf32<1>(s32, lane); break;
                    case 64: sort_buf32<2>(s32, lane); break;
                    case 128: sort_buf32<4>(s32, lane); break;
                    default: sort_buf32<8>(s32, lane); break;
                }
                __syncwarp();
                for (int i = lane; i < n2; i += 32) {
                    const uint32_t x = s32[i];
                    sb[i] = x == INF ? ~0ull : ((uint64_t)(kmin + (x >> 8)) << 32) | (x & 255u);
                }
            } else {
                for (int i = lane; i < n2; i += 32)
                    sb[i] = i < nr ? (((uint64_t)W.rkey[r0 + i] << 32) | (uint32_t)i) : ~0ull;
                __syncwarp();
                switch (n2) {
                    case 32: sort_buf<1>(sb, lane); break;
                    case 64: sort_buf<2>(sb, lane); break;
                    case 128: sort_buf<4>(sb, lane); break;
                    default: sort_buf<8>(sb, lane); break;
                }
            }
            __syncwarp();
            // lane l: sorted positions [l * pp, l * pp + pp)
            const int pp = n2 / 32;
            uint64_t myT = 0;
            uint32_t myN = 0;
            for (int j = 0; j < pp; j++) {
                const int p = lane * pp + j;
                if (p < nr) {
                    const uint32_t c = W.rcnt[r0 + (uint32_t)sb[p]];
                    myT += c;
                    myN += c > 0 ? 1u : 0u;
                }
            }
            uint64_t totT, totN;
            uint64_t accT = S0 + warp_exscan64(myT, lane, totT);
            uint64_t accN = NE0 + warp_exscan64(myN, lane, totN);
            int hit = -1;
            uint64_t hN = 0;
            for (int j = 0; j < pp; j++) {
                const int p = lane * pp + j;
                if (p >= nr) break;
                const uint32_t c = W.rcnt[r0 + (uint32_t)sb[p]];
                const uint64_t nT = accT + c, nN = accN + (c > 0 ? 1u : 0u);
                const uint64_t wb = sc ? accN : N0 + (uint64_t)p, wa = sc ? nN : N0 + (uint64_t)p + 1;
                const bool before = accT >= needT || wb >= needW, after = nT >= needT || wa >= needW;
                if (after && !before && hit < 0) {
                    hit = p;
                    hN = nN;
                }
                accT = nT;
                accN = nN;
            }
            const unsigned hm = __ballot_sync(FULL, hit >= 0);
            if (hm == 0u) {
                defer_q();
                continue;
            }
            const int src = __ffs(hm) - 1;
            pcut = __shfl_sync(FULL, hit, src);
            nev = shfl64(hN, src);
            nv = N0 + (uint64_t)pcut + 1;
            // a cut at or past the smallest key outside the prefix grid needs
            // the complete lists: the block-wide kernel sorts them
            const uint32_t kap = (uint32_t)(sb[pcut] >> 32);
            if (kap >= bound) {
                defer_q();
                continue;
            }
        } else if (!whole) {
            // the prefix grid is exhausted but other cells exist
            defer_q();
            continue;
        }

        mark(2);
        // (4) the visited non-empty cells -> (cell, prefix) list in the
        // query's pool region: the earlier rounds in rank order, then the
        // last round (up to the cut) in key order
        const int rA = trig ? r0 : nrec, nB = trig ? pcut + 1 : 0;
        const int nvis = (int)nev;
        const uint32_t need = (uint32_t)nvis + 1u;
        uint32_t off = (uint32_t)q * a.pool_stride;
        int err = 0;
        if (need > a.pool_stride) {
            uint32_t o = 0;
            if (lane == 0) o = atomicAdd(a.pool_over, need);
            o = __shfl_sync(FULL, o, 0);
            if ((uint64_t)o + need <= (uint64_t)a.pool_over_cap) {
                off = (uint32_t)a.nq * a.pool_stride + o;
            } else {
                err = 1;
                if (lane == 0) atomicOr(a.status, ST_POOL);
            }
        }
        uint32_t runc = 0;
        if (!err) {
            uint32_t *vc = a.pool_cell + off, *vp = a.pool_pre + off;
            uint32_t pos = 0;
            // entry e: record e (e < rA) or the sorted last round's e - rA
            for (int e0 = 0; e0 < rA + nB; e0 += 32) {
                const int e = e0 + lane;
                uint32_t c = 0, cell = 0;
                if (e < rA + nB) {
                    const uint32_t r = e < rA ? (uint32_t)e : (uint32_t)r0 + (uint32_t)sb[e - rA];
                    c = W.rcnt[r];
                    cell = W.rcell[r];
                }
                const bool f = c > 0;
                const unsigned m = __ballot_sync(FULL, f);
                uint64_t tot;
                const uint32_t ex = (uint32_t)warp_exscan64(c, lane, tot);
                if (f) {
                    const uint32_t p = pos + (uint32_t)__popc(m & lt);
                    vc[p] = cell;
                    vp[p] = runc + ex;
                }
                pos += (uint32_t)__popc(m);
                runc += (uint32_t)tot;
            }
            if (lane == 0) vp[nvis] = runc;
        }
        mark(3);
        finish(off, nvis, runc, err, runc, nv - nev);
    }
}

}  // namespace

bool select_warp_serves(int mode, int kc) {
    return (mode == SCG_IVFADC || mode == SCG_IMI || mode == SCG_SC2) && coarse_sort_width(kc) > 0;
}

int select_warp_launch(const SearchArgs &a, int *defer, int grid, cudaStream_t s) {
    k_select_warp<<<grid, WS_WARPS * 32, 0, s>>>(a, defer);
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

int select_warp_blocks_per_sm() {
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_select_warp, WS_WARPS * 32, 0) != cudaSuccess) return 0;
    return n;
}

}  // namespace scg
