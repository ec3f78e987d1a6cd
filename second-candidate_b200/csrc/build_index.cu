// Index build on the GPU: the bucketing of Encoder::distribution /
// SCEncoder::distribution (encoder.cpp:170-305, sc_encoder.cpp:17-182) and
// the CSR that PQQuery::load_encoded_data builds from the .edat_ file
// (query.cpp:82-165), without the host.
//
// Each row's cell is h = sum over parts of h * kc + cid[part] (vector_base,
// sc_utilities.h:156-166; second candidate: nn1 * kc + nn2).  Rows are
// ordered by cell and, inside a cell, by row id -- the order the reference's
// writer produces -- with a least-significant-digit radix sort of the cell
// keys (8-bit digits), each pass a stable counting sort: per-tile digit
// histograms, one exclusive scan of them (digit-major), and a scatter whose
// in-tile ranks keep the row order (warp match + per-warp digit counters,
// warps in tile order).  Cell offsets come from a histogram of the keys and
// the same scan.
#include "scg_internal.cuh"

namespace scg {

namespace {

constexpr int BT = 256;             // threads per block
constexpr int ITEMS = 4;            // elements per thread per tile
constexpr int TILE = BT * ITEMS;    // elements per tile
constexpr int NW = BT / 32;

__global__ void k_cell_ids(const uint16_t *__restrict__ cid, int64_t n, int parts, int kc, uint32_t *__restrict__ key,
                           uint32_t *__restrict__ val) {
    const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n) return;
    uint64_t h = 0;
    for (int i = 0; i < parts; i++) h = h * (uint64_t)kc + cid[(size_t)r * parts + i];
    key[r] = (uint32_t)h;
    val[r] = (uint32_t)r;
}

__global__ void k_count(const uint32_t *__restrict__ key, int64_t n, uint32_t *__restrict__ cnt) {
    const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (r < n) atomicAdd(cnt + key[r], 1u);
}

// Exclusive scan, level 1: each block scans TILE elements (blocked, ITEMS
// per thread) and writes the tile total.
__global__ void __launch_bounds__(BT) k_scan_tiles(const uint32_t *__restrict__ in, int64_t n,
                                                   uint32_t *__restrict__ out, uint32_t *__restrict__ sums) {
    __shared__ uint32_t ws[NW];
    const int64_t base = (int64_t)blockIdx.x * TILE + (int64_t)threadIdx.x * ITEMS;
    uint32_t v[ITEMS], t = 0;
#pragma unroll
    for (int j = 0; j < ITEMS; j++) {
        v[j] = base + j < n ? in[base + j] : 0u;
        t += v[j];
    }
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    uint32_t x = t;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) ws[w] = x;
    __syncthreads();
    uint32_t wpre = 0, tot = 0;
    for (int i = 0; i < NW; i++) {
        if (i < w) wpre += ws[i];
        tot += ws[i];
    }
    uint32_t run = wpre + x - t;
#pragma unroll
    for (int j = 0; j < ITEMS; j++) {
        if (base + j < n) out[base + j] = run;
        run += v[j];
    }
    if (threadIdx.x == 0) sums[blockIdx.x] = tot;
}

// Level 2: one block scans the tile totals in place (exclusive).
__global__ void __launch_bounds__(BT) k_scan_sums(uint32_t *__restrict__ sums, int64_t m) {
    __shared__ uint32_t ws[NW];
    __shared__ uint32_t carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int64_t c0 = 0; c0 < m; c0 += BT) {
        const int64_t i = c0 + threadIdx.x;
        const uint32_t t = i < m ? sums[i] : 0u;
        uint32_t x = t;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) ws[w] = x;
        __syncthreads();
        uint32_t wpre = 0, tot = 0;
        for (int k = 0; k < NW; k++) {
            if (k < w) wpre += ws[k];
            tot += ws[k];
        }
        if (i < m) sums[i] = carry + wpre + x - t;
        __syncthreads();
        if (threadIdx.x == 0) carry += tot;
        __syncthreads();
    }
}

__global__ void k_scan_add(uint32_t *__restrict__ out, int64_t n, const uint32_t *__restrict__ sums) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] += sums[i / TILE];
}

// Radix pass, histograms: hist[digit * nb + tile].
__global__ void __launch_bounds__(BT) k_digit_hist(const uint32_t *__restrict__ key, int64_t n, int shift,
                                                   uint32_t *__restrict__ hist, int64_t nb) {
    __shared__ uint32_t h[256];
    h[threadIdx.x] = 0;
    __syncthreads();
    const int64_t base = (int64_t)blockIdx.x * TILE;
    for (int j = threadIdx.x; j < TILE; j += BT) {
        const int64_t i = base + j;
        if (i < n) atomicAdd(&h[(key[i] >> shift) & 255u], 1u);
    }
    __syncthreads();
    hist[(size_t)threadIdx.x * nb + blockIdx.x] = h[threadIdx.x];
}

// Radix pass, stable scatter.  Warp w of tile b handles elements
// [b TILE + w 32 ITEMS, ... + 32 ITEMS) in ITEMS rounds of 32 consecutive
// elements; an element's rank among equal digits = the digit's count in
// earlier warps + in earlier rounds of its warp + earlier lanes of its round.
__global__ void __launch_bounds__(BT) k_digit_scatter(const uint32_t *__restrict__ kin, const uint32_t *__restrict__ vin,
                                                      int64_t n, int shift, const uint32_t *__restrict__ off,
                                                      int64_t nb, uint32_t *__restrict__ kout,
                                                      uint32_t *__restrict__ vout) {
    __shared__ uint32_t cnt[NW][257];
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int i = threadIdx.x; i < NW * 257; i += BT) (&cnt[0][0])[i] = 0;
    __syncthreads();
    const int64_t base = (int64_t)blockIdx.x * TILE + (int64_t)w * 32 * ITEMS;
    uint32_t k[ITEMS], v[ITEMS], d[ITEMS], rank[ITEMS];
#pragma unroll
    for (int r = 0; r < ITEMS; r++) {
        const int64_t i = base + r * 32 + lane;
        const bool ok = i < n;
        k[r] = ok ? kin[i] : 0u;
        v[r] = ok ? vin[i] : 0u;
        d[r] = ok ? ((k[r] >> shift) & 255u) : 256u;
        const unsigned peers = __match_any_sync(FULL, d[r]);
        rank[r] = cnt[w][d[r]] + __popc(peers & ((1u << lane) - 1u));
        __syncwarp();
        if (lane == __ffs(peers) - 1) cnt[w][d[r]] += __popc(peers);
        __syncwarp();
    }
    __syncthreads();
    // counts of earlier warps, per digit (exclusive over warps)
    {
        const int dg = threadIdx.x;  // BT == 256 digits
        uint32_t run = 0;
        for (int ww = 0; ww < NW; ww++) {
            const uint32_t c = cnt[ww][dg];
            cnt[ww][dg] = run;
            run += c;
        }
    }
    __syncthreads();
#pragma unroll
    for (int r = 0; r < ITEMS; r++) {
        if (d[r] < 256u) {
            const uint32_t pos = off[(size_t)d[r] * nb + blockIdx.x] + cnt[w][d[r]] + rank[r];
            kout[pos] = k[r];
            vout[pos] = v[r];
        }
    }
}

__global__ void k_gather_rows(const uint32_t *__restrict__ order, int64_t n, int mp, const uint8_t *__restrict__ codes,
                              int *__restrict__ pid, uint8_t *__restrict__ codes_out) {
    const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    const uint32_t r = order[p];
    pid[p] = (int)r;
    for (int j = 0; j < mp; j++) codes_out[(size_t)p * mp + j] = codes[(size_t)r * mp + j];
}

void exclusive_scan(const uint32_t *in, int64_t n, uint32_t *out, uint32_t *tile_sums, cudaStream_t s) {
    const int64_t tiles = (n + TILE - 1) / TILE;
    k_scan_tiles<<<(unsigned)tiles, BT, 0, s>>>(in, n, out, tile_sums);
    k_scan_sums<<<1, BT, 0, s>>>(tile_sums, tiles);
    k_scan_add<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(out, n, tile_sums);
}

}  // namespace

size_t build_work_bytes(int64_t n, int64_t ncells) {
    const int64_t nb = (n + TILE - 1) / TILE;
    const int64_t scan_n = std::max<int64_t>(256 * nb, ncells + 1);
    return 4ull * n * 4                       // keys, values (two buffers each)
           + 4ull * 256 * nb * 2              // digit histograms and their scan
           + 4ull * ((scan_n + TILE - 1) / TILE + 1)  // tile sums
           + 4ull * (ncells + 1) + 6 * 256;   // cell counts
}

// Orders rows by cell (ties by row) and fills off[ncells + 1], pid[n],
// codes_out[n][mp] from cid[n][parts] and codes[n][mp].
void launch_build_csr(const uint16_t *cid, const uint8_t *codes, int64_t n, int parts, int kc, int mp,
                      int64_t ncells, unsigned char *work, uint32_t *off, int *pid, uint8_t *codes_out, cudaStream_t s) {
    const int64_t nb = (n + TILE - 1) / TILE;
    const int64_t scan_n = std::max<int64_t>(256 * nb, ncells + 1);
    unsigned char *cur = work;
    auto take = [&](size_t bytes) {
        unsigned char *p = cur;
        cur += (bytes + 255) & ~(size_t)255;
        return p;
    };
    uint32_t *k0 = (uint32_t *)take(4ull * n), *k1 = (uint32_t *)take(4ull * n);
    uint32_t *v0 = (uint32_t *)take(4ull * n), *v1 = (uint32_t *)take(4ull * n);
    uint32_t *hist = (uint32_t *)take(4ull * 256 * nb), *hoff = (uint32_t *)take(4ull * 256 * nb);
    uint32_t *tsum = (uint32_t *)take(4ull * ((scan_n + TILE - 1) / TILE + 1));
    uint32_t *cnt = (uint32_t *)take(4ull * (ncells + 1));
    const unsigned g = (unsigned)((n + 255) / 256);
    k_cell_ids<<<g, 256, 0, s>>>(cid, n, parts, kc, k0, v0);
    // cell offsets: counts, exclusive scan (off[ncells] = n)
    cudaMemsetAsync(cnt, 0, 4ull * (ncells + 1), s);
    k_count<<<g, 256, 0, s>>>(k0, n, cnt);
    exclusive_scan(cnt, ncells + 1, off, tsum, s);
    // LSD radix sort of the cell keys, 8 bits per pass
    int bits = 1;
    while (bits < 32 && (1ull << bits) < (uint64_t)ncells) bits++;
    for (int shift = 0; shift < bits; shift += 8) {
        k_digit_hist<<<(unsigned)nb, BT, 0, s>>>(k0, n, shift, hist, nb);
        exclusive_scan(hist, 256 * nb, hoff, tsum, s);
        k_digit_scatter<<<(unsigned)nb, BT, 0, s>>>(k0, v0, n, shift, hoff, nb, k1, v1);
        std::swap(k0, k1);
        std::swap(v0, v1);
    }
    k_gather_rows<<<g, 256, 0, s>>>(v0, n, mp, codes, pid, codes_out);
}

}  // namespace scg
