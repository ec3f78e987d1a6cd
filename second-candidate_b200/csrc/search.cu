// Host dispatch of the search kernels: shared-memory size, occupancy and
// launch of the fused kernel (part 0), the selection-only kernel (part 1) or
// the scan-only kernel (part 2) with the requested candidates per lane (the
// variants are compiled in search_u2.cu, search_u4.cu, search_u8.cu and
// search_sel.cu).
#include <map>
#include <mutex>
#include <tuple>

#include "search_impl.cuh"

namespace scg {

int search_launch_u2(const SearchArgs &a, int part, int grid, size_t smem, cudaStream_t s);
int search_launch_u4(const SearchArgs &a, int part, int grid, size_t smem, cudaStream_t s);
int search_launch_u8(const SearchArgs &a, int part, int grid, size_t smem, cudaStream_t s);
int search_launch_select(const SearchArgs &a, int grid, size_t smem, cudaStream_t s);
int search_occupancy_u2(int mp, int part, size_t smem, int var);
int search_occupancy_u4(int mp, int part, size_t smem, int var);
int search_occupancy_u8(int mp, int part, size_t smem, int var);
int search_occupancy_select(size_t smem);

size_t search_smem_bytes(int mode, int kc, int mp, int kp, int part, int rot, int qdim) {
    return carve(mode, kc, mp, kp, part, rot, qdim, nullptr, nullptr);
}

bool search_rot_form(int precision, int mp, int kp) { return rot_form(precision, mp, kp); }

static int occupancy_query(int mode, int kc, int mp, int kp, int upl, int part, int rot, int qdim) {
    const size_t smem = search_smem_bytes(mode, kc, mp, kp, part, rot, qdim);
    if (part == 1) return search_occupancy_select(smem);
    // the variant the launch picks: exact-distance scan, the fast form's
    // scan-only kernel (rotated LUT), or the general ADC kernel
    const int var = qdim > 0 ? V_EXACT : ((part == 2 && rot) ? V_FAST256 : V_ADC);
    switch (upl) {
        case 2: return search_occupancy_u2(mp, part, smem, var);
        case 8: return search_occupancy_u8(mp, part, smem, var);
        default: return search_occupancy_u4(mp, part, smem, var);
    }
}

// Resident CTAs per SM, asked of the runtime once per device and shape.
int search_max_blocks_per_sm(int mode, int kc, int mp, int kp, int upl, int part, int rot, int qdim) {
    static std::mutex mu;
    static std::map<std::tuple<int, int, int, int, int, int, int, int, int>, int> cache;
    int dev = 0;
    cudaGetDevice(&dev);
    if (part == 1) rot = qdim = 0;  // the selection kernel has no LUT
    if (qdim > 0) rot = 0;          // the exact-distance scan has none either
    const auto key = std::make_tuple(dev, mode, kc, mp, kp, upl, part, rot, qdim);
    {
        std::lock_guard<std::mutex> g(mu);
        auto it = cache.find(key);
        if (it != cache.end()) return it->second;
    }
    const int nb = occupancy_query(mode, kc, mp, kp, upl, part, rot, qdim);
    std::lock_guard<std::mutex> g(mu);
    if (nb > 0) cache[key] = nb;
    return nb;
}

int search_launch(const SearchArgs &a, int part, int grid, cudaStream_t s) {
    const size_t smem = search_smem_bytes(a.mode, a.kc, a.mp, a.kp, part, part == 1 ? 0 : a.rot,
                                          part == 1 ? 0 : a.raw_dim);
    if (part == 1) return search_launch_select(a, grid, smem, s);
    switch (a.upl) {
        case 2: return search_launch_u2(a, part, grid, smem, s);
        case 8: return search_launch_u8(a, part, grid, smem, s);
        default: return search_launch_u4(a, part, grid, smem, s);
    }
}

}  // namespace scg
