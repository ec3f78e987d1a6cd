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
int search_occupancy_u2(int mp, int part, size_t smem);
int search_occupancy_u4(int mp, int part, size_t smem);
int search_occupancy_u8(int mp, int part, size_t smem);
int search_occupancy_select(size_t smem);

size_t search_smem_bytes(int mode, int kc, int mp, int kp, int part) {
    return carve(mode, kc, mp, kp, part, nullptr, nullptr);
}

static int occupancy_query(int mode, int kc, int mp, int kp, int upl, int part) {
    const size_t smem = search_smem_bytes(mode, kc, mp, kp, part);
    if (part == 1) return search_occupancy_select(smem);
    switch (upl) {
        case 2: return search_occupancy_u2(mp, part, smem);
        case 8: return search_occupancy_u8(mp, part, smem);
        default: return search_occupancy_u4(mp, part, smem);
    }
}

// Resident CTAs per SM, asked of the runtime once per device and shape.
int search_max_blocks_per_sm(int mode, int kc, int mp, int kp, int upl, int part) {
    static std::mutex mu;
    static std::map<std::tuple<int, int, int, int, int, int, int>, int> cache;
    int dev = 0;
    cudaGetDevice(&dev);
    const auto key = std::make_tuple(dev, mode, kc, mp, kp, upl, part);
    {
        std::lock_guard<std::mutex> g(mu);
        auto it = cache.find(key);
        if (it != cache.end()) return it->second;
    }
    const int nb = occupancy_query(mode, kc, mp, kp, upl, part);
    std::lock_guard<std::mutex> g(mu);
    if (nb > 0) cache[key] = nb;
    return nb;
}

int search_launch(const SearchArgs &a, int part, int grid, cudaStream_t s) {
    const size_t smem = search_smem_bytes(a.mode, a.kc, a.mp, a.kp, part);
    if (part == 1) return search_launch_select(a, grid, smem, s);
    switch (a.upl) {
        case 2: return search_launch_u2(a, part, grid, smem, s);
        case 8: return search_launch_u8(a, part, grid, smem, s);
        default: return search_launch_u4(a, part, grid, smem, s);
    }
}

}  // namespace scg
