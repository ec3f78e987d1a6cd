// Host dispatch of the fused search kernel: shared-memory size, occupancy and
// launch of the variant with the requested candidates per lane (the variants
// are compiled in search_u2.cu, search_u4.cu and search_u8.cu).
#include "search_impl.cuh"

namespace scg {

int search_launch_u2(const SearchArgs &a, int grid, size_t smem, cudaStream_t s);
int search_launch_u4(const SearchArgs &a, int grid, size_t smem, cudaStream_t s);
int search_launch_u8(const SearchArgs &a, int grid, size_t smem, cudaStream_t s);
int search_occupancy_u2(int mp, size_t smem);
int search_occupancy_u4(int mp, size_t smem);
int search_occupancy_u8(int mp, size_t smem);

size_t search_smem_bytes(int mode, int kc, int mp, int kp) { return carve(mode, kc, mp, kp, nullptr, nullptr); }

int search_max_blocks_per_sm(int mode, int kc, int mp, int kp, int upl) {
    const size_t smem = search_smem_bytes(mode, kc, mp, kp);
    switch (upl) {
        case 2: return search_occupancy_u2(mp, smem);
        case 8: return search_occupancy_u8(mp, smem);
        default: return search_occupancy_u4(mp, smem);
    }
}

int search_launch(const SearchArgs &a, int grid, cudaStream_t s) {
    const size_t smem = search_smem_bytes(a.mode, a.kc, a.mp, a.kp);
    switch (a.upl) {
        case 2: return search_launch_u2(a, grid, smem, s);
        case 8: return search_launch_u8(a, grid, smem, s);
        default: return search_launch_u4(a, grid, smem, s);
    }
}

}  // namespace scg
