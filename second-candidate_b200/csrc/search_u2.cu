// Instantiations of the fused (part 0) and scan-only (part 2) search kernels
// with 2 candidates per lane per scan chunk (one translation unit per
// variant, so that they compile in parallel).
#include "search_impl.cuh"

namespace scg {

int search_launch_u2(const SearchArgs &a, int part, int grid, size_t smem, cudaStream_t s) {
    return part == 2 ? launch_mp<2, 2>(a, grid, smem, s) : launch_mp<2, 0>(a, grid, smem, s);
}
int search_occupancy_u2(int mp, int part, size_t smem, int var) {
    return part == 2 ? occupancy_mp<2, 2>(mp, smem, var) : occupancy_mp<2, 0>(mp, smem, var);
}

}  // namespace scg
