// Instantiations of the fused search kernel with 2 candidates per lane per
// scan chunk (one translation unit per variant, so they compile in parallel).
#include "search_impl.cuh"

namespace scg {

int search_launch_u2(const SearchArgs &a, int grid, size_t smem, cudaStream_t s) { return launch_mp<2>(a, grid, smem, s); }
int search_occupancy_u2(int mp, size_t smem) { return occupancy_mp<2>(mp, smem); }

}  // namespace scg
