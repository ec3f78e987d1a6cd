// Instantiations of the fused search kernel with 8 candidates per lane per
// scan chunk (one translation unit per variant, so they compile in parallel).
#include "search_impl.cuh"

namespace scg {

int search_launch_u8(const SearchArgs &a, int grid, size_t smem, cudaStream_t s) { return launch_mp<8>(a, grid, smem, s); }
int search_occupancy_u8(int mp, size_t smem) { return occupancy_mp<8>(mp, smem); }

}  // namespace scg
