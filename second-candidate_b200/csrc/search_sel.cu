// Instantiation of the selection-only search kernel (part 1); it has no scan,
// so one variant serves every code width and chunking.
#include "search_impl.cuh"

namespace scg {

int search_launch_select(const SearchArgs &a, int grid, size_t smem, cudaStream_t s) {
    return launch<0, 4, 1>(a, grid, smem, s);
}
int search_occupancy_select(size_t smem) { return occupancy<0, 4, 1>(smem); }

}  // namespace scg
