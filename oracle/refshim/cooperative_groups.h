// cooperative_groups.h -- host stand-in for the cooperative-groups calls of the reference
// rasterizer (TEST INFRASTRUCTURE ONLY): grid and block handles with thread_rank(), and
// tiled_partition<N> (a tile of N consecutive threads; its reduction is emulated in
// cooperative_groups/reduce.h).
#pragma once

namespace cooperative_groups {

struct grid_group {
    unsigned long long thread_rank() const {
        return (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x;
    }
};
struct thread_block {
    unsigned thread_rank() const { return threadIdx.x; }
};
template <unsigned N>
struct thread_block_tile {
    unsigned thread_rank() const { return threadIdx.x % N; }
};

inline grid_group this_grid() { return grid_group{}; }
inline thread_block this_thread_block() { return thread_block{}; }
template <unsigned N>
inline thread_block_tile<N> tiled_partition(const thread_block&) {
    return thread_block_tile<N>{};
}

}  // namespace cooperative_groups
