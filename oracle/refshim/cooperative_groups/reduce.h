// cooperative_groups/reduce.h -- host stand-in (TEST INFRASTRUCTURE ONLY).
// The launch emulation runs the lanes of a warp one after another, from lane 31 down to
// lane 0 (refshim_prelude.h).  Every lane of a tile makes the same sequence of reduce
// calls, so the k-th call of each lane adds its value into slot k, and lane 0, which runs
// last, receives the total ((v31 + v30) + ... + v1) + v0 and clears the slot.  The other
// lanes receive their own value (in the reference only lane 0 uses the result).  A tile
// of one thread returns the value itself.
#pragma once
#include <cstdlib>

namespace cooperative_groups {

template <class T>
struct plus {
    T operator()(T a, T b) const { return a + b; }
};

template <unsigned N, class T, class Op>
inline T reduce(const thread_block_tile<N>& tile, T v, Op op) {
    if (N == 1) return v;
    constexpr int kSlots = 64;
    thread_local T slot[kSlots] = {};
    thread_local unsigned long long epoch = ~0ull;
    thread_local int calls = 0;
    if (epoch != ref_thread_epoch) {
        epoch = ref_thread_epoch;
        calls = 0;
    }
    const int k = calls++;
    if (k >= kSlots) std::abort();
    if (tile.thread_rank() == N - 1) slot[k] = T();  // the first lane of the tile to run
    if (tile.thread_rank() != 0) {
        slot[k] = op(slot[k], v);
        return v;
    }
    const T total = op(slot[k], v);
    slot[k] = T();
    return total;
}

}  // namespace cooperative_groups
