// cooperative_groups/reduce.h -- host stand-in (TEST INFRASTRUCTURE ONLY): reduce over a
// one-thread tile is the value itself; wider tiles are never reached on the host.
#pragma once
#include <cstdlib>

namespace cooperative_groups {

template <class T>
struct plus {
    T operator()(T a, T b) const { return a + b; }
};

template <unsigned N, class T, class Op>
inline T reduce(const thread_block_tile<N>&, T v, Op) {
    if (N != 1) std::abort();
    return v;
}

}  // namespace cooperative_groups
