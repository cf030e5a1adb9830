// cuBQL/traversal/fixedBoxQuery.h -- host stand-in for cuBQL's box queries as the
// reference calls them (forward.cu:150,209, backward.cu:243,378).  TEST INFRASTRUCTURE
// ONLY.  The declared candidate set is used: a primitive is visited iff its closed box
// overlaps the closed query box, each once, in ascending primitive index.  forEachLeaf
// hands all of them over as one leaf (a leaf holding exactly the primitives inside the
// query box; the reference's kernels spread a leaf's primitives over the lanes of a warp).
#pragma once
#include <algorithm>
#include <vector>

#include "../bvh.h"
#include "../refshim_grid.h"

namespace cuBQL {
namespace fixedBoxQuery {

// per-thread candidate list, reused across queries
inline std::vector<uint32_t>& query_ids() {
    thread_local std::vector<uint32_t> ids;
    return ids;
}

template <typename T, int D, class F>
inline void forEachPrim(F&& f, const bvh3f& bvh, const box3f& q) {
    std::vector<uint32_t>& ids = query_ids();
    bvh.grid->query(q, ids);
    for (uint32_t id : ids) f((int)id);
}

// The reference calls forEachLeaf from every lane of a warp with the same box (one
// Gaussian per warp); on the GPU those lanes traverse in lockstep.  The host runs the
// lanes one after another, so a query repeating the previous one of the same block on
// the same index reuses its list instead of traversing again.
template <typename T, int D, class F>
inline void forEachLeaf(F&& f, const bvh3f& bvh, const box3f& q) {
    thread_local std::vector<uint32_t> ids;
    thread_local box3f last_q;
    thread_local const RefGrid* last_grid = nullptr;
    thread_local uint3 last_block{~0u, 0u, 0u};
    const bool same = last_grid == bvh.grid && last_block.x == blockIdx.x && last_q.lower.x == q.lower.x &&
                      last_q.lower.y == q.lower.y && last_q.lower.z == q.lower.z && last_q.upper.x == q.upper.x &&
                      last_q.upper.y == q.upper.y && last_q.upper.z == q.upper.z;
    if (!same) {
        bvh.grid->query(q, ids);
        last_q = q;
        last_grid = bvh.grid;
        last_block = blockIdx;
    }
    if (!ids.empty()) f(ids.data(), (int)ids.size());
}

}  // namespace fixedBoxQuery
}  // namespace cuBQL
