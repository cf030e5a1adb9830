// cuBQL/traversal/fixedBoxQuery.h -- host stand-in for cuBQL's box queries as the
// reference calls them (forward.cu:150,209, backward.cu:243,378).  TEST INFRASTRUCTURE
// ONLY.  The declared candidate set is used: a primitive is visited iff its closed box
// overlaps the closed query box, each once, in ascending primitive index.  forEachLeaf
// hands every such primitive over as a leaf of one primitive (the leaf-size-1 limit of
// the reference's sample BVH).
#pragma once
#include <algorithm>
#include <vector>

#include "../bvh.h"
#include "../refshim_grid.h"

namespace cuBQL {
namespace fixedBoxQuery {

template <typename T, int D, class F>
inline void forEachPrim(F&& f, const bvh3f& bvh, const box3f& q) {
    std::vector<uint32_t> ids;
    bvh.grid->query(q, ids);
    for (uint32_t id : ids) f((int)id);
}

template <typename T, int D, class F>
inline void forEachLeaf(F&& f, const bvh3f& bvh, const box3f& q) {
    std::vector<uint32_t> ids;
    bvh.grid->query(q, ids);
    for (uint32_t id : ids) {
        uint32_t one = id;
        f(&one, 1);
    }
}

}  // namespace fixedBoxQuery
}  // namespace cuBQL
