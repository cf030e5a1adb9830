// cuBQL/bvh.h -- host stand-in for the two cuBQL types the reference's rasterizer passes
// around (TEST INFRASTRUCTURE ONLY; cuBQL is not vendored with the reference and no
// version is pinned).  box3f is a closed axis-aligned box; bvh3f does not hold a
// hierarchy here but a uniform-grid index over the primitive boxes (refshim_grid.h),
// which answers the same queries: every primitive whose closed box overlaps the query.
#pragma once
#include <cstdint>

namespace cuBQL {

struct vec3f {
    float x, y, z;
    vec3f() : x(0.f), y(0.f), z(0.f) {}
    vec3f(float a, float b, float c) : x(a), y(b), z(c) {}
};

struct box3f {
    vec3f lower, upper;
    box3f() {}
    explicit box3f(vec3f p) : lower(p), upper(p) {}
    box3f(vec3f lo, vec3f hi) : lower(lo), upper(hi) {}
};

struct RefGrid;  // refshim_grid.h

struct bvh3f {
    const RefGrid* grid = nullptr;
};

}  // namespace cuBQL
