// refshim_grid.h -- uniform-grid index over closed primitive boxes, standing in for the
// cuBQL hierarchy in the host build of the reference rasterizer.  TEST INFRASTRUCTURE
// ONLY.  Cell of a coordinate: floor((c - lo) * inv) clamped to [0, n - 1]; the map is
// monotonic, so a box containing a point is registered in that point's cell.
#pragma once
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <vector>

#include "bvh.h"

namespace cuBQL {

struct RefGrid {
    float lo[3] = {0.f, 0.f, 0.f}, inv[3] = {0.f, 0.f, 0.f};
    int n[3] = {1, 1, 1};
    std::vector<int64_t> start;  // CSR over cells
    std::vector<uint32_t> ids;
    std::vector<box3f> boxes;

    int cell(int a, float c) const {
        float f = (c - lo[a]) * inv[a];
        if (!(f >= 0.f)) return 0;  // below the range or NaN
        const int i = (int)std::floor(f);
        return i >= n[a] ? n[a] - 1 : i;
    }

    static bool overlap(const box3f& a, const box3f& b) {
        return a.lower.x <= b.upper.x && a.upper.x >= b.lower.x && a.lower.y <= b.upper.y &&
               a.upper.y >= b.lower.y && a.lower.z <= b.upper.z && a.upper.z >= b.lower.z;
    }

    // Primitive boxes as float[6] (lo xyz, hi xyz).  A cell is about half the median box
    // extent on each axis (a box then spans about 3 x 3 x 3 cells).  Cells are filled in
    // parallel and each cell's list is then sorted, so the index does not depend on the
    // thread count.
    void build(const float* b6, int64_t count) {
        boxes.resize(count);
        float L[3] = {INFINITY, INFINITY, INFINITY}, H[3] = {-INFINITY, -INFINITY, -INFINITY};
        for (int64_t i = 0; i < count; i++) {
            boxes[i] = box3f(vec3f(b6[6 * i], b6[6 * i + 1], b6[6 * i + 2]),
                             vec3f(b6[6 * i + 3], b6[6 * i + 4], b6[6 * i + 5]));
            for (int a = 0; a < 3; a++) {
                L[a] = std::min(L[a], b6[6 * i + a]);
                H[a] = std::max(H[a], b6[6 * i + 3 + a]);
            }
        }
        for (int a = 0; a < 3; a++) {
            std::vector<float> e;
            e.reserve(std::min<int64_t>(count, 100000));
            const int64_t stride = count > 100000 ? count / 100000 : 1;
            for (int64_t i = 0; i < count; i += stride) {
                const float w = b6[6 * i + 3 + a] - b6[6 * i + a];
                if (w >= 0.f) e.push_back(w);
            }
            float med = 0.f;
            if (!e.empty()) {
                std::nth_element(e.begin(), e.begin() + e.size() / 2, e.end());
                med = e[e.size() / 2];
            }
            lo[a] = count ? L[a] : 0.f;
            const float ext = count ? H[a] - L[a] : 0.f;
            const double want = med > 0.f ? (double)ext / (0.5 * med) : std::cbrt((double)count);
            n[a] = ext > 0.f ? (int)std::max(1.0, std::min(1024.0, want)) : 1;
            inv[a] = ext > 0.f ? (float)n[a] / ext : 0.f;
        }
        const int64_t nc = (int64_t)n[0] * n[1] * n[2];
        std::vector<int64_t> cnt(nc + 1, 0);
        auto visit = [&](int64_t i, bool fill) {
            const box3f& b = boxes[i];
            if (!(b.lower.x <= b.upper.x && b.lower.y <= b.upper.y && b.lower.z <= b.upper.z)) return;
            const int x0 = cell(0, b.lower.x), x1 = cell(0, b.upper.x), y0 = cell(1, b.lower.y),
                      y1 = cell(1, b.upper.y), z0 = cell(2, b.lower.z), z1 = cell(2, b.upper.z);
            for (int z = z0; z <= z1; z++)
                for (int y = y0; y <= y1; y++)
                    for (int x = x0; x <= x1; x++) {
                        const int64_t c = ((int64_t)z * n[1] + y) * n[0] + x;
                        int64_t slot;
#pragma omp atomic capture
                        slot = cnt[c]++;
                        if (fill) ids[start[c] + slot] = (uint32_t)i;
                    }
        };
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < count; i++) visit(i, false);
        start.assign(nc + 1, 0);
        for (int64_t c = 0; c < nc; c++) start[c + 1] = start[c] + cnt[c];
        ids.resize(start[nc]);
        std::fill(cnt.begin(), cnt.end(), 0);
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < count; i++) visit(i, true);
#pragma omp parallel for schedule(dynamic, 256)
        for (int64_t c = 0; c < nc; c++) std::sort(ids.begin() + start[c], ids.begin() + start[c + 1]);
    }

    // Every primitive whose closed box overlaps q, ascending, each once.
    void query(const box3f& q, std::vector<uint32_t>& out) const {
        out.clear();
        if (boxes.empty()) return;
        const int x0 = cell(0, q.lower.x), x1 = cell(0, q.upper.x), y0 = cell(1, q.lower.y), y1 = cell(1, q.upper.y),
                  z0 = cell(2, q.lower.z), z1 = cell(2, q.upper.z);
        for (int z = z0; z <= z1; z++)
            for (int y = y0; y <= y1; y++)
                for (int x = x0; x <= x1; x++) {
                    const int64_t c = ((int64_t)z * n[1] + y) * n[0] + x;
                    for (int64_t k = start[c]; k < start[c + 1]; k++)
                        if (overlap(boxes[ids[k]], q)) out.push_back(ids[k]);
                }
        if (x0 != x1 || y0 != y1 || z0 != z1) {
            std::sort(out.begin(), out.end());
            out.erase(std::unique(out.begin(), out.end()), out.end());
        }
    }
};

}  // namespace cuBQL
