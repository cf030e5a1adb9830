// knn.cu -- mean squared distance to the three nearest other points.
//
// This is the initial-scale rule of the training code: scene/gaussian_model.py:175-179
// (create_from_pcd) and :729-733 (densify_in_empty) call simple-knn's distCUDA2, a
// third-party extension that is not part of the reference tree.  Its published
// behaviour, restated: for every point, the three smallest squared Euclidean distances
// to any other index (duplicates count with distance 0), kept in ascending order and
// averaged as (b0 + b1 + b2) / 3 in float32; neighbours that do not exist (n < 4)
// count as FLT_MAX.
//
// B200 design: the points become degenerate leaf boxes of the library's LBVH (30-bit
// Morton keys, stable radix sort, Karras hierarchy, 64-byte nodes holding both child
// boxes).  One thread per Morton-sorted query: the 3rd-best distance among its +-3
// Morton neighbours bounds the search, then a near-child-first traversal prunes every
// child whose box distance exceeds min(bound, current 3rd best).  Distances are
// rounded after every operation (no FMA contraction), which makes a box's distance
// never exceed the distance of any point inside it, so the pruning is exact and the
// result is bit-identical to the CPU restatement.
#include <float.h>

#include "lbvh.cuh"
#include "render.cuh"

namespace gvc {

namespace {

constexpr int kKnnStack = 64;  // Karras depth is bounded by the 62 key + index bits

__global__ void __launch_bounds__(256) k_point_boxes(int64_t n, const float* __restrict__ pts,
                                                     float4* __restrict__ boxes) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 p = make_float4(pts[3 * i], pts[3 * i + 1], pts[3 * i + 2], 0.f);
    boxes[2 * i] = p;
    boxes[2 * i + 1] = p;
}

// Squared distance from q to the box [lo, hi]; for a degenerate box (a point) this is
// the point's squared distance ((dx*dx + dy*dy) + dz*dz, every operation rounded).
__device__ __forceinline__ float box_dist2(float qx, float qy, float qz, float lx, float ly, float lz, float hx,
                                           float hy, float hz) {
    const float gx = fmaxf(fmaxf(__fsub_rn(lx, qx), __fsub_rn(qx, hx)), 0.f);
    const float gy = fmaxf(fmaxf(__fsub_rn(ly, qy), __fsub_rn(qy, hy)), 0.f);
    const float gz = fmaxf(fmaxf(__fsub_rn(lz, qz), __fsub_rn(qz, hz)), 0.f);
    return __fadd_rn(__fadd_rn(__fmul_rn(gx, gx), __fmul_rn(gy, gy)), __fmul_rn(gz, gz));
}

__device__ __forceinline__ void keep3(float d, float& b0, float& b1, float& b2) {
    if (d < b2) {
        if (d < b1) {
            b2 = b1;
            if (d < b0) {
                b1 = b0;
                b0 = d;
            } else {
                b1 = d;
            }
        } else {
            b2 = d;
        }
    }
}

__global__ void __launch_bounds__(128) k_knn3(int64_t n, const float4* __restrict__ sorted_boxes,
                                              const int32_t* __restrict__ perm, const BvhNode* __restrict__ nodes,
                                              float* __restrict__ out, int* status) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 q = __ldg(sorted_boxes + 2 * i);
    float b0 = FLT_MAX, b1 = FLT_MAX, b2 = FLT_MAX;
    // bound from the Morton neighbours i-3 .. i+3
    const int64_t j0 = i >= 3 ? i - 3 : 0, j1 = i + 3 < n ? i + 3 : n - 1;
    for (int64_t j = j0; j <= j1; j++) {
        if (j == i) continue;
        const float4 p = __ldg(sorted_boxes + 2 * j);
        keep3(box_dist2(q.x, q.y, q.z, p.x, p.y, p.z, p.x, p.y, p.z), b0, b1, b2);
    }
    const float reject = b2;
    b0 = b1 = b2 = FLT_MAX;

    int stack[kKnnStack];
    float sdist[kKnnStack];
    int sp = 0;
    int node = 0;
    while (true) {
        const float4* np = reinterpret_cast<const float4*>(nodes + node);
        const float4 a = __ldg(np), b = __ldg(np + 1), c = __ldg(np + 2), d = __ldg(np + 3);
        const uint32_t cl = __float_as_uint(a.w), cr = __float_as_uint(b.w);
        const float dl = box_dist2(q.x, q.y, q.z, a.x, a.y, a.z, b.x, b.y, b.z);
        const float dr = box_dist2(q.x, q.y, q.z, c.x, c.y, c.z, d.x, d.y, d.z);
        // leaves: the box distance is the point distance
        if ((cl & kLeafBit) && (int64_t)(cl & ~kLeafBit) != i) keep3(dl, b0, b1, b2);
        if ((cr & kLeafBit) && (int64_t)(cr & ~kLeafBit) != i) keep3(dr, b0, b1, b2);
        const float bound = fminf(reject, b2);
        const bool gl = !(cl & kLeafBit) && dl <= bound;
        const bool gr = !(cr & kLeafBit) && dr <= bound;
        if (gl && gr) {
            const bool left_first = dl <= dr;
            if (sp < kKnnStack) {
                stack[sp] = (int)(left_first ? cr : cl);
                sdist[sp] = left_first ? dr : dl;
                sp++;
            } else {
                atomicOr(status, kStatusStackOverflow);
            }
            node = (int)(left_first ? cl : cr);
            continue;
        }
        if (gl || gr) {
            node = (int)(gl ? cl : cr);
            continue;
        }
        // pop the next subtree that can still hold a closer point
        bool found = false;
        while (sp > 0) {
            sp--;
            if (sdist[sp] <= fminf(reject, b2)) {
                node = stack[sp];
                found = true;
                break;
            }
        }
        if (!found) break;
    }
    out[perm[i]] = __fdiv_rn(__fadd_rn(__fadd_rn(b0, b1), b2), 3.0f);
}

inline unsigned nblk(int64_t n, int t) { return (unsigned)((n + t - 1) / t); }

}  // namespace

cudaError_t launch_point_boxes(int64_t n, const float* pts, float4* boxes, cudaStream_t st) {
    if (n <= 0) return cudaSuccess;
    k_point_boxes<<<nblk(n, 256), 256, 0, st>>>(n, pts, boxes); gvc::note_launch();
    return cudaGetLastError();
}

cudaError_t launch_knn3(int64_t n, const float4* sorted_boxes, const int32_t* perm, const BvhNode* nodes, float* out,
                        int* status, cudaStream_t st) {
    if (n <= 0) return cudaSuccess;
    k_knn3<<<nblk(n, 128), 128, 0, st>>>(n, sorted_boxes, perm, nodes, out, status); gvc::note_launch();
    return cudaGetLastError();
}

}  // namespace gvc
