// traverse.cuh -- warp-cooperative LBVH traversals: with a shared-memory node stack
// (warp_traverse) and stackless by escape edges (warp_traverse_stackless, below).
//
// One warp answers one box query (a 32-sample tile box, or one Gaussian's AABB).
// Each round the warp pops up to 32 internal nodes (one per lane), tests both
// children's boxes of every popped node against the query box in parallel, and
// compacts the hits with ballots: internal children go back on the warp's stack,
// leaves go to a candidate buffer.  Whenever 32 candidates are buffered the visitor
// evaluates them as one batch.  The whole loop is warp-uniform (no per-thread
// stacks, no divergence in the traversal itself), so a query issues one round of
// independent node loads per tree level instead of one dependent load per node.
//
// Replaces cuBQL::fixedBoxQuery::forEachLeaf / forEachPrim as used at
// diff-gaussian-rasterization/cuda_rasterizer/forward.cu:150,209 and
// backward.cu:243,378 (closed-box overlap; candidates are then tested per lane).
#pragma once
#include "gvc_internal.cuh"

namespace gvc {

__device__ __forceinline__ uint32_t lane_lt_mask() {
    uint32_t m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

__device__ __forceinline__ bool box_overlap(float4 lo, float4 hi, float3 qlo, float3 qhi) {
    return lo.x <= qhi.x && hi.x >= qlo.x && lo.y <= qhi.y && hi.y >= qlo.y && lo.z <= qhi.z && hi.z >= qlo.z;
}

// Candidate buffer capacity: a round adds at most 64 leaves to at most 31 pending.
constexpr int kCandCap = 96;
// Headroom kept free on the stack so that the remaining descent (one node popped
// per round, at most one net push per level) cannot overflow.
constexpr int kStackHeadroom = 128;

// Returns 0, or kStatusStackOverflow if nodes had to be dropped (results invalid).
// `visit(const int* cand, int nb)` is warp-collective and must end with __syncwarp().
// Per-warp traversal counters (warp-uniform values).
struct TravCount {
    int max_sp = 0;   // deepest stack
    int nodes = 0;    // internal nodes popped
    int leaves = 0;   // leaves handed to the visitor
};

template <class Visitor>
__device__ __forceinline__ int warp_traverse(const BvhNode* __restrict__ nodes, float3 qlo, float3 qhi,
                                             int* __restrict__ stack, int* __restrict__ cand, Visitor& visit,
                                             TravCount& tc) {
    const int lane = threadIdx.x & 31;
    const uint32_t lt = lane_lt_mask();
    int status = 0;
    int sp = 1;
    if (lane == 0) stack[0] = 0;
    __syncwarp();
    int nc = 0;
    while (sp > 0) {
        int k = min(sp, 32);
        const int room = kStackCap - kStackHeadroom - sp;
        if (k > room) k = max(room, 1);
        const int base = sp - k;
        tc.nodes += k;
        const int node = (lane < k) ? stack[base + lane] : 0;
        __syncwarp();
        sp = base;
        bool hl = false, hr = false;
        uint32_t cl = 0, cr = 0;
        if (lane < k) {
            const float4* np = reinterpret_cast<const float4*>(nodes + node);
            const float4 a = __ldg(np), b = __ldg(np + 1), c = __ldg(np + 2), d = __ldg(np + 3);
            cl = __float_as_uint(a.w);
            cr = __float_as_uint(b.w);
            hl = box_overlap(a, b, qlo, qhi);
            hr = box_overlap(c, d, qlo, qhi);
        }
        const bool ll = hl && (cl & kLeafBit), lr = hr && (cr & kLeafBit);
        const bool il = hl && !(cl & kLeafBit), ir = hr && !(cr & kLeafBit);
        const uint32_t mll = __ballot_sync(0xffffffffu, ll), mlr = __ballot_sync(0xffffffffu, lr);
        const uint32_t mil = __ballot_sync(0xffffffffu, il), mir = __ballot_sync(0xffffffffu, ir);
        const int nll = __popc(mll), nlr = __popc(mlr), nil = __popc(mil), nir = __popc(mir);
        if (ll) cand[nc + __popc(mll & lt)] = (int)(cl & ~kLeafBit);
        if (lr) cand[nc + nll + __popc(mlr & lt)] = (int)(cr & ~kLeafBit);
        nc += nll + nlr;
        tc.leaves += nll + nlr;
        if (sp + nil + nir > kStackCap) {
            status = kStatusStackOverflow;
        } else {
            if (il) stack[sp + __popc(mil & lt)] = (int)cl;
            if (ir) stack[sp + nil + __popc(mir & lt)] = (int)cr;
            sp += nil + nir;
        }
        tc.max_sp = max(tc.max_sp, sp);
        __syncwarp();
        while (nc >= 32) {
            visit(cand + nc - 32, 32);
            nc -= 32;
        }
    }
    if (nc > 0) visit(cand, nc);
    return status;
}

// ---------------------------------------------------------------------------------------
// Stackless variant.  An edge (k, s) links internal node k to its child s (0 left, 1
// right); its box is the child's box, held in node k, and its code is 2k + s.  Walking
// the edges in pre-order needs no stack: after edge (k, 0) and its subtree comes (k, 1);
// after (k, 1) and its subtree comes the escape edge of node k, stored in node k's c.w
// (k_pack_nodes): (p, 1) for the nearest ancestor-or-self of k that is a left child of
// p, kEdgeEnd on the root's right spine.  Node k's d.w repeats its right child, so one
// edge is two float4: (a, b) for s = 0 (child in a.w), (c, d) for s = 1 (child in d.w,
// escape in c.w).
//
// The warp first descends level by level from the root, one overlapping internal node
// per lane, while a level's overlapping internal children fit 32 lanes (every node's
// two children tested in parallel, as in warp_traverse).  When the next level would
// not fit, each lane walks the subtree of its node by escape edges: edge (k, 0) up to
// node k's escape edge, one edge per step, the 32 walks in parallel.  Leaves found in
// either phase go through the same candidate buffer and visitor, so the candidate set
// equals warp_traverse's (the order differs).  Nothing is stored per node visited: no
// capacity can overflow.
// ---------------------------------------------------------------------------------------
constexpr uint32_t kEdgeEnd = 0xffffffffu;

// Lane index of the (r + 1)-th set bit of m (r < popc(m)): binary search on prefix counts.
__device__ __forceinline__ int nth_set_bit(uint32_t m, int r) {
    int p = 0;
#pragma unroll
    for (int b = 16; b > 0; b >>= 1)
        if (__popc(m & ((1u << (p + b)) - 1u)) <= r) p += b;
    return p;
}

// n_internal: internal nodes of the tree.  A level count or a lane's walk longer than
// the tree allows (2 n_internal edges) can only come from corrupt links; the traversal
// then stops and returns kStatusStackOverflow instead of looping.
template <class Visitor>
__device__ __forceinline__ int warp_traverse_stackless(const BvhNode* __restrict__ nodes, int64_t n_internal,
                                                       float3 qlo, float3 qhi, int* __restrict__ cand,
                                                       Visitor& visit, TravCount& tc) {
    const int lane = threadIdx.x & 31;
    const uint32_t lt = lane_lt_mask();
    int status = 0;
    int nc = 0;
    int nf = 1;           // overlapping internal nodes of the current level, one per lane
    uint32_t fnode = 0u;  // this lane's node (lane < nf)
    uint32_t fesc = kEdgeEnd;
    bool walk = false;
    for (int64_t level = 0; nf > 0; level++) {
        if (level > n_internal) {
            status = kStatusStackOverflow;
            break;
        }
        bool hl = false, hr = false;
        uint32_t cl = 0, cr = 0;
        if (lane < nf) {
            const float4* np = reinterpret_cast<const float4*>(nodes + fnode);
            const float4 a = __ldg(np), b = __ldg(np + 1), c = __ldg(np + 2), d = __ldg(np + 3);
            cl = __float_as_uint(a.w);
            cr = __float_as_uint(b.w);
            fesc = __float_as_uint(c.w);
            hl = box_overlap(a, b, qlo, qhi);
            hr = box_overlap(c, d, qlo, qhi);
        }
        const bool il = hl && !(cl & kLeafBit), ir = hr && !(cr & kLeafBit);
        const uint32_t mil = __ballot_sync(0xffffffffu, il), mir = __ballot_sync(0xffffffffu, ir);
        const int nil = __popc(mil), nir = __popc(mir);
        if (nil + nir > 32) {  // warp-uniform: the next level does not fit; walk this level's subtrees
            walk = true;
            break;
        }
        tc.nodes += nf;
        const bool ll = hl && (cl & kLeafBit), lr = hr && (cr & kLeafBit);
        const uint32_t mll = __ballot_sync(0xffffffffu, ll), mlr = __ballot_sync(0xffffffffu, lr);
        const int nll = __popc(mll), nlr = __popc(mlr);
        if (ll) cand[nc + __popc(mll & lt)] = (int)(cl & ~kLeafBit);
        if (lr) cand[nc + nll + __popc(mlr & lt)] = (int)(cr & ~kLeafBit);
        nc += nll + nlr;
        tc.leaves += nll + nlr;
        // next level: lane j takes the j-th overlapping internal child, left children first
        const bool from_left = lane < nil;
        const int rank = from_left ? lane : lane - nil;
        const int src = (lane < nil + nir) ? nth_set_bit(from_left ? mil : mir, rank) : 0;
        const uint32_t vl = __shfl_sync(0xffffffffu, cl, src);
        const uint32_t vr = __shfl_sync(0xffffffffu, cr, src);
        fnode = from_left ? vl : vr;
        nf = nil + nir;
        __syncwarp();
        while (nc >= 32) {
            visit(cand + nc - 32, 32);
            nc -= 32;
        }
    }
    if (walk) {
        bool act = lane < nf;
        uint32_t cur = 2u * fnode;
        const uint32_t stop = fesc;
        const int64_t max_steps = 2 * n_internal;
        for (int64_t step = 0; __any_sync(0xffffffffu, act); step++) {
            if (step > max_steps) {
                status = kStatusStackOverflow;
                break;
            }
            tc.nodes += __popc(__ballot_sync(0xffffffffu, act && !(cur & 1u)));
            bool leaf = false;
            uint32_t lid = 0;
            if (act) {
                const uint32_t k = cur >> 1, s = cur & 1u;
                const float4* np = reinterpret_cast<const float4*>(nodes + k) + 2 * s;
                const float4 lo = __ldg(np), hi = __ldg(np + 1);
                const uint32_t child = __float_as_uint(s ? hi.w : lo.w);
                const bool hit = box_overlap(lo, hi, qlo, qhi);
                if (hit && !(child & kLeafBit)) {
                    cur = 2u * child;
                } else {
                    leaf = hit;
                    lid = child & ~kLeafBit;
                    cur = s ? __float_as_uint(lo.w) : (cur | 1u);
                }
                act = cur != stop;
            }
            const uint32_t m = __ballot_sync(0xffffffffu, leaf);
            if (leaf) cand[nc + __popc(m & lt)] = (int)lid;
            nc += __popc(m);
            tc.leaves += __popc(m);
            __syncwarp();
            if (nc >= 32) {
                visit(cand + nc - 32, 32);
                nc -= 32;
            }
        }
    }
    if (nc > 0) visit(cand, nc);
    return status;
}

// The kernels' STACKLESS template parameter picks the traversal at compile time.
template <bool STACKLESS, class Visitor>
__device__ __forceinline__ int warp_traverse_sel(const BvhNode* __restrict__ nodes, int64_t n_internal, float3 qlo,
                                                 float3 qhi, int* __restrict__ stack, int* __restrict__ cand,
                                                 Visitor& visit, TravCount& tc) {
    if constexpr (STACKLESS)
        return warp_traverse_stackless(nodes, n_internal, qlo, qhi, cand, visit, tc);
    else
        return warp_traverse(nodes, qlo, qhi, stack, cand, visit, tc);
}

// Sum of 16 per-lane values across the warp with 16 shuffles (recursive halving):
// on return lanes 2k and 2k+1 hold the warp total of value k.
__device__ __forceinline__ float warp_transpose_reduce16(float (&v)[16]) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int i = 0; i < 8; i++) {
        const bool up = lane & 16;
        float send = up ? v[i] : v[i + 8];
        float keep = up ? v[i + 8] : v[i];
        v[i] = keep + __shfl_xor_sync(0xffffffffu, send, 16);
    }
#pragma unroll
    for (int i = 0; i < 4; i++) {
        const bool up = lane & 8;
        float send = up ? v[i] : v[i + 4];
        float keep = up ? v[i + 4] : v[i];
        v[i] = keep + __shfl_xor_sync(0xffffffffu, send, 8);
    }
#pragma unroll
    for (int i = 0; i < 2; i++) {
        const bool up = lane & 4;
        float send = up ? v[i] : v[i + 2];
        float keep = up ? v[i + 2] : v[i];
        v[i] = keep + __shfl_xor_sync(0xffffffffu, send, 4);
    }
    {
        const bool up = lane & 2;
        float send = up ? v[0] : v[1];
        float keep = up ? v[1] : v[0];
        v[0] = keep + __shfl_xor_sync(0xffffffffu, send, 2);
    }
    return v[0] + __shfl_xor_sync(0xffffffffu, v[0], 1);
}

}  // namespace gvc
