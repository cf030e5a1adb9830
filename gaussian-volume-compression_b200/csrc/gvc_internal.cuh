// gvc_internal.cuh -- shared device helpers, constants and the context layout.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <string>

#include "gvc.h"

namespace gvc {

// diff-gaussian-rasterization/cuda_rasterizer/config.h:9
constexpr float kWeightCutoff = 1e-2f;
// forward.cu:166 / forward.cu:235: power window [-14, 0]
constexpr float kPowerFloor = -14.0f;
// Tile of Morton-sorted samples handled by one warp.
constexpr int kTile = 32;
// Each tile is split into at most this many lane groups at Morton-order jumps; the
// sample-side LBVH has one leaf slot per (tile, group).
constexpr int kGroups = 4;
// Per-warp traversal stack (entries of int32) in shared memory.
constexpr int kStackCap = 512;
// Gaussians whose covariance condition estimate exceeds this get an FP64 inverse.
constexpr float kCondFp64 = 1.0e2f;

// Counts kernel launches issued by this library (reported by gvc_launch_count()).
void note_launch(int n = 1);

// Device status bits (OR-ed into ctx->d_status).
constexpr int kStatusStackOverflow = 1;
constexpr int kStatusTimeout = 2;  // a bounded wait gave up (mbarrier, radix-sort look-back)

// Gaussian evaluation record, one per Gaussian in LBVH (Morton) order: 80 bytes.
//   r0 = (mu.x, mu.y, mu.z, w)
//   r1 = (c0, c1, c2, c3)  -- conic xx, xy, xz, yy as written to the conics output
//   r2 = (c4, c5, v, 0)    -- conic yz, zz, value
//   r3 = (lo.x, lo.y, lo.z, 0), r4 = (hi.x, hi.y, hi.z, 0): the AABB
struct __align__(16) GaussRec {
    float4 r0, r1, r2, r3, r4;
};

// LBVH internal node with both children's boxes: 64 bytes.
//   a = (L.lo.xyz, left child bits), b = (L.hi.xyz, right child bits),
//   c = (R.lo.xyz, escape edge),     d = (R.hi.xyz, right child bits)
// Child encoding: internal node k >= 0; leaf i stored as (i | 0x80000000).  The escape
// edge (2p + s: child s of node p, 0xffffffff for none) is the edge that follows this
// node's subtree in pre-order; the stackless traversal (traverse.cuh) walks by it.
struct __align__(16) BvhNode {
    float4 a, b, c, d;
};

constexpr uint32_t kLeafBit = 0x80000000u;

// Growable device buffer owned by the context.
struct DevBuf {
    void* ptr = nullptr;
    size_t bytes = 0;
    cudaError_t ensure(size_t need) {
        if (need <= bytes && ptr) return cudaSuccess;
        if (ptr) {
            cudaError_t e = cudaFree(ptr);
            if (e != cudaSuccess) return e;
            ptr = nullptr;
            bytes = 0;
        }
        size_t n = need < 256 ? 256 : need;
        n = (n + 255) & ~size_t(255);
        cudaError_t e = cudaMalloc(&ptr, n);
        if (e == cudaSuccess) bytes = n;
        return e;
    }
    template <class T>
    T* as() const { return reinterpret_cast<T*>(ptr); }
    void release() {
        if (ptr) cudaFree(ptr);
        ptr = nullptr;
        bytes = 0;
    }
};

// Radix-sort workspace and LBVH storage for one set of boxes.
struct Lbvh {
    int64_t n = 0;
    DevBuf keys, keys_alt, perm, perm_alt;  // sorted keys / permutation (sorted pos -> input idx)
    DevBuf boxes;                           // input boxes [n] as 2 x float4 (lo, hi)
    DevBuf sorted_boxes;                    // leaf boxes in sorted order, 2 x float4
    DevBuf left, right, parent, flags;      // Karras hierarchy + refit counters
    DevBuf node_boxes;                      // [n-1] internal node boxes, 2 x float4
    DevBuf nodes;                           // [n-1] BvhNode
    DevBuf hist, bounds;                    // sort histograms, centroid bounds
    DevBuf onesweep;                        // one-kernel-per-pass sort: digit counts, tickets, look-back words
    int* status = nullptr;                  // device status word; null keeps the three-kernel sort passes
};

}  // namespace gvc

struct gvc_ctx {
    int device = 0;
    std::string err;
    // options
    int cov_grad_mode = 0;
    int bwd_mode = 0;
    int eval_path = 0;
    int traversal = 0;      // 0 = node stack, 1 = stackless (GVC_OPT_TRAVERSAL)
    int cand_log = 1;       // GVC_OPT_CAND_LOG
    int count_pairs = 0;
    int time_kernels = 0;   // record CUDA events around the evaluation kernels
    double fwd_kernel_ms = 0.0, bwd_kernel_ms = 0.0;
    int64_t fwd_kernel_calls = 0, bwd_kernel_calls = 0;
    cudaEvent_t ev_pool[64];  // pairs of (start, stop) events pending read-out
    int ev_kind[32];          // 0 = forward, 1 = backward
    int ev_pending = 0;
    bool ev_init = false;
    // sample state (gvc_build_bvh)
    const float* samples = nullptr;
    int64_t S = 0;
    int64_t n_tiles = 0;
    bool samples_ready = false;
    // candidate log of the last block-group forward (for the tensor-core backward)
    gvc::DevBuf clog, cend;
    bool clog_ready = false;
    // (out, W) per sorted slot as the last FP32 block-group forward wrote them, and the
    // output arrays it wrote them to (the backward uses the copy for those arrays only)
    gvc::DevBuf fwd_sorted;
    const float* fwd_out_cells = nullptr;
    const float* fwd_out_weights = nullptr;
    bool fwd_sorted_ready = false;
    // the Gaussian arrays of the last forward: its AABBs (gtmp) and records (grec) are
    // reused by a backward handed the same arrays
    const float* fwd_means = nullptr;
    const float* fwd_scales = nullptr;
    const float* fwd_rots = nullptr;
    const float* fwd_values = nullptr;
    const float* fwd_weights = nullptr;
    const float* fwd_conics = nullptr;
    float fwd_scale_mod = 0.f;
    bool fwd_recs_ready = false;
    gvc::DevBuf s_sorted;   // [n_tiles*32] float4 (x, y, z, bits of caller index or -1)
    gvc::DevBuf tile_boxes; // [n_tiles * kGroups] group boxes, 2 x float4 (empty for unused slots)
    gvc::DevBuf tile_keys;  // [n_tiles * kGroups] uint32 Morton key of each group's first sample
    gvc::DevBuf tile_gdesc; // [n_tiles] group starts: bytes 0..2 = start lane of groups 1..3
                            // (32 if unused), byte 3 = number of groups
    gvc::DevBuf blk_desc;   // [ceil(S/128)] uint2 block-group descriptors (CTA kernels)
    gvc::DevBuf blk_boxes;  // [ceil(S/128) * 8] block-group boxes, 2 x float4
    gvc::DevBuf blk_desc_b;   // the same with the backward's finer split (built on first use)
    gvc::DevBuf blk_boxes_b;
    bool blk_b_ready = false;
    bool tiles_ready = false;        // sample-group LBVH built for the current samples
    bool tile_groups_ready = false;  // tile lane groups built for the current samples
    gvc::DevBuf s_grad;     // [n_tiles*32] float4 (x, y, z, gx) backward sample records
    gvc::DevBuf s_gyz;      // [n_tiles*32] float gyz (see k_sample_grads)
    gvc::DevBuf s_ok;       // [n_tiles*32] uint8 1 iff W > 0.01 (pair statistics only)
    gvc::Lbvh s_sort;       // sample sort (keys/perm only)
    gvc::Lbvh tiles;        // tile LBVH
    // Gaussian state (forward)
    int64_t P = 0;
    bool gauss_ready = false;
    gvc::Lbvh gbvh;         // Gaussian LBVH
    gvc::DevBuf grec;       // [P] GaussRec in LBVH order
    gvc::DevBuf gtmp;       // preprocess scratch: AABBs in caller order
    // mesh sampler
    gvc::Lbvh cells;
    // three-nearest-neighbour distances (point LBVH and its leaf boxes)
    gvc::Lbvh knn;
    gvc::DevBuf knn_boxes;
    // training sample batches: unsorted points, Morton / batch key words, FP64 values
    gvc::Lbvh ts_sort;
    gvc::DevBuf ts_points, ts_words, ts_gt64;
    gvc::DevBuf m_out_sorted;
    // status and statistics
    int* d_status = nullptr;          // device status word
    unsigned long long* d_stats = nullptr;  // [16] device counters
    int* h_status = nullptr;          // pinned mirror
};
