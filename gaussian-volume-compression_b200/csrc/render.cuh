// render.cuh -- launch interfaces of the forward / backward evaluation kernels and
// of the preprocessing kernels (prep.cu).
#pragma once
#include "gvc_internal.cuh"

namespace gvc {

struct FwdArgs {
    const float4* s_sorted;
    const float4* tile_boxes;  // group boxes [n_tiles * kGroups]
    const uint32_t* gdesc;     // [n_tiles]
    int64_t n_tiles;
    const BvhNode* gnodes;
    const GaussRec* recs;
    float* out_cells;
    float* out_weights;
    int* status;
    unsigned long long* stats;
    bool count;
};

struct BwdArgs {
    int64_t P;
    const int32_t* gorder;  // processing order (sorted pos -> caller idx) or null
    const int32_t* gperm;   // LBVH order -> caller idx (atomic mode)
    const float* means;
    const float* values;
    const float* weights;
    const float* conics;
    const float4* boxes;  // caller order, lo/hi
    const float4* s_sorted;
    const float4* s_grad;      // (x, y, z, gx) per sorted slot
    const float* s_gyz;        // gyz per sorted slot
    const uint8_t* s_ok;       // W > 0.01 per sorted slot (pair statistics)
    const float4* tile_boxes;  // group boxes [n_tiles * kGroups]
    const uint32_t* gdesc;     // [n_tiles]
    int64_t n_tiles;
    const BvhNode* tnodes;  // sample-group LBVH
    const BvhNode* gnodes;  // Gaussian LBVH (atomic and tensor-core modes)
    int64_t g_internal;     // its internal nodes
    bool stackless;         // tensor-core mode: traverse by escape edges (warp_traverse_stackless)
    const int32_t* clog;    // tensor-core mode: the forward's candidate log (null: traverse)
    const int32_t* cend;
    const uint2* cdesc;     // the forward's block groups (the log's groups)
    const GaussRec* recs;   // LBVH order (atomic mode)
    float* gacc;            // [P][16] caller order
    int* status;
    unsigned long long* stats;
    bool count;
};

cudaError_t launch_forward(const FwdArgs& a, cudaStream_t st);

// Candidate log of the block-group forwards, read by the tensor-core backward instead of
// walking the Gaussian LBVH again: the forward's producer appends the candidates of a
// block's groups in order to the block's kCandLogPerBlock slots, and group g's candidates
// end at cend[blk * 8 + g]; a block with more candidates than slots gets -1 for every
// group, and the backward walks the tree for it.
constexpr int kCandLogPerBlock = 4096;

struct CandLog {
    int32_t* ids = nullptr;  // this block's slots, or null (no log)
    int pos = 0;             // candidates appended (warp-uniform)
    bool over = false;
    int gend = 0;  // on lane g: end of group g

    __device__ __forceinline__ void append(const int* c, int nb) {
        if (!ids) return;
        const int lane = threadIdx.x & 31;
        if (pos + nb <= kCandLogPerBlock) {
            if (lane < nb) ids[pos + lane] = c[lane];
        } else {
            over = true;
        }
        pos += nb;
    }
    __device__ __forceinline__ void end_group(int g) {
        if ((threadIdx.x & 31) == g) gend = pos;
    }
    __device__ __forceinline__ void finish(int32_t* cend_blk, int ng) {
        if (ids && (int)(threadIdx.x & 31) < ng) cend_blk[threadIdx.x & 31] = over ? -1 : gend;
    }
};

// cta.cu: CTA-level forward on 128-sample blocks (tensor-core or SIMT exponent)
struct CtaArgs {
    const float4* s_sorted;
    int64_t S;
    const uint2* bdesc;    // [n_blocks] block-group descriptors
    const float4* bboxes;  // [n_blocks * 8] block-group boxes (lo, hi)
    const BvhNode* gnodes;
    int64_t n_internal;    // internal nodes of gnodes
    bool stackless;        // traverse by escape edges (warp_traverse_stackless)
    int32_t* clog;         // candidate log [n_blocks * kCandLogPerBlock], or null
    int32_t* cend;         // group ends of the log [n_blocks * 8]
    const GaussRec* recs;
    float* out_cells;
    float* out_weights;
    float2* out_sorted;    // (out, W) per sorted slot, read by the backward's sample records; or null
    int* status;
    unsigned long long* stats;
    bool count;
};
// Block groups split where both halves' boxes have at most `ratio` of the whole's
// half-perimeter: kBlockSplitForward for the forward, kBlockSplitBackward (finer) for the
// tensor-core backward.
constexpr float kBlockSplitForward = 0.45f;
constexpr float kBlockSplitBackward = 0.65f;
// Block groups with `ratio`; with bdesc2 also a second set with `ratio2` from the same
// loaded rows (one launch).
cudaError_t launch_sample_blocks(int64_t S, const float4* s_sorted, const uint32_t* skeys, uint2* bdesc,
                                 float4* bboxes, float ratio, cudaStream_t st, uint2* bdesc2 = nullptr,
                                 float4* bboxes2 = nullptr, float ratio2 = 0.f);
cudaError_t launch_forward_cta(const CtaArgs& a, bool tc, cudaStream_t st);
// fwd_tc.cu: the forward with the exponent on tcgen05 (launch_forward_cta(a, true) calls it)
cudaError_t launch_forward_tc(const CtaArgs& a, cudaStream_t st);
cudaError_t launch_tc_gemm_test(const void* A, const void* B, int N, float* D, int* status, cudaStream_t st);
// One block waiting on an mbarrier nothing arrives on: the bounded wait runs out and
// records kStatusTimeout (tests the host-side report of device timeouts).
cudaError_t launch_wait_timeout_test(int* status, cudaStream_t st);
cudaError_t launch_backward_gauss(const BwdArgs& a, cudaStream_t st);
// bwd_tc.cu: backward on 128-sample blocks with the reduction over samples on tcgen05
cudaError_t launch_backward_cta(const BwdArgs& a, int64_t n_blocks, const uint2* bdesc, const float4* bboxes,
                                cudaStream_t st);
cudaError_t launch_backward_tiles(const BwdArgs& a, cudaStream_t st);
cudaError_t launch_finalize(int64_t P, const float* gacc, const float* scales, const float* rots, const float* conics,
                            float sm, int ref_compat, float* dmeans, float* dscales, float* drots, float* dvalues,
                            float* dweights, cudaStream_t st);

// prep.cu (compiled without FMA contraction so that its arithmetic matches the oracle)
cudaError_t launch_preprocess(int64_t P, const float* means, const float* scales, const float* rots,
                              const float* weights, float sm, float* conics_out, float4* boxes_out, cudaStream_t st);
cudaError_t launch_gather_recs(int64_t P, const int32_t* perm, const float* means, const float* values,
                               const float* weights, const float* conics, const float4* boxes, GaussRec* recs,
                               cudaStream_t st);
cudaError_t launch_sample_tiles(int64_t S, int64_t n_tiles, const float* samples, const int32_t* perm,
                                const uint32_t* skeys, float4* s_sorted, float4* group_boxes, uint32_t* group_keys,
                                uint32_t* gdesc, bool with_groups, cudaStream_t st);
// out_sorted: the forward's (out, W) per sorted slot when the caller's out_cells /
// out_weights are that forward's outputs (else null: they are gathered).
cudaError_t launch_sample_grads(int64_t n_slots, const float4* s_sorted, const float2* out_sorted,
                                const float* out_cells, const float* out_weights, const float* gout, const float* gw,
                                float4* s_grad, float* s_gyz, uint8_t* s_ok, cudaStream_t st);
cudaError_t launch_fill_zero_outputs(int64_t S, float* out_cells, float* out_weights, cudaStream_t st);

// mesh.cu
cudaError_t launch_sample_uniform(const int64_t dims[3], const float origin[3], const float spacing[3],
                                  const void* values, int dtype, int64_t N, const float* samples, void* out,
                                  cudaStream_t st);
cudaError_t launch_tet_boxes(int64_t C, const float* pts, const int32_t* conn4, float4* boxes, cudaStream_t st);
cudaError_t launch_cell_boxes(int64_t C, const float* pts, const uint8_t* types, const int64_t* offsets,
                              const int32_t* conn, float4* boxes, cudaStream_t st);
cudaError_t launch_sample_cells(int64_t N, const float* samples, const int32_t* sperm, const float* pts,
                                const uint8_t* types, const int64_t* offsets, const int32_t* conn,
                                const double* values, const BvhNode* cnodes, const int32_t* cperm, int64_t C,
                                double* out, int64_t* cell_ids, int* status, cudaStream_t st);
cudaError_t launch_sample_tets(int64_t N, const float* samples, const int32_t* sperm, const float* pts,
                               const int32_t* conn4, const double* values, const BvhNode* cnodes,
                               const int32_t* cperm, int64_t C, double* out, int64_t* cell_ids, int* status,
                               cudaStream_t st);

// trainsamp.cu
cudaError_t launch_tet_points(int64_t N, int64_t S, uint64_t seed, const float* pts, const int32_t* conn4, int64_t C,
                              float* out, uint32_t* w_lo, uint32_t* w_hi, uint32_t* w_batch, cudaStream_t st);
cudaError_t launch_gather_points(int64_t N, const float* src, const int32_t* perm, float* dst, cudaStream_t st);
cudaError_t launch_to_f32(int64_t N, const double* src, float* dst, cudaStream_t st);

// knn.cu
cudaError_t launch_point_boxes(int64_t n, const float* pts, float4* boxes, cudaStream_t st);
cudaError_t launch_knn3(int64_t n, const float4* sorted_boxes, const int32_t* perm, const BvhNode* nodes, float* out,
                        int* status, cudaStream_t st);

}  // namespace gvc
