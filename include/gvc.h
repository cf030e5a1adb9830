/*
 * gvc.h -- C ABI of the B200 Gaussian-mixture volume path (libgvc.so).
 *
 * Plain pointers and sizes only: every float / int pointer below is a DEVICE pointer
 * on the context's device unless stated otherwise, and `stream` is a cudaStream_t
 * passed as void* (NULL = legacy default stream).  All calls are stream-ordered and
 * do not synchronise the device unless `debug` is non-zero.
 *
 * Each entry point names the reference interface it replaces (paths inside the
 * reference project schakrabarti-lanl/gaussian-volume-compression).
 *
 * Return value: 0 (GVC_OK) or a gvc_status code; gvc_last_error() gives the message.
 * Device-side failures (a traversal stack overflow) are recorded in a status word and
 * reported by gvc_sync_status() and by the next call on the same context.
 */
#ifndef GVC_H_INCLUDED
#define GVC_H_INCLUDED

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct gvc_ctx gvc_ctx;

typedef enum {
    GVC_OK = 0,
    GVC_ERR_ARG = 1,         /* bad argument (shape, size, null pointer, dtype)      */
    GVC_ERR_CUDA = 2,        /* a CUDA runtime call failed                            */
    GVC_ERR_CAPACITY = 3,    /* a size exceeds a documented maximum                   */
    GVC_ERR_TRAVERSAL = 4,   /* a BVH traversal stack overflowed (results invalid)    */
    GVC_ERR_UNSUPPORTED = 5, /* unsupported cell type / dtype                         */
    GVC_ERR_STATE = 6,       /* call order violated (forward before build_bvh, ...)   */
    GVC_ERR_TIMEOUT = 7      /* a bounded device-side wait ran out (results invalid) */
} gvc_status;

/* Options for gvc_set_option. */
typedef enum {
    GVC_OPT_COV_GRAD = 1,   /* 0 = true gradient of the forward (default),
                               1 = reference-compatible formula of
                                   diff-gaussian-rasterization/cuda_rasterizer/backward.cu:50-124 */
    GVC_OPT_BWD_MODE = 2,   /* 0 = follow use_gaussian_bvh (default):
                                   use_gaussian_bvh == 0 -> Gaussian-owned segmented reduction
                                   (deterministic, no atomics; mirrors backward.cu:127-337),
                                   use_gaussian_bvh != 0 -> sample-tile traversal with warp
                                   pre-reduction + FP32 atomics (mirrors backward.cu:339-559);
                                   (with GVC_OPT_EVAL_PATH = 1: the tensor-core reduction, 3);
                               1 = always deterministic, 2 = always sample-tile atomic,
                               3 = tensor core: per 128-sample block, the per-Gaussian sums
                                   over samples as a tcgen05 BF16 3-way split GEMM in TMEM,
                                   FP32 atomics (not bitwise reproducible)                  */
    GVC_OPT_EVAL_PATH = 3,  /* forward evaluation kernel (all compute the same field):
                               0 = FP32 exponent, one CTA per 128-sample block: a producer warp
                                   walks the Gaussian LBVH and stages batches, two consumer
                                   warps evaluate two samples per thread (default, fastest),
                               1 = tensor-core exponent: the same pipeline with the power as a
                                   tcgen05 BF16 3-way split MMA into TMEM,
                               2 = FP32 exponent, one warp per 32-sample tile               */
    GVC_OPT_COUNT_PAIRS = 4,/* 1 = record per-call pair counts (gvc_get_stats)            */
    GVC_OPT_TIME_KERNELS = 5,/* 1 = time the evaluation kernels with CUDA events on the
                                caller's stream (gvc_get_stats)                          */
    GVC_OPT_TRAVERSAL = 6,  /* Gaussian-LBVH traversal of the block-group forwards (eval
                               paths 0 and 1) and of the tensor-core backward (same
                               candidates, same results up to summation order):
                               0 = warp-cooperative with a shared-memory node stack (default),
                               1 = stackless: level-synchronous descent while a level's
                                   overlapping nodes fit the warp, then one subtree per lane
                                   walked by escape edges stored in the nodes              */
    GVC_OPT_CAND_LOG = 7    /* 1 (default) = when the tensor-core backward is selected, the
                               block-group forward records every block's candidate Gaussians
                               (kCandLogPerBlock = 4096 per 128-sample block, 16 KB) and the
                               backward reads them back instead of walking the Gaussian LBVH
                               again (each of its finer block groups keeps the candidates of
                               the enclosing forward group whose boxes overlap its own);
                               blocks with more candidates are walked, and without device
                               memory for the log the forward runs without it.
                               0 = always walk.                                            */
} gvc_option;

typedef struct {
    int64_t fwd_candidates;   /* (sample, Gaussian) pairs with the sample inside the AABB   */
    int64_t fwd_contributing; /* ... and -14 <= power <= 0                                  */
    int64_t bwd_contributing; /* contributing pairs of samples with W > 0.01                */
    int32_t max_stack_fwd;    /* deepest traversal stack seen (entries)                     */
    int32_t max_stack_bwd;
    double fwd_kernel_ms;     /* summed duration of the forward evaluation kernel          */
    double bwd_kernel_ms;     /* summed duration of the backward evaluation kernel         */
    int64_t fwd_kernel_calls; /* launches timed since the option was set                   */
    int64_t bwd_kernel_calls;
    int64_t fwd_leaf_hits;    /* (tile, Gaussian) pairs evaluated by the forward            */
    int64_t fwd_node_visits;  /* internal LBVH nodes popped by the forward traversal        */
    int64_t bwd_leaf_hits;    /* (Gaussian or tile) leaves evaluated by the backward        */
    int64_t bwd_node_visits;
    int64_t fwd_lane_evals;   /* (sample, Gaussian) lane slots the forward evaluated (CTA paths) */
    int64_t bwd_rows;         /* (sample, Gaussian) rows the deterministic backward evaluated   */
} gvc_stats;

/* Context: owns the sample ordering, both LBVHs and all workspace (no per-call
   cudaMalloc once sizes stop growing).  Replaces the module statics samples_bvh,
   gaussian_bvh and stored_samples of diff-gaussian-rasterization/ext.cu:8-10.
   A context belongs to the device current at creation; use one context per thread. */
int gvc_ctx_create(gvc_ctx** out);
void gvc_ctx_destroy(gvc_ctx* ctx);
const char* gvc_last_error(const gvc_ctx* ctx);
int gvc_set_option(gvc_ctx* ctx, int option, int value);
int gvc_get_stats(gvc_ctx* ctx, gvc_stats* out, void* stream); /* synchronises `stream` */
/* Number of kernel launches this library has issued in the process so far (all
   contexts); no counterpart in the reference. */
int64_t gvc_launch_count(void);
/* Waits for `stream`, returns the device status word (GVC_OK, GVC_ERR_TRAVERSAL, or
   GVC_ERR_TIMEOUT when a kernel's bounded wait on a pipeline barrier or on another
   block's published count ran out) and clears it. */
int gvc_sync_status(gvc_ctx* ctx, void* stream);

/* Replaces BuildBVH (diff-gaussian-rasterization/ext.cu:28-65).
   samples: [S,3] float32.  The context keeps the POINTER: the caller keeps the buffer
   alive and unchanged until the next gvc_build_bvh (the reference keeps a tensor
   reference, ext.cu:29).  Sorts the samples by a 30-bit Morton key, forms 32-sample
   tiles and builds the tile LBVH (the reference's leaf threshold 257, ext.cu:51, has
   no counterpart: tiles are 32 samples). */
int gvc_build_bvh(gvc_ctx* ctx, const float* samples, int64_t S, int debug, int use_gaussian_bvh, void* stream);

/* Replaces RasterizeGaussiansCUDAWrapper / RasterizeGaussiansCUDA
   (diff-gaussian-rasterization/ext.cu:67-105, rasterize_points.cu:17-73).
   means3D [P,3], scales [P,3], rotations [P,4] (r,x,y,z), values [P], weights [P];
   bounds = {min_x, min_y, min_z, max_x, max_y, max_z} and bg are accepted and unused,
   as in the reference.  Outputs (caller-allocated): out_cells [S], out_weights [S],
   conics [6P].  P == 0 writes zeros (rasterize_points.cu:51). */
int gvc_rasterize_gaussians(gvc_ctx* ctx, int64_t P, const float* means3D, const float* scales,
                            const float* rotations, const float* values, const float* weights, float scale_modifier,
                            const float* bounds /* host, 6 floats, may be NULL */, float bg, int use_gaussian_bvh,
                            int debug, float* out_cells, float* out_weights, float* conics, void* stream);

/* Replaces RasterizeGaussiansBackwardCUDAWrapper / RasterizeGaussiansBackwardCUDA
   (diff-gaussian-rasterization/ext.cu:107-147, rasterize_points.cu:75-137).
   Outputs (caller-allocated, overwritten): dmeans [P,3], dscales [P,3], drots [P,4],
   dvalues [P], dweights [P]. */
int gvc_rasterize_gaussians_backward(gvc_ctx* ctx, int64_t P, const float* means3D, const float* scales,
                                     const float* rotations, const float* conics, const float* values,
                                     const float* weights, const float* out_cells, const float* out_weights,
                                     float scale_modifier, const float* bounds, float bg, const float* dL_dout_cells,
                                     const float* dL_dout_weights, int use_gaussian_bvh, int debug, float* dmeans,
                                     float* dscales, float* drots, float* dvalues, float* dweights, void* stream);

/* Value dtypes of the structured sampler (gpu_sampling/sample_mesh.cu:76-115). */
typedef enum { GVC_F64 = 0, GVC_F32 = 1, GVC_U16 = 2, GVC_U8 = 3 } gvc_dtype;

/* Replaces sample_mesh (gpu_sampling/sample_mesh.cu:26-240): uniform point field of
   dims nx*ny*nz (x fastest), trilinear interpolation, invalid = -1 cast to the dtype.
   dims/origin/spacing are HOST arrays; values/samples/out are device pointers. */
int gvc_sample_uniform(gvc_ctx* ctx, const int64_t* dims, const float* origin, const float* spacing,
                       const void* values, int dtype, int64_t N, const float* samples, void* out, void* stream);

/* Replaces the tetrahedral case of sample_meshu (gpu_sampling/sample_mesh.cu:242-414,
   VTK_TETRA = 10).  conn4: [C,4] int32 vertex ids; values: [npts] float64.
   out: [N] float64 (value or -1); cell_ids: [N] int64 (lowest containing tet or -1),
   may be NULL. */
int gvc_sample_tets(gvc_ctx* ctx, int64_t npts, const float* pts, int64_t C, const int32_t* conn4,
                    const double* values, int64_t N, const float* samples, double* out, int64_t* cell_ids,
                    void* stream);

/* Replaces sample_meshu for mixed explicit meshes (gpu_sampling/sample_mesh.cu:242-414,
   cell types mapped at :300-336).  cell_types [C] uint8 VTK ids: 10 tetra, 12 hexahedron,
   13 wedge, 14 pyramid are located (isoparametric, Newton inversion in double); 1 vertex,
   3 line, 5 triangle, 9 quad have no volume and never contain a probe point.
   cell_offsets [C] int64: first connectivity entry of each cell; conn int32 vertex ids;
   values [npts] float64.  out [N] float64 (value or -1), cell_ids [N] int64 (lowest
   containing cell or -1, may be NULL).  All device pointers. */
int gvc_sample_cells(gvc_ctx* ctx, int64_t npts, const float* pts, int64_t C, const uint8_t* cell_types,
                     const int64_t* cell_offsets, const int32_t* conn, const double* values, int64_t N,
                     const float* samples, double* out, int64_t* cell_ids, void* stream);

/* Mean squared distance to the three nearest other points, one value per point: the
   initial Gaussian scale rule, replacing simple-knn's distCUDA2 (a third-party
   extension outside the reference tree, called at scene/gaussian_model.py:175-179 and
   :729-733).  pts [n][3] float32, out [n] float32, both device pointers.  Exact: the
   three smallest float32 squared distances ((dx*dx + dy*dy) + dz*dz, each operation
   rounded) to any other index, summed in ascending order and divided by 3 in float32;
   when fewer than three other points exist the missing ones count as FLT_MAX (so n <= 2
   gives +inf).  A traversal overflow (impossible for the LBVH's depth) is reported by
   gvc_sync_status. */
int gvc_knn3_mean_dist2(gvc_ctx* ctx, int64_t n, const float* pts, float* out, void* stream);

/* Training sample batches generated on the device, replacing train.py:34-61
   (sample_mesh_points: random tetrahedron uniform over cells, sorted-uniform barycentric
   weights), :273-282 (ground truth through gpu_sampleu) and :286-315 (per-batch 21-bit
   Morton sort, clamped to [0,1]).  Mesh: pts [npts][3] float32, conn4 [C][4] int32 vertex
   ids in [0, npts), values [npts] float64, all device pointers.  Output: samples_out
   [num_batches][batch_size][3] float32, each batch sorted stably by its 63-bit Morton
   code, and gt_out [num_batches][batch_size] float32, the point field interpolated at each
   sample by the tetrahedral locator (lowest containing cell, -1 outside), or NULL to skip
   it.  Random numbers: Philox4x32-10 keyed by `seed`, so the same seed gives the same
   batches on every device.  num_batches * batch_size must stay below 2^31 - 4096.  The
   workspace (about 48 bytes per sample) stays with the context until gvc_ctx_destroy. */
int gvc_training_samples(gvc_ctx* ctx, int64_t npts, const float* pts, int64_t C, const int32_t* conn4,
                         const double* values, int64_t num_batches, int64_t batch_size, uint64_t seed,
                         float* samples_out, float* gt_out, void* stream);

/* No counterpart in the reference.  Tetrahedral sampling for callers that cannot
   allocate device memory (their memory belongs to another allocator, or cudaMalloc's
   device-wide synchronisation is unacceptable where they call).  Same inputs, outputs
   and results as gvc_sample_tets, but no context and no allocation: the scratch is one
   static device array of about 6.4 MB in every device that loads the library, which
   limits the mesh to C <= 32768 cells (larger meshes are rejected with
   GVC_ERR_CAPACITY and a message in errbuf).  The first call on a device looks up the
   array's device address; under CUDA's default lazy module loading that is also when
   the driver loads the library's device code there and reserves the array, so that
   first call reserves device memory once.  A call with N = 0 does only this set-up:
   make it at start-up (or run with CUDA_MODULE_LOADING=EAGER), and before any stream
   capture on that device.  Later calls allocate nothing.  Calls share the array: calls
   that overlap on the GPU race, so issue them one after another.  Samples are traversed
   in the caller's order; the call returns after `stream` has finished its work (it
   reads the traversal status back).  errbuf (host, may be NULL) receives a message. */
int gvc_sample_tets_static(int64_t npts, const float* pts, int64_t C, const int32_t* conn4, const double* values,
                           int64_t N, const float* samples, double* out, int64_t* cell_ids, void* stream,
                           char* errbuf, int64_t errbuf_len);

/* Test hook: builds the LBVH over n boxes [n,6] (lo xyz, hi xyz) exactly as the
   forward does over Gaussian AABBs, and copies the result out (device pointers):
   keys_sorted [n] uint32, perm [n] int32, left/right [n-1] int32 (leaf i encoded as
   i | 0x80000000), node_boxes [(n-1),6]. No counterpart in the reference (its
   builder is cuBQL::cuda::radixBuilder, rasterizer_impl.cu:82). */
int gvc_debug_lbvh(gvc_ctx* ctx, int64_t n, const float* boxes, uint32_t* keys_sorted, int32_t* perm,
                   int32_t* left, int32_t* right, float* node_boxes, void* stream);

/* Test hook: the escape edges of the stackless traversal in the tree of the last
   gvc_debug_lbvh call: escape [max(n-1, 1)] int32 (device), per internal node the edge
   2p + s (child s of node p) that follows its subtree in pre-order, -1 for none.  No
   counterpart in the reference. */
int gvc_debug_lbvh_escape(gvc_ctx* ctx, int32_t* escape, void* stream);

/* Test hook: the forward's preprocess (FORWARD::preprocess, forward.cu:10-114) alone:
   conics [6P] and AABBs [P,6] in the caller's order. */
int gvc_debug_preprocess(gvc_ctx* ctx, int64_t P, const float* means3D, const float* scales, const float* rotations,
                         const float* weights, float scale_modifier, float* conics, float* aabbs, void* stream);

/* Test hook: D[128 x N] = A[128 x 16] * B[N x 16]^T with BF16 inputs and FP32 output on
   the tensor cores (tcgen05.mma, one CTA); N a multiple of 32 in [32, 256]; row-major
   device arrays.  No counterpart in the reference. */
int gvc_debug_tc_gemm(gvc_ctx* ctx, const void* A, const void* B, int N, float* D, void* stream);

/* Test hook: one block waits on a pipeline barrier (mbarrier) that nothing completes,
   with the same bounded wait as the evaluation kernels (about 0.1 s), records the
   timeout in the device status word and returns; the next gvc_sync_status reports
   GVC_ERR_TIMEOUT.  No counterpart in the reference. */
int gvc_debug_wait_timeout(gvc_ctx* ctx, void* stream);

/* Test hook: the sample ordering of the last gvc_build_bvh: perm [S] int32 (sorted
   position -> caller index) and keys [S] uint32. */
int gvc_debug_sample_order(gvc_ctx* ctx, int32_t* perm, uint32_t* keys, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* GVC_H_INCLUDED */
