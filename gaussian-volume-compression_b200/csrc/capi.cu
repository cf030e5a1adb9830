// capi.cu -- extern "C" entry points of libgvc.so (declared in include/gvc.h).
//
// Host orchestration of the path that diff-gaussian-rasterization/ext.cu,
// rasterize_points.cu and cuda_rasterizer/rasterizer_impl.cu implement in the
// reference: stream-ordered, no per-call cudaMalloc once the context's buffers have
// grown to the working sizes, no device synchronisation unless debug is set (the
// reference synchronises every call through cudaMalloc/cudaFree and a D2H copy,
// rasterizer_impl.cu:121-169).
#include <atomic>
#include <cstdio>
#include <cstring>
#include <new>

#include "lbvh.cuh"
#include "render.cuh"

using namespace gvc;

static std::atomic<long long> g_launches{0};
void gvc::note_launch(int n) { g_launches.fetch_add(n, std::memory_order_relaxed); }

namespace {

struct Scratch {
    DevBuf gacc;       // [P][16] per-Gaussian gradient accumulators
    DevBuf tmp_boxes;  // debug hooks / tet boxes
    DevBuf tmp_out;
    Lbvh dbg;          // debug LBVH
    Lbvh msamp;        // Morton order of mesh sample points
};

Scratch* scratch_of(gvc_ctx* c);

int fail(gvc_ctx* c, int code, const char* msg) {
    if (c) c->err = msg;
    return code;
}

int cuda_fail(gvc_ctx* c, cudaError_t e, const char* where) {
    if (c) {
        c->err = std::string(where) + ": " + cudaGetErrorString(e);
    }
    return GVC_ERR_CUDA;
}

#define GVC_CUDA(call, where)                                   \
    do {                                                        \
        cudaError_t e_ = (call);                                \
        if (e_ != cudaSuccess) return cuda_fail(ctx, e_, where); \
    } while (0)

__global__ void k_boxes6_to_f4(int64_t n, const float* __restrict__ b6, float4* __restrict__ out) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    out[2 * i] = make_float4(b6[6 * i], b6[6 * i + 1], b6[6 * i + 2], 0.f);
    out[2 * i + 1] = make_float4(b6[6 * i + 3], b6[6 * i + 4], b6[6 * i + 5], 0.f);
}

// escape edges of the stackless traversal (BvhNode c.w)
__global__ void k_node_escape(int64_t n, const BvhNode* __restrict__ nodes, int32_t* __restrict__ out) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    out[i] = __float_as_int(nodes[i].c.w);
}

__global__ void k_f4_to_boxes6(int64_t n, const float4* __restrict__ in, float* __restrict__ b6) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    float4 lo = in[2 * i], hi = in[2 * i + 1];
    b6[6 * i] = lo.x;
    b6[6 * i + 1] = lo.y;
    b6[6 * i + 2] = lo.z;
    b6[6 * i + 3] = hi.x;
    b6[6 * i + 4] = hi.y;
    b6[6 * i + 5] = hi.z;
}

inline unsigned nb(int64_t n, int t) { return (unsigned)((n + t - 1) / t); }

// Largest element count handled with 32-bit indices inside the kernels.
constexpr int64_t kMaxElems = (int64_t(1) << 31) - 4096;

struct DebugTimer {
    bool on;
    cudaStream_t st;
    cudaEvent_t ev[8];
    int n = 0;
    DebugTimer(bool on_, cudaStream_t s) : on(on_), st(s) {
        if (on)
            for (auto& e : ev) cudaEventCreate(&e);
    }
    void mark() {
        if (on && n < 8) cudaEventRecord(ev[n++], st);
    }
    float ms(int a, int b) {
        float t = 0.f;
        if (on && b < n) cudaEventElapsedTime(&t, ev[a], ev[b]);
        return t;
    }
    ~DebugTimer() {
        if (on)
            for (auto& e : ev) cudaEventDestroy(e);
    }
};

// Kernel timing: events recorded around the evaluation kernels on the caller's stream;
// read out (after a synchronisation) by gvc_get_stats or when the pool is full.
void drain_events(gvc_ctx* ctx) {
    for (int i = 0; i < ctx->ev_pending; i++) {
        cudaEventSynchronize(ctx->ev_pool[2 * i + 1]);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, ctx->ev_pool[2 * i], ctx->ev_pool[2 * i + 1]);
        if (ctx->ev_kind[i] == 0) {
            ctx->fwd_kernel_ms += ms;
            ctx->fwd_kernel_calls++;
        } else {
            ctx->bwd_kernel_ms += ms;
            ctx->bwd_kernel_calls++;
        }
    }
    ctx->ev_pending = 0;
}

int timer_begin(gvc_ctx* ctx, cudaStream_t st, int kind) {
    if (!ctx->time_kernels) return -1;
    if (!ctx->ev_init) {
        for (auto& e : ctx->ev_pool) cudaEventCreate(&e);
        ctx->ev_init = true;
    }
    if (ctx->ev_pending == 32) drain_events(ctx);
    int i = ctx->ev_pending++;
    ctx->ev_kind[i] = kind;
    cudaEventRecord(ctx->ev_pool[2 * i], st);
    return i;
}

void timer_end(gvc_ctx* ctx, cudaStream_t st, int i) {
    if (i >= 0) cudaEventRecord(ctx->ev_pool[2 * i + 1], st);
}

int debug_check(gvc_ctx* ctx, cudaStream_t st) {
    cudaError_t e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "debug synchronize");
    e = cudaMemcpy(ctx->h_status, ctx->d_status, sizeof(int), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "status copy");
    const int s = *ctx->h_status;
    if (s == 0) return GVC_OK;
    e = cudaMemset(ctx->d_status, 0, sizeof(int));
    if (e != cudaSuccess) return cuda_fail(ctx, e, "status clear");
    if (s & kStatusStackOverflow)
        return fail(ctx, GVC_ERR_TRAVERSAL, "BVH traversal stack overflow: results are invalid");
    return fail(ctx, GVC_ERR_TIMEOUT,
                "a bounded device-side wait ran out (pipeline barrier or radix-sort look-back): results are invalid");
}

}  // namespace

struct gvc_ctx_full : gvc_ctx {
    Scratch scratch;
};

namespace {
Scratch* scratch_of(gvc_ctx* c) { return &static_cast<gvc_ctx_full*>(c)->scratch; }
}  // namespace

extern "C" {

int64_t gvc_launch_count(void) { return (int64_t)g_launches.load(std::memory_order_relaxed); }

int gvc_ctx_create(gvc_ctx** out) {
    if (!out) return GVC_ERR_ARG;
    *out = nullptr;
    gvc_ctx_full* c = new (std::nothrow) gvc_ctx_full();
    if (!c) return GVC_ERR_CAPACITY;
    gvc_ctx* ctx = c;
    GVC_CUDA(cudaGetDevice(&c->device), "cudaGetDevice");
    GVC_CUDA(cudaMalloc(&c->d_status, sizeof(int)), "cudaMalloc status");
    GVC_CUDA(cudaMemset(c->d_status, 0, sizeof(int)), "cudaMemset status");
    GVC_CUDA(cudaMalloc(&c->d_stats, sizeof(unsigned long long) * 16), "cudaMalloc stats");
    GVC_CUDA(cudaMemset(c->d_stats, 0, sizeof(unsigned long long) * 16), "cudaMemset stats");
    GVC_CUDA(cudaMallocHost(&c->h_status, sizeof(int)), "cudaMallocHost");
    Lbvh* sorted[] = {&c->s_sort, &c->tiles, &c->gbvh, &c->cells, &c->knn, &c->ts_sort, &c->scratch.dbg,
                      &c->scratch.msamp};
    for (Lbvh* L : sorted) L->status = c->d_status;
    *out = c;
    return GVC_OK;
}

void gvc_ctx_destroy(gvc_ctx* ctx) {
    if (!ctx) return;
    gvc_ctx_full* c = static_cast<gvc_ctx_full*>(ctx);
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(c->device);
    Lbvh* lbvhs[] = {&c->s_sort,  &c->tiles,      &c->gbvh,          &c->cells,
                     &c->knn,     &c->ts_sort,    &c->scratch.dbg,   &c->scratch.msamp};
    for (Lbvh* L : lbvhs) {
        DevBuf* bufs[] = {&L->keys, &L->keys_alt, &L->perm, &L->perm_alt, &L->boxes, &L->sorted_boxes, &L->left,
                          &L->right, &L->parent, &L->flags, &L->node_boxes, &L->nodes, &L->hist, &L->bounds,
                          &L->onesweep};
        for (DevBuf* b : bufs) b->release();
    }
    DevBuf* bufs[] = {&c->s_sorted, &c->fwd_sorted, &c->tile_boxes, &c->tile_keys, &c->tile_gdesc, &c->blk_desc, &c->blk_boxes, &c->blk_desc_b, &c->blk_boxes_b, &c->s_grad, &c->s_gyz, &c->s_ok, &c->grec, &c->gtmp,
                      &c->m_out_sorted, &c->knn_boxes, &c->ts_points, &c->ts_words, &c->ts_gt64, &c->scratch.gacc, &c->scratch.tmp_boxes, &c->scratch.tmp_out,
                      &c->clog, &c->cend};
    for (DevBuf* b : bufs) b->release();
    if (c->d_status) cudaFree(c->d_status);
    if (c->d_stats) cudaFree(c->d_stats);
    if (c->h_status) cudaFreeHost(c->h_status);
    if (c->ev_init)
        for (auto& e : c->ev_pool) cudaEventDestroy(e);
    cudaSetDevice(prev);
    delete c;
}

const char* gvc_last_error(const gvc_ctx* ctx) { return ctx ? ctx->err.c_str() : "null context"; }

int gvc_set_option(gvc_ctx* ctx, int option, int value) {
    if (!ctx) return GVC_ERR_ARG;
    switch (option) {
        case GVC_OPT_COV_GRAD:
            if (value < 0 || value > 1) return fail(ctx, GVC_ERR_ARG, "cov_grad must be 0 or 1");
            ctx->cov_grad_mode = value;
            return GVC_OK;
        case GVC_OPT_BWD_MODE:
            if (value < 0 || value > 3) return fail(ctx, GVC_ERR_ARG, "bwd_mode must be 0, 1, 2 or 3");
            ctx->bwd_mode = value;
            return GVC_OK;
        case GVC_OPT_EVAL_PATH:
            if (value < 0 || value > 2) return fail(ctx, GVC_ERR_ARG, "eval path must be 0, 1 or 2");
            ctx->eval_path = value;
            return GVC_OK;
        case GVC_OPT_COUNT_PAIRS:
            ctx->count_pairs = value ? 1 : 0;
            return GVC_OK;
        case GVC_OPT_CAND_LOG:
            ctx->cand_log = value ? 1 : 0;
            return GVC_OK;
        case GVC_OPT_TRAVERSAL:
            if (value < 0 || value > 1) return fail(ctx, GVC_ERR_ARG, "traversal must be 0 or 1");
            ctx->traversal = value;
            return GVC_OK;
        case GVC_OPT_TIME_KERNELS:
            drain_events(ctx);
            ctx->time_kernels = value ? 1 : 0;
            ctx->fwd_kernel_ms = ctx->bwd_kernel_ms = 0.0;
            ctx->fwd_kernel_calls = ctx->bwd_kernel_calls = 0;
            return GVC_OK;
        default:
            return fail(ctx, GVC_ERR_ARG, "unknown option");
    }
}

int gvc_get_stats(gvc_ctx* ctx, gvc_stats* out, void* stream) {
    if (!ctx || !out) return GVC_ERR_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    unsigned long long h[16];
    GVC_CUDA(cudaStreamSynchronize(st), "cudaStreamSynchronize");
    GVC_CUDA(cudaMemcpy(h, ctx->d_stats, sizeof(h), cudaMemcpyDeviceToHost), "stats copy");
    out->fwd_candidates = (int64_t)h[0];
    out->fwd_contributing = (int64_t)h[1];
    out->bwd_contributing = (int64_t)h[2];
    out->max_stack_fwd = (int32_t)h[3];
    out->max_stack_bwd = (int32_t)h[4];
    out->fwd_leaf_hits = (int64_t)h[5];
    out->fwd_node_visits = (int64_t)h[6];
    out->bwd_leaf_hits = (int64_t)h[7];
    out->bwd_node_visits = (int64_t)h[8];
    out->fwd_lane_evals = (int64_t)h[9];
    out->bwd_rows = (int64_t)h[10];
    drain_events(ctx);
    out->fwd_kernel_ms = ctx->fwd_kernel_ms;
    out->bwd_kernel_ms = ctx->bwd_kernel_ms;
    out->fwd_kernel_calls = ctx->fwd_kernel_calls;
    out->bwd_kernel_calls = ctx->bwd_kernel_calls;
    return GVC_OK;
}

int gvc_sync_status(gvc_ctx* ctx, void* stream) {
    if (!ctx) return GVC_ERR_ARG;
    return debug_check(ctx, (cudaStream_t)stream);
}

// Lane groups of the 32-sample tiles (forward per tile, sample-side backward kernels).
static int ensure_tile_groups(gvc_ctx* ctx, cudaStream_t st) {
    if (ctx->tile_groups_ready || ctx->n_tiles == 0) return GVC_OK;
    const int64_t slots_g = ctx->n_tiles * kGroups;
    GVC_CUDA(ctx->tile_boxes.ensure(sizeof(float4) * 2 * slots_g), "alloc tile_boxes");
    GVC_CUDA(ctx->tile_keys.ensure(sizeof(uint32_t) * slots_g), "alloc tile_keys");
    GVC_CUDA(ctx->tile_gdesc.ensure(sizeof(uint32_t) * ctx->n_tiles), "alloc tile_gdesc");
    // reads the context's own sorted samples (the caller's array may be gone by now)
    GVC_CUDA(launch_sample_tiles(ctx->S, ctx->n_tiles, nullptr, nullptr, ctx->s_sort.keys.as<uint32_t>(),
                                 ctx->s_sorted.as<float4>(),
                                 ctx->tile_boxes.as<float4>(), ctx->tile_keys.as<uint32_t>(),
                                 ctx->tile_gdesc.as<uint32_t>(), true, st),
             "sample tile groups");
    ctx->tile_groups_ready = true;
    return GVC_OK;
}

// The LBVH over the tile lane groups (the deterministic Gaussian-owned backward).
static int ensure_tile_lbvh(gvc_ctx* ctx, cudaStream_t st) {
    if (ctx->tiles_ready || ctx->n_tiles == 0) return GVC_OK;
    const int rc = ensure_tile_groups(ctx, st);
    if (rc != GVC_OK) return rc;
    GVC_CUDA(lbvh_hierarchy(ctx->tiles, ctx->n_tiles * kGroups, ctx->tile_keys.as<uint32_t>(),
                            ctx->tile_boxes.as<float4>(), st),
             "sample-group LBVH");
    ctx->tiles_ready = true;
    return GVC_OK;
}

int gvc_build_bvh(gvc_ctx* ctx, const float* samples, int64_t S, int debug, int use_gaussian_bvh, void* stream) {
    (void)use_gaussian_bvh;  // both reference modes use the same sample ordering here
    if (!ctx) return GVC_ERR_ARG;
    if (S < 0 || S > kMaxElems) return fail(ctx, GVC_ERR_CAPACITY, "number of samples out of range");
    if (S > 0 && !samples) return fail(ctx, GVC_ERR_ARG, "samples is null");
    cudaStream_t st = (cudaStream_t)stream;
    DebugTimer tm(debug != 0, st);
    tm.mark();
    ctx->samples = samples;
    ctx->S = S;
    ctx->n_tiles = (S + kTile - 1) / kTile;
    ctx->samples_ready = false;
    ctx->blk_b_ready = false;
    ctx->clog_ready = false;
    ctx->fwd_sorted_ready = false;
    ctx->tiles_ready = false;        // the sample-group LBVH is built by its first user
    ctx->tile_groups_ready = false;  // so are the lane groups of the 32-sample tiles
    if (S > 0) {
        GVC_CUDA(morton_sort_points(ctx->s_sort, S, samples, st), "sample sort");
        const int64_t slots = ctx->n_tiles * kTile;
        GVC_CUDA(ctx->s_sorted.ensure(sizeof(float4) * slots), "alloc s_sorted");
        // sorted samples only; the 32-sample lane groups and their LBVH are built by their
        // first user (ensure_tile_groups / ensure_tile_lbvh)
        GVC_CUDA(launch_sample_tiles(S, ctx->n_tiles, samples, ctx->s_sort.perm.as<int32_t>(),
                                     ctx->s_sort.keys.as<uint32_t>(), ctx->s_sorted.as<float4>(), nullptr, nullptr,
                                     nullptr, false, st),
                 "sample tiles");
        const int64_t n_blocks = (S + 127) / 128;
        GVC_CUDA(ctx->blk_desc.ensure(sizeof(uint2) * n_blocks), "alloc blk_desc");
        GVC_CUDA(ctx->blk_boxes.ensure(sizeof(float4) * 2 * 8 * n_blocks), "alloc blk_boxes");
        // when the options already select the tensor-core backward, its finer block groups
        // come from the same launch; otherwise that backward builds them on first use
        const bool tc_bwd = ctx->bwd_mode == 3 || (ctx->bwd_mode == 0 && ctx->eval_path == 1);
        if (tc_bwd) {
            GVC_CUDA(ctx->blk_desc_b.ensure(sizeof(uint2) * n_blocks), "alloc blk_desc_b");
            GVC_CUDA(ctx->blk_boxes_b.ensure(sizeof(float4) * 2 * 8 * n_blocks), "alloc blk_boxes_b");
        }
        GVC_CUDA(launch_sample_blocks(S, ctx->s_sorted.as<float4>(), ctx->s_sort.keys.as<uint32_t>(),
                                      ctx->blk_desc.as<uint2>(), ctx->blk_boxes.as<float4>(), kBlockSplitForward, st,
                                      tc_bwd ? ctx->blk_desc_b.as<uint2>() : nullptr,
                                      tc_bwd ? ctx->blk_boxes_b.as<float4>() : nullptr, kBlockSplitBackward),
                 "sample blocks");
        ctx->blk_b_ready = tc_bwd;
    }
    ctx->samples_ready = true;
    tm.mark();
    if (debug) {
        int rc = debug_check(ctx, st);
        printf("Sample BVH time: %g ms\n", tm.ms(0, 1));
        if (rc) return rc;
    }
    return GVC_OK;
}

int gvc_rasterize_gaussians(gvc_ctx* ctx, int64_t P, const float* means3D, const float* scales,
                            const float* rotations, const float* values, const float* weights, float scale_modifier,
                            const float* bounds, float bg, int use_gaussian_bvh, int debug, float* out_cells,
                            float* out_weights, float* conics, void* stream) {
    (void)bounds;
    (void)bg;
    (void)use_gaussian_bvh;
    if (!ctx) return GVC_ERR_ARG;
    if (!ctx->samples_ready) return fail(ctx, GVC_ERR_STATE, "build_bvh must be called before rasterize_gaussians");
    if (P < 0 || P > kMaxElems) return fail(ctx, GVC_ERR_CAPACITY, "number of Gaussians out of range");
    const int64_t S = ctx->S;
    if (S > 0 && (!out_cells || !out_weights)) return fail(ctx, GVC_ERR_ARG, "null output");
    cudaStream_t st = (cudaStream_t)stream;
    if (P == 0) {  // rasterize_points.cu:51: outputs stay zero
        GVC_CUDA(launch_fill_zero_outputs(S, out_cells, out_weights, st), "zero outputs");
        ctx->gauss_ready = false;
        ctx->clog_ready = false;
        ctx->fwd_sorted_ready = false;
        ctx->fwd_recs_ready = false;
        return GVC_OK;
    }
    if (!means3D || !scales || !rotations || !values || !weights || !conics)
        return fail(ctx, GVC_ERR_ARG, "null Gaussian parameter pointer");
    // this call rewrites the AABBs, records and sorted outputs: valid again only once it ends
    ctx->fwd_recs_ready = false;
    ctx->fwd_sorted_ready = false;
    DebugTimer tm(debug != 0, st);
    if (ctx->count_pairs) GVC_CUDA(cudaMemsetAsync(ctx->d_stats, 0, sizeof(unsigned long long) * 16, st), "stats");
    tm.mark();
    GVC_CUDA(ctx->gtmp.ensure(sizeof(float4) * 2 * P), "alloc boxes");
    float4* boxes = ctx->gtmp.as<float4>();
    GVC_CUDA(launch_preprocess(P, means3D, scales, rotations, weights, scale_modifier, conics, boxes, st),
             "preprocess");
    tm.mark();
    GVC_CUDA(lbvh_build_boxes(ctx->gbvh, P, boxes, st), "Gaussian LBVH");
    GVC_CUDA(ctx->grec.ensure(sizeof(GaussRec) * P), "alloc records");
    GVC_CUDA(launch_gather_recs(P, ctx->gbvh.perm.as<int32_t>(), means3D, values, weights, conics, boxes,
                                ctx->grec.as<GaussRec>(), st),
             "gather records");
    tm.mark();
    if (ctx->eval_path == 2) {
        const int rc = ensure_tile_groups(ctx, st);
        if (rc != GVC_OK) return rc;
    }
    FwdArgs fa{};
    fa.s_sorted = ctx->s_sorted.as<float4>();
    fa.tile_boxes = ctx->tile_boxes.as<float4>();
    fa.gdesc = ctx->tile_gdesc.as<uint32_t>();
    fa.n_tiles = ctx->n_tiles;
    fa.gnodes = ctx->gbvh.nodes.as<BvhNode>();
    fa.recs = ctx->grec.as<GaussRec>();
    fa.out_cells = out_cells;
    fa.out_weights = out_weights;
    fa.status = ctx->d_status;
    fa.stats = ctx->d_stats;
    fa.count = ctx->count_pairs != 0;
    const int tk = timer_begin(ctx, st, 0);
    if (ctx->eval_path == 2) {
        GVC_CUDA(launch_forward(fa, st), "forward");
    } else {
        CtaArgs ca{};
        ca.s_sorted = ctx->s_sorted.as<float4>();
        ca.S = ctx->S;
        ca.bdesc = ctx->blk_desc.as<uint2>();
        ca.bboxes = ctx->blk_boxes.as<float4>();
        ca.gnodes = ctx->gbvh.nodes.as<BvhNode>();
        ca.n_internal = ctx->gbvh.n > 1 ? ctx->gbvh.n - 1 : 1;
        ca.stackless = ctx->traversal == 1;
        ca.recs = ctx->grec.as<GaussRec>();
        ca.out_cells = out_cells;
        ca.out_weights = out_weights;
        ca.status = ctx->d_status;
        ca.stats = ctx->d_stats;
        ca.count = ctx->count_pairs != 0;
        // the candidates are logged for the tensor-core backward when it is the one selected
        const bool tc_bwd = ctx->bwd_mode == 3 || (ctx->bwd_mode == 0 && ctx->eval_path == 1);
        if (tc_bwd && ctx->cand_log && ctx->S > 0) {
            // 16 KB per 128 samples: where that does not fit in device memory, the forward
            // runs without the log and the backward walks the tree
            const int64_t n_blocks = (ctx->S + 127) / 128;
            if (ctx->clog.ensure(sizeof(int32_t) * kCandLogPerBlock * n_blocks) == cudaSuccess &&
                ctx->cend.ensure(sizeof(int32_t) * 8 * n_blocks) == cudaSuccess) {
                ca.clog = ctx->clog.as<int32_t>();
                ca.cend = ctx->cend.as<int32_t>();
            } else {
                (void)cudaGetLastError();  // a failed allocation is not sticky: clear it
                ctx->clog.release();
                ctx->cend.release();
            }
        }
        // the FP32 forward also stores (out, W) in sorted order for the backward's sample records
        if (ctx->eval_path == 0 && ctx->S > 0) {
            if (ctx->fwd_sorted.ensure(sizeof(float2) * ctx->n_tiles * kTile) == cudaSuccess) {
                ca.out_sorted = ctx->fwd_sorted.as<float2>();
            } else {
                (void)cudaGetLastError();
                ctx->fwd_sorted.release();
            }
        }
        GVC_CUDA(launch_forward_cta(ca, ctx->eval_path == 1, st), "forward (CTA)");
        ctx->clog_ready = ca.clog != nullptr;
        ctx->fwd_sorted_ready = ca.out_sorted != nullptr;
        ctx->fwd_out_cells = out_cells;
        ctx->fwd_out_weights = out_weights;
    }
    if (ctx->eval_path == 2) {
        ctx->clog_ready = false;
        ctx->fwd_sorted_ready = false;
    }
    timer_end(ctx, st, tk);
    tm.mark();
    ctx->P = P;
    ctx->gauss_ready = true;
    ctx->fwd_means = means3D;
    ctx->fwd_scales = scales;
    ctx->fwd_rots = rotations;
    ctx->fwd_values = values;
    ctx->fwd_weights = weights;
    ctx->fwd_conics = conics;
    ctx->fwd_scale_mod = scale_modifier;
    ctx->fwd_recs_ready = true;
    if (debug) {
        int rc = debug_check(ctx, st);
        printf("Preprocess time: %g ms\nBVH time: %g ms\nRender time: %g ms\n", tm.ms(0, 1), tm.ms(1, 2),
               tm.ms(2, 3));
        if (rc) return rc;
    }
    return GVC_OK;
}

int gvc_rasterize_gaussians_backward(gvc_ctx* ctx, int64_t P, const float* means3D, const float* scales,
                                     const float* rotations, const float* conics, const float* values,
                                     const float* weights, const float* out_cells, const float* out_weights,
                                     float scale_modifier, const float* bounds, float bg, const float* dL_dout_cells,
                                     const float* dL_dout_weights, int use_gaussian_bvh, int debug, float* dmeans,
                                     float* dscales, float* drots, float* dvalues, float* dweights, void* stream) {
    (void)bounds;
    (void)bg;
    if (!ctx) return GVC_ERR_ARG;
    if (!ctx->samples_ready)
        return fail(ctx, GVC_ERR_STATE, "build_bvh must be called before rasterize_gaussians_backward");
    if (P < 0 || P > kMaxElems) return fail(ctx, GVC_ERR_CAPACITY, "number of Gaussians out of range");
    if (P == 0) return GVC_OK;
    if (!means3D || !scales || !rotations || !conics || !values || !weights || !dmeans || !dscales || !drots ||
        !dvalues || !dweights)
        return fail(ctx, GVC_ERR_ARG, "null pointer");
    const int64_t S = ctx->S;
    if (S > 0 && (!out_cells || !out_weights || !dL_dout_cells || !dL_dout_weights))
        return fail(ctx, GVC_ERR_ARG, "null sample-side pointer");
    cudaStream_t st = (cudaStream_t)stream;
    Scratch* sc = scratch_of(ctx);
    DebugTimer tm(debug != 0, st);
    tm.mark();
    // Handed the very arrays of the last forward (and its conics), the forward's AABBs and
    // LBVH-ordered records still hold; otherwise both are rebuilt here (and no longer
    // describe that forward).
    const bool same_gauss = ctx->fwd_recs_ready && ctx->gauss_ready && ctx->P == P && means3D == ctx->fwd_means &&
                            scales == ctx->fwd_scales && rotations == ctx->fwd_rots && values == ctx->fwd_values &&
                            weights == ctx->fwd_weights && conics == ctx->fwd_conics &&
                            scale_modifier == ctx->fwd_scale_mod;
    GVC_CUDA(ctx->gtmp.ensure(sizeof(float4) * 2 * P), "alloc boxes");
    float4* boxes = ctx->gtmp.as<float4>();
    if (!same_gauss) {
        ctx->fwd_recs_ready = false;
        GVC_CUDA(launch_preprocess(P, means3D, scales, rotations, weights, scale_modifier, nullptr, boxes, st),
                 "preprocess");
    }
    GVC_CUDA(sc->gacc.ensure(sizeof(float) * 16 * P), "alloc gacc");
    float* gacc = sc->gacc.as<float>();
    // mode 3, or the tensor-core path in auto mode: reduction over samples on tcgen05
    const bool tc_bwd = ctx->bwd_mode == 3 || (ctx->bwd_mode == 0 && ctx->eval_path == 1);
    const bool atomic_mode = ctx->bwd_mode == 2 || (ctx->bwd_mode == 0 && use_gaussian_bvh);
    const bool have_order = ctx->gauss_ready && ctx->P == P;
    if (ctx->n_tiles == 0) {
        GVC_CUDA(cudaMemsetAsync(gacc, 0, sizeof(float) * 16 * P, st), "zero gacc");
    } else {
        const int64_t slots = ctx->n_tiles * kTile;
        GVC_CUDA(ctx->s_grad.ensure(sizeof(float4) * slots), "alloc s_grad");
        GVC_CUDA(ctx->s_gyz.ensure(sizeof(float) * slots), "alloc s_gyz");
        GVC_CUDA(ctx->s_ok.ensure(slots), "alloc s_ok");
        // the forward's sorted copy of (out, W) when these are the arrays it wrote
        const bool same_out = ctx->fwd_sorted_ready && have_order && out_cells == ctx->fwd_out_cells &&
                              out_weights == ctx->fwd_out_weights;
        GVC_CUDA(launch_sample_grads(slots, ctx->s_sorted.as<float4>(),
                                     same_out ? ctx->fwd_sorted.as<float2>() : nullptr, out_cells, out_weights,
                                     dL_dout_cells, dL_dout_weights, ctx->s_grad.as<float4>(), ctx->s_gyz.as<float>(),
                                     ctx->s_ok.as<uint8_t>(), st),
                 "sample grads");
        BwdArgs ba{};
        ba.P = P;
        ba.means = means3D;
        ba.values = values;
        ba.weights = weights;
        ba.conics = conics;
        ba.boxes = boxes;
        ba.s_sorted = ctx->s_sorted.as<float4>();
        ba.s_grad = ctx->s_grad.as<float4>();
        ba.s_gyz = ctx->s_gyz.as<float>();
        ba.s_ok = ctx->s_ok.as<uint8_t>();
        if (!tc_bwd) {
            // the deterministic reduction walks the sample groups; the atomic one uses their boxes
            const int rc = atomic_mode ? ensure_tile_groups(ctx, st) : ensure_tile_lbvh(ctx, st);
            if (rc != GVC_OK) return rc;
        }
        ba.tile_boxes = ctx->tile_boxes.as<float4>();
        ba.gdesc = ctx->tile_gdesc.as<uint32_t>();
        ba.n_tiles = ctx->n_tiles;
        ba.tnodes = ctx->tiles.nodes.as<BvhNode>();
        ba.gacc = gacc;
        ba.status = ctx->d_status;
        ba.stats = ctx->d_stats;
        ba.count = ctx->count_pairs != 0;
        tm.mark();
        if (tc_bwd) {
            if (!have_order) GVC_CUDA(lbvh_build_boxes(ctx->gbvh, P, boxes, st), "Gaussian LBVH");
            if (!same_gauss) {
                GVC_CUDA(ctx->grec.ensure(sizeof(GaussRec) * P), "alloc records");
                GVC_CUDA(launch_gather_recs(P, ctx->gbvh.perm.as<int32_t>(), means3D, values, weights, conics,
                                            boxes, ctx->grec.as<GaussRec>(), st),
                         "gather records");
            }
            GVC_CUDA(cudaMemsetAsync(gacc, 0, sizeof(float) * 16 * P, st), "zero gacc");
            ba.gorder = nullptr;
            ba.gperm = ctx->gbvh.perm.as<int32_t>();
            ba.gnodes = ctx->gbvh.nodes.as<BvhNode>();
            ba.g_internal = ctx->gbvh.n > 1 ? ctx->gbvh.n - 1 : 1;
            ba.stackless = ctx->traversal == 1;
            ba.recs = ctx->grec.as<GaussRec>();
            const int tk = timer_begin(ctx, st, 1);
            const int64_t n_blocks = (S + 127) / 128;
            if (!ctx->blk_b_ready) {
                GVC_CUDA(ctx->blk_desc_b.ensure(sizeof(uint2) * n_blocks), "alloc blk_desc_b");
                GVC_CUDA(ctx->blk_boxes_b.ensure(sizeof(float4) * 2 * 8 * n_blocks), "alloc blk_boxes_b");
                GVC_CUDA(launch_sample_blocks(S, ctx->s_sorted.as<float4>(), ctx->s_sort.keys.as<uint32_t>(),
                                              ctx->blk_desc_b.as<uint2>(), ctx->blk_boxes_b.as<float4>(),
                                              kBlockSplitBackward, st),
                         "backward block groups");
                ctx->blk_b_ready = true;
            }
            // the forward's candidate log, when it belongs to these Gaussians and samples,
            // replaces the backward's own walk of the tree
            if (have_order && ctx->clog_ready) {
                ba.clog = ctx->clog.as<int32_t>();
                ba.cend = ctx->cend.as<int32_t>();
                ba.cdesc = ctx->blk_desc.as<uint2>();
            }
            const uint2* bdesc = ctx->blk_desc_b.as<uint2>();
            const float4* bboxes = ctx->blk_boxes_b.as<float4>();
            GVC_CUDA(launch_backward_cta(ba, n_blocks, bdesc, bboxes, st), "backward (tensor core)");
            timer_end(ctx, st, tk);
        } else if (atomic_mode) {
            if (!have_order) GVC_CUDA(lbvh_build_boxes(ctx->gbvh, P, boxes, st), "Gaussian LBVH");
            if (!same_gauss) {
                GVC_CUDA(ctx->grec.ensure(sizeof(GaussRec) * P), "alloc records");
                GVC_CUDA(launch_gather_recs(P, ctx->gbvh.perm.as<int32_t>(), means3D, values, weights, conics,
                                            boxes, ctx->grec.as<GaussRec>(), st),
                         "gather records");
            }
            GVC_CUDA(cudaMemsetAsync(gacc, 0, sizeof(float) * 16 * P, st), "zero gacc");
            ba.gorder = nullptr;
            ba.gperm = ctx->gbvh.perm.as<int32_t>();
            ba.gnodes = ctx->gbvh.nodes.as<BvhNode>();
            ba.recs = ctx->grec.as<GaussRec>();
            const int tk = timer_begin(ctx, st, 1);
            GVC_CUDA(launch_backward_tiles(ba, st), "backward (atomic)");
            timer_end(ctx, st, tk);
        } else {
            ba.gorder = have_order ? ctx->gbvh.perm.as<int32_t>() : nullptr;
            ba.gperm = nullptr;
            ba.gnodes = nullptr;
            ba.recs = nullptr;
            const int tk = timer_begin(ctx, st, 1);
            GVC_CUDA(launch_backward_gauss(ba, st), "backward (deterministic)");
            timer_end(ctx, st, tk);
        }
    }
    tm.mark();
    GVC_CUDA(launch_finalize(P, gacc, scales, rotations, conics, scale_modifier, ctx->cov_grad_mode, dmeans, dscales,
                             drots, dvalues, dweights, st),
             "finalize");
    tm.mark();
    if (debug) {
        int rc = debug_check(ctx, st);
        printf("Backward render time: %g ms\nBackward preprocess time: %g ms\n", tm.ms(1, 2), tm.ms(2, 3));
        if (rc) return rc;
    }
    return GVC_OK;
}

int gvc_sample_uniform(gvc_ctx* ctx, const int64_t* dims, const float* origin, const float* spacing,
                       const void* values, int dtype, int64_t N, const float* samples, void* out, void* stream) {
    if (!ctx) return GVC_ERR_ARG;
    if (!dims || !origin || !spacing) return fail(ctx, GVC_ERR_ARG, "dims/origin/spacing must be host arrays");
    if (dtype < GVC_F64 || dtype > GVC_U8)
        return fail(ctx, GVC_ERR_UNSUPPORTED, "Unsupported values dtype. Expected float64, float32, uint16, or uint8.");
    for (int a = 0; a < 3; a++)
        if (dims[a] < 1) return fail(ctx, GVC_ERR_ARG, "dims must be >= 1");
    if (N < 0) return fail(ctx, GVC_ERR_ARG, "negative sample count");
    if (N > 0 && (!values || !samples || !out)) return fail(ctx, GVC_ERR_ARG, "null pointer");
    GVC_CUDA(launch_sample_uniform(dims, origin, spacing, values, dtype, N, samples, out, (cudaStream_t)stream),
             "sample_uniform");
    return GVC_OK;
}

int gvc_sample_tets(gvc_ctx* ctx, int64_t npts, const float* pts, int64_t C, const int32_t* conn4,
                    const double* values, int64_t N, const float* samples, double* out, int64_t* cell_ids,
                    void* stream) {
    if (!ctx) return GVC_ERR_ARG;
    if (npts < 0 || C < 0 || N < 0) return fail(ctx, GVC_ERR_ARG, "negative size");
    if (C > kMaxElems || N > kMaxElems) return fail(ctx, GVC_ERR_CAPACITY, "mesh or sample count out of range");
    if (N > 0 && (!samples || !out)) return fail(ctx, GVC_ERR_ARG, "null pointer");
    if (C > 0 && (!pts || !conn4 || !values)) return fail(ctx, GVC_ERR_ARG, "null mesh pointer");
    cudaStream_t st = (cudaStream_t)stream;
    Scratch* sc = scratch_of(ctx);
    if (N == 0) return GVC_OK;
    const int32_t* cperm = nullptr;
    const BvhNode* cnodes = nullptr;
    if (C > 0) {
        GVC_CUDA(sc->tmp_boxes.ensure(sizeof(float4) * 2 * C), "alloc cell boxes");
        GVC_CUDA(launch_tet_boxes(C, pts, conn4, sc->tmp_boxes.as<float4>(), st), "tet boxes");
        GVC_CUDA(lbvh_build_boxes(ctx->cells, C, sc->tmp_boxes.as<float4>(), st), "cell LBVH");
        cperm = ctx->cells.perm.as<int32_t>();
        cnodes = ctx->cells.nodes.as<BvhNode>();
    }
    GVC_CUDA(morton_sort_points(sc->msamp, N, samples, st), "sample order");
    GVC_CUDA(launch_sample_tets(N, samples, sc->msamp.perm.as<int32_t>(), pts, conn4, values, cnodes, cperm, C, out,
                                cell_ids, ctx->d_status, st),
             "sample tets");
    return GVC_OK;
}

int gvc_knn3_mean_dist2(gvc_ctx* ctx, int64_t n, const float* pts, float* out, void* stream) {
    if (!ctx) return GVC_ERR_ARG;
    if (n < 0) return fail(ctx, GVC_ERR_ARG, "negative point count");
    if (n > kMaxElems) return fail(ctx, GVC_ERR_CAPACITY, "point count out of range");
    if (n == 0) return GVC_OK;
    if (!pts || !out) return fail(ctx, GVC_ERR_ARG, "null pointer");
    cudaStream_t st = (cudaStream_t)stream;
    GVC_CUDA(ctx->knn_boxes.ensure(sizeof(float4) * 2 * n), "alloc point boxes");
    GVC_CUDA(launch_point_boxes(n, pts, ctx->knn_boxes.as<float4>(), st), "point boxes");
    GVC_CUDA(lbvh_build_boxes(ctx->knn, n, ctx->knn_boxes.as<float4>(), st), "point LBVH");
    GVC_CUDA(launch_knn3(n, ctx->knn.sorted_boxes.as<float4>(), ctx->knn.perm.as<int32_t>(),
                         ctx->knn.nodes.as<BvhNode>(), out, ctx->d_status, st),
             "knn3");
    return GVC_OK;
}

int gvc_training_samples(gvc_ctx* ctx, int64_t npts, const float* pts, int64_t C, const int32_t* conn4,
                         const double* values, int64_t num_batches, int64_t batch_size, uint64_t seed,
                         float* samples_out, float* gt_out, void* stream) {
    if (!ctx) return GVC_ERR_ARG;
    if (npts < 0 || C < 0 || num_batches < 0 || batch_size < 0) return fail(ctx, GVC_ERR_ARG, "negative size");
    if (C == 0 || npts == 0) return fail(ctx, GVC_ERR_ARG, "the mesh has no cells or no points");
    if (num_batches == 0 || batch_size == 0) return GVC_OK;
    if (C > kMaxElems || batch_size > kMaxElems || num_batches > kMaxElems / batch_size)
        return fail(ctx, GVC_ERR_CAPACITY, "num_batches * batch_size out of range");
    if (!pts || !conn4 || !samples_out || (gt_out && !values)) return fail(ctx, GVC_ERR_ARG, "null pointer");
    const int64_t N = num_batches * batch_size;
    cudaStream_t st = (cudaStream_t)stream;
    Scratch* sc = scratch_of(ctx);
    GVC_CUDA(ctx->ts_points.ensure(sizeof(float) * 3 * N), "alloc sample points");
    GVC_CUDA(ctx->ts_words.ensure(sizeof(uint32_t) * 3 * N), "alloc sort keys");
    uint32_t* w = ctx->ts_words.as<uint32_t>();
    GVC_CUDA(launch_tet_points(N, batch_size, seed, pts, conn4, C, ctx->ts_points.as<float>(), w, w + N, w + 2 * N,
                               st),
             "tet points");
    // batch index most significant, then the 63-bit Morton code (high word, low word)
    int batch_bits = 0;
    while (batch_bits < 32 && (uint64_t(1) << batch_bits) < (uint64_t)num_batches) batch_bits++;
    const uint32_t* words[3] = {w, w + N, w + 2 * N};
    const int bits[3] = {32, 31, batch_bits};
    GVC_CUDA(radix_sort_words(ctx->ts_sort, N, words, bits, batch_bits > 0 ? 3 : 2, st), "batch Morton sort");
    GVC_CUDA(launch_gather_points(N, ctx->ts_points.as<float>(), ctx->ts_sort.perm.as<int32_t>(), samples_out, st),
             "gather samples");
    if (!gt_out) return GVC_OK;
    GVC_CUDA(sc->tmp_boxes.ensure(sizeof(float4) * 2 * C), "alloc cell boxes");
    GVC_CUDA(launch_tet_boxes(C, pts, conn4, sc->tmp_boxes.as<float4>(), st), "tet boxes");
    GVC_CUDA(lbvh_build_boxes(ctx->cells, C, sc->tmp_boxes.as<float4>(), st), "cell LBVH");
    GVC_CUDA(ctx->ts_gt64.ensure(sizeof(double) * N), "alloc values");
    // the samples are Morton-sorted per batch already: locate them in that order
    GVC_CUDA(launch_sample_tets(N, samples_out, nullptr, pts, conn4, values, ctx->cells.nodes.as<BvhNode>(),
                                ctx->cells.perm.as<int32_t>(), C, ctx->ts_gt64.as<double>(), nullptr,
                                ctx->d_status, st),
             "sample tets");
    GVC_CUDA(launch_to_f32(N, ctx->ts_gt64.as<double>(), gt_out, st), "values to float32");
    return GVC_OK;
}

int gvc_sample_cells(gvc_ctx* ctx, int64_t npts, const float* pts, int64_t C, const uint8_t* cell_types,
                     const int64_t* cell_offsets, const int32_t* conn, const double* values, int64_t N,
                     const float* samples, double* out, int64_t* cell_ids, void* stream) {
    if (!ctx) return GVC_ERR_ARG;
    if (npts < 0 || C < 0 || N < 0) return fail(ctx, GVC_ERR_ARG, "negative size");
    if (C > kMaxElems || N > kMaxElems) return fail(ctx, GVC_ERR_CAPACITY, "mesh or sample count out of range");
    if (N > 0 && (!samples || !out)) return fail(ctx, GVC_ERR_ARG, "null pointer");
    if (C > 0 && (!pts || !cell_types || !cell_offsets || !conn || !values))
        return fail(ctx, GVC_ERR_ARG, "null mesh pointer");
    cudaStream_t st = (cudaStream_t)stream;
    Scratch* sc = scratch_of(ctx);
    if (N == 0) return GVC_OK;
    const int32_t* cperm = nullptr;
    const BvhNode* cnodes = nullptr;
    if (C > 0) {
        GVC_CUDA(sc->tmp_boxes.ensure(sizeof(float4) * 2 * C), "alloc cell boxes");
        GVC_CUDA(launch_cell_boxes(C, pts, cell_types, cell_offsets, conn, sc->tmp_boxes.as<float4>(), st),
                 "cell boxes");
        GVC_CUDA(lbvh_build_boxes(ctx->cells, C, sc->tmp_boxes.as<float4>(), st), "cell LBVH");
        cperm = ctx->cells.perm.as<int32_t>();
        cnodes = ctx->cells.nodes.as<BvhNode>();
    }
    GVC_CUDA(morton_sort_points(sc->msamp, N, samples, st), "sample order");
    GVC_CUDA(launch_sample_cells(N, samples, sc->msamp.perm.as<int32_t>(), pts, cell_types, cell_offsets, conn,
                                 values, cnodes, cperm, C, out, cell_ids, ctx->d_status, st),
             "sample cells");
    return GVC_OK;
}

int gvc_debug_lbvh(gvc_ctx* ctx, int64_t n, const float* boxes, uint32_t* keys_sorted, int32_t* perm,
                   int32_t* left, int32_t* right, float* node_boxes, void* stream) {
    if (!ctx) return GVC_ERR_ARG;
    if (n <= 0 || n > kMaxElems) return fail(ctx, GVC_ERR_ARG, "n out of range");
    cudaStream_t st = (cudaStream_t)stream;
    Scratch* sc = scratch_of(ctx);
    GVC_CUDA(sc->tmp_boxes.ensure(sizeof(float4) * 2 * n), "alloc");
    k_boxes6_to_f4<<<nb(n, 256), 256, 0, st>>>(n, boxes, sc->tmp_boxes.as<float4>()); gvc::note_launch();
    GVC_CUDA(lbvh_build_boxes(sc->dbg, n, sc->tmp_boxes.as<float4>(), st), "LBVH");
    if (keys_sorted)
        GVC_CUDA(cudaMemcpyAsync(keys_sorted, sc->dbg.keys.ptr, sizeof(uint32_t) * n, cudaMemcpyDeviceToDevice, st),
                 "copy keys");
    if (perm)
        GVC_CUDA(cudaMemcpyAsync(perm, sc->dbg.perm.ptr, sizeof(int32_t) * n, cudaMemcpyDeviceToDevice, st),
                 "copy perm");
    if (n > 1) {
        if (left)
            GVC_CUDA(cudaMemcpyAsync(left, sc->dbg.left.ptr, sizeof(int32_t) * (n - 1), cudaMemcpyDeviceToDevice, st),
                     "copy left");
        if (right)
            GVC_CUDA(
                cudaMemcpyAsync(right, sc->dbg.right.ptr, sizeof(int32_t) * (n - 1), cudaMemcpyDeviceToDevice, st),
                "copy right");
        if (node_boxes) k_f4_to_boxes6<<<nb(n - 1, 256), 256, 0, st>>>(n - 1, sc->dbg.node_boxes.as<float4>(), node_boxes); gvc::note_launch();
    }
    GVC_CUDA(cudaGetLastError(), "debug lbvh");
    return GVC_OK;
}

int gvc_debug_lbvh_escape(gvc_ctx* ctx, int32_t* escape, void* stream) {
    if (!ctx || !escape) return GVC_ERR_ARG;
    Scratch* sc = scratch_of(ctx);
    const int64_t n = sc->dbg.n;
    if (n <= 0) return fail(ctx, GVC_ERR_STATE, "gvc_debug_lbvh has not built a tree");
    const int64_t ni = n > 1 ? n - 1 : 1;
    cudaStream_t st = (cudaStream_t)stream;
    k_node_escape<<<nb(ni, 256), 256, 0, st>>>(ni, sc->dbg.nodes.as<BvhNode>(), escape); gvc::note_launch();
    GVC_CUDA(cudaGetLastError(), "debug lbvh escape");
    return GVC_OK;
}

int gvc_debug_preprocess(gvc_ctx* ctx, int64_t P, const float* means3D, const float* scales, const float* rotations,
                         const float* weights, float scale_modifier, float* conics, float* aabbs, void* stream) {
    if (!ctx) return GVC_ERR_ARG;
    if (P <= 0 || P > kMaxElems) return fail(ctx, GVC_ERR_ARG, "P out of range");
    cudaStream_t st = (cudaStream_t)stream;
    Scratch* sc = scratch_of(ctx);
    GVC_CUDA(sc->tmp_boxes.ensure(sizeof(float4) * 2 * P), "alloc");
    GVC_CUDA(launch_preprocess(P, means3D, scales, rotations, weights, scale_modifier, conics,
                               sc->tmp_boxes.as<float4>(), st),
             "preprocess");
    if (aabbs) k_f4_to_boxes6<<<nb(P, 256), 256, 0, st>>>(P, sc->tmp_boxes.as<float4>(), aabbs); gvc::note_launch();
    GVC_CUDA(cudaGetLastError(), "debug preprocess");
    return GVC_OK;
}

int gvc_debug_tc_gemm(gvc_ctx* ctx, const void* A, const void* B, int N, float* D, void* stream) {
    if (!ctx) return GVC_ERR_ARG;
    if (N < 32 || N > 256 || N % 32) return fail(ctx, GVC_ERR_ARG, "N must be a multiple of 32 in [32, 256]");
    if (!A || !B || !D) return fail(ctx, GVC_ERR_ARG, "null pointer");
    GVC_CUDA(launch_tc_gemm_test(A, B, N, D, ctx->d_status, (cudaStream_t)stream), "tc gemm");
    return GVC_OK;
}

int gvc_debug_wait_timeout(gvc_ctx* ctx, void* stream) {
    if (!ctx) return GVC_ERR_ARG;
    GVC_CUDA(launch_wait_timeout_test(ctx->d_status, (cudaStream_t)stream), "wait timeout");
    return GVC_OK;
}

int gvc_debug_sample_order(gvc_ctx* ctx, int32_t* perm, uint32_t* keys, void* stream) {
    if (!ctx) return GVC_ERR_ARG;
    if (!ctx->samples_ready) return fail(ctx, GVC_ERR_STATE, "no samples");
    cudaStream_t st = (cudaStream_t)stream;
    if (ctx->S == 0) return GVC_OK;
    if (perm)
        GVC_CUDA(cudaMemcpyAsync(perm, ctx->s_sort.perm.ptr, sizeof(int32_t) * ctx->S, cudaMemcpyDeviceToDevice, st),
                 "copy perm");
    if (keys)
        GVC_CUDA(cudaMemcpyAsync(keys, ctx->s_sort.keys.ptr, sizeof(uint32_t) * ctx->S, cudaMemcpyDeviceToDevice, st),
                 "copy keys");
    return GVC_OK;
}

}  // extern "C"
