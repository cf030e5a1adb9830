// cta.cu -- CTA-level forward evaluation in FP32 (SIMT), the 128-sample block groups the
// CTA kernels run on, and a tcgen05 GEMM test hook.  The forward with the exponent on the
// tensor cores is in fwd_tc.cu.
//
// One CTA owns 128 consecutive Morton-sorted samples.  build_bvh splits each such block
// into at most 8 contiguous "block groups" at Z-order jumps (the rule of the 32-sample
// tiles, applied to 128 rows).  For each group the CTA walks the Gaussian LBVH (a
// producer warp, warp-cooperative traversal) and stages candidate Gaussians 32 at a time;
// two consumer warps (two rows per thread) evaluate, for the columns whose box overlaps
// their rows, the exact AABB test, the base-2 power, the window, ex2 and the sums.
#include "cta.cuh"
#include "tc.cuh"
#include "traverse.cuh"

namespace gvc {


constexpr float kHalfLog2eC = -0.72134752044448170368f;
constexpr float kLog2FloorC = -20.197570572173914f;

__device__ __forceinline__ float ex2_apx(float x) {
    float y;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

__device__ __forceinline__ float hp6(const Box6& b) { return (b.hx - b.lx) + (b.hy - b.ly) + (b.hz - b.lz); }

// Order-preserving float <-> uint32 map: a < b as floats iff ord(a) < ord(b) as integers
// (finite values and infinities; -0 orders below +0, which compare equal as floats).
__device__ __forceinline__ uint32_t ford(float f) {
    const uint32_t b = __float_as_uint(f);
    return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
__device__ __forceinline__ float ordf(uint32_t u) {
    return __uint_as_float((u & 0x80000000u) ? (u & 0x7fffffffu) : ~u);
}

// One warp per 128-row block; lane l holds rows 4l .. 4l + 3 (warp reductions only, no
// block barriers).  Box unions are min/max reductions (one redux.sync each on the ordered
// integers), so the result does not depend on the reduction order.
__device__ __forceinline__ Box6 warp_reduce_box(Box6 b) {
    b.lx = ordf(__reduce_min_sync(0xffffffffu, ford(b.lx)));
    b.ly = ordf(__reduce_min_sync(0xffffffffu, ford(b.ly)));
    b.lz = ordf(__reduce_min_sync(0xffffffffu, ford(b.lz)));
    b.hx = ordf(__reduce_max_sync(0xffffffffu, ford(b.hx)));
    b.hy = ordf(__reduce_max_sync(0xffffffffu, ford(b.hy)));
    b.hz = ordf(__reduce_max_sync(0xffffffffu, ford(b.hz)));
    return b;
}

// Box of the rows [a, b) (warp-collective).
__device__ __forceinline__ Box6 rows_box(int a, int b, const float (&x)[4], const float (&y)[4], const float (&z)[4]) {
    const int lane = threadIdx.x & 31;
    Box6 r{INFINITY, INFINITY, INFINITY, -INFINITY, -INFINITY, -INFINITY};
#pragma unroll
    for (int k = 0; k < 4; k++) {
        const int row = 4 * lane + k;
        if (row >= a && row < b) {
            r.lx = fminf(r.lx, x[k]);
            r.ly = fminf(r.ly, y[k]);
            r.lz = fminf(r.lz, z[k]);
            r.hx = fmaxf(r.hx, x[k]);
            r.hy = fmaxf(r.hy, y[k]);
            r.hz = fmaxf(r.hz, z[k]);
        }
    }
    return warp_reduce_box(r);
}

// Candidate split row of [a, b) or -1 (warp-uniform): the first row at the first Morton
// bit where the range's first and last keys differ.
__device__ __forceinline__ int rows_split_row(int a, int b, const uint32_t* keys, const uint32_t (&key)[4]) {
    if (b - a < 2) return -1;
    const uint32_t ka = keys[a], kb = keys[b - 1];
    if (ka == kb) return -1;
    const int bit = 31 - __clz(ka ^ kb);
    const int lane = threadIdx.x & 31;
    int first = kBlockRows;  // keys are sorted: the rows with the bit set are a suffix of [a, b)
#pragma unroll
    for (int k = 0; k < 4; k++) {
        const int row = 4 * lane + k;
        if (row >= a && row < b && ((key[k] >> bit) & 1u)) first = min(first, row);
    }
    return (int)__reduce_min_sync(0xffffffffu, (unsigned)first);
}

constexpr int kBlocksPerCta = 8;  // 128-row blocks (warps) per CTA of k_sample_blocks

__device__ __forceinline__ Box6 shfl_box(const Box6& b, int src) {
    return Box6{__shfl_sync(0xffffffffu, b.lx, src), __shfl_sync(0xffffffffu, b.ly, src),
                __shfl_sync(0xffffffffu, b.lz, src), __shfl_sync(0xffffffffu, b.hx, src),
                __shfl_sync(0xffffffffu, b.hy, src), __shfl_sync(0xffffffffu, b.hz, src)};
}

// Split tree of one block's valid rows [0, nvalid): node 1 is the block, nodes 2i and
// 2i + 1 are the halves of node i, three levels (at most 8 groups).  A range splits at its
// Morton split row when both halves' boxes have at most `ratio` of its half-perimeter.
// A split taken with some ratio is taken with every larger one at the same row, so the tree
// is built once with the larger of the two ratios, recording each node's two half-perimeter
// figures, and each ratio's groups are the leaves of the subtree whose splits pass its own
// test (the same float comparison as a tree built with that ratio alone).  Box unions are
// exact, so each node's box is computed once.  Lane i holds node i's fields.
struct SplitTree {
    Box6 box;    // box of node i
    int a, b;    // rows [a, b) of node i
    float h12;   // max(hp(half 1), hp(half 2)), +inf where node i has no split row
    float h;     // hp(node i)
};

__device__ __forceinline__ SplitTree split_tree_build(int nvalid, float rmax, const uint32_t* keys,
                                                      const uint32_t (&key)[4], const float (&x)[4],
                                                      const float (&y)[4], const float (&z)[4]) {
    const int lane = threadIdx.x & 31;
    SplitTree T;
    T.box = rows_box(0, nvalid, x, y, z);
    T.a = 0;
    T.b = nvalid;
    T.h12 = INFINITY;
    T.h = 0.f;
    bool ex[16];
#pragma unroll
    for (int i = 0; i < 16; i++) ex[i] = i == 1;
#pragma unroll
    for (int i = 1; i < 8; i++) {
        if (!ex[i]) continue;  // warp-uniform
        const int ai = __shfl_sync(0xffffffffu, T.a, i), bi = __shfl_sync(0xffffffffu, T.b, i);
        const int m = rows_split_row(ai, bi, keys, key);
        if (m < 0) continue;
        const Box6 B = shfl_box(T.box, i);
        const Box6 B1 = rows_box(ai, m, x, y, z);
        const Box6 B2 = rows_box(m, bi, x, y, z);
        const float h12 = fmaxf(hp6(B1), hp6(B2)), h = hp6(B);
        if (lane == i) {
            T.h12 = h12;
            T.h = h;
        }
        if (h12 <= rmax * h) {
            ex[2 * i] = ex[2 * i + 1] = true;
            if (lane == 2 * i) {
                T.box = B1;
                T.a = ai;
                T.b = m;
            }
            if (lane == 2 * i + 1) {
                T.box = B2;
                T.a = m;
                T.b = bi;
            }
        }
    }
    return T;
}

// Groups of `ratio` from the tree: bdesc[blk] = (starts of groups 1..7 as bytes, 128 if
// unused; byte 7 = group count), bboxes[blk * 8 + g] = (lo, hi) of group g (empty box if
// unused).
__device__ __forceinline__ void split_tree_store(const SplitTree& T, int64_t blk, float ratio,
                                                 uint2* __restrict__ bdesc, float4* __restrict__ bboxes) {
    const int lane = threadIdx.x & 31;
    const bool splits = T.h12 <= ratio * T.h;  // lane i: node i splits with this ratio
    const uint32_t sm = __ballot_sync(0xffffffffu, splits);
    int ids[kBlockGroups];
    int nr = 1;
    ids[0] = 1;
    for (int depth = 0; depth < 3; depth++) {
        int nid[kBlockGroups];
        int nn = 0;
        for (int k = 0; k < nr; k++) {
            const int i = ids[k];
            if ((sm >> i) & 1u) {
                nid[nn++] = 2 * i;
                nid[nn++] = 2 * i + 1;
            } else {
                nid[nn++] = i;
            }
        }
        for (int k = 0; k < nn; k++) ids[k] = nid[k];
        nr = nn;
    }
    const int mine = lane < nr ? ids[lane] : 0;
    const Box6 G = shfl_box(T.box, mine);
    const int start = __shfl_sync(0xffffffffu, T.a, mine);
    if (lane < kBlockGroups) {
        Box6 B{INFINITY, INFINITY, INFINITY, -INFINITY, -INFINITY, -INFINITY};
        if (lane < nr) B = G;
        bboxes[2 * (blk * kBlockGroups + lane)] = make_float4(B.lx, B.ly, B.lz, 0.f);
        bboxes[2 * (blk * kBlockGroups + lane) + 1] = make_float4(B.hx, B.hy, B.hz, 0.f);
    }
    uint32_t starts[kBlockGroups];
#pragma unroll
    for (int g = 0; g < kBlockGroups; g++) {
        const int sg = __shfl_sync(0xffffffffu, start, g);
        starts[g] = g < nr ? (uint32_t)sg : (uint32_t)kBlockRows;
    }
    if (lane == 0) {
        uint2 d;
        d.x = starts[1] | (starts[2] << 8) | (starts[3] << 16) | (starts[4] << 24);
        d.y = starts[5] | (starts[6] << 8) | (starts[7] << 16) | ((uint32_t)nr << 24);
        bdesc[blk] = d;
    }
}

// One warp per 128-row block: the rows are loaded once and split with `ratio` into
// (bdesc, bboxes) and, when bdesc2 is given, also with `ratio2` into (bdesc2, bboxes2).
__global__ void __launch_bounds__(32 * kBlocksPerCta) k_sample_blocks(const float4* __restrict__ s_sorted,
                                                                      const uint32_t* __restrict__ skeys, int64_t S,
                                                                      int64_t n_blocks, uint2* __restrict__ bdesc,
                                                                      float4* __restrict__ bboxes, float ratio,
                                                                      uint2* __restrict__ bdesc2,
                                                                      float4* __restrict__ bboxes2, float ratio2) {
    __shared__ uint32_t s_keys[kBlocksPerCta][kBlockRows];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t blk = (int64_t)blockIdx.x * kBlocksPerCta + warp;
    if (blk >= n_blocks) return;
    uint32_t* keys = s_keys[warp];
    float x[4], y[4], z[4];
    uint32_t key[4];
#pragma unroll
    for (int k = 0; k < 4; k++) {
        const int64_t row = blk * kBlockRows + 4 * lane + k;
        x[k] = y[k] = z[k] = NAN;
        key[k] = 0xffffffffu;
        if (row < S) {
            const float4 p = s_sorted[row];
            x[k] = p.x;
            y[k] = p.y;
            z[k] = p.z;
            key[k] = skeys[row];
        }
        keys[4 * lane + k] = key[k];
    }
    __syncwarp();
    const int64_t rem = S - blk * kBlockRows;
    const int nvalid = rem < kBlockRows ? (int)rem : kBlockRows;
    const SplitTree T = split_tree_build(nvalid, bdesc2 ? fmaxf(ratio, ratio2) : ratio, keys, key, x, y, z);
    split_tree_store(T, blk, ratio, bdesc, bboxes);
    if (bdesc2) split_tree_store(T, blk, ratio2, bdesc2, bboxes2);
}

// ---------------------------------------------------------------------------------------
// tcgen05 GEMM test hook: D[128 x N] = A[128 x 16] * B[N x 16]^T (bf16 in, fp32 out).
// ---------------------------------------------------------------------------------------
__global__ void __launch_bounds__(128) k_tc_gemm_test(const __nv_bfloat16* __restrict__ A,
                                                      const __nv_bfloat16* __restrict__ B, int N,
                                                      float* __restrict__ D, int* status) {
    __shared__ __align__(1024) unsigned char sA[kBlockRows * 32];
    __shared__ __align__(1024) unsigned char sB[256 * 32];
    __shared__ __align__(8) uint64_t bar;
    __shared__ uint32_t tmem_base;
    const int t = threadIdx.x, w = t >> 5;
    __nv_bfloat16 row[16];
    for (int k = 0; k < 16; k++) row[k] = A[t * 16 + k];
    store_row_k16(sA, t, row);
    for (int r = t; r < N; r += 128) {
        for (int k = 0; k < 16; k++) row[k] = B[r * 16 + k];
        store_row_k16(sB, r, row);
    }
    fence_proxy_async_smem();
    uint32_t ncols = 32;
    while ((int)ncols < N) ncols <<= 1;
    if (w == 0) {
        tmem_alloc(&tmem_base, ncols);
        tmem_relinquish();
    }
    if (t == 0) {
        mbar_init(&bar, 1);
        fence_mbar_init();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tb = tmem_base;
    if (t == 0) {
        umma_bf16(tb, smem_desc_k16(sA), smem_desc_k16(sB), idesc_bf16_f32(128, N), 0u);
        umma_commit(&bar);
    }
    const bool ok = mbar_wait(&bar, 0, status);
    tc_fence_after();
    if (ok) {
        for (int c = 0; c < N; c += 32) {
            float v[32];
            tmem_ld32(tb + ((uint32_t)(32 * w) << 16) + (uint32_t)c, v);
            for (int j = 0; j < 32; j++) D[(int64_t)t * N + c + j] = v[j];
        }
    }
    tc_fence_before();
    __syncthreads();
    if (w == 0) tmem_dealloc(tb, ncols);
}

// ---------------------------------------------------------------------------------------
// CTA forward (FP32): warp-specialised pipeline.
//   warp 2 (producer): walks the Gaussian LBVH with each group's box (warp-cooperative
//     traversal), copies each batch of up to 32 candidate records into one of kStages
//     stages with cp.async and, one call later, finalises it (base-2 conic, per-consumer
//     warp column masks);
//   warps 0-1 (consumers): thread (w, lane) owns rows (2 w + k) * 32 + lane, k = 0, 1;
//     for every column whose box overlaps the warp's rows of the group: the exact AABB
//     test of both rows, a warp vote per row chain, and for the chains with a row inside
//     the 9-FMA power, the window, ex2 and the sums, all in registers.
//   full[s]  completes when the producer has finalised s;
//   empty[s] completes when both consumer warps have released s.
// ---------------------------------------------------------------------------------------
constexpr int kStages = 4;            // batches in flight
constexpr int kBatch = 32;            // Gaussians per batch
constexpr int kRowsPerThread = 2;     // each staged record (80 bytes broadcast) serves two samples
constexpr int kConsumerWarps = 4 / kRowsPerThread;
// Resident CTAs per SM requested from the register allocator: 14 (40 registers; fewer
// spill loads than asking for 16: 16.82 against 17.00 ms at 2M x 16M).
constexpr int kCtaMinBlocks = 14;

struct CtaSmem {
    float4 gd[kStages][kBatch][5];       // (mu, w), C'(0..3), (C'4, C'5, v, -), lo, hi
    uint8_t colmask[kStages][kBatch];    // bit w: column overlaps consumer warp w's rows
    int2 desc[kStages];                  // (number of columns or -1 at the end, group)
    Box6 wb[kConsumerWarps];             // boxes of the current group's rows of each consumer warp
    int stack[kStackCap];
    int cand[kCandCap];
    uint64_t full[kStages], empty[kStages];
};

// Producer warp: traversal visitor that stages batches.  Batch k goes to stage k % kStages;
// its records are copied into shared memory with cp.async as soon as the traversal hands
// them over, and the batch is finalised (coefficients, masks) one call later, while the
// next batch's copies are in flight.
struct Producer {
    CtaSmem& sm;
    const GaussRec* __restrict__ recs;
    int* status;
    uint32_t total;  // batches handed to stages so far
    bool pending;
    int pend_stage, pend_nb;
    int g;
    bool failed;
    CandLog log;  // the block's candidates for the tensor-core backward (ids null: off)

    // waits until the consumers have released the previous use of the stage of batch n
    __device__ __forceinline__ bool acquire_batch(uint32_t n) {
        const uint32_t k = n / kStages;
        if (k == 0) return true;
        return mbar_wait(&sm.empty[n % kStages], (k - 1) & 1u, status);
    }

    __device__ __forceinline__ void finalize(int s, int nb) {
        const int lane = threadIdx.x & 31;
        uint8_t cm = 0;
        if (lane < nb) {
            const float4 r1 = sm.gd[s][lane][1], r2 = sm.gd[s][lane][2], r3 = sm.gd[s][lane][3],
                         r4 = sm.gd[s][lane][4];
            const float k = kHalfLog2eC;
            const float c0 = k * r1.x, c1 = k * r1.y, c2 = k * r1.z, c3 = k * r1.w, c4 = k * r2.x, c5 = k * r2.y;
            sm.gd[s][lane][1] = make_float4(c0, 2.f * c1, 2.f * c2, c3);
            sm.gd[s][lane][2] = make_float4(2.f * c4, c5, r2.z, 0.f);
#pragma unroll
            for (int ww = 0; ww < kConsumerWarps; ww++)
                cm |= overlap6(sm.wb[ww], r3, r4) ? (uint8_t)(1u << ww) : (uint8_t)0;
        }
        sm.colmask[s][lane] = cm;
        if (lane == 0) sm.desc[s] = make_int2(nb, g);
        __syncwarp();
        if (lane == 0) mbar_arrive(&sm.full[s]);
        __syncwarp();
    }

    __device__ __forceinline__ void flush() {
        if (pending) {
            cp_async_wait<0>();
            __syncwarp();
            finalize(pend_stage, pend_nb);
            pending = false;
        }
    }

    // waits until every batch handed out so far has been consumed
    __device__ __forceinline__ void drain() {
        for (uint32_t n = total >= kStages ? total - kStages : 0; n < total; n++)
            if (!acquire_batch(n + kStages)) failed = true;
    }

    __device__ __forceinline__ void operator()(const int* c, int nb) {
        const int lane = threadIdx.x & 31;
        log.append(c, nb);
        if (failed || !acquire_batch(total)) {
            failed = true;
            __syncwarp();
            return;
        }
        const int s = (int)(total % kStages);
        if (lane < nb) {
            const float4* src = reinterpret_cast<const float4*>(recs + c[lane]);
#pragma unroll
            for (int q = 0; q < 5; q++) cp_async16(&sm.gd[s][lane][q], src + q);
        }
        cp_async_commit();
        if (pending) {
            cp_async_wait<1>();
            __syncwarp();
            finalize(pend_stage, pend_nb);
        }
        pending = true;
        pend_stage = s;
        pend_nb = nb;
        total++;
        __syncwarp();
    }
};

template <bool COUNT, bool STACKLESS>
__global__ void __launch_bounds__(kConsumerWarps * 32 + 32, kCtaMinBlocks)
    k_forward_cta(const float4* __restrict__ s_sorted, int64_t S, const uint2* __restrict__ bdesc,
                  const float4* __restrict__ bboxes, const BvhNode* __restrict__ nodes, int64_t n_internal,
                  const GaussRec* __restrict__ recs, float* __restrict__ out_cells, float* __restrict__ out_weights,
                  float2* __restrict__ out_sorted, int32_t* __restrict__ clog, int32_t* __restrict__ cend, int* status,
                  unsigned long long* stats) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    CtaSmem& sm = *reinterpret_cast<CtaSmem*>(smem_raw);
    constexpr int RPT = kRowsPerThread;
    const int t = threadIdx.x, w = t >> 5, lane = t & 31;
    const int64_t blk = blockIdx.x;
    const uint2 bd = bdesc[blk];
    const int ng = group_count(bd);
    if (t == 0) {
        for (int s = 0; s < kStages; s++) {
            mbar_init(&sm.full[s], 1);
            mbar_init(&sm.empty[s], kConsumerWarps);
        }
        fence_mbar_init();
    }
    __syncthreads();

    if (w == kConsumerWarps) {
        // ---------------- producer ----------------
        Producer pr{sm, recs, status, 0u, false, 0, 0, 0, false};
        if (clog) pr.log.ids = clog + blk * kCandLogPerBlock;
        TravCount tc;
        int st = 0;
        for (int g = 0; g < ng && !pr.failed; g++) {
            // the column masks of the previous group's batches use sm.wb: consume them first
            pr.flush();
            pr.drain();
            if (pr.failed) break;
            const int ra = group_start(bd, g), rb = group_start(bd, g + 1);
            const float4 glo = bboxes[2 * (blk * kBlockGroups + g)], ghi = bboxes[2 * (blk * kBlockGroups + g) + 1];
            pr.g = g;
#pragma unroll
            for (int q = 0; q < 4; q++) {
                // row r belongs to consumer warp q / RPT
                const int r = 32 * q + lane;
                const int64_t row = blk * kBlockRows + r;
                const bool in = row < S && r >= ra && r < rb;
                float4 p = make_float4(0.f, 0.f, 0.f, 0.f);
                if (in) p = s_sorted[row];
                const Box6 bq = warp_box6(in, p.x, p.y, p.z);
                if (lane == 0) {
                    if (q % RPT == 0) {
                        sm.wb[q / RPT] = bq;
                    } else {
                        Box6& u = sm.wb[q / RPT];
                        u.lx = fminf(u.lx, bq.lx);
                        u.ly = fminf(u.ly, bq.ly);
                        u.lz = fminf(u.lz, bq.lz);
                        u.hx = fmaxf(u.hx, bq.hx);
                        u.hy = fmaxf(u.hy, bq.hy);
                        u.hz = fmaxf(u.hz, bq.hz);
                    }
                }
            }
            __syncwarp();
            st |= warp_traverse_sel<STACKLESS>(nodes, n_internal, make_float3(glo.x, glo.y, glo.z),
                                               make_float3(ghi.x, ghi.y, ghi.z), sm.stack, sm.cand, pr, tc);
            pr.log.end_group(g);
        }
        if (pr.failed || st) pr.log.over = true;
        if (clog) pr.log.finish(cend + blk * kBlockGroups, ng);
        pr.flush();
        if (st && lane == 0) atomicOr(status, st);
        // end marker
        if (pr.acquire_batch(pr.total)) {
            const int s = (int)(pr.total % kStages);
            if (lane == 0) {
                sm.desc[s] = make_int2(-1, 0);
                mbar_arrive(&sm.full[s]);
            }
        }
        __syncwarp();
        if (COUNT && lane == 0) {
            atomicMax(&stats[3], (unsigned long long)tc.max_sp);
            atomicAdd(&stats[5], (unsigned long long)tc.leaves);
            atomicAdd(&stats[6], (unsigned long long)tc.nodes);
        }
    } else {
        // ---------------- consumers: thread (w, lane) owns rows (w * RPT + k) * 32 + lane ----------------
        float xr[RPT], yr[RPT], zr[RPT], Wr[RPT], Vr[RPT];
        int orig[RPT];
        bool valid[RPT];
#pragma unroll
        for (int k = 0; k < RPT; k++) {
            const int64_t row = blk * kBlockRows + (w * RPT + k) * 32 + lane;
            valid[k] = row < S;
            float4 spv = make_float4(NAN, NAN, NAN, __int_as_float(-1));
            if (valid[k]) spv = s_sorted[row];
            xr[k] = spv.x;
            yr[k] = spv.y;
            zr[k] = spv.z;
            orig[k] = __float_as_int(spv.w);
            Wr[k] = 0.f;
            Vr[k] = 0.f;
        }
        int ncand = 0, ncontrib = 0, nlane = 0;
        uint32_t n = 0;  // batches consumed
        while (true) {
            const int stage = (int)(n % kStages);
            const bool ok = mbar_wait(&sm.full[stage], (n / kStages) & 1u, status);
            if (!__all_sync(0xffffffffu, ok)) break;
            const int2 d = sm.desc[stage];
            if (d.x < 0) break;
            const int ra = group_start(bd, d.y), rb = group_start(bd, d.y + 1);
            bool ing[RPT];
#pragma unroll
            for (int k = 0; k < RPT; k++) {
                const int r = (w * RPT + k) * 32 + lane;
                ing[k] = valid[k] && r >= ra && r < rb;
            }
            const uint8_t cm = sm.colmask[stage][lane];
            const uint32_t wm = __ballot_sync(0xffffffffu, (cm >> w) & 1u);
            if (COUNT) nlane += 32 * RPT * __popc(wm);
            uint32_t mm = wm;
            while (mm) {
                const int j = __ffs(mm) - 1;
                mm &= mm - 1;
                const float4 lo = sm.gd[stage][j][3], hi = sm.gd[stage][j][4];
                bool inr[RPT];
                uint32_t kany = 0;
#pragma unroll
                for (int k = 0; k < RPT; k++) {
                    const float x = xr[k], y = yr[k], z = zr[k];
                    inr[k] = ing[k] && lo.x <= x && x <= hi.x && lo.y <= y && y <= hi.y && lo.z <= z && z <= hi.z;
                    kany |= __any_sync(0xffffffffu, inr[k]) ? (1u << k) : 0u;
                }
                // the column's box overlaps the warp's rows, but often no row lies inside it; a
                // vote per row chain also skips the chain none of whose rows is inside
                if (!kany) continue;
                const float4 r0 = sm.gd[stage][j][0], r1 = sm.gd[stage][j][1], r2 = sm.gd[stage][j][2];
#pragma unroll
                for (int k = 0; k < RPT; k++) {
                    if (!((kany >> k) & 1u)) continue;
                    const float x = xr[k], y = yr[k], z = zr[k];
                    const bool in = inr[k];
                    const float dx = x - r0.x, dy = y - r0.y, dz = z - r0.z;
                    const float p2 = dx * fmaf(r1.x, dx, fmaf(r1.y, dy, r1.z * dz)) + dy * fmaf(r1.w, dy, r2.x * dz) +
                                     dz * (r2.y * dz);
                    const bool cc = in && p2 >= kLog2FloorC && p2 <= 0.0f;
                    const float wt = cc ? r0.w * ex2_apx(p2) : 0.f;
                    Wr[k] += wt;
                    Vr[k] = fmaf(wt, r2.z, Vr[k]);
                    if (COUNT) {
                        ncand += in ? 1 : 0;
                        ncontrib += cc ? 1 : 0;
                    }
                }
            }
            __syncwarp();
            if (lane == 0) mbar_arrive(&sm.empty[stage]);
            n++;
        }
#pragma unroll
        for (int k = 0; k < RPT; k++) {
            if (valid[k]) {
                float o, ww;
                if (Wr[k] <= kWeightCutoff) {
                    o = -1.0f;
                    ww = 0.0f;
                } else {
                    o = Vr[k] / Wr[k];
                    ww = Wr[k];
                }
                out_cells[orig[k]] = o;
                out_weights[orig[k]] = ww;
                // the same pair in sorted order (coalesced), so that the backward's sample
                // records need not gather them back
                if (out_sorted) out_sorted[blk * kBlockRows + (w * RPT + k) * 32 + lane] = make_float2(o, ww);
            }
        }
        if (COUNT) {
            unsigned long long a = (unsigned long long)ncand, b = (unsigned long long)ncontrib;
            for (int off = 16; off > 0; off >>= 1) {
                a += __shfl_xor_sync(0xffffffffu, a, off);
                b += __shfl_xor_sync(0xffffffffu, b, off);
            }
            if (lane == 0) {
                atomicAdd(&stats[0], a);
                atomicAdd(&stats[1], b);
                atomicAdd(&stats[9], (unsigned long long)nlane);
            }
        }
    }
}

static inline unsigned nblk128(int64_t n) { return (unsigned)((n + kBlockRows - 1) / kBlockRows); }

cudaError_t launch_sample_blocks(int64_t S, const float4* s_sorted, const uint32_t* skeys, uint2* bdesc,
                                 float4* bboxes, float ratio, cudaStream_t st, uint2* bdesc2, float4* bboxes2,
                                 float ratio2) {
    if (S <= 0) return cudaSuccess;
    const int64_t nb = (S + kBlockRows - 1) / kBlockRows;
    k_sample_blocks<<<(unsigned)((nb + kBlocksPerCta - 1) / kBlocksPerCta), 32 * kBlocksPerCta, 0, st>>>(
        s_sorted, skeys, S, nb, bdesc, bboxes, ratio, bdesc2, bboxes2, ratio2);
    gvc::note_launch();
    return cudaGetLastError();
}

template <bool COUNT, bool STACKLESS>
static cudaError_t launch_cta_impl(const CtaArgs& a, cudaStream_t st) {
    const size_t smem = sizeof(CtaSmem);
    cudaError_t e =
        cudaFuncSetAttribute(k_forward_cta<COUNT, STACKLESS>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    k_forward_cta<COUNT, STACKLESS><<<nblk128(a.S), kConsumerWarps * 32 + 32, smem, st>>>(
        a.s_sorted, a.S, a.bdesc, a.bboxes, a.gnodes, a.n_internal, a.recs, a.out_cells, a.out_weights,
        a.out_sorted, a.clog, a.cend, a.status, a.stats);
    gvc::note_launch();
    return cudaGetLastError();
}

cudaError_t launch_forward_cta(const CtaArgs& a, bool tc, cudaStream_t st) {
    if (a.S <= 0) return cudaSuccess;
    if (tc) return launch_forward_tc(a, st);
    if (a.stackless) return a.count ? launch_cta_impl<true, true>(a, st) : launch_cta_impl<false, true>(a, st);
    return a.count ? launch_cta_impl<true, false>(a, st) : launch_cta_impl<false, false>(a, st);
}

cudaError_t launch_tc_gemm_test(const void* A, const void* B, int N, float* D, int* status, cudaStream_t st) {
    k_tc_gemm_test<<<1, 128, 0, st>>>(reinterpret_cast<const __nv_bfloat16*>(A),
                                      reinterpret_cast<const __nv_bfloat16*>(B), N, D, status); gvc::note_launch();
    return cudaGetLastError();
}

__global__ void __launch_bounds__(32) k_wait_timeout_test(int* status) {
    __shared__ __align__(8) uint64_t bar;
    if (threadIdx.x == 0) {
        mbar_init(&bar, 1);
        fence_mbar_init();
    }
    __syncwarp();
    // nothing arrives on `bar`: phase 0 never completes and the wait gives up
    if (threadIdx.x == 0) (void)mbar_wait(&bar, 0, status);
    __syncwarp();
}

cudaError_t launch_wait_timeout_test(int* status, cudaStream_t st) {
    k_wait_timeout_test<<<1, 32, 0, st>>>(status); gvc::note_launch();
    return cudaGetLastError();
}

}  // namespace gvc
