// cta.cu -- CTA-level forward evaluation with a tensor-core (tcgen05) or FP32 SIMT
// exponent, the 128-sample block groups it runs on, and a tcgen05 GEMM test hook.
//
// One CTA (4 warps) owns 128 consecutive Morton-sorted samples.  build_bvh splits each
// such block into at most 8 contiguous "block groups" at Z-order jumps (the rule of the
// 32-sample tiles, applied to 128 rows).  For each group the CTA walks the Gaussian LBVH
// (a producer warp, warp-cooperative traversal) and stages candidate Gaussians 32 at a time.
//
// Tensor-core exponent: with x0 the centre of the group box, u = x - x0 and m = mu - x0,
//   log2-power p2 = -0.5 log2(e) (x - mu)^T C (x - mu) = phi(u) . beta(m, C)
//   phi  = [ux^2, uy^2, uz^2, ux uy, ux uz, uy uz, ux, uy, uz, 1, 0 x 6]        (A, 128 x 16)
//   beta = k [C00, C11, C22, 2C01, 2C02, 2C12, -2(Cm)x, -2(Cm)y, -2(Cm)z, m^T C m, 0 x 6]
//          with k = -0.5 log2(e)                                                (B, 64 x 16)
// Both operands are split into three BF16 parts (hi + mid + lo, ~24 bits); the six
// products with i + j <= 2 are accumulated in FP32 in tensor memory by tcgen05.mma
// (M = 128, N = 32, K = 16).  Columns whose term bound sum_k |beta_k| max|phi_k| exceeds
// kTcMaxTerm are recomputed in FP32 SIMT (the FP32 accumulation error grows with the
// terms, not with the result).  The epilogue applies the exact AABB test, the power
// window, ex2 and the accumulation in FP32, visiting only columns whose box overlaps the
// warp's own samples.  The SIMT variant runs the identical structure with the quadratic
// form evaluated in FP32 per lane.
#include "render.cuh"
#include "tc.cuh"
#include "traverse.cuh"

namespace gvc {

constexpr int kBlockRows = 128;
constexpr int kBlockGroups = 8;
constexpr float kTcMaxTerm = 256.0f;  // term bound above which a column is evaluated in SIMT

constexpr float kHalfLog2eC = -0.72134752044448170368f;
constexpr float kLog2FloorC = -20.197570572173914f;

__device__ __forceinline__ float ex2_apx(float x) {
    float y;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

struct Box6 {
    float lx, ly, lz, hx, hy, hz;
};

__device__ __forceinline__ Box6 warp_box6(bool in, float x, float y, float z) {
    Box6 b{in ? x : INFINITY, in ? y : INFINITY, in ? z : INFINITY, in ? x : -INFINITY, in ? y : -INFINITY,
           in ? z : -INFINITY};
    for (int off = 16; off > 0; off >>= 1) {
        b.lx = fminf(b.lx, __shfl_xor_sync(0xffffffffu, b.lx, off));
        b.ly = fminf(b.ly, __shfl_xor_sync(0xffffffffu, b.ly, off));
        b.lz = fminf(b.lz, __shfl_xor_sync(0xffffffffu, b.lz, off));
        b.hx = fmaxf(b.hx, __shfl_xor_sync(0xffffffffu, b.hx, off));
        b.hy = fmaxf(b.hy, __shfl_xor_sync(0xffffffffu, b.hy, off));
        b.hz = fmaxf(b.hz, __shfl_xor_sync(0xffffffffu, b.hz, off));
    }
    return b;
}

__device__ __forceinline__ float hp6(const Box6& b) { return (b.hx - b.lx) + (b.hy - b.ly) + (b.hz - b.lz); }

// One warp per 128-row block; lane l holds rows 4l .. 4l + 3 (shuffles only, no block
// barriers).  Box unions are min/max reductions, so the result does not depend on the
// reduction order.
__device__ __forceinline__ Box6 warp_reduce_box(Box6 b) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        b.lx = fminf(b.lx, __shfl_xor_sync(0xffffffffu, b.lx, off));
        b.ly = fminf(b.ly, __shfl_xor_sync(0xffffffffu, b.ly, off));
        b.lz = fminf(b.lz, __shfl_xor_sync(0xffffffffu, b.lz, off));
        b.hx = fmaxf(b.hx, __shfl_xor_sync(0xffffffffu, b.hx, off));
        b.hy = fmaxf(b.hy, __shfl_xor_sync(0xffffffffu, b.hy, off));
        b.hz = fmaxf(b.hz, __shfl_xor_sync(0xffffffffu, b.hz, off));
    }
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

// Split row of [a, b) or -1 (warp-uniform): at the first Morton bit where the range's
// first and last keys differ, taken when both halves' boxes have at most half the
// half-perimeter of the whole.
__device__ int rows_split(int a, int b, const uint32_t* keys, const uint32_t (&key)[4], const float (&x)[4],
                          const float (&y)[4], const float (&z)[4], float ratio) {
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
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) first = min(first, __shfl_xor_sync(0xffffffffu, first, off));
    const int m = first;
    const Box6 B = rows_box(a, b, x, y, z);
    const Box6 B1 = rows_box(a, m, x, y, z);
    const Box6 B2 = rows_box(m, b, x, y, z);
    return fmaxf(hp6(B1), hp6(B2)) <= ratio * hp6(B) ? m : -1;
}

constexpr int kBlocksPerCta = 8;  // 128-row blocks (warps) per CTA of k_sample_blocks

// Splits the block's valid rows [0, nvalid) three times (every range of a level in
// order, at most 8 groups) with `ratio` and writes bdesc[blk] = (starts of groups 1..7
// as bytes, 128 if unused; byte 7 = group count) and bboxes[blk * 8 + g] = (lo, hi) of
// group g (empty box if unused).
__device__ __forceinline__ void block_split_store(int64_t blk, int nvalid, const uint32_t* keys,
                                                  const uint32_t (&key)[4], const float (&x)[4],
                                                  const float (&y)[4], const float (&z)[4], float ratio,
                                                  uint2* __restrict__ bdesc, float4* __restrict__ bboxes) {
    const int lane = threadIdx.x & 31;
    int ra[kBlockGroups], rb[kBlockGroups];
    int nr = 1;
    ra[0] = 0;
    rb[0] = nvalid;
    for (int depth = 0; depth < 3; depth++) {
        int na[kBlockGroups], nbb[kBlockGroups];
        int nn = 0;
        for (int i = 0; i < nr; i++) {
            const int m = rows_split(ra[i], rb[i], keys, key, x, y, z, ratio);
            if (m >= 0) {
                na[nn] = ra[i];
                nbb[nn++] = m;
                na[nn] = m;
                nbb[nn++] = rb[i];
            } else {
                na[nn] = ra[i];
                nbb[nn++] = rb[i];
            }
        }
        for (int i = 0; i < nn; i++) {
            ra[i] = na[i];
            rb[i] = nbb[i];
        }
        nr = nn;
    }
    uint32_t starts[kBlockGroups];
    for (int g = 0; g < kBlockGroups; g++) starts[g] = g < nr ? (uint32_t)ra[g] : (uint32_t)kBlockRows;
    for (int g = 0; g < kBlockGroups; g++) {
        Box6 B{INFINITY, INFINITY, INFINITY, -INFINITY, -INFINITY, -INFINITY};
        if (g < nr) B = rows_box(ra[g], rb[g], x, y, z);
        if (lane == 0) {
            bboxes[2 * (blk * kBlockGroups + g)] = make_float4(B.lx, B.ly, B.lz, 0.f);
            bboxes[2 * (blk * kBlockGroups + g) + 1] = make_float4(B.hx, B.hy, B.hz, 0.f);
        }
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
    block_split_store(blk, nvalid, keys, key, x, y, z, ratio, bdesc, bboxes);
    if (bdesc2) block_split_store(blk, nvalid, keys, key, x, y, z, ratio2, bdesc2, bboxes2);
}

__device__ __forceinline__ int group_start(uint2 d, int g) {
    if (g == 0) return 0;
    if (g >= kBlockGroups) return kBlockRows;
    if (g <= 4) return (int)((d.x >> (8 * (g - 1))) & 0xffu);
    return (int)((d.y >> (8 * (g - 5))) & 0xffu);
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
// CTA forward: warp-specialised pipeline.
//   warp 4 (producer): per block group writes the A operand, walks the Gaussian LBVH with
//     the group box (warp-cooperative traversal), stages 32 candidates per batch (records,
//     base-2 conic, tensor-core coefficients, per-warp column masks) into one of two
//     stages and issues the six MMAs of that batch into the stage's 32 TMEM columns;
//   warps 0-3 (consumers): own TMEM lanes 32w..32w+31 = rows 32w..32w+31; per batch they
//     read their accumulator columns and run the FP32 epilogue, then release the stage.
//   full[s]  completes when the producer has staged s (arrive) and its MMAs are done (commit);
//   empty[s] completes when the four consumer warps have released s.
// ---------------------------------------------------------------------------------------
// Batches in flight: 4 for the SIMT variant; 2 for the tensor-core variant, whose smaller
// operand ring lets 6 CTAs share an SM (24.6 ms instead of 26.2 ms at 2M x 16M).
template <bool TC>
constexpr int kStagesOf = TC ? 2 : 4;
constexpr int kBatch = 32;  // Gaussians per MMA batch (N)

__device__ __forceinline__ bool overlap6(const Box6& b, float4 lo, float4 hi) {
    return lo.x <= b.hx && hi.x >= b.lx && lo.y <= b.hy && hi.y >= b.ly && lo.z <= b.hz && hi.z >= b.lz;
}

// Tensor-core operands (first in the block, 1024-byte aligned); absent in the SIMT variant,
// whose smaller footprint lets more CTAs share an SM.
template <bool TC>
struct CtaTcOperands {
    unsigned char A[3][kBlockRows * 32];       // phi(u), three bf16 parts
    unsigned char B[kStagesOf<TC>][3][kBatch * 32];  // beta, three bf16 parts, per stage
};
template <>
struct CtaTcOperands<false> {};

template <bool TC>
struct CtaSmem : CtaTcOperands<TC> {
    float4 gd[kStagesOf<TC>][kBatch][5];                 // (mu, w), C'(0..3), (C'4, C'5, v, -), lo, hi
    uint8_t colmask[kStagesOf<TC>][kBatch];              // bits 0..3: column overlaps warp w; bit 4: SIMT fallback
    int2 desc[kStagesOf<TC>];                            // (number of columns or -1 at the end, group)
    Box6 wb[4];                                    // boxes of the current group's rows of each consumer warp
    int stack[kStackCap];
    int cand[kCandCap];
    uint64_t full[kStagesOf<TC>], empty[kStagesOf<TC>];
    uint32_t tmem_base;
};

__device__ __forceinline__ void cp_async16(void* dst, const void* src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// Producer warp: traversal visitor that stages batches.  Batch k goes to stage k % kStages;
// its records are copied into shared memory with cp.async as soon as the traversal hands
// them over, and the batch is finalised (coefficients, masks, MMAs) one call later, while
// the next batch's copies are in flight.
template <bool TC, bool COUNT, int NCW>
struct Producer {
    static constexpr int kStages = kStagesOf<TC>;
    CtaSmem<TC>& sm;
    const GaussRec* __restrict__ recs;
    int* status;
    uint32_t tmem;
    uint32_t total;  // batches handed to stages so far
    bool pending;
    int pend_stage, pend_nb;
    int g;
    float x0, y0, z0, ex, ey, ez;
    bool failed;

    // waits until the consumers have released the previous use of the stage of batch n
    __device__ __forceinline__ bool acquire_batch(uint32_t n) {
        const uint32_t k = n / kStages;
        if (k == 0) return true;
        return mbar_wait(&sm.empty[n % kStages], (k - 1) & 1u, status);
    }

    __device__ __forceinline__ void finalize(int s, int nb) {
        const int lane = threadIdx.x & 31;
        if (TC) tc_fence_after();
        uint8_t cm = 0;
        if (lane < nb) {
            const float4 r0 = sm.gd[s][lane][0], r1 = sm.gd[s][lane][1], r2 = sm.gd[s][lane][2],
                         r3 = sm.gd[s][lane][3], r4 = sm.gd[s][lane][4];
            const float k = kHalfLog2eC;
            const float c0 = k * r1.x, c1 = k * r1.y, c2 = k * r1.z, c3 = k * r1.w, c4 = k * r2.x, c5 = k * r2.y;
            sm.gd[s][lane][1] = make_float4(c0, 2.f * c1, 2.f * c2, c3);
            sm.gd[s][lane][2] = make_float4(2.f * c4, c5, r2.z, 0.f);
#pragma unroll
            for (int ww = 0; ww < NCW; ww++) cm |= overlap6(sm.wb[ww], r3, r4) ? (uint8_t)(1u << ww) : (uint8_t)0;
            if constexpr (TC) {
                const float mx = r0.x - x0, my = r0.y - y0, mz = r0.z - z0;
                const float cmx = c0 * mx + c1 * my + c2 * mz;
                const float cmy = c1 * mx + c3 * my + c4 * mz;
                const float cmz = c2 * mx + c4 * my + c5 * mz;
                float beta[16];
                beta[0] = c0;
                beta[1] = c3;
                beta[2] = c5;
                beta[3] = 2.f * c1;
                beta[4] = 2.f * c2;
                beta[5] = 2.f * c4;
                beta[6] = -2.f * cmx;
                beta[7] = -2.f * cmy;
                beta[8] = -2.f * cmz;
                beta[9] = mx * cmx + my * cmy + mz * cmz;
#pragma unroll
                for (int q = 10; q < 16; q++) beta[q] = 0.f;
                const float bound = fabsf(beta[0]) * ex * ex + fabsf(beta[1]) * ey * ey + fabsf(beta[2]) * ez * ez +
                                    fabsf(beta[3]) * ex * ey + fabsf(beta[4]) * ex * ez + fabsf(beta[5]) * ey * ez +
                                    fabsf(beta[6]) * ex + fabsf(beta[7]) * ey + fabsf(beta[8]) * ez + fabsf(beta[9]);
                if (!(bound <= kTcMaxTerm)) cm |= 16;
                __nv_bfloat16 h[16], m[16], l[16];
                split_bf16(beta, h, m, l);
                store_row_k16(sm.B[s][0], lane, h);
                store_row_k16(sm.B[s][1], lane, m);
                store_row_k16(sm.B[s][2], lane, l);
            }
        } else if constexpr (TC) {
            __nv_bfloat16 zz[16];
#pragma unroll
            for (int q = 0; q < 16; q++) zz[q] = __float2bfloat16_rn(0.f);
            store_row_k16(sm.B[s][0], lane, zz);
            store_row_k16(sm.B[s][1], lane, zz);
            store_row_k16(sm.B[s][2], lane, zz);
        }
        sm.colmask[s][lane] = cm;
        if (lane == 0) sm.desc[s] = make_int2(nb, g);
        if (TC) fence_proxy_async_smem();
        __syncwarp();
        if (lane == 0) {
            if constexpr (TC) {
                const uint32_t idesc = idesc_bf16_f32(kBlockRows, kBatch);
                const uint32_t d = tmem + (uint32_t)(s * kBatch);
                const uint64_t a0 = smem_desc_k16(sm.A[0]), a1 = smem_desc_k16(sm.A[1]), a2 = smem_desc_k16(sm.A[2]);
                const uint64_t b0 = smem_desc_k16(sm.B[s][0]), b1 = smem_desc_k16(sm.B[s][1]),
                               b2 = smem_desc_k16(sm.B[s][2]);
                umma_bf16(d, a2, b0, idesc, 0u);  // lo * hi
                umma_bf16(d, a1, b1, idesc, 1u);  // mid * mid
                umma_bf16(d, a0, b2, idesc, 1u);  // hi * lo
                umma_bf16(d, a1, b0, idesc, 1u);  // mid * hi
                umma_bf16(d, a0, b1, idesc, 1u);  // hi * mid
                umma_bf16(d, a0, b0, idesc, 1u);  // hi * hi
                umma_commit(&sm.full[s]);
            }
            mbar_arrive(&sm.full[s]);
            if (!TC) mbar_arrive(&sm.full[s]);
        }
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

// Resident CTAs per SM requested from the register allocator.  The tensor-core variant
// (4 consumer warps, one row per thread) runs 6; the SIMT
// variant with one row per thread fits 8 (40 warps), with two rows per thread 16
// (48 warps, 40 registers).
constexpr int kCtaMinBlocksTc = 6;
constexpr int kCtaMinBlocksSimt1 = 8;
constexpr int kCtaMinBlocksSimt2 = 14;
// Rows per consumer thread of the SIMT variant: each staged record (80 bytes broadcast to
// every lane) then serves two samples, halving the shared-memory datapath traffic.
constexpr int kSimtRowsPerThread = 2;

template <bool TC, bool COUNT, int RPT>
__global__ void __launch_bounds__((4 / RPT) * 32 + 32,
                                  TC ? kCtaMinBlocksTc : (RPT == 1 ? kCtaMinBlocksSimt1 : kCtaMinBlocksSimt2))
    k_forward_cta(
    const float4* __restrict__ s_sorted, int64_t S, const uint2* __restrict__ bdesc,
    const float4* __restrict__ bboxes, const BvhNode* __restrict__ nodes, const GaussRec* __restrict__ recs,
    float* __restrict__ out_cells, float* __restrict__ out_weights, int* status, unsigned long long* stats) {
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    CtaSmem<TC>& sm = *reinterpret_cast<CtaSmem<TC>*>(smem_raw);
    static_assert(!TC || RPT == 1, "the tensor-core variant owns one row (TMEM lane) per thread");
    constexpr int kStages = kStagesOf<TC>;
    static_assert(!TC || tmem_cols_ok(kStages * kBatch), "TMEM columns must be a power of two >= 32");
    constexpr int NCW = 4 / RPT;  // consumer warps; warp NCW is the producer
    const int t = threadIdx.x, w = t >> 5, lane = t & 31;
    const int64_t blk = blockIdx.x;
    const uint2 bd = bdesc[blk];
    const int ng = (int)(bd.y >> 24);
    if (t == 0) {
        for (int s = 0; s < kStages; s++) {
            mbar_init(&sm.full[s], 2);
            mbar_init(&sm.empty[s], NCW);
        }
        fence_mbar_init();
    }
    if (TC && w == 0) {
        tmem_alloc(&sm.tmem_base, kStages * kBatch);
        tmem_relinquish();
    }
    if (TC) tc_fence_before();
    __syncthreads();
    if (TC) tc_fence_after();
    const uint32_t tmem = TC ? sm.tmem_base : 0u;

    if (w == NCW) {
        // ---------------- producer ----------------
        Producer<TC, COUNT, NCW> pr{sm, recs, status, tmem, 0u, false, 0, 0, 0, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, false};
        TravCount tc;
        int st = 0;
        for (int g = 0; g < ng && !pr.failed; g++) {
            // every issued batch must be consumed before A is rewritten
            pr.flush();
            pr.drain();
            if (pr.failed) break;
            const int ra = group_start(bd, g), rb = group_start(bd, g + 1);
            const float4 glo = bboxes[2 * (blk * kBlockGroups + g)], ghi = bboxes[2 * (blk * kBlockGroups + g) + 1];
            pr.g = g;
            pr.x0 = 0.5f * (glo.x + ghi.x);
            pr.y0 = 0.5f * (glo.y + ghi.y);
            pr.z0 = 0.5f * (glo.z + ghi.z);
            pr.ex = 0.5f * (ghi.x - glo.x);
            pr.ey = 0.5f * (ghi.y - glo.y);
            pr.ez = 0.5f * (ghi.z - glo.z);
            if (TC) tc_fence_after();
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
                if constexpr (TC) {
                    float phi[16];
                    const float ux = in ? p.x - pr.x0 : 0.f, uy = in ? p.y - pr.y0 : 0.f, uz = in ? p.z - pr.z0 : 0.f;
                    phi[0] = ux * ux;
                    phi[1] = uy * uy;
                    phi[2] = uz * uz;
                    phi[3] = ux * uy;
                    phi[4] = ux * uz;
                    phi[5] = uy * uz;
                    phi[6] = ux;
                    phi[7] = uy;
                    phi[8] = uz;
                    phi[9] = in ? 1.f : 0.f;
#pragma unroll
                    for (int k = 10; k < 16; k++) phi[k] = 0.f;
                    __nv_bfloat16 h[16], m[16], l[16];
                    split_bf16(phi, h, m, l);
                    store_row_k16(sm.A[0], r, h);
                    store_row_k16(sm.A[1], r, m);
                    store_row_k16(sm.A[2], r, l);
                }
            }
            if (TC) fence_proxy_async_smem();
            __syncwarp();
            st |= warp_traverse(nodes, make_float3(glo.x, glo.y, glo.z), make_float3(ghi.x, ghi.y, ghi.z), sm.stack,
                                sm.cand, pr, tc);
        }
        pr.flush();
        if (st && lane == 0) atomicOr(status, st);
        // end marker
        if (pr.acquire_batch(pr.total)) {
            const int s = (int)(pr.total % kStages);
            if (lane == 0) {
                sm.desc[s] = make_int2(-1, 0);
                mbar_arrive(&sm.full[s]);
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
            if constexpr (TC) {
                const float x = xr[0], y = yr[0], z = zr[0];
                float W = Wr[0], V = Vr[0];
                const uint32_t fb = __ballot_sync(0xffffffffu, (cm >> 4) & 1u);
                tc_fence_after();
                float v[32];
                tmem_ld32(tmem + ((uint32_t)(32 * w) << 16) + (uint32_t)(stage * kBatch), v);
#pragma unroll
                for (int j = 0; j < kBatch; j++) {
                    if (!((wm >> j) & 1u)) continue;
                    const float4 lo = sm.gd[stage][j][3], hi = sm.gd[stage][j][4];
                    const bool in = ing[0] && lo.x <= x && x <= hi.x && lo.y <= y && y <= hi.y && lo.z <= z && z <= hi.z;
                    const float4 r0 = sm.gd[stage][j][0];
                    float p2 = v[j];
                    if ((fb >> j) & 1u) {
                        const float4 r1 = sm.gd[stage][j][1], r2 = sm.gd[stage][j][2];
                        const float dx = x - r0.x, dy = y - r0.y, dz = z - r0.z;
                        p2 = dx * fmaf(r1.x, dx, fmaf(r1.y, dy, r1.z * dz)) + dy * fmaf(r1.w, dy, r2.x * dz) +
                             dz * (r2.y * dz);
                    }
                    const bool cc = in && p2 >= kLog2FloorC && p2 <= 0.0f;
                    const float wt = cc ? r0.w * ex2_apx(p2) : 0.f;
                    W += wt;
                    V = fmaf(wt, sm.gd[stage][j][2].z, V);
                    if (COUNT) {
                        ncand += in ? 1 : 0;
                        ncontrib += cc ? 1 : 0;
                    }
                }
                Wr[0] = W;
                Vr[0] = V;
                tc_fence_before();
            } else {
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
                        const float p2 = dx * fmaf(r1.x, dx, fmaf(r1.y, dy, r1.z * dz)) +
                                         dy * fmaf(r1.w, dy, r2.x * dz) + dz * (r2.y * dz);
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
    if (TC) tc_fence_before();
    __syncthreads();
    if (TC) {
        tc_fence_after();
        if (w == 0) tmem_dealloc(tmem, kStages * kBatch);
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

template <bool TC, bool COUNT>
static cudaError_t launch_cta_impl(const CtaArgs& a, cudaStream_t st) {
    constexpr int RPT = TC ? 1 : kSimtRowsPerThread;
    const size_t smem = sizeof(CtaSmem<TC>) + 1024;
    cudaError_t e = cudaFuncSetAttribute(k_forward_cta<TC, COUNT, RPT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem);
    if (e != cudaSuccess) return e;
    k_forward_cta<TC, COUNT, RPT><<<nblk128(a.S), (4 / RPT) * 32 + 32, smem, st>>>(a.s_sorted, a.S, a.bdesc, a.bboxes, a.gnodes,
                                                                     a.recs, a.out_cells, a.out_weights, a.status,
                                                                     a.stats); gvc::note_launch();
    return cudaGetLastError();
}

cudaError_t launch_forward_cta(const CtaArgs& a, bool tc, cudaStream_t st) {
    if (a.S <= 0) return cudaSuccess;
    if (tc) return a.count ? launch_cta_impl<true, true>(a, st) : launch_cta_impl<true, false>(a, st);
    return a.count ? launch_cta_impl<false, true>(a, st) : launch_cta_impl<false, false>(a, st);
}

cudaError_t launch_tc_gemm_test(const void* A, const void* B, int N, float* D, int* status, cudaStream_t st) {
    k_tc_gemm_test<<<1, 128, 0, st>>>(reinterpret_cast<const __nv_bfloat16*>(A),
                                      reinterpret_cast<const __nv_bfloat16*>(B), N, D, status); gvc::note_launch();
    return cudaGetLastError();
}

}  // namespace gvc
