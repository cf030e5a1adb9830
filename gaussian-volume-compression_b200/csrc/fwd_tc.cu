// fwd_tc.cu -- forward evaluation of the mixture field with the exponent on the tensor
// cores (tcgen05, split BF16, FP32 accumulation in tensor memory).  Replaces the per-pair
// power of FORWARD::sampleRenderCUDA / renderCUDA
// (diff-gaussian-rasterization/cuda_rasterizer/forward.cu:155-170, 224-256).
//
// One CTA owns one 128-row block of Morton-sorted samples and its block groups
// (k_sample_blocks: at most 8 contiguous groups split at Z-order jumps).
//
// Exponent as a GEMM.  With x0 the centre of a group's box, u = x - x0, m = mu - x0 and
// c = -0.5 log2(e) * conic (so that the power arrives in base 2),
//   p2 = (u - m)^T c (u - m) = phi(u) . beta(m, c)
//   phi  = [ux^2, uy^2, uz^2, ux uy, ux uz, uy uz, ux, uy, uz, 1, 0 x 6]          (A: 128 x 16)
//   beta = [c00, c11, c22, 2c01, 2c02, 2c12, -2(cm)x, -2(cm)y, -2(cm)z, m^T c m, 0 x 6]
//                                                                             (B: 32 x 16)
// Every row belongs to exactly one group, so the A tile holds each row's phi relative to
// its own group's centre and is written once per CTA: the product of group g's batch with
// a row of another group is meaningless and is never read (that row is outside g).  Both
// operands are split into three BF16 parts (~24 bits); the six products with i + j <= 2
// are accumulated in FP32 (M = 128, N = 32, K = 16).  A column whose term bound
// sum_k |beta_k| max|phi_k| over the group exceeds kTcMaxTerm is evaluated in FP32 SIMT
// instead (the accumulation error grows with the terms, not with the result).
//
// Warps: 0..3 consumers (thread t owns row t and TMEM lane t), 4 stager, 5 finaliser.  The
// stager walks the Gaussian LBVH once per group with the group box (warp-cooperative
// traversal) and copies each batch of up to 32 candidate records into one of kStages
// stages with cp.async; the finaliser then computes the base-2 conic, the epilogue's
// column data (lo, w) and (hi, w v), per-consumer-warp column masks (box overlap with the
// warp's rows of the group), beta split into BF16 parts, and issues the six MMAs into the
// stage's 32 TMEM columns.  Splitting the two jobs over two warps keeps the traversal's
// load latency and the finalising arithmetic from serialising.  Consumers read their 32 columns 16 at a time and, for the columns of their
// mask, apply the exact AABB test, the power window and ex2 in FP32 and accumulate
// W and V in registers.  full[s] completes when the producer has staged s (arrive) and its
// MMAs are done (commit); empty[s] when the four consumer warps have read it.
//
// The window's upper end p <= 0 holds exactly for a positive definite conic; near the mean
// the split sum can exceed 0 by its rounding error, so powers up to kTcZeroTol count as
// 0 (e = 1) instead of dropping the pair.
#include "cta.cuh"
#include "tc.cuh"
#include "traverse.cuh"

// Batches in flight and resident CTAs per SM requested from the register allocator
// (measured at 2M x 16M: 2 stages at 6 CTAs per SM 23.7 ms, 4 stages at 4 CTAs 25.1 ms).
#ifndef GVC_FWD_TC_STAGES
#define GVC_FWD_TC_STAGES 2
#endif
#ifndef GVC_FWD_TC_MIN_BLOCKS
#define GVC_FWD_TC_MIN_BLOCKS 6
#endif

namespace gvc {

namespace {

constexpr int kStages = GVC_FWD_TC_STAGES;
constexpr int kBatch = 32;  // Gaussians per MMA (N)
constexpr int kMinBlocks = GVC_FWD_TC_MIN_BLOCKS;
constexpr float kTcMaxTerm = 256.0f;
constexpr float kTcZeroTol = 1.0f / 1024.0f;
constexpr float kHalfLog2eF = -0.72134752044448170368f;
constexpr float kLog2FloorF = -20.197570572173914f;

static_assert(tmem_cols_ok(kStages * kBatch), "TMEM columns must be a power of two >= 32");

struct __align__(1024) FwdTcSmem {
    unsigned char A[3][kBlockRows * 32];        // phi of every row, three BF16 parts
    unsigned char B[kStages][3][kBatch * 32];   // beta per stage, three BF16 parts
    float4 rec[kStages][kBatch][5];             // staged records; r1, r2 rewritten as the base-2 conic
    float4 colA[kStages][kBatch];               // (lo.x, lo.y, lo.z, w)
    float4 colB[kStages][kBatch];               // (hi.x, hi.y, hi.z, w v)
    uint32_t wmask[kStages][4];                 // columns overlapping consumer warp w's rows of the group
    uint32_t fbmask[kStages];                   // columns evaluated in FP32 SIMT
    int2 desc[kStages];                         // (columns, group) or (-1, 0) at the end
    int2 sdesc[kStages];                        // the same, from the stager to the finaliser
    int stack[kStackCap];
    int cand[kCandCap];
    uint64_t staged[kStages], full[kStages], empty[kStages];
    uint32_t tmem_base;
};

__device__ __forceinline__ float ex2f(float x) {
    float y;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

struct GroupGeom {
    float x0, y0, z0, ex, ey, ez;  // centre and half extents of the group box
};

__device__ __forceinline__ GroupGeom group_geom(const float4* bboxes, int64_t blk, int g) {
    const float4 lo = bboxes[2 * (blk * kBlockGroups + g)], hi = bboxes[2 * (blk * kBlockGroups + g) + 1];
    return GroupGeom{0.5f * (lo.x + hi.x), 0.5f * (lo.y + hi.y), 0.5f * (lo.z + hi.z),
                     0.5f * (hi.x - lo.x), 0.5f * (hi.y - lo.y), 0.5f * (hi.z - lo.z)};
}

// Warp 4: traversal visitor that copies each batch of up to 32 candidate records into the
// next stage with cp.async and publishes the previous batch once its copies have landed.
struct FwdTcStager {
    FwdTcSmem& sm;
    const GaussRec* __restrict__ recs;
    int* status;
    uint32_t total = 0;  // batches handed to stages
    bool pending = false;
    int pend_stage = 0, pend_nb = 0;
    int g = 0;
    bool failed = false;
    CandLog log;  // the block's candidates for the tensor-core backward (ids null: off)

    __device__ __forceinline__ bool acquire(uint32_t n) {
        const uint32_t k = n / kStages;
        if (k == 0) return true;
        return mbar_wait(&sm.empty[n % kStages], (k - 1) & 1u, status);
    }

    __device__ __forceinline__ void publish(int s, int nb) {
        const int lane = threadIdx.x & 31;
        __syncwarp();
        if (lane == 0) {
            sm.sdesc[s] = make_int2(nb, g);
            mbar_arrive(&sm.staged[s]);
        }
        __syncwarp();
    }

    __device__ __forceinline__ void flush() {
        if (pending) {
            cp_async_wait<0>();
            publish(pend_stage, pend_nb);
            pending = false;
        }
    }

    __device__ __forceinline__ void operator()(const int* c, int nb) {
        const int lane = threadIdx.x & 31;
        log.append(c, nb);
        if (failed || !acquire(total)) {
            failed = true;
            __syncwarp();
            return;
        }
        const int s = (int)(total % kStages);
        if (lane < nb) {
            const float4* src = reinterpret_cast<const float4*>(recs + c[lane]);
#pragma unroll
            for (int q = 0; q < 5; q++) cp_async16(&sm.rec[s][lane][q], src + q);
        }
        cp_async_commit();
        if (pending) {
            cp_async_wait<1>();
            publish(pend_stage, pend_nb);
        }
        pending = true;
        pend_stage = s;
        pend_nb = nb;
        total++;
        __syncwarp();
    }
};

// Warp 5: per staged batch, the base-2 conic, the epilogue's columns, the consumer warps'
// column masks, beta split into BF16 parts, and the six MMAs into the stage's TMEM columns.
struct FwdTcFinaliser {
    FwdTcSmem& sm;
    uint32_t tmem;
    GroupGeom geo{};
    Box6 wb[4];  // boxes of the group's rows of each consumer warp (same on every lane)

    __device__ __forceinline__ void set_group(const float4* __restrict__ s_sorted, int64_t S,
                                              const float4* __restrict__ bboxes, int64_t blk, uint2 bd, int g) {
        const int lane = threadIdx.x & 31;
        const int ra = group_start(bd, g), rb = group_start(bd, g + 1);
        geo = group_geom(bboxes, blk, g);
#pragma unroll
        for (int q = 0; q < 4; q++) {
            const int r = 32 * q + lane;
            const int64_t rr = blk * kBlockRows + r;
            const bool in = rr < S && r >= ra && r < rb;
            float4 p = make_float4(0.f, 0.f, 0.f, 0.f);
            if (in) p = s_sorted[rr];
            wb[q] = warp_box6(in, p.x, p.y, p.z);
        }
    }

    __device__ __forceinline__ void finalize(int s, int nb, int g) {
        const int lane = threadIdx.x & 31;
        const bool live = lane < nb;
        float4 r0 = make_float4(0.f, 0.f, 0.f, 0.f), r1 = r0, r2 = r0, lo = r0, hi = r0;
        if (live) {
            r0 = sm.rec[s][lane][0];
            r1 = sm.rec[s][lane][1];
            r2 = sm.rec[s][lane][2];
            lo = sm.rec[s][lane][3];
            hi = sm.rec[s][lane][4];
        }
        const float c0 = kHalfLog2eF * r1.x, c1 = kHalfLog2eF * r1.y, c2 = kHalfLog2eF * r1.z,
                    c3 = kHalfLog2eF * r1.w, c4 = kHalfLog2eF * r2.x, c5 = kHalfLog2eF * r2.y;
        uint32_t wm[4];
#pragma unroll
        for (int q = 0; q < 4; q++) wm[q] = __ballot_sync(0xffffffffu, live && overlap6(wb[q], lo, hi));
        const float mx = r0.x - geo.x0, my = r0.y - geo.y0, mz = r0.z - geo.z0;
        const float cmx = c0 * mx + c1 * my + c2 * mz;
        const float cmy = c1 * mx + c3 * my + c4 * mz;
        const float cmz = c2 * mx + c4 * my + c5 * mz;
        float beta[10];
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
        const float bound = fabsf(beta[0]) * geo.ex * geo.ex + fabsf(beta[1]) * geo.ey * geo.ey +
                            fabsf(beta[2]) * geo.ez * geo.ez + fabsf(beta[3]) * geo.ex * geo.ey +
                            fabsf(beta[4]) * geo.ex * geo.ez + fabsf(beta[5]) * geo.ey * geo.ez +
                            fabsf(beta[6]) * geo.ex + fabsf(beta[7]) * geo.ey + fabsf(beta[8]) * geo.ez +
                            fabsf(beta[9]);
        const uint32_t fb = __ballot_sync(0xffffffffu, live && !(bound <= kTcMaxTerm));
        if (live) {
            // the SIMT fallback's coefficients (off-diagonals doubled) and the epilogue's columns
            sm.rec[s][lane][1] = make_float4(c0, 2.f * c1, 2.f * c2, c3);
            sm.rec[s][lane][2] = make_float4(2.f * c4, c5, r2.z, 0.f);
            sm.colA[s][lane] = make_float4(lo.x, lo.y, lo.z, r0.w);
            sm.colB[s][lane] = make_float4(hi.x, hi.y, hi.z, r0.w * r2.z);
            store_features10(sm.B[s][0], sm.B[s][1], sm.B[s][2], lane, beta);
        }
        if (lane == 0) {
#pragma unroll
            for (int q = 0; q < 4; q++) sm.wmask[s][q] = wm[q];
            sm.fbmask[s] = fb;
            sm.desc[s] = make_int2(nb, g);
        }
        fence_proxy_async_smem();
        __syncwarp();
        if (lane == 0) {
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
            mbar_arrive(&sm.full[s]);
        }
        __syncwarp();
    }
};

}  // namespace

template <bool COUNT, bool STACKLESS>
__global__ void __launch_bounds__(192, kMinBlocks)
    k_forward_tc(const float4* __restrict__ s_sorted, int64_t S, const uint2* __restrict__ bdesc,
                 const float4* __restrict__ bboxes, const BvhNode* __restrict__ nodes, int64_t n_internal,
                 const GaussRec* __restrict__ recs, float* __restrict__ out_cells, float* __restrict__ out_weights,
                 int32_t* __restrict__ clog, int32_t* __restrict__ cend, int* status, unsigned long long* stats) {
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    FwdTcSmem& sm = *reinterpret_cast<FwdTcSmem*>(
        smem_raw + ((1024 - (static_cast<uint32_t>(__cvta_generic_to_shared(smem_raw)) & 1023)) & 1023));
    const int t = threadIdx.x, w = t >> 5, lane = t & 31;
    const int64_t blk = blockIdx.x;
    const uint2 bd = bdesc[blk];
    const int ng = group_count(bd);

    if (t == 0) {
        for (int s = 0; s < kStages; s++) {
            mbar_init(&sm.staged[s], 1);
            mbar_init(&sm.full[s], 2);
            mbar_init(&sm.empty[s], 4);
        }
        fence_mbar_init();
    }
    // features 10..15 of every operand row stay zero
    for (int i = t; i < (int)((sizeof(sm.A) + sizeof(sm.B)) / sizeof(uint4)); i += 192)
        reinterpret_cast<uint4*>(&sm.A[0][0])[i] = make_uint4(0u, 0u, 0u, 0u);
    __syncthreads();
    // consumer thread t: its row's phi relative to the centre of its own group
    const int64_t row = blk * kBlockRows + t;
    float x = NAN, y = NAN, z = NAN;
    int orig = -1;
    int my_group = -1;
    if (w < 4) {
        if (row < S) {
            const float4 p = s_sorted[row];
            x = p.x;
            y = p.y;
            z = p.z;
            orig = __float_as_int(p.w);
            my_group = group_of(bd, t);
        }
        float f[10] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
        if (my_group >= 0) {
            const GroupGeom gg = group_geom(bboxes, blk, my_group);
            const float ux = x - gg.x0, uy = y - gg.y0, uz = z - gg.z0;
            f[0] = ux * ux;
            f[1] = uy * uy;
            f[2] = uz * uz;
            f[3] = ux * uy;
            f[4] = ux * uz;
            f[5] = uy * uz;
            f[6] = ux;
            f[7] = uy;
            f[8] = uz;
            f[9] = 1.f;
        }
        store_features10(sm.A[0], sm.A[1], sm.A[2], t, f);
    }
    if (w == 0) {
        tmem_alloc(&sm.tmem_base, kStages * kBatch);
        tmem_relinquish();
    }
    fence_proxy_async_smem();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = sm.tmem_base;

    if (w == 4) {
        // ---------------- stager: traversal and record copies ----------------
        FwdTcStager sg{sm, recs, status};
        if (clog) sg.log.ids = clog + blk * kCandLogPerBlock;
        TravCount tc;
        int st = 0;
        for (int g = 0; g < ng && !sg.failed; g++) {
            sg.flush();  // the pending batch belongs to the previous group
            sg.g = g;
            const float4 glo = bboxes[2 * (blk * kBlockGroups + g)], ghi = bboxes[2 * (blk * kBlockGroups + g) + 1];
            st |= warp_traverse_sel<STACKLESS>(nodes, n_internal, make_float3(glo.x, glo.y, glo.z),
                                               make_float3(ghi.x, ghi.y, ghi.z), sm.stack, sm.cand, sg, tc);
            sg.log.end_group(g);
        }
        if (sg.failed || st) sg.log.over = true;
        if (clog) sg.log.finish(cend + blk * kBlockGroups, ng);
        sg.flush();
        if (st && lane == 0) atomicOr(status, st);
        if (!sg.failed && sg.acquire(sg.total)) {
            const int s = (int)(sg.total % kStages);
            if (lane == 0) {
                sm.sdesc[s] = make_int2(-1, 0);
                mbar_arrive(&sm.staged[s]);
            }
        }
        __syncwarp();
        if (COUNT && lane == 0) {
            atomicMax(&stats[3], (unsigned long long)tc.max_sp);
            atomicAdd(&stats[5], (unsigned long long)tc.leaves);
            atomicAdd(&stats[6], (unsigned long long)tc.nodes);
        }
    } else if (w == 5) {
        // ---------------- finaliser: coefficients, masks, MMAs ----------------
        FwdTcFinaliser fz{sm, tmem};
        int cur = -1;
        for (uint32_t n = 0;; n++) {
            const int s = (int)(n % kStages);
            const bool ok = mbar_wait(&sm.staged[s], (n / kStages) & 1u, status);
            if (!__all_sync(0xffffffffu, ok)) break;
            const int2 d = sm.sdesc[s];
            if (d.x < 0) {
                if (lane == 0) {
                    sm.desc[s] = make_int2(-1, 0);
                    mbar_arrive(&sm.full[s]);
                    mbar_arrive(&sm.full[s]);
                }
                __syncwarp();
                break;
            }
            if (d.y != cur) {
                cur = d.y;
                fz.set_group(s_sorted, S, bboxes, blk, bd, cur);
            }
            fz.finalize(s, d.x, d.y);
        }
    } else {
        // ---------------- consumers: thread t owns row t ----------------
        float W = 0.f, V = 0.f;
        long long ncand = 0, ncontrib = 0, nlane = 0;
        const uint32_t lane_base = tmem + ((uint32_t)(32 * w) << 16);
        for (uint32_t n = 0;; n++) {
            const int s = (int)(n % kStages);
            const bool ok = mbar_wait(&sm.full[s], (n / kStages) & 1u, status);
            if (!__all_sync(0xffffffffu, ok)) break;
            const int2 d = sm.desc[s];
            if (d.x < 0) break;
            const bool ing = my_group == d.y;
            const uint32_t wm = sm.wmask[s][w];
            const uint32_t fb = sm.fbmask[s] & wm;
            const uint32_t tm = wm & ~fb;
            if (COUNT) nlane += 32 * __popc(wm);
            tc_fence_after();
#pragma unroll
            for (int h = 0; h < 2; h++) {
                const uint32_t m16 = (tm >> (16 * h)) & 0xffffu;
                if (m16 == 0u) continue;  // warp-uniform
                float v[16];
                tmem_ld16(lane_base + (uint32_t)(s * kBatch + 16 * h), v);
#pragma unroll
                for (int j = 0; j < 16; j++) {
                    if (!((m16 >> j) & 1u)) continue;
                    const float p2 = v[j];
                    const bool win = ing && p2 >= kLog2FloorF && p2 <= kTcZeroTol;
                    // the window needs no column data: a column none of whose rows in this
                    // warp is in it contributes nothing here, box test or not
                    if (!COUNT && !__any_sync(0xffffffffu, win)) continue;
                    const float4 a = sm.colA[s][16 * h + j], b = sm.colB[s][16 * h + j];
                    const bool in = ing && a.x <= x && x <= b.x && a.y <= y && y <= b.y && a.z <= z && z <= b.z;
                    const bool c = in && win;
                    const float e = c ? ex2f(fminf(p2, 0.f)) : 0.f;
                    W = fmaf(a.w, e, W);
                    V = fmaf(b.w, e, V);
                    if (COUNT) {
                        ncand += in ? 1 : 0;
                        ncontrib += c ? 1 : 0;
                    }
                }
            }
            // columns whose terms are too large for the split accumulation: FP32 SIMT
            uint32_t f = fb;
            while (f) {
                const int j = __ffs(f) - 1;
                f &= f - 1;
                const float4 a = sm.colA[s][j], b = sm.colB[s][j];
                const float4 r0 = sm.rec[s][j][0], r1 = sm.rec[s][j][1], r2 = sm.rec[s][j][2];
                const bool in = ing && a.x <= x && x <= b.x && a.y <= y && y <= b.y && a.z <= z && z <= b.z;
                const float dx = x - r0.x, dy = y - r0.y, dz = z - r0.z;
                const float p2 = dx * fmaf(r1.x, dx, fmaf(r1.y, dy, r1.z * dz)) + dy * fmaf(r1.w, dy, r2.x * dz) +
                                 dz * (r2.y * dz);
                const bool c = in && p2 >= kLog2FloorF && p2 <= 0.0f;
                const float e = c ? ex2f(p2) : 0.f;
                W = fmaf(a.w, e, W);
                V = fmaf(b.w, e, V);
                if (COUNT) {
                    ncand += in ? 1 : 0;
                    ncontrib += c ? 1 : 0;
                }
            }
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(&sm.empty[s]);
        }
        if (row < S) {
            float o, ww;
            if (W <= kWeightCutoff) {
                o = -1.0f;
                ww = 0.0f;
            } else {
                o = V / W;
                ww = W;
            }
            out_cells[orig] = o;
            out_weights[orig] = ww;
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
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (w == 0) tmem_dealloc(tmem, kStages * kBatch);
}

template <bool COUNT, bool STACKLESS>
static cudaError_t launch_fwd_tc_impl(const CtaArgs& a, cudaStream_t st) {
    const size_t smem = sizeof(FwdTcSmem) + 1024;
    cudaError_t e =
        cudaFuncSetAttribute(k_forward_tc<COUNT, STACKLESS>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    const unsigned nb = (unsigned)((a.S + kBlockRows - 1) / kBlockRows);
    k_forward_tc<COUNT, STACKLESS><<<nb, 192, smem, st>>>(a.s_sorted, a.S, a.bdesc, a.bboxes, a.gnodes, a.n_internal,
                                                          a.recs, a.out_cells, a.out_weights, a.clog, a.cend,
                                                          a.status, a.stats);
    gvc::note_launch();
    return cudaGetLastError();
}

cudaError_t launch_forward_tc(const CtaArgs& a, cudaStream_t st) {
    if (a.S <= 0) return cudaSuccess;
    if (a.stackless) return a.count ? launch_fwd_tc_impl<true, true>(a, st) : launch_fwd_tc_impl<false, true>(a, st);
    return a.count ? launch_fwd_tc_impl<true, false>(a, st) : launch_fwd_tc_impl<false, false>(a, st);
}

}  // namespace gvc
