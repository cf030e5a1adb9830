// render.cu -- fused traversal + Gaussian evaluation (forward) and the adjoint
// (backward) of the mixture field at Morton-sorted sample tiles.
//
// Forward (replaces FORWARD::sampleRenderCUDA / renderCUDA + normalizeCUDA,
// diff-gaussian-rasterization/cuda_rasterizer/forward.cu:116-274): one warp per tile of
// 32 Morton-sorted samples walks the Gaussian LBVH with the tile's box; candidate
// Gaussians are staged 32 at a time in shared memory and every lane evaluates its own
// sample against each of them, accumulating W and V in registers (no atomics).
//
// Backward, deterministic (replaces BACKWARD::renderCUDA, backward.cu:127-337): one
// warp per Gaussian walks the sample-group LBVH with the Gaussian's AABB; the rows of the
// candidate groups are packed densely onto the lanes; per-lane partial moments are
// reduced once per Gaussian (a fixed-order segmented reduction, no atomics).
//
// Backward, atomic (replaces BACKWARD::sampleRenderCUDA, backward.cu:339-559): one warp
// per sample tile re-walks the Gaussian LBVH; the 11 per-pair terms are pre-reduced over
// the tile with 16 shuffles and added with one FP32 atomic per field and Gaussian.
//
// Pair math follows forward.cu:224-256 and backward.cu:252-298; the per-sample factors
// 1/W, -out/W are folded into the sample record once per sample.
#include "pair.cuh"
#include "render.cuh"
#include "traverse.cuh"

namespace gvc {

constexpr int kWarpsPerBlock = 4;

// --------------------------------------------------------------------------------
// Forward
// --------------------------------------------------------------------------------
template <bool COUNT>
struct FwdVisitor {
    const GaussRec* __restrict__ recs;
    float4* batch;  // shared [32 * 5]
    float x, y, z;
    bool valid;
    float W, V;
    int ncand, ncontrib;

    __device__ __forceinline__ void operator()(const int* c, int nb) {
        const int lane = threadIdx.x & 31;
        if (lane < nb) {
            // stage one record per lane; the conic becomes base-2 power coefficients with
            // the off-diagonal entries doubled (symmetric quadratic form in 9 operations)
            const float4* rp = reinterpret_cast<const float4*>(recs + c[lane]);
            const float4 r0 = __ldg(rp), r1 = __ldg(rp + 1), r2 = __ldg(rp + 2), r3 = __ldg(rp + 3),
                         r4 = __ldg(rp + 4);
            batch[lane * 5 + 0] = r0;
            batch[lane * 5 + 1] = make_float4(kHalfLog2e * r1.x, 2.f * kHalfLog2e * r1.y, 2.f * kHalfLog2e * r1.z,
                                              kHalfLog2e * r1.w);
            batch[lane * 5 + 2] = make_float4(2.f * kHalfLog2e * r2.x, kHalfLog2e * r2.y, r2.z, 0.f);
            batch[lane * 5 + 3] = r3;
            batch[lane * 5 + 4] = r4;
        }
        __syncwarp();
        // Four Gaussians per step, branch-free inside the step: four independent
        // dependency chains per lane; a step is skipped only when no lane of the warp is
        // inside any of the four boxes.
        for (int g0 = 0; g0 < nb; g0 += 4) {
            bool in[4];
#pragma unroll
            for (int j = 0; j < 4; j++) {
                const int g = g0 + j;
                in[j] = false;
                if (g < nb) {
                    const float4 r3 = batch[g * 5 + 3], r4 = batch[g * 5 + 4];
                    in[j] = valid && r3.x <= x && x <= r4.x && r3.y <= y && y <= r4.y && r3.z <= z && z <= r4.z;
                }
            }
            if (!__any_sync(0xffffffffu, in[0] | in[1] | in[2] | in[3])) continue;
#pragma unroll
            for (int j = 0; j < 4; j++) {
                const int g = min(g0 + j, nb - 1);
                const float4 r0 = batch[g * 5 + 0], r1 = batch[g * 5 + 1], r2 = batch[g * 5 + 2];
                const float dx = x - r0.x, dy = y - r0.y, dz = z - r0.z;
                const float p2 = dx * fmaf(r1.x, dx, fmaf(r1.y, dy, r1.z * dz)) + dy * fmaf(r1.w, dy, r2.x * dz) +
                                 dz * (r2.y * dz);
                const bool c = in[j] && p2 >= kLog2Floor && p2 <= 0.0f;
                const float wt = c ? r0.w * ex2_approx(p2) : 0.0f;
                W += wt;
                V = fmaf(wt, r2.z, V);
                if (COUNT) {
                    ncand += in[j] ? 1 : 0;
                    ncontrib += c ? 1 : 0;
                }
            }
        }
        __syncwarp();
    }
};

// Lane group of this lane in a tile with descriptor gd (see k_sample_tiles).
__device__ __forceinline__ int lane_group(uint32_t gd, int lane) {
    return (lane >= (int)(gd & 0xffu)) + (lane >= (int)((gd >> 8) & 0xffu)) + (lane >= (int)((gd >> 16) & 0xffu));
}

template <bool COUNT>
__global__ void __launch_bounds__(kWarpsPerBlock * 32) k_forward(const float4* __restrict__ s_sorted,
                                                                 const float4* __restrict__ group_boxes,
                                                                 const uint32_t* __restrict__ gdesc, int n_tiles,
                                                                 const BvhNode* __restrict__ nodes,
                                                                 const GaussRec* __restrict__ recs,
                                                                 float* __restrict__ out_cells,
                                                                 float* __restrict__ out_weights, int* status,
                                                                 unsigned long long* stats) {
    __shared__ int s_stack[kWarpsPerBlock][kStackCap];
    __shared__ int s_cand[kWarpsPerBlock][kCandCap];
    __shared__ float4 s_batch[kWarpsPerBlock][32 * 5];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int tile = blockIdx.x * kWarpsPerBlock + warp;
    if (tile >= n_tiles) return;
    const float4 sp = s_sorted[(int64_t)tile * 32 + lane];
    const int orig = __float_as_int(sp.w);
    const uint32_t gd = gdesc[tile];
    const int ng = (int)(gd >> 24), mygroup = lane_group(gd, lane);
    FwdVisitor<COUNT> vis{recs, s_batch[warp], sp.x, sp.y, sp.z, false, 0.f, 0.f, 0, 0};
    TravCount tc;
    int st = 0;
    for (int g = 0; g < ng; g++) {
        const int64_t slot = (int64_t)tile * kGroups + g;
        const float4 tlo = group_boxes[2 * slot], thi = group_boxes[2 * slot + 1];
        vis.valid = orig >= 0 && mygroup == g;
        st |= warp_traverse(nodes, make_float3(tlo.x, tlo.y, tlo.z), make_float3(thi.x, thi.y, thi.z),
                            s_stack[warp], s_cand[warp], vis, tc);
    }
    if (orig >= 0) {
        float o, w;
        if (vis.W <= kWeightCutoff) {
            o = -1.0f;
            w = 0.0f;
        } else {
            o = vis.V / vis.W;
            w = vis.W;
        }
        out_cells[orig] = o;
        out_weights[orig] = w;
    }
    if (st && lane == 0) atomicOr(status, st);
    if (COUNT) {
        unsigned long long a = (unsigned long long)vis.ncand, b = (unsigned long long)vis.ncontrib;
        for (int off = 16; off > 0; off >>= 1) {
            a += __shfl_xor_sync(0xffffffffu, a, off);
            b += __shfl_xor_sync(0xffffffffu, b, off);
        }
        if (lane == 0) {
            atomicAdd(&stats[0], a);
            atomicAdd(&stats[1], b);
            atomicMax(&stats[3], (unsigned long long)tc.max_sp);
            atomicAdd(&stats[5], (unsigned long long)tc.leaves);
            atomicAdd(&stats[6], (unsigned long long)tc.nodes);
        }
    }
}

// --------------------------------------------------------------------------------
// Backward, deterministic Gaussian-owned reduction with densely packed sample rows.
// --------------------------------------------------------------------------------
// A candidate leaf is one lane group of a sample tile (rows [start, end) of the tile).
// Groups hold 1..32 rows, so mapping lanes to a group's rows leaves lanes idle; instead
// the rows of successive candidate groups are appended to a per-warp ring and evaluated
// kFlush at a time (kRowsPerLane rows per lane, all loads issued before the arithmetic:
// the kernel is bound by the latency of these gathers).  The order in which rows reach
// lanes depends only on the traversal order, so the sums are deterministic.
constexpr int kRowsPerLane = 2;
constexpr int kFlush = 32 * kRowsPerLane;  // rows per evaluation
constexpr int kRing = 2 * kFlush;          // queued rows stay below kFlush + 32

template <bool COUNT>
struct BwdDenseVisitor {
    const float4* __restrict__ s_grad;
    const float* __restrict__ s_gyz;
    const uint8_t* __restrict__ s_ok;
    const uint32_t* __restrict__ gdesc;
    int* ring;     // shared [kRing]
    int4* leaves;  // shared [32]: (first slot of tile, start lane, end lane, rows queued through this leaf)
    uint32_t head, tail;
    GaussB g;
    float m[11];
    int npairs;
    int nrows;  // rows evaluated (warp-uniform, statistics)

    // evaluates the n (1..kFlush) rows at the ring head
    __device__ __forceinline__ void eval(int n) {
        const int lane = threadIdx.x & 31;
        float4 p[kRowsPerLane];
        float y[kRowsPerLane];
        int r[kRowsPerLane];
#pragma unroll
        for (int k = 0; k < kRowsPerLane; k++) {
            p[k] = make_float4(0.f, 0.f, 0.f, 0.f);
            y[k] = 0.f;
            r[k] = -1;
            if (lane + 32 * k < n) {
                r[k] = ring[(head + (uint32_t)(32 * k + lane)) & (kRing - 1)];
                p[k] = __ldg(s_grad + r[k]);
                y[k] = __ldg(s_gyz + r[k]);
            }
        }
#pragma unroll
        for (int k = 0; k < kRowsPerLane; k++) {
            if (32 * k < n) {
                const bool c = pair_moments(g, p[k], y[k], m);
                if (COUNT && c && r[k] >= 0 && s_ok[r[k]]) npairs++;
            }
        }
        if (COUNT) nrows += n;
        head += (uint32_t)n;
    }

    __device__ __forceinline__ void operator()(const int* c, int nb) {
        const int lane = threadIdx.x & 31;
        int sz = 0;
        int4 L = make_int4(0, 0, 0, 0);
        if (lane < nb) {
            const int leaf = c[lane];
            const int t = leaf >> 2;  // leaf = tile * kGroups + group
            const int gi = leaf & 3;
            const uint32_t gd = __ldg(gdesc + t);
            const int start = gi == 0 ? 0 : (int)((gd >> (8 * (gi - 1))) & 0xffu);
            const int end = gi < 3 ? (int)((gd >> (8 * gi)) & 0xffu) : 32;
            sz = end - start;
            L = make_int4(t * 32, start, end, 0);
        }
        int incl = sz;
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
            const int v = __shfl_up_sync(0xffffffffu, incl, off);
            if (lane >= off) incl += v;
        }
        L.w = incl;
        leaves[lane] = L;
        __syncwarp();
        const uint32_t base = tail;
        for (int j = 0; j < nb; j++) {
            const int4 q = leaves[j];
            const int excl = q.w - (q.z - q.y);
            if (lane >= q.y && lane < q.z) ring[(base + (uint32_t)(excl + lane - q.y)) & (kRing - 1)] = q.x + lane;
            if (base + (uint32_t)q.w - head >= (uint32_t)kFlush) {
                __syncwarp();
                eval(kFlush);
            }
        }
        tail = base + (uint32_t)__shfl_sync(0xffffffffu, incl, 31);
        __syncwarp();
    }

    __device__ __forceinline__ void drain() {
        while (tail != head) {
            __syncwarp();
            const uint32_t n = tail - head;
            eval(n < (uint32_t)kFlush ? (int)n : kFlush);
        }
        __syncwarp();
    }
};

// Warps (consecutive Gaussians in Morton order) per block: neighbouring Gaussians gather
// overlapping sample rows, which then hit in the SM's L1.
constexpr int kBwdWarps = 4;

template <bool COUNT>
__global__ void __launch_bounds__(kBwdWarps * 32) k_backward_gauss(
    int P, const int32_t* __restrict__ gorder, const float* __restrict__ means, const float* __restrict__ values,
    const float* __restrict__ weights, const float* __restrict__ conics, const float4* __restrict__ boxes,
    const float4* __restrict__ s_grad, const float* __restrict__ s_gyz, const uint8_t* __restrict__ s_ok,
    const uint32_t* __restrict__ gdesc, const BvhNode* __restrict__ tnodes, float* __restrict__ gacc, int* status,
    unsigned long long* stats) {
    __shared__ int s_stack[kBwdWarps][kStackCap];
    __shared__ int s_cand[kBwdWarps][kCandCap];
    __shared__ int s_ring[kBwdWarps][kRing];
    __shared__ int4 s_leaves[kBwdWarps][32];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int gi = blockIdx.x * kBwdWarps + warp;
    if (gi >= P) return;
    const int64_t o = gorder ? gorder[gi] : gi;
    BwdDenseVisitor<COUNT> vis;
    vis.s_grad = s_grad;
    vis.s_gyz = s_gyz;
    vis.s_ok = s_ok;
    vis.gdesc = gdesc;
    vis.ring = s_ring[warp];
    vis.leaves = s_leaves[warp];
    vis.head = vis.tail = 0u;
    const float* cp = conics + 6 * o;
    const float4 lo = __ldg(boxes + 2 * o), hi = __ldg(boxes + 2 * o + 1);
    vis.g = gauss_b(__ldg(means + 3 * o), __ldg(means + 3 * o + 1), __ldg(means + 3 * o + 2), __ldg(values + o),
                    __ldg(cp), __ldg(cp + 1), __ldg(cp + 2), __ldg(cp + 3), __ldg(cp + 4), __ldg(cp + 5), lo, hi);
#pragma unroll
    for (int k = 0; k < 11; k++) vis.m[k] = 0.f;
    vis.npairs = 0;
    vis.nrows = 0;
    TravCount tc;
    const int st = warp_traverse(tnodes, make_float3(lo.x, lo.y, lo.z), make_float3(hi.x, hi.y, hi.z), s_stack[warp],
                                 s_cand[warp], vis, tc);
    vis.drain();
    float v16[16];
#pragma unroll
    for (int k = 0; k < 16; k++) v16[k] = k < 11 ? vis.m[k] : 0.f;
    const float tot = warp_transpose_reduce16(v16);
    const float term = moments_to_terms(tot, __ldg(weights + o), __ldg(cp), __ldg(cp + 1), __ldg(cp + 2),
                                        __ldg(cp + 3), __ldg(cp + 4), __ldg(cp + 5));
    if (!(lane & 1)) gacc[16 * o + (lane >> 1)] = term;
    if (st && lane == 0) atomicOr(status, st);
    if (COUNT) {
        unsigned long long a = (unsigned long long)vis.npairs;
        for (int off = 16; off > 0; off >>= 1) a += __shfl_xor_sync(0xffffffffu, a, off);
        if (lane == 0) {
            atomicAdd(&stats[2], a);
            atomicMax(&stats[4], (unsigned long long)tc.max_sp);
            atomicAdd(&stats[7], (unsigned long long)tc.leaves);
            atomicAdd(&stats[8], (unsigned long long)tc.nodes);
            atomicAdd(&stats[10], (unsigned long long)vis.nrows);
        }
    }
}

// --------------------------------------------------------------------------------
// Backward, sample-tile traversal with warp pre-reduction + FP32 atomics.
// --------------------------------------------------------------------------------
struct BwdTileVisitor {
    const GaussRec* __restrict__ recs;
    const int32_t* __restrict__ gperm;
    float4* batch;  // shared [32 * 5]
    float4 p;       // (x, y, z, gx); gx = 0 outside the current group
    float gyz;      // 0 outside the current group
    bool act;       // lane in the current group
    bool ok;
    float* __restrict__ gacc;
    int npairs;

    __device__ __forceinline__ void operator()(const int* c, int nb) {
        const int lane = threadIdx.x & 31;
        if (lane < nb) {
            const float4* rp = reinterpret_cast<const float4*>(recs + c[lane]);
            batch[lane * 5 + 0] = __ldg(rp);
            batch[lane * 5 + 1] = __ldg(rp + 1);
            batch[lane * 5 + 2] = __ldg(rp + 2);
            batch[lane * 5 + 3] = __ldg(rp + 3);
            batch[lane * 5 + 4] = __ldg(rp + 4);
        }
        __syncwarp();
        for (int gi = 0; gi < nb; gi++) {
            const float4 r0 = batch[gi * 5 + 0], r1 = batch[gi * 5 + 1], r2 = batch[gi * 5 + 2];
            const GaussB g = gauss_b(r0.x, r0.y, r0.z, r2.z, r1.x, r1.y, r1.z, r1.w, r2.x, r2.y, batch[gi * 5 + 3],
                                     batch[gi * 5 + 4]);
            float m[11];
#pragma unroll
            for (int k = 0; k < 11; k++) m[k] = 0.f;
            const bool hit = pair_moments(g, p, gyz, m) && act;
            if (!__any_sync(0xffffffffu, hit)) continue;
            npairs += (hit && ok) ? 1 : 0;
            float v16[16];
#pragma unroll
            for (int k = 0; k < 16; k++) v16[k] = k < 11 ? m[k] : 0.f;
            const float tot = warp_transpose_reduce16(v16);
            const float term = moments_to_terms(tot, r0.w, r1.x, r1.y, r1.z, r1.w, r2.x, r2.y);
            const int k = lane >> 1;
            if (!(lane & 1) && k < 11) {
                const int o = gperm[c[gi]];
                atomicAdd(gacc + 16 * (int64_t)o + k, term);
            }
        }
        __syncwarp();
    }
};

template <bool COUNT>
__global__ void __launch_bounds__(kWarpsPerBlock * 32) k_backward_tiles(
    const float4* __restrict__ s_grad, const float* __restrict__ s_gyz, const uint8_t* __restrict__ s_ok,
    const float4* __restrict__ group_boxes, const uint32_t* __restrict__ gdesc, int n_tiles,
    const BvhNode* __restrict__ gnodes, const GaussRec* __restrict__ recs, const int32_t* __restrict__ gperm,
    float* __restrict__ gacc, int* status, unsigned long long* stats) {
    __shared__ int s_stack[kWarpsPerBlock][kStackCap];
    __shared__ int s_cand[kWarpsPerBlock][kCandCap];
    __shared__ float4 s_batch[kWarpsPerBlock][32 * 5];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int tile = blockIdx.x * kWarpsPerBlock + warp;
    if (tile >= n_tiles) return;
    BwdTileVisitor vis;
    vis.recs = recs;
    vis.gperm = gperm;
    vis.batch = s_batch[warp];
    const int64_t slot = (int64_t)tile * 32 + lane;
    const float4 sp = s_grad[slot];
    const float syz = s_gyz[slot];
    vis.ok = s_ok[slot] != 0;
    vis.gacc = gacc;
    vis.npairs = 0;
    const uint32_t gd = gdesc[tile];
    const int ng = (int)(gd >> 24), mygroup = lane_group(gd, lane);
    TravCount tc;
    int st = 0;
    for (int g = 0; g < ng; g++) {
        const int64_t gslot = (int64_t)tile * kGroups + g;
        const float4 tlo = group_boxes[2 * gslot], thi = group_boxes[2 * gslot + 1];
        // lanes outside the group carry zero gradients and are not counted
        vis.act = mygroup == g;
        vis.p = make_float4(sp.x, sp.y, sp.z, vis.act ? sp.w : 0.f);
        vis.gyz = vis.act ? syz : 0.f;
        st |= warp_traverse(gnodes, make_float3(tlo.x, tlo.y, tlo.z), make_float3(thi.x, thi.y, thi.z),
                            s_stack[warp], s_cand[warp], vis, tc);
    }
    if (st && lane == 0) atomicOr(status, st);
    if (COUNT) {
        unsigned long long a = (unsigned long long)vis.npairs;
        for (int off = 16; off > 0; off >>= 1) a += __shfl_xor_sync(0xffffffffu, a, off);
        if (lane == 0) {
            atomicAdd(&stats[2], a);
            atomicMax(&stats[4], (unsigned long long)tc.max_sp);
            atomicAdd(&stats[7], (unsigned long long)tc.leaves);
            atomicAdd(&stats[8], (unsigned long long)tc.nodes);
        }
    }
}

// --------------------------------------------------------------------------------
// Finalize: gacc [P][16] (caller order) -> dmeans, dvalues, dweights and the
// covariance adjoint dconic -> dscales, drots (one thread per Gaussian).
// --------------------------------------------------------------------------------
__device__ __forceinline__ void rot_cols(float r, float x, float y, float z, float Rc[3][3]) {
    // Rc[col][row]: glm's column-major fill of forward.cu:40-44
    Rc[0][0] = 1.f - 2.f * (y * y + z * z);
    Rc[0][1] = 2.f * (x * y - r * z);
    Rc[0][2] = 2.f * (x * z + r * y);
    Rc[1][0] = 2.f * (x * y + r * z);
    Rc[1][1] = 1.f - 2.f * (x * x + z * z);
    Rc[1][2] = 2.f * (y * z - r * x);
    Rc[2][0] = 2.f * (x * z - r * y);
    Rc[2][1] = 2.f * (y * z + r * x);
    Rc[2][2] = 1.f - 2.f * (x * x + y * y);
}

// True gradient of conic = inv(Sigma + eps I), Sigma = M^T M, M = diag(s) Rg.
__device__ void cov_adjoint_true(const float s_in[3], const float q[4], float sm, const float c6[6],
                                 const float u[6], float ds[3], float dq[4]) {
    float Rc[3][3];
    rot_cols(q[0], q[1], q[2], q[3], Rc);
    float Rg[3][3];  // Rg[i][j] = row i, col j
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) Rg[i][j] = Rc[j][i];
    const float sv[3] = {sm * s_in[0], sm * s_in[1], sm * s_in[2]};
    float M[3][3];
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) M[i][j] = sv[i] * Rg[i][j];
    float Sd[3];
    for (int i = 0; i < 3; i++) Sd[i] = M[0][i] * M[0][i] + M[1][i] * M[1][i] + M[2][i] * M[2][i];
    const float C[3][3] = {{c6[0], c6[1], c6[2]}, {c6[1], c6[3], c6[4]}, {c6[2], c6[4], c6[5]}};
    const float G[3][3] = {{u[0], 0.5f * u[1], 0.5f * u[2]}, {0.5f * u[1], u[3], 0.5f * u[4]}, {0.5f * u[2], 0.5f * u[4], u[5]}};
    float T[3][3], H[3][3];
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) T[i][j] = G[i][0] * C[0][j] + G[i][1] * C[1][j] + G[i][2] * C[2][j];
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) H[i][j] = -(C[i][0] * T[0][j] + C[i][1] * T[1][j] + C[i][2] * T[2][j]);
    const float a0 = fabsf(Sd[0]), a1 = fabsf(Sd[1]), a2 = fabsf(Sd[2]);
    int kmax = 0;
    if (a1 > a0) kmax = 1;
    if (a2 > (kmax == 0 ? a0 : a1)) kmax = 2;
    const float trH = H[0][0] + H[1][1] + H[2][2];
    const float sk = Sd[kmax];
    const float sgn = sk > 0.f ? 1.f : (sk < 0.f ? -1.f : 0.f);
    H[kmax][kmax] += trH * 1e-5f * sgn;
    float dM[3][3];
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) dM[i][j] = 2.f * (M[i][0] * H[0][j] + M[i][1] * H[1][j] + M[i][2] * H[2][j]);
    float GR[3][3];  // gradient wrt the textbook rotation R_std = Rg^T
    for (int k = 0; k < 3; k++) {
        ds[k] = (dM[k][0] * Rg[k][0] + dM[k][1] * Rg[k][1] + dM[k][2] * Rg[k][2]) * sm;
        for (int j = 0; j < 3; j++) GR[j][k] = sv[k] * dM[k][j];
    }
    const float r = q[0], x = q[1], y = q[2], z = q[3];
    dq[0] = 2.f * (-z * GR[0][1] + y * GR[0][2] + z * GR[1][0] - x * GR[1][2] - y * GR[2][0] + x * GR[2][1]);
    dq[1] = 2.f * (y * GR[0][1] + z * GR[0][2] + y * GR[1][0] - 2.f * x * GR[1][1] - r * GR[1][2] + z * GR[2][0] +
                   r * GR[2][1] - 2.f * x * GR[2][2]);
    dq[2] = 2.f * (-2.f * y * GR[0][0] + x * GR[0][1] + r * GR[0][2] + x * GR[1][0] + z * GR[1][2] - r * GR[2][0] +
                   z * GR[2][1] - 2.f * y * GR[2][2]);
    dq[3] = 2.f * (-2.f * z * GR[0][0] - r * GR[0][1] + x * GR[0][2] + r * GR[1][0] - 2.f * z * GR[1][1] +
                   y * GR[1][2] + x * GR[2][0] + y * GR[2][1]);
}

// Reference-compatible covariance adjoint: backward.cu:50-124 with glm's
// column-major conventions ((A*B)[c][r] = sum_k A[k][r] * B[c][k]).
__device__ void cov_adjoint_ref(const float s_in[3], const float q[4], float sm, const float c6[6],
                                const float u[6], float ds[3], float dq[4]) {
    float Rc[3][3];
    const float r = q[0], x = q[1], y = q[2], z = q[3];
    rot_cols(r, x, y, z, Rc);
    const float sv[3] = {sm * s_in[0], sm * s_in[1], sm * s_in[2]};
    auto mul = [](const float A[3][3], const float B[3][3], float O[3][3]) {
        for (int c = 0; c < 3; c++)
            for (int rr = 0; rr < 3; rr++) O[c][rr] = A[0][rr] * B[c][0] + A[1][rr] * B[c][1] + A[2][rr] * B[c][2];
    };
    float Sm[3][3] = {{sv[0], 0.f, 0.f}, {0.f, sv[1], 0.f}, {0.f, 0.f, sv[2]}};
    float M[3][3], Mt[3][3], Sigma[3][3];
    mul(Sm, Rc, M);
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) Mt[i][j] = M[j][i];
    mul(Mt, M, Sigma);
    const float C[3][3] = {{c6[0], c6[1], c6[2]}, {c6[1], c6[3], c6[4]}, {c6[2], c6[4], c6[5]}};
    const float G[3][3] = {{u[0], u[1], u[2]}, {u[1], u[3], u[4]}, {u[2], u[4], u[5]}};
    float negC[3][3], T1[3][3], dS[3][3];
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) negC[i][j] = -C[i][j];
    mul(negC, G, T1);
    mul(T1, C, dS);
    const float dc[6] = {dS[0][0], dS[0][1], dS[0][2], dS[1][1], dS[1][2], dS[2][2]};
    const float a0 = fabsf(Sigma[0][0]), a1 = fabsf(Sigma[1][1]), a2 = fabsf(Sigma[2][2]);
    auto sgn = [](float v) { return v > 0.f ? 1.f : (v < 0.f ? -1.f : 0.f); };
    const float de0 = (a0 >= a1 && a0 >= a2) ? 1e-5f * sgn(Sigma[0][0]) : 0.f;
    const float de1 = (a1 >= a0 && a1 >= a2) ? 1e-5f * sgn(Sigma[1][1]) : 0.f;
    const float de2 = (a2 >= a0 && a2 >= a1) ? 1e-5f * sgn(Sigma[2][2]) : 0.f;
    const float tr = dc[0] + dc[3] + dc[5];
    const float dLdS[3][3] = {{dc[0] + tr * de0, dc[1], dc[2]}, {dc[1], dc[3] + tr * de1, dc[4]}, {dc[2], dc[4], dc[5] + tr * de2}};
    float dM[3][3], Rt[3][3], dSm[3][3];
    mul(dLdS, M, dM);
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) dM[i][j] *= 2.f;
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) Rt[i][j] = Rc[j][i];
    mul(dM, Rt, dSm);
    ds[0] = dSm[0][0] * sm;
    ds[1] = dSm[1][1] * sm;
    ds[2] = dSm[2][2] * sm;
    for (int k = 0; k < 3; k++)
        for (int rr = 0; rr < 3; rr++) dM[k][rr] *= sv[k];
    dq[0] = 2 * z * (dM[1][0] - dM[0][1]) + 2 * y * (dM[0][2] - dM[2][0]) + 2 * x * (dM[2][1] - dM[1][2]);
    dq[1] = 2 * y * (dM[0][1] + dM[1][0]) + 2 * z * (dM[0][2] + dM[2][0]) + 2 * r * (dM[2][1] - dM[1][2]) -
            4 * x * (dM[2][2] + dM[1][1]);
    dq[2] = 2 * x * (dM[0][1] + dM[1][0]) + 2 * r * (dM[0][2] - dM[2][0]) + 2 * z * (dM[2][1] + dM[1][2]) -
            4 * y * (dM[2][2] + dM[0][0]);
    dq[3] = 2 * r * (dM[1][0] - dM[0][1]) + 2 * x * (dM[0][2] + dM[2][0]) + 2 * y * (dM[2][1] + dM[1][2]) -
            4 * z * (dM[1][1] + dM[0][0]);
}

__global__ void __launch_bounds__(256) k_finalize(int P, const float* __restrict__ gacc, const float* __restrict__ scales,
                                                  const float* __restrict__ rots, const float* __restrict__ conics,
                                                  float sm, int ref_compat, float* __restrict__ dmeans,
                                                  float* __restrict__ dscales, float* __restrict__ drots,
                                                  float* __restrict__ dvalues, float* __restrict__ dweights) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P) return;
    const float4* a = reinterpret_cast<const float4*>(gacc + 16 * (int64_t)i);
    const float4 a0 = a[0], a1 = a[1], a2 = a[2];
    dvalues[i] = a0.x;
    dweights[i] = a0.y;
    dmeans[3 * (int64_t)i] = a0.z;
    dmeans[3 * (int64_t)i + 1] = a0.w;
    dmeans[3 * (int64_t)i + 2] = a1.x;
    const float u[6] = {a1.y, a1.z, a1.w, a2.x, a2.y, a2.z};
    const float s[3] = {scales[3 * (int64_t)i], scales[3 * (int64_t)i + 1], scales[3 * (int64_t)i + 2]};
    const float q[4] = {rots[4 * (int64_t)i], rots[4 * (int64_t)i + 1], rots[4 * (int64_t)i + 2], rots[4 * (int64_t)i + 3]};
    float c6[6];
    for (int k = 0; k < 6; k++) c6[k] = conics[6 * (int64_t)i + k];
    float ds[3], dq[4];
    if (ref_compat) cov_adjoint_ref(s, q, sm, c6, u, ds, dq);
    else cov_adjoint_true(s, q, sm, c6, u, ds, dq);
    dscales[3 * (int64_t)i] = ds[0];
    dscales[3 * (int64_t)i + 1] = ds[1];
    dscales[3 * (int64_t)i + 2] = ds[2];
    drots[4 * (int64_t)i] = dq[0];
    drots[4 * (int64_t)i + 1] = dq[1];
    drots[4 * (int64_t)i + 2] = dq[2];
    drots[4 * (int64_t)i + 3] = dq[3];
}

// --------------------------------------------------------------------------------
// Launchers
// --------------------------------------------------------------------------------
static inline unsigned nblk(int64_t n, int per) { return (unsigned)((n + per - 1) / per); }

cudaError_t launch_forward(const FwdArgs& a, cudaStream_t st) {
    if (a.n_tiles <= 0) return cudaSuccess;
    if (a.count) {
        k_forward<true><<<nblk(a.n_tiles, kWarpsPerBlock), kWarpsPerBlock * 32, 0, st>>>(
            a.s_sorted, a.tile_boxes, a.gdesc, (int)a.n_tiles, a.gnodes, a.recs, a.out_cells, a.out_weights, a.status,
            a.stats);
    } else {
        k_forward<false><<<nblk(a.n_tiles, kWarpsPerBlock), kWarpsPerBlock * 32, 0, st>>>(
            a.s_sorted, a.tile_boxes, a.gdesc, (int)a.n_tiles, a.gnodes, a.recs, a.out_cells, a.out_weights, a.status,
            a.stats);
    }
    gvc::note_launch();
    return cudaGetLastError();
}

cudaError_t launch_backward_gauss(const BwdArgs& a, cudaStream_t st) {
    if (a.P <= 0) return cudaSuccess;
    if (a.count) {
        k_backward_gauss<true><<<nblk(a.P, kBwdWarps), kBwdWarps * 32, 0, st>>>(
            (int)a.P, a.gorder, a.means, a.values, a.weights, a.conics, a.boxes, a.s_grad, a.s_gyz, a.s_ok, a.gdesc,
            a.tnodes, a.gacc, a.status, a.stats);
    } else {
        k_backward_gauss<false><<<nblk(a.P, kBwdWarps), kBwdWarps * 32, 0, st>>>(
            (int)a.P, a.gorder, a.means, a.values, a.weights, a.conics, a.boxes, a.s_grad, a.s_gyz, a.s_ok, a.gdesc,
            a.tnodes, a.gacc, a.status, a.stats);
    }
    gvc::note_launch();
    return cudaGetLastError();
}

cudaError_t launch_backward_tiles(const BwdArgs& a, cudaStream_t st) {
    if (a.n_tiles <= 0) return cudaSuccess;
    if (a.count) {
        k_backward_tiles<true><<<nblk(a.n_tiles, kWarpsPerBlock), kWarpsPerBlock * 32, 0, st>>>(
            a.s_grad, a.s_gyz, a.s_ok, a.tile_boxes, a.gdesc, (int)a.n_tiles, a.gnodes, a.recs, a.gperm, a.gacc,
            a.status, a.stats);
    } else {
        k_backward_tiles<false><<<nblk(a.n_tiles, kWarpsPerBlock), kWarpsPerBlock * 32, 0, st>>>(
            a.s_grad, a.s_gyz, a.s_ok, a.tile_boxes, a.gdesc, (int)a.n_tiles, a.gnodes, a.recs, a.gperm, a.gacc,
            a.status, a.stats);
    }
    gvc::note_launch();
    return cudaGetLastError();
}

cudaError_t launch_finalize(int64_t P, const float* gacc, const float* scales, const float* rots, const float* conics,
                            float sm, int ref_compat, float* dmeans, float* dscales, float* drots, float* dvalues,
                            float* dweights, cudaStream_t st) {
    if (P <= 0) return cudaSuccess;
    k_finalize<<<nblk(P, 256), 256, 0, st>>>((int)P, gacc, scales, rots, conics, sm, ref_compat, dmeans, dscales,
                                             drots, dvalues, dweights); gvc::note_launch();
    return cudaGetLastError();
}

}  // namespace gvc
