// bwd_tc.cu -- backward of the mixture field on 128-sample blocks with the per-Gaussian
// reduction over samples on the tensor cores (replaces BACKWARD::sampleRenderCUDA,
// diff-gaussian-rasterization/cuda_rasterizer/backward.cu:339-559: sample-side
// traversal, per-Gaussian sums added atomically).
//
// One CTA owns the 128 Morton-sorted samples of a block and the block groups of the
// forward (k_sample_blocks).  A producer warp walks the Gaussian LBVH once per group and
// hands out the candidate Gaussians 128 at a time; consumer thread t owns candidate t of
// a batch (and TMEM lane t).  For a group with centre x0 and a sample row with u = x - x0,
//   phi(u) = [1, ux, uy, uz, ux ux, ux uy, ux uz, uy uy, uy uz, uz uz]
//   Psi(row) = [gx phi(u), gyz phi(u), 0 x 12]                     (B: 32 x rows)
// and with e the pair's exponential (the forward's base-2 power, window and AABB test),
//   D[gaussian][k] = sum over rows of e(row, gaussian) Psi(row)[k]  (A = E: 128 x rows)
// is one GEMM per batch, accumulated in FP32 in tensor memory by tcgen05.mma (M = 128,
// N = 32, K = 16 rows per chunk).  E is split into two BF16 parts (e to ~2^-16 relative)
// and Psi into three; the five products hi*hi, hi*mid, mid*hi, hi*lo and mid*mid are
// accumulated (the third part of E measured 10 % slower for no gain within tolerance).  Thread t then reads its
// own row of D, turns the moments about x0 into the moments about its mean (pair.cuh)
// and adds its eleven gradient terms with FP32 atomics.  An MMA warp issues the products
// while the consumers compute the next 16-row chunks (three A buffers); batches alternate
// between two TMEM accumulators, so that a batch's read-out waits until the next batch's
// chunks are issued and its last MMAs drain meanwhile.
#include "pair.cuh"
#include "render.cuh"
#include "tc.cuh"
#include "traverse.cuh"

namespace gvc {

constexpr int kBRows = 128;            // sample rows per block (the forward's blocks)
constexpr int kBGroups = 8;            // block groups per block
constexpr int kBBatch = 128;           // candidate Gaussians per batch (consumer threads)
constexpr int kBStages = 4;            // candidate batches in flight
constexpr int kBChunks = kBRows / 16;  // K chunks of 16 rows
constexpr int kMom = 32;               // B rows: 20 moment features + zero padding

struct BwdSmem {
    unsigned char A[3][2][kBBatch * 32];        // E chunk (128 x 16 bf16), two parts, three buffers
    unsigned char B[kBChunks][3][kMom * 32];    // Psi (32 x 16 bf16) per chunk, three parts
    float rx[kBRows], ry[kBRows], rz[kBRows];  // coordinates of the block's rows (pairs load as float2)
    uint8_t rok[kBRows];                        // W > 0.01 (pair statistics only)
    int cand[kBStages][kBBatch];                // candidate Gaussians (LBVH leaf = record index)
    int2 desc[kBStages];                        // (count or -1 at the end, group)
    int stack[kStackCap];
    int tcand[kCandCap];
    uint64_t full[kBStages], empty[kBStages], aready[3], afree[3], dready[2], dfree[2];
    uint32_t tmem_base;
};

__device__ __forceinline__ int bgroup_start(uint2 d, int g) {
    if (g == 0) return 0;
    if (g >= kBGroups) return kBRows;
    if (g <= 4) return (int)((d.x >> (8 * (g - 1))) & 0xffu);
    return (int)((d.y >> (8 * (g - 5))) & 0xffu);
}

// Producer: collects candidates into 128-entry batches (stage n % kBStages for batch n).
struct BwdProducer {
    BwdSmem& sm;
    int* status;
    uint32_t total;  // batches published
    int fill;        // entries in the open batch
    int g;           // current group
    bool failed;

    __device__ __forceinline__ bool acquire(uint32_t n) {
        const uint32_t k = n / kBStages;
        if (k == 0) return true;
        return mbar_wait(&sm.empty[n % kBStages], (k - 1) & 1u, status);
    }

    __device__ __forceinline__ void publish(int count) {
        const int lane = threadIdx.x & 31;
        __syncwarp();
        if (lane == 0) {
            sm.desc[total % kBStages] = make_int2(count, g);
            mbar_arrive(&sm.full[total % kBStages]);
        }
        total++;
        fill = 0;
        if (!acquire(total)) failed = true;
        __syncwarp();
    }

    __device__ __forceinline__ void operator()(const int* c, int nb) {
        const int lane = threadIdx.x & 31;
        int done = 0;
        while (done < nb && !failed) {
            const int take = min(nb - done, kBBatch - fill);
            if (lane < take) sm.cand[total % kBStages][fill + lane] = c[done + lane];
            fill += take;
            done += take;
            if (fill == kBBatch) publish(kBBatch);
        }
        __syncwarp();
    }
};

// Splits 16 fp32 values into three bf16 parts and stores them as row r of the three tiles.
__device__ __forceinline__ void store_split_row(unsigned char* t0, unsigned char* t1, unsigned char* t2, int r,
                                                const float (&v)[16]) {
    __nv_bfloat16 h[16], m[16], l[16];
    split_bf16(v, h, m, l);
    store_row_k16(t0, r, h);
    store_row_k16(t1, r, m);
    store_row_k16(t2, r, l);
}

template <bool COUNT, bool STACKLESS>
__global__ void __launch_bounds__(kBRows + 64, 4) k_backward_cta(
    int64_t n_slots, const uint2* __restrict__ bdesc, const float4* __restrict__ bboxes,
    const BvhNode* __restrict__ gnodes, int64_t n_internal, const GaussRec* __restrict__ recs,
    const int32_t* __restrict__ gperm,
    const float4* __restrict__ s_grad, const float* __restrict__ s_gyz, const uint8_t* __restrict__ s_ok,
    const int32_t* __restrict__ clog, const int32_t* __restrict__ cend, const uint2* __restrict__ cdesc,
    float* __restrict__ gacc, int* status, unsigned long long* stats) {
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    BwdSmem& sm = *reinterpret_cast<BwdSmem*>(smem_raw);
    const int t = threadIdx.x, w = t >> 5, lane = t & 31;
    const int64_t blk = blockIdx.x;
    const uint2 bd = bdesc[blk];
    const int ng = (int)(bd.y >> 24);
    if (t == 0) {
        for (int s = 0; s < kBStages; s++) {
            mbar_init(&sm.full[s], 1);
            mbar_init(&sm.empty[s], 5);  // the four consumer warps and the MMA warp
        }
        for (int b = 0; b < 3; b++) {
            mbar_init(&sm.aready[b], 4);
            mbar_init(&sm.afree[b], 1);
        }
        for (int b = 0; b < 2; b++) {
            mbar_init(&sm.dready[b], 1);
            mbar_init(&sm.dfree[b], 4);
        }
        fence_mbar_init();
    }
    // features 20..31 of every Psi tile stay zero
    for (int i = t; i < (int)(sizeof(sm.B) / sizeof(uint4)); i += kBRows + 64)
        reinterpret_cast<uint4*>(&sm.B[0][0][0])[i] = make_uint4(0u, 0u, 0u, 0u);
    fence_proxy_async_smem();
    if (t < kBRows) {
        const int64_t row = blk * kBRows + t;
        // rows past the end at +inf (outside every box); + 0 turns -0 into +0, which the
        // sign-bit box test below needs
        float4 p = make_float4(INFINITY, INFINITY, INFINITY, 0.f);
        if (row < n_slots) {
            const float4 q = s_grad[row];
            p = make_float4(q.x + 0.0f, q.y + 0.0f, q.z + 0.0f, s_ok[row] ? 1.f : 0.f);
        }
        sm.rx[t] = p.x;
        sm.ry[t] = p.y;
        sm.rz[t] = p.z;
        sm.rok[t] = p.w != 0.f;
    }
    if (w == 0) {
        static_assert(tmem_cols_ok(2 * kMom), "TMEM columns must be a power of two >= 32");
        tmem_alloc(&sm.tmem_base, 2 * kMom);
        tmem_relinquish();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = sm.tmem_base;

    if (w == 4) {
        // ---------------- producer ----------------
        BwdProducer pr{sm, status, 0u, 0, 0, false};
        TravCount tc;
        int st = 0;
        // With the forward's candidate log, the block's candidates are read back instead of
        // walking the tree.  The log holds the candidates of the forward's groups (cdesc),
        // each of which contains whole groups of this kernel: a group keeps the candidates
        // of its enclosing forward group whose boxes overlap its own, 128 per round trip.
        const uint2 cd = clog ? cdesc[blk] : make_uint2(0u, 0u);
        const int cng = (int)(cd.y >> 24);
        const int gend = (clog && lane < cng) ? cend[blk * kBGroups + lane] : -1;
        const bool from_log = clog && __shfl_sync(0xffffffffu, gend, 0) >= 0;
        const int32_t* blog = clog ? clog + blk * kCandLogPerBlock : nullptr;
        const uint32_t lt = lane_lt_mask();
        for (int g = 0; g < ng && !pr.failed; g++) {
            pr.g = g;
            const float4 glo = bboxes[2 * (blk * kBGroups + g)], ghi = bboxes[2 * (blk * kBGroups + g) + 1];
            if (from_log) {
                const int ra = bgroup_start(bd, g);
                int G = 0;
                for (int k = 1; k < cng; k++)
                    if (ra >= bgroup_start(cd, k)) G = k;
                const int a = G > 0 ? __shfl_sync(0xffffffffu, gend, G - 1) : 0;
                const int b = __shfl_sync(0xffffffffu, gend, G);
                const float3 qlo = make_float3(glo.x, glo.y, glo.z), qhi = make_float3(ghi.x, ghi.y, ghi.z);
                for (int off = a; off < b && !pr.failed; off += 128) {
                    int ids[4];
#pragma unroll
                    for (int u = 0; u < 4; u++) {
                        const int i = off + 32 * u + lane;
                        ids[u] = i < b ? __ldg(blog + i) : -1;
                    }
                    bool hit[4];
#pragma unroll
                    for (int u = 0; u < 4; u++) {
                        hit[u] = false;
                        if (ids[u] >= 0) {
                            const float4* rp = reinterpret_cast<const float4*>(recs + ids[u]);
                            hit[u] = box_overlap(__ldg(rp + 3), __ldg(rp + 4), qlo, qhi);
                        }
                    }
#pragma unroll
                    for (int u = 0; u < 4; u++) {
                        const uint32_t m = __ballot_sync(0xffffffffu, hit[u]);  // warp-uniform
                        if (m) {
                            if (hit[u]) sm.tcand[__popc(m & lt)] = ids[u];
                            __syncwarp();
                            pr(sm.tcand, __popc(m));
                            tc.leaves += __popc(m);
                        }
                    }
                }
            } else {
                st |= warp_traverse_sel<STACKLESS>(gnodes, n_internal, make_float3(glo.x, glo.y, glo.z),
                                                   make_float3(ghi.x, ghi.y, ghi.z), sm.stack, sm.tcand, pr, tc);
            }
            if (pr.fill > 0 && !pr.failed) pr.publish(pr.fill);
        }
        if (lane == 0) {
            if (st) atomicOr(status, st);
            if (!pr.failed) {
                sm.desc[pr.total % kBStages] = make_int2(-1, 0);
                mbar_arrive(&sm.full[pr.total % kBStages]);
            }
            if (COUNT) {
                atomicMax(&stats[4], (unsigned long long)tc.max_sp);
                atomicAdd(&stats[7], (unsigned long long)tc.leaves);
                atomicAdd(&stats[8], (unsigned long long)tc.nodes);
            }
        }
        __syncwarp();
    } else if (w == 5) {
        // ---------------- MMA issuer ----------------
        if (lane == 0) {
            const uint32_t idesc = idesc_bf16_f32(kBBatch, kMom);
            uint32_t j = 0;  // chunk counter (same sequence as the consumers)
            for (uint32_t n = 0;; n++) {
                const int s = (int)(n % kBStages);
                if (!mbar_wait(&sm.full[s], (n / kBStages) & 1u, status)) break;
                const int2 d = sm.desc[s];
                if (d.x < 0) break;
                mbar_arrive(&sm.empty[s]);  // its descriptor is read
                const int ra = bgroup_start(bd, d.y), rb = bgroup_start(bd, d.y + 1);
                const int q0 = ra >> 4, q1 = (rb - 1) >> 4;
                if (n >= 2 && !mbar_wait(&sm.dfree[n & 1u], ((n >> 1) - 1) & 1u, status)) break;
                const uint32_t tmem_d = tmem + (n & 1u) * kMom;
                bool ok = true;
                for (int q = q0; q <= q1; q++, j++) {
                    const int b = (int)(j % 3u);
                    if (!mbar_wait(&sm.aready[b], (j / 3u) & 1u, status)) {
                        ok = false;
                        break;
                    }
                    tc_fence_after();
                    const uint64_t a0 = smem_desc_k16(sm.A[b][0]), a1 = smem_desc_k16(sm.A[b][1]);
                    const uint64_t b0 = smem_desc_k16(sm.B[q][0]), b1 = smem_desc_k16(sm.B[q][1]),
                                   b2 = smem_desc_k16(sm.B[q][2]);
                    umma_bf16(tmem_d, a1, b1, idesc, q == q0 ? 0u : 1u);  // mid * mid
                    umma_bf16(tmem_d, a0, b2, idesc, 1u);                 // hi * lo
                    umma_bf16(tmem_d, a1, b0, idesc, 1u);                 // mid * hi
                    umma_bf16(tmem_d, a0, b1, idesc, 1u);                 // hi * mid
                    umma_bf16(tmem_d, a0, b0, idesc, 1u);                 // hi * hi
                    umma_commit(&sm.afree[b]);
                }
                if (!ok) break;
                umma_commit(&sm.dready[n & 1u]);
            }
        }
        __syncwarp();
    } else {
        // ---------------- consumers: thread t owns candidate t of each batch ----------------
        int cur_group = -1;
        float x0 = 0.f, y0 = 0.f, z0 = 0.f;
        uint32_t j = 0;
        int ncand = 0, ncontrib = 0;
        long long nlane = 0;  // lane slots evaluated (warp-uniform)
        // The previous batch's read-out is deferred until this batch's chunks are issued,
        // so that its last MMAs drain meanwhile (two TMEM accumulators, by batch parity).
        bool pending = false;
        uint32_t pend_n = 0;
        int pend_leaf = -1;
        float px0 = 0.f, py0 = 0.f, pz0 = 0.f;
        auto drain = [&]() -> bool {
            const uint32_t pb = pend_n & 1u;
            pending = false;
            const bool okd = mbar_wait(&sm.dready[pb], (pend_n >> 1) & 1u, status);
            if (!__all_sync(0xffffffffu, okd)) return false;
            tc_fence_after();
            float v[32];
            tmem_ld32(tmem + pb * kMom + ((uint32_t)(32 * w) << 16), v);
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(&sm.dfree[pb]);
            // a Gaussian without a contributing pair has an all-zero row of D
            bool anyc = false;
#pragma unroll
            for (int k = 0; k < 20; k++) anyc |= v[k] != 0.f;
            if (anyc && pend_leaf >= 0) {
                const float4* rp = reinterpret_cast<const float4*>(recs + pend_leaf);
                const float4 r0 = __ldg(rp), r1 = __ldg(rp + 1), r2 = __ldg(rp + 2);
                // moments about the group centre -> moments about the mean (d = u - a)
                const float ax = r0.x - px0, ay = r0.y - py0, az = r0.z - pz0;
                float S[10];
#pragma unroll
                for (int k = 0; k < 10; k++) S[k] = fmaf(r2.z, v[k], v[10 + k]);
                float m[11];
                m[0] = v[0];
                m[1] = S[0];
                m[2] = S[1] - ax * S[0];
                m[3] = S[2] - ay * S[0];
                m[4] = S[3] - az * S[0];
                m[5] = S[4] - 2.f * ax * S[1] + ax * ax * S[0];
                m[6] = S[5] - ax * S[2] - ay * S[1] + ax * ay * S[0];
                m[7] = S[6] - ax * S[3] - az * S[1] + ax * az * S[0];
                m[8] = S[7] - 2.f * ay * S[2] + ay * ay * S[0];
                m[9] = S[8] - ay * S[3] - az * S[2] + ay * az * S[0];
                m[10] = S[9] - 2.f * az * S[3] + az * az * S[0];
                float tm[11];
                moments_to_terms_lane(m, r0.w, r1.x, r1.y, r1.z, r1.w, r2.x, r2.y, tm);
                float4* dst = reinterpret_cast<float4*>(gacc + 16 * (int64_t)gperm[pend_leaf]);
                atomicAdd(dst, make_float4(tm[0], tm[1], tm[2], tm[3]));
                atomicAdd(dst + 1, make_float4(tm[4], tm[5], tm[6], tm[7]));
                atomicAdd(dst + 2, make_float4(tm[8], tm[9], tm[10], 0.f));
            }
            return true;
        };
        for (uint32_t n = 0;; n++) {
            const int s = (int)(n % kBStages);
            const bool okw = mbar_wait(&sm.full[s], (n / kBStages) & 1u, status);
            if (!__all_sync(0xffffffffu, okw)) break;
            const int2 d = sm.desc[s];
            if (d.x < 0) break;
            const int ra = bgroup_start(bd, d.y), rb = bgroup_start(bd, d.y + 1);
            const int q0 = ra >> 4, q1 = (rb - 1) >> 4;
            if (d.y != cur_group) {
                // Psi of this warp's rows (chunks 2w, 2w + 1) for the new group; every MMA of
                // the previous group has completed once its last batch is drained.
                if (pending && !drain()) break;
                cur_group = d.y;
                const float4 glo = bboxes[2 * (blk * kBGroups + d.y)], ghi = bboxes[2 * (blk * kBGroups + d.y) + 1];
                x0 = 0.5f * (glo.x + ghi.x);
                y0 = 0.5f * (glo.y + ghi.y);
                z0 = 0.5f * (glo.z + ghi.z);
                const int r = 32 * w + lane;
                const bool in = r >= ra && r < rb && blk * kBRows + r < n_slots;
                float gx = 0.f, gyz = 0.f, ux = 0.f, uy = 0.f, uz = 0.f;
                if (in) {
                    const float4 q = s_grad[blk * kBRows + r];
                    gx = q.w;
                    gyz = s_gyz[blk * kBRows + r];
                    ux = q.x - x0;
                    uy = q.y - y0;
                    uz = q.z - z0;
                }
                const float ph[10] = {1.f, ux, uy, uz, ux * ux, ux * uy, ux * uz, uy * uy, uy * uz, uz * uz};
                // row r is column k = r % 16 of chunk r / 16; feature n is tile row n
                const int q = r >> 4, k = r & 15;
                const int koff = (k >> 3) * 128 + (k & 7) * 2;
#pragma unroll
                for (int n = 0; n < 20; n++) {
                    const float v = in ? (n < 10 ? gx : gyz) * ph[n < 10 ? n : n - 10] : 0.f;
                    const __nv_bfloat16 h = __float2bfloat16_rn(v);
                    const float r1 = v - __bfloat162float(h);
                    const __nv_bfloat16 m = __float2bfloat16_rn(r1);
                    const __nv_bfloat16 l = __float2bfloat16_rn(r1 - __bfloat162float(m));
                    const int off = (n >> 3) * 256 + (n & 7) * 16 + koff;
                    *reinterpret_cast<__nv_bfloat16*>(sm.B[q][0] + off) = h;
                    *reinterpret_cast<__nv_bfloat16*>(sm.B[q][1] + off) = m;
                    *reinterpret_cast<__nv_bfloat16*>(sm.B[q][2] + off) = l;
                }
                fence_proxy_async_smem();
                __syncwarp();
            }
            // this thread's Gaussian (an empty box when the batch is not full)
            float4 r0 = make_float4(0.f, 0.f, 0.f, 0.f), r1 = r0, r2 = r0;
            float4 blo = make_float4(INFINITY, INFINITY, INFINITY, 0.f), bhi = make_float4(-INFINITY, -INFINITY, -INFINITY, 0.f);
            int leaf = -1;
            if (t < d.x) {
                leaf = sm.cand[s][t];
                const float4* rp = reinterpret_cast<const float4*>(recs + leaf);
                r0 = __ldg(rp);
                r1 = __ldg(rp + 1);
                r2 = __ldg(rp + 2);
                blo = __ldg(rp + 3);
                bhi = __ldg(rp + 4);
            }
            __syncwarp();
            if (lane == 0) mbar_arrive(&sm.empty[s]);  // the stage's candidates are read
            const GaussB g = gauss_b(r0.x, r0.y, r0.z, r2.z, r1.x, r1.y, r1.z, r1.w, r2.x, r2.y, blo, bhi);
            const float2 nmx = make_float2(-g.mx, -g.mx), nmy = make_float2(-g.my, -g.my),
                         nmz = make_float2(-g.mz, -g.mz);
            const float2 Q0 = make_float2(g.q0, g.q0), Q1 = make_float2(g.q1, g.q1), Q2 = make_float2(g.q2, g.q2),
                         Q3 = make_float2(g.q3, g.q3), Q4 = make_float2(g.q4, g.q4), Q5 = make_float2(g.q5, g.q5);
            // box and window as signs of differences: lo <= x <=> x - lo has its sign bit clear,
            // exact for finite values once neither x nor hi is -0 (rows and hi get + 0)
            const float2 NLX = make_float2(-g.lx, -g.lx), NLY = make_float2(-g.ly, -g.ly),
                         NLZ = make_float2(-g.lz, -g.lz);
            const float2 HX = make_float2(g.hx + 0.0f, g.hx + 0.0f), HY = make_float2(g.hy + 0.0f, g.hy + 0.0f),
                         HZ = make_float2(g.hz + 0.0f, g.hz + 0.0f);
            bool okc = true;
            for (int q = q0; q <= q1; q++, j++) {
                const int b = (int)(j % 3u);
                if (j >= 3) {
                    const bool okf = mbar_wait(&sm.afree[b], ((j / 3u) - 1) & 1u, status);
                    if (!__all_sync(0xffffffffu, okf)) {
                        okc = false;
                        break;
                    }
                }
                // branch-free over the 16 rows: independent chains the scheduler can interleave
                // (a per-row warp vote to skip missing rows measured 15 % slower)
                // rows of the chunk inside the group (warp-uniform bit mask)
                const int c0 = max(ra - 16 * q, 0), c1 = min(rb - 16 * q, 16);
                const uint32_t rmask = c1 > c0 ? (((1u << (c1 - c0)) - 1u) << c0) : 0u;
                // Rows two at a time: the coordinates load as float2 pairs and the power runs
                // on packed f32x2 FMAs (the AABB test, window and ex2 per row).
                uint32_t hw[8], mw[8];
#pragma unroll
                for (int k = 0; k < 16; k += 2) {
                    const int r = 16 * q + k;
                    const float2 X = *reinterpret_cast<const float2*>(&sm.rx[r]);
                    const float2 Y = *reinterpret_cast<const float2*>(&sm.ry[r]);
                    const float2 Z = *reinterpret_cast<const float2*>(&sm.rz[r]);
                    // rows of the chunk outside the group need no mask: their Psi rows are zero
                    const float2 M1 = make_float2(-1.0f, -1.0f);
                    const float2 lx2 = __fadd2_rn(X, NLX), ly2 = __fadd2_rn(Y, NLY), lz2 = __fadd2_rn(Z, NLZ);
                    const float2 hx2 = __ffma2_rn(X, M1, HX), hy2 = __ffma2_rn(Y, M1, HY), hz2 = __ffma2_rn(Z, M1, HZ);
                    const uint32_t b0 = __float_as_uint(lx2.x) | __float_as_uint(ly2.x) | __float_as_uint(lz2.x) |
                                        __float_as_uint(hx2.x) | __float_as_uint(hy2.x) | __float_as_uint(hz2.x);
                    const uint32_t b1 = __float_as_uint(lx2.y) | __float_as_uint(ly2.y) | __float_as_uint(lz2.y) |
                                        __float_as_uint(hx2.y) | __float_as_uint(hy2.y) | __float_as_uint(hz2.y);
                    const float2 dX = __fadd2_rn(X, nmx), dY = __fadd2_rn(Y, nmy), dZ = __fadd2_rn(Z, nmz);
                    // p2 = dx (q0 dx + q1 dy + q2 dz) + dy (q3 dy + q4 dz) + dz (q5 dz)
                    float2 a = __ffma2_rn(Q0, dX, __ffma2_rn(Q1, dY, __fmul2_rn(Q2, dZ)));
                    a = __fmul2_rn(dX, a);
                    a = __ffma2_rn(dY, __ffma2_rn(Q3, dY, __fmul2_rn(Q4, dZ)), a);
                    const float2 P2 = __ffma2_rn(dZ, __fmul2_rn(Q5, dZ), a);
                    // window kLog2Floor <= p2 <= 0: p2 - floor and 0 - p2 (as -p2 + 0: +0 for p2 = -0)
                    const float2 wl = __fadd2_rn(P2, make_float2(-kLog2Floor, -kLog2Floor));
                    const float2 wh = __ffma2_rn(P2, M1, make_float2(0.0f, 0.0f));
                    const bool c0 = (int)(b0 | __float_as_uint(wl.x) | __float_as_uint(wh.x)) >= 0;
                    const bool c1 = (int)(b1 | __float_as_uint(wl.y) | __float_as_uint(wh.y)) >= 0;
                    const float e0 = c0 ? ex2_approx(P2.x) : 0.f, e1 = c1 ? ex2_approx(P2.y) : 0.f;
                    // E in two BF16 parts (~16 bits: e to 2^-16 relative); Psi keeps three
                    const __nv_bfloat162 H = __floats2bfloat162_rn(e0, e1);
                    const __nv_bfloat162 M = __floats2bfloat162_rn(e0 - __low2float(H), e1 - __high2float(H));
                    hw[k >> 1] = *reinterpret_cast<const uint32_t*>(&H);
                    mw[k >> 1] = *reinterpret_cast<const uint32_t*>(&M);
                    if (COUNT) {
                        const bool g0 = (rmask >> k) & 1u, g1 = (rmask >> (k + 1)) & 1u;
                        ncand += ((g0 && (int)b0 >= 0) ? 1 : 0) + ((g1 && (int)b1 >= 0) ? 1 : 0);
                        ncontrib += ((g0 && c0 && sm.rok[r]) ? 1 : 0) + ((g1 && c1 && sm.rok[r + 1]) ? 1 : 0);
                        nlane += 64;
                    }
                }
                tc_fence_after();
                {
                    unsigned char* a0 = sm.A[b][0] + (t >> 3) * 256 + (t & 7) * 16;
                    unsigned char* a1 = sm.A[b][1] + (t >> 3) * 256 + (t & 7) * 16;
                    *reinterpret_cast<uint4*>(a0) = make_uint4(hw[0], hw[1], hw[2], hw[3]);
                    *reinterpret_cast<uint4*>(a0 + 128) = make_uint4(hw[4], hw[5], hw[6], hw[7]);
                    *reinterpret_cast<uint4*>(a1) = make_uint4(mw[0], mw[1], mw[2], mw[3]);
                    *reinterpret_cast<uint4*>(a1 + 128) = make_uint4(mw[4], mw[5], mw[6], mw[7]);
                }
                fence_proxy_async_smem();
                __syncwarp();
                if (lane == 0) mbar_arrive(&sm.aready[b]);
            }
            if (!okc) break;
            if (pending && !drain()) break;
            pending = true;
            pend_n = n;
            pend_leaf = leaf;
            px0 = x0;
            py0 = y0;
            pz0 = z0;
        }
        if (pending) drain();
        if (COUNT) {
            unsigned long long a = (unsigned long long)ncand, c = (unsigned long long)ncontrib;
            for (int off = 16; off > 0; off >>= 1) {
                a += __shfl_xor_sync(0xffffffffu, a, off);
                c += __shfl_xor_sync(0xffffffffu, c, off);
            }
            (void)a;
            if (lane == 0) {
                atomicAdd(&stats[2], c);
                atomicAdd(&stats[10], (unsigned long long)nlane);
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (w == 0) tmem_dealloc(tmem, 2 * kMom);
}

template <bool COUNT, bool STACKLESS>
static cudaError_t launch_bwd_cta_impl(const BwdArgs& a, int64_t n_blocks, const uint2* bdesc, const float4* bboxes,
                                       cudaStream_t st) {
    const size_t smem = sizeof(BwdSmem) + 1024;
    cudaError_t e =
        cudaFuncSetAttribute(k_backward_cta<COUNT, STACKLESS>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    k_backward_cta<COUNT, STACKLESS><<<(unsigned)n_blocks, kBRows + 64, smem, st>>>(
        a.n_tiles * kTile, bdesc, bboxes, a.gnodes, a.g_internal, a.recs, a.gperm, a.s_grad, a.s_gyz, a.s_ok,
        a.clog, a.cend, a.cdesc, a.gacc, a.status, a.stats);
    gvc::note_launch();
    return cudaGetLastError();
}

cudaError_t launch_backward_cta(const BwdArgs& a, int64_t n_blocks, const uint2* bdesc, const float4* bboxes,
                                cudaStream_t st) {
    if (n_blocks <= 0 || a.P <= 0) return cudaSuccess;
    if (a.stackless)
        return a.count ? launch_bwd_cta_impl<true, true>(a, n_blocks, bdesc, bboxes, st)
                       : launch_bwd_cta_impl<false, true>(a, n_blocks, bdesc, bboxes, st);
    return a.count ? launch_bwd_cta_impl<true, false>(a, n_blocks, bdesc, bboxes, st)
                   : launch_bwd_cta_impl<false, false>(a, n_blocks, bdesc, bboxes, st);
}

}  // namespace gvc
