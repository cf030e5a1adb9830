// prep.cu -- per-Gaussian preprocessing and the sample-side gathers.
//
// This file is compiled with --fmad=false: every float and double expression rounds
// after each operation, exactly like the oracle compiled with -ffp-contract=off, so
// the conic output and the AABBs are reproducible bit for bit on the CPU.
#include "render.cuh"

namespace gvc {

__device__ __forceinline__ void rot_cols_p(float r, float x, float y, float z, float Rc[3][3]) {
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

// conic = adj(Sigma + eps I) / det in float (forward.cu:46-76); when the Frobenius
// condition estimate ||Sigma'||_F ||conic||_F exceeds kCondFp64 the inverse is
// recomputed in double from the float scales and quaternion and rounded once.
__device__ void conic_select(const float s_in[3], const float q[4], float sm, float c[6]) {
    float Rc[3][3];
    rot_cols_p(q[0], q[1], q[2], q[3], Rc);
    const float sv[3] = {sm * s_in[0], sm * s_in[1], sm * s_in[2]};
    float M[3][3];  // M[col][row] = sv[row] * Rc[col][row]
    for (int ci = 0; ci < 3; ci++)
        for (int r = 0; r < 3; r++) M[ci][r] = sv[r] * Rc[ci][r];
    float Sg[3][3];
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) {
            float acc = M[i][0] * M[j][0];
            acc = acc + M[i][1] * M[j][1];
            acc = acc + M[i][2] * M[j][2];
            Sg[i][j] = acc;
        }
    const float eps = (float)((double)fmaxf(fmaxf(fabsf(Sg[0][0]), fabsf(Sg[1][1])), fabsf(Sg[2][2])) * 1e-5);
    const float a = Sg[0][0] + eps, b = Sg[0][1], cc = Sg[0][2];
    const float d = Sg[1][1] + eps, e = Sg[1][2], f = Sg[2][2] + eps;
    const float det = a * (d * f - e * e) - b * (b * f - cc * e) + cc * (b * e - cc * d);
    const float inv = (float)(1.0 / (double)det);
    c[0] = (d * f - e * e) * inv;
    c[1] = (cc * e - b * f) * inv;
    c[2] = (b * e - cc * d) * inv;
    c[3] = (a * f - cc * cc) * inv;
    c[4] = (b * cc - a * e) * inv;
    c[5] = (a * d - b * b) * inv;
    float nS = a * a;
    nS = nS + d * d;
    nS = nS + f * f;
    float oS = b * b;
    oS = oS + cc * cc;
    oS = oS + e * e;
    nS = nS + 2.f * oS;
    float nC = c[0] * c[0];
    nC = nC + c[3] * c[3];
    nC = nC + c[5] * c[5];
    float oC = c[1] * c[1];
    oC = oC + c[2] * c[2];
    oC = oC + c[4] * c[4];
    nC = nC + 2.f * oC;
    const float cond2 = nS * nC;
    if (cond2 <= kCondFp64 * kCondFp64) return;
    // FP64 inverse (Gaussians with a large condition estimate, or non-finite values)
    const double r = q[0], x = q[1], y = q[2], z = q[3];
    const double Rs[3][3] = {{1.0 - 2.0 * (y * y + z * z), 2.0 * (x * y - r * z), 2.0 * (x * z + r * y)},
                             {2.0 * (x * y + r * z), 1.0 - 2.0 * (x * x + z * z), 2.0 * (y * z - r * x)},
                             {2.0 * (x * z - r * y), 2.0 * (y * z + r * x), 1.0 - 2.0 * (x * x + y * y)}};
    const double sd[3] = {(double)sv[0], (double)sv[1], (double)sv[2]};
    double S[3][3];
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) {
            double acc = 0.0;
            for (int k = 0; k < 3; k++) acc += (sd[k] * Rs[i][k]) * (sd[k] * Rs[j][k]);
            S[i][j] = acc;
        }
    const double ep = fmax(fmax(fabs(S[0][0]), fabs(S[1][1])), fabs(S[2][2])) * 1e-5;
    const double A = S[0][0] + ep, B = S[0][1], CC = S[0][2];
    const double D = S[1][1] + ep, E = S[1][2], F = S[2][2] + ep;
    const double dt = A * (D * F - E * E) - B * (B * F - CC * E) + CC * (B * E - CC * D);
    const double iv = 1.0 / dt;
    c[0] = (float)((D * F - E * E) * iv);
    c[1] = (float)((CC * E - B * F) * iv);
    c[2] = (float)((B * E - CC * D) * iv);
    c[3] = (float)((A * F - CC * CC) * iv);
    c[4] = (float)((B * CC - A * E) * iv);
    c[5] = (float)((A * D - B * B) * iv);
}

// Oriented-box AABB (forward.cu:78-113): corners mu +- m s_k Rc[k] walk the glm
// columns (rows of the textbook rotation), m = sqrt(-2 ln(1e-3 / w)) evaluated in
// double and rounded once; min/max ignore NaN (w < 1e-3 collapses the box to mu).
__device__ void aabb_of(const float mu[3], const float s_in[3], const float q[4], float w, float sm, float lo[3],
                        float hi[3]) {
    float Rc[3][3];
    rot_cols_p(q[0], q[1], q[2], q[3], Rc);
    const float S0 = sm * s_in[0], S1 = sm * s_in[1], S2 = sm * s_in[2];
    // (0.1 * WEIGHT_CUTOFF) with the reference's double literal 1e-2 (config.h:9)
    const float arg = (float)((0.1 * 1e-2) / (double)w);
    const float m = (float)sqrt(-2.0 * log((double)arg));
    const float ss0 = S0 * m, ss1 = S1 * m, ss2 = S2 * m;
    const float n[2] = {-1.0f, 1.0f};
    for (int a = 0; a < 3; a++) {
        lo[a] = mu[a];
        hi[a] = mu[a];
    }
    for (int i = 0; i < 2; i++)
        for (int j = 0; j < 2; j++)
            for (int k = 0; k < 2; k++)
                for (int a = 0; a < 3; a++) {
                    float t0 = n[i] * Rc[0][a];
                    t0 = t0 * ss0;
                    float t1 = n[j] * Rc[1][a];
                    t1 = t1 * ss1;
                    float t2 = n[k] * Rc[2][a];
                    t2 = t2 * ss2;
                    float c = mu[a] + t0;
                    c = c + t1;
                    c = c + t2;
                    lo[a] = fminf(lo[a], c);
                    hi[a] = fmaxf(hi[a], c);
                }
}

__global__ void __launch_bounds__(256) k_preprocess(int64_t P, const float* __restrict__ means,
                                                    const float* __restrict__ scales, const float* __restrict__ rots,
                                                    const float* __restrict__ weights, float sm,
                                                    float* __restrict__ conics_out, float4* __restrict__ boxes_out) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= P) return;
    const float s[3] = {scales[3 * i], scales[3 * i + 1], scales[3 * i + 2]};
    const float q[4] = {rots[4 * i], rots[4 * i + 1], rots[4 * i + 2], rots[4 * i + 3]};
    if (conics_out) {
        float c[6];
        conic_select(s, q, sm, c);
        for (int k = 0; k < 6; k++) conics_out[6 * i + k] = c[k];
    }
    if (boxes_out) {
        const float mu[3] = {means[3 * i], means[3 * i + 1], means[3 * i + 2]};
        float lo[3], hi[3];
        aabb_of(mu, s, q, weights[i], sm, lo, hi);
        boxes_out[2 * i] = make_float4(lo[0], lo[1], lo[2], 0.f);
        boxes_out[2 * i + 1] = make_float4(hi[0], hi[1], hi[2], 0.f);
    }
}

__global__ void __launch_bounds__(256) k_gather_recs(int64_t P, const int32_t* __restrict__ perm,
                                                     const float* __restrict__ means, const float* __restrict__ values,
                                                     const float* __restrict__ weights,
                                                     const float* __restrict__ conics, const float4* __restrict__ boxes,
                                                     GaussRec* __restrict__ recs) {
    const int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (g >= P) return;
    const int64_t o = perm[g];
    GaussRec r;
    r.r0 = make_float4(means[3 * o], means[3 * o + 1], means[3 * o + 2], weights[o]);
    r.r1 = make_float4(conics[6 * o], conics[6 * o + 1], conics[6 * o + 2], conics[6 * o + 3]);
    r.r2 = make_float4(conics[6 * o + 4], conics[6 * o + 5], values[o], 0.f);
    r.r3 = boxes[2 * o];
    r.r4 = boxes[2 * o + 1];
    recs[g] = r;
}

// Sorted sample slots: (x, y, z, caller index as int bits); padding slots carry NaN
// coordinates and index -1.  One warp per tile of 32 slots also splits the tile into at
// most kGroups contiguous lane groups: a group [a, b) is split at the Morton bit where
// its first and last keys first differ when both halves' boxes are at most half the
// group's size (half-perimeter).  A tile that straddles a jump of the Z-order curve thus
// becomes compact groups instead of one box spanning the jump.  Writes one box and
// key per group slot (unused slots: empty box, key of the last sample) and the group
// descriptor of the tile.
struct WBox {
    float lx, ly, lz, hx, hy, hz;
};

__device__ __forceinline__ WBox warp_box(bool in, float x, float y, float z) {
    WBox b;
    b.lx = in ? x : INFINITY;
    b.ly = in ? y : INFINITY;
    b.lz = in ? z : INFINITY;
    b.hx = in ? x : -INFINITY;
    b.hy = in ? y : -INFINITY;
    b.hz = in ? z : -INFINITY;
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

__device__ __forceinline__ float half_perimeter(const WBox& b) {
    return (b.hx - b.lx) + (b.hy - b.ly) + (b.hz - b.lz);
}

// A lane group is split when both halves' boxes have at most this fraction of the whole's
// half-perimeter (0.65 measured best for the backward's candidate rows: 0.5 gathers 9.4e9
// rows at 2M x 16M, 0.65 8.5e9; from 0.8 on the extra leaves cost more than they save).
constexpr float kTileSplitRatio = 0.65f;

// Split lane of group [a, b), or -1 (warp-uniform).
__device__ int try_split(int a, int b, uint32_t key, int lane, float x, float y, float z) {
    if (b - a < 2) return -1;
    const uint32_t ka = __shfl_sync(0xffffffffu, key, a), kb = __shfl_sync(0xffffffffu, key, b - 1);
    if (ka == kb) return -1;
    const int bit = 31 - __clz(ka ^ kb);
    const bool in = lane >= a && lane < b;
    const uint32_t hi = __ballot_sync(0xffffffffu, in && ((key >> bit) & 1u));
    const int m = __ffs(hi) - 1;  // keys are sorted: a < m < b
    const WBox B = warp_box(in, x, y, z);
    const WBox B1 = warp_box(in && lane < m, x, y, z);
    const WBox B2 = warp_box(in && lane >= m, x, y, z);
    const float h = half_perimeter(B);
    return fmaxf(half_perimeter(B1), half_perimeter(B2)) <= kTileSplitRatio * h ? m : -1;
}

__global__ void __launch_bounds__(256) k_sample_tiles(int64_t S, int64_t n_tiles, const float* __restrict__ samples,
                                                      const int32_t* __restrict__ perm,
                                                      const uint32_t* __restrict__ skeys, float4* __restrict__ s_sorted,
                                                      float4* __restrict__ group_boxes, uint32_t* __restrict__ group_keys,
                                                      uint32_t* __restrict__ gdesc, int with_groups) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int64_t t = i >> 5;
    if (t >= n_tiles) return;
    const int lane = threadIdx.x & 31;
    float x = NAN, y = NAN, z = NAN;
    int o = -1;
    uint32_t key = 0xffffffffu;
    if (!with_groups) {
        // pass 1 (build_bvh): gather the sorted samples
        if (i < S) {
            o = perm[i];
            x = samples[3 * (int64_t)o];
            y = samples[3 * (int64_t)o + 1];
            z = samples[3 * (int64_t)o + 2];
        }
        s_sorted[i] = make_float4(x, y, z, __int_as_float(o));
        return;  // warp-uniform
    }
    // pass 2 (first user of the lane groups): read them back from s_sorted
    const float4 sp = s_sorted[i];
    x = sp.x;
    y = sp.y;
    z = sp.z;
    o = __float_as_int(sp.w);
    if (i < S) key = skeys[i];
    const int nvalid = __popc(__ballot_sync(0xffffffffu, o >= 0));
    int starts[kGroups + 1];
    int ng = 1;
    starts[0] = 0;
    const int m = try_split(0, nvalid, key, lane, x, y, z);
    if (m >= 0) {
        const int m1 = try_split(0, m, key, lane, x, y, z);
        const int m2 = try_split(m, nvalid, key, lane, x, y, z);
        if (m1 >= 0) starts[ng++] = m1;
        starts[ng++] = m;
        if (m2 >= 0) starts[ng++] = m2;
    }
    for (int g = ng; g <= kGroups; g++) starts[g] = 32;
    const uint32_t last_key = __shfl_sync(0xffffffffu, key, nvalid - 1);
    for (int g = 0; g < kGroups; g++) {
        const int a = starts[g], b = (g + 1 < ng) ? starts[g + 1] : nvalid;
        WBox B;
        uint32_t k = last_key;
        if (g < ng) {
            B = warp_box(lane >= a && lane < b, x, y, z);
            k = __shfl_sync(0xffffffffu, key, a);
        } else {
            B.lx = B.ly = B.lz = INFINITY;
            B.hx = B.hy = B.hz = -INFINITY;
        }
        if (lane == 0) {
            group_boxes[2 * (kGroups * t + g)] = make_float4(B.lx, B.ly, B.lz, 0.f);
            group_boxes[2 * (kGroups * t + g) + 1] = make_float4(B.hx, B.hy, B.hz, 0.f);
            group_keys[kGroups * t + g] = k;
        }
    }
    if (lane == 0)
        gdesc[t] = (uint32_t)starts[1] | ((uint32_t)starts[2] << 8) | ((uint32_t)starts[3] << 16) |
                   ((uint32_t)ng << 24);
}

// Per sorted sample: (gO / W, -gO * out / W, gW, 1) if W > 0.01, else zeros
// (backward.cu:260-263 and :268-279).
// Backward sample records in sorted order: (x, y, z, gx) with gx = dL/dout / W, gyz =
// -dL/dout * out / W + dL/dW (backward.cu:252-298 folds the same factors per pair), and
// ok = W > 0.01.  Samples below the cutoff get gx = gyz = 0, so their pairs add exactly
// nothing; tile padding gets finite coordinates (0) and zero gradients for the same reason.
// With out_sorted (the forward's (out, W) per sorted slot) only dL/dout and dL/dW are
// gathered from the caller's order.
__global__ void __launch_bounds__(256) k_sample_grads(int64_t n_slots, const float4* __restrict__ s_sorted,
                                                      const float2* __restrict__ out_sorted,
                                                      const float* __restrict__ out_cells,
                                                      const float* __restrict__ out_weights,
                                                      const float* __restrict__ gout, const float* __restrict__ gw,
                                                      float4* __restrict__ s_grad, float* __restrict__ s_gyz,
                                                      uint8_t* __restrict__ s_ok) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n_slots) return;
    const float4 sp = s_sorted[i];
    const int o = __float_as_int(sp.w);
    float gx = 0.f, gyz = 0.f;
    uint8_t ok = 0;
    float4 r = make_float4(0.f, 0.f, 0.f, 0.f);
    if (o >= 0) {
        const float2 ow = out_sorted ? out_sorted[i] : make_float2(0.f, out_weights[o]);
        const float W = ow.y;
        if (W > kWeightCutoff) {
            const float g = gout[o];
            gx = g / W;
            gyz = -(g * (out_sorted ? ow.x : out_cells[o])) / W + gw[o];
            ok = 1;
        }
        r = make_float4(sp.x, sp.y, sp.z, gx);
    }
    s_grad[i] = r;
    s_gyz[i] = gyz;
    s_ok[i] = ok;
}

static inline unsigned nb256(int64_t n) { return (unsigned)((n + 255) / 256); }

cudaError_t launch_preprocess(int64_t P, const float* means, const float* scales, const float* rots,
                              const float* weights, float sm, float* conics_out, float4* boxes_out, cudaStream_t st) {
    if (P <= 0) return cudaSuccess;
    k_preprocess<<<nb256(P), 256, 0, st>>>(P, means, scales, rots, weights, sm, conics_out, boxes_out); gvc::note_launch();
    return cudaGetLastError();
}

cudaError_t launch_gather_recs(int64_t P, const int32_t* perm, const float* means, const float* values,
                               const float* weights, const float* conics, const float4* boxes, GaussRec* recs,
                               cudaStream_t st) {
    if (P <= 0) return cudaSuccess;
    k_gather_recs<<<nb256(P), 256, 0, st>>>(P, perm, means, values, weights, conics, boxes, recs); gvc::note_launch();
    return cudaGetLastError();
}

cudaError_t launch_sample_tiles(int64_t S, int64_t n_tiles, const float* samples, const int32_t* perm,
                                const uint32_t* skeys, float4* s_sorted, float4* group_boxes, uint32_t* group_keys,
                                uint32_t* gdesc, bool with_groups, cudaStream_t st) {
    if (n_tiles <= 0) return cudaSuccess;
    k_sample_tiles<<<nb256(n_tiles * 32), 256, 0, st>>>(S, n_tiles, samples, perm, skeys, s_sorted, group_boxes,
                                                        group_keys, gdesc, with_groups ? 1 : 0); gvc::note_launch();
    return cudaGetLastError();
}

cudaError_t launch_sample_grads(int64_t n_slots, const float4* s_sorted, const float2* out_sorted,
                                const float* out_cells, const float* out_weights, const float* gout, const float* gw,
                                float4* s_grad, float* s_gyz, uint8_t* s_ok, cudaStream_t st) {
    if (n_slots <= 0) return cudaSuccess;
    k_sample_grads<<<nb256(n_slots), 256, 0, st>>>(n_slots, s_sorted, out_sorted, out_cells, out_weights, gout, gw,
                                                   s_grad, s_gyz, s_ok); gvc::note_launch();
    return cudaGetLastError();
}

cudaError_t launch_fill_zero_outputs(int64_t S, float* out_cells, float* out_weights, cudaStream_t st) {
    if (S <= 0) return cudaSuccess;
    cudaError_t e = cudaMemsetAsync(out_cells, 0, sizeof(float) * S, st);
    if (e != cudaSuccess) return e;
    return cudaMemsetAsync(out_weights, 0, sizeof(float) * S, st);
}

}  // namespace gvc
