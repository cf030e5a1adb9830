// pair.cuh -- the arithmetic of one (sample, Gaussian) pair shared by the forward and the
// backward kernels: the base-2 power with staged coefficients, its window, and the
// backward's moment accumulation.
#pragma once
#include "gvc_internal.cuh"

namespace gvc {

__device__ __forceinline__ float ex2_approx(float x) {
    float y;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

// -0.5 * log2(e): folds the -1/2 of the power (forward.cu:234) and the change of base
// of the exponential into the staged conic, so the power arrives in base 2.
constexpr float kHalfLog2e = -0.72134752044448170368f;
// The power floor -14 (forward.cu:235) in base 2.
constexpr float kLog2Floor = -20.197570572173914f;

// --------------------------------------------------------------------------------
// Backward pair math.  For a pair (sample x, Gaussian g) with d = x - mu and the base-2
// power p2 evaluated exactly as in the forward (same staged coefficients, same window),
// e = 2^p2 and gs = (v gx + gyz) e, the Gaussian accumulates eleven moments
//   m0 = sum gx e, m1 = sum gs, m2..4 = sum gs d, m5..10 = sum gs (dx dx, dx dy, dx dz, dy dy, dy dz, dz dz)
// and moments_to_terms() turns them into the per-Gaussian sums of backward.cu:252-298:
//   dL/dv = w m0, dL/dw = m1, dL/dmu = w C (m2, m3, m4),
//   dL/dconic (unique entries, off-diagonals counted twice) = -w/2 m5, -w m6, -w m7, -w/2 m8, -w m9, -w/2 m10.
// The weight w and the conic multiply once per Gaussian instead of once per pair.
// --------------------------------------------------------------------------------
struct GaussB {
    float mx, my, mz, v;
    float q0, q1, q2, q3, q4, q5;  // base-2 power coefficients, off-diagonals doubled
    float lx, ly, lz, hx, hy, hz;  // AABB
};

__device__ __forceinline__ GaussB gauss_b(float mx, float my, float mz, float v, float c0, float c1, float c2,
                                          float c3, float c4, float c5, float4 lo, float4 hi) {
    GaussB g;
    g.mx = mx; g.my = my; g.mz = mz; g.v = v;
    g.q0 = kHalfLog2e * c0;
    g.q1 = 2.f * (kHalfLog2e * c1);
    g.q2 = 2.f * (kHalfLog2e * c2);
    g.q3 = kHalfLog2e * c3;
    g.q4 = 2.f * (kHalfLog2e * c4);
    g.q5 = kHalfLog2e * c5;
    g.lx = lo.x; g.ly = lo.y; g.lz = lo.z;
    g.hx = hi.x; g.hy = hi.y; g.hz = hi.z;
    return g;
}

// p = (x, y, z, gx) with finite coordinates; gx = gyz = 0 makes every term exactly 0.
// Branch-free: a pair outside the box or the power window gets e = 0.  Returns whether
// the pair is inside the box and the window.
__device__ __forceinline__ bool pair_moments(const GaussB& g, float4 p, float gyz, float (&m)[11]) {
    const bool in = g.lx <= p.x && p.x <= g.hx && g.ly <= p.y && p.y <= g.hy && g.lz <= p.z && p.z <= g.hz;
    const float dx = p.x - g.mx, dy = p.y - g.my, dz = p.z - g.mz;
    const float p2 = dx * fmaf(g.q0, dx, fmaf(g.q1, dy, g.q2 * dz)) + dy * fmaf(g.q3, dy, g.q4 * dz) + dz * (g.q5 * dz);
    const bool c = in && p2 >= kLog2Floor && p2 <= 0.0f;
    const float e = c ? ex2_approx(p2) : 0.0f;
    m[0] = fmaf(p.w, e, m[0]);
    const float gs = fmaf(g.v, p.w, gyz) * e;
    m[1] += gs;
    const float gx = gs * dx, gy = gs * dy, gz = gs * dz;
    m[2] += gx;
    m[3] += gy;
    m[4] += gz;
    m[5] = fmaf(gx, dx, m[5]);
    m[6] = fmaf(gx, dy, m[6]);
    m[7] = fmaf(gx, dz, m[7]);
    m[8] = fmaf(gy, dy, m[8]);
    m[9] = fmaf(gy, dz, m[9]);
    m[10] = fmaf(gz, dz, m[10]);
    return c;
}

// After warp_transpose_reduce16 lanes 2k, 2k+1 hold moment k; returns gradient field k
// (0 dv, 1 dw, 2..4 dmean, 5..10 dconic; 0 for k >= 11).  Warp-collective.
__device__ __forceinline__ float moments_to_terms(float tot, float w, float c0, float c1, float c2, float c3,
                                                  float c4, float c5) {
    const int k = (threadIdx.x & 31) >> 1;
    const float a2 = __shfl_sync(0xffffffffu, tot, 4), a3 = __shfl_sync(0xffffffffu, tot, 6),
                a4 = __shfl_sync(0xffffffffu, tot, 8);
    if (k == 0) return w * tot;
    if (k == 1) return tot;
    if (k == 2) return w * (c0 * a2 + c1 * a3 + c2 * a4);
    if (k == 3) return w * (c1 * a2 + c3 * a3 + c4 * a4);
    if (k == 4) return w * (c2 * a2 + c4 * a3 + c5 * a4);
    if (k == 5 || k == 8 || k == 10) return -0.5f * w * tot;
    if (k == 6 || k == 7 || k == 9) return -w * tot;
    return 0.f;
}

// Per-lane form of moments_to_terms: all eleven gradient fields of one Gaussian from its
// own moments m (0 dv, 1 dw, 2..4 dmean, 5..10 dconic).
__device__ __forceinline__ void moments_to_terms_lane(const float (&m)[11], float w, float c0, float c1, float c2,
                                                      float c3, float c4, float c5, float (&t)[11]) {
    t[0] = w * m[0];
    t[1] = m[1];
    t[2] = w * (c0 * m[2] + c1 * m[3] + c2 * m[4]);
    t[3] = w * (c1 * m[2] + c3 * m[3] + c4 * m[4]);
    t[4] = w * (c2 * m[2] + c4 * m[3] + c5 * m[4]);
    t[5] = -0.5f * w * m[5];
    t[6] = -w * m[6];
    t[7] = -w * m[7];
    t[8] = -0.5f * w * m[8];
    t[9] = -w * m[9];
    t[10] = -0.5f * w * m[10];
}

}  // namespace gvc
