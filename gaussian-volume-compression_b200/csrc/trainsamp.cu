// trainsamp.cu -- training sample batches generated on the device.
//
// The reference builds its training samples once, with host round trips in between
// (train.py:34-61 sample_mesh_points, :273-282 ground truth through gpu_sampleu on host
// arrays, :286-315 per-batch 21-bit Morton sort):
//   1. pick a random tetrahedron of the triangulated mesh for every point, uniform over
//      cells; draw three uniforms, sort them, take their gaps as barycentric weights
//      (b0 = u0, b1 = u1 - u0, b2 = u2 - u1, b3 = 1 - u2) and interpolate the vertices;
//   2. sample the mesh's point field at the points (locate + interpolate, -1 outside);
//   3. per batch, sort points and values by the 63-bit Morton code of the clamped
//      coordinates (q = int64(clamp(x, 0, 1) * (2^21 - 1)) per axis, interleaved).
// Here all three run on the device with no host copy.  Differences, declared:
//   * random numbers come from Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel
//     random numbers: as easy as 1, 2, 3", SC 2011), counter = (point index, 0, block, 0),
//     key = the 64-bit seed, instead of torch's generator state: the same distribution,
//     not the same stream.  The cell is floor(r64 * C / 2^64) from two 32-bit words; a
//     uniform is (r >> 8) * 2^-24, a multiple of 2^-24 in [0, 1), so the gaps are exact;
//   * the vertex interpolation is ((b0 v0 + b1 v1) + b2 v2) + b3 v3 per axis, every
//     operation rounded;
//   * the Morton sort is stable (the reference's argsort is not: points with equal codes
//     may come out in another order there);
//   * the ground truth is located in the sorted order (coherent traversal) and converted
//     to float32, as the reference's torch.tensor(big_gt, dtype=float) does.
#include "lbvh.cuh"
#include "render.cuh"

namespace gvc {

namespace {

__device__ __forceinline__ void philox4x32_10(uint32_t c[4], uint32_t k0, uint32_t k1) {
#pragma unroll
    for (int r = 0; r < 10; r++) {
        if (r) {
            k0 += 0x9E3779B9u;
            k1 += 0xBB67AE85u;
        }
        const uint32_t lo0 = 0xD2511F53u * c[0], hi0 = __umulhi(0xD2511F53u, c[0]);
        const uint32_t lo1 = 0xCD9E8D57u * c[2], hi1 = __umulhi(0xCD9E8D57u, c[2]);
        const uint32_t n0 = hi1 ^ c[1] ^ k0, n2 = hi0 ^ c[3] ^ k1;
        c[0] = n0;
        c[1] = lo1;
        c[2] = n2;
        c[3] = lo0;
    }
}

__device__ __forceinline__ float unit24(uint32_t r) { return __uint2float_rn(r >> 8) * 5.9604644775390625e-8f; }

__device__ __forceinline__ uint64_t part1by2_21(uint64_t n) {
    n &= 0x1fffffull;
    n = (n | (n << 32)) & 0x1f00000000ffffull;
    n = (n | (n << 16)) & 0x1f0000ff0000ffull;
    n = (n | (n << 8)) & 0x100f00f00f00f00full;
    n = (n | (n << 4)) & 0x10c30c30c30c30c3ull;
    n = (n | (n << 2)) & 0x1249249249249249ull;
    return n;
}

__device__ __forceinline__ uint64_t quant21(float x) {
    // clamp to [0, 1] (NaN stays NaN and converts to 0), times 2^21 - 1 in float32, truncate
    const float c = fminf(fmaxf(x, 0.f), 1.f);
    const float v = __fmul_rn(c, 2097151.0f);
    return v == v ? (uint64_t)v : 0ull;
}

// One thread per point t of batch t / S: random tet, barycentric point, Morton words.
__global__ void __launch_bounds__(256) k_tet_points(int64_t N, int64_t S, uint64_t seed, const float* __restrict__ pts,
                                                    const int32_t* __restrict__ conn4, int64_t C,
                                                    float* __restrict__ out, uint32_t* __restrict__ w_lo,
                                                    uint32_t* __restrict__ w_hi, uint32_t* __restrict__ w_batch) {
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t >= N) return;
    const uint32_t k0 = (uint32_t)seed, k1 = (uint32_t)(seed >> 32);
    uint32_t a[4] = {(uint32_t)t, (uint32_t)((uint64_t)t >> 32), 0u, 0u};
    uint32_t b[4] = {(uint32_t)t, (uint32_t)((uint64_t)t >> 32), 1u, 0u};
    philox4x32_10(a, k0, k1);
    philox4x32_10(b, k0, k1);
    const uint64_t r64 = ((uint64_t)a[0] << 32) | a[1];
    const int64_t cell = (int64_t)__umul64hi(r64, (uint64_t)C);
    float u0 = unit24(a[2]), u1 = unit24(a[3]), u2 = unit24(b[0]);
    // sort three values ascending
    float lo = fminf(u0, u1), hi = fmaxf(u0, u1);
    u0 = fminf(lo, u2);
    const float m = fmaxf(lo, u2);
    u1 = fminf(m, hi);
    u2 = fmaxf(m, hi);
    const float w[4] = {u0, __fsub_rn(u1, u0), __fsub_rn(u2, u1), __fsub_rn(1.0f, u2)};
    const int32_t* cv = conn4 + 4 * cell;
    float p[3];
#pragma unroll
    for (int ax = 0; ax < 3; ax++) {
        float s = __fmul_rn(w[0], pts[3 * (int64_t)cv[0] + ax]);
        s = __fadd_rn(s, __fmul_rn(w[1], pts[3 * (int64_t)cv[1] + ax]));
        s = __fadd_rn(s, __fmul_rn(w[2], pts[3 * (int64_t)cv[2] + ax]));
        s = __fadd_rn(s, __fmul_rn(w[3], pts[3 * (int64_t)cv[3] + ax]));
        p[ax] = s;
        out[3 * t + ax] = s;
    }
    const uint64_t key = part1by2_21(quant21(p[0])) | (part1by2_21(quant21(p[1])) << 1) |
                         (part1by2_21(quant21(p[2])) << 2);
    w_lo[t] = (uint32_t)key;
    w_hi[t] = (uint32_t)(key >> 32);
    w_batch[t] = (uint32_t)(t / S);
}

__global__ void __launch_bounds__(256) k_gather_points(int64_t N, const float* __restrict__ src,
                                                       const int32_t* __restrict__ perm, float* __restrict__ dst) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= N) return;
    const int64_t s = perm[i];
    dst[3 * i] = src[3 * s];
    dst[3 * i + 1] = src[3 * s + 1];
    dst[3 * i + 2] = src[3 * s + 2];
}

__global__ void __launch_bounds__(256) k_to_f32(int64_t N, const double* __restrict__ src, float* __restrict__ dst) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < N) dst[i] = (float)src[i];
}

inline unsigned nblk(int64_t n, int t) { return (unsigned)((n + t - 1) / t); }

}  // namespace

cudaError_t launch_tet_points(int64_t N, int64_t S, uint64_t seed, const float* pts, const int32_t* conn4, int64_t C,
                              float* out, uint32_t* w_lo, uint32_t* w_hi, uint32_t* w_batch, cudaStream_t st) {
    if (N <= 0) return cudaSuccess;
    k_tet_points<<<nblk(N, 256), 256, 0, st>>>(N, S, seed, pts, conn4, C, out, w_lo, w_hi, w_batch);
    gvc::note_launch();
    return cudaGetLastError();
}

cudaError_t launch_gather_points(int64_t N, const float* src, const int32_t* perm, float* dst, cudaStream_t st) {
    if (N <= 0) return cudaSuccess;
    k_gather_points<<<nblk(N, 256), 256, 0, st>>>(N, src, perm, dst); gvc::note_launch();
    return cudaGetLastError();
}

cudaError_t launch_to_f32(int64_t N, const double* src, float* dst, cudaStream_t st) {
    if (N <= 0) return cudaSuccess;
    k_to_f32<<<nblk(N, 256), 256, 0, st>>>(N, src, dst); gvc::note_launch();
    return cudaGetLastError();
}

}  // namespace gvc
