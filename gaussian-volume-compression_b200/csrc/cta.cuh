// cta.cuh -- pieces shared by the CTA-level kernels on 128-sample blocks (the FP32 forward
// in cta.cu, the tensor-core forward in fwd_tc.cu): block-group descriptors, box helpers.
#pragma once
#include "render.cuh"

namespace gvc {

constexpr int kBlockRows = 128;
constexpr int kBlockGroups = 8;

struct Box6 {
    float lx, ly, lz, hx, hy, hz;
};

// Box of the lanes with `in` set (empty box if none), on every lane of the warp.
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

__device__ __forceinline__ bool overlap6(const Box6& b, float4 lo, float4 hi) {
    return lo.x <= b.hx && hi.x >= b.lx && lo.y <= b.hy && hi.y >= b.ly && lo.z <= b.hz && hi.z >= b.lz;
}

// First row of block group g (kBlockRows past the last group) from the block descriptor
// written by k_sample_blocks: bytes 0..6 = starts of groups 1..7, byte 7 = group count.
__device__ __forceinline__ int group_start(uint2 d, int g) {
    if (g == 0) return 0;
    if (g >= kBlockGroups) return kBlockRows;
    if (g <= 4) return (int)((d.x >> (8 * (g - 1))) & 0xffu);
    return (int)((d.y >> (8 * (g - 5))) & 0xffu);
}

__device__ __forceinline__ int group_count(uint2 d) { return (int)(d.y >> 24); }

// The group of row r (rows of a group are contiguous; groups are in order).
__device__ __forceinline__ int group_of(uint2 d, int r) {
    const int ng = group_count(d);
    int g = 0;
#pragma unroll
    for (int k = 1; k < kBlockGroups; k++)
        if (k < ng && r >= group_start(d, k)) g = k;
    return g;
}

__device__ __forceinline__ void cp_async16(void* dst, const void* src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(static_cast<uint32_t>(__cvta_generic_to_shared(dst))),
                 "l"(src)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

}  // namespace gvc
