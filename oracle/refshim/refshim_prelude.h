// refshim_prelude.h -- host stand-ins that let the reference's CUDA rasterizer sources
// (diff-gaussian-rasterization/cuda_rasterizer/forward.cu, backward.cu) compile as plain
// C++ for the CPU.  TEST INFRASTRUCTURE ONLY (oracle/_ref, built by oracle/build_ref.py).
//
// What is emulated:
//   * CUDA qualifiers (__global__, __device__, __forceinline__) become host inline code;
//   * the built-in vector types float3/float4, dim3 and the thread coordinates
//     threadIdx/blockIdx/blockDim/gridDim (thread-local, set by ref_launch);
//   * a kernel launch `k<<<grid, block>>>(args)` (rewritten by the recipe into
//     ref_launch(grid, block, k, args)) runs every thread of every block in turn, blocks
//     spread over OpenMP threads.  Within each warp the lanes run from 31 down to 0, so
//     that a warp reduction (cooperative_groups/reduce.h) can hand lane 0 the sum of the
//     lanes that ran before it; the kernels use no shared memory and no block barriers;
//   * CUDA's float min/max (fminf/fmaxf: a NaN operand is dropped) and atomicAdd;
//   * the float overloads of exp/abs/sqrt that CUDA device code resolves to.
#pragma once
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <iostream>
#include <stdexcept>
#include <utility>
#ifdef _OPENMP
#include <omp.h>
#endif

#define __global__
#define __device__
#define __host__
#define __forceinline__ inline

using std::abs;
using std::exp;
using std::sqrt;

typedef unsigned int uint;

struct float3 {
    float x, y, z;
};
struct float4 {
    float x, y, z, w;
};
struct uint3 {
    unsigned x, y, z;
};
struct dim3 {
    unsigned x, y, z;
    dim3(unsigned x_ = 1, unsigned y_ = 1, unsigned z_ = 1) : x(x_), y(y_), z(z_) {}
};
inline float3 make_float3(float x, float y, float z) { return float3{x, y, z}; }
inline float4 make_float4(float x, float y, float z, float w) { return float4{x, y, z, w}; }

// CUDA's min/max on floats are fminf/fmaxf; the integer forms are the usual ones.
inline float min(float a, float b) { return fminf(a, b); }
inline float max(float a, float b) { return fmaxf(a, b); }
inline int min(int a, int b) { return a < b ? a : b; }
inline int max(int a, int b) { return a > b ? a : b; }

extern thread_local uint3 threadIdx;
extern thread_local uint3 blockIdx;
extern thread_local dim3 blockDim;
extern thread_local dim3 gridDim;

// Set by the driver: when nonzero, atomicAdd is a plain add and launches run on one
// thread in launch order (reproducible sums).
extern int ref_serial;
// Incremented before every emulated thread runs (resets the warp-reduction call count).
extern thread_local unsigned long long ref_thread_epoch;

inline float atomicAdd(float* p, float v) {
    float old;
    if (ref_serial) {
        old = *p;
        *p = old + v;
        return old;
    }
#pragma omp atomic capture
    {
        old = *p;
        *p += v;
    }
    return old;
}
inline int atomicAdd(int* p, int v) {
    int old;
#pragma omp atomic capture
    {
        old = *p;
        *p += v;
    }
    return old;
}

template <class K, class... A>
inline void ref_run_block(long b, dim3 grid, dim3 block, K kernel, A... args) {
    blockIdx = uint3{(unsigned)b, 0u, 0u};
    blockDim = block;
    gridDim = grid;
    for (unsigned w = 0; w * 32 < block.x; w++) {
        for (int l = 31; l >= 0; l--) {
            const unsigned t = w * 32 + (unsigned)l;
            if (t >= block.x) continue;
            threadIdx = uint3{t, 0u, 0u};
            ref_thread_epoch++;
            kernel(args...);
        }
    }
}

template <class K, class... A>
void ref_launch(dim3 grid, dim3 block, K kernel, A... args) {
    const long nb = (long)grid.x;
    if (ref_serial) {
        for (long b = 0; b < nb; b++) ref_run_block(b, grid, block, kernel, args...);
        return;
    }
#pragma omp parallel for schedule(dynamic, 4)
    for (long b = 0; b < nb; b++) ref_run_block(b, grid, block, kernel, args...);
}
