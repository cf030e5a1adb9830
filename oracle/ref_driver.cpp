// ref_driver.cpp -- C entry points over the reference's own rasterizer code compiled for
// the host (TEST INFRASTRUCTURE ONLY; built into oracle/_ref/libgvc_ref.so by
// oracle/build_ref.py, never linked into the product library).
//
// The functions called here are the reference's, from its unmodified source text:
//   FORWARD::preprocess  diff-gaussian-rasterization/cuda_rasterizer/forward.cu:276-295
//                        (preprocessCUDA, forward.cu:10-114: conic and AABB)
//   FORWARD::render      forward.cu:297-324 with use_gaussian_bvh = true
//                        (sampleRenderCUDA, forward.cu:185-259: per-pair power, window,
//                        exp, accumulation and the 0.01 cutoff)
//   BACKWARD::render     backward.cu:561-622 with use_gaussian_bvh = true
//                        (sampleRenderCUDA, backward.cu:339-559: per-pair adjoint with
//                        atomicAdd; preprocessCUDA, backward.cu:9-125: covariance adjoint)
// in the order rasterizer_impl.cu:65-104 and :288-312 call them.  What stands in for the
// absent third-party code: the BVH is a uniform-grid index answering the same box query
// (every Gaussian whose closed AABB contains the sample, ascending index); glm is a
// minimal column-major stand-in; kernel launches loop over the threads on the host.
#include <cstring>
#include <vector>

#include "backward.h"
#include "cuBQL/refshim_grid.h"
#include "forward.h"

thread_local uint3 threadIdx;
thread_local uint3 blockIdx;
thread_local dim3 blockDim;
thread_local dim3 gridDim;
int ref_serial = 0;

extern "C" {

// 1 when built with OpenMP.
int gvc_ref_openmp(void) {
#ifdef _OPENMP
    return 1;
#else
    return 0;
#endif
}

// nthreads > 0 sets the OpenMP thread count; serial != 0 runs every launch on one thread
// in launch order (then the backward's atomic sums are reproducible).
void gvc_ref_config(int nthreads, int serial) {
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#else
    (void)nthreads;
#endif
    ref_serial = serial;
}

// conics [P*6], aabbs [P*6] (lo xyz, hi xyz).
void gvc_ref_preprocess(int P, const float* means, const float* scales, float scale_modifier, const float* rots,
                        const float* weights, float* conics, float* aabbs) {
    if (P <= 0) return;
    FORWARD::preprocess(P, means, reinterpret_cast<const glm::vec3*>(scales), scale_modifier,
                        reinterpret_cast<const glm::vec4*>(rots), weights, conics,
                        reinterpret_cast<cuBQL::box3f*>(aabbs));
}

// Gaussian-BVH forward: out, outw [S]; counts [S] may be null.
void gvc_ref_forward(int P, int S, const float* means, const float* values, const float* weights,
                     const float* samples, const float* conics, const float* aabbs, float* out, float* outw,
                     int* counts) {
    if (S <= 0) return;
    cuBQL::RefGrid grid;
    grid.build(aabbs, P);
    cuBQL::bvh3f bvh;
    bvh.grid = &grid;
    std::vector<int> cnt(counts ? 0 : S);
    FORWARD::render(P, S, means, values, weights, samples, conics, reinterpret_cast<const cuBQL::box3f*>(aabbs),
                    bvh, out, outw, counts ? counts : cnt.data(), true);
}

// Gaussian-BVH backward.  Every gradient output is zeroed here first (the reference's
// wrapper allocates them with torch::zeros, rasterize_points.cu:102-106).
void gvc_ref_backward(int P, int S, const float* means, const float* scales, float scale_modifier,
                      const float* rots, const float* conics, const float* values, const float* weights,
                      const float* aabbs, const float* samples, const float* out_cells, const float* out_weights,
                      const float* dL_dout, const float* dL_doutw, float* dmeans, float* dvalues, float* dweights,
                      float* dscales, float* drots, float* dconics) {
    std::memset(dmeans, 0, sizeof(float) * 3 * (size_t)P);
    std::memset(dvalues, 0, sizeof(float) * (size_t)P);
    std::memset(dweights, 0, sizeof(float) * (size_t)P);
    std::memset(dscales, 0, sizeof(float) * 3 * (size_t)P);
    std::memset(drots, 0, sizeof(float) * 4 * (size_t)P);
    std::memset(dconics, 0, sizeof(float) * 6 * (size_t)P);
    if (P <= 0) return;
    cuBQL::RefGrid grid;
    grid.build(aabbs, P);
    cuBQL::bvh3f bvh;
    bvh.grid = &grid;
    std::vector<int> cnt(S > 0 ? S : 1);
    const float3 zero{0.f, 0.f, 0.f};
    BACKWARD::render(P, S, means, reinterpret_cast<const glm::vec3*>(scales), scale_modifier,
                     reinterpret_cast<const glm::vec4*>(rots), conics, values, weights, zero, zero, samples, bvh,
                     out_cells, out_weights, dL_dout, dL_doutw, dmeans, dvalues, dweights,
                     reinterpret_cast<glm::vec3*>(dscales), reinterpret_cast<glm::vec4*>(drots), dconics, cnt.data(),
                     true);
}

}  // extern "C"
