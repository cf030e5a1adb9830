// ref_driver.cpp -- C entry points over the reference's own rasterizer code compiled for
// the host (TEST INFRASTRUCTURE ONLY; built into oracle/_ref/libgvc_ref.so by
// oracle/build_ref.py, never linked into the product library).
//
// The functions called here are the reference's, from its unmodified source text:
//   FORWARD::preprocess  diff-gaussian-rasterization/cuda_rasterizer/forward.cu:276-295
//                        (preprocessCUDA, forward.cu:10-114: conic and AABB)
//   FORWARD::render      forward.cu:297-348, both modes:
//                        use_gaussian_bvh = true: sampleRenderCUDA (forward.cu:185-259,
//                        thread per sample: power, window, exp, sums, 0.01 cutoff);
//                        false: renderCUDA + normalizeCUDA (forward.cu:116-182, 261-274,
//                        warp per Gaussian, atomicAdd into the samples)
//   BACKWARD::render     backward.cu:561-659, both modes:
//                        true: sampleRenderCUDA (backward.cu:339-559, thread per sample,
//                        atomicAdd into the Gaussians); false: renderCUDA (backward.cu:
//                        127-337, warp per Gaussian, warp reductions); then
//                        preprocessCUDA (backward.cu:9-125: covariance adjoint)
// in the order rasterizer_impl.cu:65-104 and :288-312 call them.  What stands in for the
// absent third-party code: each BVH is a uniform-grid index answering the same box
// queries (the Gaussians whose closed AABB contains a sample; the samples inside a
// Gaussian's closed AABB; ascending index); glm is a minimal column-major stand-in;
// kernel launches loop over the threads on the host.
#include <cstring>
#include <vector>

#include "backward.h"
#include "cuBQL/refshim_grid.h"
#include "forward.h"

// The Gaussian index: the reference builds its Gaussian BVH in the forward
// (rasterizer_impl.cu:79-83) and the backward reuses that module-global BVH
// (ext.cu:8-10); gvc_ref_forward builds this index and gvc_ref_backward reuses it when
// it was built over the same boxes.
// The sample index stands in for the sample BVH that build_bvh makes once per batch
// (ext.cu:28-65) and both passes use.
struct CachedIndex {
    cuBQL::RefGrid grid;
    std::vector<float> key;
};
static CachedIndex g_gauss, g_samples;

static const cuBQL::RefGrid& index_for(CachedIndex& c, const std::vector<float>& boxes, int64_t n) {
    if (c.key.size() != boxes.size() || std::memcmp(c.key.data(), boxes.data(), boxes.size() * sizeof(float)) != 0) {
        c.key = boxes;
        c.grid = cuBQL::RefGrid();
        c.grid.build(boxes.data(), n);
    }
    return c.grid;
}

static const cuBQL::RefGrid& gaussian_index(const float* aabbs, int P) {
    return index_for(g_gauss, std::vector<float>(aabbs, aabbs + 6 * (size_t)P), P);
}

static const cuBQL::RefGrid& sample_index(const float* samples, int S) {
    std::vector<float> b(6 * (size_t)S);
    for (int64_t i = 0; i < S; i++)
        for (int a = 0; a < 3; a++) b[6 * i + a] = b[6 * i + 3 + a] = samples[3 * i + a];
    return index_for(g_samples, b, S);
}

thread_local uint3 threadIdx;
thread_local uint3 blockIdx;
thread_local dim3 blockDim;
thread_local dim3 gridDim;
thread_local unsigned long long ref_thread_epoch = 0;
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

// Forward: out, outw [S] (zeroed here first, as the wrapper's torch::zeros,
// rasterize_points.cu:44-45); counts (S entries in the Gaussian-BVH mode, P otherwise)
// may be null.
void gvc_ref_forward(int P, int S, const float* means, const float* values, const float* weights,
                     const float* samples, const float* conics, const float* aabbs, float* out, float* outw,
                     int* counts, int use_gaussian_bvh) {
    std::memset(out, 0, sizeof(float) * (size_t)(S > 0 ? S : 0));
    std::memset(outw, 0, sizeof(float) * (size_t)(S > 0 ? S : 0));
    if (S <= 0 || P <= 0) return;
    cuBQL::bvh3f bvh;
    bvh.grid = use_gaussian_bvh ? &gaussian_index(aabbs, P) : &sample_index(samples, S);
    std::vector<int> cnt(counts ? 0 : (use_gaussian_bvh ? S : P));
    FORWARD::render(P, S, means, values, weights, samples, conics, reinterpret_cast<const cuBQL::box3f*>(aabbs),
                    bvh, out, outw, counts ? counts : cnt.data(), use_gaussian_bvh != 0);
}

// Backward.  Every gradient output is zeroed here first (the reference's
// wrapper allocates them with torch::zeros, rasterize_points.cu:102-106).
void gvc_ref_backward(int P, int S, const float* means, const float* scales, float scale_modifier,
                      const float* rots, const float* conics, const float* values, const float* weights,
                      const float* aabbs, const float* samples, const float* out_cells, const float* out_weights,
                      const float* dL_dout, const float* dL_doutw, float* dmeans, float* dvalues, float* dweights,
                      float* dscales, float* drots, float* dconics, int use_gaussian_bvh) {
    std::memset(dmeans, 0, sizeof(float) * 3 * (size_t)P);
    std::memset(dvalues, 0, sizeof(float) * (size_t)P);
    std::memset(dweights, 0, sizeof(float) * (size_t)P);
    std::memset(dscales, 0, sizeof(float) * 3 * (size_t)P);
    std::memset(drots, 0, sizeof(float) * 4 * (size_t)P);
    std::memset(dconics, 0, sizeof(float) * 6 * (size_t)P);
    if (P <= 0) return;
    cuBQL::bvh3f bvh;
    bvh.grid = use_gaussian_bvh ? &gaussian_index(aabbs, P) : &sample_index(samples, S);
    std::vector<int> cnt(use_gaussian_bvh ? (S > 0 ? S : 1) : P);
    const float3 zero{0.f, 0.f, 0.f};
    BACKWARD::render(P, S, means, reinterpret_cast<const glm::vec3*>(scales), scale_modifier,
                     reinterpret_cast<const glm::vec4*>(rots), conics, values, weights, zero, zero, samples, bvh,
                     out_cells, out_weights, dL_dout, dL_doutw, dmeans, dvalues, dweights,
                     reinterpret_cast<glm::vec3*>(dscales), reinterpret_cast<glm::vec4*>(drots), dconics, cnt.data(),
                     use_gaussian_bvh != 0);
}

}  // extern "C"
