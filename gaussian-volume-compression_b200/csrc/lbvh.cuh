// lbvh.cuh -- LBVH builder interface shared by the Gaussian, sample-tile and cell BVHs.
#pragma once
#include "gvc_internal.cuh"

namespace gvc {

// Stable radix sort of L.keys[0..n) (uint32); result in L.keys (sorted) and L.perm
// (sorted position -> input index).
cudaError_t radix_sort_pairs(Lbvh& L, int64_t n, cudaStream_t st);

// Stable LSD sort of n indices by a key of several 32-bit words (words[0] least
// significant); bits[w] = significant bits of word w (ceil(bits / 8) radix passes).
// Result in L.perm (sorted position -> input index); L.keys / keys_alt are scratch.
cudaError_t radix_sort_words(Lbvh& L, int64_t n, const uint32_t* const* words, const int* bits, int nwords,
                             cudaStream_t st);

// 30-bit Morton keys of box centroids over the centroid bounds, then sort.
cudaError_t morton_sort_boxes(Lbvh& L, int64_t n, const float4* boxes, cudaStream_t st);
// Same for points [n][3].
cudaError_t morton_sort_points(Lbvh& L, int64_t n, const float* pts, cudaStream_t st);

// Karras hierarchy + refit + node packing over keys/leaf boxes already in sorted order.
cudaError_t lbvh_hierarchy(Lbvh& L, int64_t n, const uint32_t* sorted_keys, const float4* sorted_leaf_boxes,
                           cudaStream_t st);

// Full build from boxes in input order: keys, sort, gather, hierarchy.
cudaError_t lbvh_build_boxes(Lbvh& L, int64_t n, const float4* boxes, cudaStream_t st);

}  // namespace gvc
