// lbvh.cuh -- LBVH builder interface shared by the Gaussian, sample-tile and cell BVHs.
#pragma once
#include "gvc_internal.cuh"

namespace gvc {

// Radix sort tile: 8 warps x 16 iterations x 32 lanes = 4096 keys per block.
constexpr int kRsWarps = 8;
constexpr int kRsIters = 16;
constexpr int kRsTile = kRsWarps * kRsIters * 32;

// Bytes each Lbvh buffer must hold for an LBVH build over n boxes (lbvh_build_boxes);
// the builder sizes its buffers with exactly these, and callers that provide the buffers
// themselves (the allocation-free sampler) check their views against them.
struct LbvhBytes {
    static constexpr int64_t internal(int64_t n) { return n > 1 ? n - 1 : 1; }
    static constexpr size_t keys(int64_t n) { return sizeof(uint32_t) * (size_t)n; }  // keys, keys_alt, perm, perm_alt
    static constexpr size_t hist(int64_t n) {
        return sizeof(uint32_t) * (256 * (size_t)((n + kRsTile - 1) / kRsTile) + 256);
    }
    static constexpr size_t bounds() { return sizeof(uint32_t) * 8; }
    static constexpr size_t sorted_boxes(int64_t n) { return 2 * 16 * (size_t)n; }
    static constexpr size_t child(int64_t n) { return sizeof(int32_t) * (size_t)internal(n); }  // left, right, flags
    static constexpr size_t parent(int64_t n) { return sizeof(int32_t) * 2 * (size_t)n; }
    static constexpr size_t node_boxes(int64_t n) { return 2 * 16 * (size_t)internal(n); }
    static constexpr size_t nodes(int64_t n) { return sizeof(BvhNode) * (size_t)internal(n); }
};

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
