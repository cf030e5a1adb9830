// lbvh.cu -- on-device LBVH construction: 30-bit Morton keys, stable LSD radix sort
// (8-bit digits, warp-aggregated stable ranking; one kernel per pass with decoupled
// look-back, or per-pass block histograms + scan + scatter where no status word is
// given), Karras 2012 hierarchy, atomic bottom-up refit and node packing.
//
// Replaces cuBQL::cuda::radixBuilder as called from
// diff-gaussian-rasterization/cuda_rasterizer/rasterizer_impl.cu:78-83 (Gaussian AABBs)
// and diff-gaussian-rasterization/ext.cu:50-54 (sample points).  The declared ordering
// (keys, tie-break, tree) is restated on the CPU by the oracle and checked bit for bit.
#include "lbvh.cuh"

namespace gvc {

// ----------------------------------------------------------------------------------
// Ordered float <-> uint mapping for atomic min/max of floats.
// ----------------------------------------------------------------------------------
__device__ __forceinline__ uint32_t f2ord(float f) {
    uint32_t b = __float_as_uint(f);
    return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
__device__ __forceinline__ float ord2f(uint32_t u) {
    uint32_t b = (u & 0x80000000u) ? (u & 0x7fffffffu) : ~u;
    return __uint_as_float(b);
}

__device__ __forceinline__ uint32_t expand10(uint32_t v) {
    v &= 0x3ffu;
    v = (v | (v << 16)) & 0x030000FFu;
    v = (v | (v << 8)) & 0x0300F00Fu;
    v = (v | (v << 4)) & 0x030C30C3u;
    v = (v | (v << 2)) & 0x09249249u;
    return v;
}

__device__ __forceinline__ uint32_t quant10(float c, float lo, float scale) {
    float t = __fmul_rn(__fsub_rn(c, lo), scale);
    if (!(t >= 0.0f)) return 0u;
    if (t >= 1023.0f) return 1023u;
    return (uint32_t)t;
}

// Centroid of box i ((lo + hi) * 0.5f) or the point itself.
struct BoxSrc {
    const float4* boxes;  // [n][2] lo, hi
    __device__ __forceinline__ void centroid(int64_t i, float c[3]) const {
        float4 lo = boxes[2 * i], hi = boxes[2 * i + 1];
        c[0] = __fmul_rn(__fadd_rn(lo.x, hi.x), 0.5f);
        c[1] = __fmul_rn(__fadd_rn(lo.y, hi.y), 0.5f);
        c[2] = __fmul_rn(__fadd_rn(lo.z, hi.z), 0.5f);
    }
};
struct PointSrc {
    const float* pts;  // [n][3]
    __device__ __forceinline__ void centroid(int64_t i, float c[3]) const {
        // (p + p) * 0.5f == p exactly for finite p, as for a degenerate box
        float x = pts[3 * i], y = pts[3 * i + 1], z = pts[3 * i + 2];
        c[0] = __fmul_rn(__fadd_rn(x, x), 0.5f);
        c[1] = __fmul_rn(__fadd_rn(y, y), 0.5f);
        c[2] = __fmul_rn(__fadd_rn(z, z), 0.5f);
    }
};

__global__ void k_bounds_init(uint32_t* b) {
    if (threadIdx.x < 3) b[threadIdx.x] = 0xffffffffu;
    else if (threadIdx.x < 6) b[threadIdx.x] = 0u;
}

template <class Src>
__global__ void __launch_bounds__(256) k_bounds(Src src, int64_t n, uint32_t* bounds) {
    uint32_t mn[3] = {0xffffffffu, 0xffffffffu, 0xffffffffu}, mx[3] = {0u, 0u, 0u};
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        float c[3];
        src.centroid(i, c);
#pragma unroll
        for (int a = 0; a < 3; a++) {
            if (c[a] == c[a]) {  // NaN centroids do not move the bounds (fminf semantics)
                uint32_t o = f2ord(c[a]);
                mn[a] = min(mn[a], o);
                mx[a] = max(mx[a], o);
            }
        }
    }
#pragma unroll
    for (int a = 0; a < 3; a++) {
        for (int off = 16; off > 0; off >>= 1) {
            mn[a] = min(mn[a], __shfl_xor_sync(0xffffffffu, mn[a], off));
            mx[a] = max(mx[a], __shfl_xor_sync(0xffffffffu, mx[a], off));
        }
    }
    if ((threadIdx.x & 31) == 0) {
#pragma unroll
        for (int a = 0; a < 3; a++) {
            atomicMin(&bounds[a], mn[a]);
            atomicMax(&bounds[3 + a], mx[a]);
        }
    }
}

template <class Src>
__global__ void __launch_bounds__(256) k_keys(Src src, int64_t n, const uint32_t* bounds, uint32_t* keys) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    float lo[3], scale[3];
#pragma unroll
    for (int a = 0; a < 3; a++) {
        uint32_t ulo = bounds[a], uhi = bounds[3 + a];
        if (ulo == 0xffffffffu) {  // every centroid was NaN
            lo[a] = 0.f;
            scale[a] = 0.f;
            continue;
        }
        lo[a] = ord2f(ulo);
        float hi = ord2f(uhi);
        float ext = __fsub_rn(hi, lo[a]);
        scale[a] = ext > 0.0f ? __fdiv_rn(1024.0f, ext) : 0.0f;
    }
    float c[3];
    src.centroid(i, c);
    uint32_t q0 = quant10(c[0], lo[0], scale[0]);
    uint32_t q1 = quant10(c[1], lo[1], scale[1]);
    uint32_t q2 = quant10(c[2], lo[2], scale[2]);
    keys[i] = expand10(q0) | (expand10(q1) << 1) | (expand10(q2) << 2);
}

// ----------------------------------------------------------------------------------
// Stable LSD radix sort of (uint32 key, int32 value) pairs, 8-bit digits.
//   tile = 8 warps x 16 iterations x 32 lanes = 4096 elements per block.
//   per pass: k_rs_hist (per-block digit counts of the current order),
//   k_rs_scan (per-digit exclusive scan over blocks + digit totals),
//   k_rs_scatter (stable ranks: (warp, iteration, lane) = input order).
// ----------------------------------------------------------------------------------

__device__ __forceinline__ uint32_t lanemask_lt() {
    uint32_t m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

__global__ void __launch_bounds__(256) k_rs_hist(const uint32_t* __restrict__ keys, int64_t n, int nb, int pass,
                                                 uint32_t* __restrict__ hist) {
    __shared__ uint32_t cnt[256];
    for (int t = threadIdx.x; t < 256; t += blockDim.x) cnt[t] = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int shift = 8 * pass;
    int64_t base = (int64_t)blockIdx.x * kRsTile + (int64_t)warp * (kRsIters * 32);
#pragma unroll 4
    for (int it = 0; it < kRsIters; it++) {
        int64_t idx = base + it * 32 + lane;
        bool valid = idx < n;
        uint32_t key = valid ? keys[idx] : 0u;
        uint32_t d = (key >> shift) & 255u;
        uint32_t tag = valid ? d : (256u + lane);
        uint32_t peers = __match_any_sync(0xffffffffu, tag);
        if (valid && (__ffs(peers) - 1) == lane) atomicAdd(&cnt[d], (uint32_t)__popc(peers));
    }
    __syncthreads();
    for (int d = threadIdx.x; d < 256; d += blockDim.x) hist[(int64_t)d * nb + blockIdx.x] = cnt[d];
}

// grid (256 digits), 1024 threads: in-place exclusive scan of one digit's row.
__global__ void __launch_bounds__(1024) k_rs_scan(uint32_t* __restrict__ hist, int nb, uint32_t* __restrict__ totals) {
    const int d = blockIdx.x;
    uint32_t* row = hist + (int64_t)d * nb;
    const int per = (nb + blockDim.x - 1) / blockDim.x;
    const int b0 = threadIdx.x * per;
    uint32_t local = 0;
    for (int k = 0; k < per; k++) {
        int b = b0 + k;
        if (b < nb) local += row[b];
    }
    __shared__ uint32_t wsum[32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t incl = local;
    for (int off = 1; off < 32; off <<= 1) {
        uint32_t v = __shfl_up_sync(0xffffffffu, incl, off);
        if (lane >= off) incl += v;
    }
    if (lane == 31) wsum[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        uint32_t v = lane < (int)(blockDim.x >> 5) ? wsum[lane] : 0u;
        uint32_t vi = v;
        for (int off = 1; off < 32; off <<= 1) {
            uint32_t t = __shfl_up_sync(0xffffffffu, vi, off);
            if (lane >= off) vi += t;
        }
        wsum[lane] = vi - v;  // exclusive warp offsets
        if (lane == 31) totals[d] = vi;
    }
    __syncthreads();
    uint32_t run = wsum[warp] + incl - local;
    for (int k = 0; k < per; k++) {
        int b = b0 + k;
        if (b < nb) {
            uint32_t v = row[b];
            row[b] = run;
            run += v;
        }
    }
}

__global__ void __launch_bounds__(256) k_rs_scatter(const uint32_t* __restrict__ keys_in,
                                                    const int32_t* __restrict__ vals_in, uint32_t* __restrict__ keys_out,
                                                    int32_t* __restrict__ vals_out, int64_t n, int nb, int pass,
                                                    const uint32_t* __restrict__ hist,
                                                    const uint32_t* __restrict__ totals) {
    __shared__ uint32_t wcnt[kRsWarps][256];
    __shared__ uint32_t dbase[256];
    __shared__ uint32_t bstart[256];
    __shared__ uint32_t wsum[kRsWarps];
    __shared__ uint32_t skey[kRsTile];
    __shared__ int32_t sval[kRsTile];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int shift = 8 * pass;
    for (int t = threadIdx.x; t < kRsWarps * 256; t += blockDim.x) (&wcnt[0][0])[t] = 0;
    // digit bases: exclusive scan of the 256 digit totals + this block's row offset
    if (warp == 0) {
        uint32_t run = 0;
        for (int chunk = 0; chunk < 8; chunk++) {
            int d = chunk * 32 + lane;
            uint32_t v = totals[d];
            uint32_t incl = v;
            for (int off = 1; off < 32; off <<= 1) {
                uint32_t t = __shfl_up_sync(0xffffffffu, incl, off);
                if (lane >= off) incl += t;
            }
            dbase[d] = run + incl - v + hist[(int64_t)d * nb + blockIdx.x];
            run += __shfl_sync(0xffffffffu, incl, 31);
        }
    }
    __syncthreads();
    const int64_t base = (int64_t)blockIdx.x * kRsTile + (int64_t)warp * (kRsIters * 32);
    uint32_t kreg[kRsIters];
    int32_t vreg[kRsIters];
    uint32_t rreg[kRsIters];  // (local rank << 8) | digit, or 0xffffffff if invalid
#pragma unroll
    for (int it = 0; it < kRsIters; it++) {
        int64_t idx = base + it * 32 + lane;
        bool valid = idx < n;
        uint32_t key = valid ? keys_in[idx] : 0u;
        int32_t val = valid ? (vals_in ? vals_in[idx] : (int32_t)idx) : 0;
        uint32_t d = (key >> shift) & 255u;
        uint32_t tag = valid ? d : (256u + lane);
        uint32_t peers = __match_any_sync(0xffffffffu, tag);
        uint32_t rank = __popc(peers & lanemask_lt());
        uint32_t pre = valid ? wcnt[warp][d] : 0u;
        __syncwarp();
        if (valid && (__ffs(peers) - 1) == lane) wcnt[warp][d] = pre + __popc(peers);
        __syncwarp();
        kreg[it] = key;
        vreg[it] = val;
        rreg[it] = valid ? (((pre + rank) << 8) | d) : 0xffffffffu;
    }
    __syncthreads();
    // exclusive prefix over warps for each digit; run = this block's count of digit d
    uint32_t run = 0;
    {
        const int d = threadIdx.x;  // 256 threads == 256 digits
#pragma unroll
        for (int w = 0; w < kRsWarps; w++) {
            const uint32_t t = wcnt[w][d];
            wcnt[w][d] = run;
            run += t;
        }
    }
    // block-local start of each digit: exclusive scan of the 256 counts
    {
        uint32_t incl = run;
        for (int off = 1; off < 32; off <<= 1) {
            const uint32_t t = __shfl_up_sync(0xffffffffu, incl, off);
            if (lane >= off) incl += t;
        }
        if (lane == 31) wsum[warp] = incl;
        __syncthreads();
        uint32_t wbase = 0;
        for (int w = 0; w < warp; w++) wbase += wsum[w];
        bstart[threadIdx.x] = wbase + incl - run;
    }
    __syncthreads();
    // place every key at its block-local sorted position, then write the block out in that
    // order: consecutive threads write consecutive addresses of each digit's run
#pragma unroll
    for (int it = 0; it < kRsIters; it++) {
        const uint32_t r = rreg[it];
        if (r != 0xffffffffu) {
            const uint32_t d = r & 255u;
            const uint32_t sp = bstart[d] + wcnt[warp][d] + (r >> 8);
            skey[sp] = kreg[it];
            sval[sp] = vreg[it];
        }
    }
    __syncthreads();
    const int64_t rem = n - (int64_t)blockIdx.x * kRsTile;
    const int cnt = rem < kRsTile ? (int)rem : kRsTile;
    for (int sp = threadIdx.x; sp < cnt; sp += blockDim.x) {
        const uint32_t key = skey[sp];
        const uint32_t d = (key >> shift) & 255u;
        const uint32_t pos = dbase[d] + ((uint32_t)sp - bstart[d]);
        keys_out[pos] = key;
        vals_out[pos] = sval[sp];
    }
}

// ----------------------------------------------------------------------------------
// One kernel per pass (the onesweep scheme of Adinets & Merrill 2022): the digit counts
// of all four passes come from one read of the keys (k_os_hist); in each pass the tiles
// take tickets in the order their blocks start, rank their keys as k_rs_scatter does,
// publish their per-digit counts and find the counts of every tile before them by
// decoupled look-back (Merrill & Garland 2016): the words of the preceding tiles are
// read from the nearest backwards, adding aggregates until an inclusive prefix is met.
// A word packs a 2-bit state (not ready / aggregate / inclusive) with a 30-bit count, so
// n < 2^30.  A tile only waits on tiles with smaller tickets, whose blocks are already
// running and wait only on tiles before their own, so the look-back ends; its spin is
// bounded all the same (kStatusTimeout, results invalid).  Same stable order as the
// three-kernel passes: tile t holds keys [t * kRsTile, (t + 1) * kRsTile) of the pass's
// input whatever block takes ticket t.
// ----------------------------------------------------------------------------------
constexpr uint32_t kOsAggregate = 1u << 30;
constexpr uint32_t kOsInclusive = 2u << 30;
constexpr uint32_t kOsCount = (1u << 30) - 1u;
constexpr long long kOsSpinCycles = 200000000LL;  // ~0.1 s at 2 GHz
constexpr int kOsWindow = 16;                    // look-back words loaded together

__device__ __forceinline__ uint32_t ld_relaxed_gpu(const uint32_t* p) {
    uint32_t v;
    asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_relaxed_gpu(uint32_t* p, uint32_t v) {
    asm volatile("st.relaxed.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// ghist[pass * 256 + digit] += count over keys[0, n) (ghist zeroed by the caller).
__global__ void __launch_bounds__(256) k_os_hist(const uint32_t* __restrict__ keys, int64_t n,
                                                 uint32_t* __restrict__ ghist) {
    __shared__ uint32_t cnt[4 * 256];
    for (int i = threadIdx.x; i < 4 * 256; i += blockDim.x) cnt[i] = 0u;
    __syncthreads();
    const int64_t nv = n >> 2;  // uint4 loads (the buffer is 256-byte aligned), then the tail
    const uint4* k4 = reinterpret_cast<const uint4*>(keys);
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nv + 4; i += stride) {
        uint32_t k[4];
        int m = 0;
        if (i < nv) {
            const uint4 q = k4[i];
            k[0] = q.x;
            k[1] = q.y;
            k[2] = q.z;
            k[3] = q.w;
            m = 4;
        } else if (4 * nv + (i - nv) < n) {
            k[0] = keys[4 * nv + (i - nv)];
            m = 1;
        }
        for (int j = 0; j < m; j++) {
            atomicAdd(&cnt[k[j] & 255u], 1u);
            atomicAdd(&cnt[256 + ((k[j] >> 8) & 255u)], 1u);
            atomicAdd(&cnt[512 + ((k[j] >> 16) & 255u)], 1u);
            atomicAdd(&cnt[768 + (k[j] >> 24)], 1u);
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < 4 * 256; i += blockDim.x) {
        const uint32_t v = cnt[i];
        if (v) atomicAdd(&ghist[i], v);
    }
}

__global__ void __launch_bounds__(256, 4) k_os_scatter(const uint32_t* __restrict__ keys_in,
                                                    const int32_t* __restrict__ vals_in,
                                                    uint32_t* __restrict__ keys_out, int32_t* __restrict__ vals_out,
                                                    int64_t n, int pass, const uint32_t* __restrict__ ghist,
                                                    uint32_t* __restrict__ look, uint32_t* __restrict__ ticket,
                                                    int* __restrict__ status) {
    __shared__ uint32_t wcnt[kRsWarps][256];
    __shared__ uint32_t dbase[256];
    __shared__ uint32_t bstart[256];
    __shared__ uint32_t wsum[kRsWarps];
    __shared__ uint32_t skey[kRsTile];
    __shared__ int32_t sval[kRsTile];
    __shared__ uint32_t s_tile;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int shift = 8 * pass;
    if (threadIdx.x == 0) s_tile = atomicAdd(ticket, 1u);
    for (int t = threadIdx.x; t < kRsWarps * 256; t += blockDim.x) (&wcnt[0][0])[t] = 0;
    // first position of each digit in the output: exclusive scan of the pass's digit counts
    if (warp == 0) {
        uint32_t run = 0;
        for (int chunk = 0; chunk < 8; chunk++) {
            const int d = chunk * 32 + lane;
            const uint32_t v = ghist[pass * 256 + d];
            uint32_t incl = v;
            for (int off = 1; off < 32; off <<= 1) {
                const uint32_t t = __shfl_up_sync(0xffffffffu, incl, off);
                if (lane >= off) incl += t;
            }
            dbase[d] = run + incl - v;
            run += __shfl_sync(0xffffffffu, incl, 31);
        }
    }
    __syncthreads();
    const int64_t tile = s_tile;
    const int64_t base = tile * kRsTile + (int64_t)warp * (kRsIters * 32);
    uint32_t kreg[kRsIters];
    int32_t vreg[kRsIters];
    uint32_t rreg[kRsIters];  // (local rank << 8) | digit, or 0xffffffff if invalid
#pragma unroll
    for (int it = 0; it < kRsIters; it++) {
        const int64_t idx = base + it * 32 + lane;
        const bool valid = idx < n;
        const uint32_t key = valid ? keys_in[idx] : 0u;
        const int32_t val = valid ? (vals_in ? vals_in[idx] : (int32_t)idx) : 0;
        const uint32_t d = (key >> shift) & 255u;
        const uint32_t tag = valid ? d : (256u + lane);
        const uint32_t peers = __match_any_sync(0xffffffffu, tag);
        const uint32_t rank = __popc(peers & lanemask_lt());
        const uint32_t pre = valid ? wcnt[warp][d] : 0u;
        __syncwarp();
        if (valid && (__ffs(peers) - 1) == lane) wcnt[warp][d] = pre + __popc(peers);
        __syncwarp();
        kreg[it] = key;
        vreg[it] = val;
        rreg[it] = valid ? (((pre + rank) << 8) | d) : 0xffffffffu;
    }
    __syncthreads();
    // exclusive prefix over warps for each digit; run = this tile's count of digit d
    const int d = threadIdx.x;  // 256 threads == 256 digits
    uint32_t run = 0;
#pragma unroll
    for (int w = 0; w < kRsWarps; w++) {
        const uint32_t t = wcnt[w][d];
        wcnt[w][d] = run;
        run += t;
    }
    // publish this tile's count of digit d at once, so that later tiles can pass over it
    uint32_t* mine = look + tile * 256 + d;
    st_relaxed_gpu(mine, (tile == 0 ? kOsInclusive : kOsAggregate) | run);
    // tile-local start of each digit: exclusive scan of the 256 counts
    {
        uint32_t incl = run;
        for (int off = 1; off < 32; off <<= 1) {
            const uint32_t t = __shfl_up_sync(0xffffffffu, incl, off);
            if (lane >= off) incl += t;
        }
        if (lane == 31) wsum[warp] = incl;
        __syncthreads();
        uint32_t wbase = 0;
        for (int w = 0; w < warp; w++) wbase += wsum[w];
        bstart[threadIdx.x] = wbase + incl - run;
    }
    __syncthreads();
    // the keys go to their tile-local sorted slots before the look-back (their registers
    // are free for the look-back's window)
#pragma unroll
    for (int it = 0; it < kRsIters; it++) {
        const uint32_t r = rreg[it];
        if (r != 0xffffffffu) {
            const uint32_t dd = r & 255u;
            const uint32_t sp = bstart[dd] + wcnt[warp][dd] + (r >> 8);
            skey[sp] = kreg[it];
            sval[sp] = vreg[it];
        }
    }
    // look back for the count of digit d in all tiles before this one, kOsWindow words
    // loaded together: aggregates are added until an inclusive prefix is met; a tile not
    // ready yet ends this window (the words before it are kept) and is read again
    if (tile > 0) {
        uint32_t excl = 0;
        int64_t k = tile - 1;  // nearest tile not accounted for yet
        const long long t0 = clock64();
        bool ok = true;
        while (true) {
            uint32_t v[kOsWindow];
#pragma unroll
            for (int i = 0; i < kOsWindow; i++) v[i] = k - i >= 0 ? ld_relaxed_gpu(look + (k - i) * 256 + d) : kOsInclusive;
            uint32_t add = 0;
            int taken = 0;
            bool inclusive = false, blocked = false;
#pragma unroll
            for (int i = 0; i < kOsWindow; i++) {
                if (!inclusive && !blocked) {
                    const uint32_t state = v[i] & ~kOsCount;
                    if (state == 0u) {
                        blocked = true;
                    } else {
                        add += v[i] & kOsCount;
                        taken++;
                        inclusive = state == kOsInclusive;
                    }
                }
            }
            excl += add;
            if (inclusive) break;
            k -= taken;
            if (blocked) {
                if (clock64() - t0 > kOsSpinCycles) {
                    ok = false;
                    break;
                }
                __nanosleep(32);
            }
        }
        if (!ok) atomicOr(status, kStatusTimeout);
        st_relaxed_gpu(mine, kOsInclusive | ((excl + run) & kOsCount));
        dbase[d] += excl;
    }
    __syncthreads();
    const int64_t rem = n - tile * kRsTile;
    const int cnt = rem < kRsTile ? (int)rem : kRsTile;
    for (int sp = threadIdx.x; sp < cnt; sp += blockDim.x) {
        const uint32_t key = skey[sp];
        const uint32_t dd = (key >> shift) & 255u;
        const uint32_t pos = dbase[dd] + ((uint32_t)sp - bstart[dd]);
        // pos < n always (a timed-out look-back only undercounts); the test costs nothing
        if (pos < (uint64_t)n) {
            keys_out[pos] = key;
            vals_out[pos] = sval[sp];
        }
    }
}

static cudaError_t radix_sort_onesweep(Lbvh& L, int64_t n, cudaStream_t st) {
    const int64_t T = (n + kRsTile - 1) / kRsTile;
    const size_t head = sizeof(uint32_t) * (4 * 256 + 64);  // digit counts [4][256], tickets [4] (padded)
    const size_t look = sizeof(uint32_t) * 256 * (size_t)T;  // one word per (tile, digit) and pass
    cudaError_t e;
    if ((e = L.keys_alt.ensure(LbvhBytes::keys(n))) != cudaSuccess) return e;
    if ((e = L.perm.ensure(LbvhBytes::keys(n))) != cudaSuccess) return e;
    if ((e = L.perm_alt.ensure(LbvhBytes::keys(n))) != cudaSuccess) return e;
    if ((e = L.onesweep.ensure(head + 4 * look)) != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(L.onesweep.ptr, 0, head + 4 * look, st)) != cudaSuccess) return e;
    uint32_t* ghist = L.onesweep.as<uint32_t>();
    uint32_t* tickets = ghist + 4 * 256;
    uint32_t* look0 = ghist + head / sizeof(uint32_t);
    const unsigned hb = (unsigned)(T < 148 * 4 ? T : 148 * 4);
    k_os_hist<<<hb, 256, 0, st>>>(L.keys.as<uint32_t>(), n, ghist); gvc::note_launch();
    uint32_t* kin = L.keys.as<uint32_t>();
    uint32_t* kout = L.keys_alt.as<uint32_t>();
    int32_t* vin = nullptr;
    int32_t* vout = L.perm_alt.as<int32_t>();
    for (int pass = 0; pass < 4; pass++) {
        k_os_scatter<<<(unsigned)T, 256, 0, st>>>(kin, vin, kout, vout, n, pass, ghist,
                                                  look0 + (size_t)pass * 256 * (size_t)T, tickets + pass,
                                                  L.status); gvc::note_launch();
        // ping-pong as in radix_sort_pairs: the result ends in L.keys / L.perm
        uint32_t* tk = kin;
        kin = kout;
        kout = tk;
        vin = vout;
        vout = (vout == L.perm_alt.as<int32_t>()) ? L.perm.as<int32_t>() : L.perm_alt.as<int32_t>();
    }
    return cudaGetLastError();
}

cudaError_t radix_sort_pairs(Lbvh& L, int64_t n, cudaStream_t st) {
    // Input: L.keys [n]. Output: L.keys sorted, L.perm (sorted pos -> input index).
    if (n <= 0) return cudaSuccess;
    // one kernel per pass where a status word can take the look-back's timeout report
    if (L.status && n <= (int64_t)kOsCount) return radix_sort_onesweep(L, n, st);
    const int nb = (int)((n + kRsTile - 1) / kRsTile);
    cudaError_t e;
    if ((e = L.keys_alt.ensure(LbvhBytes::keys(n))) != cudaSuccess) return e;
    if ((e = L.perm.ensure(LbvhBytes::keys(n))) != cudaSuccess) return e;
    if ((e = L.perm_alt.ensure(LbvhBytes::keys(n))) != cudaSuccess) return e;
    if ((e = L.hist.ensure(LbvhBytes::hist(n))) != cudaSuccess) return e;
    uint32_t* hist = L.hist.as<uint32_t>();
    uint32_t* totals = hist + 256 * (size_t)nb;
    uint32_t* kin = L.keys.as<uint32_t>();
    uint32_t* kout = L.keys_alt.as<uint32_t>();
    int32_t* vin = nullptr;
    int32_t* vout = L.perm_alt.as<int32_t>();
    for (int pass = 0; pass < 4; pass++) {
        k_rs_hist<<<nb, 256, 0, st>>>(kin, n, nb, pass, hist); gvc::note_launch();
        k_rs_scan<<<256, 1024, 0, st>>>(hist, nb, totals); gvc::note_launch();
        k_rs_scatter<<<nb, 256, 0, st>>>(kin, vin, kout, vout, n, nb, pass, hist, totals); gvc::note_launch();
        // ping-pong: pass 0 keys->alt, 1 alt->keys, 2 keys->alt, 3 alt->keys
        uint32_t* tk = kin;
        kin = kout;
        kout = tk;
        vin = vout;
        vout = (vout == L.perm_alt.as<int32_t>()) ? L.perm.as<int32_t>() : L.perm_alt.as<int32_t>();
    }
    return cudaGetLastError();
}

__global__ void __launch_bounds__(256) k_gather_u32(int64_t n, const uint32_t* __restrict__ src,
                                                    const int32_t* __restrict__ perm, uint32_t* __restrict__ dst) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < n) dst[i] = src[perm[i]];
}

cudaError_t radix_sort_words(Lbvh& L, int64_t n, const uint32_t* const* words, const int* bits, int nwords,
                             cudaStream_t st) {
    if (n <= 0) return cudaSuccess;
    const int nb = (int)((n + kRsTile - 1) / kRsTile);
    cudaError_t e;
    if ((e = L.keys.ensure(sizeof(uint32_t) * n)) != cudaSuccess) return e;
    if ((e = L.keys_alt.ensure(LbvhBytes::keys(n))) != cudaSuccess) return e;
    if ((e = L.perm.ensure(LbvhBytes::keys(n))) != cudaSuccess) return e;
    if ((e = L.perm_alt.ensure(LbvhBytes::keys(n))) != cudaSuccess) return e;
    if ((e = L.hist.ensure(LbvhBytes::hist(n))) != cudaSuccess) return e;
    uint32_t* hist = L.hist.as<uint32_t>();
    uint32_t* totals = hist + 256 * (size_t)nb;
    uint32_t* kin = L.keys.as<uint32_t>();
    uint32_t* kout = L.keys_alt.as<uint32_t>();
    int32_t* vin = nullptr;  // identity before the first pass
    int32_t* vout = L.perm_alt.as<int32_t>();
    const unsigned gb = (unsigned)((n + 255) / 256);
    // one kernel per pass (as radix_sort_pairs) where a status word takes the look-back's report
    const bool os = L.status && n <= (int64_t)kOsCount;
    const size_t os_head = sizeof(uint32_t) * (4 * 256 + 64);
    const size_t os_look = sizeof(uint32_t) * 256 * (size_t)nb;
    if (os && (e = L.onesweep.ensure(os_head + 4 * os_look)) != cudaSuccess) return e;
    uint32_t* ghist = os ? L.onesweep.as<uint32_t>() : nullptr;
    for (int w = 0; w < nwords; w++) {
        const int passes = (bits[w] + 7) / 8;
        if (passes <= 0) continue;
        // this word's keys in the current order
        if (vin) {
            k_gather_u32<<<gb, 256, 0, st>>>(n, words[w], vin, kin); gvc::note_launch();
        } else if ((e = cudaMemcpyAsync(kin, words[w], sizeof(uint32_t) * n, cudaMemcpyDeviceToDevice, st)) !=
                   cudaSuccess) {
            return e;
        }
        if (os) {
            if ((e = cudaMemsetAsync(ghist, 0, os_head + (size_t)passes * os_look, st)) != cudaSuccess) return e;
            k_os_hist<<<(unsigned)(nb < 148 * 4 ? nb : 148 * 4), 256, 0, st>>>(kin, n, ghist); gvc::note_launch();
        }
        for (int pass = 0; pass < passes; pass++) {
            if (os) {
                k_os_scatter<<<(unsigned)nb, 256, 0, st>>>(kin, vin, kout, vout, n, pass, ghist,
                                                           ghist + os_head / sizeof(uint32_t) +
                                                               (size_t)pass * 256 * (size_t)nb,
                                                           ghist + 4 * 256 + pass, L.status); gvc::note_launch();
            } else {
                k_rs_hist<<<nb, 256, 0, st>>>(kin, n, nb, pass, hist); gvc::note_launch();
                k_rs_scan<<<256, 1024, 0, st>>>(hist, nb, totals); gvc::note_launch();
                k_rs_scatter<<<nb, 256, 0, st>>>(kin, vin, kout, vout, n, nb, pass, hist, totals); gvc::note_launch();
            }
            uint32_t* tk = kin;
            kin = kout;
            kout = tk;
            int32_t* tv = vin;
            vin = vout;
            vout = tv ? tv : (vin == L.perm_alt.as<int32_t>() ? L.perm.as<int32_t>() : L.perm_alt.as<int32_t>());
        }
    }
    if (!vin) return cudaErrorInvalidValue;  // no word had any bits
    if (vin != L.perm.as<int32_t>() &&
        (e = cudaMemcpyAsync(L.perm.ptr, vin, sizeof(int32_t) * n, cudaMemcpyDeviceToDevice, st)) != cudaSuccess)
        return e;
    return cudaGetLastError();
}

// ----------------------------------------------------------------------------------
// Karras 2012 ("Maximizing parallelism in the construction of BVHs, octrees and k-d
// trees", HPG 2012, Fig. 4).  Equal keys are disambiguated by position.
// parent: [2n-1]: parent[k] of internal node k (k < n-1), parent[n-1+i] of leaf i.
// ----------------------------------------------------------------------------------
__device__ __forceinline__ int delta(const uint32_t* k, int64_t n, int64_t i, int64_t j) {
    if (j < 0 || j >= n) return -1;
    uint32_t a = k[i], b = k[j];
    if (a == b) return 32 + __clz((uint32_t)(i ^ j));
    return __clz(a ^ b);
}

__global__ void __launch_bounds__(256) k_karras(const uint32_t* __restrict__ keys, int64_t n, int32_t* __restrict__ left,
                                                int32_t* __restrict__ right, int32_t* __restrict__ parent) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n - 1) return;
    const int64_t d = (delta(keys, n, i, i + 1) - delta(keys, n, i, i - 1)) >= 0 ? 1 : -1;
    const int dmin = delta(keys, n, i, i - d);
    int64_t lmax = 2;
    while (delta(keys, n, i, i + lmax * d) > dmin) lmax *= 2;
    int64_t l = 0;
    for (int64_t t = lmax / 2; t >= 1; t /= 2)
        if (delta(keys, n, i, i + (l + t) * d) > dmin) l += t;
    const int64_t j = i + l * d;
    const int dnode = delta(keys, n, i, j);
    int64_t s = 0, t = l;
    do {
        t = (t + 1) / 2;
        if (delta(keys, n, i, i + (s + t) * d) > dnode) s += t;
    } while (t > 1);
    const int64_t gamma = i + s * d + (d < 0 ? d : 0);
    const int64_t lo = min(i, j), hi = max(i, j);
    if (lo == gamma) {
        left[i] = (int32_t)((uint32_t)gamma | kLeafBit);
        parent[n - 1 + gamma] = (int32_t)i;
    } else {
        left[i] = (int32_t)gamma;
        parent[gamma] = (int32_t)i;
    }
    if (hi == gamma + 1) {
        right[i] = (int32_t)((uint32_t)(gamma + 1) | kLeafBit);
        parent[n - 1 + gamma + 1] = (int32_t)i;
    } else {
        right[i] = (int32_t)(gamma + 1);
        parent[gamma + 1] = (int32_t)i;
    }
    if (i == 0) parent[0] = -1;
}

__device__ __forceinline__ void load_child_box(int32_t c, const float4* __restrict__ leaf_boxes,
                                               const float4* node_boxes, float4& lo, float4& hi) {
    if ((uint32_t)c & kLeafBit) {
        int li = (int)((uint32_t)c & ~kLeafBit);
        lo = __ldcg(leaf_boxes + 2 * li);
        hi = __ldcg(leaf_boxes + 2 * li + 1);
    } else {
        lo = __ldcg(node_boxes + 2 * c);
        hi = __ldcg(node_boxes + 2 * c + 1);
    }
}

// Bottom-up refit: the second thread to reach a node computes its box (min/max,
// independent of arrival order).
__global__ void __launch_bounds__(256) k_refit(int n, const int32_t* __restrict__ left, const int32_t* __restrict__ right,
                                               const int32_t* __restrict__ parent, const float4* __restrict__ leaf_boxes,
                                               float4* node_boxes, uint32_t* flags) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int node = parent[n - 1 + i];
    while (node >= 0) {
        // acquire-release at GPU scope: the first child's box (stored before its arrival)
        // is visible to the second arriver, which goes on with the node
        uint32_t old;
        asm volatile("atom.acq_rel.gpu.global.add.u32 %0, [%1], 1;" : "=r"(old) : "l"(flags + node) : "memory");
        if (old == 0) return;
        float4 alo, ahi, blo, bhi;
        load_child_box(left[node], leaf_boxes, node_boxes, alo, ahi);
        load_child_box(right[node], leaf_boxes, node_boxes, blo, bhi);
        float4 lo = make_float4(fminf(alo.x, blo.x), fminf(alo.y, blo.y), fminf(alo.z, blo.z), 0.f);
        float4 hi = make_float4(fmaxf(ahi.x, bhi.x), fmaxf(ahi.y, bhi.y), fmaxf(ahi.z, bhi.z), 0.f);
        __stcg(node_boxes + 2 * node, lo);
        __stcg(node_boxes + 2 * node + 1, hi);
        node = parent[node];
    }
}

// Packs node k with both children's boxes, and the links of the stackless traversal:
// c.w = the escape edge of node k (the edge that follows k's subtree in pre-order, edge
// code 2p + s for child s of node p): (p, 1) for the nearest ancestor-or-self of k that
// is the left child of p, 0xffffffff when k lies on the root's right spine; d.w = the
// right child again.
__global__ void __launch_bounds__(256) k_pack_nodes(int n, const int32_t* __restrict__ left,
                                                    const int32_t* __restrict__ right,
                                                    const int32_t* __restrict__ parent,
                                                    const float4* __restrict__ leaf_boxes,
                                                    const float4* __restrict__ node_boxes, BvhNode* __restrict__ nodes) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (n == 1) {
        // a single leaf: a root whose right child can never overlap anything
        if (k == 0) {
            float4 lo = leaf_boxes[0], hi = leaf_boxes[1];
            BvhNode nd;
            nd.a = make_float4(lo.x, lo.y, lo.z, __uint_as_float(0u | kLeafBit));
            nd.b = make_float4(hi.x, hi.y, hi.z, __uint_as_float(0u | kLeafBit));
            nd.c = make_float4(INFINITY, INFINITY, INFINITY, __uint_as_float(0xffffffffu));
            nd.d = make_float4(-INFINITY, -INFINITY, -INFINITY, __uint_as_float(0u | kLeafBit));
            nodes[0] = nd;
        }
        return;
    }
    if (k >= n - 1) return;
    int32_t l = left[k], r = right[k];
    float4 alo, ahi, blo, bhi;
    load_child_box(l, leaf_boxes, node_boxes, alo, ahi);
    load_child_box(r, leaf_boxes, node_boxes, blo, bhi);
    BvhNode nd;
    nd.a = make_float4(alo.x, alo.y, alo.z, __int_as_float(l));
    nd.b = make_float4(ahi.x, ahi.y, ahi.z, __int_as_float(r));
    // escape edge: climb while the node is its parent's right child (at most the depth)
    int32_t x = k, p = parent[k];
    for (int depth = 0; p >= 0 && right[p] == x && depth < n; depth++) {
        x = p;
        p = parent[p];
    }
    const uint32_t esc = p < 0 ? 0xffffffffu : 2u * (uint32_t)p + 1u;
    nd.c = make_float4(blo.x, blo.y, blo.z, __uint_as_float(esc));
    nd.d = make_float4(bhi.x, bhi.y, bhi.z, __int_as_float(r));
    nodes[k] = nd;
}

__global__ void __launch_bounds__(256) k_gather_boxes(int64_t n, const int32_t* __restrict__ perm,
                                                      const float4* __restrict__ boxes, float4* __restrict__ out) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    int64_t p = perm[i];
    out[2 * i] = boxes[2 * p];
    out[2 * i + 1] = boxes[2 * p + 1];
}

static inline unsigned blocks_for(int64_t n, int t) { return (unsigned)((n + t - 1) / t); }

cudaError_t lbvh_hierarchy(Lbvh& L, int64_t n, const uint32_t* sorted_keys, const float4* sorted_leaf_boxes,
                           cudaStream_t st) {
    cudaError_t e;
    int64_t ni = n > 1 ? n - 1 : 1;
    if ((e = L.left.ensure(LbvhBytes::child(n))) != cudaSuccess) return e;
    if ((e = L.right.ensure(LbvhBytes::child(n))) != cudaSuccess) return e;
    if ((e = L.parent.ensure(LbvhBytes::parent(n))) != cudaSuccess) return e;
    if ((e = L.flags.ensure(LbvhBytes::child(n))) != cudaSuccess) return e;
    if ((e = L.node_boxes.ensure(LbvhBytes::node_boxes(n))) != cudaSuccess) return e;
    if ((e = L.nodes.ensure(LbvhBytes::nodes(n))) != cudaSuccess) return e;
    L.n = n;
    if (n > 1) {
        k_karras<<<blocks_for(n - 1, 256), 256, 0, st>>>(sorted_keys, n, L.left.as<int32_t>(),
                                                         L.right.as<int32_t>(), L.parent.as<int32_t>()); gvc::note_launch();
        if ((e = cudaMemsetAsync(L.flags.ptr, 0, sizeof(uint32_t) * (n - 1), st)) != cudaSuccess) return e;
        k_refit<<<blocks_for(n, 256), 256, 0, st>>>((int)n, L.left.as<int32_t>(), L.right.as<int32_t>(),
                                                    L.parent.as<int32_t>(), sorted_leaf_boxes,
                                                    L.node_boxes.as<float4>(), L.flags.as<uint32_t>()); gvc::note_launch();
    }
    k_pack_nodes<<<blocks_for(ni, 256), 256, 0, st>>>((int)n, L.left.as<int32_t>(), L.right.as<int32_t>(),
                                                     L.parent.as<int32_t>(), sorted_leaf_boxes, L.node_boxes.as<float4>(),
                                                     L.nodes.as<BvhNode>()); gvc::note_launch();
    return cudaGetLastError();
}

cudaError_t morton_sort_boxes(Lbvh& L, int64_t n, const float4* boxes, cudaStream_t st) {
    cudaError_t e;
    if ((e = L.keys.ensure(LbvhBytes::keys(n))) != cudaSuccess) return e;
    if ((e = L.bounds.ensure(LbvhBytes::bounds())) != cudaSuccess) return e;
    k_bounds_init<<<1, 32, 0, st>>>(L.bounds.as<uint32_t>()); gvc::note_launch();
    unsigned nbk = blocks_for(n, 256);
    if (nbk > 148u * 8u) nbk = 148u * 8u;
    k_bounds<BoxSrc><<<nbk, 256, 0, st>>>(BoxSrc{boxes}, n, L.bounds.as<uint32_t>()); gvc::note_launch();
    k_keys<BoxSrc><<<blocks_for(n, 256), 256, 0, st>>>(BoxSrc{boxes}, n, L.bounds.as<uint32_t>(),
                                                       L.keys.as<uint32_t>()); gvc::note_launch();
    return radix_sort_pairs(L, n, st);
}

cudaError_t morton_sort_points(Lbvh& L, int64_t n, const float* pts, cudaStream_t st) {
    cudaError_t e;
    if ((e = L.keys.ensure(LbvhBytes::keys(n))) != cudaSuccess) return e;
    if ((e = L.bounds.ensure(LbvhBytes::bounds())) != cudaSuccess) return e;
    k_bounds_init<<<1, 32, 0, st>>>(L.bounds.as<uint32_t>()); gvc::note_launch();
    unsigned nbk = blocks_for(n, 256);
    if (nbk > 148u * 8u) nbk = 148u * 8u;
    k_bounds<PointSrc><<<nbk, 256, 0, st>>>(PointSrc{pts}, n, L.bounds.as<uint32_t>()); gvc::note_launch();
    k_keys<PointSrc><<<blocks_for(n, 256), 256, 0, st>>>(PointSrc{pts}, n, L.bounds.as<uint32_t>(),
                                                         L.keys.as<uint32_t>()); gvc::note_launch();
    return radix_sort_pairs(L, n, st);
}

cudaError_t lbvh_build_boxes(Lbvh& L, int64_t n, const float4* boxes, cudaStream_t st) {
    cudaError_t e;
    if (n <= 0) {
        L.n = 0;
        return cudaSuccess;
    }
    if ((e = morton_sort_boxes(L, n, boxes, st)) != cudaSuccess) return e;
    if ((e = L.sorted_boxes.ensure(LbvhBytes::sorted_boxes(n))) != cudaSuccess) return e;
    k_gather_boxes<<<blocks_for(n, 256), 256, 0, st>>>(n, L.perm.as<int32_t>(), boxes, L.sorted_boxes.as<float4>()); gvc::note_launch();
    return lbvh_hierarchy(L, n, L.keys.as<uint32_t>(), L.sorted_boxes.as<float4>(), st);
}

}  // namespace gvc
