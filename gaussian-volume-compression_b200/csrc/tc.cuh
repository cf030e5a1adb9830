// tc.cuh -- sm_100a tensor-core (tcgen05 / TMEM) and mbarrier primitives in inline PTX.
//
// Conventions follow the PTX ISA for tcgen05 (cta_group::1, kind::f16 with BF16 operands,
// FP32 accumulation in tensor memory) and the shared-memory matrix descriptor of sm_100:
//   operands are K-major without swizzle ("interleaved" canonical layout): an operand tile
//   of R rows x 16 bf16 is stored as core matrices of 8 rows x 16 bytes; element (r, k)
//   lives at byte (r / 8) * 256 + (k / 8) * 128 + (r % 8) * 16 + (k % 8) * 2, i.e. the
//   leading (K) byte offset is 128 and the stride (8-row group) byte offset is 256.
// Every wait is bounded: a timeout sets a status bit and the caller stops waiting.
#pragma once
#include <cuda_bf16.h>

#include "gvc_internal.cuh"

namespace gvc {

// Bounded spin for mbarrier waits: ~0.1 s at 2 GHz.
constexpr long long kSpinCycles = 200000000LL;

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// ---- mbarrier -------------------------------------------------------------------------
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.release.cta.shared::cta.b64 st, [%0];\n\t}" ::"r"(smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void fence_mbar_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t phase) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(phase)
        : "memory");
    return ok != 0;
}

// Waits for the phase with the given parity to complete; false (and a status bit) on timeout.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t phase, int* status) {
    const long long t0 = clock64();
    while (!mbar_try_wait(bar, phase)) {
        if (clock64() - t0 > kSpinCycles) {
            atomicOr(status, kStatusTimeout);
            return false;
        }
    }
    return true;
}

// ---- tensor memory --------------------------------------------------------------------
// Warp-wide: allocates ncols (power of 2, >= 32) columns; the TMEM address goes to *dst.
// A TMEM allocation is a power of two of at least 32 columns (anything else is an
// illegal instruction); callers check their column counts with this at compile time.
__host__ __device__ constexpr bool tmem_cols_ok(uint32_t n) { return n >= 32 && n <= 512 && (n & (n - 1)) == 0; }

__device__ __forceinline__ void tmem_alloc(uint32_t* dst, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(dst)),
                 "r"(ncols)
                 : "memory");
}
__device__ __forceinline__ void tmem_relinquish() {
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}
__device__ __forceinline__ void tc_fence_before() {
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
// Makes this thread's generic-proxy shared-memory writes visible to the tensor cores.
__device__ __forceinline__ void fence_proxy_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// ---- descriptors ------------------------------------------------------------------------
// Shared-memory matrix descriptor: K-major, no swizzle, LBO = 128 B, SBO = 256 B, sm_100.
__device__ __forceinline__ uint64_t smem_desc_k16(const void* tile) {
    const uint32_t a = smem_u32(tile);
    uint64_t d = 0;
    d |= (uint64_t)((a >> 4) & 0x3FFFu);
    d |= (uint64_t)((128u >> 4) & 0x3FFFu) << 16;
    d |= (uint64_t)((256u >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1u << 46;  // descriptor version for sm_100
    return d;                 // base offset 0, legacy LBO mode, layout type 0 (no swizzle)
}

// Instruction descriptor: kind::f16, A = B = BF16, D = F32, both K-major, dense.
__host__ __device__ constexpr uint32_t idesc_bf16_f32(int M, int N) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

// D[tmem] (+)= A[smem] * B[smem]^T, issued by one thread.
__device__ __forceinline__ void umma_bf16(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                          uint32_t accumulate) {
    const uint32_t z = 0;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
        :
        : "r"(d_tmem), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(z), "r"(z), "r"(z), "r"(z)
        : "memory");
}

// Arrives on the mbarrier once every MMA issued so far by this thread has completed.
__device__ __forceinline__ void umma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

// Warp-wide: thread t receives columns [col, col + 32) of TMEM lane (lane base + t).
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32]) {
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
        "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
        "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 32; i++) v[i] = __uint_as_float(r[i]);
}

// ---- operand tiles -------------------------------------------------------------------------
// Writes row r (16 bf16 values) of a K-major no-swizzle operand tile.
__device__ __forceinline__ void store_row_k16(unsigned char* tile, int r, const __nv_bfloat16 (&v)[16]) {
    uint4 lo, hi;
    __nv_bfloat162 p[8];
#pragma unroll
    for (int i = 0; i < 8; i++) p[i] = __halves2bfloat162(v[2 * i], v[2 * i + 1]);
    lo.x = *reinterpret_cast<uint32_t*>(&p[0]);
    lo.y = *reinterpret_cast<uint32_t*>(&p[1]);
    lo.z = *reinterpret_cast<uint32_t*>(&p[2]);
    lo.w = *reinterpret_cast<uint32_t*>(&p[3]);
    hi.x = *reinterpret_cast<uint32_t*>(&p[4]);
    hi.y = *reinterpret_cast<uint32_t*>(&p[5]);
    hi.z = *reinterpret_cast<uint32_t*>(&p[6]);
    hi.w = *reinterpret_cast<uint32_t*>(&p[7]);
    unsigned char* base = tile + (r >> 3) * 256 + (r & 7) * 16;
    *reinterpret_cast<uint4*>(base) = lo;
    *reinterpret_cast<uint4*>(base + 128) = hi;
}

// Splits 16 fp32 values into `terms` bf16 parts (hi, mid, lo): v = sum of parts to ~8*terms bits.
__device__ __forceinline__ void split_bf16(const float (&v)[16], __nv_bfloat16 (&h)[16], __nv_bfloat16 (&m)[16],
                                           __nv_bfloat16 (&l)[16]) {
#pragma unroll
    for (int i = 0; i < 16; i++) {
        h[i] = __float2bfloat16_rn(v[i]);
        const float r1 = v[i] - __bfloat162float(h[i]);
        m[i] = __float2bfloat16_rn(r1);
        const float r2 = r1 - __bfloat162float(m[i]);
        l[i] = __float2bfloat16_rn(r2);
    }
}

// ---- split-BF16 operand rows and narrower TMEM reads ------------------------------------
__device__ __forceinline__ uint32_t bf2_bits(__nv_bfloat162 v) { return *reinterpret_cast<uint32_t*>(&v); }

// Splits (a, b) into three BF16 parts each: a = h.x + m.x + l.x (~24 bits), same for b.
__device__ __forceinline__ void split3_pair(float a, float b, uint32_t& h, uint32_t& m, uint32_t& l) {
    const __nv_bfloat162 H = __floats2bfloat162_rn(a, b);
    const float ra = a - __low2float(H), rb = b - __high2float(H);
    const __nv_bfloat162 M = __floats2bfloat162_rn(ra, rb);
    const float sa = ra - __low2float(M), sb = rb - __high2float(M);
    const __nv_bfloat162 L = __floats2bfloat162_rn(sa, sb);
    h = bf2_bits(H);
    m = bf2_bits(M);
    l = bf2_bits(L);
}

// Writes the ten features f[0..9] of row r into the three parts of a K-major no-swizzle
// tile (element (r, k) at (r / 8) * 256 + (k / 8) * 128 + (r % 8) * 16 + (k % 8) * 2);
// features 10..15 are left as they are (zero).
__device__ __forceinline__ void store_features10(unsigned char* t0, unsigned char* t1, unsigned char* t2, int r,
                                                 const float (&f)[10]) {
    uint32_t h[5], m[5], l[5];
#pragma unroll
    for (int i = 0; i < 5; i++) split3_pair(f[2 * i], f[2 * i + 1], h[i], m[i], l[i]);
    const int off = (r >> 3) * 256 + (r & 7) * 16;
    *reinterpret_cast<uint4*>(t0 + off) = make_uint4(h[0], h[1], h[2], h[3]);
    *reinterpret_cast<uint4*>(t1 + off) = make_uint4(m[0], m[1], m[2], m[3]);
    *reinterpret_cast<uint4*>(t2 + off) = make_uint4(l[0], l[1], l[2], l[3]);
    *reinterpret_cast<uint32_t*>(t0 + off + 128) = h[4];
    *reinterpret_cast<uint32_t*>(t1 + off + 128) = m[4];
    *reinterpret_cast<uint32_t*>(t2 + off + 128) = l[4];
}

// Warp-wide: thread t receives columns [col, col + 16) of TMEM lane (lane base + t).
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
        "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; i++) v[i] = __uint_as_float(r[i]);
}

}  // namespace gvc
