// Blackwell (sm_100a) tensor-core building blocks: TMEM allocation,
// shared-memory matrix descriptors, tcgen05.mma issue / commit, TMEM loads
// and bounded mbarrier waits.  Inline PTX only.
//
// Operand layout used throughout: K-major, no swizzle ("interleaved" core
// matrices).  A core matrix is 8 rows x 16 bytes (8 sixteen-bit elements of
// K), stored contiguously (row r at byte 16 r).  For a tile of R rows
// (multiple of 8) and KT K-elements (multiple of 8) the core matrices are
// laid out chunk-major:
//     byte(r, k) = (k / 8) * (R / 8) * 128 + (r / 8) * 128 + (r % 8) * 16 + (k % 8) * 2
// so the stride between 8-row groups (SBO) is 128 bytes and between the two
// 8-element K chunks of one MMA (LBO) is R * 16 bytes.  The MMA over K
// elements [16 j, 16 j + 16) starts at byte 2 j * R * 16.
#pragma once

#include <cstdint>
#include <cuda_bf16.h>
#include <cuda_fp16.h>

namespace gs {
namespace tc {

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Byte offset of element (r, k) in the interleaved K-major tile of R rows.
__host__ __device__ __forceinline__ uint32_t kmajor_off(int r, int k, int R) {
    return (uint32_t)((k >> 3) * (R >> 3) * 128 + (r >> 3) * 128 + (r & 7) * 16 + (k & 7) * 2);
}

// Byte offset of element (mn, k) in an MN-major, no-swizzle operand: core
// matrices of 8 K-rows x 16 bytes (8 sixteen-bit MN elements), the 8-element
// MN groups `sbo` bytes apart and the 8-row K groups `lbo` bytes apart (the
// descriptor's stride and leading byte offsets for this major-ness).  The
// MMA over K elements [16 j, 16 j + 16) starts at byte 2 j lbo.
__host__ __device__ __forceinline__ uint32_t mnmajor_off(int mn, int k, uint32_t sbo, uint32_t lbo) {
    return (uint32_t)((mn >> 3) * sbo + (k >> 3) * lbo + (k & 7) * 16 + (mn & 7) * 2);
}

// Shared-memory matrix descriptor: start address, leading (K-chunk) and
// stride (8-row group) byte offsets, descriptor version 1, no swizzle.
__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
    d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1 << 46;  // version
    return d;                // base offset 0, legacy LBO mode, layout SWIZZLE_NONE
}

// Instruction descriptor of kind::f16 with f32 accumulation, both operands
// K-major; ab_bf16 selects BF16 (1) or FP16 (0) for A and B alike.
__host__ __device__ constexpr uint32_t idesc_f16(int M, int N, int ab_bf16) {
    return (1u << 4)                          // D format f32
           | ((uint32_t)ab_bf16 << 7)         // A format
           | ((uint32_t)ab_bf16 << 10)        // B format
           | ((uint32_t)(N >> 3) << 17)       // N / 8
           | ((uint32_t)(M >> 4) << 24);      // M / 16
}
// The same with A and / or B MN-major (bits 15 and 16).
__host__ __device__ constexpr uint32_t idesc_f16_major(int M, int N, int ab_bf16, int a_mn, int b_mn) {
    return idesc_f16(M, N, ab_bf16) | ((uint32_t)a_mn << 15) | ((uint32_t)b_mn << 16);
}

// ---- mbarrier ----
__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_mbar_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
// Waits until the barrier's phase with the given parity has completed; gives
// up after `limit` polls (returns false).
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, uint32_t limit) {
    const uint32_t a = smem_u32(bar);
    for (uint32_t it = 0; it < limit; ++it) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(a), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

__device__ __forceinline__ uint64_t globaltimer_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Waits until the barrier's phase with the given parity has completed,
// suspending the thread inside try_wait (up to `hint_ns` per attempt, woken
// when the phase completes) instead of spinning, so a waiting warp takes no
// issue slots; gives up after `limit_ns` of wall time (returns false).
__device__ __forceinline__ bool mbar_wait_suspend(uint64_t* bar, uint32_t parity, uint32_t hint_ns,
                                                  uint64_t limit_ns) {
    const uint32_t a = smem_u32(bar);
    const uint64_t t0 = globaltimer_ns();
    for (;;) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(a), "r"(parity), "r"(hint_ns)
            : "memory");
        if (done) return true;
        if (globaltimer_ns() - t0 > limit_ns) return false;
    }
}

// Waits until the barrier's phase with the given parity has completed,
// polling with a short sleep in between (one thread, its warp issuing little
// meanwhile); gives up after `limit_ns` of wall time (returns false).
__device__ __forceinline__ bool mbar_wait_backoff(uint64_t* bar, uint32_t parity, uint64_t limit_ns) {
    const uint32_t a = smem_u32(bar);
    const uint64_t t0 = globaltimer_ns();
    for (;;) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(a), "r"(parity)
            : "memory");
        if (done) return true;
        if (globaltimer_ns() - t0 > limit_ns) return false;
        __nanosleep(64);
    }
}

// ---- fences ----
// st.shared writes -> visible to the tensor core's (async proxy) reads
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// ---- TMEM allocation (one full warp) ----
__device__ __forceinline__ void tmem_alloc(uint32_t* dst_smem, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(dst_smem)),
                 "r"(ncols)
                 : "memory");
}
__device__ __forceinline__ void tmem_relinquish() {
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

// ---- MMA (one thread issues) ----
__device__ __forceinline__ void mma_f16(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                        uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
        : "memory");
}
// Arrive on `bar` once all previously issued MMAs of this thread complete.
__device__ __forceinline__ void mma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

// ---- TMEM -> registers: 32 lanes x 16 consecutive 32-bit columns ----
// Warp w of a warpgroup may read lanes [32 (w % 4), 32 (w % 4) + 32).
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
        "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}
__device__ __forceinline__ void tmem_ld_wait() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// ---- TMEM -> registers: 32 lanes x 32 consecutive 32-bit columns (no wait) ----
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t* r) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
        "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
}

// ---- split of an f32 pair into (hi, lo) 16-bit pairs: x = hi + lo + O(2^-16 x) ----
template <bool kBf16>
struct Split;

template <>
struct Split<true> {
    __device__ __forceinline__ static void run(float a, float b, uint32_t& hi, uint32_t& lo) {
        __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
        const float2 hf = __bfloat1622float2(h);
        __nv_bfloat162 l = __floats2bfloat162_rn(a - hf.x, b - hf.y);
        hi = *reinterpret_cast<uint32_t*>(&h);
        lo = *reinterpret_cast<uint32_t*>(&l);
    }
};

template <>
struct Split<false> {
    __device__ __forceinline__ static void run(float a, float b, uint32_t& hi, uint32_t& lo) {
        __half2 h = __floats2half2_rn(a, b);
        const float2 hf = __half22float2(h);
        __half2 l = __floats2half2_rn(a - hf.x, b - hf.y);
        hi = *reinterpret_cast<uint32_t*>(&h);
        lo = *reinterpret_cast<uint32_t*>(&l);
    }
};

}  // namespace tc
}  // namespace gs
