// Persistent correlation kernel with the N2-point DFT stage on the tensor
// cores (tcgen05, split 16-bit precision, f32 accumulation in TMEM).
//
// Same work queue, dependencies, scratch ring and bounded waits as
// k_corr_persistent (corr.cuh); the tiles differ.  The length-L inverse DFT
// of a vector (L = 16 N2) is taken in four steps with n = N2 a + b and
// k = ka + 16 kb:
//   1. for each b: 16-point DFT over a in FP32 registers (regfft.cuh), then
//      the twiddle exp(+2 pi i b ka / L)            -> Y[v][ka][b]
//   2. for each (v, ka): N2-point DFT over b as a real GEMM on the tensor
//      cores: D[(v,ka)][(kb,c')] = sum_(b,c) Y[(v,ka)][(b,c)] F[(kb,c')][(b,c)]
//      with F the real form of exp(+2 pi i b kb / N2).
// Both Y and F are split into 16-bit (hi, lo) parts and D accumulates
// hi*hi + lo*hi + hi*lo, so the stage keeps about 16 (BF16) or 22 (FP16)
// significant bits per operand.  FP16 needs bounded data (see a_scale).
//
// A tile is 8 vectors (rows in the row pass, columns in the column pass):
// the GEMM has M = 8 x 16 = 128 rows (row index ka * 8 + v), K = N = 2 N2
// rounded up to 16.  A CTA (one per SM) runs three independent pipelines,
// one per warpgroup of 128 threads: each claims its own work items, has its
// own A operand buffers, mbarrier, TMEM column slice and named barrier, and
// all three share one copy of the DFT matrix, so one pipeline's MMAs overlap
// the others' FP32 work with 12 warps per SM.  In a pipeline one thread
// issues the MMAs, one lane per warp polls the mbarrier their commit arrives
// on, and every warp then reads its 32 TMEM lanes.  Operands are K-major
// interleaved tiles (tc.cuh).
#pragma once

#include "corr.cuh"
#include "tc.cuh"

namespace gs {

constexpr int kTcWgThreads = 128;               // threads of one pipeline (warpgroup)
constexpr int kTcWarps = kTcWgThreads / 32;     // warps per tile

template <int N2, bool kBf16>
struct TcCfg {
    static constexpr int L = 16 * N2;
    static constexpr int V = 8;                         // vectors per tile
    static constexpr int T = L / V;                     // tiles per pass of one unit
    static constexpr int KP = ((2 * N2 + 15) / 16) * 16;  // GEMM K = N
    static constexpr int M = 128;
    static constexpr uint32_t idesc = tc::idesc_f16(M, KP, kBf16 ? 1 : 0);
    // FP16 keeps the data operand inside its range (max 65504) by an exact
    // power-of-two prescale, undone by the matrix: (A / 16) (16 F) = A F.
    // With amplitude-normalised spectra (phase_flip 1) the data stays below
    // about 2e4 at l <= 768.
    static constexpr float a_scale = kBf16 ? 1.0f : 0.0625f;
    static constexpr float b_scale = kBf16 ? 1.0f : 16.0f;
    // products per K step: both operands split (hi*hi + lo*hi + hi*lo).  A
    // DFT matrix rounded once to FP16 (hi*F + lo*F, one matrix copy less and
    // three CTAs per SM) gives about 2e-4 score error and moves peaks between
    // near-equal pixels, which changes picks; it is not used.
    static constexpr int kProducts = 3;
    static constexpr int kWg = 3;                          // pipelines per CTA
    static constexpr int kThreads = kWg * kTcWgThreads;
    // shared memory: shared DFT matrix and twiddles, then per pipeline its A
    // operand (hi, lo), then the mbarriers and the small slots
    static constexpr size_t a_bytes = (size_t)M * KP * 2;   // one of hi / lo
    static constexpr size_t b_bytes = (size_t)KP * KP * 2;
    static constexpr size_t off_b_hi = 0;
    static constexpr size_t off_b_lo = off_b_hi + b_bytes;
    static constexpr size_t off_tw = off_b_lo + b_bytes;
    static constexpr size_t tw_bytes = (size_t)16 * N2 * sizeof(float2);
    static constexpr size_t off_a = ((off_tw + tw_bytes + 127) / 128) * 128;
    static constexpr size_t off_bar = off_a + (size_t)kWg * 2 * a_bytes;
    static constexpr size_t off_misc = off_bar + 8 * kWg;  // tmem slot, then 4 broadcast slots per pipeline
    static constexpr size_t bytes = off_misc + 16 + (size_t)16 * kWg;
    static constexpr uint32_t tmem_cols = KP <= 64 ? 64 : 128;   // per pipeline
    static constexpr uint32_t tmem_alloc_cols = kWg * tmem_cols <= 128 ? 128 : kWg * tmem_cols <= 256 ? 256 : 512;
    static_assert(L % V == 0, "tile");
    static_assert(KP <= 256 && KP % 16 == 0, "N");
    static_assert(kWg * tmem_cols <= 512, "TMEM");
    static_assert(bytes <= 227 * 1024, "shared memory");
};

// One pipeline (warpgroup) of a CTA: its thread index, operand buffers,
// mbarrier, TMEM columns and broadcast slots.
struct TcWg {
    int g, wt;                 // pipeline, thread within it
    unsigned char* a_hi;
    unsigned char* a_lo;
    uint64_t* bar;
    uint32_t tmem;
    int* ish;
};

// Barrier of one pipeline's 128 threads (named barrier g + 1; 0 is the CTA's).
__device__ __forceinline__ void wg_sync(int g) {
    asm volatile("bar.sync %0, %1;" ::"r"(g + 1), "r"(kTcWgThreads) : "memory");
}

// Step 1 of a tile: FP32 16-point DFTs + twiddle, split and stored into the
// A operand.  Lane mapping v = task % 8, b = task / 8 keeps both the global
// loads (8 rows x 4 consecutive b, or 4 rows x 8 consecutive columns) and
// the 4-byte shared stores (banks (v, b % 4)) conflict-free.
template <int N2, bool kBf16, class Load>
__device__ __forceinline__ void tc_step1(const Load& load, const TcWg& w, const float2* twt) {
    using C = TcCfg<N2, kBf16>;
    unsigned char* a_hi = w.a_hi;
    unsigned char* a_lo = w.a_lo;
    for (int task = w.wt; task < C::V * N2; task += kTcWgThreads) {
        const int v = task & 7, b = task >> 3;
        float2 x[16];
#pragma unroll
        for (int a = 0; a < 16; ++a) x[a] = load(v, N2 * a + b);
        rf::rfft<16, 1, true>(x);
        rf::static_for<16>([&](auto kc) {
            constexpr int ka = decltype(kc)::value;
            float2 y = ka ? cmul(x[rf::rpos<16>(ka)], twt[ka * N2 + b]) : x[rf::rpos<16>(ka)];
            if (!kBf16) y = cscale(y, C::a_scale);
            uint32_t hi, lo;
            tc::Split<kBf16>::run(y.x, y.y, hi, lo);
            const uint32_t off = tc::kmajor_off(ka * 8 + v, 2 * b, C::M);
            *reinterpret_cast<uint32_t*>(a_hi + off) = hi;
            *reinterpret_cast<uint32_t*>(a_lo + off) = lo;
        });
    }
}

// Step 2: the split GEMM, issued by thread 0, completion on the mbarrier.
template <int N2, bool kBf16>
__device__ __forceinline__ void tc_issue(const TcWg& w, unsigned char* sm) {
    using C = TcCfg<N2, kBf16>;
    if (w.wt != 0) return;
    const uint32_t tmem = w.tmem;
    uint64_t* bar = w.bar;
    const uint32_t a_hi = tc::smem_u32(w.a_hi), a_lo = tc::smem_u32(w.a_lo);
    const uint32_t b_hi = tc::smem_u32(sm + C::off_b_hi), b_lo = tc::smem_u32(sm + C::off_b_lo);
    constexpr uint32_t lbo_a = C::M * 16, lbo_b = C::KP * 16;
    uint32_t acc = 0;
#pragma unroll
    for (int j = 0; j < C::KP / 16; ++j) {
        const uint32_t oa = 2 * j * lbo_a, ob = 2 * j * lbo_b;
        tc::mma_f16(tmem, tc::smem_desc(a_hi + oa, lbo_a, 128), tc::smem_desc(b_hi + ob, lbo_b, 128), C::idesc, acc);
        acc = 1;
        tc::mma_f16(tmem, tc::smem_desc(a_lo + oa, lbo_a, 128), tc::smem_desc(b_hi + ob, lbo_b, 128), C::idesc, 1);
        if (C::kProducts == 3)
            tc::mma_f16(tmem, tc::smem_desc(a_hi + oa, lbo_a, 128), tc::smem_desc(b_lo + ob, lbo_b, 128), C::idesc, 1);
    }
    tc::mma_commit(bar);
}

// Publish step 1 to the tensor core, run step 2, wait for it.  Returns false
// when the bounded wait gave up (the error flag is raised by the caller).
template <int N2, bool kBf16>
__device__ __forceinline__ bool tc_gemm(const TcWg& w, unsigned char* sm, uint32_t& phase) {
    tc::fence_async_smem();
    tc::fence_before_sync();
    wg_sync(w.g);
    tc::fence_after_sync();
    tc_issue<N2, kBf16>(w, sm);
    __syncwarp();
    // one lane per warp polls the barrier (128 pollers of one shared word
    // throttle the shared-memory pipe); the warp then synchronises with it
    int ok = 1;
    if ((threadIdx.x & 31) == 0) ok = tc::mbar_wait(w.bar, phase, 1u << 24) ? 1 : 0;
    ok = __shfl_sync(0xffffffffu, ok, 0);
    phase ^= 1u;
    tc::fence_after_sync();
    return ok != 0;
}

// This thread's GEMM row (KP columns = KP / 2 complex outputs kb) from TMEM,
// all loads issued before one wait.
template <int KP>
__device__ __forceinline__ void tc_read_row(const TcWg& w, uint32_t* r) {
    // warp k of a pipeline (CTA warp 4 g + k) may read TMEM lanes 32 k .. 32 k + 31
    const uint32_t base = w.tmem + ((uint32_t)(32 * (w.wt >> 5)) << 16);
#pragma unroll
    for (int q = 0; q < KP / 32; ++q) tc::tmem_ld32(base + 32 * q, r + 32 * q);
    tc::tmem_ld_wait();
}

// Publishes one warp's share of a tile: its stores or atomics, then the
// counter increment with release semantics.
__device__ __forceinline__ void publish_warp(int* counter) {
    __syncwarp();
    if ((threadIdx.x & 31) == 0) asm volatile("red.release.gpu.global.add.s32 [%0], 1;" ::"l"(counter) : "memory");
}

template <int N2, bool kBf16>
__device__ __forceinline__ bool tc_row_tile(const CorrArgs& a, int u, int t, const TcWg& w, unsigned char* sm,
                                            const float2* twt, uint32_t& phase) {
    using C = TcCfg<N2, kBf16>;
    constexpr int L = C::L;
    const int2 wp = a.unit_wp[u];
    const float2* Wr = a.W + (long long)wp.x * a.L2;
    const float2* Pr = a.P + (long long)wp.y * a.L2;
    float2* Rs = a.R + (long long)(u % a.S) * a.L2;
    const int r0 = t * C::V;
    const unsigned long long keep = l2_policy_evict_last();
    auto load = [&](int v, int n) {
        const long long o = (long long)(r0 + v) * L + n;
        return cmulc(ld_l2hint(Wr + o, keep), __ldg(Pr + o));
    };
    tc_step1<N2, kBf16>(load, w, twt);
    const bool ok = tc_gemm<N2, kBf16>(w, sm, phase);
    const int r = w.wt, ka = r >> 3, v = r & 7;
    float2* dst = Rs + (long long)(r0 + v) * L + ka;
    uint32_t o[C::KP];
    tc_read_row<C::KP>(w, o);
#pragma unroll
    for (int kb = 0; kb < N2; ++kb)
        st_l2hint(dst + 16 * kb, make_float2(__uint_as_float(o[2 * kb]), __uint_as_float(o[2 * kb + 1])), keep);
    publish_warp(&a.done_rows[u]);
    return ok;
}

template <int N2, bool kBf16>
__device__ __forceinline__ bool tc_col_tile(const CorrArgs& a, int u, int t, const TcWg& w, unsigned char* sm,
                                            const float2* twt, uint32_t& phase, bool* last_out) {
    using C = TcCfg<N2, kBf16>;
    constexpr int L = C::L;
    constexpr int h = L / 2;
    const float2* Rs = a.R + (long long)(u % a.S) * a.L2;
    const int c0 = t * C::V;
    const unsigned long long drop = l2_policy_evict_first();
    auto load = [&](int v, int n) { return ld_l2hint(Rs + (long long)n * L + c0 + v, drop); };
    tc_step1<N2, kBf16>(load, w, twt);
    const bool ok = tc_gemm<N2, kBf16>(w, sm, phase);
    const int r = w.wt, ka = r >> 3, v = r & 7;
    const int x = c0 + v;
    const bool xin = (unsigned)(x - a.yb0) > (unsigned)(a.yb1 - a.yb0);
    float best1 = 0.0f, best2 = 0.0f;
    int bk1 = -1, bk2 = -1;
    float s1a = 0.f, s2a = 0.f, s1b = 0.f, s2b = 0.f;
    {
        uint32_t o[C::KP];
        tc_read_row<C::KP>(w, o);
#pragma unroll
        for (int kb = 0; kb < N2; ++kb) {
            const int y = ka + 16 * kb;
            const bool in = xin && ((unsigned)(y - a.yb0) > (unsigned)(a.yb1 - a.yb0));
            const float v1 = ((L / 2) % 2 == 0) ? __uint_as_float(o[2 * kb]) : -__uint_as_float(o[2 * kb]);
            const float v2 = ((L / 2) % 2 == 0) ? __uint_as_float(o[2 * kb + 1]) : -__uint_as_float(o[2 * kb + 1]);
            const bool g1 = in && v1 > best1, g2 = in && v2 > best2;
            best1 = g1 ? v1 : best1;
            bk1 = g1 ? kb : bk1;
            best2 = g2 ? v2 : best2;
            bk2 = g2 ? kb : bk2;
            s1a += v1; s2a = fmaf(v1, v1, s2a);
            s1b += v2; s2b = fmaf(v2, v2, s2b);
        }
    }
    const int X = x + h < L ? x + h : x - h;
    unsigned long long ka_key = 0ull, kb_key = 0ull;
    if (bk1 >= 0) {
        const int y = ka + 16 * bk1;
        const int Y = y + h < L ? y + h : y - h;
        ka_key = argmax_key(best1, Y * L + X);
    }
    if (bk2 >= 0) {
        const int y = ka + 16 * bk2;
        const int Y = y + h < L ? y + h : y - h;
        kb_key = argmax_key(best2, Y * L + X);
    }
    double d1a = warp_sum((double)s1a), d2a = warp_sum((double)s2a);
    double d1b = warp_sum((double)s1b), d2b = warp_sum((double)s2b);
    ka_key = warp_max_u64(ka_key);
    kb_key = warp_max_u64(kb_key);
    bool last = false;
    if ((threadIdx.x & 31) == 0) {
        UnitAcc* ac = a.acc + 2 * (long long)u;
        if (ka_key) atomicMax(&ac[0].key, ka_key);
        atomicAdd(&ac[0].s1, d1a);
        atomicAdd(&ac[0].s2, d2a);
        if (kb_key) atomicMax(&ac[1].key, kb_key);
        atomicAdd(&ac[1].s1, d1b);
        atomicAdd(&ac[1].s2, d2b);
        int prev;
        asm volatile("atom.acq_rel.gpu.global.add.s32 %0, [%1], 1;" : "=r"(prev) : "l"(&a.done_cols[u]) : "memory");
        last = prev == kTcWarps * C::T - 1;
    }
    *last_out = last;
    return ok;
}

// The pipeline leader waits until *p >= target (bounded like wait_counter_warp).
__device__ __forceinline__ void tc_wait_counter(const int* p, int target, int* error) {
    if (ld_acquire_gpu(p) >= target) return;
    for (int it = 0; it < (1 << 22); ++it) {
        __nanosleep(256);
        if (ld_acquire_gpu(p) >= target) {
            __threadfence();
            return;
        }
    }
    atomicExch(error, 1);
}

// Called by a pipeline's leader thread only.
template <int N2, bool kBf16>
__device__ __forceinline__ void tc_wait_for(const CorrArgs& a, int item) {
    using C = TcCfg<N2, kBf16>;
    const int s = item / (2 * C::T), j = item - s * (2 * C::T);
    if (j < C::T) {
        if (s < a.nu && s >= a.S) tc_wait_counter(a.done_cols + (s - a.S), kTcWarps * C::T, a.error);
    } else {
        const int u = s - a.lag;
        if (u >= 0 && u < a.nu) tc_wait_counter(a.done_rows + u, kTcWarps * C::T, a.error);
    }
}

template <int N2, bool kBf16>
__global__ void __launch_bounds__(TcCfg<N2, kBf16>::kThreads, 1) k_corr_tc(CorrArgs a) {
    using C = TcCfg<N2, kBf16>;
    extern __shared__ __align__(128) unsigned char smt[];
    float2* twt = reinterpret_cast<float2*>(smt + C::off_tw);
    uint64_t* bars = reinterpret_cast<uint64_t*>(smt + C::off_bar);
    uint32_t* tslot = reinterpret_cast<uint32_t*>(smt + C::off_misc);
    // twiddles exp(+2 pi i b ka / L), table [ka][b]
    for (int i = threadIdx.x; i < 16 * N2; i += C::kThreads) {
        const int ka = i / N2, b = i - ka * N2;
        double sn, cs;
        sincospi(2.0 * (double)((b * ka) % C::L) / (double)C::L, &sn, &cs);
        twt[i] = make_float2((float)cs, (float)sn);
    }
    // DFT-N2 matrix (inverse sign), real form, split; rows (kb, c'), columns (b, c)
    for (int i = threadIdx.x; i < C::KP * C::KP / 2; i += C::kThreads) {
        const int row = (2 * i) / C::KP, col = (2 * i) % C::KP;  // col even: (b, re), (b, im)
        const int kb = row >> 1, cp = row & 1, b = col >> 1;
        float e0 = 0.f, e1 = 0.f;
        if (kb < N2 && b < N2) {
            double sn, cs;
            sincospi(2.0 * (double)((b * kb) % N2) / (double)N2, &sn, &cs);
            // out_re = x_re cos - x_im sin ; out_im = x_re sin + x_im cos
            e0 = cp ? (float)sn : (float)cs;
            e1 = cp ? (float)cs : (float)-sn;
        }
        e0 *= C::b_scale;
        e1 *= C::b_scale;
        uint32_t hi, lo;
        tc::Split<kBf16>::run(e0, e1, hi, lo);
        const uint32_t off = tc::kmajor_off(row, col, C::KP);
        *reinterpret_cast<uint32_t*>(smt + C::off_b_hi + off) = hi;
        *reinterpret_cast<uint32_t*>(smt + C::off_b_lo + off) = lo;
    }
    // K padding of every pipeline's A operand stays zero (step 1 writes only b < N2)
    for (int i = threadIdx.x; i < C::kWg * C::M * C::KP / 2; i += C::kThreads) {
        const int g = i / (C::M * C::KP / 2), k = i - g * (C::M * C::KP / 2);
        const int row = (2 * k) / C::KP, col = (2 * k) % C::KP;
        if ((col >> 1) >= N2) {
            const uint32_t off = tc::kmajor_off(row, col, C::M);
            unsigned char* base = smt + C::off_a + (size_t)g * 2 * C::a_bytes;
            *reinterpret_cast<uint32_t*>(base + off) = 0u;
            *reinterpret_cast<uint32_t*>(base + C::a_bytes + off) = 0u;
        }
    }
    if ((threadIdx.x >> 5) == 0) {
        tc::tmem_alloc(tslot, C::tmem_alloc_cols);
        tc::tmem_relinquish();
    }
    if (threadIdx.x == 0) {
        for (int g = 0; g < C::kWg; ++g) tc::mbar_init(bars + g, 1);
        tc::fence_mbar_init();
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    TcWg w;
    w.g = threadIdx.x / kTcWgThreads;
    w.wt = threadIdx.x - w.g * kTcWgThreads;
    w.a_hi = smt + C::off_a + (size_t)w.g * 2 * C::a_bytes;
    w.a_lo = w.a_hi + C::a_bytes;
    w.bar = bars + w.g;
    w.tmem = *tslot + (uint32_t)w.g * C::tmem_cols;
    w.ish = reinterpret_cast<int*>(smt + C::off_misc + 16) + 4 * w.g;
    const int total = (a.nu + a.lag) * 2 * C::T;
    if (w.wt == 0) {
        const int first = atomicAdd(a.next_item, 1);
        if (first < total) tc_wait_for<N2, kBf16>(a, first);
        w.ish[0] = first;
    }
    wg_sync(w.g);
    uint32_t phase = 0;
    bool ok = true;
    int item = w.ish[0];
    for (int iter = 1; item < total; ++iter) {
        int nxt = 0;
        if (w.wt == 0) nxt = atomicAdd(a.next_item, 1);
        const int s = item / (2 * C::T), j = item - s * (2 * C::T);
        if (j < C::T) {
            if (s < a.nu) ok &= tc_row_tile<N2, kBf16>(a, s, j, w, smt, twt, phase);
        } else {
            const int u = s - a.lag;
            if (u >= 0 && u < a.nu) {
                bool last = false;
                ok &= tc_col_tile<N2, kBf16>(a, u, j - C::T, w, smt, twt, phase, &last);
                if ((threadIdx.x & 31) == 0 && last) {
                    __threadfence();
                    const int2 wp = a.unit_wp[u];
                    const UnitAcc* ac = a.acc + 2 * (long long)u;
                    for (int q = 0; q < 2; ++q) {
                        const long long o = unit_out_index(wp.y, q, wp.x, a.pairs, a.ntmpl, a.out_stride);
                        if (o < 0) break;
                        UnitAcc v;
                        v.key = __ldcg(&ac[q].key);
                        v.s1 = __ldcg(&ac[q].s1);
                        v.s2 = __ldcg(&ac[q].s2);
                        a.out[o] = unit_score(v, C::L);
                    }
                }
            }
        }
        if (w.wt == 0) {
            if (nxt < total) tc_wait_for<N2, kBf16>(a, nxt);
            w.ish[iter & 3] = nxt;
        }
        // this pipeline's A operand and TMEM columns are free again (all reads
        // done) and its next item is published
        tc::fence_before_sync();
        wg_sync(w.g);
        tc::fence_after_sync();
        item = w.ish[iter & 3];
    }
    if (!ok && w.wt == 0) atomicExch(a.error, 1);
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    if ((threadIdx.x >> 5) == 0) tc::tmem_dealloc(*tslot, C::tmem_alloc_cols);
}

}  // namespace gs
