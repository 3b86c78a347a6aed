// Persistent correlation kernel with every DFT stage on the tensor cores:
// window l = 720 = 16 x 45, both passes of the 2D inverse transform as
// prime-factor (Good-Thomas) transforms, each pass two GEMMs on tcgen05:
//
//   stage 1 (45-point over n2):  D1[(v, n1)][(k2, c')] = sum_(n2, c) A1[(v, n1)][(n2, c)] F45[(k2, c')][(n2, c)]
//   stage 2 (16-point over n1):  D2[(k2, v)][(k1, c')] = sum_(n1, c) A2[(k2, v)][(n1, c)] F16[(k1, c')][(n1, c)]
//
// for the V = 8 vectors (spectrum rows in the row pass, map columns in the
// column pass) of a tile; F are the real forms of exp(+2 pi i n k / N).  The
// prime-factor index maps leave no twiddles between the stages (the same
// orders as the FP32 kernel at window 720: spectra stored with their columns
// in the input order PfaCols, spectrum rows read in that order, outputs in
// map coordinates (A1 k1 + A2 k2) mod 720).
//
// Operands are FP16: the data is rounded once per GEMM and the DFT matrices
// are either rounded once (kProducts = 1) or split into (hi, lo) with both
// products accumulated (kProducts = 2); accumulation is FP32 in TMEM.  To
// keep FP16 in range each unit's spectrum is scaled by an exact power of two
// s with max |W| max |P| s <= 1 (then every intermediate stays below
// 45 x 720 = 32400); the scores are scale free and peak / sigma are returned
// unscaled.  Row-pass maps are stored as FP16 in the scratch ring, each row
// in blocks of 8 columns [re x 8][im x 8] so that a column tile's 8 columns
// land in shared memory as an MN-major operand with plain 16-byte copies.
//
// Work queue, scratch ring, dependency counters and bounded waits are those
// of k_corr_persistent (corr.cuh); a CTA runs kWg independent pipelines of
// 128 threads (one warpgroup each: its own A operand buffer, mbarrier, TMEM
// columns and claims), so that one pipeline's SIMT work overlaps another's
// MMAs.  In a pipeline: SIMT fills A1 -> one thread issues stage 1 ->
// every thread reads its TMEM lane (row (v, n1)) and writes A2 -> stage 2 ->
// every thread reads its lanes of the three stage-2 tiles (rows (k2, v)) and
// runs the epilogue (row pass: FP16 map rows to the scratch ring; column
// pass: border-masked peak, its position and the sum of squares of both
// templates of the pair).
#pragma once

#include "corr.cuh"
#include "tc.cuh"

namespace gs {

struct Tc2Args {
    const float2* W;         // window spectra (PfaCols column order), Nw x L2
    const float2* P;         // template-pair spectra of the launch's angles (PfaCols order), (angles x pairs) x L2
    const __half2* W16;      // the same in FP16, row-tile order (k_to_half_tiles), scaled by s_w
    const __half2* P16;      // the same for the pairs, scaled by s_p
    __half2* R;              // scratch ring, S x L2 half2 (FP16 re, im in 8-column blocks)
    const float* wmax;       // per window max |W|
    const float* pmax;       // per pair max |P|
    const int2* unit_wp;     // unit -> (window, angle x pairs + pair)
    int* done_rows;          // per unit, row-tile warps finished
    int* done_cols;          // per unit, column-tile warps finished
    UnitAcc* acc;            // per unit, 2 templates (key, s2 of the scaled map)
    UnitOut* out;            // results, index angle * out_stride + w * ntmpl + J
    int* next_item;          // claim counter
    int* error;              // set when a bounded wait gives up
    int nu, ntmpl, S, lag;
    long long L2;
    int yb0, yb1;            // border interval of unshifted indices (both axes)
    int pairs;               // template pairs per angle
    long long out_stride;    // results per angle (windows x templates)
};

template <int kProducts_>
struct Tc2Cfg {
    static constexpr int kProducts = kProducts_;
    static constexpr int N1 = 16, N2 = 45, L = 720;
    using Pfa = CorrCfg<45, 16>;                // index maps of the FP32 kernel at window 720
    static constexpr int V = 8;                 // vectors per tile
    static constexpr int T = L / V;             // tiles per pass of one unit
    static constexpr int K1 = 96;               // stage 1: K = N = 2 x 48 (n2, k2 padded to 48)
    static constexpr int N2P = 48;
    static constexpr int M2 = V * N2P;          // stage-2 rows (k2, v), 384
    static constexpr int MT2 = M2 / 128;        // stage-2 M-tiles
    static constexpr int K2 = 32;               // stage 2: K = N = 2 x 16
    static constexpr int kWg = 5;               // pipelines per CTA
    static constexpr int kThreads = 128 * kWg;
    static constexpr int kDone = T;             // tile completions per pass of a unit
    static constexpr int kBatch = 2;            // items claimed (and published) together
    // stage-1 operand, row pass: K-major, 8-row groups 128 B apart, 8-element
    // K groups LBO1R apart (padded so that a warp's 4-byte stores of 32
    // consecutive columns hit distinct banks)
    static constexpr uint32_t LBO1R = 16 * 128 + 16;
    // stage-1 operand, column pass: MN-major, 8-column groups (one per n1)
    // SBO1C apart, 8-row K groups 128 B apart
    static constexpr uint32_t SBO1C = N2P * 32;  // 1536
    // stage-2 operand: K-major over 384 rows, K groups LBO2 apart
    static constexpr uint32_t LBO2 = (M2 / 8) * 128;  // 6144
    static constexpr uint32_t a_bytes = 12 * LBO1R > 4 * LBO2 ? 12 * LBO1R : 4 * LBO2;  // A1 and A2 alias
    static constexpr uint32_t b45_bytes = K1 * K1 * 2;   // one product
    static constexpr uint32_t b16_bytes = K2 * K2 * 2;
    static constexpr size_t off_b45 = 0;
    static constexpr size_t off_b16 = off_b45 + (size_t)kProducts * b45_bytes;
    static constexpr size_t off_a = ((off_b16 + (size_t)kProducts * b16_bytes + 127) / 128) * 128;
    static constexpr size_t off_bar = off_a + (size_t)kWg * a_bytes;
    static constexpr size_t off_misc = off_bar + 8 * kWg;  // tmem slot (16 B), then 4 claim slots per pipeline
    static constexpr size_t bytes = off_misc + 16 + (size_t)16 * kWg;
    static constexpr uint32_t tmem_cols = 96;             // per pipeline (stage 1 N = 96; stage 2 3 x 32, aliased)
    static constexpr uint32_t idesc1r = tc::idesc_f16_major(128, K1, 0, 0, 0);
    static constexpr uint32_t idesc1c = tc::idesc_f16_major(128, K1, 0, 1, 0);
    static constexpr uint32_t idesc2 = tc::idesc_f16_major(128, K2, 0, 0, 0);
    static_assert(bytes <= 227 * 1024, "shared memory");
    static_assert(kWg * tmem_cols <= 512, "TMEM");
    static_assert(kProducts == 1 || kProducts == 2, "products");
};

struct Tc2Wg {
    int g, wt;            // pipeline, thread within it
    unsigned char* a;     // A1 / A2
    uint32_t as;          // the same as a shared-window address
    uint64_t* bar;
    uint32_t tmem;
    int* ish;
};

// Exact power-of-two scale of one spectrum from its max |.|: max |.| x s in
// [1/2, 1) (1 for an all-zero or non-finite maximum).  A unit's map is
// computed from the product of its window's and its pair's scaled spectra,
// so its scale is s_w s_p and every intermediate stays below 45 x 720.
__host__ __device__ __forceinline__ float tc2_scale1(float m) {
    if (!(m > 1e-30f) || !(m < 1e30f)) return 1.0f;
    int e;
    frexpf(m, &e);  // m = f 2^e, f in [0.5, 1)
    return ldexpf(1.0f, -e);
}
__device__ __forceinline__ float tc2_scale(float wm, float pm) { return tc2_scale1(wm) * tc2_scale1(pm); }

// Stores to shared memory by 32-bit shared-window address.
__device__ __forceinline__ void sts32(uint32_t addr, uint32_t v) {
    asm volatile("st.shared.b32 [%0], %1;" ::"r"(addr), "r"(v) : "memory");
}
// st.shared.b32 when `pred` is nonzero (predicated inside the instruction,
// no branch around it).
__device__ __forceinline__ void sts32_if(uint32_t addr, uint32_t v, uint32_t pred) {
    asm volatile("{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %2, 0;\n\t@p st.shared.b32 [%0], %1;\n\t}"
                 ::"r"(addr), "r"(v), "r"(pred) : "memory");
}
__device__ __forceinline__ void sts128(uint32_t addr, uint4 v) {
    asm volatile("st.shared.v4.b32 [%0], {%1, %2, %3, %4};" ::"r"(addr), "r"(v.x), "r"(v.y), "r"(v.z), "r"(v.w)
                 : "memory");
}

__device__ __forceinline__ uint32_t pack_half2(float re, float im) {
    __half2 h = __floats2half2_rn(re, im);
    return *reinterpret_cast<uint32_t*>(&h);
}

// DFT matrices (inverse sign), real form, K-major, rows (k, c'), columns (n, c),
// rounded to FP16 once, or as (hi, lo) for two products.
template <class C>
__device__ void tc2_fill_dft(unsigned char* sm) {
    for (int i = threadIdx.x; i < C::K1 * C::K1; i += blockDim.x) {
        const int row = i / C::K1, col = i % C::K1;
        const int k = row >> 1, cp = row & 1, n = col >> 1, c = col & 1;
        float e = 0.0f;
        if (k < C::N2 && n < C::N2) {
            double sn, cs;
            sincospi(2.0 * (double)((k * n) % C::N2) / (double)C::N2, &sn, &cs);
            // out_re = x_re cos - x_im sin ; out_im = x_re sin + x_im cos
            e = cp ? (c ? (float)cs : (float)sn) : (c ? (float)-sn : (float)cs);
        }
        const __half hi = __float2half_rn(e);
        const uint32_t off = tc::kmajor_off(row, col, C::K1);
        *reinterpret_cast<__half*>(sm + C::off_b45 + off) = hi;
        if (C::kProducts == 2)
            *reinterpret_cast<__half*>(sm + C::off_b45 + C::b45_bytes + off) = __float2half_rn(e - __half2float(hi));
    }
    for (int i = threadIdx.x; i < C::K2 * C::K2; i += blockDim.x) {
        const int row = i / C::K2, col = i % C::K2;
        const int k = row >> 1, cp = row & 1, n = col >> 1, c = col & 1;
        double sn, cs;
        sincospi(2.0 * (double)((k * n) % C::N1) / (double)C::N1, &sn, &cs);
        const float e = cp ? (c ? (float)cs : (float)sn) : (c ? (float)-sn : (float)cs);
        const __half hi = __float2half_rn(e);
        const uint32_t off = tc::kmajor_off(row, col, C::K2);
        *reinterpret_cast<__half*>(sm + C::off_b16 + off) = hi;
        if (C::kProducts == 2)
            *reinterpret_cast<__half*>(sm + C::off_b16 + C::b16_bytes + off) = __float2half_rn(e - __half2float(hi));
    }
}

// Named barrier of one pipeline (ids 1 .. kWg; 0 is the CTA's).  bar.sync is
// the warp-aligned form: the warp is reconverged first (one lane may arrive
// from a wait the others skipped).
__device__ __forceinline__ void tc2_sync(int g) {
    __syncwarp();
    asm volatile("bar.sync %0, 128;" ::"r"(g + 1) : "memory");
}

// Bounded (about a second); gives up at once when another wait of the
// launch has already given up (error flag set), so a failed launch ends soon.
template <class C>
__device__ __forceinline__ void tc2_wait_counter(const int* p, int target, int* error) {
    if (ld_acquire_gpu(p) >= target) return;
    for (int it = 0; it < (1 << 22); ++it) {
        __nanosleep(256);
        if (ld_acquire_gpu(p) >= target) return;
        if ((it & 1023) == 1023 && *(volatile int*)error) return;
    }
    atomicExch(error, 1);
}

// Issue a GEMM stage (thread 0 of the pipeline), commit, wait for it (lane
// 0 of every warp waits on the mbarrier itself, so the warps resume as soon
// as the MMAs complete, without a pipeline barrier).  Returns false when this
// warp's bounded wait gave up.
template <class C, bool kStage2, bool kColPass>
__device__ __forceinline__ bool tc2_gemm(const Tc2Wg& w, unsigned char* sm, uint32_t& phase, int* a_error,
                                         const int* dep = nullptr) {
    tc::fence_async_smem();
    tc::fence_before_sync();
    tc2_sync(w.g);
    tc::fence_after_sync();
    int ok = 1;
    if (w.wt == 0) {
        const uint32_t a = tc::smem_u32(w.a);
        if (!kStage2) {
            const uint32_t b = tc::smem_u32(sm + C::off_b45);
            constexpr uint32_t lbo_b = C::K1 * 16;
#pragma unroll
            for (int j = 0; j < C::K1 / 16; ++j) {
                const uint64_t ad = kColPass ? tc::smem_desc(a + 2 * j * 128, 128, C::SBO1C)
                                             : tc::smem_desc(a + 2 * j * C::LBO1R, C::LBO1R, 128);
#pragma unroll
                for (int p = 0; p < C::kProducts; ++p)
                    tc::mma_f16(w.tmem, ad, tc::smem_desc(b + p * C::b45_bytes + 2 * j * lbo_b, lbo_b, 128),
                                kColPass ? C::idesc1c : C::idesc1r, (j | p) ? 1u : 0u);
            }
        } else {
            const uint32_t b = tc::smem_u32(sm + C::off_b16);
            constexpr uint32_t lbo_b = C::K2 * 16;
            // the three M-tiles' accumulators are independent: interleave
            // them so that consecutive MMAs do not wait on one another
#pragma unroll
            for (int j = 0; j < C::K2 / 16; ++j)
#pragma unroll
                for (int p = 0; p < C::kProducts; ++p)
#pragma unroll
                    for (int t = 0; t < C::MT2; ++t)
                        tc::mma_f16(w.tmem + 32 * t, tc::smem_desc(a + t * 2048 + 2 * j * C::LBO2, C::LBO2, 128),
                                    tc::smem_desc(b + p * C::b16_bytes + 2 * j * lbo_b, lbo_b, 128), C::idesc2,
                                    (j | p) ? 1u : 0u);
        }
        tc::mma_commit(w.bar);
    }
    // every warp waits for the MMAs itself (its lane 0, sleeping between
    // polls; bounded: 2 s, or 1 ms once any wait of the launch has given up)
    // and checks the dependency, so that no pipeline barrier follows
    if ((w.wt & 31) == 0) {
        const int dv = dep ? ld_acquire_gpu(dep) : C::kDone;
        const uint64_t limit = *(volatile const int*)a_error ? 1000000ull : 2000000000ull;
        if (!tc::mbar_wait_backoff(w.bar, phase, limit)) {
            ok = 0;
            atomicExch(a_error, 1);
        }
        if (dv < C::kDone) tc2_wait_counter<C>(dep, C::kDone, a_error);
    }
    phase ^= 1u;
    __syncwarp();
    tc::fence_after_sync();
    return ok != 0;
}

// Stage 1 -> stage 2: this thread's TMEM lane m = (v, n1) = (m % 8, m / 8)
// holds the 48 (k2) complex outputs; they become A2 entries (k2 v, n1).
template <class C>
__device__ __forceinline__ void tc2_transition(const Tc2Wg& w) {
    const int m = w.wt, v = m & 7, n1 = m >> 3;
    const uint32_t lane_base = w.tmem + ((uint32_t)(32 * (w.wt >> 5)) << 16);
    const uint32_t dst = w.as + (uint32_t)(n1 >> 2) * C::LBO2 + (uint32_t)v * 16 + (uint32_t)(n1 & 3) * 4;
    // A1 (aliased by A2) is no longer read: the stage-1 MMAs completed.  The
    // next 32 columns are loaded while the current ones are converted and
    // stored (tcgen05.wait::ld waits for every load issued before it).
    uint32_t r0[32], r1[32];
    tc::tmem_ld32(lane_base, r0);
    tc::tmem_ld_wait();
    tc::tmem_ld32(lane_base + 32, r1);
#pragma unroll
    for (int i = 0; i < 16; ++i)
        sts32(dst + (uint32_t)i * 128, pack_half2(__uint_as_float(r0[2 * i]), __uint_as_float(r0[2 * i + 1])));
    tc::tmem_ld_wait();
    tc::tmem_ld32(lane_base + 64, r0);
#pragma unroll
    for (int i = 0; i < 16; ++i)
        sts32(dst + (uint32_t)(16 + i) * 128, pack_half2(__uint_as_float(r1[2 * i]), __uint_as_float(r1[2 * i + 1])));
    tc::tmem_ld_wait();
#pragma unroll
    for (int i = 0; i < 16; ++i)
        sts32(dst + (uint32_t)(32 + i) * 128, pack_half2(__uint_as_float(r0[2 * i]), __uint_as_float(r0[2 * i + 1])));
}

// Conjugate product of two FP16 complex numbers (re, im) in half2
// arithmetic: w conj(p) = (w_re p_re + w_im p_im, w_im p_re - w_re p_im).
__device__ __forceinline__ uint32_t cmulc_h2(uint32_t wu, uint32_t pu) {
    const __half2 w = *reinterpret_cast<const __half2*>(&wu);
    const __half2 p = *reinterpret_cast<const __half2*>(&pu);
    const __half2 pre = __low2half2(p);                                     // (p_re, p_re)
    const __half2 pim = __hmul2(__high2half2(p), __floats2half2_rn(1.0f, -1.0f));  // (p_im, -p_im)
    const __half2 r = __hfma2(__lowhigh2highlow(w), pim, __hmul2(w, pre));
    return *reinterpret_cast<const uint32_t*>(&r);
}

// Row tile t of unit u from the FP16 spectra in tile order (k_to_half_tiles):
// rows 8 t .. 8 t + 7 hold spectrum rows spectrum_row(8 t + v), each as 16
// groups n1 of 48 values n2 (45 and three zeros), in A1's K order.  A task
// is 4 consecutive n2 of one (v, n1): two 16-byte loads, four conjugate
// products in half2 arithmetic, one 16-byte store at A1's (K group n2 / 4,
// row m = v + 8 n1).  The K padding comes from the zeros.  Consecutive lanes
// take consecutive groups: coalesced loads, and LBO1R = 16 mod 128 keeps
// the stores conflict-free.  Two rounds of six tasks per thread.
template <class C>
__device__ __forceinline__ void tc2_row_fill(const Tc2Args& a, int u, int t, const Tc2Wg& w) {
    constexpr int G = C::N2P / 4;               // 12 groups of 4 per (v, n1)
    constexpr int kRow = 16 * C::N2P;           // 768 values per row
    constexpr int kTasks = C::V * 16 * G;       // 1536
    constexpr int kRounds = 2;
    constexpr int kPer = kTasks / 128 / kRounds;  // 6 per round
    static_assert(kTasks % (128 * kRounds) == 0, "tasks");
    const int2 wp = __ldg(a.unit_wp + u);
    const uint4* Wt = reinterpret_cast<const uint4*>(a.W16 + ((long long)wp.x * C::L + 8 * t) * kRow);
    const uint4* Pt = reinterpret_cast<const uint4*>(a.P16 + ((long long)wp.y * C::L + 8 * t) * kRow);
    const unsigned long long keep = l2_policy_evict_last();
#pragma unroll 1
    for (int round = 0; round < kRounds; ++round) {
        uint4 wv[kPer], pv[kPer];
#pragma unroll
        for (int i = 0; i < kPer; ++i) {
            const int q = w.wt + 128 * (kPer * round + i);   // (v, n1, g), g fastest: uint4 index q
            asm volatile("ld.global.L1::no_allocate.L2::cache_hint.v4.u32 {%0, %1, %2, %3}, [%4], %5;"
                         : "=r"(wv[i].x), "=r"(wv[i].y), "=r"(wv[i].z), "=r"(wv[i].w) : "l"(Wt + q), "l"(keep));
            pv[i] = __ldg(Pt + q);
        }
#pragma unroll
        for (int i = 0; i < kPer; ++i) {
            const int q = w.wt + 128 * (kPer * round + i);
            const int g = q % G, vn = q / G, n1 = vn & 15, v = vn >> 4;
            const uint4 x = make_uint4(cmulc_h2(wv[i].x, pv[i].x), cmulc_h2(wv[i].y, pv[i].y),
                                       cmulc_h2(wv[i].z, pv[i].z), cmulc_h2(wv[i].w, pv[i].w));
            sts128(w.as + (uint32_t)g * C::LBO1R + (uint32_t)n1 * 128 + (uint32_t)v * 16, x);
        }
    }
}

// Column tile t of unit u: the 8 columns 8 t .. 8 t + 7 of the scratch map,
// every row r = n2 + 45 n1, into A1 (column pass layout, MN-major): 16-byte
// copies of each row's [re x 8] and [im x 8] halves.
template <class C>
__device__ __forceinline__ void tc2_col_fill(const Tc2Args& a, int u, int t, const Tc2Wg& w) {
    const __half2* Rs = a.R + (long long)(u % a.S) * a.L2;
    const unsigned long long drop = l2_policy_evict_first();
    constexpr int kChunks = 2 * C::L;  // (row, half)
    constexpr int kPer = 6;            // 16-byte chunks in flight per thread
    static_assert(kChunks <= 2 * kPer * 128, "two rounds");
    for (int base = 0; base < kChunks; base += kPer * 128) {
    uint4 vals[kPer];
#pragma unroll
    for (int i = 0; i < kPer; ++i) {
        const int q = min(base + w.wt + 128 * i, kChunks - 1);  // past the end: re-read the last chunk
        const int r = q >> 1, h = q & 1;
        const uint4* src = reinterpret_cast<const uint4*>(Rs + (long long)r * C::L + 8 * t) + h;
        asm volatile("ld.global.L1::no_allocate.L2::cache_hint.v4.u32 {%0, %1, %2, %3}, [%4], %5;"
                     : "=r"(vals[i].x), "=r"(vals[i].y), "=r"(vals[i].z), "=r"(vals[i].w)
                     : "l"(src), "l"(drop));
    }
#pragma unroll
    for (int i = 0; i < kPer; ++i) {
        const int q = min(base + w.wt + 128 * i, kChunks - 1);  // a repeated chunk stores the same bytes again
        const int r = q >> 1, h = q & 1;
        const int n1 = r / C::N2, n2 = r - n1 * C::N2;
        sts128(w.as + (uint32_t)n1 * C::SBO1C + (uint32_t)n2 * 32 + (uint32_t)h * 16, vals[i]);
    }
    }
    // K padding rows n2 = 45 .. 47 of every n1 group: zero
    for (int i = w.wt; i < 16 * 3 * 2; i += 128) {
        const int n1 = i / 6, rest = i - n1 * 6, n2 = 45 + (rest >> 1), h = rest & 1;
        sts128(w.as + (uint32_t)n1 * C::SBO1C + (uint32_t)n2 * 32 + (uint32_t)h * 16, make_uint4(0u, 0u, 0u, 0u));
    }
}

// Row-pass epilogue: stage-2 rows (k2, v) of the three M-tiles -> FP16 map
// row 8 t + v, physical columns 16 k2 .. 16 k2 + 15 (two 8-column blocks).
template <class C>
__device__ __forceinline__ void tc2_row_out(const Tc2Args& a, int u, int t, const Tc2Wg& w) {
    __half2* Rs = a.R + (long long)(u % a.S) * a.L2;
    const uint32_t lane_base = w.tmem + ((uint32_t)(32 * (w.wt >> 5)) << 16);
    const int v = w.wt & 7;
    const unsigned long long keep = l2_policy_evict_last();
    // one stage-2 tile's 16 k1 values of row (k2, v): two 8-column blocks
    // [re x 8][im x 8] of FP16 map row 8 t + v
    auto put = [&](const uint32_t* r, int ti) {
        const int k2 = 16 * ti + (w.wt >> 3);
        if (k2 >= C::N2) return;
        uint32_t o[16];
#pragma unroll
        for (int blk = 0; blk < 2; ++blk)
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                const int k1 = 8 * blk + 2 * i;
                o[8 * blk + i] = pack_half2(__uint_as_float(r[2 * k1]), __uint_as_float(r[2 * k1 + 2]));          // re
                o[8 * blk + 4 + i] = pack_half2(__uint_as_float(r[2 * k1 + 1]), __uint_as_float(r[2 * k1 + 3]));  // im
            }
        uint4* dst = reinterpret_cast<uint4*>(Rs + (long long)(8 * t + v) * C::L + 16 * k2);
#pragma unroll
        for (int i = 0; i < 4; ++i)
            asm volatile("st.global.L1::no_allocate.L2::cache_hint.v4.u32 [%0], {%1, %2, %3, %4}, %5;"
                         ::"l"(dst + i), "r"(o[4 * i]), "r"(o[4 * i + 1]), "r"(o[4 * i + 2]), "r"(o[4 * i + 3]),
                         "l"(keep) : "memory");
    };
    // the next tile's columns are loaded while the current ones are stored
    uint32_t r0[32], r1[32];
    tc::tmem_ld32(lane_base, r0);
    tc::tmem_ld_wait();
    tc::tmem_ld32(lane_base + 32, r1);
    put(r0, 0);
    tc::tmem_ld_wait();
    tc::tmem_ld32(lane_base + 64, r0);
    put(r1, 1);
    tc::tmem_ld_wait();
    put(r0, 2);
}

// Border mask of the map rows this thread's stage-2 lanes hold: bit k1 of
// word ti is set when map row (A1 k1 + A2 k2) mod L, k2 = 16 ti + wt / 8, lies
// inside the maximum's interior (outside the border interval [yb0, yb1]).
// Fixed for the life of the kernel.
struct Tc2Masks {
    uint32_t m[3];
};
template <class C>
__device__ __forceinline__ Tc2Masks tc2_row_masks(int wt, int yb0, int yb1) {
    Tc2Masks mk;
#pragma unroll
    for (int ti = 0; ti < C::MT2; ++ti) {
        const int k2 = 16 * ti + (wt >> 3);
        uint32_t m = 0u;
        if (k2 < C::N2)
            for (int k1 = 0; k1 < 16; ++k1) {
                const int y = C::Pfa::map_coord(k1, k2);
                if ((unsigned)(y - yb0) > (unsigned)(yb1 - yb0)) m |= 1u << k1;
            }
        mk.m[ti] = m;
    }
    return mk;
}

// Column-pass epilogue: values of map column x (physical column 8 t + v),
// rows map_coord(k1, k2), both templates of the pair: the sum of squares and
// the border-masked maximum (starting at 0, as the reference's peak) with its
// position, per thread (the position as (tile, k1), k1 a compile-time
// constant; among equal values the first in (tile, k1) order), then per warp
// (smallest map index among equal values), added to the unit's accumulators.
template <class C>
__device__ __forceinline__ void tc2_col_out(const Tc2Args& a, int u, int t, const Tc2Wg& w, const Tc2Masks mb) {
    constexpr int L = C::L, h = L / 2;
    static_assert((L / 2) % 2 == 0, "sign of the fftshift: (-1)^(L/2) = +1");
    const uint32_t lane_base = w.tmem + ((uint32_t)(32 * (w.wt >> 5)) << 16);
    const int pc = 8 * t + (w.wt & 7);                           // physical column
    const int x = C::Pfa::map_coord(pc & 15, pc >> 4);           // map column
    const bool xin = (unsigned)(x - a.yb0) <= (unsigned)(a.yb1 - a.yb0);  // column in the border
    float b1 = 0.0f, b2 = 0.0f, s2a = 0.0f, s2b = 0.0f;
    int k1a = -1, k1b = -1, tia = 0, tib = 0;
    // eight k1 values (half `hf` of tile ti); rows k2 >= 45 hold zeros and no bits
    auto take = [&](const float* r, int ti, int hf) {
        const uint32_t bits = xin ? 0u : (mb.m[ti] >> (8 * hf));
        const float b1_0 = b1, b2_0 = b2;
#pragma unroll
        for (int kk = 0; kk < 8; ++kk) {
            const int k1 = 8 * hf + kk;
            const float v1 = r[2 * kk], v2 = r[2 * kk + 1];
            const bool in = (bits >> kk) & 1u;
            const bool g1 = in && v1 > b1, g2 = in && v2 > b2;
            b1 = g1 ? v1 : b1;
            k1a = g1 ? k1 : k1a;
            b2 = g2 ? v2 : b2;
            k1b = g2 ? k1 : k1b;
            s2a = fmaf(v1, v1, s2a);
            s2b = fmaf(v2, v2, s2b);
        }
        // the maximum only grows strictly: it changed iff it now lies here
        tia = b1 != b1_0 ? ti : tia;
        tib = b2 != b2_0 ? ti : tib;
    };
    // 16-column halves, the next one loaded while the current one is reduced
    // (tcgen05.wait::ld waits for every load issued before it)
    float ra[16], rb[16];
    tc::tmem_ld16(lane_base, ra);
    tc::tmem_ld_wait();
    tc::tmem_ld16(lane_base + 16, rb);
    take(ra, 0, 0);
    tc::tmem_ld_wait();
    tc::tmem_ld16(lane_base + 32, ra);
    take(rb, 0, 1);
    tc::tmem_ld_wait();
    tc::tmem_ld16(lane_base + 48, rb);
    take(ra, 1, 0);
    tc::tmem_ld_wait();
    tc::tmem_ld16(lane_base + 64, ra);
    take(rb, 1, 1);
    tc::tmem_ld_wait();
    tc::tmem_ld16(lane_base + 80, rb);
    take(ra, 2, 0);
    tc::tmem_ld_wait();
    take(rb, 2, 1);
    const int X = x + h < L ? x + h : x - h;
    auto key_of = [&](float b, int k1, int ti) -> unsigned long long {
        if (k1 < 0) return 0ull;
        const int k2 = 16 * ti + (w.wt >> 3);
        const int y = C::Pfa::map_coord(k1, k2);
        const int Y = y + h < L ? y + h : y - h;
        return argmax_key(b, Y * L + X);
    };
    unsigned long long ka = key_of(b1, k1a, tia), kb = key_of(b2, k1b, tib);
    float fa = s2a, fb = s2b;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        fa += __shfl_xor_sync(0xffffffffu, fa, o);
        fb += __shfl_xor_sync(0xffffffffu, fb, o);
        const unsigned long long oa = __shfl_xor_sync(0xffffffffu, ka, o);
        const unsigned long long ob = __shfl_xor_sync(0xffffffffu, kb, o);
        ka = oa > ka ? oa : ka;
        kb = ob > kb ? ob : kb;
    }
    if ((threadIdx.x & 31) == 0) {
        UnitAcc* ac = a.acc + 2 * (long long)u;
        if (ka) atomicMax(&ac[0].key, ka);
        atomicAdd(&ac[0].s2, (double)fa);
        if (kb) atomicMax(&ac[1].key, kb);
        atomicAdd(&ac[1].s2, (double)fb);
    }
}

// The last column-tile warp of unit u: scores from the accumulators (scaled
// map, scale s), the maps' plain sums from the spectrum's DC term.
template <class C>
__device__ __forceinline__ void tc2_finish_unit(const Tc2Args& a, int u) {
    const int2 wp = a.unit_wp[u];
    const UnitAcc* ac = a.acc + 2 * (long long)u;
    const float s = tc2_scale(__ldg(a.wmax + wp.x), __ldg(a.pmax + wp.y));
    const float2 w0 = __ldg(a.W + (long long)wp.x * a.L2);
    const float2 p0 = __ldg(a.P + (long long)wp.y * a.L2);
    const double l2 = (double)a.L2;
    const double sums[2] = {l2 * ((double)w0.x * p0.x + (double)w0.y * p0.y),
                            l2 * ((double)w0.y * p0.x - (double)w0.x * p0.y)};
    const double inv = 1.0 / (double)s;
    for (int q = 0; q < 2; ++q) {
        const long long o = unit_out_index(wp.y, q, wp.x, a.pairs, a.ntmpl, a.out_stride);
        if (o < 0) break;
        UnitAcc v;
        v.key = __ldcg(&ac[q].key);
        v.s2 = __ldcg(&ac[q].s2) * inv * inv;
        // unscaled peak: the key's value is s x peak, exactly (s a power of two)
        const float pk = key_value(v.key) * (float)inv;
        v.key = v.key ? argmax_key(pk, key_index(v.key)) : 0ull;
        a.out[o] = unit_score(v, sums[q], C::L);
    }
}

// Called by a pipeline's leader thread only; a pipeline barrier follows.  A
// column tile reads its unit's row maps, so it waits before the item; a row
// tile needs its scratch slot only for its output, and checks that inside
// its stage-2 GEMM (tc2_row_dep).
template <class C>
__device__ __forceinline__ void tc2_wait_for(const Tc2Args& a, int item) {
    const int s = item / (2 * C::T), j = item - s * (2 * C::T);
    if (j >= C::T) {
        const int u = s - a.lag;
        if (u >= 0 && u < a.nu) tc2_wait_counter<C>(a.done_rows + u, C::kDone, a.error);
    }
}
// The counter a row tile of unit s waits for before writing slot s % S (the
// column tiles of unit s - S), or nullptr.
template <class C>
__device__ __forceinline__ const int* tc2_row_dep(const Tc2Args& a, int s) {
    return s >= a.S ? a.done_cols + (s - a.S) : nullptr;
}

// Count one finished tile (one thread of the pipeline, after a release fence
// that orders the pipeline's earlier stores and atomics before it); the last
// column tile of a unit computes its scores.
template <class C>
__device__ __forceinline__ void tc2_publish(const Tc2Args& a, int item) {
    const int s = item / (2 * C::T), j = item - s * (2 * C::T);
    if (j < C::T) {
        if (s < a.nu) atomicAdd(&a.done_rows[s], 1);
        return;
    }
    const int u = s - a.lag;
    if (u < 0 || u >= a.nu) return;
    const int prev = atomicAdd(&a.done_cols[u], 1);
    if (prev == C::kDone - 1) {
        // acquire: the other pipelines' accumulator atomics, published before their counts
        asm volatile("fence.acq_rel.gpu;" ::: "memory");
        tc2_finish_unit<C>(a, u);
    }
}

template <int kProducts>
__global__ void __launch_bounds__(Tc2Cfg<kProducts>::kThreads, 1) k_corr_tc2(Tc2Args a) {
    using C = Tc2Cfg<kProducts>;
    extern __shared__ __align__(128) unsigned char sm[];
    uint64_t* bars = reinterpret_cast<uint64_t*>(sm + C::off_bar);
    uint32_t* tslot = reinterpret_cast<uint32_t*>(sm + C::off_misc);
    tc2_fill_dft<C>(sm);
    if ((threadIdx.x >> 5) == 0) {
        tc::tmem_alloc(tslot, 512);
        tc::tmem_relinquish();
    }
    if (threadIdx.x == 0) {
        for (int g = 0; g < C::kWg; ++g) tc::mbar_init(bars + g, 1);
        tc::fence_mbar_init();
    }
    tc::fence_async_smem();
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    Tc2Wg w;
    w.g = threadIdx.x >> 7;
    w.wt = threadIdx.x & 127;
    w.a = sm + C::off_a + (size_t)w.g * C::a_bytes;
    w.as = tc::smem_u32(w.a);
    w.bar = bars + w.g;
    w.tmem = *tslot + (uint32_t)w.g * C::tmem_cols;
    w.ish = reinterpret_cast<int*>(sm + C::off_misc + 16) + 4 * w.g;
    const Tc2Masks ymask = tc2_row_masks<C>(w.wt, a.yb0, a.yb1);
    const int total = (a.nu + a.lag) * 2 * C::T;
    // The pipeline leader claims batches of kBatch consecutive items (one
    // atomic per batch), the pipeline processes them in order and one thread
    // publishes the whole batch after its last item (one release for all of
    // them, after the barrier that orders every warp's stores and
    // accumulator atomics before it).  Deferring within a batch cannot
    // deadlock: an item's dependency lies at least (lag - 1) x 2T items
    // earlier, far more than a batch spans, so no item waits for another item
    // of its own batch, and the earliest unpublished item's pipeline always
    // gets through the rest of its batch.
    // Claims start at 0 and advance by kBatch, so a batch starts at a
    // multiple of kBatch: every thread tells the batch's last item from the
    // item index alone (the extra barrier below must be taken by all).
    int pre = 0;  // the leader's claim of the next batch
    if (w.wt == 0) {
        const int first = atomicAdd(a.next_item, C::kBatch);
        if (first < total) tc2_wait_for<C>(a, first);
        w.ish[0] = first;
    }
    tc2_sync(w.g);
    uint32_t phase = 0;
    bool ok = true;
    int item = w.ish[0];
    for (int iter = 1; item < total; ++iter) {
        const bool last_of_batch = (item % C::kBatch == C::kBatch - 1) || (item + 1 >= total);
        // the next batch is claimed at this batch's first item, well before it is needed
        if (w.wt == 0 && item % C::kBatch == 0) pre = atomicAdd(a.next_item, C::kBatch);
        const int s = item / (2 * C::T), j = item - s * (2 * C::T);
        if (j < C::T) {
            if (s < a.nu) {
                tc2_row_fill<C>(a, s, j, w);
                ok &= tc2_gemm<C, false, false>(w, sm, phase, a.error);
                tc2_transition<C>(w);
                ok &= tc2_gemm<C, true, false>(w, sm, phase, a.error, tc2_row_dep<C>(a, s));
                tc2_row_out<C>(a, s, j, w);
            }
        } else {
            const int u = s - a.lag;
            if (u >= 0 && u < a.nu) {
                tc2_col_fill<C>(a, u, j - C::T, w);
                ok &= tc2_gemm<C, false, true>(w, sm, phase, a.error);
                tc2_transition<C>(w);
                ok &= tc2_gemm<C, true, true>(w, sm, phase, a.error);
                tc2_col_out<C>(a, u, j - C::T, w, ymask);
            }
        }
        if (last_of_batch) {
            // every warp's stores and atomics of the batch before the release
            tc2_sync(w.g);
            // published by lane 0 of the pipeline's last warp, so that its
            // fence and atomics overlap the leader's wait for the next item
            if (w.wt == 96) {
                // release: the batch's stores and atomics (ordered before by
                // the barrier) before its counts
                asm volatile("fence.acq_rel.gpu;" ::: "memory");
                for (int q = item - item % C::kBatch; q <= item; ++q) tc2_publish<C>(a, q);
            }
        }
        if (w.wt == 0) {
            const int nxt = last_of_batch ? pre : item + 1;
            if (nxt < total) tc2_wait_for<C>(a, nxt);
            w.ish[iter & 3] = nxt;
        }
        // this pipeline's operand buffer and TMEM columns are free again and
        // its next item's dependency is resolved
        tc::fence_before_sync();
        tc2_sync(w.g);
        tc::fence_after_sync();
        item = w.ish[iter & 3];
    }
    if (!ok && w.wt == 0) atomicExch(a.error, 1);
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    if ((threadIdx.x >> 5) == 0) tc::tmem_dealloc(*tslot, 512);
}

// FP16 copy of `count` window or pair spectra (PfaCols column order, natural
// row order) in the all-tensor-core row tiles' order: image i scaled by the
// exact power of two tc2_scale1(maxabs[i]); row r of the copy holds spectrum
// row spectrum_row(r) as 16 groups n1 of 48 values (physical columns
// 45 n1 .. 45 n1 + 44, then three zeros).
__global__ void k_to_half_tiles(const float2* __restrict__ z, const float* __restrict__ maxabs,
                                __half2* __restrict__ out) {
    using F = CorrCfg<45, 16>;
    constexpr int L = 720, kRow = 16 * 48;
    const float s = tc2_scale1(__ldg(maxabs + blockIdx.y));
    const float2* img = z + (long long)blockIdx.y * L * L;
    __half2* o = out + (long long)blockIdx.y * L * kRow;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < L * kRow; i += gridDim.x * blockDim.x) {
        const int r = i / kRow, rest = i - r * kRow, n1 = rest / 48, n2 = rest - n1 * 48;
        float2 v = make_float2(0.0f, 0.0f);
        if (n2 < 45) v = img[(long long)F::spectrum_row(r) * L + 45 * n1 + n2];
        o[i] = __floats2half2_rn(v.x * s, v.y * s);
    }
}

// Per-row-block maximum of |z| of `count` images of l2 complex values each,
// as float bits (non-negative floats order like their bit patterns).
__global__ void k_max_abs(const float2* __restrict__ z, long long l2, float* __restrict__ out) {
    const float2* img = z + (long long)blockIdx.y * l2;
    float m = 0.0f;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < l2; i += (long long)gridDim.x * blockDim.x) {
        const float2 v = img[i];
        m = fmaxf(m, fmaxf(fabsf(v.x), fabsf(v.y)));
    }
    for (int o = 16; o; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) atomicMax(reinterpret_cast<unsigned int*>(out) + blockIdx.y, __float_as_uint(m));
}

}  // namespace gs
