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
    const float2* P;         // template-pair spectra of this angle (PfaCols order), Np x L2
    __half2* R;              // scratch ring, S x L2 half2 (FP16 re, im in 8-column blocks)
    const float* wmax;       // per window max |W|
    const float* pmax;       // per pair max |P|
    const int2* unit_wp;     // unit -> (window, pair)
    int* done_rows;          // per unit, row-tile warps finished
    int* done_cols;          // per unit, column-tile warps finished
    UnitAcc* acc;            // per unit, 2 templates (key, s2 of the scaled map)
    UnitOut* out;            // this angle's results, index w * ntmpl + J
    int* next_item;          // claim counter
    int* error;              // set when a bounded wait gives up
    int nu, ntmpl, S, lag;
    long long L2;
    int yb0, yb1;            // border interval of unshifted indices (both axes)
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
    static constexpr int kBatch = 4;            // items claimed (and published) together
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
    uint64_t* bar;
    uint32_t tmem;
    int* ish;
};

// exact power-of-two scale s of a unit: max |W| max |P| s in (1/2, 1]
__device__ __forceinline__ float tc2_scale(float wm, float pm) {
    const float m = wm * pm;
    if (!(m > 1e-30f) || !(m < 1e30f)) return 1.0f;
    int e;
    frexpf(m, &e);          // m = f 2^e, f in [0.5, 1)
    return ldexpf(1.0f, -e);
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

// Named barrier of one pipeline (ids 1 .. kWg; 0 is the CTA's).
__device__ __forceinline__ void tc2_sync(int g) { asm volatile("bar.sync %0, 128;" ::"r"(g + 1) : "memory"); }

// Issue a GEMM stage (thread 0 of the pipeline), commit, wait for it (one
// lane per warp polls the mbarrier).  Returns false when the bounded wait gave up.
template <class C, bool kStage2, bool kColPass>
__device__ __forceinline__ bool tc2_gemm(const Tc2Wg& w, unsigned char* sm, uint32_t& phase, const int* a_error) {
    tc::fence_async_smem();
    tc::fence_before_sync();
    tc2_sync(w.g);
    tc::fence_after_sync();
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
    __syncwarp();
    int ok = 1;
    // once any wait of the launch has given up, later waits end quickly
    // lane 0 sleeps in try_wait until the MMAs complete (bounded: 2 s, or
    // 1 ms once any wait of the launch has given up)
    if ((threadIdx.x & 31) == 0)
        ok = tc::mbar_wait_suspend(w.bar, phase, 100000u,
                                   *(volatile int*)a_error ? 1000000ull : 2000000000ull) ? 1 : 0;
    if (!ok && (threadIdx.x & 31) == 0) atomicExch(const_cast<int*>(a_error), 1);
    ok = __shfl_sync(0xffffffffu, ok, 0);
    phase ^= 1u;
    tc::fence_after_sync();
    return ok != 0;
}

// Stage 1 -> stage 2: this thread's TMEM lane m = (v, n1) = (m % 8, m / 8)
// holds the 48 (k2) complex outputs; they become A2 entries (k2 v, n1).
template <class C>
__device__ __forceinline__ void tc2_transition(const Tc2Wg& w) {
    const int m = w.wt, v = m & 7, n1 = m >> 3;
    const uint32_t lane_base = w.tmem + ((uint32_t)(32 * (w.wt >> 5)) << 16);
    uint32_t r[32];
    unsigned char* dst = w.a + (uint32_t)(n1 >> 2) * C::LBO2 + (uint32_t)v * 16 + (uint32_t)(n1 & 3) * 4;
#pragma unroll 1
    for (int q = 0; q < 3; ++q) {
        tc::tmem_ld32(lane_base + 32 * q, r);
        tc::tmem_ld_wait();
#pragma unroll
        for (int i = 0; i < 16; ++i) {
            // A1 (aliased by A2) is no longer read: the stage-1 MMAs completed
            const int k2 = 16 * q + i;
            *reinterpret_cast<uint32_t*>(dst + (uint32_t)k2 * 128) =
                pack_half2(__uint_as_float(r[2 * i]), __uint_as_float(r[2 * i + 1]));
        }
    }
}

// Per-thread constants of the row fill: column chunk i of warp w covers
// columns c = 32 (w + 4 i) + lane (23 chunks per row, the last 16 wide); its
// A1 offset (row group n1, K position (n2, re/im)) without the row v, and
// whether the column exists.
struct Tc2FillMap {
    uint32_t off[6];
    uint32_t valid;  // bit i
};
template <class C>
__device__ __forceinline__ Tc2FillMap tc2_fill_map(int wt) {
    Tc2FillMap f;
    f.valid = 0u;
    const int warp = wt >> 5, lane = wt & 31;
#pragma unroll
    for (int i = 0; i < 6; ++i) {
        const int c = 32 * (warp + 4 * i) + lane;
        const int n1 = c / C::N2, n2 = c - n1 * C::N2;
        f.off[i] = (uint32_t)(n2 >> 2) * C::LBO1R + (uint32_t)n1 * 128 + (uint32_t)(n2 & 3) * 4;
        if (c < C::L) f.valid |= 1u << i;
    }
    return f;
}

// Row tile t of unit u: spectrum rows spectrum_row(8 t + v), product with the
// pair spectrum, scaled, into A1 (row pass layout: row m = v + 8 n1 of the
// operand is 8-row group n1, row v in it).  Row by row, the six column
// chunks of a row are loaded together (one base pointer per row, the chunks
// at fixed offsets) before any is used.
template <class C>
__device__ __forceinline__ void tc2_row_fill(const Tc2Args& a, int u, int t, const Tc2Wg& w, float s,
                                             const Tc2FillMap& fm) {
    const int2 wp = __ldg(a.unit_wp + u);
    const int warp = w.wt >> 5, lane = w.wt & 31;
    const float2* Wr = a.W + (long long)wp.x * a.L2 + 32 * warp + lane;
    const float2* Pr = a.P + (long long)wp.y * a.L2 + 32 * warp + lane;
    const unsigned long long keep = l2_policy_evict_last();
#pragma unroll 1
    for (int v = 0; v < C::V; ++v) {
        const int row = C::Pfa::spectrum_row(8 * t + v) * C::L;
        const float2* pw = Wr + row;
        const float2* pp = Pr + row;
        float2 wv[6], pv[6];
#pragma unroll
        for (int i = 0; i < 6; ++i)
            if ((fm.valid >> i) & 1u) {
                wv[i] = ld_l2hint(pw + 128 * i, keep);
                pv[i] = __ldg(pp + 128 * i);
            }
        unsigned char* dst = w.a + (uint32_t)v * 16;
#pragma unroll
        for (int i = 0; i < 6; ++i)
            if ((fm.valid >> i) & 1u) {
                const float2 x = cmulc(wv[i], pv[i]);
                *reinterpret_cast<uint32_t*>(dst + fm.off[i]) = pack_half2(x.x * s, x.y * s);
            }
    }
    // K padding n2 = 45 .. 47 (K group 11, entries 1 .. 3): zero (their B rows are zero too)
    for (int i = w.wt; i < 128 * 3; i += 128) {
        const int m = i / 3, n2 = 45 + (i - (i / 3) * 3);
        *reinterpret_cast<uint32_t*>(w.a + 11u * C::LBO1R + (uint32_t)(m >> 3) * 128 + (uint32_t)(m & 7) * 16 +
                                     (uint32_t)(n2 & 3) * 4) = 0u;
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
    static_assert(kChunks <= 2 * kPer * 128, "two batches");
    for (int base = 0; base < kChunks; base += kPer * 128) {
    uint4 vals[kPer];
#pragma unroll
    for (int i = 0; i < kPer; ++i) {
        const int q = base + w.wt + 128 * i;
        if (q < kChunks) {
            const int r = q >> 1, h = q & 1;
            const uint4* src = reinterpret_cast<const uint4*>(Rs + (long long)r * C::L + 8 * t) + h;
            asm volatile("ld.global.L1::no_allocate.L2::cache_hint.v4.u32 {%0, %1, %2, %3}, [%4], %5;"
                         : "=r"(vals[i].x), "=r"(vals[i].y), "=r"(vals[i].z), "=r"(vals[i].w)
                         : "l"(src), "l"(drop));
        }
    }
#pragma unroll
    for (int i = 0; i < kPer; ++i) {
        const int q = base + w.wt + 128 * i;
        if (q < kChunks) {
            const int r = q >> 1, h = q & 1;
            const int n1 = r / C::N2, n2 = r - n1 * C::N2;
            *reinterpret_cast<uint4*>(w.a + (uint32_t)n1 * C::SBO1C + (uint32_t)n2 * 32 + (uint32_t)h * 16) = vals[i];
        }
    }
    }
    // K padding rows n2 = 45 .. 47 of every n1 group: zero
    for (int i = w.wt; i < 16 * 3 * 2; i += 128) {
        const int n1 = i / 6, rest = i - n1 * 6, n2 = 45 + (rest >> 1), h = rest & 1;
        *reinterpret_cast<uint4*>(w.a + (uint32_t)n1 * C::SBO1C + (uint32_t)n2 * 32 + (uint32_t)h * 16) =
            make_uint4(0u, 0u, 0u, 0u);
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
#pragma unroll 1
    for (int ti = 0; ti < C::MT2; ++ti) {
        uint32_t r[32];
        tc::tmem_ld32(lane_base + 32 * ti, r);
        tc::tmem_ld_wait();
        const int k2 = 16 * ti + (w.wt >> 3);
        if (k2 >= C::N2) continue;
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
        for (int i = 0; i < 4; ++i) {
            const uint4 val = make_uint4(o[4 * i], o[4 * i + 1], o[4 * i + 2], o[4 * i + 3]);
            asm volatile("st.global.L1::no_allocate.L2::cache_hint.v4.u32 [%0], {%1, %2, %3, %4}, %5;"
                         ::"l"(dst + i), "r"(val.x), "r"(val.y), "r"(val.z), "r"(val.w), "l"(keep) : "memory");
        }
    }
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
// the border-masked maximum (starting at 0, as the reference's peak) per
// thread, the maximum reduced over the warp, and only the lanes holding the
// warp's maximum look for its position (re-reading their TMEM lanes); the
// warp then adds its share to the unit's accumulators.
template <class C>
__device__ __forceinline__ void tc2_col_out(const Tc2Args& a, int u, int t, const Tc2Wg& w, const Tc2Masks mb) {
    constexpr int L = C::L, h = L / 2;
    static_assert((L / 2) % 2 == 0, "sign of the fftshift: (-1)^(L/2) = +1");
    const uint32_t lane_base = w.tmem + ((uint32_t)(32 * (w.wt >> 5)) << 16);
    const int pc = 8 * t + (w.wt & 7);                           // physical column
    const int x = C::Pfa::map_coord(pc & 15, pc >> 4);           // map column
    const bool xin = (unsigned)(x - a.yb0) <= (unsigned)(a.yb1 - a.yb0);  // column in the border
    float m1 = 0.0f, m2 = 0.0f, s2a = 0.0f, s2b = 0.0f;
    // the tile loops stay rolled: one 32-register array is live at a time
#pragma unroll 1
    for (int ti = 0; ti < C::MT2; ++ti) {
        uint32_t r[32];
        tc::tmem_ld32(lane_base + 32 * ti, r);
        tc::tmem_ld_wait();
        // rows k2 >= 45 hold zeros and no bits
        const uint32_t bits = xin ? 0u : (ti == 0 ? mb.m[0] : ti == 1 ? mb.m[1] : mb.m[2]);
#pragma unroll
        for (int k1 = 0; k1 < 16; ++k1) {
            const float v1 = __uint_as_float(r[2 * k1]), v2 = __uint_as_float(r[2 * k1 + 1]);
            const bool in = (bits >> k1) & 1u;
            m1 = fmaxf(m1, in ? v1 : 0.0f);
            m2 = fmaxf(m2, in ? v2 : 0.0f);
            s2a = fmaf(v1, v1, s2a);
            s2b = fmaf(v2, v2, s2b);
        }
    }
    float M1 = m1, M2 = m2;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        M1 = fmaxf(M1, __shfl_xor_sync(0xffffffffu, M1, o));
        M2 = fmaxf(M2, __shfl_xor_sync(0xffffffffu, M2, o));
    }
    unsigned long long ka = 0ull, kb = 0ull;
    if (M1 > 0.0f || M2 > 0.0f) {   // warp-uniform: every lane re-reads its TMEM lanes
        const bool look1 = M1 > 0.0f && m1 == M1, look2 = M2 > 0.0f && m2 == M2;
        const int X = x + h < L ? x + h : x - h;
        int i1 = 0x7fffffff, i2 = 0x7fffffff;
#pragma unroll 1
        for (int ti = 0; ti < C::MT2; ++ti) {
            uint32_t r[32];
            tc::tmem_ld32(lane_base + 32 * ti, r);
            tc::tmem_ld_wait();
            if (!(look1 || look2)) continue;
            const uint32_t bits = xin ? 0u : (ti == 0 ? mb.m[0] : ti == 1 ? mb.m[1] : mb.m[2]);
            const int k2 = 16 * ti + (w.wt >> 3);
#pragma unroll
            for (int k1 = 0; k1 < 16; ++k1) {
                if (!((bits >> k1) & 1u)) continue;
                const float v1 = __uint_as_float(r[2 * k1]), v2 = __uint_as_float(r[2 * k1 + 1]);
                if (!((look1 && v1 == M1) || (look2 && v2 == M2))) continue;
                const int y = C::Pfa::map_coord(k1, k2);
                const int Y = y + h < L ? y + h : y - h;
                const int idx = Y * L + X;
                if (look1 && v1 == M1) i1 = min(i1, idx);
                if (look2 && v2 == M2) i2 = min(i2, idx);
            }
        }
        if (i1 != 0x7fffffff) ka = argmax_key(M1, i1);
        if (i2 != 0x7fffffff) kb = argmax_key(M2, i2);
    }
    const double d2a = warp_sum((double)s2a), d2b = warp_sum((double)s2b);
    ka = warp_max_u64(ka);
    kb = warp_max_u64(kb);
    if ((threadIdx.x & 31) == 0) {
        UnitAcc* ac = a.acc + 2 * (long long)u;
        if (ka) atomicMax(&ac[0].key, ka);
        atomicAdd(&ac[0].s2, d2a);
        if (kb) atomicMax(&ac[1].key, kb);
        atomicAdd(&ac[1].s2, d2b);
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
        const int J = 2 * wp.y + q;
        if (J >= a.ntmpl) break;
        UnitAcc v;
        v.key = __ldcg(&ac[q].key);
        v.s2 = __ldcg(&ac[q].s2) * inv * inv;
        // unscaled peak: the key's value is s x peak, exactly (s a power of two)
        const float pk = key_value(v.key) * (float)inv;
        v.key = v.key ? argmax_key(pk, key_index(v.key)) : 0ull;
        a.out[(long long)wp.x * a.ntmpl + J] = unit_score(v, sums[q], C::L);
    }
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

// Called by a pipeline's leader thread only; a pipeline barrier follows.
template <class C>
__device__ __forceinline__ void tc2_wait_for(const Tc2Args& a, int item) {
    const int s = item / (2 * C::T), j = item - s * (2 * C::T);
    if (j < C::T) {
        if (s < a.nu && s >= a.S) tc2_wait_counter<C>(a.done_cols + (s - a.S), C::kDone, a.error);
    } else {
        const int u = s - a.lag;
        if (u >= 0 && u < a.nu) tc2_wait_counter<C>(a.done_rows + u, C::kDone, a.error);
    }
}

// Count one finished tile (leader thread, after a __threadfence that orders
// the pipeline's earlier stores and atomics before it); the last column tile
// of a unit computes its scores.
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
        __threadfence();  // the other pipelines' accumulator atomics, published before their counts
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
    w.bar = bars + w.g;
    w.tmem = *tslot + (uint32_t)w.g * C::tmem_cols;
    w.ish = reinterpret_cast<int*>(sm + C::off_misc + 16) + 4 * w.g;
    const Tc2Masks ymask = tc2_row_masks<C>(w.wt, a.yb0, a.yb1);
    const Tc2FillMap fmap = tc2_fill_map<C>(w.wt);
    const int total = (a.nu + a.lag) * 2 * C::T;
    // The pipeline leader claims batches of kBatch consecutive items (one
    // atomic per batch), the pipeline processes them in order and the leader
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
        if (w.wt == 0 && last_of_batch) pre = atomicAdd(a.next_item, C::kBatch);  // used after this item
        const int s = item / (2 * C::T), j = item - s * (2 * C::T);
        if (j < C::T) {
            if (s < a.nu) {
                const int2 wp = __ldg(a.unit_wp + s);
                const float sc = tc2_scale(__ldg(a.wmax + wp.x), __ldg(a.pmax + wp.y));
                tc2_row_fill<C>(a, s, j, w, sc, fmap);
                ok &= tc2_gemm<C, false, false>(w, sm, phase, a.error);
                tc2_transition<C>(w);
                ok &= tc2_gemm<C, true, false>(w, sm, phase, a.error);
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
            if (w.wt == 0) {
                __threadfence();
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
