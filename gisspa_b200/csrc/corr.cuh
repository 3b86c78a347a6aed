// Persistent correlation kernel: the row pass and the column pass of every
// (window, template pair) unit of one in-plane angle in a single launch.
//
// Work items, claimed in increasing order from one atomic counter:
//   slot s (0 <= s < Nu + lag) = [T row tiles of unit s] [T column tiles of unit s - lag]
// with T = l / V tiles of V vectors (V = 16 or 8, CorrCfg).  A row tile takes V
// spectrum rows of unit u: S = W_w conj(P_p), inverse FFT along x (the
// four-step l = 16 N2 transform of fastfft.cuh), written to scratch map slot
// u % S (for odd N2 prime-factor transforms along both axes, CorrCfg::kPfa).
// A column tile takes V columns of that map: inverse FFT along y and the score
// epilogue (border-masked peak and its position, sum of squares, for both
// templates of the pair), reduced into the unit's accumulators; the last
// column tile of a unit computes the two scores, taking the maps' plain sums
// from the spectrum's DC term (sum of the map = L^2 S(0, 0)).
//
// Dependencies and why they cannot deadlock: a column tile of u waits until
// all T row tiles of u are done; a row tile of u >= S waits until all
// column tiles of u - S are done (its scratch slot is free).  Completion is
// counted per tile or per warp (CorrCfg::kWarpPub).  Per tile: after the CTA
// barrier that ends a tile, one thread (the publisher, the CTA's last thread,
// which has the lightest share of step 1 when the tasks do not divide evenly)
// increments the unit's counter, so a pass of a unit is done at T
// increments, claims the CTA's next-but-one item (written into the CTA's
// ring of claimed items just before the following barrier, so its warp does
// not wait for the atomic), and each warp checks the dependency of its CTA's
// next item itself before starting it.  Per warp: every warp counts its own share
// before that barrier (a pass is done at warps x T increments), and thread 0
// waits for the next item's dependency before it.  Both dependencies point at
// items that come earlier in the claim order, and an item is claimed only by
// a running CTA that finishes and publishes it before it waits for anything
// later, so the earliest unpublished item can always proceed.  Every wait is
// bounded; a wait that gives up raises the error flag (reported as
// GS_ERR_TIMEOUT) and the item still completes and is published, so no other
// CTA is left waiting on it.
//
// Memory ordering: producers store the maps bypassing L1 (st.global with an
// L2 cache hint) and add their accumulator atomics; the CTA barrier that ends
// the tile (per warp: __syncwarp) orders every thread's stores before the
// release increment (acquire-release for column tiles, whose last increment also
// computes the unit's scores), which therefore makes all of them visible
// (release is cumulative).  On the consumer side lane 0 of each warp (per
// warp: thread 0) spins with ld.acquire.gpu and __syncwarp() (the barrier)
// extends the acquire to its warp (CTA), whose threads read the maps with L1::no_allocate loads (L2, never a stale L1
// line from an earlier occupant of the slot).  A column tile costs two CTA
// barriers (step 1 -> step 2 of the FFT, whose vectors are columns spread
// over all warps for coalesced loads, and the end-of-item barrier); a row
// tile only the end-of-item barrier, as each warp owns two whole rows.
#pragma once

#include "fastfft.cuh"

namespace gs {

struct CorrArgs {
    const float2* W;         // window spectra, Nw x L2
    const float2* P;         // template-pair spectra of the launch's angles, (angles x pairs) x L2
    float2* R;               // scratch ring, S x L2
    const int2* unit_wp;     // unit -> (window, angle x pairs + pair)
    int* done_rows;          // per unit, row tiles finished
    int* done_cols;          // per unit, column tiles finished
    UnitAcc* acc;            // per unit, 2 templates
    UnitOut* out;            // results, index angle * out_stride + w * ntmpl + J
    int* next_item;          // claim counter
    int* error;              // set when a bounded wait gives up
    int nu, ntmpl, S, lag;
    long long L2;
    int yb0, yb1;            // border interval of unshifted indices (both axes)
    int pairs;               // template pairs per angle
    long long out_stride;    // results per angle (windows x templates)
};

// Results slot of template q (0, 1) of pair index y = angle x pairs + pair
// for window w, or -1 when the pair has no second template (odd count).
__device__ __forceinline__ long long unit_out_index(int y, int q, int w, int pairs, int ntmpl,
                                                    long long out_stride) {
    const int an = y / pairs, J = 2 * (y - an * pairs) + q;
    return J < ntmpl ? an * out_stride + (long long)w * ntmpl + J : -1;
}

__device__ __forceinline__ int ld_acquire_gpu(const int* p) {
    int v;
    asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// The calling thread waits until *p >= target (bounded: about a second or
// more, then it flags the error and gives up).  A barrier must follow before
// other threads rely on the condition.
__device__ __forceinline__ void wait_counter(const int* p, int target, int* error) {
    if (ld_acquire_gpu(p) >= target) return;
    bool ok = false;
    for (int it = 0; it < (1 << 22) && !ok; ++it) {
        __nanosleep(256);
        ok = ld_acquire_gpu(p) >= target;
    }
    if (!ok) atomicExch(error, 1);
}

// The calling warp waits until *p >= target: lane 0 spins (bounded, about a
// second or more, then flags the error and gives up) and __syncwarp()
// extends its acquire to the warp.  Every lane must call it.
__device__ __forceinline__ void wait_counter_warp(const int* p, int target, int* error) {
    if ((threadIdx.x & 31) == 0) wait_counter(p, target, error);
    __syncwarp();
}

// b^-1 mod m for gcd(b, m) = 1 (compile time, m small)
constexpr int inv_mod(int b, int m) {
    for (int x = 1; x < m; ++x)
        if ((b * x) % m == 1) return x;
    return m == 1 ? 0 : -1;
}

// Tile geometry: V vectors per tile (16 or 8), 16 V threads per CTA (step 2
// has one (vector, k1) task per thread), 512 / (16 V) CTAs per SM.  A pass of
// one unit is T = L / V tiles.
template <int N2, int V_>
struct CorrCfg {
    static constexpr int L = 16 * N2;
    static constexpr int V = V_;
    static constexpr int BP = (N2 % 2) ? N2 : N2 + 1;  // odd block pitch
    static constexpr int VP = 16 * BP + 1;             // vector pitch
    static constexpr int kThreads = 16 * V;
    static constexpr int kWarps = kThreads / 32;
    static constexpr int T = L / V;
    // Publication protocol.  When step 1's tasks do not divide evenly over
    // the threads (odd N2), per tile: one thread publishes after the
    // end-of-item barrier -- the CTA's last thread, whose step-1 share is the
    // lightest, so the release fence it waits for costs no barrier time --
    // and every warp checks its next item's dependency itself.  Otherwise
    // (kWarpPub) per warp: lane 0 of every warp counts its own share before
    // that barrier, and thread 0 waits for the next item's dependency while
    // the CTA finishes the current one.  Each was measured faster where used.
    static constexpr bool kWarpPub = (V * N2) % (16 * V) == 0;
    static constexpr int kDone = kWarpPub ? (V / 2) * T : T;  // completions that finish one pass of a unit
    static constexpr int kCtasPerSm = 512 / kThreads;
    static_assert(V == 8 || V == 16, "tile width");
    static_assert(V == 2 * kWarps, "a row tile gives each warp two rows");
    // Odd N2 (l = 720 = 16 x 45): 16 and N2 are coprime, so both passes use
    // the Good-Thomas mapping and need no twiddles between their two DFT
    // steps.  Along x the spectra arrive in that mapping's input order
    // (PfaCols: physical column n2 + N2 n1 holds frequency (N2 n1 + 16 n2)
    // mod L).  Along y the column pass's input row n2 + N2 n1 must hold
    // spectrum row (N2 n1 + 16 n2) mod L, so the row pass reads the spectrum
    // rows in that order.  Either pass's output k1 + 16 k2 is map coordinate
    // (A1 k1 + A2 k2) mod L, A1 = 1 mod 16, 0 mod N2 and A2 = 0 mod 16, 1 mod N2.
    static constexpr bool kPfa = (N2 % 2) == 1;
    static constexpr int A1 = kPfa ? (N2 * inv_mod(N2 % 16, 16)) % L : 1;
    static constexpr int A2 = kPfa ? (16 * inv_mod(16 % N2, N2)) % L : 16;
    // spectrum row that physical row r of the scratch map holds
    __host__ __device__ __forceinline__ static int spectrum_row(int r) {
        if constexpr (kPfa) {
            const int n1 = r / N2, n2 = r - n1 * N2;
            const int q = N2 * n1 + 16 * n2;
            return q < L ? q : q - L;  // N2 n1 + 16 n2 < 2 L
        } else {
            return r;
        }
    }
    // map coordinate of pass output (k1, k2): x of physical column k1 + 16 k2,
    // y of column-pass output k2 of thread k1
    __host__ __device__ static constexpr int map_coord(int k1, int k2) { return (A1 * k1 + A2 * k2) % L; }
};

template <int N2, int V>
struct CorrSmem {
    using C = CorrCfg<N2, V>;
    static constexpr size_t tile = (size_t)C::V * C::VP * sizeof(float2);
    static constexpr size_t tw = C::kPfa ? 0 : (size_t)16 * N2 * sizeof(float2);  // no twiddles with kPfa
    static constexpr size_t red = 128 * sizeof(double);
    static constexpr size_t bytes = tile + tw + red + 32;
};

// L2 eviction-priority hints: scratch maps are stored "evict last" (they are
// read again shortly) and loaded "evict first" by their only reader; the
// window spectra, reused by every pair of a window block, are loaded
// "evict last".
__device__ __forceinline__ unsigned long long l2_policy_evict_last() {
    unsigned long long p;
    asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
    return p;
}
__device__ __forceinline__ unsigned long long l2_policy_evict_first() {
    unsigned long long p;
    asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
    return p;
}
__device__ __forceinline__ float2 ld_l2hint(const float2* ptr, unsigned long long pol) {
    float2 v;
    asm volatile("ld.global.L1::no_allocate.L2::cache_hint.v2.f32 {%0, %1}, [%2], %3;"
                 : "=f"(v.x), "=f"(v.y) : "l"(ptr), "l"(pol));
    return v;
}
__device__ __forceinline__ void st_l2hint(float2* ptr, float2 v, unsigned long long pol) {
    asm volatile("st.global.L1::no_allocate.L2::cache_hint.v2.f32 [%0], {%1, %2}, %3;"
                 :: "l"(ptr), "f"(v.x), "f"(v.y), "l"(pol) : "memory");
}

// Drops one 128-byte line from L2 without writing it back (its contents
// become undefined).  Used on scratch-map lines that have been consumed and
// will be rewritten before they are read again.
__device__ __forceinline__ void l2_discard128(const void* p) {
    asm volatile("discard.global.L2 [%0], 128;" ::"l"(p) : "memory");
}

template <int N2, int V>
__device__ __forceinline__ void corr_row_tile(const CorrArgs& a, int u, int t, float2* tile, const float2* twt,
                                              int2 wp) {
    using F = CorrCfg<N2, V>;
    constexpr int L = F::L;
    const float2* Wr = a.W + (long long)wp.x * a.L2;
    const float2* Pr = a.P + (long long)wp.y * a.L2;
    float2* Rs = a.R + (long long)(u % a.S) * a.L2;
    const int r0 = t * F::V;
    const unsigned long long keep = l2_policy_evict_last();
    // each warp transforms its own two rows (vectors 2w, 2w + 1) through its
    // own part of the tile buffer, so step 1 -> step 2 needs only __syncwarp
    const int w2 = 2 * (threadIdx.x >> 5), lane = threadIdx.x & 31;
    for (int task = lane; task < 2 * N2; task += 32) {
        const int v = w2 + (task >= N2), n2 = task - (task >= N2) * N2;
        const long long base = (long long)F::spectrum_row(r0 + v) * L + n2;
        float2 x[16];
#pragma unroll
        for (int n1 = 0; n1 < 16; ++n1)
            x[n1] = cmulc(ld_l2hint(Wr + base + N2 * n1, keep), __ldg(Pr + base + N2 * n1));
        rf::rfft<16, 1, true>(x);
        float2* dst = tile + v * F::VP + n2;
        const float2* tw = twt + n2;
        rf::static_for<16>([&](auto kc) {
            constexpr int k1 = decltype(kc)::value;
            constexpr int r = rf::rpos<16>(k1);
            dst[k1 * F::BP] = (k1 && !F::kPfa) ? cmul(x[r], tw[k1 * N2]) : x[r];
        });
    }
    __syncwarp();
    {
        const int v = threadIdx.x >> 4, k1 = threadIdx.x & 15;  // v = w2 + lane / 16
        float2 b[N2];
        const float2* src = tile + v * F::VP + k1 * F::BP;
#pragma unroll
        for (int n2 = 0; n2 < N2; ++n2) b[n2] = src[n2];
        rf::rfft<N2, 1, true>(b);
        float2* dst = Rs + (long long)(r0 + v) * L + k1;
        rf::static_for<N2>([&](auto kc) {
            constexpr int k2 = decltype(kc)::value;
            st_l2hint(dst + 16 * k2, b[rf::rpos<N2>(k2)], keep);
        });
    }
}

// Border mask of the map rows one column-pass thread produces: bit k2 is set
// when map row map_coord(k1, k2) lies outside the border interval [yb0, yb1]
// (the thread's k1 is fixed for the life of the kernel).
template <int N2, int V>
__device__ __forceinline__ uint2 corr_row_mask(int yb0, int yb1) {
    using F = CorrCfg<N2, V>;
    const int k1 = V == 16 ? (threadIdx.x >> 4) : (threadIdx.x & 15);
    uint2 m = make_uint2(0u, 0u);
    for (int k2 = 0; k2 < N2; ++k2) {
        const int y = F::map_coord(k1, k2);
        if ((unsigned)(y - yb0) > (unsigned)(yb1 - yb0)) {
            if (k2 < 32) m.x |= 1u << k2;
            else m.y |= 1u << (k2 - 32);
        }
    }
    return m;
}

template <int N2, int V>
__device__ __forceinline__ void corr_col_tile(const CorrArgs& a, int u, int t, float2* tile, const float2* twt,
                                              uint2 ymask) {
    using F = CorrCfg<N2, V>;
    constexpr int L = F::L;
    constexpr int h = L / 2;
    const float2* Rs = a.R + (long long)(u % a.S) * a.L2;
    const int c0 = t * F::V;
    const unsigned long long drop = l2_policy_evict_first();
    for (int task = threadIdx.x; task < F::V * N2; task += F::kThreads) {
        const int n2 = task / F::V, v = task - n2 * F::V;
        const float2* src = Rs + (long long)n2 * L + c0 + v;
        float2 x[16];
#pragma unroll
        for (int n1 = 0; n1 < 16; ++n1) x[n1] = ld_l2hint(src + (long long)N2 * n1 * L, drop);
        rf::rfft<16, 1, true>(x);
        float2* dst = tile + v * F::VP + n2;
        const float2* tw = twt + n2;
        rf::static_for<16>([&](auto kc) {
            constexpr int k1 = decltype(kc)::value;
            constexpr int r = rf::rpos<16>(k1);
            dst[k1 * F::BP] = (k1 && !F::kPfa) ? cmul(x[r], tw[k1 * N2]) : x[r];
        });
    }
    __syncthreads();
    // every line of this tile's 16 columns has been read (the barrier orders
    // the loads before the discards): drop them from L2 instead of letting
    // them be written back; the slot is rewritten before its next read.  An
    // 8-column tile owns only half of each line and leaves them alone.
    if (V == 16)
        for (int r = threadIdx.x; r < L; r += F::kThreads) l2_discard128(Rs + (long long)r * L + c0);
    // step-2 task: (vector, k1); both orders read distinct banks per half-warp
    // for their width
    const int v = V == 16 ? (threadIdx.x & 15) : (threadIdx.x >> 4);
    const int k1 = V == 16 ? (threadIdx.x >> 4) : (threadIdx.x & 15);
    // map column held by physical column c0 + v (the row pass's output order)
    const int x = F::kPfa ? F::map_coord((c0 + v) & 15, (c0 + v) >> 4) : c0 + v;
    // column outside the border: the rows of ymask count, else none
    if ((unsigned)(x - a.yb0) <= (unsigned)(a.yb1 - a.yb0)) ymask = make_uint2(0u, 0u);
    constexpr float sgn = ((L / 2) % 2 == 0) ? 1.0f : -1.0f;
    // Per point the border-masked maximum with its k2 and the sum of squares;
    // the map's plain sum is L^2 times its spectrum's DC term, taken when the
    // unit's scores are computed.
    float best1 = 0.0f, best2 = 0.0f;   // reference peak = max(0, masked max)
    int bk1 = -1, bk2 = -1;
    float s2a = 0.f, s2b = 0.f;
    {
        float2 b[N2];
        const float2* src = tile + v * F::VP + k1 * F::BP;
#pragma unroll
        for (int n2 = 0; n2 < N2; ++n2) b[n2] = src[n2];
        rf::rfft<N2, 1, true>(b);
        rf::static_for<N2>([&](auto kc) {
            constexpr int k2 = decltype(kc)::value;
            const float2 val = b[rf::rpos<N2>(k2)];
            const bool in = (((k2 < 32 ? ymask.x : ymask.y) >> (k2 & 31)) & 1u) != 0u;
            const float v1 = sgn * val.x, v2 = sgn * val.y;
            const bool g1 = in && v1 > best1, g2 = in && v2 > best2;
            best1 = g1 ? v1 : best1;
            bk1 = g1 ? k2 : bk1;
            best2 = g2 ? v2 : best2;
            bk2 = g2 ? k2 : bk2;
            s2a = fmaf(v1, v1, s2a);
            s2b = fmaf(v2, v2, s2b);
        });
    }
    // keys: value bits high, ~flat index low (among equal values the smallest
    // index wins across threads; within one thread, the first in k2 order)
    const int X = x + h < L ? x + h : x - h;
    unsigned long long ka = 0ull, kb = 0ull;
    if (bk1 >= 0) {
        const int y = F::map_coord(k1, bk1);
        const int Y = y + h < L ? y + h : y - h;
        ka = argmax_key(best1, Y * L + X);
    }
    if (bk2 >= 0) {
        const int y = F::map_coord(k1, bk2);
        const int Y = y + h < L ? y + h : y - h;
        kb = argmax_key(best2, Y * L + X);
    }
    // warp-level reduction
    const double d2a = warp_sum((double)s2a), d2b = warp_sum((double)s2b);
    ka = warp_max_u64(ka);
    kb = warp_max_u64(kb);
    // one set of atomics per warp (published with the tile)
    if ((threadIdx.x & 31) == 0) {
        UnitAcc* ac = a.acc + 2 * (long long)u;
        if (ka) atomicMax(&ac[0].key, ka);
        atomicAdd(&ac[0].s2, d2a);
        if (kb) atomicMax(&ac[1].key, kb);
        atomicAdd(&ac[1].s2, d2b);
    }
}

// Score of one template from its accumulators (main.cu:869-876); s1 is the
// sum of the whole map.
__device__ __forceinline__ UnitOut unit_score(const UnitAcc& ac, double s1, int l) {
    const float peak = key_value(ac.key);
    UnitOut u;
    u.peak = peak;
    u.pos = key_index(ac.key);
    const double ra = s1 - peak;
    const double rb = ac.s2 - (double)peak * peak;
    const double rc = (double)l * l - 1.0;
    const double sd = sqrt(rb / rc - (ra / rc) * (ra / rc));
    u.sigma = (float)sd;
    u.score = sd > 0.0 ? (float)(peak / sd) : __int_as_float(0x7fc00000);
    return u;
}
__device__ __forceinline__ UnitOut unit_score(const UnitAcc& ac, int l) { return unit_score(ac, ac.s1, l); }

// The counter whose completions `item` waits for (kDone of them), or nullptr.
template <int N2, int V>
__device__ __forceinline__ const int* corr_dep(const CorrArgs& a, int item) {
    using C = CorrCfg<N2, V>;
    const int s = item / (2 * C::T), j = item - s * (2 * C::T);
    if (j < C::T) return (s < a.nu && s >= a.S) ? a.done_cols + (s - a.S) : nullptr;
    const int u = s - a.lag;
    return (u >= 0 && u < a.nu) ? a.done_rows + u : nullptr;
}

// (window, pair) of the unit whose row tile `item` is ({0, 0} for column
// tiles and the padding items past the last unit).  unit_wp is written by the
// host before the launch, so this load needs no ordering.
template <int N2, int V>
__device__ __forceinline__ int2 corr_item_wp(const CorrArgs& a, int item, int total) {
    using C = CorrCfg<N2, V>;
    if (item >= total) return make_int2(0, 0);
    const int s = item / (2 * C::T), j = item - s * (2 * C::T);
    return (j < C::T && s < a.nu) ? __ldg(a.unit_wp + s) : make_int2(0, 0);
}

// Per-tile protocol: each warp checks the dependency of `item` before
// working on it.
template <int N2, int V>
__device__ __forceinline__ void corr_wait_for(const CorrArgs& a, int item) {
    using C = CorrCfg<N2, V>;
    const int* p = corr_dep<N2, V>(a, item);
    if (p) wait_counter_warp(p, C::kDone, a.error);
}

// Count a finished tile (or one warp's share of it, kWarpPub); the last
// count of a unit's column pass computes its two scores.
template <int N2, int V>
__device__ __forceinline__ void corr_publish(const CorrArgs& a, int item) {
    using F = CorrCfg<N2, V>;
    const int s = item / (2 * F::T), j = item - s * (2 * F::T);
    if (j < F::T) {
        if (s < a.nu) asm volatile("red.release.gpu.global.add.s32 [%0], 1;" ::"l"(&a.done_rows[s]) : "memory");
        return;
    }
    const int u = s - a.lag;
    if (u < 0 || u >= a.nu) return;
    int prev;
    asm volatile("atom.acq_rel.gpu.global.add.s32 %0, [%1], 1;" : "=r"(prev) : "l"(&a.done_cols[u]) : "memory");
    if (prev != F::kDone - 1) return;
    const int2 wp = a.unit_wp[u];
    const UnitAcc* ac = a.acc + 2 * (long long)u;
    // sum of the map c1 + i c2 = L^2 S(0, 0), S = W conj(P)
    // (frequency (0, 0) sits at element 0 in either column order)
    const float2 w0 = __ldg(a.W + (long long)wp.x * a.L2);
    const float2 p0 = __ldg(a.P + (long long)wp.y * a.L2);
    const double sg = ((F::L / 2) % 2 == 0) ? 1.0 : -1.0;
    const double l2 = (double)a.L2;
    const double sums[2] = {sg * l2 * ((double)w0.x * p0.x + (double)w0.y * p0.y),
                            sg * l2 * ((double)w0.y * p0.x - (double)w0.x * p0.y)};
    for (int q = 0; q < 2; ++q) {
        const long long o = unit_out_index(wp.y, q, wp.x, a.pairs, a.ntmpl, a.out_stride);
        if (o < 0) break;
        UnitAcc v;
        v.key = __ldcg(&ac[q].key);
        v.s2 = __ldcg(&ac[q].s2);
        a.out[o] = unit_score(v, sums[q], F::L);
    }
}

template <int N2, int V>
__global__ void __launch_bounds__(CorrCfg<N2, V>::kThreads, CorrCfg<N2, V>::kCtasPerSm) k_corr_persistent(CorrArgs a) {
    using F = CorrCfg<N2, V>;
    using SM = CorrSmem<N2, V>;
    constexpr int kPub = F::kThreads - 1;  // the publisher
    extern __shared__ __align__(16) unsigned char smc[];
    float2* tile = reinterpret_cast<float2*>(smc);
    float2* twt = reinterpret_cast<float2*>(smc + SM::tile);
    int* ish = reinterpret_cast<int*>(smc + SM::tile + SM::tw + SM::red);  // ring of 4 claimed items
    // inverse twiddles W_L^{-n2 k1} = exp(+2 pi i n2 k1 / L), table [k1][n2]
    for (int i = threadIdx.x; i < (F::kPfa ? 0 : 16 * N2); i += F::kThreads) {
        const int k1 = i / N2, n2 = i - k1 * N2;
        double sn, cs;
        sincospi(2.0 * (double)((n2 * k1) % F::L) / (double)F::L, &sn, &cs);
        twt[i] = make_float2((float)cs, (float)sn);
    }
    const uint2 ymask = corr_row_mask<N2, V>(a.yb0, a.yb1);
    const int total = (a.nu + a.lag) * 2 * F::T;
    if constexpr (F::kWarpPub) {
        // per-warp protocol: thread 0 claims the next item while the CTA works
        // on the current one and resolves its dependency before the barrier
        // that ends the current one (each warp has counted its share by then,
        // thread 0's own warp included, so nothing of this CTA is pending)
        if (threadIdx.x == 0) {
            const int first = atomicAdd(a.next_item, 1);
            const int* p = first < total ? corr_dep<N2, V>(a, first) : nullptr;
            if (p) wait_counter(p, F::kDone, a.error);
            ish[0] = first;
        }
        __syncthreads();
        int item = ish[0];
        for (int iter = 1; item < total; ++iter) {
            int nxt = 0;
            if (threadIdx.x == 0) nxt = atomicAdd(a.next_item, 1);  // consumed after the tile
            const int s = item / (2 * F::T), j = item - s * (2 * F::T);
            if (j < F::T) {
                if (s < a.nu) corr_row_tile<N2, V>(a, s, j, tile, twt, a.unit_wp[s]);
            } else {
                const int u = s - a.lag;
                if (u >= 0 && u < a.nu) corr_col_tile<N2, V>(a, u, j - F::T, tile, twt, ymask);
            }
            __syncwarp();  // the warp's stores and atomics before its count
            if ((threadIdx.x & 31) == 0) corr_publish<N2, V>(a, item);
            if (threadIdx.x == 0) {
                const int* p = nxt < total ? corr_dep<N2, V>(a, nxt) : nullptr;
                if (p) wait_counter(p, F::kDone, a.error);
                ish[iter & 3] = nxt;
            }
            // the tile buffer is free and the next item (dependency satisfied)
            // published; slot iter & 3 is not rewritten before every thread has
            // passed at least one more barrier
            __syncthreads();
            item = ish[iter & 3];
        }
        return;
    }
    // per-tile protocol: the CTA always holds its current item and the next one
    if (threadIdx.x == kPub) {
        ish[0] = atomicAdd(a.next_item, 1);
        ish[1] = atomicAdd(a.next_item, 1);
    }
    __syncthreads();
    int item = ish[0];
    int claimed = 0;  // the publisher's claim for slot (iter + 1) & 3, made after the previous barrier
    for (int iter = 0; item < total; ++iter) {
        // the unit's (window, pair) is read-only in this launch: its load is
        // issued before the dependency wait and overlaps it
        const int2 wp = corr_item_wp<N2, V>(a, item, total);
        corr_wait_for<N2, V>(a, item);
        const int s = item / (2 * F::T), j = item - s * (2 * F::T);
        if (j < F::T) {
            if (s < a.nu) corr_row_tile<N2, V>(a, s, j, tile, twt, wp);
        } else {
            const int u = s - a.lag;
            if (u >= 0 && u < a.nu) corr_col_tile<N2, V>(a, u, j - F::T, tile, twt, ymask);
        }
        // the claim made after the previous barrier enters the ring only now,
        // so the publisher's warp did not wait for the atomic's return
        if (threadIdx.x == kPub && iter > 0) ish[(iter + 1) & 3] = claimed;
        // every thread is done with the item: the tile buffer is free, the
        // item's stores and atomics are ordered before its publication, and
        // slot (iter + 1) & 3 holds the next item; slot (iter + 2) & 3 was
        // last read two iterations ago
        __syncthreads();
        const int next = ish[(iter + 1) & 3];
        if (threadIdx.x == kPub) {
            corr_publish<N2, V>(a, item);
            claimed = atomicAdd(a.next_item, 1);  // for slot (iter + 2) & 3
        }
        item = next;
    }
}

}  // namespace gs
