// Persistent correlation kernel: the row pass and the column pass of every
// (window, template pair) unit of one in-plane angle in a single launch.
//
// Work items, claimed in increasing order from one atomic counter:
//   slot s (0 <= s < Nu + lag) = [N2 row tiles of unit s] [N2 column tiles of unit s - lag]
// A row tile takes 16 spectrum rows of unit u: S = W_w conj(P_p), inverse FFT
// along x (fastfft.cuh four-step), written to scratch map slot u % S.  A
// column tile takes 16 columns of that map: inverse FFT along y and the score
// epilogue (border-masked peak and position, sum and sum of squares of both
// templates of the pair), reduced into the unit's accumulators; the last
// column tile of a unit computes the two scores.
//
// Dependencies and why they cannot deadlock: a column tile of u waits until
// all N2 row tiles of u are done; a row tile of u >= S waits until all
// column tiles of u - S are done (its scratch slot is free).  Both wait only
// on items that come earlier in the claim order, and an item is claimed only
// by a running CTA that finishes it before claiming another, so the earliest
// unfinished item can always proceed.  Every wait is bounded; a wait that
// gives up raises the error flag (reported as GS_ERR_TIMEOUT) and the item
// still completes and signals, so no other CTA is left waiting on it.
//
// Memory ordering: producers store the maps with st.global.cg, then
// __syncthreads(), and one thread issues __threadfence() + atomicAdd on the
// unit's counter; consumers spin with ld.acquire.gpu, __syncthreads(), and
// read the maps with ld.global.cg (L2, never a stale L1 line from an earlier
// occupant of the slot).
#pragma once

#include "fastfft.cuh"

namespace gs {

struct CorrArgs {
    const float2* W;         // window spectra, Nw x L2
    const float2* P;         // template-pair spectra of this angle, Np x L2
    float2* R;               // scratch ring, S x L2
    const int2* unit_wp;     // unit -> (window, pair)
    int* done_rows;          // per unit, row tiles finished
    int* done_cols;          // per unit, column tiles finished
    UnitAcc* acc;            // per unit, 2 templates
    UnitOut* out;            // this angle's results, index w * ntmpl + J
    int* next_item;          // claim counter
    int* error;              // set when a bounded wait gives up
    int nu, ntmpl, S, lag;
    long long L2;
    int yb0, yb1;            // border interval of unshifted indices (both axes)
};

__device__ __forceinline__ int ld_acquire_gpu(const int* p) {
    int v;
    asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// Thread 0 waits until *p >= target; bounded (about a second or more), then
// flags the error and gives up.  Must be followed by __syncthreads().
__device__ __forceinline__ void wait_counter(const int* p, int target, int* error) {
    if (threadIdx.x != 0) return;
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

template <int N2>
struct CorrSmem {
    using F = Fast16<N2>;
    static constexpr size_t tile = (size_t)F::V * F::VP * sizeof(float2);
    static constexpr size_t tw = (size_t)16 * N2 * sizeof(float2);
    static constexpr size_t red = 128 * sizeof(double);
    static constexpr size_t bytes = tile + tw + red + 16;
};

template <int N2>
__device__ __forceinline__ void corr_row_tile(const CorrArgs& a, int u, int t, float2* tile, const float2* twt) {
    using F = Fast16<N2>;
    constexpr int L = F::L;
    const int2 wp = a.unit_wp[u];
    const float2* Wr = a.W + (long long)wp.x * a.L2;
    const float2* Pr = a.P + (long long)wp.y * a.L2;
    float2* Rs = a.R + (long long)(u % a.S) * a.L2;
    const int r0 = t * F::V;
    for (int task = threadIdx.x; task < F::V * N2; task += F::kThreads) {
        const int v = task / N2, n2 = task - v * N2;
        const long long base = (long long)(r0 + v) * L + n2;
        float2 x[16];
#pragma unroll
        for (int n1 = 0; n1 < 16; ++n1) x[n1] = cmulc(__ldg(Wr + base + N2 * n1), __ldg(Pr + base + N2 * n1));
        rf::rfft<16, 1, true>(x);
        float2* dst = tile + v * F::VP + n2;
        const float2* tw = twt + n2;
        rf::static_for<16>([&](auto kc) {
            constexpr int k1 = decltype(kc)::value;
            constexpr int r = rf::rpos<16>(k1);
            dst[k1 * F::BP] = k1 ? cmul(x[r], tw[k1 * N2]) : x[r];
        });
    }
    __syncthreads();
    {
        const int v = threadIdx.x >> 4, k1 = threadIdx.x & 15;
        float2 b[N2];
        const float2* src = tile + v * F::VP + k1 * F::BP;
#pragma unroll
        for (int n2 = 0; n2 < N2; ++n2) b[n2] = src[n2];
        rf::rfft<N2, 1, true>(b);
        float2* dst = Rs + (long long)(r0 + v) * L + k1;
        rf::static_for<N2>([&](auto kc) {
            constexpr int k2 = decltype(kc)::value;
            __stcg(dst + 16 * k2, b[rf::rpos<N2>(k2)]);
        });
    }
}

template <int N2>
__device__ __forceinline__ void corr_col_tile(const CorrArgs& a, int u, int t, float2* tile, const float2* twt,
                                              double* red, bool* last_out) {
    using F = Fast16<N2>;
    constexpr int L = F::L;
    constexpr int h = L / 2;
    const float2* Rs = a.R + (long long)(u % a.S) * a.L2;
    const int c0 = t * F::V;
    for (int task = threadIdx.x; task < F::V * N2; task += F::kThreads) {
        const int n2 = task / F::V, v = task - n2 * F::V;
        const float2* src = Rs + (long long)n2 * L + c0 + v;
        float2 x[16];
#pragma unroll
        for (int n1 = 0; n1 < 16; ++n1) x[n1] = __ldcg(src + (long long)N2 * n1 * L);
        rf::rfft<16, 1, true>(x);
        float2* dst = tile + v * F::VP + n2;
        const float2* tw = twt + n2;
        rf::static_for<16>([&](auto kc) {
            constexpr int k1 = decltype(kc)::value;
            constexpr int r = rf::rpos<16>(k1);
            dst[k1 * F::BP] = k1 ? cmul(x[r], tw[k1 * N2]) : x[r];
        });
    }
    __syncthreads();
    const int v = threadIdx.x & 15, k1 = threadIdx.x >> 4;
    const int x = c0 + v;
    const bool xin = (unsigned)(x - a.yb0) > (unsigned)(a.yb1 - a.yb0);  // column outside the border
    float best1 = 0.0f, best2 = 0.0f;   // reference peak = max(0, masked max)
    int bk1 = -1, bk2 = -1;
    float s1a = 0.f, s2a = 0.f, s1b = 0.f, s2b = 0.f;
    {
        float2 b[N2];
        const float2* src = tile + v * F::VP + k1 * F::BP;
#pragma unroll
        for (int n2 = 0; n2 < N2; ++n2) b[n2] = src[n2];
        rf::rfft<N2, 1, true>(b);
        rf::static_for<N2>([&](auto kc) {
            constexpr int k2 = decltype(kc)::value;
            const float2 val = b[rf::rpos<N2>(k2)];
            const int y = k1 + 16 * k2;
            const bool in = xin && ((unsigned)(y - a.yb0) > (unsigned)(a.yb1 - a.yb0));
            const float v1 = ((L / 2) % 2 == 0) ? val.x : -val.x;
            const float v2 = ((L / 2) % 2 == 0) ? val.y : -val.y;
            const bool g1 = in && v1 > best1, g2 = in && v2 > best2;
            best1 = g1 ? v1 : best1;
            bk1 = g1 ? k2 : bk1;
            best2 = g2 ? v2 : best2;
            bk2 = g2 ? k2 : bk2;
            s1a += v1; s2a = fmaf(v1, v1, s2a);
            s1b += v2; s2b = fmaf(v2, v2, s2b);
        });
    }
    // keys: value bits high, ~flat index low (smallest index wins among equal values)
    const int X = x + h < L ? x + h : x - h;
    unsigned long long ka = 0ull, kb = 0ull;
    if (bk1 >= 0) {
        const int y = k1 + 16 * bk1;
        const int Y = y + h < L ? y + h : y - h;
        ka = argmax_key(best1, Y * L + X);
    }
    if (bk2 >= 0) {
        const int y = k1 + 16 * bk2;
        const int Y = y + h < L ? y + h : y - h;
        kb = argmax_key(best2, Y * L + X);
    }
    double s[4] = {s1a, s2a, s1b, s2b};
    ka = warp_max_u64(ka);
    kb = warp_max_u64(kb);
    block_sum<4>(s, red);
    unsigned long long* ks = reinterpret_cast<unsigned long long*>(red);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) { ks[warp] = ka; ks[32 + warp] = kb; }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w2 = 0; w2 < F::kThreads / 32; ++w2) {
            ka = ks[w2] > ka ? ks[w2] : ka;
            kb = ks[32 + w2] > kb ? ks[32 + w2] : kb;
        }
        UnitAcc* ac = a.acc + 2 * (long long)u;
        if (ka) atomicMax(&ac[0].key, ka);
        atomicAdd(&ac[0].s1, s[0]);
        atomicAdd(&ac[0].s2, s[1]);
        if (kb) atomicMax(&ac[1].key, kb);
        atomicAdd(&ac[1].s1, s[2]);
        atomicAdd(&ac[1].s2, s[3]);
        __threadfence();
        *last_out = atomicAdd(&a.done_cols[u], 1) == N2 - 1;
    }
}

// Score of one template from its accumulators (main.cu:869-876).
__device__ __forceinline__ UnitOut unit_score(const UnitAcc& ac, int l) {
    const float peak = key_value(ac.key);
    UnitOut u;
    u.peak = peak;
    u.pos = key_index(ac.key);
    const double ra = ac.s1 - peak;
    const double rb = ac.s2 - (double)peak * peak;
    const double rc = (double)l * l - 1.0;
    const double sd = sqrt(rb / rc - (ra / rc) * (ra / rc));
    u.sigma = (float)sd;
    u.score = sd > 0.0 ? (float)(peak / sd) : __int_as_float(0x7fc00000);
    return u;
}

template <int N2>
__global__ void __launch_bounds__(256, 2) k_corr_persistent(CorrArgs a) {
    using F = Fast16<N2>;
    using SM = CorrSmem<N2>;
    extern __shared__ __align__(16) unsigned char smc[];
    float2* tile = reinterpret_cast<float2*>(smc);
    float2* twt = reinterpret_cast<float2*>(smc + SM::tile);
    double* red = reinterpret_cast<double*>(smc + SM::tile + SM::tw);
    int* ish = reinterpret_cast<int*>(smc + SM::tile + SM::tw + SM::red);
    bool* last = reinterpret_cast<bool*>(ish + 2);
    // inverse twiddles W_L^{-n2 k1} = exp(+2 pi i n2 k1 / L), table [k1][n2]
    for (int i = threadIdx.x; i < 16 * N2; i += F::kThreads) {
        const int k1 = i / N2, n2 = i - k1 * N2;
        double s, c;
        sincospi(2.0 * (double)((n2 * k1) % F::L) / (double)F::L, &s, &c);
        twt[i] = make_float2((float)c, (float)s);
    }
    const int total = (a.nu + a.lag) * 2 * N2;
    if (threadIdx.x == 0) ish[0] = atomicAdd(a.next_item, 1);
    __syncthreads();
    int item = ish[0];
    __syncthreads();  // every thread has read ish[0] before thread 0 writes it again
    while (item < total) {
        int nxt = 0;
        if (threadIdx.x == 0) nxt = atomicAdd(a.next_item, 1);  // consumed after the tile
        const int s = item / (2 * N2), j = item - s * (2 * N2);
        if (j < N2) {
            const int u = s;
            if (u < a.nu) {
                if (u >= a.S) wait_counter(a.done_cols + (u - a.S), N2, a.error);
                __syncthreads();
                corr_row_tile<N2>(a, u, j, tile, twt);
                __syncthreads();
                if (threadIdx.x == 0) {
                    __threadfence();
                    atomicAdd(&a.done_rows[u], 1);
                }
            }
        } else {
            const int u = s - a.lag;
            if (u >= 0 && u < a.nu) {
                wait_counter(a.done_rows + u, N2, a.error);
                __syncthreads();
                corr_col_tile<N2>(a, u, j - N2, tile, twt, red, last);
                __syncthreads();
                if (threadIdx.x == 0 && *last) {
                    __threadfence();
                    const int2 wp = a.unit_wp[u];
                    const UnitAcc* ac = a.acc + 2 * (long long)u;
                    for (int q = 0; q < 2; ++q) {
                        const int J = 2 * wp.y + q;
                        if (J >= a.ntmpl) break;
                        UnitAcc v;
                        v.key = __ldcg(&ac[q].key);
                        v.s1 = __ldcg(&ac[q].s1);
                        v.s2 = __ldcg(&ac[q].s2);
                        a.out[(long long)wp.x * a.ntmpl + J] = unit_score(v, F::L);
                    }
                }
            }
        }
        if (threadIdx.x == 0) ish[0] = nxt;
        __syncthreads();
        item = ish[0];
        __syncthreads();  // as above: no thread may still be reading ish[0] when it changes
    }
}

}  // namespace gs
