// Four-step l = 16 * N2 FFT kernels for the correlation hot path.
//
// One CTA (256 threads) transforms a tile of 16 vectors (rows, or columns
// of row-major l x l images).  For each vector x of length l:
//   step 1  thread (v, n2):  16-point DFT of x[n2 + N2 n1] in registers,
//           twiddle by W_l^{n2 k1}, write to shared memory;
//   step 2  thread (v, k1):  N2-point DFT of the 16 x N2 block row k1 in
//           registers; X[k1 + 16 k2] is its output k2.
// Global loads of step 1 and stores of step 2 are coalesced (consecutive
// threads touch consecutive addresses), there is one shared-memory exchange
// per transform, and the shared layout (block pitch BP odd, vector pitch
// 16 BP + 1) makes both the step-1 writes and the step-2 reads of a
// half-warp hit distinct banks.  All twiddles inside the register DFTs are
// compile-time constants (regfft.cuh); the W_l^{n2 k1} twiddles are built
// from one table entry per thread by at most three complex products.
#pragma once

#include <type_traits>

#include "fft.cuh"
#include "kernels.cuh"
#include "regfft.cuh"

namespace gs {

template <int N2>
struct Fast16 {
    static constexpr int L = 16 * N2;
    static constexpr int V = 16;                       // vectors per CTA tile
    static constexpr int BP = (N2 % 2) ? N2 : N2 + 1;  // odd block pitch
    static constexpr int VP = 16 * BP + 1;             // vector pitch
    static constexpr int kThreads = 256;
    static constexpr size_t smem_bytes() {
        return (size_t)V * VP * sizeof(float2) + kFftRedDoubles * sizeof(double);
    }
};

// W_l^{n2 k1} for k1 = 0..15 from w1 = W_l^{n2}: w2 = w1^2, w4 = w2^2,
// w8 = w4^2 and w_k = products of those (at most three products deep).
__device__ __forceinline__ void twiddle16(float2 w1, float2 (&w)[16]) {
    w[0] = make_float2(1.0f, 0.0f);
    w[1] = w1;
    w[2] = cmul(w1, w1);
    w[3] = cmul(w[2], w1);
    w[4] = cmul(w[2], w[2]);
    w[5] = cmul(w[4], w1);
    w[6] = cmul(w[4], w[2]);
    w[7] = cmul(w[4], w[3]);
    w[8] = cmul(w[4], w[4]);
#pragma unroll
    for (int k = 9; k < 16; ++k) w[k] = cmul(w[8], w[k - 8]);
}

// IO functors with `static constexpr bool kStaged = true` store a row
// transform's outputs in their own column order (column(k) for output k)
// through shared memory (store_at(img, v, column, value)).
template <class T, class = void>
struct IoStaged : std::false_type {};
template <class T>
struct IoStaged<T, std::void_t<decltype(T::kStaged)>> : std::bool_constant<T::kStaged> {};

template <int N2, bool kInv, bool kCols, class IO>
__global__ void __launch_bounds__(256, 2) k_fft16(const float2* __restrict__ tw, IO io_param) {
    using F = Fast16<N2>;
    extern __shared__ float2 sm16[];
    IO io = io_param;
    const int img = blockIdx.y;
    const int v0 = blockIdx.x * F::V;
    // ---- step 1: 16-point DFTs down the stride-N2 columns of each vector
    for (int task = threadIdx.x; task < F::V * N2; task += F::kThreads) {
        int v, n2;
        if (kCols) { n2 = task / F::V; v = task - n2 * F::V; }
        else { v = task / N2; n2 = task - v * N2; }
        float2 a[16];
#pragma unroll
        for (int n1 = 0; n1 < 16; ++n1) a[n1] = io.load(img, v0 + v, N2 * n1 + n2);
        rf::rfft<16, 1, kInv>(a);
        float2 w[16];
        twiddle16(twiddle(tw, n2, kInv), w);
        float2* dst = sm16 + v * F::VP + n2;
        rf::static_for<16>([&](auto kc) {
            constexpr int k1 = decltype(kc)::value;
            constexpr int r = rf::rpos<16>(k1);
            dst[k1 * F::BP] = k1 ? cmul(a[r], w[k1]) : a[r];
        });
    }
    __syncthreads();
    // ---- step 2: N2-point DFT of block row k1 of each vector
    {
        int v, k1;
        if (kCols) { v = threadIdx.x & 15; k1 = threadIdx.x >> 4; }
        else { v = threadIdx.x >> 4; k1 = threadIdx.x & 15; }
        float2 b[N2];
        const float2* src = sm16 + v * F::VP + k1 * F::BP;
#pragma unroll
        for (int n2 = 0; n2 < N2; ++n2) b[n2] = src[n2];
        rf::rfft<N2, 1, kInv>(b);
        if constexpr (IoStaged<IO>::value) {
            // permuted output order: through shared memory, so that the
            // global stores stay coalesced
            __syncthreads();  // every step-2 read of the tile is done
            rf::static_for<N2>([&](auto kc) {
                constexpr int k2 = decltype(kc)::value;
                sm16[v * F::VP + io.column(k1 + 16 * k2)] = b[rf::rpos<N2>(k2)];
            });
        } else {
            rf::static_for<N2>([&](auto kc) {
                constexpr int k2 = decltype(kc)::value;
                io.store(img, v0 + v, k1 + 16 * k2, b[rf::rpos<N2>(k2)]);
            });
        }
    }
    if constexpr (IoStaged<IO>::value) {
        __syncthreads();
        for (int e = threadIdx.x; e < F::V * F::L; e += F::kThreads) {
            const int vv = e / F::L, p = e - vv * F::L;
            io.store_at(img, v0 + vv, p, sm16[vv * F::VP + p]);
        }
    }
    io.finish(reinterpret_cast<double*>(sm16 + F::V * F::VP));
}

// ---- IO functors: (img, v, k) -> element k of vector v of image img ----

// Column order of spectra fed to a prime-factor inverse transform along x
// (L = 16 N2, N2 odd, so 16 and N2 are coprime): physical column
// p = n2 + N2 n1 holds frequency (N2 n1 + 16 n2) mod L, the Good-Thomas input
// map, so that the transform reads its 16-point groups at stride N2 exactly
// like the four-step kernels.  N2 = 0 means natural order.
struct PfaCols {
    int L = 0, N2 = 0;
    int i16 = 0;  // N2^-1 mod 16
    int iN = 0;   // 16^-1 mod N2
    static PfaCols make(int l) {
        PfaCols c;
        if (l % 16 || (l / 16) % 2 == 0) return c;
        c.L = l;
        c.N2 = l / 16;
        for (int x = 1; x < 16; ++x)
            if ((c.N2 * x) % 16 == 1) c.i16 = x;
        for (int x = 1; x < c.N2; ++x)
            if ((16 * x) % c.N2 == 1) c.iN = x;
        return c;
    }
    // frequency held by physical column p
    __host__ __device__ int logical(int p) const {
        const int n1 = p / N2, n2 = p - n1 * N2;
        const int q = N2 * n1 + 16 * n2;
        return q < L ? q : q - L;
    }
    // physical column of frequency k = k1 + 16 k2: n1 = k1 / N2 mod 16,
    // n2 = k / 16 mod N2 = k1 iN + k2 mod N2
    __host__ __device__ int physical(int k) const {
        const int k1 = k & 15;
        const int n1 = (k1 * i16) & 15;
        const int n2 = (k1 * iN + (k >> 4)) % N2;
        return n2 + N2 * n1;
    }
};

// In place, every row of `rows` rows of length L: to_physical moves
// natural-order columns to the PfaCols order, otherwise back.
__global__ void k_pfa_permute_rows(float2* __restrict__ data, long long rows, PfaCols pc, bool to_physical) {
    extern __shared__ float2 prow[];
    const int L = pc.L;
    for (long long r = blockIdx.x; r < rows; r += gridDim.x) {
        float2* row = data + r * L;
        for (int i = threadIdx.x; i < L; i += blockDim.x) prow[i] = row[i];
        __syncthreads();
        for (int i = threadIdx.x; i < L; i += blockDim.x) row[i] = prow[to_physical ? pc.logical(i) : pc.physical(i)];
        __syncthreads();
    }
}

template <bool kCols>
__device__ __forceinline__ long long f16_addr(int L, long long L2, int img, int v, int k) {
    return (long long)img * L2 + (kCols ? (long long)k * L + v : (long long)v * L + k);
}

// In place, output scaled.
template <bool kCols>
struct F16Complex {
    float2* data;
    int L;
    long long L2;
    float scale;
    __device__ float2 load(int img, int v, int k) const { return data[f16_addr<kCols>(L, L2, img, v, k)]; }
    __device__ void store(int img, int v, int k, float2 x) const {
        data[f16_addr<kCols>(L, L2, img, v, k)] = cscale(x, scale);
    }
    __device__ void finish(double*) const {}
};

// Per-image scale on load (scale[img]), in place.
template <bool kCols>
struct F16ScaleIn {
    float2* data;
    const double* scale;
    int L;
    long long L2;
    __device__ float2 load(int img, int v, int k) const {
        return cscale(data[f16_addr<kCols>(L, L2, img, v, k)], (float)scale[img]);
    }
    __device__ void store(int img, int v, int k, float2 x) const { data[f16_addr<kCols>(L, L2, img, v, k)] = x; }
    __device__ void finish(double*) const {}
};

// Complex in, real part out (float image with the same geometry).
template <bool kCols>
struct F16RealOut {
    const float2* in;
    float* out;
    int L;
    long long L2;
    __device__ float2 load(int img, int v, int k) const { return in[f16_addr<kCols>(L, L2, img, v, k)]; }
    __device__ void store(int img, int v, int k, float2 x) const { out[f16_addr<kCols>(L, L2, img, v, k)] = x.x; }
    __device__ void finish(double*) const {}
};

// Rows of the template-pair images: z = t1n - i t2n with per-template
// (mean, 1/sd) normalisation on load (see IoPairNorm), in place.
struct F16PairNorm {
    float2* data;
    const float4* coef;
    int L;
    long long L2;
    __device__ float2 load(int img, int v, int k) const {
        const float4 c = coef[img];
        const float2 z = data[f16_addr<false>(L, L2, img, v, k)];
        return make_float2((z.x - c.x) * c.y, -(z.y - c.z) * c.w);
    }
    __device__ void store(int img, int v, int k, float2 x) const { data[f16_addr<false>(L, L2, img, v, k)] = x; }
    __device__ void finish(double*) const {}
};

// The same row pass, its spectra stored in the PfaCols column order of the
// prime-factor correlation kernel.
struct F16PairNormPfa : F16PairNorm {
    PfaCols pfa;
    static constexpr bool kStaged = true;
    __device__ int column(int k) const { return pfa.physical(k); }
    __device__ void store_at(int img, int v, int p, float2 x) const { data[f16_addr<false>(L, L2, img, v, p)] = x; }
};

// Row pass of the correlation: S = W_w conj(P_p), inverse FFT along x,
// stored to the scratch map R_p (same role as IoPass1).
struct F16Pass1 {
    const float2* W;
    const float2* P;
    float2* R;
    int L;
    long long L2;
    __device__ float2 load(int img, int v, int k) const {
        const long long off = (long long)v * L + k;
        return cmulc(__ldg(W + off), __ldcs(P + (long long)img * L2 + off));
    }
    __device__ void store(int img, int v, int k, float2 x) const {
        __stcg(R + (long long)img * L2 + (long long)v * L + k, x);
    }
    __device__ void finish(double*) const {}
};

// Column pass of the correlation with the score epilogue (same reduction
// as IoPass2): vector v = map column x, element k = map row y.
struct F16Pass2 {
    const float2* R;
    UnitAcc* acc;
    int L, ntmpl;
    long long L2;
    float q_lo, q_hi, sgn;
    unsigned long long k1 = 0ull, k2 = 0ull;
    float s1a = 0.f, s2a = 0.f, s1b = 0.f, s2b = 0.f;

    __device__ float2 load(int img, int v, int k) const {
        return __ldcs(R + (long long)img * L2 + (long long)k * L + v);
    }
    __device__ void store(int, int v, int k, float2 val) {
        const int h = L >> 1;
        int X = v + h; if (X >= L) X -= L;
        int Y = k + h; if (Y >= L) Y -= L;
        const float v1 = sgn * val.x, v2 = sgn * val.y;
        const bool border = (float)X < q_lo || (float)X > q_hi || (float)Y < q_lo || (float)Y > q_hi;
        if (!border) {
            const int pos = Y * L + X;
            const unsigned long long a = argmax_key(v1, pos), b = argmax_key(v2, pos);
            k1 = a > k1 ? a : k1;
            k2 = b > k2 ? b : k2;
        }
        s1a += v1; s2a = fmaf(v1, v1, s2a);
        s1b += v2; s2b = fmaf(v2, v2, s2b);
    }
    __device__ void finish(double* scratch) {
        double s[4] = {s1a, s2a, s1b, s2b};
        unsigned long long ka = warp_max_u64(k1), kb = warp_max_u64(k2);
        block_sum<4>(s, scratch);
        unsigned long long* ks = reinterpret_cast<unsigned long long*>(scratch);
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
        if (lane == 0) { ks[warp] = ka; ks[32 + warp] = kb; }
        __syncthreads();
        if (threadIdx.x == 0) {
            for (int w2 = 0; w2 < nw; ++w2) {
                ka = ks[w2] > ka ? ks[w2] : ka;
                kb = ks[32 + w2] > kb ? ks[32 + w2] : kb;
            }
            const int p = blockIdx.y;
            const int J1 = 2 * p, J2 = 2 * p + 1;
            if (ka) atomicMax(&acc[J1].key, ka);
            atomicAdd(&acc[J1].s1, s[0]);
            atomicAdd(&acc[J1].s2, s[1]);
            if (J2 < ntmpl) {
                if (kb) atomicMax(&acc[J2].key, kb);
                atomicAdd(&acc[J2].s1, s[2]);
                atomicAdd(&acc[J2].s2, s[3]);
            }
        }
    }
};

}  // namespace gs
