// Register-resident small FFTs with compile-time twiddles.
//
// rfft<N, S, kInv, OFF>(a) transforms the N complex values a[OFF + n*S]
// (n < N) of a register array in place.  N is split recursively as
// N = P * Q with P a base radix (2, 3, 4, 5, 8):
//     X[k1 + P k2] = sum_{n2} W_Q^{n2 k2} W_N^{n2 k1} sum_{n1} x[n2 + Q n1] W_P^{n1 k1}
// (P-point DFTs at stride Q, twiddles, Q-point DFTs on contiguous blocks), so
// the result X[k] lands at register position OFF + rpos<N>(k) * S.  All
// indices and twiddles are compile-time constants: the twiddles come from a
// constexpr double-precision sine/cosine (Taylor series) rounded to float,
// so no table is loaded and every array index resolves to a register.
#pragma once

#include <utility>

#include "common.cuh"
#include "fft.cuh"

namespace gs {
namespace rf {

constexpr double kPiD = 3.14159265358979323846264338327950288;

// sin(x) for |x| <= pi/2 by its Taylor series (error < 1e-17)
constexpr double taylor_sin(double x) {
    double term = x, sum = x;
    for (int n = 1; n < 20; ++n) {
        term *= -x * x / ((2.0 * n) * (2.0 * n + 1.0));
        if (term < 1e-30 && term > -1e-30) break;  // negligible; also keeps the evaluation free of denormals
        sum += term;
    }
    return sum;
}
// sin(2 pi m / n) and cos(2 pi m / n), exact reduction on the integers first
constexpr double sin2pi(long m, long n) {
    m %= n;
    if (m < 0) m += n;
    if (m == 0 || 2 * m == n) return 0.0;
    if (4 * m == n) return 1.0;
    if (4 * m == 3 * n) return -1.0;
    // angle in [0, 2pi): reduce to [-pi/2, pi/2] using sin(pi - x) = sin(x)
    const double x = 2.0 * kPiD * (double)m / (double)n;
    if (4 * m <= n) return taylor_sin(x);                   // [0, pi/2]
    if (4 * m <= 3 * n) return taylor_sin(kPiD - x);        // (pi/2, 3pi/2]
    return taylor_sin(x - 2.0 * kPiD);                      // (3pi/2, 2pi)
}
constexpr double cos2pi(long m, long n) { return sin2pi(4 * m + n, 4 * n); }

template <int N, int M, bool kInv>
__host__ __device__ __forceinline__ float2 twc() {
    constexpr float c = (float)cos2pi(M, N);
    constexpr float s = (float)(kInv ? sin2pi(M, N) : -sin2pi(M, N));
    return make_float2(c, s);
}

template <int I, int N>
struct StaticFor {
    template <class F>
    __host__ __device__ __forceinline__ static void run(F&& f) {
        f(std::integral_constant<int, I>{});
        StaticFor<I + 1, N>::run(f);
    }
};
template <int N>
struct StaticFor<N, N> {
    template <class F>
    __host__ __device__ __forceinline__ static void run(F&&) {}
};
template <int N, class F>
__host__ __device__ __forceinline__ void static_for(F&& f) {
    StaticFor<0, N>::run(f);
}

constexpr bool is_base(int n) { return n == 2 || n == 3 || n == 4 || n == 5 || n == 8; }
constexpr int first_factor(int n) {
    return (n % 4 == 0 && n > 8) ? 4 : (n % 5 == 0 && n > 5) ? 5 : (n % 3 == 0 && n > 3) ? 3
         : (n % 2 == 0 && n > 8) ? 2 : n;
}
// register position of output k of an N-point rfft (unit stride)
template <int N>
constexpr int rpos(int k) {
    if constexpr (is_base(N)) {
        return k;
    } else {
        constexpr int P = first_factor(N), Q = N / P;
        return Q * (k % P) + rpos<Q>(k / P);
    }
}

template <int R, int S, bool kInv, int OFF>
__host__ __device__ __forceinline__ void base_dft(float2* a) {
    if constexpr (R == 2) {
        dft2<kInv>(a[OFF], a[OFF + S]);
    } else if constexpr (R == 3) {
        dft3<kInv>(a[OFF], a[OFF + S], a[OFF + 2 * S]);
    } else if constexpr (R == 4) {
        dft4<kInv>(a[OFF], a[OFF + S], a[OFF + 2 * S], a[OFF + 3 * S]);
    } else if constexpr (R == 5) {
        dft5<kInv>(a[OFF], a[OFF + S], a[OFF + 2 * S], a[OFF + 3 * S], a[OFF + 4 * S]);
    } else {
        float2 t[8];
#pragma unroll
        for (int q = 0; q < 8; ++q) t[q] = a[OFF + q * S];
        dft8<kInv>(t);
#pragma unroll
        for (int q = 0; q < 8; ++q) a[OFF + q * S] = t[q];
    }
}

template <int N, int S, bool kInv, int OFF = 0>
__host__ __device__ __forceinline__ void rfft(float2* a) {
    if constexpr (is_base(N)) {
        base_dft<N, S, kInv, OFF>(a);
    } else {
        constexpr int P = first_factor(N), Q = N / P;
        static_for<Q>([&](auto n2c) {
            constexpr int n2 = decltype(n2c)::value;
            base_dft<P, S * Q, kInv, OFF + n2 * S>(a);
        });
        static_for<Q>([&](auto n2c) {
            constexpr int n2 = decltype(n2c)::value;
            static_for<P>([&](auto k1c) {
                constexpr int k1 = decltype(k1c)::value;
                if constexpr ((n2 * k1) % N != 0) {
                    const float2 w = twc<N, n2 * k1, kInv>();
                    a[OFF + (n2 + Q * k1) * S] = cmul(a[OFF + (n2 + Q * k1) * S], w);
                }
            });
        });
        static_for<P>([&](auto k1c) {
            constexpr int k1 = decltype(k1c)::value;
            rfft<Q, S, kInv, OFF + Q * k1 * S>(a);
        });
    }
}

}  // namespace rf
}  // namespace gs
