// Register-resident small FFTs with compile-time twiddles.
//
// rfft<N, S, kInv, OFF>(a) transforms the N complex values a[OFF + n*S]
// (n < N) of a register array in place.  N is split recursively as
// N = P * Q with P a base radix (2, 3, 4, 5, 8).  When P and Q share a factor
// (Cooley-Tukey):
//     X[k1 + P k2] = sum_{n2} W_Q^{n2 k2} W_N^{n2 k1} sum_{n1} x[n2 + Q n1] W_P^{n1 k1}
// (P-point DFTs at stride Q, twiddles, Q-point DFTs on contiguous blocks).
// When they are coprime (Good-Thomas prime-factor mapping, no twiddles):
//     X[(a1 k1 + a2 k2) mod N] = sum_{n2} W_Q^{n2 k2} sum_{n1} W_P^{n1 k1} x[(Q n1 + P n2) mod N]
// with a1 = 1 mod P, 0 mod Q and a2 = 0 mod P, 1 mod Q (Chinese remainders).
// Either way the result X[k] lands at register position OFF + rpos<N>(k) * S.
// All indices and twiddles are compile-time constants: the twiddles come from
// a constexpr double-precision sine/cosine (Taylor series) rounded to float,
// twiddles of +-1 and +-i become sign changes and swaps, so no table is
// loaded and every array index resolves to a register.
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
constexpr int gcd_c(int a, int b) { return b == 0 ? a : gcd_c(b, a % b); }
// prime-factor split of N = first_factor(N) x rest (coprime factors)
template <int N>
constexpr bool is_pfa() {
    if constexpr (is_base(N)) {
        return false;
    } else {
        return gcd_c(first_factor(N), N / first_factor(N)) == 1;
    }
}
// register position of output k of an N-point rfft (unit stride)
template <int N>
constexpr int rpos(int k) {
    if constexpr (is_base(N)) {
        return k;
    } else {
        constexpr int P = first_factor(N), Q = N / P;
        if constexpr (is_pfa<N>())
            return (Q * (k % P) + P * rpos<Q>(k % Q)) % N;
        else
            return Q * (k % P) + rpos<Q>(k / P);
    }
}

// a * W_N^M (M != 0 mod N) with the constant twiddle of the transform's
// direction; quarter turns are exact swaps and sign changes
template <int N, int M, bool kInv>
__host__ __device__ __forceinline__ float2 twiddle_mul(float2 a) {
    constexpr int m = ((M % N) + N) % N;
    if constexpr (2 * m == N) {
        return make_float2(-a.x, -a.y);
    } else if constexpr (4 * m == N) {
        return mul_mi<kInv>(a);  // W_N^{N/4} = -i forward, +i inverse
    } else if constexpr (4 * m == 3 * N) {
        return mul_mi<!kInv>(a);
    } else {
        return cmul(a, twc<N, m, kInv>());
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
__host__ __device__ __forceinline__ void rfft(float2* a);

// Good-Thomas split N = P x Q, gcd(P, Q) = 1: P-point DFTs over n1 at the
// positions (Q n1 + P n2) mod N, then Q-point DFTs over n2 at (Q k1 + P n2)
// mod N, each gathered into a temporary (register renaming, no moves once
// unrolled).  Output k ends at position (Q (k mod P) + P rpos<Q>(k mod Q)) mod N.
template <int N, int S, bool kInv, int OFF>
__host__ __device__ __forceinline__ void rfft_pfa(float2* a) {
    constexpr int P = first_factor(N), Q = N / P;
    static_for<Q>([&](auto n2c) {
        constexpr int n2 = decltype(n2c)::value;
        float2 t[P];
        static_for<P>([&](auto jc) {
            constexpr int j = decltype(jc)::value;
            t[j] = a[OFF + ((Q * j + P * n2) % N) * S];
        });
        base_dft<P, 1, kInv, 0>(t);
        static_for<P>([&](auto jc) {
            constexpr int j = decltype(jc)::value;
            a[OFF + ((Q * j + P * n2) % N) * S] = t[j];
        });
    });
    static_for<P>([&](auto k1c) {
        constexpr int k1 = decltype(k1c)::value;
        float2 t[Q];
        static_for<Q>([&](auto jc) {
            constexpr int j = decltype(jc)::value;
            t[j] = a[OFF + ((Q * k1 + P * j) % N) * S];
        });
        rfft<Q, 1, kInv, 0>(t);
        static_for<Q>([&](auto jc) {
            constexpr int j = decltype(jc)::value;
            a[OFF + ((Q * k1 + P * j) % N) * S] = t[j];
        });
    });
}

template <int N, int S, bool kInv, int OFF>
__host__ __device__ __forceinline__ void rfft(float2* a) {
    if constexpr (is_base(N)) {
        base_dft<N, S, kInv, OFF>(a);
    } else if constexpr (is_pfa<N>()) {
        rfft_pfa<N, S, kInv, OFF>(a);
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
                if constexpr ((n2 * k1) % N != 0)
                    a[OFF + (n2 + Q * k1) * S] = twiddle_mul<N, n2 * k1, kInv>(a[OFF + (n2 + Q * k1) * S]);
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
