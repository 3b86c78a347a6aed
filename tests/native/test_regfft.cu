// Host-side check of the register FFTs (gisspa_b200/csrc/regfft.cuh): every
// supported length, both directions, against a double-precision DFT.  Built
// with nvcc and run on the CPU by tests/test_native.py.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <random>

#include "regfft.cuh"

using namespace gs;

template <int N, bool kInv>
static double check(std::mt19937& rng) {
    std::normal_distribution<double> nd;
    double xr[N], xi[N];
    float2 a[N];
    for (int n = 0; n < N; ++n) {
        xr[n] = nd(rng);
        xi[n] = nd(rng);
        a[n] = make_float2((float)xr[n], (float)xi[n]);
    }
    rf::rfft<N, 1, kInv>(a);
    double err = 0, ref = 0;
    for (int k = 0; k < N; ++k) {
        double sr = 0, si = 0;
        for (int n = 0; n < N; ++n) {
            const double ang = (kInv ? 2.0 : -2.0) * M_PI * (double)((long)n * k % N) / N;
            sr += (double)(float)xr[n] * cos(ang) - (double)(float)xi[n] * sin(ang);
            si += (double)(float)xr[n] * sin(ang) + (double)(float)xi[n] * cos(ang);
        }
        const float2 g = a[rf::rpos<N>(k)];
        err = fmax(err, hypot(g.x - sr, g.y - si));
        ref = fmax(ref, hypot(sr, si));
    }
    return err / ref;
}

template <int N>
static int run(std::mt19937& rng) {
    double e = fmax(check<N, false>(rng), check<N, true>(rng));
    // permutation check: rpos is a bijection on [0, N)
    int seen[N] = {0};
    for (int k = 0; k < N; ++k) seen[rf::rpos<N>(k)]++;
    for (int k = 0; k < N; ++k)
        if (seen[k] != 1) { printf("N=%d rpos not a permutation\n", N); return 1; }
    printf("N=%d max rel err %.3g\n", N, e);
    return e < 2e-6 ? 0 : 1;
}

int main() {
    std::mt19937 rng(1234);
    int bad = 0;
    bad |= run<2>(rng); bad |= run<3>(rng); bad |= run<4>(rng); bad |= run<5>(rng); bad |= run<8>(rng);
    bad |= run<9>(rng); bad |= run<12>(rng); bad |= run<15>(rng); bad |= run<16>(rng);
    bad |= run<20>(rng); bad |= run<24>(rng); bad |= run<30>(rng); bad |= run<32>(rng);
    bad |= run<36>(rng); bad |= run<40>(rng); bad |= run<45>(rng); bad |= run<48>(rng);
    bad |= run<60>(rng); bad |= run<64>(rng);
    // constexpr trig against libm
    double te = 0;
    for (int n = 1; n < 200; ++n)
        for (int m = -n; m <= 2 * n; ++m) {
            te = fmax(te, fabs(rf::sin2pi(m, n) - sin(2 * M_PI * m / n)));
            te = fmax(te, fabs(rf::cos2pi(m, n) - cos(2 * M_PI * m / n)));
        }
    printf("constexpr trig max abs err %.3g\n", te);
    bad |= te > 1e-14;
    printf(bad ? "FAIL\n" : "OK\n");
    return bad;
}
