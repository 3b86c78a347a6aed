// Host-side check of the prime-factor (Good-Thomas) index maps of the
// window-720 correlation (gisspa_b200/csrc/corr.cuh CorrCfg, fastfft.cuh
// PfaCols): the column order of the stored spectra is a permutation whose
// inverse is PfaCols::physical, the row-read order is a permutation, and an
// inverse transform done the kernel's way (16-point DFTs over physical index
// n2 + 45 n1, then 45-point DFTs over n2 with no twiddles, output k1 + 16 k2
// landing on map_coord(k1, k2)) equals a direct double-precision inverse DFT.
// Built with nvcc and run on the CPU by tests/test_native.py.
#include <cmath>
#include <cstdio>
#include <random>
#include <vector>

#include "corr.cuh"

using namespace gs;

int main() {
    constexpr int N2 = 45, L = 16 * N2;
    using F = CorrCfg<N2, 16>;
    static_assert(F::kPfa, "window 720 is a prime-factor size");
    int bad = 0;
    const PfaCols pc = PfaCols::make(L);
    if (pc.N2 != N2) { printf("PfaCols::make(720) did not select the prime-factor order\n"); return 1; }
    if (PfaCols::make(512).N2 != 0 || PfaCols::make(768).N2 != 0) { printf("PfaCols for even N2\n"); bad = 1; }
    std::vector<int> seen(L, 0), seen_row(L, 0), seen_map(L, 0);
    for (int p = 0; p < L; ++p) {
        const int k = pc.logical(p);
        if (k < 0 || k >= L) { printf("logical(%d) = %d out of range\n", p, k); return 1; }
        seen[k]++;
        if (pc.physical(k) != p) { printf("physical(logical(%d)) = %d\n", p, pc.physical(k)); bad = 1; }
        const int r = F::spectrum_row(p);
        if (r != k) { printf("spectrum_row(%d) = %d != logical %d\n", p, r, k); bad = 1; }
        seen_row[r]++;
    }
    for (int k1 = 0; k1 < 16; ++k1)
        for (int k2 = 0; k2 < N2; ++k2) seen_map[F::map_coord(k1, k2)]++;
    for (int k = 0; k < L; ++k)
        if (seen[k] != 1 || seen_row[k] != 1 || seen_map[k] != 1) { printf("not a permutation at %d\n", k); bad = 1; }
    if (F::A1 % 16 != 1 || F::A1 % N2 != 0 || F::A2 % 16 != 0 || F::A2 % N2 != 1) { printf("CRT constants\n"); bad = 1; }

    // one 720-point inverse transform the kernel's way against a direct DFT
    std::mt19937 rng(720);
    std::normal_distribution<double> nd;
    std::vector<double> xr(L), xi(L);   // spectrum, natural frequency order
    for (int k = 0; k < L; ++k) { xr[k] = nd(rng); xi[k] = nd(rng); }
    std::vector<float2> phys(L);        // stored in PfaCols order
    for (int p = 0; p < L; ++p) phys[p] = make_float2((float)xr[pc.logical(p)], (float)xi[pc.logical(p)]);
    float2 tile[16][N2];
    for (int n2 = 0; n2 < N2; ++n2) {
        float2 x[16];
        for (int n1 = 0; n1 < 16; ++n1) x[n1] = phys[n2 + N2 * n1];
        rf::rfft<16, 1, true>(x);
        for (int k1 = 0; k1 < 16; ++k1) tile[k1][n2] = x[rf::rpos<16>(k1)];
    }
    double emax = 0, ref = 0;
    for (int k1 = 0; k1 < 16; ++k1) {
        float2 b[N2];
        for (int n2 = 0; n2 < N2; ++n2) b[n2] = tile[k1][n2];
        rf::rfft<N2, 1, true>(b);
        for (int k2 = 0; k2 < N2; ++k2) {
            const int y = F::map_coord(k1, k2);
            double sr = 0, si = 0;
            for (int k = 0; k < L; ++k) {
                const double a = 2.0 * M_PI * (double)((long)k * y % L) / L;
                sr += (double)(float)xr[k] * cos(a) - (double)(float)xi[k] * sin(a);
                si += (double)(float)xr[k] * sin(a) + (double)(float)xi[k] * cos(a);
            }
            const float2 g = b[rf::rpos<N2>(k2)];
            emax = fmax(emax, hypot(g.x - sr, g.y - si));
            ref = fmax(ref, hypot(sr, si));
        }
    }
    printf("720-point prime-factor inverse vs double DFT: max rel err %.3g\n", emax / ref);
    bad |= !(emax / ref < 2e-6);
    printf(bad ? "FAIL\n" : "OK\n");
    return bad;
}
