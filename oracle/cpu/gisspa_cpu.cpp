// C++/OpenMP FP32 restatement of the search's correlation and scoring, with
// its own FFT: the CPU baseline that bench.py times.  Test and measurement
// infrastructure only; the product never links or calls it.
//
// Per (window, template) unit, as the reference computes it (main.cu:824-876,
// GPU_func.cu:584-615 and 667-708): cc = inverse FFT (unnormalised) of
// W conj(T) (-1)^(x+y) (the checkerboard puts the peak at the particle
// centre), peak = max(0, max of cc over pixels at least d_m / 4 from the
// edges), pos = its index, sigma = standard deviation of cc without the peak
// (rc = l^2 - 1), score = peak / sigma (NaN when sigma <= 0).  Two templates
// share one complex transform: IFFT(W (conj T_a + i conj T_b) chk) =
// cc_a + i cc_b, both maps being real.
//
// FFT: Stockham self-sorting, mixed radix 4 / 2 / 3 / 5 (E. Bainville's
// formulation: stage with radix R and span p maps x[i + r n / R] to
// y[(i - k) R + k + r p], k = i mod p, after the twiddles
// exp(s 2 pi i r k / (R p))); the 2D transform runs the rows, transposes in
// 32 x 32 blocks, runs the rows again (the score reads the transposed map
// with the indices swapped).
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstring>
#include <vector>

#include <omp.h>

namespace {

using cf = std::complex<float>;

struct Stage {
    int R, p;
    std::vector<cf> tw;  // [k][r], r = 1 .. R-1
};

struct Plan {
    int n = 0;
    std::vector<Stage> st;
};

Plan make_plan(int n, int sign) {
    Plan pl;
    pl.n = n;
    int m = n, p = 1;
    auto add = [&](int R) {
        Stage s;
        s.R = R;
        s.p = p;
        s.tw.resize((size_t)p * (R - 1));
        for (int k = 0; k < p; ++k)
            for (int r = 1; r < R; ++r) {
                const double a = sign * 2.0 * M_PI * (double)r * k / ((double)R * p);
                s.tw[(size_t)k * (R - 1) + r - 1] = cf((float)cos(a), (float)sin(a));
            }
        pl.st.push_back(std::move(s));
        p *= R;
        m /= R;
    };
    while (m % 4 == 0) add(4);
    while (m % 2 == 0) add(2);
    while (m % 3 == 0) add(3);
    while (m % 5 == 0) add(5);
    if (m != 1) pl.n = 0;  // unsupported size
    return pl;
}

// One transform of length n, in -> out (in is destroyed), sign of the plan.
void fft1(const Plan& pl, cf* in, cf* out, int sign) {
    const int n = pl.n;
    cf* x = in;
    cf* y = out;
    const float sg = (float)sign;
    for (const Stage& s : pl.st) {
        const int R = s.R, p = s.p, q = n / R;
        for (int i = 0; i < q; ++i) {
            const int k = i % p;
            const cf* tw = s.tw.data() + (size_t)k * (R - 1);
            const int j = (i - k) * R + k;
            if (R == 4) {
                cf u0 = x[i], u1 = x[i + q] * tw[0], u2 = x[i + 2 * q] * tw[1], u3 = x[i + 3 * q] * tw[2];
                const cf a = u0 + u2, b = u0 - u2, c = u1 + u3, d = u1 - u3;
                const cf jd(-sg * d.imag(), sg * d.real());  // sign * i * d
                y[j] = a + c;
                y[j + p] = b + jd;
                y[j + 2 * p] = a - c;
                y[j + 3 * p] = b - jd;
            } else if (R == 2) {
                const cf u0 = x[i], u1 = x[i + q] * tw[0];
                y[j] = u0 + u1;
                y[j + p] = u0 - u1;
            } else if (R == 3) {
                const cf u0 = x[i], u1 = x[i + q] * tw[0], u2 = x[i + 2 * q] * tw[1];
                const float c1 = -0.5f, s1 = sg * 0.86602540378443864676f;
                const cf t = u1 + u2, dd = u1 - u2;
                const cf m1 = u0 + c1 * t;
                const cf m2(-s1 * dd.imag(), s1 * dd.real());
                y[j] = u0 + t;
                y[j + p] = m1 + m2;
                y[j + 2 * p] = m1 - m2;
            } else {  // R == 5
                const cf u0 = x[i], u1 = x[i + q] * tw[0], u2 = x[i + 2 * q] * tw[1], u3 = x[i + 3 * q] * tw[2],
                         u4 = x[i + 4 * q] * tw[3];
                const float c1 = 0.30901699437494742410f, c2 = -0.80901699437494742410f;
                const float s1 = sg * 0.95105651629515357212f, s2 = sg * 0.58778525229247312917f;
                const cf a1 = u1 + u4, b1 = u1 - u4, a2 = u2 + u3, b2 = u2 - u3;
                const cf m1 = u0 + c1 * a1 + c2 * a2, m2 = u0 + c2 * a1 + c1 * a2;
                const cf t1 = s1 * b1 + s2 * b2, t2 = s2 * b1 - s1 * b2;
                const cf n1(-t1.imag(), t1.real()), n2(-t2.imag(), t2.real());
                y[j] = u0 + a1 + a2;
                y[j + p] = m1 + n1;
                y[j + 4 * p] = m1 - n1;
                y[j + 2 * p] = m2 + n2;
                y[j + 3 * p] = m2 - n2;
            }
        }
        std::swap(x, y);
    }
    if (x != out) std::memcpy(out, x, sizeof(cf) * n);
}

void transpose(const cf* a, cf* b, int l) {
    constexpr int B = 32;
    for (int y0 = 0; y0 < l; y0 += B)
        for (int x0 = 0; x0 < l; x0 += B)
            for (int y = y0; y < std::min(l, y0 + B); ++y)
                for (int x = x0; x < std::min(l, x0 + B); ++x) b[(size_t)x * l + y] = a[(size_t)y * l + x];
}

struct Work {
    std::vector<cf> a, b, t;
};

// Inverse 2D transform of img (l x l) in place; on return `img` holds the
// TRANSPOSED map (element [x * l + y] is map (x, y)).
void ifft2_transposed(const Plan& pl, cf* img, Work& w, int l) {
    for (int y = 0; y < l; ++y) {
        std::memcpy(w.t.data(), img + (size_t)y * l, sizeof(cf) * l);
        fft1(pl, w.t.data(), img + (size_t)y * l, +1);
    }
    transpose(img, w.b.data(), l);
    for (int x = 0; x < l; ++x) {
        std::memcpy(w.t.data(), w.b.data() + (size_t)x * l, sizeof(cf) * l);
        fft1(pl, w.t.data(), img + (size_t)x * l, +1);
    }
}

void score_map(const cf* mt, int l, float d_m, bool imag, float* score, int* pos) {
    const float q_lo = d_m / 4.0f, q_hi = (float)l - q_lo;
    const int h = l / 2;
    double s1 = 0.0, s2 = 0.0;
    float best = 0.0f;
    int bpos = 0;
    for (int x = 0; x < l; ++x) {
        // map index (x, y) is stored as fftshifted particle-centre position
        // (X, Y) = ((x + h) mod l, (y + h) mod l) once the checkerboard is applied
        // to the spectrum; here the spectrum already carries it, so (x, y) IS
        // the centre position
        const bool xb = (float)x < q_lo || (float)x > q_hi;
        const cf* col = mt + (size_t)x * l;
        for (int y = 0; y < l; ++y) {
            const float v = imag ? col[y].imag() : col[y].real();
            s1 += v;
            s2 += (double)v * v;
            if (!xb && !((float)y < q_lo || (float)y > q_hi)) {
                const int idx = y * l + x;
                if (v > best || (v == best && v > 0.0f && idx < bpos)) {
                    best = v;
                    bpos = idx;
                }
            }
        }
    }
    (void)h;
    const double peak = best;
    const double ra = s1 - peak, rb = s2 - peak * peak, rc = (double)l * l - 1.0;
    const double sd = std::sqrt(rb / rc - (ra / rc) * (ra / rc));
    *score = sd > 0.0 ? (float)(peak / sd) : NAN;
    *pos = bpos;
}

}  // namespace

extern "C" {

// Correlation and scores of nw windows x nt templates.  W: nw x l x l
// complex window spectra; T: nt x l x l complex template spectra (both
// interleaved float32, natural order, as the search builds them).  Outputs
// score[w * nt + J], pos[w * nt + J].  threads <= 0: all.  Returns 0, or -1
// for a window size the FFT does not handle (factors other than 2, 3, 5).
int gsc_correlate(const float* W, int nw, const float* T, int nt, int l, float d_m, float* score, int* pos,
                  int threads) {
    const Plan pl = make_plan(l, +1);
    if (pl.n != l) return -1;
    const size_t l2 = (size_t)l * l;
    const cf* Wc = reinterpret_cast<const cf*>(W);
    const cf* Tc = reinterpret_cast<const cf*>(T);
    const int np = (nt + 1) / 2;
    const long long units = (long long)nw * np;
    if (threads <= 0) threads = omp_get_max_threads();
#pragma omp parallel num_threads(threads)
    {
        Work wk;
        wk.b.resize(l2);
        wk.t.resize(l);
        std::vector<cf> img(l2);
#pragma omp for schedule(dynamic, 1)
        for (long long u = 0; u < units; ++u) {
            const int w = (int)(u / np), pp = (int)(u % np);
            const int ja = 2 * pp, jb = 2 * pp + 1;
            const cf* Ww = Wc + (size_t)w * l2;
            const cf* Ta = Tc + (size_t)ja * l2;
            const cf* Tb = jb < nt ? Tc + (size_t)jb * l2 : nullptr;
            for (int y = 0; y < l; ++y) {
                const float cy = (y & 1) ? -1.0f : 1.0f;
                for (int x = 0; x < l; ++x) {
                    const size_t i = (size_t)y * l + x;
                    const float c = (x & 1) ? -cy : cy;
                    cf s = std::conj(Ta[i]);
                    if (Tb) s += cf(0.0f, 1.0f) * std::conj(Tb[i]);
                    img[i] = Ww[i] * s * c;
                }
            }
            ifft2_transposed(pl, img.data(), wk, l);
            score_map(img.data(), l, d_m, false, score + (size_t)w * nt + ja, pos + (size_t)w * nt + ja);
            if (Tb) score_map(img.data(), l, d_m, true, score + (size_t)w * nt + jb, pos + (size_t)w * nt + jb);
        }
    }
    return 0;
}

int gsc_max_threads(void) { return omp_get_max_threads(); }

}  // extern "C"
