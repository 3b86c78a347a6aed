// Off-grid score of a pick and its gradient (adjoint), batched over picks.
//
// The objective continues the search's score off its grid of angles and
// pixels (no reference counterpart).  For pick p (window w, template J, map
// position x0, in-plane angle e, sub-pixel shift d, CTF theta = (defocus,
// dfdiff, dfang) of the template weight):
//   B   = FFT(b_J) / l^2                 b_J: padded, edge-normalised,
//                                        whitened template (main.cu:182-431)
//   F1  = B w(k; theta)                  band-pass x |CTF| Wiener weight
//                                        (GPU_func.cu:249-290)
//   t   = Re IFFT(F1 / a), a = sqrt(sum_sel |F1|^2) / cnt  (main.cu:447-463)
//   tm  = mask . rotate_bilinear(t, e)   (GPU_func.cu:496-560, 229-247)
//   tn  = (tm - mean) / sd               full frame (main.cu:697-710)
//   F   = FFT(tn) / l^2
//   c   = Re sum_k W(k) conj(F(k)) exp(2 pi i k.(x0 + d) / l), k signed
//   sig = sqrt(sum_k |W|^2 |F|^2)        map standard deviation (Parseval)
//   s   = sgn c / sig
// The adjoint runs the same chain backwards; it recomputes nothing it can
// keep from the forward of the same call (the per-pick buffers B, F1, tn and
// F stay in device memory for the backward) and stores no map.
#pragma once

#include "common.cuh"

namespace gs {

// One pick: inputs of the objective.
struct RefinePickDev {
    int window, tmpl, x0, y0;  // x0, y0: unshifted map position
    float e, dx, dy;           // degrees, pixels
    float defocus, dfdiff, dfang;  // um (positive underfocus), um, degrees
};

// Per-pick accumulators (double sums) and results.
struct RefineAcc {
    double asum;        // sum_sel |F1|^2
    double m1, m2;      // sum tm, sum tm^2
    double c, sig2, cdx, cdy;
    double g1, g2;      // sum gamma, sum gamma tn
    double de;          // d s / d e
    double abar;        // -Re sum Fbar2 conj(F1)
    double dth[3];      // d s / d theta
};

struct RefineConsts {
    int l;
    long long L2;
    float apix, lambda, cs, ampconst, kk, a, b, b2, bf, bf2, bf3, hp, lp, ds;
    float d_m;
    float cnt;  // number of (r < l/2, x <= l/2) bins
};

// Weight w(k; theta) and, optionally, its theta derivatives (float; the
// value path is the same arithmetic as k_weight_map).
__device__ __forceinline__ float refine_weight(int x, int y, const RefineConsts& rc, const RefinePickDev& pk,
                                               bool* insel, float dw[3]) {
    const int l = rc.l;
    float rf;
    const int r = shell_index(x, y, l, l, &rf);
    const float band = bandpass<false>(r, rc.hp, rc.lp);
    *insel = (r < l / 2 && r >= 0);
    dw[0] = dw[1] = dw[2] = 0.0f;
    if (!*insel) return band;
    // CTF geometry of ctf_ast(x, (y + l/2) % l)
    int x1 = x, y1 = (y + l / 2) % l;
    y1 = x1 > l / 2 ? l - y1 : y1;
    x1 = min(x1, l - x1);
    const float fx = (float)x1, fy = (float)(y1 - l / 2);
    const float ss = (fx * fx / (float)(l * l) + fy * fy / (float)(l * l)) / (rc.apix * rc.apix);
    const float ag = atan2f(fy, fx);
    const float D = -pk.defocus;
    const float dfu = D + pk.dfdiff, dfv = D - pk.dfdiff;
    const float ang2 = (float)(2.0 * ((double)pk.dfang * kPiRef / 180.0 - (double)ag));
    const float cs2 = cosf(ang2);
    const float df_ast = 0.5f * (dfu + dfv + 2.0f * pk.dfdiff * cs2);
    const double lam = (double)rc.lambda;
    const float gamma = (float)(-2.0 * kPiRef *
                                ((double)rc.cs * 2.5e6 * lam * lam * lam * (double)ss * (double)ss +
                                 (double)df_ast * 5000.0 * lam * (double)ss));
    const float sa = sqrtf(1.0f - rc.ampconst * rc.ampconst);
    float sg, cg;
    sincosf(gamma, &sg, &cg);
    const float V = sa * sg + rc.ampconst * cg;
    const float v = fabsf(V);
    const float ssw = rf * rc.ds;
    const float signal = expf(rc.bf * ssw * ssw + rc.bf2 * ssw + rc.bf3) / (rc.kk + 1.0f);
    const float ncurve = expf(rc.a * ssw * ssw + rc.b * ssw + rc.b2) / signal;
    const float den = ncurve + rc.kk * v * v;
    const float w = v * sqrtf(1.0f / den);
    // d w / d gamma = band * ncurve den^-3/2 * sign(V) (sa cos g - a sin g)
    const float dwdg = band * ncurve / (den * sqrtf(den)) * (V >= 0.0f ? 1.0f : -1.0f) *
                       (sa * cg - rc.ampconst * sg);
    const float dgdf = (float)(-2.0 * kPiRef * 5000.0 * lam * (double)ss);  // d gamma / d df_ast
    dw[0] = dwdg * dgdf * -1.0f;                                            // d df_ast / d defocus = -1
    dw[1] = dwdg * dgdf * cs2;                                              // d df_ast / d dfdiff
    dw[2] = dwdg * dgdf * (-2.0f * pk.dfdiff * sinf(ang2)) * (float)(kPiRef / 180.0);
    return band * w;
}

// ---- forward ----

// Row pass input of B = FFT(b_J): real base template of the pick's template.
struct IoBaseIn {
    const float* base;     // N x L2
    const RefinePickDev* pk;
    float2* out;           // picks x L2 (complex)
    long long L2;
    __device__ float2 load(int img, int, int, long long a) const {
        return make_float2(base[(long long)pk[img].tmpl * L2 + (a - (long long)img * L2)], 0.0f);
    }
    __device__ void store(int, int, int, long long a, float2 v) const { out[a] = v; }
    __device__ void finish(double*, int, int) const {}
};

// F1 = B w(theta); sum_sel |F1|^2 per pick.  Grid (pixel chunks, picks).
__global__ void __launch_bounds__(256) k_ref_weight(const float2* __restrict__ B, float2* __restrict__ F1,
                                                    const RefinePickDev* __restrict__ pks, RefineConsts rc,
                                                    RefineAcc* __restrict__ acc) {
    __shared__ double red[32];
    const int p = blockIdx.y;
    const RefinePickDev pk = pks[p];
    const int l = rc.l;
    double s = 0.0;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < rc.L2; i += (long long)gridDim.x * blockDim.x) {
        const int x = (int)(i % l), y = (int)(i / l);
        bool insel;
        float dw[3];
        const float w = refine_weight(x, y, rc, pk, &insel, dw);
        const float2 v = cscale(B[p * rc.L2 + i], w);
        F1[p * rc.L2 + i] = v;
        if (insel && x <= l / 2) s += (double)v.x * v.x + (double)v.y * v.y;
    }
    double v1[1] = {s};
    block_sum<1>(v1, red);
    if (threadIdx.x == 0) atomicAdd(&acc[p].asum, v1[0]);
}

// t = Re IFFT(F1 / a) (row pass: in F1 scaled by 1/a into T; column pass real out).
struct IoInvA {
    const float2* F1;
    float2* T;
    const RefineAcc* acc;
    float cnt;
    long long L2;
    __device__ float2 load(int img, int, int, long long a) const {
        const float inva = (float)((double)cnt / sqrt(acc[img].asum));
        return cscale(F1[a], inva);
    }
    __device__ void store(int, int, int, long long a, float2 v) const { T[a] = v; }
    __device__ void finish(double*, int, int) const {}
};

// Source coordinates of rotate_subIMG for output pixel (i, j) and angle e.
__device__ __forceinline__ void rot_src(int i, int j, int l, float c, float s, float* x2, float* y2) {
    const float h = (float)(l / 2);
    const float x = (float)(i - l / 2), y = (float)(j - l / 2);
    *x2 = fmaf(c, x, s * y) + h;
    *y2 = fmaf(-s, x, c * y) + h;
}

// Bilinear sample with the reference's index rules; corner indices and
// weights for the adjoint.
struct Bilin {
    int k[4];
    float w[4];
    float dt, du;  // d value / d (fractional x), d value / d (fractional y) factors
    bool inb;
};

__device__ __forceinline__ Bilin bilin(float x2, float y2, int l) {
    Bilin b;
    b.inb = !(x2 < 0.0f || x2 > (float)(l - 1) || y2 < 0.0f || y2 > (float)(l - 1));
    int ii = (int)floorf(x2), jj = (int)floorf(y2);
    ii = min(max(ii, 0), l - 1);
    jj = min(max(jj, 0), l - 1);
    const float t = x2 - (float)ii, u = y2 - (float)jj;
    int k0 = ii + jj * l, k1 = k0 + 1, k2 = k0 + l + 1, k3 = k0 + l;
    if (ii == l - 1) { k1 -= 1; k2 -= 1; }
    if (jj == l - 1) { k2 -= l; k3 -= l; }
    b.k[0] = k0; b.k[1] = k1; b.k[2] = k2; b.k[3] = k3;
    b.w[0] = (1.0f - t) * (1.0f - u);
    b.w[1] = t * (1.0f - u);
    b.w[2] = t * u;
    b.w[3] = (1.0f - t) * u;
    b.dt = t;
    b.du = u;
    return b;
}

// tm = mask . rotate(t, e) into TM (real), sums of tm and tm^2.
__global__ void __launch_bounds__(256) k_ref_rotate(const float2* __restrict__ T, float* __restrict__ TM,
                                                    const RefinePickDev* __restrict__ pks, RefineConsts rc,
                                                    const float* __restrict__ mask, RefineAcc* __restrict__ acc) {
    __shared__ double red[64];
    const int p = blockIdx.y;
    const int l = rc.l;
    const double ang = (double)pks[p].e * kPiRef / 180.0;
    const float c = (float)cos(ang), s = (float)sin(ang);
    const float2* src = T + p * rc.L2;
    double a2[2] = {0.0, 0.0};
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < rc.L2; i += (long long)gridDim.x * blockDim.x) {
        const int x = (int)(i % l), y = (int)(i / l);
        float x2, y2;
        rot_src(x, y, l, c, s, &x2, &y2);
        const Bilin b = bilin(x2, y2, l);
        float v = 0.0f;
        if (b.inb)
            v = src[b.k[0]].x * b.w[0] + src[b.k[1]].x * b.w[1] + src[b.k[3]].x * b.w[3] + src[b.k[2]].x * b.w[2];
        v *= mask[i];
        TM[p * rc.L2 + i] = v;
        a2[0] += v;
        a2[1] += (double)v * v;
    }
    block_sum<2>(a2, red);
    if (threadIdx.x == 0) {
        atomicAdd(&acc[p].m1, a2[0]);
        atomicAdd(&acc[p].m2, a2[1]);
    }
}

__device__ __forceinline__ void ref_moments(const RefineAcc& a, double L2, double* mu, double* sd) {
    *mu = a.m1 / L2;
    const double var = a.m2 / L2 - *mu * *mu;
    *sd = sqrt(var > 0.0 ? var : 1.0);
}

// Row pass input of F = FFT(tn): normalised tm.
struct IoNormIn {
    const float* TM;
    const RefineAcc* acc;
    float2* out;
    long long L2;
    __device__ float2 load(int img, int, int, long long a) const {
        double mu, sd;
        ref_moments(acc[img], (double)L2, &mu, &sd);
        return make_float2((float)(((double)TM[a] - mu) / sd), 0.0f);
    }
    __device__ void store(int, int, int, long long a, float2 v) const { out[a] = v; }
    __device__ void finish(double*, int, int) const {}
};

// Phase exp(2 pi i (kx (x0 + dx) + ky (y0 + dy)) / l) with signed k; the
// integer part of the phase in integer arithmetic.
__device__ __forceinline__ float2 ref_phase(int kx, int ky, int l, const RefinePickDev& pk, int* kxs, int* kys) {
    const int sx = kx < (l + 1) / 2 ? kx : kx - l;
    const int sy = ky < (l + 1) / 2 ? ky : ky - l;
    *kxs = sx;
    *kys = sy;
    long long ip = ((long long)sx * pk.x0 + (long long)sy * pk.y0) % l;
    if (ip < 0) ip += l;
    const double frac = ((double)ip + (double)sx * pk.dx + (double)sy * pk.dy) / (double)l;
    double sn, cs;
    sincospi(2.0 * (frac - floor(frac)), &sn, &cs);
    return make_float2((float)cs, (float)sn);
}

// c, sigma^2 and d c / d (dx, dy): reductions over the spectrum.
__global__ void __launch_bounds__(256) k_ref_score(const float2* __restrict__ W, const float2* __restrict__ F,
                                                   const RefinePickDev* __restrict__ pks, RefineConsts rc,
                                                   RefineAcc* __restrict__ acc) {
    __shared__ double red[4 * 32];
    const int p = blockIdx.y;
    const RefinePickDev pk = pks[p];
    const int l = rc.l;
    const float2* Wp = W + (long long)pk.window * rc.L2;
    const float2* Fp = F + p * rc.L2;
    double a4[4] = {0.0, 0.0, 0.0, 0.0};
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < rc.L2; i += (long long)gridDim.x * blockDim.x) {
        const int kx = (int)(i % l), ky = (int)(i / l);
        int sx, sy;
        const float2 E = ref_phase(kx, ky, l, pk, &sx, &sy);
        const float2 G = cmulc(Wp[i], Fp[i]);          // W conj(F)
        const float2 GE = cmul(G, E);
        a4[0] += GE.x;
        const float w2 = Wp[i].x * Wp[i].x + Wp[i].y * Wp[i].y;
        const float f2 = Fp[i].x * Fp[i].x + Fp[i].y * Fp[i].y;
        a4[1] += (double)w2 * f2;
        // d/d dx of Re(GE) = Re(GE * 2 pi i kx / l) = -Im(GE) 2 pi kx / l
        a4[2] += -(double)GE.y * (2.0 * kPiRef * sx / l);
        a4[3] += -(double)GE.y * (2.0 * kPiRef * sy / l);
    }
    block_sum<4>(a4, red);
    if (threadIdx.x == 0) {
        atomicAdd(&acc[p].c, a4[0]);
        atomicAdd(&acc[p].sig2, a4[1]);
        atomicAdd(&acc[p].cdx, a4[2]);
        atomicAdd(&acc[p].cdy, a4[3]);
    }
}

// ---- backward ----

// Fbar = (sgn / sig) W E - (sgn c / sig^3) |W|^2 F, then (column pass of) the
// inverse transform: gamma = Re IFFT(Fbar) / l^2.
struct IoFbarIn {
    const float2* W;
    const float2* F;
    const RefinePickDev* pk;
    const RefineAcc* acc;
    float2* out;
    int l;
    long long L2;
    float sgn;
    __device__ float2 load(int img, int, int, long long a) const {
        const long long i = a - (long long)img * L2;
        const int kx = (int)(i % l), ky = (int)(i / l);
        int sx, sy;
        const RefinePickDev q = pk[img];
        const float2 E = ref_phase(kx, ky, l, q, &sx, &sy);
        const float2 w = W[(long long)q.window * L2 + i];
        const float2 f = F[a];
        const double sig = sqrt(acc[img].sig2);
        const float c1 = (float)(sgn / sig);
        const float c2 = (float)(sgn * acc[img].c / (sig * sig * sig));
        const float w2 = w.x * w.x + w.y * w.y;
        const float2 we = cmul(w, E);
        return make_float2(c1 * we.x - c2 * w2 * f.x, c1 * we.y - c2 * w2 * f.y);
    }
    __device__ void store(int, int, int, long long a, float2 v) const { out[a] = v; }
    __device__ void finish(double*, int, int) const {}
};

// sums of gamma and gamma tn (gamma = real part of G, already / l^2).
__global__ void __launch_bounds__(256) k_ref_gsum(const float2* __restrict__ Gm, const float* __restrict__ TM,
                                                  RefineConsts rc, RefineAcc* __restrict__ acc) {
    __shared__ double red[64];
    const int p = blockIdx.y;
    double mu, sd;
    ref_moments(acc[p], (double)rc.L2, &mu, &sd);
    double a2[2] = {0.0, 0.0};
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < rc.L2; i += (long long)gridDim.x * blockDim.x) {
        const double g = Gm[p * rc.L2 + i].x;
        const double tn = ((double)TM[p * rc.L2 + i] - mu) / sd;
        a2[0] += g;
        a2[1] += g * tn;
    }
    block_sum<2>(a2, red);
    if (threadIdx.x == 0) {
        atomicAdd(&acc[p].g1, a2[0]);
        atomicAdd(&acc[p].g2, a2[1]);
    }
}

// Normalisation, mask and rotation adjoints: d s / d e (reduction) and
// tbar (scatter-add into TB, real parts, zeroed beforehand).
__global__ void __launch_bounds__(256) k_ref_rot_adj(const float2* __restrict__ Gm, const float* __restrict__ TM,
                                                     const float2* __restrict__ T, const RefinePickDev* __restrict__ pks,
                                                     RefineConsts rc, const float* __restrict__ mask,
                                                     RefineAcc* __restrict__ acc, float* __restrict__ TB) {
    __shared__ double red[32];
    const int p = blockIdx.y;
    const int l = rc.l;
    double mu, sd;
    ref_moments(acc[p], (double)rc.L2, &mu, &sd);
    const double L2 = (double)rc.L2;
    const double mg = acc[p].g1 / L2, mgt = acc[p].g2 / L2;
    const double ang = (double)pks[p].e * kPiRef / 180.0;
    const float c = (float)cos(ang), s = (float)sin(ang);
    const float2* src = T + p * rc.L2;
    float* tb = TB + p * rc.L2;
    const float dr = (float)(kPiRef / 180.0);
    double de = 0.0;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < rc.L2; i += (long long)gridDim.x * blockDim.x) {
        const int x = (int)(i % l), y = (int)(i / l);
        const double g = Gm[p * rc.L2 + i].x;
        const double tn = ((double)TM[p * rc.L2 + i] - mu) / sd;
        const float gm = (float)((g - mg - tn * mgt) / sd) * mask[i];  // d s / d rotated pixel
        if (gm == 0.0f) continue;
        float x2, y2;
        rot_src(x, y, l, c, s, &x2, &y2);
        const Bilin b = bilin(x2, y2, l);
        if (!b.inb) continue;
        const float v0 = src[b.k[0]].x, v1 = src[b.k[1]].x, v2 = src[b.k[2]].x, v3 = src[b.k[3]].x;
        // value = (1-t)(1-u) v0 + t(1-u) v1 + t u v2 + (1-t) u v3
        const float dvdt = (1.0f - b.du) * (v1 - v0) + b.du * (v2 - v3);
        const float dvdu = (1.0f - b.dt) * (v3 - v0) + b.dt * (v2 - v1);
        const float xf = (float)(x - l / 2), yf = (float)(y - l / 2);
        const float dx2 = dr * (-s * xf + c * yf), dy2 = dr * (-c * xf - s * yf);
        de += (double)gm * (dvdt * dx2 + dvdu * dy2);
#pragma unroll
        for (int q = 0; q < 4; ++q) atomicAdd(&tb[b.k[q]], gm * b.w[q]);
    }
    double v1[1] = {de};
    block_sum<1>(v1, red);
    if (threadIdx.x == 0) atomicAdd(&acc[p].de, v1[0]);
}

// Row pass input of Fbar2 = FFT(tbar) (real).
struct IoRealIn2 {
    const float* src;
    float2* out;
    __device__ float2 load(int, int, int, long long a) const { return make_float2(src[a], 0.0f); }
    __device__ void store(int, int, int, long long a, float2 v) const { out[a] = v; }
    __device__ void finish(double*, int, int) const {}
};

// abar = -Re sum Fbar2 conj(F1) / a^2 (only the sum here).
__global__ void __launch_bounds__(256) k_ref_abar(const float2* __restrict__ Fb2, const float2* __restrict__ F1,
                                                  RefineConsts rc, RefineAcc* __restrict__ acc) {
    __shared__ double red[32];
    const int p = blockIdx.y;
    double s = 0.0;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < rc.L2; i += (long long)gridDim.x * blockDim.x) {
        const float2 u = Fb2[p * rc.L2 + i], v = F1[p * rc.L2 + i];
        s += (double)u.x * v.x + (double)u.y * v.y;
    }
    double v1[1] = {s};
    block_sum<1>(v1, red);
    if (threadIdx.x == 0) atomicAdd(&acc[p].abar, v1[0]);
}

// Fbar1 = Fbar2 / a + abar_total F1 sel / (cnt^2 a); theta gradient
// reductions; Bbar = Fbar1 w written over Fb2 (for the template gradient).
__global__ void __launch_bounds__(256) k_ref_theta(float2* __restrict__ Fb2, const float2* __restrict__ F1,
                                                   const float2* __restrict__ B, const RefinePickDev* __restrict__ pks,
                                                   RefineConsts rc, RefineAcc* __restrict__ acc) {
    __shared__ double red[3 * 32];
    const int p = blockIdx.y;
    const RefinePickDev pk = pks[p];
    const int l = rc.l;
    const double a = sqrt(acc[p].asum) / (double)rc.cnt;
    const double abar = -acc[p].abar / (a * a);
    const double k2 = abar / ((double)rc.cnt * (double)rc.cnt * a);
    double t3[3] = {0.0, 0.0, 0.0};
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < rc.L2; i += (long long)gridDim.x * blockDim.x) {
        const int x = (int)(i % l), y = (int)(i / l);
        bool insel;
        float dw[3];
        const float w = refine_weight(x, y, rc, pk, &insel, dw);
        const float2 f1 = F1[p * rc.L2 + i];
        float2 fb = cscale(Fb2[p * rc.L2 + i], (float)(1.0 / a));
        if (insel && x <= l / 2) {
            fb.x += (float)(k2 * f1.x);
            fb.y += (float)(k2 * f1.y);
        }
        const float2 bb = B[p * rc.L2 + i];
        const double re = (double)fb.x * bb.x + (double)fb.y * bb.y;  // Re(Fbar1 conj(B))
        t3[0] += re * dw[0];
        t3[1] += re * dw[1];
        t3[2] += re * dw[2];
        Fb2[p * rc.L2 + i] = cscale(fb, w);
    }
    block_sum<3>(t3, red);
    if (threadIdx.x == 0) {
        atomicAdd(&acc[p].dth[0], t3[0]);
        atomicAdd(&acc[p].dth[1], t3[1]);
        atomicAdd(&acc[p].dth[2], t3[2]);
    }
}

}  // namespace gs
