// Element-wise, reduction and fused-IO kernels of the GisSPA search.
//
// Each kernel cites the reference code whose result it reproduces.  The
// reference runs every step as a separate pass over HBM with host round
// trips for its reductions; here reductions stay on the device (FP64
// accumulators), and products / normalisation / the score epilogue are fused
// into the FFT kernels through IO functors.
#pragma once

#include "common.cuh"
#include "fft.cuh"

namespace gs {

// ---------------------------------------------------------------------------
// Templates (once per run)
// ---------------------------------------------------------------------------

// Pad a tx x ty template into l x l at ((l-tx)/2, (l-ty)/2) and edge-normalise
// it: (t - ring mean) / std(full l x l frame), the ring being the 1-px annulus
// (r-1)^2 <= d^2 <= (r+1)^2, r = l/2 - 2, around (l/2, l/2).
// Reference: readAndPaddingTemplate + edgeNormalize (main.cu:182-223,
// 311-385; kernels GPU_func.cu:3-94).  One CTA per template.
__global__ void __launch_bounds__(256) k_tmpl_pad_edge(const float* __restrict__ raw, int tx, int ty, int l,
                                                        float2* __restrict__ out) {
    __shared__ double red[4 * 32];
    const int J = blockIdx.x;
    const float* src = raw + (size_t)J * tx * ty;
    float2* dst = out + (size_t)J * l * l;
    const int sx = (l - tx) / 2, sy = (l - ty) / 2;
    const float r = (float)l / 2.0f - 2.0f;
    float up = 0.0f, low = 0.0f;
    if (r > 1.0f) {
        up = (r + 1.0f) * (r + 1.0f);
        low = (r - 1.0f) * (r - 1.0f);
    }
    const int h = l / 2;
    const int npix = l * l;
    double acc[4] = {0.0, 0.0, 0.0, 0.0};  // ring sum, ring count, sum, sum of squares
    for (int i = threadIdx.x; i < npix; i += blockDim.x) {
        const int x = i % l, y = i / l;
        float v = 0.0f;
        if (x >= sx && x < sx + tx && y >= sy && y < sy + ty) v = src[(y - sy) * tx + (x - sx)];
        const float rr = (float)((x - h) * (x - h) + (y - h) * (y - h));
        if (rr >= low && rr <= up) {
            acc[0] += v;
            acc[1] += 1.0;
        }
        acc[2] += v;
        acc[3] += (double)v * v;
    }
    block_sum<4>(acc, red);
    const double em = acc[1] > 0 ? acc[0] / acc[1] : 0.0;
    const double mean = acc[2] / npix;
    double sigma = sqrt(acc[3] / npix - mean * mean);
    if (!(sigma >= 0.0) || !isfinite(sigma)) sigma = 0.0;
    const bool scale = fabs(sigma) >= 1e-8;  // EPS of GPU_func.cuh:28
    for (int i = threadIdx.x; i < npix; i += blockDim.x) {
        const int x = i % l, y = i / l;
        float v = 0.0f;
        if (x >= sx && x < sx + tx && y >= sy && y < sy + ty) v = src[(y - sy) * tx + (x - sx)];
        if (scale) v = (float)(((double)v - em) / sigma);
        dst[i] = make_float2(v, 0.0f);
    }
}

// Radial-shell RMS of one template spectrum over the half plane x <= l/2:
// div[r] = sqrt(sum |F|^2 / count) for shells 0 <= r < l/2.
// Reference: SQRSum_by_circle, mode 0 (GPU_func.cu:98-128).  One CTA per
// template; shared memory holds the shell histogram (l/2 doubles + counts).
__global__ void __launch_bounds__(256) k_tmpl_shells(const float2* __restrict__ F, int l, float* __restrict__ div) {
    extern __shared__ double sh[];
    const int ns = l / 2;
    double* ra = sh;
    unsigned* rb = reinterpret_cast<unsigned*>(sh + ns);
    for (int r = threadIdx.x; r < ns; r += blockDim.x) {
        ra[r] = 0.0;
        rb[r] = 0u;
    }
    __syncthreads();
    const int J = blockIdx.x;
    const float2* src = F + (size_t)J * l * l;
    const int hw = l / 2 + 1;  // x <= l/2
    for (int i = threadIdx.x; i < hw * l; i += blockDim.x) {
        const int y = i / hw, x = i % hw;
        const int r = shell_index(x, y, l, l);
        if (r >= 0 && r < ns) {
            const float2 v = src[y * l + x];
            atomicAdd(&ra[r], (double)v.x * v.x + (double)v.y * v.y);
            atomicAdd(&rb[r], 1u);
        }
    }
    __syncthreads();
    for (int r = threadIdx.x; r < ns; r += blockDim.x)
        div[(size_t)J * ns + r] = (float)sqrt(ra[r] / (double)rb[r]);
}

struct WeightConsts {
    float hp, lp;        // l*apix/highres, l*apix/lowres (float)
    float ds;            // 1/(apix * configured window size)
    float kk, a, b, b2, bf, bf2, bf3;
};

// Per-bin band-pass x |CTF| x Wiener factor of the template weighting,
// identical for every template.  Reference: apply_weighting_function
// (GPU_func.cu:249-290), CTF of the first micrograph.
__global__ void k_weight_map(float* __restrict__ wmap, int l, WeightConsts wc, CtfDev c) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= l * l) return;
    const int x = i % l, y = i / l;
    float rf;
    const int r = shell_index(x, y, l, l, &rf);
    float f = bandpass<false>(r, wc.hp, wc.lp);
    if (r < l / 2 && r >= 0) {
        const float ss = rf * wc.ds;
        const float v = ctf_ast(x, (y + l / 2) % l, l, l, c, 2);
        const float signal = expf(wc.bf * ss * ss + wc.bf2 * ss + wc.bf3) / (wc.kk + 1.0f);
        const float ncurve = expf(wc.a * ss * ss + wc.b * ss + wc.b2) / signal;
        f *= v * sqrtf(1.0f / (ncurve + wc.kk * v * v));
    }
    wmap[i] = f;
}

// The whitened template spectrum alone (F / shell RMS, no weight), written
// to B: the base that the off-grid refinement re-weights with other CTF
// parameters.  Same whitening as k_tmpl_apply (whiten_Tmp, GPU_func.cu:130-152).
__global__ void __launch_bounds__(256) k_tmpl_whiten(const float2* __restrict__ F, int l, const float* __restrict__ div,
                                                     float2* __restrict__ B) {
    const int J = blockIdx.y;
    const int ns = l / 2;
    const float2* d = F + (size_t)J * l * l;
    const float* dv = div + (size_t)J * ns;
    const int npix = l * l;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < npix; i += gridDim.x * blockDim.x) {
        const int x = i % l, y = i / l;
        const int r = shell_index(x, y, l, l);
        float2 v = d[i];
        if (r >= 0 && r < ns) v = cscale(v, 1.0f / dv[r]);
        B[(size_t)J * l * l + i] = v;
    }
}

// Whiten by the shell RMS, apply the weight map, and accumulate per template
// sum |F|^2 and the count over r < l/2, x <= l/2.
// Reference: whiten_Tmp + apply_weighting_function + compute_area_sum_ofSQR
// (GPU_func.cu:130-152, 249-290, 318-362).  Grid (pixel chunks, templates).
__global__ void __launch_bounds__(256) k_tmpl_apply(float2* __restrict__ F, int l, const float* __restrict__ div,
                                                    const float* __restrict__ wmap, double* __restrict__ sumsq) {
    __shared__ double red[2 * 32];
    const int J = blockIdx.y;
    const int ns = l / 2;
    float2* d = F + (size_t)J * l * l;
    const float* dv = div + (size_t)J * ns;
    double acc[2] = {0.0, 0.0};
    const int npix = l * l;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < npix; i += gridDim.x * blockDim.x) {
        const int x = i % l, y = i / l;
        const int r = shell_index(x, y, l, l);
        float2 v = d[i];
        if (r >= 0 && r < ns) v = cscale(v, 1.0f / dv[r]);
        v = cscale(v, wmap[i]);
        d[i] = v;
        if (r >= 0 && r < ns && x <= l / 2) {
            acc[0] += (double)v.x * v.x + (double)v.y * v.y;
            acc[1] += 1.0;
        }
    }
    block_sum<2>(acc, red);
    if (threadIdx.x == 0) {
        atomicAdd(&sumsq[2 * J], acc[0]);
        atomicAdd(&sumsq[2 * J + 1], acc[1]);
    }
}

// 1 / m with m = sqrt(sum / count^2) (1 when m == 0).  Reference: the host
// loop after compute_area_sum_ofSQR and `normalize` (main.cu:446-456,
// GPU_func.cu:409-422).
__global__ void k_inv_amp_norm(const double* __restrict__ sumsq, int n, double* __restrict__ inv) {
    const int J = blockIdx.x * blockDim.x + threadIdx.x;
    if (J >= n) return;
    const double c = sumsq[2 * J + 1];
    const double m = sqrt(sumsq[2 * J] / (c * c));
    inv[J] = (m != 0.0 && isfinite(m)) ? 1.0 / m : 1.0;
}

// ---------------------------------------------------------------------------
// Micrograph (per micrograph)
// ---------------------------------------------------------------------------
struct MicStats {
    float avg;
    int up, low;
    int enabled;
};

// Per-pixel quotients of the reference's host statistics loop
// (main.cu:530-535): cur/nx/ny and cur*cur/nx/ny, IEEE float32 each.
__global__ void k_mic_quot(const float* __restrict__ img, long long n, int nx, int ny, float* __restrict__ q1,
                           float* __restrict__ q2) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float v = img[i];
    q1[i] = __fdiv_rn(__fdiv_rn(v, (float)nx), (float)ny);
    q2[i] = __fdiv_rn(__fdiv_rn(__fmul_rn(v, v), (float)nx), (float)ny);
}

// The two float32 running sums of main.cu:530-535 in their exact sequential
// order (float addition is not associative, and the reference's clamp bounds
// are integers cut from these sums, main.cu:536-543).  One CTA: thread 0 adds
// the terms in order from a shared-memory chunk while warps 1.. stage the
// next chunk (double buffer); the two sums are independent chains, so the
// loop runs at about one add latency per term.
constexpr int kSeqChunk = 2048;
__global__ void __launch_bounds__(1024) k_mic_seq(const float* __restrict__ q1, const float* __restrict__ q2,
                                                  long long n, MicStats* __restrict__ out) {
    __shared__ __align__(16) float b1[2][kSeqChunk];
    __shared__ __align__(16) float b2[2][kSeqChunk];
    const int tid = threadIdx.x;
    float s1 = 0.0f, s2 = 0.0f;
    // stage chunk 0
    for (int i = tid; i < kSeqChunk; i += blockDim.x) {
        const long long g = i;
        b1[0][i] = g < n ? q1[g] : 0.0f;
        b2[0][i] = g < n ? q2[g] : 0.0f;
    }
    int buf = 0;
    for (long long base = 0; base < n; base += kSeqChunk) {
        __syncthreads();  // chunk `buf` is staged; chunk buf^1 is free
        if (tid == 0) {
            const int cnt = (int)min((long long)kSeqChunk, n - base);
            const float4* v1 = reinterpret_cast<const float4*>(b1[buf]);
            const float4* v2 = reinterpret_cast<const float4*>(b2[buf]);
            int i = 0;
            for (; i + 4 <= cnt; i += 4) {
                const float4 a = v1[i >> 2], c = v2[i >> 2];
                s1 = __fadd_rn(s1, a.x); s2 = __fadd_rn(s2, c.x);
                s1 = __fadd_rn(s1, a.y); s2 = __fadd_rn(s2, c.y);
                s1 = __fadd_rn(s1, a.z); s2 = __fadd_rn(s2, c.z);
                s1 = __fadd_rn(s1, a.w); s2 = __fadd_rn(s2, c.w);
            }
            for (; i < cnt; ++i) {
                s1 = __fadd_rn(s1, b1[buf][i]);
                s2 = __fadd_rn(s2, b2[buf][i]);
            }
        } else if (tid >= 32) {
            const long long nb = base + kSeqChunk;
            for (int i = tid - 32; i < kSeqChunk; i += blockDim.x - 32) {
                const long long g = nb + i;
                b1[buf ^ 1][i] = g < n ? q1[g] : 0.0f;
                b2[buf ^ 1][i] = g < n ? q2[g] : 0.0f;
            }
        }
        buf ^= 1;
    }
    if (tid == 0) {
        const float avg = s1;
        const float aa = __fmul_rn(avg, avg);
        const float var = __fsqrt_rn(__fsub_rn(s2, aa));
        const float six = __fmul_rn(6.0f, var);
        MicStats st;
        st.avg = avg;
        st.up = isnan(var) ? 0 : (int)__fadd_rn(avg, six);
        st.low = isnan(var) ? 0 : (int)__fsub_rn(avg, six);
        st.enabled = s2 > aa ? 1 : 0;
        *out = st;
    }
}

// Hot-pixel clamp to the mean, optional inversion, real -> complex.
// Reference: init_d_image host loops + float2Complex (main.cu:541-551).
__global__ void k_mic_clamp(const float* __restrict__ img, long long n, const MicStats* __restrict__ st, int invert,
                            float2* __restrict__ out) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float v = img[i];
    const MicStats s = *st;
    if (s.enabled && (v > (float)s.up || v < (float)s.low)) v = s.avg;
    if (invert == 1) v = -v;
    out[i] = make_float2(v, 0.0f);
}

// Phase flip by sign(CTF) and the radial shell sums of |F|^2 over x <= nx/2,
// shells 0 <= r < max(nx,ny)/2 (pixel-index radius, anisotropic for
// nx != ny).  Reference: do_phase_flip + SQRSum_by_circle mode 1
// (GPU_func.cu:785-796, 98-128).  Each CTA owns a row range and keeps its
// histogram in shared memory.
__global__ void __launch_bounds__(256) k_mic_flip_shells(float2* __restrict__ F, int nx, int ny, CtfDev c,
                                                         double* __restrict__ ra, unsigned* __restrict__ rb) {
    extern __shared__ double sh[];
    const int ns = max(nx, ny) / 2;
    double* sra = sh;
    unsigned* srb = reinterpret_cast<unsigned*>(sh + ns);
    for (int r = threadIdx.x; r < ns; r += blockDim.x) {
        sra[r] = 0.0;
        srb[r] = 0u;
    }
    __syncthreads();
    const int rows_per = (ny + gridDim.x - 1) / gridDim.x;
    const int y0 = blockIdx.x * rows_per, y1 = min(ny, y0 + rows_per);
    for (long long i = (long long)y0 * nx + threadIdx.x; i < (long long)y1 * nx; i += blockDim.x) {
        const int y = (int)(i / nx), x = (int)(i % nx);
        float2 v = F[i];
        const float sgn = ctf_ast(x, (y + ny / 2) % ny, nx, ny, c, 0);
        v = cscale(v, sgn);
        F[i] = v;
        if (x <= nx / 2) {
            const int r = shell_index(x, y, nx, ny);
            if (r >= 0 && r < ns) {
                atomicAdd(&sra[r], (double)v.x * v.x + (double)v.y * v.y);
                atomicAdd(&srb[r], 1u);
            }
        }
    }
    __syncthreads();
    for (int r = threadIdx.x; r < ns; r += blockDim.x) {
        if (srb[r]) {
            atomicAdd(&ra[r], sra[r]);
            atomicAdd(&rb[r], srb[r]);
        }
    }
}

struct MicWhitenConsts {
    float apix, hp, lp, damp;  // hp/lp/damp = L*apix/highres, L*apix/lowres, L*apix/6 (float), L = max(nx,ny)
    float kk, a, b, b2, bf, bf2, bf3;
};

// Whitening by the shell RMS with the CTF/SNR model, exp(-100 s^2) damping
// beyond L*apix/6, band-pass, Wiener weight, then DC := 0.
// Reference: whiten_filetr_weight_Img + set_0Hz_to_0_at_RI
// (GPU_func.cu:155-227).
__global__ void k_mic_whiten(float2* __restrict__ F, int nx, int ny, CtfDev c, MicWhitenConsts w,
                             const double* __restrict__ ra, const unsigned* __restrict__ rb) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (long long)nx * ny) return;
    const int y = (int)(i / nx), x = (int)(i % nx);
    const float dx = (float)min(x, nx - x), dy = (float)min(y, ny - y);
    const int r = (int)floor((double)hypotf(dx, dy) + 0.5) - 1;
    const float ss = sqrtf((dx * dx / (float)(nx * nx) + dy * dy / (float)(ny * ny)) / (w.apix * w.apix));
    const int L = max(nx, ny);
    float f = 1.0f, v = 0.0f, signal = 1.0f, ncurve = 0.0f;
    const bool in = r < L / 2 && r >= 0;
    if (in) {
        v = ctf_ast(x, (y + ny / 2) % ny, nx, ny, c, 2);
        signal = expf(w.bf * ss * ss + w.bf2 * ss + w.bf3);
        ncurve = expf(w.a * ss * ss + w.b * ss + w.b2);
        f = sqrtf((signal * v * v + ncurve) / signal) / sqrtf((float)(ra[r] / (double)rb[r]));
        if ((float)r > w.damp) f *= expf(-100.0f * ss * ss);
    }
    f *= bandpass<true>(r, w.hp, w.lp);
    if (in) {
        signal /= (w.kk + 1.0f);
        ncurve /= signal;
        f *= sqrtf(1.0f / (ncurve + w.kk * v * v));
    }
    F[i] = (i == 0) ? make_float2(0.0f, 0.0f) : cscale(F[i], f);
}

__global__ void k_set_dc_zero(float2* F) { F[0] = make_float2(0.0f, 0.0f); }

// Cut l x l windows (window w = i + j*bx at (offx[i], offy[j]); zero beyond
// the image).  Reference: split_IMG (GPU_func.cu:564-581).
__global__ void k_extract_windows(const float* __restrict__ img, int nx, int ny, const int* __restrict__ offx,
                                  const int* __restrict__ offy, int bx, int l, float2* __restrict__ W) {
    const int w = blockIdx.y;
    const int i = w % bx, j = w / bx;
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < l * l; p += gridDim.x * blockDim.x) {
        const int x = p % l, y = p / l;
        const int px = offx[i] + x, py = offy[j] + y;
        const float v = (px < nx && py < ny) ? img[(size_t)py * nx + px] : 0.0f;
        W[(size_t)w * l * l + p] = make_float2(v, 0.0f);
    }
}

// Per-window sum |W|^2 and count over r < l/2, x <= l/2 (for the amplitude
// normalisation of split_normalize_image, main.cu:617-653).
__global__ void __launch_bounds__(256) k_win_sumsq(const float2* __restrict__ W, int l, double* __restrict__ out) {
    __shared__ double red[2 * 32];
    const int w = blockIdx.y;
    const float2* d = W + (size_t)w * l * l;
    double acc[2] = {0.0, 0.0};
    const int hw = l / 2 + 1;
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < hw * l; p += gridDim.x * blockDim.x) {
        const int y = p / hw, x = p % hw;
        const int r = shell_index(x, y, l, l);
        if (r >= 0 && r < l / 2) {
            const float2 v = d[y * l + x];
            acc[0] += (double)v.x * v.x + (double)v.y * v.y;
            acc[1] += 1.0;
        }
    }
    block_sum<2>(acc, red);
    if (threadIdx.x == 0) {
        atomicAdd(&out[2 * w], acc[0]);
        atomicAdd(&out[2 * w + 1], acc[1]);
    }
}

// Multiply image g by scale[g] (float).
__global__ void k_scale_images(float2* __restrict__ d, long long per_img, const double* __restrict__ scale) {
    const int g = blockIdx.y;
    const float s = (float)scale[g];
    float2* p = d + (size_t)g * per_img;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < per_img; i += (long long)gridDim.x * blockDim.x)
        p[i] = cscale(p[i], s);
}

// ---------------------------------------------------------------------------
// Per in-plane angle: template pair spectra
// ---------------------------------------------------------------------------

// Bilinear in-plane rotation + soft circular mask of both templates of pair
// p, written as (t_2p, t_2p+1) in one complex image, with FP64 sums and sums of
// squares of each template over the full l x l frame.
// Reference: rotate_subIMG + apply_mask + compute_sum_sqr
// (GPU_func.cu:496-560, 229-247, 363-407; main.cu:669-685).
// Several angles in one launch: with `cs` set, blockIdx.z selects angle z of
// the group ((cos, sin) = cs[z]), its images start at out + z Np l^2 and its
// sums at stats + 2 z ntmpl; without it, (cose, sine) and one angle.
__global__ void __launch_bounds__(256) k_pair_rotate(const float* __restrict__ tmpl, int ntmpl, int l, float cose,
                                                     float sine, const float2* __restrict__ cs, float d_m,
                                                     float2* __restrict__ out, double* __restrict__ stats) {
    __shared__ double red[4 * 32];
    const int p = blockIdx.y;
    const int J1 = 2 * p, J2 = 2 * p + 1;
    const bool has2 = J2 < ntmpl;
    const float* t1 = tmpl + (size_t)J1 * l * l;
    const float* t2 = tmpl + (size_t)(has2 ? J2 : J1) * l * l;
    if (cs) {
        const float2 c = cs[blockIdx.z];
        cose = c.x;
        sine = c.y;
        out += (size_t)blockIdx.z * gridDim.y * l * l;
        stats += (size_t)blockIdx.z * 2 * ntmpl;
    }
    float2* o = out + (size_t)p * l * l;
    const int h = l / 2;
    const float dm = 1.5f * d_m;
    const float rin = dm / 2.0f, rout = dm / 2.0f + 12.0f;
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    const int npix = l * l;
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < npix; q += gridDim.x * blockDim.x) {
        const int i = q % l, j = q / l;
        // mask first: outside radius rout the product with the mask is 0
        // whatever the rotated value, so its gathers are skipped
        const float r = hypotf((float)(i - h), (float)(j - h));
        float m = 1.0f;
        if (r > rout) m = 0.0f;
        else if (r >= rin) m = (float)(0.5 * (double)cosf((float)(kPiRef * (double)(r - rin) / 12.0)) + 0.5);
        const float x = (float)(i - h), y = (float)(j - h);
        const float x2 = (cose * x + sine * y) + h;
        const float y2 = (-sine * x + cose * y) + h;
        float v1 = 0.0f, v2 = 0.0f;
        if (m != 0.0f && !(x2 < 0 || x2 > l - 1.0f || y2 < 0 || y2 > l - 1.0f)) {
            const int ii = (int)floorf(x2), jj = (int)floorf(y2);
            const int k0 = ii + jj * l;
            int k1 = k0 + 1, k2 = k0 + l + 1, k3 = k0 + l;
            if (ii == l - 1) { k1--; k2--; }
            if (jj == l - 1) { k2 -= l; k3 -= l; }
            const float t = x2 - (float)ii, u = y2 - (float)jj;
            const float tt = 1.0f - t, uu = 1.0f - u;
            v1 = __ldg(t1 + k0) * tt * uu + __ldg(t1 + k1) * t * uu + __ldg(t1 + k2) * t * u + __ldg(t1 + k3) * tt * u;
            if (has2)
                v2 = __ldg(t2 + k0) * tt * uu + __ldg(t2 + k1) * t * uu + __ldg(t2 + k2) * t * u + __ldg(t2 + k3) * tt * u;
        }
        v1 *= m;
        v2 *= m;
        o[q] = make_float2(v1, v2);
        acc[0] += v1;
        acc[1] += (double)v1 * v1;
        acc[2] += v2;
        acc[3] += (double)v2 * v2;
    }
    block_sum<4>(acc, red);
    if (threadIdx.x == 0) {
        atomicAdd(&stats[2 * J1], acc[0]);
        atomicAdd(&stats[2 * J1 + 1], acc[1]);
        if (has2) {
            atomicAdd(&stats[2 * J2], acc[2]);
            atomicAdd(&stats[2 * J2 + 1], acc[3]);
        }
    }
}

// Per-template (mean, 1/sd) over the full frame; mean subtraction skipped if
// the mean is 0 and scaling skipped if the variance is 0, as in
// substract_by_mean / divided_by_var (GPU_func.cu:424-443, main.cu:696-707).
// `nang` angles one after the other: pair p of angle z at coef[z Np + p],
// from stats + 2 z ntmpl.
__global__ void k_pair_coef(const double* __restrict__ stats, int ntmpl, int l, float4* __restrict__ coef,
                            int nang) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int np = (ntmpl + 1) / 2;
    if (i >= np * nang) return;
    const int z = i / np, p = i - z * np;
    stats += (size_t)z * 2 * ntmpl;
    coef += (size_t)z * np;
    const double n = (double)l * l;
    float c[4] = {0.0f, 1.0f, 0.0f, 0.0f};
    for (int k = 0; k < 2; ++k) {
        const int J = 2 * p + k;
        if (J >= ntmpl) break;
        const double mean = stats[2 * J] / n;
        const double var = stats[2 * J + 1] / n - mean * mean;
        c[2 * k] = (float)mean;
        c[2 * k + 1] = var != 0.0 ? (float)(1.0 / sqrt(var)) : 1.0f;
    }
    coef[p] = make_float4(c[0], c[1], c[2], c[3]);
}

// Loader of the pair spectra: z = t1n - i t2n, where tkn is template k
// normalised to zero mean / unit variance, so that one complex FFT gives
// P = T1 - i T2 and W conj(P) = W conj(T1) + i W conj(T2).
struct IoPairNorm {
    float2* data;
    const float4* coef;
    long long img_elems;
    __device__ float2 load(int img, int, int, long long a) const {
        const float4 c = coef[img];
        const float2 z = data[a];
        return make_float2((z.x - c.x) * c.y, -(z.y - c.z) * c.w);
    }
    __device__ void store(int, int, int, long long a, float2 v) const { data[a] = v; }
    __device__ void finish(double*, int, int) const {}
};

// ---------------------------------------------------------------------------
// Correlation passes (per angle, per window)
// ---------------------------------------------------------------------------

// Row pass: S = W_w conj(P_p) on each spectrum row, inverse FFT along x,
// stored to the scratch map R_p.  Reference: compute_corner_CCG (its
// checkerboard is applied as an index shift and sign in the column pass)
// fused with the first half of the inverse cufftExecC2C (GPU_func.cu:584-615,
// main.cu:845-848).
struct IoPass1 {
    const float2* W;   // spectrum of this window, l x l
    const float2* P;   // pair spectra, img stride l*l
    float2* R;         // scratch, same layout as P
    long long l2;
    __device__ float2 load(int img, int, int, long long a) const {
        const long long off = a - (long long)img * l2;
        return cmulc(__ldg(W + off), P[a]);
    }
    __device__ void store(int, int, int, long long a, float2 v) const { R[a] = v; }
    __device__ void finish(double*, int, int) const {}
};

// Per (window, template) accumulators of the column pass.
struct UnitAcc {
    unsigned long long key;  // argmax_key of the border-masked max
    double s1, s2;           // sum and sum of squares of the whole map
};

// Column pass: inverse FFT along y, then the score epilogue on each output.
// The reference's map is out(X, Y) = (-1)^(l/2) s((X + l/2) mod l,
// (Y + l/2) mod l) for the unshifted inverse s (GPU_func.cu:607-614);
// template 2p is Re s, template 2p+1 is Im s.  The max ignores pixels with X
// or Y < d_m/4 or > l - d_m/4 (GPU_func.cu:681); sum and sum of squares take
// all l^2 pixels (GPU_func.cu:683-684).  Reference: get_peak_and_SUM +
// the host loop of pickPartcles_IMG_NORM (main.cu:850-866).
struct IoPass2 {
    const float2* R;
    UnitAcc* acc;
    int l, ntmpl;
    float q_lo, q_hi;
    float sgn;
    // per-thread state
    unsigned long long k1 = 0ull, k2 = 0ull;
    float s1a = 0.f, s2a = 0.f, s1b = 0.f, s2b = 0.f;
    int cur_img = -1;

    __device__ float2 load(int, int, int, long long a) const { return R[a]; }
    __device__ void store(int img, int v, int k, long long, float2 val) {
        cur_img = img;
        const int h = l / 2;
        int X = v + h; if (X >= l) X -= l;
        int Y = k + h; if (Y >= l) Y -= l;
        const int pos = Y * l + X;
        const float v1 = sgn * val.x, v2 = sgn * val.y;
        const bool border = (float)X < q_lo || (float)X > q_hi || (float)Y < q_lo || (float)Y > q_hi;
        if (!border) {
            const unsigned long long a = argmax_key(v1, pos), b = argmax_key(v2, pos);
            k1 = a > k1 ? a : k1;
            k2 = b > k2 ? b : k2;
        }
        s1a += v1; s2a += v1 * v1;
        s1b += v2; s2b += v2 * v2;
    }
    __device__ void finish(double* scratch, int, int) {
        double s[4] = {s1a, s2a, s1b, s2b};
        unsigned long long ka = warp_max_u64(k1), kb = warp_max_u64(k2);
        block_sum<4>(s, scratch);
        // block max of the keys through shared memory (scratch reused after block_sum's barrier)
        unsigned long long* ks = reinterpret_cast<unsigned long long*>(scratch);
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
        if (lane == 0) { ks[warp] = ka; ks[32 + warp] = kb; }
        __syncthreads();
        if (threadIdx.x == 0) {
            for (int w2 = 1; w2 < nw; ++w2) {
                ka = ks[w2] > ka ? ks[w2] : ka;
                kb = ks[32 + w2] > kb ? ks[32 + w2] : kb;
            }
            ka = ks[0] > ka ? ks[0] : ka;
            kb = ks[32] > kb ? ks[32] : kb;
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

struct UnitOut {
    float score;
    int pos;
    float peak;
    float sigma;
};

// Score of each (window, template): peak = max(0, masked max), sigma of the
// map without the peak (rc = l^2 - 1).  Reference: main.cu:869-876.
__global__ void k_finalize(const UnitAcc* __restrict__ acc, int ntmpl, int l, UnitOut* __restrict__ out) {
    const int J = blockIdx.x * blockDim.x + threadIdx.x;
    if (J >= ntmpl) return;
    const UnitAcc a = acc[J];
    const float peak = key_value(a.key);
    const int pos = key_index(a.key);
    const double ra = a.s1 - peak;
    const double rb = a.s2 - (double)peak * peak;
    const double rc = (double)l * l - 1.0;
    const double var = rb / rc - (ra / rc) * (ra / rc);
    const double sd = sqrt(var);  // NaN for var < 0, as sqrt in the reference
    UnitOut u;
    u.peak = peak;
    u.pos = pos;
    u.sigma = (float)sd;
    u.score = sd > 0.0 ? (float)(peak / sd) : __int_as_float(0x7fc00000);
    out[J] = u;
}

struct PickDev {
    long long unit;  // (angle * n_windows + window) * n_templates + template
    float cx, cy, score;
    int pad;
};

// Threshold + border test of every unit, compacted with an atomic counter
// (order restored on the host by sorting on `unit`).  Reference:
// main.cu:878-890.
// Threshold + centre test of the units of one micrograph (main.cu:869-891).
// The micrograph owns windows [w0, w0 + nw) of a units table laid out
// [angle][NW windows][nt templates]; pick.unit is its local index
// (angle, window, template), the reference's line order.
__global__ void k_compact(const UnitOut* __restrict__ units, long long total, int nw, int nt, int bx,
                          const int* __restrict__ offx, const int* __restrict__ offy, int l, float d_m, int nx, int ny,
                          float thres, PickDev* __restrict__ picks, unsigned long long* __restrict__ count,
                          long long cap, int NW, int w0) {
    const long long u = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (u >= total) return;
    const long long per = (long long)nw * nt;
    const long long ai = u / per, rem = u - ai * per;
    const UnitOut r = units[(ai * NW + w0) * nt + rem];
    if (!(r.score >= thres)) return;
    const int w = (int)(rem / nt);
    const int i = w % bx, j = w / bx;
    const float cx = (float)(offx[i] + r.pos % l);
    const float cy = (float)(offy[j] + r.pos / l);
    if (cx >= d_m && cx < (float)nx - d_m && cy >= d_m && cy < (float)ny - d_m) {
        const unsigned long long slot = atomicAdd(count, 1ull);
        if ((long long)slot < cap) {
            PickDev pk;
            pk.unit = u;
            pk.cx = cx;
            pk.cy = cy;
            pk.score = r.score;
            pk.pad = 0;
            picks[slot] = pk;
        }
    }
}

}  // namespace gs
