// Batched 1D complex FFTs in shared memory: mixed-radix Stockham autosort.
//
// Replaces the reference's cuFFT plans (main.cu:305, 504, 518): one CTA
// transforms a tile of vectors (rows, or columns of a row-major image) held
// in shared memory, stage by stage.  Each stage of radix r takes, for
// butterfly j of a vector of length n (m = n/r butterflies, L = product of
// the radices already applied, k = j mod L):
//     a_q = x[j + q*m] * w_{L r}^{q k}            q = 0..r-1
//     X   = DFT_r(a)
//     y[(j - k) r + k + p L] = X_p                p = 0..r-1
// which leaves the result in natural order after the last stage.
// Forward = exp(-2 pi i jk/n), inverse = exp(+2 pi i jk/n), both unscaled
// (cuFFT's convention); callers apply 1/n where the reference does.
//
// Loading and storing go through an IO functor so that products, scaling,
// normalisation and reductions fuse into the transform instead of costing
// separate passes over HBM.
#pragma once

#include "common.cuh"

namespace gs {

constexpr int kFftMaxStages = 24;

// Factorisation of one transform length plus its twiddle table
// tw[k] = exp(-2 pi i k / n), k < n (computed in double on the host).
struct FftDesc {
    int n;
    int nst;
    int radix[kFftMaxStages];
    const float2* tw;
};

__device__ __forceinline__ float2 twiddle(const float2* tw, int idx, bool inv) {
    float2 w = __ldg(tw + idx);
    return inv ? make_float2(w.x, -w.y) : w;
}

template <bool kInv>
__host__ __device__ __forceinline__ void dft2(float2& a0, float2& a1) {
    float2 t = a0;
    a0 = cadd(t, a1);
    a1 = csub(t, a1);
}

template <bool kInv>
__host__ __device__ __forceinline__ void dft3(float2& a0, float2& a1, float2& a2) {
    const float s = 0.86602540378443864676f;
    float2 t1 = cadd(a1, a2);
    float2 t2 = make_float2(a0.x - 0.5f * t1.x, a0.y - 0.5f * t1.y);
    float2 d = csub(a1, a2);
    float2 rot = cscale(mul_mi<kInv>(d), s);
    a0 = cadd(a0, t1);
    a1 = cadd(t2, rot);
    a2 = csub(t2, rot);
}

template <bool kInv>
__host__ __device__ __forceinline__ void dft4(float2& a0, float2& a1, float2& a2, float2& a3) {
    float2 s02 = cadd(a0, a2), d02 = csub(a0, a2);
    float2 s13 = cadd(a1, a3), d13 = mul_mi<kInv>(csub(a1, a3));
    a0 = cadd(s02, s13);
    a2 = csub(s02, s13);
    a1 = cadd(d02, d13);
    a3 = csub(d02, d13);
}

template <bool kInv>
__host__ __device__ __forceinline__ void dft5(float2& a0, float2& a1, float2& a2, float2& a3, float2& a4) {
    const float c1 = 0.30901699437494742410f;   // cos(2 pi / 5)
    const float c2 = -0.80901699437494742410f;  // cos(4 pi / 5)
    const float s1 = 0.95105651629515357212f;   // sin(2 pi / 5)
    const float s2 = 0.58778525229247312917f;   // sin(4 pi / 5)
    float2 p14 = cadd(a1, a4), m14 = csub(a1, a4);
    float2 p23 = cadd(a2, a3), m23 = csub(a2, a3);
    float2 b1 = make_float2(a0.x + c1 * p14.x + c2 * p23.x, a0.y + c1 * p14.y + c2 * p23.y);
    float2 b2 = make_float2(a0.x + c2 * p14.x + c1 * p23.x, a0.y + c2 * p14.y + c1 * p23.y);
    // forward: X1 = b1 - i(s1 m14 + s2 m23), X2 = b2 - i(s2 m14 - s1 m23)
    float2 e1 = make_float2(s1 * m14.x + s2 * m23.x, s1 * m14.y + s2 * m23.y);
    float2 e2 = make_float2(s2 * m14.x - s1 * m23.x, s2 * m14.y - s1 * m23.y);
    e1 = mul_mi<kInv>(e1);
    e2 = mul_mi<kInv>(e2);
    a0 = cadd(a0, cadd(p14, p23));
    a1 = cadd(b1, e1);
    a4 = csub(b1, e1);
    a2 = cadd(b2, e2);
    a3 = csub(b2, e2);
}

template <bool kInv>
__host__ __device__ __forceinline__ void dft8(float2* a) {
    const float h = 0.70710678118654752440f;
    // even / odd radix-4 halves
    float2 e0 = a[0], e1 = a[2], e2 = a[4], e3 = a[6];
    float2 o0 = a[1], o1 = a[3], o2 = a[5], o3 = a[7];
    dft4<kInv>(e0, e1, e2, e3);
    dft4<kInv>(o0, o1, o2, o3);
    // w8^1 = h(1 -+ i), w8^2 = -+i, w8^3 = h(-1 -+ i)
    float2 w1o1 = kInv ? make_float2(h * (o1.x - o1.y), h * (o1.x + o1.y))
                       : make_float2(h * (o1.x + o1.y), h * (o1.y - o1.x));
    float2 w2o2 = mul_mi<kInv>(o2);
    float2 w3o3 = kInv ? make_float2(-h * (o3.x + o3.y), h * (o3.x - o3.y))
                       : make_float2(h * (o3.y - o3.x), -h * (o3.x + o3.y));
    a[0] = cadd(e0, o0);
    a[4] = csub(e0, o0);
    a[1] = cadd(e1, w1o1);
    a[5] = csub(e1, w1o1);
    a[2] = cadd(e2, w2o2);
    a[6] = csub(e2, w2o2);
    a[3] = cadd(e3, w3o3);
    a[7] = csub(e3, w3o3);
}

// One Stockham stage of radix R for butterfly j of one vector.
template <int R, bool kInv>
__device__ __forceinline__ void stage_fixed(const float2* __restrict__ in, float2* __restrict__ out, int m,
                                            int k, int L, int twstep, const float2* tw) {
    float2 a[R];
#pragma unroll
    for (int q = 0; q < R; ++q) a[q] = in[q * m];
    if (k != 0) {
#pragma unroll
        for (int q = 1; q < R; ++q) a[q] = cmul(a[q], twiddle(tw, q * k * twstep, kInv));
    }
    if (R == 2) dft2<kInv>(a[0], a[1]);
    if (R == 3) dft3<kInv>(a[0], a[1], a[2]);
    if (R == 4) dft4<kInv>(a[0], a[1], a[2], a[3]);
    if (R == 5) dft5<kInv>(a[0], a[1], a[2], a[3], a[4]);
    if (R == 8) dft8<kInv>(a);
#pragma unroll
    for (int p = 0; p < R; ++p) out[p * L] = a[p];
}

// Generic prime radix: O(r^2), inputs twiddled in place first (each input of a
// stage belongs to exactly one butterfly, so no other thread reads them).
template <bool kInv>
__device__ __forceinline__ void stage_generic(float2* in, float2* __restrict__ out, int r, int m, int k, int L,
                                              int twstep, int n, const float2* tw) {
    if (k != 0) {
        for (int q = 1; q < r; ++q) in[q * m] = cmul(in[q * m], twiddle(tw, q * k * twstep, kInv));
    }
    const int nr = n / r;
    for (int p = 0; p < r; ++p) {
        float2 acc = in[0];
        int e = 0;
        for (int q = 1; q < r; ++q) {
            e += p;
            if (e >= r) e -= r;
            acc = cadd(acc, cmul(in[q * m], twiddle(tw, e * nr, kInv)));
        }
        out[p * L] = acc;
    }
}

// Transform `nvec` vectors stored at buf[v * pitch + k] (k < n).  All threads
// of the block must call it.  Returns the buffer (buf or alt) holding the
// result.
template <bool kInv>
__device__ float2* block_fft(float2* buf, float2* alt, int nvec, int pitch, const FftDesc& P) {
    const int n = P.n;
    int L = 1;
    float2* src = buf;
    float2* dst = alt;
    for (int s = 0; s < P.nst; ++s) {
        const int r = P.radix[s];
        const int m = n / r;
        const int twstep = n / (L * r);
        const int total = nvec * m;
        for (int b = threadIdx.x; b < total; b += blockDim.x) {
            const int v = b / m;
            const int j = b - v * m;
            const int k = j % L;
            float2* in = src + v * pitch + j;
            float2* out = dst + v * pitch + (j - k) * r + k;
            switch (r) {
                case 2: stage_fixed<2, kInv>(in, out, m, k, L, twstep, P.tw); break;
                case 3: stage_fixed<3, kInv>(in, out, m, k, L, twstep, P.tw); break;
                case 4: stage_fixed<4, kInv>(in, out, m, k, L, twstep, P.tw); break;
                case 5: stage_fixed<5, kInv>(in, out, m, k, L, twstep, P.tw); break;
                case 8: stage_fixed<8, kInv>(in, out, m, k, L, twstep, P.tw); break;
                default: stage_generic<kInv>(in, out, r, m, k, L, twstep, n, P.tw); break;
            }
        }
        __syncthreads();
        float2* t = src;
        src = dst;
        dst = t;
        L *= r;
    }
    return src;
}

// Addressing of a batch of vectors: vector v of image g starts at
// g * img_stride + v * vec_stride and steps elem_stride between elements.
struct VecGeom {
    int nvec;             // vectors per image
    long long vec_stride;
    long long elem_stride;
    long long img_stride;
};

__host__ __device__ __forceinline__ long long vec_addr(const VecGeom& g, int img, int v, int k) {
    return (long long)img * g.img_stride + (long long)v * g.vec_stride + (long long)k * g.elem_stride;
}

// Generic batched-FFT kernel.  Grid: (ceil(nvec / tile), n_images).  The IO
// functor provides load(img, v, k, addr) -> float2 and store(img, v, k, addr,
// value), plus finish(smem) called once by all threads at the end.
template <bool kInv, class IO>
__global__ void __launch_bounds__(256) fft_batched_kernel(FftDesc P, VecGeom g, int tile, IO io_param) {
    extern __shared__ float2 smem_fft[];
    IO io = io_param;  // per-thread copy: reducing IO functors keep state in it
    const int pitch = P.n + 1;
    float2* buf = smem_fft;
    float2* alt = smem_fft + (size_t)tile * pitch;
    const int img = blockIdx.y;
    const int v0 = blockIdx.x * tile;
    const int nv = min(tile, g.nvec - v0);
    const int n = P.n;
    const int tot = nv * n;
    const bool contiguous = g.elem_stride == 1;
    for (int i = threadIdx.x; i < tot; i += blockDim.x) {
        int t, k;
        if (contiguous) { t = i / n; k = i - t * n; }
        else { k = i / nv; t = i - k * nv; }
        buf[t * pitch + k] = io.load(img, v0 + t, k, vec_addr(g, img, v0 + t, k));
    }
    __syncthreads();
    float2* res = block_fft<kInv>(buf, alt, nv, pitch, P);
    for (int i = threadIdx.x; i < tot; i += blockDim.x) {
        int t, k;
        if (contiguous) { t = i / n; k = i - t * n; }
        else { k = i / nv; t = i - k * nv; }
        io.store(img, v0 + t, k, vec_addr(g, img, v0 + t, k), res[t * pitch + k]);
    }
    io.finish(reinterpret_cast<double*>(smem_fft + 2 * (size_t)tile * pitch), v0, nv);
}

// Shared memory of fft_batched_kernel: two ping-pong buffers of tile x (n+1)
// complex values, then kFftRedDoubles doubles of reduction scratch for finish().
constexpr int kFftRedDoubles = 128;
__host__ __device__ inline size_t fft_smem_bytes(int n, int tile) {
    return 2 * (size_t)tile * (n + 1) * sizeof(float2) + kFftRedDoubles * sizeof(double);
}

// ---- IO functors shared by several call sites ----

// In place complex, output scaled.
struct IoComplex {
    float2* data;
    float scale;
    __device__ float2 load(int, int, int, long long a) const { return data[a]; }
    __device__ void store(int, int, int, long long a, float2 v) const { data[a] = cscale(v, scale); }
    __device__ void finish(double*, int, int) const {}
};

// Real input (float) -> complex output, output scaled.
struct IoRealIn {
    const float* in;
    float2* out;
    float scale;
    __device__ float2 load(int, int, int, long long a) const { return make_float2(in[a], 0.0f); }
    __device__ void store(int, int, int, long long a, float2 v) const { out[a] = cscale(v, scale); }
    __device__ void finish(double*, int, int) const {}
};

// Complex input -> real part stored as float, scaled.
struct IoRealOut {
    const float2* in;
    float* out;
    float scale;
    __device__ float2 load(int, int, int, long long a) const { return in[a]; }
    __device__ void store(int, int, int, long long a, float2 v) const { out[a] = v.x * scale; }
    __device__ void finish(double*, int, int) const {}
};

// Complex input scaled per image on load (scale[img]), in place.
struct IoScaleIn {
    float2* data;
    const double* inv_scale;  // per image
    __device__ float2 load(int img, int, int, long long a) const {
        float s = (float)inv_scale[img];
        return cscale(data[a], s);
    }
    __device__ void store(int, int, int, long long a, float2 v) const { data[a] = v; }
    __device__ void finish(double*, int, int) const {}
};

}  // namespace gs
