// Shared device/host helpers for the GisSPA B200 kernels.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <math.h>

namespace gs {

// The reference's PI literal (GPU_func.cuh:29); every angle and CTF phase
// in the reference is formed with it, so the kernels use it too.
constexpr double kPiRef = 3.141592654;

__host__ __device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__host__ __device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__host__ __device__ __forceinline__ float2 cscale(float2 a, float s) { return make_float2(a.x * s, a.y * s); }
__host__ __device__ __forceinline__ float2 cmul(float2 a, float2 b) {
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// a * conj(b)
__host__ __device__ __forceinline__ float2 cmulc(float2 a, float2 b) {
    return make_float2(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}
// multiply by -i (kInv=false) or +i (kInv=true)
template <bool kInv>
__host__ __device__ __forceinline__ float2 mul_mi(float2 a) {
    return kInv ? make_float2(-a.y, a.x) : make_float2(a.y, -a.x);
}

// Radial shell index of the reference's whitening / band-pass code
// (GPU_func.cu:119,138,167,268-269): floor(hypotf(dy, dx) + 0.5) - 1 with
// dx = min(x, nx-x), dy = min(y, ny-y).
__device__ __forceinline__ int shell_index(int x, int y, int nx, int ny, float* rf_out = nullptr) {
    const float rf = hypotf((float)min(y, ny - y), (float)min(x, nx - x));
    if (rf_out) *rf_out = rf;
    return (int)floor((double)rf + 0.5) - 1;
}

// Order-preserving key for a (value, flat index) arg-max over values > 0:
// high word = float bits (monotone for positive floats), low word = ~index so
// that equal values resolve to the smallest index.  Key 0 = "no positive value".
__device__ __forceinline__ unsigned long long argmax_key(float v, int idx) {
    if (!(v > 0.0f)) return 0ull;
    return ((unsigned long long)__float_as_uint(v) << 32) | (unsigned long long)(~(unsigned)idx);
}
__host__ __device__ __forceinline__ float key_value(unsigned long long k) {
#ifdef __CUDA_ARCH__
    return k ? __uint_as_float((unsigned)(k >> 32)) : 0.0f;
#else
    unsigned u = (unsigned)(k >> 32);
    float f;
    memcpy(&f, &u, 4);
    return k ? f : 0.0f;
#endif
}
__host__ __device__ __forceinline__ int key_index(unsigned long long k) {
    return k ? (int)(~(unsigned)(k & 0xffffffffull)) : 0;
}

template <class T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ unsigned long long warp_max_u64(unsigned long long v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        unsigned long long w = __shfl_xor_sync(0xffffffffu, v, o);
        v = w > v ? w : v;
    }
    return v;
}

// Block-wide sum of NV doubles; every thread gets the totals.  `scratch`
// needs NV * 32 doubles of shared memory.  Must be called by all threads.
template <int NV>
__device__ __forceinline__ void block_sum(double (&v)[NV], double* scratch) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int nw = (blockDim.x + 31) >> 5;
#pragma unroll
    for (int k = 0; k < NV; ++k) v[k] = warp_sum(v[k]);
    __syncthreads();
    if (lane == 0) {
#pragma unroll
        for (int k = 0; k < NV; ++k) scratch[k * 32 + warp] = v[k];
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < NV; ++k) {
        double t = lane < nw ? scratch[k * 32 + lane] : 0.0;
        v[k] = warp_sum(t);
    }
    __syncthreads();
}

// CTF parameters of one micrograph, in the reference's units
// (struct Parameters fields lambda, dfu, dfv, dfdiff, dfang, ...).
struct CtfDev {
    float apix, dfu, dfv, dfdiff, dfang, lambda, cs, ampconst;
};

// Astigmatic CTF at integer FFT index (x1, y1) of an nx x ny spectrum whose y
// index has been shifted by ny/2, as the reference's CTF model takes it
// (GPU_func.cu:292-315).  mode 0: sign (+1/-1), 2: |CTF|, else the value.
__device__ __forceinline__ float ctf_ast(int x1, int y1, int nx, int ny, const CtfDev& c, int mode) {
    y1 = x1 > nx / 2 ? ny - y1 : y1;
    x1 = min(x1, nx - x1);
    const float dx = (float)x1;
    const float dy = (float)(y1 - ny / 2);
    const float ss = (dx * dx / (float)(nx * nx) + dy * dy / (float)(ny * ny)) / (c.apix * c.apix);
    const float ag = atan2f(dy, dx);
    const float df_ast = 0.5f * (c.dfu + c.dfv +
                                 2.0f * c.dfdiff * cosf((float)(2.0 * ((double)c.dfang * kPiRef / 180.0 - (double)ag))));
    const double lam = (double)c.lambda;
    const float gamma = (float)(-2.0 * kPiRef *
                                ((double)c.cs * 2.5e6 * lam * lam * lam * (double)ss * (double)ss +
                                 (double)df_ast * 5000.0 * lam * (double)ss));
    const float v = sqrtf(1.0f - c.ampconst * c.ampconst) * sinf(gamma) + c.ampconst * cosf(gamma);
    if (mode == 0) return v > 0.0f ? 1.0f : -1.0f;
    if (mode == 2) return fabsf(v);
    return v;
}

// Band-pass factor on shell index r with 8-px cosine edges (hp = l*apix/highres,
// lp = l*apix/lowres, both formed in float).  Template form has no low cut
// (GPU_func.cu:270-278); micrograph form passes only lp <= r < hp
// (GPU_func.cu:183-191).
template <bool kLowCut>
__device__ __forceinline__ float bandpass(int r, float hp, float lp) {
    const float rf = (float)r;
    const bool pass = kLowCut ? (rf < hp && rf >= lp) : (rf < hp && r >= 0);
    if (pass) return 1.0f;
    if (rf >= hp && rf < hp + 8.0f) return 0.5f * cosf((float)(kPiRef * (double)(rf - hp) / 16.0)) + 0.5f;
    if (rf >= lp - 8.0f && rf < lp && r >= 0) return 0.5f * cosf((float)(kPiRef * (double)(lp - rf) / 16.0)) + 0.5f;
    return 0.0f;
}

}  // namespace gs
