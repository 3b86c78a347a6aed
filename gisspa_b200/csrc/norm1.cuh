// norm_type 1: correlation values z-scored per window pixel over all
// templates and angles (reference main.cu:718-821, 1170-1229;
// GPU_func.cu:617-662, 711-745).
//
// Sweep 1 accumulates, per window pixel, sum and sum of squares of cc / l^2
// over every template and angle (column-pass epilogue, float atomics like
// the reference's float CCG_sum).  k_norm1_moments turns them into mean and
// standard deviation.  Sweep 2 recomputes every map, z-scores each value and
// reduces every 1024-element block of the flat map to its maximum and
// position (no border mask), as an order-preserving 64-bit key per
// (template, block); k_norm1_compact writes the threshold picks.
#pragma once

#include "fastfft.cuh"
#include "kernels.cuh"

namespace gs {

// Order-preserving map of any finite float to uint32 (negative values too).
__device__ __forceinline__ unsigned int float_order(float v) {
    const unsigned int u = __float_as_uint(v);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__host__ __device__ __forceinline__ float float_unorder(unsigned int m) {
    const unsigned int u = (m & 0x80000000u) ? (m & 0x7fffffffu) : ~m;
#ifdef __CUDA_ARCH__
    return __uint_as_float(u);
#else
    float f;
    memcpy(&f, &u, 4);
    return f;
#endif
}

struct Norm1Stats {
    float* s1;  // this window, l^2
    float* s2;
    int L, ntmpl;
    float l2f, sgn;
    __device__ __forceinline__ void put(int img, int x, int y, float2 val) const {
        const int h = L >> 1;
        int X = x + h; if (X >= L) X -= L;
        int Y = y + h; if (Y >= L) Y -= L;
        const int pos = Y * L + X;
        const float c1 = (sgn * val.x) / l2f;   // add_CCG_to_sum: cc / l^2
        float a = c1, b = c1 * c1;
        if (2 * img + 1 < ntmpl) {
            const float c2 = (sgn * val.y) / l2f;
            a += c2;
            b += c2 * c2;
        }
        atomicAdd(s1 + pos, a);
        atomicAdd(s2 + pos, b);
    }
};

struct Norm1Blocks {
    const float* avg;  // this window, l^2
    const float* sd;
    unsigned long long* keys;  // this window: ntmpl x nblk
    int L, ntmpl, nblk;
    float lf, sgn;
    __device__ __forceinline__ void put(int img, int x, int y, float2 val) const {
        const int h = L >> 1;
        int X = x + h; if (X >= L) X -= L;
        int Y = y + h; if (Y >= L) Y -= L;
        const int pos = Y * L + X;
        const float m = avg[pos], s = sd[pos];
        for (int q = 0; q < 2; ++q) {
            const int J = 2 * img + q;
            if (J >= ntmpl) break;
            const float cur = ((sgn * (q ? val.y : val.x)) / lf) / lf;  // update_CCG: cc / l / l
            const float z = s > 0.0f ? (cur - m) / s : 0.0f;
            const unsigned long long key = ((unsigned long long)float_order(z) << 32) | (unsigned)(~pos);
            atomicMax(keys + (long long)J * nblk + (pos >> 10), key);
        }
    }
};

// Column-pass IO of the generic kernel (fft_batched_kernel): vector = map
// column x, element = map row y.
template <class Epi>
struct IoNorm1 {
    const float2* R;
    Epi epi;
    __device__ float2 load(int, int, int, long long a) const { return R[a]; }
    __device__ void store(int img, int v, int k, long long, float2 val) const { epi.put(img, v, k, val); }
    __device__ void finish(double*, int, int) const {}
};

// Column-pass IO of the l = 16 N2 kernels.
template <class Epi>
struct F16Norm1 {
    const float2* R;
    Epi epi;
    int L;
    long long L2;
    __device__ float2 load(int img, int v, int k) const { return R[(long long)img * L2 + (long long)k * L + v]; }
    __device__ void store(int img, int v, int k, float2 val) const { epi.put(img, v, k, val); }
    __device__ void finish(double*) const {}
};

// mean and standard deviation per pixel from the sums (set_CCG_mean,
// GPU_func.cu:635-646), in place, float like the reference.
__global__ void k_norm1_moments(float* s1, float* s2, long long n, float total) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float avg = s1[i] / total;
    const float var = sqrtf(s2[i] / total - avg * avg);
    s1[i] = avg;
    s2[i] = var;
}

struct BlockPickDev {
    long long key;  // ((angle * nw + window) * ntmpl + template) * nblk + block
    float cx, cy, score;
    int pad;
};

// Threshold + centre test of every (template, block) of one window
// (main.cu:800-817).
__global__ void k_norm1_compact(const unsigned long long* __restrict__ keys, int ntmpl, int nblk, int L,
                                int offx, int offy, float d_m, int nx, int ny, float thres, long long key0,
                                BlockPickDev* __restrict__ picks, unsigned long long* __restrict__ count,
                                long long cap) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)ntmpl * nblk) return;
    const unsigned long long k = keys[t];
    if (!k) return;
    const float z = float_unorder((unsigned)(k >> 32));
    if (!(z >= thres)) return;
    const int pos = (int)(~(unsigned)(k & 0xffffffffull));
    const float cx = (float)(offx + pos % L), cy = (float)(offy + pos / L);
    if (cx >= d_m && cx < (float)nx - d_m && cy >= d_m && cy < (float)ny - d_m) {
        const unsigned long long slot = atomicAdd(count, 1ull);
        if ((long long)slot < cap) {
            BlockPickDev pk;
            pk.key = key0 + t;
            pk.cx = cx;
            pk.cy = cy;
            pk.score = z;
            pk.pad = 0;
            picks[slot] = pk;
        }
    }
}

}  // namespace gs
