// Per-pixel maximum of the normalised correlation over (template, angle):
// the map behind gs_get_pixel_max.  No reference counterpart (the
// reference keeps one peak per map, main.cu:856-891); its values are the
// search's own normalisation, cc / sigma with sigma the map's standard
// deviation without its peak (main.cu:869-876), so at a map's peak pixel the
// value is that unit's score.
//
// Only units whose score reaches the threshold are recomputed: a unit's
// score is the maximum of cc / sigma over the pixels the map looks at (or 0),
// so no pixel of a unit below the threshold can reach it.  Their maps are
// rebuilt with the two-pass kernels (row pass of the selected template pairs,
// then the column pass with the epilogue below), and every pixel at or above
// the threshold is merged into a micrograph-sized array of order-preserving
// 64-bit keys (value bits high, ~(angle * ntmpl + template) low: among equal
// values the smallest (angle, template) wins) by atomicMax.
#pragma once

#include "fastfft.cuh"
#include "kernels.cuh"
#include "norm1.cuh"

namespace gs {

// Row pass of selected pairs (l = 16 N2 kernels): image q is pair pairs[q];
// its row map goes to scratch slot q.
struct F16Pass1Sel {
    const float2* W;
    const float2* P;
    float2* R;
    const int* pairs;
    int L;
    long long L2;
    __device__ float2 load(int img, int v, int k) const {
        const long long off = (long long)v * L + k;
        return cmulc(__ldg(W + off), __ldcs(P + (long long)__ldg(pairs + img) * L2 + off));
    }
    __device__ void store(int img, int v, int k, float2 x) const {
        __stcg(R + (long long)img * L2 + (long long)v * L + k, x);
    }
    __device__ void finish(double*) const {}
};

// The same for the generic mixed-radix kernel (element address a is
// img * l^2 + offset).
struct IoPass1Sel {
    const float2* W;
    const float2* P;
    float2* R;
    const int* pairs;
    long long l2;
    __device__ float2 load(int img, int, int, long long a) const {
        const long long off = a - (long long)img * l2;
        return cmulc(__ldg(W + off), P[(long long)__ldg(pairs + img) * l2 + off]);
    }
    __device__ void store(int, int, int, long long a, float2 v) const { R[a] = v; }
    __device__ void finish(double*, int, int) const {}
};

// Column-pass epilogue: value (x, y) of the map of scratch slot `img` (pair
// pairs[img], real part template 2p, imaginary part 2p + 1).
struct PixelMaxEpi {
    unsigned long long* keys;  // micrograph, ny x nx
    const UnitOut* out;        // this (angle, window): ntmpl results of the search
    const int* pairs;
    int L, ntmpl, nx, offx, offy;
    unsigned int idx0;         // angle index * ntmpl
    float q_lo, q_hi, thres, sgn;
    __device__ __forceinline__ void put(int img, int x, int y, float2 val) const {
        const int h = L >> 1;
        int X = x + h; if (X >= L) X -= L;
        int Y = y + h; if (Y >= L) Y -= L;
        // the border the score's maximum leaves out (GPU_func.cu:681)
        if ((float)X < q_lo || (float)X > q_hi || (float)Y < q_lo || (float)Y > q_hi) return;
        const int pair = __ldg(pairs + img);
        for (int q = 0; q < 2; ++q) {
            const int J = 2 * pair + q;
            if (J >= ntmpl) break;
            const float sd = __ldg(&out[J].sigma), sc = __ldg(&out[J].score);
            if (!(sc >= thres) || !(sd > 0.0f)) continue;
            const float z = (sgn * (q ? val.y : val.x)) / sd;
            if (!(z >= thres)) continue;
            const unsigned long long key =
                ((unsigned long long)float_order(z) << 32) | (unsigned int)(~(idx0 + (unsigned int)J));
            atomicMax(keys + (long long)(offy + Y) * nx + offx + X, key);
        }
    }
};

}  // namespace gs
