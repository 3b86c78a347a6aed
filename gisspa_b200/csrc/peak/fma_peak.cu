// FP32 FMA throughput microbenchmark: the roofline denominator for the
// correlation kernels, which are bound by FP32 instruction issue.  Built as
// its own small library (gisspa_b200/lib/libgisspa_peak.so) for bench.py; it
// is measurement infrastructure, not part of the search's C ABI.
//
// Every thread runs kChains independent dependency chains of fma.rn.f32, so
// each SM sub-partition can issue one warp-wide FMA per clock once a few
// warps are resident; the result is written only when it equals a value it
// cannot take, which keeps the chains alive without memory traffic.
#include <cuda_runtime.h>

namespace {

constexpr int kChains = 8;
constexpr int kUnroll = 16;
constexpr int kThreads = 256;

__global__ void __launch_bounds__(kThreads) k_fma_peak(float* sink, int iters, float seed) {
    float a[kChains];
#pragma unroll
    for (int c = 0; c < kChains; ++c) a[c] = seed + 1e-3f * (float)(threadIdx.x + c);
    const float m = 0.999999f, d = 1e-7f;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int u = 0; u < kUnroll; ++u) {
#pragma unroll
            for (int c = 0; c < kChains; ++c) asm volatile("fma.rn.f32 %0, %0, %1, %2;" : "+f"(a[c]) : "f"(m), "f"(d));
        }
    }
    float s = 0.0f;
#pragma unroll
    for (int c = 0; c < kChains; ++c) s += a[c];
    if (s == -12345.0f) sink[blockIdx.x * kThreads + threadIdx.x] = s;
}

}  // namespace

extern "C" {

// Runs blocks_per_sm x SM-count CTAs of 256 threads, each thread doing
// iters x 16 x 8 FMAs, `repeats` times after one warm-up launch; returns the
// best launch's time (ms) and its FP32 FLOP count (2 per FMA).  0 = ok, else a
// cudaError_t value.
int gs_peak_fp32_fma(int device, int iters, int blocks_per_sm, int repeats, double* best_ms, double* flops) {
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) return (int)e;
    int sms = 0;
    if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device)) != cudaSuccess) return (int)e;
    const int blocks = sms * blocks_per_sm;
    float* sink = nullptr;
    if ((e = cudaMalloc(&sink, sizeof(float) * (size_t)blocks * kThreads)) != cudaSuccess) return (int)e;
    cudaEvent_t t0, t1;
    cudaEventCreate(&t0);
    cudaEventCreate(&t1);
    float best = 1e30f;
    for (int r = 0; r <= repeats; ++r) {
        cudaEventRecord(t0);
        k_fma_peak<<<blocks, kThreads>>>(sink, iters, 1.0f);
        cudaEventRecord(t1);
        if ((e = cudaEventSynchronize(t1)) != cudaSuccess) break;
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, t0, t1);
        if (r > 0 && ms < best) best = ms;  // launch 0 is the warm-up
    }
    if (e == cudaSuccess) e = cudaGetLastError();
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    cudaFree(sink);
    if (e != cudaSuccess) return (int)e;
    *best_ms = best;
    *flops = 2.0 * (double)blocks * kThreads * (double)iters * kUnroll * kChains;
    return 0;
}

}  // extern "C"
