// Device check of the tcgen05 building blocks (gisspa_b200/csrc/tc.cuh):
// one CTA computes D = A B^T (M x N, K deep) from f32 inputs split into
// 16-bit (hi, lo) parts, accumulating in TMEM, and the result is compared
// with a double-precision product on the host.  Both 16-bit formats, with the
// single hi*hi product and with the three-product split (hi*hi + lo*hi +
// hi*lo).  Built for sm_100a and run on a B200 by tests/test_gpu_tc.py.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <random>
#include <vector>

#include "tc.cuh"

using namespace gs;

template <int M, int N, int K, bool kBf16>
__global__ void __launch_bounds__(128) k_gemm(const float* __restrict__ A, const float* __restrict__ B,
                                              float* __restrict__ D, int nprod, int* __restrict__ err) {
    extern __shared__ __align__(128) unsigned char sm[];
    unsigned char* a_hi = sm;
    unsigned char* a_lo = a_hi + M * K * 2;
    unsigned char* b_hi = a_lo + M * K * 2;
    unsigned char* b_lo = b_hi + N * K * 2;
    uint64_t* bar = reinterpret_cast<uint64_t*>(b_lo + N * K * 2);
    uint32_t* slot = reinterpret_cast<uint32_t*>(bar + 1);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

    for (int i = tid; i < M * K / 2; i += blockDim.x) {
        const int r = (2 * i) / K, k = (2 * i) % K;
        uint32_t hi, lo;
        tc::Split<kBf16>::run(A[r * K + k], A[r * K + k + 1], hi, lo);
        *reinterpret_cast<uint32_t*>(a_hi + tc::kmajor_off(r, k, M)) = hi;
        *reinterpret_cast<uint32_t*>(a_lo + tc::kmajor_off(r, k, M)) = lo;
    }
    for (int i = tid; i < N * K / 2; i += blockDim.x) {
        const int r = (2 * i) / K, k = (2 * i) % K;
        uint32_t hi, lo;
        tc::Split<kBf16>::run(B[r * K + k], B[r * K + k + 1], hi, lo);
        *reinterpret_cast<uint32_t*>(b_hi + tc::kmajor_off(r, k, N)) = hi;
        *reinterpret_cast<uint32_t*>(b_lo + tc::kmajor_off(r, k, N)) = lo;
    }
    tc::fence_async_smem();
    if (warp == 0) {
        tc::tmem_alloc(slot, 128);
        tc::tmem_relinquish();
    }
    if (tid == 0) {
        tc::mbar_init(bar, 1);
        tc::fence_mbar_init();
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tbase = *slot;
    if (tid == 0) {
        constexpr uint32_t idesc = tc::idesc_f16(M, N, kBf16 ? 1 : 0);
        const unsigned char* as[3] = {a_hi, a_lo, a_hi};
        const unsigned char* bs[3] = {b_hi, b_hi, b_lo};
        uint32_t acc = 0;
        for (int j = 0; j < K / 16; ++j)
            for (int p = 0; p < nprod; ++p) {
                const uint64_t ad = tc::smem_desc(tc::smem_u32(as[p]) + 2 * j * M * 16, M * 16, 128);
                const uint64_t bd = tc::smem_desc(tc::smem_u32(bs[p]) + 2 * j * N * 16, N * 16, 128);
                tc::mma_f16(tbase, ad, bd, idesc, acc);
                acc = 1;
            }
        tc::mma_commit(bar);
    }
    __syncwarp();
    const bool ok = tc::mbar_wait(bar, 0, 1u << 22);
    tc::fence_after_sync();
    if (!ok && lane == 0) atomicExch(err, 1);
    for (int c0 = 0; c0 < N; c0 += 16) {
        float v[16];
        tc::tmem_ld16(tbase + ((uint32_t)(32 * warp) << 16) + (uint32_t)c0, v);
        tc::tmem_ld_wait();
        for (int i = 0; i < 16; ++i) D[(32 * warp + lane) * N + c0 + i] = v[i];
    }
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0) tc::tmem_dealloc(tbase, 128);
}

// A in MN-major layout (element (m, k) at mnmajor_off(m, k, SBO_A, 128): the
// layout a column tile's map rows land in) and / or a taller K-major A of
// MT x 128 rows addressed tile by tile (LBO = MT * 128 * 16), one fp16
// product per K step, or two with B split into (hi, lo).  D tile t holds rows
// 128 t .. 128 t + 127 at TMEM columns t N .. t N + N - 1.
template <int MT, int N, int K, bool kAmn>
__global__ void __launch_bounds__(128) k_gemm_layouts(const float* __restrict__ A, const float* __restrict__ B,
                                                      float* __restrict__ D, int nprod, int* __restrict__ err) {
    constexpr int M = 128 * MT;
    constexpr uint32_t SBO_A = K * 16;  // MN-major: one 8-column group holds all K rows
    extern __shared__ __align__(128) unsigned char sm[];
    unsigned char* a = sm;
    unsigned char* b_hi = a + M * K * 2;
    unsigned char* b_lo = b_hi + N * K * 2;
    uint64_t* bar = reinterpret_cast<uint64_t*>(b_lo + N * K * 2);
    uint32_t* slot = reinterpret_cast<uint32_t*>(bar + 1);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    for (int i = tid; i < M * K; i += blockDim.x) {
        const int r = i / K, k = i % K;
        const uint32_t off = kAmn ? tc::mnmajor_off(r, k, SBO_A, 128) : tc::kmajor_off(r, k, M);
        *reinterpret_cast<__half*>(a + off) = __float2half_rn(A[r * K + k]);
    }
    for (int i = tid; i < N * K / 2; i += blockDim.x) {
        const int r = (2 * i) / K, k = (2 * i) % K;
        uint32_t hi, lo;
        tc::Split<false>::run(B[r * K + k], B[r * K + k + 1], hi, lo);
        *reinterpret_cast<uint32_t*>(b_hi + tc::kmajor_off(r, k, N)) = hi;
        *reinterpret_cast<uint32_t*>(b_lo + tc::kmajor_off(r, k, N)) = lo;
    }
    tc::fence_async_smem();
    if (warp == 0) {
        tc::tmem_alloc(slot, 256);
        tc::tmem_relinquish();
    }
    if (tid == 0) {
        tc::mbar_init(bar, 1);
        tc::fence_mbar_init();
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tbase = *slot;
    if (tid == 0) {
        constexpr uint32_t idesc = tc::idesc_f16_major(128, N, 0, kAmn ? 1 : 0, 0);
        for (int t = 0; t < MT; ++t) {
            uint32_t acc = 0;
            for (int j = 0; j < K / 16; ++j)
                for (int p = 0; p < nprod; ++p) {
                    const uint64_t ad = kAmn ? tc::smem_desc(tc::smem_u32(a) + 2 * j * 128, 128, SBO_A)
                                             : tc::smem_desc(tc::smem_u32(a) + t * 2048 + 2 * j * M * 16, M * 16, 128);
                    const uint64_t bd = tc::smem_desc(tc::smem_u32(p ? b_lo : b_hi) + 2 * j * N * 16, N * 16, 128);
                    tc::mma_f16(tbase + t * N, ad, bd, idesc, acc);
                    acc = 1;
                }
        }
        tc::mma_commit(bar);
    }
    __syncwarp();
    const bool ok = tc::mbar_wait(bar, 0, 1u << 22);
    tc::fence_after_sync();
    if (!ok && lane == 0) atomicExch(err, 1);
    for (int t = 0; t < MT; ++t)
        for (int c0 = 0; c0 < N; c0 += 16) {
            float v[16];
            tc::tmem_ld16(tbase + ((uint32_t)(32 * warp) << 16) + (uint32_t)(t * N + c0), v);
            tc::tmem_ld_wait();
            for (int i = 0; i < 16; ++i) D[(128 * t + 32 * warp + lane) * N + c0 + i] = v[i];
        }
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0) tc::tmem_dealloc(tbase, 256);
}

#define CK(x)                                                                        \
    do {                                                                             \
        cudaError_t e_ = (x);                                                        \
        if (e_ != cudaSuccess) {                                                     \
            printf("CUDA error %s at %s:%d\n", cudaGetErrorString(e_), __FILE__, __LINE__); \
            return 2;                                                                \
        }                                                                            \
    } while (0)

template <bool kBf16>
static int run(int nprod, double tol, const char* name) {
    constexpr int M = 128, N = 96, K = 96;
    std::mt19937 rng(7 + nprod + (kBf16 ? 100 : 0));
    std::normal_distribution<float> nd;
    std::vector<float> A(M * K), B(N * K), D(M * N);
    for (auto& x : A) x = nd(rng);
    for (auto& x : B) x = nd(rng);
    float *dA, *dB, *dD;
    int* dErr;
    CK(cudaMalloc(&dA, A.size() * 4));
    CK(cudaMalloc(&dB, B.size() * 4));
    CK(cudaMalloc(&dD, D.size() * 4));
    CK(cudaMalloc(&dErr, 4));
    CK(cudaMemcpy(dA, A.data(), A.size() * 4, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(dB, B.data(), B.size() * 4, cudaMemcpyHostToDevice));
    CK(cudaMemset(dErr, 0, 4));
    CK(cudaMemset(dD, 0, D.size() * 4));
    const size_t smem = 2 * (M + N) * K * 2 + 16;
    auto kern = k_gemm<M, N, K, kBf16>;
    CK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    kern<<<1, 128, smem>>>(dA, dB, dD, nprod, dErr);
    CK(cudaGetLastError());
    CK(cudaDeviceSynchronize());
    int err = 0;
    CK(cudaMemcpy(&err, dErr, 4, cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(D.data(), dD, D.size() * 4, cudaMemcpyDeviceToHost));
    cudaFree(dA);
    cudaFree(dB);
    cudaFree(dD);
    cudaFree(dErr);
    if (err) {
        printf("%s: mbarrier wait gave up\n", name);
        return 1;
    }
    double emax = 0, ref = 0;
    for (int m = 0; m < M; ++m)
        for (int n = 0; n < N; ++n) {
            double s = 0;
            for (int k = 0; k < K; ++k) s += (double)A[m * K + k] * (double)B[n * K + k];
            emax = fmax(emax, fabs(s - D[m * N + n]));
            ref = fmax(ref, fabs(s));
        }
    printf("%s: nprod=%d max abs err %.3e (max |D| %.3e, rel %.3e, tol %.1e)\n", name, nprod, emax, ref,
           emax / ref, tol);
    return emax / ref <= tol ? 0 : 1;
}

template <int MT, int N, int K, bool kAmn>
static int run_layout(int nprod, double tol, const char* name) {
    constexpr int M = 128 * MT;
    std::mt19937 rng(11 + nprod + MT);
    std::normal_distribution<float> nd;
    std::vector<float> A(M * K), B(N * K), D(M * N);
    for (auto& x : A) x = (float)__half2float(__float2half_rn(nd(rng)));  // exactly representable in fp16
    for (auto& x : B) x = nd(rng);
    float *dA, *dB, *dD;
    int* dErr;
    CK(cudaMalloc(&dA, A.size() * 4));
    CK(cudaMalloc(&dB, B.size() * 4));
    CK(cudaMalloc(&dD, D.size() * 4));
    CK(cudaMalloc(&dErr, 4));
    CK(cudaMemcpy(dA, A.data(), A.size() * 4, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(dB, B.data(), B.size() * 4, cudaMemcpyHostToDevice));
    CK(cudaMemset(dErr, 0, 4));
    CK(cudaMemset(dD, 0, D.size() * 4));
    const size_t smem = (size_t)M * K * 2 + 2 * (size_t)N * K * 2 + 16;
    auto kern = k_gemm_layouts<MT, N, K, kAmn>;
    CK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    kern<<<1, 128, smem>>>(dA, dB, dD, nprod, dErr);
    CK(cudaGetLastError());
    CK(cudaDeviceSynchronize());
    int err = 0;
    CK(cudaMemcpy(&err, dErr, 4, cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(D.data(), dD, D.size() * 4, cudaMemcpyDeviceToHost));
    cudaFree(dA);
    cudaFree(dB);
    cudaFree(dD);
    cudaFree(dErr);
    if (err) {
        printf("%s: mbarrier wait gave up\n", name);
        return 1;
    }
    double emax = 0, ref = 0;
    for (int m = 0; m < M; ++m)
        for (int n = 0; n < N; ++n) {
            double s = 0;
            for (int k = 0; k < K; ++k) s += (double)A[m * K + k] * (double)B[n * K + k];
            emax = fmax(emax, fabs(s - D[m * N + n]));
            ref = fmax(ref, fabs(s));
        }
    printf("%s: nprod=%d max abs err %.3e (max |D| %.3e, rel %.3e, tol %.1e)\n", name, nprod, emax, ref,
           emax / ref, tol);
    return emax / ref <= tol ? 0 : 1;
}

int main() {
    int bad = 0;
    bad |= run<true>(1, 1e-2, "bf16");   // one product: about 2^-8 relative per operand
    bad |= run<true>(3, 1e-4, "bf16");   // hi/lo split: about 2^-16
    bad |= run<false>(1, 2e-3, "fp16");
    bad |= run<false>(3, 1e-5, "fp16");
    // operand A exact in fp16: one product leaves only B's rounding (2^-12),
    // B split into (hi, lo) leaves about 2^-22
    bad |= run_layout<1, 96, 96, true>(1, 2e-3, "fp16 A MN-major, M 128 N 96 K 96");
    bad |= run_layout<1, 96, 96, true>(2, 1e-5, "fp16 A MN-major, M 128 N 96 K 96");
    bad |= run_layout<3, 32, 32, false>(1, 2e-3, "fp16 A K-major 384 rows as 3 M-tiles, N 32 K 32");
    bad |= run_layout<3, 32, 32, false>(2, 1e-5, "fp16 A K-major 384 rows as 3 M-tiles, N 32 K 32");
    printf(bad ? "FAILED\n" : "OK\n");
    return bad;
}
