// gs_correlate_window_noalloc: the correlation passes of one window without
// any device allocation.
//
// Who needs this: callers that cannot call cudaMalloc while they run, e.g.
// code inside a CUDA graph capture or an allocator-free real-time section of
// a larger pipeline, or a host that hands this library pre-allocated device
// buffers and forbids it to grow its footprint.  They keep their own input
// and output buffers; the library's intermediate maps, arg-max/sum
// accumulators and twiddle table live in one file-scope device array of fixed
// size that every GPU which loads this library holds until the process exits.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include <algorithm>
#include <map>
#include <mutex>
#include <type_traits>
#include <utility>

#include "gisspa.h"

// The kernel headers define non-template kernels too; this translation unit
// gets private copies (internal linkage) so that they do not clash with the
// library's main translation unit at link time.
namespace {
#include "fastfft.cuh"
}  // namespace

using namespace gs;

namespace {

// Fixed scratch: twiddles (first 64 KiB), accumulators (next 1 MiB), then the
// row-pass maps.  Shared by every call on a device and never cleared between
// calls except for what the call itself zeroes.
constexpr size_t kScratchBytes = GS_NOALLOC_SCRATCH_BYTES;
constexpr size_t kTwBytes = 64u << 10;
constexpr size_t kAccBytes = 1u << 20;
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

// Device addresses of the scratch array, one per CUDA context.  The module
// holding the array is loaded once per context, so a context created anew
// (e.g. the primary context after cudaDeviceReset) has a new address: the
// cache is keyed by the context's unique ID, not by the device ordinal.
std::map<unsigned long long, void*> g_scratch_addr;
std::mutex g_scratch_mu;

// Unique ID of the calling thread's current context (driver API, reached
// through the runtime so that the library needs no libcuda link), or 0 when
// no context is current or the driver cannot tell.
unsigned long long current_context_id() {
    using GetCurrent = int (*)(void**);
    using GetId = int (*)(void*, unsigned long long*);
    static GetCurrent get_current = nullptr;
    static GetId get_id = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_current = reinterpret_cast<GetCurrent>(f);
        f = nullptr;
        q = cudaDriverEntryPointSymbolNotFound;
        if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_id = reinterpret_cast<GetId>(f);
        cudaGetLastError();
    });
    void* ctx = nullptr;
    unsigned long long id = 0;
    if (!get_current || !get_id || get_current(&ctx) != 0 || !ctx || get_id(ctx, &id) != 0) return 0;
    return id;
}

// Device address of the scratch array in the current context.  The
// host-side name g_noalloc_scratch is only a stand-in symbol, so the address
// is looked up with cudaGetSymbolAddress once per context (the first call in
// a context; that lookup also makes the device's primary context current if
// no runtime call has yet in this thread).
int scratch_for_current_device(unsigned char** out) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        cudaGetLastError();
        return GS_ERR_CUDA;
    }
    std::lock_guard<std::mutex> lk(g_scratch_mu);
    unsigned long long id = current_context_id();
    auto it = id ? g_scratch_addr.find(id) : g_scratch_addr.end();
    if (it != g_scratch_addr.end()) {
        *out = static_cast<unsigned char*>(it->second);
        return GS_OK;
    }
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) {
        cudaGetLastError();
        return GS_ERR_CUDA;
    }
    if (!id) id = current_context_id();  // the lookup may have made the context current
    if (id) g_scratch_addr[id] = p;      // without an ID nothing is cached: looked up every call
    *out = static_cast<unsigned char*>(p);
    return GS_OK;
}

// tw[k] = exp(-2 pi i k / n) from double-precision sincospi.
__global__ void k_noalloc_twiddles(float2* tw, int n) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    double s, c;
    sincospi(-2.0 * (double)k / (double)n, &s, &c);
    tw[k] = make_float2((float)c, (float)s);
}

int factorize_noalloc(int n, int* radix) {
    int ns = 0, m = n;
    while (m % 8 == 0 && m > 1) { radix[ns++] = 8; m /= 8; }
    while (m % 4 == 0) { radix[ns++] = 4; m /= 4; }
    while (m % 2 == 0) { radix[ns++] = 2; m /= 2; }
    for (int f : {3, 5}) while (m % f == 0) { radix[ns++] = f; m /= f; }
    for (int f = 7; (long long)f * f <= m; f += 2)
        while (m % f == 0) { radix[ns++] = f; m /= f; }
    if (m > 1) radix[ns++] = m;
    return ns;
}

template <int N2, bool kInv, bool kCols, class IO>
cudaError_t launch_fast(const float2* tw, int nimg, IO io, cudaStream_t st) {
    using F = Fast16<N2>;
    auto kern = k_fft16<N2, kInv, kCols, IO>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)F::smem_bytes());
    if (e != cudaSuccess) return e;
    kern<<<dim3(N2, nimg), F::kThreads, F::smem_bytes(), st>>>(tw, io);
    return cudaGetLastError();
}

template <bool kInv, class IO>
cudaError_t launch_generic(const FftDesc& d, VecGeom g, int nimg, IO io, cudaStream_t st) {
    const size_t per = 2 * (size_t)(d.n + 1) * sizeof(float2);
    size_t tile = std::max<size_t>(1, (96u << 10) / per);
    tile = std::min<size_t>(tile, 16);
    tile = std::min<size_t>(tile, (size_t)g.nvec);
    const size_t smem = fft_smem_bytes(d.n, (int)tile);
    if (smem > (227u << 10)) return cudaErrorInvalidValue;
    auto kern = fft_batched_kernel<kInv, IO>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    kern<<<dim3((unsigned)((g.nvec + tile - 1) / tile), nimg), 256, smem, st>>>(d, g, (int)tile, io);
    return cudaGetLastError();
}

}  // namespace

extern "C" int gs_correlate_window_noalloc(const float* d_window_spectrum, const float* d_pair_spectra,
                                           int n_templates, int l, float d_m, gs_unit* d_units, void* stream) {
    if (!d_window_spectrum || !d_pair_spectra || !d_units || n_templates <= 0 || l < 2 || (l & 1) ||
        !(d_m > 0.0f))
        return GS_ERR_ARG;
    const size_t l2 = (size_t)l * l;
    if ((size_t)l * sizeof(float2) > kTwBytes || l2 * sizeof(float2) > kScratchBytes - kTwBytes - kAccBytes)
        return GS_ERR_UNSUPPORTED;  // beyond the fixed scratch: l <= GS_NOALLOC_MAX_WINDOW
    FftDesc desc{};
    desc.n = l;
    desc.nst = factorize_noalloc(l, desc.radix);
    if (desc.nst > kFftMaxStages) return GS_ERR_UNSUPPORTED;
    const int n2 = l / 16;
    const bool fast = (l % 16 == 0) && (n2 == 32 || n2 == 45 || n2 == 48);
    if (!fast && 2 * (size_t)(l + 1) * sizeof(float2) + kFftRedDoubles * sizeof(double) > (227u << 10))
        return GS_ERR_UNSUPPORTED;
    unsigned char* base = nullptr;
    int st = scratch_for_current_device(&base);
    if (st != GS_OK) return st;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    float2* tw = reinterpret_cast<float2*>(base);
    UnitAcc* acc = reinterpret_cast<UnitAcc*>(base + kTwBytes);
    float2* R = reinterpret_cast<float2*>(base + kTwBytes + kAccBytes);
    desc.tw = tw;
    const int npairs = (n_templates + 1) / 2;
    const size_t chunk_by_maps = (kScratchBytes - kTwBytes - kAccBytes) / (l2 * sizeof(float2));
    const size_t chunk_by_acc = kAccBytes / (2 * sizeof(UnitAcc));
    const int chunk = (int)std::min<size_t>(std::min(chunk_by_maps, chunk_by_acc), 65535);
    const float2* W = reinterpret_cast<const float2*>(d_window_spectrum);
    const float2* Pall = reinterpret_cast<const float2*>(d_pair_spectra);
    const float q_lo = d_m / 4.0f, q_hi = (float)l - q_lo;
    const float sgn = ((l / 2) % 2 == 0) ? 1.0f : -1.0f;

    k_noalloc_twiddles<<<(l + 255) / 256, 256, 0, s>>>(tw, l);
    if (cudaGetLastError() != cudaSuccess) return GS_ERR_CUDA;
    for (int p0 = 0; p0 < npairs; p0 += chunk) {
        const int np = std::min(chunk, npairs - p0);
        const int nt = std::min(n_templates - 2 * p0, 2 * np);
        const float2* P = Pall + (size_t)p0 * l2;
        // accumulators start at zero for every chunk
        if (cudaMemsetAsync(acc, 0, sizeof(UnitAcc) * 2 * (size_t)np, s) != cudaSuccess) return GS_ERR_CUDA;
        cudaError_t e;
        if (fast) {
            F16Pass1 io1{W, P, R, l, (long long)l2};
            F16Pass2 io2;
            io2.R = R; io2.acc = acc; io2.L = l; io2.ntmpl = nt; io2.L2 = (long long)l2;
            io2.q_lo = q_lo; io2.q_hi = q_hi; io2.sgn = sgn;
            switch (n2) {
                case 32: e = launch_fast<32, true, false>(tw, np, io1, s);
                         if (e == cudaSuccess) e = launch_fast<32, true, true>(tw, np, io2, s); break;
                case 45: e = launch_fast<45, true, false>(tw, np, io1, s);
                         if (e == cudaSuccess) e = launch_fast<45, true, true>(tw, np, io2, s); break;
                default: e = launch_fast<48, true, false>(tw, np, io1, s);
                         if (e == cudaSuccess) e = launch_fast<48, true, true>(tw, np, io2, s); break;
            }
        } else {
            const VecGeom rows{l, (long long)l, 1, (long long)l2};
            const VecGeom cols{l, 1, (long long)l, (long long)l2};
            IoPass1 io1{W, P, R, (long long)l2};
            IoPass2 io2;
            io2.R = R; io2.acc = acc; io2.l = l; io2.ntmpl = nt; io2.q_lo = q_lo; io2.q_hi = q_hi; io2.sgn = sgn;
            e = launch_generic<true>(desc, rows, np, io1, s);
            if (e == cudaSuccess) e = launch_generic<true>(desc, cols, np, io2, s);
        }
        if (e != cudaSuccess) return GS_ERR_CUDA;
        k_finalize<<<(nt + 127) / 128, 128, 0, s>>>(acc, nt, l, reinterpret_cast<UnitOut*>(d_units) + 2 * (size_t)p0);
        if (cudaGetLastError() != cudaSuccess) return GS_ERR_CUDA;
    }
    return GS_OK;
}
