// C-ABI implementation of the GisSPA B200 search (include/gisspa.h).
//
// Host orchestration of the kernels in kernels.cuh / fft.cuh.  One context
// = one device + one stream + the device buffers of the run.  The flow of a
// search follows the reference's main.cu:1149-1269 for norm_type 0:
// micrograph preprocessing, window spectra, then for every in-plane angle the
// template-pair spectra and, for every window, the fused correlation passes.
#include "gisspa.h"
#include "corr.cuh"
#include "fastfft.cuh"
#include "kernels.cuh"
#include "norm1.cuh"
#include "pixmax.cuh"
#include "tccorr.cuh"
#include "tccorr2.cuh"
#include "refine.cuh"

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <string>
#include <vector>

using namespace gs;

namespace {

struct FftPlan {
    FftDesc d;
    float2* tw = nullptr;
};

struct DBuf {
    void* p = nullptr;
    size_t cap = 0;
};

}  // namespace

struct CorrTuningSaved {
    int slots, lag, window_block, ctas, tile;
};

namespace {

}  // namespace

struct gs_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaStream_t side = nullptr;    // second stream: pair spectra while micrographs are prepared
    cudaEvent_t side_ev[2] = {nullptr, nullptr};  // search start on `stream`; pair spectra done on `side`
    std::string err;
    std::map<int, FftPlan> plans;
    // templates
    bool have_tmpl = false;
    gs_params p{};
    gs_ctf ctf0{};
    int l = 0, ntmpl = 0, tx = 0, ty = 0;
    DBuf tmpl;  // ntmpl x l x l float (real templates after preprocessing)
    DBuf tbase; // ntmpl x l x l float (whitened templates before the CTF weight)
    // per-search buffers
    DBuf in, q, cimg, img, stats, ra, rb, off, win, wsum, winv;
    DBuf tspec, scratch, pstats, coef, acc, units, picks, count;
    // last search
    int last_na = 0, last_nw = 0, last_nt = 0;
    bool have_units = false;
    struct MicGeom {
        int nx, ny, w0;
        std::vector<int> offx, offy;
    };
    std::vector<MicGeom> last_mics;  // micrographs of the last norm_type 0 search
    DBuf pix_keys, pix_pairs, pix_R;  // gs_get_pixel_max buffers
    float timings[GS_TIMING_COUNT] = {0, 0, 0, 0, 0, 0, 0, 0};
    bool kernel_timing = false;
    bool generic_fft = false;
    bool two_pass = false;
    int window_block = 4;
    int corr_slots = 16, corr_lag = 6;
    bool corr_ring_set = false;        // slots / lag set through gs_set_option
    bool window_block_set = false;     // window block set through gs_set_option
    bool corr_tile_set = false;        // tile width set through gs_set_option
    int corr_ctas = 0;                 // resident CTAs per SM of the persistent kernels (0 = as many as fit)
    int corr_tile = 16;                // vectors per tile of the FP32 persistent kernel (16 or 8)
    int corr_ctas_override = 0;        // value used by the launch in progress
    bool use_graph = false;            // capture the angle loop as one CUDA graph
    bool autotune = false;             // tune the persistent kernels' scheduling on first use
    std::map<long long, struct CorrTuningSaved> tuned;
    int angles_per_launch = 0;         // in-plane angles per persistent launch (0 = from the unit count)
    std::map<long long, int> tuned_angles;  // the autotuner's angles per launch, same key as `tuned`
    int last_tuning[6] = {0, 0, 0, 0, 0, 0};
    unsigned long long graph_kernel_launches = 0;
    DBuf unit_wp, dep_counters, pacc, flags;
    DBuf tc2_wmax, tc2_pmax;  // per window / per pair max |spectrum| (all-tensor-core path)
    DBuf tc2_w16, tc2_p16;    // their FP16 copies, scaled by powers of two
    DBuf rot_cs;              // (cos, sin) of every in-plane angle of the search
    // off-grid refinement (refine.cuh): per-pick chunk buffers
    DBuf rf_pk, rf_acc, rf_B, rf_F1, rf_T, rf_TM, rf_F, rf_G, rf_TB, rf_mask;
    std::vector<cudaEvent_t> kev;  // pool of events for per-kernel timing
    gs_stats counters{0, 0, 0};
};

namespace {

int set_err(gs_ctx* c, int code, const char* fmt, ...) {
    if (c) {
        char buf[512];
        va_list ap;
        va_start(ap, fmt);
        vsnprintf(buf, sizeof buf, fmt, ap);
        va_end(ap);
        c->err = buf;
    }
    return code;
}

#define CK(expr)                                                                                       \
    do {                                                                                               \
        cudaError_t e_ = (expr);                                                                       \
        if (e_ != cudaSuccess) return set_err(ctx, GS_ERR_CUDA, "%s: %s", #expr, cudaGetErrorString(e_)); \
    } while (0)
#define CKL() CK(cudaGetLastError())
#define TRY(...)                   \
    do {                           \
        int s_ = (__VA_ARGS__);    \
        if (s_ != GS_OK) return s_; \
    } while (0)

int ensure(gs_ctx* ctx, DBuf& b, size_t bytes) {
    if (bytes == 0) bytes = 16;
    if (b.cap >= bytes) return GS_OK;
    if (b.p) cudaFree(b.p);
    b.p = nullptr;
    b.cap = 0;
    cudaError_t e = cudaMalloc(&b.p, bytes);
    if (e != cudaSuccess) {
        cudaGetLastError();
        b.p = nullptr;
        return set_err(ctx, GS_ERR_OOM, "cudaMalloc(%zu bytes) failed: %s", bytes, cudaGetErrorString(e));
    }
    b.cap = bytes;
    return GS_OK;
}

template <class T>
T* P(DBuf& b) { return reinterpret_cast<T*>(b.p); }

void free_buf(DBuf& b) {
    if (b.p) cudaFree(b.p);
    b.p = nullptr;
    b.cap = 0;
}

// Radix order: 8s while they divide, then 4, 2, 3, 5, then any other prime.
int factorize(int n, int* radix) {
    int ns = 0;
    int m = n;
    while (m % 8 == 0 && m > 1) { radix[ns++] = 8; m /= 8; }
    while (m % 4 == 0) { radix[ns++] = 4; m /= 4; }
    while (m % 2 == 0) { radix[ns++] = 2; m /= 2; }
    for (int f : {3, 5}) while (m % f == 0) { radix[ns++] = f; m /= f; }
    for (int f = 7; (long long)f * f <= m; f += 2)
        while (m % f == 0) { radix[ns++] = f; m /= f; }
    if (m > 1) radix[ns++] = m;
    return ns;
}

int get_plan(gs_ctx* ctx, int n, FftPlan** out) {
    auto it = ctx->plans.find(n);
    if (it != ctx->plans.end()) {
        *out = &it->second;
        return GS_OK;
    }
    FftPlan pl;
    pl.d.n = n;
    pl.d.nst = factorize(n, pl.d.radix);
    if (pl.d.nst > kFftMaxStages) return set_err(ctx, GS_ERR_UNSUPPORTED, "FFT length %d has too many factors", n);
    for (int s = 0; s < pl.d.nst; ++s)
        if (pl.d.radix[s] > 4096) return set_err(ctx, GS_ERR_UNSUPPORTED, "FFT length %d has prime factor %d", n, pl.d.radix[s]);
    std::vector<float2> tw(n);
    for (int k = 0; k < n; ++k) {
        const double a = -2.0 * M_PI * (double)k / (double)n;
        tw[k] = make_float2((float)cos(a), (float)sin(a));
    }
    CK(cudaMalloc(&pl.tw, sizeof(float2) * n));
    CK(cudaMemcpy(pl.tw, tw.data(), sizeof(float2) * n, cudaMemcpyHostToDevice));
    pl.d.tw = pl.tw;
    auto res = ctx->plans.emplace(n, pl);
    *out = &res.first->second;
    return GS_OK;
}

constexpr int kFftThreads = 256;
constexpr size_t kFftSmemBudget = 96 * 1024;
constexpr size_t kMaxSmem = 227 * 1024;

template <bool kInv, class IO>
int run_fft(gs_ctx* ctx, int n, VecGeom g, int nimg, IO io, int max_tile = 16) {
    FftPlan* pl = nullptr;
    TRY(get_plan(ctx, n, &pl));
    const size_t per = 2 * (size_t)(n + 1) * sizeof(float2);
    size_t tile = std::max<size_t>(1, kFftSmemBudget / per);
    if (per > kFftSmemBudget) tile = 1;
    tile = std::min<size_t>(tile, (size_t)max_tile);
    tile = std::min<size_t>(tile, (size_t)g.nvec);
    const size_t smem = fft_smem_bytes(n, (int)tile);
    if (smem > kMaxSmem) return set_err(ctx, GS_ERR_UNSUPPORTED, "FFT length %d exceeds shared memory", n);
    if (nimg > 65535) return set_err(ctx, GS_ERR_UNSUPPORTED, "too many images in one FFT batch (%d)", nimg);
    auto kern = fft_batched_kernel<kInv, IO>;
    CK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    dim3 grid((unsigned)((g.nvec + tile - 1) / tile), (unsigned)nimg);
    kern<<<grid, kFftThreads, smem, ctx->stream>>>(pl->d, g, (int)tile, io);
    ++ctx->counters.kernel_launches;
    CKL();
    return GS_OK;
}

// Specialised l = 16 * N2 kernels (fastfft.cuh) exist for these sizes.
bool fast_ok(const gs_ctx* ctx, int l) {
    if (ctx->generic_fft || l % 16) return false;
    const int n2 = l / 16;
    return n2 == 32 || n2 == 45 || n2 == 48;
}

template <int N2, bool kInv, bool kCols, class IO>
int launch_fast_n2(gs_ctx* ctx, const float2* tw, int nimg, IO io) {
    using F = Fast16<N2>;
    auto kern = k_fft16<N2, kInv, kCols, IO>;
    const size_t smem = F::smem_bytes();
    CK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    dim3 grid(N2, (unsigned)nimg);
    kern<<<grid, F::kThreads, smem, ctx->stream>>>(tw, io);
    ++ctx->counters.kernel_launches;
    CKL();
    return GS_OK;
}

// Batched l x l transform along rows (kCols = false) or columns of nimg
// images through the specialised kernels; fast_ok(l) must hold.
template <bool kInv, bool kCols, class IO>
int run_fast(gs_ctx* ctx, int l, int nimg, IO io) {
    FftPlan* pl = nullptr;
    TRY(get_plan(ctx, l, &pl));
    if (nimg > 65535) return set_err(ctx, GS_ERR_UNSUPPORTED, "too many images in one FFT batch (%d)", nimg);
    switch (l / 16) {
        case 32: return launch_fast_n2<32, kInv, kCols>(ctx, pl->tw, nimg, io);
        case 45: return launch_fast_n2<45, kInv, kCols>(ctx, pl->tw, nimg, io);
        case 48: return launch_fast_n2<48, kInv, kCols>(ctx, pl->tw, nimg, io);
        default: return set_err(ctx, GS_ERR_UNSUPPORTED, "no specialised FFT for %d", l);
    }
}

template <int N2, int V>
int launch_corr_nv(gs_ctx* ctx, const CorrArgs& a) {
    using C = CorrCfg<N2, V>;
    const size_t smem = CorrSmem<N2, V>::bytes;
    auto kern = k_corr_persistent<N2, V>;
    CK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int per_sm = 0, nsm = 0, dev = 0;
    CK(cudaGetDevice(&dev));
    CK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, C::kThreads, smem));
    if (per_sm < 1) return set_err(ctx, GS_ERR_UNSUPPORTED, "persistent kernel does not fit on an SM");
    if (ctx->corr_ctas_override > 0) per_sm = std::min(per_sm, ctx->corr_ctas_override);
    const long long total_items = (long long)(a.nu + a.lag) * 2 * C::T;
    const long long grid = std::min<long long>((long long)nsm * per_sm, total_items);
    kern<<<(unsigned)grid, C::kThreads, smem, ctx->stream>>>(a);
    ++ctx->counters.kernel_launches;
    CKL();
    return GS_OK;
}

// Persistent FP32 correlation with tiles of `tile` vectors (16 or 8).
int launch_corr(gs_ctx* ctx, int l, int tile, const CorrArgs& a) {
    const bool wide = tile != 8;
    switch (l / 16) {
        case 32: return wide ? launch_corr_nv<32, 16>(ctx, a) : launch_corr_nv<32, 8>(ctx, a);
        case 45: return wide ? launch_corr_nv<45, 16>(ctx, a) : launch_corr_nv<45, 8>(ctx, a);
        case 48: return wide ? launch_corr_nv<48, 16>(ctx, a) : launch_corr_nv<48, 8>(ctx, a);
        default: return set_err(ctx, GS_ERR_UNSUPPORTED, "no persistent kernel for %d", l);
    }
}

template <int N2, bool kBf16>
int launch_corr_tc_n2(gs_ctx* ctx, const CorrArgs& a, long long total_items) {
    using C = TcCfg<N2, kBf16>;
    auto kern = k_corr_tc<N2, kBf16>;
    CK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)C::bytes));
    int per_sm = 0, nsm = 0, dev = 0;
    CK(cudaGetDevice(&dev));
    CK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    CK(cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, cudaSharedmemCarveoutMaxShared));
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, C::kThreads, C::bytes));
    if (per_sm < 1) return set_err(ctx, GS_ERR_UNSUPPORTED, "tensor-core kernel does not fit on an SM");
    // one CTA per SM: it runs C::kWg pipelines and holds the TMEM columns of
    // all of them (a second CTA would not fit in shared memory)
    const long long grid = std::min<long long>((long long)nsm, total_items);
    kern<<<(unsigned)grid, C::kThreads, C::bytes, ctx->stream>>>(a);
    ++ctx->counters.kernel_launches;
    CKL();
    return GS_OK;
}

// Persistent correlation with every DFT stage on the tensor cores (window
// 720, tccorr2.cuh).  One CTA per SM: it allocates all 512 TMEM columns.
template <int kProducts>
int launch_corr_tc2_p(gs_ctx* ctx, const Tc2Args& a) {
    using C = Tc2Cfg<kProducts>;
    static_assert(2 * C::bytes > 228 * 1024, "a second CTA must not fit on an SM (TMEM is allocated whole)");
    auto kern = k_corr_tc2<kProducts>;
    CK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)C::bytes));
    int nsm = 0, dev = 0;
    CK(cudaGetDevice(&dev));
    CK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    const long long total = (long long)(a.nu + a.lag) * 2 * C::T;
    const long long grid = std::min<long long>((long long)nsm, total);
    kern<<<(unsigned)grid, C::kThreads, C::bytes, ctx->stream>>>(a);
    ++ctx->counters.kernel_launches;
    CKL();
    return GS_OK;
}

// Persistent correlation with the tensor-core N2-point stage (tccorr.cuh).
int launch_corr_tc(gs_ctx* ctx, int l, bool bf16, const CorrArgs& a) {
    const int T = l / 8;
    const long long total = (long long)(a.nu + a.lag) * 2 * T;
    switch (l / 16) {
        case 32: return bf16 ? launch_corr_tc_n2<32, true>(ctx, a, total) : launch_corr_tc_n2<32, false>(ctx, a, total);
        case 45: return bf16 ? launch_corr_tc_n2<45, true>(ctx, a, total) : launch_corr_tc_n2<45, false>(ctx, a, total);
        case 48: return bf16 ? launch_corr_tc_n2<48, true>(ctx, a, total) : launch_corr_tc_n2<48, false>(ctx, a, total);
        default: return set_err(ctx, GS_ERR_UNSUPPORTED, "no tensor-core kernel for window %d", l);
    }
}

// Row / column geometry of a batch of row-major h x w images (vectors of
// length w for rows, h for columns).
VecGeom rows_of(int w, int h) { return VecGeom{h, (long long)w, 1, (long long)w * h}; }
VecGeom cols_of(int w, int h) { return VecGeom{w, 1, (long long)w, (long long)w * h}; }

std::vector<int> window_offsets(int n, int l, int overlap) {
    // main.cu:228-250 (interval > 0 is checked by the caller)
    const int interval = l - overlap;
    std::vector<int> offs{0};
    int off = 0;
    while (off + l < n) {
        off += interval;
        if (off + l >= n) off = n - l;
        offs.push_back(off);
    }
    return offs;
}

std::vector<float> angle_list(float step) {
    // main.cu:1232: float accumulation
    std::vector<float> out;
    for (float e = 0.0f; e < 360.0f; e += step) out.push_back(e);
    return out;
}

float printed_phi(float e) {
    float cur = 360.0f - e;  // main.cu:1254-1256
    if (cur >= 360.0f) cur -= 360.0f;
    return cur;
}

CtfDev make_ctf(const gs_params& p, const gs_ctf& c, int padding_for_ds, float* ds_out) {
    // main.cu:150-155 + DataReader.cpp:375-385
    CtfDev d;
    const float defocus = -c.defocus;
    d.apix = p.apix;
    d.dfu = defocus + c.dfdiff;
    d.dfv = defocus - c.dfdiff;
    d.dfdiff = c.dfdiff;
    d.dfang = c.dfang;
    d.lambda = (float)(12.2639 / sqrt((double)p.energy * 1000.0 + 0.97845 * (double)p.energy * (double)p.energy));
    d.cs = p.cs;
    d.ampconst = p.ampconst;
    if (ds_out) *ds_out = 1.0f / (p.apix * (float)padding_for_ds);
    return d;
}

int adjust_padding(int window, int tx, int ty) {
    // main.cu:158-178
    if (window < tx || window < ty) {
        int l = 0;
        while (l < tx || l < ty) l += 32;
        return l;
    }
    return window;
}

unsigned blocks_for(long long n, int threads, unsigned cap = 1u << 30) {
    long long b = (n + threads - 1) / threads;
    if (b < 1) b = 1;
    return (unsigned)std::min<long long>(b, cap);
}

}  // namespace

// ===========================================================================
// C ABI
// ===========================================================================
// Template-pair spectra of one in-plane angle (rotate_template + the
// normalisation and FFT of main.cu:1236-1249): TS[p] = FFT(t_2p - i t_2p+1) / l^2
// with each rotated, masked template mean/variance normalised.
// pfa: store the spectra in the PfaCols column order of the prime-factor
// correlation kernel (window 720) instead of natural order.
// (cos, sin) of in-plane angle e (degrees) as the rotation takes them.
static float2 rotation_cs(float e) {
    const double ang = (double)e * kPiRef / 180.0;
    return make_float2((float)cos(ang), (float)sin(ang));
}
// The spectra of `nang` consecutive angles in one pass (angle z's at
// TS + z Np l^2; pstats and coef hold nang angles): cs = their (cos, sin) on
// the device, or nullptr for the single angle e.
static int pair_spectra_n(gs_ctx* ctx, float e, const float2* cs, int nang, float2* TS, bool pfa) {
    const int l = ctx->l, N = ctx->ntmpl, Np = (N + 1) / 2;
    const long long l2 = (long long)l * l;
    const float2 c = rotation_cs(e);
    const int nimg = Np * nang;
    CK(cudaMemsetAsync(ctx->pstats.p, 0, sizeof(double) * 2 * N * nang, ctx->stream));
    dim3 g(blocks_for(l2, 256, 32), Np, nang);
    k_pair_rotate<<<g, 256, 0, ctx->stream>>>(P<float>(ctx->tmpl), N, l, c.x, c.y, cs, ctx->p.d_m, TS,
                                              P<double>(ctx->pstats));
    ++ctx->counters.kernel_launches;
    k_pair_coef<<<blocks_for(nimg, 128), 128, 0, ctx->stream>>>(P<double>(ctx->pstats), N, l,
                                                                P<float4>(ctx->coef), nang);
    ++ctx->counters.kernel_launches;
    CKL();
    if (fast_ok(ctx, l)) {
        const F16PairNorm rows{TS, P<float4>(ctx->coef), l, l2};
        if (pfa)
            TRY(run_fast<false, false>(ctx, l, nimg, F16PairNormPfa{rows, PfaCols::make(l)}));
        else
            TRY(run_fast<false, false>(ctx, l, nimg, rows));
        TRY(run_fast<false, true>(ctx, l, nimg, F16Complex<true>{TS, l, l2, (float)(1.0 / (double)l2)}));
    } else {
        TRY(run_fft<false>(ctx, l, rows_of(l, l), nimg, IoPairNorm{TS, P<float4>(ctx->coef), l2}));
        TRY(run_fft<false>(ctx, l, cols_of(l, l), nimg, IoComplex{TS, (float)(1.0 / (double)l2)}));
    }
    return GS_OK;
}
static int pair_spectra(gs_ctx* ctx, float e, float2* TS, bool pfa = false) {
    return pair_spectra_n(ctx, e, nullptr, 1, TS, pfa);
}

// Row pass of the correlation of window spectrum Ww with the Np pair spectra
// into the scratch maps R (inverse FFT along x of Ww conj(TS_p)).
static int corr_rows(gs_ctx* ctx, const float2* Ww, const float2* TS, float2* R) {
    const int l = ctx->l, Np = (ctx->ntmpl + 1) / 2;
    const long long l2 = (long long)l * l;
    if (fast_ok(ctx, l)) return run_fast<true, false>(ctx, l, Np, F16Pass1{Ww, TS, R, l, l2});
    return run_fft<true>(ctx, l, rows_of(l, l), Np, IoPass1{Ww, TS, R, l2});
}

// Column pass of the correlation with a per-value epilogue (norm1.cuh).
template <class Epi>
static int corr_cols(gs_ctx* ctx, const float2* R, const Epi& epi) {
    const int l = ctx->l, Np = (ctx->ntmpl + 1) / 2;
    const long long l2 = (long long)l * l;
    if (fast_ok(ctx, l)) return run_fast<true, true>(ctx, l, Np, F16Norm1<Epi>{R, epi, l, l2});
    return run_fft<true>(ctx, l, cols_of(l, l), Np, IoNorm1<Epi>{R, epi});
}

// norm_type 1 (pickPartcles_CCG_NORM path, main.cu:1170-1229): sweep 1 sums
// cc / l^2 and its square per window pixel over all templates and angles
// (compute_CCG_sum, main.cu:724-749) and turns them into mean and standard
// deviation (compute_CCG_mean); sweep 2 recomputes every map, z-scores it
// and reports the maximum of every 1024-element block (main.cu:770-820).
// Picks come out in the reference's order: angle, window row, window
// column, template, block.
static int search_norm1(gs_ctx* ctx, const float2* W, int nx, int ny, const std::vector<int>& offx,
                        const std::vector<int>& offy, const std::vector<float>& angles, float* ms_spec,
                        float* ms_corr, std::vector<gs_pick>* out) {
    const int l = ctx->l, N = ctx->ntmpl;
    const long long l2 = (long long)l * l;
    const int bx = (int)offx.size(), nw = bx * (int)offy.size(), na = (int)angles.size();
    const int nblk = (int)(l2 / 1024);
    const float sgn = ((l / 2) % 2 == 0) ? 1.0f : -1.0f;
    float2* TS = P<float2>(ctx->tspec);
    float2* R = P<float2>(ctx->scratch);
    TRY(ensure(ctx, ctx->pacc, sizeof(float) * 2 * l2 * nw));        // window moments
    TRY(ensure(ctx, ctx->units, sizeof(unsigned long long) * (size_t)nw * N * nblk));  // block keys
    TRY(ensure(ctx, ctx->picks, sizeof(BlockPickDev) * (size_t)nw * N * nblk));
    TRY(ensure(ctx, ctx->count, sizeof(unsigned long long)));
    float* s1 = P<float>(ctx->pacc);
    float* s2 = s1 + l2 * nw;
    unsigned long long* keys = P<unsigned long long>(ctx->units);
    CK(cudaMemsetAsync(s1, 0, sizeof(float) * 2 * l2 * nw, ctx->stream));
    cudaEvent_t ea, eb, ec;
    CK(cudaEventCreate(&ea));
    CK(cudaEventCreate(&eb));
    CK(cudaEventCreate(&ec));
    struct EvGuard3 { cudaEvent_t a, b, c; ~EvGuard3() { cudaEventDestroy(a); cudaEventDestroy(b); cudaEventDestroy(c); } } eg3{ea, eb, ec};
    auto elapsed = [&](void) -> int {
        CK(cudaEventSynchronize(ec));
        float t1 = 0, t2 = 0;
        cudaEventElapsedTime(&t1, ea, eb);
        cudaEventElapsedTime(&t2, eb, ec);
        *ms_spec += t1;
        *ms_corr += t2;
        return GS_OK;
    };
    // ---- sweep 1: moments ----
    for (int ai = 0; ai < na; ++ai) {
        CK(cudaEventRecord(ea, ctx->stream));
        TRY(pair_spectra(ctx, angles[ai], TS));
        CK(cudaEventRecord(eb, ctx->stream));
        for (int w = 0; w < nw; ++w) {
            TRY(corr_rows(ctx, W + (size_t)w * l2, TS, R));
            Norm1Stats e{s1 + (size_t)w * l2, s2 + (size_t)w * l2, l, N, (float)l2, sgn};
            TRY(corr_cols(ctx, R, e));
        }
        CK(cudaEventRecord(ec, ctx->stream));
        TRY(elapsed());
    }
    {
        const long long n = l2 * nw;
        k_norm1_moments<<<blocks_for(n, 256), 256, 0, ctx->stream>>>(s1, s2, n, (float)N * (float)na);
        ++ctx->counters.kernel_launches;
        CKL();
    }
    // ---- sweep 2: z-scores, block maxima, picks ----
    const long long nkeys = (long long)N * nblk;
    std::vector<BlockPickDev> hp;
    for (int ai = 0; ai < na; ++ai) {
        CK(cudaEventRecord(ea, ctx->stream));
        TRY(pair_spectra(ctx, angles[ai], TS));
        CK(cudaEventRecord(eb, ctx->stream));
        CK(cudaMemsetAsync(keys, 0, sizeof(unsigned long long) * nkeys * nw, ctx->stream));
        CK(cudaMemsetAsync(ctx->count.p, 0, sizeof(unsigned long long), ctx->stream));
        for (int w = 0; w < nw; ++w) {
            TRY(corr_rows(ctx, W + (size_t)w * l2, TS, R));
            Norm1Blocks e{s1 + (size_t)w * l2, s2 + (size_t)w * l2, keys + (size_t)w * nkeys, l, N, nblk,
                          (float)l, sgn};
            TRY(corr_cols(ctx, R, e));
            k_norm1_compact<<<blocks_for(nkeys, 256), 256, 0, ctx->stream>>>(
                keys + (size_t)w * nkeys, N, nblk, l, offx[w % bx], offy[w / bx], ctx->p.d_m, nx, ny, ctx->p.thres,
                ((long long)ai * nw + w) * nkeys, P<BlockPickDev>(ctx->picks), P<unsigned long long>(ctx->count),
                nkeys * nw);
            ++ctx->counters.kernel_launches;
            CKL();
        }
        CK(cudaEventRecord(ec, ctx->stream));
        TRY(elapsed());
        unsigned long long cnt = 0;
        CK(cudaMemcpy(&cnt, ctx->count.p, sizeof cnt, cudaMemcpyDeviceToHost));
        if (cnt) {
            const size_t o = hp.size();
            hp.resize(o + cnt);
            CK(cudaMemcpy(hp.data() + o, ctx->picks.p, sizeof(BlockPickDev) * cnt, cudaMemcpyDeviceToHost));
        }
    }
    std::sort(hp.begin(), hp.end(), [](const BlockPickDev& a, const BlockPickDev& b) { return a.key < b.key; });
    out->resize(hp.size());
    for (size_t k = 0; k < hp.size(); ++k) {
        const long long u = hp[k].key / nblk;
        const int J = (int)(u % N);
        const int w = (int)((u / N) % nw);
        const int ai = (int)(u / ((long long)N * nw));
        gs_pick& o = (*out)[k];
        o.angle_index = ai;
        o.phi = printed_phi(angles[ai]);
        o.window_x = w % bx;
        o.window_y = w / bx;
        o.template_index = J;
        o.center_x = hp[k].cx;
        o.center_y = hp[k].cy;
        o.score = hp[k].score;
    }
    return GS_OK;
}

// Soft mask factor of apply_mask (GPU_func.cu:229-247), the arithmetic of
// k_pair_rotate.
__global__ void k_ref_mask(float* __restrict__ mask, int l, float d_m) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= l * l) return;
    const int h = l / 2;
    const int i = q % l, j = q / l;
    const float dm = 1.5f * d_m;
    const float rin = dm / 2.0f, rout = dm / 2.0f + 12.0f;
    const float r = hypotf((float)(i - h), (float)(j - h));
    float m = 1.0f;
    if (r > rout) m = 0.0f;
    else if (r >= rin) m = (float)(0.5 * (double)cosf((float)(kPiRef * (double)(r - rin) / 12.0)) + 0.5);
    mask[q] = m;
}

// Objective (and with grad, its gradient) of n picks, chunked.  tgrad: host
// n x l x l floats or null.
static int score_grad_impl(gs_ctx* ctx, const gs_refine_pick* picks, int n, bool grad, gs_refine_result* out,
                           float* tgrad) {
    const gs_params& p = ctx->p;
    const int l = ctx->l;
    const long long l2 = (long long)l * l;
    if (!ctx->have_units || ctx->last_nw <= 0)
        return set_err(ctx, GS_ERR_STATE, "the window spectra of a norm_type 0 search are needed (search first)");
    for (int i = 0; i < n; ++i) {
        const gs_refine_pick& q = picks[i];
        if (q.window < 0 || q.window >= ctx->last_nw || q.template_index < 0 || q.template_index >= ctx->ntmpl ||
            q.pos < 0 || (long long)q.pos >= l2)
            return set_err(ctx, GS_ERR_ARG, "pick %d: window, template or position out of range", i);
        if (!std::isfinite(q.angle) || !std::isfinite(q.dx) || !std::isfinite(q.dy) || !std::isfinite(q.defocus) ||
            !std::isfinite(q.dfdiff) || !std::isfinite(q.dfang))
            return set_err(ctx, GS_ERR_ARG, "pick %d: parameter not finite", i);
    }
    // per-pick bytes: 6 complex + 2 real maps
    const long long per = l2 * (6 * (long long)sizeof(float2) + 2 * (long long)sizeof(float));
    const int chunk = (int)std::max<long long>(1, std::min<long long>(n, (2ll << 30) / per));
    TRY(ensure(ctx, ctx->rf_pk, sizeof(RefinePickDev) * chunk));
    TRY(ensure(ctx, ctx->rf_acc, sizeof(RefineAcc) * chunk));
    TRY(ensure(ctx, ctx->rf_B, sizeof(float2) * l2 * chunk));
    TRY(ensure(ctx, ctx->rf_F1, sizeof(float2) * l2 * chunk));
    TRY(ensure(ctx, ctx->rf_T, sizeof(float2) * l2 * chunk));
    TRY(ensure(ctx, ctx->rf_TM, sizeof(float) * l2 * chunk));
    TRY(ensure(ctx, ctx->rf_F, sizeof(float2) * l2 * chunk));
    TRY(ensure(ctx, ctx->rf_G, sizeof(float2) * l2 * chunk));
    TRY(ensure(ctx, ctx->rf_TB, sizeof(float) * l2 * chunk));
    TRY(ensure(ctx, ctx->rf_mask, sizeof(float) * l2));
    k_ref_mask<<<blocks_for(l2, 256), 256, 0, ctx->stream>>>(P<float>(ctx->rf_mask), l, p.d_m);
    ++ctx->counters.kernel_launches;
    CKL();
    RefineConsts rc;
    rc.l = l;
    rc.L2 = l2;
    {
        float ds = 0.0f;
        CtfDev c0 = make_ctf(p, ctx->ctf0, p.window_size, &ds);
        rc.apix = c0.apix; rc.lambda = c0.lambda; rc.cs = c0.cs; rc.ampconst = c0.ampconst;
        rc.ds = ds;
    }
    rc.kk = p.kk; rc.a = p.a; rc.b = p.b; rc.b2 = p.b2;
    rc.bf = p.bfactor; rc.bf2 = p.bfactor2; rc.bf3 = p.bfactor3;
    rc.hp = ((float)l * p.apix) / p.highres;
    rc.lp = ((float)l * p.apix) / p.lowres;
    rc.d_m = p.d_m;
    {
        // bins with 0 <= shell < l/2 and x <= l/2 (the amplitude normalisation's count)
        long long cnt = 0;
        for (int y = 0; y < l; ++y)
            for (int x = 0; x <= l / 2; ++x) {
                const float dy = (float)std::min(y, l - y), dx = (float)std::min(x, l - x);
                const int r = (int)floorf(hypotf(dy, dx) + 0.5f) - 1;
                if (r >= 0 && r < l / 2) ++cnt;
            }
        rc.cnt = (float)cnt;
    }
    const float sgn = ((l / 2) % 2 == 0) ? 1.0f : -1.0f;
    RefinePickDev* d_pk = P<RefinePickDev>(ctx->rf_pk);
    RefineAcc* d_acc = P<RefineAcc>(ctx->rf_acc);
    float2* B = P<float2>(ctx->rf_B);
    float2* F1 = P<float2>(ctx->rf_F1);
    float2* T = P<float2>(ctx->rf_T);
    float* TM = P<float>(ctx->rf_TM);
    float2* F = P<float2>(ctx->rf_F);
    float2* Gm = P<float2>(ctx->rf_G);
    float* TB = P<float>(ctx->rf_TB);
    const float* mask = P<float>(ctx->rf_mask);
    const float2* W = P<float2>(ctx->win);
    const float inv_l2 = (float)(1.0 / (double)l2);
    std::vector<RefinePickDev> hp(chunk);
    std::vector<RefineAcc> ha(chunk);
    for (int c0 = 0; c0 < n; c0 += chunk) {
        const int nc = std::min(chunk, n - c0);
        for (int i = 0; i < nc; ++i) {
            const gs_refine_pick& q = picks[c0 + i];
            RefinePickDev& d = hp[i];
            d.window = q.window;
            d.tmpl = q.template_index;
            d.x0 = ((q.pos % l) - l / 2 + l) % l;
            d.y0 = ((q.pos / l) - l / 2 + l) % l;
            d.e = q.angle; d.dx = q.dx; d.dy = q.dy;
            d.defocus = q.defocus; d.dfdiff = q.dfdiff; d.dfang = q.dfang;
        }
        CK(cudaMemcpyAsync(d_pk, hp.data(), sizeof(RefinePickDev) * nc, cudaMemcpyHostToDevice, ctx->stream));
        CK(cudaMemsetAsync(d_acc, 0, sizeof(RefineAcc) * nc, ctx->stream));
        const dim3 g(blocks_for(l2, 256, 128), nc);
        // forward
        TRY(run_fft<false>(ctx, l, rows_of(l, l), nc, IoBaseIn{P<float>(ctx->tbase), d_pk, B, l2}));
        TRY(run_fft<false>(ctx, l, cols_of(l, l), nc, IoComplex{B, inv_l2}));
        k_ref_weight<<<g, 256, 0, ctx->stream>>>(B, F1, d_pk, rc, d_acc);
        ++ctx->counters.kernel_launches;
        TRY(run_fft<true>(ctx, l, rows_of(l, l), nc, IoInvA{F1, T, d_acc, rc.cnt, l2}));
        TRY(run_fft<true>(ctx, l, cols_of(l, l), nc, IoComplex{T, 1.0f}));
        k_ref_rotate<<<g, 256, 0, ctx->stream>>>(T, TM, d_pk, rc, mask, d_acc);
        ++ctx->counters.kernel_launches;
        TRY(run_fft<false>(ctx, l, rows_of(l, l), nc, IoNormIn{TM, d_acc, F, l2}));
        TRY(run_fft<false>(ctx, l, cols_of(l, l), nc, IoComplex{F, inv_l2}));
        k_ref_score<<<g, 256, 0, ctx->stream>>>(W, F, d_pk, rc, d_acc);
        ++ctx->counters.kernel_launches;
        CKL();
        if (grad) {
            TRY(run_fft<true>(ctx, l, rows_of(l, l), nc, IoFbarIn{W, F, d_pk, d_acc, Gm, l, l2, sgn}));
            TRY(run_fft<true>(ctx, l, cols_of(l, l), nc, IoComplex{Gm, inv_l2}));
            k_ref_gsum<<<g, 256, 0, ctx->stream>>>(Gm, TM, rc, d_acc);
            ++ctx->counters.kernel_launches;
            CK(cudaMemsetAsync(TB, 0, sizeof(float) * l2 * nc, ctx->stream));
            k_ref_rot_adj<<<g, 256, 0, ctx->stream>>>(Gm, TM, T, d_pk, rc, mask, d_acc, TB);
            ++ctx->counters.kernel_launches;
            // Fbar2 = FFT(tbar), into Gm (gamma no longer needed)
            TRY(run_fft<false>(ctx, l, rows_of(l, l), nc, IoRealIn2{TB, Gm}));
            TRY(run_fft<false>(ctx, l, cols_of(l, l), nc, IoComplex{Gm, 1.0f}));
            k_ref_abar<<<g, 256, 0, ctx->stream>>>(Gm, F1, rc, d_acc);
            ++ctx->counters.kernel_launches;
            k_ref_theta<<<g, 256, 0, ctx->stream>>>(Gm, F1, B, d_pk, rc, d_acc);
            ++ctx->counters.kernel_launches;
            CKL();
            if (tgrad) {
                // bbar = Re IFFT(Bbar) / l^2, real maps into TB
                TRY(run_fft<true>(ctx, l, rows_of(l, l), nc, IoComplex{Gm, 1.0f}));
                TRY(run_fft<true>(ctx, l, cols_of(l, l), nc, IoRealOut{Gm, TB, inv_l2}));
                CK(cudaMemcpyAsync(tgrad + (size_t)c0 * l2, TB, sizeof(float) * l2 * nc, cudaMemcpyDeviceToHost,
                                   ctx->stream));
            }
        }
        CK(cudaMemcpyAsync(ha.data(), d_acc, sizeof(RefineAcc) * nc, cudaMemcpyDeviceToHost, ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
        for (int i = 0; i < nc; ++i) {
            const RefineAcc& a = ha[i];
            gs_refine_result& o = out[c0 + i];
            const double sig = sqrt(a.sig2);
            o.score = sig > 0.0 ? (float)(sgn * a.c / sig) : 0.0f;
            o.d_angle = (float)a.de;
            o.d_dx = sig > 0.0 ? (float)(sgn * a.cdx / sig) : 0.0f;
            o.d_dy = sig > 0.0 ? (float)(sgn * a.cdy / sig) : 0.0f;
            o.d_defocus = (float)a.dth[0];
            o.d_dfdiff = (float)a.dth[1];
            o.d_dfang = (float)a.dth[2];
            if (!grad) o.d_angle = o.d_dx = o.d_dy = o.d_defocus = o.d_dfdiff = o.d_dfang = 0.0f;
        }
    }
    return GS_OK;
}

// Gradient ascent of every pick's objective (no reference counterpart):
// per step a move of length eta in scaled units (scale: 0.5 deg, 0.25 px,
// 0.005 um, 0.005 um, 5 deg) along the scaled gradient; a step that lowers
// the score is undone and eta halved for that pick.
static int refine_impl(gs_ctx* ctx, gs_refine_pick* picks, int n, int steps, gs_refine_result* out) {
    const double sc[6] = {0.5, 0.25, 0.25, 0.005, 0.005, 5.0};
    std::vector<gs_refine_pick> cur(picks, picks + n), trial(cur);
    std::vector<gs_refine_result> rc(n), rt(n);
    std::vector<double> eta(n, 0.5);
    TRY(score_grad_impl(ctx, cur.data(), n, true, rc.data(), nullptr));
    auto get = [](const gs_refine_pick& q, int k) -> double {
        switch (k) {
            case 0: return q.angle;
            case 1: return q.dx;
            case 2: return q.dy;
            case 3: return q.defocus;
            case 4: return q.dfdiff;
            default: return q.dfang;
        }
    };
    auto set = [](gs_refine_pick& q, int k, double v) {
        switch (k) {
            case 0: q.angle = (float)v; break;
            case 1: q.dx = (float)v; break;
            case 2: q.dy = (float)v; break;
            case 3: q.defocus = (float)v; break;
            case 4: q.dfdiff = (float)v; break;
            default: q.dfang = (float)v; break;
        }
    };
    auto grad_of = [](const gs_refine_result& r, int k) -> double {
        switch (k) {
            case 0: return r.d_angle;
            case 1: return r.d_dx;
            case 2: return r.d_dy;
            case 3: return r.d_defocus;
            case 4: return r.d_dfdiff;
            default: return r.d_dfang;
        }
    };
    for (int it = 0; it < steps; ++it) {
        for (int i = 0; i < n; ++i) {
            double g2 = 0.0;
            for (int k = 0; k < 6; ++k) {
                const double gk = grad_of(rc[i], k) * sc[k];
                g2 += gk * gk;
            }
            trial[i] = cur[i];
            if (g2 > 0.0 && std::isfinite(g2)) {
                const double norm = sqrt(g2);
                for (int k = 0; k < 6; ++k)
                    set(trial[i], k, get(cur[i], k) + eta[i] * sc[k] * sc[k] * grad_of(rc[i], k) / norm);
            }
            // keep the shift inside one pixel and the astigmatism magnitude non-negative
            trial[i].dx = std::max(-1.0f, std::min(1.0f, trial[i].dx));
            trial[i].dy = std::max(-1.0f, std::min(1.0f, trial[i].dy));
            trial[i].dfdiff = std::max(0.0f, trial[i].dfdiff);
        }
        TRY(score_grad_impl(ctx, trial.data(), n, true, rt.data(), nullptr));
        for (int i = 0; i < n; ++i) {
            if (rt[i].score > rc[i].score) {
                cur[i] = trial[i];
                rc[i] = rt[i];
            } else {
                eta[i] *= 0.5;
            }
        }
    }
    for (int i = 0; i < n; ++i) {
        picks[i] = cur[i];
        out[i] = rc[i];
    }
    return GS_OK;
}

extern "C" {

const char* gs_status_string(int s) {
    switch (s) {
        case GS_OK: return "ok";
        case GS_ERR_ARG: return "invalid argument";
        case GS_ERR_OOM: return "out of memory";
        case GS_ERR_CUDA: return "CUDA error";
        case GS_ERR_STATE: return "invalid call order";
        case GS_ERR_UNSUPPORTED: return "unsupported input";
        case GS_ERR_TIMEOUT: return "device wait timed out";
        case GS_ERR_IO: return "I/O error";
        default: return "unknown status";
    }
}

int gs_version(void) { return 10000; }

int gs_params_default(gs_params* p) {
    if (!p) return GS_ERR_ARG;
    // DataReader.h:16-42
    p->apix = -1; p->phi_step = -1; p->kk = -1; p->energy = -1; p->cs = -1;
    p->highres = -1; p->lowres = -1; p->d_m = -1;
    p->thres = 7.0f;
    p->window_size = 320;
    p->overlap = -1;
    p->phase_flip = 0;
    p->norm_type = 0;
    p->invert = 0;
    p->ampconst = 0.07f;
    p->a = -9.32f; p->b = 2.65f; p->b2 = 0.01908f;
    p->bfactor = -78.7757f; p->bfactor2 = -12.9121f; p->bfactor3 = 1.28732f;
    p->precision = GS_PREC_FP32;
    return GS_OK;
}

int gs_ctx_create(int device, gs_ctx** out) {
    if (!out) return GS_ERR_ARG;
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return GS_ERR_CUDA;
    }
    if (device < 0 || device >= ndev) return GS_ERR_ARG;
    gs_ctx* ctx = new gs_ctx();
    ctx->device = device;
    if (cudaSetDevice(device) != cudaSuccess || cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithFlags(&ctx->side, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&ctx->side_ev[0], cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&ctx->side_ev[1], cudaEventDisableTiming) != cudaSuccess) {
        cudaGetLastError();
        if (ctx->side_ev[0]) cudaEventDestroy(ctx->side_ev[0]);
        if (ctx->side) cudaStreamDestroy(ctx->side);
        if (ctx->stream) cudaStreamDestroy(ctx->stream);
        delete ctx;
        return GS_ERR_CUDA;
    }
    *out = ctx;
    return GS_OK;
}

int gs_ctx_destroy(gs_ctx* ctx) {
    if (!ctx) return GS_ERR_ARG;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    cudaStreamSynchronize(ctx->side);
    for (auto& kv : ctx->plans) cudaFree(kv.second.tw);
    DBuf* bufs[] = {&ctx->tmpl, &ctx->in, &ctx->q, &ctx->cimg, &ctx->img, &ctx->stats, &ctx->ra, &ctx->rb,
                    &ctx->off, &ctx->win, &ctx->wsum, &ctx->winv, &ctx->tspec, &ctx->scratch, &ctx->pstats,
                    &ctx->coef, &ctx->acc, &ctx->units, &ctx->picks, &ctx->count, &ctx->unit_wp,
                    &ctx->dep_counters, &ctx->pacc, &ctx->flags, &ctx->tbase, &ctx->rf_pk, &ctx->rf_acc,
                    &ctx->rf_B, &ctx->rf_F1, &ctx->rf_T, &ctx->rf_TM, &ctx->rf_F, &ctx->rf_G, &ctx->rf_TB,
                    &ctx->rf_mask, &ctx->pix_keys, &ctx->pix_pairs, &ctx->pix_R, &ctx->tc2_wmax,
                    &ctx->tc2_pmax, &ctx->tc2_w16, &ctx->tc2_p16, &ctx->rot_cs};
    for (DBuf* b : bufs) free_buf(*b);
    for (cudaEvent_t e : ctx->kev) cudaEventDestroy(e);
    for (cudaEvent_t e : ctx->side_ev) cudaEventDestroy(e);
    cudaStreamDestroy(ctx->side);
    cudaStreamDestroy(ctx->stream);
    delete ctx;
    return GS_OK;
}

const char* gs_ctx_last_error(gs_ctx* ctx) { return ctx ? ctx->err.c_str() : "null context"; }

static int validate_params(gs_ctx* ctx, const gs_params* p) {
    if (!(p->apix > 0) || !(p->phi_step > 0) || !(p->kk >= 0) || !(p->energy > 0) || !(p->cs >= 0) ||
        !(p->highres > 0) || !(p->lowres > 0) || !(p->d_m > 0))
        return set_err(ctx, GS_ERR_ARG, "required parameter missing or not positive");
    if (p->norm_type != 0 && p->norm_type != 1)
        return set_err(ctx, GS_ERR_ARG, "norm_type must be 0 or 1 (got %d)", p->norm_type);
    if (p->precision != GS_PREC_FP32 && p->precision != GS_PREC_TC_BF16 && p->precision != GS_PREC_TC_FP16 &&
        p->precision != GS_PREC_TC_FULL && p->precision != GS_PREC_TC_FULL_1P)
        return set_err(ctx, GS_ERR_ARG, "unknown precision mode %d", p->precision);
    if (p->precision != GS_PREC_FP32 && p->norm_type != 0)
        return set_err(ctx, GS_ERR_UNSUPPORTED, "tensor-core precision modes need norm_type 0");
    if (p->precision == GS_PREC_TC_FP16 && p->phase_flip != 1)
        return set_err(ctx, GS_ERR_UNSUPPORTED,
                       "GS_PREC_TC_FP16 needs phase_flip 1 (amplitude-normalised spectra keep the data in FP16 range)");
    if (p->window_size <= 0) return set_err(ctx, GS_ERR_ARG, "window_size must be positive");
    if (360.0f / p->phi_step > 1e6f) return set_err(ctx, GS_ERR_ARG, "phistep too small");
    return GS_OK;
}

int gs_set_templates(gs_ctx* ctx, const gs_params* p, const float* host_templates, int n, int tx, int ty,
                     const gs_ctf* first_ctf) {
    if (!ctx || !p || !host_templates || !first_ctf || n <= 0 || tx <= 0 || ty <= 0)
        return set_err(ctx, GS_ERR_ARG, "null pointer or empty template stack");
    TRY(validate_params(ctx, p));
    if (n > 2 * 65535) return set_err(ctx, GS_ERR_UNSUPPORTED, "at most %d templates", 2 * 65535);
    CK(cudaSetDevice(ctx->device));
    const int l = adjust_padding(p->window_size, tx, ty);
    if (l % 2) return set_err(ctx, GS_ERR_UNSUPPORTED, "window size %d must be even", l);
    // norm_type 1 reduces 1024-element blocks of the flat l x l map
    // (GPU_func.cu:711-745 with the launch at main.cu:798)
    if (p->norm_type == 1 && ((long long)l * l) % 1024)
        return set_err(ctx, GS_ERR_UNSUPPORTED, "norm_type 1 needs window*window to be a multiple of 1024 (window %d)", l);
    ctx->have_tmpl = false;
    ctx->have_units = false;
    ctx->p = *p;
    ctx->ctf0 = *first_ctf;
    ctx->l = l;
    ctx->ntmpl = n;
    ctx->tx = tx;
    ctx->ty = ty;
    const size_t l2 = (size_t)l * l;
    TRY(ensure(ctx, ctx->tmpl, sizeof(float) * l2 * n));
    TRY(ensure(ctx, ctx->tbase, sizeof(float) * l2 * n));
    const int chunk = (int)std::max<size_t>(1, std::min<size_t>((size_t)n, (size_t)(1u << 30) / (l2 * 8)));
    DBuf raw, F, div, sumsq, inv, wmap, Fb;
    int st = GS_OK;
    do {
        if ((st = ensure(ctx, raw, sizeof(float) * (size_t)tx * ty * chunk))) break;
        if ((st = ensure(ctx, F, sizeof(float2) * l2 * chunk))) break;
        if ((st = ensure(ctx, div, sizeof(float) * (size_t)(l / 2) * chunk))) break;
        if ((st = ensure(ctx, sumsq, sizeof(double) * 2 * chunk))) break;
        if ((st = ensure(ctx, inv, sizeof(double) * chunk))) break;
        if ((st = ensure(ctx, wmap, sizeof(float) * l2))) break;
        if ((st = ensure(ctx, Fb, sizeof(float2) * l2 * chunk))) break;
        // weight map with the FIRST micrograph's CTF; ds from the configured
        // window size (main.cu:155 runs before main.cu:1116 adjusts it)
        float ds = 0.0f;
        CtfDev c0 = make_ctf(*p, *first_ctf, p->window_size, &ds);
        WeightConsts wc;
        wc.hp = ((float)l * p->apix) / p->highres;
        wc.lp = ((float)l * p->apix) / p->lowres;
        wc.ds = ds;
        wc.kk = p->kk; wc.a = p->a; wc.b = p->b; wc.b2 = p->b2;
        wc.bf = p->bfactor; wc.bf2 = p->bfactor2; wc.bf3 = p->bfactor3;
        k_weight_map<<<blocks_for((long long)l2, 256), 256, 0, ctx->stream>>>(P<float>(wmap), l, wc, c0);
        ++ctx->counters.kernel_launches;
        if ((st = (cudaGetLastError() == cudaSuccess ? GS_OK : set_err(ctx, GS_ERR_CUDA, "k_weight_map")))) break;
        for (int c0i = 0; c0i < n && st == GS_OK; c0i += chunk) {
            const int nc = std::min(chunk, n - c0i);
            cudaError_t e = cudaMemcpyAsync(P<float>(raw), host_templates + (size_t)c0i * tx * ty,
                                            sizeof(float) * (size_t)tx * ty * nc, cudaMemcpyHostToDevice, ctx->stream);
            if (e != cudaSuccess) { st = set_err(ctx, GS_ERR_CUDA, "template upload: %s", cudaGetErrorString(e)); break; }
            k_tmpl_pad_edge<<<nc, 256, 0, ctx->stream>>>(P<float>(raw), tx, ty, l, P<float2>(F));
            ++ctx->counters.kernel_launches;
            if (cudaGetLastError() != cudaSuccess) { st = set_err(ctx, GS_ERR_CUDA, "k_tmpl_pad_edge"); break; }
            if (fast_ok(ctx, l)) {
                if ((st = run_fast<false, false>(ctx, l, nc, F16Complex<false>{P<float2>(F), l, (long long)l2, 1.0f}))) break;
                if ((st = run_fast<false, true>(ctx, l, nc, F16Complex<true>{P<float2>(F), l, (long long)l2, 1.0f / (float)l2}))) break;
            } else {
                if ((st = run_fft<false>(ctx, l, rows_of(l, l), nc, IoComplex{P<float2>(F), 1.0f}))) break;
                if ((st = run_fft<false>(ctx, l, cols_of(l, l), nc, IoComplex{P<float2>(F), 1.0f / (float)l2}))) break;
            }
            const size_t shs = (size_t)(l / 2) * (sizeof(double) + sizeof(unsigned));
            if (shs > kMaxSmem) { st = set_err(ctx, GS_ERR_UNSUPPORTED, "window too large"); break; }
            cudaFuncSetAttribute(k_tmpl_shells, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shs);
            k_tmpl_shells<<<nc, 256, shs, ctx->stream>>>(P<float2>(F), l, P<float>(div));
            ++ctx->counters.kernel_launches;
            {
                // whitened base (before the weight), kept for the refinement
                dim3 gb(blocks_for((long long)l2, 256, 64), nc);
                k_tmpl_whiten<<<gb, 256, 0, ctx->stream>>>(P<float2>(F), l, P<float>(div), P<float2>(Fb));
                ++ctx->counters.kernel_launches;
                if ((st = run_fft<true>(ctx, l, rows_of(l, l), nc, IoComplex{P<float2>(Fb), 1.0f}))) break;
                if ((st = run_fft<true>(ctx, l, cols_of(l, l), nc,
                                        IoRealOut{P<float2>(Fb), P<float>(ctx->tbase) + (size_t)c0i * l2, 1.0f}))) break;
            }
            cudaMemsetAsync(P<double>(sumsq), 0, sizeof(double) * 2 * nc, ctx->stream);
            dim3 g(blocks_for((long long)l2, 256, 64), nc);
            k_tmpl_apply<<<g, 256, 0, ctx->stream>>>(P<float2>(F), l, P<float>(div), P<float>(wmap), P<double>(sumsq));
            ++ctx->counters.kernel_launches;
            k_inv_amp_norm<<<blocks_for(nc, 128), 128, 0, ctx->stream>>>(P<double>(sumsq), nc, P<double>(inv));
            ++ctx->counters.kernel_launches;
            if (cudaGetLastError() != cudaSuccess) { st = set_err(ctx, GS_ERR_CUDA, "template weighting"); break; }
            if (fast_ok(ctx, l)) {
                if ((st = run_fast<true, false>(ctx, l, nc, F16ScaleIn<false>{P<float2>(F), P<double>(inv), l, (long long)l2}))) break;
                if ((st = run_fast<true, true>(ctx, l, nc, F16RealOut<true>{P<float2>(F), P<float>(ctx->tmpl) + (size_t)c0i * l2,
                                                                            l, (long long)l2}))) break;
            } else {
                if ((st = run_fft<true>(ctx, l, rows_of(l, l), nc, IoScaleIn{P<float2>(F), P<double>(inv)}))) break;
                if ((st = run_fft<true>(ctx, l, cols_of(l, l), nc,
                                        IoRealOut{P<float2>(F), P<float>(ctx->tmpl) + (size_t)c0i * l2, 1.0f}))) break;
            }
        }
        if (st) break;
        cudaError_t e = cudaStreamSynchronize(ctx->stream);
        if (e != cudaSuccess) st = set_err(ctx, GS_ERR_CUDA, "template preprocessing: %s", cudaGetErrorString(e));
    } while (0);
    cudaStreamSynchronize(ctx->stream);
    free_buf(raw); free_buf(F); free_buf(div); free_buf(sumsq); free_buf(inv); free_buf(wmap); free_buf(Fb);
    if (st == GS_OK) ctx->have_tmpl = true;
    return st;
}

int gs_get_geometry(gs_ctx* ctx, int nx, int ny, gs_geometry* out) {
    if (!ctx || !out || nx <= 0 || ny <= 0) return set_err(ctx, GS_ERR_ARG, "bad geometry query");
    if (!ctx->have_tmpl) return set_err(ctx, GS_ERR_STATE, "templates not loaded");
    const int l = ctx->l;
    if (l - ctx->p.overlap <= 0) return set_err(ctx, GS_ERR_ARG, "overlap must be smaller than the window");
    out->l = l;
    out->n_windows_x = (int)window_offsets(nx, l, ctx->p.overlap).size();
    out->n_windows_y = (int)window_offsets(ny, l, ctx->p.overlap).size();
    out->n_angles = (int)angle_list(ctx->p.phi_step).size();
    out->n_templates = ctx->ntmpl;
    return GS_OK;
}

// One micrograph of a search: its pixels, CTF, geometry, and where its
// windows sit in the window-spectrum array (windows [w0, w0 + nw)).
struct MicPlan {
    const float* host = nullptr;  // host pixels, copied to the device first
    const float* dev = nullptr;   // or device pixels
    int nx = 0, ny = 0, bx = 0, by = 0, nw = 0, w0 = 0;
    gs_ctf ctf{};
    std::vector<int> offx, offy;
};

// Micrograph preprocessing and its window spectra (init_d_image +
// split_normalize_image + fft_on_img, main.cu:523-655, 758-769), written to
// W[w0 .. w0 + nw).
static int prep_micrograph(gs_ctx* ctx, const MicPlan& mp, float2* W) {
    const gs_params& p = ctx->p;
    const int l = ctx->l;
    const long long l2 = (long long)l * l;
    const int nx = mp.nx, ny = mp.ny, bx = mp.bx, by = mp.by, nw = mp.nw;
    const long long npix = (long long)nx * ny;
    const float* d_mic = mp.dev;
    if (mp.host) {
        TRY(ensure(ctx, ctx->in, sizeof(float) * npix));
        CK(cudaMemcpyAsync(ctx->in.p, mp.host, sizeof(float) * npix, cudaMemcpyHostToDevice, ctx->stream));
        d_mic = P<float>(ctx->in);
    }
    // ---- micrograph: init_d_image (main.cu:523-586) ----
    TRY(ensure(ctx, ctx->q, sizeof(float) * 2 * npix));
    TRY(ensure(ctx, ctx->cimg, sizeof(float2) * npix));
    TRY(ensure(ctx, ctx->img, sizeof(float) * npix));
    TRY(ensure(ctx, ctx->stats, sizeof(MicStats)));
    const int ns = std::max(nx, ny) / 2;
    TRY(ensure(ctx, ctx->ra, sizeof(double) * ns));
    TRY(ensure(ctx, ctx->rb, sizeof(unsigned) * ns));
    float* q1 = P<float>(ctx->q);
    float* q2 = q1 + npix;
    k_mic_quot<<<blocks_for(npix, 256), 256, 0, ctx->stream>>>(d_mic, npix, nx, ny, q1, q2);
    ++ctx->counters.kernel_launches;
    k_mic_seq<<<1, 1024, 0, ctx->stream>>>(q1, q2, npix, P<MicStats>(ctx->stats));
    ++ctx->counters.kernel_launches;
    k_mic_clamp<<<blocks_for(npix, 256), 256, 0, ctx->stream>>>(d_mic, npix, P<MicStats>(ctx->stats), p.invert,
                                                                 P<float2>(ctx->cimg));
    ++ctx->counters.kernel_launches;
    CKL();
    float2* C = P<float2>(ctx->cimg);
    TRY(run_fft<false>(ctx, nx, rows_of(nx, ny), 1, IoComplex{C, 1.0f}));
    TRY(run_fft<false>(ctx, ny, cols_of(nx, ny), 1, IoComplex{C, (float)(1.0 / (double)npix)}));
    CtfDev cm = make_ctf(p, mp.ctf, l, nullptr);
    if (p.phase_flip == 1) {
        CK(cudaMemsetAsync(ctx->ra.p, 0, sizeof(double) * ns, ctx->stream));
        CK(cudaMemsetAsync(ctx->rb.p, 0, sizeof(unsigned) * ns, ctx->stream));
        const size_t shs = (size_t)ns * (sizeof(double) + sizeof(unsigned));
        if (shs > kMaxSmem) return set_err(ctx, GS_ERR_UNSUPPORTED, "micrograph too large for the shell histogram");
        CK(cudaFuncSetAttribute(k_mic_flip_shells, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shs));
        const unsigned nb = (unsigned)std::min(ny, 296);
        k_mic_flip_shells<<<nb, 256, shs, ctx->stream>>>(C, nx, ny, cm, P<double>(ctx->ra), P<unsigned>(ctx->rb));
        ++ctx->counters.kernel_launches;
        MicWhitenConsts w;
        const int L = std::max(nx, ny);
        w.apix = p.apix;
        w.hp = ((float)L * p.apix) / p.highres;
        w.lp = ((float)L * p.apix) / p.lowres;
        w.damp = ((float)L * p.apix) / 6.0f;
        w.kk = p.kk; w.a = p.a; w.b = p.b; w.b2 = p.b2;
        w.bf = p.bfactor; w.bf2 = p.bfactor2; w.bf3 = p.bfactor3;
        k_mic_whiten<<<blocks_for(npix, 256), 256, 0, ctx->stream>>>(C, nx, ny, cm, w, P<double>(ctx->ra),
                                                                      P<unsigned>(ctx->rb));
        ++ctx->counters.kernel_launches;
    } else {
        k_set_dc_zero<<<1, 1, 0, ctx->stream>>>(C);
        ++ctx->counters.kernel_launches;
    }
    CKL();
    TRY(run_fft<true>(ctx, ny, cols_of(nx, ny), 1, IoComplex{C, 1.0f}));
    TRY(run_fft<true>(ctx, nx, rows_of(nx, ny), 1, IoRealOut{C, P<float>(ctx->img), 1.0f}));

    // ---- windows: split_normalize_image + fft_on_img (main.cu:588-655, 758-769) ----
    TRY(ensure(ctx, ctx->off, sizeof(int) * (bx + by)));
    std::vector<int> offs(mp.offx);
    offs.insert(offs.end(), mp.offy.begin(), mp.offy.end());
    CK(cudaMemcpyAsync(ctx->off.p, offs.data(), sizeof(int) * offs.size(), cudaMemcpyHostToDevice, ctx->stream));
    const int* d_offx = P<int>(ctx->off);
    const int* d_offy = d_offx + bx;
    float2* Wm = W + (size_t)mp.w0 * l2;
    {
        dim3 g(blocks_for(l2, 256, 256), nw);
        k_extract_windows<<<g, 256, 0, ctx->stream>>>(P<float>(ctx->img), nx, ny, d_offx, d_offy, bx, l, Wm);
        ++ctx->counters.kernel_launches;
        CKL();
    }
    if (fast_ok(ctx, l)) {
        TRY(run_fast<false, false>(ctx, l, nw, F16Complex<false>{Wm, l, l2, 1.0f}));
        TRY(run_fast<false, true>(ctx, l, nw, F16Complex<true>{Wm, l, l2, (float)(1.0 / (double)l2)}));
    } else {
        TRY(run_fft<false>(ctx, l, rows_of(l, l), nw, IoComplex{Wm, 1.0f}));
        TRY(run_fft<false>(ctx, l, cols_of(l, l), nw, IoComplex{Wm, (float)(1.0 / (double)l2)}));
    }
    if (p.phase_flip == 1) {
        TRY(ensure(ctx, ctx->wsum, sizeof(double) * 2 * nw));
        TRY(ensure(ctx, ctx->winv, sizeof(double) * nw));
        CK(cudaMemsetAsync(ctx->wsum.p, 0, sizeof(double) * 2 * nw, ctx->stream));
        dim3 g(blocks_for(l2 / 2, 256, 64), nw);
        k_win_sumsq<<<g, 256, 0, ctx->stream>>>(Wm, l, P<double>(ctx->wsum));
        ++ctx->counters.kernel_launches;
        k_inv_amp_norm<<<blocks_for(nw, 128), 128, 0, ctx->stream>>>(P<double>(ctx->wsum), nw, P<double>(ctx->winv));
        ++ctx->counters.kernel_launches;
        dim3 g2(blocks_for(l2, 256, 256), nw);
        k_scale_images<<<g2, 256, 0, ctx->stream>>>(Wm, l2, P<double>(ctx->winv));
        ++ctx->counters.kernel_launches;
        CKL();
    }
    return GS_OK;
}

// Scheduling of the persistent correlation: ring slots, lag, window block,
// resident CTAs per SM (0 = as many as fit).
struct CorrTuning {
    int slots, lag, window_block, ctas, tile;
};

// Unit order: angle-major over the launch's `angles` angles (pair index
// angle x Np + pair); within an angle blocks of window_block windows, inside
// a block pair-major.
static int upload_unit_order(gs_ctx* ctx, int NW, int Np, int wbk, int limit, int angles = 1) {
    std::vector<int2> wp;
    wp.reserve((size_t)NW * Np * angles);
    wbk = std::max(1, wbk);
    for (int an = 0; an < angles; ++an)
        for (int w0 = 0; w0 < NW; w0 += wbk)
            for (int pp = 0; pp < Np; ++pp)
                for (int w = w0; w < std::min(NW, w0 + wbk); ++w) wp.push_back(make_int2(w, an * Np + pp));
    const size_t n = std::min(wp.size(), (size_t)limit);
    TRY(ensure(ctx, ctx->unit_wp, sizeof(int2) * std::max<size_t>(1, wp.size())));
    CK(cudaMemcpyAsync(ctx->unit_wp.p, wp.data(), sizeof(int2) * n, cudaMemcpyHostToDevice, ctx->stream));
    // the host vector must outlive the (staged) copy
    CK(cudaStreamSynchronize(ctx->stream));
    return GS_OK;
}

// One persistent correlation launch over the first nu units (the template-pair
// spectra of the launch's angles already in TS, angle after angle), results
// to out, out_stride results per angle.
static int corr_launch(gs_ctx* ctx, const float2* W, const float2* TS, int nu, const CorrTuning& t, UnitOut* out,
                       long long out_stride = 0) {
    const int l = ctx->l;
    const long long l2 = (long long)l * l;
    int* cnt = P<int>(ctx->dep_counters);
    CK(cudaMemsetAsync(cnt, 0, sizeof(int) * (2 * (size_t)nu + 4), ctx->stream));
    CK(cudaMemsetAsync(ctx->pacc.p, 0, sizeof(UnitAcc) * 2 * (size_t)nu, ctx->stream));
    CorrArgs ca;
    ca.W = W; ca.P = TS; ca.R = P<float2>(ctx->scratch);
    ca.unit_wp = P<int2>(ctx->unit_wp);
    ca.done_rows = cnt; ca.done_cols = cnt + nu;
    ca.acc = P<UnitAcc>(ctx->pacc);
    ca.out = out;
    ca.next_item = cnt + 2 * (size_t)nu;
    ca.error = P<int>(ctx->flags);
    ca.nu = nu; ca.ntmpl = ctx->ntmpl; ca.S = t.slots; ca.lag = t.lag; ca.L2 = l2;
    ca.pairs = (ctx->ntmpl + 1) / 2;
    ca.out_stride = out_stride;
    // border interval of unshifted indices: X = (x + l/2) mod l is masked
    // when X < d_m/4 or X > l - d_m/4 (GPU_func.cu:681)
    {
        const float q_lo = ctx->p.d_m / 4.0f, q_hi = (float)l - q_lo;
        const int h = l / 2;
        const int ya = (int)ceilf(q_lo), yb = (int)floorf(q_hi);
        ca.yb0 = yb - h + 1;
        ca.yb1 = ya + h - 1;
        if (ca.yb1 < ca.yb0) { ca.yb0 = 1; ca.yb1 = 0; }
    }
    ctx->corr_ctas_override = t.ctas;
    if (ctx->p.precision == GS_PREC_FP32) return launch_corr(ctx, l, t.tile, ca);
    if (ctx->p.precision == GS_PREC_TC_FULL || ctx->p.precision == GS_PREC_TC_FULL_1P) {
        if (l != 720) return set_err(ctx, GS_ERR_UNSUPPORTED, "the all-tensor-core path takes window 720 (got %d)", l);
        // items are claimed and published in batches of 4: every dependency
        // must lie more than a batch back (lag >= 1, slots >= lag + 2)
        if (ca.lag < 1 || ca.S < ca.lag + 2)
            return set_err(ctx, GS_ERR_UNSUPPORTED, "the all-tensor-core path needs lag >= 1 and slots >= lag + 2 "
                           "(got lag %d, slots %d)", ca.lag, ca.S);
        Tc2Args a;
        a.W = ca.W; a.P = ca.P;
        a.R = P<__half2>(ctx->scratch);
        a.wmax = P<float>(ctx->tc2_wmax);
        a.pmax = P<float>(ctx->tc2_pmax);
        a.W16 = P<__half2>(ctx->tc2_w16);
        a.P16 = P<__half2>(ctx->tc2_p16);
        a.unit_wp = ca.unit_wp; a.done_rows = ca.done_rows; a.done_cols = ca.done_cols;
        a.acc = ca.acc; a.out = ca.out; a.next_item = ca.next_item; a.error = ca.error;
        a.nu = ca.nu; a.ntmpl = ca.ntmpl; a.S = ca.S; a.lag = ca.lag; a.L2 = ca.L2;
        a.yb0 = ca.yb0; a.yb1 = ca.yb1;
        a.pairs = ca.pairs; a.out_stride = ca.out_stride;
        return ctx->p.precision == GS_PREC_TC_FULL ? launch_corr_tc2_p<2>(ctx, a) : launch_corr_tc2_p<1>(ctx, a);
    }
    return launch_corr_tc(ctx, l, ctx->p.precision == GS_PREC_TC_BF16, ca);
}

// Autotuner of the persistent correlation's scheduling (no reference
// counterpart): coordinate descent over ring slots, lag, window block and
// CTAs per SM, each candidate timed with CUDA events on angle 0 over the
// first min(nu, 8192) units of its own unit order.  The result is cached
// per (window, templates, windows, precision).
static int autotune(gs_ctx* ctx, const float2* W, const float2* TS, int NW, CorrTuning* best) {
    const int N = ctx->ntmpl, Np = (N + 1) / 2;
    const long long key = (((long long)ctx->l * 1000003 + N) * 1000003 + NW) * 4 + ctx->p.precision;
    auto it = ctx->tuned.find(key);
    if (it != ctx->tuned.end()) {
        *best = CorrTuning{it->second.slots, it->second.lag, it->second.window_block, it->second.ctas,
                           it->second.tile};
        return GS_OK;
    }
    const int nu_full = Np * NW;
    const int nu = std::min(nu_full, 8192);
    std::vector<int> slots_c = {8, 12, 16, 24, 32}, lag_c = {2, 4, 6, 10}, wb_c = {1, 2, 4, 8}, ctas_c = {0, 1};
    std::vector<int> tile_c = {16, 8};
    CorrTuning cur = *best;  // the defaults for this window and precision
    cur.ctas = 0;
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    struct G2 { cudaEvent_t a, b; ~G2() { cudaEventDestroy(a); cudaEventDestroy(b); } } g2{e0, e1};
    int order_wb = -1;
    auto time_of = [&](const CorrTuning& t, float* ms) -> int {
        if (t.window_block != order_wb) {
            TRY(upload_unit_order(ctx, NW, Np, t.window_block, nu));
            order_wb = t.window_block;
        }
        UnitOut* out = P<UnitOut>(ctx->units);
        TRY(corr_launch(ctx, W, TS, nu, t, out));  // warm-up
        CK(cudaEventRecord(e0, ctx->stream));
        TRY(corr_launch(ctx, W, TS, nu, t, out));
        CK(cudaEventRecord(e1, ctx->stream));
        CK(cudaEventSynchronize(e1));
        CK(cudaEventElapsedTime(ms, e0, e1));
        return GS_OK;
    };
    float best_ms = 0;
    TRY(time_of(cur, &best_ms));
    const int npass = ctx->p.precision == GS_PREC_FP32 ? 5 : 4;  // the tile width exists in the FP32 kernel only
    for (int pass = 0; pass < npass; ++pass) {
        const std::vector<int>& cand =
            pass == 0 ? slots_c : pass == 1 ? lag_c : pass == 2 ? wb_c : pass == 3 ? ctas_c : tile_c;
        for (int v : cand) {
            CorrTuning t = cur;
            if (pass == 0) t.slots = v;
            else if (pass == 1) t.lag = v;
            else if (pass == 2) t.window_block = v;
            else if (pass == 3) t.ctas = v;
            else t.tile = v;
            if (t.lag >= t.slots) continue;
            if (t.slots == cur.slots && t.lag == cur.lag && t.window_block == cur.window_block &&
                t.ctas == cur.ctas && t.tile == cur.tile)
                continue;
            float ms = 0;
            TRY(time_of(t, &ms));
            if (ms < best_ms) {
                best_ms = ms;
                cur = t;
            }
        }
    }
    int flag = 0;
    CK(cudaMemcpy(&flag, ctx->flags.p, sizeof(int), cudaMemcpyDeviceToHost));
    if (flag) return set_err(ctx, GS_ERR_TIMEOUT, "correlation kernel: a bounded dependency wait gave up (autotuner)");
    ctx->tuned[key] = CorrTuningSaved{cur.slots, cur.lag, cur.window_block, cur.ctas, cur.tile};
    *best = cur;
    return GS_OK;
}

// Item indices of one persistent launch over n units (2 x l/8 tiles per
// unit) must fit an int.
static bool units_fit(int l, long long n) { return (n + 64) * 2 * (l / 8) < (1ll << 31); }

// In-plane angles per persistent launch before any tuning: the option's
// count, else enough angles for about kUnitsPerLaunch units (a launch's
// ramp-up and drain, and the per-launch overhead, then weigh little against
// its work) with the pair spectra of one launch within kAngleBudget bytes;
// at most na, and within the item-index limit.
static int launch_angles(const gs_ctx* ctx, int nu, int na, bool tc2) {
    constexpr long long kUnitsPerLaunch = 16384;
    constexpr double kAngleBudget = 8.0 * (1ull << 30);
    const int l = ctx->l, Np = (ctx->ntmpl + 1) / 2;
    const long long l2 = (long long)l * l;
    const double angle_bytes = (double)sizeof(float2) * l2 * Np +
                               (tc2 ? (double)sizeof(__half2) * l * 768 * Np + sizeof(float) * Np : 0.0);
    int A;
    if (ctx->angles_per_launch > 0) {
        A = ctx->angles_per_launch;
    } else {
        A = (int)std::max(1ll, kUnitsPerLaunch / nu);
        A = (int)std::min<double>(A, std::max(1.0, std::floor(kAngleBudget / angle_bytes)));
    }
    A = std::max(1, std::min(A, na));
    while (A > 1 && !units_fit(l, (long long)A * nu)) --A;
    return A;
}

// Every angle's (cos, sin) on the device, for the pair spectra of a group of
// angles in one pass (synchronous: before any capture).
static int upload_rotations(gs_ctx* ctx, const std::vector<float>& angles) {
    const int na = (int)angles.size();
    std::vector<float2> cs(std::max(1, na));
    for (int i = 0; i < na; ++i) cs[i] = rotation_cs(angles[i]);
    TRY(ensure(ctx, ctx->rot_cs, sizeof(float2) * cs.size()));
    CK(cudaMemcpy(ctx->rot_cs.p, cs.data(), sizeof(float2) * na, cudaMemcpyHostToDevice));
    return GS_OK;
}

// The first persistent launch's pair spectra, enqueued on the side stream
// so that they overlap the micrograph preparation that follows on the main
// stream (its exact-order statistics keep one SM busy for milliseconds).
// *count = angles prefetched, 0 when the correlation tunes first (the tuner
// times its own pair spectra), has no persistent launch, or norm_type 1.
// side_ev[1] marks their completion.
static int prefetch_pair_spectra(gs_ctx* ctx, int NW, const std::vector<float>& angles, int* count) {
    *count = 0;
    const gs_params& p = ctx->p;
    const int l = ctx->l, N = ctx->ntmpl, Np = (N + 1) / 2, na = (int)angles.size();
    const long long l2 = (long long)l * l;
    const bool tc2 = p.precision == GS_PREC_TC_FULL || p.precision == GS_PREC_TC_FULL_1P;
    const bool persistent = fast_ok(ctx, l) && !ctx->two_pass;
    if (!persistent || ctx->autotune || p.norm_type == 1 || na == 0 || (tc2 && l != 720)) return GS_OK;
    const int nu = Np * NW;
    if (!units_fit(l, nu)) return GS_OK;  // the correlation reports it
    const bool pfa = (p.precision == GS_PREC_FP32 || tc2) && PfaCols::make(l).N2 != 0;
    const int A = launch_angles(ctx, nu, na, tc2);
    TRY(ensure(ctx, ctx->tspec, sizeof(float2) * l2 * Np * A));
    TRY(ensure(ctx, ctx->pstats, sizeof(double) * 2 * N * A));
    TRY(ensure(ctx, ctx->coef, sizeof(float4) * Np * A));
    TRY(upload_rotations(ctx, angles));
    FftPlan* plan = nullptr;
    TRY(get_plan(ctx, l, &plan));  // created (synchronously) before the side work
    // after everything already on the main stream (an earlier search's
    // correlation still reading the pair spectra)
    CK(cudaEventRecord(ctx->side_ev[0], ctx->stream));
    CK(cudaStreamWaitEvent(ctx->side, ctx->side_ev[0], 0));
    // the launch helpers enqueue on ctx->stream: point it at the side stream
    std::swap(ctx->stream, ctx->side);
    int st = GS_OK;
    constexpr int kImgs = 32768;
    const int per = std::max(1, kImgs / Np);
    float2* TS = P<float2>(ctx->tspec);
    for (int k = 0; k < A && st == GS_OK; k += per)
        st = pair_spectra_n(ctx, angles[k], P<float2>(ctx->rot_cs) + k, std::min(per, A - k),
                            TS + (size_t)k * Np * l2, pfa);
    std::swap(ctx->stream, ctx->side);
    CK(cudaEventRecord(ctx->side_ev[1], ctx->side));
    if (st != GS_OK) {
        // whatever was enqueued stays ordered before the main stream's later work
        cudaStreamWaitEvent(ctx->stream, ctx->side_ev[1], 0);
        return st;
    }
    *count = A;
    return GS_OK;
}

// Correlation of every window with every template over all angles (the
// angle loop of main.cu:1232-1257): per angle the template-pair spectra, then
// either one persistent launch over all (window, pair) units or per-window
// row and column launches.  Results to ctx->units [angle][NW][N].
static int correlate_all(gs_ctx* ctx, float2* W, int NW, const std::vector<float>& angles, float* t_spec,
                         float* t_corr, float kt[4], int prefetched = 0) {
    const gs_params& p = ctx->p;
    const int l = ctx->l;
    const long long l2 = (long long)l * l;
    const int N = ctx->ntmpl, Np = (N + 1) / 2;
    const int na = (int)angles.size();
    const long long total_units = (long long)na * NW * N;
    const bool persistent = fast_ok(ctx, l) && !ctx->two_pass;
    // the FP32 persistent kernel at window 720 takes prime-factor transforms
    // and reads its spectra in PfaCols column order
    const bool tc2 = p.precision == GS_PREC_TC_FULL || p.precision == GS_PREC_TC_FULL_1P;
    if (tc2 && l != 720)
        return set_err(ctx, GS_ERR_UNSUPPORTED, "the all-tensor-core path takes window 720 (got %d)", l);
    const bool pfa = persistent && (p.precision == GS_PREC_FP32 || tc2) && PfaCols::make(l).N2 != 0;
    if (p.precision != GS_PREC_FP32 && !persistent)
        return set_err(ctx, GS_ERR_UNSUPPORTED,
                       "tensor-core precision needs window 512, 720 or 768 and the persistent path (window %d)", l);
    const int nu = Np * NW;
    if (!units_fit(l, nu))
        return set_err(ctx, GS_ERR_UNSUPPORTED, "too many (window, template pair) units in one search (%d)", nu);
    int A = persistent ? launch_angles(ctx, nu, na, tc2) : 1;
    // pair spectra of the first launch already enqueued on the side stream
    // (prefetch_pair_spectra): used when the group matches, else awaited
    // and recomputed
    if (prefetched && prefetched != A) {
        CK(cudaStreamWaitEvent(ctx->stream, ctx->side_ev[1], 0));
        prefetched = 0;
    }
    TRY(ensure(ctx, ctx->tspec, sizeof(float2) * l2 * Np * A));
    TRY(ensure(ctx, ctx->pstats, sizeof(double) * 2 * N * A));
    TRY(ensure(ctx, ctx->coef, sizeof(float4) * Np * A));
    // (a prefetch uploaded them already, and its kernels may still read them)
    if (!prefetched) TRY(upload_rotations(ctx, angles));
    TRY(ensure(ctx, ctx->acc, sizeof(UnitAcc) * N));
    TRY(ensure(ctx, ctx->units, sizeof(UnitOut) * std::max<long long>(1, total_units)));
    float2* TS = P<float2>(ctx->tspec);
    UnitOut* units = P<UnitOut>(ctx->units);
    FftPlan* plan = nullptr;
    TRY(get_plan(ctx, l, &plan));  // before any capture: plan creation copies synchronously
    CorrTuning tune{ctx->corr_slots, ctx->corr_lag, ctx->window_block, ctx->corr_ctas, ctx->corr_tile};
    // the all-tensor-core kernel keeps about twice as many items in flight
    // (five pipelines per SM, items claimed in pairs): its own defaults
    // unless the caller set the ring explicitly
    if (tc2 && !ctx->corr_ring_set) {
        tune.slots = 24;
        tune.lag = 12;
    }
    // window 512, FP32 kernel: the autotuner's choice on both measured
    // workloads there (the reference's 1024^2 case, 34.6 against 32.6
    // micrographs/s, and the 32-micrograph batch): 8-vector tiles, a deeper
    // ring and blocks of 8 windows, unless the caller set them
    if (l == 512 && p.precision == GS_PREC_FP32) {
        if (!ctx->corr_ring_set) {
            tune.slots = 32;
            tune.lag = 10;
        }
        if (!ctx->window_block_set) tune.window_block = 8;
        if (!ctx->corr_tile_set) tune.tile = 8;
    }
    // window spectra in PfaCols order for the duration of the correlation,
    // natural order again afterwards (on every return path)
    struct PfaWindows {
        gs_ctx* ctx;
        float2* W;
        long long rows;
        PfaCols pc;
        bool on = false;
        int set(bool to_physical) {
            const int threads = 256, blocks = (int)std::min<long long>(rows, 148 * 8);
            k_pfa_permute_rows<<<blocks, threads, sizeof(float2) * pc.L, ctx->stream>>>(W, rows, pc, to_physical);
            ++ctx->counters.kernel_launches;
            if (cudaGetLastError() != cudaSuccess) return set_err(ctx, GS_ERR_CUDA, "k_pfa_permute_rows");
            on = to_physical;
            return GS_OK;
        }
        ~PfaWindows() {
            if (on) set(false);
        }
    } pfa_w{ctx, W, (long long)NW * l, PfaCols::make(l)};
    if (pfa) TRY(pfa_w.set(true));
    if (tc2) {
        // per-window max |W| for the FP16 scaling of each unit
        TRY(ensure(ctx, ctx->tc2_wmax, sizeof(float) * NW));
        TRY(ensure(ctx, ctx->tc2_pmax, sizeof(float) * Np * A));
        // FP16 copies in the row tiles' order: l rows of 16 x 48 values
        TRY(ensure(ctx, ctx->tc2_w16, sizeof(__half2) * (size_t)l * 768 * NW));
        TRY(ensure(ctx, ctx->tc2_p16, sizeof(__half2) * (size_t)l * 768 * Np * A));
        CK(cudaMemsetAsync(ctx->tc2_wmax.p, 0, sizeof(float) * NW, ctx->stream));
        k_max_abs<<<dim3(64, NW), 256, 0, ctx->stream>>>(W, l2, P<float>(ctx->tc2_wmax));
        k_to_half_tiles<<<dim3(64, NW), 256, 0, ctx->stream>>>(W, P<float>(ctx->tc2_wmax), P<__half2>(ctx->tc2_w16));
        ctx->counters.kernel_launches += 2;
        CKL();
    }
    if (persistent) {
        TRY(ensure(ctx, ctx->dep_counters, sizeof(int) * (2 * (size_t)nu * A + 4)));
        TRY(ensure(ctx, ctx->pacc, sizeof(UnitAcc) * 2 * (size_t)nu * A));
        TRY(ensure(ctx, ctx->flags, sizeof(int) * 4));
        CK(cudaMemsetAsync(ctx->flags.p, 0, sizeof(int) * 4, ctx->stream));
        if (ctx->autotune) {
            TRY(ensure(ctx, ctx->scratch, sizeof(float2) * l2 * 32));
            TRY(pair_spectra(ctx, angles[0], TS, pfa));
            if (tc2) {
                CK(cudaMemsetAsync(ctx->tc2_pmax.p, 0, sizeof(float) * Np, ctx->stream));
                k_max_abs<<<dim3(64, Np), 256, 0, ctx->stream>>>(TS, l2, P<float>(ctx->tc2_pmax));
                k_to_half_tiles<<<dim3(64, Np), 256, 0, ctx->stream>>>(TS, P<float>(ctx->tc2_pmax),
                                                                      P<__half2>(ctx->tc2_p16));
                ctx->counters.kernel_launches += 2;
                CKL();
            }
            TRY(autotune(ctx, W, TS, NW, &tune));
        }
        // angle-major: a launch of fewer angles takes a prefix of this order
        TRY(upload_unit_order(ctx, NW, Np, tune.window_block, nu * A, A));
        TRY(ensure(ctx, ctx->scratch, sizeof(float2) * l2 * tune.slots));
    } else {
        TRY(ensure(ctx, ctx->scratch, sizeof(float2) * l2 * Np));
    }
    ctx->last_tuning[0] = tune.slots;
    ctx->last_tuning[1] = tune.lag;
    ctx->last_tuning[2] = tune.window_block;
    ctx->last_tuning[3] = tune.ctas;
    ctx->last_tuning[4] = p.precision == GS_PREC_FP32 ? tune.tile : 8;
    float2* R = P<float2>(ctx->scratch);
    UnitAcc* acc = P<UnitAcc>(ctx->acc);
    const float q_lo = p.d_m / 4.0f;
    const float q_hi = (float)l - q_lo;
    const float sgn = ((l / 2) % 2 == 0) ? 1.0f : -1.0f;
    const bool timing = ctx->kernel_timing && !ctx->use_graph;
    if (timing && (int)ctx->kev.size() < 4 * NW) {
        while ((int)ctx->kev.size() < 4 * NW) {
            cudaEvent_t e;
            CK(cudaEventCreate(&e));
            ctx->kev.push_back(e);
        }
    }
    cudaEvent_t ea, eb, ec;
    CK(cudaEventCreate(&ea));
    CK(cudaEventCreate(&eb));
    CK(cudaEventCreate(&ec));
    struct EvGuard3 { cudaEvent_t a, b, c; ~EvGuard3() { cudaEventDestroy(a); cudaEventDestroy(b); cudaEventDestroy(c); } } eg3{ea, eb, ec};
    float k1ms = 0, k2ms = 0;
    long long k1n = 0, k2n = 0;

    bool capturing = false;  // enqueue_group is being captured into the graph
    // the work of angles a0 .. a0 + ag - 1 (ag = 1 without the persistent
    // kernel), enqueued on the context's stream: their pair spectra one
    // after the other in TS, then one correlation launch over all their units
    auto enqueue_group = [&](int a0, int ag, bool rec) -> int {
        if (rec) CK(cudaEventRecord(ea, ctx->stream));
        // pair spectra of the group, in passes of at most kImgs images (the
        // first group's may come from the side stream: in the stream loop
        // the main stream waits for them here, a graph waits before capture)
        constexpr int kImgs = 32768;
        const int per = std::max(1, kImgs / Np);
        const bool have = prefetched && a0 == 0;
        if (have && !capturing) CK(cudaStreamWaitEvent(ctx->stream, ctx->side_ev[1], 0));
        for (int k = 0; k < ag && !have; k += per) {
            const int n = std::min(per, ag - k);
            TRY(pair_spectra_n(ctx, angles[a0 + k], P<float2>(ctx->rot_cs) + a0 + k, n,
                               TS + (size_t)k * Np * l2, pfa));
        }
        for (int k = 0; k < ag; ++k) {
            float2* TSk = TS + (size_t)k * Np * l2;
            if (tc2) {
                float* pm = P<float>(ctx->tc2_pmax) + (size_t)k * Np;
                CK(cudaMemsetAsync(pm, 0, sizeof(float) * Np, ctx->stream));
                k_max_abs<<<dim3(64, Np), 256, 0, ctx->stream>>>(TSk, l2, pm);
                k_to_half_tiles<<<dim3(64, Np), 256, 0, ctx->stream>>>(
                    TSk, pm, P<__half2>(ctx->tc2_p16) + (size_t)k * Np * l * 768);
                ctx->counters.kernel_launches += 2;
                CKL();
            }
        }
        if (rec) CK(cudaEventRecord(eb, ctx->stream));
        if (persistent) {
            if (timing) CK(cudaEventRecord(ctx->kev[0], ctx->stream));
            TRY(corr_launch(ctx, W, TS, nu * ag, tune, units + (size_t)a0 * NW * N, (long long)NW * N));
            if (timing) CK(cudaEventRecord(ctx->kev[1], ctx->stream));
            return GS_OK;
        }
        const int ai = a0;
        for (int w = 0; w < NW; ++w) {
            CK(cudaMemsetAsync(acc, 0, sizeof(UnitAcc) * N, ctx->stream));
            const bool fast = fast_ok(ctx, l);
            if (timing) CK(cudaEventRecord(ctx->kev[4 * w + 0], ctx->stream));
            if (fast) TRY(run_fast<true, false>(ctx, l, Np, F16Pass1{W + (size_t)w * l2, TS, R, l, l2}));
            else TRY(run_fft<true>(ctx, l, rows_of(l, l), Np, IoPass1{W + (size_t)w * l2, TS, R, l2}));
            if (timing) CK(cudaEventRecord(ctx->kev[4 * w + 1], ctx->stream));
            if (timing) CK(cudaEventRecord(ctx->kev[4 * w + 2], ctx->stream));
            if (fast) {
                F16Pass2 io2;
                io2.R = R; io2.acc = acc; io2.L = l; io2.ntmpl = N; io2.L2 = l2;
                io2.q_lo = q_lo; io2.q_hi = q_hi; io2.sgn = sgn;
                TRY(run_fast<true, true>(ctx, l, Np, io2));
            } else {
                IoPass2 io2;
                io2.R = R; io2.acc = acc; io2.l = l; io2.ntmpl = N; io2.q_lo = q_lo; io2.q_hi = q_hi; io2.sgn = sgn;
                TRY(run_fft<true>(ctx, l, cols_of(l, l), Np, io2));
            }
            if (timing) CK(cudaEventRecord(ctx->kev[4 * w + 3], ctx->stream));
            k_finalize<<<blocks_for(N, 128), 128, 0, ctx->stream>>>(acc, N, l, units + ((size_t)ai * NW + w) * N);
            ++ctx->counters.kernel_launches;
            CKL();
        }
        return GS_OK;
    };

    // Autotuner, angles per launch (when the default groups angles): each
    // candidate's first group (pair spectra and correlation of angles
    // 0 .. A - 1) timed once after one warm-up group, time per angle
    // compared; the choice is cached with the scheduling.
    if (persistent && ctx->autotune && ctx->angles_per_launch == 0 && A > 1) {
        const long long key = (((long long)l * 1000003 + N) * 1000003 + NW) * 4 + p.precision;
        auto it = ctx->tuned_angles.find(key);
        if (it != ctx->tuned_angles.end()) {
            A = std::max(1, std::min(A, it->second));
        } else {
            std::vector<int> cand = {1, std::max(1, A / 4), std::max(1, A / 2), A};
            cand.erase(std::unique(cand.begin(), cand.end()), cand.end());
            TRY(enqueue_group(0, cand[0], false));  // warm-up
            float best = 0.0f;
            int best_a = A;
            for (int c : cand) {
                CK(cudaEventRecord(ea, ctx->stream));
                TRY(enqueue_group(0, c, false));
                CK(cudaEventRecord(ec, ctx->stream));
                CK(cudaEventSynchronize(ec));
                float ms = 0.0f;
                CK(cudaEventElapsedTime(&ms, ea, ec));
                const float per = ms / (float)c;
                if (c == cand[0] || per < best) {
                    best = per;
                    best_a = c;
                }
            }
            ctx->tuned_angles[key] = best_a;
            A = best_a;
        }
    }
    ctx->last_tuning[5] = A;

    if (ctx->use_graph) {
        // the whole angle loop as one CUDA graph: captured once, launched once
        cudaGraph_t graph = nullptr;
        cudaGraphExec_t exec = nullptr;
        const unsigned long long launches0 = ctx->counters.kernel_launches;
        if (prefetched) CK(cudaStreamWaitEvent(ctx->stream, ctx->side_ev[1], 0));
        capturing = true;
        CK(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
        int st = GS_OK;
        for (int ai = 0; ai < na && st == GS_OK; ai += A) st = enqueue_group(ai, std::min(A, na - ai), false);
        const cudaError_t ce = cudaStreamEndCapture(ctx->stream, &graph);
        capturing = false;
        if (st != GS_OK) {
            if (graph) cudaGraphDestroy(graph);
            return st;
        }
        if (ce != cudaSuccess) return set_err(ctx, GS_ERR_CUDA, "graph capture: %s", cudaGetErrorString(ce));
        struct GGuard { cudaGraph_t g; cudaGraphExec_t* e; ~GGuard() { if (*e) cudaGraphExecDestroy(*e); cudaGraphDestroy(g); } } gg{graph, &exec};
        CK(cudaGraphInstantiate(&exec, graph, 0));
        ctx->graph_kernel_launches = ctx->counters.kernel_launches - launches0;
        CK(cudaEventRecord(eb, ctx->stream));
        CK(cudaGraphLaunch(exec, ctx->stream));
        CK(cudaEventRecord(ec, ctx->stream));
        CK(cudaEventSynchronize(ec));
        float t = 0;
        cudaEventElapsedTime(&t, eb, ec);
        *t_corr += t;
    } else {
        for (int ai = 0; ai < na; ai += A) {
            TRY(enqueue_group(ai, std::min(A, na - ai), true));
            CK(cudaEventRecord(ec, ctx->stream));
            CK(cudaEventSynchronize(ec));
            float t1 = 0, t2 = 0;
            cudaEventElapsedTime(&t1, ea, eb);
            cudaEventElapsedTime(&t2, eb, ec);
            *t_spec += t1;
            *t_corr += t2;
            if (timing && persistent) {
                float a = 0;
                cudaEventElapsedTime(&a, ctx->kev[0], ctx->kev[1]);
                k1ms += a;
                k1n += 1;
            } else if (timing) {
                for (int w = 0; w < NW; ++w) {
                    float a = 0, b = 0;
                    cudaEventElapsedTime(&a, ctx->kev[4 * w + 0], ctx->kev[4 * w + 1]);
                    cudaEventElapsedTime(&b, ctx->kev[4 * w + 2], ctx->kev[4 * w + 3]);
                    k1ms += a;
                    k2ms += b;
                }
                k1n += NW;
                k2n += NW;
            }
        }
    }
    if (persistent) {
        int flag = 0;
        CK(cudaMemcpyAsync(&flag, ctx->flags.p, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
        if (flag) return set_err(ctx, GS_ERR_TIMEOUT, "correlation kernel: a bounded dependency wait gave up");
    }
    kt[0] = k1ms;
    kt[1] = (float)k1n;
    kt[2] = k2ms;
    kt[3] = (float)k2n;
    return GS_OK;
}

// Threshold picks of one micrograph (main.cu:869-891), in the reference's
// line order (angle, window row, window column, template).
static int compact_picks(gs_ctx* ctx, const MicPlan& mp, int NW, const std::vector<float>& angles,
                         std::vector<gs_pick>* out) {
    const gs_params& p = ctx->p;
    const int N = ctx->ntmpl, na = (int)angles.size();
    const long long total = (long long)na * mp.nw * N;
    TRY(ensure(ctx, ctx->picks, sizeof(PickDev) * std::max<long long>(1, total)));
    TRY(ensure(ctx, ctx->count, sizeof(unsigned long long)));
    TRY(ensure(ctx, ctx->off, sizeof(int) * (mp.bx + mp.by)));
    std::vector<int> offs(mp.offx);
    offs.insert(offs.end(), mp.offy.begin(), mp.offy.end());
    CK(cudaMemcpyAsync(ctx->off.p, offs.data(), sizeof(int) * offs.size(), cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemsetAsync(ctx->count.p, 0, sizeof(unsigned long long), ctx->stream));
    if (total > 0) {
        const int* d_offx = P<int>(ctx->off);
        k_compact<<<blocks_for(total, 256), 256, 0, ctx->stream>>>(
            P<UnitOut>(ctx->units), total, mp.nw, N, mp.bx, d_offx, d_offx + mp.bx, ctx->l, p.d_m, mp.nx, mp.ny,
            p.thres, P<PickDev>(ctx->picks), P<unsigned long long>(ctx->count), total, NW, mp.w0);
        ++ctx->counters.kernel_launches;
        CKL();
    }
    unsigned long long cnt = 0;
    CK(cudaMemcpyAsync(&cnt, ctx->count.p, sizeof cnt, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    std::vector<PickDev> hp(cnt);
    if (cnt) CK(cudaMemcpy(hp.data(), ctx->picks.p, sizeof(PickDev) * cnt, cudaMemcpyDeviceToHost));
    std::sort(hp.begin(), hp.end(), [](const PickDev& a, const PickDev& b) { return a.unit < b.unit; });
    out->resize(cnt);
    for (size_t k = 0; k < cnt; ++k) {
        const long long u = hp[k].unit;
        const int J = (int)(u % N);
        const int w = (int)((u / N) % mp.nw);
        const int ai = (int)(u / ((long long)N * mp.nw));
        gs_pick& o = (*out)[k];
        o.angle_index = ai;
        o.phi = printed_phi(angles[ai]);
        o.window_x = w % mp.bx;
        o.window_y = w / mp.bx;
        o.template_index = J;
        o.center_x = hp[k].cx;
        o.center_y = hp[k].cy;
        o.score = hp[k].score;
    }
    return GS_OK;
}

// A search over one or more micrographs with the loaded templates.  The
// windows of all micrographs share one window-spectrum array and every angle's
// template-pair spectra; each micrograph's picks come out in the reference's
// order, micrographs in the given order.
static int search_many(gs_ctx* ctx, std::vector<MicPlan>& mics, std::vector<std::vector<gs_pick>>* res) {
    const gs_params& p = ctx->p;
    const int l = ctx->l;
    const long long l2 = (long long)l * l;
    const int N = ctx->ntmpl;
    if (l - p.overlap <= 0) return set_err(ctx, GS_ERR_ARG, "overlap must be smaller than the window");
    int NW = 0;
    for (MicPlan& mp : mics) {
        if (std::max(mp.nx, mp.ny) / 2 > 1 << 20) return set_err(ctx, GS_ERR_UNSUPPORTED, "micrograph too large");
        mp.offx = window_offsets(mp.nx, l, p.overlap);
        mp.offy = window_offsets(mp.ny, l, p.overlap);
        mp.bx = (int)mp.offx.size();
        mp.by = (int)mp.offy.size();
        mp.nw = mp.bx * mp.by;
        mp.w0 = NW;
        NW += mp.nw;
    }
    if (p.norm_type == 1 && mics.size() != 1)
        return set_err(ctx, GS_ERR_UNSUPPORTED, "norm_type 1 searches one micrograph per call");
    const std::vector<float> angles = angle_list(p.phi_step);
    const int na = (int)angles.size();
    const long long total_units = (long long)na * NW * N;
    ctx->have_units = false;

    cudaEvent_t ev[4];
    for (auto& e : ev) CK(cudaEventCreate(&e));
    struct EvGuard { cudaEvent_t* e; ~EvGuard() { for (int i = 0; i < 4; ++i) cudaEventDestroy(e[i]); } } evg{ev};
    CK(cudaEventRecord(ev[0], ctx->stream));
    // the first launch's pair spectra on the side stream during the
    // micrograph preparation; whatever path the search takes, the main
    // stream's later work is ordered after them
    int prefetched = 0;
    TRY(prefetch_pair_spectra(ctx, NW, angles, &prefetched));
    struct SideJoin {
        gs_ctx* ctx;
        const int* on;
        ~SideJoin() { if (*on) cudaStreamWaitEvent(ctx->stream, ctx->side_ev[1], 0); }
    } side_join{ctx, &prefetched};
    TRY(ensure(ctx, ctx->win, sizeof(float2) * l2 * NW));
    float2* W = P<float2>(ctx->win);
    for (const MicPlan& mp : mics) TRY(prep_micrograph(ctx, mp, W));
    CK(cudaEventRecord(ev[1], ctx->stream));

    float t_spec = 0.0f, t_corr = 0.0f, kt[4] = {0, 0, 0, 0};
    res->assign(mics.size(), std::vector<gs_pick>());
    if (p.norm_type == 1) {
        const int Np = (N + 1) / 2;
        TRY(ensure(ctx, ctx->tspec, sizeof(float2) * l2 * Np));
        TRY(ensure(ctx, ctx->scratch, sizeof(float2) * l2 * Np));
        TRY(ensure(ctx, ctx->pstats, sizeof(double) * 2 * N));
        TRY(ensure(ctx, ctx->coef, sizeof(float4) * Np));
        const MicPlan& mp = mics[0];
        TRY(search_norm1(ctx, W, mp.nx, mp.ny, mp.offx, mp.offy, angles, &t_spec, &t_corr, &(*res)[0]));
    } else {
        TRY(correlate_all(ctx, W, NW, angles, &t_spec, &t_corr, kt, prefetched));
        ctx->last_na = na;
        ctx->last_nw = NW;
        ctx->last_nt = N;
        ctx->have_units = true;
        ctx->last_mics.clear();
        for (const MicPlan& mp : mics) ctx->last_mics.push_back(gs_ctx::MicGeom{mp.nx, mp.ny, mp.w0, mp.offx, mp.offy});
        for (size_t m = 0; m < mics.size(); ++m) TRY(compact_picks(ctx, mics[m], NW, angles, &(*res)[m]));
    }
    CK(cudaEventRecord(ev[3], ctx->stream));
    CK(cudaEventSynchronize(ev[3]));
    float t_prep = 0, t_tot = 0;
    cudaEventElapsedTime(&t_prep, ev[0], ev[1]);
    cudaEventElapsedTime(&t_tot, ev[0], ev[3]);
    const float t[GS_TIMING_COUNT] = {t_prep, t_spec, t_corr, t_tot, kt[0], kt[1], kt[2], kt[3]};
    memcpy(ctx->timings, t, sizeof t);
    ctx->counters.searches += 1;
    ctx->counters.units += (unsigned long long)total_units;
    return GS_OK;
}

// Per-pixel maximum of cc / sigma over (angle, template) for micrograph `mic`
// of the last search (pixmax.cuh): the units whose score reaches `thres` are
// recomputed with the two-pass FP32 kernels, angle by angle, window by window.
static int pixel_max_impl(gs_ctx* ctx, int mic, float thres, float* value, int* tmpl, int* angle_out) {
    const gs_params& p = ctx->p;
    const int l = ctx->l;
    const long long l2 = (long long)l * l;
    const int N = ctx->ntmpl, Np = (N + 1) / 2, NW = ctx->last_nw, na = ctx->last_na;
    const gs_ctx::MicGeom& mg = ctx->last_mics[mic];
    const int bx = (int)mg.offx.size(), nwm = bx * (int)mg.offy.size();
    const std::vector<float> angles = angle_list(p.phi_step);
    if ((int)angles.size() != na) return set_err(ctx, GS_ERR_STATE, "parameters changed since the search");
    // this micrograph's units, every angle
    std::vector<UnitOut> u((size_t)na * nwm * N);
    for (int a = 0; a < na; ++a)
        CK(cudaMemcpyAsync(u.data() + (size_t)a * nwm * N,
                           P<UnitOut>(ctx->units) + ((size_t)a * NW + mg.w0) * N, sizeof(UnitOut) * (size_t)nwm * N,
                           cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    const size_t npix = (size_t)mg.nx * mg.ny;
    TRY(ensure(ctx, ctx->pix_keys, sizeof(unsigned long long) * npix));
    TRY(ensure(ctx, ctx->pix_pairs, sizeof(int) * Np));
    const int chunk = (int)std::max<long long>(1, std::min<long long>(Np, (1ll << 30) / (l2 * (long long)sizeof(float2))));
    TRY(ensure(ctx, ctx->pix_R, sizeof(float2) * l2 * chunk));
    TRY(ensure(ctx, ctx->tspec, sizeof(float2) * l2 * Np));
    TRY(ensure(ctx, ctx->pstats, sizeof(double) * 2 * N));
    TRY(ensure(ctx, ctx->coef, sizeof(float4) * Np));
    CK(cudaMemsetAsync(ctx->pix_keys.p, 0, sizeof(unsigned long long) * npix, ctx->stream));
    unsigned long long* keys = P<unsigned long long>(ctx->pix_keys);
    int* d_pairs = P<int>(ctx->pix_pairs);
    float2* R = P<float2>(ctx->pix_R);
    float2* TS = P<float2>(ctx->tspec);
    const float2* W = P<float2>(ctx->win);
    const float q_lo = p.d_m / 4.0f, q_hi = (float)l - q_lo;
    const float sgn = ((l / 2) % 2 == 0) ? 1.0f : -1.0f;
    std::vector<int> pairs;
    for (int a = 0; a < na; ++a) {
        bool any = false;
        for (size_t i = (size_t)a * nwm * N; i < (size_t)(a + 1) * nwm * N && !any; ++i)
            any = u[i].score >= thres && u[i].sigma > 0.0f;
        if (!any) continue;
        TRY(pair_spectra(ctx, angles[a], TS, false));
        for (int wl = 0; wl < nwm; ++wl) {
            const UnitOut* uw = u.data() + ((size_t)a * nwm + wl) * N;
            pairs.clear();
            for (int pp = 0; pp < Np; ++pp) {
                bool sel = false;
                for (int q = 0; q < 2 && 2 * pp + q < N; ++q)
                    sel = sel || (uw[2 * pp + q].score >= thres && uw[2 * pp + q].sigma > 0.0f);
                if (sel) pairs.push_back(pp);
            }
            if (pairs.empty()) continue;
            const int w = mg.w0 + wl;
            const float2* Ww = W + (long long)w * l2;
            PixelMaxEpi epi;
            epi.keys = keys;
            epi.out = P<UnitOut>(ctx->units) + ((size_t)a * NW + w) * N;
            epi.L = l;
            epi.ntmpl = N;
            epi.nx = mg.nx;
            epi.offx = mg.offx[wl % bx];
            epi.offy = mg.offy[wl / bx];
            epi.idx0 = (unsigned int)a * (unsigned int)N;
            epi.q_lo = q_lo;
            epi.q_hi = q_hi;
            epi.thres = thres;
            epi.sgn = sgn;
            for (size_t c0 = 0; c0 < pairs.size(); c0 += (size_t)chunk) {
                const int nc = (int)std::min<size_t>((size_t)chunk, pairs.size() - c0);
                // pageable source: the copy has completed when the call returns
                CK(cudaMemcpyAsync(d_pairs, pairs.data() + c0, sizeof(int) * nc, cudaMemcpyHostToDevice, ctx->stream));
                epi.pairs = d_pairs;
                if (fast_ok(ctx, l)) {
                    TRY(run_fast<true, false>(ctx, l, nc, F16Pass1Sel{Ww, TS, R, d_pairs, l, l2}));
                    TRY(run_fast<true, true>(ctx, l, nc, F16Norm1<PixelMaxEpi>{R, epi, l, l2}));
                } else {
                    TRY(run_fft<true>(ctx, l, rows_of(l, l), nc, IoPass1Sel{Ww, TS, R, d_pairs, l2}));
                    TRY(run_fft<true>(ctx, l, cols_of(l, l), nc, IoNorm1<PixelMaxEpi>{R, epi}));
                }
                CK(cudaStreamSynchronize(ctx->stream));  // d_pairs is rewritten by the next chunk
            }
        }
    }
    std::vector<unsigned long long> hk(npix);
    CK(cudaMemcpyAsync(hk.data(), keys, sizeof(unsigned long long) * npix, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    for (size_t i = 0; i < npix; ++i) {
        if (!hk[i]) {
            value[i] = 0.0f;
            if (tmpl) tmpl[i] = -1;
            if (angle_out) angle_out[i] = -1;
            continue;
        }
        value[i] = float_unorder((unsigned int)(hk[i] >> 32));
        const unsigned int idx = ~(unsigned int)(hk[i] & 0xffffffffull);
        if (tmpl) tmpl[i] = (int)(idx % (unsigned int)N);
        if (angle_out) angle_out[i] = (int)(idx / (unsigned int)N);
    }
    return GS_OK;
}

// Concatenated picks in a library-owned array.
static int hand_out(gs_ctx* ctx, const std::vector<std::vector<gs_pick>>& res, gs_pick** picks, size_t* n_picks,
                    size_t* per_mic) {
    size_t n = 0;
    for (size_t m = 0; m < res.size(); ++m) {
        if (per_mic) per_mic[m] = res[m].size();
        n += res[m].size();
    }
    gs_pick* out = nullptr;
    if (n) {
        out = (gs_pick*)malloc(sizeof(gs_pick) * n);
        if (!out) return set_err(ctx, GS_ERR_OOM, "host allocation of %zu picks", n);
        size_t k = 0;
        for (const auto& v : res) {
            if (!v.empty()) memcpy(out + k, v.data(), sizeof(gs_pick) * v.size());
            k += v.size();
        }
    }
    *picks = out;
    *n_picks = n;
    return GS_OK;
}

int gs_search_device(gs_ctx* ctx, const float* device_micrograph, int nx, int ny, const gs_ctf* ctf, gs_pick** picks,
                     size_t* n_picks) {
    if (!ctx || !device_micrograph || !ctf || !picks || !n_picks || nx <= 0 || ny <= 0)
        return set_err(ctx, GS_ERR_ARG, "null pointer or empty micrograph");
    *picks = nullptr;
    *n_picks = 0;
    if (!ctx->have_tmpl) return set_err(ctx, GS_ERR_STATE, "gs_set_templates must come first");
    CK(cudaSetDevice(ctx->device));
    std::vector<MicPlan> mics(1);
    mics[0].dev = device_micrograph;
    mics[0].nx = nx;
    mics[0].ny = ny;
    mics[0].ctf = *ctf;
    std::vector<std::vector<gs_pick>> res;
    TRY(search_many(ctx, mics, &res));
    return hand_out(ctx, res, picks, n_picks, nullptr);
}

int gs_search(gs_ctx* ctx, const float* host_micrograph, int nx, int ny, const gs_ctf* ctf, gs_pick** picks,
              size_t* n_picks) {
    if (!ctx || !host_micrograph || !ctf || !picks || !n_picks || nx <= 0 || ny <= 0)
        return set_err(ctx, GS_ERR_ARG, "null pointer or empty micrograph");
    *picks = nullptr;
    *n_picks = 0;
    if (!ctx->have_tmpl) return set_err(ctx, GS_ERR_STATE, "gs_set_templates must come first");
    CK(cudaSetDevice(ctx->device));
    std::vector<MicPlan> mics(1);
    mics[0].host = host_micrograph;
    mics[0].nx = nx;
    mics[0].ny = ny;
    mics[0].ctf = *ctf;
    std::vector<std::vector<gs_pick>> res;
    TRY(search_many(ctx, mics, &res));
    return hand_out(ctx, res, picks, n_picks, nullptr);
}

int gs_search_batch(gs_ctx* ctx, int n_micrographs, const float* const* host_micrographs, const int* nx,
                    const int* ny, const gs_ctf* ctfs, gs_pick** picks, size_t* n_picks, size_t* picks_per_micrograph) {
    if (!ctx || n_micrographs <= 0 || !host_micrographs || !nx || !ny || !ctfs || !picks || !n_picks ||
        !picks_per_micrograph)
        return set_err(ctx, GS_ERR_ARG, "null pointer or empty batch");
    *picks = nullptr;
    *n_picks = 0;
    for (int m = 0; m < n_micrographs; ++m) {
        picks_per_micrograph[m] = 0;
        if (!host_micrographs[m] || nx[m] <= 0 || ny[m] <= 0)
            return set_err(ctx, GS_ERR_ARG, "micrograph %d: null pointer or empty", m);
    }
    if (!ctx->have_tmpl) return set_err(ctx, GS_ERR_STATE, "gs_set_templates must come first");
    CK(cudaSetDevice(ctx->device));
    std::vector<std::vector<gs_pick>> res(n_micrographs);
    if (ctx->p.norm_type == 1) {
        // per-pixel statistics are per micrograph: one search each
        for (int m = 0; m < n_micrographs; ++m) {
            std::vector<MicPlan> one(1);
            one[0].host = host_micrographs[m];
            one[0].nx = nx[m];
            one[0].ny = ny[m];
            one[0].ctf = ctfs[m];
            std::vector<std::vector<gs_pick>> r1;
            TRY(search_many(ctx, one, &r1));
            res[m] = std::move(r1[0]);
        }
    } else {
        std::vector<MicPlan> mics(n_micrographs);
        for (int m = 0; m < n_micrographs; ++m) {
            mics[m].host = host_micrographs[m];
            mics[m].nx = nx[m];
            mics[m].ny = ny[m];
            mics[m].ctf = ctfs[m];
        }
        TRY(search_many(ctx, mics, &res));
    }
    return hand_out(ctx, res, picks, n_picks, picks_per_micrograph);
}

int gs_get_units(gs_ctx* ctx, gs_unit* host_out, size_t cap, size_t* n_out) {
    if (!ctx || !n_out) return set_err(ctx, GS_ERR_ARG, "null pointer");
    if (!ctx->have_units)
        return set_err(ctx, GS_ERR_STATE, "no norm_type 0 search has run (units are its per-template maxima)");
    const size_t total = (size_t)ctx->last_na * ctx->last_nw * ctx->last_nt;
    *n_out = total;
    if (!host_out) return GS_OK;
    if (cap < total) return set_err(ctx, GS_ERR_ARG, "capacity %zu < %zu units", cap, total);
    static_assert(sizeof(gs_unit) == sizeof(UnitOut), "gs_unit layout");
    CK(cudaSetDevice(ctx->device));
    CK(cudaMemcpy(host_out, ctx->units.p, sizeof(gs_unit) * total, cudaMemcpyDeviceToHost));
    return GS_OK;
}

int gs_get_pixel_max(gs_ctx* ctx, int micrograph, float thres, float* value, int* template_index,
                     int* angle_index) {
    if (!ctx || !value) return set_err(ctx, GS_ERR_ARG, "null pointer");
    if (!std::isfinite(thres)) return set_err(ctx, GS_ERR_ARG, "threshold not finite");
    if (!ctx->have_units)
        return set_err(ctx, GS_ERR_STATE, "no norm_type 0 search has run (the map needs its units)");
    if (micrograph < 0 || micrograph >= (int)ctx->last_mics.size())
        return set_err(ctx, GS_ERR_ARG, "micrograph %d not in the last search", micrograph);
    CK(cudaSetDevice(ctx->device));
    return pixel_max_impl(ctx, micrograph, thres, value, template_index, angle_index);
}

void gs_picks_free(gs_pick* p) { free(p); }

int gs_get_stats(gs_ctx* ctx, gs_stats* out) {
    if (!ctx || !out) return GS_ERR_ARG;
    *out = ctx->counters;
    return GS_OK;
}

int gs_get_timings(gs_ctx* ctx, float* out, int n) {
    if (!ctx || !out || n < 0) return GS_ERR_ARG;
    for (int i = 0; i < n && i < GS_TIMING_COUNT; ++i) out[i] = ctx->timings[i];
    return GS_OK;
}

int gs_set_option(gs_ctx* ctx, int option, int value) {
    if (!ctx) return GS_ERR_ARG;
    switch (option) {
        case GS_OPT_GENERIC_FFT: ctx->generic_fft = value != 0; return GS_OK;
        case GS_OPT_TWO_PASS: ctx->two_pass = value != 0; return GS_OK;
        case GS_OPT_CORR_SLOTS:
            if (value <= ctx->corr_lag) return set_err(ctx, GS_ERR_ARG, "slots must exceed the lag");
            ctx->corr_slots = value;
            ctx->corr_ring_set = true;
            return GS_OK;
        case GS_OPT_CORR_LAG:
            if (value < 0 || value >= ctx->corr_slots) return set_err(ctx, GS_ERR_ARG, "lag must be in [0, slots)");
            ctx->corr_lag = value;
            ctx->corr_ring_set = true;
            return GS_OK;
        case GS_OPT_WINDOW_BLOCK:
            if (value < 1) return set_err(ctx, GS_ERR_ARG, "window block must be >= 1");
            ctx->window_block = value;
            ctx->window_block_set = true;
            return GS_OK;
        case GS_OPT_CORR_CTAS:
            if (value < 0) return set_err(ctx, GS_ERR_ARG, "CTAs per SM must be >= 0");
            ctx->corr_ctas = value;
            return GS_OK;
        case GS_OPT_GRAPH: ctx->use_graph = value != 0; return GS_OK;
        case GS_OPT_CORR_TILE:
            if (value != 8 && value != 16) return set_err(ctx, GS_ERR_ARG, "tile width must be 8 or 16");
            ctx->corr_tile = value;
            ctx->corr_tile_set = true;
            return GS_OK;
        case GS_OPT_AUTOTUNE: ctx->autotune = value != 0; return GS_OK;
        case GS_OPT_ANGLES_PER_LAUNCH:
            if (value < 0) return set_err(ctx, GS_ERR_ARG, "angles per launch must be >= 0");
            ctx->angles_per_launch = value;
            return GS_OK;
        default: return set_err(ctx, GS_ERR_ARG, "unknown option %d", option);
    }
}

int gs_score_grad(gs_ctx* ctx, const gs_refine_pick* picks, int n, int with_gradient, gs_refine_result* out,
                  float* template_gradients) {
    if (!ctx || (!picks && n > 0) || (!out && n > 0) || n < 0) return set_err(ctx, GS_ERR_ARG, "null pointer or n < 0");
    if (n == 0) return GS_OK;
    if (!ctx->have_tmpl) return set_err(ctx, GS_ERR_STATE, "gs_set_templates must come first");
    CK(cudaSetDevice(ctx->device));
    return score_grad_impl(ctx, picks, n, with_gradient != 0, out, with_gradient ? template_gradients : nullptr);
}

int gs_refine(gs_ctx* ctx, gs_refine_pick* picks, int n, int steps, gs_refine_result* out) {
    if (!ctx || (!picks && n > 0) || (!out && n > 0) || n < 0 || steps < 0)
        return set_err(ctx, GS_ERR_ARG, "null pointer, n < 0 or steps < 0");
    if (n == 0) return GS_OK;
    if (!ctx->have_tmpl) return set_err(ctx, GS_ERR_STATE, "gs_set_templates must come first");
    CK(cudaSetDevice(ctx->device));
    return refine_impl(ctx, picks, n, steps, out);
}

int gs_get_tuning(gs_ctx* ctx, int* out, int n) {
    if (!ctx || !out || n < 0) return set_err(ctx, GS_ERR_ARG, "null pointer or n < 0");
    for (int i = 0; i < n && i < 6; ++i) out[i] = ctx->last_tuning[i];
    return GS_OK;
}

int gs_set_kernel_timing(gs_ctx* ctx, int enable) {
    if (!ctx) return GS_ERR_ARG;
    ctx->kernel_timing = enable != 0;
    return GS_OK;
}

}  // extern "C"
