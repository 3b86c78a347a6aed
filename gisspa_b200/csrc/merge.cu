// Duplicate merging of picks: gs_merge_duplicates (include/gisspa.h).
//
// Follows the reference's python_scripts/remove_repeat_particles_from_list.py
// (grouping :22-35, visit order :36-50, centre test :53-57, orientation
// distance :59-135, removal rule :136-140).  The pair tests are independent
// and run on the GPU in FP64 (the script's float64): one thread per pick i
// tests every later pick j of its group and lists the duplicate pairs (i, j)
// in j order.  The removal sweep depends on visit order and runs on the host
// over that (sparse) pair list: pick i, if still kept when its turn comes,
// removes each listed j still kept and scoring lower, or is itself removed
// when j scores at least as high, and goes on comparing either way.
#include "gisspa.h"

#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

namespace {

constexpr double kPiScript = 3.14159265359;  // the script's constant

// Rotation angle in degrees between two orientations (alt, az, phi in
// degrees); negative when the script skips the pair.
__device__ double euler_distance(double a1, double z1, double p1, double a2, double z2, double p2) {
    const double alt = a1 * kPiScript / 180, az = z1 * kPiScript / 180, phi = p1 * kPiScript / 180;
    const double alt_o = a2 * kPiScript / 180, az_o = z2 * kPiScript / 180, phi_o = p2 * kPiScript / 180;
    const double ca = cos(alt), sa = sin(alt), cz = cos(az), sz = sin(az), cp = cos(phi), sp = sin(phi);
    const double cao = cos(alt_o), sao = sin(alt_o), czo = cos(az_o), szo = sin(az_o), cpo = cos(phi_o),
                 spo = sin(phi_o);
    double mo[9], m[9], r[9];
    mo[0] = cpo * czo - spo * cao * szo;
    mo[1] = cpo * szo + spo * cao * czo;
    mo[2] = spo * sao;
    mo[3] = -spo * czo - cpo * cao * szo;
    mo[4] = -spo * szo + cpo * cao * czo;
    mo[5] = cpo * sao;
    mo[6] = sao * szo;
    mo[7] = -sao * czo;
    mo[8] = cao;
    m[0] = cp * cz - sp * ca * sz;
    m[1] = -sp * cz - cp * ca * sz;
    m[2] = sa * sz;
    m[3] = cp * sz + sp * ca * cz;
    m[4] = -sp * sz + cp * ca * cz;
    m[5] = -sa * cz;
    m[6] = sp * sa;
    m[7] = cp * sa;
    m[8] = ca;
    r[0] = m[0] * mo[0] + m[3] * mo[1] + m[6] * mo[2];
    r[1] = mo[0] * m[1] + mo[1] * m[4] + mo[2] * m[7];
    r[2] = mo[0] * m[2] + mo[1] * m[5] + mo[2] * m[8];
    r[3] = mo[3] * m[0] + mo[4] * m[3] + mo[5] * m[6];
    r[4] = mo[3] * m[1] + mo[4] * m[4] + mo[5] * m[7];
    r[5] = mo[3] * m[2] + mo[4] * m[5] + mo[5] * m[8];
    r[6] = mo[6] * m[0] + mo[7] * m[3] + mo[8] * m[6];
    r[7] = mo[6] * m[1] + mo[7] * m[4] + mo[8] * m[7];
    r[8] = mo[6] * m[2] + mo[7] * m[5] + mo[8] * m[8];
    const double tr = r[0] + r[4] + r[8];
    double q0 = 0.0;
    if (tr > 0) {
        const double t = sqrt(1 + tr) * 2;
        if (t == 0) return -1.0;
        q0 = 0.25 * t;
    } else {
        // the script's first branch (r0 largest) is evaluated, and may skip the
        // pair, but its q0 is always overridden by the next one
        if (r[0] >= r[4] && r[0] >= r[8]) {
            const double v = 1 + r[0] - r[4] - r[8];
            if (v < 0) return -1.0;  // the script's sqrt would raise here
            if (sqrt(v) * 2 == 0) return -1.0;
        }
        if (r[4] > r[8]) {
            const double v = 1 - r[0] + r[4] - r[8];
            if (v < 0) return -1.0;
            const double t = sqrt(v) * 2;
            if (t == 0) return -1.0;
            q0 = (r[2] - r[6]) / t;
        } else {
            const double v = 1 - r[0] - r[4] + r[8];
            if (v < 0) return -1.0;
            const double t = sqrt(v) * 2;
            if (t == 0) return -1.0;
            q0 = (r[3] - r[1]) / t;
        }
    }
    if (!(q0 <= 1 && q0 >= -1)) return -1.0;
    return fabs(acos(q0) * 2 * 180 / kPiScript);
}

__device__ bool duplicate(const gs_merge_item& p, const gs_merge_item& q, double center, double thres) {
    const double dx = q.x - p.x, dy = q.y - p.y;
    const double dist = fabs(sqrt(dx * dx + dy * dy));
    if (!(dist < center)) return false;
    const double ed = euler_distance(p.alt, p.az, p.phi, q.alt, q.az, q.phi);
    if (ed < 0) return false;
    double d2 = fmod(ed, 180.0);
    if (d2 > thres + 1) d2 = 180 - d2;
    return ed < thres || d2 < thres;
}

// pass 0: count duplicates of each i; pass 1: write them at off[i] in j order
__global__ void k_merge_pairs(const gs_merge_item* __restrict__ it, long long n, const long long* __restrict__ gend,
                              double center, double thres, int pass, unsigned long long* __restrict__ cnt,
                              const unsigned long long* __restrict__ off, long long* __restrict__ pairs) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const gs_merge_item p = it[i];
    const long long end = gend[i];
    unsigned long long c = 0, o = pass ? off[i] : 0;
    for (long long j = i + 1; j < end; ++j) {
        if (duplicate(p, it[j], center, thres)) {
            if (pass) pairs[o + c] = j;
            ++c;
        }
    }
    if (!pass) cnt[i] = c;
}

struct DevMem {
    void* p = nullptr;
    ~DevMem() { if (p) cudaFree(p); }
};

int cuda_status(cudaError_t e) { return e == cudaSuccess ? GS_OK : GS_ERR_CUDA; }

}  // namespace

extern "C" int gs_merge_duplicates(int device, const gs_merge_item* items, size_t n, double center,
                                   double euler_thres, unsigned char* keep) {
    if ((!items || !keep) && n) return GS_ERR_ARG;
    if (n == 0) return GS_OK;
    if (cudaSetDevice(device) != cudaSuccess) return GS_ERR_CUDA;
    // end of each pick's group (runs of equal group ids)
    std::vector<long long> gend(n);
    for (size_t a = 0; a < n;) {
        size_t b = a;
        while (b < n && items[b].group == items[a].group) ++b;
        for (size_t k = a; k < b; ++k) gend[k] = (long long)b;
        a = b;
    }
    DevMem d_it, d_end, d_cnt, d_off, d_pairs;
    if (cudaMalloc(&d_it.p, sizeof(gs_merge_item) * n) != cudaSuccess ||
        cudaMalloc(&d_end.p, sizeof(long long) * n) != cudaSuccess ||
        cudaMalloc(&d_cnt.p, sizeof(unsigned long long) * n) != cudaSuccess ||
        cudaMalloc(&d_off.p, sizeof(unsigned long long) * n) != cudaSuccess)
        return GS_ERR_OOM;
    int st;
    if ((st = cuda_status(cudaMemcpy(d_it.p, items, sizeof(gs_merge_item) * n, cudaMemcpyHostToDevice)))) return st;
    if ((st = cuda_status(cudaMemcpy(d_end.p, gend.data(), sizeof(long long) * n, cudaMemcpyHostToDevice)))) return st;
    const unsigned blocks = (unsigned)((n + 255) / 256);
    k_merge_pairs<<<blocks, 256>>>((const gs_merge_item*)d_it.p, (long long)n, (const long long*)d_end.p, center,
                                   euler_thres, 0, (unsigned long long*)d_cnt.p, nullptr, nullptr);
    if ((st = cuda_status(cudaGetLastError()))) return st;
    std::vector<unsigned long long> cnt(n), off(n);
    if ((st = cuda_status(cudaMemcpy(cnt.data(), d_cnt.p, sizeof(unsigned long long) * n, cudaMemcpyDeviceToHost))))
        return st;
    unsigned long long total = 0;
    for (size_t k = 0; k < n; ++k) {
        off[k] = total;
        total += cnt[k];
    }
    std::vector<long long> pairs(total);
    if (total) {
        if (cudaMalloc(&d_pairs.p, sizeof(long long) * total) != cudaSuccess) return GS_ERR_OOM;
        if ((st = cuda_status(cudaMemcpy(d_off.p, off.data(), sizeof(unsigned long long) * n, cudaMemcpyHostToDevice))))
            return st;
        k_merge_pairs<<<blocks, 256>>>((const gs_merge_item*)d_it.p, (long long)n, (const long long*)d_end.p, center,
                                       euler_thres, 1, nullptr, (const unsigned long long*)d_off.p,
                                       (long long*)d_pairs.p);
        if ((st = cuda_status(cudaGetLastError()))) return st;
        if ((st = cuda_status(cudaMemcpy(pairs.data(), d_pairs.p, sizeof(long long) * total, cudaMemcpyDeviceToHost))))
            return st;
    }
    // the order-dependent removal sweep (:41-49, 136-140)
    std::vector<unsigned char> removed(n, 0);
    for (size_t i = 0; i < n; ++i) {
        if (removed[i]) continue;
        for (unsigned long long k = off[i]; k < off[i] + cnt[i]; ++k) {
            const long long j = pairs[k];
            if (removed[j]) continue;
            if (items[i].score > items[j].score) removed[j] = 1;
            else removed[i] = 1;
        }
    }
    for (size_t k = 0; k < n; ++k) keep[k] = removed[k] ? 0 : 1;
    return GS_OK;
}
