// Pair-potential tables built on the device (vd_set_scoring_device).
//
// Same tables and operation order as the host build (tables.cpp,
// precalculate.h:121-140, 255-283): one thread per (type pair, entry)
// evaluates the weighted XS energy at its own and its neighbouring sample
// distances in FP64 and writes
//   se[i], sd[i] = (e[i+1]-e[i-1]) / ((r[i+1]-r[i-1]) r[i]), fast[i] = (e[i]+e[i+1])/2
// in double (copied back for the host-side consumers) plus the device copies
// the kernels read: fast in FP32 and FP64, smooth as {e_i, dor_i, e_i+1, dor_i+1}.
// This file is compiled without FMA contraction so the arithmetic rounds like
// the host build; only exp() may differ from the host's, by an ulp.
#include <cfloat>
#include <chrono>

#include "common.h"
#include "xs_terms.h"

namespace vd {
namespace {

struct TableParams {
    double w[6];
    double* fast;     // [kPairTypes][kN]
    double* se;
    double* sd;
    float* fast_f;    // [kPairTypes][kBins]
    double* fast_d;   // [kPairTypes][kBins]
    float4* smooth;   // [kPairTypes][kBins]
};

__device__ __forceinline__ double sample_r(int k) { return sqrt(k / 32.0); }

__global__ void __launch_bounds__(256) tables_kernel(TableParams p) {
    const int gid = blockIdx.x * blockDim.x + threadIdx.x;
    if (gid >= kPairTypes * kN) return;
    const int tp = gid / kN, i = gid - tp * kN;
    int t2 = 0;
    while ((t2 + 1) * (t2 + 2) / 2 <= tp) ++t2;  // tp = t1 + t2 (t2 + 1) / 2, t1 <= t2
    const int t1 = tp - t2 * (t2 + 1) / 2;
    auto energy = [&](int k) { return fmin(DBL_MAX, xs_weighted_energy(p.w, t1, t2, sample_r(k))); };
    auto dor = [&](int k, double em, double ep) {
        return (k == 0 || k == kN - 1) ? 0.0 : (ep - em) / ((sample_r(k + 1) - sample_r(k - 1)) * sample_r(k));
    };
    const double e_i = energy(i);
    const double e_m = i > 0 ? energy(i - 1) : 0.0;
    const double e_p = i + 1 < kN ? energy(i + 1) : 0.0;
    const double sd_i = dor(i, e_m, e_p);
    const double fast_i = (e_p + e_i) / 2;
    const size_t o = size_t(tp) * kN + i;
    p.se[o] = e_i;
    p.sd[o] = sd_i;
    p.fast[o] = fast_i;
    if (i < kBins) {  // i + 2 <= kN - 1: the next entry's derivative is defined
        const double sd_p = dor(i + 1, e_i, energy(i + 2));
        const size_t ob = size_t(tp) * kBins + i;
        p.fast_f[ob] = float(fast_i);
        p.fast_d[ob] = fast_i;
        p.smooth[ob] = make_float4(float(e_i), float(sd_i), float(e_p), float(sd_p));
    }
}

}  // namespace

vd_status build_tables_device(Ctx& c, const double w[6]) {
    const size_t n = size_t(kPairTypes) * kN, nb = size_t(kPairTypes) * kBins;
    vd_status st = VD_OK;
    if (!c.d_fast && (st = dev_alloc(c, &c.d_fast, nb * sizeof(float), "pair tables")) != VD_OK) return st;
    if (!c.d_smooth && (st = dev_alloc(c, &c.d_smooth, nb * sizeof(float4), "pair tables")) != VD_OK) return st;
    if (!c.d_fastd && (st = dev_alloc(c, &c.d_fastd, nb * sizeof(double), "pair tables")) != VD_OK) return st;
    st = ensure_scratch(&c, 3 * n * sizeof(double));
    if (st != VD_OK) return st;
    TableParams p{};
    for (int k = 0; k < 6; ++k) p.w[k] = w[k];
    p.fast = static_cast<double*>(c.d_scratch);
    p.se = p.fast + n;
    p.sd = p.se + n;
    p.fast_f = c.d_fast;
    p.fast_d = c.d_fastd;
    p.smooth = c.d_smooth;
    tables_kernel<<<unsigned((n + 255) / 256), 256, 0, c.stream>>>(p);
    VD_CUDA(cudaGetLastError());
    c.fast.resize(n);
    c.se.resize(n);
    c.sd.resize(n);
    VD_CUDA(cudaMemcpyAsync(c.fast.data(), p.fast, n * sizeof(double), cudaMemcpyDeviceToHost, c.stream));
    VD_CUDA(cudaMemcpyAsync(c.se.data(), p.se, n * sizeof(double), cudaMemcpyDeviceToHost, c.stream));
    VD_CUDA(cudaMemcpyAsync(c.sd.data(), p.sd, n * sizeof(double), cudaMemcpyDeviceToHost, c.stream));
    VD_CUDA(cudaStreamSynchronize(c.stream));
    return VD_OK;
}

}  // namespace vd
