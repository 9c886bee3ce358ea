// Pair-potential tables for the XS scoring function.
//
// For each unordered XS type pair (t1 <= t2, index t1 + t2*(t2+1)/2) and each
// r_i = sqrt(i/32), i < 2051 (precalculate.h:255-283, 334-339):
//   smooth_e[i]   = sum_k w_k * term_k(t1, t2, r_i)          (weighted_terms.cpp:64-69)
//   smooth_dor[i] = (e[i+1]-e[i-1]) / ((r[i+1]-r[i-1]) r[i])  (precalculate.h:121-140)
//   fast[i]       = (e[i] + e[i+1]) / 2
// with the five enabled terms of everything.cpp:381-479 on the surface
// distance d = r - R1 - R2 (XS radii, atom_constants.h:209-235).
// Computed in double on the host, in the reference's operation order, so the
// grid maps built from `fast` bin for bin match the reference's CPU grid
// (tables_device.cu builds the same tables on the device for weight sweeps).
#include <cmath>
#include <limits>

#include "common.h"
#include "xs_terms.h"

namespace vd {

void build_tables(const double w[6], std::vector<double>& fast, std::vector<double>& se,
                  std::vector<double>& sd) {
    const double kMaxD = std::numeric_limits<double>::max();
    fast.assign(size_t(kPairTypes) * kN, 0.0);
    se.assign(size_t(kPairTypes) * kN, 0.0);
    sd.assign(size_t(kPairTypes) * kN, 0.0);
    std::vector<double> rs(kN);
    for (int i = 0; i < kN; ++i) rs[i] = std::sqrt(i / 32.0);
    for (int t2 = 0; t2 < kTypes; ++t2)
        for (int t1 = 0; t1 <= t2; ++t1) {
            const size_t b = size_t(tri_index(t1, t2)) * kN;
            for (int i = 0; i < kN; ++i) se[b + i] = std::fmin(kMaxD, xs_weighted_energy(w, t1, t2, rs[i]));
            for (int i = 0; i < kN; ++i) {
                sd[b + i] = (i == 0 || i == kN - 1)
                                ? 0.0
                                : (se[b + i + 1] - se[b + i - 1]) / ((rs[i + 1] - rs[i - 1]) * rs[i]);
                const double nxt = (i + 1 >= kN) ? 0.0 : se[b + i + 1];
                fast[b + i] = (nxt + se[b + i]) / 2;
            }
        }
}

float pair_force_scale(const std::vector<double>& sd) {
    // A pair force is the lerp of two derivative entries times r (at most
    // r_{i+1} in bin i); the kernels sum up to 127 of them per atom.
    double bound = 0.0;
    for (int p = 0; p < kPairTypes; ++p)
        for (int i = 0; i + 1 < kBins; ++i) {
            const size_t b = size_t(p) * kN + i;
            bound = std::fmax(bound, std::fmax(std::fabs(sd[b]), std::fabs(sd[b + 1])) * std::sqrt((i + 1) / 32.0));
        }
    int k = 24;  // finest scale used: 2^-24 kcal/mol/A
    while (k > -24 && 128.0 * bound * std::ldexp(1.0, k) >= 1073741824.0) --k;
    return float(std::ldexp(1.0, k));
}

}  // namespace vd
