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
// grid maps built from `fast` bin for bin match the reference's CPU grid.
#include <cmath>
#include <limits>

#include "common.h"

namespace vd {
namespace {

const double kRadius[kTypes] = {1.9, 1.9, 1.8, 1.8, 1.8, 1.8, 1.7, 1.7, 1.7,
                                1.7, 2.0, 2.1, 1.5, 1.8, 2.0, 2.2, 1.2};

bool hydrophobic(int t) { return t == 0 || t == 12 || t == 13 || t == 14 || t == 15; }
bool acceptor(int t) { return t == 4 || t == 5 || t == 8 || t == 9; }
bool donor(int t) { return t == 3 || t == 5 || t == 7 || t == 9 || t == 16; }

// Linear ramp from 0 at `bad` to 1 at `good` (everything.cpp:128-138).
double ramp(double bad, double good, double x) {
    if (bad < good) {
        if (x <= bad) return 0;
        if (x >= good) return 1;
    } else {
        if (x >= bad) return 0;
        if (x <= good) return 1;
    }
    return (x - bad) / (good - bad);
}

double weighted_energy(const double w[6], int t1, int t2, double r) {
    const double opt = kRadius[t1] + kRadius[t2];
    const double g1 = std::exp(-((r - (opt + 0)) / 0.5) * ((r - (opt + 0)) / 0.5));
    const double g2 = std::exp(-((r - (opt + 3)) / 2.0) * ((r - (opt + 3)) / 2.0));
    const double d = r - (opt + 0.0);
    const double rep = (d > 0) ? 0 : d * d;
    const double hyd = (hydrophobic(t1) && hydrophobic(t2)) ? ramp(1.5, 0.5, r - opt) : 0;
    const bool hb = (donor(t1) && acceptor(t2)) || (donor(t2) && acceptor(t1));
    const double hbond = hb ? ramp(0, -0.7, r - opt) : 0;
    double acc = 0;
    acc += w[0] * g1;
    acc += w[1] * g2;
    acc += w[2] * rep;
    acc += w[3] * hyd;
    acc += w[4] * hbond;
    return acc;
}

}  // namespace

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
            for (int i = 0; i < kN; ++i) se[b + i] = std::fmin(kMaxD, weighted_energy(w, t1, t2, rs[i]));
            for (int i = 0; i < kN; ++i) {
                sd[b + i] = (i == 0 || i == kN - 1)
                                ? 0.0
                                : (se[b + i + 1] - se[b + i - 1]) / ((rs[i + 1] - rs[i - 1]) * rs[i]);
                const double nxt = (i + 1 >= kN) ? 0.0 : se[b + i + 1];
                fast[b + i] = (nxt + se[b + i]) / 2;
            }
        }
}

}  // namespace vd
