// XS pair energy as a function of distance, shared by the host table build
// (tables.cpp) and the device one (tables_device.cu): the five enabled terms of
// everything.cpp:381-479 on the surface distance d = r - R1 - R2 with the XS
// radii of atom_constants.h:209-235, weighted as in weighted_terms.cpp:64-69.
#pragma once

#include <cmath>

#include <cuda_runtime.h>

namespace vd {

__host__ __device__ inline double xs_radius(int t) {
    switch (t) {
        case 0: case 1: return 1.9;                        // C_H, C_P
        case 2: case 3: case 4: case 5: return 1.8;        // N_P, N_D, N_A, N_DA
        case 6: case 7: case 8: case 9: return 1.7;        // O_P, O_D, O_A, O_DA
        case 10: return 2.0;                               // S_P
        case 11: return 2.1;                               // P_P
        case 12: return 1.5;                               // F_H
        case 13: return 1.8;                               // Cl_H
        case 14: return 2.0;                               // Br_H
        case 15: return 2.2;                               // I_H
        default: return 1.2;                               // Met_D
    }
}
__host__ __device__ inline bool xs_hydrophobic(int t) { return t == 0 || t == 12 || t == 13 || t == 14 || t == 15; }
__host__ __device__ inline bool xs_acceptor(int t) { return t == 4 || t == 5 || t == 8 || t == 9; }
__host__ __device__ inline bool xs_donor(int t) { return t == 3 || t == 5 || t == 7 || t == 9 || t == 16; }

// Linear ramp from 0 at `bad` to 1 at `good` (everything.cpp:128-138).
__host__ __device__ inline double xs_ramp(double bad, double good, double x) {
    if (bad < good) {
        if (x <= bad) return 0;
        if (x >= good) return 1;
    } else {
        if (x >= bad) return 0;
        if (x <= good) return 1;
    }
    return (x - bad) / (good - bad);
}

// sum_k w_k * term_k(t1, t2, r); weights gauss1, gauss2, repulsion,
// hydrophobic, hydrogen bond (w[5], the rotor weight, is not a pair term).
__host__ __device__ inline double xs_weighted_energy(const double w[6], int t1, int t2, double r) {
    const double opt = xs_radius(t1) + xs_radius(t2);
    const double g1 = exp(-((r - (opt + 0)) / 0.5) * ((r - (opt + 0)) / 0.5));
    const double g2 = exp(-((r - (opt + 3)) / 2.0) * ((r - (opt + 3)) / 2.0));
    const double d = r - (opt + 0.0);
    const double rep = (d > 0) ? 0 : d * d;
    const double hyd = (xs_hydrophobic(t1) && xs_hydrophobic(t2)) ? xs_ramp(1.5, 0.5, r - opt) : 0;
    const bool hb = (xs_donor(t1) && xs_acceptor(t2)) || (xs_donor(t2) && xs_acceptor(t1));
    const double hbond = hb ? xs_ramp(0, -0.7, r - opt) : 0;
    double acc = 0;
    acc += w[0] * g1;
    acc += w[1] * g2;
    acc += w[2] * rep;
    acc += w[3] * hyd;
    acc += w[4] * hbond;
    return acc;
}

}  // namespace vd
