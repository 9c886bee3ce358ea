/*
 * ORACLE -- test infrastructure only (see vina_oracle.h for the contract).
 * CPU double-precision restatement of the reference's scoring, grid,
 * kinematics, optimiser and search code.  Paths below are relative to the
 * reference tree Vina-CUDA_v1.1/.  Compile with -ffp-contract=off so the
 * double arithmetic follows the reference's operation order without fused
 * multiply-adds (the reference is built for plain x86-64 without FMA).
 */
#include "vina_oracle.h"

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstring>
#include <limits>
#include <thread>
#include <vector>

namespace {

const double kPi = 3.1415926535897931;
const double kEps = std::numeric_limits<double>::epsilon();
const double kMax = std::numeric_limits<double>::max();
const int kTypes = 17;                        // XS_TYPE_SIZE, lib/atom_constants.h:88
const int kPairs = kTypes * (kTypes + 1) / 2; // 153
const double kCutoff = 8.0;                   // lib/everything.cpp:310
const double kFactor = 32.0;                  // lib/precalculate.h:255
const int kN = int(kFactor * kCutoff * kCutoff) + 3;  // 2051, precalculate.h:257

struct V3 {
    double d[3];
    V3() { d[0] = d[1] = d[2] = 0; }
    V3(double a, double b, double c) { d[0] = a; d[1] = b; d[2] = c; }
    double& operator[](int i) { return d[i]; }
    double operator[](int i) const { return d[i]; }
};
inline V3 operator+(const V3& a, const V3& b) { return V3(a[0] + b[0], a[1] + b[1], a[2] + b[2]); }
inline V3 operator-(const V3& a, const V3& b) { return V3(a[0] - b[0], a[1] - b[1], a[2] - b[2]); }
inline V3 operator*(double s, const V3& a) { return V3(s * a[0], s * a[1], s * a[2]); }
inline V3& operator+=(V3& a, const V3& b) { a[0] += b[0]; a[1] += b[1]; a[2] += b[2]; return a; }
inline V3& operator-=(V3& a, const V3& b) { a[0] -= b[0]; a[1] -= b[1]; a[2] -= b[2]; return a; }
inline double sqr(double x) { return x * x; }
inline double dot(const V3& a, const V3& b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
inline double sqr(const V3& a) { return sqr(a[0]) + sqr(a[1]) + sqr(a[2]); }       // common.h:294
inline double dist_sqr(const V3& a, const V3& b) {                                  // common.h:286
    return sqr(a[0] - b[0]) + sqr(a[1] - b[1]) + sqr(a[2] - b[2]);
}
inline V3 cross(const V3& a, const V3& b) {
    return V3(a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]);
}

// ---------------------------------------------------------------- quaternions
// lib/quaternion.cpp; boost::math::quaternion is plain Hamilton arithmetic.
struct Q { double a, b, c, d; };
const Q kQid = {1, 0, 0, 0};
inline Q qmul(const Q& x, const Q& y) {
    return {x.a * y.a - x.b * y.b - x.c * y.c - x.d * y.d,
            x.a * y.b + x.b * y.a + x.c * y.d - x.d * y.c,
            x.a * y.c - x.b * y.d + x.c * y.a + x.d * y.b,
            x.a * y.d + x.b * y.c - x.c * y.b + x.d * y.a};
}
inline double qnorm_sqr(const Q& q) { return sqr(q.a) + sqr(q.b) + sqr(q.c) + sqr(q.d); }

void normalize_angle(double& x) {  // common.h:316-340
    if (x > 3 * kPi) {
        double n = (x - kPi) / (2 * kPi);
        x -= 2 * kPi * std::ceil(n);
        normalize_angle(x);
    } else if (x < -3 * kPi) {
        double n = (-x - kPi) / (2 * kPi);
        x += 2 * kPi * std::ceil(n);
        normalize_angle(x);
    } else if (x > kPi) {
        x -= 2 * kPi;
    } else if (x < -kPi) {
        x += 2 * kPi;
    }
}
inline double normalized_angle(double x) { normalize_angle(x); return x; }

Q angle_to_quaternion(const V3& axis, double angle) {  // quaternion.cpp:65-74
    normalize_angle(angle);
    double c = std::cos(angle / 2), s = std::sin(angle / 2);
    return {c, s * axis[0], s * axis[1], s * axis[2]};
}
Q angle_to_quaternion(const V3& rot) {  // quaternion.cpp:89-97
    double angle = std::sqrt(sqr(rot));
    if (angle > kEps) {
        V3 axis = (1 / angle) * rot;
        return angle_to_quaternion(axis, angle);
    }
    return kQid;
}
void quaternion_normalize_approx(Q& q, double tol = 1e-6) {  // quaternion.h:120-133
    double s = qnorm_sqr(q);
    if (std::abs(s - 1) < tol) return;
    double a = std::sqrt(s);
    double inv = 1 / a;
    q.a *= inv; q.b *= inv; q.c *= inv; q.d *= inv;
}
void quaternion_increment(Q& q, const V3& rot) {  // quaternion.cpp:235-240
    q = qmul(angle_to_quaternion(rot), q);
    quaternion_normalize_approx(q);
}
struct M3 { double m[9]; };  // m[i + 3*j] = row i, column j (lib/matrix.h)
M3 quaternion_to_r3(const Q& q) {  // quaternion.cpp:155-192
    const double a = q.a, b = q.b, c = q.c, d = q.d;
    const double aa = a * a, ab = a * b, ac = a * c, ad = a * d, bb = b * b, bc = b * c,
                 bd = b * d, cc = c * c, cd = c * d, dd = d * d;
    M3 t;
    t.m[0 + 0] = aa + bb - cc - dd;
    t.m[0 + 3] = 2 * (-ad + bc);
    t.m[0 + 6] = 2 * (ac + bd);
    t.m[1 + 0] = 2 * (ad + bc);
    t.m[1 + 3] = aa - bb + cc - dd;
    t.m[1 + 6] = 2 * (-ab + cd);
    t.m[2 + 0] = 2 * (-ac + bd);
    t.m[2 + 3] = 2 * (ab + cd);
    t.m[2 + 6] = aa - bb - cc + dd;
    return t;
}
inline V3 mv(const M3& m, const V3& v) {
    return V3(m.m[0] * v[0] + m.m[3] * v[1] + m.m[6] * v[2],
              m.m[1] * v[0] + m.m[4] * v[1] + m.m[7] * v[2],
              m.m[2] * v[0] + m.m[5] * v[1] + m.m[8] * v[2]);
}

// ------------------------------------------------------------ scoring terms
// lib/atom_constants.h:209-278 (XS radii and predicates)
const double kXsRadius[kTypes] = {1.9, 1.9, 1.8, 1.8, 1.8, 1.8, 1.7, 1.7, 1.7,
                                  1.7, 2.0, 2.1, 1.5, 1.8, 2.0, 2.2, 1.2};
inline bool xs_hydrophobic(int t) { return t == 0 || t == 12 || t == 13 || t == 14 || t == 15; }
inline bool xs_acceptor(int t) { return t == 4 || t == 5 || t == 8 || t == 9; }
inline bool xs_donor(int t) { return t == 3 || t == 5 || t == 7 || t == 9 || t == 16; }
inline bool xs_hbond(int a, int b) {
    return (xs_donor(a) && xs_acceptor(b)) || (xs_donor(b) && xs_acceptor(a));
}
inline double slope_step(double bad, double good, double x) {  // everything.cpp:128-138
    if (bad < good) {
        if (x <= bad) return 0;
        if (x >= good) return 1;
    } else {
        if (x >= bad) return 0;
        if (x <= good) return 1;
    }
    return (x - bad) / (good - bad);
}
// The five enabled usable terms, everything.cpp:381-479, in weight order.
void raw_terms(int t1, int t2, double r, double out[5]) {
    const double opt = kXsRadius[t1] + kXsRadius[t2];       // everything.cpp:97-99
    out[0] = std::exp(-sqr((r - (opt + 0)) / 0.5));          // gauss(0, 0.5) 101-110
    out[1] = std::exp(-sqr((r - (opt + 3)) / 2.0));          // gauss(3, 2.0)
    double d = r - (opt + 0.0);                              // repulsion(0) 115-126
    out[2] = (d > 0) ? 0 : d * d;
    out[3] = (xs_hydrophobic(t1) && xs_hydrophobic(t2)) ? slope_step(1.5, 0.5, r - opt) : 0;  // 141-152
    out[4] = xs_hbond(t1, t2) ? slope_step(0, -0.7, r - opt) : 0;  // non_dir_h_bond 205-216
}
inline int tri_index(int t1, int t2) {  // triangular_matrix_index.h
    return (t1 <= t2) ? t1 + t2 * (t2 + 1) / 2 : t2 + t1 * (t1 + 1) / 2;
}
inline double curl(double& e, double v) {  // curl.h:42-47, returns the scale
    if (e > 0 && v < 0.1 * kMax) {
        double tmp = (v < kEps) ? 0 : (v / (v + e));
        e *= tmp;
        return tmp;
    }
    return 1.0;
}

// ------------------------------------------------------------ precalculate
struct Precalc {  // precalculate.h:255-283
    std::vector<double> fast, se, sd;  // [kPairs*kN]
    void build(const double w[5]) {
        fast.assign(size_t(kPairs) * kN, 0);
        se.assign(size_t(kPairs) * kN, 0);
        sd.assign(size_t(kPairs) * kN, 0);
        std::vector<double> rs(kN);
        for (int i = 0; i < kN; ++i) rs[i] = std::sqrt(i / kFactor);  // calculate_rs 334-339
        for (int t1 = 0; t1 < kTypes; ++t1)
            for (int t2 = t1; t2 < kTypes; ++t2) {
                const size_t base = size_t(tri_index(t1, t2)) * kN;
                for (int i = 0; i < kN; ++i) {
                    double t[5];
                    raw_terms(t1, t2, rs[i], t);
                    double acc = 0;  // weighted_terms.cpp:64-69
                    for (int k = 0; k < 5; ++k) acc += w[k] * t[k];
                    se[base + i] = std::min(kMax, acc);
                }
                for (int i = 0; i < kN; ++i) {  // init_from_smooth_fst 121-140
                    double& dor = sd[base + i];
                    if (i == 0 || i == kN - 1) dor = 0;
                    else {
                        double delta = rs[i + 1] - rs[i - 1];
                        double r = rs[i];
                        dor = (se[base + i + 1] - se[base + i - 1]) / (delta * r);
                    }
                    double f1 = se[base + i];
                    double f2 = (i + 1 >= kN) ? 0 : se[base + i + 1];
                    fast[base + i] = (f2 + f1) / 2;
                }
            }
    }
    double eval_fast(int tp, double r2) const {  // precalculate.h:55-60
        size_t i = size_t(kFactor * r2);
        return fast[size_t(tp) * kN + i];
    }
    void eval_deriv(int tp, double r2, double& e, double& dor) const {  // precalculate.h:80-95
        double rf = kFactor * r2;
        size_t i1 = size_t(rf), i2 = i1 + 1;
        double rem = rf - i1;
        const size_t b = size_t(tp) * kN;
        e = se[b + i1] + rem * (se[b + i2] - se[b + i1]);
        dor = sd[b + i1] + rem * (sd[b + i2] - sd[b + i1]);
    }
};

// ------------------------------------------------------------ grids
struct GridDim { double begin = 0, end = 0; int n = 0; };  // grid_dim.h

struct CellList {  // szv_grid.cpp:28-131
    double init[3], range[3];
    int dim[3];
    std::vector<std::vector<int>> cells;
    V3 index_to_coord(int i, int j, int k) const {  // szv_grid.cpp:109-118
        int idx[3] = {i, j, k};
        V3 t;
        for (int n = 0; n < 3; ++n) t[n] = init[n] + range[n] * idx[n] / dim[n];
        return t;
    }
    static double brick_dsqr(const V3& b, const V3& e, const V3& v) {  // brick.h:33-49
        V3 c;
        for (int i = 0; i < 3; ++i) c[i] = (v[i] <= b[i]) ? b[i] : ((v[i] >= e[i]) ? e[i] : v[i]);
        return dist_sqr(c, v);
    }
    void build(const GridDim gd[3], const std::vector<V3>& xyz, const std::vector<int>& xs) {
        V3 end;
        for (int i = 0; i < 3; ++i) {  // szv_grid_dims 120-131
            init[i] = gd[i].begin;
            end[i] = gd[i].end;
            double n_fl = (gd[i].end - gd[i].begin) / 3;
            int n_int = int(n_fl);
            dim[i] = (n_int < 1) ? 1 : n_int;
        }
        for (int i = 0; i < 3; ++i) range[i] = end[i] - init[i];
        V3 vinit(init[0], init[1], init[2]);
        std::vector<int> relevant;
        for (size_t i = 0; i < xyz.size(); ++i)
            if (xs[i] >= 0 && xs[i] < kTypes && brick_dsqr(vinit, end, xyz[i]) < kCutoff * kCutoff)
                relevant.push_back(int(i));
        cells.assign(size_t(dim[0]) * dim[1] * dim[2], {});
        for (int x = 0; x < dim[0]; ++x)
            for (int y = 0; y < dim[1]; ++y)
                for (int z = 0; z < dim[2]; ++z) {
                    V3 b = index_to_coord(x, y, z), e = index_to_coord(x + 1, y + 1, z + 1);
                    auto& c = cells[x + dim[0] * (y + size_t(dim[1]) * z)];
                    for (int i : relevant)
                        if (brick_dsqr(b, e, xyz[i]) < kCutoff * kCutoff) c.push_back(i);
                }
    }
    static size_t fl_to_sz(double x, size_t max_sz) {  // common.h:242-247
        if (x <= 0) return 0;
        if (x >= double(max_sz)) return max_sz;
        return std::min(size_t(x), max_sz);
    }
    const std::vector<int>& possibilities(const V3& c) const {  // szv_grid.cpp:92-107
        size_t idx[3];
        for (int i = 0; i < 3; ++i)
            idx[i] = fl_to_sz((c[i] - init[i]) * dim[i] / range[i], size_t(dim[i] - 1));
        return cells[idx[0] + dim[0] * (idx[1] + size_t(dim[1]) * idx[2])];
    }
};

struct Grid {  // grid.h / grid.cpp
    double init[3], range[3], factor[3], dmo[3], finv[3];
    int n[3];  // points per dim (intervals + 1)
    std::vector<double> data;
    void setup(const GridDim gd[3]) {  // grid.cpp:29-43
        for (int i = 0; i < 3; ++i) {
            n[i] = gd[i].n + 1;
            init[i] = gd[i].begin;
            range[i] = gd[i].end - gd[i].begin;
            dmo[i] = n[i] - 1.0;
        }
        for (int i = 0; i < 3; ++i) {
            factor[i] = dmo[i] / range[i];
            finv[i] = 1 / factor[i];
        }
    }
    double at(int x, int y, int z) const { return data[x + size_t(n[0]) * (y + size_t(n[1]) * z)]; }
    V3 index_to_argument(int x, int y, int z) const {  // grid.h:48-52
        return V3(init[0] + finv[0] * x, init[1] + finv[1] * y, init[2] + finv[2] * z);
    }
    // grid.cpp:50-160
    double evaluate(const V3& loc, double slope, double v, V3* deriv) const {
        V3 s;
        for (int i = 0; i < 3; ++i) s[i] = (loc[i] - init[i]) * factor[i];
        V3 miss;
        int region[3];
        size_t a[3];
        for (int i = 0; i < 3; ++i) {
            if (s[i] < 0) {
                miss[i] = -s[i]; region[i] = -1; a[i] = 0; s[i] = 0;
            } else if (s[i] >= dmo[i]) {
                miss[i] = s[i] - dmo[i]; region[i] = 1; a[i] = n[i] - 2; s[i] = 1;
            } else {
                region[i] = 0; a[i] = size_t(s[i]); s[i] -= a[i];
            }
        }
        const double penalty = slope * (miss[0] * finv[0] + miss[1] * finv[1] + miss[2] * finv[2]);
        const int x0 = int(a[0]), y0 = int(a[1]), z0 = int(a[2]);
        const int x1 = x0 + 1, y1 = y0 + 1, z1 = z0 + 1;
        const double f000 = at(x0, y0, z0), f100 = at(x1, y0, z0), f010 = at(x0, y1, z0),
                     f110 = at(x1, y1, z0), f001 = at(x0, y0, z1), f101 = at(x1, y0, z1),
                     f011 = at(x0, y1, z1), f111 = at(x1, y1, z1);
        const double x = s[0], y = s[1], z = s[2];
        const double mx = 1 - x, my = 1 - y, mz = 1 - z;
        double f = f000 * mx * my * mz + f100 * x * my * mz + f010 * mx * y * mz +
                   f110 * x * y * mz + f001 * mx * my * z + f101 * x * my * z +
                   f011 * mx * y * z + f111 * x * y * z;
        if (deriv) {
            const double x_g = f000 * (-1) * my * mz + f100 * 1 * my * mz + f010 * (-1) * y * mz +
                               f110 * 1 * y * mz + f001 * (-1) * my * z + f101 * 1 * my * z +
                               f011 * (-1) * y * z + f111 * 1 * y * z;
            const double y_g = f000 * mx * (-1) * mz + f100 * x * (-1) * mz + f010 * mx * 1 * mz +
                               f110 * x * 1 * mz + f001 * mx * (-1) * z + f101 * x * (-1) * z +
                               f011 * mx * 1 * z + f111 * x * 1 * z;
            const double z_g = f000 * mx * my * (-1) + f100 * x * my * (-1) + f010 * mx * y * (-1) +
                               f110 * x * y * (-1) + f001 * mx * my * 1 + f101 * x * my * 1 +
                               f011 * mx * y * 1 + f111 * x * y * 1;
            V3 grad(x_g, y_g, z_g);
            double sc = curl(f, v);
            grad = (sc * sc) * grad;
            for (int i = 0; i < 3; ++i) {
                double ge = (region[i] == 0) ? grad[i] : 0;
                (*deriv)[i] = factor[i] * ge + slope * region[i];
            }
            return f + penalty;
        }
        curl(f, v);
        return f + penalty;
    }
};

// ------------------------------------------------------------ ligand model
struct Pair { int a, b, tp; };
struct Lig {
    int na = 0, nn = 0;
    std::vector<V3> local;        // coords relative to the owning node's origin
    std::vector<int> xs, el, node;
    std::vector<int> parent, nbegin, nend;
    std::vector<std::vector<int>> children;
    std::vector<V3> origin0, rel_origin, rel_axis;
    std::vector<Pair> pairs;
    double num_tors = 0;
    int ntors() const { return nn - 1; }
};

struct Frames {
    std::vector<V3> origin, axis;
    std::vector<Q> q;
    std::vector<M3> R;
    std::vector<V3> coords;
};

// tree.h:282-292 (segment::set_conf), 165-171 (rigid_body), 395-400 (heterotree)
void set_conf(const Lig& L, const double* conf, Frames& F) {
    F.origin.resize(L.nn); F.axis.resize(L.nn); F.q.resize(L.nn); F.R.resize(L.nn);
    F.coords.resize(L.na);
    F.origin[0] = V3(conf[0], conf[1], conf[2]);
    F.q[0] = {conf[3], conf[4], conf[5], conf[6]};
    F.R[0] = quaternion_to_r3(F.q[0]);
    for (int k = 1; k < L.nn; ++k) {  // DFS pre-order == node index order
        const int p = L.parent[k];
        F.origin[k] = F.origin[p] + mv(F.R[p], L.rel_origin[k]);
        F.axis[k] = mv(F.R[p], L.rel_axis[k]);
        Q t = qmul(angle_to_quaternion(F.axis[k], conf[7 + k - 1]), F.q[p]);
        quaternion_normalize_approx(t);
        F.q[k] = t;
        F.R[k] = quaternion_to_r3(t);
    }
    for (int i = 0; i < L.na; ++i) {
        const int k = L.node[i];
        F.coords[i] = F.origin[k] + mv(F.R[k], L.local[i]);
    }
}

// tree.h:169-178, 341-348, 373-380, 416-422: bottom-up force/torque sums.
void derivative_rec(const Lig& L, const Frames& F, const std::vector<V3>& f, int k, V3& force,
                    V3& torque, double* g) {
    force = V3(); torque = V3();
    for (int i = L.nbegin[k]; i < L.nend[k]; ++i) {
        force += f[i];
        torque += cross(F.coords[i] - F.origin[k], f[i]);
    }
    for (int c : L.children[k]) {
        V3 cf, ct;
        derivative_rec(L, F, f, c, cf, ct, g);
        force += cf;
        torque += cross(F.origin[c] - F.origin[k], cf) + ct;
    }
    if (k > 0) g[6 + k - 1] = dot(torque, F.axis[k]);
}
void derivative(const Lig& L, const Frames& F, const std::vector<V3>& f, double* g) {
    V3 force, torque;
    derivative_rec(L, F, f, 0, force, torque, g);
    for (int i = 0; i < 3; ++i) { g[i] = force[i]; g[3 + i] = torque[i]; }
}

// conf.h:367-372 (ligand_conf::increment): conf += factor * change
void conf_increment(int ntors, double* x, const double* c, double factor) {
    for (int i = 0; i < 3; ++i) x[i] += factor * c[i];
    V3 rot(factor * c[3], factor * c[4], factor * c[5]);
    Q q = {x[3], x[4], x[5], x[6]};
    quaternion_increment(q, rot);
    x[3] = q.a; x[4] = q.b; x[5] = q.c; x[6] = q.d;
    for (int i = 0; i < ntors; ++i) {  // conf.h:31-37
        x[7 + i] += normalized_angle(factor * c[6 + i]);
        normalize_angle(x[7 + i]);
    }
}

// ------------------------------------------------------------ Philox
inline void mulhilo(uint32_t a, uint32_t b, uint32_t& hi, uint32_t& lo) {
    uint64_t p = uint64_t(a) * b;
    hi = uint32_t(p >> 32); lo = uint32_t(p);
}
void philox(const uint32_t c_in[4], const uint32_t k_in[2], uint32_t out[4]) {
    uint32_t c[4] = {c_in[0], c_in[1], c_in[2], c_in[3]};
    uint32_t k0 = k_in[0], k1 = k_in[1];
    for (int r = 0; r < 10; ++r) {
        uint32_t hi0, lo0, hi1, lo1;
        mulhilo(0xD2511F53u, c[0], hi0, lo0);
        mulhilo(0xCD9E8D57u, c[2], hi1, lo1);
        uint32_t n0 = hi1 ^ c[1] ^ k0, n2 = hi0 ^ c[3] ^ k1;
        c[0] = n0; c[1] = lo1; c[2] = n2; c[3] = lo0;
        k0 += 0x9E3779B9u; k1 += 0xBB67AE85u;
    }
    for (int i = 0; i < 4; ++i) out[i] = c[i];
}
inline double u01(uint32_t u) { return double(float(u >> 8) * (1.0f / 16777216.0f)); }
inline double u01_open(uint32_t u) { return double(float((u >> 8) + 1) * (1.0f / 16777216.0f)); }

}  // namespace

// ------------------------------------------------------------ context
struct or_ctx {
    double w[6];
    Precalc prec;
    std::vector<V3> rec_xyz;
    std::vector<int> rec_xs;
    GridDim gd[3];
    bool has_box = false;
    CellList cl;
    bool cl_ready = false;
    Grid grids[kTypes];
    bool grid_ok[kTypes] = {};
    std::vector<Lig> ligs;
};

namespace {

void ensure_cells(or_ctx* c) {
    if (!c->cl_ready) { c->cl.build(c->gd, c->rec_xyz, c->rec_xs); c->cl_ready = true; }
}

// cache.cpp:148-208 for the listed types, points [x_begin, x_end) of dim 0.
void populate_range(or_ctx* c, const std::vector<int>& needed, int x_begin, int x_end) {
    Grid& g = c->grids[needed.front()];
    const double cutoff_sqr = kCutoff * kCutoff;
    std::vector<double> aff(needed.size());
    for (int x = x_begin; x < x_end; ++x)
        for (int y = 0; y < g.n[1]; ++y)
            for (int z = 0; z < g.n[2]; ++z) {
                std::fill(aff.begin(), aff.end(), 0.0);
                V3 probe = g.index_to_argument(x, y, z);
                const std::vector<int>& poss = c->cl.possibilities(probe);
                for (int i : poss) {
                    const int t1 = c->rec_xs[i];
                    if (t1 < 0 || t1 >= kTypes) continue;
                    const double r2 = dist_sqr(c->rec_xyz[i], probe);
                    if (r2 <= cutoff_sqr)
                        for (size_t j = 0; j < needed.size(); ++j)
                            aff[j] += c->prec.eval_fast(tri_index(t1, needed[j]), r2);
                }
                for (size_t j = 0; j < needed.size(); ++j)
                    c->grids[needed[j]].data[x + size_t(g.n[0]) * (y + size_t(g.n[1]) * z)] = aff[j];
            }
}

void build_grids(or_ctx* c, const std::vector<int>& needed, int threads) {
    ensure_cells(c);
    for (int t : needed) {
        c->grids[t].setup(c->gd);
        c->grids[t].data.assign(size_t(c->grids[t].n[0]) * c->grids[t].n[1] * c->grids[t].n[2], 0.0);
        c->grid_ok[t] = true;
    }
    const int nx = c->grids[needed.front()].n[0];
    if (threads <= 1) { populate_range(c, needed, 0, nx); return; }
    std::vector<std::thread> th;
    std::atomic<int> next(0);
    for (int t = 0; t < threads; ++t)
        th.emplace_back([&]() {
            for (;;) {
                int x = next.fetch_add(1);
                if (x >= nx) break;
                populate_range(c, needed, x, x + 1);
            }
        });
    for (auto& t : th) t.join();
}

// model.cpp:1324-1333 with cache::eval_deriv (cache.cpp:73-88) and
// eval_interacting_pairs_deriv (model.cpp:1241-1256).
double eval_deriv_cache(const or_ctx* c, const Lig& L, const double* conf, const double v[3],
                        double slope, double* g, Frames& F, std::vector<V3>& f) {
    set_conf(L, conf, F);
    f.assign(L.na, V3());
    double e = 0;
    for (int i = 0; i < L.na; ++i) {
        const int t = L.xs[i];
        if (t < 0 || t >= kTypes) continue;
        V3 d;
        e += c->grids[t].evaluate(F.coords[i], slope, v[1], g ? &d : nullptr);
        f[i] = d;
    }
    const double cutoff_sqr = kCutoff * kCutoff;
    for (const Pair& p : L.pairs) {
        V3 r = F.coords[p.b] - F.coords[p.a];
        double r2 = sqr(r);
        if (r2 < cutoff_sqr) {
            double pe, dor;
            c->prec.eval_deriv(p.tp, r2, pe, dor);
            V3 force = dor * r;
            double sc = curl(pe, v[0]);
            force = (sc * sc) * force;
            e += pe;
            f[p.a] -= force;
            f[p.b] += force;
        }
    }
    if (g) derivative(L, F, f, g);
    return e;
}

// non_cache.cpp:82-128 (eval_deriv) plus the same intra pair term.
double eval_deriv_noncache(const or_ctx* c, const Lig& L, const double* conf, const double v[3],
                           double slope, double* g, Frames& F, std::vector<V3>& f) {
    set_conf(L, conf, F);
    f.assign(L.na, V3());
    double e = 0;
    const double cutoff_sqr = kCutoff * kCutoff;
    for (int i = 0; i < L.na; ++i) {
        const int t1 = L.xs[i];
        if (t1 < 0 || t1 >= kTypes) continue;
        double this_e = 0;
        V3 deriv, oob_deriv;
        double oob = 0;
        const V3& ac = F.coords[i];
        V3 adj = ac;
        for (int j = 0; j < 3; ++j) {
            if (c->gd[j].n > 0) {
                if (ac[j] < c->gd[j].begin) { adj[j] = c->gd[j].begin; oob_deriv[j] = -1; oob += std::abs(ac[j] - c->gd[j].begin); }
                else if (ac[j] > c->gd[j].end) { adj[j] = c->gd[j].end; oob_deriv[j] = 1; oob += std::abs(ac[j] - c->gd[j].end); }
            }
        }
        oob *= slope;
        oob_deriv = slope * oob_deriv;
        for (int j : c->cl.possibilities(adj)) {
            const int t2 = c->rec_xs[j];
            if (t2 < 0 || t2 >= kTypes) continue;
            V3 r_ba = adj - c->rec_xyz[j];
            double r2 = sqr(r_ba);
            if (r2 < cutoff_sqr) {
                double pe, dor;
                c->prec.eval_deriv(tri_index(t1, t2), r2, pe, dor);
                this_e += pe;
                deriv += dor * r_ba;
            }
        }
        double sc = curl(this_e, v[1]);
        deriv = (sc * sc) * deriv;
        f[i] = deriv + oob_deriv;
        e += this_e + oob;
    }
    for (const Pair& p : L.pairs) {
        V3 r = F.coords[p.b] - F.coords[p.a];
        double r2 = sqr(r);
        if (r2 < cutoff_sqr) {
            double pe, dor;
            c->prec.eval_deriv(p.tp, r2, pe, dor);
            V3 force = dor * r;
            double sc = curl(pe, v[0]);
            force = (sc * sc) * force;
            e += pe;
            f[p.a] -= force;
            f[p.b] += force;
        }
    }
    if (g) derivative(L, F, f, g);
    return e;
}

// non_cache.cpp:20-55 (non_cache::eval) on given coordinates.
double nc_eval_coords(const or_ctx* c, const Lig& L, const std::vector<V3>& xyz, double v, double slope) {
    double e = 0;
    const double cutoff_sqr = kCutoff * kCutoff;
    for (int i = 0; i < L.na; ++i) {
        const int t1 = L.xs[i];
        if (t1 < 0 || t1 >= kTypes) continue;
        double this_e = 0, oob = 0;
        const V3& ac = xyz[i];
        V3 adj = ac;
        for (int j = 0; j < 3; ++j)
            if (c->gd[j].n > 0) {
                if (ac[j] < c->gd[j].begin) { adj[j] = c->gd[j].begin; oob += std::abs(ac[j] - c->gd[j].begin); }
                else if (ac[j] > c->gd[j].end) { adj[j] = c->gd[j].end; oob += std::abs(ac[j] - c->gd[j].end); }
            }
        oob *= slope;
        for (int j : c->cl.possibilities(adj)) {
            const int t2 = c->rec_xs[j];
            if (t2 < 0 || t2 >= kTypes) continue;
            V3 r_ba = adj - c->rec_xyz[j];
            double r2 = sqr(r_ba);
            if (r2 < cutoff_sqr) this_e += c->prec.eval_fast(tri_index(t1, t2), r2);
        }
        curl(this_e, v);
        e += this_e + oob;
    }
    return e;
}
// model.cpp:1206-1219 (eval_interacting_pairs)
double intra_fast_coords(const or_ctx* c, const Lig& L, const std::vector<V3>& xyz, double v) {
    double e = 0;
    for (const Pair& p : L.pairs) {
        double r2 = dist_sqr(xyz[p.a], xyz[p.b]);
        if (r2 < kCutoff * kCutoff) {
            double t = c->prec.eval_fast(p.tp, r2);
            curl(t, v);
            e += t;
        }
    }
    return e;
}
bool nc_within(const or_ctx* c, const Lig& L, const std::vector<V3>& xyz, double margin = 0.0001) {
    for (int i = 0; i < L.na; ++i) {  // non_cache.cpp:57-66
        if (L.el[i] == 0) continue;
        for (int j = 0; j < 3; ++j)
            if (c->gd[j].n > 0)
                if (xyz[i][j] < c->gd[j].begin - margin || xyz[i][j] > c->gd[j].end + margin) return false;
    }
    return true;
}
// weighted_terms.cpp:83-89 + everything.cpp:294-301 (num_tors_div)
double conf_independent(const or_ctx* c, const Lig& L, double x) {
    double w = 0.1 * (c->w[5] + 1);
    double y = 1 + w * L.num_tors / 5.0;
    if (std::abs(x) < kEps) return 0;
    if (std::abs(y) < kEps) return (x * y > 0) ? kMax : -kMax;
    return x / y;
}

typedef double (*EvalFn)(const or_ctx*, const Lig&, const double*, const double*, double, double*,
                         Frames&, std::vector<V3>&);

struct Objective {
    const or_ctx* c;
    const Lig* L;
    const double* v;
    double slope;
    EvalFn fn;
    int64_t evals = 0;
    Frames F;
    std::vector<V3> f;
    double operator()(const double* x, double* g) {
        ++evals;
        return fn(c, *L, x, v, slope, g, F, f);
    }
};

inline double sp(const double* a, const double* b, int n) {
    double t = 0;
    for (int i = 0; i < n; ++i) t += a[i] * b[i];
    return t;
}

// quasi_newton.cuh:1710-1806 (Lewis-Overton line search), in double.
int line_search_lo(Objective& obj, int ntors, int n, double& stp, double* x, double& f, double* g,
                   const double* d, const double* xp, const double* gp) {
    int count = 0;
    bool brackt = false;
    double mu = 0.0, nu = 1.0e+20;
    const int nc = 7 + ntors;
    double dginit = sp(gp, d, n);
    if (0.0 < dginit) return -1;
    const double finit = f, dgtest = 1.0e-4 * dginit, dstest = 0.1 * dginit;
    for (;;) {
        std::memcpy(x, xp, sizeof(double) * nc);
        conf_increment(ntors, x, d, stp);
        f = obj(x, g);
        ++count;
        if (f > finit + stp * dgtest) {
            nu = stp;
            brackt = true;
        } else {
            if (sp(g, d, n) < dstest) mu = stp;
            else return count;
        }
        if (10 <= count) return (f > finit) ? -1 : count;
        if (brackt) stp = 0.5 * (mu + nu);
        else stp *= 2.0;
    }
}

// quasi_newton.cuh:2172-2389 (rilc_bfgs_update), in double.
double rilc_bfgs(Objective& obj, int ntors, double* x, int max_steps) {
    const int n = 6 + ntors, nc = 7 + ntors;
    std::vector<double> g(n), d(n), xp(nc), gp(n), x_orig(nc), g_orig(n), s(n), y(n);
    double fx = obj(x, g.data());
    const double fx_orig = fx;
    g_orig = g;
    std::memcpy(x_orig.data(), x, sizeof(double) * nc);
    for (int i = 0; i < n; ++i) d[i] = -g[i];
    if (!(std::sqrt(sp(g.data(), g.data(), n)) >= 1e-5)) return fx;
    double step = 1.0 / std::sqrt(sp(d.data(), d.data(), n));
    int k = 1;
    for (;;) {
        std::memcpy(xp.data(), x, sizeof(double) * nc);
        gp = g;
        const double fxp = fx;
        int ls = line_search_lo(obj, ntors, n, step, x, fx, g.data(), d.data(), xp.data(), gp.data());
        if (ls < 0) {
            std::memcpy(x, xp.data(), sizeof(double) * nc);
            g = gp;
            fx = fxp;
            break;
        }
        if (!(std::sqrt(sp(g.data(), g.data(), n)) >= 1e-5)) return fx;
        if (max_steps != 0 && max_steps <= k) break;
        ++k;
        for (int i = 0; i < n; ++i) { s[i] = step * d[i]; y[i] = g[i] - gp[i]; }
        double ys = sp(y.data(), s.data(), n), yy = sp(y.data(), y.data(), n);
        for (int i = 0; i < n; ++i) d[i] = -g[i];
        double cau = sp(s.data(), s.data(), n) * std::sqrt(sp(gp.data(), gp.data(), n)) * 1.0e-6;
        if (ys > cau) {
            double alpha = sp(s.data(), d.data(), n) / ys;
            for (int i = 0; i < n; ++i) d[i] += alpha * y[i];
            for (int i = 0; i < n; ++i) d[i] *= ys / yy;
            double beta = sp(y.data(), d.data(), n) / ys;
            for (int i = 0; i < n; ++i) d[i] += (alpha - beta) * s[i];
        }
        step = 1.0;
    }
    if (!(fx <= fx_orig)) {
        fx = fx_orig;
        std::memcpy(x, x_orig.data(), sizeof(double) * nc);
    }
    return fx;
}

// lib/bfgs.h:95-140 (dense BFGS, Armijo backtracking line_search 65-82).
double dense_bfgs(Objective& obj, int ntors, double* x, int max_steps) {
    const int n = 6 + ntors, nc = 7 + ntors;
    std::vector<double> h(size_t(n) * n, 0.0);  // symmetric, full storage
    for (int i = 0; i < n; ++i) h[i * n + i] = 1;
    std::vector<double> g(n), g_new(n), x_new(nc), g_orig, x_orig(x, x + nc), p(n), y(n), minus_hy(n);
    double f0 = obj(x, g.data());
    const double f_orig = f0;
    g_orig = g;
    for (int step = 0; step < max_steps; ++step) {
        for (int i = 0; i < n; ++i) {  // minus_mat_vec_product
            double sum = 0;
            for (int j = 0; j < n; ++j) sum += h[i * n + j] * g[j];
            p[i] = -sum;
        }
        double f1 = 0, alpha = 1;
        const double pg = sp(p.data(), g.data(), n);
        for (int trial = 0; trial < 10; ++trial) {
            std::memcpy(x_new.data(), x, sizeof(double) * nc);
            conf_increment(ntors, x_new.data(), p.data(), alpha);
            f1 = obj(x_new.data(), g_new.data());
            if (f1 - f0 < 0.0001 * alpha * pg) break;
            alpha *= 0.5;
        }
        for (int i = 0; i < n; ++i) y[i] = g_new[i] - g[i];
        f0 = f1;
        std::memcpy(x, x_new.data(), sizeof(double) * nc);
        if (!(std::sqrt(sp(g.data(), g.data(), n)) >= 1e-5)) break;
        g = g_new;
        if (step == 0) {
            const double yy = sp(y.data(), y.data(), n);
            if (std::abs(yy) > kEps) {
                const double dg = alpha * sp(y.data(), p.data(), n) / yy;
                for (int i = 0; i < n; ++i) h[i * n + i] = dg;
            }
        }
        // bfgs_update, bfgs.h:49-63
        const double yp = sp(y.data(), p.data(), n);
        if (alpha * yp < kEps) continue;
        for (int i = 0; i < n; ++i) {
            double sum = 0;
            for (int j = 0; j < n; ++j) sum += h[i * n + j] * y[j];
            minus_hy[i] = -sum;
        }
        const double yhy = -sp(y.data(), minus_hy.data(), n);
        const double r = 1 / (alpha * yp);
        for (int i = 0; i < n; ++i)
            for (int j = i; j < n; ++j) {
                double upd = alpha * r * (minus_hy[i] * p[j] + minus_hy[j] * p[i]) +
                             alpha * alpha * (r * r * yhy + r) * p[i] * p[j];
                h[i * n + j] += upd;
                if (j != i) h[j * n + i] = h[i * n + j];
            }
    }
    if (!(f0 <= f_orig)) {
        f0 = f_orig;
        std::memcpy(x, x_orig.data(), sizeof(double) * nc);
    }
    return f0;
}

// Random draws shared bit-for-bit with the GPU search kernel.
struct Draw {
    uint32_t u[4];
    Draw(uint32_t seed, uint32_t lig, uint32_t chain, uint32_t step, uint32_t tag) {
        uint32_t ctr[4] = {chain, step, tag, 0x5644u}, key[2] = {seed, lig};
        philox(ctr, key, u);
    }
};
const uint32_t kInitStep = 0xFFFFFFFFu;

void init_conf(const or_ctx* c, const Lig& L, uint32_t seed, uint32_t lig, uint32_t chain, double* x) {
    Draw p(seed, lig, chain, kInitStep, 0);
    for (int i = 0; i < 3; ++i) {  // random_in_box
        double lo = c->gd[i].begin, hi = c->gd[i].end;
        x[i] = lo + u01(p.u[i]) * (hi - lo);
    }
    Draw q(seed, lig, chain, kInitStep, 1);  // random_orientation: normalised 4-D Gaussian
    double r0 = std::sqrt(-2.0 * std::log(u01_open(q.u[0]))), r1 = std::sqrt(-2.0 * std::log(u01_open(q.u[2])));
    double a0 = 2 * kPi * u01(q.u[1]), a1 = 2 * kPi * u01(q.u[3]);
    double n4[4] = {r0 * std::cos(a0), r0 * std::sin(a0), r1 * std::cos(a1), r1 * std::sin(a1)};
    double nrm = std::sqrt(n4[0] * n4[0] + n4[1] * n4[1] + n4[2] * n4[2] + n4[3] * n4[3]);
    if (!(nrm > 1e-6)) { n4[0] = 1; n4[1] = n4[2] = n4[3] = 0; nrm = 1; }
    for (int i = 0; i < 4; ++i) x[3 + i] = n4[i] / nrm;
    for (int t = 0; t < L.ntors(); t += 4) {
        Draw d(seed, lig, chain, kInitStep, 2 + t / 4);
        for (int j = 0; j < 4 && t + j < L.ntors(); ++j) x[7 + t + j] = -kPi + 2 * kPi * u01(d.u[j]);
    }
}

V3 sphere_point(uint32_t u1, uint32_t u2, uint32_t u3) {  // uniform inside the unit ball
    double z = 2.0 * u01(u1) - 1.0, phi = 2 * kPi * u01(u2), r = std::cbrt(u01(u3));
    double s = std::sqrt(std::max(0.0, 1.0 - z * z));
    return V3(r * s * std::cos(phi), r * s * std::sin(phi), r * z);
}

double gyration_radius(const Lig& L, const Frames& F) {  // model.cpp:1161-1175
    double acc = 0;
    int cnt = 0;
    for (int i = 0; i < L.na; ++i)
        if (L.el[i] != 0) { acc += dist_sqr(F.coords[i], F.origin[0]); ++cnt; }
    return cnt > 0 ? std::sqrt(acc / cnt) : 0;
}

// mutate.cpp:62-127 with a Philox-driven choice; returns nothing.
void mutate(const Lig& L, double* x, uint32_t seed, uint32_t lig, uint32_t chain, uint32_t step,
            double amplitude, Frames& F) {
    Draw a(seed, lig, chain, step, 0), b(seed, lig, chain, step, 1);
    const int ntors = L.ntors();
    const int m = 2 + ntors;
    int which = int(u01(a.u[0]) * m);
    if (which > m - 1) which = m - 1;
    V3 sp3 = sphere_point(a.u[1], a.u[2], a.u[3]);
    if (which == 0) {
        for (int i = 0; i < 3; ++i) x[i] += amplitude * sp3[i];
        return;
    }
    if (which == 1) {
        set_conf(L, x, F);
        double gr = gyration_radius(L, F);
        if (gr > kEps) {
            V3 rot = (amplitude / gr) * sp3;
            Q q = {x[3], x[4], x[5], x[6]};
            quaternion_increment(q, rot);
            x[3] = q.a; x[4] = q.b; x[5] = q.c; x[6] = q.d;
        }
        return;
    }
    x[7 + which - 2] = -kPi + 2 * kPi * u01(b.u[0]);
}

// kernel2.cu:219-426: MC chain with RILC-BFGS local search; with s.dense,
// kernel2.cu:427-563: dense BFGS (bfgs_optimized, quasi_newton.cuh:2391-2499)
// and no effective re-optimisation of an accepted pose that beats the best:
// that branch re-optimises a copy (`candidate`) and then keeps `tmp`, whose
// energy it did not change (kernel2.cu:526-552), so the best pose and energy
// are the accepted candidate's.
double mc_chain(const or_ctx* c, const Lig& L, const or_search& s, uint32_t chain, double* best,
                int64_t& evals) {
    if (s.dense) {
        const int nc = 7 + L.ntors();
        Objective obj{c, &L, s.hunt_cap, s.slope, eval_deriv_cache};
        std::vector<double> tmp(nc), cand(nc);
        init_conf(c, L, s.seed, s.lig_uid, chain, tmp.data());
        double tmp_e = kMax, best_e = std::numeric_limits<double>::infinity();
        std::memcpy(best, tmp.data(), sizeof(double) * nc);
        for (int step = 0; step < s.search_depth; ++step) {
            cand = tmp;
            mutate(L, cand.data(), s.seed, s.lig_uid, chain, uint32_t(step), s.amplitude, obj.F);
            const double ce = dense_bfgs(obj, L.ntors(), cand.data(), s.max_bfgs_steps);
            Draw b(s.seed, s.lig_uid, chain, uint32_t(step), 1);
            const bool acc = step == 0 || ce < tmp_e || u01(b.u[1]) < std::exp((tmp_e - ce) / s.temperature);
            if (acc) {
                tmp = cand;
                tmp_e = ce;
                if (tmp_e < best_e) {
                    best_e = tmp_e;
                    std::memcpy(best, tmp.data(), sizeof(double) * nc);
                }
            }
        }
        evals += obj.evals;
        return best_e;
    }
    const int nc = 7 + L.ntors();
    Objective obj{c, &L, s.hunt_cap, s.slope, eval_deriv_cache};
    std::vector<double> tmp(nc), cand(nc), g(6 + L.ntors());
    init_conf(c, L, s.seed, s.lig_uid, chain, tmp.data());
    double tmp_e = kMax, best_e = std::numeric_limits<double>::infinity();
    std::memcpy(best, tmp.data(), sizeof(double) * nc);
    // QuickVina2-CUDA's visited history (visited.cuh:48-227): rilc_bfgs_update
    // evaluates the entry pose, and unless interesting() holds returns it with
    // that energy (quasi_newton.cuh:1937-1943); interesting() is true until the
    // history holds 10*(6+ntors) entries (one add() per optimisation run) and
    // then consults check(), which returns false on every path
    // (visited.cuh:91-166).  So a chain runs its first 10*(6+ntors)
    // optimisations and keeps every later candidate's entry energy.
    const int history = 10 * (6 + L.ntors());
    int runs = 0;
    auto local_search = [&](double* x) {
        if (s.visited && runs >= history) return obj(x, g.data());
        ++runs;
        return rilc_bfgs(obj, L.ntors(), x, s.max_bfgs_steps);
    };
    for (int step = 0; step < s.search_depth; ++step) {
        cand = tmp;
        mutate(L, cand.data(), s.seed, s.lig_uid, chain, uint32_t(step), s.amplitude, obj.F);
        double ce = local_search(cand.data());
        Draw b(s.seed, s.lig_uid, chain, uint32_t(step), 1);
        bool acc = step == 0 || ce < tmp_e ||
                   u01(b.u[1]) < std::exp((tmp_e - ce) / s.temperature);  // kernel2.cu:63-71
        if (acc) {
            tmp = cand;
            tmp_e = ce;
            if (tmp_e < best_e) {
                tmp_e = local_search(tmp.data());
                if (tmp_e < best_e) {
                    best_e = tmp_e;
                    std::memcpy(best, tmp.data(), sizeof(double) * nc);
                }
            }
        }
    }
    evals += obj.evals;
    return best_e;
}

Lig make_lig(const or_ligand* d) {
    Lig L;
    L.na = d->n_atoms;
    L.nn = d->n_nodes;
    std::vector<V3> xyz(L.na);
    for (int i = 0; i < L.na; ++i) xyz[i] = V3(d->xyz[3 * i], d->xyz[3 * i + 1], d->xyz[3 * i + 2]);
    L.xs.assign(d->xs, d->xs + L.na);
    L.el.assign(d->el, d->el + L.na);
    L.node.assign(d->atom_node, d->atom_node + L.na);
    L.parent.assign(d->node_parent, d->node_parent + L.nn);
    L.nbegin.assign(L.nn, L.na);
    L.nend.assign(L.nn, 0);
    for (int i = 0; i < L.na; ++i) {
        L.nbegin[L.node[i]] = std::min(L.nbegin[L.node[i]], i);
        L.nend[L.node[i]] = std::max(L.nend[L.node[i]], i + 1);
    }
    for (int k = 0; k < L.nn; ++k) if (L.nbegin[k] > L.nend[k]) L.nbegin[k] = L.nend[k] = 0;
    L.children.assign(L.nn, {});
    for (int k = 1; k < L.nn; ++k) L.children[L.parent[k]].push_back(k);
    L.origin0.resize(L.nn);
    L.rel_origin.resize(L.nn);
    L.rel_axis.resize(L.nn);
    for (int k = 0; k < L.nn; ++k) L.origin0[k] = xyz[d->node_origin_atom[k]];
    for (int k = 1; k < L.nn; ++k) {  // tree.h:230-237 (axis_frame), 258-262 (segment)
        V3 diff = L.origin0[k] - xyz[d->node_axis_atom[k]];
        double nrm = std::sqrt(sqr(diff));
        L.rel_axis[k] = (1 / nrm) * diff;
        L.rel_origin[k] = L.origin0[k] - L.origin0[L.parent[k]];
    }
    L.local.resize(L.na);
    for (int i = 0; i < L.na; ++i) L.local[i] = xyz[i] - L.origin0[L.node[i]];
    for (int p = 0; p < d->n_pairs; ++p) {
        int a = d->pairs[2 * p], b = d->pairs[2 * p + 1];
        if (L.xs[a] < 0 || L.xs[b] < 0) continue;
        L.pairs.push_back({a, b, tri_index(L.xs[a], L.xs[b])});
    }
    L.num_tors = d->num_tors;
    return L;
}

std::vector<V3> to_v3(const double* p, int n) {
    std::vector<V3> v(n);
    for (int i = 0; i < n; ++i) v[i] = V3(p[3 * i], p[3 * i + 1], p[3 * i + 2]);
    return v;
}

}  // namespace

// ------------------------------------------------------------ C API
extern "C" {

or_ctx* or_create(const double weights[6]) {
    or_ctx* c = new or_ctx();
    std::memcpy(c->w, weights, sizeof(c->w));
    c->prec.build(weights);
    return c;
}
void or_destroy(or_ctx* c) { delete c; }

void or_tables(or_ctx* c, double* fast, double* se, double* sd) {
    const size_t n = size_t(kPairs) * kN;
    if (fast) std::memcpy(fast, c->prec.fast.data(), n * sizeof(double));
    if (se) std::memcpy(se, c->prec.se.data(), n * sizeof(double));
    if (sd) std::memcpy(sd, c->prec.sd.data(), n * sizeof(double));
}

int or_set_receptor(or_ctx* c, int n, const double* xyz, const int32_t* xs) {
    c->rec_xyz = to_v3(xyz, n);
    c->rec_xs.assign(xs, xs + n);
    c->cl_ready = false;
    for (bool& b : c->grid_ok) b = false;
    return 0;
}

int or_set_box(or_ctx* c, const double center[3], const double size[3]) {
    const double granularity = 0.375;  // main.cpp:864-876
    for (int i = 0; i < 3; ++i) {
        c->gd[i].n = int(std::ceil(size[i] / granularity));
        double real_span = granularity * c->gd[i].n;
        c->gd[i].begin = center[i] - real_span / 2;
        c->gd[i].end = c->gd[i].begin + real_span;
    }
    c->has_box = true;
    c->cl_ready = false;
    for (bool& b : c->grid_ok) b = false;
    return 0;
}

void or_grid_info(or_ctx* c, int32_t npts[3], double begin[3], double end[3]) {
    for (int i = 0; i < 3; ++i) {
        npts[i] = c->gd[i].n + 1;
        begin[i] = c->gd[i].begin;
        end[i] = c->gd[i].end;
    }
}

int or_build_grids(or_ctx* c, const int32_t* types, int n_types) {
    if (!c->has_box || n_types <= 0) return -1;
    std::vector<int> needed(types, types + n_types);
    unsigned hw = std::thread::hardware_concurrency();
    build_grids(c, needed, int(hw ? hw : 1));
    return 0;
}

double or_grid_seconds(or_ctx* c, const int32_t* types, int n_types, int threads) {
    std::vector<int> needed(types, types + n_types);
    ensure_cells(c);
    auto t0 = std::chrono::steady_clock::now();
    build_grids(c, needed, threads);
    auto t1 = std::chrono::steady_clock::now();
    return std::chrono::duration<double>(t1 - t0).count();
}

int or_get_grid(or_ctx* c, int t, double* out) {
    if (t < 0 || t >= kTypes || !c->grid_ok[t]) return -1;
    std::memcpy(out, c->grids[t].data.data(), c->grids[t].data.size() * sizeof(double));
    return 0;
}

int or_add_ligand(or_ctx* c, const or_ligand* d) {
    ensure_cells(c);
    c->ligs.push_back(make_lig(d));
    return int(c->ligs.size()) - 1;
}
int or_ligand_ntors(or_ctx* c, int lig) { return c->ligs[lig].ntors(); }

// 1 when a map exists for every heavy-atom type of the ligand (the cached
// evaluation reads them); entry points that need the maps return NaN / -1
// otherwise instead of reading an empty map.
int or_maps_ready(or_ctx* c, int lig) {
    for (int t : c->ligs[lig].xs)
        if (t >= 0 && t < kTypes && c->grids[t].data.empty()) return 0;
    return 1;
}

double or_eval_deriv(or_ctx* c, int lig, const double* conf, const double v[3], double slope, double* grad) {
    if (!or_maps_ready(c, lig)) return std::nan("");
    Frames F;
    std::vector<V3> f;
    return eval_deriv_cache(c, c->ligs[lig], conf, v, slope, grad, F, f);
}

double or_nc_eval_deriv(or_ctx* c, int lig, const double* conf, const double v[3], double slope, double* grad) {
    Frames F;
    std::vector<V3> f;
    return eval_deriv_noncache(c, c->ligs[lig], conf, v, slope, grad, F, f);
}

void or_coords(or_ctx* c, int lig, const double* conf, double* out) {
    Frames F;
    const Lig& L = c->ligs[lig];
    set_conf(L, conf, F);
    for (int i = 0; i < L.na; ++i)
        for (int j = 0; j < 3; ++j) out[3 * i + j] = F.coords[i][j];
}

double or_eval_intramolecular(or_ctx* c, int lig, const double* conf, double v_intra) {
    Frames F;
    const Lig& L = c->ligs[lig];
    set_conf(L, conf, F);  // model.cpp:1375-1420 (ligand part)
    return intra_fast_coords(c, L, F.coords, v_intra);
}

double or_intramolecular_coords(or_ctx* c, int lig, const double* xyz) {
    const Lig& L = c->ligs[lig];
    return intra_fast_coords(c, L, to_v3(xyz, L.na), 1000.0);
}

// model.cpp:1428-1431: conf_independent(eval(c) - intra_best) with authentic_v
double or_eval_adjusted_coords(or_ctx* c, int lig, const double* xyz, double intra_best) {
    const Lig& L = c->ligs[lig];
    std::vector<V3> v = to_v3(xyz, L.na);
    double e = nc_eval_coords(c, L, v, 1000.0, 1e6) + intra_fast_coords(c, L, v, 1000.0);
    return conf_independent(c, L, e - intra_best);
}
// terms.cpp:385-446 (evale_robust): the five unweighted intermolecular
// terms, evaluated analytically at each ligand-receptor heavy-atom distance
// up to the 8 A cutoff (what --score_only prints, main.cpp:191-218).
void or_term_values_coords(or_ctx* c, int lig, const double* xyz, double out[5]) {
    const Lig& L = c->ligs[lig];
    const std::vector<V3> v = to_v3(xyz, L.na);
    for (int k = 0; k < 5; ++k) out[k] = 0;
    for (int i = 0; i < L.na; ++i) {
        if (L.xs[i] < 0 || L.xs[i] >= kTypes) continue;
        for (size_t j = 0; j < c->rec_xyz.size(); ++j) {
            const int t2 = c->rec_xs[j];
            if (t2 < 0 || t2 >= kTypes) continue;
            const double d2 = dist_sqr(v[i], c->rec_xyz[j]);
            if (d2 > kCutoff * kCutoff) continue;
            double t[5];
            raw_terms(L.xs[i], t2, std::sqrt(d2), t);
            for (int k = 0; k < 5; ++k) out[k] += t[k];
        }
    }
}
double or_conf_independent(or_ctx* c, int lig, double x) { return conf_independent(c, c->ligs[lig], x); }

double or_eval_adjusted(or_ctx* c, int lig, const double* conf, double intra_best) {
    Frames F;
    const Lig& L = c->ligs[lig];
    set_conf(L, conf, F);
    double e = nc_eval_coords(c, L, F.coords, 1000.0, 1e6) + intra_fast_coords(c, L, F.coords, 1000.0);
    return conf_independent(c, L, e - intra_best);
}

// model.cpp:1509-1523
double or_rmsd_upper(or_ctx* c, int lig, const double* a, const double* b) {
    const Lig& L = c->ligs[lig];
    double sum = 0;
    int cnt = 0;
    for (int i = 0; i < L.na; ++i)
        if (L.el[i] != 0) {
            sum += sqr(a[3 * i] - b[3 * i]) + sqr(a[3 * i + 1] - b[3 * i + 1]) + sqr(a[3 * i + 2] - b[3 * i + 2]);
            ++cnt;
        }
    return cnt ? std::sqrt(sum / cnt) : 0;
}
// model.cpp:1485-1507
static double rmsd_lb_asym(const Lig& L, const double* x, const double* y) {
    double sum = 0;
    int cnt = 0;
    for (int i = 0; i < L.na; ++i) {
        if (L.el[i] == 0) continue;
        double r2 = kMax;
        for (int j = 0; j < L.na; ++j)
            if (L.el[i] == L.el[j] && L.el[j] != 0) {
                double t = sqr(x[3 * i] - y[3 * j]) + sqr(x[3 * i + 1] - y[3 * j + 1]) + sqr(x[3 * i + 2] - y[3 * j + 2]);
                if (t < r2) r2 = t;
            }
        sum += r2;
        ++cnt;
    }
    return cnt ? std::sqrt(sum / cnt) : 0;
}
double or_rmsd_lower(or_ctx* c, int lig, const double* a, const double* b) {
    const Lig& L = c->ligs[lig];
    return std::max(rmsd_lb_asym(L, a, b), rmsd_lb_asym(L, b, a));
}

double or_rilc_bfgs(or_ctx* c, int lig, double* conf, const double v[3], double slope, int max_steps,
                    int64_t* evals) {
    if (!or_maps_ready(c, lig)) return std::nan("");
    const Lig& L = c->ligs[lig];
    Objective obj{c, &L, v, slope, eval_deriv_cache};
    double e = rilc_bfgs(obj, L.ntors(), conf, max_steps);
    if (evals) *evals = obj.evals;
    return e;
}

double or_bfgs(or_ctx* c, int lig, double* conf, const double v[3], double slope, int max_steps,
               int use_noncache, int64_t* evals) {
    if (!use_noncache && !or_maps_ready(c, lig)) return std::nan("");
    const Lig& L = c->ligs[lig];
    Objective obj{c, &L, v, slope, use_noncache ? eval_deriv_noncache : eval_deriv_cache};
    double e = dense_bfgs(obj, L.ntors(), conf, max_steps);
    if (evals) *evals = obj.evals;
    return e;
}

void or_init_conf(or_ctx* c, int lig, uint32_t seed, uint32_t lig_uid, uint32_t chain, double* conf) {
    init_conf(c, c->ligs[lig], seed, lig_uid, chain, conf);
}

int64_t or_mc_chains(or_ctx* c, int lig, const or_search* s, int cb, int ce, double* out_conf,
                     double* out_e, int threads) {
    if (!or_maps_ready(c, lig)) return -1;
    const Lig& L = c->ligs[lig];
    const int nc = 7 + L.ntors();
    std::atomic<int> next(cb);
    std::atomic<int64_t> total(0);
    auto work = [&]() {
        int64_t ev = 0;
        for (;;) {
            int ch = next.fetch_add(1);
            if (ch >= ce) break;
            out_e[ch - cb] = mc_chain(c, L, *s, uint32_t(ch), out_conf + size_t(ch - cb) * nc, ev);
        }
        total += ev;
    };
    if (threads <= 1) work();
    else {
        std::vector<std::thread> th;
        for (int t = 0; t < threads; ++t) th.emplace_back(work);
        for (auto& t : th) t.join();
    }
    return total.load();
}

// main.cpp:139-157 (refine_structure) with the authentic cap (1000).
double or_refine(or_ctx* c, int lig, double* conf, int max_steps, int64_t* evals) {
    const Lig& L = c->ligs[lig];
    const double v[3] = {1000, 1000, 1000};
    int64_t ev = 0;
    double e = 0;
    Frames F;
    for (int p = 0; p < 5; ++p) {
        double slope = 100 * std::pow(10.0, 2.0 * p);
        Objective obj{c, &L, v, slope, eval_deriv_noncache};
        e = dense_bfgs(obj, L.ntors(), conf, max_steps);
        ev += obj.evals;
        set_conf(L, conf, F);
        if (nc_within(c, L, F.coords)) break;
    }
    set_conf(L, conf, F);
    if (!nc_within(c, L, F.coords)) e = kMax;
    if (evals) *evals = ev;
    return e;
}

int or_cluster(or_ctx* c, int lig, int n, const double* confs, const double* e, double min_rmsd,
               int max_keep, int32_t* kept) {
    const Lig& L = c->ligs[lig];
    const int nc = 7 + L.ntors();
    std::vector<int> order(n);
    for (int i = 0; i < n; ++i) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return e[a] < e[b]; });
    std::vector<std::vector<double>> kc;
    Frames F;
    int nk = 0;
    for (int idx : order) {
        if (nk >= max_keep) break;
        set_conf(L, confs + size_t(idx) * nc, F);
        std::vector<double> xyz(3 * L.na);
        for (int i = 0; i < L.na; ++i)
            for (int j = 0; j < 3; ++j) xyz[3 * i + j] = F.coords[i][j];
        bool close = false;
        for (auto& k : kc)
            if (or_rmsd_upper(c, lig, xyz.data(), k.data()) < min_rmsd) { close = true; break; }
        if (close) continue;
        kc.push_back(xyz);
        kept[nk++] = idx;
    }
    return nk;
}

void or_philox(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) { philox(ctr, key, out); }

}  // extern "C"
