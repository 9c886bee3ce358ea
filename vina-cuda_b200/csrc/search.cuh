// Warp-level local optimisation and Monte-Carlo moves (FP32).
//
// Vectors of the 6+ntors pose space are spread over the warp: component c
// lives in lane c%32, slot c/32.  The pose (7+ntors floats) lives in shared
// memory because the kinematics of every lane reads it.
#pragma once

#include <cfloat>

#include "eval.cuh"

namespace vd {

constexpr float kPiF = 3.14159265358979f;

// ---------------------------------------------------------------- Philox
// Philox4x32-10 (Salmon et al., SC'11); the oracle uses the same streams.
__host__ __device__ __forceinline__ void philox4x32(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3,
                                                    uint32_t k0, uint32_t k1, uint32_t out[4]) {
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        const uint64_t p0 = uint64_t(0xD2511F53u) * c0, p1 = uint64_t(0xCD9E8D57u) * c2;
        const uint32_t hi0 = uint32_t(p0 >> 32), lo0 = uint32_t(p0), hi1 = uint32_t(p1 >> 32), lo1 = uint32_t(p1);
        const uint32_t n0 = hi1 ^ c1 ^ k0, n2 = hi0 ^ c3 ^ k1;
        c0 = n0; c1 = lo1; c2 = n2; c3 = lo0;
        k0 += 0x9E3779B9u; k1 += 0xBB67AE85u;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}
constexpr uint32_t kInitStep = 0xFFFFFFFFu;
constexpr uint32_t kStreamTag = 0x5644u;
__device__ __forceinline__ void draw(uint32_t seed, uint32_t lig, uint32_t chain, uint32_t step, uint32_t tag,
                                     uint32_t u[4]) {
    philox4x32(chain, step, tag, kStreamTag, seed, lig, u);
}
__device__ __forceinline__ float u01(uint32_t u) { return float(u >> 8) * (1.0f / 16777216.0f); }
__device__ __forceinline__ float u01_open(uint32_t u) { return float((u >> 8) + 1) * (1.0f / 16777216.0f); }

// ---------------------------------------------------------------- helpers
__device__ __forceinline__ float norm_angle(float x) {  // common.h:316-340
    if (x > 3.f * kPiF) x -= 2.f * kPiF * ceilf((x - kPiF) / (2.f * kPiF));
    else if (x < -3.f * kPiF) x += 2.f * kPiF * ceilf((-x - kPiF) / (2.f * kPiF));
    if (x > kPiF) x -= 2.f * kPiF;
    else if (x < -kPiF) x += 2.f * kPiF;
    return x;
}
// q <- angle_to_quaternion(rot) * q, normalised (quaternion.cpp:235-240)
__device__ __forceinline__ float4 quat_increment(float4 q, float r0, float r1, float r2) {
    const float ang = sqrtf(r0 * r0 + r1 * r1 + r2 * r2);
    if (ang > FLT_EPSILON) {
        const float inv = __fdividef(1.f, ang);
        float s, c;
        __sincosf(0.5f * norm_angle(ang), &s, &c);
        q = qmul(make_float4(c, s * r0 * inv, s * r1 * inv, s * r2 * inv), q);
    }
    const float n2 = q.x * q.x + q.y * q.y + q.z * q.z + q.w * q.w;
    if (fabsf(n2 - 1.f) >= 1e-6f) {
        const float inv = rsqrtf(n2);
        q = make_float4(q.x * inv, q.y * inv, q.z * inv, q.w * inv);
    }
    return q;
}

struct Vec2 {  // one lane's share of a pose-space vector
    float a, b;
};
__device__ __forceinline__ float lane_dot(Vec2 x, Vec2 y) { return x.a * y.a + x.b * y.b; }
__device__ __forceinline__ float vdot(Vec2 x, Vec2 y) { return warp_sum(lane_dot(x, y)); }
// N independent dot products in one butterfly: each sum takes the same
// steps as warp_sum, so the values equal N separate vdot calls.
template <int N>
__device__ __forceinline__ void warp_sum_n(float (&v)[N]) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
#pragma unroll
        for (int j = 0; j < N; ++j) v[j] += __shfl_xor_sync(0xffffffffu, v[j], o);
}
// Six sums over the warp, every lane getting all six: a reduce-scatter
// (lanes exchange half of their partial sums with the lane 16, 8, then 4
// away, so each lane ends with one of the sums over 8 lanes), a butterfly
// over the remaining 4 lanes, then one broadcast per sum: 15 shuffles
// instead of the 30 of six butterflies.
__device__ __forceinline__ void warp_sum6(float (&v)[6], int lane) {
    const unsigned full = 0xffffffffu;
    const bool h16 = lane & 16, h8 = lane & 8, h4 = lane & 4;
    const float w[8] = {v[0], v[1], v[2], v[3], v[4], v[5], 0.f, 0.f};
    float a[4], b[2];
#pragma unroll
    for (int j = 0; j < 4; ++j) {  // sums 4*h16 + j
        const float keep = h16 ? w[j + 4] : w[j], give = h16 ? w[j] : w[j + 4];
        a[j] = keep + __shfl_xor_sync(full, give, 16);
    }
#pragma unroll
    for (int j = 0; j < 2; ++j) {  // sums 4*h16 + 2*h8 + j
        const float keep = h8 ? a[j + 2] : a[j], give = h8 ? a[j] : a[j + 2];
        b[j] = keep + __shfl_xor_sync(full, give, 8);
    }
    float c = (h4 ? b[1] : b[0]) + __shfl_xor_sync(full, h4 ? b[0] : b[1], 4);  // sum 4*h16 + 2*h8 + h4
    c += __shfl_xor_sync(full, c, 2);
    c += __shfl_xor_sync(full, c, 1);
#pragma unroll
    for (int j = 0; j < 6; ++j) v[j] = __shfl_sync(full, c, (j & 7) << 2);
}
__device__ __forceinline__ Vec2 vload(const float* g, int n, int lane) {
    Vec2 v;
    v.a = (lane < n) ? g[lane] : 0.f;
    v.b = (lane + 32 < n) ? g[lane + 32] : 0.f;
    return v;
}

// x = xp + alpha * d (conf.h:367-372); xp, x in shared memory.  Lanes 0-2
// step the position components they hold; lane 3 rotates the orientation
// by the rotation vector in lanes 3-5.
__device__ __forceinline__ void conf_step(const float* xp, float* x, Vec2 d, float alpha, int nt, int lane) {
    const float d4 = __shfl_down_sync(0xffffffffu, d.a, 1), d5 = __shfl_down_sync(0xffffffffu, d.a, 2);
    if (lane < 3) x[lane] = xp[lane] + alpha * d.a;
    if (lane == 3) {
        const float4 q = quat_increment(make_float4(xp[3], xp[4], xp[5], xp[6]), alpha * d.a, alpha * d4, alpha * d5);
        x[3] = q.x; x[4] = q.y; x[5] = q.z; x[6] = q.w;
    }
    const int t0 = lane - 6, t1 = lane + 26;  // torsion held in slot a / b
    if (t0 >= 0 && t0 < nt) x[7 + t0] = norm_angle(xp[7 + t0] + norm_angle(alpha * d.a));
    if (t1 < nt) x[7 + t1] = norm_angle(xp[7 + t1] + norm_angle(alpha * d.b));
    __syncwarp();
}

__device__ __forceinline__ void copy_conf(const float* src, float* dst, int nc, int lane) {
    for (int i = lane; i < nc; i += 32) dst[i] = src[i];
    __syncwarp();
}

struct SearchMem {  // per-warp shared memory of the optimiser
    WarpMem m;      // m.x is the working pose
    float* xp;      // previous pose in the line search
    float* xo;      // pose at entry (restored if the run got worse)
};

// quasi_newton.cuh:2172-2389 (RILC-BFGS) with the Lewis-Overton line search
// of quasi_newton.cuh:1710-1806, on the pose in s.m.x.  Returns the energy;
// s.m.x holds the optimised pose.  *evals counts energy+gradient calls
// (a trial whose adjoint is skipped counts as one, as the reference's
// evaluation count does).
//
// The loop has one evaluation site: the entry evaluation and every
// line-search trial run through the same inlined copy of the evaluation
// (about 30 KB of code), so the search kernel's hot code fits the
// instruction caches better.  The operations and their order are those of
// the straight-line form: entry evaluation, then per iteration a line search
// (start, trials) and the direction update.
// entry_only: evaluate the entry pose and return its energy without
// optimising it (the visited-history policy's skipped calls,
// quasi_newton.cuh:1937-1939).
__device__ inline float rilc_bfgs(const LigView& L, const SearchMem& s, const MapView& G, const float4* smooth,
                           const EvalParams ep, int max_steps, int lane, int& evals, bool entry_only = false) {
    const int n = 6 + L.nt, nc = 7 + L.nt;
    if (max_steps <= 0) max_steps = 1000;  // the reference's 0 means unbounded
    float fx = 0.f, fx_orig = 0.f, fxp = 0.f, step = 0.f;
    Vec2 g = {0.f, 0.f}, gp = {0.f, 0.f}, d = {0.f, 0.f};
    // line-search state
    int count = 0, k = 1;
    bool brackt = false, first = true;
    float mu = 0.f, nu = 1.0e20f, finit = 0.f, dgtest = 0.f, dstest = 0.f;
    for (;;) {
        if (!first) conf_step(s.xp, s.m.x, d, step, L.nt, lane);  // the line search's trial pose
        // a trial that fails the Armijo test before the tenth reads no
        // gradient: its adjoint is skipped
        const float armijo = finit + step * dgtest;  // one value for the skip and the test below
        fx = eval_pose<true, true>(L, s.m, G, smooth, ep, lane,
                                   SkipAbove{(!first && count + 1 < 10) ? armijo : INFINITY});
        ++evals;
        g = vload(s.m.g, n, lane);
        if (first) {
            if (entry_only) return fx;
            first = false;
            fx_orig = fx;
            copy_conf(s.m.x, s.xo, nc, lane);
            d = Vec2{-g.a, -g.b};
            const float gg = vdot(g, g);  // = d.d (d = -g)
            if (!(sqrtf(gg) >= 1e-5f)) return fx;
            step = 1.f / sqrtf(gg);
        } else {
            ++count;
            bool accept = false;
            if (fx > armijo) {
                nu = step;
                brackt = true;
            } else {
                if (vdot(g, d) < dstest) mu = step;
                else accept = true;
            }
            if (!accept && count >= 10) {
                if (fx > finit) {  // the line search failed: back to its start
                    copy_conf(s.xp, s.m.x, nc, lane);
                    g = gp;
                    fx = fxp;
                    break;
                }
                accept = true;
            }
            if (!accept) {
                step = brackt ? 0.5f * (mu + nu) : 2.f * step;
                continue;
            }
            // the update's dot products that do not depend on one another, in one
            // reduction: g.g, y.s, y.y, s.s, gp.gp and s.d with d = -g
            const Vec2 sv = {step * d.a, step * d.b};
            const Vec2 yv = {g.a - gp.a, g.b - gp.b};
            const Vec2 dn = {-g.a, -g.b};
            float dots[6] = {lane_dot(g, g), lane_dot(yv, sv), lane_dot(yv, yv), lane_dot(sv, sv), lane_dot(gp, gp),
                             lane_dot(sv, dn)};
            warp_sum6(dots, lane);
            if (!(sqrtf(dots[0]) >= 1e-5f)) return fx;
            if (max_steps <= k) break;
            ++k;
            const float ys = dots[1], yy = dots[2];
            d = dn;
            const float cau = dots[3] * sqrtf(dots[4]) * 1.0e-6f;
            if (ys > cau) {
                const float alpha = dots[5] / ys;
                d.a += alpha * yv.a; d.b += alpha * yv.b;
                const float sc = ys / yy;
                d.a *= sc; d.b *= sc;
                const float beta = vdot(yv, d) / ys;
                d.a += (alpha - beta) * sv.a; d.b += (alpha - beta) * sv.b;
            }
            step = 1.f;
        }
        // start a line search from the current pose
        copy_conf(s.m.x, s.xp, nc, lane);
        gp = g;
        fxp = fx;
        count = 0;
        brackt = false;
        mu = 0.f;
        nu = 1.0e20f;
        const float dginit = vdot(gp, d);
        if (0.f < dginit) {  // not a descent direction
            copy_conf(s.xp, s.m.x, nc, lane);
            g = gp;
            fx = fxp;
            break;
        }
        finit = fx;
        dgtest = 1.0e-4f * dginit;
        dstest = 0.1f * dginit;
    }
    if (!(fx <= fx_orig)) {
        fx = fx_orig;
        copy_conf(s.xo, s.m.x, nc, lane);
    }
    return fx;
}

// Adjoint skip of the dense line search: a trial whose Armijo test
// (bfgs.h:72) fails.
struct SkipArmijo {
    float f0, c;
    bool on;
    __device__ __forceinline__ bool operator()(float e) const { return on && !(e - f0 < c); }
};

// bfgs.h:95-140 (dense BFGS, Armijo backtracking line_search 65-82,
// bfgs_update 49-63) and its GPU form bfgs_optimized
// (quasi_newton.cuh:2391-2499, line_search_optimized 1859-1916), warp-
// parallel: the inverse Hessian H (n x n, full storage) and the vectors gc,
// pv, yv, mhy (n floats each) in the warp's shared memory.  Used by the
// refinement (direct-sum score) and by the Monte-Carlo search with
// --rilc_bfgs 0 (grid maps).  pair_atomics as in eval_pose_t.
template <bool pair_atomics = false, class Inter>
__device__ float dense_bfgs(const LigView& L, const SearchMem& s, float* H, float* gc, float* pv, float* yv,
                           float* mhy, const Inter& inter, const float4* smooth, float v_intra, float fix,
                           float inv_fix, int max_steps, int lane, int& evals) {
    const int n = 6 + L.nt, nc = 7 + L.nt;
    for (int i = lane; i < n * n; i += 32) H[i] = (i / n == i % n) ? 1.f : 0.f;
    // One evaluation site (the entry evaluation and every line-search trial),
    // as in rilc_bfgs; the operations and their order are the straight-line
    // algorithm's.  As in the reference's line search, a trial that fails
    // the Armijo test halves alpha, the tenth failure included, and the step
    // keeps the last trial pose.
    float f0 = 0.f, f_orig = 0.f, alpha = 1.f, pg = 0.f;
    Vec2 p = {0.f, 0.f}, g = {0.f, 0.f};
    int step = 0, trial = 0;
    bool first = true;
    for (;;) {
        if (!first) conf_step(s.xp, s.m.x, p, alpha, L.nt, lane);
        // a trial that fails the Armijo test before the tenth reads no
        // gradient: its adjoint is skipped
        const float armijo = 0.0001f * alpha * pg;
        const float fe = eval_pose_t<true, pair_atomics>(L, s.m, inter, smooth, v_intra, fix, inv_fix, lane,
                                                         SkipArmijo{f0, armijo, !first && trial + 1 < 10});
        ++evals;
        if (first) {
            first = false;
            f0 = fe;
            for (int i = lane; i < n; i += 32) gc[i] = s.m.g[i];
            f_orig = f0;
            copy_conf(s.m.x, s.xo, nc, lane);
        } else {
            if (!(fe - f0 < armijo)) {  // line_search, bfgs.h:65-82
                alpha *= 0.5f;
                if (++trial < 10) continue;
            }
            const Vec2 gn = vload(s.m.g, n, lane);
            const Vec2 y = {gn.a - g.a, gn.b - g.b};
            f0 = fe;
            if (!(sqrtf(vdot(g, g)) >= 1e-5f)) break;
            for (int i = lane; i < n; i += 32) { gc[i] = s.m.g[i]; yv[i] = s.m.g[i] - (i < 32 ? g.a : g.b); }
            __syncwarp();
            if (step == 0) {
                const float yy = vdot(y, y);
                if (fabsf(yy) > FLT_EPSILON) {
                    const float dg = alpha * vdot(y, p) / yy;
                    for (int i = lane; i < n; i += 32) H[i * n + i] = dg;
                    __syncwarp();
                }
            }
            const float yp = vdot(y, p);  // bfgs_update, bfgs.h:49-63
            if (!(alpha * yp < FLT_EPSILON)) {
                for (int i = lane; i < n; i += 32) {
                    float sum = 0.f;
                    for (int j = 0; j < n; ++j) sum += H[i * n + j] * yv[j];
                    mhy[i] = -sum;
                }
                __syncwarp();
                const float yhy = -vdot(y, vload(mhy, n, lane));
                const float r = 1.f / (alpha * yp);
                const float c2 = alpha * alpha * (r * r * yhy + r);
                for (int idx = lane; idx < n * n; idx += 32) {
                    const int i = idx / n, j = idx % n;
                    H[idx] += alpha * r * (mhy[i] * pv[j] + mhy[j] * pv[i]) + c2 * pv[i] * pv[j];
                }
                __syncwarp();
            }
            ++step;
        }
        if (step >= max_steps) break;
        for (int i = lane; i < n; i += 32) {  // p = -H g
            float sum = 0.f;
            for (int j = 0; j < n; ++j) sum += H[i * n + j] * gc[j];
            pv[i] = -sum;
        }
        __syncwarp();
        copy_conf(s.m.x, s.xp, nc, lane);
        p = vload(pv, n, lane);
        g = vload(gc, n, lane);
        pg = vdot(p, g);
        alpha = 1.f;
        trial = 0;
    }
    if (!(f0 <= f_orig)) {
        f0 = f_orig;
        copy_conf(s.xo, s.m.x, nc, lane);
    }
    return f0;
}

// Random initial pose (conf.h:137-140 rigid_conf::randomize, torsions in
// [-pi, pi]) from the chain's Philox stream; written to x.
__device__ __forceinline__ void init_pose(float* x, int nt, uint32_t seed, uint32_t lig, uint32_t chain,
                                          const float lo[3], const float hi[3], int lane) {
    uint32_t u[4], q[4];
    draw(seed, lig, chain, kInitStep, 0, u);
    draw(seed, lig, chain, kInitStep, 1, q);
    if (lane == 0) {
        for (int i = 0; i < 3; ++i) x[i] = lo[i] + u01(u[i]) * (hi[i] - lo[i]);
        const float r0 = sqrtf(-2.f * logf(u01_open(q[0]))), r1 = sqrtf(-2.f * logf(u01_open(q[2])));
        float s0, c0, s1, c1;
        sincosf(2.f * kPiF * u01(q[1]), &s0, &c0);
        sincosf(2.f * kPiF * u01(q[3]), &s1, &c1);
        float n4[4] = {r0 * c0, r0 * s0, r1 * c1, r1 * s1};
        float nrm = sqrtf(n4[0] * n4[0] + n4[1] * n4[1] + n4[2] * n4[2] + n4[3] * n4[3]);
        if (!(nrm > 1e-6f)) { n4[0] = 1.f; n4[1] = n4[2] = n4[3] = 0.f; nrm = 1.f; }
        for (int i = 0; i < 4; ++i) x[3 + i] = n4[i] / nrm;
    }
    for (int t = lane; t < nt; t += 32) {
        uint32_t v[4];
        draw(seed, lig, chain, kInitStep, 2 + t / 4, v);
        x[7 + t] = -kPiF + 2.f * kPiF * u01(v[t & 3]);
    }
    __syncwarp();
}

// mutate.cpp:62-127: one of position (2 A ball), orientation (2/Rg ball,
// Rg = heavy-atom gyration radius about the root origin, model.cpp:1161),
// or one torsion set uniformly in [-pi, pi].
__device__ __forceinline__ void mutate_pose(const LigView& L, const WarpMem& m, uint32_t seed, uint32_t lig,
                                            uint32_t chain, uint32_t step, float amplitude, int lane) {
    uint32_t a[4], b[4];
    draw(seed, lig, chain, step, 0, a);
    draw(seed, lig, chain, step, 1, b);
    const int mm = 2 + L.nt;
    int which = int(u01(a[0]) * float(mm));
    if (which > mm - 1) which = mm - 1;
    const float z = 2.f * u01(a[1]) - 1.f, phi = 2.f * kPiF * u01(a[2]), r = cbrtf(u01(a[3]));
    float sp, cp;
    sincosf(phi, &sp, &cp);
    const float sz = sqrtf(fmaxf(0.f, 1.f - z * z));
    const float s0 = r * sz * cp, s1 = r * sz * sp, s2 = r * z;
    if (which == 0) {
        if (lane == 0) { m.x[0] += amplitude * s0; m.x[1] += amplitude * s1; m.x[2] += amplitude * s2; }
    } else if (which == 1) {
        kinematics(L, m, lane);
        float acc = 0.f;
        for (int i = lane; i < L.na; i += 32) {
            const float dx = m.c[i].x - m.x[0], dy = m.c[i].y - m.x[1], dz = m.c[i].z - m.x[2];
            acc += dx * dx + dy * dy + dz * dz;
        }
        acc = warp_sum(acc);
        const float gr = sqrtf(acc / float(L.na));
        if (gr > FLT_EPSILON && lane == 0) {
            const float f = amplitude / gr;
            const float4 q = quat_increment(make_float4(m.x[3], m.x[4], m.x[5], m.x[6]), f * s0, f * s1, f * s2);
            m.x[3] = q.x; m.x[4] = q.y; m.x[5] = q.z; m.x[6] = q.w;
        }
    } else {
        if (lane == 0) m.x[7 + which - 2] = -kPiF + 2.f * kPiF * u01(b[0]);
    }
    __syncwarp();
}

}  // namespace vd
