// Warp-level energy and adjoint of one ligand pose (FP32).
//
// One warp owns one pose.  Per evaluation:
//   1. lanes = rigid bodies: local rotation aa_k = (cos t/2, sin t/2 u_k)
//   2. lanes = rigid bodies: each walks its ancestor path to get its frame
//        q_k = q_root * aa_j1 * ... * aa_k,  o_k = o_root + R_root * w_k
//      (rotation about a body-fixed axis; equals tree.h:282-292)
//   3. lanes = atoms: coordinates, trilinear grid term (grid.cpp:50-160)
//   4. intra pair term (model.cpp:1241-1256), two pairs per lane per
//      iteration.  The search (pair_atomics) walks the ligand's search
//      schedule: rounds of one pair per lane in which few lanes share an
//      atom, both atoms' forces added with shared-memory atomics.  The pose
//      kernels walk per-lane segments of the pair list sorted by second atom,
//      the second atom's force summed in registers while it repeats, the
//      first atom's added with an atomic.  Pair forces are summed in 32-bit
//      fixed point (EvalParams::fix units per kcal/mol/A, set from the tables
//      so that no atom's sum can overflow): integer sums are exact, so the
//      result does not depend on the order in which the atomics land, and
//      32-bit integer shared atomics are the cheapest kind on B200 (FP32 and
//      64-bit ones cost more per lane); atomics of several lanes of one
//      instruction to the same address serialise, which the schedule avoids
//   6. lanes = contiguous atom ranges: warp prefix sums over the heavy atoms
//      of force and moment about the root origin
//   7. lanes = bodies: subtree sums as differences of two prefixes (a
//        subtree's atoms are one contiguous range: atoms are grouped by body
//        in pre-order), torque T_k = M_k - (o_k - o_root) x F_k,
//        dE/dtorsion = T_k . axis_k (the bottom-up recursion of
//        tree.h:169-178, 341-348, 373-422)
//   8. warp butterfly sum of the energy (deterministic).
// The per-body and subtree sums run in a fixed order, so every result is
// reproducible run to run and across launch shapes.
#pragma once

#include "checks.cuh"
#include "common.h"

namespace vd {

struct MapView {
    const float* map[kTypes];   // per XS type (nullptr if not built)
    const float* cell[kTypes];  // same maps as 32-byte corner cells (nullptr: read map)
    float init[3], factor[3], finv[3], dmo[3];
    int32_t n[3];
    int32_t pitch;
};

struct EvalParams {
    float v_intra, v_inter, slope;
    float fix, inv_fix;  // fixed-point units per kcal/mol/A of the pair forces (a power of two), 1/fix
};

struct LigView {
    const float4* atoms;
    const NodeRec* nodes;
    const int2* pairs;
    const int4* lpairs;         // per-lane segments, two pairs per entry, interleaved by lane
    const int2* spairs;         // search schedule: rounds of one pair per lane, two rounds per entry
    int32_t na, nn, np, nt;
    int32_t sp_iters;           // schedule entries per lane
    float num_tors;
};

__device__ __forceinline__ LigView lig_view(const float4* pool, int64_t off) {
    const float4* b = pool + off;
    const LigHeader* h = reinterpret_cast<const LigHeader*>(b);
    LigView L;
    L.na = h->n_atoms;
    L.nn = h->n_nodes;
    L.np = h->n_pairs;
    L.nt = h->ntors;
    L.num_tors = h->num_tors;
    L.atoms = b + h->off_atoms;
    L.nodes = reinterpret_cast<const NodeRec*>(b + h->off_nodes);
    L.pairs = reinterpret_cast<const int2*>(b + h->off_pairs);
    L.lpairs = reinterpret_cast<const int4*>(b + h->off_lpairs);
    L.spairs = reinterpret_cast<const int2*>(b + h->off_spairs);
    L.sp_iters = h->sp_iters;
    return L;
}

// Body frame in shared memory, 20 floats: three rows [R(i,0) R(i,1) R(i,2) o_i]
// (so an atom position is three 128-bit loads), 4 unused, and the local
// rotation about the body's torsion axis.  The 80-byte stride puts the
// 128-bit rows of 8 consecutive bodies in distinct bank groups.
constexpr int kNodeF = 20;
constexpr int kNdAA = 16;

__host__ __device__ inline int pad4(int n) { return (n + 3) & ~3; }
// Shared-memory floats one warp needs for a ligand of the given size.
__host__ __device__ inline int warp_floats(int na, int nn, int np, int nt) {
    return pad4(7 + nt) + kNodeF * nn + 4 * na + 3 * pad4(na) + 3 * pad4(na) + pad4(6 + nt);
}

struct WarpMem {
    float* x;
    float* nd;
    float4* c;          // heavy-atom coordinates (w unused)
    float *fx, *fy, *fz;  // [pad4(na)] grid-term forces, then prefix forces
    float* ns;          // [3][pad4(na)] fixed-point pair forces, then prefix moments
    float* g;
};

__device__ __forceinline__ WarpMem carve(float* p, int na, int nn, int np, int nt) {
    WarpMem m;
    m.x = p; p += pad4(7 + nt);
    m.nd = p; p += kNodeF * nn;
    const int a4 = pad4(na);
    m.c = reinterpret_cast<float4*>(p); p += 4 * na;
    m.fx = p; p += a4;
    m.fy = p; p += a4;
    m.fz = p; p += a4;
    m.ns = p; p += 3 * pad4(na);  // prefix moments [3][pad4(na)] (prefix forces overwrite fx/fy/fz)
    m.g = p;
    return m;
}

// Fixed point of the intra-pair forces, `fix` units per kcal/mol/A: the
// host picks the largest power of two for which 128 times the tables' largest
// pair force stays below 2^30 (pair_force_scale), so an atom's sum over at
// most 127 partners cannot overflow; 2^19 for the default weights.
__device__ __forceinline__ int to_fixed(float v, float fix) { return __float2int_rn(v * fix); }
__device__ __forceinline__ float from_fixed(int v, float inv_fix) { return float(v) * inv_fix; }

__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Hamilton product a*b, (w,x,y,z).
__device__ __forceinline__ float4 qmul(float4 a, float4 b) {
    return make_float4(a.x * b.x - a.y * b.y - a.z * b.z - a.w * b.w,
                       a.x * b.y + a.y * b.x + a.z * b.w - a.w * b.z,
                       a.x * b.z - a.y * b.w + a.z * b.x + a.w * b.y,
                       a.x * b.w + a.y * b.z - a.z * b.y + a.w * b.x);
}
// Rotates v by unit quaternion q: v + 2 w x (w x v + s v), w = (q.y,q.z,q.w), s = q.x.
__device__ __forceinline__ float3 qrot(float4 q, float3 v) {
    const float tx = q.z * v.z - q.w * v.y + q.x * v.x;
    const float ty = q.w * v.x - q.y * v.z + q.x * v.y;
    const float tz = q.y * v.y - q.z * v.x + q.x * v.z;
    return make_float3(v.x + 2.f * (q.z * tz - q.w * ty), v.y + 2.f * (q.w * tx - q.y * tz),
                       v.z + 2.f * (q.y * ty - q.z * tx));
}
// Body frame from a unit quaternion (rotation matrix as quaternion.cpp:155-192)
// and origin o, written as three 128-bit rows [R(i,0) R(i,1) R(i,2) o_i].
__device__ __forceinline__ void store_frame(float4 q, float3 o, float* nd) {
    const float a = q.x, b = q.y, c = q.z, d = q.w;
    const float aa = a * a, ab = a * b, ac = a * c, ad = a * d, bb = b * b, bc = b * c, bd = b * d,
                cc = c * c, cd = c * d, dd = d * d;
    float4* r = reinterpret_cast<float4*>(nd);
    r[0] = make_float4(aa + bb - cc - dd, 2.f * (-ad + bc), 2.f * (ac + bd), o.x);
    r[1] = make_float4(2.f * (ad + bc), aa - bb + cc - dd, 2.f * (-ab + cd), o.y);
    r[2] = make_float4(2.f * (-ac + bd), 2.f * (ab + cd), aa - bb - cc + dd, o.z);
}

// Node words as 128-bit loads (NodeRec: {origin, parent}, {axis, first
// atom}, {atom end, subtree end, depth, subtree atom end}).
__device__ __forceinline__ float4 node_word(const NodeRec* nodes, int k, int w) {
    return __ldg(reinterpret_cast<const float4*>(nodes + k) + w);
}

// Phases 1-2: rigid-body frames from the pose in m.x.
__device__ __forceinline__ void frames(const LigView& L, const WarpMem& m, int lane) {
    // 1: local rotation of each body about its axis (angle_to_quaternion)
    for (int k = lane; k < L.nn; k += 32) {
        float4 aa = make_float4(1.f, 0.f, 0.f, 0.f);
        if (k > 0) {
            float s, c;
            __sincosf(0.5f * m.x[7 + k - 1], &s, &c);  // |angle| <= pi/2, abs error < 1e-6
            const float4 ax = node_word(L.nodes, k, 1);
            aa = make_float4(c, s * ax.x, s * ax.y, s * ax.z);
        }
        *reinterpret_cast<float4*>(m.nd + kNodeF * k + kNdAA) = aa;
    }
    __syncwarp();
    // 2: frames by walking the ancestor path
    // the pose's position and orientation: two broadcast 128-bit loads (m.x is
    // 16-byte aligned and holds at least 8 floats)
    const float4 x0 = *reinterpret_cast<const float4*>(m.x), x1 = *reinterpret_cast<const float4*>(m.x + 4);
    const float4 qr = make_float4(x0.w, x1.x, x1.y, x1.z);
    const float3 orr = make_float3(x0.x, x0.y, x0.z);
    for (int k = lane; k < L.nn; k += 32) {
        float4 P = make_float4(1.f, 0.f, 0.f, 0.f);
        float3 w = make_float3(0.f, 0.f, 0.f);
        if (k > 0) {
            P = *reinterpret_cast<const float4*>(m.nd + kNodeF * k + kNdAA);
            const float4 ok = node_word(L.nodes, k, 0);
            w = make_float3(ok.x, ok.y, ok.z);
            int j = VD_DCLAMP(__float_as_int(ok.w), 0, k - 1, kChkParent);
            while (j > 0) {
                const float4 aj = *reinterpret_cast<const float4*>(m.nd + kNodeF * j + kNdAA);
                const float4 oj = node_word(L.nodes, j, 0);
                const float3 r = qrot(aj, w);
                w = make_float3(oj.x + r.x, oj.y + r.y, oj.z + r.z);
                P = qmul(aj, P);
                j = VD_DCLAMP(__float_as_int(oj.w), 0, j - 1, kChkParent);
            }
        }
        float4 q = qmul(qr, P);
        const float inv = rsqrtf(q.x * q.x + q.y * q.y + q.z * q.z + q.w * q.w);
        q = make_float4(q.x * inv, q.y * inv, q.z * inv, q.w * inv);
        const float3 ro = qrot(qr, w);
        store_frame(q, make_float3(orr.x + ro.x, orr.y + ro.y, orr.z + ro.z), m.nd + kNodeF * k);
    }
    __syncwarp();
}

// Phase 3a for one heavy atom: its coordinates from its body's frame.
__device__ __forceinline__ float4 atom_position(const LigView& L, const WarpMem& m, float4 a) {
    const int k = VD_DCLAMP((__float_as_int(a.w) >> 8) & 0xff, 0, L.nn - 1, kChkAtomBody);
    const float4* nd = reinterpret_cast<const float4*>(m.nd + kNodeF * k);
    const float4 r0 = nd[0], r1 = nd[1], r2 = nd[2];
    return make_float4(r0.w + (r0.x * a.x + r0.y * a.y + r0.z * a.z), r1.w + (r1.x * a.x + r1.y * a.y + r1.z * a.z),
                       r2.w + (r2.x * a.x + r2.y * a.y + r2.z * a.z), 0.f);
}

// Phases 1-3a: rigid-body frames and heavy-atom coordinates from the pose in m.x.
__device__ __forceinline__ void kinematics(const LigView& L, const WarpMem& m, int lane) {
    frames(L, m, lane);
    for (int i = lane; i < L.na; i += 32) m.c[i] = atom_position(L, m, __ldg(&L.atoms[i]));
    __syncwarp();
}

// grid.cpp:50-160 in FP32: trilinear value, gradient, curl, out-of-box
// penalty.  Outside the box a coordinate is clamped to the nearest cell
// (fraction 0 below, 1 above), the gradient component is replaced by
// slope * region and the penalty adds slope * distance outside.
// The eight corners of trilinear cell (a0, a1, a2): from the corner-cell
// layout, one 256-bit load of one 32-byte sector (x fastest, then y, then z:
// f000 f100 f010 f110 f001 f101 f011 f111); else eight loads from the map.
struct Corners {
    float f000, f100, f010, f110, f001, f101, f011, f111;
};
__device__ __forceinline__ Corners load_corners(const MapView& G, const float* map, const float* cell, int a0, int a1,
                                                int a2) {
    Corners k;
    if (cell) {
        const float* c = cell + ((size_t(a2) * (G.n[1] - 1) + a1) * (G.n[0] - 1) + a0) * 8;
        unsigned long long w0, w1, w2, w3;
        // not allocated in L1: the cells of a 70 A box span 1.67 GB and are
        // rarely re-read from L1, where they would evict the pair table
        asm("ld.global.nc.L1::no_allocate.v4.b64 {%0,%1,%2,%3}, [%4];" : "=l"(w0), "=l"(w1), "=l"(w2), "=l"(w3) : "l"(c));
        k.f000 = __int_as_float(int(w0 & 0xffffffffull)); k.f100 = __int_as_float(int(w0 >> 32));
        k.f010 = __int_as_float(int(w1 & 0xffffffffull)); k.f110 = __int_as_float(int(w1 >> 32));
        k.f001 = __int_as_float(int(w2 & 0xffffffffull)); k.f101 = __int_as_float(int(w2 >> 32));
        k.f011 = __int_as_float(int(w3 & 0xffffffffull)); k.f111 = __int_as_float(int(w3 >> 32));
    } else {
        const size_t row = size_t(G.pitch);
        const size_t plane = row * size_t(G.n[1]);
        const float* b = map + size_t(a2) * plane + size_t(a1) * row + a0;
        k.f000 = __ldg(b); k.f100 = __ldg(b + 1);
        k.f010 = __ldg(b + row); k.f110 = __ldg(b + row + 1);
        k.f001 = __ldg(b + plane); k.f101 = __ldg(b + plane + 1);
        k.f011 = __ldg(b + plane + row); k.f111 = __ldg(b + plane + row + 1);
    }
    return k;
}

__device__ __forceinline__ float grid_term(const MapView& G, const float* map, const float* cell, float px, float py,
                                           float pz, float v, float slope, float& gx, float& gy, float& gz) {
    const float pc[3] = {px, py, pz};
    float fr[3], miss = 0.f, reg[3];
    int a[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        const float s = (pc[d] - G.init[d]) * G.factor[d];
        const float lo = fmaxf(-s, 0.f), hi = fmaxf(s - G.dmo[d], 0.f);
        miss += (lo + hi) * G.finv[d];
        reg[d] = (s < 0.f) ? -1.f : ((s >= G.dmo[d]) ? 1.f : 0.f);
        const float sc = fminf(fmaxf(s, 0.f), G.dmo[d]);
        const int ai = min(int(sc), G.n[d] - 2);
        a[d] = ai;
        fr[d] = (s >= G.dmo[d]) ? 1.f : sc - float(ai);
    }
    const float penalty = slope * miss;
    const Corners k = load_corners(G, map, cell, a[0], a[1], a[2]);
    const float f000 = k.f000, f100 = k.f100, f010 = k.f010, f110 = k.f110;
    const float f001 = k.f001, f101 = k.f101, f011 = k.f011, f111 = k.f111;
    const float x = fr[0], y = fr[1], z = fr[2];
    const float mx = 1.f - x, my = 1.f - y, mz = 1.f - z;
    float f = f000 * mx * my * mz + f100 * x * my * mz + f010 * mx * y * mz + f110 * x * y * mz +
              f001 * mx * my * z + f101 * x * my * z + f011 * mx * y * z + f111 * x * y * z;
    float xg = (f100 - f000) * my * mz + (f110 - f010) * y * mz + (f101 - f001) * my * z + (f111 - f011) * y * z;
    float yg = (f010 - f000) * mx * mz + (f110 - f100) * x * mz + (f011 - f001) * mx * z + (f111 - f101) * x * z;
    float zg = (f001 - f000) * mx * my + (f101 - f100) * x * my + (f011 - f010) * mx * y + (f111 - f110) * x * y;
    const float t = (f > 0.f) ? __fdividef(v, v + f) : 1.f;  // curl (curl.h:31-40)
    f *= t;
    const float t2 = t * t;
    gx = (reg[0] == 0.f) ? G.factor[0] * xg * t2 : slope * reg[0];
    gy = (reg[1] == 0.f) ? G.factor[1] * yg * t2 : slope * reg[1];
    gz = (reg[2] == 0.f) ? G.factor[2] * zg * t2 : slope * reg[2];
    return f + penalty;
}

// Energy (and, when want_grad, the gradient into m.g) of the pose in m.x.
// Returns the same value in every lane.
// Inter-molecular term of one atom on the cached grid maps.
struct GridInter {
    const MapView* G;
    float v, slope;
    __device__ __forceinline__ float operator()(int t, float px, float py, float pz, float& gx, float& gy,
                                                float& gz) const {
#ifdef VD_CHECKS
        if (t < 0 || t >= kTypes || !G->map[t]) {
            VD_DCHECK(false, kChkMapMissing);
            gx = gy = gz = 0.f;
            return 0.f;
        }
#endif
        return grid_term(*G, G->map[t], G->cell[t], px, py, pz, v, slope, gx, gy, gz);
    }
};

// Adjoint-skip tests for eval_pose_t (below).  NoSkip: always compute it.
struct NoSkip {
    __device__ __forceinline__ bool operator()(float) const { return false; }
};
// Skip when the energy exceeds a threshold (+inf: never; a NaN energy never
// exceeds it).
struct SkipAbove {
    float thr;
    __device__ __forceinline__ bool operator()(float e) const { return e > thr; }
};

// pair_atomics: pairs from the search schedule, both atoms' forces by
// atomics (no per-lane flush when the second atom changes: shorter, less
// divergent code, which the latency-bound search prefers); otherwise the
// second atom's force is summed in registers along b-sorted segments, which
// the pose kernels, bound by L1 wavefronts, prefer (fewer atomics and
// coordinate loads).
// skip(e): called with the energy (the same in every lane) once it is
// known; when it returns true the adjoint phases (prefix sums, torques) are
// skipped and m.g is left as it was.  The line searches pass a test that
// holds exactly when the trial's gradient will not be read (a failed Armijo
// test that is not the search's last trial).
template <bool want_grad, bool pair_atomics = false, class Inter, class Skip = NoSkip>
__device__ inline float eval_pose_t(const LigView& L, const WarpMem& m, const Inter& inter, const float4* smooth,
                             float v_intra, float fix, float inv_fix, int lane, const Skip& skip = Skip()) {
    frames(L, m, lane);
    float e = 0.f;
    // 3: per atom its coordinates (kept for the pair phase) and the grid
    // term, whose gradient seeds the atom's force
    for (int i = lane; i < L.na; i += 32) {
        const float4 a = __ldg(&L.atoms[i]);
        const float4 ci = atom_position(L, m, a);
        m.c[i] = ci;
        const int t = __float_as_int(a.w) & 0xff;
        float gx, gy, gz;
        e += inter(t, ci.x, ci.y, ci.z, gx, gy, gz);
        if (want_grad) {
            int* const q = reinterpret_cast<int*>(m.ns);  // pair-force accumulators start at zero
            const int a4 = pad4(L.na);
            m.fx[i] = gx; m.fy[i] = gy; m.fz[i] = gz;
            q[i] = 0; q[a4 + i] = 0; q[2 * a4 + i] = 0;
        }
    }
    __syncwarp();
    // 4: intra pairs, two per lane per iteration (two table gathers in
    // flight); table indices are clamped and pairs past the cutoff masked
    // (their table loads predicated off).
    //  - pair_atomics (the search): the ligand's search schedule, one pair per
    //    lane per round; both atoms' forces go to their accumulators with
    //    atomics, and the rounds are built so few lanes share an atom;
    //  - otherwise: pairs sorted by their second atom b, each lane a
    //    contiguous segment, b's coordinates and force kept in registers
    //    while b repeats, the force on a added with an atomic.
    if (pair_atomics) {
        int* const qx = reinterpret_cast<int*>(m.ns);
        int* const qy = qx + pad4(L.na);
        int* const qz = qy + pad4(L.na);
        const int2* sp = L.spairs + lane;
        for (int k = 0; k < L.sp_iters; ++k, sp += 32) {
            const int2 qq = __ldg(sp);  // coalesced across the warp
            const bool v0 = qq.x >= 0, v1 = qq.y >= 0;  // unused slots are negative (atoms 0, 0)
            const int a0 = VD_DCLAMP(qq.x & 0xff, 0, L.na - 1, kChkPairAtom);
            const int b0 = VD_DCLAMP((qq.x >> 8) & 0xff, 0, L.na - 1, kChkPairAtom);
            const int a1 = VD_DCLAMP(qq.y & 0xff, 0, L.na - 1, kChkPairAtom);
            const int b1 = VD_DCLAMP((qq.y >> 8) & 0xff, 0, L.na - 1, kChkPairAtom);
            const float4 ca0 = m.c[a0], cb0 = m.c[b0], ca1 = m.c[a1], cb1 = m.c[b1];
            const float r0x = cb0.x - ca0.x, r0y = cb0.y - ca0.y, r0z = cb0.z - ca0.z;
            const float r1x = cb1.x - ca1.x, r1y = cb1.y - ca1.y, r1z = cb1.z - ca1.z;
            const float d0 = r0x * r0x + r0y * r0y + r0z * r0z, d1 = r1x * r1x + r1y * r1y + r1z * r1z;
            const float rf0 = fminf(32.f * d0, 2047.5f), rf1 = fminf(32.f * d1, 2047.5f);
            const int i0 = VD_DCLAMP(int(rf0), 0, kBins - 2, kChkTableBin);
            const int i1 = VD_DCLAMP(int(rf1), 0, kBins - 2, kChkTableBin);
            const int tp0 = VD_DCLAMP(v0 ? (qq.x >> 16) : 0, 0, kPairTypes - 1, kChkPairType);
            const int tp1 = VD_DCLAMP(v1 ? (qq.y >> 16) : 0, 0, kPairTypes - 1, kChkPairType);
            const bool in0 = v0 && d0 < 64.f, in1 = v1 && d1 < 64.f;
            float4 t0 = make_float4(0.f, 0.f, 0.f, 0.f), t1 = t0;
            if (in0) t0 = __ldg(smooth + size_t(tp0) * kBins + i0);  // no gather past the cutoff
            if (in1) t1 = __ldg(smooth + size_t(tp1) * kBins + i1);
            const float w0 = rf0 - float(i0), w1 = rf1 - float(i1);
            float e0 = t0.x + w0 * (t0.z - t0.x), g0 = t0.y + w0 * (t0.w - t0.y);
            float e1 = t1.x + w1 * (t1.z - t1.x), g1 = t1.y + w1 * (t1.w - t1.y);
            const float c0 = (e0 > 0.f) ? __fdividef(v_intra, v_intra + e0) : 1.f;
            const float c1 = (e1 > 0.f) ? __fdividef(v_intra, v_intra + e1) : 1.f;
            e0 = in0 ? e0 * c0 : 0.f;
            e1 = in1 ? e1 * c1 : 0.f;
            e += e0 + e1;
            if (want_grad) {
                // fixed point: fix is a power of two, so (g * fix) * r rounds exactly like (g * r) * fix
                const float gf0 = in0 ? g0 * c0 * c0 * fix : 0.f, gf1 = in1 ? g1 * c1 * c1 * fix : 0.f;
                if (in0) {
                    const int Fx = __float2int_rn(gf0 * r0x), Fy = __float2int_rn(gf0 * r0y), Fz = __float2int_rn(gf0 * r0z);
                    atomicAdd(&qx[a0], -Fx); atomicAdd(&qy[a0], -Fy); atomicAdd(&qz[a0], -Fz);
                    atomicAdd(&qx[b0], Fx); atomicAdd(&qy[b0], Fy); atomicAdd(&qz[b0], Fz);
                }
                if (in1) {
                    const int Fx = __float2int_rn(gf1 * r1x), Fy = __float2int_rn(gf1 * r1y), Fz = __float2int_rn(gf1 * r1z);
                    atomicAdd(&qx[a1], -Fx); atomicAdd(&qy[a1], -Fy); atomicAdd(&qz[a1], -Fz);
                    atomicAdd(&qx[b1], Fx); atomicAdd(&qy[b1], Fy); atomicAdd(&qz[b1], Fz);
                }
            }
        }
    } else {
        const int len = (((lane + 1) * L.np) >> 5) - ((lane * L.np) >> 5);
        const int4* lp = L.lpairs + lane;
        int cur_b = -1;
        float bx = 0.f, by = 0.f, bz = 0.f;
        int* const qx = reinterpret_cast<int*>(m.ns);
        int* const qy = qx + pad4(L.na);
        int* const qz = qy + pad4(L.na);
        auto flush = [&](int nb) {
            if (want_grad && cur_b >= 0) {
                atomicAdd(&qx[cur_b], to_fixed(bx, fix)); atomicAdd(&qy[cur_b], to_fixed(by, fix));
                atomicAdd(&qz[cur_b], to_fixed(bz, fix));
            }
            cur_b = nb;
            bx = by = bz = 0.f;
        };
        float4 cb = make_float4(0.f, 0.f, 0.f, 0.f);  // coordinates of cur_b
        for (int p = 0; p < len; p += 2, lp += 32) {
            const bool two = p + 1 < len;
            const int4 qq = __ldg(lp);  // coalesced across the warp
            const int2 q0 = make_int2(qq.x, qq.y);
            const int2 q1 = two ? make_int2(qq.z, qq.w) : q0;
            const int a0 = VD_DCLAMP(q0.x & 0xffff, 0, L.na - 1, kChkPairAtom);
            const int b0 = VD_DCLAMP(q0.x >> 16, 0, L.na - 1, kChkPairAtom);
            const int a1 = VD_DCLAMP(q1.x & 0xffff, 0, L.na - 1, kChkPairAtom);
            const int b1 = VD_DCLAMP(q1.x >> 16, 0, L.na - 1, kChkPairAtom);
            if (b0 != cur_b) {  // b repeats along the segment: its coordinates stay in registers
                flush(b0);
                cb = m.c[b0];
            }
            const float4 cb0 = cb, cb1 = (b1 != b0) ? m.c[b1] : cb;
            const float4 ca0 = m.c[a0], ca1 = m.c[a1];
            const float r0x = cb0.x - ca0.x, r0y = cb0.y - ca0.y, r0z = cb0.z - ca0.z;
            const float r1x = cb1.x - ca1.x, r1y = cb1.y - ca1.y, r1z = cb1.z - ca1.z;
            const float d0 = r0x * r0x + r0y * r0y + r0z * r0z, d1 = r1x * r1x + r1y * r1y + r1z * r1z;
            const float rf0 = fminf(32.f * d0, 2047.5f), rf1 = fminf(32.f * d1, 2047.5f);
            const int i0 = VD_DCLAMP(int(rf0), 0, kBins - 2, kChkTableBin);
            const int i1 = VD_DCLAMP(int(rf1), 0, kBins - 2, kChkTableBin);
            const int tp0 = VD_DCLAMP(q0.y, 0, kPairTypes - 1, kChkPairType);
            const int tp1 = VD_DCLAMP(q1.y, 0, kPairTypes - 1, kChkPairType);
            const bool in0 = d0 < 64.f, in1 = two && d1 < 64.f;
            float4 t0 = make_float4(0.f, 0.f, 0.f, 0.f), t1 = t0;
            if (in0) t0 = __ldg(smooth + size_t(tp0) * kBins + i0);  // no gather past the cutoff
            if (in1) t1 = __ldg(smooth + size_t(tp1) * kBins + i1);
            const float w0 = rf0 - float(i0), w1 = rf1 - float(i1);
            float e0 = t0.x + w0 * (t0.z - t0.x), g0 = t0.y + w0 * (t0.w - t0.y);
            float e1 = t1.x + w1 * (t1.z - t1.x), g1 = t1.y + w1 * (t1.w - t1.y);
            const float c0 = (e0 > 0.f) ? __fdividef(v_intra, v_intra + e0) : 1.f;
            const float c1 = (e1 > 0.f) ? __fdividef(v_intra, v_intra + e1) : 1.f;
            e0 = in0 ? e0 * c0 : 0.f;
            e1 = in1 ? e1 * c1 : 0.f;
            g0 = in0 ? g0 * c0 * c0 : 0.f;
            g1 = in1 ? g1 * c1 * c1 : 0.f;
            e += e0 + e1;
            if (!want_grad && two && b1 != cur_b) {
                cur_b = b1;
                cb = cb1;
            }
            if (want_grad) {
                if (in0) {
                    const float Fx = g0 * r0x, Fy = g0 * r0y, Fz = g0 * r0z;
                    atomicAdd(&qx[a0], to_fixed(-Fx, fix)); atomicAdd(&qy[a0], to_fixed(-Fy, fix));
                    atomicAdd(&qz[a0], to_fixed(-Fz, fix));
                    bx += Fx; by += Fy; bz += Fz;
                }
                if (two) {
                    if (b1 != cur_b) {
                        flush(b1);
                        cb = cb1;
                    }
                    if (in1) {
                        const float Fx = g1 * r1x, Fy = g1 * r1y, Fz = g1 * r1z;
                        atomicAdd(&qx[a1], to_fixed(-Fx, fix)); atomicAdd(&qy[a1], to_fixed(-Fy, fix));
                        atomicAdd(&qz[a1], to_fixed(-Fz, fix));
                        bx += Fx; by += Fy; bz += Fz;
                    }
                }
            }
        }
        flush(-1);
    }
    e = warp_sum(e);
    if (!want_grad || skip(e)) return e;
    __syncwarp();
    // 6: prefix sums over the heavy atoms of force and moment about the root
    // origin.  Atoms are grouped by body in pre-order, so a subtree's atoms
    // are one contiguous range and its sums are a difference of two prefixes.
    // Lane l owns atoms [l*A, l*A + A); prefix forces overwrite fx/fy/fz.
    const float4 xo4 = *reinterpret_cast<const float4*>(m.x);
    const float ox = xo4.x, oy = xo4.y, oz = xo4.z;
    {
        const int A = (L.na + 31) >> 5, a0 = lane * A, a1 = min(L.na, a0 + A);
        const int a4 = pad4(L.na);
        float* mx = m.ns;
        float* my = m.ns + a4;
        float* mz = m.ns + 2 * a4;
        auto contrib = [&](int i, float v[6]) {
            const float4 ci = m.c[i];
            const int* q = reinterpret_cast<const int*>(m.ns);  // read before this lane overwrites it
            const float fx = m.fx[i] + from_fixed(q[i], inv_fix), fy = m.fy[i] + from_fixed(q[a4 + i], inv_fix),
                        fz = m.fz[i] + from_fixed(q[2 * a4 + i], inv_fix);
            const float dx = ci.x - ox, dy = ci.y - oy, dz = ci.z - oz;
            v[0] = fx; v[1] = fy; v[2] = fz;
            v[3] = dy * fz - dz * fy;
            v[4] = dz * fx - dx * fz;
            v[5] = dx * fy - dy * fx;
        };
        auto scan = [&](float (&run)[6]) {  // inclusive scan of the lane totals
#pragma unroll
            for (int off = 1; off < 32; off <<= 1) {
#pragma unroll
                for (int j = 0; j < 6; ++j) {
                    const float o = __shfl_up_sync(0xffffffffu, run[j], off);
                    if (lane >= off) run[j] += o;
                }
            }
        };
        if (A == 1) {  // up to 32 atoms: a lane's inclusive scan value is its atom's prefix
            float run[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
            if (a0 < a1) contrib(a0, run);
            scan(run);
            if (a0 < a1) {
                m.fx[a0] = run[0]; m.fy[a0] = run[1]; m.fz[a0] = run[2];
                mx[a0] = run[3]; my[a0] = run[4]; mz[a0] = run[5];
            }
        } else {  // lane totals, their exclusive scan, then each atom's prefix
            float run[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
            for (int i = a0; i < a1; ++i) {
                float v[6];
                contrib(i, v);
#pragma unroll
                for (int j = 0; j < 6; ++j) run[j] += v[j];
            }
            scan(run);
            float acc[6];
#pragma unroll
            for (int j = 0; j < 6; ++j) acc[j] = __shfl_up_sync(0xffffffffu, run[j], 1);
            if (lane == 0)
#pragma unroll
                for (int j = 0; j < 6; ++j) acc[j] = 0.f;
            for (int i = a0; i < a1; ++i) {
                float v[6];
                contrib(i, v);
#pragma unroll
                for (int j = 0; j < 6; ++j) acc[j] += v[j];
                m.fx[i] = acc[0]; m.fy[i] = acc[1]; m.fz[i] = acc[2];
                mx[i] = acc[3]; my[i] = acc[4]; mz[i] = acc[5];
            }
        }
    }
    __syncwarp();
    // 7: subtree sums (prefix differences), torques and the pose gradient
    for (int k = lane; k < L.nn; k += 32) {
        const float4 w1 = node_word(L.nodes, k, 1);  // {axis, first atom}
        const int e1 = VD_DCLAMP(__float_as_int(node_word(L.nodes, k, 2).w), 0, L.na, kChkSubtree);
        const int b = VD_DCLAMP(__float_as_int(w1.w), 0, e1, kChkSubtree);
        const int a4 = pad4(L.na);
        float F0 = 0.f, F1 = 0.f, F2 = 0.f, M0 = 0.f, M1 = 0.f, M2 = 0.f;
        if (e1 > b) {
            const int hi = e1 - 1;
            F0 = m.fx[hi]; F1 = m.fy[hi]; F2 = m.fz[hi];
            M0 = m.ns[hi]; M1 = m.ns[a4 + hi]; M2 = m.ns[2 * a4 + hi];
            if (b > 0) {
                const int lo = b - 1;
                F0 -= m.fx[lo]; F1 -= m.fy[lo]; F2 -= m.fz[lo];
                M0 -= m.ns[lo]; M1 -= m.ns[a4 + lo]; M2 -= m.ns[2 * a4 + lo];
            }
        }
        if (k == 0) {
            m.g[0] = F0; m.g[1] = F1; m.g[2] = F2; m.g[3] = M0; m.g[4] = M1; m.g[5] = M2;
        } else {
            const float4* nd = reinterpret_cast<const float4*>(m.nd + kNodeF * k);
            const float4 r0 = nd[0], r1 = nd[1], r2 = nd[2];
            const float dx = r0.w - ox, dy = r1.w - oy, dz = r2.w - oz;
            const float T0 = M0 - (dy * F2 - dz * F1);
            const float T1 = M1 - (dz * F0 - dx * F2);
            const float T2 = M2 - (dx * F1 - dy * F0);
            const float u0 = w1.x, u1 = w1.y, u2 = w1.z;
            const float a0 = r0.x * u0 + r0.y * u1 + r0.z * u2;
            const float a1 = r1.x * u0 + r1.y * u1 + r1.z * u2;
            const float a2 = r2.x * u0 + r2.y * u1 + r2.z * u2;
            m.g[6 + k - 1] = T0 * a0 + T1 * a1 + T2 * a2;
        }
    }
    __syncwarp();
    return e;
}

template <bool want_grad, bool pair_atomics = false, class Skip = NoSkip>
__device__ __forceinline__ float eval_pose(const LigView& L, const WarpMem& m, const MapView& G,
                                           const float4* smooth, const EvalParams ep, int lane,
                                           const Skip& skip = Skip()) {
    const GridInter gi{&G, ep.v_inter, ep.slope};
    return eval_pose_t<want_grad, pair_atomics>(L, m, gi, smooth, ep.v_intra, ep.fix, ep.inv_fix, lane, skip);
}

}  // namespace vd
