// Warp-level energy and adjoint of one ligand pose (FP32).
//
// One warp owns one pose.  Per evaluation:
//   1. lanes = rigid bodies: local rotation aa_k = (cos t/2, sin t/2 u_k)
//   2. lanes = rigid bodies: each walks its ancestor path to get its frame
//        q_k = q_root * aa_j1 * ... * aa_k,  o_k = o_root + R_root * w_k
//      (rotation about a body-fixed axis; equals tree.h:282-292)
//   3. lanes = atoms: coordinates, trilinear grid term (grid.cpp:50-160)
//   4. lanes = pairs: intra pair term and pair force (model.cpp:1241-1256)
//   5. lanes = atoms: per-atom force = grid gradient + incident pair forces
//   6. lanes = bodies: own force and moment about the root origin
//   7. lanes = bodies: subtree sums over the pre-order range [k, end_k),
//        torque T_k = M_k - (o_k - o_root) x F_k, dE/dtorsion = T_k . axis_k
//      (the bottom-up recursion of tree.h:169-178, 341-348, 373-422)
//   8. warp butterfly sum of the energy (deterministic).
// All sums run in a fixed order, so results are bit-reproducible.
#pragma once

#include "common.h"

namespace vd {

struct MapView {
    const float* map[kTypes];   // per XS type (nullptr if not built)
    float init[3], factor[3], finv[3], dmo[3];
    int32_t n[3];
    int32_t pitch;
};

struct EvalParams {
    float v_intra, v_inter, slope;
};

struct LigView {
    const float4* atoms;
    const NodeRec* nodes;
    const int2* pairs;
    const int32_t* csr_off;
    const int32_t* csr;
    int32_t na, nn, np, nt;
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
    L.num_tors = h->conf_indep;
    L.atoms = b + h->off_atoms;
    L.nodes = reinterpret_cast<const NodeRec*>(b + h->off_nodes);
    L.pairs = reinterpret_cast<const int2*>(b + h->off_pairs);
    L.csr_off = reinterpret_cast<const int32_t*>(b + h->off_csr);
    L.csr = reinterpret_cast<const int32_t*>(b + h->off_csr_list);
    return L;
}

constexpr int kNodeF = 20;  // q[4], o[3], R[9], aa[4]

__host__ __device__ inline int pad4(int n) { return (n + 3) & ~3; }
// Shared-memory floats one warp needs for a ligand of the given size.
__host__ __device__ inline int warp_floats(int na, int nn, int np, int nt) {
    return pad4(7 + nt) + kNodeF * nn + 6 * pad4(na) + 3 * pad4(np) + pad4(6 * nn) + pad4(6 + nt);
}

struct WarpMem {
    float* x;
    float* nd;
    float *cx, *cy, *cz;
    float *fx, *fy, *fz;
    float *px, *py, *pz;
    float* ns;
    float* g;
};

__device__ __forceinline__ WarpMem carve(float* p, int na, int nn, int np, int nt) {
    WarpMem m;
    m.x = p; p += pad4(7 + nt);
    m.nd = p; p += kNodeF * nn;
    const int a4 = pad4(na), p4 = pad4(np);
    m.cx = p; p += a4;
    m.cy = p; p += a4;
    m.cz = p; p += a4;
    m.fx = p; p += a4;
    m.fy = p; p += a4;
    m.fz = p; p += a4;
    m.px = p; p += p4;
    m.py = p; p += p4;
    m.pz = p; p += p4;
    m.ns = p; p += pad4(6 * nn);
    m.g = p;
    return m;
}

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
// quaternion.cpp:155-192 layout: R[i + 3j] = row i, column j.
__device__ __forceinline__ void qmat(float4 q, float* R) {
    const float a = q.x, b = q.y, c = q.z, d = q.w;
    const float aa = a * a, ab = a * b, ac = a * c, ad = a * d, bb = b * b, bc = b * c, bd = b * d,
                cc = c * c, cd = c * d, dd = d * d;
    R[0] = aa + bb - cc - dd;
    R[3] = 2.f * (-ad + bc);
    R[6] = 2.f * (ac + bd);
    R[1] = 2.f * (ad + bc);
    R[4] = aa - bb + cc - dd;
    R[7] = 2.f * (-ab + cd);
    R[2] = 2.f * (-ac + bd);
    R[5] = 2.f * (ab + cd);
    R[8] = aa - bb - cc + dd;
}

// Phases 1-3a: rigid-body frames and heavy-atom coordinates from the pose in m.x.
__device__ __forceinline__ void kinematics(const LigView& L, const WarpMem& m, int lane) {
    // 1: local rotation of each body about its axis (angle_to_quaternion)
    for (int k = lane; k < L.nn; k += 32) {
        float4 aa = make_float4(1.f, 0.f, 0.f, 0.f);
        if (k > 0) {
            float s, c;
            sincosf(0.5f * m.x[7 + k - 1], &s, &c);
            const NodeRec& n = L.nodes[k];
            aa = make_float4(c, s * __ldg(&n.axis[0]), s * __ldg(&n.axis[1]), s * __ldg(&n.axis[2]));
        }
        float* nd = m.nd + kNodeF * k;
        nd[16] = aa.x; nd[17] = aa.y; nd[18] = aa.z; nd[19] = aa.w;
    }
    __syncwarp();
    // 2: frames by walking the ancestor path
    const float4 qr = make_float4(m.x[3], m.x[4], m.x[5], m.x[6]);
    const float3 orr = make_float3(m.x[0], m.x[1], m.x[2]);
    for (int k = lane; k < L.nn; k += 32) {
        float4 P = make_float4(1.f, 0.f, 0.f, 0.f);
        float3 w = make_float3(0.f, 0.f, 0.f);
        if (k > 0) {
            const float* ndk = m.nd + kNodeF * k;
            P = make_float4(ndk[16], ndk[17], ndk[18], ndk[19]);
            const NodeRec& nk = L.nodes[k];
            w = make_float3(__ldg(&nk.rel_origin[0]), __ldg(&nk.rel_origin[1]), __ldg(&nk.rel_origin[2]));
            int j = __ldg(&nk.parent);
            while (j > 0) {
                const float* ndj = m.nd + kNodeF * j;
                const float4 aj = make_float4(ndj[16], ndj[17], ndj[18], ndj[19]);
                const NodeRec& nj = L.nodes[j];
                const float3 r = qrot(aj, w);
                w = make_float3(__ldg(&nj.rel_origin[0]) + r.x, __ldg(&nj.rel_origin[1]) + r.y,
                                __ldg(&nj.rel_origin[2]) + r.z);
                P = qmul(aj, P);
                j = __ldg(&nj.parent);
            }
        }
        float4 q = qmul(qr, P);
        const float inv = rsqrtf(q.x * q.x + q.y * q.y + q.z * q.z + q.w * q.w);
        q = make_float4(q.x * inv, q.y * inv, q.z * inv, q.w * inv);
        const float3 ro = qrot(qr, w);
        float* nd = m.nd + kNodeF * k;
        nd[0] = q.x; nd[1] = q.y; nd[2] = q.z; nd[3] = q.w;
        nd[4] = orr.x + ro.x; nd[5] = orr.y + ro.y; nd[6] = orr.z + ro.z;
        qmat(q, nd + 7);
    }
    __syncwarp();
    // 3a: heavy-atom coordinates
    for (int i = lane; i < L.na; i += 32) {
        const float4 a = __ldg(&L.atoms[i]);
        const int k = (__float_as_int(a.w) >> 8) & 0xff;
        const float* nd = m.nd + kNodeF * k;
        const float* R = nd + 7;
        m.cx[i] = nd[4] + (R[0] * a.x + R[3] * a.y + R[6] * a.z);
        m.cy[i] = nd[5] + (R[1] * a.x + R[4] * a.y + R[7] * a.z);
        m.cz[i] = nd[6] + (R[2] * a.x + R[5] * a.y + R[8] * a.z);
    }
    __syncwarp();
}

// grid.cpp:50-160 in FP32: trilinear value, gradient, curl, out-of-box penalty.
__device__ __forceinline__ float grid_term(const MapView& G, const float* map, float px, float py, float pz,
                                           float v, float slope, float& gx, float& gy, float& gz) {
    float s[3] = {(px - G.init[0]) * G.factor[0], (py - G.init[1]) * G.factor[1], (pz - G.init[2]) * G.factor[2]};
    float miss[3] = {0.f, 0.f, 0.f};
    int region[3], a[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        if (s[d] < 0.f) {
            miss[d] = -s[d]; region[d] = -1; a[d] = 0; s[d] = 0.f;
        } else if (s[d] >= G.dmo[d]) {
            miss[d] = s[d] - G.dmo[d]; region[d] = 1; a[d] = G.n[d] - 2; s[d] = 1.f;
        } else {
            region[d] = 0; a[d] = int(s[d]); s[d] -= float(a[d]);
        }
    }
    const float penalty = slope * (miss[0] * G.finv[0] + miss[1] * G.finv[1] + miss[2] * G.finv[2]);
    const size_t row = size_t(G.pitch);
    const size_t plane = row * size_t(G.n[1]);
    const float* b = map + size_t(a[2]) * plane + size_t(a[1]) * row + a[0];
    const float f000 = __ldg(b), f100 = __ldg(b + 1);
    const float f010 = __ldg(b + row), f110 = __ldg(b + row + 1);
    const float f001 = __ldg(b + plane), f101 = __ldg(b + plane + 1);
    const float f011 = __ldg(b + plane + row), f111 = __ldg(b + plane + row + 1);
    const float x = s[0], y = s[1], z = s[2];
    const float mx = 1.f - x, my = 1.f - y, mz = 1.f - z;
    float f = f000 * mx * my * mz + f100 * x * my * mz + f010 * mx * y * mz + f110 * x * y * mz +
              f001 * mx * my * z + f101 * x * my * z + f011 * mx * y * z + f111 * x * y * z;
    float xg = (f100 - f000) * my * mz + (f110 - f010) * y * mz + (f101 - f001) * my * z + (f111 - f011) * y * z;
    float yg = (f010 - f000) * mx * mz + (f110 - f100) * x * mz + (f011 - f001) * mx * z + (f111 - f101) * x * z;
    float zg = (f001 - f000) * mx * my + (f101 - f100) * x * my + (f011 - f010) * mx * y + (f111 - f110) * x * y;
    if (f > 0.f) {  // curl (curl.h:31-40)
        const float t = v / (v + f);
        f *= t;
        const float t2 = t * t;
        xg *= t2; yg *= t2; zg *= t2;
    }
    gx = G.factor[0] * (region[0] == 0 ? xg : 0.f) + slope * float(region[0]);
    gy = G.factor[1] * (region[1] == 0 ? yg : 0.f) + slope * float(region[1]);
    gz = G.factor[2] * (region[2] == 0 ? zg : 0.f) + slope * float(region[2]);
    return f + penalty;
}

// Intra pair term from the smooth table (precalculate.h:80-95), curl with v.
__device__ __forceinline__ float pair_term(const float4* smooth, int tp, float r2, float v, float& dor) {
    const float rf = 32.f * r2;
    const int i1 = int(rf);
    const float rem = rf - float(i1);
    const float4 t = __ldg(smooth + size_t(tp) * kBins + i1);
    float e = t.x + rem * (t.z - t.x);
    dor = t.y + rem * (t.w - t.y);
    if (e > 0.f) {
        const float c = v / (v + e);
        e *= c;
        dor *= c * c;
    }
    return e;
}

// Energy (and, when want_grad, the gradient into m.g) of the pose in m.x.
// Returns the same value in every lane.
// Inter-molecular term of one atom on the cached grid maps.
struct GridInter {
    const MapView* G;
    float v, slope;
    __device__ __forceinline__ float operator()(int t, float px, float py, float pz, float& gx, float& gy,
                                                float& gz) const {
        return grid_term(*G, G->map[t], px, py, pz, v, slope, gx, gy, gz);
    }
};

template <bool want_grad, class Inter>
__device__ inline float eval_pose_t(const LigView& L, const WarpMem& m, const Inter& inter, const float4* smooth,
                             float v_intra, int lane) {
    kinematics(L, m, lane);
    float e = 0.f;
    // 3b: grid term per atom
    float gxs[4], gys[4], gzs[4];
#pragma unroll
    for (int s = 0; s < 4; ++s) {
        const int i = lane + 32 * s;
        gxs[s] = gys[s] = gzs[s] = 0.f;
        if (i < L.na) {
            const int t = __float_as_int(__ldg(&L.atoms[i].w)) & 0xff;
            e += inter(t, m.cx[i], m.cy[i], m.cz[i], gxs[s], gys[s], gzs[s]);
        }
    }
    // 4: intra pairs
    for (int p = lane; p < L.np; p += 32) {
        const int2 pr = __ldg(&L.pairs[p]);
        const int a = pr.x & 0xffff, b = pr.x >> 16;
        const float rx = m.cx[b] - m.cx[a], ry = m.cy[b] - m.cy[a], rz = m.cz[b] - m.cz[a];
        const float r2 = rx * rx + ry * ry + rz * rz;
        float Fx = 0.f, Fy = 0.f, Fz = 0.f;
        if (r2 < 64.f) {
            float dor;
            e += pair_term(smooth, pr.y, r2, v_intra, dor);
            Fx = dor * rx; Fy = dor * ry; Fz = dor * rz;
        }
        if (want_grad) { m.px[p] = Fx; m.py[p] = Fy; m.pz[p] = Fz; }
    }
    e = warp_sum(e);
    if (!want_grad) return e;
    __syncwarp();
    // 5: per-atom forces
#pragma unroll
    for (int s = 0; s < 4; ++s) {
        const int i = lane + 32 * s;
        if (i < L.na) {
            float fx = gxs[s], fy = gys[s], fz = gzs[s];
            const int b0 = __ldg(&L.csr_off[i]), b1 = __ldg(&L.csr_off[i + 1]);
            for (int q = b0; q < b1; ++q) {
                const int ent = __ldg(&L.csr[q]);
                const int p = ent >> 1;
                if (ent & 1) { fx += m.px[p]; fy += m.py[p]; fz += m.pz[p]; }
                else { fx -= m.px[p]; fy -= m.py[p]; fz -= m.pz[p]; }
            }
            m.fx[i] = fx; m.fy[i] = fy; m.fz[i] = fz;
        }
    }
    __syncwarp();
    // 6: own force and moment about the root origin per body
    const float ox = m.x[0], oy = m.x[1], oz = m.x[2];
    for (int k = lane; k < L.nn; k += 32) {
        const int b0 = __ldg(&L.nodes[k].atom_begin), b1 = __ldg(&L.nodes[k].atom_end);
        float F0 = 0.f, F1 = 0.f, F2 = 0.f, M0 = 0.f, M1 = 0.f, M2 = 0.f;
        for (int i = b0; i < b1; ++i) {
            const float fx = m.fx[i], fy = m.fy[i], fz = m.fz[i];
            const float dx = m.cx[i] - ox, dy = m.cy[i] - oy, dz = m.cz[i] - oz;
            F0 += fx; F1 += fy; F2 += fz;
            M0 += dy * fz - dz * fy;
            M1 += dz * fx - dx * fz;
            M2 += dx * fy - dy * fx;
        }
        float* ns = m.ns + 6 * k;
        ns[0] = F0; ns[1] = F1; ns[2] = F2; ns[3] = M0; ns[4] = M1; ns[5] = M2;
    }
    __syncwarp();
    // 7: subtree sums, torques and the pose gradient
    for (int k = lane; k < L.nn; k += 32) {
        const int e1 = __ldg(&L.nodes[k].subtree_end);
        float F0 = 0.f, F1 = 0.f, F2 = 0.f, M0 = 0.f, M1 = 0.f, M2 = 0.f;
        for (int j = k; j < e1; ++j) {
            const float* ns = m.ns + 6 * j;
            F0 += ns[0]; F1 += ns[1]; F2 += ns[2]; M0 += ns[3]; M1 += ns[4]; M2 += ns[5];
        }
        if (k == 0) {
            m.g[0] = F0; m.g[1] = F1; m.g[2] = F2; m.g[3] = M0; m.g[4] = M1; m.g[5] = M2;
        } else {
            const float* nd = m.nd + kNodeF * k;
            const float dx = nd[4] - ox, dy = nd[5] - oy, dz = nd[6] - oz;
            const float T0 = M0 - (dy * F2 - dz * F1);
            const float T1 = M1 - (dz * F0 - dx * F2);
            const float T2 = M2 - (dx * F1 - dy * F0);
            const float* R = nd + 7;
            const NodeRec& n = L.nodes[k];
            const float u0 = __ldg(&n.axis[0]), u1 = __ldg(&n.axis[1]), u2 = __ldg(&n.axis[2]);
            const float a0 = R[0] * u0 + R[3] * u1 + R[6] * u2;
            const float a1 = R[1] * u0 + R[4] * u1 + R[7] * u2;
            const float a2 = R[2] * u0 + R[5] * u1 + R[8] * u2;
            m.g[6 + k - 1] = T0 * a0 + T1 * a1 + T2 * a2;
        }
    }
    __syncwarp();
    return e;
}

template <bool want_grad>
__device__ __forceinline__ float eval_pose(const LigView& L, const WarpMem& m, const MapView& G,
                                           const float4* smooth, const EvalParams ep, int lane) {
    const GridInter gi{&G, ep.v_inter, ep.slope};
    return eval_pose_t<want_grad>(L, m, gi, smooth, ep.v_intra, lane);
}

}  // namespace vd
