// Post-processing of the chain results on the GPU, replacing the host tail
// of the reference (main_procedure_cu.cpp:896-926, main.cpp:423-489):
//   cluster : energy-sorted greedy selection of up to 20 poses whose
//             heavy-atom RMSD to every kept pose is >= min_rmsd
//             (add_to_output_container semantics, coords.cpp:47-62, applied
//             in energy order)
//   refine  : refine_structure (main.cpp:139-157): dense BFGS (bfgs.h:95-140)
//             on the direct-sum score (non_cache.cpp:82-128) with the slope
//             ramp 100*10^(2p), authentic caps (1000)
//   score   : eval_intramolecular of the best mode and eval_adjusted
//             (model.cpp:1375-1431) in double, remove_redundant, the
//             num_modes / energy_range cut and RMSD bounds to mode 1
// dock_pipeline runs the docking launch and these kernels; the batched form
// records the whole sequence, with its uploads and downloads, into one CUDA
// graph per call (updated in place for the next call of the same shape).
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstring>
#include <functional>
#include <string>

#include "dock.h"
#include "launch.h"
#include "search.cuh"

namespace vd {
namespace {

// ------------------------------------------------------------ receptor view
struct RecView {
    const float4* rec;          // relevant receptor atoms {x,y,z,type}
    const double4* recd;        // same in double
    const int32_t* cell_start;  // [cells+1]
    const int32_t* cell_list;   // atom indices per cell
    double init[3], range[3];   // szv_grid cell geometry
    int32_t dim[3];
    double gb[3], ge[3];        // box (non_cache gd)
};

__device__ __forceinline__ int cell_of(const RecView& R, double x, double y, double z) {
    const double c[3] = {x, y, z};
    int idx[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {  // szv_grid.cpp:92-107, fl_to_sz
        const double t = (c[d] - R.init[d]) * R.dim[d] / R.range[d];
        const int mx = R.dim[d] - 1;
        idx[d] = (t <= 0) ? 0 : ((t >= mx) ? mx : min(int(t), mx));
    }
    return VD_DCLAMP(idx[0] + R.dim[0] * (idx[1] + R.dim[1] * idx[2]), 0, R.dim[0] * R.dim[1] * R.dim[2] - 1, kChkCell);
}

// non_cache::eval_deriv term of one atom (FP32), smooth table, curl v.
struct DirectInter {
    const RecView* R;
    const float4* smooth;
    float v, slope;
    __device__ __forceinline__ float operator()(int t1, float px, float py, float pz, float& gx, float& gy,
                                                float& gz) const {
        float a[3] = {px, py, pz}, od[3] = {0.f, 0.f, 0.f};
        float oob = 0.f;
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            const float b = float(R->gb[d]), e = float(R->ge[d]);
            if (a[d] < b) { oob += fabsf(a[d] - b); a[d] = b; od[d] = -1.f; }
            else if (a[d] > e) { oob += fabsf(a[d] - e); a[d] = e; od[d] = 1.f; }
        }
        const int c = cell_of(*R, a[0], a[1], a[2]);
        const int q0 = __ldg(&R->cell_start[c]), q1 = __ldg(&R->cell_start[c + 1]);
        float this_e = 0.f, dx = 0.f, dy = 0.f, dz = 0.f;
        for (int q = q0; q < q1; ++q) {
            const float4 b = __ldg(&R->rec[__ldg(&R->cell_list[q])]);
            const float rx = a[0] - b.x, ry = a[1] - b.y, rz = a[2] - b.z;
            const float r2 = rx * rx + ry * ry + rz * rz;
            if (r2 < 64.f) {
                const int t2 = int(b.w);
                const int tp = (t1 <= t2) ? t1 + t2 * (t2 + 1) / 2 : t2 + t1 * (t1 + 1) / 2;
                const float rf = 32.f * r2;
                const int i1 = int(rf);
                const float rem = rf - float(i1);
                const float4 tv = __ldg(smooth + size_t(tp) * kBins + i1);
                this_e += tv.x + rem * (tv.z - tv.x);
                const float dor = tv.y + rem * (tv.w - tv.y);
                dx += dor * rx; dy += dor * ry; dz += dor * rz;
            }
        }
        if (this_e > 0.f) {
            const float tt = v / (v + this_e);
            this_e *= tt;
            dx *= tt * tt; dy *= tt * tt; dz *= tt * tt;
        }
        gx = dx + slope * od[0];
        gy = dy + slope * od[1];
        gz = dz + slope * od[2];
        return this_e + slope * oob;
    }
};

// ------------------------------------------------------------ cluster
struct ClusterParams {
    const float4* pool;
    const int64_t* lig_off;
    const int32_t* prefix;      // items of ligand i: [prefix[i], prefix[i+1])
    const float* conf;          // [items][stride]
    const float* e;
    int32_t stride;
    float min_rmsd;
    int32_t max_keep;
    int32_t* kept;              // [n_ligs][20] item indices, -1 padded
    int32_t sort_n;             // power of two >= chains per ligand
    int32_t warp_floats;
};

__device__ __forceinline__ uint32_t ordered(float f) {
    const uint32_t u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}

__global__ void __launch_bounds__(256) cluster_kernel(ClusterParams p) {
    extern __shared__ float4 smem4[];
    unsigned long long* keys = reinterpret_cast<unsigned long long*>(smem4);
    const int li = blockIdx.x;
    const int b0 = p.prefix[li], n = p.prefix[li + 1] - b0;
    for (int i = threadIdx.x; i < p.sort_n; i += blockDim.x) {
        unsigned long long k = ~0ull;
        if (i < n) {
            const float e = p.e[b0 + i];
            if (e == e && e < FLT_MAX) k = (static_cast<unsigned long long>(ordered(e)) << 32) | uint32_t(i);
        }
        keys[i] = k;
    }
    __syncthreads();
    for (int size = 2; size <= p.sort_n; size <<= 1)  // bitonic sort, ascending
        for (int stride = size >> 1; stride > 0; stride >>= 1) {
            for (int i = threadIdx.x; i < p.sort_n; i += blockDim.x) {
                const int j = i ^ stride;
                if (j > i) {
                    const bool up = (i & size) == 0;
                    const unsigned long long a = keys[i], b = keys[j];
                    if ((a > b) == up) { keys[i] = b; keys[j] = a; }
                }
            }
            __syncthreads();
        }
    if (threadIdx.x >= 32) return;
    const int lane = threadIdx.x;
    const LigView L = lig_view(p.pool, p.lig_off[li]);
    float* wbase = reinterpret_cast<float*>(keys + p.sort_n);
    WarpMem m = carve(wbase, L.na, L.nn, L.np, L.nt);
    float* kc = wbase + p.warp_floats;  // kept coordinates [20][na][3]
    int nk = 0;
    const int nc = 7 + L.nt;
    for (int r = 0; r < n && nk < p.max_keep; ++r) {
        const unsigned long long k = keys[r];
        if (k == ~0ull) break;
        const int item = b0 + VD_DCLAMP(int(uint32_t(k)), 0, n - 1, kChkClusterKept);
        for (int i = lane; i < nc; i += 32) m.x[i] = p.conf[size_t(item) * p.stride + i];
        __syncwarp();
        kinematics(L, m, lane);
        bool close = false;
        for (int j = 0; j < nk && !close; ++j) {
            const float* c = kc + size_t(j) * 3 * L.na;
            float acc = 0.f;
            for (int i = lane; i < L.na; i += 32) {
                const float dx = m.c[i].x - c[3 * i], dy = m.c[i].y - c[3 * i + 1], dz = m.c[i].z - c[3 * i + 2];
                acc += dx * dx + dy * dy + dz * dz;
            }
            acc = warp_sum(acc);
            close = sqrtf(acc / float(L.na)) < p.min_rmsd;
        }
        if (close) continue;
        float* c = kc + size_t(nk) * 3 * L.na;
        for (int i = lane; i < L.na; i += 32) { c[3 * i] = m.c[i].x; c[3 * i + 1] = m.c[i].y; c[3 * i + 2] = m.c[i].z; }
        if (lane == 0) p.kept[li * VD_MAX_MODES + nk] = item;
        ++nk;
        __syncwarp();
    }
    for (int j = nk + lane; j < VD_MAX_MODES; j += 32) p.kept[li * VD_MAX_MODES + j] = -1;
}

// ------------------------------------------------------------ refine
struct RefineParams {
    const float4* pool;
    const int64_t* lig_off;     // per ligand in batch
    const int32_t* pose_lig;    // [n_poses] ligand (batch index) of each pose
    float* poses;               // [n_poses][stride] in/out
    float* e_out;               // [n_poses]
    int32_t stride;
    int32_t n_poses;
    int32_t max_steps_default;
    const int32_t* max_steps;   // per ligand (may be null)
    RecView R;
    const float4* smooth;
    float fix, inv_fix;         // fixed-point scale of the pair forces (EvalParams::fix) and 1/fix
    int32_t warp_floats;
    unsigned long long* evals;
    int32_t skip_invalid;       // leave poses whose e_out is FLT_MAX untouched
};

constexpr int kRefineWarps = 4;

__device__ __forceinline__ bool m_out(float v, double b, double e) {
    return v < float(b - 1e-4) || v > float(e + 1e-4);
}

__global__ void __launch_bounds__(32 * kRefineWarps) refine_kernel(RefineParams p) {
    extern __shared__ float4 smem4[];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    float* base = reinterpret_cast<float*>(smem4) + size_t(wid) * p.warp_floats;
    int evals = 0;
    for (int pose = blockIdx.x * kRefineWarps + wid; pose < p.n_poses; pose += gridDim.x * kRefineWarps) {
        const int li = p.pose_lig ? p.pose_lig[pose] : 0;
        if (p.skip_invalid && !(p.e_out[pose] < FLT_MAX)) continue;
        const LigView L = lig_view(p.pool, p.lig_off[li]);
        const int n = 6 + L.nt, nc = 7 + L.nt;
        SearchMem s;
        s.m = carve(base, L.na, L.nn, L.np, L.nt);
        s.xp = base + warp_floats(L.na, L.nn, L.np, L.nt);
        s.xo = s.xp + pad4(nc);
        float* H = s.xo + pad4(nc);
        float* gc = H + pad4(n * n);
        float* pv = gc + pad4(n);
        float* yv = pv + pad4(n);
        float* mhy = yv + pad4(n);
        float* x = p.poses + size_t(pose) * p.stride;
        for (int i = lane; i < nc; i += 32) s.m.x[i] = x[i];
        __syncwarp();
        const int max_steps = p.max_steps ? p.max_steps[li] : p.max_steps_default;
        float e = FLT_MAX;
        bool inside = false;
        for (int ramp = 0; ramp < 5; ++ramp) {
            const float slope = 100.f * powf(10.f, 2.f * ramp);
            const DirectInter di{&p.R, p.smooth, 1000.f, slope};
            e = dense_bfgs(L, s, H, gc, pv, yv, mhy, di, p.smooth, 1000.f, p.fix, p.inv_fix, max_steps, lane, evals);
            kinematics(L, s.m, lane);
            bool ok = true;  // non_cache::within, margin 1e-4
            for (int i = lane; i < L.na; i += 32) {
                if (m_out(s.m.c[i].x, p.R.gb[0], p.R.ge[0]) || m_out(s.m.c[i].y, p.R.gb[1], p.R.ge[1]) ||
                    m_out(s.m.c[i].z, p.R.gb[2], p.R.ge[2]))
                    ok = false;
            }
            inside = __all_sync(0xffffffffu, ok);
            if (inside) break;
        }
        if (!inside) e = FLT_MAX;
        for (int i = lane; i < nc; i += 32) x[i] = s.m.x[i];
        if (lane == 0) p.e_out[pose] = e;
        __syncwarp();
    }
    if (lane == 0 && evals) atomicAdd(p.evals, (unsigned long long)evals);
}

// ------------------------------------------------------------ score (double)
struct ScoreParams {
    const float4* pool;
    const int64_t* lig_off;
    const float* poses;         // [n_ligs][20][stride] refined poses
    const float* e_ref;         // [n_ligs][20] refined energies (FLT_MAX = rejected)
    const int32_t* n_in;        // [n_ligs] poses per ligand
    int32_t stride;
    RecView R;
    const double* fastd;        // [153][kBins]
    double w_rot;               // 0.1 * (weights[5] + 1)
    int32_t num_modes;
    double energy_range;
    double min_rmsd;
    vd_dock_result* out;        // [n_ligs]
};

// Heavy-atom coordinates of a pose in double (same frame walk as kinematics).
__device__ void coords_d(const LigView& L, const float* pose, double* nd, double* c, int lane) {
    for (int k = lane; k < L.nn; k += 32) {
        double* a = nd + 8 * k;
        a[0] = 1; a[1] = a[2] = a[3] = 0;
        if (k > 0) {
            const double th = 0.5 * double(pose[7 + k - 1]);
            const double s = sin(th), co = cos(th);
            a[0] = co; a[1] = s * double(L.nodes[k].axis[0]); a[2] = s * double(L.nodes[k].axis[1]);
            a[3] = s * double(L.nodes[k].axis[2]);
        }
    }
    __syncwarp();
    double* fr = nd + 8 * L.nn;  // per node: q[4], o[3]
    const double qr[4] = {pose[3], pose[4], pose[5], pose[6]};
    for (int k = lane; k < L.nn; k += 32) {
        double P[4] = {1, 0, 0, 0}, w[3] = {0, 0, 0};
        if (k > 0) {
            for (int i = 0; i < 4; ++i) P[i] = nd[8 * k + i];
            for (int i = 0; i < 3; ++i) w[i] = L.nodes[k].rel_origin[i];
            int j = L.nodes[k].parent;
            while (j > 0) {
                const double* A = nd + 8 * j;
                // w = rel_origin_j + rot(A) w
                const double tx = A[2] * w[2] - A[3] * w[1] + A[0] * w[0];
                const double ty = A[3] * w[0] - A[1] * w[2] + A[0] * w[1];
                const double tz = A[1] * w[1] - A[2] * w[0] + A[0] * w[2];
                const double r0 = w[0] + 2 * (A[2] * tz - A[3] * ty), r1 = w[1] + 2 * (A[3] * tx - A[1] * tz),
                             r2 = w[2] + 2 * (A[1] * ty - A[2] * tx);
                w[0] = L.nodes[j].rel_origin[0] + r0;
                w[1] = L.nodes[j].rel_origin[1] + r1;
                w[2] = L.nodes[j].rel_origin[2] + r2;
                const double n0 = A[0] * P[0] - A[1] * P[1] - A[2] * P[2] - A[3] * P[3];
                const double n1 = A[0] * P[1] + A[1] * P[0] + A[2] * P[3] - A[3] * P[2];
                const double n2 = A[0] * P[2] - A[1] * P[3] + A[2] * P[0] + A[3] * P[1];
                const double n3 = A[0] * P[3] + A[1] * P[2] - A[2] * P[1] + A[3] * P[0];
                P[0] = n0; P[1] = n1; P[2] = n2; P[3] = n3;
                j = L.nodes[j].parent;
            }
        }
        double q[4] = {qr[0] * P[0] - qr[1] * P[1] - qr[2] * P[2] - qr[3] * P[3],
                       qr[0] * P[1] + qr[1] * P[0] + qr[2] * P[3] - qr[3] * P[2],
                       qr[0] * P[2] - qr[1] * P[3] + qr[2] * P[0] + qr[3] * P[1],
                       qr[0] * P[3] + qr[1] * P[2] - qr[2] * P[1] + qr[3] * P[0]};
        const double inv = 1.0 / sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
        for (int i = 0; i < 4; ++i) q[i] *= inv;
        const double tx = qr[2] * w[2] - qr[3] * w[1] + qr[0] * w[0];
        const double ty = qr[3] * w[0] - qr[1] * w[2] + qr[0] * w[1];
        const double tz = qr[1] * w[1] - qr[2] * w[0] + qr[0] * w[2];
        double* f = fr + 8 * k;
        for (int i = 0; i < 4; ++i) f[i] = q[i];
        f[4] = double(pose[0]) + w[0] + 2 * (qr[2] * tz - qr[3] * ty);
        f[5] = double(pose[1]) + w[1] + 2 * (qr[3] * tx - qr[1] * tz);
        f[6] = double(pose[2]) + w[2] + 2 * (qr[1] * ty - qr[2] * tx);
    }
    __syncwarp();
    for (int i = lane; i < L.na; i += 32) {
        const float4 a = L.atoms[i];
        const int k = (__float_as_int(a.w) >> 8) & 0xff;
        const double* f = fr + 8 * k;
        const double v[3] = {a.x, a.y, a.z};
        const double tx = f[2] * v[2] - f[3] * v[1] + f[0] * v[0];
        const double ty = f[3] * v[0] - f[1] * v[2] + f[0] * v[1];
        const double tz = f[1] * v[1] - f[2] * v[0] + f[0] * v[2];
        c[3 * i] = f[4] + v[0] + 2 * (f[2] * tz - f[3] * ty);
        c[3 * i + 1] = f[5] + v[1] + 2 * (f[3] * tx - f[1] * tz);
        c[3 * i + 2] = f[6] + v[2] + 2 * (f[1] * ty - f[2] * tx);
    }
    __syncwarp();
}

__device__ __forceinline__ double warp_sum_d(double v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// model.cpp:1206-1219 (eval_interacting_pairs, eval_fast, curl 1000)
__device__ double intra_fast(const LigView& L, const double* c, const double* fastd, int lane) {
    double e = 0;
    for (int p = lane; p < L.np; p += 32) {
        const int2 pr = L.pairs[p];
        const int a = pr.x & 0xffff, b = pr.x >> 16;
        const double dx = c[3 * a] - c[3 * b], dy = c[3 * a + 1] - c[3 * b + 1], dz = c[3 * a + 2] - c[3 * b + 2];
        const double r2 = (dx * dx + dy * dy) + dz * dz;
        if (r2 < 64.0) {
            double t = fastd[size_t(pr.y) * kBins + int(32.0 * r2)];
            if (t > 0) t *= 1000.0 / (1000.0 + t);
            e += t;
        }
    }
    return warp_sum_d(e);
}

// non_cache.cpp:20-55 (non_cache::eval, eval_fast, curl 1000, slope 1e6)
__device__ double inter_fast(const LigView& L, const RecView& R, const double* c, const double* fastd, int lane) {
    double e = 0;
    for (int i = lane; i < L.na; i += 32) {
        const int t1 = __float_as_int(L.atoms[i].w) & 0xff;
        double a[3] = {c[3 * i], c[3 * i + 1], c[3 * i + 2]}, oob = 0;
        for (int d = 0; d < 3; ++d) {
            if (a[d] < R.gb[d]) { oob += fabs(a[d] - R.gb[d]); a[d] = R.gb[d]; }
            else if (a[d] > R.ge[d]) { oob += fabs(a[d] - R.ge[d]); a[d] = R.ge[d]; }
        }
        oob *= 1e6;
        const int ce = cell_of(R, a[0], a[1], a[2]);
        double this_e = 0;
        for (int q = R.cell_start[ce]; q < R.cell_start[ce + 1]; ++q) {
            const double4 b = R.recd[R.cell_list[q]];
            const double rx = a[0] - b.x, ry = a[1] - b.y, rz = a[2] - b.z;
            const double r2 = (rx * rx + ry * ry) + rz * rz;
            if (r2 < 64.0) {
                const int t2 = int(b.w);
                const int tp = (t1 <= t2) ? t1 + t2 * (t2 + 1) / 2 : t2 + t1 * (t1 + 1) / 2;
                this_e += fastd[size_t(tp) * kBins + int(32.0 * r2)];
            }
        }
        if (this_e > 0) this_e *= 1000.0 / (1000.0 + this_e);
        e += this_e + oob;
    }
    return warp_sum_d(e);
}

// Kept chain results -> refinement buffer ([ligand][20] slots).
__global__ void gather_kernel(const int32_t* kept, const float* conf, const float* e, int stride, int n_slots,
                              float* rp, float* re) {
    const int slot = blockIdx.x;
    if (slot >= n_slots) return;
    const int item = kept[slot];
    for (int i = threadIdx.x; i < stride; i += blockDim.x)
        rp[size_t(slot) * stride + i] = item >= 0 ? conf[size_t(item) * stride + i] : 0.f;
    if (threadIdx.x == 0) re[slot] = item >= 0 ? e[item] : FLT_MAX;
}

// model.cpp:1485-1523: RMSD upper bound (each heavy atom to the same atom)
// and lower bound (each heavy atom to the nearest atom of the same element,
// the larger of the two directions) between heavy-atom coordinate sets a and
// b ([na][3] floats); sums in double.  Same value in every lane.
__device__ void rmsd_bounds(const LigView& L, const float* a, const float* b, int lane, double& lb, double& ub) {
    double su = 0, s1 = 0, s2 = 0;
    for (int i = lane; i < L.na; i += 32) {
        const int ei = (__float_as_int(L.atoms[i].w) >> 16) & 0xff;
        double d2 = 0, m1 = DBL_MAX, m2 = DBL_MAX;
        for (int d = 0; d < 3; ++d) d2 += double(a[3 * i + d] - b[3 * i + d]) * double(a[3 * i + d] - b[3 * i + d]);
        for (int q = 0; q < L.na; ++q) {
            if (((__float_as_int(L.atoms[q].w) >> 16) & 0xff) != ei) continue;
            double t1 = 0, t2 = 0;
            for (int d = 0; d < 3; ++d) {
                t1 += double(a[3 * i + d] - b[3 * q + d]) * double(a[3 * i + d] - b[3 * q + d]);
                t2 += double(b[3 * i + d] - a[3 * q + d]) * double(b[3 * i + d] - a[3 * q + d]);
            }
            m1 = fmin(m1, t1);
            m2 = fmin(m2, t2);
        }
        su += d2; s1 += m1; s2 += m2;
    }
    su = warp_sum_d(su); s1 = warp_sum_d(s1); s2 = warp_sum_d(s2);
    ub = sqrt(su / L.na);
    lb = fmax(sqrt(s1 / L.na), sqrt(s2 / L.na));
}

// RMSD bounds of poses to pose 0 (vd_rmsd_bounds): heavy-atom coordinates in
// double, stored as floats as the output stage stores its kept modes.
__global__ void __launch_bounds__(32) rmsd_poses_kernel(const float4* pool, const int64_t* off, const float* poses,
                                                         int n, int stride, double* out) {
    extern __shared__ double smemd[];
    const int lane = threadIdx.x;
    const LigView L = lig_view(pool, off[0]);
    double* nd = smemd;
    double* c = nd + 16 * L.nn;
    float* k0 = reinterpret_cast<float*>(c + 3 * L.na);
    float* ki = k0 + 3 * L.na;
    coords_d(L, poses, nd, c, lane);
    for (int a = lane; a < 3 * L.na; a += 32) k0[a] = float(c[a]);
    __syncwarp();
    for (int i = 0; i < n; ++i) {
        coords_d(L, poses + size_t(i) * stride, nd, c, lane);
        for (int a = lane; a < 3 * L.na; a += 32) ki[a] = float(c[a]);
        __syncwarp();
        double lb, ub;
        rmsd_bounds(L, ki, k0, lane, lb, ub);
        if (lane == 0) {
            out[2 * i] = lb;
            out[2 * i + 1] = ub;
        }
        __syncwarp();
    }
}

// Adjusted score and intramolecular energy of up to 20 poses (vd_score).
__global__ void __launch_bounds__(32) score_poses_kernel(const float4* pool, const int64_t* off, const float* poses,
                                                          int n, int stride, RecView R, const double* fastd,
                                                          double w_rot, double* out) {
    extern __shared__ double smemd[];
    const int lane = threadIdx.x;
    const LigView L = lig_view(pool, off[0]);
    double* nd = smemd;
    double* c = nd + 16 * L.nn;
    double intra0 = 0;
    for (int i = 0; i < n; ++i) {
        coords_d(L, poses + size_t(i) * stride, nd, c, lane);
        const double intra = intra_fast(L, c, fastd, lane);
        if (i == 0) intra0 = intra;
        const double e = inter_fast(L, R, c, fastd, lane) + intra;
        const double x = e - intra0, y = 1 + w_rot * double(L.num_tors) / 5.0;
        if (lane == 0) {
            out[2 * i] = (fabs(x) < DBL_EPSILON) ? 0.0 : x / y;
            out[2 * i + 1] = intra;
        }
        __syncwarp();
    }
}

__global__ void __launch_bounds__(32) score_kernel(ScoreParams p) {
    extern __shared__ double smemd[];
    const int li = blockIdx.x, lane = threadIdx.x;
    const LigView L = lig_view(p.pool, p.lig_off[li]);
    double* nd = smemd;                        // [nn][8] + [nn][8]
    double* c = nd + 16 * L.nn;                // [na][3]
    float* kc = reinterpret_cast<float*>(c + 3 * L.na);  // [20][na][3]
    __shared__ int order[VD_MAX_MODES], kept[VD_MAX_MODES];
    __shared__ double adj[VD_MAX_MODES];
    const int n = p.n_in[li];
    const float* poses = p.poses + size_t(li) * VD_MAX_MODES * p.stride;
    const float* er = p.e_ref + size_t(li) * VD_MAX_MODES;
    vd_dock_result* out = p.out + li;
    if (lane == 0) {
        for (int i = 0; i < n; ++i) order[i] = i;
        for (int i = 1; i < n; ++i)  // stable insertion sort by refined energy
            for (int j = i; j > 0 && er[order[j]] < er[order[j - 1]]; --j) {
                const int t = order[j]; order[j] = order[j - 1]; order[j - 1] = t;
            }
    }
    __syncwarp();
    double intra_best = 0;
    if (n > 0) {
        coords_d(L, poses + size_t(order[0]) * p.stride, nd, c, lane);
        intra_best = intra_fast(L, c, p.fastd, lane);
    }
    for (int i = 0; i < n; ++i) {
        double v = DBL_MAX;
        if (er[i] < FLT_MAX) {
            coords_d(L, poses + size_t(i) * p.stride, nd, c, lane);
            const double e = inter_fast(L, p.R, c, p.fastd, lane) + intra_fast(L, c, p.fastd, lane);
            const double x = e - intra_best, y = 1 + p.w_rot * double(L.num_tors) / 5.0;
            v = (fabs(x) < DBL_EPSILON) ? 0.0 : x / y;  // smooth_div, everything.cpp:232-236
        }
        if (lane == 0) adj[i] = v;
    }
    __syncwarp();
    if (lane == 0) {
        for (int i = 0; i < n; ++i) order[i] = i;
        for (int i = 1; i < n; ++i)
            for (int j = i; j > 0 && adj[order[j]] < adj[order[j - 1]]; --j) {
                const int t = order[j]; order[j] = order[j - 1]; order[j - 1] = t;
            }
    }
    __syncwarp();
    int nk = 0;  // remove_redundant (main.cpp:172-178) then the mode cut
    for (int r = 0; r < n; ++r) {
        const int i = order[r];
        if (!(adj[i] < 0.1 * DBL_MAX)) break;
        if (nk >= p.num_modes) break;
        if (nk > 0 && adj[i] > adj[kept[0]] + p.energy_range) break;
        coords_d(L, poses + size_t(i) * p.stride, nd, c, lane);
        bool close = false;
        for (int j = 0; j < nk && !close; ++j) {
            const float* k = kc + size_t(j) * 3 * L.na;
            double acc = 0;
            for (int a = lane; a < L.na; a += 32)
                for (int d = 0; d < 3; ++d) acc += (c[3 * a + d] - k[3 * a + d]) * (c[3 * a + d] - k[3 * a + d]);
            acc = warp_sum_d(acc);
            close = sqrt(acc / L.na) < p.min_rmsd;
        }
        if (close) continue;
        float* k = kc + size_t(nk) * 3 * L.na;
        for (int a = lane; a < 3 * L.na; a += 32) k[a] = float(c[a]);
        if (lane == 0) kept[nk] = i;
        ++nk;
        __syncwarp();
    }
    __syncwarp();
    // outputs with RMSD bounds to mode 1 (model.cpp:1485-1523)
    for (int j = 0; j < nk; ++j) {
        double lb, ub;
        rmsd_bounds(L, kc + size_t(j) * 3 * L.na, kc, lane, lb, ub);
        const int i = kept[j];
        if (lane == 0) {
            out->energy[j] = float(adj[i]);
            out->rmsd_ub[j] = float(ub);
            out->rmsd_lb[j] = float(lb);
        }
        for (int q = lane; q < 7 + L.nt; q += 32) out->pose[j][q] = poses[size_t(i) * p.stride + q];
    }
    if (lane == 0) {
        out->n_modes = nk;
        out->ntors = L.nt;
    }
}

}  // namespace
}  // namespace vd

namespace vd {

// szv_grid over the box (szv_grid.cpp:28-74, 120-131), uploaded once per
// receptor and box.
vd_status ensure_receptor_cells(Ctx* c) {
    if (c->rec_dev_ready) return VD_OK;
    VD_CHECK(c->has_box, VD_ERR_ARG, "no box set");
    const GridGeom& g = c->geom;
    double init[3], range[3], end[3];
    int dim[3];
    for (int d = 0; d < 3; ++d) {
        init[d] = g.begin[d];
        end[d] = g.end[d];
        const int n_int = int((g.end[d] - g.begin[d]) / 3);
        dim[d] = n_int < 1 ? 1 : n_int;
    }
    for (int d = 0; d < 3; ++d) range[d] = end[d] - init[d];
    auto brick = [](const double* b, const double* e, const double* v) {
        double d2 = 0;
        for (int i = 0; i < 3; ++i) {
            const double q = (v[i] <= b[i]) ? b[i] : ((v[i] >= e[i]) ? e[i] : v[i]);
            d2 += (q - v[i]) * (q - v[i]);
        }
        return d2;
    };
    std::vector<int> rel;
    const int n_rec = int(c->rec_xs.size());
    for (int i = 0; i < n_rec; ++i)
        if (c->rec_xs[i] >= 0 && brick(init, end, &c->rec_xyz[3 * size_t(i)]) < kCutoff2) rel.push_back(i);
    const int ncell = dim[0] * dim[1] * dim[2];
    std::vector<std::vector<int>> cells(ncell);
    auto coord = [&](int d, int i) { return init[d] + range[d] * i / dim[d]; };
    for (int r = 0; r < int(rel.size()); ++r) {
        const double* a = &c->rec_xyz[3 * size_t(rel[r])];
        int lo[3], hi[3];
        for (int d = 0; d < 3; ++d) {  // candidate cells within the cutoff, then the exact test
            lo[d] = std::max(0, int(std::floor((a[d] - 8.0 - init[d]) * dim[d] / range[d])) - 1);
            hi[d] = std::min(dim[d] - 1, int(std::floor((a[d] + 8.0 - init[d]) * dim[d] / range[d])) + 1);
        }
        for (int z = lo[2]; z <= hi[2]; ++z)
            for (int y = lo[1]; y <= hi[1]; ++y)
                for (int x = lo[0]; x <= hi[0]; ++x) {
                    const double b[3] = {coord(0, x), coord(1, y), coord(2, z)};
                    const double e[3] = {coord(0, x + 1), coord(1, y + 1), coord(2, z + 1)};
                    if (brick(b, e, a) < kCutoff2) cells[x + dim[0] * (y + dim[1] * z)].push_back(r);
                }
    }
    std::vector<int32_t> start(ncell + 1, 0), list;
    for (int i = 0; i < ncell; ++i) {
        start[i + 1] = start[i] + int(cells[i].size());
        list.insert(list.end(), cells[i].begin(), cells[i].end());
    }
    std::vector<float4> rf(std::max<size_t>(1, rel.size()));
    std::vector<double4> rd(std::max<size_t>(1, rel.size()));
    for (size_t r = 0; r < rel.size(); ++r) {
        const double* a = &c->rec_xyz[3 * size_t(rel[r])];
        rf[r] = make_float4(float(a[0]), float(a[1]), float(a[2]), float(c->rec_xs[rel[r]]));
        rd[r] = make_double4(a[0], a[1], a[2], double(c->rec_xs[rel[r]]));
    }
    dev_release(*c, c->d_rec);
    dev_release(*c, c->d_recd);
    dev_release(*c, c->d_cell_start);
    dev_release(*c, c->d_cell_list);
    vd_status st = dev_alloc(*c, &c->d_rec, rf.size() * sizeof(float4), "receptor cells");
    if (st == VD_OK) st = dev_alloc(*c, &c->d_recd, rd.size() * sizeof(double4), "receptor cells");
    if (st == VD_OK) st = dev_alloc(*c, &c->d_cell_start, start.size() * sizeof(int32_t), "receptor cells");
    if (st == VD_OK)
        st = dev_alloc(*c, &c->d_cell_list, std::max<size_t>(1, list.size()) * sizeof(int32_t), "receptor cells");
    if (st != VD_OK) {
        dev_release(*c, c->d_rec);
        dev_release(*c, c->d_recd);
        dev_release(*c, c->d_cell_start);
        dev_release(*c, c->d_cell_list);
        return st;
    }
    VD_CUDA(cudaMemcpy(c->d_rec, rf.data(), rf.size() * sizeof(float4), cudaMemcpyHostToDevice));
    VD_CUDA(cudaMemcpy(c->d_recd, rd.data(), rd.size() * sizeof(double4), cudaMemcpyHostToDevice));
    VD_CUDA(cudaMemcpy(c->d_cell_start, start.data(), start.size() * sizeof(int32_t), cudaMemcpyHostToDevice));
    if (!list.empty())
        VD_CUDA(cudaMemcpy(c->d_cell_list, list.data(), list.size() * sizeof(int32_t), cudaMemcpyHostToDevice));
    for (int d = 0; d < 3; ++d) {
        c->cell_dim[d] = dim[d];
        c->cell_init[d] = init[d];
        c->cell_range[d] = range[d];
    }
    c->n_rec_dev = int(rel.size());
    c->rec_dev_ready = true;
    return VD_OK;
}

namespace {

RecView rec_view(const Ctx& c) {
    RecView R;
    R.rec = c.d_rec;
    R.recd = c.d_recd;
    R.cell_start = c.d_cell_start;
    R.cell_list = c.d_cell_list;
    for (int d = 0; d < 3; ++d) {
        R.init[d] = c.cell_init[d];
        R.range[d] = c.cell_range[d];
        R.dim[d] = c.cell_dim[d];
        R.gb[d] = c.geom.begin[d];
        R.ge[d] = c.geom.end[d];
    }
    return R;
}

int refine_warp_floats(const HostLigand& L) {
    const int n = 6 + L.h.ntors, nc = 7 + L.h.ntors;
    return lig_warp_floats(L) + 2 * pad4(nc) + pad4(n * n) + 4 * pad4(n);
}

inline size_t al256(size_t b) { return (b + 255) & ~size_t(255); }

// Host side of cluster -> gather -> refine -> score for the ligands of one
// dock launch: parameters, device layout in the dock's extra scratch
// (params: off | prefix | steps | pose ligand | n_in, then kept poses and
// results) and the kernel launches; no stream operation.
struct PostPlan {
    std::vector<unsigned char> h_params;
    void* d_params = nullptr;
    vd_dock_result* d_out = nullptr;
    int n = 0;
    std::function<cudaError_t(cudaStream_t)> launch;
};

vd_status prepare_post(Ctx& c, const std::vector<int>& ligs, const vd_search_params& sp, const DockBuffers& db,
                       PostPlan& pp) {
    vd_status st = ensure_receptor_cells(&c);
    if (st != VD_OK) return st;
    const int n = int(ligs.size());
    int max_chains = 0, max_wf = 0, max_rwf = 0, max_na = 0, max_nn = 0;
    std::vector<int64_t> off(n);
    std::vector<int32_t> steps(n), depth(n);
    for (int i = 0; i < n; ++i) {
        const HostLigand& L = c.ligs[ligs[i]];
        off[i] = L.pool_offset;
        search_defaults(L, sp, depth[i], steps[i]);
        max_chains = std::max(max_chains, db.prefix[i + 1] - db.prefix[i]);
        max_wf = std::max(max_wf, lig_warp_floats(L));
        max_rwf = std::max(max_rwf, refine_warp_floats(L));
        max_na = std::max(max_na, L.h.n_atoms);
        max_nn = std::max(max_nn, L.h.n_nodes);
    }
    int sort_n = 2;  // >= 2: the warp's arrays after the 8-byte keys start 16-byte aligned
    while (sort_n < max_chains) sort_n <<= 1;
    VD_CHECK(sort_n <= 16384, VD_ERR_CAPACITY, "more than 16384 chains per ligand");
    std::vector<int32_t> plig(size_t(n) * VD_MAX_MODES), nin(n, VD_MAX_MODES);
    for (int i = 0; i < n * VD_MAX_MODES; ++i) plig[i] = i / VD_MAX_MODES;
    // parameter arrays (host), mirrored at the start of the extra scratch
    size_t o = 0;
    const size_t b_par = al256(n * sizeof(int64_t)) + al256((n + 1) * sizeof(int32_t)) + al256(n * sizeof(int32_t)) +
                         al256(plig.size() * sizeof(int32_t)) + al256(n * sizeof(int32_t));
    pp.h_params.assign(b_par, 0);
    char* s = db.d_extra;
    pp.d_params = s;
    auto put = [&](const void* src, size_t bytes) {
        std::memcpy(pp.h_params.data() + o, src, bytes);
        char* d = s + o;
        o += al256(bytes);
        return d;
    };
    const int64_t* d_off = reinterpret_cast<const int64_t*>(put(off.data(), n * sizeof(int64_t)));
    const int32_t* d_pre = reinterpret_cast<const int32_t*>(put(db.prefix.data(), (n + 1) * sizeof(int32_t)));
    const int32_t* d_steps = reinterpret_cast<const int32_t*>(put(steps.data(), n * sizeof(int32_t)));
    const int32_t* d_plig = reinterpret_cast<const int32_t*>(put(plig.data(), plig.size() * sizeof(int32_t)));
    const int32_t* d_nin = reinterpret_cast<const int32_t*>(put(nin.data(), n * sizeof(int32_t)));
    s += b_par;
    int32_t* d_kept = reinterpret_cast<int32_t*>(s); s += al256(size_t(n) * VD_MAX_MODES * sizeof(int32_t));
    float* d_rp = reinterpret_cast<float*>(s); s += al256(size_t(n) * VD_MAX_MODES * db.stride * sizeof(float));
    float* d_re = reinterpret_cast<float*>(s); s += al256(size_t(n) * VD_MAX_MODES * sizeof(float));
    vd_dock_result* d_out = reinterpret_cast<vd_dock_result*>(s);
    pp.d_out = d_out;
    pp.n = n;
    // cluster
    ClusterParams cp{};
    cp.pool = c.d_pool;
    cp.lig_off = d_off;
    cp.prefix = d_pre;
    cp.conf = db.d_conf;
    cp.e = db.d_e;
    cp.stride = db.stride;
    cp.min_rmsd = float(sp.min_rmsd > 0 ? sp.min_rmsd : 1.0);
    cp.max_keep = VD_MAX_MODES;
    cp.kept = d_kept;
    cp.sort_n = sort_n;
    cp.warp_floats = max_wf;
    const size_t smem_c = size_t(sort_n) * 8 + size_t(max_wf) * 4 + size_t(VD_MAX_MODES) * 3 * max_na * 4;
    VD_CHECK(smem_c <= 227 * 1024, VD_ERR_CAPACITY, "cluster kernel shared memory exceeds 227 KB");
    VD_CUDA(cudaFuncSetAttribute(cluster_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem_c)));
    // refine
    const bool refine = sp.refine != 0;
    RefineParams rp{};
    size_t smem_r = 0;
    int blocks_r = 0;
    if (refine) {
        rp.pool = c.d_pool;
        rp.lig_off = d_off;
        rp.pose_lig = d_plig;
        rp.poses = d_rp;
        rp.e_out = d_re;
        rp.stride = db.stride;
        rp.n_poses = n * VD_MAX_MODES;
        rp.max_steps = d_steps;
        rp.R = rec_view(c);
        rp.smooth = c.d_smooth;
        rp.fix = c.fix_scale;
        rp.inv_fix = 1.f / c.fix_scale;
        rp.warp_floats = max_rwf;
        rp.evals = reinterpret_cast<unsigned long long*>(c.d_counter + 4);
        rp.skip_invalid = 1;
        smem_r = size_t(max_rwf) * kRefineWarps * 4;
        VD_CHECK(smem_r <= 227 * 1024, VD_ERR_CAPACITY, "refine kernel shared memory exceeds 227 KB");
        VD_CUDA(cudaFuncSetAttribute(refine_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem_r)));
        blocks_r = (n * VD_MAX_MODES + kRefineWarps - 1) / kRefineWarps;
    }
    // score
    ScoreParams sc{};
    sc.pool = c.d_pool;
    sc.lig_off = d_off;
    sc.poses = d_rp;
    sc.e_ref = d_re;
    sc.n_in = d_nin;
    sc.stride = db.stride;
    sc.R = rec_view(c);
    sc.fastd = c.d_fastd;
    sc.w_rot = 0.1 * (c.weights[5] + 1);
    sc.num_modes = std::max(1, std::min(VD_MAX_MODES, sp.num_modes > 0 ? sp.num_modes : 9));
    sc.energy_range = sp.energy_range > 0 ? sp.energy_range : 3.0;
    sc.min_rmsd = 1.0;
    sc.out = d_out;
    const size_t smem_s = size_t(16 * max_nn + 3 * max_na) * 8 + size_t(VD_MAX_MODES) * 3 * max_na * 4;
    VD_CUDA(cudaFuncSetAttribute(score_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem_s)));
    const int stride = db.stride;
    const float* conf = db.d_conf;
    const float* e = db.d_e;
    pp.launch = [=](cudaStream_t stream) {
        cluster_kernel<<<n, 256, smem_c, stream>>>(cp);
        // gather kept poses (missing slots get e = FLT_MAX)
        gather_kernel<<<n * VD_MAX_MODES, 64, 0, stream>>>(d_kept, conf, e, stride, n * VD_MAX_MODES, d_rp, d_re);
        if (refine) refine_kernel<<<blocks_r, 32 * kRefineWarps, smem_r, stream>>>(rp);
        score_kernel<<<n, 32, smem_s, stream>>>(sc);
        return cudaGetLastError();
    };
    return VD_OK;
}

// Stream side: parameter upload, the kernels (ending at c.ev2), the results
// to out (host, pinned for graph capture).
vd_status enqueue_post(Ctx& c, const PostPlan& pp, const void* params_src, vd_dock_result* out,
                       cudaStream_t stream) {
    VD_CUDA(cudaMemcpyAsync(pp.d_params, params_src, pp.h_params.size(), cudaMemcpyHostToDevice, stream));
    VD_CUDA(pp.launch(stream));
    VD_CUDA(record_event(c.ev2, stream));
    VD_CUDA(cudaMemcpyAsync(out, pp.d_out, pp.n * sizeof(vd_dock_result), cudaMemcpyDeviceToHost, stream));
    return VD_OK;
}

// Ends a stream capture left open by an early return.
struct CaptureGuard {
    cudaStream_t s;
    bool open;
    ~CaptureGuard() {
        if (open) {
            cudaGraph_t g = nullptr;
            cudaStreamEndCapture(s, &g);
            if (g) cudaGraphDestroy(g);
        }
    }
};

}  // namespace

size_t post_scratch_bytes(int n_ligs, int stride) {
    return al256(n_ligs * 8) + al256((n_ligs + 1) * 4) + 3 * al256(size_t(n_ligs) * VD_MAX_MODES * 4) +
           2 * al256(n_ligs * 4) + al256(size_t(n_ligs) * VD_MAX_MODES * stride * 4) +
           al256(size_t(n_ligs) * VD_MAX_MODES * 4) + al256(n_ligs * sizeof(vd_dock_result)) + 1024;
}

// Docking of a ligand list followed by the post-processing.  The batched
// (persistent) form records the whole sequence -- parameter uploads from a
// pinned stage, the docking kernel, cluster / gather / refine / score and
// the result download -- into one CUDA graph, updated in place when the
// next call records the same topology, and submits it with one launch; the
// plain form issues the same operations directly, one ligand per launch.
vd_status dock_pipeline(Ctx& c, const std::vector<int>& ligs, const vd_search_params& sp, bool persistent,
                        vd_dock_result* out) {
    VD_CUDA(cudaSetDevice(c.device));
    for (int l : ligs) VD_CHECK(l >= 0 && l < int(c.ligs.size()), VD_ERR_ARG, "bad ligand id");
    int max_nt = 0;
    for (int l : ligs) max_nt = std::max(max_nt, c.ligs[l].h.ntors);
    const int n = int(ligs.size());
    DockBuffers db;
    db.extra_bytes = post_scratch_bytes(n, 7 + max_nt);
    vd_status st = prepare_dock(c, ligs, sp, persistent, db);
    if (st != VD_OK) return st;
    PostPlan pp;
    st = prepare_post(c, ligs, sp, db, pp);
    if (st != VD_OK) return st;
    // pinned stage: [dock params | post params | results | counters]
    const size_t b_dp = al256(db.h_params.size()), b_pp = al256(pp.h_params.size());
    const size_t b_res = al256(n * sizeof(vd_dock_result)), b_cnt = al256((2 + n) * sizeof(unsigned long long));
    st = ensure_host_stage(&c, b_dp + b_pp + b_res + b_cnt);
    if (st != VD_OK) return st;
    unsigned char* hs = static_cast<unsigned char*>(c.h_stage);
    std::memcpy(hs, db.h_params.data(), db.h_params.size());
    std::memcpy(hs + b_dp, pp.h_params.data(), pp.h_params.size());
    vd_dock_result* h_res = reinterpret_cast<vd_dock_result*>(hs + b_dp + b_pp);
    unsigned long long* h_cnt = reinterpret_cast<unsigned long long*>(hs + b_dp + b_pp + b_res);
    auto enqueue_all = [&](cudaStream_t s) -> vd_status {
        vd_status e = enqueue_dock(c, db, hs, s);
        if (e != VD_OK) return e;
        e = enqueue_post(c, pp, hs + b_dp, h_res, s);
        if (e != VD_OK) return e;
        VD_CUDA(cudaMemcpyAsync(h_cnt, c.d_counter + 2, 2 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, s));
        VD_CUDA(cudaMemcpyAsync(h_cnt + 2, db.d_lig_evals, n * sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                                s));
        return VD_OK;
    };
    if (persistent) {
        CaptureGuard guard{c.stream, false};
        VD_CUDA(cudaStreamBeginCapture(c.stream, cudaStreamCaptureModeThreadLocal));
        guard.open = true;
        st = enqueue_all(c.stream);
        if (st != VD_OK) return st;
        cudaGraph_t graph = nullptr;
        guard.open = false;
        VD_CUDA(cudaStreamEndCapture(c.stream, &graph));
        bool updated = false;
        if (c.pipe_exec) {
            cudaGraphExecUpdateResultInfo info{};
            updated = cudaGraphExecUpdate(c.pipe_exec, graph, &info) == cudaSuccess;
            if (!updated) {
                cudaGetLastError();  // clear the update failure; a new executable replaces it
                cudaGraphExecDestroy(c.pipe_exec);
                c.pipe_exec = nullptr;
            }
        }
        cudaError_t e = cudaSuccess;
        if (!updated) {
            e = cudaGraphInstantiate(&c.pipe_exec, graph, 0);
            ++c.stats.graph_instantiations;
        }
        cudaGraphDestroy(graph);
        if (e != cudaSuccess) {
            c.pipe_exec = nullptr;
            set_error(std::string("CUDA graph instantiation failed: ") + cudaGetErrorString(e));
            return VD_ERR_CUDA;
        }
        VD_CUDA(cudaGraphLaunch(c.pipe_exec, c.stream));
        ++c.stats.graph_launches;
    } else {
        st = enqueue_all(c.stream);
        if (st != VD_OK) return st;
    }
    VD_CUDA(cudaStreamSynchronize(c.stream));
    if ((st = dock_take_checks("docking kernel")) != VD_OK) return st;
    if ((st = take_device_checks("post-processing kernels")) != VD_OK) return st;
    float dock_ms = 0, post_ms = 0;
    VD_CUDA(cudaEventElapsedTime(&dock_ms, c.ev0, c.ev1));
    VD_CUDA(cudaEventElapsedTime(&post_ms, c.ev1, c.ev2));
    std::memcpy(out, h_res, n * sizeof(vd_dock_result));
    c.stats.dock_ms = dock_ms;
    c.stats.post_ms = post_ms;
    c.stats.bfgs_evals += int64_t(h_cnt[0] + h_cnt[1]);
    dock_tune_report(c, db, dock_ms, h_cnt + 2);
    for (int i = 0; i < n; ++i) out[i].bfgs_evals = int64_t(h_cnt[2 + i]);  // search evaluations
    return VD_OK;
}

}  // namespace vd

using namespace vd;

extern "C" {

vd_status vd_dock_plain(vd_ctx* h, int32_t lig, const vd_search_params* sp, vd_dock_result* out) {
    VD_CHECK(h && sp && out, VD_ERR_ARG, "vd_dock_plain: NULL argument");
    return dock_pipeline(h->c, {lig}, *sp, false, out);
}

vd_status vd_dock_batched(vd_ctx* h, const int32_t* ligs, int32_t n, const vd_search_params* sp,
                          vd_dock_result* out) {
    VD_CHECK(h && ligs && sp && out && n > 0, VD_ERR_ARG, "vd_dock_batched: bad arguments");
    Ctx& c = h->c;
    for (int i = 0; i < n; ++i) VD_CHECK(ligs[i] >= 0 && ligs[i] < int(c.ligs.size()), VD_ERR_ARG, "bad ligand id");
    // The work queue hands out ligands in the order given; most expensive
    // chains first shortens the tail (a chain's result does not depend on
    // its position in the batch).  Cost = MC steps x BFGS steps x bytes
    // touched per evaluation.
    std::vector<int> order(n);
    std::vector<double> cost(n);
    for (int i = 0; i < n; ++i) {
        const HostLigand& L = c.ligs[ligs[i]];
        int depth = 0, steps = 0;
        search_defaults(L, *sp, depth, steps);
        order[i] = i;
        // depth 0 here means no MC step (a negative search_depth): one evaluation's bytes
        cost[i] = double(depth > 0 ? double(depth) * steps : 1.0) * (32.0 * L.h.n_atoms + 16.0 * L.h.n_pairs);
    }
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return cost[a] > cost[b]; });
    std::vector<int> v(n);
    for (int i = 0; i < n; ++i) v[i] = ligs[order[i]];
    std::vector<vd_dock_result> tmp(n);
    vd_status st = dock_pipeline(c, v, *sp, true, tmp.data());
    if (st != VD_OK) return st;
    for (int i = 0; i < n; ++i) out[order[i]] = tmp[i];
    return VD_OK;
}

vd_status vd_refine(vd_ctx* h, int32_t lig, int32_t n, float* poses, int32_t max_steps, float* e_out) {
    VD_CHECK(h && poses && e_out && n >= 0, VD_ERR_ARG, "vd_refine: bad arguments");
    Ctx& c = h->c;
    VD_CHECK(lig >= 0 && lig < int(c.ligs.size()), VD_ERR_ARG, "vd_refine: bad ligand id");
    if (n == 0) return VD_OK;
    VD_CUDA(cudaSetDevice(c.device));
    vd_status st = sync_pool(&c);
    if (st != VD_OK) return st;
    st = ensure_receptor_cells(&c);
    if (st != VD_OK) return st;
    const HostLigand& L = c.ligs[lig];
    const int nc = 7 + L.h.ntors;
    st = ensure_scratch(&c, al256(size_t(n) * nc * 4) + al256(n * 4) + al256(n * 4) + 256);
    if (st != VD_OK) return st;
    char* s = static_cast<char*>(c.d_scratch);
    float* d_p = reinterpret_cast<float*>(s); s += al256(size_t(n) * nc * 4);
    float* d_e = reinterpret_cast<float*>(s); s += al256(n * 4);
    int64_t* d_off = reinterpret_cast<int64_t*>(s);
    int32_t* d_plig = reinterpret_cast<int32_t*>(s + 16);
    VD_CUDA(cudaMemcpyAsync(d_p, poses, size_t(n) * nc * 4, cudaMemcpyHostToDevice, c.stream));
    const int64_t off = L.pool_offset;
    VD_CUDA(cudaMemcpyAsync(d_off, &off, 8, cudaMemcpyHostToDevice, c.stream));
    VD_CUDA(cudaMemsetAsync(d_plig, 0, n * 4 > 0 ? 4 : 4, c.stream));
    RefineParams rp{};
    rp.pool = c.d_pool;
    rp.lig_off = d_off;
    rp.pose_lig = nullptr;
    rp.poses = d_p;
    rp.e_out = d_e;
    rp.stride = nc;
    rp.n_poses = n;
    rp.max_steps_default = max_steps > 0 ? max_steps : (30 + L.n_all_atoms) / 3;
    rp.max_steps = nullptr;
    rp.R = rec_view(c);
    rp.smooth = c.d_smooth;
    rp.fix = c.fix_scale;
    rp.inv_fix = 1.f / c.fix_scale;
    rp.warp_floats = refine_warp_floats(L);
    rp.evals = reinterpret_cast<unsigned long long*>(c.d_counter + 4);
    rp.skip_invalid = 0;
    const size_t smem_r = size_t(rp.warp_floats) * kRefineWarps * 4;
    VD_CHECK(smem_r <= 227 * 1024, VD_ERR_CAPACITY, "refine kernel shared memory exceeds 227 KB");
    VD_CUDA(cudaFuncSetAttribute(refine_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem_r)));
    refine_kernel<<<(n + kRefineWarps - 1) / kRefineWarps, 32 * kRefineWarps, smem_r, c.stream>>>(rp);
    VD_CUDA(cudaGetLastError());
    VD_CUDA(cudaMemcpyAsync(poses, d_p, size_t(n) * nc * 4, cudaMemcpyDeviceToHost, c.stream));
    VD_CUDA(cudaMemcpyAsync(e_out, d_e, n * 4, cudaMemcpyDeviceToHost, c.stream));
    VD_CUDA(cudaStreamSynchronize(c.stream));
    { const vd_status cs = take_device_checks("refinement kernel"); if (cs != VD_OK) return cs; }
    return VD_OK;
}

vd_status vd_score(vd_ctx* h, int32_t lig, int32_t n, const float* poses, float* adjusted, float* intra) {
    VD_CHECK(h && poses && n >= 0 && n <= VD_MAX_MODES, VD_ERR_ARG, "vd_score: 0..20 poses");
    Ctx& c = h->c;
    VD_CHECK(lig >= 0 && lig < int(c.ligs.size()), VD_ERR_ARG, "vd_score: bad ligand id");
    if (n == 0) return VD_OK;
    VD_CUDA(cudaSetDevice(c.device));
    vd_status st = sync_pool(&c);
    if (st != VD_OK) return st;
    st = ensure_receptor_cells(&c);
    if (st != VD_OK) return st;
    const HostLigand& L = c.ligs[lig];
    const int nc = 7 + L.h.ntors;
    st = ensure_scratch(&c, al256(size_t(n) * nc * 4) + al256(size_t(n) * 16) + 512);
    if (st != VD_OK) return st;
    char* s = static_cast<char*>(c.d_scratch);
    float* d_p = reinterpret_cast<float*>(s); s += al256(size_t(n) * nc * 4);
    double* d_o = reinterpret_cast<double*>(s); s += al256(size_t(n) * 16);
    int64_t* d_off = reinterpret_cast<int64_t*>(s);
    VD_CUDA(cudaMemcpyAsync(d_p, poses, size_t(n) * nc * 4, cudaMemcpyHostToDevice, c.stream));
    const int64_t off = L.pool_offset;
    VD_CUDA(cudaMemcpyAsync(d_off, &off, 8, cudaMemcpyHostToDevice, c.stream));
    score_poses_kernel<<<1, 32, size_t(16 * L.h.n_nodes + 3 * L.h.n_atoms) * 8, c.stream>>>(
        c.d_pool, d_off, d_p, n, nc, rec_view(c), c.d_fastd, 0.1 * (c.weights[5] + 1), d_o);
    VD_CUDA(cudaGetLastError());
    std::vector<double> o(size_t(n) * 2);
    VD_CUDA(cudaMemcpyAsync(o.data(), d_o, o.size() * 8, cudaMemcpyDeviceToHost, c.stream));
    VD_CUDA(cudaStreamSynchronize(c.stream));
    { const vd_status cs = take_device_checks("scoring kernel"); if (cs != VD_OK) return cs; }
    for (int i = 0; i < n; ++i) {
        if (adjusted) adjusted[i] = float(o[2 * i]);
        if (intra) intra[i] = float(o[2 * i + 1]);
    }
    return VD_OK;
}

vd_status vd_rmsd_bounds(vd_ctx* h, int32_t lig, int32_t n, const float* poses, float* lb_out, float* ub_out) {
    VD_CHECK(h && poses && lb_out && ub_out && n >= 0, VD_ERR_ARG, "vd_rmsd_bounds: bad arguments");
    Ctx& c = h->c;
    VD_CHECK(lig >= 0 && lig < int(c.ligs.size()), VD_ERR_ARG, "vd_rmsd_bounds: bad ligand id");
    if (n == 0) return VD_OK;
    VD_CUDA(cudaSetDevice(c.device));
    vd_status st = sync_pool(&c);
    if (st != VD_OK) return st;
    const HostLigand& L = c.ligs[lig];
    const int nc = 7 + L.h.ntors;
    st = ensure_scratch(&c, al256(size_t(n) * nc * 4) + al256(size_t(n) * 16) + 512);
    if (st != VD_OK) return st;
    char* s = static_cast<char*>(c.d_scratch);
    float* d_p = reinterpret_cast<float*>(s); s += al256(size_t(n) * nc * 4);
    double* d_o = reinterpret_cast<double*>(s); s += al256(size_t(n) * 16);
    int64_t* d_off = reinterpret_cast<int64_t*>(s);
    VD_CUDA(cudaMemcpyAsync(d_p, poses, size_t(n) * nc * 4, cudaMemcpyHostToDevice, c.stream));
    const int64_t off = L.pool_offset;
    VD_CUDA(cudaMemcpyAsync(d_off, &off, 8, cudaMemcpyHostToDevice, c.stream));
    const size_t smem = size_t(16 * L.h.n_nodes + 3 * L.h.n_atoms) * 8 + size_t(6 * L.h.n_atoms) * 4;
    rmsd_poses_kernel<<<1, 32, smem, c.stream>>>(c.d_pool, d_off, d_p, n, nc, d_o);
    VD_CUDA(cudaGetLastError());
    std::vector<double> o(size_t(n) * 2);
    VD_CUDA(cudaMemcpyAsync(o.data(), d_o, o.size() * 8, cudaMemcpyDeviceToHost, c.stream));
    VD_CUDA(cudaStreamSynchronize(c.stream));
    { const vd_status cs = take_device_checks("RMSD kernel"); if (cs != VD_OK) return cs; }
    for (int i = 0; i < n; ++i) {
        lb_out[i] = float(o[2 * i]);
        ub_out[i] = float(o[2 * i + 1]);
    }
    return VD_OK;
}

}  // extern "C"
