// Pose batches: forward energy kernel, adjoint kernel (energy + gradient,
// recomputing atom coordinates from the torsion tree), coordinates, and
// one RILC-BFGS local optimisation per pose.  One warp per pose.
#include <cstring>

#include "launch.h"
#include "search.cuh"

namespace vd {
namespace {

constexpr int kPoseWarps = 4;

struct PoseParams {
    const float4* pool;
    int64_t lig_off;
    MapView G;
    const float4* smooth;
    EvalParams ep;
    const float* poses;
    int32_t n_poses;
    float* e_out;
    float* g_out;       // adjoint only
    float* xyz_out;     // coords only
    float* poses_out;   // local opt
    int32_t max_steps;
    unsigned long long* evals;
    int32_t warp_floats;
};

// mode 0: energy, 1: energy+gradient, 2: coordinates, 3: local optimisation.
// Modes 0-2 are held to 64 registers (8 blocks of 4 warps per SM):
// they fit without spills, and the adjoint (mode 1) left free takes 72 and
// loses a block per SM.
constexpr int pose_min_blocks(int mode) { return mode == 3 ? 1 : 8; }
template <int mode>
__global__ void __launch_bounds__(32 * kPoseWarps, pose_min_blocks(mode)) pose_kernel(PoseParams p) {
    extern __shared__ float4 smem4[];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    float* base = reinterpret_cast<float*>(smem4) + size_t(wid) * p.warp_floats;
    const LigView L = lig_view(p.pool, p.lig_off);
    SearchMem s;
    s.m = carve(base, L.na, L.nn, L.np, L.nt);
    s.xp = base + warp_floats(L.na, L.nn, L.np, L.nt);
    s.xo = s.xp + pad4(7 + L.nt);
    const int nc = 7 + L.nt, n = 6 + L.nt;
    int evals = 0;
    for (int pose = blockIdx.x * kPoseWarps + wid; pose < p.n_poses; pose += gridDim.x * kPoseWarps) {
        const float* src = p.poses + size_t(pose) * nc;
        for (int i = lane; i < nc; i += 32) s.m.x[i] = src[i];
        __syncwarp();
        if (mode == 0) {
            const float e = eval_pose<false>(L, s.m, p.G, p.smooth, p.ep, lane);
            if (lane == 0) p.e_out[pose] = e;
        } else if (mode == 1) {
            const float e = eval_pose<true>(L, s.m, p.G, p.smooth, p.ep, lane);
            if (lane == 0) p.e_out[pose] = e;
            for (int i = lane; i < n; i += 32) p.g_out[size_t(pose) * n + i] = s.m.g[i];
        } else if (mode == 2) {
            kinematics(L, s.m, lane);
            float* dst = p.xyz_out + size_t(pose) * 3 * L.na;
            for (int i = lane; i < L.na; i += 32) {
                dst[3 * i] = s.m.c[i].x;
                dst[3 * i + 1] = s.m.c[i].y;
                dst[3 * i + 2] = s.m.c[i].z;
            }
        } else {
            const float e = rilc_bfgs(L, s, p.G, p.smooth, p.ep, p.max_steps, lane, evals);
            if (lane == 0) p.e_out[pose] = e;
            for (int i = lane; i < nc; i += 32) p.poses_out[size_t(pose) * nc + i] = s.m.x[i];
        }
        __syncwarp();
    }
    if (mode == 3 && lane == 0 && evals) atomicAdd(p.evals, (unsigned long long)evals);
}

template <int mode>
vd_status run_pose_kernel(Ctx& c, int lig, int n_poses, const float* d_poses, const vd_eval_params* ep,
                          float* d_e, float* d_g, float* d_xyz, float* d_out, int max_steps,
                          cudaStream_t stream) {
    VD_CHECK(lig >= 0 && lig < int(c.ligs.size()), VD_ERR_ARG, "bad ligand id");
    VD_CHECK(n_poses >= 0, VD_ERR_ARG, "negative pose count");
    if (n_poses == 0) return VD_OK;
    vd_status st = sync_pool(&c);
    if (st != VD_OK) return st;
    PoseParams p{};
    if (mode != 2) {
        st = make_map_view(c, p.G);
        if (st != VD_OK) return st;
        st = check_ligand_maps(c, lig);
        if (st != VD_OK) return st;
    }
    const HostLigand& L = c.ligs[lig];
    p.pool = c.d_pool;
    p.lig_off = L.pool_offset;
    p.smooth = c.d_smooth;
    const vd_eval_params def = {10.0, 10.0, 1e6};
    const vd_eval_params* e = ep ? ep : &def;
    p.ep = {float(e->v_intra), float(e->v_inter), float(e->slope), c.fix_scale, 1.f / c.fix_scale};
    p.poses = d_poses;
    p.n_poses = n_poses;
    p.e_out = d_e;
    p.g_out = d_g;
    p.xyz_out = d_xyz;
    p.poses_out = d_out;
    p.max_steps = max_steps;
    p.evals = reinterpret_cast<unsigned long long*>(c.d_counter + 8);
    p.warp_floats = lig_warp_floats(L) + 2 * pad4(7 + L.h.ntors);
    const size_t smem = size_t(p.warp_floats) * kPoseWarps * sizeof(float);
    VD_CHECK(smem <= 227 * 1024, VD_ERR_CAPACITY, "ligand too large for the pose kernel");
    auto kern = pose_kernel<mode>;
    VD_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
    if (mode != 3) VD_CUDA(prefer_l1(kern, c.device, pose_min_blocks(mode), smem));
    int dev_sms = 148;
    cudaDeviceGetAttribute(&dev_sms, cudaDevAttrMultiProcessorCount, c.device);
    const int blocks = std::min((n_poses + kPoseWarps - 1) / kPoseWarps, dev_sms * 16);
    kern<<<blocks, 32 * kPoseWarps, smem, stream>>>(p);
    VD_CUDA(cudaGetLastError());
    return VD_OK;
}

}  // namespace
}  // namespace vd

using namespace vd;

extern "C" {

vd_status vd_energy_grad_device(vd_ctx* h, int32_t lig, int32_t n, const float* poses, const vd_eval_params* ep,
                                float* e, float* g, void* stream) {
    VD_CHECK(h && poses && e && g, VD_ERR_ARG, "vd_energy_grad_device: NULL argument");
    Ctx& c = h->c;
    VD_CUDA(cudaSetDevice(c.device));
    cudaStream_t s = static_cast<cudaStream_t>(stream);  // NULL: the CUDA default stream
    return run_pose_kernel<1>(c, lig, n, poses, ep, e, g, nullptr, nullptr, 0, s);
}

vd_status vd_energy_device(vd_ctx* h, int32_t lig, int32_t n, const float* poses, const vd_eval_params* ep,
                           float* e, void* stream) {
    VD_CHECK(h && poses && e, VD_ERR_ARG, "vd_energy_device: NULL argument");
    Ctx& c = h->c;
    VD_CUDA(cudaSetDevice(c.device));
    cudaStream_t s = static_cast<cudaStream_t>(stream);  // NULL: the CUDA default stream
    return run_pose_kernel<0>(c, lig, n, poses, ep, e, nullptr, nullptr, nullptr, 0, s);
}

static vd_status pose_host(vd_ctx* h, int32_t lig, int32_t n, const float* poses, const vd_eval_params* ep,
                           float* e_out, float* g_out, float* xyz_out, int mode, int max_steps,
                           float* poses_out, int64_t* evals) {
    VD_CHECK(h && poses, VD_ERR_ARG, "pose call: NULL argument");
    Ctx& c = h->c;
    VD_CHECK(lig >= 0 && lig < int(c.ligs.size()), VD_ERR_ARG, "bad ligand id");
    if (n <= 0) return n == 0 ? VD_OK : VD_ERR_ARG;
    VD_CUDA(cudaSetDevice(c.device));
    const HostLigand& L = c.ligs[lig];
    const size_t nc = 7 + L.h.ntors, ng = 6 + L.h.ntors, na = L.h.n_atoms;
    const size_t b_pose = ((n * nc * 4 + 255) / 256) * 256, b_e = ((n * 4 + 255) / 256) * 256;
    const size_t b_g = ((n * ng * 4 + 255) / 256) * 256, b_x = ((n * na * 12 + 255) / 256) * 256;
    vd_status st = ensure_scratch(&c, 2 * b_pose + b_e + b_g + b_x);
    if (st != VD_OK) return st;
    char* s = static_cast<char*>(c.d_scratch);
    float* d_pose = reinterpret_cast<float*>(s);
    float* d_out = reinterpret_cast<float*>(s + b_pose);
    float* d_e = reinterpret_cast<float*>(s + 2 * b_pose);
    float* d_g = reinterpret_cast<float*>(s + 2 * b_pose + b_e);
    float* d_x = reinterpret_cast<float*>(s + 2 * b_pose + b_e + b_g);
    VD_CUDA(cudaMemcpyAsync(d_pose, poses, n * nc * 4, cudaMemcpyHostToDevice, c.stream));
    if (mode == 3) VD_CUDA(cudaMemsetAsync(c.d_counter + 8, 0, 8, c.stream));
    switch (mode) {
        case 0: st = run_pose_kernel<0>(c, lig, n, d_pose, ep, d_e, nullptr, nullptr, nullptr, 0, c.stream); break;
        case 1: st = run_pose_kernel<1>(c, lig, n, d_pose, ep, d_e, d_g, nullptr, nullptr, 0, c.stream); break;
        case 2: st = run_pose_kernel<2>(c, lig, n, d_pose, ep, nullptr, nullptr, d_x, nullptr, 0, c.stream); break;
        default: st = run_pose_kernel<3>(c, lig, n, d_pose, ep, d_e, nullptr, nullptr, d_out, max_steps, c.stream);
    }
    if (st != VD_OK) return st;
    if (e_out) VD_CUDA(cudaMemcpyAsync(e_out, d_e, n * 4, cudaMemcpyDeviceToHost, c.stream));
    if (g_out) VD_CUDA(cudaMemcpyAsync(g_out, d_g, n * ng * 4, cudaMemcpyDeviceToHost, c.stream));
    if (xyz_out) VD_CUDA(cudaMemcpyAsync(xyz_out, d_x, n * na * 12, cudaMemcpyDeviceToHost, c.stream));
    if (poses_out) VD_CUDA(cudaMemcpyAsync(poses_out, d_out, n * nc * 4, cudaMemcpyDeviceToHost, c.stream));
    unsigned long long ev = 0;
    if (mode == 3) VD_CUDA(cudaMemcpyAsync(&ev, c.d_counter + 8, 8, cudaMemcpyDeviceToHost, c.stream));
    VD_CUDA(cudaStreamSynchronize(c.stream));
    { const vd_status cs = take_device_checks("pose kernel"); if (cs != VD_OK) return cs; }
    if (evals) *evals = int64_t(ev);
    c.stats.bfgs_evals += int64_t(ev) + (mode == 1 ? n : 0);
    return VD_OK;
}

vd_status vd_energy(vd_ctx* h, int32_t lig, int32_t n, const float* poses, const vd_eval_params* ep, float* e) {
    VD_CHECK(e, VD_ERR_ARG, "vd_energy: NULL output");
    return pose_host(h, lig, n, poses, ep, e, nullptr, nullptr, 0, 0, nullptr, nullptr);
}
vd_status vd_energy_grad(vd_ctx* h, int32_t lig, int32_t n, const float* poses, const vd_eval_params* ep,
                         float* e, float* g) {
    VD_CHECK(e && g, VD_ERR_ARG, "vd_energy_grad: NULL output");
    return pose_host(h, lig, n, poses, ep, e, g, nullptr, 1, 0, nullptr, nullptr);
}
vd_status vd_pose_coords(vd_ctx* h, int32_t lig, int32_t n, const float* poses, float* xyz) {
    VD_CHECK(xyz, VD_ERR_ARG, "vd_pose_coords: NULL output");
    return pose_host(h, lig, n, poses, nullptr, nullptr, nullptr, xyz, 2, 0, nullptr, nullptr);
}
vd_status vd_local_opt(vd_ctx* h, int32_t lig, int32_t n, float* poses, const vd_eval_params* ep,
                       int32_t max_steps, float* e, int64_t* evals) {
    VD_CHECK(e, VD_ERR_ARG, "vd_local_opt: NULL output");
    return pose_host(h, lig, n, poses, ep, e, nullptr, nullptr, 3, max_steps, poses, evals);
}

}  // extern "C"
