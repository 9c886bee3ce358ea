// Monte-Carlo search: replaces kernel_monte / kernel2_update (kernel2.cu:219-426).
//
// One warp runs one chain: `search_depth` steps of mutate -> RILC-BFGS ->
// Metropolis (T = 1.2), re-optimising an accepted pose that beats the
// chain's best, exactly the control flow of kernel2.cu:290-421; or, with
// vd_search_params.dense_bfgs (--rilc_bfgs 0), mutate -> dense BFGS ->
// Metropolis as kernel2.cu:427-563, whose re-optimisation of an accepted
// pose that beats the best is discarded there (it re-optimises a copy and
// keeps the accepted pose and energy, kernel2.cu:526-552), so it is not run
// here: same best poses and energies, fewer evaluations.  Random
// numbers come from a Philox stream keyed by (seed, ligand, chain), so the
// plain (one ligand per launch, one warp per chain) and the batched
// (persistent, work queue over (ligand, chain) items) forms compute the same
// chains.
#include <algorithm>
#include <cstring>
#include <mutex>
#include <numeric>
#include <string>

#include "dock.h"
#include "launch.h"
#include "search.cuh"

namespace vd {
namespace {

struct DockParams {
    const float4* pool;
    const int64_t* lig_off;      // [n_ligs] blob offsets, in batch order
    const int32_t* prefix;       // [n_ligs+1] first item of each ligand
    const uint32_t* lig_uid;     // [n_ligs] Philox stream id
    const int32_t* depth;        // [n_ligs]
    const int32_t* bfgs_steps;   // [n_ligs]
    int32_t n_ligs;
    int32_t total_items;
    MapView G;
    const float4* smooth;
    EvalParams ep;
    uint32_t seed;
    float temperature, amplitude;
    float lo[3], hi[3];
    float* out_conf;             // [items][stride]
    int32_t stride;
    float* out_e;                // [items]
    int32_t* queue;
    unsigned long long* evals;
    unsigned long long* lig_evals;  // [n_ligs] evaluations per ligand
    int32_t warp_floats;
    int32_t warps_per_block;
    int32_t visited;             // QuickVina2-CUDA's visited history (RILC-BFGS only)
};

__device__ __forceinline__ int find_ligand(const int32_t* prefix, int n, int item) {
    int lo = 0, hi = n - 1;
    while (lo < hi) {  // last ligand with prefix <= item
        const int mid = (lo + hi + 1) >> 1;
        if (__ldg(&prefix[mid]) <= item) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// MINB: 4-warp blocks per SM the register budget targets (8/10/12/6/4 ->
// 64/48/40/80/128 registers per thread); the autotuner picks one per
// workload.  The small budgets keep more chains resident for large batches;
// the large ones drop the register spills (ptxas: 84 bytes of spill stores
// at 64, none at 128), which pays when a launch has few chains per SM.
// Per-warp shared memory: the evaluation's arrays, then the poses xp, xo,
// xt, xb (pad4(7 + ntors) floats each), then kChainWords chain scalars,
// then (dense BFGS) the inverse Hessian and four pose-space vectors
// (dense_floats).
// chain scalar slots (ints, then floats)
enum : int { kCsItem, kCsLig, kCsChain, kCsUid, kCsDepth, kCsSteps, kCsEvals0, kCsStep, kCsRuns, kCsFloats };
enum : int { kCfCurrent, kCfBest };
static_assert(kCsFloats + kCfBest + 1 <= kChainWords, "chain scalars exceed their shared words");

template <bool persistent, int MINB, bool dense = false>
__global__ void __launch_bounds__(128, MINB) dock_kernel(DockParams p) {
    extern __shared__ float4 smem4[];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    float* base = reinterpret_cast<float*>(smem4) + size_t(wid) * p.warp_floats;
    int evals = 0;
    int item = persistent ? 0 : blockIdx.x * p.warps_per_block + wid;
    for (;;) {
        if (persistent) {
            int v = 0;
            if (lane == 0) v = atomicAdd(p.queue, 1);
            item = __shfl_sync(0xffffffffu, v, 0);
        }
        if (item >= p.total_items) break;
        const int li0 = VD_DCLAMP(find_ligand(p.prefix, p.n_ligs, item), 0, p.n_ligs - 1, kChkItem);
        const LigView L = lig_view(p.pool, __ldg(&p.lig_off[li0]));
        const int nc = 7 + L.nt, nc4 = pad4(nc);
        SearchMem s;
        s.m = carve(base, L.na, L.nn, L.np, L.nt);
        s.xp = base + warp_floats(L.na, L.nn, L.np, L.nt);
        s.xo = s.xp + nc4;
        float* xt = s.xo + nc4;      // current (accepted) pose
        float* xb = xt + nc4;        // chain best
        // The chain's scalars live in shared memory, not in registers across
        // the optimiser calls: the evaluation needs every register it can get
        // (at 64 registers per thread this halves the spills to local memory,
        // whose reloads miss L1), and these are read once per MC step.
        int* cs = reinterpret_cast<int*>(xb + nc4);
        float* cf = reinterpret_cast<float*>(cs + kCsFloats);
        if (lane == 0) {
            cs[kCsItem] = item;
            cs[kCsLig] = li0;
            cs[kCsChain] = int(item - __ldg(&p.prefix[li0]));
            cs[kCsUid] = int(__ldg(&p.lig_uid[li0]));
            cs[kCsDepth] = __ldg(&p.depth[li0]);
            cs[kCsSteps] = __ldg(&p.bfgs_steps[li0]);
            cs[kCsEvals0] = evals;
            cs[kCsRuns] = 0;
            cf[kCfCurrent] = FLT_MAX;
            cf[kCfBest] = INFINITY;
        }
        __syncwarp();
        init_pose(xt, L.nt, p.seed, uint32_t(cs[kCsUid]), uint32_t(cs[kCsChain]), p.lo, p.hi, lane);
        copy_conf(xt, xb, nc, lane);
        for (int step = 0; step < cs[kCsDepth]; ++step) {
            __syncwarp();  // every lane has read the previous step index
            if (lane == 0) cs[kCsStep] = step;
            copy_conf(xt, s.m.x, nc, lane);
            mutate_pose(L, s.m, p.seed, uint32_t(cs[kCsUid]), uint32_t(cs[kCsChain]), uint32_t(step), p.amplitude,
                        lane);
            // pass 0 optimises the candidate; pass 1 re-optimises an accepted
            // candidate that beats the chain's best (one optimiser call site)
            for (int pass = 0; pass < 2; ++pass) {
                float ce;
                if (dense) {
                    const int n = 6 + L.nt;
                    float* H = reinterpret_cast<float*>(cs + kChainWords);  // after the chain scalars
                    float* gc = H + pad4(n * n);
                    float* pv = gc + pad4(n);
                    float* yv = pv + pad4(n);
                    float* mhy = yv + pad4(n);
                    const GridInter gi{&p.G, p.ep.v_inter, p.ep.slope};
                    ce = dense_bfgs<true>(L, s, H, gc, pv, yv, mhy, gi, p.smooth, p.ep.v_intra, p.ep.fix,
                                          p.ep.inv_fix, cs[kCsSteps], lane, evals);
                } else {
                    // visited history (visited.cuh:48-227, quasi_newton.cuh:1937-1943):
                    // interesting() holds until 10 x (6 + ntors) runs have been
                    // added to the history, then check() returns false on every
                    // path, so later calls keep the candidate at its entry energy
                    const int runs = cs[kCsRuns];
                    const bool skip = p.visited && runs >= 10 * (6 + L.nt);
                    __syncwarp();
                    if (lane == 0 && !skip) cs[kCsRuns] = runs + 1;
                    ce = rilc_bfgs(L, s, p.G, p.smooth, p.ep, cs[kCsSteps], lane, evals, skip);
                }
                const int stp = cs[kCsStep];
                float tmp_e = cf[kCfCurrent], best_e = cf[kCfBest];
                if (pass == 0) {
                    uint32_t b[4];
                    draw(p.seed, uint32_t(cs[kCsUid]), uint32_t(cs[kCsChain]), uint32_t(stp), 1, b);
                    const bool accept = stp == 0 || ce < tmp_e ||
                                        u01(b[1]) < __expf((tmp_e - ce) / p.temperature);  // kernel2.cu:63-71
                    if (!accept) break;
                    tmp_e = ce;
                    __syncwarp();
                    if (lane == 0) cf[kCfCurrent] = tmp_e;
                    if (dense || !(tmp_e < best_e)) {
                        if (dense && tmp_e < best_e) {  // kernel2.cu:518-552: the accepted pose is the best
                            if (lane == 0) cf[kCfBest] = tmp_e;
                            copy_conf(s.m.x, xb, nc, lane);
                        }
                        copy_conf(s.m.x, xt, nc, lane);
                        break;
                    }
                } else {
                    tmp_e = ce;
                    __syncwarp();
                    if (lane == 0) cf[kCfCurrent] = tmp_e;
                    if (tmp_e < best_e) {
                        if (lane == 0) cf[kCfBest] = tmp_e;
                        copy_conf(s.m.x, xb, nc, lane);
                    }
                    copy_conf(s.m.x, xt, nc, lane);
                }
                __syncwarp();
            }
            step = cs[kCsStep];  // reloaded: not held in a register across the optimiser
        }
        const int it = cs[kCsItem], li = cs[kCsLig];
        float* dst = p.out_conf + size_t(it) * p.stride;
        for (int i = lane; i < nc; i += 32) dst[i] = xb[i];
        if (lane == 0) {
            p.out_e[it] = cf[kCfBest];
            atomicAdd(&p.lig_evals[li], (unsigned long long)(evals - cs[kCsEvals0]));
        }
        __syncwarp();
        if (!persistent) break;
    }
    if (lane == 0 && evals) atomicAdd(p.evals, (unsigned long long)evals);
}

// Resident 4-warp blocks per SM each launch shape's register budget targets.
constexpr int kShapeBlocks[] = {8, 10, 12, 6, 4};

using DockFn = void (*)(DockParams);
template <bool persistent>
DockFn dock_fn(int shape) {
    switch (shape) {
        case 1: return dock_kernel<persistent, 10>;
        case 2: return dock_kernel<persistent, 12>;
        case 3: return dock_kernel<persistent, 6>;
        case 4: return dock_kernel<persistent, 4>;
        default: return dock_kernel<persistent, 8>;
    }
}
// Dense-BFGS search: built at the three register budgets the autotuner
// explores (64 / 80 / 128); a pinned 48- or 40-register shape runs at 64.
template <bool persistent>
DockFn dense_dock_fn(int& shape) {
    switch (shape) {
        case 3: return dock_kernel<persistent, 6, true>;
        case 4: return dock_kernel<persistent, 4, true>;
        default: shape = 0; return dock_kernel<persistent, 8, true>;
    }
}

// Shared-memory floats of the dense optimiser's state: H (n x n) and the
// four vectors gc, pv, yv, mhy, n = 6 + ntors.
int dense_floats(int ntors) {
    const int n = 6 + ntors;
    return pad4(n * n) + 4 * pad4(n);
}

}  // namespace

// The autotuner's candidates: 64, 80 and 128 registers.  The 48- and
// 40-register shapes spill heavily and were slower on every measured
// workload (wide-box screen, single ligand, uneven batch); they stay
// available to callers that pin a shape.
constexpr int kTunedShapes[] = {0, 3, 4};
constexpr int kNumTuned = int(sizeof(kTunedShapes) / sizeof(kTunedShapes[0]));

int dock_shape_for(Ctx& c, const vd_search_params& sp, uint64_t key) {
    if (sp.launch_shape >= 1 && sp.launch_shape <= kDockShapes) return sp.launch_shape - 1;
    return kTunedShapes[c.dock_tune.pick(key, kNumTuned)];
}

void dock_tune_report(Ctx& c, const DockBuffers& b, double ms, const unsigned long long* lig_evals) {
    if (!b.tuned) return;
    double work = 0;
    for (size_t i = 0; i < b.eval_bytes.size(); ++i) work += double(lig_evals[i]) * b.eval_bytes[i];
    if (!(work > 0)) return;
    for (int i = 0; i < kNumTuned; ++i)
        if (kTunedShapes[i] == b.shape) c.dock_tune.report(b.tune_key, i, ms / work);
}

// Heuristics of main.cpp:354-391 (atoms = all ligand atoms): search depth
// (0.24 atoms + 0.29 torsions - 3.41) x 2 and (30 + atoms)/3 BFGS steps for
// RILC-BFGS; x 2.4 and (25 + atoms)/3 for dense BFGS (--rilc_bfgs 0).
void search_defaults(const HostLigand& L, const vd_search_params& sp, int& depth, int& bfgs_steps) {
    const bool dense = sp.dense_bfgs != 0;
    depth = sp.search_depth;
    if (depth < 0) {  // no MC steps: each chain returns its initial pose
        depth = 0;
    } else if (depth == 0) {
        double t = (0.24 * L.n_all_atoms + 0.29 * L.h.ntors - 3.41) * (dense ? 2.4 : 2.0);
        if (t < 1) t = 1;
        depth = int(t);
    }
    bfgs_steps = sp.max_bfgs_steps > 0 ? sp.max_bfgs_steps : int(unsigned((dense ? 25 : 30) + L.n_all_atoms) / 3);
}

// Host side of a docking launch: checks, heuristics, device scratch layout
// and the packed parameter arrays; no stream operation (so the enqueue can be
// recorded into a CUDA graph).  Scratch layout:
//   [params: off | prefix | uid | depth | steps] [conf] [e] [lig_evals] [extra]
vd_status prepare_dock(Ctx& c, const std::vector<int>& ligs, const vd_search_params& sp, bool persistent,
                       DockBuffers& out) {
    VD_CHECK(!ligs.empty(), VD_ERR_ARG, "no ligands");
    VD_CHECK(sp.n_chains > 0, VD_ERR_ARG, "n_chains must be positive");
    VD_CHECK(sp.visited_history == 0 || (sp.visited_history == 1 && !sp.dense_bfgs), VD_ERR_ARG,
             "visited_history must be 0, or 1 with RILC-BFGS (QuickVina2-CUDA has no dense-BFGS search)");
    VD_CHECK(int64_t(ligs.size()) * sp.n_chains <= (int64_t(1) << 30), VD_ERR_CAPACITY,
             "more than 2^30 (ligand, chain) work items in one call");
    VD_CHECK(c.has_box, VD_ERR_ARG, "no box set");
    vd_status st = sync_pool(&c);
    if (st != VD_OK) return st;
    DockParams p{};
    st = make_map_view(c, p.G);
    if (st != VD_OK) return st;
    const int n = int(ligs.size());
    std::vector<int64_t> off(n);
    std::vector<int32_t> prefix(n + 1, 0), depth(n), steps(n);
    std::vector<uint32_t> uid(n);
    int max_wf = 0, max_nt = 0;
    for (int i = 0; i < n; ++i) {
        st = check_ligand_maps(c, ligs[i]);
        if (st != VD_OK) return st;
        const HostLigand& L = c.ligs[ligs[i]];
        off[i] = L.pool_offset;
        uid[i] = uint32_t(ligs[i]);
        search_defaults(L, sp, depth[i], steps[i]);
        prefix[i + 1] = prefix[i] + sp.n_chains;
        out.eval_bytes.push_back(32.0 * L.h.n_atoms + 16.0 * L.h.n_pairs);
        max_wf = std::max(max_wf, lig_warp_floats(L) + 4 * pad4(7 + L.h.ntors) + kChainWords +
                                      (sp.dense_bfgs ? dense_floats(L.h.ntors) : 0));
        max_nt = std::max(max_nt, L.h.ntors);
    }
    const int items = prefix[n];
    out.items = items;
    out.stride = 7 + max_nt;
    out.prefix = prefix;
    auto al = [](size_t b) { return (b + 255) & ~size_t(255); };
    const size_t b_off = n * sizeof(int64_t), b_pre = (n + 1) * sizeof(int32_t), b_arr = n * sizeof(int32_t);
    const size_t b_conf = size_t(items) * out.stride * sizeof(float), b_e = size_t(items) * sizeof(float);
    const size_t b_lev = n * sizeof(unsigned long long);
    const size_t b_par = al(b_off) + al(b_pre) + 3 * al(b_arr);
    const size_t total = b_par + al(b_conf) + al(b_e) + al(b_lev) + out.extra_bytes;
    st = ensure_scratch(&c, total);
    if (st != VD_OK) return st;
    // packed parameter arrays (host) and their device copies at the scratch start
    out.h_params.assign(b_par, 0);
    size_t o = 0;
    auto put = [&](const void* src, size_t bytes) {
        std::memcpy(out.h_params.data() + o, src, bytes);
        o += al(bytes);
    };
    char* s = static_cast<char*>(c.d_scratch);
    out.d_params = s;
    const int64_t* d_off = reinterpret_cast<const int64_t*>(s + o); put(off.data(), b_off);
    const int32_t* d_pre = reinterpret_cast<const int32_t*>(s + o); put(prefix.data(), b_pre);
    const uint32_t* d_uid = reinterpret_cast<const uint32_t*>(s + o); put(uid.data(), b_arr);
    const int32_t* d_depth = reinterpret_cast<const int32_t*>(s + o); put(depth.data(), b_arr);
    const int32_t* d_steps = reinterpret_cast<const int32_t*>(s + o); put(steps.data(), b_arr);
    s += b_par;
    out.d_conf = reinterpret_cast<float*>(s); s += al(b_conf);
    out.d_e = reinterpret_cast<float*>(s); s += al(b_e);
    out.d_lig_evals = reinterpret_cast<unsigned long long*>(s); s += al(b_lev);
    out.d_extra = s;
    p.pool = c.d_pool;
    p.lig_off = d_off;
    p.prefix = d_pre;
    p.lig_uid = d_uid;
    p.depth = d_depth;
    p.bfgs_steps = d_steps;
    p.n_ligs = n;
    p.total_items = items;
    p.smooth = c.d_smooth;
    p.ep = {float(sp.hunt_cap[0]), float(sp.hunt_cap[1]), 1e6f, c.fix_scale, 1.f / c.fix_scale};
    p.seed = sp.seed;
    p.temperature = float(sp.temperature > 0 ? sp.temperature : 1.2);
    p.amplitude = float(sp.amplitude > 0 ? sp.amplitude : 2.0);
    for (int d = 0; d < 3; ++d) {
        p.lo[d] = float(c.geom.begin[d]);
        p.hi[d] = float(c.geom.end[d]);
    }
    p.out_conf = out.d_conf;
    p.stride = out.stride;
    p.out_e = out.d_e;
    p.queue = c.d_counter;
    p.evals = reinterpret_cast<unsigned long long*>(c.d_counter + 2);
    p.lig_evals = out.d_lig_evals;
    p.warp_floats = max_wf;
    p.visited = sp.visited_history;
    // launch shape: register budget from the caller or the autotuner, keyed
    // by form, work items and shared memory per chain
    const int wpb = 4;
    const size_t smem = size_t(max_wf) * wpb * sizeof(float);
    VD_CHECK(smem <= 227 * 1024, VD_ERR_CAPACITY, "ligand too large for the docking kernel");
    p.warps_per_block = wpb;
    out.tune_key = (uint64_t(persistent) << 40) | (uint64_t(ceil_log2(uint64_t(items))) << 32) |
                   uint64_t(max_wf > 1024);  // above 4 KB per chain, shared memory caps the occupancy
    out.tune_key |= uint64_t(sp.dense_bfgs != 0) << 41;
    out.tuned = sp.launch_shape == 0;
    out.shape = dock_shape_for(c, sp, out.tune_key);
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c.device);
    const DockFn k = sp.dense_bfgs ? (persistent ? dense_dock_fn<true>(out.shape) : dense_dock_fn<false>(out.shape))
                                   : (persistent ? dock_fn<true>(out.shape) : dock_fn<false>(out.shape));
    VD_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
    VD_CUDA(prefer_l1(k, c.device, kShapeBlocks[out.shape], smem));
    int blocks = (items + wpb - 1) / wpb;
    if (persistent) {
        int per_sm = 0;
        VD_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, 32 * wpb, smem));
        blocks = std::min(sms * std::max(1, per_sm), blocks);
    }
    out.launch = [k, blocks, wpb, smem, p](cudaStream_t stream) {
        k<<<blocks, 32 * wpb, smem, stream>>>(p);
        return cudaGetLastError();
    };
    c.stats.dock_blocks = blocks;
    c.stats.dock_shape = out.shape + 1;
    c.stats.dock_warps_per_block = wpb;
    return VD_OK;
}

// Stream side of a docking launch: parameter upload (from params_src, the
// packed arrays or a pinned copy of them), counter resets, the kernel
// bracketed by c.ev0 / c.ev1.
vd_status enqueue_dock(Ctx& c, const DockBuffers& b, const void* params_src, cudaStream_t stream) {
    VD_CUDA(cudaMemcpyAsync(b.d_params, params_src, b.h_params.size(), cudaMemcpyHostToDevice, stream));
    VD_CUDA(cudaMemsetAsync(b.d_lig_evals, 0, (b.prefix.size() - 1) * sizeof(unsigned long long), stream));
    VD_CUDA(cudaMemsetAsync(c.d_counter, 0, 16, stream));
    VD_CUDA(record_event(c.ev0, stream));
    VD_CUDA(b.launch(stream));
    VD_CUDA(record_event(c.ev1, stream));
    return VD_OK;
}

vd_status launch_dock(Ctx& c, const std::vector<int>& ligs, const vd_search_params& sp, bool persistent,
                      DockBuffers& out, cudaStream_t stream) {
    vd_status st = prepare_dock(c, ligs, sp, persistent, out);
    if (st != VD_OK) return st;
    return enqueue_dock(c, out, out.h_params.data(), stream);
}

}  // namespace vd

namespace vd {
// the docking kernel's check word lives in this file; launches from other
// files (the batched pipeline) read it through here
vd_status dock_take_checks(const char* where) { return take_device_checks(where); }
}  // namespace vd

using namespace vd;

extern "C" {

vd_status vd_mc_chains(vd_ctx* h, int32_t lig, const vd_search_params* sp, float* poses_out, float* e_out,
                       int64_t* evals) {
    VD_CHECK(h && sp && poses_out && e_out, VD_ERR_ARG, "vd_mc_chains: NULL argument");
    Ctx& c = h->c;
    VD_CHECK(lig >= 0 && lig < int(c.ligs.size()), VD_ERR_ARG, "vd_mc_chains: bad ligand id");
    VD_CUDA(cudaSetDevice(c.device));
    DockBuffers b;
    vd_status st = launch_dock(c, {lig}, *sp, false, b, c.stream);
    if (st != VD_OK) return st;
    const int nc = 7 + c.ligs[lig].h.ntors;
    VD_CUDA(cudaMemcpy2DAsync(poses_out, nc * sizeof(float), b.d_conf, b.stride * sizeof(float), nc * sizeof(float),
                              b.items, cudaMemcpyDeviceToHost, c.stream));
    VD_CUDA(cudaMemcpyAsync(e_out, b.d_e, b.items * sizeof(float), cudaMemcpyDeviceToHost, c.stream));
    unsigned long long ev = 0;
    VD_CUDA(cudaMemcpyAsync(&ev, c.d_counter + 2, 8, cudaMemcpyDeviceToHost, c.stream));
    VD_CUDA(cudaStreamSynchronize(c.stream));
    if ((st = take_device_checks("docking kernel")) != VD_OK) return st;
    float ms = 0;
    VD_CUDA(cudaEventElapsedTime(&ms, c.ev0, c.ev1));
    c.stats.dock_ms = ms;
    c.stats.bfgs_evals += int64_t(ev);
    dock_tune_report(c, b, ms, &ev);
    if (evals) *evals = int64_t(ev);
    return VD_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Monte-Carlo chains without any device allocation.
//
// Some callers cannot call cudaMalloc at the moment they dock: host
// applications that reserve their whole device-memory budget up front (a
// memory pool that owns every free byte, or a service that must not grow its
// footprint once it is admitted to a shared GPU), and latency-sensitive hosts
// that cannot afford the device-wide synchronisation an allocation or free may
// imply.  This entry point keeps its launch parameters, counters and
// per-chain results in one statically sized device array instead of the
// context's growable scratch.
//
// Limits and sharing: the array holds VD_NOALLOC_SCRATCH_BYTES; a call whose
// chains do not fit is rejected with VD_ERR_CAPACITY.  Every GPU that loads
// the library holds the array until the process exits.  All calls on a
// device share it and it keeps the previous call's contents (counters are
// cleared by each call), so calls whose GPU work overlaps race with each
// other: serialise them.  The first call on a device looks up the array's
// device address with that device current (one-time set-up); make that first
// call before any stream capture.  The kernel always runs at the 64-register
// launch shape (sp->launch_shape is not read); chains do not depend on the
// shape.
namespace {

static __device__ __align__(256) unsigned char g_noalloc_scratch[VD_NOALLOC_SCRATCH_BYTES];

std::mutex g_noalloc_mu;
void* g_noalloc_addr[64] = {};

vd_status noalloc_address(int device, char** out) {
    VD_CHECK(device >= 0 && device < 64, VD_ERR_ARG, "vd_mc_chains_noalloc: device index out of range");
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (!g_noalloc_addr[device]) {
        void* p = nullptr;
        VD_CUDA(cudaGetSymbolAddress(&p, g_noalloc_scratch));  // the device is current here
        g_noalloc_addr[device] = p;
    }
    *out = static_cast<char*>(g_noalloc_addr[device]);
    return VD_OK;
}

}  // namespace

extern "C" vd_status vd_mc_chains_noalloc(vd_ctx* h, int32_t lig, const vd_search_params* sp, float* poses_out,
                                          float* e_out, int64_t* evals) {
    VD_CHECK(h && sp && poses_out && e_out, VD_ERR_ARG, "vd_mc_chains_noalloc: NULL argument");
    Ctx& c = h->c;
    VD_CHECK(lig >= 0 && lig < int(c.ligs.size()), VD_ERR_ARG, "vd_mc_chains_noalloc: bad ligand id");
    VD_CHECK(sp->n_chains > 0, VD_ERR_ARG, "vd_mc_chains_noalloc: n_chains must be positive");
    VD_CHECK(sp->visited_history == 0 || (sp->visited_history == 1 && !sp->dense_bfgs), VD_ERR_ARG,
             "vd_mc_chains_noalloc: visited_history must be 0, or 1 with RILC-BFGS");
    VD_CHECK(c.has_box, VD_ERR_ARG, "vd_mc_chains_noalloc: no box set");
    VD_CHECK(!c.pool_dirty && c.d_pool, VD_ERR_ARG,
             "vd_mc_chains_noalloc: ligands not on the device yet; make one allocating call "
             "(e.g. vd_mc_chains or vd_energy) after vd_add_ligand");
    VD_CUDA(cudaSetDevice(c.device));
    char* base = nullptr;
    vd_status st = noalloc_address(c.device, &base);
    if (st != VD_OK) return st;
    DockParams p{};
    st = make_map_view(c, p.G);
    if (st != VD_OK) return st;
    st = check_ligand_maps(c, lig);
    if (st != VD_OK) return st;
    const HostLigand& L = c.ligs[lig];
    int depth = 0, steps = 0;
    search_defaults(L, *sp, depth, steps);
    const int n = sp->n_chains, nc = 7 + L.h.ntors;
    // layout: [0,256) counters | [256,512) launch parameters | [512,..) results
    const size_t conf_bytes = ((size_t(n) * nc * sizeof(float)) + 255) & ~size_t(255);
    const size_t need = 512 + conf_bytes + size_t(n) * sizeof(float);
    VD_CHECK(need <= VD_NOALLOC_SCRATCH_BYTES, VD_ERR_CAPACITY,
             "vd_mc_chains_noalloc: " + std::to_string(n) + " chains of " + std::to_string(nc) +
                 " floats exceed the static scratch of VD_NOALLOC_SCRATCH_BYTES");
    unsigned long long* d_cnt = reinterpret_cast<unsigned long long*>(base);
    char* prm = base + 256;
    int64_t* d_off = reinterpret_cast<int64_t*>(prm);
    int32_t* d_pre = reinterpret_cast<int32_t*>(prm + 16);
    uint32_t* d_uid = reinterpret_cast<uint32_t*>(prm + 32);
    int32_t* d_depth = reinterpret_cast<int32_t*>(prm + 48);
    int32_t* d_steps = reinterpret_cast<int32_t*>(prm + 64);
    float* d_conf = reinterpret_cast<float*>(base + 512);
    float* d_e = reinterpret_cast<float*>(base + 512 + conf_bytes);
    struct {
        int64_t off;
        int64_t pad0;
        int32_t pre[4];
        uint32_t uid[4];
        int32_t depth[4];
        int32_t steps[4];
    } hp = {L.pool_offset, 0, {0, n, 0, 0}, {uint32_t(lig), 0, 0, 0}, {depth, 0, 0, 0}, {steps, 0, 0, 0}};
    VD_CUDA(cudaMemsetAsync(d_cnt, 0, 256, c.stream));  // counters start at zero on every call
    VD_CUDA(cudaMemcpyAsync(prm, &hp, sizeof(hp), cudaMemcpyHostToDevice, c.stream));
    p.pool = c.d_pool;
    p.lig_off = d_off;
    p.prefix = d_pre;
    p.lig_uid = d_uid;
    p.depth = d_depth;
    p.bfgs_steps = d_steps;
    p.n_ligs = 1;
    p.total_items = n;
    p.smooth = c.d_smooth;
    p.ep = {float(sp->hunt_cap[0]), float(sp->hunt_cap[1]), 1e6f, c.fix_scale, 1.f / c.fix_scale};
    p.seed = sp->seed;
    p.temperature = float(sp->temperature > 0 ? sp->temperature : 1.2);
    p.amplitude = float(sp->amplitude > 0 ? sp->amplitude : 2.0);
    for (int d = 0; d < 3; ++d) {
        p.lo[d] = float(c.geom.begin[d]);
        p.hi[d] = float(c.geom.end[d]);
    }
    p.out_conf = d_conf;
    p.stride = nc;
    p.out_e = d_e;
    p.queue = nullptr;  // one warp per chain: no work queue
    p.visited = sp->visited_history;
    p.evals = d_cnt;
    p.lig_evals = d_cnt + 1;
    p.warp_floats = lig_warp_floats(L) + 4 * pad4(nc) + kChainWords + (sp->dense_bfgs ? dense_floats(L.h.ntors) : 0);
    const int wpb = 4;
    const size_t smem = size_t(p.warp_floats) * wpb * sizeof(float);
    VD_CHECK(smem <= 227 * 1024, VD_ERR_CAPACITY, "vd_mc_chains_noalloc: ligand too large for the kernel");
    p.warps_per_block = wpb;
    auto k = sp->dense_bfgs ? dock_kernel<false, 8, true> : dock_kernel<false, 8>;
    VD_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
    k<<<(n + wpb - 1) / wpb, 32 * wpb, smem, c.stream>>>(p);
    VD_CUDA(cudaGetLastError());
    VD_CUDA(cudaMemcpyAsync(poses_out, d_conf, size_t(n) * nc * sizeof(float), cudaMemcpyDeviceToHost, c.stream));
    VD_CUDA(cudaMemcpyAsync(e_out, d_e, size_t(n) * sizeof(float), cudaMemcpyDeviceToHost, c.stream));
    unsigned long long ev = 0;
    VD_CUDA(cudaMemcpyAsync(&ev, d_cnt, sizeof(ev), cudaMemcpyDeviceToHost, c.stream));
    VD_CUDA(cudaStreamSynchronize(c.stream));
    if ((st = take_device_checks("vd_mc_chains_noalloc")) != VD_OK) return st;
    c.stats.bfgs_evals += int64_t(ev);
    if (evals) *evals = int64_t(ev);
    return VD_OK;
}
