// Docking launch interface shared by dock.cu and post.cu.
#pragma once

#include <functional>
#include <vector>

#include "common.h"

namespace vd {

struct DockBuffers {
    int items = 0;
    int stride = 0;                 // floats per pose in d_conf
    std::vector<int32_t> prefix;    // first item of each ligand (host)
    float* d_conf = nullptr;        // [items][stride] chain best poses
    float* d_e = nullptr;           // [items] chain best energies
    unsigned long long* d_lig_evals = nullptr;  // [n_ligs] evaluations per ligand
    size_t extra_bytes = 0;         // caller-requested scratch after the outputs
    char* d_extra = nullptr;
    uint64_t tune_key = 0;          // autotuner key of the launch
    std::vector<double> eval_bytes; // per ligand: algorithmic bytes of one evaluation (tuner cost unit)
    int shape = 0;                  // launch shape used (0-based)
    bool tuned = false;             // shape came from the autotuner
    std::vector<unsigned char> h_params;  // packed parameter arrays (host)
    void* d_params = nullptr;             // their device copy
    std::function<cudaError_t(cudaStream_t)> launch;  // the kernel launch
};

constexpr int kDockShapes = 5;      // register budgets 64/48/40/80/128 per thread
constexpr int kChainWords = 16;     // per-warp shared words for a chain's scalars (dock_kernel)

void search_defaults(const HostLigand& L, const vd_search_params& sp, int& depth, int& bfgs_steps);
// prepare_dock: host work and device layout (no stream operation);
// enqueue_dock: upload, counter resets and the kernel between c.ev0 and c.ev1;
// launch_dock: both.
vd_status prepare_dock(Ctx& c, const std::vector<int>& ligs, const vd_search_params& sp, bool persistent,
                       DockBuffers& out);
vd_status enqueue_dock(Ctx& c, const DockBuffers& b, const void* params_src, cudaStream_t stream);
vd_status launch_dock(Ctx& c, const std::vector<int>& ligs, const vd_search_params& sp, bool persistent,
                      DockBuffers& out, cudaStream_t stream);
// Feeds a finished launch's kernel time to the autotuner, per unit of work:
// ms / sum over ligands of (evaluations x algorithmic bytes per evaluation),
// so shapes tried on different ligands of one workload compare fairly.
// lig_evals: evaluations per ligand of the launch, in batch order.
void dock_tune_report(Ctx& c, const DockBuffers& b, double ms, const unsigned long long* lig_evals);
// Reads and clears the docking kernel's device bounds-check word (checked
// build only; VD_OK otherwise).
vd_status dock_take_checks(const char* where);

}  // namespace vd
