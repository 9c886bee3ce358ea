// Docking launch interface shared by dock.cu and post.cu.
#pragma once

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
};

void search_defaults(const HostLigand& L, const vd_search_params& sp, int& depth, int& bfgs_steps);
vd_status launch_dock(Ctx& c, const std::vector<int>& ligs, const vd_search_params& sp, bool persistent,
                      DockBuffers& out, cudaStream_t stream, int warps_per_block_override);

}  // namespace vd
