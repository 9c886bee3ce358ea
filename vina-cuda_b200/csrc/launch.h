// Host helpers shared by the kernel launchers.
#pragma once

#include "common.h"
#include "eval.cuh"

namespace vd {

inline vd_status make_map_view(Ctx& c, MapView& G) {
    VD_CHECK(c.n_maps > 0, VD_ERR_ARG, "grid maps not built (vd_build_grids)");
    for (int t = 0; t < kTypes; ++t) {
        G.map[t] = (c.map_slot[t] >= 0) ? c.d_maps + size_t(c.map_slot[t]) * c.map_stride : nullptr;
        G.cell[t] = (c.map_slot[t] >= 0 && c.d_cells) ? c.d_cells + size_t(c.map_slot[t]) * c.cell_stride : nullptr;
    }
    for (int d = 0; d < 3; ++d) {
        G.init[d] = float(c.geom.init[d]);
        G.factor[d] = float(c.geom.factor[d]);
        G.finv[d] = float(c.geom.finv[d]);
        G.dmo[d] = float(c.geom.dmo[d]);
        G.n[d] = c.geom.n[d];
    }
    G.pitch = c.geom.pitch;
    return VD_OK;
}

// Checks a ligand's atom types all have maps.
inline vd_status check_ligand_maps(Ctx& c, int lig) {
    VD_CHECK(lig >= 0 && lig < int(c.ligs.size()), VD_ERR_ARG, "bad ligand id");
    const HostLigand& L = c.ligs[lig];
    const float4* atoms = L.blob.data() + L.h.off_atoms;
    for (int i = 0; i < L.h.n_atoms; ++i) {
        int w;
        std::memcpy(&w, &atoms[i].w, sizeof(int));
        VD_CHECK(c.map_slot[w & 0xff] >= 0, VD_ERR_ARG,
                 "ligand atom XS type " + std::to_string(w & 0xff) + " has no grid map (vd_build_grids)");
    }
    return VD_OK;
}

inline int lig_warp_floats(const HostLigand& L) {
    return warp_floats(L.h.n_atoms, L.h.n_nodes, L.h.n_pairs, L.h.ntors);
}

}  // namespace vd
