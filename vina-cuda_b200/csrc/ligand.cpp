// Ligand ingestion: validates a vd_ligand_desc and packs the device blob
// (heavy atoms only, rigid bodies in pre-order, intra pairs).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <system_error>
#include <thread>

#include "common.h"
#include "schedule.h"

namespace vd {

// Uploads the ligands added since the last call.  Offsets are fixed when a
// ligand is added, so the upload is append-only: only new blobs cross PCIe
// (growing the buffer copies the old contents device to device).
vd_status sync_pool(Ctx* c) {
    if (!c->pool_dirty) return VD_OK;
    const int64_t words = c->pool_words;
    if (words > c->pool_cap || !c->d_pool) {
        const int64_t cap = std::max<int64_t>(words + words / 2, 4096);
        float4* fresh = nullptr;
        vd_status st = dev_alloc(*c, &fresh, size_t(cap) * sizeof(float4), "ligand pool");
        if (st != VD_OK) return st;
        int64_t keep = 0;
        if (c->pool_synced > 0) {
            const HostLigand& last = c->ligs[c->pool_synced - 1];
            keep = last.pool_offset + int64_t(last.blob.size());
        }
        if (c->d_pool && keep > 0)
            VD_CUDA(cudaMemcpyAsync(fresh, c->d_pool, size_t(keep) * sizeof(float4), cudaMemcpyDeviceToDevice,
                                    c->stream));
        VD_CUDA(cudaStreamSynchronize(c->stream));
        dev_release(*c, c->d_pool);
        c->d_pool = fresh;
        c->pool_cap = cap;
    }
    const size_t first = c->pool_synced;
    if (first < c->ligs.size()) {
        const int64_t begin = c->ligs[first].pool_offset;
        std::vector<float4> host(size_t(words - begin));
        for (size_t i = first; i < c->ligs.size(); ++i) {
            const HostLigand& L = c->ligs[i];
            std::memcpy(&host[size_t(L.pool_offset - begin)], L.blob.data(), L.blob.size() * sizeof(float4));
        }
        VD_CUDA(cudaMemcpyAsync(c->d_pool + begin, host.data(), host.size() * sizeof(float4), cudaMemcpyHostToDevice,
                                c->stream));
        VD_CUDA(cudaStreamSynchronize(c->stream));
    }
    c->pool_synced = c->ligs.size();
    c->pool_dirty = false;
    return VD_OK;
}

namespace {

// Checks that rigid bodies are numbered in depth-first pre-order, the order
// in which torsions are stored in a pose (tree.h:395-400).
bool preorder_ok(const int32_t* parent, int nn) {
    if (nn < 1 || parent[0] != -1) return false;
    std::vector<int> stack{0};
    for (int k = 1; k < nn; ++k) {
        const int p = parent[k];
        while (!stack.empty() && stack.back() != p) stack.pop_back();
        if (stack.empty()) return false;
        stack.push_back(k);
    }
    return true;
}

// Orders pairs by their second atom b.  The energy kernel gives each lane a
// contiguous segment of this list and keeps atom b's coordinates and force in
// registers while b stays the same; inside a row of equal b, the first atoms
// are rotated by b so lanes entering new rows do not all hit the same atom.
std::vector<int2> order_pairs(const std::vector<int2>& in) {
    std::vector<int2> out(in);
    std::stable_sort(out.begin(), out.end(), [](const int2& x, const int2& y) {
        return (x.x >> 16) != (y.x >> 16) ? (x.x >> 16) < (y.x >> 16) : (x.x & 0xffff) < (y.x & 0xffff);
    });
    for (size_t r0 = 0; r0 < out.size();) {
        size_t r1 = r0;
        while (r1 < out.size() && (out[r1].x >> 16) == (out[r0].x >> 16)) ++r1;
        const size_t len = r1 - r0;
        std::rotate(out.begin() + r0, out.begin() + r0 + (size_t(out[r0].x >> 16) * 13) % len, out.begin() + r1);
        r0 = r1;
    }
    return out;
}

// Validates one ligand descriptor and builds its device blob and host
// copies; touches no context state, so ligands can be built concurrently.
vd_status build_ligand(const vd_ligand_desc* d, HostLigand& L) {
    VD_CHECK(d, VD_ERR_ARG, "vd_add_ligand: NULL argument");
    const int na = d->n_atoms, nn = d->n_nodes, np = d->n_pairs;
    VD_CHECK(na >= 1 && nn >= 1 && np >= 0, VD_ERR_ARG, "vd_add_ligand: empty ligand");
    VD_CHECK(d->xyz && d->xs && d->el && d->atom_node && d->node_parent && d->node_origin_atom &&
                 d->node_axis_atom && (np == 0 || d->pairs),
             VD_ERR_ARG, "vd_add_ligand: NULL array");
    VD_CHECK(nn - 1 <= kMaxTors, VD_ERR_CAPACITY, "vd_add_ligand: more than 48 torsions");
    VD_CHECK(preorder_ok(d->node_parent, nn), VD_ERR_ARG,
             "vd_add_ligand: rigid bodies must be numbered in depth-first pre-order");
    std::vector<int32_t> heavy_of(na, -1), heavy_index;
    for (int i = 0; i < na; ++i) {
        VD_CHECK(d->xs[i] >= -1 && d->xs[i] < kTypes, VD_ERR_ARG, "vd_add_ligand: XS type out of range");
        VD_CHECK(d->atom_node[i] >= 0 && d->atom_node[i] < nn, VD_ERR_ARG, "vd_add_ligand: atom_node out of range");
        VD_CHECK(std::isfinite(d->xyz[3 * size_t(i)]) && std::isfinite(d->xyz[3 * size_t(i) + 1]) &&
                     std::isfinite(d->xyz[3 * size_t(i) + 2]),
                 VD_ERR_ARG, "vd_add_ligand: non-finite coordinate");
        VD_CHECK(i == 0 || d->atom_node[i] >= d->atom_node[i - 1], VD_ERR_ARG,
                 "vd_add_ligand: atoms must be grouped by rigid body in body order");
        if (d->xs[i] >= 0) {
            heavy_of[i] = int32_t(heavy_index.size());
            heavy_index.push_back(i);
        }
    }
    const int nh = int(heavy_index.size());
    VD_CHECK(nh >= 1, VD_ERR_ARG, "vd_add_ligand: no typed (heavy) atoms");
    VD_CHECK(nh <= kMaxHeavy, VD_ERR_CAPACITY, "vd_add_ligand: more than 128 heavy atoms");
    for (int k = 0; k < nn; ++k) {
        VD_CHECK(d->node_origin_atom[k] >= 0 && d->node_origin_atom[k] < na, VD_ERR_ARG,
                 "vd_add_ligand: node_origin_atom out of range");
        VD_CHECK(k == 0 || (d->node_axis_atom[k] >= 0 && d->node_axis_atom[k] < na), VD_ERR_ARG,
                 "vd_add_ligand: node_axis_atom out of range");
    }
    // pairs between heavy atoms
    std::vector<int2> pairs;
    for (int p = 0; p < np; ++p) {
        const int a = d->pairs[2 * p], b = d->pairs[2 * p + 1];
        VD_CHECK(a >= 0 && a < na && b >= 0 && b < na && a != b, VD_ERR_ARG, "vd_add_ligand: pair index out of range");
        if (heavy_of[a] < 0 || heavy_of[b] < 0) continue;
        pairs.push_back(make_int2(heavy_of[a] | (heavy_of[b] << 16), tri_index(d->xs[a], d->xs[b])));
    }
    const int P = int(pairs.size());
    VD_CHECK(P <= kMaxPairs, VD_ERR_CAPACITY, "vd_add_ligand: more than 4096 intra pairs");
    pairs = order_pairs(pairs);

    auto xyz = [&](int i, int k) { return d->xyz[3 * size_t(i) + k]; };
    // body geometry (tree.h:230-262): origin, unit axis from the parent-side atom
    std::vector<NodeRec> nodes(nn);
    std::vector<int> depth(nn, 0), sub_end(nn, 0);
    for (int k = 0; k < nn; ++k) {
        NodeRec& r = nodes[k];
        std::memset(&r, 0, sizeof(r));
        r.parent = d->node_parent[k];
        depth[k] = (k == 0) ? 0 : depth[r.parent] + 1;
        r.depth = depth[k];
        const int o = d->node_origin_atom[k];
        if (k > 0) {
            const int po = d->node_origin_atom[r.parent];
            const int ax = d->node_axis_atom[k];
            double diff[3], nrm = 0;
            for (int j = 0; j < 3; ++j) {
                r.rel_origin[j] = float(xyz(o, j) - xyz(po, j));
                diff[j] = xyz(o, j) - xyz(ax, j);
                nrm += diff[j] * diff[j];
            }
            nrm = std::sqrt(nrm);
            VD_CHECK(nrm > 1e-6, VD_ERR_ARG, "vd_add_ligand: zero-length torsion axis");
            for (int j = 0; j < 3; ++j) r.axis[j] = float((1 / nrm) * diff[j]);
        }
        r.atom_begin = nh;
        r.atom_end = 0;
    }
    for (int k = nn - 1; k >= 0; --k) {  // pre-order: subtree is [k, sub_end)
        sub_end[k] = k + 1;
        for (int j = k + 1; j < nn && depth[j] > depth[k]; ++j) sub_end[k] = j + 1;
    }
    int max_depth = 0;
    for (int k = 0; k < nn; ++k) {
        nodes[k].subtree_end = sub_end[k];
        max_depth = std::max(max_depth, depth[k]);
    }
    std::vector<float4> atoms(nh);
    for (int hi = 0; hi < nh; ++hi) {
        const int i = heavy_index[hi];
        const int k = d->atom_node[i];
        const int o = d->node_origin_atom[k];
        NodeRec& r = nodes[k];
        r.atom_begin = std::min(r.atom_begin, hi);
        r.atom_end = std::max(r.atom_end, hi + 1);
        float4 a;
        a.x = float(xyz(i, 0) - xyz(o, 0));
        a.y = float(xyz(i, 1) - xyz(o, 1));
        a.z = float(xyz(i, 2) - xyz(o, 2));
        VD_CHECK(d->el[i] >= 0 && d->el[i] < 256, VD_ERR_ARG, "vd_add_ligand: element type out of range");
        int packed = d->xs[i] | (k << 8) | (d->el[i] << 16);
        std::memcpy(&a.w, &packed, sizeof(int));
        atoms[hi] = a;
    }
    // heavy atoms are grouped by body in pre-order: body k owns [hb[k], hb[k+1])
    // and its subtree [hb[k], hb[subtree_end])
    std::vector<int> hb(nn + 1, 0);
    for (int hi = 0; hi < nh; ++hi) ++hb[d->atom_node[heavy_index[hi]] + 1];
    for (int k = 0; k < nn; ++k) hb[k + 1] += hb[k];
    for (int k = 0; k < nn; ++k) {
        nodes[k].atom_begin = hb[k];
        nodes[k].atom_end = hb[k + 1];
        nodes[k].sub_atom_end = hb[sub_end[k]];
    }
    L = HostLigand{};
    LigHeader& H = L.h;
    std::memset(&H, 0, sizeof(H));
    H.n_atoms = nh;
    H.n_nodes = nn;
    H.n_pairs = P;
    H.ntors = nn - 1;
    H.max_depth = max_depth;
    auto words = [](size_t bytes) { return int32_t((bytes + 15) / 16); };
    H.off_atoms = 4;
    H.off_nodes = H.off_atoms + nh;
    H.off_pairs = H.off_nodes + 3 * nn;
    H.off_lpairs = H.off_pairs + std::max<int32_t>(1, words(size_t(P) * sizeof(int2)));
    int max_seg = 0;
    for (int l = 0; l < 32; ++l) max_seg = std::max(max_seg, ((l + 1) * P >> 5) - (l * P >> 5));
    H.lp_iters = (max_seg + 1) / 2;
    std::vector<int4> lpairs(size_t(32) * H.lp_iters, make_int4(0, 0, 0, 0));
    for (int l = 0; l < 32; ++l) {
        const int p0 = l * P >> 5, p1 = (l + 1) * P >> 5;
        for (int p = p0, k = 0; p < p1; p += 2, ++k) {
            const int2 q0 = pairs[p], q1 = p + 1 < p1 ? pairs[p + 1] : q0;
            lpairs[size_t(k) * 32 + l] = make_int4(q0.x, q0.y, q1.x, q1.y);
        }
    }
    H.off_spairs = H.off_lpairs + std::max<int32_t>(1, int32_t(lpairs.size()));
    const std::vector<std::vector<int2>> rounds = schedule_pairs(pairs, nh);
    H.sp_iters = int32_t((rounds.size() + 1) / 2);
    static_assert(kMaxHeavy <= 256 && kPairTypes < 32768, "schedule word fields");
    // one 32-bit word per scheduled pair: a | b << 8 | type pair << 16
    // (heavy atoms < 128, type pairs < 153).  An unused slot has atoms 0 and
    // 0 and type field 0xffff (a negative word): the kernel loads both atoms'
    // coordinates before it tests the slot, so its atom fields must index
    // real atoms.
    constexpr int kUnusedSlot = -65536;  // 0xffff0000
    std::vector<int2> spairs(size_t(32) * H.sp_iters, make_int2(kUnusedSlot, kUnusedSlot));
    for (size_t r = 0; r < rounds.size(); ++r)
        for (size_t l = 0; l < rounds[r].size(); ++l) {
            const int2 q = rounds[r][l];
            if (q.y < 0) continue;  // empty lane
            const int w = (q.x & 0xff) | (((q.x >> 16) & 0xff) << 8) | (q.y << 16);
            int2& e = spairs[(r / 2) * 32 + l];
            if (r % 2 == 0) e.x = w;
            else e.y = w;
        }
    const int32_t total = H.off_spairs + std::max<int32_t>(1, words(spairs.size() * sizeof(int2)));
    H.num_tors = float(d->num_tors);
    L.blob.assign(size_t(total), make_float4(0, 0, 0, 0));
    char* base = reinterpret_cast<char*>(L.blob.data());
    std::memcpy(base, &H, sizeof(H));
    std::memcpy(base + 16 * size_t(H.off_atoms), atoms.data(), atoms.size() * sizeof(float4));
    std::memcpy(base + 16 * size_t(H.off_nodes), nodes.data(), nodes.size() * sizeof(NodeRec));
    if (P) std::memcpy(base + 16 * size_t(H.off_pairs), pairs.data(), pairs.size() * sizeof(int2));
    if (!lpairs.empty()) std::memcpy(base + 16 * size_t(H.off_lpairs), lpairs.data(), lpairs.size() * sizeof(int4));
    if (!spairs.empty()) std::memcpy(base + 16 * size_t(H.off_spairs), spairs.data(), spairs.size() * sizeof(int2));
    L.heavy_index = heavy_index;
    L.n_all_atoms = na;
    L.num_tors = d->num_tors;
    return VD_OK;
}

// Appends a built ligand to the context's pool (its blob's offset is fixed
// here; the next docking call uploads it).
int32_t append_ligand(Ctx& c, HostLigand&& L) {
    L.pool_offset = c.pool_words;
    c.pool_words += int64_t(L.blob.size());
    c.ligs.push_back(std::move(L));
    c.pool_dirty = true;
    return int32_t(c.ligs.size()) - 1;
}

}  // namespace
}  // namespace vd

using namespace vd;

extern "C" {

vd_status vd_add_ligand(vd_ctx* h, const vd_ligand_desc* d, int32_t* lig_id) {
    VD_CHECK(h && d && lig_id, VD_ERR_ARG, "vd_add_ligand: NULL argument");
    HostLigand L;
    const vd_status st = build_ligand(d, L);
    if (st != VD_OK) return st;
    *lig_id = append_ligand(h->c, std::move(L));
    return VD_OK;
}

vd_status vd_add_ligands(vd_ctx* h, const vd_ligand_desc* descs, int32_t n, int32_t* lig_ids) {
    VD_CHECK(h && n >= 0 && (n == 0 || (descs && lig_ids)), VD_ERR_ARG, "vd_add_ligands: NULL argument");
    std::vector<HostLigand> built(size_t(n) > 0 ? size_t(n) : 0);
    std::vector<vd_status> status(built.size(), VD_OK);
    std::vector<std::string> message(built.size());
    const int hw = int(std::max(1u, std::thread::hardware_concurrency()));
    const int workers = std::max(1, std::min({n, hw, 32}));
    auto work = [&](int w) {
        for (int i = w; i < n; i += workers) {  // interleaved: sizes vary along a list
            status[i] = build_ligand(&descs[i], built[i]);
            if (status[i] != VD_OK) message[i] = vd_last_error();  // this worker's message
        }
    };
    if (workers == 1) {
        work(0);
    } else {
        // threads that cannot be started leave their share to this thread
        std::vector<std::thread> pool;
        std::vector<int> unstarted;
        for (int w = 0; w < workers; ++w) {
            try {
                pool.emplace_back(work, w);
            } catch (const std::system_error&) {
                unstarted.push_back(w);
            }
        }
        for (int w : unstarted) work(w);
        for (auto& t : pool) t.join();
    }
    for (int i = 0; i < n; ++i)
        if (status[i] != VD_OK) {
            set_error("vd_add_ligands: ligand " + std::to_string(i) + ": " + message[i]);
            return status[i];
        }
    for (int i = 0; i < n; ++i) lig_ids[i] = append_ligand(h->c, std::move(built[i]));
    return VD_OK;
}

vd_status vd_ligand_info(vd_ctx* h, int32_t lig, int32_t* n_heavy, int32_t* ntors, int32_t* n_pairs) {
    VD_CHECK(h && lig >= 0 && lig < int32_t(h->c.ligs.size()), VD_ERR_ARG, "vd_ligand_info: bad ligand id");
    const LigHeader& H = h->c.ligs[lig].h;
    if (n_heavy) *n_heavy = H.n_atoms;
    if (ntors) *ntors = H.ntors;
    if (n_pairs) *n_pairs = H.n_pairs;
    return VD_OK;
}

vd_status vd_clear_ligands(vd_ctx* h) {
    VD_CHECK(h, VD_ERR_ARG, "vd_clear_ligands: NULL context");
    h->c.ligs.clear();
    h->c.pool_words = 0;
    h->c.pool_synced = 0;
    h->c.pool_dirty = true;
    return VD_OK;
}

}  // extern "C"
