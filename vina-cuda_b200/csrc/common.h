// Internal declarations shared by the vdock host code and CUDA kernels.
#pragma once

#include <cstddef>
#include <cstdint>
#include <cstdio>
#include <string>
#include <unordered_map>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/vdock.h"
#include "tune.h"

namespace vd {

constexpr int kTypes = 17;                       // XS_TYPE_SIZE
constexpr int kPairTypes = kTypes * (kTypes + 1) / 2;  // 153
constexpr int kN = 2051;                         // int(32*64)+3 table entries
constexpr int kBins = 2049;                      // bins reachable for r^2 <= 64
constexpr double kCutoff2 = 64.0;
constexpr int kMaxHeavy = VD_MAX_ATOMS;
constexpr int kMaxTors = VD_MAX_TORS;
constexpr int kMaxNodes = VD_MAX_TORS + 1;
constexpr int kMaxPairs = VD_MAX_PAIRS;

inline int tri_index(int t1, int t2) {
    return (t1 <= t2) ? t1 + t2 * (t2 + 1) / 2 : t2 + t1 * (t1 + 1) / 2;
}

// ---------------------------------------------------------------- errors
void set_error(const std::string& msg);
#define VD_CUDA(call)                                                              \
    do {                                                                           \
        cudaError_t e_ = (call);                                                   \
        if (e_ != cudaSuccess) {                                                   \
            ::vd::set_error(std::string(#call) + ": " + cudaGetErrorString(e_));   \
            return VD_ERR_CUDA;                                                    \
        }                                                                          \
    } while (0)
#define VD_CHECK(cond, code, msg)                                                  \
    do {                                                                           \
        if (!(cond)) {                                                             \
            ::vd::set_error(msg);                                                  \
            return code;                                                           \
        }                                                                          \
    } while (0)

// ---------------------------------------------------------------- device ligand
// One ligand is one contiguous blob of 16-byte words in the ligand pool:
//   LigHeader | atoms (float4) | nodes (NodeRec) | pairs (int2) | lane pairs (int4)
//   | search schedule (int4)
// The lane-pair array holds the same pairs split into the 32 per-lane
// segments the energy kernel walks (lane l: pairs [l*P/32, (l+1)*P/32) of the
// ordered list), two pairs per int4, interleaved so that iteration k of every
// lane reads entry k*32 + l: one coalesced 512-byte warp load per two pairs.
// A lane's odd last pair is repeated in the int4's second half.
// The search schedule holds the same pairs again in rounds of up to 32, one
// pair per lane per round, each pair one 32-bit word (a | b << 8 | type pair
// << 16), two rounds per int2 (entry k*32 + l: rounds 2k and 2k+1 of lane
// l, one coalesced 256-byte warp load), arranged so that the lanes of a
// round touch as few equal atoms as possible: the search adds both atoms'
// pair forces with shared-memory atomics, and on B200 atomics of several
// lanes to one address serialise.  An unused slot is 0xffff0000 (atoms 0
// and 0, negative as a signed word).
// Only heavy atoms (XS type >= 0) are on the device; hydrogens carry no
// energy and are placed on the host when output files are written.
struct LigHeader {
    int32_t n_atoms;      // heavy atoms
    int32_t n_nodes;
    int32_t n_pairs;
    int32_t ntors;
    int32_t off_atoms;    // in 16-byte words from the blob start
    int32_t off_nodes;
    int32_t off_pairs;    // int2 entries start (16-byte word offset)
    int32_t max_depth;
    int32_t off_lpairs;   // lane-pair int4 entries start (16-byte word offset)
    int32_t lp_iters;     // int4 entries per lane (longest segment, two pairs each)
    int32_t off_spairs;   // search-schedule int2 entries start (16-byte word offset)
    int32_t sp_iters;     // int2 entries per lane of the search schedule (two rounds each)
    float num_tors;       // N_tors of the conf-independent term
    float pad3, pad4, pad5;
};
static_assert(sizeof(LigHeader) == 64, "header size");

// Atom word: local coords (relative to its rigid body's origin) and
// (xs type | node << 8 | element << 16) stored in .w as int bits.
// Rigid body record: origin relative to parent frame, torsion axis in the
// parent frame, parent index, atom range and subtree end (pre-order).
// Three 16-byte words, grouped by use so the evaluation reads each with one
// 128-bit load: {origin, parent} per step of the ancestor walk, {axis,
// first atom} for the local rotation and the torsion derivative, and the
// ranges (sub_atom_end last) for the subtree sums.
struct NodeRec {
    float rel_origin[3];
    int32_t parent;
    float axis[3];
    int32_t atom_begin;
    int32_t atom_end;
    int32_t subtree_end;  // nodes [k, subtree_end) form k's subtree
    int32_t depth;
    int32_t sub_atom_end;  // heavy atoms [atom_begin, sub_atom_end) belong to k's subtree
};
static_assert(sizeof(NodeRec) == 48, "node size");
static_assert(offsetof(NodeRec, parent) == 12 && offsetof(NodeRec, atom_begin) == 28 &&
                  offsetof(NodeRec, sub_atom_end) == 44,
              "node words");

struct HostLigand {
    LigHeader h;
    std::vector<float4> blob;      // whole blob incl. header
    // host-side copies for helpers
    std::vector<int32_t> heavy_index;  // device atom -> input atom index
    int32_t n_all_atoms = 0;
    int64_t pool_offset = 0;       // in float4 words
    double num_tors = 0;
};

// Grid geometry exactly as main.cpp:864-876 / grid.cpp:29-43 (double).
struct GridGeom {
    int32_t n[3];          // points per dim
    double begin[3], end[3];
    double init[3], factor[3], finv[3], dmo[3];
    int32_t pitch;         // x pitch in floats (multiple of 4)
};

struct Ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr, ev2 = nullptr;
    bool scoring = false;
    double weights[6];
    std::vector<double> fast, se, sd;     // [153][2051] double (host)
    float* d_fast = nullptr;              // [153][2049] float (rescoring, eval_fast)
    float4* d_smooth = nullptr;           // [153][2049] {e_i, dor_i, e_i+1, dor_i+1}
    float fix_scale = 524288.f;           // fixed-point units per kcal/mol/A of the pair forces
    double* d_fastd = nullptr;            // [153][2049] double (final rescoring)
    // receptor
    std::vector<double> rec_xyz;
    std::vector<int32_t> rec_xs;
    bool has_box = false;
    GridGeom geom{};
    // grids
    float* d_maps = nullptr;              // [n_maps][nz][ny][pitch]
    size_t map_stride = 0;                // floats per map
    // the same maps as trilinear cells for the evaluation kernels: per map
    // [nz-1][ny-1][nx-1] cells of the 8 corner values (32 bytes, one sector),
    // null when the box is too large for them (the kernels then read d_maps)
    float* d_cells = nullptr;
    size_t cell_stride = 0;               // floats per map
    int map_slot[kTypes];                 // xs type -> map index or -1
    int n_maps = 0;
    // direct-sum receptor cell list (non_cache): ~3 A cells over the box,
    // each listing the receptor atoms within 8 A of it (szv_grid.cpp:28-74)
    float4* d_rec = nullptr;              // relevant receptor atoms {x,y,z,type}
    double4* d_recd = nullptr;            // same in double
    int32_t* d_cell_start = nullptr;      // [cells+1]
    int32_t* d_cell_list = nullptr;       // atom indices
    int32_t cell_dim[3] = {0, 0, 0};
    double cell_init[3], cell_range[3];
    int32_t n_rec_dev = 0;
    bool rec_dev_ready = false;
    // ligands
    std::vector<HostLigand> ligs;
    float4* d_pool = nullptr;
    int64_t pool_words = 0, pool_cap = 0;   // words of all added ligands / device capacity
    size_t pool_synced = 0;                 // ligands already on the device
    bool pool_dirty = false;
    // scratch
    void* d_scratch = nullptr;
    size_t scratch_bytes = 0;
    int32_t* d_counter = nullptr;         // work queue + error words
    // batched pipeline: pinned staging of its uploads and results, and the
    // executable CUDA graph it is recorded into (updated in place per call)
    void* h_stage = nullptr;
    size_t h_stage_bytes = 0;
    cudaGraphExec_t pipe_exec = nullptr;
    vd_stats stats{};
    // device memory owned by the context (dev_alloc / dev_free): bytes in use
    // per allocation, and an optional cap (0 = none) that turns an allocation
    // past it into VD_ERR_NOMEM
    std::unordered_map<void*, size_t> dev_bytes;
    size_t dev_used = 0, dev_cap = 0;
    // launch-shape autotuners (tune.h); grid_shape_fixed > 0 pins the grid tile
    Tuner dock_tune, grid_tune;
    int grid_shape_fixed = 0;
};

// Event record that becomes an event node (usable for timing) when the stream
// is being captured into a CUDA graph, and a plain record otherwise.
inline cudaError_t record_event(cudaEvent_t e, cudaStream_t s) {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    const cudaError_t r = cudaStreamIsCapturing(s, &cs);
    if (r != cudaSuccess) return r;
    return cs == cudaStreamCaptureStatusActive ? cudaEventRecordWithFlags(e, s, cudaEventRecordExternal)
                                               : cudaEventRecord(e, s);
}

// Each SM's on-chip data memory is split between shared memory and L1.  Asks
// for the smallest shared-memory carve-out that holds `blocks` resident
// blocks of `smem` bytes each (plus the driver's per-block reservation); the
// percentage is rounded up and the driver rounds it up again to a capacity
// it supports.  The rest is L1, which caches the kernels' table and grid
// gathers.
template <class K>
inline cudaError_t prefer_l1(K kernel, int device, int blocks, size_t smem) {
    int max_sm = 0, reserved = 0;
    cudaError_t r = cudaDeviceGetAttribute(&max_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, device);
    if (r == cudaSuccess) r = cudaDeviceGetAttribute(&reserved, cudaDevAttrReservedSharedMemoryPerBlock, device);
    if (r != cudaSuccess || max_sm <= 0) return r;
    const size_t need = size_t(blocks) * (smem + size_t(reserved));
    size_t pct = (need * 100 + size_t(max_sm) - 1) / size_t(max_sm);
    if (pct > 100) pct = 100;
    return cudaFuncSetAttribute(kernel, cudaFuncAttributePreferredSharedMemoryCarveout, int(pct));
}

vd_status ensure_scratch(Ctx* c, size_t bytes);
// Context-owned device allocation: VD_ERR_NOMEM past the context's cap or
// when the device is out of memory; *p is null on failure.
vd_status dev_alloc(Ctx& c, void** p, size_t bytes, const char* what);
template <class T>
vd_status dev_alloc(Ctx& c, T** p, size_t bytes, const char* what) {
    void* q = nullptr;
    const vd_status st = dev_alloc(c, &q, bytes, what);
    *p = static_cast<T*>(q);
    return st;
}
// Frees a dev_alloc allocation (null is fine) and sets the pointer to null.
void dev_free(Ctx& c, void* p);
template <class T>
void dev_release(Ctx& c, T*& p) {
    dev_free(c, p);
    p = nullptr;
}
vd_status ensure_host_stage(Ctx* c, size_t bytes);
vd_status sync_pool(Ctx* c);
vd_status ensure_receptor_cells(Ctx* c);
void build_tables(const double w[6], std::vector<double>& fast, std::vector<double>& se,
                  std::vector<double>& sd);
// Largest power of two (at most 2^24) for which 128 times the largest pair
// force of the derivative table stays below 2^30: the fixed-point scale of
// the kernels' per-atom pair-force sums.
float pair_force_scale(const std::vector<double>& sd);
// Same tables built on the device into the context's device copies, with
// the double tables copied back to c.fast / c.se / c.sd.
vd_status build_tables_device(Ctx& c, const double w[6]);

}  // namespace vd

struct vd_ctx {
    vd::Ctx c;
};
