// Grid-map precompute: replaces kernel_grid / kernel1 (kernel1.cu:93-249).
//
// Value of map t at grid point p (cache.cpp:148-208):
//   G_t(p) = sum over receptor atoms a with r^2 = |a - p|^2 <= 64 of
//            fast[pair(t_a, t)][int(32 r^2)]
// The bin index must match the reference's double computation bit for bit,
// so p = init + finv*i and r^2 = ((ax-px)^2 + (ay-py)^2) + (az-pz)^2 are
// evaluated in double with explicitly rounded operations (no FMA
// contraction); the table values are FP32 and the sums are FP32.
//
// Launch: one CTA per tile of 16(x) x 8(y) x TZ(z) points (TZ = 8 or 4,
// autotuned), 32*TZ threads, each thread owning 4 consecutive x points so
// every map store is one 128-bit store; one launch per group of up to 8 maps.  The CTA stages, in shared
// memory, the receptor atoms whose brick distance to the tile is below the
// cutoff, taken from per-type 4 A cell lists in deterministic (receptor type,
// cell, index) order.  The bin index floor(32 r^2) comes from a rounded-down
// FP64 add of 2^52 (no FP64->int conversion), every point within the cutoff
// then reads one 32-byte table row (predicated loads, so a thread's four
// issue together) and the accumulators are packed FP32 pairs added with
// add.rn.f32x2.
#include <algorithm>
#include <cmath>
#include <cstring>

#include "checks.cuh"
#include "common.h"

namespace vd {
namespace {

constexpr int kTileX = 16, kTileY = 8;  // z tile (TZ = 8 or 4) is a launch shape; threads = 32 * TZ
constexpr int kStageCap = 128;    // atoms staged per chunk (4 KB; a 70 A tile keeps ~60, larger counts loop)
constexpr double kCellSize = 4.0;
constexpr int kLutRows = kBins + 1;  // table rows per receptor type; the last (zero) row is padding

struct StagedAtom {
    double x, y, z;
    int32_t type;
    int32_t pad;
};

struct GridParams {
    double init[3], finv[3];
    int32_t n[3];
    int32_t pitch;
    size_t map_stride;
    float* maps;                  // first map of this type group
    const float* lut;             // this group's [receptor types present][kLutRows][NTG]
    int32_t n_out;                // maps written by this group (<= NTG)
    const StagedAtom* atoms;      // relevant receptor atoms sorted by (type, cell)
    const int32_t* cell_start;    // [n_rtypes][cells+1] per receptor type
    int32_t n_rtypes;             // receptor types present
    int32_t n_cells;
    double cell_org[3];
    int32_t cell_dim[3];
};

__device__ __forceinline__ double probe_coord(double init, double finv, int i) {
    return __dadd_rn(init, __dmul_rn(finv, double(i)));
}

constexpr int kMaxRows = 36;            // (cell rows in y) x (cell rows in z) per tile
constexpr int kMaxCombos = kTypes * kMaxRows;
// Block-wide exclusive scan of cnt[0..n) into off[0..n]; n <= kMaxCombos.
template <int kThreads>
__device__ __forceinline__ void block_scan(const int32_t* cnt, int32_t* off, int32_t* s_warp, int n) {
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const int per = (n + kThreads - 1) / kThreads;
    const int j0 = min(n, t * per), j1 = min(n, j0 + per);
    int sum = 0;
    for (int j = j0; j < j1; ++j) sum += cnt[j];
    int incl = sum;
    for (int o = 1; o < 32; o <<= 1) {
        const int v = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += v;
    }
    if (lane == 31) s_warp[warp] = incl;
    __syncthreads();
    int run = incl - sum;
    for (int w = 0; w < warp; ++w) run += s_warp[w];
    for (int j = j0; j < j1; ++j) {
        off[j] = run;
        run += cnt[j];
    }
    if (t == kThreads - 1) off[n] = run;
    __syncthreads();
}

// floor(32 * r2) for 0 <= r2 <= 64 on the FP64 pipe: 32 * r2 is exact, and
// adding 2^52 rounded toward -inf leaves the floor in the low mantissa word.
__device__ __forceinline__ int bin_of(double r2) {
    return __double2loint(__fma_rd(r2, 32.0, 4503599627370496.0));
}

// Two FP32 accumulators in one 64-bit register, added with one packed
// instruction (each lane rounds exactly like a scalar FP32 add).
__device__ __forceinline__ unsigned long long add2(unsigned long long a, unsigned long long b) {
    unsigned long long d;
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}

// acc[0..NTG/2) += table row v (NTG floats, 32- or 16-byte aligned).
template <int NTG>
__device__ __forceinline__ void add_row(unsigned long long (&acc)[NTG / 2], const float* v) {
    if constexpr (NTG == 8) {
        unsigned long long a0, a1, a2, a3;
        asm("ld.global.nc.v4.b64 {%0,%1,%2,%3}, [%4];" : "=l"(a0), "=l"(a1), "=l"(a2), "=l"(a3) : "l"(v));
        acc[0] = add2(acc[0], a0);
        acc[1] = add2(acc[1], a1);
        acc[2] = add2(acc[2], a2);
        acc[3] = add2(acc[3], a3);
    } else {
        unsigned long long a0, a1;
        asm("ld.global.nc.v2.b64 {%0,%1}, [%2];" : "=l"(a0), "=l"(a1) : "l"(v));
        acc[0] = add2(acc[0], a0);
        acc[1] = add2(acc[1], a1);
    }
}

// TZ = 8: 256 threads, 2 blocks per SM (120 registers); TZ = 4: 128 threads,
// 4 blocks per SM, twice the blocks for small boxes.
template <int NTG, int TZ>
__global__ void __launch_bounds__(32 * TZ, 16 / TZ) grid_build_kernel(GridParams p) {
    constexpr int kThreads = 32 * TZ, kTileZ = TZ;
    __shared__ StagedAtom s_atoms[kStageCap];
    __shared__ int32_t s_cnt[kMaxCombos];
    __shared__ int32_t s_b[kMaxCombos];
    __shared__ int32_t s_off[kMaxCombos + 1];
    __shared__ int32_t s_warp[kThreads / 32];
    __shared__ int32_t s_keep[kThreads / 32];

    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const int xq = t & 3, ly = (t >> 2) & 7, lz = t >> 5;
    const int x0 = blockIdx.x * kTileX + xq * 4;
    const int y = blockIdx.y * kTileY + ly;
    const int z = blockIdx.z * kTileZ + lz;

    // Tile bounding box (double) and the cell rows covering it +- 8 A.
    const int tx_lo = blockIdx.x * kTileX, ty_lo = blockIdx.y * kTileY, tz_lo = blockIdx.z * kTileZ;
    const int tx_hi = min(tx_lo + kTileX - 1, p.n[0] - 1);
    const int ty_hi = min(ty_lo + kTileY - 1, p.n[1] - 1);
    const int tz_hi = min(tz_lo + kTileZ - 1, p.n[2] - 1);
    const double lo[3] = {probe_coord(p.init[0], p.finv[0], tx_lo), probe_coord(p.init[1], p.finv[1], ty_lo),
                          probe_coord(p.init[2], p.finv[2], tz_lo)};
    const double hi[3] = {probe_coord(p.init[0], p.finv[0], tx_hi), probe_coord(p.init[1], p.finv[1], ty_hi),
                          probe_coord(p.init[2], p.finv[2], tz_hi)};
    int c_lo[3], c_hi[3];
    for (int d = 0; d < 3; ++d) {
        c_lo[d] = max(0, int(floor((lo[d] - 8.0 - p.cell_org[d]) / kCellSize)));
        c_hi[d] = min(p.cell_dim[d] - 1, int(floor((hi[d] + 8.0 - p.cell_org[d]) / kCellSize)));
    }
    const int ry = max(0, c_hi[1] - c_lo[1] + 1), rz = max(0, c_hi[2] - c_lo[2] + 1);
    // rows <= kMaxRows: the host checks the tile span against the cell size
    VD_DCHECK(c_lo[0] > c_hi[0] || ry * rz <= kMaxRows, kChkGridRows);
    const int n_rows = (c_lo[0] <= c_hi[0]) ? min(kMaxRows, ry * rz) : 0;
    const int n_combo = p.n_rtypes * n_rows;  // (receptor type, row), type-major

    // Candidate ranges per combo, then their exclusive prefix: candidates are
    // numbered in (type, cz, cy, cx, index) order.
    for (int j = t; j < n_combo; j += kThreads) {
        const int tr = j / n_rows, r = j - tr * n_rows;
        const int cy = c_lo[1] + r % ry, cz = c_lo[2] + r / ry;
        const int32_t* cs = p.cell_start + size_t(tr) * (p.n_cells + 1) + p.cell_dim[0] * (cy + p.cell_dim[1] * cz);
        const int b = __ldg(cs + c_lo[0]), e = __ldg(cs + c_hi[0] + 1);
        s_b[j] = b;
        s_cnt[j] = e - b;
    }
    __syncthreads();
    block_scan<kThreads>(s_cnt, s_off, s_warp, n_combo);
    const int n_cand = s_off[n_combo];

    const bool active = (x0 < p.n[0]) && (y < p.n[1]) && (z < p.n[2]);
    double px[4];
    for (int k = 0; k < 4; ++k) px[k] = probe_coord(p.init[0], p.finv[0], x0 + k);
    const double py = probe_coord(p.init[1], p.finv[1], y);
    const double pz = probe_coord(p.init[2], p.finv[2], z);

    unsigned long long acc[4][NTG / 2];  // maps (2j, 2j+1) of point k
#pragma unroll
    for (int k = 0; k < 4; ++k)
#pragma unroll
        for (int j = 0; j < NTG / 2; ++j) acc[k][j] = 0ull;

    for (int chunk = 0;; chunk += kStageCap) {
        // Stage the kept candidates with ranks [chunk, chunk + kStageCap),
        // in candidate order (a block-wide stream compaction).
        int kept = 0;
        for (int base = 0; base < n_cand; base += kThreads) {
            const int i = base + t;
            bool k = false;
            StagedAtom a;
            if (i < n_cand) {
                int lo_j = 0, hi_j = n_combo;  // last j with s_off[j] <= i
                while (hi_j - lo_j > 1) {
                    const int mid = (lo_j + hi_j) >> 1;
                    if (s_off[mid] <= i) lo_j = mid;
                    else hi_j = mid;
                }
                a = p.atoms[s_b[lo_j] + (i - s_off[lo_j])];
                double d2 = 0;
                const double c[3] = {a.x, a.y, a.z};
                for (int d = 0; d < 3; ++d) {
                    const double q = c[d] < lo[d] ? lo[d] - c[d] : (c[d] > hi[d] ? c[d] - hi[d] : 0.0);
                    d2 += q * q;
                }
                k = d2 < kCutoff2 + 1e-6;  // conservative: the per-point test below is exact
            }
            const unsigned m = __ballot_sync(0xffffffffu, k);
            if (lane == 0) s_keep[warp] = __popc(m);
            __syncthreads();
            int rank = kept + __popc(m & ((1u << lane) - 1u));
            int step = 0;
            for (int w = 0; w < kThreads / 32; ++w) {
                const int cw = s_keep[w];
                rank += (w < warp) ? cw : 0;
                step += cw;
            }
            const int slot = rank - chunk;
            if (k && slot >= 0 && slot < kStageCap) s_atoms[slot] = a;
            kept += step;
            __syncthreads();
        }
        const int n_here = min(kStageCap, kept - chunk);
        if (active) {
            for (int a = 0; a < n_here; ++a) {
                const StagedAtom at = s_atoms[a];
                const double dy = __dsub_rn(at.y, py), dz = __dsub_rn(at.z, pz);
                const double dy2 = __dmul_rn(dy, dy), dz2 = __dmul_rn(dz, dz);
                if (__dadd_rn(dy2, dz2) > kCutoff2) continue;  // exact: sums are monotone
                // Each point within the cutoff loads its row; the loads are
                // predicated per point (no branch), so those of a thread still
                // issue back to back, and points beyond the cutoff cost no L1
                // wavefront (the kernel's limit).
                const float* row_base = p.lut + VD_DCLAMP(at.type, 0, p.n_rtypes - 1, kChkGridType) * (kLutRows * NTG);
                int bin[4];
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    const double dx = __dsub_rn(at.x, px[k]);
                    const double r2 = __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), dy2), dz2);
                    bin[k] = r2 <= kCutoff2 ? bin_of(r2) : kBins;
                }
#pragma unroll
                for (int k = 0; k < 4; ++k)
                    if (bin[k] < kBins) add_row<NTG>(acc[k], row_base + bin[k] * NTG);
            }
        }
        if (kept <= chunk + kStageCap) break;
        __syncthreads();
    }
    if (!active) return;
    const size_t off = (size_t(z) * p.n[1] + y) * p.pitch + x0;
#pragma unroll
    for (int j = 0; j < NTG; ++j) {
        if (j >= p.n_out) break;
        const int h = j & 1, q = j >> 1;
        auto f = [&](int k) { return __int_as_float(int(h ? acc[k][q] >> 32 : acc[k][q] & 0xffffffffull)); };
        *reinterpret_cast<float4*>(p.maps + size_t(j) * p.map_stride + off) = make_float4(f(0), f(1), f(2), f(3));
    }
}

// Corner cells for the evaluation kernels: cell (x, y, z) of map j holds the
// map values at its 8 corners (x fastest, then y, then z), 32 bytes, so a
// trilinear lookup reads one sector instead of eight scattered floats.  One
// thread per cell; consecutive threads write consecutive cells.
__global__ void __launch_bounds__(256) corner_cells_kernel(const float* maps, size_t map_stride, float* cells,
                                                           size_t cell_stride, int n_maps, int nx, int ny, int nz,
                                                           int pitch) {
    const int cx = nx - 1, cy = ny - 1, cz = nz - 1;
    const size_t per_map = size_t(cx) * cy * cz;
    const size_t total = per_map * size_t(n_maps);
    for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < total; i += size_t(gridDim.x) * blockDim.x) {
        const int j = int(i / per_map);
        const size_t r = i - size_t(j) * per_map;
        const int x = int(r % size_t(cx));
        const size_t yz = r / size_t(cx);
        const int y = int(yz % size_t(cy)), z = int(yz / size_t(cy));
        const float* b = maps + size_t(j) * map_stride + (size_t(z) * ny + y) * pitch + x;
        const size_t row = size_t(pitch), plane = row * size_t(ny);
        const float4 lo = make_float4(b[0], b[1], b[row], b[row + 1]);
        const float4 hi = make_float4(b[plane], b[plane + 1], b[plane + row], b[plane + row + 1]);
        float4* d = reinterpret_cast<float4*>(cells + size_t(j) * cell_stride + r * 8);
        d[0] = lo;
        d[1] = hi;
    }
}

// Corner cells are built when all of them fit in this many bytes (a 150 A
// box of 17 maps is about 11 GB); larger boxes keep the plain maps only.
constexpr size_t kMaxCellBytes = size_t(16) << 30;

}  // namespace
}  // namespace vd

using namespace vd;

extern "C" {

vd_status vd_build_grids(vd_ctx* h, const int32_t* types, int32_t n_types) {
    VD_CHECK(h && types && n_types > 0 && n_types <= kTypes, VD_ERR_ARG, "vd_build_grids: bad type list");
    Ctx& c = h->c;
    VD_CHECK(c.has_box, VD_ERR_ARG, "vd_build_grids: call vd_set_box first");
    VD_CHECK(c.scoring, VD_ERR_ARG, "vd_build_grids: scoring not set");
    std::vector<int> needed;
    for (int i = 0; i < n_types; ++i) {
        VD_CHECK(types[i] >= 0 && types[i] < kTypes, VD_ERR_ARG, "vd_build_grids: XS type out of range");
        if (std::find(needed.begin(), needed.end(), types[i]) == needed.end()) needed.push_back(types[i]);
    }
    VD_CUDA(cudaSetDevice(c.device));
    const GridGeom& g = c.geom;
    const int nt = int(needed.size());

    // Relevant receptor atoms (szv_grid.cpp:28-42 rule) binned into 4 A cells
    // spanning the box grown by the cutoff.
    double org[3];
    int cd[3];
    for (int d = 0; d < 3; ++d) {
        org[d] = g.begin[d] - 8.0 - 1e-3;
        cd[d] = std::max(1, int(std::ceil((g.end[d] - g.begin[d] + 16.0 + 2e-3) / kCellSize)));
    }
    std::vector<StagedAtom> rel;
    std::vector<int> cell_of;
    const int n_rec = int(c.rec_xs.size());
    for (int i = 0; i < n_rec; ++i) {
        if (c.rec_xs[i] < 0) continue;
        const double* a = &c.rec_xyz[3 * size_t(i)];
        double d2 = 0;
        for (int d = 0; d < 3; ++d) {
            double q = (a[d] <= g.begin[d]) ? g.begin[d] : ((a[d] >= g.end[d]) ? g.end[d] : a[d]);
            d2 += (q - a[d]) * (q - a[d]);
        }
        if (!(d2 < kCutoff2)) continue;
        int ci[3];
        for (int d = 0; d < 3; ++d)
            ci[d] = std::min(cd[d] - 1, std::max(0, int(std::floor((a[d] - org[d]) / kCellSize))));
        rel.push_back({a[0], a[1], a[2], c.rec_xs[i], 0});
        cell_of.push_back(ci[0] + cd[0] * (ci[1] + cd[1] * ci[2]));
    }
    // per receptor type present: cell list over the same cells, atoms sorted
    // by (type, cell) so a tile stages them type by type
    const int n_cells = cd[0] * cd[1] * cd[2];
    std::vector<int> present;
    for (int tr = 0; tr < kTypes; ++tr)
        for (const auto& a : rel)
            if (a.type == tr) { present.push_back(tr); break; }
    if (present.empty()) present.push_back(0);
    std::vector<int32_t> start(present.size() * size_t(n_cells + 1), 0);
    std::vector<StagedAtom> sorted(rel.size());
    {
        size_t base_atom = 0;
        for (size_t ti = 0; ti < present.size(); ++ti) {
            int32_t* st = &start[ti * size_t(n_cells + 1)];
            for (size_t i = 0; i < rel.size(); ++i)
                if (rel[i].type == present[ti]) st[cell_of[i] + 1]++;
            st[0] = int32_t(base_atom);
            for (int i = 0; i < n_cells; ++i) st[i + 1] += st[i];
            std::vector<int32_t> fill(st, st + n_cells);
            for (size_t i = 0; i < rel.size(); ++i)
                if (rel[i].type == present[ti]) sorted[fill[cell_of[i]]++] = rel[i];
            base_atom = size_t(st[n_cells]);
        }
    }
    // remap staged atom types to table rows of the present types
    std::vector<int> row_of(kTypes, 0);
    for (size_t ti = 0; ti < present.size(); ++ti) row_of[present[ti]] = int(ti);
    for (auto& a : sorted) a.type = row_of[a.type];
    // Table slices per group of up to 8 maps: [receptor types present][kLutRows][w]
    // with w = 8, or 4 for a last group of at most 4 maps.
    std::vector<int> grp_w, grp_off;
    size_t lut_floats = 0;
    for (int g0 = 0; g0 < nt; g0 += 8) {
        grp_w.push_back(nt - g0 <= 4 ? 4 : 8);
        grp_off.push_back(int(lut_floats));
        lut_floats += present.size() * kLutRows * size_t(grp_w.back());
    }
    std::vector<float> lut(lut_floats, 0.f);
    for (size_t gi = 0; gi < grp_w.size(); ++gi) {
        const int w = grp_w[gi];
        for (size_t ti = 0; ti < present.size(); ++ti)
            for (int j = 0; j < w && 8 * int(gi) + j < nt; ++j) {
                const size_t b = size_t(tri_index(present[ti], needed[8 * gi + j])) * kN;
                for (int i = 0; i < kBins; ++i)
                    lut[grp_off[gi] + (ti * kLutRows + i) * w + j] = float(c.fast[b + i]);
            }
    }

    const size_t map_stride = size_t(g.pitch) * g.n[1] * g.n[2];
    const size_t bytes_maps = map_stride * nt * sizeof(float);
    const size_t bytes_atoms = std::max<size_t>(1, sorted.size()) * sizeof(StagedAtom);
    const size_t bytes_start = start.size() * sizeof(int32_t);
    const size_t bytes_lut = lut.size() * sizeof(float);
    dev_release(c, c.d_maps);
    dev_release(c, c.d_cells);
    c.n_maps = 0;
    for (int i = 0; i < kTypes; ++i) c.map_slot[i] = -1;
    vd_status st0 = dev_alloc(c, &c.d_maps, bytes_maps, "vd_build_grids: maps");
    if (st0 != VD_OK) return st0;
    vd_status st = ensure_scratch(&c, bytes_atoms + bytes_start + bytes_lut + 256);
    if (st != VD_OK) return st;
    char* s = static_cast<char*>(c.d_scratch);
    StagedAtom* d_atoms = reinterpret_cast<StagedAtom*>(s);
    int32_t* d_start = reinterpret_cast<int32_t*>(s + ((bytes_atoms + 255) & ~size_t(255)));
    float* d_lut = reinterpret_cast<float*>(reinterpret_cast<char*>(d_start) + ((bytes_start + 255) & ~size_t(255)));
    if (!sorted.empty())
        VD_CUDA(cudaMemcpyAsync(d_atoms, sorted.data(), sorted.size() * sizeof(StagedAtom), cudaMemcpyHostToDevice, c.stream));
    VD_CUDA(cudaMemcpyAsync(d_start, start.data(), bytes_start, cudaMemcpyHostToDevice, c.stream));
    VD_CUDA(cudaMemcpyAsync(d_lut, lut.data(), bytes_lut, cudaMemcpyHostToDevice, c.stream));

    GridParams p{};
    for (int d = 0; d < 3; ++d) {
        p.init[d] = g.init[d];
        p.finv[d] = g.finv[d];
        p.n[d] = g.n[d];
        p.cell_org[d] = org[d];
        p.cell_dim[d] = cd[d];
    }
    p.pitch = g.pitch;
    p.map_stride = map_stride;
    p.atoms = d_atoms;
    p.cell_start = d_start;
    p.n_rtypes = int(present.size());
    p.n_cells = n_cells;
    for (int d = 1; d < 3; ++d)  // cell rows a tile can touch in y and z: floor(span / cell) + 2 <= 6
        VD_CHECK(int(std::floor(((kTileY - 1) * g.finv[d] + 16.0) / kCellSize)) + 2 <= 6, VD_ERR_CAPACITY,
                 "vd_build_grids: grid spacing too large for the tile");
    // Launch shapes (z tile 8 or 4) give bit-identical maps: a point sums its
    // atoms in global (type, cell, index) order whatever the tile.  The first
    // build of a box size times both and keeps the faster.
    const uint64_t key = (uint64_t(ceil_log2(uint64_t(g.n[0]) * g.n[1] * g.n[2])) << 8) | uint64_t((nt + 7) / 8);
    std::vector<int> shapes;
    if (c.grid_shape_fixed > 0) shapes.push_back(c.grid_shape_fixed - 1);
    else if (c.grid_tune.best(key) >= 0) shapes.push_back(c.grid_tune.best(key));
    else shapes = {0, 1};
    // shared-memory carve-out for the blocks each tile keeps resident (2 of
    // 256 threads or 4 of 128), the rest of the SM's data memory as L1
    auto carve = [&](auto kern, int blocks) -> cudaError_t {
        cudaFuncAttributes fa{};
        const cudaError_t r = cudaFuncGetAttributes(&fa, kern);
        return r != cudaSuccess ? r : prefer_l1(kern, c.device, blocks, fa.sharedSizeBytes);
    };
    VD_CUDA(carve(grid_build_kernel<4, 8>, 2));
    VD_CUDA(carve(grid_build_kernel<8, 8>, 2));
    VD_CUDA(carve(grid_build_kernel<4, 4>, 4));
    VD_CUDA(carve(grid_build_kernel<8, 4>, 4));
    float best_ms = -1;
    for (int shape : shapes) {
        const int tz = shape == 0 ? 8 : 4;
        dim3 grid((g.n[0] + kTileX - 1) / kTileX, (g.n[1] + kTileY - 1) / kTileY, (g.n[2] + tz - 1) / tz);
        VD_CUDA(cudaEventRecord(c.ev0, c.stream));
        for (int g0 = 0; g0 < nt; g0 += 8) {
            p.maps = c.d_maps + size_t(g0) * map_stride;
            p.lut = d_lut + grp_off[g0 / 8];
            p.n_out = std::min(8, nt - g0);
            const bool narrow = nt - g0 <= 4;
            if (shape == 0) {
                if (narrow) grid_build_kernel<4, 8><<<grid, 256, 0, c.stream>>>(p);
                else grid_build_kernel<8, 8><<<grid, 256, 0, c.stream>>>(p);
            } else {
                if (narrow) grid_build_kernel<4, 4><<<grid, 128, 0, c.stream>>>(p);
                else grid_build_kernel<8, 4><<<grid, 128, 0, c.stream>>>(p);
            }
            VD_CUDA(cudaGetLastError());
        }
        VD_CUDA(cudaEventRecord(c.ev1, c.stream));
        VD_CUDA(cudaEventSynchronize(c.ev1));
        if ((st = take_device_checks("grid kernel")) != VD_OK) return st;
        float ms = 0;
        VD_CUDA(cudaEventElapsedTime(&ms, c.ev0, c.ev1));
        c.grid_tune.pick(key, 2);
        c.grid_tune.report(key, shape, ms);
        if (best_ms < 0 || ms < best_ms) best_ms = ms;
        c.stats.grid_shape = shape + 1;
    }
    c.stats.grid_ms = best_ms;
    // corner cells of the new maps (timed separately: cells_ms)
    const size_t n_cells_map = size_t(g.n[0] - 1) * (g.n[1] - 1) * (g.n[2] - 1);
    const size_t bytes_cells = n_cells_map * 8 * sizeof(float) * nt;
    c.stats.cells_ms = 0;
    if (bytes_cells <= kMaxCellBytes) {
        st = dev_alloc(c, &c.d_cells, bytes_cells, "vd_build_grids: corner cells");
        if (st != VD_OK) return st;
        c.cell_stride = n_cells_map * 8;
        int sms = 148;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c.device);
        const size_t total = n_cells_map * nt;
        const int blocks = int(std::min<size_t>((total + 255) / 256, size_t(sms) * 8));
        VD_CUDA(cudaEventRecord(c.ev0, c.stream));
        corner_cells_kernel<<<blocks, 256, 0, c.stream>>>(c.d_maps, map_stride, c.d_cells, c.cell_stride, nt, g.n[0],
                                                            g.n[1], g.n[2], g.pitch);
        VD_CUDA(cudaGetLastError());
        VD_CUDA(cudaEventRecord(c.ev1, c.stream));
        VD_CUDA(cudaEventSynchronize(c.ev1));
        float ms = 0;
        VD_CUDA(cudaEventElapsedTime(&ms, c.ev0, c.ev1));
        c.stats.cells_ms = ms;
    }
    c.map_stride = map_stride;
    c.n_maps = nt;
    for (int i = 0; i < kTypes; ++i) c.map_slot[i] = -1;
    for (int j = 0; j < nt; ++j) c.map_slot[needed[j]] = j;
    return VD_OK;
}

vd_status vd_set_grid_shape(vd_ctx* h, int32_t shape) {
    VD_CHECK(h && shape >= 0 && shape <= 2, VD_ERR_ARG, "vd_set_grid_shape: shape must be 0, 1 or 2");
    h->c.grid_shape_fixed = shape;
    return VD_OK;
}

vd_status vd_get_grid(vd_ctx* h, int32_t t, float* out) {
    VD_CHECK(h && out, VD_ERR_ARG, "vd_get_grid: NULL argument");
    Ctx& c = h->c;
    VD_CHECK(t >= 0 && t < kTypes && c.map_slot[t] >= 0, VD_ERR_ARG, "vd_get_grid: map not built");
    VD_CUDA(cudaSetDevice(c.device));
    const GridGeom& g = c.geom;
    const float* src = c.d_maps + size_t(c.map_slot[t]) * c.map_stride;
    VD_CUDA(cudaMemcpy2DAsync(out, size_t(g.n[0]) * sizeof(float), src, size_t(g.pitch) * sizeof(float),
                              size_t(g.n[0]) * sizeof(float), size_t(g.n[1]) * g.n[2], cudaMemcpyDeviceToHost,
                              c.stream));
    VD_CUDA(cudaStreamSynchronize(c.stream));
    return VD_OK;
}

}  // extern "C"
