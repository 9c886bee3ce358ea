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
// Launch: one CTA per tile of 16(x) x 8(y) x 8(z) points, 256 threads, each
// thread owning 4 consecutive x points so every map store is one 128-bit
// store.  The CTA stages, in shared memory, the receptor atoms whose brick
// distance to the tile is below the cutoff, taken from a 4 A cell list in
// deterministic (cell, index) order.
#include <algorithm>
#include <cmath>
#include <cstring>

#include "common.h"

namespace vd {
namespace {

constexpr int kTileX = 16, kTileY = 8, kTileZ = 8, kThreads = 256;
constexpr int kStageCap = 1280;   // atoms staged per chunk (40 KB)
constexpr double kCellSize = 4.0;

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
    const float* lut;             // [17][kBins][ntp]
    int32_t ntp;                  // lut row width (multiple of 8)
    int32_t col0;                 // first lut column of this group
    int32_t n_out;                // maps written by this group (<= NTG)
    const StagedAtom* atoms;      // relevant receptor atoms sorted by cell
    const int32_t* cell_start;    // [cells+1]
    double cell_org[3];
    int32_t cell_dim[3];
};

__device__ __forceinline__ double probe_coord(double init, double finv, int i) {
    return __dadd_rn(init, __dmul_rn(finv, double(i)));
}

template <int NTG>
__global__ void __launch_bounds__(kThreads) grid_build_kernel(GridParams p) {
    __shared__ StagedAtom s_atoms[kStageCap];
    __shared__ int32_t s_row_count[64];
    __shared__ int32_t s_row_off[65];
    __shared__ int32_t s_row_begin[64], s_row_end[64];

    const int t = threadIdx.x;
    const int xq = t & 3, ly = (t >> 2) & 7, lz = t >> 5;
    const int x0 = blockIdx.x * kTileX + xq * 4;
    const int y = blockIdx.y * kTileY + ly;
    const int z = blockIdx.z * kTileZ + lz;

    // Tile bounding box (double) and the cell rows covering it +- 8 A.
    const int tx_lo = blockIdx.x * kTileX, ty_lo = blockIdx.y * kTileY, tz_lo = blockIdx.z * kTileZ;
    const int tx_hi = min(tx_lo + kTileX - 1, p.n[0] - 1);
    const int ty_hi = min(ty_lo + kTileY - 1, p.n[1] - 1);
    const int tz_hi = min(tz_lo + kTileZ - 1, p.n[2] - 1);
    double lo[3] = {probe_coord(p.init[0], p.finv[0], tx_lo), probe_coord(p.init[1], p.finv[1], ty_lo),
                    probe_coord(p.init[2], p.finv[2], tz_lo)};
    double hi[3] = {probe_coord(p.init[0], p.finv[0], tx_hi), probe_coord(p.init[1], p.finv[1], ty_hi),
                    probe_coord(p.init[2], p.finv[2], tz_hi)};
    int c_lo[3], c_hi[3];
    for (int d = 0; d < 3; ++d) {
        c_lo[d] = max(0, int(floor((lo[d] - 8.0 - p.cell_org[d]) / kCellSize)));
        c_hi[d] = min(p.cell_dim[d] - 1, int(floor((hi[d] + 8.0 - p.cell_org[d]) / kCellSize)));
    }
    const int ry = max(0, c_hi[1] - c_lo[1] + 1), rz = max(0, c_hi[2] - c_lo[2] + 1);
    const int n_rows = ry * rz;  // <= 36 for the cell and tile sizes above
    if (t < n_rows) {
        const int cy = c_lo[1] + t % ry, cz = c_lo[2] + t / ry;
        const int base = p.cell_dim[0] * (cy + p.cell_dim[1] * cz);
        s_row_begin[t] = (c_lo[0] <= c_hi[0]) ? p.cell_start[base + c_lo[0]] : 0;
        s_row_end[t] = (c_lo[0] <= c_hi[0]) ? p.cell_start[base + c_hi[0] + 1] : 0;
    }
    __syncthreads();

    const int warp = t >> 5, lane = t & 31;
    auto keep = [&](const StagedAtom& a) {
        double d2 = 0;
        const double c[3] = {a.x, a.y, a.z};
        for (int d = 0; d < 3; ++d) {
            double q = c[d] < lo[d] ? lo[d] - c[d] : (c[d] > hi[d] ? c[d] - hi[d] : 0.0);
            d2 += q * q;
        }
        return d2 < 64.0 + 1e-6;  // conservative: the per-point test below is exact
    };
    // Pass 1: per-row counts of atoms near the tile.
    for (int r = warp; r < n_rows; r += kThreads / 32) {
        int cnt = 0;
        for (int i = s_row_begin[r]; i < s_row_end[r]; i += 32) {
            const bool k = (i + lane < s_row_end[r]) && keep(p.atoms[i + lane]);
            cnt += __popc(__ballot_sync(0xffffffffu, k));
        }
        if (lane == 0) s_row_count[r] = cnt;
    }
    __syncthreads();
    if (t == 0) {
        int acc = 0;
        for (int r = 0; r < n_rows; ++r) { s_row_off[r] = acc; acc += s_row_count[r]; }
        s_row_off[n_rows] = acc;
    }
    __syncthreads();
    const int total = s_row_off[n_rows];

    const bool active = (x0 < p.n[0]) && (y < p.n[1]) && (z < p.n[2]);
    double px[4];
    for (int k = 0; k < 4; ++k) px[k] = probe_coord(p.init[0], p.finv[0], x0 + k);
    const double py = probe_coord(p.init[1], p.finv[1], y);
    const double pz = probe_coord(p.init[2], p.finv[2], z);

    float acc[4][NTG];
#pragma unroll
    for (int k = 0; k < 4; ++k)
#pragma unroll
        for (int j = 0; j < NTG; ++j) acc[k][j] = 0.f;

    for (int chunk = 0; chunk < total; chunk += kStageCap) {
        // Pass 2: compact the atoms of this chunk into shared memory in order.
        for (int r = warp; r < n_rows; r += kThreads / 32) {
            int out = s_row_off[r];
            for (int i = s_row_begin[r]; i < s_row_end[r]; i += 32) {
                StagedAtom a;
                bool k = false;
                if (i + lane < s_row_end[r]) {
                    a = p.atoms[i + lane];
                    k = keep(a);
                }
                const unsigned m = __ballot_sync(0xffffffffu, k);
                const int slot = out + __popc(m & ((1u << lane) - 1u)) - chunk;
                if (k && slot >= 0 && slot < kStageCap) s_atoms[slot] = a;
                out += __popc(m);
            }
        }
        __syncthreads();
        const int n_here = min(kStageCap, total - chunk);
        if (active) {
            for (int a = 0; a < n_here; ++a) {
                const StagedAtom at = s_atoms[a];
                const double dy = __dsub_rn(at.y, py), dz = __dsub_rn(at.z, pz);
                const double dy2 = __dmul_rn(dy, dy), dz2 = __dmul_rn(dz, dz);
                if (__dadd_rn(dy2, dz2) > kCutoff2) continue;  // exact: sums are monotone
                const float* row_base = p.lut + size_t(at.type) * kBins * p.ntp + p.col0;
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    const double dx = __dsub_rn(at.x, px[k]);
                    const double r2 = __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), dy2), dz2);
                    if (r2 <= kCutoff2) {
                        const int bin = __double2int_rz(__dmul_rn(32.0, r2));
                        const float4* v = reinterpret_cast<const float4*>(row_base + size_t(bin) * p.ntp);
#pragma unroll
                        for (int j = 0; j < NTG / 4; ++j) {
                            const float4 q = __ldg(v + j);
                            acc[k][4 * j + 0] += q.x;
                            acc[k][4 * j + 1] += q.y;
                            acc[k][4 * j + 2] += q.z;
                            acc[k][4 * j + 3] += q.w;
                        }
                    }
                }
            }
        }
        __syncthreads();
    }
    if (!active) return;
    const size_t off = (size_t(z) * p.n[1] + y) * p.pitch + x0;
#pragma unroll
    for (int j = 0; j < NTG; ++j) {
        if (j >= p.n_out) break;
        float4 v = make_float4(acc[0][j], acc[1][j], acc[2][j], acc[3][j]);
        *reinterpret_cast<float4*>(p.maps + size_t(j) * p.map_stride + off) = v;
    }
}

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
    const int ntp = (nt + 7) & ~7;

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
    const int n_cells = cd[0] * cd[1] * cd[2];
    std::vector<int32_t> start(n_cells + 1, 0);
    for (int ce : cell_of) start[ce + 1]++;
    for (int i = 0; i < n_cells; ++i) start[i + 1] += start[i];
    std::vector<StagedAtom> sorted(rel.size());
    {
        std::vector<int32_t> fill(start.begin(), start.end() - 1);
        for (size_t i = 0; i < rel.size(); ++i) sorted[fill[cell_of[i]]++] = rel[i];
    }
    // Table slice [17][kBins][ntp] for the needed ligand types.
    std::vector<float> lut(size_t(kTypes) * kBins * ntp, 0.f);
    for (int tr = 0; tr < kTypes; ++tr)
        for (int j = 0; j < nt; ++j) {
            const size_t b = size_t(tri_index(tr, needed[j])) * kN;
            for (int i = 0; i < kBins; ++i) lut[(size_t(tr) * kBins + i) * ntp + j] = float(c.fast[b + i]);
        }

    const size_t map_stride = size_t(g.pitch) * g.n[1] * g.n[2];
    const size_t bytes_maps = map_stride * nt * sizeof(float);
    const size_t bytes_atoms = std::max<size_t>(1, sorted.size()) * sizeof(StagedAtom);
    const size_t bytes_start = start.size() * sizeof(int32_t);
    const size_t bytes_lut = lut.size() * sizeof(float);
    if (c.d_maps) VD_CUDA(cudaFree(c.d_maps));
    c.d_maps = nullptr;
    VD_CUDA(cudaMalloc(&c.d_maps, bytes_maps));
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
    p.lut = d_lut;
    p.ntp = ntp;
    p.atoms = d_atoms;
    p.cell_start = d_start;
    dim3 grid((g.n[0] + kTileX - 1) / kTileX, (g.n[1] + kTileY - 1) / kTileY, (g.n[2] + kTileZ - 1) / kTileZ);
    VD_CUDA(cudaEventRecord(c.ev0, c.stream));
    for (int g0 = 0; g0 < nt; g0 += 8) {
        p.maps = c.d_maps + size_t(g0) * map_stride;
        p.col0 = g0;
        p.n_out = std::min(8, nt - g0);
        if (nt - g0 <= 4) grid_build_kernel<4><<<grid, kThreads, 0, c.stream>>>(p);
        else grid_build_kernel<8><<<grid, kThreads, 0, c.stream>>>(p);
        VD_CUDA(cudaGetLastError());
    }
    VD_CUDA(cudaEventRecord(c.ev1, c.stream));
    VD_CUDA(cudaStreamSynchronize(c.stream));
    float ms = 0;
    VD_CUDA(cudaEventElapsedTime(&ms, c.ev0, c.ev1));
    c.stats.grid_ms = ms;
    c.map_stride = map_stride;
    c.n_maps = nt;
    for (int i = 0; i < kTypes; ++i) c.map_slot[i] = -1;
    for (int j = 0; j < nt; ++j) c.map_slot[needed[j]] = j;
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
