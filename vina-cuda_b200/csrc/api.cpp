// Context lifetime, errors, scoring tables, receptor and box set-up.
#include <algorithm>
#include <cmath>
#include <chrono>
#include <cstring>
#include <mutex>
#include <string>

#include "common.h"

namespace vd {

static thread_local std::string g_last_error;
void set_error(const std::string& msg) { g_last_error = msg; }

vd_status dev_alloc(Ctx& c, void** p, size_t bytes, const char* what) {
    *p = nullptr;
    if (c.dev_cap > 0 && c.dev_used + bytes > c.dev_cap) {
        set_error(std::string(what) + ": " + std::to_string(bytes) + " bytes would exceed the context's device memory cap (" +
                  std::to_string(c.dev_used) + " of " + std::to_string(c.dev_cap) + " in use)");
        return VD_ERR_NOMEM;
    }
    const cudaError_t e = cudaMalloc(p, std::max<size_t>(bytes, 1));
    if (e == cudaErrorMemoryAllocation) {
        cudaGetLastError();  // not sticky: clear it so the context stays usable
        *p = nullptr;
        set_error(std::string(what) + ": out of device memory for " + std::to_string(bytes) + " bytes");
        return VD_ERR_NOMEM;
    }
    if (e != cudaSuccess) {
        *p = nullptr;
        set_error(std::string(what) + ": cudaMalloc: " + cudaGetErrorString(e));
        return VD_ERR_CUDA;
    }
    c.dev_bytes[*p] = bytes;
    c.dev_used += bytes;
    return VD_OK;
}

void dev_free(Ctx& c, void* p) {
    if (!p) return;
    auto it = c.dev_bytes.find(p);
    if (it != c.dev_bytes.end()) {
        c.dev_used -= it->second;
        c.dev_bytes.erase(it);
    }
    cudaFree(p);
}

vd_status ensure_scratch(Ctx* c, size_t bytes) {
    if (c->scratch_bytes >= bytes) return VD_OK;
    dev_release(*c, c->d_scratch);
    c->scratch_bytes = 0;
    size_t want = bytes + bytes / 4;
    if (c->dev_cap > 0 && c->dev_used + want > c->dev_cap && c->dev_used + bytes <= c->dev_cap)
        want = bytes;  // under a cap, give up the growth headroom before failing
    vd_status st = dev_alloc(*c, &c->d_scratch, want, "scratch");
    if (st != VD_OK) return st;
    c->scratch_bytes = want;
    return VD_OK;
}

vd_status ensure_host_stage(Ctx* c, size_t bytes) {
    if (c->h_stage_bytes >= bytes) return VD_OK;
    if (c->h_stage) VD_CUDA(cudaFreeHost(c->h_stage));
    c->h_stage = nullptr;
    c->h_stage_bytes = 0;
    const size_t want = bytes + bytes / 4;
    VD_CUDA(cudaMallocHost(&c->h_stage, want));
    c->h_stage_bytes = want;
    return VD_OK;
}

}  // namespace vd

using namespace vd;

extern "C" {

const char* vd_last_error(void) { return g_last_error.c_str(); }

vd_status vd_create(vd_ctx** out, int device) {
    VD_CHECK(out != nullptr, VD_ERR_ARG, "vd_create: out is NULL");
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess || n == 0) {
        set_error(std::string("vd_create: no CUDA device: ") + cudaGetErrorString(e));
        return VD_ERR_CUDA;
    }
    VD_CHECK(device >= 0 && device < n, VD_ERR_ARG, "vd_create: device index out of range");
    VD_CUDA(cudaSetDevice(device));
    cudaDeviceProp prop;
    VD_CUDA(cudaGetDeviceProperties(&prop, device));
    if (prop.major < 10) {
        set_error("vd_create: this build targets sm_100a (B200); device is sm_" +
                  std::to_string(prop.major) + std::to_string(prop.minor));
        return VD_ERR_CUDA;
    }
    vd_ctx* h = new vd_ctx();
    Ctx& c = h->c;
    c.device = device;
    for (int i = 0; i < kTypes; ++i) c.map_slot[i] = -1;
    if (cudaStreamCreateWithFlags(&c.stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreate(&c.ev0) != cudaSuccess || cudaEventCreate(&c.ev1) != cudaSuccess ||
        cudaEventCreate(&c.ev2) != cudaSuccess ||
        cudaMalloc(&c.d_counter, 64 * sizeof(int32_t)) != cudaSuccess) {
        set_error("vd_create: stream/event/counter allocation failed");
        delete h;
        return VD_ERR_CUDA;
    }
    const double w[6] = {-0.035579, -0.005156, 0.840245, -0.035069, -0.587439, 5 * 0.05846 / 0.1 - 1};
    *out = h;
    return vd_set_scoring(h, w);
}

vd_status vd_destroy(vd_ctx* h) {
    if (!h) return VD_OK;
    Ctx& c = h->c;
    cudaSetDevice(c.device);
    cudaFree(c.d_fast);
    cudaFree(c.d_smooth);
    cudaFree(c.d_maps);
    cudaFree(c.d_cells);
    cudaFree(c.d_rec);
    cudaFree(c.d_recd);
    cudaFree(c.d_cell_start);
    cudaFree(c.d_cell_list);
    cudaFree(c.d_fastd);
    cudaFree(c.d_pool);
    cudaFree(c.d_scratch);
    cudaFree(c.d_counter);
    if (c.pipe_exec) cudaGraphExecDestroy(c.pipe_exec);
    if (c.h_stage) cudaFreeHost(c.h_stage);
    if (c.ev0) cudaEventDestroy(c.ev0);
    if (c.ev1) cudaEventDestroy(c.ev1);
    if (c.ev2) cudaEventDestroy(c.ev2);
    if (c.stream) cudaStreamDestroy(c.stream);
    delete h;
    return VD_OK;
}

vd_status vd_set_memory_cap(vd_ctx* h, int64_t bytes) {
    VD_CHECK(h && bytes >= 0, VD_ERR_ARG, "vd_set_memory_cap: bad arguments");
    h->c.dev_cap = size_t(bytes);
    return VD_OK;
}

vd_status vd_get_stats(vd_ctx* h, vd_stats* out) {
    VD_CHECK(h && out, VD_ERR_ARG, "vd_get_stats: NULL argument");
    h->c.stats.device_bytes = int64_t(h->c.dev_used);
    h->c.stats.pair_force_scale = h->c.fix_scale;
    h->c.stats.ligand_bytes = h->c.pool_words * int64_t(sizeof(float4));
    *out = h->c.stats;
    return VD_OK;
}

// After new tables: maps built with the old weights are stale.
static void scoring_changed(Ctx& c, std::chrono::steady_clock::time_point t0) {
    c.scoring = true;
    c.fix_scale = pair_force_scale(c.sd);
    c.n_maps = 0;
    for (int i = 0; i < kTypes; ++i) c.map_slot[i] = -1;
    c.stats.scoring_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
}

vd_status vd_set_scoring(vd_ctx* h, const double weights[6]) {
    VD_CHECK(h && weights, VD_ERR_ARG, "vd_set_scoring: NULL argument");
    for (int i = 0; i < 6; ++i) VD_CHECK(std::isfinite(weights[i]), VD_ERR_ARG, "vd_set_scoring: non-finite weight");
    Ctx& c = h->c;
    const auto t0 = std::chrono::steady_clock::now();
    VD_CUDA(cudaSetDevice(c.device));
    std::memcpy(c.weights, weights, sizeof(c.weights));
    build_tables(weights, c.fast, c.se, c.sd);
    std::vector<float> f(size_t(kPairTypes) * kBins);
    std::vector<float4> s(size_t(kPairTypes) * kBins);
    for (int p = 0; p < kPairTypes; ++p)
        for (int i = 0; i < kBins; ++i) {
            const size_t b = size_t(p) * kN;
            f[size_t(p) * kBins + i] = float(c.fast[b + i]);
            s[size_t(p) * kBins + i] = make_float4(float(c.se[b + i]), float(c.sd[b + i]),
                                                   float(c.se[b + i + 1]), float(c.sd[b + i + 1]));
        }
    vd_status st = VD_OK;
    if (!c.d_fast && (st = dev_alloc(c, &c.d_fast, f.size() * sizeof(float), "pair tables")) != VD_OK) return st;
    if (!c.d_smooth && (st = dev_alloc(c, &c.d_smooth, s.size() * sizeof(float4), "pair tables")) != VD_OK)
        return st;
    std::vector<double> fd(size_t(kPairTypes) * kBins);
    for (int p = 0; p < kPairTypes; ++p)
        for (int i = 0; i < kBins; ++i) fd[size_t(p) * kBins + i] = c.fast[size_t(p) * kN + i];
    if (!c.d_fastd && (st = dev_alloc(c, &c.d_fastd, fd.size() * sizeof(double), "pair tables")) != VD_OK)
        return st;
    VD_CUDA(cudaMemcpy(c.d_fastd, fd.data(), fd.size() * sizeof(double), cudaMemcpyHostToDevice));
    VD_CUDA(cudaMemcpy(c.d_fast, f.data(), f.size() * sizeof(float), cudaMemcpyHostToDevice));
    VD_CUDA(cudaMemcpy(c.d_smooth, s.data(), s.size() * sizeof(float4), cudaMemcpyHostToDevice));
    scoring_changed(c, t0);
    return VD_OK;
}

vd_status vd_set_scoring_device(vd_ctx* h, const double weights[6]) {
    VD_CHECK(h && weights, VD_ERR_ARG, "vd_set_scoring_device: NULL argument");
    for (int i = 0; i < 6; ++i)
        VD_CHECK(std::isfinite(weights[i]), VD_ERR_ARG, "vd_set_scoring_device: non-finite weight");
    Ctx& c = h->c;
    const auto t0 = std::chrono::steady_clock::now();
    VD_CUDA(cudaSetDevice(c.device));
    std::memcpy(c.weights, weights, sizeof(c.weights));
    vd_status st = build_tables_device(c, weights);
    if (st != VD_OK) return st;
    scoring_changed(c, t0);
    return VD_OK;
}

vd_status vd_get_tables(vd_ctx* h, double* fast, double* se, double* sd) {
    VD_CHECK(h, VD_ERR_ARG, "vd_get_tables: NULL context");
    const size_t n = size_t(kPairTypes) * kN * sizeof(double);
    if (fast) std::memcpy(fast, h->c.fast.data(), n);
    if (se) std::memcpy(se, h->c.se.data(), n);
    if (sd) std::memcpy(sd, h->c.sd.data(), n);
    return VD_OK;
}

vd_status vd_set_receptor(vd_ctx* h, int32_t n, const double* xyz, const int32_t* xs) {
    VD_CHECK(h && n >= 0 && (n == 0 || (xyz && xs)), VD_ERR_ARG, "vd_set_receptor: bad arguments");
    Ctx& c = h->c;
    for (int i = 0; i < n; ++i) {
        VD_CHECK(xs[i] >= -1 && xs[i] < kTypes, VD_ERR_ARG, "vd_set_receptor: XS type out of range");
        VD_CHECK(std::isfinite(xyz[3 * size_t(i)]) && std::isfinite(xyz[3 * size_t(i) + 1]) &&
                     std::isfinite(xyz[3 * size_t(i) + 2]),
                 VD_ERR_ARG, "vd_set_receptor: non-finite coordinate");
    }
    c.rec_xyz.assign(xyz, xyz + 3 * size_t(n));
    c.rec_xs.assign(xs, xs + n);
    c.n_maps = 0;
    for (int i = 0; i < kTypes; ++i) c.map_slot[i] = -1;
    c.rec_dev_ready = false;
    return VD_OK;
}

vd_status vd_set_box(vd_ctx* h, const double center[3], const double size[3]) {
    VD_CHECK(h && center && size, VD_ERR_ARG, "vd_set_box: NULL argument");
    Ctx& c = h->c;
    GridGeom& g = c.geom;
    for (int i = 0; i < 3; ++i) {
        VD_CHECK(size[i] > 0, VD_ERR_ARG, "vd_set_box: search space dimensions must be positive");
        VD_CHECK(std::isfinite(center[i]) && std::isfinite(size[i]), VD_ERR_ARG,
                 "vd_set_box: center and size must be finite");
        VD_CHECK(size[i] <= 1e5, VD_ERR_CAPACITY, "vd_set_box: box too large for one map (2^31 points)");
        const double granularity = 0.375;
        const int n = int(std::ceil(size[i] / granularity));
        const double real_span = granularity * n;
        g.begin[i] = center[i] - real_span / 2;
        g.end[i] = g.begin[i] + real_span;
        g.n[i] = n + 1;
        g.init[i] = g.begin[i];
        g.dmo[i] = g.n[i] - 1.0;
    }
    for (int i = 0; i < 3; ++i) {
        g.factor[i] = g.dmo[i] / (g.end[i] - g.begin[i]);
        g.finv[i] = 1 / g.factor[i];
    }
    g.pitch = (g.n[0] + 3) & ~3;
    VD_CHECK(size_t(g.pitch) * g.n[1] * g.n[2] < (size_t(1) << 31), VD_ERR_CAPACITY,
             "vd_set_box: box too large for one map (2^31 points)");
    c.has_box = true;
    c.n_maps = 0;
    for (int i = 0; i < kTypes; ++i) c.map_slot[i] = -1;
    c.rec_dev_ready = false;
    return VD_OK;
}

vd_status vd_grid_dims(vd_ctx* h, int32_t npts[3], double begin[3], double end[3]) {
    VD_CHECK(h && h->c.has_box, VD_ERR_ARG, "vd_grid_dims: no box set");
    for (int i = 0; i < 3; ++i) {
        if (npts) npts[i] = h->c.geom.n[i];
        if (begin) begin[i] = h->c.geom.begin[i];
        if (end) end[i] = h->c.geom.end[i];
    }
    return VD_OK;
}

}  // extern "C"
