// C-ABI runtime: context, resident meshes, job queue, persistent launches.
//
// Replaces the reference's per-A-scan worker RunGPUi (src/main.cu:43-660).
// The reference allocates ~50 device buffers, uploads the whole mesh and
// frees everything again for every A-scan, then relaunches its kernel in
// 50,000-step slices polled from the host.  Here a mesh is uploaded once
// and stays resident until released; a job (one A-scan) owns only its
// tally block and its RNG lanes (shared between jobs with the same seed and
// lane count); every job queued when a launch starts runs in that one
// persistent launch, which ends when the last packet of the last job ends.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cfloat>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "kernel_iface.h"
#include "octmps_host.h"

using namespace octmps;

namespace {

// Resident blocks per SM the default kernel variant is compiled for, and the
// share of a warp's live lanes (in 32nds) that must wait for the scattering
// half of their step before the warp runs it; both the best of a sweep on
// the B-scan workload (2 blocks: 128-register cap, no spills).
constexpr int kDefaultMinBlocks = 2;
constexpr int kDefaultScatterShare = 16;

double now_ms() {
    return std::chrono::duration<double, std::milli>(
               std::chrono::steady_clock::now().time_since_epoch())
        .count();
}

struct MeshDev {
    int32_t n_tets = 0;
    std::vector<int32_t> region;  // host copy: region of each tet
    int32_t max_region = 0;
    void *planes_f = nullptr;      // float4[4*n_tets]
    void *planes_d = nullptr;      // double[16*n_tets], built on first FP64 job
    int32_t *adj = nullptr;        // int4[n_tets] packed
    std::vector<double> planes_host;  // signed planes in double, for the FP64 build
    int refs = 0;                  // jobs in flight using it
    bool released = false;
};

struct RngDev {
    uint64_t *x = nullptr, *xR = nullptr, *xS = nullptr;
    uint32_t *a = nullptr, *aR = nullptr, *aS = nullptr;
    uint32_t n_lanes = 0;
    int refs = 0;
};

struct Launch;

struct Job {
    octmps_job_id id = 0;
    octmps_mesh_id mesh = 0;
    octmps_sim sim;
    int precision = 0;
    double probe[3] = {0, 0, 0};
    int32_t root = 0;
    uint64_t n_photons = 0;
    uint64_t seed = 0;
    uint32_t n_lanes = 0;
    std::shared_ptr<RngDev> rng;
    void *regions = nullptr;   // RegionConst<T>[n_regions]
    void *tally = nullptr;     // tally block
    unsigned long long *stats = nullptr;
    size_t tally_bytes = 0;
    std::shared_ptr<Launch> launch;
    double t_submit = 0, t_done = 0;
    bool done = false;
    octmps_status status = OCTMPS_OK;
    JobDesc desc;
};

struct Launch {
    void *buf = nullptr;  // jobs, unit_base, counter, error word
    cudaEvent_t start = nullptr, stop = nullptr;
    bool complete = false;
    unsigned int error = 0;
    float ms = 0;
    unsigned int *error_host = nullptr;  // pinned
};

}  // namespace

struct octmps_ctx {
    int device = 0;
    int n_sm = 0;
    cudaStream_t stream = nullptr;
    std::vector<uint32_t> multipliers;
    std::map<octmps_mesh_id, std::unique_ptr<MeshDev>> meshes;
    std::map<octmps_job_id, std::unique_ptr<Job>> jobs;
    std::map<std::pair<uint64_t, uint32_t>, std::shared_ptr<RngDev>> rng_cache;
    std::vector<octmps_job_id> pending;
    octmps_mesh_id next_mesh = 1;
    octmps_job_id next_job = 1;
    octmps_launch_config cfg;
    uint64_t budget = 0;
    uint64_t in_use = 0;
    std::string err;
    std::recursive_mutex mu;
    void *record_buf = nullptr;  // optional per-lane records of the next launch
};

namespace {

octmps_status fail(octmps_ctx *c, octmps_status st, const std::string &msg) {
    if (c) c->err = msg;
    return st;
}

octmps_status cuda_fail(octmps_ctx *c, cudaError_t e, const char *what) {
    return fail(c, e == cudaErrorMemoryAllocation ? OCTMPS_ERR_OOM : OCTMPS_ERR_DEVICE,
                std::string(what) + ": " + cudaGetErrorString(e));
}

#define CK(call, what)                                   \
    do {                                                 \
        cudaError_t e_ = (call);                         \
        if (e_ != cudaSuccess) return cuda_fail(ctx, e_, what); \
    } while (0)

template <typename T>
void fill_regions(const octmps_sim &s, std::vector<unsigned char> &out) {
    std::vector<RegionConst<T>> r(s.n_regions);
    for (int i = 0; i < s.n_regions; ++i) {
        // read_simulation_data (src/octmps_io.cpp:625-626) and
        // InitDeviceConstantMemory (src/octmps_kernel.cuh:204-214).
        const double mutr = (s.regions[i].mus == 0.0) ? DBL_MAX
                                                      : 1.0 / (s.regions[i].mua + s.regions[i].mus);
        r[i].n = (T)s.regions[i].n;
        r[i].muas = (T)(1.0 / mutr);
        r[i].rmuas = (T)mutr;
        r[i].mua_muas = (T)(s.regions[i].mua * mutr);
        r[i].g = (T)s.regions[i].g;
    }
    out.resize(sizeof(RegionConst<T>) * r.size());
    memcpy(out.data(), r.data(), out.size());
}

double div_rd(double a, double b) {
    double q = a / b;
    if (!std::isfinite(q) || q == 0.0) return q;
    double r = std::fma(-q, b, a);
    if (r != 0.0 && ((r < 0.0) == (b > 0.0))) q = std::nextafter(q, -INFINITY);
    return q;
}

octmps_status finish_launch(octmps_ctx *ctx, const std::shared_ptr<Launch> &L) {
    if (L->complete) return OCTMPS_OK;
    cudaError_t e = cudaEventSynchronize(L->stop);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "launch");
    cudaEventElapsedTime(&L->ms, L->start, L->stop);
    L->error = *L->error_host;
    L->complete = true;
    cudaFreeAsync(L->buf, ctx->stream);
    cudaFreeHost(L->error_host);
    L->error_host = nullptr;
    cudaEventDestroy(L->start);
    cudaEventDestroy(L->stop);
    return OCTMPS_OK;
}

octmps_status ensure_planes_d(octmps_ctx *ctx, MeshDev &m) {
    if (m.planes_d) return OCTMPS_OK;
    CK(cudaMallocAsync(&m.planes_d, m.planes_host.size() * sizeof(double), ctx->stream), "planes");
    CK(cudaMemcpyAsync(m.planes_d, m.planes_host.data(), m.planes_host.size() * sizeof(double),
                       cudaMemcpyHostToDevice, ctx->stream),
       "planes upload");
    CK(cudaStreamSynchronize(ctx->stream), "planes upload");
    return OCTMPS_OK;
}

octmps_status flush_locked(octmps_ctx *ctx) {
    if (ctx->pending.empty()) return OCTMPS_OK;
    // One launch per precision present in the queue.
    for (int prec = 0; prec < 3; ++prec) {
        std::vector<Job *> js;
        for (octmps_job_id id : ctx->pending) {
            Job *j = ctx->jobs[id].get();
            if (j->precision == prec) js.push_back(j);
        }
        if (js.empty()) continue;
        const int nj = (int)js.size();
        auto L = std::make_shared<Launch>();
        const size_t jobs_bytes = sizeof(JobDesc) * nj;
        const size_t base_off = (jobs_bytes + 15) & ~size_t(15);
        const size_t ctr_off = base_off + (((nj + 1) * sizeof(uint64_t) + 15) & ~size_t(15));
        const size_t total = ctr_off + 16;
        CK(cudaMallocAsync(&L->buf, total, ctx->stream), "launch buffer");
        std::vector<unsigned char> hb(total, 0);
        uint64_t *ub = reinterpret_cast<uint64_t *>(hb.data() + base_off);
        uint64_t units = 0;
        for (int k = 0; k < nj; ++k) {
            memcpy(hb.data() + sizeof(JobDesc) * k, &js[k]->desc, sizeof(JobDesc));
            ub[k] = units;
            units += js[k]->n_lanes;
        }
        ub[nj] = units;
        CK(cudaMemcpyAsync(L->buf, hb.data(), total, cudaMemcpyHostToDevice, ctx->stream),
           "launch upload");
        CK(cudaMallocHost(&L->error_host, sizeof(unsigned int)), "pinned");
        *L->error_host = 0;
        LaunchArgs a;
        a.jobs = reinterpret_cast<const JobDesc *>(L->buf);
        a.unit_base = reinterpret_cast<const uint64_t *>((char *)L->buf + base_off);
        a.n_jobs = nj;
        a.total_units = units;
        a.next_unit = reinterpret_cast<unsigned long long *>((char *)L->buf + ctr_off);
        a.error = reinterpret_cast<unsigned int *>((char *)L->buf + ctr_off + 8);
        // A packet needs ~10^2-10^4 steps; a photon caught in degenerate
        // geometry (stepping s = 0 around an edge) is stopped and flagged.
        a.step_cap = 1ull << 26;
        a.scatter_share = ctx->cfg.scatter_share > 0 ? ctx->cfg.scatter_share : kDefaultScatterShare;
        // Variant compiled for 2 or 3 resident blocks per SM (register cap
        // 128 or 80); the FP64 form has only the first.
        int min_blocks = ctx->cfg.blocks_per_sm == 2 || ctx->cfg.blocks_per_sm == 3
                             ? ctx->cfg.blocks_per_sm
                             : kDefaultMinBlocks;
        if (prec == kFP64 || ctx->record_buf) min_blocks = 2;
        int regs = 0, per_sm = 0;
        int st = photon_kernel_attributes(prec, 256, min_blocks, &regs, &per_sm);
        if (st) return cuda_fail(ctx, (cudaError_t)st, "kernel attributes");
        if (per_sm < 1) per_sm = 1;
        const uint64_t max_useful = (units + 255) / 256;
        int grid = ctx->n_sm * per_sm;
        if ((uint64_t)grid > max_useful) grid = (int)std::max<uint64_t>(1, max_useful);
        CK(cudaEventCreate(&L->start), "event");
        CK(cudaEventCreate(&L->stop), "event");
        CK(cudaEventRecord(L->start, ctx->stream), "event");
        st = launch_photon_kernel(prec, min_blocks, a, grid, 256, ctx->stream, ctx->record_buf);
        if (st) return cuda_fail(ctx, (cudaError_t)st, "photon kernel launch");
        CK(cudaMemcpyAsync(L->error_host, a.error, sizeof(unsigned int), cudaMemcpyDeviceToHost,
                           ctx->stream),
           "error word");
        CK(cudaEventRecord(L->stop, ctx->stream), "event");
        for (Job *j : js) j->launch = L;
    }
    ctx->pending.clear();
    ctx->record_buf = nullptr;
    return OCTMPS_OK;
}

void release_job_device(octmps_ctx *ctx, Job *j) {
    if (j->regions) cudaFreeAsync(j->regions, ctx->stream);
    if (j->tally) cudaFreeAsync(j->tally, ctx->stream);
    j->regions = nullptr;
    j->tally = nullptr;
    j->stats = nullptr;
    if (ctx->in_use >= j->tally_bytes) ctx->in_use -= j->tally_bytes;
    if (j->rng) {
        if (--j->rng->refs == 0) {
            for (auto it = ctx->rng_cache.begin(); it != ctx->rng_cache.end(); ++it)
                if (it->second == j->rng) {
                    ctx->rng_cache.erase(it);
                    break;
                }
            if (j->rng.use_count() <= 1) {
                cudaFreeAsync(j->rng->x, ctx->stream);
            }
        }
        j->rng.reset();
    }
    auto mi = ctx->meshes.find(j->mesh);
    if (mi != ctx->meshes.end()) {
        MeshDev &m = *mi->second;
        if (--m.refs == 0 && m.released) {
            cudaFreeAsync(m.planes_f, ctx->stream);
            if (m.planes_d) cudaFreeAsync(m.planes_d, ctx->stream);
            cudaFreeAsync(m.adj, ctx->stream);
            ctx->meshes.erase(mi);
        }
    }
}

}  // namespace

extern "C" {

const char *octmps_status_string(octmps_status st) {
    switch (st) {
        case OCTMPS_OK: return "ok";
        case OCTMPS_ERR_INVALID_ARG: return "invalid argument";
        case OCTMPS_ERR_OOM: return "out of memory";
        case OCTMPS_ERR_DEVICE: return "CUDA device error";
        case OCTMPS_ERR_TIMEOUT: return "timeout";
        case OCTMPS_ERR_NOT_FOUND: return "not found";
        case OCTMPS_ERR_IO: return "file I/O error";
        case OCTMPS_ERR_NO_DEVICE: return "no usable CUDA device";
        case OCTMPS_ERR_BUDGET: return "HBM budget exceeded";
        case OCTMPS_ERR_KERNEL: return "kernel reported an error";
    }
    return "unknown status";
}

const char *octmps_last_error(const octmps_ctx *ctx) { return ctx ? ctx->err.c_str() : ""; }

octmps_status octmps_ctx_create(int device, octmps_ctx **out) {
    if (!out) return OCTMPS_ERR_INVALID_ARG;
    *out = nullptr;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n <= device || device < 0)
        return OCTMPS_ERR_NO_DEVICE;
    cudaDeviceProp p;
    if (cudaGetDeviceProperties(&p, device) != cudaSuccess) return OCTMPS_ERR_NO_DEVICE;
    if (p.major < 10) return OCTMPS_ERR_NO_DEVICE;  // built for sm_100a only
    std::unique_ptr<octmps_ctx> c(new octmps_ctx());
    c->device = device;
    c->n_sm = p.multiProcessorCount;
    memset(&c->cfg, 0, sizeof c->cfg);
    if (cudaSetDevice(device) != cudaSuccess) return OCTMPS_ERR_DEVICE;
    if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess)
        return OCTMPS_ERR_DEVICE;
    size_t fr = 0, tot = 0;
    cudaMemGetInfo(&fr, &tot);
    c->budget = (uint64_t)(0.8 * (double)fr);
    *out = c.release();
    return OCTMPS_OK;
}

octmps_status octmps_ctx_destroy(octmps_ctx *ctx) {
    if (!ctx) return OCTMPS_ERR_INVALID_ARG;
    {
        std::lock_guard<std::recursive_mutex> g(ctx->mu);
        cudaSetDevice(ctx->device);
        cudaStreamSynchronize(ctx->stream);
        for (auto &kv : ctx->jobs) {
            Job *j = kv.second.get();
            if (j->launch) finish_launch(ctx, j->launch);
            j->launch.reset();
        }
        std::vector<octmps_job_id> ids;
        for (auto &kv : ctx->jobs) ids.push_back(kv.first);
        for (auto id : ids) release_job_device(ctx, ctx->jobs[id].get());
        ctx->jobs.clear();
        for (auto &kv : ctx->meshes) {
            cudaFreeAsync(kv.second->planes_f, ctx->stream);
            if (kv.second->planes_d) cudaFreeAsync(kv.second->planes_d, ctx->stream);
            cudaFreeAsync(kv.second->adj, ctx->stream);
        }
        ctx->meshes.clear();
        cudaStreamSynchronize(ctx->stream);
        cudaStreamDestroy(ctx->stream);
    }
    delete ctx;
    return OCTMPS_OK;
}

octmps_status octmps_ctx_set_multipliers(octmps_ctx *ctx, const uint32_t *a, uint64_t count) {
    if (!ctx || !a || count < 6) return OCTMPS_ERR_INVALID_ARG;
    std::lock_guard<std::recursive_mutex> g(ctx->mu);
    ctx->multipliers.assign(a, a + count);
    return OCTMPS_OK;
}

octmps_status octmps_ctx_configure(octmps_ctx *ctx, const octmps_launch_config *cfg) {
    if (!ctx || !cfg) return OCTMPS_ERR_INVALID_ARG;
    std::lock_guard<std::recursive_mutex> g(ctx->mu);
    if (cfg->block_size != 0 && cfg->block_size != 256)
        return fail(ctx, OCTMPS_ERR_INVALID_ARG, "block_size must be 256");
    ctx->cfg = *cfg;
    if (cfg->hbm_budget_bytes) ctx->budget = cfg->hbm_budget_bytes;
    return OCTMPS_OK;
}

octmps_status octmps_mesh_upload(octmps_ctx *ctx, const octmps_mesh_desc *m, octmps_mesh_id *out) {
    if (!ctx || !m || !out || m->n_tets < 1 || m->n_faces < 1 || !m->tet_region || !m->tet_faces ||
        !m->tet_signs || !m->tet_adj || !m->face_plane)
        return OCTMPS_ERR_INVALID_ARG;
    std::lock_guard<std::recursive_mutex> g(ctx->mu);
    cudaSetDevice(ctx->device);
    if (m->n_tets >= kMaxTetsPacked)
        return fail(ctx, OCTMPS_ERR_INVALID_ARG, "mesh has too many tets (limit 2^24)");
    const int32_t T = m->n_tets;
    std::unique_ptr<MeshDev> d(new MeshDev());
    d->n_tets = T;
    d->region.assign(m->tet_region, m->tet_region + T);
    std::vector<float> pf((size_t)T * 16);
    d->planes_host.resize((size_t)T * 16);
    std::vector<int32_t> adj((size_t)T * 4);
    for (int32_t t = 0; t < T; ++t) {
        const int32_t r = m->tet_region[t];
        if (r < 0 || r >= OCTMPS_MAX_REGIONS)
            return fail(ctx, OCTMPS_ERR_INVALID_ARG, "tet region out of range");
        d->max_region = std::max(d->max_region, r);
        for (int k = 0; k < 4; ++k) {
            const int32_t f = m->tet_faces[4 * (size_t)t + k];
            const int32_t s = m->tet_signs[4 * (size_t)t + k];
            const int32_t n = m->tet_adj[4 * (size_t)t + k];
            if (f < 0 || f >= m->n_faces || (s != 1 && s != -1) || n < -1 || n >= T)
                return fail(ctx, OCTMPS_ERR_INVALID_ARG, "mesh face/sign/neighbour out of range");
            for (int c = 0; c < 4; ++c) {
                const double v = m->face_plane[4 * (size_t)f + c] * (double)s;
                d->planes_host[(size_t)t * 16 + 4 * k + c] = v;
                pf[(size_t)t * 16 + 4 * k + c] = (float)v;
            }
            adj[4 * (size_t)t + k] =
                n < 0 ? -1 : (int32_t)((uint32_t)n | ((uint32_t)m->tet_region[n] << kAdjIndexBits));
        }
    }
    CK(cudaMallocAsync(&d->planes_f, pf.size() * sizeof(float), ctx->stream), "mesh planes");
    CK(cudaMallocAsync((void **)&d->adj, adj.size() * sizeof(int32_t), ctx->stream), "mesh adjacency");
    CK(cudaMemcpyAsync(d->planes_f, pf.data(), pf.size() * sizeof(float), cudaMemcpyHostToDevice,
                       ctx->stream),
       "mesh upload");
    CK(cudaMemcpyAsync(d->adj, adj.data(), adj.size() * sizeof(int32_t), cudaMemcpyHostToDevice,
                       ctx->stream),
       "mesh upload");
    CK(cudaStreamSynchronize(ctx->stream), "mesh upload");
    const octmps_mesh_id id = ctx->next_mesh++;
    ctx->meshes[id] = std::move(d);
    *out = id;
    return OCTMPS_OK;
}

octmps_status octmps_mesh_release(octmps_ctx *ctx, octmps_mesh_id id) {
    if (!ctx) return OCTMPS_ERR_INVALID_ARG;
    std::lock_guard<std::recursive_mutex> g(ctx->mu);
    auto it = ctx->meshes.find(id);
    if (it == ctx->meshes.end() || it->second->released) return OCTMPS_ERR_NOT_FOUND;
    it->second->released = true;
    if (it->second->refs == 0) {
        cudaFreeAsync(it->second->planes_f, ctx->stream);
        if (it->second->planes_d) cudaFreeAsync(it->second->planes_d, ctx->stream);
        cudaFreeAsync(it->second->adj, ctx->stream);
        ctx->meshes.erase(it);
    }
    return OCTMPS_OK;
}

octmps_status octmps_job_submit(octmps_ctx *ctx, const octmps_job *job, octmps_job_id *out) {
    if (!ctx || !job || !job->sim || !out) return OCTMPS_ERR_INVALID_ARG;
    std::lock_guard<std::recursive_mutex> g(ctx->mu);
    cudaSetDevice(ctx->device);
    auto mi = ctx->meshes.find(job->mesh);
    if (mi == ctx->meshes.end() || mi->second->released)
        return fail(ctx, OCTMPS_ERR_NOT_FOUND, "unknown mesh id");
    MeshDev &m = *mi->second;
    const octmps_sim &s = *job->sim;
    if (job->precision < 0 || job->precision > 2)
        return fail(ctx, OCTMPS_ERR_INVALID_ARG, "precision must be 0, 1 or 2");
    if (s.n_regions < 2 || s.n_regions > OCTMPS_MAX_REGIONS || m.max_region >= s.n_regions)
        return fail(ctx, OCTMPS_ERR_INVALID_ARG, "mesh regions exceed the simulation's regions");
    if (s.num_optical_depth_length_steps < 1)
        return fail(ctx, OCTMPS_ERR_INVALID_ARG, "no depth bins");
    if (job->root_tet < 0 || job->root_tet >= m.n_tets)
        return fail(ctx, OCTMPS_ERR_INVALID_ARG, "root tet out of range");
    for (int i = 1; i < s.n_regions; ++i)
        if (s.regions[i].mus == 0.0 && job->precision != OCTMPS_PREC_FP64)
            return fail(ctx, OCTMPS_ERR_INVALID_ARG,
                        "a region with mus = 0 (glass) needs precision FP64");
    const uint64_t n_ph = job->n_photons ? job->n_photons : s.number_of_photons;
    if (n_ph == 0) return fail(ctx, OCTMPS_ERR_INVALID_ARG, "zero photons");
    uint32_t lanes = job->n_lanes;
    if (lanes == 0) {
        const uint64_t def = ctx->cfg.default_lanes > 0 ? (uint64_t)ctx->cfg.default_lanes : 88800ull;
        lanes = (uint32_t)std::min<uint64_t>(n_ph, def);
    }
    if ((uint64_t)lanes > n_ph) lanes = (uint32_t)n_ph;
    if (n_ph / lanes >= 0xffffffffull)
        return fail(ctx, OCTMPS_ERR_INVALID_ARG, "more than 2^32 packets per RNG lane");
    if (ctx->multipliers.size() < 3 + 3 * (uint64_t)lanes)
        return fail(ctx, OCTMPS_ERR_INVALID_ARG, "multiplier table too short for the lane count");
    const uint64_t seed = job->seed ? job->seed : 985456376ull;
    if (job->precision == OCTMPS_PREC_FP64) {
        octmps_status st = ensure_planes_d(ctx, m);
        if (st != OCTMPS_OK) return st;
    }

    std::unique_ptr<Job> j(new Job());
    j->id = ctx->next_job++;
    j->mesh = job->mesh;
    j->sim = s;
    j->precision = job->precision;
    j->probe[0] = job->probe_x;
    j->probe[1] = job->probe_y;
    j->probe[2] = job->probe_z;
    j->root = job->root_tet;
    j->n_photons = n_ph;
    j->seed = seed;
    j->n_lanes = lanes;
    j->t_submit = now_ms();

    const size_t psize = job->precision == OCTMPS_PREC_FP32 ? sizeof(float) : sizeof(double);
    const TallyLayout TL = tally_layout(s.num_optical_depth_length_steps, psize);
    const size_t stats_off = TL.bytes;
    j->tally_bytes = stats_off + 4 * sizeof(unsigned long long);
    // RNG lanes: cached per (seed, lanes).
    auto key = std::make_pair(seed, lanes);
    auto ri = ctx->rng_cache.find(key);
    uint64_t need = j->tally_bytes;
    if (ri == ctx->rng_cache.end()) need += (uint64_t)lanes * 36;
    if (ctx->in_use + need > ctx->budget)
        return fail(ctx, OCTMPS_ERR_BUDGET, "job does not fit the HBM budget");
    if (ri != ctx->rng_cache.end()) {
        j->rng = ri->second;
    } else {
        auto r = std::make_shared<RngDev>();
        r->n_lanes = lanes;
        std::vector<uint64_t> hx(lanes), hxR(lanes), hxS(lanes);
        std::vector<uint32_t> ha(lanes), haR(lanes), haS(lanes);
        octmps_rng_lanes rl{hx.data(), ha.data(), hxR.data(), haR.data(), hxS.data(), haS.data()};
        octmps_status st =
            octmps_rng_init(ctx->multipliers.data(), ctx->multipliers.size(), lanes, seed, &rl);
        if (st != OCTMPS_OK) return fail(ctx, st, "RNG seeding failed (invalid seed?)");
        void *buf = nullptr;
        const size_t n8 = (size_t)lanes * 8, n4 = (size_t)lanes * 4;
        CK(cudaMallocAsync(&buf, 3 * n8 + 3 * n4 + 64, ctx->stream), "rng lanes");
        char *b = (char *)buf;
        r->x = (uint64_t *)b;
        r->xR = (uint64_t *)(b + n8);
        r->xS = (uint64_t *)(b + 2 * n8);
        r->a = (uint32_t *)(b + 3 * n8);
        r->aR = (uint32_t *)(b + 3 * n8 + n4);
        r->aS = (uint32_t *)(b + 3 * n8 + 2 * n4);
        CK(cudaMemcpyAsync(r->x, hx.data(), n8, cudaMemcpyHostToDevice, ctx->stream), "rng");
        CK(cudaMemcpyAsync(r->xR, hxR.data(), n8, cudaMemcpyHostToDevice, ctx->stream), "rng");
        CK(cudaMemcpyAsync(r->xS, hxS.data(), n8, cudaMemcpyHostToDevice, ctx->stream), "rng");
        CK(cudaMemcpyAsync(r->a, ha.data(), n4, cudaMemcpyHostToDevice, ctx->stream), "rng");
        CK(cudaMemcpyAsync(r->aR, haR.data(), n4, cudaMemcpyHostToDevice, ctx->stream), "rng");
        CK(cudaMemcpyAsync(r->aS, haS.data(), n4, cudaMemcpyHostToDevice, ctx->stream), "rng");
        CK(cudaStreamSynchronize(ctx->stream), "rng upload");  // host vectors go out of scope
        ctx->rng_cache[key] = r;
        j->rng = r;
    }
    j->rng->refs++;

    std::vector<unsigned char> regions;
    if (job->precision == OCTMPS_PREC_FP64) fill_regions<double>(s, regions);
    else fill_regions<float>(s, regions);
    CK(cudaMallocAsync(&j->regions, regions.size(), ctx->stream), "regions");
    CK(cudaMemcpyAsync(j->regions, regions.data(), regions.size(), cudaMemcpyHostToDevice,
                       ctx->stream),
       "regions");
    CK(cudaMallocAsync(&j->tally, j->tally_bytes, ctx->stream), "tally");
    CK(cudaMemsetAsync(j->tally, 0, j->tally_bytes, ctx->stream), "tally");
    CK(cudaStreamSynchronize(ctx->stream), "job upload");
    j->stats = reinterpret_cast<unsigned long long *>((char *)j->tally + stats_off);
    ctx->in_use += j->tally_bytes;
    m.refs++;

    JobDesc &D = j->desc;
    memset(&D, 0, sizeof D);
    D.planes = job->precision == OCTMPS_PREC_FP64 ? m.planes_d : m.planes_f;
    D.adj = m.adj;
    D.regions = j->regions;
    D.rng_x = j->rng->x;
    D.rng_a = j->rng->a;
    D.rng_xR = j->rng->xR;
    D.rng_aR = j->rng->aR;
    D.rng_xS = j->rng->xS;
    D.rng_aS = j->rng->aS;
    D.tally = j->tally;
    D.stats = j->stats;
    D.n_photons = n_ph;
    D.n_lanes = lanes;
    D.n_tets = m.n_tets;
    D.probe_x = job->probe_x;
    D.probe_y = job->probe_y;
    D.probe_z = job->probe_z;
    const double n0 = s.regions[0].n, nr = s.regions[m.region[job->root_tet]].n;
    const double rs = (n0 - nr) / (n0 + nr);  // Rspecular, src/main.cu:29-37
    D.w0 = 1.0 - rs * rs;
    D.tdmin = s.target_depth_min;
    D.tdmax = s.target_depth_max;
    D.bias_a = s.backward_bias_coefficient;
    D.p_bias = s.probability_additional_bias;
    D.cos_collect = cos(s.max_collecting_angle_deg * 3.14159265359 / 180.0);
    D.radius = s.max_collecting_radius;
    D.rnd_step = s.rnd_step_size_in_tissue;
    D.n_ambient = s.regions[0].n;
    D.shift = s.optical_depth_shift;
    D.bin_width = div_rd(s.coherence_length_source, 6.0);
    D.half_lc = div_rd(s.coherence_length_source, 2.0);
    D.root_tet = job->root_tet;
    D.root_region = m.region[job->root_tet];
    D.type_bias = s.type_bias;
    D.nbins = s.num_optical_depth_length_steps;

    *out = j->id;
    ctx->pending.push_back(j->id);
    ctx->jobs[j->id] = std::move(j);
    return OCTMPS_OK;
}

octmps_status octmps_ctx_flush(octmps_ctx *ctx) {
    if (!ctx) return OCTMPS_ERR_INVALID_ARG;
    std::lock_guard<std::recursive_mutex> g(ctx->mu);
    cudaSetDevice(ctx->device);
    return flush_locked(ctx);
}

// Test hook: per-lane records of the first packets of the first job of the
// next launch (device buffer of n_lanes records, 80 bytes each).
octmps_status octmps_debug_record_next_launch(octmps_ctx *ctx, void *device_records) {
    if (!ctx) return OCTMPS_ERR_INVALID_ARG;
    std::lock_guard<std::recursive_mutex> g(ctx->mu);
    ctx->record_buf = device_records;
    return OCTMPS_OK;
}

octmps_status octmps_job_wait(octmps_ctx *ctx, octmps_job_id id, int32_t timeout_ms) {
    if (!ctx) return OCTMPS_ERR_INVALID_ARG;
    std::shared_ptr<Launch> L;
    {
        std::lock_guard<std::recursive_mutex> g(ctx->mu);
        cudaSetDevice(ctx->device);
        auto it = ctx->jobs.find(id);
        if (it == ctx->jobs.end()) return fail(ctx, OCTMPS_ERR_NOT_FOUND, "unknown job id");
        Job *j = it->second.get();
        if (j->done) return j->status;
        if (!j->launch) {
            octmps_status st = flush_locked(ctx);
            if (st != OCTMPS_OK) return st;
        }
        L = j->launch;
    }
    const double t0 = now_ms();
    for (;;) {
        cudaError_t q;
        {
            std::lock_guard<std::recursive_mutex> g(ctx->mu);
            if (L->complete) break;
            q = cudaEventQuery(L->stop);
            if (q == cudaSuccess) {
                octmps_status st = finish_launch(ctx, L);
                if (st != OCTMPS_OK) return st;
                break;
            }
            if (q != cudaErrorNotReady) return cuda_fail(ctx, q, "launch");
        }
        if (timeout_ms >= 0 && now_ms() - t0 > timeout_ms)
            return fail(ctx, OCTMPS_ERR_TIMEOUT, "job not finished within the timeout");
        std::this_thread::sleep_for(std::chrono::microseconds(200));
    }
    std::lock_guard<std::recursive_mutex> g(ctx->mu);
    Job *j = ctx->jobs[id].get();
    if (!j->done) {
        j->done = true;
        j->t_done = now_ms();
        if (L->error) {
            j->status = OCTMPS_ERR_KERNEL;
            char msg[96];
            snprintf(msg, sizeof msg, "kernel error word 0x%x", L->error);
            ctx->err = msg;
        }
    }
    return j->status;
}

octmps_status octmps_job_fetch(octmps_ctx *ctx, octmps_job_id id, octmps_tally *out) {
    if (!ctx || !out) return OCTMPS_ERR_INVALID_ARG;
    octmps_status st = octmps_job_wait(ctx, id, -1);
    if (st != OCTMPS_OK) return st;
    std::lock_guard<std::recursive_mutex> g(ctx->mu);
    Job *j = ctx->jobs[id].get();
    if (!j->tally) return fail(ctx, OCTMPS_ERR_NOT_FOUND, "job already released");
    std::vector<unsigned char> h(j->tally_bytes);
    CK(cudaMemcpyAsync(h.data(), j->tally, j->tally_bytes, cudaMemcpyDeviceToHost, ctx->stream),
       "tally download");
    CK(cudaStreamSynchronize(ctx->stream), "tally download");
    const int nb = j->sim.num_optical_depth_length_steps;
    const bool f32 = j->precision == OCTMPS_PREC_FP32;
    const TallyLayout TL = tally_layout(nb, f32 ? sizeof(float) : sizeof(double));
    const uint64_t *tot = reinterpret_cast<const uint64_t *>(h.data() + TL.totals);
    out->num_filtered = tot[0];
    out->num_filtered_class1 = tot[1];
    out->num_filtered_class2 = tot[2];
    auto copy_u = [&](uint64_t *dst, size_t off) {
        if (dst) memcpy(dst, h.data() + off, (nb + 1) * sizeof(uint64_t));
    };
    auto copy_p = [&](double *dst, size_t off) {
        if (!dst) return;
        for (int i = 0; i < nb + 2; ++i) {
            if (f32) {
                float v;
                memcpy(&v, h.data() + off + 4 * i, 4);
                dst[i] = v;
            } else {
                memcpy(&dst[i], h.data() + off + 8 * i, 8);
            }
        }
    };
    copy_u(out->count1, TL.count1);
    copy_u(out->count2, TL.count2);
    copy_p(out->sum1, TL.sum1);
    copy_p(out->sumsq1, TL.sumsq1);
    copy_p(out->max1, TL.max1);
    copy_p(out->sum2, TL.sum2);
    copy_p(out->sumsq2, TL.sumsq2);
    copy_p(out->max2, TL.max2);
    return OCTMPS_OK;
}

octmps_status octmps_job_fetch_stats(octmps_ctx *ctx, octmps_job_id id, octmps_job_stats *out) {
    if (!ctx || !out) return OCTMPS_ERR_INVALID_ARG;
    octmps_status st = octmps_job_wait(ctx, id, -1);
    if (st != OCTMPS_OK && st != OCTMPS_ERR_KERNEL) return st;
    std::lock_guard<std::recursive_mutex> g(ctx->mu);
    Job *j = ctx->jobs[id].get();
    if (!j->stats) return fail(ctx, OCTMPS_ERR_NOT_FOUND, "job already released");
    unsigned long long s[4];
    CK(cudaMemcpyAsync(s, j->stats, sizeof s, cudaMemcpyDeviceToHost, ctx->stream), "stats");
    CK(cudaStreamSynchronize(ctx->stream), "stats");
    out->steps = s[0];
    out->restores = s[1];
    out->packets = s[2];
    out->device_ms = j->launch ? j->launch->ms : 0.0;
    out->submit_to_done_ms = j->t_done - j->t_submit;
    return st;
}

octmps_status octmps_job_release(octmps_ctx *ctx, octmps_job_id id) {
    if (!ctx) return OCTMPS_ERR_INVALID_ARG;
    std::lock_guard<std::recursive_mutex> g(ctx->mu);
    auto it = ctx->jobs.find(id);
    if (it == ctx->jobs.end()) return OCTMPS_ERR_NOT_FOUND;
    Job *j = it->second.get();
    if (!j->launch) {
        // still queued: drop it from the queue
        ctx->pending.erase(std::remove(ctx->pending.begin(), ctx->pending.end(), id),
                           ctx->pending.end());
    } else if (!j->launch->complete) {
        octmps_status st = finish_launch(ctx, j->launch);
        if (st != OCTMPS_OK) return st;
    }
    release_job_device(ctx, j);
    ctx->jobs.erase(it);
    return OCTMPS_OK;
}

}  // extern "C"
