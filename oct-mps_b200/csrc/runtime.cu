// C-ABI runtime: context, resident meshes, continuous batching of jobs.
//
// Replaces the reference's per-A-scan worker RunGPUi (src/main.cu:43-660).
// The reference allocates ~50 device buffers, uploads the whole mesh and
// frees everything again for every A-scan, then relaunches its kernel in
// 50,000-step slices polled from the host.  Here a mesh is uploaded once
// and stays resident until released; a job (one A-scan) owns only its tally
// block and its RNG lanes (shared between jobs with the same seed and lane
// count).
//
// Jobs go into a device-resident job table per precision.  A persistent
// launch works through the table's units (RNG lanes); a job submitted while
// the launch runs is appended to the table and taken up by the running
// kernel as its threads free up (continuous batching), so its work overlaps
// the work already on the GPU.  A kernel thread that finds no unit left
// keeps retrying for new jobs while any thread of its block has work and
// then for linger_us, and exits early only when the host drains the launch,
// so a stream of submissions keeps one launch at full width.  A launch whose threads have
// begun to leave may be down to a few of them; work arriving then also
// starts another launch over the same table (up to kMaxLaunches at once,
// each on its own stream), whose blocks take SM slots as the older launch's
// blocks leave.  A job is finished when all of its lanes have reported back,
// which can be well before the launch ends.  When every unit of the table
// has been handed out and every launch has ended, the table is reset for the
// next batch; jobs arriving while the table is full wait for that.
//
// Nothing on the submit path runs a kernel (device buffers are filled by
// copies, not memsets): a kernel queued behind a persistent launch that holds
// every SM would wait for that launch to end.
//
// Device memory released while a launch runs is freed only once no launch
// runs (deferred frees).  A running launch may hold lines of that memory in
// its SMs' L1 caches, which are not coherent; were the memory handed to a
// new job's buffers in the same launch, its threads could read the stale
// lines instead of the new job's data.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cfloat>
#include <cstdio>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "kernel_iface.h"
#include "octmps_host.h"
#include "region_consts.h"

using namespace octmps;

namespace {

constexpr int kTableSlots = 4096;       // jobs per table between resets
constexpr int kMaxLaunches = 4;         // launches in flight per table
constexpr double kRefreshMs = 0.2;      // slot states are read back at most this often
constexpr int kDefaultLingerUs = 2000;  // idle kernel threads wait this long for new jobs
constexpr size_t kCtrlBytes = 256;      // control words, then the incident record at word 8
static_assert(8 * sizeof(unsigned long long) + sizeof(Incident) <= kCtrlBytes, "control area");

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

// One persistent launch of a table.
struct LaunchRec {
    cudaEvent_t start = nullptr, stop = nullptr;
    bool ended = false;
    float ms = 0;
    int64_t seq = 0;
    int stream = 0;
    ~LaunchRec() {
        if (start) cudaEventDestroy(start);
        if (stop) cudaEventDestroy(stop);
    }
};

struct Job {
    octmps_job_id id = 0;
    octmps_mesh_id mesh = 0;
    octmps_sim sim;
    int precision = 0;
    int32_t root = 0;
    uint64_t n_photons = 0;
    uint64_t seed = 0;
    uint32_t n_lanes = 0;
    std::shared_ptr<RngDev> rng;
    void *regions = nullptr;   // RegionConst<T>[n_regions]
    void *tally = nullptr;     // tally block + 4 statistics words
    unsigned long long *stats = nullptr;
    PhotonRecordDev *records = nullptr;  // RecordPhotonsFlag records, in the tally buffer
    uint64_t record_cap = 0;
    size_t tally_bytes = 0;
    int slot = -1;             // slot in its table, -1 while waiting for one
    std::shared_ptr<LaunchRec> launch;  // launch that finished its last lane
    double t_submit = 0, t_done = 0;
    bool done = false;
    octmps_status status = OCTMPS_OK;
    JobDesc desc;
};

// Device job table of one precision.
struct Table {
    int prec = 0;
    cudaStream_t streams[kMaxLaunches] = {};
    JobDesc *d_jobs = nullptr;
    uint64_t *d_base = nullptr;            // [kTableSlots]
    unsigned long long *d_ctrl = nullptr;  // next, total, error; incident at word 8
    uint2 *d_state = nullptr;              // [kTableSlots] units finished, finishing launch
    uint2 *h_state = nullptr;              // pinned copy of d_state[0, n_used)
    unsigned long long *h_ctrl = nullptr;  // pinned copy of the control words
    double state_at = -1e30;               // host time of the last copy
    int n_used = 0;
    uint64_t total = 0;                    // units appended
    uint64_t total_at_launch = 0;          // total when the newest launch started
    uint64_t next = 0;                     // units handed out (exact while none runs)
    unsigned error = 0;                    // error word of this table's current batch
    std::vector<octmps_job_id> slot_job;
    std::deque<octmps_job_id> waiting;     // jobs waiting for a free slot
    void *splits[kMaxLaunches] = {};       // split copies of the pooled kernel, per stream
    std::vector<std::shared_ptr<LaunchRec>> running;  // launches in flight
    std::vector<std::shared_ptr<LaunchRec>> batch;    // launches since the last reset
    Incident last_incident{};              // kept across resets
    octmps_job_id incident_job = 0;
};

}  // namespace

struct octmps_ctx {
    int device = 0;
    int n_sm = 0;
    cudaStream_t stream = nullptr;  // uploads, downloads and table updates
    std::vector<uint32_t> multipliers;
    std::map<octmps_mesh_id, std::unique_ptr<MeshDev>> meshes;
    std::map<octmps_job_id, std::unique_ptr<Job>> jobs;
    std::map<std::pair<uint64_t, uint32_t>, std::shared_ptr<RngDev>> rng_cache;
    std::unique_ptr<Table> tables[3];
    octmps_mesh_id next_mesh = 1;
    octmps_job_id next_job = 1;
    int64_t launches = 0;
    octmps_launch_config cfg;
    uint64_t budget = 0;
    uint64_t in_use = 0;
    uint64_t record_capacity = 0;  // RecordPhotonsFlag records per job (0 = packets)
    std::string err;
    std::recursive_mutex mu;
    void *record_buf = nullptr;  // optional per-lane records of the next launch
    bool completion_queue = false;         // on after the first octmps_ctx_poll
    std::deque<octmps_job_id> completed;   // finished jobs not yet returned by a poll
    // pinned host bytes of value 0x00 / 0xff that device buffers are filled
    // from by copy; outgrown buffers are kept until the context is destroyed
    // (freeing pinned memory waits for the device)
    unsigned char *h_fill[2] = {nullptr, nullptr};
    size_t h_fill_cap[2] = {0, 0};
    std::vector<void *> h_fill_old;
    std::vector<void *> deferred;  // device buffers to free once no launch runs
    uint64_t deferred_bytes = 0;   // their share of the HBM budget
    JobDesc *h_desc = nullptr;   // pinned staging (1 slot)
    uint64_t *h_base = nullptr;  // pinned staging (2 words)
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

// Fills device bytes with 0x00 or 0xff (value 0 or 1) through the copy
// engine on the context stream; the caller synchronises the stream.
octmps_status fill_device(octmps_ctx *ctx, void *dst, int value, size_t bytes) {
    if (bytes == 0) return OCTMPS_OK;
    if (ctx->h_fill_cap[value] < bytes) {
        const size_t cap = std::max<size_t>(bytes, 1 << 20);
        void *p = nullptr;
        CK(cudaMallocHost(&p, cap), "pinned fill buffer");
        memset(p, value ? 0xff : 0x00, cap);
        if (ctx->h_fill[value]) ctx->h_fill_old.push_back(ctx->h_fill[value]);
        ctx->h_fill[value] = static_cast<unsigned char *>(p);
        ctx->h_fill_cap[value] = cap;
    }
    CK(cudaMemcpyAsync(dst, ctx->h_fill[value], bytes, cudaMemcpyHostToDevice, ctx->stream),
       "device fill");
    return OCTMPS_OK;
}

#define FILL(dst, value, bytes)                                        \
    do {                                                               \
        octmps_status st_ = fill_device(ctx, (dst), (value), (bytes)); \
        if (st_ != OCTMPS_OK) return st_;                              \
    } while (0)

template <typename T>
void fill_regions(const octmps_sim &s, std::vector<unsigned char> &out) {
    std::vector<RegionConst<T>> r(s.n_regions);
    fill_region_consts<T>(s, r.data());
    out.resize(sizeof(RegionConst<T>) * r.size());
    memcpy(out.data(), r.data(), out.size());
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

octmps_status table_get(octmps_ctx *ctx, int prec, Table **out) {
    std::unique_ptr<Table> &T = ctx->tables[prec];
    if (!T) {
        std::unique_ptr<Table> t(new Table());
        t->prec = prec;
        for (auto &s : t->streams)
            CK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking), "stream");
        const size_t jb = sizeof(JobDesc) * kTableSlots;
        const size_t bb = sizeof(uint64_t) * kTableSlots;
        const size_t sb = sizeof(uint2) * kTableSlots;
        char *p = nullptr;
        CK(cudaMalloc((void **)&p, jb + bb + kCtrlBytes + sb), "job table");
        t->d_jobs = reinterpret_cast<JobDesc *>(p);
        t->d_base = reinterpret_cast<uint64_t *>(p + jb);
        t->d_ctrl = reinterpret_cast<unsigned long long *>(p + jb + bb);
        t->d_state = reinterpret_cast<uint2 *>(p + jb + bb + kCtrlBytes);
        CK(cudaMallocHost(&t->h_state, sb), "job table");
        CK(cudaMallocHost(&t->h_ctrl, kCtrlBytes), "job table");
        FILL(t->d_base, 1, bb);
        FILL(t->d_ctrl, 0, kCtrlBytes + sb);
        CK(cudaStreamSynchronize(ctx->stream), "job table");
        T = std::move(t);
    }
    *out = T.get();
    return OCTMPS_OK;
}

// Collects the table's ended launches; after any has ended, reads back the
// control words (the next-unit counter is exact once none runs).
octmps_status table_poll(octmps_ctx *ctx, Table &T) {
    bool any = false;
    for (size_t i = 0; i < T.running.size();) {
        LaunchRec &L = *T.running[i];
        cudaError_t q = cudaEventQuery(L.stop);
        if (q == cudaErrorNotReady) {
            ++i;
            continue;
        }
        if (q != cudaSuccess) return cuda_fail(ctx, q, "photon kernel");
        cudaEventElapsedTime(&L.ms, L.start, L.stop);
        L.ended = true;
        T.running.erase(T.running.begin() + i);
        any = true;
    }
    if (!any) return OCTMPS_OK;
    CK(cudaMemcpyAsync(T.h_ctrl, T.d_ctrl, 3 * sizeof(unsigned long long),
                       cudaMemcpyDeviceToHost, ctx->stream),
       "control words");
    CK(cudaStreamSynchronize(ctx->stream), "control words");
    T.next = T.h_ctrl[0];
    T.error = (unsigned)T.h_ctrl[2];
    return OCTMPS_OK;
}

// Starts a launch over the table: when none runs and units are left (its
// threads first take the next units in order), or when units were appended
// since the newest launch started (its blocks claim units from the shared
// counter).
octmps_status table_launch(octmps_ctx *ctx, Table &T) {
    if (ctx->record_buf && !T.running.empty() && T.total > T.total_at_launch) {
        // a recording launch runs alone, so that its threads (and no others)
        // take the recorded job's units: wait for the running ones to end
        for (auto &r : T.running) CK(cudaEventSynchronize(r->stop), "launch");
        octmps_status st = table_poll(ctx, T);
        if (st != OCTMPS_OK) return st;
    }
    const bool fresh = T.running.empty();
    if (fresh ? T.next >= T.total
              : (T.total <= T.total_at_launch || (int)T.running.size() >= kMaxLaunches))
        return OCTMPS_OK;
    // The per-lane kernel (default): 2, 3 or 4 resident 256-thread blocks per
    // SM (register caps 128, 80, 64), 6, 7 or 8 of 128 threads (caps 80, 72,
    // 64) or 2 of 512 (cap 64); its FP64 form and recording variant only
    // 256 x 2.  The pooled kernel: 4, 5 or 6 resident 128-thread blocks (caps
    // 128, 96, 80), the FP64 form 2 or 3, the recording variant 2.
    const bool pooled = ctx->cfg.kernel_form == 1;
    int min_blocks;
    int lane_block = ctx->cfg.block_size > 0 ? ctx->cfg.block_size : kDefaultBlock;
    if (pooled) {
        const int want = ctx->cfg.blocks_per_sm;
        if (T.prec == kFP64) min_blocks = (want == 2 || want == 3) ? want : kDefaultPooledMinBlocksFP64;
        else min_blocks = (want >= 4 && want <= 6) ? want : kDefaultPooledMinBlocks;
        if (ctx->record_buf) min_blocks = 2;
    } else {
        min_blocks = ctx->cfg.blocks_per_sm > 0 ? ctx->cfg.blocks_per_sm
                     : lane_block == kDefaultBlock ? kDefaultMinBlocks
                     : lane_block == 128          ? 6
                                                  : 2;
        if (T.prec == kFP64 || ctx->record_buf) {
            lane_block = 256;
            min_blocks = 2;
        }
    }
    int regs = 0, per_sm = 0;
    int st = pooled ? pooled_kernel_attributes(T.prec, min_blocks, ctx->record_buf != nullptr, &regs,
                                               &per_sm)
                    : photon_kernel_attributes(T.prec, lane_block, min_blocks, &regs, &per_sm);
    if (st) return cuda_fail(ctx, (cudaError_t)st, "kernel attributes");
    if (per_sm < 1) per_sm = 1;
    if (pooled && per_sm > 6) per_sm = 6;  // the split-copy buffers hold 6 blocks per SM
    const int block = pooled ? kPooledBlock : lane_block;
    const uint64_t grid = (uint64_t)ctx->n_sm * per_sm;
    // units the launch's threads take first: one per thread (per-lane), two
    // per thread (pooled)
    const uint64_t threads = grid * block * (pooled ? kPooledPerThread : 1);
    int si = 0;
    while (si < kMaxLaunches) {
        bool used = false;
        for (auto &r : T.running) used |= r->stream == si;
        if (!used) break;
        ++si;
    }
    if (pooled && !T.splits[si]) {
        // sized for the largest grid of any pooled variant and form (6 blocks
        // per SM, FP64 split copies); the stream's launches reuse it
        CK(cudaMallocAsync(&T.splits[si], pooled_split_bytes(kFP64, ctx->n_sm * 6), ctx->stream),
           "split copies");
        CK(cudaStreamSynchronize(ctx->stream), "split copies");
    }
    LaunchArgs a;
    a.jobs = T.d_jobs;
    a.unit_base = T.d_base;
    a.n_slots = kTableSlots;
    a.ctrl = T.d_ctrl;
    a.slot_state = T.d_state;
    a.incident = reinterpret_cast<Incident *>(T.d_ctrl + 8);
    if (fresh) {
        // thread t takes unit next + t; the counter starts past them (no
        // launch runs, so the copy races with nothing)
        T.h_ctrl[0] = std::min<uint64_t>(T.total, T.next + threads);
        CK(cudaMemcpyAsync(T.d_ctrl, T.h_ctrl, sizeof(unsigned long long),
                           cudaMemcpyHostToDevice, ctx->stream),
           "control words");
        CK(cudaStreamSynchronize(ctx->stream), "control words");
        a.start_unit = T.next;
        a.initial_total = T.total;
    } else {
        a.start_unit = 0;
        a.initial_total = 0;
    }
    // A packet needs ~10^2-10^4 steps; a photon caught in degenerate
    // geometry (stepping s = 0 around an edge) is stopped and flagged.
    a.step_cap = 1ull << 26;
    a.scatter_share = ctx->cfg.scatter_share > 0 ? ctx->cfg.scatter_share : kDefaultScatterShare;
    a.linger_us = ctx->cfg.linger_us < 0    ? 0u
                  : ctx->cfg.linger_us == 0 ? (uint32_t)kDefaultLingerUs
                                            : (uint32_t)ctx->cfg.linger_us;
    auto L = std::make_shared<LaunchRec>();
    L->seq = ++ctx->launches;
    L->stream = si;
    a.launch_seq = (uint32_t)L->seq;
    a.record_slot = T.n_used - 1;
    cudaStream_t s = T.streams[si];
    CK(cudaEventCreate(&L->start), "event");
    CK(cudaEventCreate(&L->stop), "event");
    CK(cudaEventRecord(L->start, s), "event");
    st = pooled ? launch_pooled_kernel(T.prec, min_blocks, a, (int)grid, s, ctx->record_buf,
                                       T.splits[si])
                : launch_photon_kernel(T.prec, min_blocks, a, (int)grid, block, s, ctx->record_buf);
    if (st) return cuda_fail(ctx, (cudaError_t)st, "photon kernel launch");
    CK(cudaEventRecord(L->stop, s), "event");
    T.total_at_launch = T.total;
    T.running.push_back(L);
    T.batch.push_back(L);
    ctx->record_buf = nullptr;
    return OCTMPS_OK;
}

// Appends a job to a free slot: descriptor and unit base first, then the
// total that makes the kernel hand out its units.
octmps_status table_append(octmps_ctx *ctx, Table &T, Job &j) {
    const int slot = T.n_used++;
    j.slot = slot;
    if ((int)T.slot_job.size() <= slot) T.slot_job.resize(slot + 1);
    T.slot_job[slot] = j.id;
    memcpy(ctx->h_desc, &j.desc, sizeof(JobDesc));
    ctx->h_base[0] = T.total;
    T.total += j.n_lanes;
    ctx->h_base[1] = T.total;
    CK(cudaMemcpyAsync(T.d_jobs + slot, ctx->h_desc, sizeof(JobDesc), cudaMemcpyHostToDevice,
                       ctx->stream),
       "job table");
    CK(cudaMemcpyAsync(T.d_base + slot, ctx->h_base, sizeof(uint64_t), cudaMemcpyHostToDevice,
                       ctx->stream),
       "job table");
    CK(cudaMemcpyAsync(T.d_ctrl + 1, ctx->h_base + 1, sizeof(uint64_t), cudaMemcpyHostToDevice,
                       ctx->stream),
       "job table");
    CK(cudaStreamSynchronize(ctx->stream), "job table");
    return OCTMPS_OK;
}

void mark_done(octmps_ctx *ctx, Job &j) {
    j.done = true;
    j.t_done = now_ms();
    if (ctx->completion_queue) ctx->completed.push_back(j.id);
}

// Reads back every slot's state (units finished, finishing launch) and the
// error word, and marks the jobs whose lanes have all reported as done.
octmps_status table_refresh(octmps_ctx *ctx, Table &T) {
    if (T.n_used == 0) return OCTMPS_OK;
    CK(cudaMemcpyAsync(T.h_state, T.d_state, sizeof(uint2) * T.n_used, cudaMemcpyDeviceToHost,
                       ctx->stream),
       "job state");
    CK(cudaMemcpyAsync(T.h_ctrl + 3, T.d_ctrl + 2, sizeof(unsigned long long),
                       cudaMemcpyDeviceToHost, ctx->stream),
       "error word");
    CK(cudaStreamSynchronize(ctx->stream), "job state");
    T.state_at = now_ms();
    const unsigned err = (unsigned)T.h_ctrl[3];
    for (int s = 0; s < T.n_used; ++s) {
        auto it = ctx->jobs.find(T.slot_job[s]);
        if (it == ctx->jobs.end() || it->second->done) continue;
        Job &j = *it->second;
        const uint2 st = T.h_state[s];
        // the finishing launch stamps its number just after the last count
        if (st.x < j.n_lanes || st.y == 0) continue;
        mark_done(ctx, j);
        for (auto &L : T.batch)
            if (L->seq == (int64_t)st.y) j.launch = L;
        if (err) {
            j.status = OCTMPS_ERR_KERNEL;
            char msg[96];
            snprintf(msg, sizeof msg, "kernel error word 0x%x", err);
            ctx->err = msg;
        }
    }
    return OCTMPS_OK;
}

// A table whose launches have all ended with every unit handed out holds
// only finished jobs: they are marked done and the slots are freed.
octmps_status table_try_reset(octmps_ctx *ctx, Table &T) {
    if (!T.running.empty() || T.n_used == 0 || T.next < T.total) return OCTMPS_OK;
    octmps_status st = table_refresh(ctx, T);
    if (st != OCTMPS_OK) return st;
    for (int s = 0; s < T.n_used; ++s) {
        auto it = ctx->jobs.find(T.slot_job[s]);
        if (it == ctx->jobs.end()) continue;
        Job &j = *it->second;
        if (!j.done) {  // cannot happen unless the kernel lost units
            mark_done(ctx, j);
            j.status = OCTMPS_ERR_KERNEL;
            ctx->err = "job lanes missing at the end of the launches";
        }
        j.slot = -1;
    }
    // keep the incident record (if any) of the batch before clearing it
    Incident inc;
    CK(cudaMemcpyAsync(&inc, T.d_ctrl + 8, sizeof inc, cudaMemcpyDeviceToHost, ctx->stream),
       "incident");
    CK(cudaStreamSynchronize(ctx->stream), "incident");
    if (inc.flag) {
        T.last_incident = inc;
        T.incident_job = (int)inc.slot < T.n_used ? T.slot_job[inc.slot] : 0;
    }
    FILL(T.d_base, 1, sizeof(uint64_t) * T.n_used);
    FILL(T.d_state, 0, sizeof(uint2) * T.n_used);
    FILL(T.d_ctrl, 0, kCtrlBytes);
    CK(cudaStreamSynchronize(ctx->stream), "job table");
    T.n_used = 0;
    T.total = T.next = T.total_at_launch = 0;
    T.error = 0;
    T.slot_job.clear();
    T.batch.clear();
    // jobs that were waiting for a slot move in
    while (!T.waiting.empty() && T.n_used < kTableSlots) {
        auto it = ctx->jobs.find(T.waiting.front());
        T.waiting.pop_front();
        if (it == ctx->jobs.end()) continue;
        st = table_append(ctx, T, *it->second);
        if (st != OCTMPS_OK) return st;
    }
    return OCTMPS_OK;
}

// One scheduling round of a table: collect ended launches, free the table
// if drained, launch if work is waiting.
void free_deferred(octmps_ctx *ctx);

octmps_status table_step(octmps_ctx *ctx, Table &T) {
    octmps_status st = table_poll(ctx, T);
    if (st != OCTMPS_OK) return st;
    free_deferred(ctx);
    st = table_try_reset(ctx, T);
    if (st != OCTMPS_OK) return st;
    return table_launch(ctx, T);
}

// Whether a job has finished: all of its lanes reported (read back from the
// device while launches may still run).
octmps_status job_check(octmps_ctx *ctx, Job &j) {
    if (j.done) return OCTMPS_OK;
    Table &T = *ctx->tables[j.precision];
    octmps_status st = table_step(ctx, T);
    if (st != OCTMPS_OK || j.done || j.slot < 0) return st;
    if (now_ms() - T.state_at < kRefreshMs) return OCTMPS_OK;
    return table_refresh(ctx, T);
}

void defer_free(octmps_ctx *ctx, void *p, uint64_t budget_bytes) {
    if (!p) return;
    ctx->deferred.push_back(p);
    ctx->deferred_bytes += budget_bytes;
}

bool any_launch_running(octmps_ctx *ctx) {
    for (auto &t : ctx->tables)
        if (t && !t->running.empty()) return true;
    return false;
}

// Frees the deferred buffers once no launch runs.
void free_deferred(octmps_ctx *ctx) {
    if (ctx->deferred.empty() || any_launch_running(ctx)) return;
    for (void *p : ctx->deferred) cudaFreeAsync(p, ctx->stream);
    ctx->deferred.clear();
    ctx->deferred_bytes = 0;
}

void free_mesh_device(octmps_ctx *ctx, MeshDev &m) {
    defer_free(ctx, m.planes_f, 0);
    defer_free(ctx, m.planes_d, 0);
    defer_free(ctx, m.adj, 0);
    m.planes_f = m.planes_d = nullptr;
    m.adj = nullptr;
    free_deferred(ctx);
}

void release_job_device(octmps_ctx *ctx, Job *j) {
    defer_free(ctx, j->regions, 0);
    defer_free(ctx, j->tally, j->tally ? j->tally_bytes : 0);
    j->regions = nullptr;
    j->tally = nullptr;
    j->stats = nullptr;
    j->records = nullptr;
    if (ctx->in_use >= j->tally_bytes) ctx->in_use -= j->tally_bytes;
    if (j->rng) {
        if (--j->rng->refs == 0) {
            for (auto it = ctx->rng_cache.begin(); it != ctx->rng_cache.end(); ++it)
                if (it->second == j->rng) {
                    ctx->rng_cache.erase(it);
                    break;
                }
            if (j->rng.use_count() <= 1) {
                const uint64_t rb = (uint64_t)j->rng->n_lanes * 36;
                defer_free(ctx, j->rng->x, rb);
                ctx->in_use = ctx->in_use >= rb ? ctx->in_use - rb : 0;
            }
        }
        j->rng.reset();
    }
    auto mi = ctx->meshes.find(j->mesh);
    if (mi != ctx->meshes.end()) {
        MeshDev &m = *mi->second;
        if (--m.refs == 0 && m.released) {
            free_mesh_device(ctx, m);
            ctx->meshes.erase(mi);
        }
    }
    free_deferred(ctx);
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
    if (cudaMallocHost(&c->h_desc, sizeof(JobDesc)) != cudaSuccess ||
        cudaMallocHost(&c->h_base, 2 * sizeof(uint64_t)) != cudaSuccess)
        return OCTMPS_ERR_OOM;
    size_t fr = 0, tot = 0;
    cudaMemGetInfo(&fr, &tot);
    c->budget = (uint64_t)(0.8 * (double)fr);
    // Job buffers come from the device's stream-ordered pool.  Memory freed
    // there stays mapped (no release threshold): handing it back to the
    // driver at each synchronisation would unmap pages while a launch runs,
    // which stalls the launch; the pool is bounded by the HBM budget anyway.
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
        uint64_t keep = UINT64_MAX;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
    *out = c.release();
    return OCTMPS_OK;
}

octmps_status octmps_ctx_destroy(octmps_ctx *ctx) {
    if (!ctx) return OCTMPS_ERR_INVALID_ARG;
    {
        std::lock_guard<std::recursive_mutex> g(ctx->mu);
        cudaSetDevice(ctx->device);
        for (auto &t : ctx->tables)
            if (t)
                for (auto s : t->streams) cudaStreamSynchronize(s);
        cudaStreamSynchronize(ctx->stream);
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
        for (void *p : ctx->deferred) cudaFreeAsync(p, ctx->stream);  // every launch has ended
        ctx->deferred.clear();
        cudaStreamSynchronize(ctx->stream);
        for (auto &t : ctx->tables)
            if (t) {
                t->running.clear();
                t->batch.clear();
                cudaFree(t->d_jobs);
                for (void *p : t->splits)
                    if (p) cudaFree(p);
                cudaFreeHost(t->h_state);
                cudaFreeHost(t->h_ctrl);
                for (auto s : t->streams) cudaStreamDestroy(s);
                t.reset();
            }
        cudaStreamDestroy(ctx->stream);
        cudaFreeHost(ctx->h_desc);
        cudaFreeHost(ctx->h_base);
        for (void *p : ctx->h_fill)
            if (p) cudaFreeHost(p);
        for (void *p : ctx->h_fill_old) cudaFreeHost(p);
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
    if (cfg->kernel_form < 0 || cfg->kernel_form > 1)
        return fail(ctx, OCTMPS_ERR_INVALID_ARG, "kernel_form must be 0 (per-lane) or 1 (pooled)");
    if (cfg->kernel_form == 1) {
        if (cfg->block_size != 0 && cfg->block_size != kPooledBlock)
            return fail(ctx, OCTMPS_ERR_INVALID_ARG, "block_size must be 0 or 128 (pooled kernel)");
        if (cfg->blocks_per_sm != 0 && (cfg->blocks_per_sm < 2 || cfg->blocks_per_sm > 6))
            return fail(ctx, OCTMPS_ERR_INVALID_ARG, "blocks_per_sm must be 0 or 2..6 (pooled kernel)");
    } else {
        const int b = cfg->block_size > 0 ? cfg->block_size : kDefaultBlock;
        const int m = cfg->blocks_per_sm > 0 ? cfg->blocks_per_sm
                      : b == kDefaultBlock ? kDefaultMinBlocks
                      : b == 128          ? 6
                                          : 2;
        // the mixed form's variants (the FP32 form has the same ones; the
        // FP64 form always runs 256 x 2)
        if (cfg->block_size < 0 || cfg->blocks_per_sm < 0 || !photon_kernel_variant(kMixed, b, m))
            return fail(ctx, OCTMPS_ERR_INVALID_ARG,
                        "per-lane kernel: block_size x blocks_per_sm must be 256 x 2..4, "
                        "128 x 6..8 or 512 x 2 (0 = default)");
    }
    if (cfg->scatter_share < 0 || cfg->scatter_share > 32)
        return fail(ctx, OCTMPS_ERR_INVALID_ARG, "scatter_share must be 0..32");
    if (cfg->linger_us < -1 || cfg->linger_us > 1000000)
        return fail(ctx, OCTMPS_ERR_INVALID_ARG, "linger_us must be -1..1000000");
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
        free_mesh_device(ctx, *it->second);
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
    Table *T = nullptr;
    {
        octmps_status st = table_get(ctx, job->precision, &T);
        if (st != OCTMPS_OK) return st;
    }
    if (job->precision == OCTMPS_PREC_FP64) {
        octmps_status st = ensure_planes_d(ctx, m);
        if (st != OCTMPS_OK) return st;
    }

    std::unique_ptr<Job> j(new Job());
    j->id = ctx->next_job++;
    j->mesh = job->mesh;
    j->sim = s;
    j->precision = job->precision;
    j->root = job->root_tet;
    j->n_photons = n_ph;
    j->seed = seed;
    j->n_lanes = lanes;
    j->t_submit = now_ms();

    const size_t psize = job->precision == OCTMPS_PREC_FP32 ? sizeof(float) : sizeof(double);
    const TallyLayout TL = tally_layout(s.num_optical_depth_length_steps, psize);
    const size_t stats_off = TL.bytes;
    // RecordPhotonsFlag: a record buffer after the statistics words (detections
    // are at most about one per packet; more are counted, not kept)
    const uint64_t rec_cap =
        s.record_photons_flag
            ? std::min<uint64_t>(ctx->record_capacity ? ctx->record_capacity : n_ph, 0xffffffffull)
            : 0;
    const size_t rec_off = stats_off + kStatsWords * sizeof(unsigned long long);
    j->record_cap = rec_cap;
    j->tally_bytes = rec_off + rec_cap * sizeof(PhotonRecordDev);
    // RNG lanes: cached per (seed, lanes).
    auto key = std::make_pair(seed, lanes);
    auto ri = ctx->rng_cache.find(key);
    uint64_t need = j->tally_bytes;
    if (ri == ctx->rng_cache.end()) need += (uint64_t)lanes * 36;
    // memory released while a launch runs counts until no launch runs
    for (auto &t : ctx->tables)
        if (t) {
            octmps_status st = table_poll(ctx, *t);
            if (st != OCTMPS_OK) return st;
        }
    free_deferred(ctx);
    if (ctx->in_use + ctx->deferred_bytes + need > ctx->budget)
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
        ctx->in_use += (uint64_t)lanes * 36;
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
    FILL(j->tally, 0, rec_off);  // tally and statistics; records are written before read
    CK(cudaStreamSynchronize(ctx->stream), "job upload");
    j->stats = reinterpret_cast<unsigned long long *>((char *)j->tally + stats_off);
    j->records = rec_cap ? reinterpret_cast<PhotonRecordDev *>((char *)j->tally + rec_off) : nullptr;
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
    D.n_regions = s.n_regions;
    D.record_cap = (uint32_t)j->record_cap;
    D.photon_records = j->records;
    D.type_bias = s.type_bias;
    D.nbins = s.num_optical_depth_length_steps;

    Job &jr = *j;
    *out = j->id;
    ctx->jobs[j->id] = std::move(j);
    // Into the table now (a running launch takes it up), or into the queue
    // of jobs waiting for a slot.
    octmps_status st = table_poll(ctx, *T);
    if (st == OCTMPS_OK) st = table_try_reset(ctx, *T);
    if (st != OCTMPS_OK) return st;
    if (T->n_used < kTableSlots && T->waiting.empty()) return table_append(ctx, *T, jr);
    T->waiting.push_back(jr.id);
    return OCTMPS_OK;
}

octmps_status octmps_ctx_flush(octmps_ctx *ctx) {
    if (!ctx) return OCTMPS_ERR_INVALID_ARG;
    std::lock_guard<std::recursive_mutex> g(ctx->mu);
    cudaSetDevice(ctx->device);
    for (auto &t : ctx->tables) {
        if (!t) continue;
        octmps_status st = table_step(ctx, *t);
        if (st != OCTMPS_OK) return st;
    }
    return OCTMPS_OK;
}

octmps_status octmps_ctx_synchronize(octmps_ctx *ctx) {
    if (!ctx) return OCTMPS_ERR_INVALID_ARG;
    std::lock_guard<std::recursive_mutex> g(ctx->mu);
    cudaSetDevice(ctx->device);
    for (auto &t : ctx->tables) {
        if (!t) continue;
        octmps_status st = table_step(ctx, *t);
        if (st != OCTMPS_OK) return st;
        if (t->running.empty()) continue;
        // idle threads exit at once instead of lingering (drain word)
        FILL(t->d_ctrl + 3, 1, sizeof(unsigned long long));
        CK(cudaStreamSynchronize(ctx->stream), "drain");
        // a launch that ends with units left (jobs appended as its threads
        // were leaving) is followed by another, which this waits for too
        while (st == OCTMPS_OK && !t->running.empty()) {
            CK(cudaEventSynchronize(t->running.front()->stop), "launch");
            st = table_step(ctx, *t);
        }
        if (st != OCTMPS_OK) return st;
        FILL(t->d_ctrl + 3, 0, sizeof(unsigned long long));
        CK(cudaStreamSynchronize(ctx->stream), "drain");
    }
    return OCTMPS_OK;
}

octmps_status octmps_ctx_poll(octmps_ctx *ctx, octmps_job_id *done, int32_t max_ids,
                              int32_t *n_done) {
    if (!ctx || !n_done || max_ids < 0 || (max_ids > 0 && !done)) return OCTMPS_ERR_INVALID_ARG;
    std::lock_guard<std::recursive_mutex> g(ctx->mu);
    cudaSetDevice(ctx->device);
    *n_done = 0;
    if (!ctx->completion_queue) {
        // jobs that finished before the first poll are reported too
        ctx->completion_queue = true;
        for (auto &kv : ctx->jobs)
            if (kv.second->done) ctx->completed.push_back(kv.first);
    }
    for (auto &t : ctx->tables) {
        if (!t) continue;
        octmps_status st = table_step(ctx, *t);
        if (st == OCTMPS_OK && t->n_used > 0 && now_ms() - t->state_at >= kRefreshMs)
            st = table_refresh(ctx, *t);
        if (st != OCTMPS_OK) return st;
    }
    while (*n_done < max_ids && !ctx->completed.empty()) {
        const octmps_job_id id = ctx->completed.front();
        ctx->completed.pop_front();
        if (ctx->jobs.count(id)) done[(*n_done)++] = id;
    }
    return OCTMPS_OK;
}

octmps_status octmps_debug_incident(octmps_ctx *ctx, int32_t precision, octmps_incident *out) {
    if (!ctx || !out || precision < 0 || precision > 2) return OCTMPS_ERR_INVALID_ARG;
    std::lock_guard<std::recursive_mutex> g(ctx->mu);
    cudaSetDevice(ctx->device);
    memset(out, 0, sizeof *out);
    Table *T = ctx->tables[precision].get();
    if (!T) return OCTMPS_OK;
    Incident inc;
    CK(cudaMemcpyAsync(&inc, T->d_ctrl + 8, sizeof inc, cudaMemcpyDeviceToHost, ctx->stream),
       "incident");
    CK(cudaStreamSynchronize(ctx->stream), "incident");
    octmps_job_id jid = 0;
    if (inc.flag) {
        jid = (int)inc.slot < T->n_used ? T->slot_job[inc.slot] : 0;
    } else {
        inc = T->last_incident;  // from a batch already reset
        jid = T->incident_job;
    }
    if (!inc.flag) return OCTMPS_OK;
    out->stopped = (int32_t)inc.flag;
    out->job = jid;
    auto it = ctx->jobs.find(jid);
    if (it != ctx->jobs.end()) {
        out->seed = it->second->seed;
        out->n_lanes = it->second->n_lanes;
        out->n_photons = it->second->n_photons;
    }
    out->lane = inc.lane;
    out->packets_left = inc.packets_left;
    out->steps = inc.steps;
    out->tet = inc.tet;
    for (int k = 0; k < 3; ++k) {
        out->pos[k] = inc.pos[k];
        out->dir[k] = inc.dir[k];
    }
    out->weight = inc.w;
    out->step_left = inc.sleft;
    return OCTMPS_OK;
}

// Test hook: per-lane records of the first packets of the most recently
// submitted job, run by the next launch, which waits for the table's running
// launches to end first (device buffer of n_lanes records, 80 bytes each).
octmps_status octmps_debug_record_next_launch(octmps_ctx *ctx, void *device_records) {
    if (!ctx) return OCTMPS_ERR_INVALID_ARG;
    std::lock_guard<std::recursive_mutex> g(ctx->mu);
    ctx->record_buf = device_records;
    return OCTMPS_OK;
}

octmps_status octmps_job_wait(octmps_ctx *ctx, octmps_job_id id, int32_t timeout_ms) {
    if (!ctx) return OCTMPS_ERR_INVALID_ARG;
    const double t0 = now_ms();
    for (;;) {
        {
            std::lock_guard<std::recursive_mutex> g(ctx->mu);
            cudaSetDevice(ctx->device);
            auto it = ctx->jobs.find(id);
            if (it == ctx->jobs.end()) return fail(ctx, OCTMPS_ERR_NOT_FOUND, "unknown job id");
            Job &j = *it->second;
            octmps_status st = job_check(ctx, j);
            if (st != OCTMPS_OK) return st;
            if (j.done) return j.status;
        }
        if (timeout_ms >= 0 && now_ms() - t0 > timeout_ms)
            return fail(ctx, OCTMPS_ERR_TIMEOUT, "job not finished within the timeout");
        std::this_thread::sleep_for(std::chrono::microseconds(100));
    }
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
    out->num_nonfinite = tot[3];
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
    out->stopped = s[3];
    // device time of the launch the job finished in, once that launch has
    // ended (a job can finish well before the launch does; this never waits)
    out->device_ms = -1.0;
    out->launch_id = 0;
    if (j->launch) {
        if (!j->launch->ended && cudaEventQuery(j->launch->stop) == cudaSuccess) {
            cudaEventElapsedTime(&j->launch->ms, j->launch->start, j->launch->stop);
            j->launch->ended = true;
        }
        if (j->launch->ended) out->device_ms = j->launch->ms;
        out->launch_id = j->launch->seq;
    }
    out->submit_to_done_ms = j->t_done - j->t_submit;
    return st;
}

octmps_status octmps_ctx_set_photon_record_capacity(octmps_ctx *ctx, uint64_t capacity) {
    if (!ctx || capacity > 0xffffffffull) return OCTMPS_ERR_INVALID_ARG;
    std::lock_guard<std::recursive_mutex> g(ctx->mu);
    ctx->record_capacity = capacity;
    return OCTMPS_OK;
}

octmps_status octmps_job_photon_records(octmps_ctx *ctx, octmps_job_id id,
                                        octmps_photon_record *out, uint64_t max,
                                        uint64_t *n_kept, uint64_t *n_detected) {
    static_assert(sizeof(octmps_photon_record) == sizeof(PhotonRecordDev),
                  "record layouts differ");
    if (!ctx || !n_kept || !n_detected || (max && !out)) return OCTMPS_ERR_INVALID_ARG;
    octmps_status st = octmps_job_wait(ctx, id, -1);
    if (st != OCTMPS_OK) return st;
    std::lock_guard<std::recursive_mutex> g(ctx->mu);
    Job *j = ctx->jobs[id].get();
    if (!j->stats) return fail(ctx, OCTMPS_ERR_NOT_FOUND, "job already released");
    unsigned long long s[kStatsWords];
    CK(cudaMemcpyAsync(s, j->stats, sizeof s, cudaMemcpyDeviceToHost, ctx->stream), "stats");
    CK(cudaStreamSynchronize(ctx->stream), "stats");
    *n_detected = j->records ? s[4] : 0;
    *n_kept = std::min<uint64_t>(*n_detected, j->record_cap);
    const uint64_t n = std::min<uint64_t>(*n_kept, max);
    if (n) {
        CK(cudaMemcpyAsync(out, j->records, n * sizeof(PhotonRecordDev), cudaMemcpyDeviceToHost,
                           ctx->stream),
           "records");
        CK(cudaStreamSynchronize(ctx->stream), "records");
    }
    return OCTMPS_OK;
}

octmps_status octmps_job_release(octmps_ctx *ctx, octmps_job_id id) {
    if (!ctx) return OCTMPS_ERR_INVALID_ARG;
    std::lock_guard<std::recursive_mutex> g(ctx->mu);
    auto it = ctx->jobs.find(id);
    if (it == ctx->jobs.end()) return OCTMPS_ERR_NOT_FOUND;
    Job *j = it->second.get();
    if (!j->done) {
        // A job in the table runs to its end (its device buffers are in use);
        // one still waiting for a slot is simply dropped.
        Table &T = *ctx->tables[j->precision];
        auto w = std::find(T.waiting.begin(), T.waiting.end(), id);
        if (w != T.waiting.end()) {
            T.waiting.erase(w);
        } else {
            octmps_status st = octmps_job_wait(ctx, id, -1);
            if (st != OCTMPS_OK && st != OCTMPS_ERR_KERNEL) return st;
        }
    }
    // The job's buffers may still be named by its table slot until the table
    // resets, but the kernel no longer touches them once every lane of the
    // job has reported (its last writes are fenced before the report), so
    // they are freed without waiting for the launch to end.
    release_job_device(ctx, j);
    ctx->jobs.erase(it);
    return OCTMPS_OK;
}

}  // extern "C"
