// A-scan entry point that allocates no memory.
//
// Some callers of this library cannot call cudaMalloc: an application that
// hands the library a fixed device arena at start-up and forbids any other
// allocation (real-time or certified pipelines, or a host framework whose own
// caching allocator owns all of device memory), or a caller running inside a
// section where a device allocation could stall behind other work.  For them
// this file runs one A-scan through the same photon kernel as
// octmps_job_submit, with everything the kernel needs beyond the caller's
// inputs and outputs (job descriptor, work-unit table, work counter, error
// word, statistics, region constants) placed in one file-scope device array
// of fixed size instead of in allocated memory.
//
// That array exists once per GPU that loads the library and stays allocated
// until the process exits.  Every call on a device shares it and it keeps
// the previous call's contents; the call rewrites all of it before the launch.
// Two calls whose work overlaps on the GPU (different streams, or calls from
// several host threads) race on it: serialise them.
#include <cuda_runtime.h>

#include <cmath>
#include <cfloat>
#include <cstring>
#include <mutex>

#include "kernel_iface.h"
#include "octmps_host.h"
#include "region_consts.h"

using namespace octmps;

namespace {

// Scratch layout inside the array (offsets in bytes).
constexpr size_t kJobOff = 0;                                        // JobDesc
constexpr size_t kUnitOff = 512;                                     // uint64 unit_base[2]
constexpr size_t kCtrlOff = 544;     // u64 next unit, total units, error word
constexpr size_t kStatsOff = 576;                                    // u64 stats[4]
constexpr size_t kRegionOff = 640;                                   // RegionConst<float>[...]
constexpr size_t kScratchBytes = kRegionOff + OCTMPS_NOALLOC_MAX_REGIONS * sizeof(RegionConst<float>);

static_assert(sizeof(JobDesc) <= kUnitOff - kJobOff, "job descriptor does not fit its slot");
static_assert(kScratchBytes == OCTMPS_NOALLOC_SCRATCH_BYTES, "scratch size differs from the header");

__device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
unsigned char *g_scratch_addr[kMaxDevices] = {nullptr};

// Device address of the scratch array on the current device (looked up once
// per device; the host-side symbol is not a device address).  The address is
// kept for the life of the process: after cudaDeviceReset (or anything else
// that replaces the device's primary context) it is stale, and calls on that
// device are not supported.
cudaError_t scratch_address(int device, unsigned char **out) {
    std::lock_guard<std::mutex> g(g_mu);
    if (!g_scratch_addr[device]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return e;
        g_scratch_addr[device] = static_cast<unsigned char *>(p);
    }
    *out = g_scratch_addr[device];
    return cudaSuccess;
}

// The caller's neighbour entries, checked on the device before any photon
// follows them: each is -1 (ambient) or names a tet below n_tets and a
// region in [1, n_regions).  A bad entry sets kErrBadNeighbour in the
// scratch error word.
__global__ void validate_adj(const int32_t *adj, int64_t n, int32_t n_tets, int32_t n_regions,
                             unsigned int *err) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int32_t e = adj[i];
        if (e == -1) continue;
        const uint32_t idx = (uint32_t)e & kAdjIndexMask;
        const uint32_t reg = (uint32_t)e >> kAdjIndexBits;
        if (idx >= (uint32_t)n_tets || reg < 1u || reg >= (uint32_t)n_regions)
            atomicOr(err, kErrBadNeighbour);
    }
}

}  // namespace

static_assert(OCTMPS_NOALLOC_TALLY_BYTES(600) == 32 + 2 * 4816 + 6 * 4816,
              "tally size formula");

extern "C" octmps_status octmps_ascan_run_noalloc(const octmps_noalloc_ascan *a, void *stream) {
    if (!a || !a->sim || !a->planes || !a->adj || !a->rng_x || !a->rng_a || !a->rng_xR ||
        !a->rng_aR || !a->rng_xS || !a->rng_aS || !a->tally)
        return OCTMPS_ERR_INVALID_ARG;
    const octmps_sim &s = *a->sim;
    if (s.n_regions < 2 || s.n_regions > OCTMPS_NOALLOC_MAX_REGIONS)
        return OCTMPS_ERR_INVALID_ARG;  // the region table must fit the fixed scratch
    if (a->n_tets < 1 || a->n_tets >= kMaxTetsPacked || a->root_tet < 0 ||
        a->root_tet >= a->n_tets || a->root_region < 1 || a->root_region >= s.n_regions ||
        a->n_lanes == 0 || a->n_photons < a->n_lanes || s.num_optical_depth_length_steps < 1)
        return OCTMPS_ERR_INVALID_ARG;
    for (int i = 1; i < s.n_regions; ++i)
        if (s.regions[i].mus == 0.0) return OCTMPS_ERR_INVALID_ARG;  // glass needs FP64

    int device = 0;
    if (cudaGetDevice(&device) != cudaSuccess || device < 0 || device >= kMaxDevices)
        return OCTMPS_ERR_NO_DEVICE;
    unsigned char *scratch = nullptr;
    if (scratch_address(device, &scratch) != cudaSuccess) return OCTMPS_ERR_DEVICE;
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);

    // Host image of the scratch area (stack memory; no allocation).
    unsigned char img[kScratchBytes];
    memset(img, 0, sizeof img);
    // the region constants as octmps_job_submit derives them (region_consts.h)
    fill_region_consts<float>(s, reinterpret_cast<RegionConst<float> *>(img + kRegionOff));
    JobDesc D;
    memset(&D, 0, sizeof D);
    D.planes = a->planes;
    D.adj = a->adj;
    D.regions = scratch + kRegionOff;
    D.rng_x = const_cast<uint64_t *>(a->rng_x);
    D.rng_a = const_cast<uint32_t *>(a->rng_a);
    D.rng_xR = const_cast<uint64_t *>(a->rng_xR);
    D.rng_aR = const_cast<uint32_t *>(a->rng_aR);
    D.rng_xS = const_cast<uint64_t *>(a->rng_xS);
    D.rng_aS = const_cast<uint32_t *>(a->rng_aS);
    D.tally = a->tally;
    D.stats = reinterpret_cast<unsigned long long *>(scratch + kStatsOff);
    D.n_photons = a->n_photons;
    D.n_lanes = a->n_lanes;
    D.n_tets = a->n_tets;
    D.probe_x = a->probe_x;
    D.probe_y = a->probe_y;
    D.probe_z = a->probe_z;
    const double n0 = s.regions[0].n, nr = s.regions[a->root_region].n;
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
    D.root_tet = a->root_tet;
    D.root_region = a->root_region;
    D.n_regions = s.n_regions;
    D.type_bias = s.type_bias;
    D.nbins = s.num_optical_depth_length_steps;
    memcpy(img + kJobOff, &D, sizeof D);
    uint64_t *ub = reinterpret_cast<uint64_t *>(img + kUnitOff);
    ub[0] = 0;
    ub[1] = a->n_lanes;
    int sms = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess)
        return OCTMPS_ERR_DEVICE;
    int regs = 0, per_sm = 0;
    if (photon_kernel_attributes(kMixed, 256, kDefaultMinBlocks, &regs, &per_sm) != 0 || per_sm < 1)
        per_sm = 1;
    uint64_t grid = (uint64_t)sms * per_sm;
    const uint64_t useful = (a->n_lanes + 255) / 256;
    if (grid > useful) grid = useful;
    // thread t runs unit t first; the counter starts past those units
    uint64_t *ctrl = reinterpret_cast<uint64_t *>(img + kCtrlOff);
    ctrl[0] = grid * 256 < a->n_lanes ? grid * 256 : a->n_lanes;
    ctrl[1] = a->n_lanes;
    // error word and statistics start at zero (img is zeroed)

    if (cudaMemcpyAsync(scratch, img, sizeof img, cudaMemcpyHostToDevice, st) != cudaSuccess)
        return OCTMPS_ERR_DEVICE;
    if (tally_layout(D.nbins, sizeof(double)).bytes != OCTMPS_NOALLOC_TALLY_BYTES(D.nbins))
        return OCTMPS_ERR_INVALID_ARG;
    if (cudaMemsetAsync(a->tally, 0, OCTMPS_NOALLOC_TALLY_BYTES(D.nbins), st) != cudaSuccess)
        return OCTMPS_ERR_DEVICE;
    unsigned int *err_word = reinterpret_cast<unsigned int *>(scratch + kCtrlOff + 16);
    {
        const int64_t n = 4 * (int64_t)a->n_tets;
        const int64_t blocks = (n + 255) / 256 < (int64_t)sms * 4 ? (n + 255) / 256 : (int64_t)sms * 4;
        validate_adj<<<(unsigned)blocks, 256, 0, st>>>(a->adj, n, a->n_tets, s.n_regions, err_word);
        unsigned int bad = 0;
        if (cudaGetLastError() != cudaSuccess ||
            cudaMemcpyAsync(&bad, err_word, sizeof bad, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
            cudaStreamSynchronize(st) != cudaSuccess)
            return OCTMPS_ERR_DEVICE;
        if (bad) return OCTMPS_ERR_INVALID_ARG;  // a neighbour entry names no tet or region
    }
    LaunchArgs L;
    L.jobs = reinterpret_cast<const JobDesc *>(scratch + kJobOff);
    L.unit_base = reinterpret_cast<const uint64_t *>(scratch + kUnitOff);
    L.n_slots = 1;
    L.ctrl = reinterpret_cast<unsigned long long *>(scratch + kCtrlOff);
    L.slot_state = nullptr;
    L.incident = nullptr;
    L.start_unit = 0;
    L.initial_total = a->n_lanes;
    L.step_cap = 1ull << 26;
    L.scatter_share = kDefaultScatterShare;
    L.launch_seq = 1;
    L.record_slot = -1;
    L.linger_us = 0;
    if (launch_photon_kernel(kMixed, kDefaultMinBlocks, L, (int)grid, 256, st, nullptr) != 0)
        return OCTMPS_ERR_DEVICE;
    unsigned int err = 0;
    if (cudaMemcpyAsync(&err, scratch + kCtrlOff + 16, sizeof err, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
        return OCTMPS_ERR_DEVICE;
    return err ? OCTMPS_ERR_KERNEL : OCTMPS_OK;
}
