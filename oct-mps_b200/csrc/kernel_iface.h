// Device-side job table shared by the runtime (runtime.cu) and the photon
// kernel (photon_kernel.cu).
#ifndef OCTMPS_KERNEL_IFACE_H
#define OCTMPS_KERNEL_IFACE_H

#include <cstdint>

namespace octmps {

// Neighbour entry of the packed mesh: -1 for the ambient medium, else the
// neighbour tet index in the low 24 bits and its region in the high 8.
constexpr int kAdjIndexBits = 24;
constexpr uint32_t kAdjIndexMask = (1u << kAdjIndexBits) - 1u;
constexpr int kMaxTetsPacked = 1 << kAdjIndexBits;

// Per-region constants as InitDeviceConstantMemory derives them
// (src/octmps_kernel.cuh:204-214), in the job's geometry precision.
template <typename T>
struct RegionConst {
    T n, muas, rmuas, mua_muas, g;
};

// One job (one A-scan) of a launch.  All pointers are device pointers.
struct JobDesc {
    const void *planes;   // per tet 4 inward planes (nx, ny, nz, d), float or double
    const int32_t *adj;   // per tet 4 packed neighbour entries (int4-aligned)
    const void *regions;  // RegionConst<T>[n_regions]
    uint64_t *rng_x;      // this job's lanes: general stream
    uint32_t *rng_a;
    uint64_t *rng_xR;     // reflect/transmit stream
    uint32_t *rng_aR;
    uint64_t *rng_xS;     // spin stream
    uint32_t *rng_aS;
    void *tally;          // tally block, layout below
    unsigned long long *stats;  // [0] steps [1] restores [2] packets [3] capped
    uint64_t n_photons;
    uint32_t n_lanes;
    int32_t n_tets;
    double probe_x, probe_y, probe_z;
    double w0;            // 1 - Rspecular
    double tdmin, tdmax, bias_a, p_bias;
    double cos_collect;   // cos(MaxCollectingAngleDeg * PI_const / 180)
    double radius;        // MaxCollectingRadius
    double rnd_step;      // rndStepSizeInTissue
    double n_ambient;
    double shift, bin_width, half_lc;  // OpticalDepthShift, Lc/6, Lc/2 (round-down)
    int32_t root_tet, root_region, type_bias, nbins;
};

// Tally block of one job (P = double or float):
//   uint64 totals[4]     NumFilteredPhotons, ...ClassI, ...ClassII, pad
//   uint64 count1[nb+1], count2[nb+1]
//   P      sum1[nb+2], sumsq1[nb+2], sum2[nb+2], sumsq2[nb+2]
//   P      max1[nb+2], max2[nb+2]  (kept as unsigned bit patterns: the
//          values are >= 0, so integer max on the bits is max on the values)
struct TallyLayout {
    size_t totals, count1, count2, sum1, sumsq1, sum2, sumsq2, max1, max2, bytes;
};

#ifdef __CUDACC__
#define OCTMPS_HD __host__ __device__
#else
#define OCTMPS_HD
#endif

OCTMPS_HD inline size_t tally_round16(size_t n) { return (n + 15) & ~size_t(15); }

OCTMPS_HD inline TallyLayout tally_layout(int nbins, size_t psize) {
    TallyLayout L;
    const size_t cnt = tally_round16((size_t)(nbins + 1) * 8);
    const size_t val = tally_round16((size_t)(nbins + 2) * psize);
    L.totals = 0;
    L.count1 = 32;
    L.count2 = L.count1 + cnt;
    L.sum1 = L.count2 + cnt;
    L.sumsq1 = L.sum1 + val;
    L.sum2 = L.sumsq1 + val;
    L.sumsq2 = L.sum2 + val;
    L.max1 = L.sumsq2 + val;
    L.max2 = L.max1 + val;
    L.bytes = L.max2 + val;
    return L;
}

struct LaunchArgs {
    const JobDesc *jobs;
    const uint64_t *unit_base;  // [n_jobs+1]: first work unit (RNG lane) of each job
    int32_t n_jobs;
    uint64_t total_units;
    unsigned long long *next_unit;  // work counter, zeroed before the launch
    unsigned int *error;            // error word, zeroed before the launch
    uint64_t step_cap;              // steps allowed per packet
    int32_t scatter_share;          // a warp runs the scattering halves of its steps once
                                    // at least scatter_share/32 of its live lanes wait
};

// Error bits reported through LaunchArgs::error.
constexpr unsigned int kErrNoExitFace = 1u;   // a hit with no face toward the photon
constexpr unsigned int kErrStepCap = 2u;      // a packet exceeded step_cap
constexpr unsigned int kErrBadNeighbour = 4u; // neighbour index out of range

enum Precision { kMixed = 0, kFP32 = 1, kFP64 = 2 };

// Host-callable launcher (photon_kernel.cu).
// min_blocks (2 or 3) selects the variant compiled for that many resident
// blocks per SM; records (test hook) selects the recording variant.
int launch_photon_kernel(int precision, int min_blocks, const LaunchArgs &args, int grid,
                         int block, void *stream, void *records);
int photon_kernel_attributes(int precision, int block, int min_blocks, int *regs,
                             int *max_blocks_per_sm);

}  // namespace octmps

#endif
