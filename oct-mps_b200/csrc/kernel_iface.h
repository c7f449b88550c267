// Device-side job table shared by the runtime (runtime.cu) and the photon
// kernel (photon_kernel.cu).
#ifndef OCTMPS_KERNEL_IFACE_H
#define OCTMPS_KERNEL_IFACE_H

#include <cstdint>

#include <vector_types.h>

namespace octmps {

// Neighbour entry of the packed mesh: -1 for the ambient medium, else the
// neighbour tet index in the low 24 bits and its region in the high 8.
constexpr int kAdjIndexBits = 24;
constexpr uint32_t kAdjIndexMask = (1u << kAdjIndexBits) - 1u;
constexpr int kMaxTetsPacked = 1 << kAdjIndexBits;

// Per-region constants as InitDeviceConstantMemory derives them
// (src/octmps_kernel.cuh:204-214), in the job's geometry precision, followed
// by the two job-invariant terms of the biased spin that cost a square root
// or a logarithm (region_consts.h derives them): sqrt(1 + b^2) of the job's
// bias coefficient b, and the distance -log(rndStepSizeInTissue) / mu_t.
// (Terms that take an add or a multiply are cheaper computed than loaded.)
template <typename T>
struct RegionConst {
    T n, muas, rmuas, mua_muas, g;
    T b_sq1p2;  // sqrt(mad(b, b, 1))
    T far;      // +inf when rndStepSizeInTissue is 0
};

// One job (one A-scan) of a launch.  All pointers are device pointers.
// A slot is exactly two 128-byte cache lines of its own: a launch reads a
// slot that the host filled while the launch ran, and no line of it may have
// been cached in L1 before (a line shared with the neighbouring slot would
// be, stale).
struct alignas(256) JobDesc {
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
    unsigned long long *stats;  // kStatsWords statistics words (below)
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
    int32_t n_regions;    // entries of regions[]; a neighbour's region must be below it
    uint32_t record_cap;  // detected-packet records kept (RecordPhotonsFlag)
    struct PhotonRecordDev *photon_records;  // null: none kept; index from stats[4]
};

// One detected packet (RecordPhotonsFlag), laid out as octmps_photon_record.
struct PhotonRecordDev {
    double weight, likelihood, radius, cos_angle, optical_path, max_depth;
};

// Statistics words after a job's tally block: [0] steps [1] restores
// [2] packets [3] stopped [4] detections recorded (the record index; may pass
// record_cap), [5..7] unused.
constexpr int kStatsWords = 8;

static_assert(sizeof(JobDesc) == 256, "a job slot is two cache lines");

// Tally block of one job (P = double or float):
//   uint64 totals[4]     NumFilteredPhotons, ...ClassI, ...ClassII, and the
//                        number of NaN or infinite contributions added
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

// The first packet a table's launches stopped (flag 1: step cap; 2: no
// progress), for diagnosis; written once, cleared when the table is reset.
struct Incident {
    unsigned int flag;
    unsigned int slot;
    int32_t tet;
    uint32_t packets_left;  // packets of the lane still to run, this one included
    uint64_t lane;
    uint64_t steps;
    double pos[3], dir[3];
    double w, sleft;
};

// A launch works through a job table that may grow while it runs: the host
// fills a free slot (descriptor and unit base) and only then raises the
// total number of units, so a kernel thread that takes unit u < total always
// finds u's slot complete.  Threads take units by compare-and-swap on the
// next-unit counter, which therefore never passes the total.  A thread that
// finds no unit left retries (jobs submitted meanwhile are taken up by the
// running launch) until its block has been idle for linger_us or the host
// raises the drain word, and then exits.  Several launches may work
// through one table at once: the host starts another when work arrives while
// the running one may be down to its last threads, and the new launch's
// blocks take SM slots as the older launch's blocks leave.
struct LaunchArgs {
    const JobDesc *jobs;            // job slots
    const uint64_t *unit_base;      // [n_slots]: first unit of each slot; ~0 for empty slots
    int32_t n_slots;                // table capacity (binary search range)
    unsigned long long *ctrl;       // [0] next unit to hand out, [1] total units, [2] error
                                    // word, [3] nonzero: idle threads exit (drain)
    uint2 *slot_state;              // per slot: x = units (RNG lanes) finished, y = launch_seq
                                    // of the launch that finished the last one; may be null
    Incident *incident;             // may be null
    uint64_t start_unit;            // at launch thread t takes unit start_unit + t ...
    uint64_t initial_total;         // ... if that is below the total at launch; 0 for a
                                    // launch beside a running one (blocks claim runs)
    uint64_t step_cap;              // steps allowed per packet
    int32_t scatter_share;          // a warp runs the scattering halves of its steps once
                                    // at least scatter_share/32 of its live lanes wait
    uint32_t launch_seq;            // nonzero
    int32_t record_slot;            // recording variant: the slot whose lanes are recorded
    uint32_t linger_us;             // a thread that finds no unit retries for this long
                                    // (about 1 us granularity) before it exits
};

// Error bits reported through LaunchArgs::error.
constexpr unsigned int kErrNoExitFace = 1u;   // a hit with no face toward the photon
constexpr unsigned int kErrStepCap = 2u;      // a packet exceeded step_cap
constexpr unsigned int kErrBadNeighbour = 4u; // neighbour index out of range

enum Precision { kMixed = 0, kFP32 = 1, kFP64 = 2 };

// Block size and resident blocks per SM of the default kernel variant, and
// the share of a warp's live lanes (in 32nds) that must wait for the
// scattering half of their step before the warp runs it: the best of a sweep
// on 8 A-scans of the B-scan workload (steps/s, mixed form): 3 blocks
// (80-register cap) 33.0-33.6 G at shares 10-14, against 28.8-29.3 G with 2
// blocks and 28.4-29.1 G with 4.
constexpr int kDefaultBlock = 256;
constexpr int kDefaultMinBlocks = 3;
constexpr int kDefaultScatterShare = 12;

// Host-callable launcher (photon_kernel.cu).  (block, min_blocks) selects the
// variant compiled for that block size and that many resident blocks per SM:
// 256 x 2, 3 or 4; 128 x 6, 7 or 8; 512 x 2 (FP32 geometry forms); the FP64
// form and the recording variant (records, a test hook) only 256 x 2.
int launch_photon_kernel(int precision, int min_blocks, const LaunchArgs &args, int grid,
                         int block, void *stream, void *records);
int photon_kernel_attributes(int precision, int block, int min_blocks, int *regs,
                             int *max_blocks_per_sm);
// Whether a per-lane variant exists (for configuration checks).
bool photon_kernel_variant(int precision, int block, int min_blocks);

// Pooled kernel (photon_kernel.cu): 128-thread blocks, each warp holding
// kPooledPerThread photons per lane in shared memory; min_blocks 4, 5 or 6
// (FP32 geometry forms), 2 or 3 (FP64 form); the recording variant runs 2.
// `splits`: a device buffer of pooled_split_bytes(precision, grid) bytes for
// the photons' split copies, private to the launch.
constexpr int kPooledBlock = 128;
constexpr int kPooledPerThread = 2;
constexpr int kDefaultPooledMinBlocks = 4;
constexpr int kDefaultPooledMinBlocksFP64 = 2;
size_t pooled_split_bytes(int precision, int grid);
int launch_pooled_kernel(int precision, int min_blocks, const LaunchArgs &args, int grid,
                         void *stream, void *records, void *splits);
int pooled_kernel_attributes(int precision, int min_blocks, bool record, int *regs,
                             int *max_blocks_per_sm);

}  // namespace octmps

#endif
