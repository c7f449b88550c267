/*
 * oracle.h - CPU restatement of OCT-MPS's per-photon Monte Carlo method.
 *
 * TEST INFRASTRUCTURE ONLY.  Only the tests, the smoke check and the
 * bench's CPU-baseline leg may load this library; the product never links
 * it and has no CPU fallback to it.
 *
 * What it restates: the device path of the reference,
 * src/octmps_kernel.cuh:475-1402 (LaunchPhoton, ComputeStepSize,
 * HitBoundary, Hop, Drop, FastReflectTransmit with the Class I/II tally,
 * Spin, SpinTheta, SpinThetaForwardFstBias, SpinBias, roulette with split
 * restore) and the MWC generator (:10-29), in three precisions:
 *   precision 0 (MIXED): geometry/scattering FP32, path and tallies FP64
 *   precision 1 (FP32) : everything FP32
 *   precision 2 (FP64) : everything FP64, as the reference
 * with one deterministic numerical method shared, by specification only,
 * with the CUDA kernels: every FMA is written out, division and square root
 * are IEEE (FP64 divisions round down, like the reference's FAST_DIV), and
 * log / sin / cos are computed by the project's own series (atanh series
 * for log, Taylor series after an exact or Cody-Waite reduction for sin and
 * cos), so host and device results agree bit for bit.
 *
 * Parity pinning: the FP64 form is checked against the reference's own
 * routine compiled for the host (oracle/_ref, built by oracle/Makefile from
 * the reference tree) on the fixtures in tests/golden/.
 */
#ifndef OCTMPS_ORACLE_H
#define OCTMPS_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ORACLE_MAX_REGIONS 100

typedef struct {
    int32_t n_regions; /* including the ambient region 0 */
    double region_n[ORACLE_MAX_REGIONS];
    double region_mua[ORACLE_MAX_REGIONS];
    double region_mus[ORACLE_MAX_REGIONS];
    double region_g[ORACLE_MAX_REGIONS];
    int32_t type_bias;
    int32_t nbins; /* NumOpticalDepthLengthSteps */
    double target_depth_min, target_depth_max;
    double backward_bias_coefficient;
    double max_collecting_angle_deg, max_collecting_radius;
    double probability_additional_bias;
    double optical_depth_shift, coherence_length_source;
    double rnd_step_size_in_tissue;
} OracleParams;

/* Mesh in SerializeGraph's layout (src/mesh.cpp:294-359). */
typedef struct {
    int32_t n_tets;
    int32_t n_faces;
    const int32_t *region; /* [n_tets] */
    const int32_t *faces;  /* [n_tets*4] */
    const int32_t *signs;  /* [n_tets*4] */
    const int32_t *adj;    /* [n_tets*4] */
    const double *planes;  /* [n_faces*4] Nx, Ny, Nz, d */
} OracleMesh;

typedef struct {
    uint64_t num_filtered, num_filtered_class1, num_filtered_class2;
    uint64_t *count1, *count2;    /* [nbins+1] */
    double *sum1, *max1, *sumsq1; /* [nbins+2] */
    double *sum2, *max2, *sumsq2; /* [nbins+2] */
    uint64_t steps, restores, packets, capped;
} OracleTally;

/* One packet (a launch and every split copy it resumes) summarised so that
 * event sequences can be compared exactly. */
typedef struct {
    uint64_t hash;       /* FNV-1a over (tet << 8 | event) per step */
    uint64_t x, xR, xS;  /* generator states when the packet ends */
    uint32_t steps, hits, scatters, restores, detections, survivals;
    double contribution; /* sum of detected w*(1-R)*LR, in order */
    double optical_path; /* optical path when the packet ends */
} OraclePacket;

enum {
    ORACLE_EV_SCATTER = 1,
    ORACLE_EV_TRANSMIT = 2,
    ORACLE_EV_REFLECT = 3,
    ORACLE_EV_EXIT = 4,
    ORACLE_EV_DETECT = 8,
    ORACLE_EV_SURVIVE = 16,
    ORACLE_EV_RESTORE = 32,
    ORACLE_EV_END = 64
};

/* Runs one A-scan: n_photons packets spread over n_lanes RNG lanes, lane v
 * taking n_photons/n_lanes packets plus one if v < n_photons % n_lanes, each
 * lane's packets drawn in order from that lane's three MWC streams.
 * first (optional, [n_lanes]) receives lane v's first packet.  Returns 0 on
 * success. */
int oracle_run(const OracleParams *p, const OracleMesh *m, double probe_x, double probe_y,
               double probe_z, int32_t root, uint64_t n_photons, uint32_t n_lanes,
               const uint64_t *x, const uint32_t *a, const uint64_t *xR, const uint32_t *aR,
               const uint64_t *xS, const uint32_t *aS, int precision, int n_threads,
               OracleTally *out, OraclePacket *first);

/* Per-step state of one lane's packet number packet_index (0 = its first;
 * diagnostics): per step 12 doubles tet, event, x, y, z, ux, uy, uz, w, s,
 * optical path, likelihood ratio; at most max_steps steps (the dumped packet
 * ends there).  Returns the number of steps written. */
int oracle_dump_lane(const OracleParams *p, const OracleMesh *m, double probe_x, double probe_y,
                     double probe_z, int32_t root, uint64_t x, uint32_t a, uint64_t xR,
                     uint32_t aR, uint64_t xS, uint32_t aS, int precision, double *out,
                     uint32_t max_steps, uint64_t packet_index);

/* The math kernels of the method, exposed for unit tests. */
float oracle_logf(float x);
double oracle_log(double x);
void oracle_sincos_turn_f(float turns, float *s, float *c); /* sin, cos of 2*pi*turns */
void oracle_sincos_d(double psi, double *s, double *c);
double oracle_div_rd(double a, double b);
float oracle_uint2float_rz(uint32_t u);

/* MWC multiplier list: every a < 2^32 with a*2^32 - 1 and a*2^31 - 1 prime,
 * descending from 2^32 - 1 (the first column of the reference's missing
 * safeprimes_base32.txt, src/octmps_kernel.cuh:74-105).  0 on success. */
int oracle_safeprimes(uint32_t *out, uint64_t count);

/* One detected packet (RecordPhotonsFlag): weight leaving (w (1 - R)),
 * likelihood ratio, radius and cosine (-uz) at the exit, optical path,
 * maximum depth; the fields BiasParam.mco lists for FilteredPhotons.mco
 * (src/octmps_io.cpp:259-270). */
typedef struct {
    double weight, likelihood, radius, cos_angle, optical_path, max_depth;
} OraclePhotonRecord;

/* Runs that follow append their detected-packet records to `buf` (at most
 * `cap`; buf NULL: none) and count every detection; returns the count since
 * the last call and resets it. */
uint64_t oracle_set_photon_records(OraclePhotonRecord *buf, uint64_t cap);

#ifdef __cplusplus
}
#endif

#endif
