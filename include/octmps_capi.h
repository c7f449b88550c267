/*
 * octmps_capi.h - C ABI of the B200 OCT-MPS photon-transport library.
 *
 * The reference (SSSherif/OCT-MPS) has no library interface: its host
 * program calls a per-GPU worker, RunGPUi(HostThreadState*)
 * (src/main.cu:43), which allocates every device buffer, uploads the mesh,
 * runs the kernels and copies the tallies back, once per A-scan.  This
 * header is the boundary that replaces it.  Plain C types and pointers only;
 * every call returns an octmps_status and never exits the process.
 *
 * Units are the reference's: lengths in cm, coefficients in 1/cm.
 *
 * Entry point                      replaces (reference file:line)
 * -------------------------------  -----------------------------------------
 * octmps_ctx_create/destroy        device setup / cudaDeviceReset in main
 *                                  (src/main.cu:877-888, 1054)
 * octmps_mesh_build_file           MeshGraph + FindRootofGraph +
 * octmps_mesh_find_root            SerializeGraph (src/mesh.cpp:86-359)
 * octmps_mesh_upload/release       mesh upload inside RunGPUi
 *                                  (src/main.cu:447-465), made resident
 * octmps_rng_init                  init_RNG (src/octmps_kernel.cuh:52-172)
 * octmps_job_submit/wait/fetch     RunGPUi (src/main.cu:43-660) with
 *                                  InitDeviceConstantMemory
 *                                  (src/octmps_kernel.cuh:177-220) and
 *                                  CopyDeviceToHostMem (:225-300)
 * octmps_read_opt / octmps_read_mci read_simulation_data
 *                                  (src/octmps_io.cpp:504-645), Bias_Read
 *                                  (src/bias.cpp:9-110)
 * octmps_write_result              Write_Bias_Parameters + WriteResult
 *                                  (src/octmps_io.cpp:237-437)
 */
#ifndef OCTMPS_CAPI_H
#define OCTMPS_CAPI_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    OCTMPS_OK = 0,
    OCTMPS_ERR_INVALID_ARG = 1, /* bad pointer, size or parameter */
    OCTMPS_ERR_OOM = 2,         /* device or host allocation failed */
    OCTMPS_ERR_DEVICE = 3,      /* CUDA error; the message says which */
    OCTMPS_ERR_TIMEOUT = 4,     /* octmps_job_wait ran out of time */
    OCTMPS_ERR_NOT_FOUND = 5,   /* unknown mesh or job id */
    OCTMPS_ERR_IO = 6,          /* file could not be read or written */
    OCTMPS_ERR_NO_DEVICE = 7,   /* no CUDA device, or not sm_100 */
    OCTMPS_ERR_BUDGET = 8,      /* admission refused: HBM budget exceeded */
    OCTMPS_ERR_KERNEL = 9       /* a kernel reported an internal error word */
} octmps_status;

/* Arithmetic of one job.  MIXED: geometry, direction, weight and scattering
 * in FP32, optical path length, depth bin and tally sums in FP64 (the
 * default).  FP32: everything in FP32.  FP64: everything in FP64, the
 * precision of the reference. */
typedef enum { OCTMPS_PREC_MIXED = 0, OCTMPS_PREC_FP32 = 1, OCTMPS_PREC_FP64 = 2 } octmps_precision;

typedef struct octmps_ctx octmps_ctx;
typedef int32_t octmps_mesh_id;
typedef int64_t octmps_job_id;

/* ---- mesh ---------------------------------------------------------------
 * A tetrahedral mesh in the layout SerializeGraph produces
 * (TetrahedronStructGPU and TriangleFaces, src/octmps.h:52-57,193-196):
 * per tet its 1-based region, 4 face indices, 4 orientation signs (+1/-1)
 * and 4 neighbour tets (-1 = boundary, the ambient medium); per face the
 * plane Nx*x + Ny*y + Nz*z + d = 0.  Sign s on face f orients the plane so
 * that (N*s).x + d*s > 0 inside the tet. */
typedef struct {
    int32_t n_tets;
    int32_t n_faces;
    const int32_t *tet_region; /* [n_tets] */
    const int32_t *tet_faces;  /* [n_tets*4] */
    const int32_t *tet_signs;  /* [n_tets*4] */
    const int32_t *tet_adj;    /* [n_tets*4] */
    const double *face_plane;  /* [n_faces*4]: Nx, Ny, Nz, d */
} octmps_mesh_desc;

/* Host-side mesh built from a .mesh file; arrays owned by the library,
 * freed by octmps_mesh_host_free. */
typedef struct {
    int32_t n_vertices;
    int32_t n_tets;
    int32_t n_faces;     /* 4*n_tets slots, as the reference sizes them */
    int32_t n_distinct;  /* faces actually used */
    int32_t *tet_region;
    int32_t *tet_faces;
    int32_t *tet_signs;
    int32_t *tet_adj;
    double *face_plane;
} octmps_host_mesh;

/* ---- simulation parameters (SimulationStruct, src/octmps.h:77-128) ---- */
typedef struct {
    double n, mua, mus, g; /* as read from the .opt file */
} octmps_region;

#define OCTMPS_MAX_REGIONS 100 /* including the ambient region 0 */

typedef struct {
    double start_x, step_x, end_x; /* probe scan, x only (y = z = 0) */
    uint32_t number_of_photons;
    int32_t n_regions;                          /* including ambient region 0 */
    octmps_region regions[OCTMPS_MAX_REGIONS];  /* [0].n = ambient index */
    int32_t type_simulation;
    int32_t type_bias; /* 0: HG only; 37: biased toward the probe; 3: no split */
    int32_t record_photons_flag;
    int32_t num_optical_depth_length_steps; /* depth bins, NBINS */
    double backward_bias_coefficient;
    double target_depth_min, target_depth_max;
    double coherence_length_source;
    double max_collecting_radius;
    double max_collecting_angle_deg;
    double probability_additional_bias;
    double max_relative_contribution;
    double max_filtered_optical_depth;
    double optical_depth_shift;
    /* Never read from input by the reference (src/octmps.h:124); it reads
     * an uninitialised value that is 0 in practice.  0 here. */
    double rnd_step_size_in_tissue;
} octmps_sim;

/* ---- RNG state of one lane: the three MWC streams of init_RNG ---------- */
typedef struct {
    uint64_t *x;  /* general stream: step size, roulette */
    uint32_t *a;
    uint64_t *xR; /* reflect/transmit stream */
    uint32_t *aR;
    uint64_t *xS; /* spin stream */
    uint32_t *aS;
} octmps_rng_lanes;

/* ---- one job: one A-scan (one probe position) -------------------------- */
typedef struct {
    octmps_mesh_id mesh;
    const octmps_sim *sim;  /* copied at submit */
    double probe_x, probe_y, probe_z;
    int32_t root_tet;       /* from octmps_mesh_find_root */
    uint64_t n_photons;     /* packets; 0 = sim->number_of_photons */
    uint64_t seed;          /* general-stream seed (-S); 0 = 985456376 */
    uint32_t n_lanes;       /* RNG lanes (virtual lanes) for this job; 0 = auto */
    int32_t precision;      /* octmps_precision */
} octmps_job;

/* Tally of one job, laid out like SimState's tally arrays
 * (src/octmps.h:155-170).  Caller-allocated arrays. */
typedef struct {
    uint64_t num_filtered;
    uint64_t num_filtered_class1;
    uint64_t num_filtered_class2;
    uint64_t *count1; /* [nbins+1] NumClassI_PhotonsFilteredInRange */
    uint64_t *count2; /* [nbins+1] */
    double *sum1;     /* [nbins+2] ReflectanceClassI_Sum */
    double *max1;     /* [nbins+2] */
    double *sumsq1;   /* [nbins+2] */
    double *sum2;     /* [nbins+2] ReflectanceClassII_Sum */
    double *max2;     /* [nbins+2] */
    double *sumsq2;   /* [nbins+2] */
    uint64_t num_nonfinite; /* detections whose contribution was NaN or infinite (added
                               to the sums like any other); filled by octmps_job_fetch */
} octmps_tally;

/* Per-job statistics filled by octmps_job_fetch_stats. */
typedef struct {
    uint64_t packets;     /* packets launched (equals n_photons) */
    uint64_t steps;       /* propagation steps taken */
    uint64_t restores;    /* split copies resumed */
    double device_ms;     /* kernel time of the launch the job finished in, or -1
                             while that launch still runs (never waits) */
    double submit_to_done_ms;
    int64_t launch_id;    /* sequence number (per context) of that launch */
    uint64_t stopped;     /* packets stopped: at the step cap (2^26 steps, an error) or
                             after 1000 boundary hits in a row that did not move the
                             photon (a packet the reference would run forever) */
} octmps_job_stats;

/* One detected packet of a job whose sim sets record_photons_flag: the fields
 * that BiasParam.mco describes for FilteredPhotons.mco ("Weight |
 * LikelihoodRatio | Radius | AngleRad | OpticalPath | MaxDepth",
 * src/octmps_io.cpp:259-270; the reference creates the file but writes no
 * record).  Values in the job's geometry precision, widened exactly. */
typedef struct {
    double weight;        /* w (1 - R): the packet weight that leaves through the face */
    double likelihood;    /* the packet's likelihood ratio */
    double radius;        /* distance from the probe axis at the exit */
    double cos_angle;     /* -uz at the exit; the angle to the probe axis is acos of it */
    double optical_path;
    double max_depth;
} octmps_photon_record;

/* ---- context ------------------------------------------------------------ */
octmps_status octmps_ctx_create(int device, octmps_ctx **out);
octmps_status octmps_ctx_destroy(octmps_ctx *ctx);
const char *octmps_last_error(const octmps_ctx *ctx);
const char *octmps_status_string(octmps_status st);

/* Multiplier table of the MWC generators: the first column of
 * safeprimes_base32.txt (src/octmps_kernel.cuh:74-105).  Needed before any
 * job is submitted; at least 3 + 3*n_lanes entries. */
octmps_status octmps_ctx_set_multipliers(octmps_ctx *ctx, const uint32_t *a, uint64_t count);

/* Launch configuration (0 = default).  Two forms of the photon kernel run
 * the same per-photon arithmetic:
 *   per-lane (kernel_form 0, the default): one photon per thread, a warp
 *     vote choosing which half of a propagation step (boundary test, or
 *     scattering) its lanes run; blocks of 256 threads (2, 3 or 4 resident
 *     per SM), 128 (6, 7 or 8) or 512 (2) in the FP32 geometry forms, 256 x 2
 *     in the FP64 form;
 *   pooled (kernel_form 1): 128-thread blocks; each warp holds two photons
 *     per lane in shared memory and runs every half-step on a full warp of
 *     photons at once (fuller warps, but more instructions and fewer
 *     resident warps: slower on the B-scan workload). */
typedef struct {
    int32_t block_size;       /* per-lane 256 (0 = 256), 128 or 512; pooled 128 (0 = 128) */
    int32_t blocks_per_sm;    /* resident blocks per SM: per-lane 256 x 2, 3 or 4 (0 = 3),
                                 128 x 6, 7 or 8 (0 = 6), 512 x 2 (0 = 2); FP64 256 x 2;
                                 pooled 4, 5 or 6 (0 = 4; the FP64 form 2 or 3, 0 = 2) */
    int32_t default_lanes;    /* RNG lanes per job when job.n_lanes = 0 */
    int32_t use_graphs;       /* reserved, 0 (a batch is one persistent launch, so
                                 there is no launch sequence to replay) */
    uint64_t hbm_budget_bytes;/* admission budget for job state; 0 = 80% of free */
    int32_t scatter_share;    /* per-lane: a warp runs its lanes' scattering step halves
                                 once at least scatter_share/32 of its live lanes wait for
                                 one; pooled: with fewer than 32 photons waiting for the
                                 boundary half, the scattering half runs once it holds at
                                 least scatter_share/32 of the warp's photons (1..32;
                                 0 = 12) */
    int32_t linger_us;        /* a kernel thread that finds no work waits this long for
                                 newly submitted jobs before it exits (0 = 2000;
                                 -1 = exit at once; at most 1000000) */
    int32_t kernel_form;      /* 0 per-lane (default), 1 pooled */
} octmps_launch_config;
octmps_status octmps_ctx_configure(octmps_ctx *ctx, const octmps_launch_config *cfg);

/* ---- meshes -------------------------------------------------------------- */
octmps_status octmps_mesh_build_file(const char *path, octmps_host_mesh *out);
void octmps_mesh_host_free(octmps_host_mesh *m);
/* Root tet of a probe position with FindRootofGraph's rule
 * (src/mesh.cpp:257-289); *root = -1 with OCTMPS_ERR_NOT_FOUND if the
 * probe is not on a boundary face. */
octmps_status octmps_mesh_find_root(const octmps_mesh_desc *m, double px, double py, double pz,
                                    int32_t *root);
octmps_status octmps_mesh_upload(octmps_ctx *ctx, const octmps_mesh_desc *m,
                                 octmps_mesh_id *out);
octmps_status octmps_mesh_release(octmps_ctx *ctx, octmps_mesh_id id);

/* ---- RNG seeding (init_RNG) ---------------------------------------------- */
octmps_status octmps_rng_init(const uint32_t *multipliers, uint64_t n_multipliers, uint32_t n_lanes,
                              uint64_t seed, octmps_rng_lanes *out);

/* ---- jobs ------------------------------------------------------------------
 * A job is one A-scan; the reference runs one per worker call (RunGPUi,
 * src/main.cu:43).  Submitted jobs go into a device job table (one per
 * precision); octmps_ctx_flush (or a wait on any job) starts a persistent
 * launch over the table if none runs.  A job submitted while a launch runs
 * is appended to the table and taken up by that launch as its threads free
 * up (continuous batching); a job is finished, and can be fetched and
 * released, as soon as all of its lanes have reported, which can be before
 * the launch ends.  octmps_ctx_synchronize waits for every launch to end.
 * octmps_ctx_poll is a completion queue: it advances the launches and
 * returns up to max_ids jobs finished since the last poll (the first poll
 * also returns jobs finished before it), without waiting. */
octmps_status octmps_job_submit(octmps_ctx *ctx, const octmps_job *job, octmps_job_id *out);
octmps_status octmps_ctx_flush(octmps_ctx *ctx);
octmps_status octmps_ctx_synchronize(octmps_ctx *ctx);
octmps_status octmps_ctx_poll(octmps_ctx *ctx, octmps_job_id *done, int32_t max_ids,
                              int32_t *n_done);
octmps_status octmps_job_wait(octmps_ctx *ctx, octmps_job_id id, int32_t timeout_ms);
octmps_status octmps_job_fetch(octmps_ctx *ctx, octmps_job_id id, octmps_tally *out);
octmps_status octmps_job_fetch_stats(octmps_ctx *ctx, octmps_job_id id, octmps_job_stats *out);
octmps_status octmps_job_release(octmps_ctx *ctx, octmps_job_id id);
/* RecordPhotonsFlag: records kept per job for jobs whose sim sets
 * record_photons_flag (0 = the job's packet count, the default); further
 * detections are counted but not kept.  Applies to jobs submitted after it. */
octmps_status octmps_ctx_set_photon_record_capacity(octmps_ctx *ctx, uint64_t capacity);
/* A finished job's detected-packet records, in detection order (which varies
 * from run to run; the set does not): copies min(kept, max) into `out`
 * (may be NULL with max 0), sets *n_kept to the records kept and
 * *n_detected to all detections.  A job without the flag has none. */
octmps_status octmps_job_photon_records(octmps_ctx *ctx, octmps_job_id id,
                                        octmps_photon_record *out, uint64_t max,
                                        uint64_t *n_kept, uint64_t *n_detected);

/* Diagnosis: the first packet of a precision's job table (its current batch,
 * else the latest batch that had one) that was stopped, with the state it
 * was stopped in; seed, n_lanes and n_photons are filled while the job is
 * not released. */
typedef struct {
    int32_t stopped;        /* 0 none, 1 step cap, 2 no progress */
    int32_t tet;
    octmps_job_id job;
    uint64_t seed, n_lanes, n_photons;
    uint64_t lane;          /* RNG lane (virtual thread) of the job */
    uint64_t packets_left;  /* packets of that lane still to run, this one included */
    uint64_t steps;
    double pos[3], dir[3];
    double weight, step_left;
} octmps_incident;
octmps_status octmps_debug_incident(octmps_ctx *ctx, int32_t precision, octmps_incident *out);

/* ---- files (the reference's formats) -------------------------------------- */
octmps_status octmps_read_opt(const char *path, octmps_sim *out);
octmps_status octmps_read_mci(const char *path, octmps_sim *inout);
/* Appends one A-scan to ClassI_Scatt.out, ClassII_Scatt.out,
 * ClassI_ScattFilt.out, ClassII_ScattFilt.out and rewrites BiasParam.mco
 * and FilteredPhotons.mco, in directory `dir` ("" = current). */
octmps_status octmps_write_result(const char *dir, const octmps_sim *sim, double probe_x,
                                  const octmps_tally *t);
/* Appends detected-packet records to FilteredPhotons.mco in `dir`, one line
 * per record: the A-scan's probe position, then Weight, LikelihoodRatio,
 * Radius, AngleRad (acos of cos_angle), OpticalPath, MaxDepth ("%G",
 * tab-separated). */
octmps_status octmps_write_filtered_photons(const char *dir, double probe_x,
                                            const octmps_photon_record *r, uint64_t n);

/* ---- one A-scan without any allocation ----------------------------------------
 * No counterpart in the reference: an addition for callers that cannot
 * allocate device memory, for instance an application that gives the
 * library a fixed device arena and forbids further cudaMalloc (real-time or
 * certified pipelines, or a host framework whose caching allocator owns all
 * of device memory), or code running where an allocation could stall.
 *
 * octmps_ascan_run_noalloc runs one A-scan (mixed precision) through the same
 * photon kernel as octmps_job_submit.  The caller passes every input and
 * output in device memory it owns; the call allocates nothing (no cudaMalloc,
 * cudaFree or allocating library routine).  What the kernel needs beyond the
 * inputs and outputs (job descriptor, work counter, error word, statistics,
 * region constants: OCTMPS_NOALLOC_SCRATCH_BYTES) lives in one fixed
 * file-scope device array that every GPU loading the library holds until the
 * process exits.  The first call on a device looks up that array's device
 * address (once per device); make that first call before any stream capture.
 * All calls on a device share the array, so calls whose work overlaps on the
 * GPU race: serialise them.  The array's device address is kept per device
 * for the life of the process, so calls after cudaDeviceReset are not
 * supported.  The call returns after the A-scan finished.  It keeps no
 * detected-packet records (RecordPhotonsFlag is ignored: they would need a
 * buffer of the caller's; use the job API for them).
 *
 * Device layouts the caller provides:
 *   planes : float, 16 per tet: for face k = 0..3 the reference's face plane
 *            (Nx, Ny, Nz, d) of tet_faces[k] times tet_signs[k]
 *   adj    : int32, 4 per tet (16-byte aligned): -1 for a boundary face, else
 *            neighbour | region_of_neighbour << 24 (meshes below 2^24 tets),
 *            with neighbour < n_tets and 1 <= region < sim->n_regions; the
 *            call checks every entry on the device before any photon runs
 *            and returns OCTMPS_ERR_INVALID_ARG on a bad one
 *   rng_*  : the lanes' generator states as octmps_rng_init fills them
 *   tally  : OCTMPS_NOALLOC_TALLY_BYTES(nbins) bytes, zeroed by the call:
 *            uint64 totals[4] (filtered, class I, class II, 0) at byte 0, then
 *            uint64 count1[nbins+1], count2[nbins+1], then double sum1, sumsq1,
 *            sum2, sumsq2, max1, max2 [nbins+2] each; every array starts on a
 *            16-byte boundary.
 * Errors: OCTMPS_ERR_INVALID_ARG for null pointers, more than
 * OCTMPS_NOALLOC_MAX_REGIONS regions, glass regions (mus = 0), n_lanes 0 or
 * above n_photons, root or tet counts out of range, a neighbour entry out of
 * range; OCTMPS_ERR_KERNEL if the
 * kernel flagged a photon; OCTMPS_ERR_DEVICE on a CUDA error. */
#define OCTMPS_NOALLOC_MAX_REGIONS 100
#define OCTMPS_NOALLOC_SCRATCH_BYTES 3440 /* per GPU, held until exit */
#define OCTMPS_NOALLOC_ROUND16(n) ((((uint64_t)(n)) + 15u) & ~(uint64_t)15u)
#define OCTMPS_NOALLOC_TALLY_BYTES(nbins) \
    (32u + 2u * OCTMPS_NOALLOC_ROUND16(((uint64_t)(nbins) + 1u) * 8u) + \
     6u * OCTMPS_NOALLOC_ROUND16(((uint64_t)(nbins) + 2u) * 8u))
typedef struct {
    const octmps_sim *sim;          /* host memory; copied by the call */
    const float *planes;            /* device */
    const int32_t *adj;             /* device */
    int32_t n_tets;
    int32_t root_tet;               /* octmps_mesh_find_root */
    int32_t root_region;            /* region of root_tet (tet_region[root_tet] of the
                                       mesh; it sets the specular weight and the
                                       first optical constants, and is not checked
                                       against adj) */
    double probe_x, probe_y, probe_z;
    uint64_t n_photons;
    uint32_t n_lanes;               /* 1 .. n_photons */
    const uint64_t *rng_x;          /* device, n_lanes each */
    const uint32_t *rng_a;
    const uint64_t *rng_xR;
    const uint32_t *rng_aR;
    const uint64_t *rng_xS;
    const uint32_t *rng_aS;
    void *tally;                    /* device */
} octmps_noalloc_ascan;
octmps_status octmps_ascan_run_noalloc(const octmps_noalloc_ascan *a, void *stream);

/* ---- A-scans of a B-scan ---------------------------------------------------
 * octmps_probe_positions: the probe positions of main()'s A-scan loop
 * (src/main.cu:948-950), x from start_x while x < end_x in double steps of
 * step_x; writes at most max_out, returns the count (-1: invalid).
 * octmps_ascans_of_gpu: the A-scans GPU `gpu` of `n_gpus` runs under the
 * CLI's -G (round robin: gpu, gpu + n_gpus, ...); replaces the per-GPU photon
 * split of DoOneSimulation (src/main.cu:665-848); writes at most max_out
 * indices, returns the count (-1: invalid). */
int64_t octmps_probe_positions(const octmps_sim *sim, double *out, uint64_t max_out);
int64_t octmps_ascans_of_gpu(uint64_t n_ascans, uint32_t n_gpus, uint32_t gpu, uint64_t *out,
                             uint64_t max_out);

/* ---- multiplier table generation (safeprimes_base32.txt) ---------------- */
int octmps_safeprimes_generate(uint32_t *out, uint64_t count);
int octmps_safeprimes_write(const char *path, uint64_t count);
/* Reads the first column of a safe-prime file; returns entries read. */
int64_t octmps_safeprimes_read(const char *path, uint32_t *out, uint64_t max_count);

#ifdef __cplusplus
}
#endif

#endif /* OCTMPS_CAPI_H */
