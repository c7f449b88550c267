// Test infrastructure only (never linked into the product).
//
// Host driver around the reference's own per-photon routine.  The
// reference's source is compiled in place from its tree (see
// oracle/Makefile): src/octmps_kernel.cuh through the CUDA-keyword shim in
// cuda_shim.h, and src/mesh.cpp, src/bias.cpp, src/octmps_io.cpp unchanged.
// This file adds only what src/main.cu would do on the host, written anew
// for a CPU: it emulates the grid of OCTMPSKernel with OpenMP, and exposes
// the reference's parsers, mesh builder, RNG seeding and writers through a
// flat C interface that the tests call with ctypes.
#include "cuda_shim.h"

#include <omp.h>

#include <chrono>
#include <vector>

#ifdef OCTMPS_REF_METHOD_MATH
// The "method" build (oracle/_ref/libocref_method.so): the reference's
// log and sincos calls (src/octmps_kernel.cuh:510, 847, 957, 1012) go to the
// oracle's own series (oracle.cpp, linked in) instead of glibc's, every other
// operation (acos included) unchanged.  The FP64 oracle and this build then
// differ only where the oracle restates the method differently, which is
// what the test of this build pins.
#include <math.h>  // its declarations before the renames below
#include <stdio.h>
#include <stdlib.h>
extern "C" double oracle_log(double x);
extern "C" void oracle_sincos_d(double psi, double *s, double *c);
static inline double octmps_method_log(double x) { return oracle_log(x); }
static inline void octmps_method_sincos(double x, double *s, double *c) { oracle_sincos_d(x, s, c); }
#define log octmps_method_log
#define sincos octmps_method_sincos
#endif
#include "octmps_kernel.cuh"
#ifdef OCTMPS_REF_METHOD_MATH
#undef log
#undef sincos
#endif

thread_local shim_dim3 blockIdx = {0, 0, 0};
thread_local shim_dim3 threadIdx = {0, 0, 0};
shim_dim3 blockDim = {NUM_THREADS_PER_BLOCK, 1, 1};
shim_dim3 gridDim = {1, 1, 1};

// Rspecular lives in src/main.cu (:29-37), which is CUDA-only host code the
// shim cannot compile; its one-line formula is restated here.
FLOAT Rspecular(FLOAT ni, FLOAT nt) {
    FLOAT temp = (ni - nt) / (ni + nt);
    return temp * temp;
}

// Flat copy of the SimulationStruct fields the path uses
// (src/octmps.h:77-128), so tests can compare parsers field by field and
// drive a run with parameters from either parser.
struct RefSim {
    double start_x, step_x, end_x;
    uint32_t number_of_photons;
    int32_t n_regions;  // including the ambient region 0
    double region_n[MAX_REGIONS], region_mua[MAX_REGIONS], region_mus[MAX_REGIONS],
        region_g[MAX_REGIONS], region_mutr[MAX_REGIONS];
    int32_t type_simulation, type_bias, record_photons_flag, num_optical_depth_length_steps;
    double backward_bias_coefficient, target_depth_min, target_depth_max,
        coherence_length_source, max_collecting_radius, max_collecting_angle_deg,
        probability_additional_bias, max_relative_contribution, max_filtered_optical_depth,
        optical_depth_shift, rnd_step_size_in_tissue;
};

// Tally block laid out as SimState's tally arrays (src/octmps.h:155-170).
struct RefTally {
    uint64_t num_filtered, num_filtered_class1, num_filtered_class2;
    uint64_t *count1, *count2;             // [nbins+1]
    double *sum1, *max1, *sumsq1;          // [nbins+2]
    double *sum2, *max2, *sumsq2;          // [nbins+2]
};

// Mesh in SerializeGraph's layout (src/mesh.cpp:294-359): per tet
// idx, region, faces[4], signs[4], adjTetras[4]; per face Nx, Ny, Nz, d.
struct RefMesh {
    int32_t n_tets, n_faces, root;
    const int32_t *tet;  // [n_tets*14]
    const double *face;  // [n_faces*4]
};

static void sim_from_flat(const RefSim *f, SimulationStruct *s, RegionStruct *regions) {
    memset(s, 0, sizeof *s);
    s->number_of_photons = f->number_of_photons;
    s->n_regions = f->n_regions;
    s->regions = regions;
    for (int i = 0; i < f->n_regions; ++i) {
        regions[i].n = f->region_n[i];
        regions[i].mua = f->region_mua[i];
        regions[i].mus = f->region_mus[i];
        regions[i].g = f->region_g[i];
        regions[i].mutr = f->region_mutr[i];
    }
    s->TypeSimulation = (short)f->type_simulation;
    s->TypeBias = (short)f->type_bias;
    s->RecordPhotonsFlag = (short)f->record_photons_flag;
    s->NumOpticalDepthLengthSteps = (short)f->num_optical_depth_length_steps;
    s->BackwardBiasCoefficient = f->backward_bias_coefficient;
    s->TargetDepthMin = f->target_depth_min;
    s->TargetDepthMax = f->target_depth_max;
    s->CoherenceLengthSource = f->coherence_length_source;
    s->MaxCollectingRadius = f->max_collecting_radius;
    s->MaxCollectingAngleDeg = f->max_collecting_angle_deg;
    s->ProbabilityAdditionalBias = f->probability_additional_bias;
    s->MaxRelativeContributionToBinPerPostProcessedSample = f->max_relative_contribution;
    s->MaxFilteredOpticalDepth = f->max_filtered_optical_depth;
    s->OpticalDepthShift = f->optical_depth_shift;
    s->rndStepSizeInTissue = f->rnd_step_size_in_tissue;
    s->probe.start_x = f->start_x;
    s->probe.distance_Ascans = f->step_x;
    s->probe.end_x = f->end_x;
    s->probe.current_scanning_x = f->start_x;
}

static void mesh_to_ref(const RefMesh *m, std::vector<TetrahedronStructGPU> &tets,
                        std::vector<TriangleFaces> &faces) {
    tets.resize(m->n_tets);
    for (int i = 0; i < m->n_tets; ++i) {
        const int32_t *t = m->tet + 14 * (size_t)i;
        tets[i].idx = t[0];
        tets[i].region = t[1];
        for (int k = 0; k < 4; ++k) {
            tets[i].faces[k] = t[2 + k];
            tets[i].signs[k] = t[6 + k];
            tets[i].adjTetras[k] = t[10 + k];
        }
    }
    faces.assign(m->n_faces, TriangleFaces());
    for (int i = 0; i < m->n_faces; ++i) {
        faces[i].idx = i;
        faces[i].Nx = m->face[4 * (size_t)i + 0];
        faces[i].Ny = m->face[4 * (size_t)i + 1];
        faces[i].Nz = m->face[4 * (size_t)i + 2];
        faces[i].d = m->face[4 * (size_t)i + 3];
    }
}

extern "C" {

int ref_num_threads_per_block(void) { return NUM_THREADS_PER_BLOCK; }

// init_RNG, src/octmps_kernel.cuh:52-172.
int ref_init_rng(uint64_t *x, uint32_t *a, uint64_t *xR, uint32_t *aR, uint64_t *xS,
                 uint32_t *aS, uint32_t n, const char *path, uint64_t seed) {
    return init_RNG((UINT64 *)x, a, (UINT64 *)xR, aR, (UINT64 *)xS, aS, n, path, seed);
}

// read_simulation_data (src/octmps_io.cpp:504-645) + Bias_Read
// (src/bias.cpp:9-110), flattened.
int ref_parse(const char *opt_path, const char *mci_path, RefSim *out) {
    SimulationStruct *sims = NULL;
    int n = read_simulation_data((char *)opt_path, &sims);
    if (n <= 0) return 1;
    if (!Bias_Read((char *)mci_path, &sims)) return 2;
    SimulationStruct *s = &sims[0];
    memset(out, 0, sizeof *out);
    out->start_x = s->probe.start_x;
    out->step_x = s->probe.distance_Ascans;
    out->end_x = s->probe.end_x;
    out->number_of_photons = s->number_of_photons;
    out->n_regions = (int32_t)s->n_regions;
    for (UINT32 i = 0; i < s->n_regions && i < MAX_REGIONS; ++i) {
        out->region_n[i] = s->regions[i].n;
        out->region_mua[i] = i ? s->regions[i].mua : 0.0;
        out->region_mus[i] = i ? s->regions[i].mus : 0.0;
        out->region_g[i] = i ? s->regions[i].g : 0.0;
        out->region_mutr[i] = i ? s->regions[i].mutr : 0.0;
    }
    out->type_simulation = s->TypeSimulation;
    out->type_bias = s->TypeBias;
    out->record_photons_flag = s->RecordPhotonsFlag;
    out->num_optical_depth_length_steps = s->NumOpticalDepthLengthSteps;
    out->backward_bias_coefficient = s->BackwardBiasCoefficient;
    out->target_depth_min = s->TargetDepthMin;
    out->target_depth_max = s->TargetDepthMax;
    out->coherence_length_source = s->CoherenceLengthSource;
    out->max_collecting_radius = s->MaxCollectingRadius;
    out->max_collecting_angle_deg = s->MaxCollectingAngleDeg;
    out->probability_additional_bias = s->ProbabilityAdditionalBias;
    out->max_relative_contribution = s->MaxRelativeContributionToBinPerPostProcessedSample;
    out->max_filtered_optical_depth = s->MaxFilteredOpticalDepth;
    out->optical_depth_shift = s->OpticalDepthShift;
    out->rnd_step_size_in_tissue = 0.0;
    return 0;
}

int ref_mesh_counts(const char *mesh_path, int32_t *n_vertices, int32_t *n_tets) {
    int nv = 0, nt = 0;
    if (!read_mesh_param((char *)mesh_path, &nv, &nt)) return 1;
    *n_vertices = nv;
    *n_tets = nt;
    return 0;
}

// MeshGraph + FindRootofGraph + SerializeGraph (src/mesh.cpp), exactly as
// main() chains them (src/main.cu:943-963).  tet_out: [n_tets*14],
// face_out: [4*n_tets*4] (faces never filled stay zero).  Returns the root
// tet index in *root (or -1 when FindRootofGraph fails).
int ref_mesh_build(const char *mesh_path, double probe_x, double probe_y, double probe_z,
                   int32_t *tet_out, double *face_out, int32_t *root) {
    int nv = 0, nt = 0;
    if (!read_mesh_param((char *)mesh_path, &nv, &nt)) return 1;
    SimulationStruct sim;
    memset(&sim, 0, sizeof sim);
    SimulationStruct *psim = &sim;
    TetrahedronStruct *graph = MeshGraph((char *)mesh_path, &psim);
    if (!graph) return 2;
    sim.probe_x = probe_x;
    sim.probe_y = probe_y;
    sim.probe_z = probe_z;
    TetrahedronStruct *r = FindRootofGraph(graph, &psim);
    *root = r ? r->index : -1;
    if (!r) r = graph;  // serialise anyway so the layout can still be compared
    std::vector<Vertex> verts(nv);
    std::vector<TriangleFaces> faces(4 * (size_t)nt);
    memset(faces.data(), 0, faces.size() * sizeof(TriangleFaces));
    std::vector<TetrahedronStructGPU> tets(nt);
    SerializeGraph(r, nv, 4 * nt, nt, verts.data(), faces.data(), tets.data());
    for (int i = 0; i < nt; ++i) {
        int32_t *t = tet_out + 14 * (size_t)i;
        t[0] = tets[i].idx;
        t[1] = tets[i].region;
        for (int k = 0; k < 4; ++k) {
            t[2 + k] = tets[i].faces[k];
            t[6 + k] = tets[i].signs[k];
            t[10 + k] = tets[i].adjTetras[k];
        }
    }
    for (size_t i = 0; i < faces.size(); ++i) {
        face_out[4 * i + 0] = faces[i].Nx;
        face_out[4 * i + 1] = faces[i].Ny;
        face_out[4 * i + 2] = faces[i].Nz;
        face_out[4 * i + 3] = faces[i].d;
    }
    return 0;
}

// MeshGraph + SerializeGraph once, then FindRootofGraph for each of n_probes
// probe positions (x, 0, 0), as main() chains them for a B-scan
// (src/main.cu:943-963, 948-955).  FindRootofGraph loops over
// SimulationStruct::num_tetrahedrons, a short (src/octmps.h:95), which
// wraps for meshes above 32,767 tets; the search here runs the same
// function over the first min(T, 32767) tets, which is the reference's
// result with a wide counter whenever the root lies among them (the
// generated meshes write the probe's surface layer first).  roots[k] = -1
// where it returns no tet.  tet_out: [n_tets*14]; face_out: [4*n_tets*4].
int ref_mesh_build_roots(const char *mesh_path, int32_t n_probes, const double *probe_x,
                         int32_t *tet_out, double *face_out, int32_t *roots) {
    int nv = 0, nt = 0;
    if (!read_mesh_param((char *)mesh_path, &nv, &nt)) return 1;
    SimulationStruct sim;
    memset(&sim, 0, sizeof sim);
    SimulationStruct *psim = &sim;
    TetrahedronStruct *graph = MeshGraph((char *)mesh_path, &psim);
    if (!graph) return 2;
    sim.num_tetrahedrons = (short)(nt < 32767 ? nt : 32767);
    for (int32_t k = 0; k < n_probes; ++k) {
        sim.probe_x = probe_x[k];
        sim.probe_y = 0.0;
        sim.probe_z = 0.0;
        TetrahedronStruct *r = FindRootofGraph(graph, &psim);
        roots[k] = r ? r->index : -1;
    }
    std::vector<Vertex> verts(nv);
    std::vector<TriangleFaces> faces(4 * (size_t)nt);
    memset(faces.data(), 0, faces.size() * sizeof(TriangleFaces));
    std::vector<TetrahedronStructGPU> tets(nt);
    SerializeGraph(graph, nv, 4 * nt, nt, verts.data(), faces.data(), tets.data());
    for (int i = 0; i < nt; ++i) {
        int32_t *t = tet_out + 14 * (size_t)i;
        t[0] = tets[i].idx;
        t[1] = tets[i].region;
        for (int k = 0; k < 4; ++k) {
            t[2 + k] = tets[i].faces[k];
            t[6 + k] = tets[i].signs[k];
            t[10 + k] = tets[i].adjTetras[k];
        }
    }
    for (size_t i = 0; i < faces.size(); ++i) {
        face_out[4 * i + 0] = faces[i].Nx;
        face_out[4 * i + 1] = faces[i].Ny;
        face_out[4 * i + 2] = faces[i].Nz;
        face_out[4 * i + 3] = faces[i].d;
    }
    return 0;
}

// One A-scan through the reference's kernels, as RunGPUi does it
// (src/main.cu:43-660): InitDeviceConstantMemory, InitThreadState over the
// grid, then OCTMPSKernel relaunched until n_photons_left reaches 0
// (src/main.cu:572-623).  Each launch runs the grid's n_blocks*600 threads
// on `n_threads` OpenMP threads.  rng_*: [n_blocks*600] per-lane state from
// init_RNG.  *seconds gets the wall time of the relaunch loop only.
int ref_run(const RefSim *fs, const RefMesh *mesh, double probe_x, double probe_y,
            double probe_z, uint32_t n_blocks, uint64_t *rng_x, uint32_t *rng_a,
            uint64_t *rng_xR, uint32_t *rng_aR, uint64_t *rng_xS, uint32_t *rng_aS,
            int n_threads, RefTally *out, double *seconds, uint32_t *launches) {
    static RegionStruct regions[MAX_REGIONS];
    SimulationStruct sim;
    sim_from_flat(fs, &sim, regions);
    std::vector<TetrahedronStructGPU> tets;
    std::vector<TriangleFaces> faces;
    mesh_to_ref(mesh, tets, faces);

    const uint32_t n_lanes = n_blocks * NUM_THREADS_PER_BLOCK;
    int region = tets[mesh->root].region;
    sim.Rspecular = Rspecular(sim.regions[0].n, sim.regions[region].n);
    sim.rootIdx = mesh->root;
    sim.probe_x = probe_x;
    sim.probe_y = probe_y;
    sim.probe_z = probe_z;
    if (InitDeviceConstantMemory(&sim)) return 1;

    const int nb = sim.NumOpticalDepthLengthSteps;
    std::vector<UINT64> c1(nb + 1, 0), c2(nb + 1, 0);
    std::vector<FLOAT> s1(nb + 2, 0), m1(nb + 2, 0), q1(nb + 2, 0), s2(nb + 2, 0),
        m2(nb + 2, 0), q2(nb + 2, 0);
    UINT32 n_left = sim.number_of_photons;
    SimState st;
    memset(&st, 0, sizeof st);
    st.probe_x = probe_x;
    st.probe_y = probe_y;
    st.probe_z = probe_z;
    st.n_photons_left = &n_left;
    st.x = (UINT64 *)rng_x;
    st.a = rng_a;
    st.xR = (UINT64 *)rng_xR;
    st.aR = rng_aR;
    st.xS = (UINT64 *)rng_xS;
    st.aS = rng_aS;
    st.NumClassI_PhotonsFilteredInRange = c1.data();
    st.NumClassII_PhotonsFilteredInRange = c2.data();
    st.ReflectanceClassI_Sum = s1.data();
    st.ReflectanceClassI_Max = m1.data();
    st.ReflectanceClassI_SumSq = q1.data();
    st.ReflectanceClassII_Sum = s2.data();
    st.ReflectanceClassII_Max = m2.data();
    st.ReflectanceClassII_SumSq = q2.data();

    // GPUThreadStates: one SoA array per field (src/octmps_kernel.h:152-217).
    std::vector<int> nt_(n_lanes), nt_c(n_lanes);
    std::vector<UINT32> u32[11];
    for (auto &v : u32) v.assign(n_lanes, 0);
    std::vector<FLOAT> f64[27];
    for (auto &v : f64) v.assign(n_lanes, 0.0);
    GPUThreadStates ts;
    memset(&ts, 0, sizeof ts);
    ts.NextTetrahedron = nt_.data();
    ts.NextTetrahedron_cont = nt_c.data();
    ts.is_active = u32[0].data();
    ts.dead = u32[1].data();
    ts.hit = u32[2].data();
    ts.photon_region = u32[3].data();
    ts.rootIdx = u32[4].data();
    ts.FstBackReflectionFlag = u32[5].data();
    ts.NumBackwardsSpecularReflections = u32[6].data();
    ts.dead_cont = u32[7].data();
    ts.rootIdx_cont = u32[8].data();
    ts.FstBackReflectionFlag_cont = u32[9].data();
    ts.NumBackwardsSpecularReflections_cont = u32[10].data();
    FLOAT **fp[] = {&ts.photon_x, &ts.photon_y, &ts.photon_z, &ts.photon_x_cont,
                    &ts.photon_y_cont, &ts.photon_z_cont, &ts.photon_ux, &ts.photon_uy,
                    &ts.photon_uz, &ts.photon_ux_cont, &ts.photon_uy_cont,
                    &ts.photon_uz_cont, &ts.photon_w, &ts.photon_s, &ts.photon_sleft,
                    &ts.photon_w_cont, &ts.photon_s_cont, &ts.photon_sleft_cont, &ts.MinCos,
                    &ts.OpticalPath, &ts.MaxDepth, &ts.LikelihoodRatio, &ts.LocationFstBias,
                    &ts.MinCos_cont, &ts.OpticalPath_cont, &ts.MaxDepth_cont,
                    &ts.LikelihoodRatio_cont};
    for (int i = 0; i < 27; ++i) *fp[i] = f64[i].data();
    std::vector<FLOAT> lr_after(n_lanes), loc_cont(n_lanes);
    ts.LikelihoodRatioAfterFstBias = lr_after.data();
    ts.LocationFstBias_cont = loc_cont.data();
    ts.tetrahedron = tets.data();
    ts.faces = faces.data();

    gridDim.x = n_blocks;
    blockDim.x = NUM_THREADS_PER_BLOCK;
    if (n_threads > 0) omp_set_num_threads(n_threads);

#pragma omp parallel for schedule(static)
    for (int64_t tid = 0; tid < (int64_t)n_lanes; ++tid) {
        blockIdx.x = (unsigned)(tid / NUM_THREADS_PER_BLOCK);
        threadIdx.x = (unsigned)(tid % NUM_THREADS_PER_BLOCK);
        InitThreadState(&ts, probe_x, probe_y, probe_z);
    }
    auto t0 = std::chrono::steady_clock::now();
    uint32_t nl = 0;
    while (__atomic_load_n(&n_left, __ATOMIC_SEQ_CST) > 0) {
#pragma omp parallel for schedule(dynamic, 64)
        for (int64_t tid = 0; tid < (int64_t)n_lanes; ++tid) {
            blockIdx.x = (unsigned)(tid / NUM_THREADS_PER_BLOCK);
            threadIdx.x = (unsigned)(tid % NUM_THREADS_PER_BLOCK);
            OCTMPSKernel(&st, &ts);
        }
        ++nl;
    }
    auto t1 = std::chrono::steady_clock::now();
    if (seconds) *seconds = std::chrono::duration<double>(t1 - t0).count();
    if (launches) *launches = nl;

    out->num_filtered = st.NumFilteredPhotons;
    out->num_filtered_class1 = st.NumFilteredPhotonsClassI;
    out->num_filtered_class2 = st.NumFilteredPhotonsClassII;
    memcpy(out->count1, c1.data(), c1.size() * sizeof(uint64_t));
    memcpy(out->count2, c2.data(), c2.size() * sizeof(uint64_t));
    memcpy(out->sum1, s1.data(), s1.size() * sizeof(double));
    memcpy(out->max1, m1.data(), m1.size() * sizeof(double));
    memcpy(out->sumsq1, q1.data(), q1.size() * sizeof(double));
    memcpy(out->sum2, s2.data(), s2.size() * sizeof(double));
    memcpy(out->max2, m2.data(), m2.size() * sizeof(double));
    memcpy(out->sumsq2, q2.data(), q2.size() * sizeof(double));
    return 0;
}

// Per-lane record of one packet (the first packet a lane launches, with
// every split copy it restores), so that event sequences can be compared
// with the restatement.  The loop body follows OCTMPSKernel
// (src/octmps_kernel.cuh:1349-1392) call for call.
struct PacketRecord {
    uint64_t hash;       // FNV-1a over (tet, event) per step
    uint64_t x, xR, xS;  // generator states when the packet ends
    uint32_t steps, hits, scatters, restores, detections, survivals;
    double contribution;  // sum of w*(1-R)*LR over the packet's detections
    double optical_path;  // OpticalPath when the packet ends
};

enum { EV_SCATTER = 1, EV_TRANSMIT = 2, EV_REFLECT = 3, EV_EXIT = 4, EV_DETECT = 8,
       EV_SURVIVE = 16, EV_RESTORE = 32, EV_END = 64 };

static inline uint64_t fnv(uint64_t h, uint64_t v) {
    for (int i = 0; i < 8; ++i) {
        h ^= (v >> (8 * i)) & 0xff;
        h *= 1099511628211ull;
    }
    return h;
}

int ref_trace_first_packets(const RefSim *fs, const RefMesh *mesh, double probe_x,
                            double probe_y, double probe_z, uint32_t n_lanes,
                            const uint64_t *rng_x, const uint32_t *rng_a,
                            const uint64_t *rng_xR, const uint32_t *rng_aR,
                            const uint64_t *rng_xS, const uint32_t *rng_aS,
                            uint32_t max_steps, PacketRecord *out, int64_t dump_lane,
                            double *dump, uint32_t dump_max) {
    static RegionStruct regions[MAX_REGIONS];
    SimulationStruct sim;
    sim_from_flat(fs, &sim, regions);
    std::vector<TetrahedronStructGPU> tets;
    std::vector<TriangleFaces> faces;
    mesh_to_ref(mesh, tets, faces);
    int region = tets[mesh->root].region;
    sim.Rspecular = Rspecular(sim.regions[0].n, sim.regions[region].n);
    sim.rootIdx = mesh->root;
    if (InitDeviceConstantMemory(&sim)) return 1;
    const int nb = sim.NumOpticalDepthLengthSteps;

#pragma omp parallel for schedule(dynamic, 16)
    for (int64_t lane = 0; lane < (int64_t)n_lanes; ++lane) {
        std::vector<UINT64> c1(nb + 1, 0), c2(nb + 1, 0);
        std::vector<FLOAT> s1(nb + 2, 0), m1(nb + 2, 0), q1(nb + 2, 0), s2(nb + 2, 0),
            m2(nb + 2, 0), q2(nb + 2, 0);
        SimState st;
        memset(&st, 0, sizeof st);
        st.NumClassI_PhotonsFilteredInRange = c1.data();
        st.NumClassII_PhotonsFilteredInRange = c2.data();
        st.ReflectanceClassI_Sum = s1.data();
        st.ReflectanceClassI_Max = m1.data();
        st.ReflectanceClassI_SumSq = q1.data();
        st.ReflectanceClassII_Sum = s2.data();
        st.ReflectanceClassII_Max = m2.data();
        st.ReflectanceClassII_SumSq = q2.data();

        UINT64 x = rng_x[lane], xR = rng_xR[lane], xS = rng_xS[lane];
        UINT32 a = rng_a[lane], aR = rng_aR[lane], aS = rng_aS[lane];
        PhotonStructGPU photon, photon_cont;
        LaunchPhoton(&photon, probe_x, probe_y, probe_z);
        photon.tetrahedron = tets.data();
        photon.faces = faces.data();
        photon_cont = photon;  // InitThreadState fills the _cont slots alike

        PacketRecord rec;
        memset(&rec, 0, sizeof rec);
        rec.hash = 14695981039346656037ull;
        for (uint32_t step = 0; step < max_steps; ++step) {
            uint32_t ev = 0;
            UINT64 det_before = st.NumFilteredPhotons;
            ComputeStepSize(&photon, &x, &a);
            photon.hit = HitBoundary(&photon);
            Hop(&photon);
            if (photon.hit) {
                ++rec.hits;
                UINT32 before = photon.rootIdx;
                int next = photon.tetrahedron[before].adjTetras[photon.NextTetrahedron];
                double w0 = photon.w;
                FastReflectTransmit(&photon, &st, &xR, &aR, probe_x, probe_y, probe_z);
                // The exterior branch taken when R < 1 (src/octmps_kernel.cuh:662)
                // is the only one that scales the weight by R.
                if (photon.rootIdx != before) ev = EV_TRANSMIT;
                else if (next == -1 && photon.w != w0) ev = EV_EXIT;
                else ev = EV_REFLECT;
                if (st.NumFilteredPhotons != det_before) {
                    ev |= EV_DETECT;
                    ++rec.detections;
                }
            } else {
                ++rec.scatters;
                ev = EV_SCATTER;
                Drop(&photon);
                switch (d_simparam.TypeBias) {
                    case 0:
                        Spin(d_regionspecs[photon.tetrahedron[photon.rootIdx].region].g,
                             &photon, &xS, &aS);
                        break;
                    case 37:
                        SpinBias(d_regionspecs[photon.tetrahedron[photon.rootIdx].region].g,
                                 photon.tetrahedron[photon.rootIdx].region, &photon,
                                 &photon_cont, &xS, &aS, probe_x, probe_y, probe_z);
                        break;
                }
            }
            bool end = false;
            if (photon.w < WEIGHT) {
                FLOAT rand = rand_MWC_co(&x, &a);
                if (photon.w != ZERO_FP && rand < CHANCE) {
                    photon.w *= (FLOAT)FAST_DIV(FP_ONE, CHANCE);
                    ev |= EV_SURVIVE;
                    ++rec.survivals;
                } else if (photon.FstBackReflectionFlag && d_simparam.TypeBias != 3) {
                    FLOAT LikelihoodRatioTmp = photon.LikelihoodRatioAfterFstBias;
                    CopyPhotonStruct(&photon_cont, &photon);
                    Spin(d_regionspecs[photon.tetrahedron[photon.rootIdx].region].g, &photon,
                         &xS, &aS);
                    if (LikelihoodRatioTmp < 1)
                        photon.LikelihoodRatio = 1 - LikelihoodRatioTmp;
                    else
                        photon.LikelihoodRatio = 1;
                    ev |= EV_RESTORE;
                    ++rec.restores;
                } else {
                    ev |= EV_END;
                    end = true;
                }
            }
            rec.hash = fnv(rec.hash, ((uint64_t)photon.rootIdx << 8) | ev);
            if (dump && lane == dump_lane && rec.steps < dump_max) {
                double *d = dump + 12 * (size_t)rec.steps;
                d[0] = photon.rootIdx; d[1] = ev; d[2] = photon.x; d[3] = photon.y; d[4] = photon.z;
                d[5] = photon.ux; d[6] = photon.uy; d[7] = photon.uz; d[8] = photon.w;
                d[9] = photon.s; d[10] = photon.OpticalPath; d[11] = photon.LikelihoodRatio;
            }
            ++rec.steps;
            if (end) break;
        }
        double total = 0;
        for (int i = 0; i < nb + 2; ++i) total += s1[i] + s2[i];
        rec.contribution = total;
        rec.optical_path = photon.OpticalPath;
        rec.x = x;
        rec.xR = xR;
        rec.xS = xS;
        out[lane] = rec;
    }
    return 0;
}

// WriteResult + Write_Bias_Parameters (src/octmps_io.cpp:237-437) for one
// A-scan at probe x, writing into the current directory as the reference
// does.
int ref_write_result(const RefSim *fs, double probe_x, const RefTally *t) {
    static RegionStruct regions[MAX_REGIONS];
    SimulationStruct sim;
    sim_from_flat(fs, &sim, regions);
    sim.probe.current_scanning_x = probe_x;
    const int nb = sim.NumOpticalDepthLengthSteps;
    SimState st;
    memset(&st, 0, sizeof st);
    st.NumFilteredPhotons = t->num_filtered;
    st.NumFilteredPhotonsClassI = t->num_filtered_class1;
    st.NumFilteredPhotonsClassII = t->num_filtered_class2;
    std::vector<UINT64> c1(t->count1, t->count1 + nb + 1), c2(t->count2, t->count2 + nb + 1);
    std::vector<FLOAT> s1(t->sum1, t->sum1 + nb + 2), m1(t->max1, t->max1 + nb + 2),
        q1(t->sumsq1, t->sumsq1 + nb + 2), s2(t->sum2, t->sum2 + nb + 2),
        m2(t->max2, t->max2 + nb + 2), q2(t->sumsq2, t->sumsq2 + nb + 2);
    std::vector<FLOAT> r1(nb, 0), r2(nb, 0), ms1(nb, 0), mq1(nb, 0), ms2(nb, 0), mq2(nb, 0);
    st.NumClassI_PhotonsFilteredInRange = c1.data();
    st.NumClassII_PhotonsFilteredInRange = c2.data();
    st.ReflectanceClassI_Sum = s1.data();
    st.ReflectanceClassI_Max = m1.data();
    st.ReflectanceClassI_SumSq = q1.data();
    st.ReflectanceClassII_Sum = s2.data();
    st.ReflectanceClassII_Max = m2.data();
    st.ReflectanceClassII_SumSq = q2.data();
    st.ReflectanceClassI = r1.data();
    st.ReflectanceClassII = r2.data();
    st.MeanReflectanceClassI_Sum = ms1.data();
    st.MeanReflectanceClassI_SumSq = mq1.data();
    st.MeanReflectanceClassII_Sum = ms2.data();
    st.MeanReflectanceClassII_SumSq = mq2.data();
    Write_Bias_Parameters(&st, &sim, 0.0f);
    if (sim.output_file_ptr) fclose(sim.output_file_ptr);
    float tr = 0;
    WriteResult(&sim, &st, &tr);
    return 0;
}

}  // extern "C"
