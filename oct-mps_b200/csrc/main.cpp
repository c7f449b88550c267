// octmps: drop-in command line for the B200 library.
//
//   octmps [-S<seed>] [-G<num GPUs>] <input opt file> <input mesh file> <input bias file>
//
// Same arguments, inputs and output files as the reference's OCT-MPS
// (main, src/main.cu:850-1056; interpret_arg, src/octmps_io.cpp:105-145):
// reads safeprimes_base32.txt from the working directory, runs one A-scan
// per probe position x = start, start+step, ... < end (y = z = 0), and
// appends ClassI_Scatt.out, ClassII_Scatt.out, ClassI_ScattFilt.out,
// ClassII_ScattFilt.out (rewriting BiasParam.mco) A-scan by A-scan.
//
// Differences: all A-scans of the scan are submitted at once and run in
// one persistent launch per GPU instead of one launch sequence each; -G
// splits the A-scans (not the photons of one A-scan) over the GPUs.
// Extension flags the reference does not have: -P<0|1|2> selects the
// arithmetic (0 mixed FP32/FP64, the default; 1 all FP32; 2 all FP64),
// -L<lanes> the RNG lanes per A-scan (default 88800, the reference's lane
// count on a 148-SM GPU), -K<k> seeds A-scan k with seed+k (the reference
// reuses one seed for every A-scan).
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <thread>
#include <vector>

#include "octmps_capi.h"

namespace {

void usage(const char *prog) {
    printf("\nUsage: %s [-S<seed>] [-G<num GPUs>] <input opt file> <input mesh file> <input bias file>\n\n",
           prog);
    printf("  -S: seed for random number generation (MT only)\n");
    printf("  -G: set the number of GPUs this program uses\n");
    printf("\n");
    fflush(stdout);
}

struct Args {
    const char *opt = nullptr, *mesh = nullptr, *mci = nullptr;
    unsigned long long seed = 985456376ull;
    unsigned int gpus = 1;
    int precision = 0;
    unsigned int lanes = 88800;
    int seed_per_ascan = 0;
};

// interpret_arg, src/octmps_io.cpp:105-145.
int parse(int argc, char **argv, Args &a) {
    for (int i = 1; i < argc; ++i) {
        char *arg = argv[i];
        if (arg[0] != '-') {
            a.opt = arg;
            a.mesh = i + 1 < argc ? argv[i + 1] : nullptr;
            a.mci = i + 2 < argc ? argv[i + 2] : nullptr;
            break;
        }
        ++arg;
        int p = 0;
        unsigned int l = 0;
        if (sscanf(arg, "S%llu", &a.seed) == 1) {
        } else if (sscanf(arg, "G%u", &a.gpus) == 1) {
        } else if (sscanf(arg, "P%d", &p) == 1) {
            a.precision = p;
        } else if (sscanf(arg, "L%u", &l) == 1) {
            a.lanes = l;
        } else if (sscanf(arg, "K%d", &p) == 1) {
            a.seed_per_ascan = p;
        }
    }
    return a.opt == nullptr || a.mesh == nullptr || a.mci == nullptr;
}

}  // namespace

int main(int argc, char **argv) {
    printf("OCT-MPS on B200: per-photon Monte Carlo of OCT in tetrahedral meshes\n");
    Args A;
    if (parse(argc, argv, A)) {
        usage(argv[0]);
        return 1;
    }
    printf("\n====================================\n");
    printf("EXECUTION MODE:\n");
    printf("  seed#1 Step + Roulette:  %llu\n", A.seed);
    printf("  seed#2 ReflectTransmit:  %lu\n", 3858638025ul);
    printf("  seed#3 Spin:             %lu\n", 2658951225ul);
    printf("  # of GPUs:               %u\n", A.gpus);
    printf("====================================\n\n");

    octmps_sim sim;
    if (octmps_read_opt(A.opt, &sim) != OCTMPS_OK) {
        printf("Something wrong with read_simulation_data!\n");
        return 1;
    }
    if (octmps_read_mci(A.mci, &sim) != OCTMPS_OK) {
        printf("Something wrong with the bias reading, check file!\n");
        return 1;
    }
    auto t0 = std::chrono::steady_clock::now();
    octmps_host_mesh hm;
    if (octmps_mesh_build_file(A.mesh, &hm) != OCTMPS_OK) {
        printf("Something wrong with the meshing parameters!\n");
        return 1;
    }
    auto t1 = std::chrono::steady_clock::now();
    printf("\n====================================\n");
    printf("Mesh Parameters:\n");
    printf("No. of nodes=%d\n", hm.n_vertices);
    printf("No. of tetrahedrons=%d\n", hm.n_tets);
    printf("No. of faces=%d\n", hm.n_faces);
    printf("====================================\n");
    printf("Mesh graph is created in %.3f seconds.\n",
           std::chrono::duration<double>(t1 - t0).count());

    const uint64_t need = 3 + 3 * (uint64_t)A.lanes;
    std::vector<uint32_t> mult(need);
    const int64_t got = octmps_safeprimes_read("safeprimes_base32.txt", mult.data(), need);
    if (got < 0) {
        printf("Could not find the file of safeprimes (%s)! Terminating!\n", "safeprimes_base32.txt");
        return 1;
    }
    if ((uint64_t)got < need) {
        printf("safeprimes_base32.txt has %lld entries; %llu lanes need %llu.\n", (long long)got,
               (unsigned long long)A.lanes, (unsigned long long)need);
        return 1;
    }

    octmps_mesh_desc md{hm.n_tets, hm.n_faces, hm.tet_region, hm.tet_faces,
                        hm.tet_signs, hm.tet_adj, hm.face_plane};
    const int64_t n_xs = octmps_probe_positions(&sim, nullptr, 0);
    if (n_xs < 0) {
        printf("Something wrong with the probe scan parameters!\n");
        return 1;
    }
    std::vector<double> xs((size_t)n_xs);
    octmps_probe_positions(&sim, xs.data(), xs.size());
    std::vector<int32_t> roots(xs.size());
    for (size_t k = 0; k < xs.size(); ++k) {
        if (octmps_mesh_find_root(&md, xs[k], 0.0, 0.0, &roots[k]) != OCTMPS_OK) {
            printf("The probe at x=%G is not on a boundary face of the mesh.\n", xs[k]);
            return 1;
        }
    }

    int dev_count = 0;
    {
        octmps_ctx *probe = nullptr;
        for (int d = 0; d < 64; ++d) {
            if (octmps_ctx_create(d, &probe) != OCTMPS_OK) break;
            octmps_ctx_destroy(probe);
            ++dev_count;
        }
    }
    if (dev_count <= 0) {
        fprintf(stderr, "No GPU available. Quit.\n");
        return 1;
    }
    unsigned int ngpu = A.gpus < 1 ? 1 : A.gpus;
    if (ngpu > (unsigned)dev_count) {
        printf("The number of GPUs available is (%d).\n", dev_count);
        ngpu = (unsigned)dev_count;
    }

    const int nb = sim.num_optical_depth_length_steps;
    struct Result {
        std::vector<uint64_t> c1, c2;
        std::vector<double> s1, m1, q1, s2, m2, q2;
        octmps_tally t;
        octmps_status st = OCTMPS_OK;
        double ms = 0;
    };
    std::vector<Result> res(xs.size());
    for (auto &r : res) {
        r.c1.assign(nb + 1, 0);
        r.c2.assign(nb + 1, 0);
        for (auto *v : {&r.s1, &r.m1, &r.q1, &r.s2, &r.m2, &r.q2}) v->assign(nb + 2, 0.0);
        r.t = octmps_tally{0, 0, 0, r.c1.data(), r.c2.data(), r.s1.data(), r.m1.data(),
                           r.q1.data(), r.s2.data(), r.m2.data(), r.q2.data()};
    }
    // RecordPhotonsFlag: FilteredPhotons.mco collects the detected-packet
    // records of every A-scan of the run, written as each A-scan finishes
    // (lines carry the probe position, so their order does not matter).
    const bool record = (short)sim.record_photons_flag != 0;
    std::mutex record_mu;
    if (record) {
        FILE *fp = fopen("FilteredPhotons.mco", "w");
        if (fp) fclose(fp);
    }
    auto ts = std::chrono::steady_clock::now();
    std::vector<std::thread> threads;
    for (unsigned int g = 0; g < ngpu; ++g) {
        threads.emplace_back([&, g]() {
            std::vector<uint64_t> mine(xs.size());
            mine.resize((size_t)octmps_ascans_of_gpu(xs.size(), ngpu, g, mine.data(), mine.size()));
            octmps_ctx *ctx = nullptr;
            if (octmps_ctx_create((int)g, &ctx) != OCTMPS_OK) {
                for (uint64_t k : mine) res[k].st = OCTMPS_ERR_NO_DEVICE;
                return;
            }
            octmps_ctx_set_multipliers(ctx, mult.data(), mult.size());
            octmps_mesh_id mid = 0;
            octmps_status st = octmps_mesh_upload(ctx, &md, &mid);
            std::vector<octmps_job_id> ids(xs.size(), 0);
            for (uint64_t k : mine) {
                if (st != OCTMPS_OK) break;
                octmps_job jb;
                memset(&jb, 0, sizeof jb);
                jb.mesh = mid;
                jb.sim = &sim;
                jb.probe_x = xs[k];
                jb.root_tet = roots[k];
                jb.n_photons = sim.number_of_photons;
                jb.seed = A.seed + (A.seed_per_ascan ? (uint64_t)k : 0);
                jb.n_lanes = A.lanes;
                jb.precision = A.precision;
                st = octmps_job_submit(ctx, &jb, &ids[k]);
                if (st != OCTMPS_OK) fprintf(stderr, "[GPU %u] %s\n", g, octmps_last_error(ctx));
            }
            for (uint64_t k : mine) {
                if (st != OCTMPS_OK) {
                    res[k].st = st;
                    continue;
                }
                res[k].st = octmps_job_fetch(ctx, ids[k], &res[k].t);
                octmps_job_stats js;
                if (octmps_job_fetch_stats(ctx, ids[k], &js) == OCTMPS_OK) res[k].ms = js.device_ms;
                uint64_t kept = 0, detected = 0;
                if (record && res[k].st == OCTMPS_OK &&
                    octmps_job_photon_records(ctx, ids[k], nullptr, 0, &kept, &detected) == OCTMPS_OK) {
                    std::vector<octmps_photon_record> recs(kept);
                    if (octmps_job_photon_records(ctx, ids[k], recs.data(), kept, &kept, &detected) ==
                        OCTMPS_OK) {
                        std::lock_guard<std::mutex> lk(record_mu);
                        octmps_write_filtered_photons("", xs[k], recs.data(), kept);
                        if (detected > kept)
                            fprintf(stderr, "A-scan %llu: %llu of %llu detected packets recorded\n",
                                    (unsigned long long)k, (unsigned long long)kept,
                                    (unsigned long long)detected);
                    }
                }
                if (res[k].st != OCTMPS_OK)
                    fprintf(stderr, "[GPU %u] failure in OCTMPSKernel: %s\n", g, octmps_last_error(ctx));
                octmps_job_release(ctx, ids[k]);
            }
            octmps_ctx_destroy(ctx);
        });
    }
    for (auto &t : threads) t.join();
    auto te = std::chrono::steady_clock::now();
    const double elapsed = std::chrono::duration<double, std::milli>(te - ts).count();
    printf("\n\n>>>>>>Simulation time: %f (ms)\n", elapsed);
    int rc = 0;
    for (size_t k = 0; k < xs.size(); ++k) {
        if (res[k].st != OCTMPS_OK) {
            rc = 1;
            continue;
        }
        if (octmps_write_result("", &sim, xs[k], &res[k].t) != OCTMPS_OK) rc = 1;
    }
    octmps_mesh_host_free(&hm);
    return rc;
}
