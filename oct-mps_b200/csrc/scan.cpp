// A-scans of a B-scan: the probe positions and their split over GPUs.
#include <cstdint>

#include "octmps_host.h"

// The probe positions of main()'s A-scan loop (src/main.cu:948-950): x from
// start_x while x < end_x, in steps of step_x added in double.  Writes at
// most max_out positions; returns how many there are (-1 for a step that
// never ends the loop).
extern "C" int64_t octmps_probe_positions(const octmps_sim *sim, double *out, uint64_t max_out) {
    if (!sim) return -1;
    if (!(sim->step_x > 0.0) && sim->start_x < sim->end_x) return -1;
    int64_t n = 0;
    for (double x = sim->start_x; x < sim->end_x; x += sim->step_x) {
        if (out && (uint64_t)n < max_out) out[n] = x;
        ++n;
    }
    return n;
}

// A-scans run by GPU `gpu` of `n_gpus` when a scan's A-scans are split over
// GPUs (the CLI's -G): round robin, k = gpu, gpu + n_gpus, ..., so that
// neighbouring positions, of similar cost, go to different GPUs.  The
// reference instead splits the photons of every A-scan over its GPUs
// (DoOneSimulation, src/main.cu:665-848).  Writes at most max_out indices;
// returns how many the GPU owns (-1 for invalid arguments).
extern "C" int64_t octmps_ascans_of_gpu(uint64_t n_ascans, uint32_t n_gpus, uint32_t gpu,
                                        uint64_t *out, uint64_t max_out) {
    if (n_gpus == 0 || gpu >= n_gpus) return -1;
    int64_t n = 0;
    for (uint64_t k = gpu; k < n_ascans; k += n_gpus) {
        if (out && (uint64_t)n < max_out) out[n] = k;
        ++n;
    }
    return n;
}
