// Seeding of the per-lane multiply-with-carry generators, bit-identical to
// init_RNG (src/octmps_kernel.cuh:52-172), with the multiplier table passed
// in memory instead of read from safeprimes_base32.txt.
//
// The first three multipliers drive three seeding generators, one per
// stream (general: seeded by the job's seed; reflect/transmit and spin:
// fixed seeds 3858638025 and 2658951225, src/octmps_kernel.h:8-9).  Lane i
// takes multipliers 3+3i, 4+3i, 5+3i and draws its carry
// floor(u/2^32 * a) and its state u' from its stream's seeding generator,
// redrawing while the pair is invalid for a generator with multiplier a.
#include <cmath>

#include "octmps_host.h"

namespace {

inline bool invalid(uint64_t x, uint32_t a) {
    return (x == 0) | (((uint32_t)(x >> 32)) >= (a - 1)) | (((uint32_t)x) >= 0xfffffffful);
}

inline uint64_t seed_lane(uint64_t *xinit, uint32_t begin, uint32_t a) {
    uint64_t x = 0;
    while (invalid(x, a)) {
        *xinit = (*xinit & 0xffffffffull) * begin + (*xinit >> 32);
        x = (uint32_t)floor((((double)((uint32_t)*xinit)) / (double)0x100000000) * a);
        x = x << 32;
        *xinit = (*xinit & 0xffffffffull) * begin + (*xinit >> 32);
        x += (uint32_t)*xinit;
    }
    return x;
}

}  // namespace

extern "C" octmps_status octmps_rng_init(const uint32_t *m, uint64_t n_multipliers, uint32_t n_lanes,
                                         uint64_t seed, octmps_rng_lanes *out) {
    if (!m || !out || !out->x || !out->a || !out->xR || !out->aR || !out->xS || !out->aS)
        return OCTMPS_ERR_INVALID_ARG;
    if (n_multipliers < 3 + 3 * (uint64_t)n_lanes) return OCTMPS_ERR_INVALID_ARG;
    const uint32_t begin = m[0], beginR = m[1], beginS = m[2];
    uint64_t xinit = seed, xinitR = 3858638025ull, xinitS = 2658951225ull;
    if ((xinit == 0ull) | (((uint32_t)(xinit >> 32)) >= (begin - 1)) |
        (((uint32_t)xinit) >= 0xfffffffful))
        return OCTMPS_ERR_INVALID_ARG;  // "not a valid seed"
    for (uint32_t i = 0; i < n_lanes; ++i) {
        const uint32_t fora = m[3 + 3 * (uint64_t)i];
        const uint32_t forR = m[4 + 3 * (uint64_t)i];
        const uint32_t forS = m[5 + 3 * (uint64_t)i];
        out->a[i] = fora;
        out->aR[i] = forR;
        out->aS[i] = forS;
        out->x[i] = seed_lane(&xinit, begin, fora);
        out->xR[i] = seed_lane(&xinitR, beginR, forR);
        out->xS[i] = seed_lane(&xinitS, beginS, forS);
    }
    return OCTMPS_OK;
}
