// Per-region constants of a job, derived on the host (runtime.cu, noalloc.cu).
//
// The first five are InitDeviceConstantMemory's (src/octmps_kernel.cuh:204-214)
// from read_simulation_data's mutr (src/octmps_io.cpp:625-626).  The other two
// are terms of the biased spin (src/octmps_kernel.cuh:881-896, 898-1086) that
// do not change during a job and cost a square root or a logarithm: sqrt(1 +
// b^2) of the bias coefficient b, and -log(rndStepSizeInTissue) / mu_t.  They
// are evaluated here with the kernel's own operations in the kernel's order
// (the FP32 forms' fused multiply-adds, the FP64 form's separately rounded
// products and sums and its round-down division, correctly rounded square
// root, the project's logarithm), so the kernel reads exactly the values it
// would otherwise recompute at every scattering.
#ifndef OCTMPS_REGION_CONSTS_H
#define OCTMPS_REGION_CONSTS_H

#include <cfloat>
#include <cmath>
#include <vector>

#include "kernel_iface.h"
#include "octmps_capi.h"
#include "photon_math.cuh"

namespace octmps {

// a / b rounded toward minus infinity (the reference's FAST_DIV in FP64,
// src/octmps_kernel.h:38): the nearest quotient, stepped down when the exact
// remainder shows it above the true value.
inline double div_rd(double a, double b) {
    double q = a / b;
    if (!std::isfinite(q) || q == 0.0) return q;
    double r = std::fma(-q, b, a);
    if (r != 0.0 && ((r < 0.0) == (b > 0.0))) q = std::nextafter(q, -INFINITY);
    return q;
}

// The kernel's DevNum<T> operations, on the host.
template <typename T>
struct HostNum;
template <>
struct HostNum<float> {
    static float mad(float a, float b, float c) { return std::fma(a, b, c); }
    static float div(float a, float b) { return a / b; }
};
template <>
struct HostNum<double> {
    static double mad(double a, double b, double c) {
        const double p = a * b;  // rounded on its own (built with -ffp-contract=off)
        return p + c;
    }
    static double div(double a, double b) { return div_rd(a, b); }
};

template <typename T>
RegionConst<T> region_const(const octmps_region &reg, const octmps_sim &s) {
    using N = HostNum<T>;
    RegionConst<T> c;
    // read_simulation_data: a region without scattering (glass) gets DBL_MAX
    const double mutr = reg.mus == 0.0 ? DBL_MAX : 1.0 / (reg.mua + reg.mus);
    c.n = (T)reg.n;
    c.muas = (T)(1.0 / mutr);
    c.rmuas = (T)mutr;
    c.mua_muas = (T)(reg.mua * mutr);
    c.g = (T)reg.g;
    const T b = (T)s.backward_bias_coefficient;
    c.b_sq1p2 = std::sqrt(N::mad(b, b, (T)1));
    const T rs = (T)s.rnd_step_size_in_tissue;
    c.far = rs == (T)0 ? (T)INFINITY : N::div(-log_method(rs), c.muas);
    return c;
}

template <typename T>
void fill_region_consts(const octmps_sim &s, RegionConst<T> *out) {
    for (int i = 0; i < s.n_regions; ++i) out[i] = region_const<T>(s.regions[i], s);
}

}  // namespace octmps

#endif
