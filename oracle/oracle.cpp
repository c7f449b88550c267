// CPU restatement of OCT-MPS's per-photon method.  TEST INFRASTRUCTURE
// ONLY: loaded by the tests, the smoke check and the bench's CPU leg, never
// by the product.  See oracle.h for what it covers and in which precisions.
//
// Build flags matter: -ffp-contract=off, so the only fused multiply-adds
// are the std::fma calls written below, and no fast-math.
#include "oracle.h"

#include <omp.h>

#include <cfloat>
#include <cmath>
#include <atomic>
#include <cstring>
#include <type_traits>
#include <vector>

namespace {

// Detected-packet records (oracle_set_photon_records), shared by all threads.
OraclePhotonRecord *g_records = nullptr;
uint64_t g_record_cap = 0;
std::atomic<uint64_t> g_record_n{0};

// ---------------------------------------------------------------- math ---

inline uint32_t f2u(float f) {
    uint32_t u;
    memcpy(&u, &f, 4);
    return u;
}
inline float u2f(uint32_t u) {
    float f;
    memcpy(&f, &u, 4);
    return f;
}
inline uint64_t d2u(double f) {
    uint64_t u;
    memcpy(&u, &f, 8);
    return u;
}
inline double u2d(uint64_t u) {
    double f;
    memcpy(&f, &u, 8);
    return f;
}

// Round-toward-minus-infinity quotient (the reference's FAST_DIV,
// src/octmps_kernel.h:38): the round-to-nearest quotient corrected by the
// sign of its exact FMA remainder.
inline double div_rd(double a, double b) {
    double q = a / b;
    if (!std::isfinite(q) || q == 0.0) return q;
    double r = std::fma(-q, b, a);
    if (r != 0.0 && ((r < 0.0) == (b > 0.0))) q = std::nextafter(q, -INFINITY);
    return q;
}

// float(u) rounded toward zero (__uint2float_rz, src/octmps_kernel.cuh:17).
inline float uint2float_rz(uint32_t u) {
    if (u >= (1u << 24)) {
        int lead = 31 - __builtin_clz(u);
        u &= ~((1u << (lead - 23)) - 1u);
    }
    return (float)u;
}

// Natural log by the atanh series.  x = m * 2^e with m in [sqrt(1/2),
// sqrt(2)); log(m) = 2 atanh(s), s = (m-1)/(m+1), |s| <= 0.1716, and
// 2 atanh(s) = 2s (1 + s^2/3 + s^4/5 + ...).  log 2 is split Cody-Waite
// style (high part with 16 significant bits, so e*LN2_HI is exact).
float logf_method(float x) {
    if (x == 0.0f) return -INFINITY;
    if (!(x > 0.0f) || std::isinf(x)) return x < 0.0f ? NAN : x;
    uint32_t b = f2u(x);
    int e = 0;
    if (b < 0x00800000u) {  // subnormal: scale by 2^23
        b = f2u(x * 0x1p23f);
        e = -23;
    }
    e += (int)(b >> 23) - 127;
    uint32_t mb = (b & 0x007fffffu) | 0x3f800000u;
    if (mb > 0x3fb504f3u) {  // m > sqrt(2): use m/2
        mb -= 0x00800000u;
        e += 1;
    }
    const float m = u2f(mb);
    const float f = m - 1.0f;  // exact
    const float s = f / (2.0f + f);
    const float z = s * s;
    const float t = s + s;
    float p = std::fma(z, 0x1.c71c72p-4f, 0x1.24924ap-3f);  // 1/9, 1/7
    p = std::fma(z, p, 0x1.99999ap-3f);                      // 1/5
    p = std::fma(z, p, 0x1.555556p-2f);                      // 1/3
    const float lm = std::fma(t * z, p, t);
    const float ef = (float)e;
    return std::fma(ef, 0x1.62e400p-1f, std::fma(ef, 0x1.7f7d1cp-20f, lm));
}

double log_method(double x) {
    if (x == 0.0) return -INFINITY;
    if (!(x > 0.0) || std::isinf(x)) return x < 0.0 ? NAN : x;
    uint64_t b = d2u(x);
    int e = 0;
    if (b < 0x0010000000000000ull) {  // subnormal: scale by 2^54
        b = d2u(x * 0x1p54);
        e = -54;
    }
    e += (int)(b >> 52) - 1023;
    uint64_t mb = (b & 0x000fffffffffffffull) | 0x3ff0000000000000ull;
    if (mb > 0x3ff6a09e667f3bcdull) {  // m > sqrt(2)
        mb -= 0x0010000000000000ull;
        e += 1;
    }
    const double m = u2d(mb);
    const double f = m - 1.0;
    const double s = f / (2.0 + f);
    const double z = s * s;
    const double t = s + s;
    double p = std::fma(z, 0x1.8618618618618p-5, 0x1.af286bca1af28p-5);  // 1/21, 1/19
    p = std::fma(z, p, 0x1.e1e1e1e1e1e1ep-5);                             // 1/17
    p = std::fma(z, p, 0x1.1111111111111p-4);                             // 1/15
    p = std::fma(z, p, 0x1.3b13b13b13b14p-4);                             // 1/13
    p = std::fma(z, p, 0x1.745d1745d1746p-4);                             // 1/11
    p = std::fma(z, p, 0x1.c71c71c71c71cp-4);                             // 1/9
    p = std::fma(z, p, 0x1.2492492492492p-3);                             // 1/7
    p = std::fma(z, p, 0x1.999999999999ap-3);                             // 1/5
    p = std::fma(z, p, 0x1.5555555555555p-2);                             // 1/3
    const double lm = std::fma(t * z, p, t);
    const double ef = (double)e;
    return std::fma(ef, 0x1.62e42fee00000p-1, std::fma(ef, 0x1.a39ef35793c76p-33, lm));
}

// Taylor polynomials of sin and cos on |r| <= pi/4 (+ a few ulps).
inline void sincos_poly_f(float r, float *s, float *c) {
    const float z = r * r;
    float ps = std::fma(z, 0x1.71de3ap-19f, -0x1.a01a02p-13f);  // 1/9!, -1/7!
    ps = std::fma(z, ps, 0x1.111112p-7f);                        // 1/5!
    ps = std::fma(z, ps, -0x1.555556p-3f);                       // -1/3!
    *s = std::fma(r * z, ps, r);
    float pc = std::fma(z, -0x1.27e4fcp-22f, 0x1.a01a02p-16f);  // -1/10!, 1/8!
    pc = std::fma(z, pc, -0x1.6c16c2p-10f);                      // -1/6!
    pc = std::fma(z, pc, 0x1.555556p-5f);                        // 1/4!
    pc = std::fma(z, pc, -0.5f);                                 // -1/2!
    *c = std::fma(z, pc, 1.0f);
}

inline void sincos_poly_d(double r, double *s, double *c) {
    const double z = r * r;
    double ps = std::fma(z, 0x1.952c77030ad4ap-49, -0x1.ae7f3e733b81fp-41);  // 1/17!, -1/15!
    ps = std::fma(z, ps, 0x1.6124613a86d09p-33);                              // 1/13!
    ps = std::fma(z, ps, -0x1.ae64567f544e4p-26);                             // -1/11!
    ps = std::fma(z, ps, 0x1.71de3a556c734p-19);                              // 1/9!
    ps = std::fma(z, ps, -0x1.a01a01a01a01ap-13);                             // -1/7!
    ps = std::fma(z, ps, 0x1.1111111111111p-7);                               // 1/5!
    ps = std::fma(z, ps, -0x1.5555555555555p-3);                              // -1/3!
    *s = std::fma(r * z, ps, r);
    double pc = std::fma(z, -0x1.6827863b97d97p-53, 0x1.ae7f3e733b81fp-45);  // -1/18!, 1/16!
    pc = std::fma(z, pc, -0x1.93974a8c07c9dp-37);                       // -1/14!
    pc = std::fma(z, pc, 0x1.1eed8eff8d898p-29);                        // 1/12!
    pc = std::fma(z, pc, -0x1.27e4fb7789f5cp-22);                       // -1/10!
    pc = std::fma(z, pc, 0x1.a01a01a01a01ap-16);                        // 1/8!
    pc = std::fma(z, pc, -0x1.6c16c16c16c17p-10);                       // -1/6!
    pc = std::fma(z, pc, 0x1.5555555555555p-5);                         // 1/4!
    pc = std::fma(z, pc, -0.5);                                         // -1/2!
    *c = std::fma(z, pc, 1.0);
}

// sin and cos of 2*pi*t for t in [0, 1): reduction in turns is exact
// (q = rint(4t), r = t - q/4), then the polynomials on 2*pi*r.
void sincos_turn_f(float t, float *s, float *c) {
    const float q = std::rint(t * 4.0f);
    const float r = std::fma(q, -0.25f, t);  // exact
    const float th = r * 0x1.921fb6p+2f;      // 2*pi rounded to float
    float sr, cr;
    sincos_poly_f(th, &sr, &cr);
    switch (((int)q) & 3) {
        case 0: *s = sr; *c = cr; break;
        case 1: *s = cr; *c = -sr; break;
        case 2: *s = -sr; *c = -cr; break;
        default: *s = -cr; *c = sr; break;
    }
}

// sin and cos of psi in [0, 2*pi): Cody-Waite reduction by pi/2 split in
// two doubles (the first product and difference are exact), then the
// polynomials.
void sincos_d(double psi, double *s, double *c) {
    const double q = std::rint(psi * 0x1.45f306dc9c883p-1);  // 2/pi
    double r = std::fma(-q, 0x1.921fb54442d18p+0, psi);      // pi/2 high
    r = std::fma(-q, 0x1.1a62633145c07p-54, r);              // pi/2 low
    double sr, cr;
    sincos_poly_d(r, &sr, &cr);
    switch (((int)q) & 3) {
        case 0: *s = sr; *c = cr; break;
        case 1: *s = cr; *c = -sr; break;
        case 2: *s = -sr; *c = -cr; break;
        default: *s = -cr; *c = sr; break;
    }
}

// -------------------------------------------------------- precision traits

template <typename T>
struct Num;

template <>
struct Num<float> {
    // a*b + c: fused (one rounding) in the FP32 forms
    static float mad(float a, float b, float c) { return std::fma(a, b, c); }
    static float div(float a, float b) { return a / b; }
    static float log(float x) { return logf_method(x); }
    // sin, cos of the azimuth 2*pi*rand (src/octmps_kernel.cuh:846-847)
    static void sincos_rand(float r, float *s, float *c) { sincos_turn_f(r, s, c); }
    static float rand_value(uint32_t u) { return uint2float_rz(u) * 0x1p-32f; }
    static constexpr float coszero = 0.999999f;
    static constexpr float cos90 = 1.0e-6f;
    static constexpr float weight = 1.0e-4f;
    static constexpr float chance = 0.1f;
    static constexpr float big = 1.0e10f;
};

template <>
struct Num<double> {
    // a*b + c: product and sum rounded separately, as the reference's
    // source evaluates it without contraction
    static double mad(double a, double b, double c) { return a * b + c; }
    static double div(double a, double b) { return div_rd(a, b); }
    static double log(double x) { return log_method(x); }
    static void sincos_rand(double r, double *s, double *c) {
        const double psi = (2.0 * 3.14159265359) * r;  // FP_TWO * PI_const * rand
        sincos_d(psi, s, c);
    }
    static double rand_value(uint32_t u) { return (double)uint2float_rz(u) * 0x1p-32; }
    static constexpr double coszero = 1.0 - 1.0e-14;  // (1.0F - 1.0E-14), src/octmps.h:29
    static constexpr double cos90 = 1.0e-6;
    static constexpr double weight = 1.0e-4;
    static constexpr double chance = 0.1;
    static constexpr double big = 1.0e10;
};

// MWC step (src/octmps_kernel.cuh:16) and the [0,1) value it yields.
template <typename T>
inline T rand_co(uint64_t *x, uint32_t a) {
    *x = (*x & 0xffffffffull) * a + (*x >> 32);
    return Num<T>::rand_value((uint32_t)*x);
}
template <typename T>
inline T rand_oc(uint64_t *x, uint32_t a) {
    return (T)1 - rand_co<T>(x, a);
}

// The FP32 forms (fused multiply-adds) also take a few cheaper but equally
// accurate formulations of the same quantities; the FP64 form keeps the
// reference's operations.
template <typename T>
struct FusedForm : std::is_same<T, float> {};
template <typename T>
constexpr bool kFused = FusedForm<T>::value;

// a.x + b.y + c.z evaluated left to right, (a.x + b.y) + c.z, as the
// reference writes its dot products; fused in the FP32 forms.
template <typename T>
inline T dot3(T a, T b, T c, T x, T y, T z) {
    return Num<T>::mad(c, z, Num<T>::mad(a, x, b * y));
}

inline uint64_t fnv(uint64_t h, uint64_t v) {
    for (int i = 0; i < 8; ++i) {
        h ^= (v >> (8 * i)) & 0xff;
        h *= 1099511628211ull;
    }
    return h;
}

// ------------------------------------------------------------ the method

template <typename T, typename P>
struct Region {
    T n, muas, rmuas, mua_muas, g;
};

template <typename T, typename P>
struct Photon {
    T x, y, z, ux, uy, uz, w, s, sleft, min_cos, max_depth, lr, lr_after, loc_fst;
    P optical_path;
    int32_t tet, next_face;
    uint32_t fst_flag, num_back;
};

template <typename T, typename P>
struct Tally {
    uint64_t nf = 0, nf1 = 0, nf2 = 0;
    std::vector<uint64_t> c1, c2;
    std::vector<P> s1, m1, q1, s2, m2, q2;
    uint64_t steps = 0, restores = 0, packets = 0, capped = 0;
    explicit Tally(int nb)
        : c1(nb + 1, 0), c2(nb + 1, 0), s1(nb + 2, 0), m1(nb + 2, 0), q1(nb + 2, 0),
          s2(nb + 2, 0), m2(nb + 2, 0), q2(nb + 2, 0) {}
};

template <typename T, typename P>
struct Setup {
    std::vector<T> planes;  // [n_tets*4*4], signed (inward) per tet and face
    const int32_t *adj;
    const int32_t *region;
    std::vector<Region<T, P>> regions;
    T n_ambient;
    int type_bias, nbins;
    T probe_x, probe_y, probe_z;
    T tdmin, tdmax, bias_a, p_bias, cos_collect, radius, w0, rnd_step;
    P shift, bin_width, half_lc;
    int32_t root;
};

template <typename T, typename P>
struct Lane {
    const Setup<T, P> &S;
    Tally<T, P> &tally;
    uint64_t x, xR, xS;
    uint32_t a, aR, aS;
    OraclePacket *rec;  // non-null while recording a packet
    double rec_contrib;
    double *dump = nullptr;  // per-step state of packet dump_packet (diagnostics)
    uint32_t dump_max = 0;
    uint64_t dump_packet = 0;
    uint64_t dump_rows = 0;

    const T *plane(int tet, int k) const { return &S.planes[(size_t)(4 * tet + k) * 4]; }

    // LaunchPhoton, src/octmps_kernel.cuh:475-503.
    void launch(Photon<T, P> &ph) {
        ph.x = S.probe_x;
        ph.y = S.probe_y;
        ph.z = S.probe_z;
        ph.ux = 0;
        ph.uy = 0;
        ph.uz = 1;
        ph.w = S.w0;
        ph.min_cos = 0;
        ph.s = 0;
        ph.sleft = 0;
        ph.optical_path = 0;
        ph.max_depth = 0;
        ph.lr = 1;
        ph.lr_after = 1;
        ph.fst_flag = 0;
        ph.loc_fst = -1;
        ph.num_back = 0;
        ph.next_face = -1;
        ph.tet = S.root;
    }

    // ComputeStepSize, src/octmps_kernel.cuh:505-515.
    void step_size(Photon<T, P> &ph) {
        const Region<T, P> &rg = S.regions[S.region[ph.tet]];
        if (ph.sleft == (T)0) {
            T r = rand_oc<T>(&x, a);
            ph.s = -Num<T>::log(r) * rg.rmuas;
        } else {
            ph.s = ph.sleft * rg.rmuas;
            ph.sleft = 0;
        }
    }

    // HitBoundary, src/octmps_kernel.cuh:517-572, on sign-folded planes.
    bool hit_boundary(Photon<T, P> &ph) {
        T cosv[4];
        for (int k = 0; k < 4; ++k) {
            const T *pl = plane(ph.tet, k);
            cosv[k] = dot3<T>(pl[0], pl[1], pl[2], ph.ux, ph.uy, ph.uz);
        }
        T min_d = Num<T>::big;
        int idx = -1;
        if (kFused<T>) {
            // FP32 forms: the nearest face by comparing perp_i / c_i against
            // perp_j / c_j as perp_i * c_j < perp_j * c_i (c = -cos > 0),
            // then one division for the winner.
            T best_perp = 0, best_c = 0;
            for (int k = 0; k < 4; ++k) {
                if (cosv[k] < (T)0) {
                    const T *pl = plane(ph.tet, k);
                    const T perp = dot3<T>(pl[0], pl[1], pl[2], ph.x, ph.y, ph.z) + pl[3];
                    const T c = -cosv[k];
                    const bool nearer = idx < 0 ? perp < Num<T>::big * c
                                                : perp * best_c < best_perp * c;
                    if (nearer) {
                        best_perp = perp;
                        best_c = c;
                        idx = k;
                    }
                }
            }
            if (idx >= 0) {
                min_d = Num<T>::div(best_perp, best_c);
                ph.min_cos = -best_c;
            }
        } else {
            for (int k = 0; k < 4; ++k) {
                if (cosv[k] < (T)0) {
                    const T *pl = plane(ph.tet, k);
                    T perp = dot3<T>(pl[0], pl[1], pl[2], ph.x, ph.y, ph.z) + pl[3];
                    T t = Num<T>::div(-perp, cosv[k]);
                    if (t < min_d) {
                        min_d = t;
                        idx = k;
                        ph.min_cos = cosv[k];
                    }
                }
            }
        }
        if (ph.s > min_d) {
            const Region<T, P> &rg = S.regions[S.region[ph.tet]];
            ph.sleft = (ph.s - min_d) * rg.muas;
            ph.s = min_d;
            ph.next_face = idx;
            return true;
        }
        ph.next_face = -1;
        return false;
    }

    // Hop, src/octmps_kernel.cuh:574-582.
    void hop(Photon<T, P> &ph) {
        ph.x = Num<T>::mad(ph.s, ph.ux, ph.x);
        ph.y = Num<T>::mad(ph.s, ph.uy, ph.y);
        ph.z = Num<T>::mad(ph.s, ph.uz, ph.z);
        ph.optical_path += (P)ph.s;
        if (ph.max_depth < ph.z) ph.max_depth = ph.z;
    }

    // Drop, src/octmps_kernel.cuh:584-588.
    void drop(Photon<T, P> &ph) {
        const Region<T, P> &rg = S.regions[S.region[ph.tet]];
        ph.w = Num<T>::mad(-ph.w, rg.mua_muas, ph.w);
    }

    // Class I/II tally, src/octmps_kernel.cuh:684-744.
    void tally_detection(const Photon<T, P> &ph, T r_fresnel, T rr) {
        tally.nf++;
        const P op = ph.optical_path;
        const P depth = Num<P>::div(op, (P)2);
        const P vpf = Num<P>::div(depth - S.shift, S.bin_width);
        // (unsigned) conversion of the bin position, saturating as the
        // device's float-to-unsigned conversion does.
        int64_t vp;
        if (!(vpf > (P)0)) vp = 0;
        else if (vpf >= (P)4294967295.0) vp = 4294967295ll;
        else vp = (int64_t)vpf;
        const bool class1 = (P)ph.max_depth > depth - S.half_lc;
        const T wt = ph.w * ((T)1 - r_fresnel);
        const T c = wt * ph.lr;
        const P cp = (P)c;
        if (g_records) {
            const uint64_t k = g_record_n.fetch_add(1, std::memory_order_relaxed);
            if (k < g_record_cap)
                g_records[k] = {(double)wt, (double)ph.lr, (double)rr, (double)-ph.uz,
                                (double)op, (double)ph.max_depth};
        }
        for (int64_t ii = vp - 3; ii < vp + 3; ++ii) {
            if (ii >= 0 && ii < S.nbins) {
                if (rec) rec_contrib += (double)cp;
                if (class1) {
                    if (ii == vp) tally.nf1++;
                    tally.s1[ii] += cp;
                    if (tally.m1[ii] < cp) tally.m1[ii] = cp;
                    tally.q1[ii] += cp * cp;
                    tally.c1[ii]++;
                } else {
                    if (ii == vp) tally.nf2++;
                    if (tally.m2[ii] < cp) tally.m2[ii] = cp;
                    tally.s2[ii] += cp;
                    tally.q2[ii] += cp * cp;
                    tally.c2[ii]++;
                }
            }
        }
    }

    // FastReflectTransmit with PARTIAL_REFLECTION, src/octmps_kernel.cuh:590-775.
    // Returns the event code.
    int reflect_transmit(Photon<T, P> &ph) {
        const T ca1 = -ph.min_cos;
        const T ni = S.regions[S.region[ph.tet]].n;
        const int next = S.adj[4 * ph.tet + ph.next_face];
        const T nt = next == -1 ? S.n_ambient : S.regions[S.region[next]].n;
        T r;
        T sa1 = std::sqrt(Num<T>::mad(-ca1, ca1, (T)1));
        if (ca1 > Num<T>::coszero) sa1 = 0;
        if (kFused<T> && ni == nt) {
            // FP32 forms, matched refractive indices: Fresnel's R is exactly
            // 0 (the formula only adds rounding noise in FP32), except for
            // the reference's grazing-incidence rule (sa2 = sa1 here).
            r = (ca1 < Num<T>::cos90 || sa1 == (T)1) ? (T)1 : (T)0;
        } else {
            const T ni_nt = Num<T>::div(ni, nt);
            const T sa2 = std::fmin(ni_nt * sa1, (T)1);
            const T ca2 = std::sqrt(Num<T>::mad(-sa2, sa2, (T)1));
            const T ca1ca2 = ca1 * ca2;
            const T sa1sa2 = sa1 * sa2;
            T sa1ca2 = sa1 * ca2;
            T ca1sa2 = ca1 * sa2;
            if (ca1 > Num<T>::coszero) {
                sa1ca2 = 1;
                ca1sa2 = ni_nt;
            }
            const T cam = ca1ca2 + sa1sa2;
            const T sap = sa1ca2 + ca1sa2;
            const T sam = sa1ca2 - ca1sa2;
            r = Num<T>::div(sam, sap * cam);
            r = r * r;
            r = r * Num<T>::mad(ca1ca2, ca1ca2, sa1sa2 * sa1sa2);
            if (ca1 < Num<T>::cos90 || sa2 == (T)1) r = 1;
        }

        const T *pl = plane(ph.tet, ph.next_face);
        const T two_ca1 = ca1 + ca1;
        const T rx = Num<T>::mad(two_ca1, pl[0], ph.ux);
        const T ry = Num<T>::mad(two_ca1, pl[1], ph.uy);
        const T rz = Num<T>::mad(two_ca1, pl[2], ph.uz);

        const T rnd = rand_co<T>(&xR, aR);
        if (next == -1 && r < (T)1) {
            int ev = ORACLE_EV_EXIT;
            if (ph.uz < (T)0) {
                bool filt = false;
                const T dx = ph.x - S.probe_x;
                const T dy = ph.y - S.probe_y;
                const T rr = std::sqrt(Num<T>::mad(dx, dx, dy * dy));
                if (rr < S.radius && -ph.uz > S.cos_collect) {
                    if (S.type_bias == 0 || S.type_bias == 3) filt = true;
                    if ((ph.fst_flag && S.type_bias == 37) ||
                        (ph.loc_fst == ph.max_depth && S.type_bias != 37) || ph.num_back > 0)
                        filt = true;
                }
                if (filt) {
                    tally_detection(ph, r, rr);
                    ev |= ORACLE_EV_DETECT;
                }
            } else {
                ph.num_back++;
            }
            ph.w *= r;
            ph.ux = rx;
            ph.uy = ry;
            ph.uz = rz;
            return ev;
        } else if (rnd > r) {
            ph.tet = next;
            ph.next_face = -1;
            return ORACLE_EV_TRANSMIT;
        } else {
            ph.next_face = -1;
            if (ph.uz > (T)0) ph.num_back++;
            ph.ux = rx;
            ph.uy = ry;
            ph.uz = rz;
            return ORACLE_EV_REFLECT;
        }
    }

    // SpinTheta, src/octmps_kernel.cuh:807-820.
    T spin_theta(T g) {
        T cost;
        if (g == (T)0) {
            cost = (T)2 * rand_oc<T>(&xS, aS) - (T)1;
        } else {
            const T r = rand_oc<T>(&xS, aS);
            const T temp = Num<T>::div(Num<T>::mad(-g, g, (T)1), Num<T>::mad(g + g, r, (T)1 - g));
            cost = Num<T>::div(Num<T>::mad(-temp, temp, Num<T>::mad(g, g, (T)1)), g + g);
            if (cost < (T)-1) cost = -1;
            else if (cost > (T)1) cost = 1;
        }
        return cost;
    }

    // SpinThetaForwardFstBias, src/octmps_kernel.cuh:881-896.
    T spin_theta_forward(T g) {
        T cost;
        if (g == (T)0) {
            cost = rand_oc<T>(&xS, aS);
        } else {
            const T r = rand_oc<T>(&xS, aS);
            const T temp = Num<T>::div(r, (T)1 - g) +
                           Num<T>::div((T)1 - r, std::sqrt(Num<T>::mad(g, g, (T)1)));
            cost = Num<T>::div(Num<T>::mad(g, g, (T)1) - Num<T>::div((T)1, temp * temp), g + g);
            if (cost < (T)-1) cost = -1;
            else if (cost > (T)1) cost = 1;
        }
        return cost;
    }

    // Rotation of (ux,uy,uz) by polar cosine cost and azimuth from one
    // draw of the spin stream (src/octmps_kernel.cuh:844-868, 1006-1026).
    void rotate(T cost, T ux, T uy, T uz, Photon<T, P> &ph, bool copysign_form) {
        const T sint = std::sqrt(Num<T>::mad(-cost, cost, (T)1));
        T sinp, cosp;
        Num<T>::sincos_rand(rand_co<T>(&xS, aS), &sinp, &cosp);
        const T stcp = sint * cosp;
        const T stsp = sint * sinp;
        if (std::fabs(uz) > Num<T>::coszero) {
            ph.ux = stcp;
            ph.uy = stsp;
            if (copysign_form) ph.uz = std::copysign(cost, uz * cost);
            else ph.uz = cost * (uz >= (T)0 ? (T)1 : (T)-1);
        } else {
            // RSQRT(x) taken as 1/sqrt(x), both correctly rounded.
            const T sq = std::sqrt(Num<T>::mad(-uz, uz, (T)1));
            const T temp = (T)1 / sq;
            ph.ux = Num<T>::mad(Num<T>::mad(stcp * ux, uz, -(stsp * uy)), temp, ux * cost);
            ph.uy = Num<T>::mad(Num<T>::mad(stcp * uy, uz, stsp * ux), temp, uy * cost);
            // FAST_DIV(-stcp, temp) is -stcp * sqrt(1 - uz^2): the FP32 forms
            // multiply, the FP64 form divides as the reference.
            ph.uz = Num<T>::mad(uz, cost, kFused<T> ? -(stcp * sq) : Num<T>::div(-stcp, temp));
        }
    }

    // Spin, src/octmps_kernel.cuh:822-879.
    void spin(T g, Photon<T, P> &ph) {
        const T cost = spin_theta(g);
        rotate(cost, ph.ux, ph.uy, ph.uz, ph, false);
    }

    // SpinBias, src/octmps_kernel.cuh:898-1086.
    void spin_bias(T g, Photon<T, P> &ph, Photon<T, P> &cont) {
        const T g2 = g * g;
        T ux = ph.ux, uy = ph.uy, uz = ph.uz;
        const T ox = ux, oy = uy, oz = uz;
        T btmp = 0;
        int reached = 0;
        bool first = false;
        if ((ph.z > S.tdmin) && (ph.z < S.tdmax) && (ph.uz > (T)0) && !ph.fst_flag) {
            cont = ph;  // CopyPhotonStruct: the saved copy resumes later
            reached = 1;
            ph.fst_flag = 1;
            ph.loc_fst = ph.z;
            btmp = S.bias_a;
            first = true;
        }
        T vx = S.probe_x - ph.x;
        T vy = S.probe_y - ph.y;
        T vz = S.probe_z - ph.z;
        const T len = std::sqrt(Num<T>::mad(vz, vz, Num<T>::mad(vx, vx, vy * vy)));
        if (kFused<T>) {
            // FP32 forms: one reciprocal, three products
            const T rl = (T)1 / len;
            vx *= rl;
            vy *= rl;
            vz *= rl;
        } else {
            vx = Num<T>::div(vx, len);
            vy = Num<T>::div(vy, len);
            vz = Num<T>::div(vz, len);
        }
        if ((ph.fst_flag || ph.num_back > 0) && !reached) {
            reached = 2;
            const Region<T, P> &rg = S.regions[S.region[ph.tet]];
            // -log(0)/mu_t is +infinity: with rndStepSizeInTissue = 0 (what the
            // reference reads, src/octmps.h:124) the distance test always holds.
            const bool far = S.rnd_step == (T)0 ||
                             Num<T>::div(-Num<T>::log(S.rnd_step), rg.muas) >= len;
            // the distance to the probe equals len (same terms, same order)
            if (far && -vz >= S.cos_collect) reached = 1;
            btmp = S.bias_a;
        }
        int sel = 0;
        T cost;
        if (reached) {
            sel = rand_co<T>(&xS, aS) <= S.p_bias ? 1 : 2;
            if (reached == 1 || sel == 1) {
                cost = spin_theta_forward(btmp);
                ux = vx;
                uy = vy;
                uz = vz;
            } else {
                cost = spin_theta(g);
            }
        } else {
            cost = spin_theta(g);
        }
        cost = std::fmax(cost, (T)-1);
        cost = std::fmin(cost, (T)1);
        rotate(cost, ux, uy, uz, ph, true);

        T costg = dot3<T>(ox, oy, oz, ph.ux, ph.uy, ph.uz);
        T costg1 = dot3<T>(vx, vy, vz, ph.ux, ph.uy, ph.uz);
        if (kFused<T>) {
            // FP32 forms, as the kernel: a direction rotated about a nearly
            // vertical axis is off unit length by a few tenths of a percent,
            // so a cosine can exceed 1 and the likelihood's square root turn
            // NaN: clamp to [-1, 1]
            costg = std::fmin(std::fmax(costg, (T)-1), (T)1);
            costg1 = std::fmin(std::fmax(costg1, (T)-1), (T)1);
        }
        if (btmp != (T)0) {
            const T opa2 = Num<T>::mad(btmp, btmp, (T)1);
            const T sq_opa2 = std::sqrt(opa2);
            T f;
            if (reached == 1) {
                // Likelihood of the first biased scattering (eq. 8 of
                // Malektaji et al., J. Biomed. Opt. 19(4) 046001, 2014).
                const T b1 = opa2 - (btmp + btmp) * cost;
                const T h1 = Num<T>::mad(g, g, (T)1) - (g + g) * costg;
                const T num = ((T)1 - g2) * (sq_opa2 - (T)1 + btmp) * std::sqrt(b1 * b1 * b1);
                const T den = (btmp + btmp) * ((T)1 - btmp) * sq_opa2 * std::sqrt(h1 * h1 * h1);
                f = Num<T>::div(num, den);
            } else {
                // Mixture likelihood of later scatterings (eq. 9, same paper).
                const T c1 = sel == 1 ? cost : costg1;
                const T c2 = sel == 1 ? costg : cost;
                const T b1 = opa2 - (btmp + btmp) * c1;
                const T pdf1 = Num<T>::div(sq_opa2 * btmp * ((T)1 - btmp),
                                           (sq_opa2 - (T)1 + btmp) * std::sqrt(b1 * b1 * b1));
                const T h2 = std::sqrt(Num<T>::mad(g, g, (T)1) - (g + g) * c2);
                const T pdf2 = Num<T>::div((T)1 - g2, (T)2 * (h2 * h2 * h2));
                f = Num<T>::div(pdf2, Num<T>::mad(S.p_bias, pdf1, ((T)1 - S.p_bias) * pdf2));
            }
            ph.lr *= f;
            if (first) ph.lr_after = ph.lr;
        }
    }

    // One lane: its packets in order, each to the end of its last split copy
    // (OCTMPSKernel loop body, src/octmps_kernel.cuh:1349-1392).
    void run(uint64_t packets, OraclePacket *first_rec) {
        Photon<T, P> ph, cont;
        // steps allowed per packet, as the kernel's step_cap; a dump ends
        // its packet at the dump's length
        const uint64_t cap = (1ull << 26);
        for (uint64_t k = 0; k < packets; ++k) {
            rec = (k == 0) ? first_rec : nullptr;
            rec_contrib = 0;
            OraclePacket r{};
            r.hash = 14695981039346656037ull;
            launch(ph);
            cont = ph;
            tally.packets++;
            uint64_t steps = 0;
            uint32_t stall = 0;  // boundary hits in a row that did not move the photon
            for (;;) {
                int ev;
                step_size(ph);
                const bool hit = hit_boundary(ph);
                stall = (hit && ph.s <= (T)0) ? stall + 1 : 0;
                hop(ph);
                if (hit) {
                    ev = reflect_transmit(ph);
                    r.hits++;
                    if (ev & ORACLE_EV_DETECT) r.detections++;
                } else {
                    ev = ORACLE_EV_SCATTER;
                    r.scatters++;
                    drop(ph);
                    const T g = S.regions[S.region[ph.tet]].g;
                    if (S.type_bias == 0) spin(g, ph);
                    else if (S.type_bias == 37) spin_bias(g, ph, cont);
                }
                bool end = false;
                if (ph.w < Num<T>::weight) {
                    const T rnd = rand_co<T>(&x, a);
                    if (ph.w != (T)0 && rnd < Num<T>::chance) {
                        ph.w *= Num<T>::div((T)1, Num<T>::chance);
                        ev |= ORACLE_EV_SURVIVE;
                        r.survivals++;
                    } else if (ph.fst_flag && S.type_bias != 3) {
                        const T lr_tmp = ph.lr_after;
                        const T keep_after = ph.lr_after;  // not part of the copy
                        ph = cont;
                        ph.lr_after = keep_after;
                        spin(S.regions[S.region[ph.tet]].g, ph);
                        ph.lr = lr_tmp < (T)1 ? (T)1 - lr_tmp : (T)1;
                        ev |= ORACLE_EV_RESTORE;
                        stall = 0;
                        r.restores++;
                        tally.restores++;
                    } else {
                        ev |= ORACLE_EV_END;
                        end = true;
                    }
                }
                r.hash = fnv(r.hash, ((uint64_t)(uint32_t)ph.tet << 8) | (uint64_t)ev);
                if (dump && k == dump_packet && r.steps < dump_max) {
                    dump_rows = r.steps + 1;
                    double *d = dump + 12 * (size_t)r.steps;
                    d[0] = ph.tet; d[1] = ev; d[2] = (double)ph.x; d[3] = (double)ph.y;
                    d[4] = (double)ph.z; d[5] = (double)ph.ux; d[6] = (double)ph.uy;
                    d[7] = (double)ph.uz; d[8] = (double)ph.w; d[9] = (double)ph.s;
                    d[10] = (double)ph.optical_path; d[11] = (double)ph.lr;
                }
                r.steps++;
                ++steps;
                if (end) break;
                // The kernel's stop rule: the step cap, or 1000 hits in a row
                // that did not move the photon (a photon on a face moving
                // parallel to it is reflected with its direction unchanged
                // by the grazing-incidence rule, again at distance 0; the
                // reference repeats that forever).
                if (steps >= cap || stall >= 1000 ||
                    (dump && k == dump_packet && steps >= dump_max)) {
                    tally.capped++;
                    break;
                }
            }
            tally.steps += steps;
            if (rec) {
                r.x = x;
                r.xR = xR;
                r.xS = xS;
                r.contribution = rec_contrib;
                r.optical_path = (double)ph.optical_path;
                *rec = r;
            }
        }
    }
};

template <typename T, typename P>
void make_setup(Setup<T, P> &S, const OracleParams *p, const OracleMesh *m, double px, double py,
                double pz, int32_t root) {
    S.planes.resize((size_t)m->n_tets * 16);
    for (int t = 0; t < m->n_tets; ++t)
        for (int k = 0; k < 4; ++k) {
            const int f = m->faces[4 * t + k];
            const double sg = (double)m->signs[4 * t + k];
            for (int c = 0; c < 4; ++c)
                S.planes[(size_t)(4 * t + k) * 4 + c] = (T)(m->planes[4 * (size_t)f + c] * sg);
        }
    S.adj = m->adj;
    S.region = m->region;
    S.regions.resize(p->n_regions);
    for (int i = 0; i < p->n_regions; ++i) {
        // read_simulation_data (src/octmps_io.cpp:625-626) and
        // InitDeviceConstantMemory (src/octmps_kernel.cuh:204-214).
        const double mutr = (p->region_mus[i] == 0.0) ? DBL_MAX
                                                      : 1.0 / (p->region_mua[i] + p->region_mus[i]);
        S.regions[i].n = (T)p->region_n[i];
        S.regions[i].muas = (T)(1.0 / mutr);
        S.regions[i].rmuas = (T)mutr;
        S.regions[i].mua_muas = (T)(p->region_mua[i] * mutr);
        S.regions[i].g = (T)p->region_g[i];
    }
    S.n_ambient = (T)p->region_n[0];
    S.type_bias = p->type_bias;
    S.nbins = p->nbins;
    S.probe_x = (T)px;
    S.probe_y = (T)py;
    S.probe_z = (T)pz;
    S.tdmin = (T)p->target_depth_min;
    S.tdmax = (T)p->target_depth_max;
    S.bias_a = (T)p->backward_bias_coefficient;
    S.p_bias = (T)p->probability_additional_bias;
    S.cos_collect = (T)std::cos(p->max_collecting_angle_deg * 3.14159265359 / 180.0);
    S.radius = (T)p->max_collecting_radius;
    S.rnd_step = (T)p->rnd_step_size_in_tissue;
    const double n0 = p->region_n[0], nr = p->region_n[m->region[root]];
    const double rs = (n0 - nr) / (n0 + nr);  // Rspecular, src/main.cu:29-37
    S.w0 = (T)(1.0 - rs * rs);
    S.shift = (P)p->optical_depth_shift;
    S.bin_width = (P)div_rd(p->coherence_length_source, 6.0);
    S.half_lc = (P)div_rd(p->coherence_length_source, 2.0);
    S.root = root;
}

template <typename T, typename P>
int run_typed(const OracleParams *p, const OracleMesh *m, double px, double py, double pz,
              int32_t root, uint64_t n_photons, uint32_t n_lanes, const uint64_t *x,
              const uint32_t *a, const uint64_t *xR, const uint32_t *aR, const uint64_t *xS,
              const uint32_t *aS, int n_threads, OracleTally *out, OraclePacket *first) {
    Setup<T, P> S;
    make_setup(S, p, m, px, py, pz, root);
    if (n_threads > 0) omp_set_num_threads(n_threads);
    const int nth = omp_get_max_threads();
    std::vector<Tally<T, P> *> tallies(nth, nullptr);
    const uint64_t base = n_lanes ? n_photons / n_lanes : 0;
    const uint64_t extra = n_lanes ? n_photons % n_lanes : 0;
#pragma omp parallel
    {
        const int tid = omp_get_thread_num();
        Tally<T, P> *tl = new Tally<T, P>(p->nbins);
        tallies[tid] = tl;
#pragma omp for schedule(static, 1)
        for (int64_t v = 0; v < (int64_t)n_lanes; ++v) {
            Lane<T, P> L{S, *tl, x[v], xR[v], xS[v], a[v], aR[v], aS[v], nullptr, 0.0};
            const uint64_t q = base + ((uint64_t)v < extra ? 1 : 0);
            L.run(q, first ? &first[v] : nullptr);
        }
    }
    // Reduce in thread order (deterministic for a fixed thread count).
    const int nb = p->nbins;
    memset(out->count1, 0, sizeof(uint64_t) * (nb + 1));
    memset(out->count2, 0, sizeof(uint64_t) * (nb + 1));
    for (double *d : {out->sum1, out->max1, out->sumsq1, out->sum2, out->max2, out->sumsq2})
        memset(d, 0, sizeof(double) * (nb + 2));
    out->num_filtered = out->num_filtered_class1 = out->num_filtered_class2 = 0;
    out->steps = out->restores = out->packets = out->capped = 0;
    std::vector<P> s1(nb + 2, 0), q1(nb + 2, 0), s2(nb + 2, 0), q2(nb + 2, 0);
    for (Tally<T, P> *t : tallies) {
        if (!t) continue;
        out->num_filtered += t->nf;
        out->num_filtered_class1 += t->nf1;
        out->num_filtered_class2 += t->nf2;
        out->steps += t->steps;
        out->restores += t->restores;
        out->packets += t->packets;
        out->capped += t->capped;
        for (int i = 0; i < nb + 1; ++i) {
            out->count1[i] += t->c1[i];
            out->count2[i] += t->c2[i];
        }
        for (int i = 0; i < nb + 2; ++i) {
            s1[i] += t->s1[i];
            q1[i] += t->q1[i];
            s2[i] += t->s2[i];
            q2[i] += t->q2[i];
            if ((double)t->m1[i] > out->max1[i]) out->max1[i] = (double)t->m1[i];
            if ((double)t->m2[i] > out->max2[i]) out->max2[i] = (double)t->m2[i];
        }
        delete t;
    }
    for (int i = 0; i < nb + 2; ++i) {
        out->sum1[i] = (double)s1[i];
        out->sumsq1[i] = (double)q1[i];
        out->sum2[i] = (double)s2[i];
        out->sumsq2[i] = (double)q2[i];
    }
    return 0;
}

template <typename T, typename P>
int dump_typed(const OracleParams *p, const OracleMesh *m, double px, double py, double pz,
               int32_t root, uint64_t x, uint32_t a, uint64_t xR, uint32_t aR, uint64_t xS,
               uint32_t aS, double *out, uint32_t max_steps, uint64_t packet_index) {
    Setup<T, P> S;
    make_setup(S, p, m, px, py, pz, root);
    Tally<T, P> tl(p->nbins);
    OraclePacket rec{};
    Lane<T, P> L{S, tl, x, xR, xS, a, aR, aS, nullptr, 0.0};
    L.dump = out;
    L.dump_max = max_steps;
    L.dump_packet = packet_index;
    L.run(packet_index + 1, &rec);
    return (int)L.dump_rows;
}

}  // namespace

extern "C" {

int oracle_run(const OracleParams *p, const OracleMesh *m, double probe_x, double probe_y,
               double probe_z, int32_t root, uint64_t n_photons, uint32_t n_lanes,
               const uint64_t *x, const uint32_t *a, const uint64_t *xR, const uint32_t *aR,
               const uint64_t *xS, const uint32_t *aS, int precision, int n_threads,
               OracleTally *out, OraclePacket *first) {
    if (!p || !m || !out || root < 0 || root >= m->n_tets || p->n_regions < 1 ||
        p->n_regions > ORACLE_MAX_REGIONS)
        return 1;
    switch (precision) {
        case 0:
            return run_typed<float, double>(p, m, probe_x, probe_y, probe_z, root, n_photons,
                                            n_lanes, x, a, xR, aR, xS, aS, n_threads, out, first);
        case 1:
            return run_typed<float, float>(p, m, probe_x, probe_y, probe_z, root, n_photons,
                                           n_lanes, x, a, xR, aR, xS, aS, n_threads, out, first);
        case 2:
            return run_typed<double, double>(p, m, probe_x, probe_y, probe_z, root, n_photons,
                                             n_lanes, x, a, xR, aR, xS, aS, n_threads, out, first);
        default:
            return 2;
    }
}

int oracle_dump_lane(const OracleParams *p, const OracleMesh *m, double probe_x, double probe_y,
                     double probe_z, int32_t root, uint64_t x, uint32_t a, uint64_t xR,
                     uint32_t aR, uint64_t xS, uint32_t aS, int precision, double *out,
                     uint32_t max_steps, uint64_t packet_index) {
    switch (precision) {
        case 0:
            return dump_typed<float, double>(p, m, probe_x, probe_y, probe_z, root, x, a, xR, aR,
                                             xS, aS, out, max_steps, packet_index);
        case 1:
            return dump_typed<float, float>(p, m, probe_x, probe_y, probe_z, root, x, a, xR, aR,
                                            xS, aS, out, max_steps, packet_index);
        case 2:
            return dump_typed<double, double>(p, m, probe_x, probe_y, probe_z, root, x, a, xR, aR,
                                              xS, aS, out, max_steps, packet_index);
    }
    return -1;
}

// Multiplier list of the MWC generators, for runs that must not load the
// product library (the bench's reference arm).  The reference reads the
// first column of safeprimes_base32.txt (src/octmps_kernel.cuh:74-105), a
// file it does not ship; a valid multiplier a < 2^32 makes a*2^32 - 1 and
// a*2^31 - 1 both prime.  The list is every such a in descending order from
// 2^32 - 1, found by trial division by the odd primes below 100 and the
// deterministic 64-bit Miller-Rabin test (bases 2, 325, 9375, 28178, 450775,
// 9780504, 1795265022, after J. Sinclair).  Returns 0 when `count` entries
// were written.
namespace {
typedef unsigned __int128 u128;
uint64_t mr_pow(uint64_t b, uint64_t e, uint64_t m) {
    uint64_t r = 1;
    b %= m;
    for (; e; e >>= 1) {
        if (e & 1) r = (uint64_t)((u128)r * b % m);
        b = (uint64_t)((u128)b * b % m);
    }
    return r;
}
bool mr_prime(uint64_t n) {
    static const uint64_t small[] = {3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37, 41, 43, 47,
                                     53, 59, 61, 67, 71, 73, 79, 83, 89, 97};
    if (n < 2) return false;
    if (n % 2 == 0) return n == 2;
    for (uint64_t q : small)
        if (n % q == 0) return n == q;
    uint64_t d = n - 1;
    int r = 0;
    while (!(d & 1)) { d >>= 1; ++r; }
    for (uint64_t a : {2ull, 325ull, 9375ull, 28178ull, 450775ull, 9780504ull, 1795265022ull}) {
        uint64_t x = mr_pow(a, d, n);
        if (x == 0 || x == 1 || x == n - 1) continue;
        bool comp = true;
        for (int i = 1; i < r && comp; ++i) {
            x = (uint64_t)((u128)x * x % n);
            if (x == n - 1) comp = false;
        }
        if (comp) return false;
    }
    return true;
}
}  // namespace

uint64_t oracle_set_photon_records(OraclePhotonRecord *buf, uint64_t cap) {
    g_records = buf;
    g_record_cap = buf ? cap : 0;
    return g_record_n.exchange(0);
}

int oracle_safeprimes(uint32_t *out, uint64_t count) {
    const uint64_t chunk = 1 << 16;
    uint64_t found = 0, top = 0xffffffffull;
    while (found < count && top >= 0x80000000ull) {
        const int nchunks = 64;
        std::vector<std::vector<uint32_t>> got(nchunks);
#pragma omp parallel for schedule(dynamic, 1)
        for (int c = 0; c < nchunks; ++c) {
            const uint64_t hi = top - (uint64_t)c * chunk;
            for (uint64_t i = 0; i < chunk; ++i) {
                const uint64_t a = hi - i;
                if (a < 0x80000000ull) break;
                if (mr_prime((a << 31) - 1) && mr_prime((a << 32) - 1))
                    got[c].push_back((uint32_t)a);
            }
        }
        for (int c = 0; c < nchunks && found < count; ++c)
            for (uint32_t a : got[c]) {
                if (found == count) break;
                out[found++] = a;
            }
        top = top >= (uint64_t)nchunks * chunk ? top - (uint64_t)nchunks * chunk : 0;
    }
    return found == count ? 0 : 1;
}

float oracle_logf(float x) { return logf_method(x); }
double oracle_log(double x) { return log_method(x); }
void oracle_sincos_turn_f(float t, float *s, float *c) { sincos_turn_f(t, s, c); }
void oracle_sincos_d(double psi, double *s, double *c) { sincos_d(psi, s, c); }
double oracle_div_rd(double a, double b) { return div_rd(a, b); }
float oracle_uint2float_rz(uint32_t u) { return uint2float_rz(u); }

}  // extern "C"
