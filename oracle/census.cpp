// Operation census of the photon method.  TEST AND MEASUREMENT
// INFRASTRUCTURE ONLY (the bench's roofline reads its result; the product
// never links it).
//
// The oracle's own code (oracle.cpp, included below) runs with its
// geometry and path types replaced by counting number types, so every
// floating-point operation the method performs on a workload is counted as
// it executes: + - x / and sqrt count 1 each, a fused multiply-add 2, log 1,
// a sine-cosine pair 2 (one transcendental each).  Comparisons, min/max,
// absolute value, sign copies, negations and conversions count 0.  Divided by
// the propagation steps taken, this is the algorithmic work per step of the
// workload's actual event mix (hits, scatterings, biased scatterings,
// roulettes, restores, detections), in FP32 and FP64 separately.
#include <cmath>
#include <cstdint>
#include <type_traits>

namespace census {
struct Counts {
    uint64_t add, mul, div, sqrt, fma, trans;
};
Counts c32 = {}, c64 = {};
template <typename U>
inline Counts &of() {
    return sizeof(U) == 4 ? c32 : c64;
}
}  // namespace census

template <typename U>
struct Cnt {
    U v;
    Cnt() = default;
    constexpr Cnt(double x) : v((U)x) {}
    constexpr Cnt(float x) : v((U)x) {}
    constexpr Cnt(int x) : v((U)x) {}
    template <typename W, typename = typename std::enable_if<!std::is_same<U, W>::value>::type>
    constexpr Cnt(Cnt<W> o) : v((U)o.v) {}
    explicit operator double() const { return (double)v; }
    explicit operator float() const { return (float)v; }
    explicit operator long() const { return (long)v; }
    explicit operator long long() const { return (long long)v; }
    explicit operator unsigned() const { return (unsigned)v; }
    Cnt operator-() const { return Cnt(-v); }
    Cnt &operator+=(Cnt o) { census::of<U>().add++; v += o.v; return *this; }
    Cnt &operator-=(Cnt o) { census::of<U>().add++; v -= o.v; return *this; }
    Cnt &operator*=(Cnt o) { census::of<U>().mul++; v *= o.v; return *this; }
    static Cnt raw(U x) { Cnt c; c.v = x; return c; }
};
template <typename U>
inline Cnt<U> operator+(Cnt<U> a, Cnt<U> b) { census::of<U>().add++; return Cnt<U>::raw(a.v + b.v); }
template <typename U>
inline Cnt<U> operator-(Cnt<U> a, Cnt<U> b) { census::of<U>().add++; return Cnt<U>::raw(a.v - b.v); }
template <typename U>
inline Cnt<U> operator*(Cnt<U> a, Cnt<U> b) { census::of<U>().mul++; return Cnt<U>::raw(a.v * b.v); }
template <typename U>
inline Cnt<U> operator/(Cnt<U> a, Cnt<U> b) { census::of<U>().div++; return Cnt<U>::raw(a.v / b.v); }
template <typename U> inline bool operator<(Cnt<U> a, Cnt<U> b) { return a.v < b.v; }
template <typename U> inline bool operator>(Cnt<U> a, Cnt<U> b) { return a.v > b.v; }
template <typename U> inline bool operator<=(Cnt<U> a, Cnt<U> b) { return a.v <= b.v; }
template <typename U> inline bool operator>=(Cnt<U> a, Cnt<U> b) { return a.v >= b.v; }
template <typename U> inline bool operator==(Cnt<U> a, Cnt<U> b) { return a.v == b.v; }
template <typename U> inline bool operator!=(Cnt<U> a, Cnt<U> b) { return a.v != b.v; }

// The oracle calls these qualified; overloads for the counting types.
namespace std {
template <typename U>
inline Cnt<U> sqrt(Cnt<U> a) { census::of<U>().sqrt++; return Cnt<U>::raw(std::sqrt(a.v)); }
template <typename U>
inline Cnt<U> fmin(Cnt<U> a, Cnt<U> b) { return Cnt<U>::raw(std::fmin(a.v, b.v)); }
template <typename U>
inline Cnt<U> fmax(Cnt<U> a, Cnt<U> b) { return Cnt<U>::raw(std::fmax(a.v, b.v)); }
template <typename U>
inline Cnt<U> fabs(Cnt<U> a) { return Cnt<U>::raw(std::fabs(a.v)); }
template <typename U>
inline Cnt<U> copysign(Cnt<U> a, Cnt<U> b) { return Cnt<U>::raw(std::copysign(a.v, b.v)); }
}  // namespace std

#include "oracle.cpp"

namespace {

typedef Cnt<float> CF;
typedef Cnt<double> CD;

template <>
struct FusedForm<CF> : std::true_type {};

// The mixed form's arithmetic (Num<float> for geometry and scattering,
// Num<double> for path and tally), counted.
template <>
struct Num<CF> {
    static CF mad(CF a, CF b, CF c) { census::c32.fma++; return CF::raw(std::fma(a.v, b.v, c.v)); }
    static CF div(CF a, CF b) { census::c32.div++; return CF::raw(a.v / b.v); }
    static CF log(CF x) { census::c32.trans++; return CF::raw(logf_method(x.v)); }
    static void sincos_rand(CF r, CF *s, CF *c) {
        census::c32.trans += 2;
        float ss, cc;
        sincos_turn_f(r.v, &ss, &cc);
        *s = CF::raw(ss);
        *c = CF::raw(cc);
    }
    static CF rand_value(uint32_t u) { census::c32.mul++; return CF::raw(uint2float_rz(u) * 0x1p-32f); }
    static constexpr CF coszero = CF(0.999999f);
    static constexpr CF cos90 = CF(1.0e-6f);
    static constexpr CF weight = CF(1.0e-4f);
    static constexpr CF chance = CF(0.1f);
    static constexpr CF big = CF(1.0e10f);
};

template <>
struct Num<CD> {
    static CD mad(CD a, CD b, CD c) { return a * b + c; }
    static CD div(CD a, CD b) { census::c64.div++; return CD::raw(div_rd(a.v, b.v)); }
    static CD log(CD x) { census::c64.trans++; return CD::raw(log_method(x.v)); }
    static void sincos_rand(CD r, CD *s, CD *c) {
        census::c64.mul += 2;  // 2 * PI_const * rand
        census::c64.trans += 2;
        double ss, cc;
        sincos_d((2.0 * 3.14159265359) * r.v, &ss, &cc);
        *s = CD::raw(ss);
        *c = CD::raw(cc);
    }
    static CD rand_value(uint32_t u) {
        census::c64.mul++;
        return CD::raw((double)uint2float_rz(u) * 0x1p-32);
    }
    static constexpr CD coszero = CD(1.0 - 1.0e-14);
    static constexpr CD cos90 = CD(1.0e-6);
    static constexpr CD weight = CD(1.0e-4);
    static constexpr CD chance = CD(0.1);
    static constexpr CD big = CD(1.0e10);
};

}  // namespace

extern "C" {

// One A-scan of the mixed form (precision 0) or the FP64 form (2) on one
// thread, with its operation counts: out[0..5] FP32 add, mul, div, sqrt,
// fma, transcendental; out[6..11] the same in FP64.  The tally goes to
// `tally` as oracle_run fills it (steps included).
int census_run(const OracleParams *p, const OracleMesh *m, double px, double py, double pz,
               int32_t root, uint64_t n_photons, uint32_t n_lanes, const uint64_t *x,
               const uint32_t *a, const uint64_t *xR, const uint32_t *aR, const uint64_t *xS,
               const uint32_t *aS, int precision, OracleTally *tally, uint64_t *out) {
    census::c32 = census::Counts{};
    census::c64 = census::Counts{};
    int st;
    if (precision == 0)
        st = run_typed<CF, CD>(p, m, px, py, pz, root, n_photons, n_lanes, x, a, xR, aR, xS, aS,
                               1, tally, nullptr);
    else if (precision == 2)
        st = run_typed<CD, CD>(p, m, px, py, pz, root, n_photons, n_lanes, x, a, xR, aR, xS, aS,
                               1, tally, nullptr);
    else
        return 2;
    const census::Counts *cs[2] = {&census::c32, &census::c64};
    for (int i = 0; i < 2; ++i) {
        out[6 * i + 0] = cs[i]->add;
        out[6 * i + 1] = cs[i]->mul;
        out[6 * i + 2] = cs[i]->div;
        out[6 * i + 3] = cs[i]->sqrt;
        out[6 * i + 4] = cs[i]->fma;
        out[6 * i + 5] = cs[i]->trans;
    }
    return st;
}

}  // extern "C"
