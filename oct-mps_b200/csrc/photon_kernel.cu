// The per-photon Monte Carlo hot path on sm_100a.
//
// One persistent kernel runs every job of a launch.  Its work unit is an RNG
// lane of a job: a thread takes the next unit from a global counter, loads
// that lane's three multiply-with-carry streams, and runs the lane's packets
// one after the other (lane v of a job with N packets over V lanes runs
// N/V packets, plus one if v < N%V), each packet to the end of its last split
// copy.  A thread whose unit is done takes the next one, so idle lanes are
// refilled until the launch's work runs out.  The method is the reference's
// OCTMPSKernel loop (src/octmps_kernel.cuh:1329-1402) and the device
// functions it calls (:475-1086), restated with the deterministic arithmetic
// of photon_math.cuh.
//
// Layout the kernel reads (built by runtime.cu):
//   planes : per tet 4 inward face planes, sign already applied
//            (float4 x4 = 64 B per tet, or double x16 = 128 B)
//   adj    : per tet int4 of packed neighbours (index | region << 24, or -1)
//   regions: RegionConst<T>[n_regions] (n, mu_t, 1/mu_t, mu_a/mu_t, g)
// The current region's constants stay in registers and are reloaded only
// when a transmission changes region.  The split copy of a photon lives in
// shared memory: it is written at the first biased scattering and read back
// at the restore, a few times per packet.
#include <cuda_runtime.h>

#include "kernel_iface.h"
#include "photon_math.cuh"

namespace octmps {

namespace {

constexpr int kBlock = 256;

// Outcomes of the first half of a step.
constexpr int kDone = 0;     // step finished, packet continues
constexpr int kEnd = 1;      // step finished, packet ended
constexpr int kPending = 2;  // no face reached: scattering still to do

template <typename T>
struct Plane4;
template <>
struct Plane4<float> {
    float v[4][4];
    __device__ __forceinline__ void load(const void *base, int tet) {
        const float4 *p = reinterpret_cast<const float4 *>(base) + 4 * (size_t)tet;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const float4 q = __ldg(p + k);
            v[k][0] = q.x;
            v[k][1] = q.y;
            v[k][2] = q.z;
            v[k][3] = q.w;
        }
    }
};
template <>
struct Plane4<double> {
    double v[4][4];
    __device__ __forceinline__ void load(const void *base, int tet) {
        const double2 *p = reinterpret_cast<const double2 *>(base) + 8 * (size_t)tet;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const double2 a = __ldg(p + 2 * k);
            const double2 b = __ldg(p + 2 * k + 1);
            v[k][0] = a.x;
            v[k][1] = a.y;
            v[k][2] = b.x;
            v[k][3] = b.y;
        }
    }
};

template <typename T, typename P>
struct SplitCopy {
    T x, y, z, ux, uy, uz, w, max_depth, lr;
    P op;
    int32_t tet, region;
    uint32_t num_back;
};

struct PacketRecordDev {
    unsigned long long hash, x, xR, xS;
    uint32_t steps, hits, scatters, restores, detections, survivals;
    double contribution, optical_path;
};

__device__ __forceinline__ unsigned long long fnv(unsigned long long h, unsigned long long v) {
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        h ^= (v >> (8 * i)) & 0xffull;
        h *= 1099511628211ull;
    }
    return h;
}

constexpr uint32_t kStallHits = 1000;    // see the stop rule in the kernel loop
constexpr uint32_t kRetryUs = 8;         // first retry interval of a thread waiting for work
constexpr uint32_t kRetryMaxUs = 512;    // the interval doubles up to this
constexpr unsigned kIdleSleepNs = 4000;  // pause of a warp whose lanes all wait

// Global timer in ticks of 1.024 us (wraps after about 73 minutes; only
// differences are used).
__device__ __forceinline__ uint32_t timer_us() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return (uint32_t)(t >> 10);
}

// Claims up to k >= 1 units from the shared counter by compare-and-swap;
// returns how many it got (0 when none is left) and the first in u.  Retries
// back off (32 ns doubling to 1 us); after 2^20 failed tries it gives up,
// which leaves the units to a later launch.
__device__ __forceinline__ unsigned claim_units(unsigned long long *ctrl, unsigned k,
                                                unsigned long long &u) {
    unsigned ns = 32;
    for (int attempt = 0; attempt < (1 << 20); ++attempt) {
        const unsigned long long cur = __ldcv(ctrl);
        const unsigned long long tot = __ldcv(ctrl + 1);
        if (cur >= tot) return 0;
        const unsigned long long c = min((unsigned long long)k, tot - cur);
        if (atomicCAS(ctrl, cur, cur + c) == cur) {
            u = cur;
            return (unsigned)c;
        }
        __nanosleep(ns);
        if (ns < 1024) ns <<= 1;
    }
    return 0;
}

// One unit for each lane of the warp that arrives here, claimed together by
// the lowest such lane (one compare-and-swap per warp instead of per thread).
__device__ __forceinline__ bool take_unit(unsigned long long *ctrl, unsigned long long &u) {
    const unsigned m = __activemask();
    const int lane = threadIdx.x & 31;
    const int leader = __ffs(m) - 1;
    const unsigned rank = __popc(m & ((1u << lane) - 1u));
    unsigned long long base = 0;
    unsigned c = 0;
    if (lane == leader) c = claim_units(ctrl, __popc(m), base);
    c = __shfl_sync(m, c, leader);
    base = __shfl_sync(m, base, leader);
    u = base + rank;
    return rank < c;
}

// Reports a finished unit of a slot; the launch that finishes the slot's
// last unit stamps its sequence number.  The unit's tallies are made visible
// before the count.
__device__ __forceinline__ void unit_finished(const LaunchArgs &args, int slot, uint32_t n_units) {
    if (!args.slot_state) return;
    __threadfence();
    const unsigned before = atomicAdd(&args.slot_state[slot].x, 1u);
    if (before + 1 == n_units) atomicExch(&args.slot_state[slot].y, args.launch_seq);
}

template <typename P>
__device__ __forceinline__ void atomic_max_bits(P *addr, P v);
template <>
__device__ __forceinline__ void atomic_max_bits<double>(double *addr, double v) {
    atomicMax(reinterpret_cast<unsigned long long *>(addr),
              (unsigned long long)__double_as_longlong(v));
}
template <>
__device__ __forceinline__ void atomic_max_bits<float>(float *addr, float v) {
    atomicMax(reinterpret_cast<unsigned int *>(addr), __float_as_uint(v));
}

// Class I/II tally of one detection, src/octmps_kernel.cuh:684-744.  Out of
// line (a detection is rare) and given its inputs by value: a member function
// would take the lane's address and keep the lane's state in local memory
// instead of registers.  Returns the number of bins the contribution went to.
template <typename T, typename P>
__device__ __noinline__ int tally_detection(const JobDesc *jd, P op, T max_depth, T w,
                                            T r_fresnel, T lr) {
    const JobDesc &J = *jd;
    const TallyLayout L = tally_layout(J.nbins, sizeof(P));
    unsigned char *base = reinterpret_cast<unsigned char *>(J.tally);
    unsigned long long *totals = reinterpret_cast<unsigned long long *>(base + L.totals);
    atomicAdd(&totals[0], 1ull);
    const P depth = DevNum<P>::div(op, (P)2);
    const P vpf = DevNum<P>::div(depth - (P)J.shift, (P)J.bin_width);
    long long vp;
    if (!(vpf > (P)0)) vp = 0;
    else if (vpf >= (P)4294967295.0) vp = 4294967295ll;
    else vp = (long long)vpf;
    const bool class1 = (P)max_depth > depth - (P)J.half_lc;
    const T c = w * ((T)1 - r_fresnel) * lr;
    const P cp = (P)c;
    // NaN or infinite: counted, and added like any other
    if (!(cp - cp == (P)0)) atomicAdd(&totals[3], 1ull);
    unsigned long long *cnt =
        reinterpret_cast<unsigned long long *>(base + (class1 ? L.count1 : L.count2));
    P *sum = reinterpret_cast<P *>(base + (class1 ? L.sum1 : L.sum2));
    P *sumsq = reinterpret_cast<P *>(base + (class1 ? L.sumsq1 : L.sumsq2));
    P *mx = reinterpret_cast<P *>(base + (class1 ? L.max1 : L.max2));
    int n = 0;
    for (long long ii = vp - 3; ii < vp + 3; ++ii) {
        if (ii >= 0 && ii < J.nbins) {
            if (ii == vp) atomicAdd(&totals[class1 ? 1 : 2], 1ull);
            atomicAdd(&sum[ii], cp);
            atomicAdd(&sumsq[ii], cp * cp);
            atomic_max_bits<P>(&mx[ii], cp);
            atomicAdd(&cnt[ii], 1ull);
            ++n;
        }
    }
    return n;
}

template <typename T, typename P, bool kRecord>
struct Lane {
    // photon
    T x, y, z, ux, uy, uz, w, s, sleft, max_depth, lr, lr_after, loc_fst;
    P op;
    int32_t tet, region;
    uint32_t fst_flag, num_back;
    // current region
    RegionConst<T> rg;
    // generators
    uint64_t xG, xR, xS;
    uint32_t aG, aR, aS;
    // job
    const JobDesc *jd;
    const RegionConst<T> *regions;
    const void *planes;
    const int4 *adj;
    T px, py, pz;
    int32_t type_bias;
    // record of the current packet (kRecord only)
    unsigned long long rhash;
    uint32_t rsteps, rhits, rscatters, rrestores, rdetections, rsurvivals;
    double rcontrib;

    __device__ __forceinline__ T rand_co_G() { return DevNum<T>::rand_value(mwc_next(xG, aG)); }
    __device__ __forceinline__ T rand_co_R() { return DevNum<T>::rand_value(mwc_next(xR, aR)); }
    __device__ __forceinline__ T rand_co_S() { return DevNum<T>::rand_value(mwc_next(xS, aS)); }

    __device__ __forceinline__ void load_region(int r) {
        const T *p = reinterpret_cast<const T *>(regions + r);
        rg.n = __ldg(p + 0);
        rg.muas = __ldg(p + 1);
        rg.rmuas = __ldg(p + 2);
        rg.mua_muas = __ldg(p + 3);
        rg.g = __ldg(p + 4);
        region = r;
    }

    // LaunchPhoton, src/octmps_kernel.cuh:475-503.
    __device__ __forceinline__ void launch() {
        x = px;
        y = py;
        z = pz;
        ux = 0;
        uy = 0;
        uz = 1;
        w = (T)jd->w0;
        s = 0;
        sleft = 0;
        op = 0;
        max_depth = 0;
        lr = 1;
        lr_after = 1;
        fst_flag = 0;
        loc_fst = -1;
        num_back = 0;
        stall = 0;
        tet = jd->root_tet;
        if (jd->root_region != region) load_region(jd->root_region);
        if (kRecord) {
            rhash = 14695981039346656037ull;
            rsteps = rhits = rscatters = rrestores = rdetections = rsurvivals = 0;
            rcontrib = 0.0;
        }
    }

    // SpinTheta, src/octmps_kernel.cuh:807-820.
    __device__ __forceinline__ T spin_theta(T g) {
        T cost;
        if (g == (T)0) {
            cost = (T)2 * ((T)1 - rand_co_S()) - (T)1;
        } else {
            const T r = (T)1 - rand_co_S();
            const T temp = DevNum<T>::div(DevNum<T>::mad(-g, g, (T)1), DevNum<T>::mad(g + g, r, (T)1 - g));
            cost = DevNum<T>::div(DevNum<T>::mad(-temp, temp, DevNum<T>::mad(g, g, (T)1)), g + g);
            if (cost < (T)-1) cost = -1;
            else if (cost > (T)1) cost = 1;
        }
        return cost;
    }

    // SpinThetaForwardFstBias, src/octmps_kernel.cuh:881-896.
    __device__ __forceinline__ T spin_theta_forward(T g) {
        T cost;
        if (g == (T)0) {
            cost = (T)1 - rand_co_S();
        } else {
            const T r = (T)1 - rand_co_S();
            const T temp = DevNum<T>::div(r, (T)1 - g) +
                           DevNum<T>::div((T)1 - r, sqrtT(DevNum<T>::mad(g, g, (T)1)));
            cost = DevNum<T>::div(DevNum<T>::mad(g, g, (T)1) - DevNum<T>::div((T)1, temp * temp), g + g);
            if (cost < (T)-1) cost = -1;
            else if (cost > (T)1) cost = 1;
        }
        return cost;
    }

    // New direction from polar cosine `cost` and a drawn azimuth about
    // (ax, ay, az) (src/octmps_kernel.cuh:844-868 and 1006-1026).
    __device__ __forceinline__ void rotate(T cost, T ax, T ay, T az, bool copysign_form) {
        const T sint = sqrtT(DevNum<T>::mad(-cost, cost, (T)1));
        T sinp, cosp;
        sincos_rand(rand_co_S(), sinp, cosp);
        const T stcp = sint * cosp;
        const T stsp = sint * sinp;
        if (fabsT(az) > DevNum<T>::coszero) {
            ux = stcp;
            uy = stsp;
            uz = copysign_form ? copysignT(cost, az * cost) : cost * (az >= (T)0 ? (T)1 : (T)-1);
        } else {
            // RSQRT(x) taken as 1/sqrt(x), both correctly rounded.
            const T sq = sqrtT(DevNum<T>::mad(-az, az, (T)1));
            const T temp = rcpT(sq);
            ux = DevNum<T>::mad(DevNum<T>::mad(stcp * ax, az, -(stsp * ay)), temp, ax * cost);
            uy = DevNum<T>::mad(DevNum<T>::mad(stcp * ay, az, stsp * ax), temp, ay * cost);
            // FAST_DIV(-stcp, temp) = -stcp * sqrt(1 - uz^2): multiplied in
            // the FP32 forms, divided in the FP64 form
            uz = DevNum<T>::mad(az, cost, kFused<T> ? -(stcp * sq) : DevNum<T>::div(-stcp, temp));
        }
    }

    // SpinBias, src/octmps_kernel.cuh:898-1086.
    __device__ void spin_bias(SplitCopy<T, P> &cont) {
        const JobDesc &J = *jd;
        const T g = rg.g;
        const T g2 = g * g;
        T ax = ux, ay = uy, az = uz;
        const T ox = ux, oy = uy, oz = uz;
        T btmp = 0;
        int reached = 0;
        bool first = false;
        if (z > (T)J.tdmin && z < (T)J.tdmax && uz > (T)0 && !fst_flag) {
            cont.x = x;
            cont.y = y;
            cont.z = z;
            cont.ux = ux;
            cont.uy = uy;
            cont.uz = uz;
            cont.w = w;
            cont.max_depth = max_depth;
            cont.lr = lr;
            cont.op = op;
            cont.tet = tet;
            cont.region = region;
            cont.num_back = num_back;
            reached = 1;
            fst_flag = 1;
            loc_fst = z;
            btmp = (T)J.bias_a;
            first = true;
        }
        T vx = px - x;
        T vy = py - y;
        T vz = pz - z;
        const T len = sqrtT(DevNum<T>::mad(vz, vz, DevNum<T>::mad(vx, vx, vy * vy)));
        if (kFused<T>) {
            const T rl = rcpT(len);  // FP32 forms: one reciprocal, three products
            vx *= rl;
            vy *= rl;
            vz *= rl;
        } else {
            vx = DevNum<T>::div(vx, len);
            vy = DevNum<T>::div(vy, len);
            vz = DevNum<T>::div(vz, len);
        }
        if ((fst_flag || num_back > 0) && !reached) {
            reached = 2;
            // -log(0)/mu_t is +infinity: with rndStepSizeInTissue = 0 the
            // distance test always holds.
            const T rs = (T)J.rnd_step;
            const bool far = rs == (T)0 || DevNum<T>::div(-log_method(rs), rg.muas) >= len;
            if (far && -vz >= (T)J.cos_collect) reached = 1;
            btmp = (T)J.bias_a;
        }
        int sel = 0;
        T cost;
        const T pb = (T)J.p_bias;
        if (reached) {
            sel = rand_co_S() <= pb ? 1 : 2;
            if (reached == 1 || sel == 1) {
                cost = spin_theta_forward(btmp);
                ax = vx;
                ay = vy;
                az = vz;
            } else {
                cost = spin_theta(g);
            }
        } else {
            cost = spin_theta(g);
        }
        cost = fmaxT(cost, (T)-1);
        cost = fminT(cost, (T)1);
        rotate(cost, ax, ay, az, true);

        T costg = dot3<T>(ox, oy, oz, ux, uy, uz);
        T costg1 = dot3<T>(vx, vy, vz, ux, uy, uz);
        if (kFused<T>) {
            // FP32 forms: a direction rotated about a nearly vertical axis is
            // off unit length by a few tenths of a percent (1 - uz*uz
            // cancels), so a cosine can exceed 1 and 1 + g*g - 2*g*cos go
            // negative under the square root (a NaN likelihood): clamp.
            costg = fminT(fmaxT(costg, (T)-1), (T)1);
            costg1 = fminT(fmaxT(costg1, (T)-1), (T)1);
        }
        if (btmp != (T)0) {
            const T opa2 = DevNum<T>::mad(btmp, btmp, (T)1);
            const T sq_opa2 = sqrtT(opa2);
            T f;
            if (reached == 1) {
                const T b1 = opa2 - (btmp + btmp) * cost;
                const T h1 = DevNum<T>::mad(g, g, (T)1) - (g + g) * costg;
                const T num = ((T)1 - g2) * (sq_opa2 - (T)1 + btmp) * sqrtT(b1 * b1 * b1);
                const T den = (btmp + btmp) * ((T)1 - btmp) * sq_opa2 * sqrtT(h1 * h1 * h1);
                f = DevNum<T>::div(num, den);
            } else {
                const T c1 = sel == 1 ? cost : costg1;
                const T c2 = sel == 1 ? costg : cost;
                const T b1 = opa2 - (btmp + btmp) * c1;
                const T pdf1 = DevNum<T>::div(sq_opa2 * btmp * ((T)1 - btmp),
                                              (sq_opa2 - (T)1 + btmp) * sqrtT(b1 * b1 * b1));
                const T h2 = sqrtT(DevNum<T>::mad(g, g, (T)1) - (g + g) * c2);
                const T pdf2 = DevNum<T>::div((T)1 - g2, (T)2 * (h2 * h2 * h2));
                f = DevNum<T>::div(pdf2, DevNum<T>::mad(pb, pdf1, ((T)1 - pb) * pdf2));
            }
            lr *= f;
            if (first) lr_after = lr;
        }
    }

    // First half of a propagation step, OCTMPSKernel's loop body
    // (src/octmps_kernel.cuh:1351-1392): step size, boundary test, hop and,
    // when a face is reached, reflection or transmission and the roulette.
    // Returns kDone, kEnd (the packet ended) or kPending (no face reached:
    // the step continues in phase_b).
    __device__ __forceinline__ int phase_a(SplitCopy<T, P> &cont, unsigned int *err) {
        int ev = 0;
        // ComputeStepSize, :505-515
        if (sleft == (T)0) {
            const T r = (T)1 - rand_co_G();
            s = -log_method(r) * rg.rmuas;
        } else {
            s = sleft * rg.rmuas;
            sleft = 0;
        }
        // HitBoundary, :517-572
        Plane4<T> pl;
        pl.load(planes, tet);
        const int4 nb = __ldg(adj + tet);
        T cosv[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) cosv[k] = dot3<T>(pl.v[k][0], pl.v[k][1], pl.v[k][2], ux, uy, uz);
        T min_d = DevNum<T>::big;
        T min_cos = 0;
        int face = -1;
        if (kFused<T>) {
            // FP32 forms: nearest face by perp_i * c_j < perp_j * c_i
            // (c = -cos > 0), one division for the winner.
            T best_perp = 0, best_c = 0;
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                if (cosv[k] < (T)0) {
                    const T perp = dot3<T>(pl.v[k][0], pl.v[k][1], pl.v[k][2], x, y, z) + pl.v[k][3];
                    const T c = -cosv[k];
                    const bool nearer = face < 0 ? perp < DevNum<T>::big * c
                                                 : perp * best_c < best_perp * c;
                    if (nearer) {
                        best_perp = perp;
                        best_c = c;
                        face = k;
                    }
                }
            }
            if (face >= 0) {
                min_d = DevNum<T>::div(best_perp, best_c);
                min_cos = -best_c;
            }
        } else {
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                if (cosv[k] < (T)0) {
                    const T perp = dot3<T>(pl.v[k][0], pl.v[k][1], pl.v[k][2], x, y, z) + pl.v[k][3];
                    const T t = DevNum<T>::div(-perp, cosv[k]);
                    if (t < min_d) {
                        min_d = t;
                        face = k;
                        min_cos = cosv[k];
                    }
                }
            }
        }
        const bool hit = s > min_d;
        if (hit) {
            sleft = (s - min_d) * rg.muas;
            s = min_d;
        }
        stall = (hit && s <= (T)0) ? stall + 1 : 0;
        // Hop, :574-582
        x = DevNum<T>::mad(s, ux, x);
        y = DevNum<T>::mad(s, uy, y);
        z = DevNum<T>::mad(s, uz, z);
        op += (P)s;
        if (max_depth < z) max_depth = z;

        if (hit) {
            if (face < 0) {
                atomicOr(err, kErrNoExitFace);
                return kEnd;
            }
            // FastReflectTransmit, :590-775
            if (kRecord) ++rhits;
            const T ca1 = -min_cos;
            const int32_t entry = face == 0 ? nb.x : face == 1 ? nb.y : face == 2 ? nb.z : nb.w;
            const int next_region = entry < 0 ? 0 : (int)((uint32_t)entry >> kAdjIndexBits);
            // A neighbour entry must name a tet of the mesh and a region of
            // the job's table: the job API checks the mesh at upload, the
            // allocation-free entry point takes the caller's array unchecked.
            if (entry >= 0 && (next_region >= jd->n_regions ||
                               (int32_t)((uint32_t)entry & kAdjIndexMask) >= jd->n_tets)) {
                atomicOr(err, kErrBadNeighbour);
                return kEnd;
            }
            const T nt = entry < 0 ? (T)jd->n_ambient
                                   : __ldg(reinterpret_cast<const T *>(regions + next_region));
            T r;
            T sa1 = sqrtT(DevNum<T>::mad(-ca1, ca1, (T)1));
            if (ca1 > DevNum<T>::coszero) sa1 = 0;
            if (kFused<T> && rg.n == nt) {
                // FP32 forms, matched refractive indices: R is exactly 0
                // except for the grazing-incidence rule (sa2 = sa1 here).
                r = (ca1 < DevNum<T>::cos90 || sa1 == (T)1) ? (T)1 : (T)0;
            } else {
                const T ni_nt = DevNum<T>::div(rg.n, nt);
                const T sa2 = fminT(ni_nt * sa1, (T)1);
                const T ca2 = sqrtT(DevNum<T>::mad(-sa2, sa2, (T)1));
                const T ca1ca2 = ca1 * ca2;
                const T sa1sa2 = sa1 * sa2;
                T sa1ca2 = sa1 * ca2;
                T ca1sa2 = ca1 * sa2;
                if (ca1 > DevNum<T>::coszero) {
                    sa1ca2 = 1;
                    ca1sa2 = ni_nt;
                }
                const T cam = ca1ca2 + sa1sa2;
                const T sap = sa1ca2 + ca1sa2;
                const T sam = sa1ca2 - ca1sa2;
                r = DevNum<T>::div(sam, sap * cam);
                r = r * r;
                r = r * DevNum<T>::mad(ca1ca2, ca1ca2, sa1sa2 * sa1sa2);
                if (ca1 < DevNum<T>::cos90 || sa2 == (T)1) r = 1;
            }

            const T fnx = face == 0 ? pl.v[0][0] : face == 1 ? pl.v[1][0] : face == 2 ? pl.v[2][0] : pl.v[3][0];
            const T fny = face == 0 ? pl.v[0][1] : face == 1 ? pl.v[1][1] : face == 2 ? pl.v[2][1] : pl.v[3][1];
            const T fnz = face == 0 ? pl.v[0][2] : face == 1 ? pl.v[1][2] : face == 2 ? pl.v[2][2] : pl.v[3][2];
            const T two_ca1 = ca1 + ca1;
            const T rx = DevNum<T>::mad(two_ca1, fnx, ux);
            const T ry = DevNum<T>::mad(two_ca1, fny, uy);
            const T rz = DevNum<T>::mad(two_ca1, fnz, uz);
            const T rnd = rand_co_R();
            if (entry < 0 && r < (T)1) {
                ev = 4;
                if (uz < (T)0) {
                    bool filt = false;
                    const T dx = x - px;
                    const T dy = y - py;
                    const T rr = sqrtT(DevNum<T>::mad(dx, dx, dy * dy));
                    if (rr < (T)jd->radius && -uz > (T)jd->cos_collect) {
                        if (type_bias == 0 || type_bias == 3) filt = true;
                        if ((fst_flag && type_bias == 37) || (loc_fst == max_depth && type_bias != 37) ||
                            num_back > 0)
                            filt = true;
                    }
                    if (filt) {
                        const int nbins_added = tally_detection<T, P>(jd, op, max_depth, w, r, lr);
                        if (kRecord) {
                            const P cp = (P)(w * ((T)1 - r) * lr);
                            for (int k = 0; k < nbins_added; ++k) rcontrib += (double)cp;
                        }
                        ev |= 8;
                        if (kRecord) ++rdetections;
                    }
                } else {
                    num_back++;
                }
                w *= r;
                ux = rx;
                uy = ry;
                uz = rz;
            } else if (rnd > r) {
                const int next = (int)((uint32_t)entry & kAdjIndexMask);
                tet = next;
                if (next_region != region) load_region(next_region);
                ev = 2;
            } else {
                if (uz > (T)0) num_back++;
                ux = rx;
                uy = ry;
                uz = rz;
                ev = 3;
            }
        } else {
            return kPending;  // the scattering half of the step runs in phase_b
        }
        return finish(ev, cont) ? kEnd : kDone;
    }

    // Second half of a step that did not reach a face: Drop, then Spin or
    // SpinBias (:1359-1369), then the roulette.  Returns true when the
    // packet ends.
    __device__ __forceinline__ bool phase_b(SplitCopy<T, P> &cont) {
        if (kRecord) ++rscatters;
        // Drop, :584-588
        w = DevNum<T>::mad(-w, rg.mua_muas, w);
        if (type_bias == 0) {
            rotate(spin_theta(rg.g), ux, uy, uz, false);
        } else if (type_bias == 37) {
            spin_bias(cont);
        }
        return finish(1, cont);
    }

    // Roulette, :1376-1392, and the step's record.  Returns true when the
    // packet ends.
    __device__ __forceinline__ bool finish(int ev, SplitCopy<T, P> &cont) {
        bool end = false;
        if (w < DevNum<T>::weight) {
            const T rnd = rand_co_G();
            if (w != (T)0 && rnd < DevNum<T>::chance) {
                w *= DevNum<T>::div((T)1, DevNum<T>::chance);
                ev |= 16;
                if (kRecord) ++rsurvivals;
            } else if (fst_flag && type_bias != 3) {
                const T lr_tmp = lr_after;
                x = cont.x;
                y = cont.y;
                z = cont.z;
                ux = cont.ux;
                uy = cont.uy;
                uz = cont.uz;
                w = cont.w;
                max_depth = cont.max_depth;
                lr = cont.lr;
                op = cont.op;
                tet = cont.tet;
                num_back = cont.num_back;
                fst_flag = 0;
                loc_fst = -1;
                sleft = 0;
                if (cont.region != region) load_region(cont.region);
                rotate(spin_theta(rg.g), ux, uy, uz, false);
                lr = lr_tmp < (T)1 ? (T)1 - lr_tmp : (T)1;
                ev |= 32;
                if (kRecord) ++rrestores;
                restores_++;
                stall = 0;
            } else {
                ev |= 64;
                end = true;
            }
        }
        if (kRecord) {
            rhash = fnv(rhash, ((unsigned long long)(uint32_t)tet << 8) | (unsigned long long)ev);
            ++rsteps;
        }
        return end;
    }
    uint32_t restores_;
    uint32_t stall;  // consecutive boundary hits that did not move the photon
};

// kMinBlocks: resident blocks per SM the register allocation must allow
// (2: up to 128 registers per thread; 3: up to 80).
template <typename T, typename P, bool kRecord, int kMinBlocks>
__global__ void __launch_bounds__(kBlock, kMinBlocks)
    photon_kernel(const LaunchArgs args, PacketRecordDev *records) {
    __shared__ SplitCopy<T, P> cont_all[kBlock];
    SplitCopy<T, P> &cont = cont_all[threadIdx.x];
    Lane<T, P, kRecord> L;
    L.jd = nullptr;
    L.region = -1;
    L.restores_ = 0;
    // packets still to run in the current unit (the runtime keeps a job's
    // packets per lane below 2^32) and steps of the current packet (capped
    // at step_cap <= 2^32)
    uint32_t packets_left = 0, steps_packet = 0;
    bool recording = false;

    // Lanes of this warp still in the loop, and whether this lane's current
    // step waits for its scattering half.  A warp runs, per iteration, either
    // the first half of a step on its lanes that have one to start, or the
    // scattering half on the lanes waiting for it; it switches to the
    // scattering half once at least kScatterShare/32 of its live lanes wait
    // (or no lane can start a step).  Each lane still performs exactly the
    // reference's sequence of operations; only the interleaving of lanes
    // changes, so the warp executes the long scattering code for many lanes
    // at once instead of on almost every iteration.
    unsigned live = 0xffffffffu;
    bool pending = false;
    const int share = args.scatter_share;
    unsigned int *const err = reinterpret_cast<unsigned int *>(args.ctrl + 2);
    // First units: in a launch started on an idle table, thread t takes unit
    // start_unit + t; in one started beside a running launch, each block
    // claims a run of units at once (a grid's worth of threads arriving
    // together would otherwise contend for the counter one by one).
    __shared__ unsigned long long s_first;
    __shared__ unsigned s_count;
    // threads of this block that hold a unit (or have not yet looked for one)
    __shared__ unsigned s_busy;
    unsigned long long first_u;
    bool first_ok;
    if (threadIdx.x == 0) {
        s_busy = kBlock;
        s_first = 0;
        s_count = 0;
        if (args.initial_total == 0) s_count = claim_units(args.ctrl, kBlock, s_first);
    }
    __syncthreads();
    if (args.initial_total == 0) {
        first_u = s_first + threadIdx.x;
        first_ok = threadIdx.x < s_count;
    } else {
        first_u = args.start_unit + (blockIdx.x * (unsigned long long)kBlock + threadIdx.x);
        first_ok = first_u < args.initial_total;
    }
    bool first_unit = true;
    // A thread that finds no unit left waits for jobs appended while the
    // launch runs: it retries after kRetryUs, doubling the interval up to
    // kRetryMaxUs (the counter's cache line is shared by every waiting warp).
    // It exits once its whole block has been without work for linger_us, or
    // at once when the host asks the launch to drain (control word 3): a
    // block stays resident until its last thread exits, so threads leaving
    // one by one would hold the block's SM slot for a few long lanes while
    // new work found no free threads.  Times from the global timer in
    // 1.024 us ticks.
    // This state, and the current unit's job slot and lane, are touched only
    // between units (and at a stop), so they live in shared memory rather
    // than in registers the propagation loop needs.
    struct UnitState {
        uint32_t idle_since, last_try, gap;
        int32_t slot;   // job slot of the current unit
        uint32_t lane;  // its RNG lane (lane counts are 32-bit)
        bool waiting, drain;
    };
    __shared__ UnitState s_unit[kBlock];
    UnitState &lg = s_unit[threadIdx.x];
    lg.waiting = lg.drain = false;
    lg.idle_since = lg.last_try = 0;
    lg.gap = kRetryUs;
    lg.slot = 0;
    lg.lane = ~0u;

    for (;;) {
        bool has_work = true;
        bool idle = false;
        if (packets_left == 0) {
            unsigned long long u = 0;
            bool got = false;
            if (first_unit) {
                first_unit = false;
                u = first_u;
                got = first_ok;
            }
            if (!got) {
                const uint32_t now = timer_us();
                if (!lg.waiting || now - lg.last_try >= lg.gap) {
                    got = take_unit(args.ctrl, u);
                    if (!got) lg.drain = __ldcv(args.ctrl + 3) != 0ull;
                    lg.last_try = now;
                    if (lg.waiting && lg.gap < kRetryMaxUs) lg.gap <<= 1;
                }
                if (!got) {
                    if (!lg.waiting) {
                        lg.waiting = true;
                        atomicSub(&s_busy, 1u);
                        lg.idle_since = now;
                    }
                    if (*reinterpret_cast<volatile unsigned *>(&s_busy) != 0u) lg.idle_since = now;
                    if (lg.drain || now - lg.idle_since >= args.linger_us) has_work = false;
                    else idle = true;
                }
            }
            if (got) {
                if (lg.waiting) atomicAdd(&s_busy, 1u);
                lg.waiting = false;
                lg.gap = kRetryUs;
                // the slot holding unit u: the last one whose base is <= u
                // (bases of empty slots are ~0); read past L1, the host may
                // have filled the slot after this launch started
                int lo = 0, hi = args.n_slots - 1;
                while (lo < hi) {
                    const int mid = (lo + hi + 1) >> 1;
                    if (__ldcg(args.unit_base + mid) <= u) lo = mid;
                    else hi = mid - 1;
                }
                lg.slot = lo;
                const JobDesc *jd = args.jobs + lo;
                const uint64_t v = u - __ldcg(args.unit_base + lo);
                if (jd != L.jd) {
                    L.jd = jd;
                    L.regions = reinterpret_cast<const RegionConst<T> *>(jd->regions);
                    L.planes = jd->planes;
                    L.adj = reinterpret_cast<const int4 *>(jd->adj);
                    L.px = (T)jd->probe_x;
                    L.py = (T)jd->probe_y;
                    L.pz = (T)jd->probe_z;
                    L.type_bias = jd->type_bias;
                    L.region = -1;
                }
                L.xG = jd->rng_x[v];
                L.aG = jd->rng_a[v];
                L.xR = jd->rng_xR[v];
                L.aR = jd->rng_aR[v];
                L.xS = jd->rng_xS[v];
                L.aS = jd->rng_aS[v];
                const uint64_t nl = jd->n_lanes;
                packets_left = (uint32_t)(jd->n_photons / nl + (v < jd->n_photons % nl ? 1 : 0));
                if (packets_left == 0) {
                    idle = true;  // a lane without packets: take another unit next time
                    unit_finished(args, lg.slot, jd->n_lanes);
                } else {
                    L.launch();
                    steps_packet = 0;
                    pending = false;
                    recording = kRecord && records && lo == args.record_slot;
                    lg.lane = (uint32_t)v;
                }
            }
        }
        // The two vote sites below are reached by every live lane in every
        // iteration.
        live = __ballot_sync(live, has_work);
        if (!has_work) break;
        const unsigned pend = __ballot_sync(live, pending && !idle);
        const unsigned ready = __ballot_sync(live, !pending && !idle);
        const bool run_b = ready == 0u || __popc(pend) * 32 >= share * __popc(live);
        if ((pend | ready) == 0u) __nanosleep(kIdleSleepNs);  // every live lane waits for work
        if (idle) continue;
        bool end;
        if (run_b) {
            if (!pending) continue;
            pending = false;
            end = L.phase_b(cont);
        } else {
            if (pending) continue;
            const int r = L.phase_a(cont, err);
            if (r == kPending) {
                pending = true;
                continue;
            }
            end = r == kEnd;
        }
        ++steps_packet;
        bool done = end;
        // A packet is stopped (its split copy too) at the step cap, an
        // error, or after kStallHits boundary hits in a row that did not
        // move it: a photon on a face moving parallel to it (the cosine of
        // incidence below the grazing limit) is reflected with its direction
        // unchanged, the same hit again at distance 0, forever.
        unsigned reason = 0;
        if (!done && steps_packet >= args.step_cap) {
            atomicOr(err, kErrStepCap);
            reason = 1;
        } else if (!done && L.stall >= kStallHits) {
            reason = 2;
        }
        if (reason) {
            atomicAdd(&L.jd->stats[3], 1ull);
            done = true;
        }
        if (reason) {
            Incident *inc = args.incident;
            if (inc && atomicCAS(&inc->flag, 0u, reason) == 0u) {
                inc->slot = (unsigned)lg.slot;
                inc->tet = L.tet;
                inc->packets_left = packets_left;
                inc->lane = lg.lane;
                inc->steps = steps_packet;
                inc->pos[0] = (double)L.x;
                inc->pos[1] = (double)L.y;
                inc->pos[2] = (double)L.z;
                inc->dir[0] = (double)L.ux;
                inc->dir[1] = (double)L.uy;
                inc->dir[2] = (double)L.uz;
                inc->w = (double)L.w;
                inc->sleft = (double)L.sleft;
            }
        }
        if (done) {
            // per-packet statistics: steps, split copies resumed, packets
            atomicAdd(&L.jd->stats[0], (unsigned long long)steps_packet);
            if (L.restores_) atomicAdd(&L.jd->stats[1], (unsigned long long)L.restores_);
            atomicAdd(&L.jd->stats[2], 1ull);
            L.restores_ = 0;
            if (kRecord && recording) {
                PacketRecordDev r;
                r.hash = L.rhash;
                r.x = L.xG;
                r.xR = L.xR;
                r.xS = L.xS;
                r.steps = L.rsteps;
                r.hits = L.rhits;
                r.scatters = L.rscatters;
                r.restores = L.rrestores;
                r.detections = L.rdetections;
                r.survivals = L.rsurvivals;
                r.contribution = L.rcontrib;
                r.optical_path = (double)L.op;
                records[lg.lane] = r;
                recording = false;
            }
            --packets_left;
            if (packets_left) {
                L.launch();
                steps_packet = 0;
            } else {
                unit_finished(args, lg.slot, L.jd->n_lanes);
            }
        }
    }
}

}  // namespace

namespace {

template <typename T, typename P>
const void *pick(int min_blocks, bool record) {
    if (record) return (const void *)photon_kernel<T, P, true, 2>;
    switch (min_blocks) {
        case 2: return (const void *)photon_kernel<T, P, false, 2>;
        case 3: return (const void *)photon_kernel<T, P, false, 3>;
        case 4: return (const void *)photon_kernel<T, P, false, 4>;
        default: return nullptr;
    }
}

const void *photon_kernel_fn(int precision, int min_blocks, bool record) {
    switch (precision) {
        case kMixed: return pick<float, double>(min_blocks, record);
        case kFP32: return pick<float, float>(min_blocks, record);
        case kFP64: return pick<double, double>(2, record);  // spills at 80 registers
        default: return nullptr;
    }
}

}  // namespace

int launch_photon_kernel(int precision, int min_blocks, const LaunchArgs &args, int grid,
                         int block, void *stream, void *records) {
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    PacketRecordDev *rec = reinterpret_cast<PacketRecordDev *>(records);
    if (block != kBlock) return (int)cudaErrorInvalidValue;
    const void *fn = photon_kernel_fn(precision, min_blocks, rec != nullptr);
    if (!fn) return (int)cudaErrorInvalidValue;
    void *params[2] = {const_cast<LaunchArgs *>(&args), &rec};
    return (int)cudaLaunchKernel(fn, dim3(grid), dim3(block), params, 0, st);
}

int photon_kernel_attributes(int precision, int block, int min_blocks, int *regs,
                             int *max_blocks_per_sm) {
    cudaFuncAttributes a;
    const void *fn = photon_kernel_fn(precision, min_blocks, false);
    if (!fn) return (int)cudaErrorInvalidValue;
    cudaError_t e = cudaFuncGetAttributes(&a, fn);
    if (e != cudaSuccess) return (int)e;
    *regs = a.numRegs;
    int nb = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, fn, block, 0);
    if (e != cudaSuccess) return (int)e;
    *max_blocks_per_sm = nb;
    return 0;
}

}  // namespace octmps
