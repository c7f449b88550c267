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

// Results of a half-step besides its event code (>= 1): no face reached, the
// scattering half still to do; or the packet ended on an error.
constexpr int kEvPending = -1;
constexpr int kEvError = -2;

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

// A photon's split copy: its state at the first biased scattering toward the
// probe (src/octmps_kernel.cuh:933-951), resumed when the photon dies
// (:1376-1392).  save() stores a lane's state, restore() puts it back (all
// but the region, which it returns).  The per-lane kernel keeps one record
// per thread in shared memory, the pooled kernel one per photon in global
// memory.
template <typename T, typename P>
struct SplitCopy {
    T x, y, z, ux, uy, uz, w, max_depth, lr;
    P op;
    int32_t tet, region;
    uint32_t num_back;
    template <class L>
    __device__ __forceinline__ void save(const L &l) {
        x = l.x;
        y = l.y;
        z = l.z;
        ux = l.ux;
        uy = l.uy;
        uz = l.uz;
        w = l.w;
        max_depth = l.max_depth;
        lr = l.lr;
        op = l.op;
        tet = l.tet;
        region = l.region;
        num_back = l.num_back;
    }
    template <class L>
    __device__ __forceinline__ int32_t restore(L &l) const {
        l.x = x;
        l.y = y;
        l.z = z;
        l.ux = ux;
        l.uy = uy;
        l.uz = uz;
        l.w = w;
        l.max_depth = max_depth;
        l.lr = lr;
        l.op = op;
        l.tet = tet;
        l.num_back = num_back;
        return region;
    }
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
// instead of registers.  With RecordPhotonsFlag (a record buffer in the job)
// it also keeps the packet's record: weight leaving, likelihood ratio, radius
// rr and cosine -uz at the exit, optical path and maximum depth.  Returns the
// number of bins the contribution went to.
template <typename T, typename P>
__device__ __noinline__ int tally_detection(const JobDesc *jd, P op, T max_depth, T w,
                                            T r_fresnel, T lr, T rr, T cos_exit) {
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
    const T wt = w * ((T)1 - r_fresnel);
    const T c = wt * lr;
    const P cp = (P)c;
    if (J.photon_records) {
        const unsigned long long k = atomicAdd(&J.stats[4], 1ull);
        if (k < J.record_cap) {
            PhotonRecordDev &rec = J.photon_records[k];
            rec.weight = (double)wt;
            rec.likelihood = (double)lr;
            rec.radius = (double)rr;
            rec.cos_angle = (double)cos_exit;
            rec.optical_path = (double)op;
            rec.max_depth = (double)max_depth;
        }
    }
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
    // photon (s_next: the step size drawn ahead for the next step, pooled kernel)
    T x, y, z, ux, uy, uz, w, s, sleft, max_depth, lr, lr_after, loc_fst, s_next;
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
    // The probe position and bias type are read from the job descriptor
    // where they are used (launches, biased scatterings, exits): held in
    // registers across the step loop they were spilled to local memory.
    __device__ __forceinline__ T px() const { return (T)__ldg(&jd->probe_x); }
    __device__ __forceinline__ T py() const { return (T)__ldg(&jd->probe_y); }
    __device__ __forceinline__ T pz() const { return (T)__ldg(&jd->probe_z); }
    __device__ __forceinline__ int32_t type_bias() const { return __ldg(&jd->type_bias); }
    // record of the current packet (kRecord only)
    unsigned long long rhash;
    uint32_t rsteps, rhits, rscatters, rrestores, rdetections, rsurvivals;
    double rcontrib;

    __device__ __forceinline__ T rand_co_G() { return DevNum<T>::rand_value(mwc_next(xG, aG)); }
    __device__ __forceinline__ T rand_co_R() { return DevNum<T>::rand_value(mwc_next(xR, aR)); }
    __device__ __forceinline__ T rand_co_S() { return DevNum<T>::rand_value(mwc_next(xS, aS)); }

    // The current region's n, mu_t and 1/mu_t stay in registers (every step
    // uses them); its other constants are read where a scattering uses them.
    __device__ __forceinline__ void load_region(int r) {
        const RegionConst<T> *c = regions + r;
        rg.n = __ldg(&c->n);
        rg.muas = __ldg(&c->muas);
        rg.rmuas = __ldg(&c->rmuas);
        region = r;
    }
    __device__ __forceinline__ const RegionConst<T> *rc() const { return regions + region; }

    // LaunchPhoton, src/octmps_kernel.cuh:475-503.
    __device__ __forceinline__ void launch() {
        x = px();
        y = py();
        z = pz();
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

    // SpinTheta, src/octmps_kernel.cuh:807-820, with the current region's g:
    // temp = (1 - g^2) / (1 + 2 g r - g), cost = (1 + g^2 - temp^2) / 2g.
    __device__ __forceinline__ T spin_theta() {
        const RegionConst<T> *c = rc();
        T cost;
        const T g = __ldg(&c->g);
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

    // SpinThetaForwardFstBias, src/octmps_kernel.cuh:881-896, with the job's
    // bias coefficient b: temp = r / (1 - b) + (1 - r) / sqrt(1 + b^2),
    // cost = (1 + b^2 - 1 / temp^2) / 2b, the root from the region constants.
    __device__ __forceinline__ T spin_theta_forward() {
        const RegionConst<T> *c = rc();
        const T b = (T)jd->bias_a;
        T cost;
        if (b == (T)0) {
            cost = (T)1 - rand_co_S();
        } else {
            const T r = (T)1 - rand_co_S();
            const T temp = DevNum<T>::div(r, (T)1 - b) + DevNum<T>::div((T)1 - r, __ldg(&c->b_sq1p2));
            cost = DevNum<T>::div(DevNum<T>::mad(b, b, (T)1) - DevNum<T>::div((T)1, temp * temp), b + b);
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
    template <class C>
    __device__ void spin_bias(C &cont) {
        const JobDesc &J = *jd;
        const RegionConst<T> *c = rc();
        T ax = ux, ay = uy, az = uz;
        const T ox = ux, oy = uy, oz = uz;
        T btmp = 0;
        int reached = 0;
        bool first = false;
        if (z > (T)J.tdmin && z < (T)J.tdmax && uz > (T)0 && !fst_flag) {
            cont.save(*this);
            reached = 1;
            fst_flag = 1;
            loc_fst = z;
            btmp = (T)J.bias_a;
            first = true;
        }
        T vx = px() - x;
        T vy = py() - y;
        T vz = pz() - z;
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
            // -log(rndStepSizeInTissue) / mu_t from the region constants
            // (+infinity for a step of 0: the distance test always holds)
            const bool far = __ldg(&c->far) >= len;
            if (far && -vz >= (T)J.cos_collect) reached = 1;
            btmp = (T)J.bias_a;
        }
        int sel = 0;
        T cost;
        const T pb = (T)J.p_bias;
        if (reached) {
            sel = rand_co_S() <= pb ? 1 : 2;
            if (reached == 1 || sel == 1) {
                cost = spin_theta_forward();
                ax = vx;
                ay = vy;
                az = vz;
            } else {
                cost = spin_theta();
            }
        } else {
            cost = spin_theta();
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
            // b = btmp (the job's coefficient); sqrt(1 + b^2) comes from the
            // region constants
            T f;
            if (reached == 1) {
                const T g = __ldg(&c->g), sq = __ldg(&c->b_sq1p2);
                const T b1 = DevNum<T>::mad(btmp, btmp, (T)1) - (btmp + btmp) * cost;
                const T h1 = DevNum<T>::mad(g, g, (T)1) - (g + g) * costg;
                const T num = ((T)1 - g * g) * (sq - (T)1 + btmp) * sqrtT(b1 * b1 * b1);
                const T den = (btmp + btmp) * ((T)1 - btmp) * sq * sqrtT(h1 * h1 * h1);
                f = DevNum<T>::div(num, den);
            } else {
                const T c1 = sel == 1 ? cost : costg1;
                const T c2 = sel == 1 ? costg : cost;
                const T g = __ldg(&c->g), sq = __ldg(&c->b_sq1p2);
                const T b1 = DevNum<T>::mad(btmp, btmp, (T)1) - (btmp + btmp) * c1;
                const T pdf1 = DevNum<T>::div(sq * btmp * ((T)1 - btmp), (sq - (T)1 + btmp) * sqrtT(b1 * b1 * b1));
                const T h2 = sqrtT(DevNum<T>::mad(g, g, (T)1) - (g + g) * c2);
                const T pdf2 = DevNum<T>::div((T)1 - g * g, (T)2 * (h2 * h2 * h2));
                f = DevNum<T>::div(pdf2, DevNum<T>::mad(pb, pdf1, ((T)1 - pb) * pdf2));
            }
            lr *= f;
            if (first) lr_after = lr;
        }
    }

    // ComputeStepSize's draw for a step that starts with sleft == 0,
    // src/octmps_kernel.cuh:505-515.  The kernels draw it at the end of the
    // previous step (after its roulette and stop checks) or at the launch:
    // the general stream's draws keep their order, and the first half of a
    // step no longer diverges on the logarithm.
    __device__ __forceinline__ void draw_step() {
        const T r = (T)1 - rand_co_G();  // in [2^-24, 1]: normal
        s_next = -log_method_normal(r) * rg.rmuas;
    }

    // First half of a propagation step, OCTMPSKernel's loop body
    // (src/octmps_kernel.cuh:1351-1392): step size, boundary test, hop and,
    // when a face is reached, reflection or transmission.  Returns the event
    // code for finish() (the roulette, called once per step by the loop),
    // kEvPending when no face was reached (the step continues in half_b) or
    // kEvError.
    __device__ __forceinline__ int half_a(unsigned int *err) {
        int ev = 0;
        // ComputeStepSize, :505-515: a fresh step's size was drawn ahead
        // (draw_step), a remaining one is converted with the current region's
        // 1/mu_t
        s = sleft == (T)0 ? s_next : sleft * rg.rmuas;
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
            // (c = -cos > 0), one division for the winner.  Starting from
            // (perp, c) = (big, 1) makes the first candidate's test
            // perp * 1 < big * c, exactly the distance test against big, and
            // leaves min_d = big / 1 = big when no face is a candidate.
            T best_perp = DevNum<T>::big, best_c = 1;
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                const T perp = dot3<T>(pl.v[k][0], pl.v[k][1], pl.v[k][2], x, y, z) + pl.v[k][3];
                const T c = -cosv[k];
                if (cosv[k] < (T)0 && perp * best_c < best_perp * c) {
                    best_perp = perp;
                    best_c = c;
                    face = k;
                }
            }
            min_d = DevNum<T>::div(best_perp, best_c);
            min_cos = -best_c;
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
        sleft = hit ? (s - min_d) * rg.muas : (T)0;
        s = hit ? min_d : s;
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
                return kEvError;
            }
            // FastReflectTransmit, :590-775
            if (kRecord) ++rhits;
            const T ca1 = -min_cos;
            const int32_t entry = face == 0 ? nb.x : face == 1 ? nb.y : face == 2 ? nb.z : nb.w;
            const int next_region = entry < 0 ? 0 : (int)((uint32_t)entry >> kAdjIndexBits);
            const T nt = entry < 0                ? (T)jd->n_ambient
                         : next_region == region ? rg.n
                                                 : __ldg(&regions[next_region].n);
            T r;
            const T sa1_sq = DevNum<T>::mad(-ca1, ca1, (T)1);
            if (kFused<T> && rg.n == nt) {
                // FP32 forms, matched refractive indices: R is exactly 0
                // except for the grazing-incidence rule (sa2 = sa1 here).
                // sa1 = sqrt(1 - ca1^2) is 1 exactly when its argument is 1
                // (the correctly rounded root of the largest float below 1
                // is below 1), and 0 when ca1 > COSZERO: no root needed.
                r = (ca1 < DevNum<T>::cos90 || (sa1_sq == (T)1 && !(ca1 > DevNum<T>::coszero)))
                        ? (T)1
                        : (T)0;
            } else {
                T sa1 = sqrtT(sa1_sq);
                if (ca1 > DevNum<T>::coszero) sa1 = 0;
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
                    const T dx = x - px();
                    const T dy = y - py();
                    const T rr = sqrtT(DevNum<T>::mad(dx, dx, dy * dy));
                    if (rr < (T)jd->radius && -uz > (T)jd->cos_collect) {
                        const int32_t tb = type_bias();
                        if (tb == 0 || tb == 3) filt = true;
                        if ((fst_flag && tb == 37) || (loc_fst == max_depth && tb != 37) ||
                            num_back > 0)
                            filt = true;
                    }
                    if (filt) {
                        const int nbins_added =
                            tally_detection<T, P>(jd, op, max_depth, w, r, lr, rr, -uz);
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
            return kEvPending;  // the scattering half of the step runs in half_b
        }
        return ev;
    }

    // Second half of a step that did not reach a face: Drop, then Spin or
    // SpinBias (:1359-1369).  Returns the event code for finish().
    template <class C>
    __device__ __forceinline__ int half_b(C &cont) {
        if (kRecord) ++rscatters;
        // Drop, :584-588
        w = DevNum<T>::mad(-w, __ldg(&rc()->mua_muas), w);
        const int32_t tb = type_bias();
        if (tb == 0) {
            rotate(spin_theta(), ux, uy, uz, false);
        } else if (tb == 37) {
            spin_bias(cont);
        }
        return 1;
    }

    // Roulette, :1376-1392, and the step's record.  Returns true when the
    // packet ends.
    template <class C>
    __device__ __forceinline__ bool finish(int ev, C &cont) {
        bool end = false;
        if (w < DevNum<T>::weight) {
            const T rnd = rand_co_G();
            if (w != (T)0 && rnd < DevNum<T>::chance) {
                w *= DevNum<T>::div((T)1, DevNum<T>::chance);
                ev |= 16;
                if (kRecord) ++rsurvivals;
            } else if (fst_flag && type_bias() != 3) {
                const T lr_tmp = lr_after;
                const int32_t cr = cont.restore(*this);
                fst_flag = 0;
                loc_fst = -1;
                sleft = 0;
                if (cr != region) load_region(cr);
                rotate(spin_theta(), ux, uy, uz, false);
                lr = lr_tmp < (T)1 ? (T)1 - lr_tmp : (T)1;
                ev |= 32;
                if (kRecord) ++rrestores;
                atomicAdd(&jd->stats[1], 1ull);  // split copies resumed (rare)
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
    uint32_t stall;  // consecutive boundary hits that did not move the photon
};

// kBlk threads per block; kMinBlocks: resident blocks per SM the register
// allocation must allow (65,536 registers per SM: 256 x 3 blocks, up to 80
// registers per thread; 128 x 7, up to 72; 256 x 2, up to 128).
template <typename T, typename P, bool kRecord, int kBlk, int kMinBlocks>
__global__ void __launch_bounds__(kBlk, kMinBlocks)
    photon_kernel(const LaunchArgs args, PacketRecordDev *records) {
    // one split copy per thread (touched only at first biased scatterings and
    // restores, so the record layout's bank conflicts cost little; a table
    // with one column per field measured 10 % slower: its base address is
    // held in registers across the loop)
    __shared__ SplitCopy<T, P> cont_all[kBlk];
    SplitCopy<T, P> &cont = cont_all[threadIdx.x];
    Lane<T, P, kRecord> L;
    L.jd = nullptr;
    L.region = -1;
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
        s_busy = kBlk;
        s_first = 0;
        s_count = 0;
        if (args.initial_total == 0) s_count = claim_units(args.ctrl, kBlk, s_first);
    }
    __syncthreads();
    if (args.initial_total == 0) {
        first_u = s_first + threadIdx.x;
        first_ok = threadIdx.x < s_count;
    } else {
        first_u = args.start_unit + (blockIdx.x * (unsigned long long)kBlk + threadIdx.x);
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
    __shared__ UnitState s_unit[kBlk];
    UnitState &lg = s_unit[threadIdx.x];
    lg.waiting = lg.drain = false;
    lg.idle_since = lg.last_try = 0;
    lg.gap = kRetryUs;
    lg.slot = 0;
    lg.lane = ~0u;

    for (;;) {
        // Lanes without a unit (at the start, after a unit's last packet,
        // while waiting for work) look for one; the warp takes this path
        // together, so an iteration in which every lane holds a unit costs
        // one vote for it.
        bool idle = false;
        unsigned idle_mask = 0u;
        if (__any_sync(live, packets_left == 0)) {
        bool has_work = true;
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
                    L.draw_step();
                    steps_packet = 0;
                    pending = false;
                    recording = kRecord && records && lo == args.record_slot;
                    lg.lane = (uint32_t)v;
                }
            }
        }
        live = __ballot_sync(live, has_work);
        if (!has_work) break;
        idle_mask = __ballot_sync(live, idle);
        if (idle_mask == live) {  // every live lane waits for work
            __nanosleep(kIdleSleepNs);
            continue;
        }
        }
        // The vote below is reached by every live lane in every iteration
        // (an idle lane is never pending).
        const unsigned pend = __ballot_sync(live, pending);
        const unsigned ready = live & ~pend & ~idle_mask;
        const bool run_b = ready == 0u || __popc(pend) * 32 >= share * __popc(live);
        if (run_b ? !pending : (pending || idle)) continue;
        int ev;
        if (run_b) {
            pending = false;
            ev = L.half_b(cont);
        } else {
            ev = L.half_a(err);
            if (ev == kEvPending) {
                pending = true;
                continue;
            }
        }
        // one roulette call site for both halves (its code inlined once)
        const bool end = ev == kEvError || L.finish(ev, cont);
        ++steps_packet;
        bool done = end;
        // A packet is stopped (its split copy too) at the step cap, an
        // error, or after kStallHits boundary hits in a row that did not
        // move it: a photon on a face moving parallel to it (the cosine of
        // incidence below the grazing limit) is reflected with its direction
        // unchanged, the same hit again at distance 0, forever.
        if (!done && (steps_packet >= args.step_cap || L.stall >= kStallHits)) {
            const unsigned reason = steps_packet >= args.step_cap ? 1u : 2u;
            if (reason == 1u) atomicOr(err, kErrStepCap);
            atomicAdd(&L.jd->stats[3], 1ull);
            done = true;
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
        if (!done && L.sleft == (T)0) L.draw_step();  // the next step's size, drawn ahead
        if (done) {
            // per-packet statistics: steps, split copies resumed, packets
            atomicAdd(&L.jd->stats[0], (unsigned long long)steps_packet);
            atomicAdd(&L.jd->stats[2], 1ull);
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
                L.draw_step();
                steps_packet = 0;
            } else {
                unit_finished(args, lg.slot, L.jd->n_lanes);
            }
        }
    }
}


// ------------------------------------------------------------------------
// Pooled kernel: photons held in shared memory, phases run in full warps.
//
// Each warp keeps up to kPool photons (two per lane) in its own slice of
// shared memory, as two stacks: photons whose next step starts with the
// boundary test (stack A, positions [0, nA)) and photons that reached no
// face and wait for their scattering half (stack B, positions
// [kPool - nB, kPool)).  Every iteration the warp pops up to 32 photons of
// one stack (B once it holds a full warp's worth, else the fuller one), runs
// that half of a step on all of them at once, and pushes each result onto
// the stack of its next half.  Both halves thus run with (nearly) every lane
// busy, where one photon per thread left a warp's lanes split between the
// halves.  A photon's arithmetic is that of the per-lane kernel above, step
// for step: only which lane runs it changes.  The step size of a step that
// starts with sleft == 0 is drawn at the end of the previous step (after its
// roulette and stop checks) or at the launch, which keeps the general
// stream's draws in order and takes the logarithm out of the boundary half.
//
// Measured on the B-scan workload (8 A-scans x 2e5 packets, B200): the
// pooled form raises active threads per warp instruction from 15.7 to 23.5,
// but spends 44 % more thread instructions (moving photon state and reloading
// job constants every half-step) and, at 128 registers, keeps 16 warps per SM
// resident against the per-lane kernel's 24 (issue active 48 % vs 60 %):
// 28.9 G against 37.7 G propagation steps/s.  It is kept as a launch variant
// (octmps_launch_config.kernel_form = 1) that the autotuner times.
//
// A photon's state is 16-byte chunks (8 for the mixed and FP32 forms, 16 for
// FP64 and the recording variant); chunk k of the photon at position q sits
// at chunk (k ^ (q & 7)) of its record, so that 8 consecutive photons read or
// write a given chunk through 8 different bank groups.  Split copies live
// in global memory, one per photon identity ("home") of the warp, which a
// photon keeps across its packets and units.

constexpr int kPoolBlock = 128;  // threads (4 warps) per block
constexpr int kPoolWarps = kPoolBlock / 32;
constexpr int kPool = 64;        // photons per warp

// Word layout of a pooled photon (32-bit words; t = words per geometry value):
//   [0, 13t)        x y z ux uy uz w sleft s_next max_depth lr lr_after loc_fst
//   META + 0..10    tet | region << 24, flags, num_back, steps of the packet,
//                   packets left (the current one included), job slot, RNG
//                   lane, home, aG, aR, aS
//   OP, XG, XR, XS  optical path (P), generator states (2 words each)
//   REC             recording variant: hash (2), steps, hits, scatters,
//                   restores, detections, survivals, contribution (2)
// flags: bit 31 fst_flag, bit 30 the packet is recorded, bits 0-29 stall.
template <typename T, typename P, bool kRecord>
struct PoolLayout {
    static constexpr int t = (int)(sizeof(T) / 4);
    static constexpr int META = 13 * t;
    static constexpr int OP = META + 11;
    static constexpr int XG = OP + 2, XR = XG + 2, XS = XR + 2;
    static constexpr int REC = XS + 2;
    static constexpr int WORDS = REC + (kRecord ? 10 : 0);
    static constexpr int USED = (WORDS + 3) / 4;           // 16-byte chunks in use
    static constexpr int CHUNKS = USED <= 8 ? 8 : 16;      // record stride (power of two)
    static constexpr int PADDED = 4 * USED;
    static_assert(USED <= 16, "a pooled photon is at most 16 chunks");
};

static_assert(PoolLayout<float, double, false>::CHUNKS == 8, "mixed form: 8 chunks");
static_assert(PoolLayout<float, float, false>::CHUNKS == 8, "FP32 form: 8 chunks");

constexpr uint32_t kFlagFst = 1u << 31;
constexpr uint32_t kFlagRec = 1u << 30;
constexpr uint32_t kStallMask = (1u << 30) - 1u;

// Per-photon fields kept beside the lane's registers while a half-step runs.
struct PoolMeta {
    int32_t slot;
    uint32_t lane, home, packets_left, steps_packet, flags;
    uint32_t aG, aR, aS;
};

__device__ __forceinline__ void put_w(uint32_t *w, int i, float v) { w[i] = __float_as_uint(v); }
__device__ __forceinline__ void put_w(uint32_t *w, int i, double v) {
    w[i] = (uint32_t)__double2loint(v);
    w[i + 1] = (uint32_t)__double2hiint(v);
}
__device__ __forceinline__ void put_w(uint32_t *w, int i, unsigned long long v) {
    w[i] = (uint32_t)v;
    w[i + 1] = (uint32_t)(v >> 32);
}
template <typename F>
__device__ __forceinline__ F get_w(const uint32_t *w, int i);
template <>
__device__ __forceinline__ float get_w<float>(const uint32_t *w, int i) { return __uint_as_float(w[i]); }
template <>
__device__ __forceinline__ double get_w<double>(const uint32_t *w, int i) {
    return __hiloint2double((int)w[i + 1], (int)w[i]);
}
template <>
__device__ __forceinline__ unsigned long long get_w<unsigned long long>(const uint32_t *w, int i) {
    return (unsigned long long)w[i] | ((unsigned long long)w[i + 1] << 32);
}

// Chunk k of the photon at position q is chunk (k ^ (q & 7)) of its record.
template <typename Lay>
__device__ __forceinline__ void pool_read(const float4 *pool, int q, uint32_t (&w)[Lay::PADDED]) {
#pragma unroll
    for (int k = 0; k < Lay::USED; ++k) {
        const float4 c = pool[q * Lay::CHUNKS + (k ^ (q & 7))];
        w[4 * k + 0] = __float_as_uint(c.x);
        w[4 * k + 1] = __float_as_uint(c.y);
        w[4 * k + 2] = __float_as_uint(c.z);
        w[4 * k + 3] = __float_as_uint(c.w);
    }
}

template <typename Lay>
__device__ __forceinline__ void pool_write(float4 *pool, int q, const uint32_t (&w)[Lay::PADDED]) {
#pragma unroll
    for (int k = 0; k < Lay::USED; ++k)
        pool[q * Lay::CHUNKS + (k ^ (q & 7))] =
            make_float4(__uint_as_float(w[4 * k + 0]), __uint_as_float(w[4 * k + 1]),
                        __uint_as_float(w[4 * k + 2]), __uint_as_float(w[4 * k + 3]));
}

// The lane's registers (and the job's constants) from a pooled photon.
template <typename T, typename P, bool kRecord>
__device__ __forceinline__ void unpack(const uint32_t *w, const LaunchArgs &args, PoolMeta &m,
                                       Lane<T, P, kRecord> &L) {
    using Lay = PoolLayout<T, P, kRecord>;
    constexpr int t = Lay::t, M = Lay::META;
    m.slot = (int32_t)w[M + 5];
    m.lane = w[M + 6];
    m.home = w[M + 7];
    m.packets_left = w[M + 4];
    m.steps_packet = w[M + 3];
    m.flags = w[M + 1];
    m.aG = w[M + 8];
    m.aR = w[M + 9];
    m.aS = w[M + 10];
    const JobDesc *jd = args.jobs + m.slot;
    L.jd = jd;
    L.regions = reinterpret_cast<const RegionConst<T> *>(jd->regions);
    L.planes = jd->planes;
    L.adj = reinterpret_cast<const int4 *>(jd->adj);
    L.x = get_w<T>(w, 0 * t);
    L.y = get_w<T>(w, 1 * t);
    L.z = get_w<T>(w, 2 * t);
    L.ux = get_w<T>(w, 3 * t);
    L.uy = get_w<T>(w, 4 * t);
    L.uz = get_w<T>(w, 5 * t);
    L.w = get_w<T>(w, 6 * t);
    L.sleft = get_w<T>(w, 7 * t);
    L.s_next = get_w<T>(w, 8 * t);
    L.max_depth = get_w<T>(w, 9 * t);
    L.lr = get_w<T>(w, 10 * t);
    L.lr_after = get_w<T>(w, 11 * t);
    L.loc_fst = get_w<T>(w, 12 * t);
    L.op = get_w<P>(w, Lay::OP);
    L.tet = (int32_t)(w[M] & kAdjIndexMask);
    L.load_region((int)(w[M] >> kAdjIndexBits));
    L.fst_flag = (m.flags & kFlagFst) ? 1u : 0u;
    L.stall = m.flags & kStallMask;
    L.num_back = w[M + 2];
    L.xG = get_w<unsigned long long>(w, Lay::XG);
    L.xR = get_w<unsigned long long>(w, Lay::XR);
    L.xS = get_w<unsigned long long>(w, Lay::XS);
    L.aG = m.aG;
    L.aR = m.aR;
    L.aS = m.aS;
    if constexpr (kRecord) {
        constexpr int R = Lay::REC;
        L.rhash = get_w<unsigned long long>(w, R);
        L.rsteps = w[R + 2];
        L.rhits = w[R + 3];
        L.rscatters = w[R + 4];
        L.rrestores = w[R + 5];
        L.rdetections = w[R + 6];
        L.rsurvivals = w[R + 7];
        L.rcontrib = get_w<double>(w, R + 8);
    }
}

template <typename T, typename P, bool kRecord>
__device__ __forceinline__ void pack(const Lane<T, P, kRecord> &L, const PoolMeta &m,
                                     uint32_t (&w)[PoolLayout<T, P, kRecord>::PADDED]) {
    using Lay = PoolLayout<T, P, kRecord>;
    constexpr int t = Lay::t, M = Lay::META;
#pragma unroll
    for (int i = Lay::WORDS; i < Lay::PADDED; ++i) w[i] = 0u;
    put_w(w, 0 * t, L.x);
    put_w(w, 1 * t, L.y);
    put_w(w, 2 * t, L.z);
    put_w(w, 3 * t, L.ux);
    put_w(w, 4 * t, L.uy);
    put_w(w, 5 * t, L.uz);
    put_w(w, 6 * t, L.w);
    put_w(w, 7 * t, L.sleft);
    put_w(w, 8 * t, L.s_next);
    put_w(w, 9 * t, L.max_depth);
    put_w(w, 10 * t, L.lr);
    put_w(w, 11 * t, L.lr_after);
    put_w(w, 12 * t, L.loc_fst);
    w[M] = (uint32_t)L.tet | ((uint32_t)L.region << kAdjIndexBits);
    w[M + 1] = (m.flags & kFlagRec) | (L.fst_flag ? kFlagFst : 0u) | (L.stall & kStallMask);
    w[M + 2] = L.num_back;
    w[M + 3] = m.steps_packet;
    w[M + 4] = m.packets_left;
    w[M + 5] = (uint32_t)m.slot;
    w[M + 6] = m.lane;
    w[M + 7] = m.home;
    w[M + 8] = m.aG;
    w[M + 9] = m.aR;
    w[M + 10] = m.aS;
    w[Lay::OP + 1] = 0u;
    put_w(w, Lay::OP, L.op);
    put_w(w, Lay::XG, (unsigned long long)L.xG);
    put_w(w, Lay::XR, (unsigned long long)L.xR);
    put_w(w, Lay::XS, (unsigned long long)L.xS);
    if constexpr (kRecord) {
        constexpr int R = Lay::REC;
        put_w(w, R, (unsigned long long)L.rhash);
        w[R + 2] = L.rsteps;
        w[R + 3] = L.rhits;
        w[R + 4] = L.rscatters;
        w[R + 5] = L.rrestores;
        w[R + 6] = L.rdetections;
        w[R + 7] = L.rsurvivals;
        put_w(w, R + 8, L.rcontrib);
    }
}

// Starts unit u (a job's RNG lane): its slot, generators and packet count,
// and its first packet, with the first step size drawn.  Returns false when
// the lane has no packets (it is reported finished at once).
template <typename T, typename P, bool kRecord>
__device__ __forceinline__ bool start_unit(const LaunchArgs &args, unsigned long long u,
                                           PacketRecordDev *records, PoolMeta &m,
                                           Lane<T, P, kRecord> &L) {
    // the slot holding unit u: the last one whose base is <= u (bases of
    // empty slots are ~0); read past L1, the host may have filled the slot
    // after this launch started
    int lo = 0, hi = args.n_slots - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (__ldcg(args.unit_base + mid) <= u) lo = mid;
        else hi = mid - 1;
    }
    const JobDesc *jd = args.jobs + lo;
    const uint64_t v = u - __ldcg(args.unit_base + lo);
    const uint64_t nl = jd->n_lanes;
    const uint32_t packets = (uint32_t)(jd->n_photons / nl + (v < jd->n_photons % nl ? 1 : 0));
    if (packets == 0) {
        unit_finished(args, lo, jd->n_lanes);
        return false;
    }
    m.slot = lo;
    m.lane = (uint32_t)v;
    m.packets_left = packets;
    m.steps_packet = 0;
    m.flags = (kRecord && records && lo == args.record_slot) ? kFlagRec : 0u;
    m.aG = jd->rng_a[v];
    m.aR = jd->rng_aR[v];
    m.aS = jd->rng_aS[v];
    L.jd = jd;
    L.regions = reinterpret_cast<const RegionConst<T> *>(jd->regions);
    L.planes = jd->planes;
    L.adj = reinterpret_cast<const int4 *>(jd->adj);
    L.region = -1;
    L.xG = jd->rng_x[v];
    L.xR = jd->rng_xR[v];
    L.xS = jd->rng_xS[v];
    L.aG = m.aG;
    L.aR = m.aR;
    L.aS = m.aS;
    L.launch();
    L.draw_step();
    return true;
}

// The n-th (from 0) set bit of the 64-bit mask hi:lo.
__device__ __forceinline__ uint32_t nth_set_bit(uint32_t lo, uint32_t hi, int n) {
    const int c = __popc(lo);
    return n < c ? (uint32_t)__fns(lo, 0, n + 1) : 32u + (uint32_t)__fns(hi, 0, n - c + 1);
}

template <typename T, typename P, bool kRecord, int kMinBlocks>
__global__ void __launch_bounds__(kPoolBlock, kMinBlocks)
    pooled_kernel(const LaunchArgs args, PacketRecordDev *records, SplitCopy<T, P> *splits) {
    using Lay = PoolLayout<T, P, kRecord>;
    extern __shared__ float4 pool_smem[];
    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    const unsigned full = 0xffffffffu;
    const unsigned below = (1u << lane) - 1u;
    float4 *const pool = pool_smem + (size_t)warp * kPool * Lay::CHUNKS;
    SplitCopy<T, P> *const wsplit = splits + ((size_t)blockIdx.x * kPoolWarps + warp) * kPool;
    unsigned int *const err = reinterpret_cast<unsigned int *>(args.ctrl + 2);
    const int share = args.scatter_share;

    // First units, two per thread, as the per-lane kernel takes them: in a
    // launch on an idle table thread t takes units start_unit + 2t and
    // start_unit + 2t + 1; a launch beside a running one claims a run of
    // 2 x kPoolBlock units per block.
    __shared__ unsigned long long s_first;
    __shared__ unsigned s_count;
    __shared__ unsigned s_busy;  // warps of this block holding photons
    if (threadIdx.x == 0) {
        s_busy = kPoolWarps;
        s_first = 0;
        s_count = 0;
        if (args.initial_total == 0) s_count = claim_units(args.ctrl, 2 * kPoolBlock, s_first);
    }
    __syncthreads();

    int nA = 0, nB = 0;                    // stack heights (warp-uniform)
    uint32_t home_lo = 0u, home_hi = 0u;   // free homes (split-copy slots) of the warp
    {
        const unsigned long long tid = (unsigned long long)blockIdx.x * kPoolBlock + threadIdx.x;
#pragma unroll 1
        for (int r = 0; r < 2; ++r) {
            unsigned long long u;
            bool got;
            if (args.initial_total == 0) {
                const unsigned idx = (unsigned)(threadIdx.x * 2 + r);
                u = s_first + idx;
                got = idx < s_count;
            } else {
                u = args.start_unit + 2 * tid + r;
                got = u < args.initial_total;
            }
            PoolMeta m;
            Lane<T, P, kRecord> L;
            if (got) got = start_unit<T, P, kRecord>(args, u, records, m, L);
            const unsigned b = __ballot_sync(full, got);
            if (got) {
                m.home = (uint32_t)(r * 32 + lane);
                uint32_t w[Lay::PADDED];
                pack(L, m, w);
                pool_write<Lay>(pool, nA + __popc(b & below), w);
            }
            if (r == 0) home_lo = ~b;
            else home_hi = ~b;
            nA += __popc(b);
        }
        __syncwarp();
    }

    // Refills and waiting: a warp with free homes takes units from the
    // counter; after an attempt that found none it retries after kRetryUs,
    // doubling up to kRetryMaxUs.  A warp without photons waits for jobs
    // appended while the launch runs; the block leaves once all its warps
    // have been without photons for linger_us, or when the host drains the
    // launch.
    bool waiting = false, last_ok = true;
    uint32_t idle_since = 0, last_try = 0, gap = kRetryUs;

#pragma unroll 1
    for (;;) {
        const int n_free = __popc(home_lo) + __popc(home_hi);
        uint32_t now = 0;  // the warp's decisions below use lane 0's clock and reads
        if (n_free > 0) {
            now = __shfl_sync(full, timer_us(), 0);
            if (last_ok || now - last_try >= gap) {
                const int want = n_free < 32 ? n_free : 32;
                unsigned long long u = 0;
                bool got = false;
                if (lane < want) got = take_unit(args.ctrl, u);
                PoolMeta m;
                Lane<T, P, kRecord> L;
                if (got) got = start_unit<T, P, kRecord>(args, u, records, m, L);
                const unsigned b = __ballot_sync(full, got);
                if (got) {
                    const int rank = __popc(b & below);
                    m.home = nth_set_bit(home_lo, home_hi, rank);
                    uint32_t w[Lay::PADDED];
                    pack(L, m, w);
                    pool_write<Lay>(pool, nA + rank, w);
                }
                for (int k = __popc(b); k > 0; --k) {  // the homes taken: the lowest free ones
                    if (home_lo) home_lo &= home_lo - 1u;
                    else home_hi &= home_hi - 1u;
                }
                nA += __popc(b);
                last_ok = b != 0u;
                if (last_ok) {
                    gap = kRetryUs;
                } else {
                    if (gap < kRetryMaxUs) gap <<= 1;
                    last_try = now;
                }
                __syncwarp();
            }
        }
        if (nA + nB == 0) {
            if (n_free == 0) now = __shfl_sync(full, timer_us(), 0);
            if (!waiting) {
                waiting = true;
                if (lane == 0) atomicSub(&s_busy, 1u);
                idle_since = now;
            }
            __syncwarp();
            unsigned busy = 0u, drain = 0u;
            if (lane == 0) {
                busy = *reinterpret_cast<volatile unsigned *>(&s_busy);
                drain = __ldcv(args.ctrl + 3) != 0ull ? 1u : 0u;
            }
            busy = __shfl_sync(full, busy, 0);
            drain = __shfl_sync(full, drain, 0);
            if (busy != 0u) idle_since = now;
            if (drain || now - idle_since >= args.linger_us) break;
            __nanosleep(kIdleSleepNs);
            continue;
        }
        if (waiting) {
            waiting = false;
            if (lane == 0) atomicAdd(&s_busy, 1u);
        }

        // ---- one half-step for up to 32 photons of one stack: B once it
        // holds a warp's worth; with fewer than 32 photons on A, B once it
        // holds at least share/32 of the warp's photons
        const bool run_b = nB >= 32 || nA == 0 || (nA < 32 && nB * 32 >= share * (nA + nB));
        const int mcount = run_b ? min(nB, 32) : min(nA, 32);
        const bool active = lane < mcount;
        PoolMeta m;
        Lane<T, P, kRecord> L;
        if (active) {
            uint32_t w[Lay::PADDED];
            pool_read<Lay>(pool, run_b ? (kPool - nB + lane) : (nA - mcount + lane), w);
            unpack(w, args, m, L);
        }
        __syncwarp();
        int to = 0;  // 0: leaves the pool, 1: stack A, 2: stack B
        if (active) {
            SplitCopy<T, P> &cont = wsplit[m.home];
            const int ev = run_b ? L.half_b(cont) : L.half_a(err);
            const bool step_done = ev != kEvPending;
            const bool end = step_done && (ev == kEvError || L.finish(ev, cont));
            if (!step_done) {
                to = 2;
            } else {
                ++m.steps_packet;
                bool done = end;
                unsigned reason = 0;
                if (!done && m.steps_packet >= args.step_cap) {
                    atomicOr(err, kErrStepCap);
                    reason = 1;
                } else if (!done && L.stall >= kStallHits) {
                    reason = 2;
                }
                if (reason) {
                    atomicAdd(&L.jd->stats[3], 1ull);
                    done = true;
                    Incident *inc = args.incident;
                    if (inc && atomicCAS(&inc->flag, 0u, reason) == 0u) {
                        inc->slot = (unsigned)m.slot;
                        inc->tet = L.tet;
                        inc->packets_left = m.packets_left;
                        inc->lane = m.lane;
                        inc->steps = m.steps_packet;
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
                if (!done) {
                    if (L.sleft == (T)0) L.draw_step();
                    to = 1;
                } else {
                    atomicAdd(&L.jd->stats[0], (unsigned long long)m.steps_packet);
                    atomicAdd(&L.jd->stats[2], 1ull);
                    if (kRecord && (m.flags & kFlagRec)) {
                        PacketRecordDev rr;
                        rr.hash = L.rhash;
                        rr.x = L.xG;
                        rr.xR = L.xR;
                        rr.xS = L.xS;
                        rr.steps = L.rsteps;
                        rr.hits = L.rhits;
                        rr.scatters = L.rscatters;
                        rr.restores = L.rrestores;
                        rr.detections = L.rdetections;
                        rr.survivals = L.rsurvivals;
                        rr.contribution = L.rcontrib;
                        rr.optical_path = (double)L.op;
                        records[m.lane] = rr;
                        m.flags &= ~kFlagRec;
                    }
                    if (--m.packets_left) {
                        // the unit's next packet, from the same generators
                        L.launch();
                        L.draw_step();
                        m.steps_packet = 0;
                        to = 1;
                    } else {
                        unit_finished(args, m.slot, L.jd->n_lanes);
                        // the next unit, in the same home
                        unsigned long long u = 0;
                        const uint32_t home = m.home;
                        if (take_unit(args.ctrl, u) &&
                            start_unit<T, P, kRecord>(args, u, records, m, L)) {
                            m.home = home;
                            to = 1;
                        }
                    }
                }
            }
        }
        // ---- push: A grows up from its popped base, B down from its end
        const int baseA = run_b ? nA : nA - mcount;
        const int baseB = run_b ? nB - mcount : nB;
        const unsigned bA = __ballot_sync(full, to == 1);
        const unsigned bB = __ballot_sync(full, to == 2);
        if (to) {
            uint32_t w[Lay::PADDED];
            pack(L, m, w);
            pool_write<Lay>(pool, to == 1 ? baseA + __popc(bA & below)
                                          : kPool - baseB - 1 - __popc(bB & below), w);
        }
        // homes of photons that left the pool become free
        const bool left = active && to == 0;
        const uint32_t h = left ? m.home : 0u;
        home_lo |= __reduce_or_sync(full, left && h < 32 ? (1u << h) : 0u);
        home_hi |= __reduce_or_sync(full, left && h >= 32 ? (1u << (h - 32)) : 0u);
        nA = baseA + __popc(bA);
        nB = baseB + __popc(bB);
        __syncwarp();
    }
}

}  // namespace

namespace {

// Per-lane variants: 256-thread blocks at 2, 3 or 4 per SM, 128-thread
// blocks at 6, 7 or 8, 512-thread blocks at 2 (FP32 geometry forms); the
// FP64 form and the recording variant run 256 x 2 (they spill at 80
// registers).
template <typename T, typename P>
const void *pick(int block, int min_blocks, bool record) {
    if (record) return block == 256 ? (const void *)photon_kernel<T, P, true, 256, 2> : nullptr;
    if constexpr (sizeof(T) == sizeof(double)) {
        return block == 256 && min_blocks == 2 ? (const void *)photon_kernel<T, P, false, 256, 2>
                                               : nullptr;
    } else {
    switch (block * 16 + min_blocks) {
        case 256 * 16 + 2: return (const void *)photon_kernel<T, P, false, 256, 2>;
        case 256 * 16 + 3: return (const void *)photon_kernel<T, P, false, 256, 3>;
        case 256 * 16 + 4: return (const void *)photon_kernel<T, P, false, 256, 4>;
        case 128 * 16 + 6: return (const void *)photon_kernel<T, P, false, 128, 6>;
        case 128 * 16 + 7: return (const void *)photon_kernel<T, P, false, 128, 7>;
        case 128 * 16 + 8: return (const void *)photon_kernel<T, P, false, 128, 8>;
        case 512 * 16 + 2: return (const void *)photon_kernel<T, P, false, 512, 2>;
        default: return nullptr;
    }
    }
}

const void *photon_kernel_fn(int precision, int block, int min_blocks, bool record) {
    switch (precision) {
        case kMixed: return pick<float, double>(block, min_blocks, record);
        case kFP32: return pick<float, float>(block, min_blocks, record);
        case kFP64: return pick<double, double>(block, min_blocks, record);
        default: return nullptr;
    }
}

// Pooled variants: 4, 5 or 6 resident 128-thread blocks per SM (register caps
// 128, 96 and 80) in the FP32 geometry forms; the FP64 form and the
// recording variant (16-chunk photon records, 64 KB of shared memory per
// block) run 2 or 3.
template <typename T, typename P>
const void *pick_pooled(int min_blocks, bool record) {
    if (record) return (const void *)pooled_kernel<T, P, true, 2>;
    if (sizeof(T) == sizeof(double)) {
        switch (min_blocks) {
            case 2: return (const void *)pooled_kernel<T, P, false, 2>;
            case 3: return (const void *)pooled_kernel<T, P, false, 3>;
            default: return nullptr;
        }
    }
    switch (min_blocks) {
        case 4: return (const void *)pooled_kernel<T, P, false, 4>;
        case 5: return (const void *)pooled_kernel<T, P, false, 5>;
        case 6: return (const void *)pooled_kernel<T, P, false, 6>;
        default: return nullptr;
    }
}

const void *pooled_kernel_fn(int precision, int min_blocks, bool record) {
    switch (precision) {
        case kMixed: return pick_pooled<float, double>(min_blocks, record);
        case kFP32: return pick_pooled<float, float>(min_blocks, record);
        case kFP64: return pick_pooled<double, double>(min_blocks, record);
        default: return nullptr;
    }
}

template <typename T, typename P, bool kRecord>
constexpr size_t pooled_smem() {
    return (size_t)kPoolWarps * kPool * PoolLayout<T, P, kRecord>::CHUNKS * 16;
}

size_t pooled_smem_bytes(int precision, bool record) {
    switch (precision) {
        case kMixed: return record ? pooled_smem<float, double, true>() : pooled_smem<float, double, false>();
        case kFP32: return record ? pooled_smem<float, float, true>() : pooled_smem<float, float, false>();
        default: return record ? pooled_smem<double, double, true>() : pooled_smem<double, double, false>();
    }
}

// Opts a pooled variant in to its dynamic shared memory (once per function).
cudaError_t pooled_prepare(const void *fn, size_t smem) {
    cudaFuncAttributes a;
    cudaError_t e = cudaFuncGetAttributes(&a, fn);
    if (e != cudaSuccess) return e;
    if ((size_t)a.maxDynamicSharedSizeBytes < smem)
        e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    return e;
}

}  // namespace

int launch_photon_kernel(int precision, int min_blocks, const LaunchArgs &args, int grid,
                         int block, void *stream, void *records) {
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    PacketRecordDev *rec = reinterpret_cast<PacketRecordDev *>(records);
    const void *fn = photon_kernel_fn(precision, block, min_blocks, rec != nullptr);
    if (!fn) return (int)cudaErrorInvalidValue;
    void *params[2] = {const_cast<LaunchArgs *>(&args), &rec};
    return (int)cudaLaunchKernel(fn, dim3(grid), dim3(block), params, 0, st);
}

bool photon_kernel_variant(int precision, int block, int min_blocks) {
    return photon_kernel_fn(precision, block, min_blocks, false) != nullptr;
}

int photon_kernel_attributes(int precision, int block, int min_blocks, int *regs,
                             int *max_blocks_per_sm) {
    cudaFuncAttributes a;
    const void *fn = photon_kernel_fn(precision, block, min_blocks, false);
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

size_t pooled_split_bytes(int precision, int grid) {
    const size_t per = precision == kFP64 ? sizeof(SplitCopy<double, double>)
                       : precision == kFP32 ? sizeof(SplitCopy<float, float>)
                                            : sizeof(SplitCopy<float, double>);
    return (size_t)grid * kPoolWarps * kPool * per;
}

int launch_pooled_kernel(int precision, int min_blocks, const LaunchArgs &args, int grid,
                         void *stream, void *records, void *splits) {
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    PacketRecordDev *rec = reinterpret_cast<PacketRecordDev *>(records);
    const void *fn = pooled_kernel_fn(precision, min_blocks, rec != nullptr);
    if (!fn || !splits) return (int)cudaErrorInvalidValue;
    const size_t smem = pooled_smem_bytes(precision, rec != nullptr);
    cudaError_t e = pooled_prepare(fn, smem);
    if (e != cudaSuccess) return (int)e;
    void *params[3] = {const_cast<LaunchArgs *>(&args), &rec, &splits};
    return (int)cudaLaunchKernel(fn, dim3(grid), dim3(kPoolBlock), params, smem, st);
}

int pooled_kernel_attributes(int precision, int min_blocks, bool record, int *regs,
                             int *max_blocks_per_sm) {
    const void *fn = pooled_kernel_fn(precision, min_blocks, record);
    if (!fn) return (int)cudaErrorInvalidValue;
    const size_t smem = pooled_smem_bytes(precision, record);
    cudaError_t e = pooled_prepare(fn, smem);
    if (e != cudaSuccess) return (int)e;
    cudaFuncAttributes a;
    e = cudaFuncGetAttributes(&a, fn);
    if (e != cudaSuccess) return (int)e;
    *regs = a.numRegs;
    int nb = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, fn, kPoolBlock, smem);
    if (e != cudaSuccess) return (int)e;
    *max_blocks_per_sm = nb;
    return 0;
}

}  // namespace octmps
