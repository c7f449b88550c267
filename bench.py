"""Benchmark of the OCT-MPS photon-transport hot path on B200.

Workload (the headline configuration): the B-scan of a 4 x 2 x 2 mm box of
tissue with an ellipsoid and two spheres, meshed as 64x32x31 Kuhn-split
cubes (380,928 tets), 256 A-scans 10 um apart, 1e6 photon packets each,
seeds 1..256, mixed precision (FP32 geometry, FP64 path length and
tallies).  One step = one batch of --batch (default 32) consecutive A-scans
of the scan run in one persistent launch; successive steps walk along the
scan.  (The whole B-scan is about 3.2e12 propagation steps, minutes of GPU
time, so a step is a slice of it.)  Synthetic inputs of
the configuration's shapes and optical properties (generated by
oct-mps_b200/meshgen.py); no dataset is involved.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

value: packets/s of the whole job, device-timed (CUDA events around the
persistent launch on the library's stream), inputs resident in HBM.
e2e: the same metric through the C-ABI a user calls: mesh upload from host
arrays, job submission (RNG lanes seeded on the host and copied), the
launch, and the download of every A-scan's tallies, wall-clock per step.
Under torchrun each rank runs its own B-scan (seeds offset by rank): weak
scaling, no collective on the data path.

roofline: issue-bound; algorithmic FLOPs per propagation step (frozen from
the oracle's operation census on this workload) x steps/s against the
non-tensor FP32 peak at the sampled clock.

--impl reference times the reference's own per-photon routine
(src/octmps_kernel.cuh relaunched as src/main.cu:572-623 does, compiled for
the host with OpenMP in oracle/_ref/) on all host cores: step k runs the
A-scans of the GPU arm's k-th launch with --ref-packets packets each, on the
mesh the reference's own MeshGraph builds (oracle/ref_mesh_cache.py), without
loading the product library.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "oct-mps_b200"))

METRIC = "photon packets/s (B-scan, 256 A-scans)"
B_STEP = 80  # algorithmic bytes per propagation step: 4 float4 planes + int4 neighbours
# Algorithmic FLOPs per propagation step on this workload, frozen from the
# oracle's operation census (oracle/census.cpp: + - x / sqrt count 1, a fused
# multiply-add 2, a transcendental 1; 1000 lanes x 2 packets at positions 0,
# 64, 128, 192 and 255 of the B-scan, 1.39e8 steps): mixed form 65.85 FP32 +
# 1.00 FP64, FP64 form 81.63.  tests/test_oracle.py re-counts a sample.
F_STEP = {0: 66.85, 1: 66.85, 2: 81.63}
F_STEP_FP64 = F_STEP[2]
N_SM = 148
# DRAM traffic of one launch, from an ncu capture (dram__bytes_read.sum + write) of 8 A-scans
# x 2e5 packets on the B-scan mesh: 65.1 MB = the mesh once (30.5 MB) + 4.33 MB per A-scan
# (its 88,800 RNG lanes, 3.2 MB, its tally and job state, write-backs).  The traffic does not
# grow with packets or steps (the mesh stays in L2), so a launch's is modelled as
# mesh + A-scans x per-A-scan bytes.
DRAM_PER_ASCAN = (65.1e6 - 30.5e6) / 8


def env_int(k, d):
    try:
        return int(os.environ.get(k, d))
    except ValueError:
        return d


def measured_hbm():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return d.get("hbm_gbs", 6650.0), "measured"
    return 6650.0, "fallback"


def fp_peak_tflops(clocks, bits):
    """Non-tensor FMA peak at the sampled SM clock: 148 SMs x 128 FP32 (or 64
    FP64) lanes x 2 FLOPs per cycle."""
    mhz = (clocks or {}).get("sm_mhz") or 1965.0
    return N_SM * (128 if bits == 32 else 64) * 2 * mhz * 1e6 / 1e12


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.t.join(2)
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None, "reasons": sorted(reasons),
                "samples": len(sm)}


def make_workload(args, workdir):
    import meshgen
    import octmps
    p = meshgen.config_bscan(workdir, n_ascans=args.ascans, n_photons=args.photons)
    sim = octmps.read_deck(p["opt"], p["mci"])
    mesh = octmps.build_mesh(p["mesh"])
    xs = octmps.probe_positions(sim)[: args.ascans]
    roots = [mesh.find_root(x) for x in xs]
    return sim, mesh, xs, roots


def tally_bytes(nbins, precision):
    ps = 4 if precision == 1 else 8
    r16 = lambda n: (n + 15) // 16 * 16  # noqa: E731
    return 32 + 2 * r16((nbins + 1) * 8) + 6 * r16((nbins + 2) * ps) + 32


def rel_error_at_peak(t, n):
    """Per-bin relative standard error of Class I at its peak bin and the mean
    over bins with >= 100 detections (src/octmps_io.cpp:310-318)."""
    import numpy as np
    s, q, c = t["sum1"][:-2], t["sumsq1"][:-2], t["count1"][:-1]
    m = s / n
    se = np.sqrt(np.maximum(q / n - m * m, 0) / (n - 1))
    k = int(np.argmax(m))
    ok = (c >= 100) & (m > 0)
    return (float(se[k] / m[k]) if m[k] > 0 else None,
            float(np.mean(se[ok] / m[ok])) if ok.any() else None)


def workload_config(args, n_xs, batch, n_tets=380928):
    return {
        "workload": f"bscan ellipsoid+2 spheres, {n_tets} tets, {n_xs} A-scans x "
                    f"{args.photons} packets, seeds 1..{n_xs}; one step = {batch} A-scans "
                    f"in one launch",
        "ascans_per_step": batch,
        "precision": {0: "mixed FP32 geometry / FP64 path+tally", 1: "FP32",
                      2: "FP64"}[args.precision],
        "parallelism": "weak (A-scan batches per rank)",
        "l2": "256 MB buffer written between timed steps",
    }


def run_ours(args, rank, world, local_rank, dist):
    import octmps
    import torch

    torch.cuda.set_device(local_rank)
    work = tempfile.mkdtemp(prefix="octmps_bench_")
    sim, mesh, xs, roots = make_workload(args, work)
    nb = sim.num_optical_depth_length_steps
    lanes = args.lanes or min(88800, args.photons)
    mult = octmps.safeprimes(3 + 3 * lanes)
    ctx = octmps.Context(local_rank, mult)
    flush_buf = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")  # > 126 MB L2
    batch = min(args.batch, len(xs))
    counter = [0]

    def run_batch(mid, sel, precision):
        """Submits the A-scans `sel`, runs them in one persistent launch and
        fetches every tally.  Returns device ms of the launch, wall ms,
        packets, propagation steps, tallies and stats.  Fails loudly if the
        batch did not run in exactly one launch (the device time is that
        launch's)."""
        t0 = time.perf_counter()
        own = mid is None
        if own:
            mid = ctx.upload_mesh(mesh)
        ids = [ctx.submit(mid, sim, xs[k], roots[k], n_photons=args.photons,
                          seed=rank * len(xs) + k + 1, n_lanes=lanes, precision=precision)
               for k in sel]
        ctx.flush()
        ts = [ctx.fetch(j, nb) for j in ids]
        ctx.synchronize()  # the launch's device time is known once it has ended
        sts = [ctx.stats(j) for j in ids]
        for j in ids:
            ctx.release(j)
        if own:
            ctx.release_mesh(mid)
        wall = (time.perf_counter() - t0) * 1e3
        launches = {s["launch_id"] for s in sts}
        if len(launches) != 1:
            raise RuntimeError(f"a bench step ran in {len(launches)} launches: {sorted(launches)}")
        return (sts[0]["device_ms"], wall, sum(s["packets"] for s in sts),
                sum(s["steps"] for s in sts), ts, sts)

    def one_step(mid):
        """The next batch of A-scans of the B-scan: step k runs positions
        k*batch .. k*batch+batch-1 (wrapping at the end of the scan)."""
        sel = step_positions(counter[0], batch, len(xs))
        counter[0] += 1
        return run_batch(mid, sel, args.precision)

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    mid = ctx.upload_mesh(mesh)
    if args.kernel_form is not None or args.blocks_per_sm or args.block_size:
        ctx.configure(kernel_form=args.kernel_form or 0, block_size=args.block_size,
                      blocks_per_sm=args.blocks_per_sm)
    tuned = None
    if args.autotune:
        tuned = autotune(ctx, mid, sim, xs, roots, args, lanes)
    for _ in range(args.warmup):
        one_step(mid)
    barrier()
    sampler = ClockSampler(local_rank)
    sampler.start()
    dev_ms, packets, steps = 0.0, 0, 0
    last, first_timed = None, counter[0]
    for _ in range(args.steps):
        flush_buf.fill_(1)  # evict L2 between timed steps
        torch.cuda.synchronize()
        d, w, p, s, ts, sts = one_step(mid)
        dev_ms += d
        packets += p
        steps += s
        last = (ts, sts)
    barrier()
    # end to end through the C-ABI: upload, submit, run, fetch, per step
    e2e_ms = 0.0
    # (the A-scans of the first timed steps again, so that e2e and value
    # cover the same propagation work)
    e2e_steps = max(1, min(args.steps, 2))
    e2e_packets = 0
    counter[0] = first_timed
    for _ in range(e2e_steps):
        flush_buf.fill_(1)
        torch.cuda.synchronize()
        _, w, p_e, _, _, _ = one_step(None)
        e2e_ms += w
        e2e_packets += p_e
    barrier()
    clocks = sampler.stop()

    # The plain single-job form: one A-scan per launch (submit, run, fetch,
    # next) on the first A-scans of the scan, each also uploading and
    # releasing the mesh end to end as the reference's per-A-scan worker does
    # (src/main.cu:447-465, 638-658).  Compared in propagation steps per
    # second (A-scans differ in steps per packet).  Untimed for the headline.
    plain = None
    if args.plain_ascans > 0:
        ctx.configure(linger_us=-1)
        p_ms, p_steps, p_packets, p_wall = 0.0, 0, 0, 0.0
        for k in range(min(args.plain_ascans, len(xs))):
            d, w, p, s, _, _ = run_batch(None, [k], args.precision)
            p_ms += d
            p_wall += w
            p_steps += s
            p_packets += p
        ctx.configure(linger_us=0)
        plain = {"ascans": min(args.plain_ascans, len(xs)),
                 "packets_per_s": p_packets / (p_ms / 1e3),
                 "propagation_steps_per_s": p_steps / (p_ms / 1e3),
                 "batched_over_plain": (steps / (dev_ms / 1e3)) / (p_steps / (p_ms / 1e3)),
                 "e2e_packets_per_s": p_packets / (p_wall / 1e3),
                 "note": "one A-scan per launch; device time, ratio of propagation steps/s; "
                         "e2e includes a mesh upload per A-scan as in the reference's worker"}

    # The FP64 form (the reference's arithmetic) beside the mixed form, on
    # the same A-scans of the first timed step, one launch each: the
    # speed-up without the precision change.
    fp64 = None
    if args.fp64_ascans > 0 and args.precision == 0:
        sel = step_positions(first_timed, batch, len(xs))[: args.fp64_ascans]
        d64, _, p64, s64, _, _ = run_batch(mid, sel, 2)
        dmx, _, pmx, smx, _, _ = run_batch(mid, sel, 0)
        fp64 = {"ascans": len(sel), "packets_per_s": p64 / (d64 / 1e3),
                "propagation_steps_per_s": s64 / (d64 / 1e3),
                "mixed_packets_per_s_same_ascans": pmx / (dmx / 1e3),
                "mixed_over_fp64": (smx / (dmx / 1e3)) / (s64 / (d64 / 1e3)),
                "f_step": F_STEP_FP64,
                "frac_of_fp64_peak": s64 / (d64 / 1e3) * F_STEP_FP64 /
                (fp_peak_tflops(clocks, 64) * 1e12)}

    # The 64 batched uneven jobs (each its own mesh of 46k-744k tets, 1.3e4-
    # 9.6e6 packets): one job table against one launch per job.
    uneven = None
    if args.uneven_jobs > 0 and world == 1:
        import batch_uneven
        t0 = time.perf_counter()
        ujobs = batch_uneven.build_jobs(args.uneven_jobs, os.path.join(work, "uneven"))
        uneven = batch_uneven.run(ctx, ujobs)
        uneven["host_mesh_build_s"] = time.perf_counter() - t0 - uneven["batched"]["wall_s"] - \
            uneven["plain"]["wall_s"]
        del ujobs

    t_dev = torch.tensor([dev_ms, e2e_ms / e2e_steps], dtype=torch.float64, device="cuda")
    if dist is not None:
        dist.all_reduce(t_dev, op=dist.ReduceOp.MAX)
    dev_ms_max, e2e_ms_step = float(t_dev[0]), float(t_dev[1])
    value = packets * world / (dev_ms_max / 1e3)
    e2e_value = (e2e_packets // e2e_steps) * world / (e2e_ms_step / 1e3)
    if plain is not None:
        plain["batched_e2e_over_plain_e2e"] = e2e_value / world / plain["e2e_packets_per_s"]
    ts, sts = last
    rel_peak, rel_mean = rel_error_at_peak(ts[len(ts) // 2], args.photons)
    launch_s = dev_ms / args.steps / 1e3
    steps_per_s = steps / args.steps / launch_s
    f_step = F_STEP[args.precision]
    peak32 = fp_peak_tflops(clocks, 64 if args.precision == 2 else 32)
    achieved = steps_per_s * f_step / 1e12
    hbm_peak, hbm_kind = measured_hbm()
    h2d = mesh.n_tets * 80 + batch * (lanes * 36 + 5 * 4 * sim.n_regions + 48)
    d2h = batch * (tally_bytes(nb, args.precision) + 32)
    ctx.release_mesh(mid)
    ctx.close()
    cfg = workload_config(args, len(xs), batch, mesh.n_tets)
    cfg["rng_lanes_per_ascan"] = lanes
    cfg["parallelism"] = f"weak x{world} (A-scan batches per rank)"
    return {
        "metric": METRIC,
        "value": value,
        "unit": "packets/s",
        "n_gpus": world,
        "impl": "ours",
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": dev_ms_max / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": {0: "f32+f64", 1: "f32", 2: "f64"}[args.precision],
        "data": "synthetic",
        "config": cfg,
        "ascans_per_s": batch * world * args.steps / (dev_ms_max / 1e3),
        "steps_per_packet": steps / packets,
        "propagation_steps_per_s": steps * world / (dev_ms_max / 1e3),
        "class1_rel_error": {"at_peak": rel_peak, "mean_bins_ge_100_counts": rel_mean,
                             "ascan": "middle A-scan, last timed step"},
        "e2e": {"value": e2e_value, "unit": "packets/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h, "ms_per_step": e2e_ms_step},
        "gpu_launches": args.steps,
        "roofline": {
            "bound": "issue", "achieved": achieved, "peak": peak32, "unit": "TFLOP/s",
            "frac": achieved / peak32,
            "traffic": mesh.n_tets * 80 + batch * DRAM_PER_ASCAN,
            "f_step": f_step,
            "note": f"algorithmic FLOPs per propagation step (F_step, the oracle's operation "
                    f"census on this workload: + - x / sqrt 1, FMA 2, transcendental 1) x "
                    f"steps/s of the photon kernel (CUDA events on its stream); peak = "
                    f"{'FP64' if args.precision == 2 else 'FP32'} lanes of 148 SMs x 2 x the "
                    f"median SM clock sampled while timing (no measured non-tensor peak is "
                    f"provided); the kernel is bound by issue latency and divergence, not "
                    f"by FLOPs",
            "traffic_note": "DRAM bytes per launch, modelled from an ncu capture of 8 A-scans "
                            "x 2e5 packets (mesh once + per-A-scan state); the mesh is "
                            "L2-resident",
            "secondary_hbm": {"achieved_gbs": steps_per_s * B_STEP / 1e9, "peak_gbs": hbm_peak,
                              "frac": steps_per_s * B_STEP / 1e9 / hbm_peak,
                              "note": f"nominal: {B_STEP} B of planes and neighbours per step "
                                      f"against the {hbm_kind} HBM copy bandwidth; served "
                                      f"from L2"},
        },
        "clocks": clocks,
        "plain_single_job": plain,
        "uneven_jobs": uneven,
        "fp64": fp64,
        "autotune": tuned,
        "first_timed_position": first_timed * batch % len(xs),
    }


def run_serving(args):
    """--serve: the served request stream (four resident meshes of 50k, 381k,
    994k and 2.0M tets; Poisson arrivals of A-scan requests of 1e5-1e7
    packets and 32-128-A-scan B-scan requests of 1e5 packets each at 3:1),
    capacity measured on a Poisson stream, then offered loads of 0.5, 0.9 and
    1.2 x capacity with --serve-requests requests each."""
    import serve
    work = tempfile.mkdtemp(prefix="octmps_serve_")
    meshes = serve.build_meshes("full", work)
    import octmps
    max_lanes = 1 << 18
    ctx = octmps.Context(0, octmps.safeprimes(3 + 3 * max_lanes))
    for m in meshes.values():
        m["id"] = ctx.upload_mesh(m["mesh"])
    sampler = ClockSampler(0)
    sampler.start()
    res = serve.serve_levels(ctx, meshes, [0.5, 0.9, 1.2], args.serve_requests, 1.0, max_lanes,
                             log=lambda d: print(json.dumps(d), file=sys.stderr, flush=True))
    clocks = sampler.stop()
    ctx.close()
    top = res["levels"][-1]
    return {
        "metric": "served stream: packets/s and p50/p99 latency per request type",
        "value": top["throughput_packets_per_s"], "unit": "packets/s", "n_gpus": 1,
        "impl": "ours", "higher_is_better": True, "dtype": "f32+f64", "data": "synthetic",
        "config": {"workload": "served stream, meshes " + ", ".join(
            f"{k} {m['n_tets']} tets" for k, m in meshes.items()) +
            f"; {args.serve_requests} requests per load level", "loads": [0.5, 0.9, 1.2]},
        "serving": res, "clocks": clocks,
        "note": "value = throughput at offered load 1.2 x capacity",
    }


def reference_inputs(args):
    """The workload as the reference itself reads it, without the product
    library: the deck files (meshgen writes input files only), parsed by the
    reference's read_simulation_data + Bias_Read; the mesh serialised by the
    reference's own MeshGraph + SerializeGraph and the roots found by its
    FindRootofGraph (cached by oracle/ref_mesh_cache.py: the O(T^2) builder
    takes about an hour at 380,928 tets); the multiplier file written by the
    oracle's generator and read by the reference's init_RNG."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle_py
    import ref_mesh_cache
    ref = oracle_py.Reference(oracle_py.REF_FAST_SO)
    work = tempfile.mkdtemp(prefix="octmps_ref_")
    p = ref_mesh_cache.bscan_deck(work, n_photons=args.photons)
    rs = ref.parse(p["opt"], p["mci"])
    cache = ref_mesh_cache.load(p["mesh"])
    mesh = {"tet": cache["tet"], "planes": cache["planes"]}
    xs = [float(x) for x in cache["xs"]][: args.ascans]
    sp = os.path.join(work, "safeprimes_base32.txt")
    n_blocks = REF_BLOCKS
    lanes = n_blocks * ref.threads_per_block
    oracle_py.Oracle().write_safeprimes(sp, 3 + 3 * lanes)
    return ref, rs, mesh, xs, [int(r) for r in cache["roots"]], sp, n_blocks, lanes


REF_BLOCKS = 2  # reference grid of the CPU runs: 2 blocks x 600 threads = 1,200 lanes


def step_positions(k, batch, n):
    """A-scan positions of bench step k (warm-up steps included): the batch
    that the GPU arm runs in its k-th launch."""
    return [(k * batch + j) % n for j in range(batch)]


def reference_step(inp, positions, packets, n_threads):
    """The reference's own per-photon routine (OCTMPSKernel relaunched until
    its photon counter runs out, src/main.cu:572-623) over the given A-scans,
    `packets` each, seeds position + 1; returns (packets, seconds of the
    relaunch loops)."""
    ref, rs, mesh, xs, roots, sp, n_blocks, lanes = inp
    rs.number_of_photons = packets
    secs = 0.0
    for k in positions:
        rng = ref.init_rng(lanes, sp, k + 1)
        t = ref.run(rs, mesh, roots[k], (xs[k], 0.0, 0.0), n_blocks, rng, n_threads=n_threads)
        secs += t["seconds"]
    return packets * len(positions), secs


def autotune(ctx, mid, sim, xs, roots, args, lanes):
    """Launch variant (kernel form, block size, blocks per SM, scatter share)
    chosen on 4 A-scans of the first position, at the workload's own lane
    count (the lane count decides which random numbers a packet draws)."""
    best, table = ctx.autotune(mid, sim, xs[0], roots[0], precision=args.precision,
                               n_photons=args.photons, n_jobs=4, n_lanes=lanes)
    return {"kernel_form": best[0], "block_size": best[1], "blocks_per_sm": best[2],
            "scatter_share": best[3],
            "table_steps_per_s": [[f, bs, b, sh, round(v)] for f, bs, b, sh, _, v in table]}


def run_reference(args, rank, world):
    """--impl reference: the reference's CPU routine on the host cores, step k
    running the same A-scan positions as the GPU arm's k-th launch, with a
    bounded number of packets per A-scan."""
    if rank != 0:
        return None
    try:
        inp = reference_inputs(args)
    except (ImportError, FileNotFoundError, ValueError) as e:
        return {"impl": "reference", "unavailable": f"reference host build or mesh cache "
                                                    f"missing: {e}"}
    threads = os.cpu_count()
    lanes = inp[7]
    n_xs = len(inp[3])
    batch = min(args.batch, n_xs)
    for k in range(args.warmup):
        reference_step(inp, step_positions(k, batch, n_xs)[:1], lanes, threads)
    packets, secs = 0, 0.0
    for k in range(args.warmup, args.warmup + args.steps):
        p, t = reference_step(inp, step_positions(k, batch, n_xs), args.ref_packets, threads)
        packets += p
        secs += t
    value = packets / secs
    sample = (f"{args.ref_packets} packets of each of the {batch} A-scans of each timed GPU step "
              f"(positions {args.warmup * batch % n_xs}..), {lanes} lanes, seeds position+1")
    return {
        "impl": "reference",
        "metric": METRIC,
        "value": value,
        "unit": "packets/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": secs / args.steps * 1e3,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic",
        "config": workload_config(args, n_xs, batch),
        "cpu_baseline": {"value": value, "unit": "packets/s", "cores": threads,
                         "kind": "reference", "sample": sample,
                         "build": "reference sources, g++ -O3 -march=x86-64-v4 -fopenmp"},
        "e2e": {"value": value, "unit": "packets/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--ascans", type=int, default=256, help="A-scans in the scan")
    ap.add_argument("--batch", type=int, default=32, help="A-scans per step (one launch)")
    ap.add_argument("--photons", type=int, default=1_000_000)
    ap.add_argument("--precision", type=int, default=0)
    ap.add_argument("--lanes", type=int, default=0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-autotune", dest="autotune", action="store_false",
                    help="skip choosing the launch variant on a sample before timing")
    ap.add_argument("--plain-ascans", type=int, default=4,
                    help="A-scans run one per launch for the batched-over-plain ratio")
    ap.add_argument("--ref-gpu-ascans", type=int, default=2,
                    help="A-scans the reference's own CUDA build runs (0: skip)")
    ap.add_argument("--uneven-jobs", type=int, default=64,
                    help="batched uneven jobs, one table vs one launch per job (0: skip)")
    ap.add_argument("--fp64-ascans", type=int, default=8,
                    help="A-scans of the first timed step rerun in the FP64 form")
    ap.add_argument("--cpu-ascans", type=int, default=8,
                    help="A-scans of the ours-arm cpu_baseline sample")
    ap.add_argument("--cpu-packets", type=int, default=4800,
                    help="packets per A-scan of the ours-arm cpu_baseline sample")
    ap.add_argument("--serve", action="store_true",
                    help="run the served-stream study instead of the B-scan bench")
    ap.add_argument("--serve-requests", type=int, default=200,
                    help="requests per offered-load level of --serve")
    ap.add_argument("--kernel-form", type=int, default=None,
                    help="0 per-lane, 1 pooled (default: the library's, or --autotune's)")
    ap.add_argument("--blocks-per-sm", type=int, default=0)
    ap.add_argument("--block-size", type=int, default=0,
                    help="threads per block (per-lane 256, 128 or 512; 0 = default)")
    ap.add_argument("--ref-packets", type=int, default=2400,
                    help="packets per A-scan of each --impl reference step")
    args = ap.parse_args()
    rank, world = env_int("RANK", 0), env_int("WORLD_SIZE", 1)
    local_rank = env_int("LOCAL_RANK", 0)

    if args.serve:
        print(json.dumps(run_serving(args)), flush=True)
        return

    if args.impl == "reference":
        out = run_reference(args, rank, world)
        if out is not None:
            print(json.dumps(out), flush=True)
        return

    dist = None
    if world > 1:
        import datetime
        import torch
        import torch.distributed as td
        torch.cuda.set_device(local_rank)
        td.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                              device_id=torch.device("cuda", local_rank))
        dist = td
    out = run_ours(args, rank, world, local_rank, dist)
    if rank == 0 and world == 1 and args.ref_gpu_ascans > 0:
        # the reference's own CUDA program on the same GPU, on the first
        # A-scans of the first timed step (baseline/run_ref_gpu.py)
        sys.path.insert(0, os.path.join(ROOT, "baseline"))
        try:
            import run_ref_gpu
            out["reference_gpu"] = run_ref_gpu.run(first=out["first_timed_position"],
                                                   ascans=args.ref_gpu_ascans,
                                                   photons=args.photons, timeout_s=600)
        except Exception as e:  # the baseline never hides the GPU result
            out["reference_gpu"] = {"unavailable": f"{type(e).__name__}: {e}"}
        rg = out["reference_gpu"]
        if rg.get("value"):
            rg["ours_over_reference"] = out["value"] / rg["value"]
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        # the reference's routine on the host cores, on the A-scans of the
        # first timed step (a bounded sample, about 10 s)
        try:
            inp = reference_inputs(args)
            n_xs = len(inp[3])
            batch = min(args.batch, n_xs)
            sel = step_positions(args.warmup, batch, n_xs)[: args.cpu_ascans]
            threads = os.cpu_count()
            p, secs = reference_step(inp, sel, args.cpu_packets, threads)
            out["cpu_baseline"] = {
                "value": p / secs, "unit": "packets/s", "cores": threads, "kind": "reference",
                "sample": f"{args.cpu_packets} packets of each of {len(sel)} A-scans of the first "
                          f"timed step (positions {sel[0]}..{sel[-1]}), {inp[7]} lanes, "
                          f"reference routine built -O3 -march=x86-64-v4 -fopenmp, mesh from the "
                          f"reference's own MeshGraph"}
        except Exception as e:  # the baseline never hides the GPU result
            out["cpu_baseline"] = {"value": None, "unit": "packets/s", "cores": os.cpu_count(),
                                   "kind": "reference", "sample": f"unavailable: {e}"}
    if rank == 0:
        print(json.dumps(out), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
