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

--impl reference times the reference's own per-photon routine
(src/octmps_kernel.cuh, compiled for the host with OpenMP in
oracle/_ref/) on all host cores, on a bounded sample of the same workload
(one A-scan of the same mesh and parameters).
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

B_STEP = 80  # algorithmic bytes per propagation step: 4 float4 planes + int4 neighbours
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


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return d.get("hbm_gbs", 6650.0), "measured"
    return 6650.0, "fallback"


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


def run_ours(args, rank, world, local_rank, dist):
    import numpy as np
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

    def one_step(resident_mid):
        """Submits the next batch of A-scans of the B-scan (positions k*batch ..
        k*batch+batch-1, wrapping at the end of the scan), runs them in one
        persistent launch and fetches every tally.  Returns device ms of the
        launch, wall ms, packets, steps and the tallies."""
        first = (counter[0] * batch) % len(xs)
        counter[0] += 1
        sel = [(first + k) % len(xs) for k in range(batch)]
        t0 = time.perf_counter()
        mid = resident_mid if resident_mid is not None else ctx.upload_mesh(mesh)
        ids = [ctx.submit(mid, sim, xs[k], roots[k], n_photons=args.photons,
                          seed=rank * len(xs) + k + 1, n_lanes=lanes, precision=args.precision)
               for k in sel]
        ctx.flush()
        ts = [ctx.fetch(j, nb) for j in ids]
        ctx.synchronize()  # the launch's device time is known once it has ended
        sts = [ctx.stats(j) for j in ids]
        for j in ids:
            ctx.release(j)
        if resident_mid is None:
            ctx.release_mesh(mid)
        wall = (time.perf_counter() - t0) * 1e3
        dev = sts[0]["device_ms"]
        return dev, wall, sum(s["packets"] for s in sts), sum(s["steps"] for s in sts), ts, sts

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    mid = ctx.upload_mesh(mesh)
    tuned = None
    if args.autotune:
        # launch variant chosen on 4 A-scans' worth of packets at the first position
        best, table = ctx.autotune(mid, sim, xs[0], roots[0], precision=args.precision,
                                   n_photons=args.photons, n_jobs=4, n_lanes=lanes)
        tuned = {"blocks_per_sm": best[0], "scatter_share": best[1],
                 "table_steps_per_s": [[b, sh, round(v)] for b, sh, v in table]}
    for _ in range(args.warmup):
        one_step(mid)
    barrier()
    sampler = ClockSampler(local_rank)
    sampler.start()
    dev_ms, packets, steps = 0.0, 0, 0
    last = None
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
    for _ in range(max(1, min(args.steps, 2))):
        flush_buf.fill_(1)
        torch.cuda.synchronize()
        _, w, p_e, _, _, _ = one_step(None)
        e2e_ms += w
    e2e_steps = max(1, min(args.steps, 2))
    barrier()
    clocks = sampler.stop()

    # The same workload one A-scan per launch (submit, run, fetch, next), on
    # the first A-scans of the scan: the batched launches' gain over the
    # plain single-job use.  Compared in propagation steps per second (the
    # A-scans differ in steps per packet).  Untimed for the headline.
    ctx.configure(linger_us=-1)
    # End to end, each A-scan also uploads and releases the mesh, as the
    # reference's per-A-scan worker does (src/main.cu:447-465, 638-658).
    plain_ms, plain_steps, plain_packets, plain_wall = 0.0, 0, 0, 0.0
    for k in range(min(args.plain_ascans, len(xs))):
        t0 = time.perf_counter()
        mid_k = ctx.upload_mesh(mesh)
        j = ctx.submit(mid_k, sim, xs[k], roots[k], n_photons=args.photons,
                       seed=rank * len(xs) + k + 1, n_lanes=lanes, precision=args.precision)
        ctx.flush()
        ctx.fetch(j, nb)
        ctx.synchronize()
        s = ctx.stats(j)
        ctx.release(j)
        ctx.release_mesh(mid_k)
        plain_wall += time.perf_counter() - t0
        plain_ms += s["device_ms"]
        plain_steps += s["steps"]
        plain_packets += s["packets"]
    ctx.configure(linger_us=0)
    plain = None
    if plain_ms > 0:
        batched_sps = steps / (dev_ms / 1e3)
        plain_sps = plain_steps / (plain_ms / 1e3)
        plain = {"ascans": min(args.plain_ascans, len(xs)), "packets_per_s": plain_packets / (plain_ms / 1e3),
                 "propagation_steps_per_s": plain_sps, "batched_over_plain": batched_sps / plain_sps,
                 "e2e_packets_per_s": plain_packets / plain_wall,
                 "note": "one A-scan per launch; device time, ratio of propagation steps/s; e2e "
                         "includes a mesh upload per A-scan as in the reference's worker"}

    t_dev = torch.tensor([dev_ms, e2e_ms / e2e_steps], dtype=torch.float64, device="cuda")
    if dist is not None:
        dist.all_reduce(t_dev, op=dist.ReduceOp.MAX)
    dev_ms_max, e2e_ms_step = float(t_dev[0]), float(t_dev[1])
    total_packets = packets * world
    value = total_packets / (dev_ms_max / 1e3)
    ms_per_step = dev_ms_max / args.steps
    e2e_value = (packets // args.steps) * world / (e2e_ms_step / 1e3)
    if plain is not None:
        plain["batched_e2e_over_plain_e2e"] = e2e_value / world / plain["e2e_packets_per_s"]
    ts, sts = last
    rel_peak, rel_mean = rel_error_at_peak(ts[len(ts) // 2], args.photons)
    launch_s = dev_ms / args.steps / 1e3
    steps_per_launch = steps / args.steps
    achieved = steps_per_launch * B_STEP / launch_s / 1e9
    peak, peak_kind = measured_peaks()
    h2d = mesh.n_tets * 80 + batch * (lanes * 36 + 5 * 4 * sim.n_regions + 48)
    d2h = batch * (tally_bytes(nb, args.precision) + 32)
    ctx.release_mesh(mid)
    ctx.close()
    return {
        "metric": "photon packets/s (B-scan, 256 A-scans)",
        "value": value,
        "unit": "packets/s",
        "n_gpus": world,
        "impl": "ours",
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms_per_step,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": {0: "f32+f64", 1: "f32", 2: "f64"}[args.precision],
        "data": "synthetic",
        "config": {
            "workload": f"bscan ellipsoid+2 spheres, {mesh.n_tets} tets, {len(xs)} A-scans x "
                        f"{args.photons} packets, seeds 1..{len(xs)}; one step = {batch} "
                        f"A-scans in one launch",
            "ascans_per_step": batch,
            "precision": {0: "mixed FP32 geometry / FP64 path+tally", 1: "FP32",
                          2: "FP64"}[args.precision],
            "rng_lanes_per_ascan": lanes,
            "parallelism": f"weak x{world} (A-scan batches per rank)",
            "l2": "256 MB buffer written between timed steps",
        },
        "ascans_per_s": batch * world * args.steps / (dev_ms_max / 1e3),
        "steps_per_packet": steps / packets,
        "propagation_steps_per_s": steps * world / (dev_ms_max / 1e3),
        "class1_rel_error": {"at_peak": rel_peak, "mean_bins_ge_100_counts": rel_mean,
                             "ascan": "middle A-scan, last timed step"},
        "e2e": {"value": e2e_value, "unit": "packets/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h, "ms_per_step": e2e_ms_step},
        "gpu_launches": args.steps * 1,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak,
                     "traffic": mesh.n_tets * 80 + batch * DRAM_PER_ASCAN,
                     "traffic_note": "DRAM bytes per launch, modelled from an ncu capture of "
                                     "8 A-scans x 2e5 packets (mesh once + per-A-scan state); "
                                     "far below the algorithmic bytes because the mesh is "
                                     "L2-resident",
                     "note": f"algorithmic {B_STEP} B per propagation step x steps per launch / "
                             f"launch time; peak = {peak_kind} HBM copy bandwidth; the mesh "
                             f"({mesh.n_tets * 80 / 1e6:.0f} MB) is L2-resident, the kernel is "
                             f"bound by instruction issue and gather latency"},
        "clocks": clocks,
        "plain_single_job": plain,
        "autotune": tuned,
    }


def cpu_sample(args, packets_hint=None, n_threads=0, target_s=12.0):
    """The reference's own routine on the host: one A-scan of the workload."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import octmps
    import oracle_py
    ref = oracle_py.Reference()
    work = tempfile.mkdtemp(prefix="octmps_ref_")
    sim, mesh, xs, roots = make_workload(argparse.Namespace(ascans=1, photons=args.photons), work)
    import meshgen  # noqa: F401
    p = os.path.join(work, "bscan")
    rs = ref.parse(p + ".opt", p + ".mci")
    sp = os.path.join(work, "safeprimes_base32.txt")
    n_blocks = 8
    lanes = n_blocks * ref.threads_per_block
    octmps.write_safeprimes(sp, 3 + 3 * lanes)
    n_threads = n_threads or os.cpu_count()

    def run(n):
        rs.number_of_photons = n
        rng = ref.init_rng(lanes, sp, 1)
        t = ref.run(rs, mesh, roots[0], (xs[0], 0.0, 0.0), n_blocks, rng, n_threads=n_threads)
        return t["seconds"]

    n0 = max(lanes * 2, 10000)
    s0 = run(n0)
    rate0 = n0 / s0
    n = packets_hint or int(max(lanes, min(5e7, rate0 * target_s)))
    return run, n, n_threads, rate0, lanes


def run_reference(args, rank, world):
    if rank != 0:
        return None
    try:
        run, n, threads, rate0, lanes = cpu_sample(args, target_s=8.0)
    except ImportError as e:
        return {"impl": "reference", "unavailable": f"reference host build missing: {e}"}
    for _ in range(args.warmup):
        run(max(lanes, n // 8))
    times = [run(n) for _ in range(args.steps)]
    tot = sum(times)
    value = n * args.steps / tot
    return {
        "impl": "reference",
        "metric": "photon packets/s (B-scan, 256 A-scans)",
        "value": value,
        "unit": "packets/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": tot / args.steps * 1e3,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": "bscan ellipsoid+2 spheres, 380928 tets; sample: 1 A-scan per step",
                   "lanes": lanes},
        "cpu_baseline": {"value": value, "unit": "packets/s", "cores": threads,
                         "kind": "reference",
                         "sample": f"{n} packets of one A-scan per step, {lanes} lanes"},
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
    ap.add_argument("--autotune", action="store_true",
                    help="choose the launch variant on a sample before timing")
    ap.add_argument("--plain-ascans", type=int, default=4,
                    help="A-scans run one per launch for the batched-over-plain ratio")
    args = ap.parse_args()
    rank, world = env_int("RANK", 0), env_int("WORLD_SIZE", 1)
    local_rank = env_int("LOCAL_RANK", 0)

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
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            run, n, threads, rate0, lanes = cpu_sample(args, target_s=12.0)
            secs = run(n)
            out["cpu_baseline"] = {"value": n / secs, "unit": "packets/s", "cores": threads,
                                   "kind": "reference",
                                   "sample": f"{n} packets of one A-scan of the workload "
                                             f"({lanes} lanes), reference routine compiled for "
                                             f"the host with OpenMP"}
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
