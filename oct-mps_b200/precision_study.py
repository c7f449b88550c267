"""Precision study: the three arithmetic forms of the kernel on one workload.

Runs the same A-scan (same seeds, same RNG lanes) in FP64, in the mixed form
(FP32 geometry and directions, FP64 path length, weights of the tally and
sums) and in FP32, and compares each form's mean Class I and Class II
reflectance per depth bin with the FP64 form's: the difference in units of
the combined standard error of the two means, and the relative difference
where the FP64 mean is resolved (relative standard error below 10 %).
Forms differ packet by packet (a last-bit difference flips a discrete
decision), so the comparison is statistical: a form is acceptable where its
per-bin differences are consistent with noise.

    python precision_study.py [--photons 10000000] [--seeds 2] [--config layers|bscan]
"""
import argparse
import json
import os
import tempfile
import time

import numpy as np

import octmps

FORMS = {2: "fp64", 0: "mixed", 1: "fp32"}


def run_form(ctx, mid, sim, x, root, nb, photons, seeds, precision, lanes):
    sums = {c: np.zeros(nb) for c in ("1", "2")}
    sq = {c: np.zeros(nb) for c in ("1", "2")}
    t0 = time.perf_counter()
    ms = 0.0
    for seed in seeds:
        j = ctx.submit(mid, sim, x, root, n_photons=photons, seed=seed, n_lanes=lanes,
                       precision=precision)
        ctx.flush()
        t = ctx.fetch(j, nb)
        ctx.synchronize()
        ms += ctx.stats(j)["device_ms"]
        ctx.release(j)
        for c in ("1", "2"):
            sums[c] += t["sum" + c][:nb]
            sq[c] += t["sumsq" + c][:nb]
    n = photons * len(seeds)
    out = {}
    for c in ("1", "2"):
        mean = sums[c] / n
        var = np.maximum(sq[c] / n - mean ** 2, 0.0) / n
        out[c] = (mean, np.sqrt(var))
    return out, ms, time.perf_counter() - t0


def compare(ref, other):
    res = {}
    for c in ("1", "2"):
        m0, s0 = ref[c]
        m1, s1 = other[c]
        se = np.sqrt(s0 ** 2 + s1 ** 2)
        ok = se > 0
        z = np.zeros_like(m0)
        z[ok] = (m1[ok] - m0[ok]) / se[ok]
        resolved = (m0 > 0) & (s0 < 0.1 * m0)
        rel = np.abs(m1[resolved] - m0[resolved]) / m0[resolved]
        res["class" + ("I" if c == "1" else "II")] = {
            "bins_compared": int(ok.sum()),
            "frac_within_3_sigma": float(np.mean(np.abs(z[ok]) <= 3.0)) if ok.any() else None,
            "max_abs_z": float(np.max(np.abs(z[ok]))) if ok.any() else None,
            "mean_z": float(np.mean(z[ok])) if ok.any() else None,
            "resolved_bins": int(resolved.sum()),
            "median_rel_diff_resolved": float(np.median(rel)) if rel.size else None,
            "median_rel_stderr_fp64_resolved":
                float(np.median(s0[resolved] / m0[resolved])) if rel.size else None,
        }
    return res


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--photons", type=int, default=10_000_000)
    ap.add_argument("--seeds", type=int, default=2)
    ap.add_argument("--lanes", type=int, default=88800)
    ap.add_argument("--config", default="layers", choices=["layers", "bscan"])
    ap.add_argument("--device", type=int, default=0)
    args = ap.parse_args()
    import meshgen
    work = tempfile.mkdtemp(prefix="octmps_prec_")
    if args.config == "layers":
        p = meshgen.config_layers(os.path.join(work, "layers"))
    else:
        p = meshgen.config_bscan(os.path.join(work, "bscan"))
    sim = octmps.read_deck(p["opt"], p["mci"])
    mesh = octmps.build_mesh(p["mesh"])
    xs = octmps.probe_positions(sim)
    x = xs[len(xs) // 2]
    root = mesh.find_root(x)
    nb = sim.num_optical_depth_length_steps
    seeds = list(range(101, 101 + args.seeds))
    mult = octmps.safeprimes(3 + 3 * args.lanes)
    with octmps.Context(args.device, mult) as ctx:
        mid = ctx.upload_mesh(mesh)
        res = {}
        timing = {}
        for prec in (2, 0, 1):
            res[prec], ms, wall = run_form(ctx, mid, sim, x, root, nb, args.photons, seeds, prec,
                                           args.lanes)
            timing[FORMS[prec]] = {"device_s": ms / 1e3,
                                   "packets_per_s": args.photons * len(seeds) / (ms / 1e3)}
        ctx.release_mesh(mid)
    print(json.dumps({
        "workload": f"{args.config}: {p['n_tets']} tets, {nb} depth bins, probe x = {x:.4f} cm, "
                    f"{args.seeds} seeds x {args.photons} packets per form",
        "timing": timing,
        "mixed_vs_fp64": compare(res[2], res[0]),
        "fp32_vs_fp64": compare(res[2], res[1]),
    }, indent=1))


if __name__ == "__main__":
    main()
