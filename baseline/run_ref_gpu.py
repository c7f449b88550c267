"""Runs the reference's own CUDA program (built by baseline/Makefile) on
A-scans of the B-scan workload and reports its photon throughput.

TEST AND MEASUREMENT INFRASTRUCTURE ONLY: the bench's ours-arm calls it to
put the reference's GPU figure beside its own; the product never does.

The deck is the benchmark's (meshgen writes the input files; no product
library is loaded), restricted to the requested A-scan positions by the
.opt file's probe range, and run as the reference's main() runs a B-scan:
one RunGPUi per A-scan, 148 blocks x 600 threads, photons re-seeded
identically per A-scan from -S (src/main.cu:948-1051).  The mesh comes
from the reference's own MeshGraph output (oracle/ref_mesh_cache.py).
Reported: packets / (sum of the per-A-scan kernel-loop times by cudaEvents)
and the reference's own wall-clock ">>>>>>Simulation time" for comparison.

    python baseline/run_ref_gpu.py [--first 96] [--ascans 4] [--photons 1000000]
"""
import argparse
import json
import os
import re
import subprocess
import sys
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
BINARY = os.path.join(HERE, "_ref", "octmps_ref")
SAFEPRIMES = os.path.join(HERE, "_ref", "safeprimes_base32.txt")
LANES = 148 * 600  # the reference's grid on a 148-SM B200 (src/main.cu:980-990)


def write_mesh_cache_bin(cache, path):
    """The binary layout baseline/mesh_cached.cpp reads."""
    with open(path, "wb") as f:
        np.array([len(cache["tet"]), len(cache["planes"]), len(cache["xs"])],
                 np.int32).tofile(f)
        np.ascontiguousarray(cache["tet"], np.int32).tofile(f)
        np.ascontiguousarray(cache["planes"], np.float64).tofile(f)
        np.ascontiguousarray(cache["xs"], np.float64).tofile(f)
        np.ascontiguousarray(cache["roots"], np.int32).tofile(f)


def ensure_safeprimes():
    """safeprimes_base32.txt for the reference's 88,800 lanes, from the
    oracle's generator (written once next to the binary)."""
    need = 3 + 3 * LANES
    if os.path.exists(SAFEPRIMES):
        with open(SAFEPRIMES) as f:
            if sum(1 for _ in f) >= need:
                return
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle_py
    oracle_py.Oracle().write_safeprimes(SAFEPRIMES, need)


def run(first=96, ascans=4, photons=1_000_000, seed=1, timeout_s=900):
    if not os.path.exists(BINARY):
        return {"unavailable": f"{BINARY} not built (baseline/Makefile needs the reference tree)"}
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import ref_mesh_cache
    work = tempfile.mkdtemp(prefix="octmps_refgpu_")
    p = ref_mesh_cache.bscan_deck(work, n_photons=photons)
    try:
        cache = ref_mesh_cache.load(p["mesh"])
    except (FileNotFoundError, ValueError) as e:
        return {"unavailable": f"reference mesh cache: {e}"}
    xs = [float(x) for x in cache["xs"]]
    sel = xs[first:first + ascans]
    # the .opt probe line: start, step, end covering exactly the selected positions
    with open(p["opt"]) as f:
        lines = f.read().split("\n")
    start, step = sel[0], 0.001  # the B-scan's A-scan spacing (meshgen.config_bscan)
    probe_idx = [i for i, ln in enumerate(lines) if ln.strip() and not ln.lstrip().startswith("#")
                 and len(ln.split()) == 3][-1]
    lines[probe_idx] = f"{start!r} {step!r} {start + step * (len(sel) - 0.5)!r}"
    with open(p["opt"], "w") as f:
        f.write("\n".join(lines))
    cache_bin = os.path.join(work, "mesh_cache.bin")
    write_mesh_cache_bin(cache, cache_bin)
    ensure_safeprimes()
    os.symlink(SAFEPRIMES, os.path.join(work, "safeprimes_base32.txt"))
    env = dict(os.environ, OCTMPS_REF_MESH_CACHE=cache_bin)
    t0 = time.time()
    r = subprocess.run(["timeout", "-k", "30", str(timeout_s), "stdbuf", "-oL", BINARY,
                        f"-S{seed}", p["opt"], p["mesh"], p["mci"]],
                       cwd=work, env=env, capture_output=True, text=True)
    wall = time.time() - t0
    loops = [(float(m.group(1)), int(m.group(2))) for m in
             re.finditer(r"kernel loop: ([0-9.]+) ms, (\d+) launches", r.stdout)]
    sims = [float(m.group(1)) for m in re.finditer(r">>>>>>Simulation time: ([0-9.]+)", r.stdout)]
    if r.returncode != 0 or len(loops) != len(sel):
        return {"unavailable": f"reference run failed (rc {r.returncode}, {len(loops)} of "
                               f"{len(sel)} A-scans): stderr: {r.stderr[-400:]!r} stdout: "
                               f"{r.stdout[-200:]!r}"}
    loop_ms = sum(ms for ms, _ in loops)
    return {
        "value": photons * len(sel) / (loop_ms / 1e3), "unit": "packets/s",
        "ascans": len(sel), "positions": [first, first + len(sel) - 1],
        "packets_per_ascan": photons, "kernel_loop_ms": [ms for ms, _ in loops],
        "launches": [n for _, n in loops],
        "wall_timer_packets_per_s": photons * len(sel) / (sum(sims) / 1e3) if sims else None,
        "process_s": wall, "lanes": LANES, "seed": seed,
        "build": "reference sources, nvcc --use_fast_math -O3 -maxrregcount=96 sm_100a; "
                 "patches: event timing around the relaunch loop, relaunch cap; mesh from the "
                 "reference's MeshGraph (cached)",
        "timing": "cudaEvents around RunGPUi's relaunch loop of OCTMPSKernel, summed over the "
                  "A-scans; value = packets / that time (FP64, the reference's arithmetic)",
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--first", type=int, default=96)
    ap.add_argument("--ascans", type=int, default=4)
    ap.add_argument("--photons", type=int, default=1_000_000)
    ap.add_argument("--timeout", type=int, default=900)
    a = ap.parse_args()
    print(json.dumps(run(a.first, a.ascans, a.photons, timeout_s=a.timeout)))


if __name__ == "__main__":
    main()
