"""Generates the per-bin reference tallies the workload-parity GPU tests
compare with, by running the reference's own per-photon routine
(src/octmps_kernel.cuh, relaunched as src/main.cu:572-623 does) compiled for
the host (oracle/_ref/libocref.so, built by oracle/Makefile from the
reference tree):

  bscan_ref_tallies.npz   the B-scan workload (380,928 tets) at A-scan
                          positions 64 and 192, 2e5 packets each, on the mesh
                          the reference's own MeshGraph builds
                          (oracle/ref_mesh_cache.py)
  layers_ref_tallies.npz  the four-layer slab (993,600 tets, 1499 depth
                          bins) at its middle position, 1e6 packets, on the
                          product builder's mesh (the reference's O(T^2)
                          builder would take about 8 hours at this size; the
                          product builder is byte-identical to it on the
                          reference's meshes and on the B-scan mesh)

Seeds and lane counts are recorded in the files.  Run where the reference
tree has been built (OCTMPS_REFERENCE=<tree> python __graft_entry__.py):

    python tests/golden/make_parity_golden.py [--part bscan|layers|all]
"""
import argparse
import os
import sys
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "oct-mps_b200"))

import oracle_py  # noqa: E402

KEYS = ("sum1", "sumsq1", "sum2", "sumsq2", "count1", "count2")
BSCAN_POSITIONS = (64, 192)
BSCAN_PACKETS = 200_000
LAYERS_PACKETS = 1_000_000


def run_ref(ref, rs, mesh, root, x, packets, n_blocks, seed, sp):
    rs.number_of_photons = packets
    rng = ref.init_rng(n_blocks * ref.threads_per_block, sp, seed)
    t0 = time.time()
    t = ref.run(rs, mesh, root, (x, 0.0, 0.0), n_blocks, rng)
    print(f"  x={x:.6f} {packets} packets in {time.time() - t0:.0f} s, "
          f"{t['num_filtered']} detections", flush=True)
    return t


def bscan(ref, work):
    import ref_mesh_cache
    p = ref_mesh_cache.bscan_deck(os.path.join(work, "bscan"))
    rs = ref.parse(p["opt"], p["mci"])
    cache = ref_mesh_cache.load(p["mesh"])
    mesh = {"tet": cache["tet"], "planes": cache["planes"]}
    n_blocks = 2
    sp = os.path.join(work, "safeprimes_bscan.txt")
    oracle_py.Oracle().write_safeprimes(sp, 3 + 3 * n_blocks * ref.threads_per_block)
    out = {}
    for k in BSCAN_POSITIONS:
        x = float(cache["xs"][k])
        seed = 5000 + k
        t = run_ref(ref, rs, mesh, int(cache["roots"][k]), x, BSCAN_PACKETS, n_blocks, seed, sp)
        for key in KEYS:
            out[f"p{k}_{key}"] = t[key]
        out[f"p{k}_packets"] = BSCAN_PACKETS
        out[f"p{k}_x"] = x
        out[f"p{k}_seed"] = seed
    out["lanes"] = n_blocks * ref.threads_per_block
    np.savez_compressed(os.path.join(HERE, "bscan_ref_tallies.npz"), **out)


def layers(ref, work):
    import meshgen
    import octmps
    p = meshgen.config_layers(os.path.join(work, "layers"))
    rs = ref.parse(p["opt"], p["mci"])
    m = octmps.build_mesh(p["mesh"])
    xs = octmps.probe_positions(octmps.read_deck(p["opt"], p["mci"]))
    x = xs[len(xs) // 2]
    n_blocks = 4
    sp = os.path.join(work, "safeprimes_layers.txt")
    oracle_py.Oracle().write_safeprimes(sp, 3 + 3 * n_blocks * ref.threads_per_block)
    seed = 7001
    t = run_ref(ref, rs, m, m.find_root(x), x, LAYERS_PACKETS, n_blocks, seed, sp)
    out = {key: t[key] for key in KEYS}
    out.update(packets=LAYERS_PACKETS, x=x, seed=seed, lanes=n_blocks * ref.threads_per_block)
    np.savez_compressed(os.path.join(HERE, "layers_ref_tallies.npz"), **out)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--part", default="all", choices=["bscan", "layers", "all"])
    args = ap.parse_args()
    ref = oracle_py.Reference()
    work = tempfile.mkdtemp(prefix="parity_golden_")
    if args.part in ("bscan", "all"):
        bscan(ref, work)
    if args.part in ("layers", "all"):
        layers(ref, work)


if __name__ == "__main__":
    main()
