"""Serialised B-scan mesh made by the reference's own mesh builder.

TEST INFRASTRUCTURE ONLY (the reference arm of bench.py and the parity
tests read it; the product never does).

The reference builds its mesh with MeshGraph, whose face matching
(CheckFaceExists, src/mesh.cpp:51-83) scans every face found so far: O(T^2)
in the tet count, about an hour at the 380,928 tets of the B-scan
workload.  Its result does not change between runs, so this script runs
MeshGraph + SerializeGraph + FindRootofGraph (src/mesh.cpp:86-359, through
oracle/_ref/libocref.so, compiled from the reference's sources) once, for
the B-scan deck that oct-mps_b200/meshgen.py writes, and stores:

  tet   (T, 14) int32   idx, region, faces[4], signs[4], adjTetras[4]
  planes (F, 4) float64 Nx, Ny, Nz, d of the F distinct faces
  roots (A,) int32      root tet of each A-scan position
  xs    (A,) float64    the A-scan positions, main()'s loop (src/main.cu:948-950)
  mesh_sha256           SHA-256 of the .mesh file it was built from

in oracle/_ref/bscan_ref_mesh.npz (git-ignored, like the rest of oracle/_ref/).

  python oracle/ref_mesh_cache.py [--out PATH]
"""
import argparse
import hashlib
import os
import sys
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CACHE = os.path.join(HERE, "_ref", "bscan_ref_mesh.npz")


def ascan_positions(start, step, end):
    """main()'s A-scan loop (src/main.cu:948-950), in the same double steps."""
    xs = []
    x = start
    while x < end:
        xs.append(x)
        x += step
    return xs


def sha256(path):
    h = hashlib.sha256()
    with open(path, "rb") as f:
        for chunk in iter(lambda: f.read(1 << 20), b""):
            h.update(chunk)
    return h.hexdigest()


def bscan_deck(out_dir, n_photons=1_000_000):
    """Writes the B-scan deck (256 A-scans) and returns its paths."""
    sys.path.insert(0, os.path.join(ROOT, "oct-mps_b200"))
    import meshgen  # writes the input files only; loads no library
    return meshgen.config_bscan(out_dir, n_ascans=256, n_photons=n_photons)


def load(mesh_path=None):
    """The cached arrays, checked against the .mesh file when one is given."""
    if not os.path.exists(CACHE):
        raise FileNotFoundError(f"{CACHE} missing; run python {os.path.relpath(__file__, ROOT)}")
    d = dict(np.load(CACHE))
    if mesh_path is not None and str(d["mesh_sha256"]) != sha256(mesh_path):
        raise ValueError(f"{CACHE} was built from a different .mesh file")
    return d


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=CACHE)
    args = ap.parse_args()
    sys.path.insert(0, HERE)
    import oracle_py
    ref = oracle_py.Reference()
    work = tempfile.mkdtemp(prefix="ref_mesh_")
    p = bscan_deck(work)
    sim = ref.parse(p["opt"], p["mci"])
    xs = ascan_positions(sim.start_x, sim.step_x, sim.end_x)
    t0 = time.time()
    m = ref.build_mesh_roots(p["mesh"], xs)
    print(f"MeshGraph + SerializeGraph + {len(xs)} roots: {time.time() - t0:.0f} s, "
          f"{len(m['tet'])} tets, {len(m['planes'])} faces", flush=True)
    if (m["roots"] < 0).any():
        raise SystemExit(f"no root for {int((m['roots'] < 0).sum())} probe positions")
    os.makedirs(os.path.dirname(args.out), exist_ok=True)
    np.savez_compressed(args.out, tet=m["tet"], planes=m["planes"], roots=m["roots"],
                        xs=np.asarray(xs), mesh_sha256=sha256(p["mesh"]))
    print(f"wrote {args.out}")


if __name__ == "__main__":
    main()
