"""Generates the golden fixtures in this directory by running the reference.

The reference has no tests and no known-answer vectors of its own, so the
fixtures are produced by the reference's own code compiled for the host
(oracle/_ref/libocref.so, built by oracle/Makefile from the reference tree
in place): its init_RNG, read_simulation_data + Bias_Read, MeshGraph +
FindRootofGraph + SerializeGraph, the per-photon routine of OCTMPSKernel
and its output writers.  Run it where the reference tree exists:

    OCTMPS_REFERENCE=<reference tree> python tests/golden/make_golden.py [--ref-input DIR]

(--ref-input defaults to the input/ directory of that tree.)

The multiplier table comes from the project's generator (the reference's
safeprimes_base32.txt is not shipped); fixtures record which entries they
used.
"""
import argparse
import hashlib
import json
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oct-mps_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import meshgen  # noqa: E402
import octmps  # noqa: E402
import oracle_py  # noqa: E402

DECKS = {
    "Sphere": ("Sphere/Sphere.opt", "Sphere/Sphere.mesh", "Sphere/BiasStartup.mci"),
    "FourLayers": ("FourLayers/FourLayers.opt", "FourLayers/FourLayers.mesh",
                   "FourLayers/BiasStartup.mci"),
    "WangBump": ("WangBump/WangBump.opt", "WangBump/WangBump.mesh", "WangBump/BiasStartup.mci"),
    "Ellipsoidand2Spheres": ("Ellipsoidand2Spheres/ellipsoid_and_two_spheres_60_degree.opt",
                             "Ellipsoidand2Spheres/ellipsoid_and_two_spheres_60_degree.mesh",
                             "Ellipsoidand2Spheres/BiasStartup.mci"),
}
SIM_FIELDS = ["start_x", "step_x", "end_x", "number_of_photons", "n_regions", "type_simulation",
              "type_bias", "record_photons_flag", "num_optical_depth_length_steps",
              "backward_bias_coefficient", "target_depth_min", "target_depth_max",
              "coherence_length_source", "max_collecting_radius", "max_collecting_angle_deg",
              "probability_additional_bias", "max_relative_contribution",
              "max_filtered_optical_depth", "optical_depth_shift"]


def digest(*arrays):
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def sim_dict(rs):
    d = {k: getattr(rs, k) for k in SIM_FIELDS}
    d["regions"] = [[rs.region_n[i], rs.region_mua[i], rs.region_mus[i], rs.region_g[i]]
                    for i in range(1, rs.n_regions)]
    d["ambient_n"] = rs.region_n[0]
    # doubles as exact hex strings
    return {k: (v.hex() if isinstance(v, float) else v) for k, v in d.items()} | {
        "regions": [[x.hex() for x in r] for r in d["regions"]], "ambient_n": d["ambient_n"].hex()}


def main():
    ap = argparse.ArgumentParser()
    tree = os.environ.get("OCTMPS_REFERENCE", "")
    ap.add_argument("--ref-input", default=os.path.join(tree, "input") if tree else None,
                    required=not tree)
    args = ap.parse_args()
    R = oracle_py.Reference()
    work = tempfile.mkdtemp()
    sp = os.path.join(work, "safeprimes_base32.txt")
    n_mult = 3 + 3 * 4000
    octmps.write_safeprimes(sp, n_mult)
    mult = octmps.read_safeprimes(sp, n_mult)

    # 1. multiplier table head + init_RNG known answers
    lanes = 64
    kat = {"multipliers_head": mult[:3 + 3 * lanes]}
    for seed in (985456376, 1, 123456789):
        r = R.init_rng(lanes, sp, seed)
        for k, v in r.items():
            kat[f"seed{seed}_{k}"] = v
    np.savez_compressed(os.path.join(HERE, "rng_kat.npz"), **kat)

    # 2. parsers and 3. mesh builder, on the shipped decks
    decks = {}
    for name, (o, m, b) in DECKS.items():
        opt, mesh, mci = (os.path.join(args.ref_input, x) for x in (o, m, b))
        rs = R.parse(opt, mci)
        px = rs.start_x
        rm = R.build_mesh(mesh, (px, 0.0, 0.0))
        nd = int(np.max(rm["faces"])) + 1
        decks[name] = {
            "files": [o, m, b],
            "sim": sim_dict(rs),
            "n_tets": int(len(rm["region"])),
            "n_distinct_faces": nd,
            "root_at_start_x": int(rm["root"]),
            "sha256_region_faces_signs_adj": digest(rm["region"], rm["faces"], rm["signs"],
                                                    rm["adj"]),
            "sha256_planes": digest(rm["planes"][:nd]),
        }
        print(name, decks[name]["n_tets"], decks[name]["root_at_start_x"])
    with open(os.path.join(HERE, "decks.json"), "w") as f:
        json.dump(decks, f, indent=1)

    # 4. first-packet records of the reference routine (FP64) on Sphere
    o, m, b = (os.path.join(args.ref_input, x) for x in DECKS["Sphere"])
    rs = R.parse(o, b)
    sim = octmps.read_deck(o, b)
    mesh = octmps.build_mesh(m)
    root = mesh.find_root(rs.start_x)
    n_tr = 2000
    rng = R.init_rng(n_tr, sp, 985456376)
    rec = R.trace(rs, mesh, root, (rs.start_x, 0.0, 0.0), rng, n_tr)
    np.savez_compressed(os.path.join(HERE, "sphere_first_packets.npz"), records=rec,
                        probe_x=rs.start_x, root=root, seed=985456376)

    # 5. full A-scans of the reference routine on the small synthetic deck
    #    (mismatched refractive indices: exercises Fresnel reflection)
    deckdir = os.path.join(work, "small")
    small = meshgen.config_small(deckdir, n_photons=20000)
    rs = R.parse(small["opt"], small["mci"])
    mesh = octmps.build_mesh(small["mesh"])
    root = mesh.find_root(rs.start_x)
    out = {}
    for rep, seed in enumerate((985456376, 2, 3, 4)):
        n_blocks = 4  # 2400 lanes
        rng = R.init_rng(n_blocks * R.threads_per_block, sp, seed)
        t = R.run(rs, mesh, root, (rs.start_x, 0.0, 0.0), n_blocks, rng, n_threads=0)
        for k, v in t.items():
            if k not in ("seconds", "launches"):
                out[f"run{rep}_{k}"] = np.asarray(v)
    np.savez_compressed(os.path.join(HERE, "small_ref_tallies.npz"), **out)

    # 6. reference writers on run 0's tallies
    t0 = {k[5:]: out[k] for k in out if k.startswith("run0_")}
    cwd = os.getcwd()
    wdir = os.path.join(work, "writer")
    os.makedirs(wdir)
    os.chdir(wdir)
    try:
        R.write_result(rs, 0.0, t0)
        R.write_result(rs, 0.001, t0)  # appended second A-scan
    finally:
        os.chdir(cwd)
    files = {fn: open(os.path.join(wdir, fn), "rb").read().decode()
             for fn in sorted(os.listdir(wdir))}
    with open(os.path.join(HERE, "small_writer_output.json"), "w") as f:
        json.dump(files, f, indent=0)
    print("fixtures written to", HERE)


if __name__ == "__main__":
    main()
