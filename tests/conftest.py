import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")


def _reference_tree():
    """Root of the reference's tree: OCTMPS_REFERENCE, else the tree the host
    build in oracle/_ref/ was compiled from (absent on machines without it)."""
    tree = os.environ.get("OCTMPS_REFERENCE", "")
    if not tree:
        rec = os.path.join(ROOT, "oracle", "_ref", "REF_TREE")
        if os.path.exists(rec):
            tree = open(rec).read().strip()
    return tree


REF_INPUT = os.path.join(_reference_tree(), "input") if _reference_tree() else ""
sys.path.insert(0, os.path.join(ROOT, "oct-mps_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an sm_100 GPU (run with -m gpu)")


@pytest.fixture(scope="session")
def octmps():
    import octmps as m
    return m


@pytest.fixture(scope="session")
def meshgen():
    import meshgen as m
    return m


@pytest.fixture(scope="session")
def oracle():
    import oracle_py
    return oracle_py.Oracle()


@pytest.fixture(scope="session")
def reference():
    import oracle_py
    try:
        return oracle_py.Reference()
    except ImportError as e:
        pytest.skip(f"reference host build unavailable: {e}")


@pytest.fixture(scope="session")
def workdir(tmp_path_factory):
    return str(tmp_path_factory.mktemp("octmps"))


@pytest.fixture(scope="session")
def multipliers(octmps):
    """The generated multiplier table (the reference's safe-prime list is not shipped)."""
    return octmps.safeprimes(3 + 3 * 88800)  # enough for the default 88,800 lanes


@pytest.fixture(scope="session")
def small_deck(octmps, meshgen, workdir):
    p = meshgen.config_small(os.path.join(workdir, "small"), n_photons=20000)
    sim = octmps.read_deck(p["opt"], p["mci"])
    mesh = octmps.build_mesh(p["mesh"])
    root = mesh.find_root(sim.start_x)
    return {"paths": p, "sim": sim, "mesh": mesh, "root": root}


@pytest.fixture(scope="session")
def small_matched_deck(octmps, meshgen, workdir):
    p = meshgen.config_small(os.path.join(workdir, "small_matched"), n_photons=20000, matched=True)
    sim = octmps.read_deck(p["opt"], p["mci"])
    mesh = octmps.build_mesh(p["mesh"])
    root = mesh.find_root(sim.start_x)
    return {"paths": p, "sim": sim, "mesh": mesh, "root": root}


def ref_deck_paths(name):
    import json
    decks = json.load(open(os.path.join(GOLDEN, "decks.json")))
    files = decks[name]["files"]
    paths = [os.path.join(REF_INPUT, f) for f in files]
    if not REF_INPUT or not all(os.path.exists(p) for p in paths):
        pytest.skip("reference input decks not present")
    return paths


def three_sigma_ok(sum_a, sumsq_a, n_a, sum_b, sumsq_b, n_b, k=3.0, min_count=None, counts=None):
    """Per-bin agreement of two Monte Carlo means within k combined standard errors.

    Mean and standard error per bin as the reference's writer computes them
    (src/octmps_io.cpp:310-318): mean = Sum/N, var = (SumSq/N - mean^2)/(N-1).
    Returns (fraction of bins within k sigma, worst |z|)."""
    ma, mb = sum_a / n_a, sum_b / n_b
    va = np.maximum(sumsq_a / n_a - ma * ma, 0) / (n_a - 1)
    vb = np.maximum(sumsq_b / n_b - mb * mb, 0) / (n_b - 1)
    se = np.sqrt(va + vb)
    sel = se > 0
    if counts is not None and min_count is not None:
        sel &= counts >= min_count
    z = np.abs(ma - mb)[sel] / se[sel]
    if len(z) == 0:
        return 1.0, 0.0
    return float(np.mean(z <= k)), float(np.max(z))


@pytest.fixture(scope="session")
def plain_2m_deck(octmps, meshgen, workdir):
    """The plain A-scan geometry on a 70 x 70 x 68 grid (1,999,200 tets)."""
    p = meshgen.config_plain_ascan(os.path.join(workdir, "plain2m"), nx=70, ny=70, nz=68)
    sim = octmps.read_deck(p["opt"], p["mci"])
    mesh = octmps.build_mesh(p["mesh"])
    return {"paths": p, "sim": sim, "mesh": mesh}


# A packet that makes no progress: on plain_2m_deck, probe x below, seed
# 2074, RNG lane 5618's first packet ends on a diagonal face of the grid,
# on a vertical grid edge, moving parallel to the face (ux == uy); the
# grazing-incidence rule reflects it there with its direction unchanged, at
# distance 0, again and again.  The stop rule ends it after 1000 such hits
# (step 6502).
STUCK_CASE = {"x": 0.0051907104324341955, "seed": 2074, "lane": 5618, "steps": 6502}


@pytest.fixture(scope="session")
def layers_deck(octmps, meshgen, workdir):
    """The four-layer slab with tilted interfaces (993,600 tets, 1499 bins)."""
    p = meshgen.config_layers(os.path.join(workdir, "layers"))
    sim = octmps.read_deck(p["opt"], p["mci"])
    mesh = octmps.build_mesh(p["mesh"])
    xs = octmps.probe_positions(sim)
    x = xs[len(xs) // 2]
    return {"paths": p, "sim": sim, "mesh": mesh, "x": x, "root": mesh.find_root(x)}


# A packet whose likelihood ratio turned NaN in the FP32 forms before cosines
# were clamped: on layers_deck, seed 102, RNG lane 36485, its packet 36 (the
# lane's 37th); its second biased scattering rotated the direction about the
# nearly vertical probe axis, off unit length by 0.24 %, and the cosine
# between the old and new directions came out as 1.0023.
NAN_CASE = {"seed": 102, "lane": 36485, "packets": 37}
