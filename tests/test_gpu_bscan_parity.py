"""Parity on the benchmarked workload: the B-scan mesh (380,928 tets,
mismatched refractive indices, ~12,000-15,000 propagation steps per packet
under total internal reflection) and the four-layer precision slab
(993,600 tets, 1499 depth bins).

* Bit-exact: the first packets of 2,000 RNG lanes at the scan's first,
  middle and last probe positions, in the mixed and FP64 forms, against the
  CPU oracle (event sequence per step, generator states, counts, optical
  path, contribution; every tally count).
* Statistical: per-bin Class I/II means of the mixed form against the FP64
  form (both on the GPU, independent seeds) and against the reference's own
  routine (src/octmps_kernel.cuh:1329-1402, committed fixtures from
  tests/golden/make_parity_golden.py), with the per-bin standard error of
  src/octmps_io.cpp:310-318 and a Bonferroni bound over the bins compared.
"""
import math
import os

import numpy as np
import pytest

from conftest import GOLDEN

import oracle_py

from test_gpu_kernel import assert_records_equal, assert_tallies_equal, run_oracle

pytestmark = pytest.mark.gpu

REC_BYTES = oracle_py.PACKET_DTYPE.itemsize
FAMILY_ALPHA = 0.01  # family-wise false-alarm rate of a per-bin comparison
MIN_COUNT = 100      # bins compared: at least this many detections in both runs


@pytest.fixture(scope="module")
def torch_cuda():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.fail("a GPU test ran without a CUDA device")
    return torch


@pytest.fixture(scope="module")
def ctx(octmps, multipliers, torch_cuda):
    c = octmps.Context(0, multipliers)
    yield c
    c.close()


@pytest.fixture(scope="module")
def bscan_deck(octmps, meshgen, workdir):
    p = meshgen.config_bscan(os.path.join(workdir, "bscan"))
    sim = octmps.read_deck(p["opt"], p["mci"])
    mesh = octmps.build_mesh(p["mesh"])
    xs = octmps.probe_positions(sim)
    return {"paths": p, "sim": sim, "mesh": mesh, "xs": xs}


def bonferroni_z(m, alpha=FAMILY_ALPHA):
    """Two-sided |z| bound with family-wise error alpha over m comparisons:
    the z with 2 * (1 - Phi(z)) = alpha / m, by bisection on erfc."""
    target = alpha / max(m, 1)
    lo, hi = 0.0, 20.0
    for _ in range(200):
        mid = 0.5 * (lo + hi)
        if math.erfc(mid / math.sqrt(2.0)) > target:
            lo = mid
        else:
            hi = mid
    return hi


def per_bin_z(a, n_a, b, n_b, nbins, c):
    """z of the per-bin mean difference of class c between two tallies, over
    the bins where both have at least MIN_COUNT detections."""
    ma, mb = a["sum" + c][:nbins] / n_a, b["sum" + c][:nbins] / n_b
    va = np.maximum(a["sumsq" + c][:nbins] / n_a - ma * ma, 0) / (n_a - 1)
    vb = np.maximum(b["sumsq" + c][:nbins] / n_b - mb * mb, 0) / (n_b - 1)
    sel = (a["count" + c][:nbins] >= MIN_COUNT) & (b["count" + c][:nbins] >= MIN_COUNT)
    sel &= (va + vb) > 0
    return (ma - mb)[sel] / np.sqrt(va + vb)[sel]


def run_job(ctx, deck, x, n, lanes, seed, precision, record=None):
    mesh, sim = deck["mesh"], deck["sim"]
    mid = ctx.upload_mesh(mesh)
    j = ctx.submit(mid, sim, x, mesh.find_root(x), n_photons=n, seed=seed, n_lanes=lanes,
                   precision=precision)
    if record is not None:
        ctx.record_next_launch(record.data_ptr())
    ctx.flush()
    t = ctx.fetch(j, sim.num_optical_depth_length_steps)
    st = ctx.stats(j)
    ctx.release(j)
    ctx.release_mesh(mid)
    return t, st


@pytest.mark.parametrize("precision", [0, 2])
@pytest.mark.parametrize("position", [0, 128, 255])
def test_bscan_first_packets_bit_exact(ctx, torch_cuda, octmps, oracle, multipliers, bscan_deck,
                                       precision, position):
    """First packets of 2,000 lanes at three probe positions of the B-scan,
    seed = position + 1 as in the benchmark."""
    d = bscan_deck
    x = d["xs"][position]
    lanes = 2000
    buf = torch_cuda.zeros(lanes * REC_BYTES, dtype=torch_cuda.uint8, device="cuda")
    t_g, st = run_job(ctx, d, x, lanes, lanes, position + 1, precision, record=buf)
    r_g = np.frombuffer(buf.cpu().numpy().tobytes(), dtype=oracle_py.PACKET_DTYPE)
    deck = {"sim": type(d["sim"]).from_buffer_copy(d["sim"]), "mesh": d["mesh"],
            "root": d["mesh"].find_root(x)}
    deck["sim"].start_x = x
    t_o, r_o = run_oracle(oracle, octmps, deck, lanes, lanes, position + 1, precision, multipliers)
    assert st["packets"] == lanes and st["stopped"] == 0
    assert st["steps"] == t_o["steps"] and st["restores"] == t_o["restores"]
    assert r_g["steps"].mean() > 5000  # the total-internal-reflection regime of the benchmark
    assert_records_equal(r_g, r_o)
    assert_tallies_equal(t_g, t_o, precision, d["sim"].num_optical_depth_length_steps)


BSCAN_STAT_POSITIONS = (64, 192)
BSCAN_STAT_PACKETS = 200_000
BSCAN_STAT_LANES = 8000


@pytest.mark.parametrize("position", BSCAN_STAT_POSITIONS)
def test_bscan_mixed_form_per_bin_against_fp64_and_reference(ctx, bscan_deck, position):
    """Per-bin Class I/II means: mixed form vs FP64 form (GPU, independent
    seeds) and vs the reference's own routine (fixture), 2e5 packets each,
    every compared bin within the Bonferroni bound at 1 % family-wise error."""
    d = bscan_deck
    nb = d["sim"].num_optical_depth_length_steps
    x = d["xs"][position]
    n = BSCAN_STAT_PACKETS
    mixed, st = run_job(ctx, d, x, n, BSCAN_STAT_LANES, 11 + position, 0)
    fp64, _ = run_job(ctx, d, x, n, BSCAN_STAT_LANES, 12 + position, 2)
    assert st["stopped"] == 0 and mixed["num_nonfinite"] == 0
    others = {"fp64": fp64}
    ref_path = os.path.join(GOLDEN, "bscan_ref_tallies.npz")
    if os.path.exists(ref_path):
        ref = np.load(ref_path)
        others["reference"] = {k: ref[f"p{position}_{k}"] for k in
                               ("sum1", "sumsq1", "sum2", "sumsq2", "count1", "count2")}
        n_ref = int(ref[f"p{position}_packets"])
        assert abs(float(ref[f"p{position}_x"]) - x) < 1e-15
    for name, o in others.items():
        n_o = n if name == "fp64" else n_ref
        zs = [per_bin_z(mixed, n, o, n_o, nb, c) for c in ("1", "2")]
        m = sum(len(z) for z in zs)
        bound = bonferroni_z(m)
        worst = max(float(np.max(np.abs(z))) for z in zs if len(z))
        assert m >= 100, (name, m)
        assert worst < bound, (name, position, m, worst, bound)


LAYERS_PACKETS = 1_000_000


def test_layers_precision_forms_per_bin(ctx, layers_deck):
    """The precision study at reduced counts: on the four-layer slab with
    tilted interfaces (993,600 tets, 1499 depth bins of 1 um), the mixed,
    FP32 and FP64 forms (GPU, independent seeds, 1e6 packets each) agree per
    Class I/II bin with one another and with the reference's own routine
    (fixture, 1e6 packets), every compared bin within the Bonferroni bound at
    1 % family-wise error; no NaN or infinite contribution in any form."""
    d = layers_deck
    nb = d["sim"].num_optical_depth_length_steps
    n = LAYERS_PACKETS
    runs = {}
    for name, prec, seed in (("mixed", 0, 8001), ("fp32", 1, 8002), ("fp64", 2, 8003)):
        t, st = run_job(ctx, d, d["x"], n, 88800, seed, prec)
        assert st["packets"] == n and t["num_nonfinite"] == 0, name
        runs[name] = (t, n)
    ref_path = os.path.join(GOLDEN, "layers_ref_tallies.npz")
    if os.path.exists(ref_path):
        ref = np.load(ref_path)
        assert abs(float(ref["x"]) - d["x"]) < 1e-15
        runs["reference"] = ({k: ref[k] for k in ("sum1", "sumsq1", "sum2", "sumsq2", "count1",
                                                   "count2")}, int(ref["packets"]))
    pairs = [("mixed", "fp64"), ("fp32", "fp64"), ("mixed", "fp32")]
    if "reference" in runs:
        pairs += [("mixed", "reference"), ("fp64", "reference")]
    for a, b in pairs:
        (ta, na), (tb, nb_) = runs[a], runs[b]
        zs = [per_bin_z(ta, na, tb, nb_, nb, c) for c in ("1", "2")]
        m = sum(len(z) for z in zs)
        bound = bonferroni_z(m)
        worst = max(float(np.max(np.abs(z))) for z in zs if len(z))
        assert m >= 200, (a, b, m)
        assert worst < bound, (a, b, m, worst, bound)
