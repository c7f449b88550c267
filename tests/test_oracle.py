"""The CPU oracle (oracle/oracle.cpp) pinned against the reference's own code.

* its math kernels against numpy in float64 (error bounds),
* its FP64 first-packet event sequences against the reference routine's on
  the Sphere deck (tests/golden/sphere_first_packets.npz),
* its per-bin Class I/II tallies, in all three precisions, against full
  A-scans of the reference routine (tests/golden/small_ref_tallies.npz)
  within 3 standard errors.
"""
import ctypes as C
import os

import numpy as np
import pytest

from conftest import GOLDEN, ref_deck_paths, three_sigma_ok

import oracle_py


def ulp32(x):
    return np.spacing(np.abs(np.float32(x))).astype(np.float64)


def test_logf_accuracy(oracle):
    rng = np.random.default_rng(1)
    xs = np.concatenate([rng.random(20000), np.float32(2.0) ** -np.arange(1, 25), [1.0]])
    xs = xs[xs > 0].astype(np.float32)
    got = np.array([oracle.L.oracle_logf(float(x)) for x in xs], np.float64)
    want = np.log(xs.astype(np.float64))
    err = np.abs(got - want) / np.maximum(ulp32(want), np.spacing(np.float32(0.5)) * 1e-30)
    assert np.max(err[want != 0]) <= 2.0
    assert oracle.L.oracle_logf(1.0) == 0.0
    assert oracle.L.oracle_logf(0.0) == -np.inf


def test_log_accuracy(oracle):
    rng = np.random.default_rng(2)
    xs = np.concatenate([rng.random(20000), 2.0 ** -np.arange(1, 60), rng.random(100) * 1e6])
    xs = xs[xs > 0]
    got = np.array([oracle.L.oracle_log(float(x)) for x in xs])
    want = np.log(xs)
    err = np.abs(got - want) / np.spacing(np.abs(want))
    assert np.max(err[want != 0]) <= 2.0
    assert oracle.L.oracle_log(0.0) == -np.inf


def test_sincos_accuracy(oracle):
    rng = np.random.default_rng(3)
    u = rng.integers(0, 2 ** 32, 20000, dtype=np.uint64)
    t = np.array([oracle.L.oracle_uint2float_rz(int(v)) for v in u], np.float64) * 2.0 ** -32
    s, c = C.c_float(), C.c_float()
    sd, cd = C.c_double(), C.c_double()
    es, ed = [], []
    for tv in t:
        oracle.L.oracle_sincos_turn_f(float(tv), C.byref(s), C.byref(c))
        es.append(max(abs(s.value - np.sin(2 * np.pi * tv)), abs(c.value - np.cos(2 * np.pi * tv))))
        psi = (2.0 * 3.14159265359) * tv
        oracle.L.oracle_sincos_d(psi, C.byref(sd), C.byref(cd))
        ed.append(max(abs(sd.value - np.sin(psi)), abs(cd.value - np.cos(psi))))
    assert max(es) < 2.5e-7  # about 4 float ulps of 1
    assert max(ed) < 5e-16


def test_div_rd_and_rz_conversion(oracle):
    from fractions import Fraction
    rng = np.random.default_rng(4)
    for a, b in zip(rng.normal(size=2000), rng.normal(size=2000)):
        q = oracle.L.oracle_div_rd(a, b)
        assert Fraction(q) <= Fraction(a) / Fraction(b) < Fraction(np.nextafter(q, np.inf))
    assert oracle.L.oracle_div_rd(1.0, 0.1) == np.nextafter(10.0, 0.0)
    for u in rng.integers(0, 2 ** 32, 5000, dtype=np.uint64):
        f = oracle.L.oracle_uint2float_rz(int(u))
        assert f <= int(u) < float(np.nextafter(np.float32(f), np.float32(np.inf)))


def first_packet_match(oracle, octmps, name="Sphere"):
    opt, mesh_path, mci = ref_deck_paths(name)
    fix = np.load(os.path.join(GOLDEN, "sphere_first_packets.npz"))
    ref = fix["records"]
    n = len(ref)
    sim = octmps.read_deck(opt, mci)
    mesh = octmps.build_mesh(mesh_path)
    root = int(fix["root"])
    assert mesh.find_root(float(fix["probe_x"])) == root
    mult = octmps.safeprimes(3 + 3 * n)
    rng = octmps.rng_init(mult, n, int(fix["seed"]))
    p = oracle_py.params_from_sim(sim)
    _, rec = oracle.run(p, mesh, (float(fix["probe_x"]), 0, 0), root, n, n, rng, 2, record=True)
    return ref, rec


def test_fp64_first_packets_match_reference(oracle, octmps):
    """Event sequences (tet visited and event kind per step, generator states
    at the end, detections, restores) of the first packet of 2000 lanes:
    the FP64 restatement against the reference routine itself.  The
    reference's log/sincos/acos are glibc's, the oracle's are its own, so a
    last-bit difference in a direction can flip a discrete decision (most
    often an exit through a matched-index face whose Fresnel R is exactly 0
    in one and ~1e-32 in the other); the fraction of identical packets is
    pinned from below."""
    ref, rec = first_packet_match(oracle, octmps)
    same = ((rec["hash"] == ref["hash"]) & (rec["x"] == ref["x"]) & (rec["xR"] == ref["xR"]) &
            (rec["xS"] == ref["xS"]) & (rec["steps"] == ref["steps"]) &
            (rec["detections"] == ref["detections"]) & (rec["restores"] == ref["restores"]))
    assert same.mean() >= 0.90, same.mean()
    c_ref, c_orc = ref["contribution"][same], rec["contribution"][same]
    nz = c_ref != 0
    assert np.all(np.abs(c_orc[nz] - c_ref[nz]) <= 1e-9 * np.abs(c_ref[nz]))
    assert np.array_equal(c_orc[~nz], c_ref[~nz])


def small_params(octmps, small_deck):
    return oracle_py.params_from_sim(small_deck["sim"])


@pytest.mark.parametrize("precision", [2, 0, 1])
def test_oracle_tallies_within_3_sigma_of_reference(oracle, octmps, small_deck, precision):
    """Full A-scans (20000 packets each) of the small mismatched-index deck:
    the oracle with seeds independent of the reference runs, per-bin Class I
    and Class II means compared within 3 combined standard errors."""
    ref = np.load(os.path.join(GOLDEN, "small_ref_tallies.npz"))
    sim = small_deck["sim"]
    n = sim.number_of_photons
    nb = sim.num_optical_depth_length_steps
    runs = 4
    ref_sum = {k: sum(ref[f"run{r}_{k}"] for r in range(runs)) for k in
               ("sum1", "sumsq1", "sum2", "sumsq2", "count1", "count2")}
    lanes = 2400
    mult = octmps.safeprimes(3 + 3 * lanes)
    p = small_params(octmps, small_deck)
    acc = None
    for seed in (11, 12, 13, 14):
        rng = octmps.rng_init(mult, lanes, seed)
        t = oracle.run(p, small_deck["mesh"], (sim.start_x, 0, 0), small_deck["root"], n, lanes,
                       rng, precision)
        assert t["packets"] == n and t["capped"] == 0
        acc = t if acc is None else {k: acc[k] + t[k] for k in acc}
    N = n * runs
    for c in ("1", "2"):
        frac, worst = three_sigma_ok(acc["sum" + c][:nb], acc["sumsq" + c][:nb], N,
                                     ref_sum["sum" + c][:nb], ref_sum["sumsq" + c][:nb], N)
        assert frac >= 0.98 and worst < 6.0, (c, frac, worst)
    # detections per packet agree within 3 sigma (Poisson)
    d_o = acc["num_filtered"]
    d_r = sum(int(ref[f"run{r}_num_filtered"]) for r in range(runs))
    assert abs(d_o - d_r) <= 3 * np.sqrt(d_o + d_r) + 1


def test_oracle_is_deterministic(oracle, octmps, small_deck):
    sim = small_deck["sim"]
    lanes = 500
    rng = octmps.rng_init(octmps.safeprimes(3 + 3 * lanes), lanes, 7)
    p = small_params(octmps, small_deck)
    a = oracle.run(p, small_deck["mesh"], (sim.start_x, 0, 0), small_deck["root"], 2000, lanes,
                   rng, 0, n_threads=3)
    b = oracle.run(p, small_deck["mesh"], (sim.start_x, 0, 0), small_deck["root"], 2000, lanes,
                   rng, 0, n_threads=3)
    for k in a:
        np.testing.assert_array_equal(a[k], b[k])


def test_oracle_stops_a_packet_that_makes_no_progress(octmps, oracle, multipliers, plain_2m_deck):
    from conftest import STUCK_CASE as S
    import oracle_py
    d = plain_2m_deck
    root = d["mesh"].find_root(S["x"])
    rng = octmps.rng_init(multipliers[: 3 + 3 * (S["lane"] + 1)], S["lane"] + 1, S["seed"])
    one = {k: v[S["lane"]:S["lane"] + 1].copy() for k, v in rng.items()}
    t, rec = oracle.run(oracle_py.params_from_sim(d["sim"]), d["mesh"], (S["x"], 0.0, 0.0), root,
                        1, 1, one, 0, record=True)
    assert t["capped"] == 1
    assert rec["steps"][0] == S["steps"]


@pytest.mark.parametrize("precision", [0, 1])
def test_oracle_fp32_forms_keep_the_likelihood_finite(octmps, oracle, multipliers, layers_deck,
                                                      precision):
    from conftest import NAN_CASE as S
    import oracle_py
    d = layers_deck
    rng = octmps.rng_init(multipliers[: 3 + 3 * (S["lane"] + 1)], S["lane"] + 1, S["seed"])
    one = {k: v[S["lane"]:S["lane"] + 1].copy() for k, v in rng.items()}
    t = oracle.run(oracle_py.params_from_sim(d["sim"]), d["mesh"], (d["x"], 0.0, 0.0), d["root"],
                   S["packets"], 1, one, precision)
    nb = d["sim"].num_optical_depth_length_steps
    assert t["num_filtered"] > 0
    for k in ("sum1", "sumsq1", "sum2", "sumsq2"):
        assert np.all(np.isfinite(t[k][:nb])), k


def test_oracle_multiplier_list_equals_the_product_generator(oracle, octmps):
    """The oracle's MWC multiplier list (used where the product library must
    not be loaded) equals the product's generator entry for entry."""
    n = 3 + 3 * 2000
    np.testing.assert_array_equal(oracle.safeprimes(n), octmps.safeprimes(n))


def test_operation_census_runs_the_oracle_and_matches_the_frozen_f_step(octmps, meshgen,
                                                                        workdir):
    """The census (the oracle's code with counting number types) gives the
    oracle's tally bit for bit, and its FLOPs per propagation step on a sample
    of the B-scan workload agree with the value the bench's roofline uses."""
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench
    p = meshgen.config_bscan(os.path.join(workdir, "bscan_census"))
    sim = octmps.read_deck(p["opt"], p["mci"])
    mesh = octmps.build_mesh(p["mesh"])
    x = octmps.probe_positions(sim)[128]
    root = mesh.find_root(x)
    par = oracle_py.params_from_sim(sim)
    lanes = 200
    mult = octmps.safeprimes(3 + 3 * lanes)
    for prec in (0, 2):
        t_c, counts = oracle_py.census(par, mesh, (x, 0, 0), root, 2 * lanes, lanes,
                                       octmps.rng_init(mult, lanes, 129), prec)
        t_o = oracle_py.Oracle().run(par, mesh, (x, 0, 0), root, 2 * lanes, lanes,
                                     octmps.rng_init(mult, lanes, 129), prec, n_threads=1)
        assert t_c["steps"] == t_o["steps"]
        for k in ("count1", "count2", "sum1", "sumsq1", "sum2", "sumsq2"):
            np.testing.assert_array_equal(t_c[k], t_o[k], err_msg=k)
        assert abs(counts["flops_per_step"] / bench.F_STEP[prec] - 1) < 0.02, counts



def method_reference():
    try:
        return oracle_py.Reference(oracle_py.REF_METHOD_SO)
    except ImportError as e:
        pytest.skip(f"reference host build unavailable: {e}")


def packets_identical(rec_r, rec_o):
    return ((rec_r["hash"] == rec_o["hash"]) & (rec_r["x"] == rec_o["x"]) &
            (rec_r["xR"] == rec_o["xR"]) & (rec_r["xS"] == rec_o["xS"]) &
            (rec_r["steps"] == rec_o["steps"]) & (rec_r["detections"] == rec_o["detections"]) &
            (rec_r["restores"] == rec_o["restores"]) &
            (rec_r["optical_path"] == rec_o["optical_path"]))


@pytest.mark.parametrize("deck", ["Sphere", "bscan"])
def test_fp64_oracle_is_the_reference_method_bit_for_bit(oracle, octmps, meshgen, workdir, deck):
    """With the reference's log and sincos routed to the oracle's series
    (oracle/_ref/libocref_method.so; acos and every other operation the
    reference's own), the FP64 restatement reproduces the reference routine
    packet for packet: event sequence, generator states, steps, detections,
    restores and optical path of every first packet identical, contributions
    equal to summation order.  So the differences against the glibc build
    (test_fp64_first_packets_match_reference) are transcendental last bits
    only.  Decks: the reference's Sphere (2000 lanes) and the B-scan workload
    at three positions (1000 lanes each, ~12,000-15,000 steps per packet)."""
    R = method_reference()
    if deck == "Sphere":
        opt, mesh_path, mci = ref_deck_paths("Sphere")
        cases = [(None, 985456376, 2000)]
    else:
        p = meshgen.config_bscan(os.path.join(workdir, "bscan_method"))
        opt, mesh_path, mci = p["opt"], p["mesh"], p["mci"]
        cases = [(k, k + 1, 1000) for k in (0, 128, 255)]
    sim = octmps.read_deck(opt, mci)
    mesh = octmps.build_mesh(mesh_path)
    rs = R.parse(opt, mci)
    xs = octmps.probe_positions(sim)
    for k, seed, n in cases:
        x = sim.start_x if k is None else xs[k]
        root = mesh.find_root(x)
        rng = octmps.rng_init(octmps.safeprimes(3 + 3 * n), n, seed)
        rec_r = R.trace(rs, mesh, root, (x, 0, 0), {a: b.copy() for a, b in rng.items()}, n)
        _, rec_o = oracle.run(oracle_py.params_from_sim(sim), mesh, (x, 0, 0), root, n, n,
                              {a: b.copy() for a, b in rng.items()}, 2, record=True)
        same = packets_identical(rec_r, rec_o)
        assert same.all(), (deck, k, np.where(~same)[0][:5])
        c_r, c_o = rec_r["contribution"], rec_o["contribution"]
        nz = c_r != 0
        assert np.all(np.abs(c_o[nz] - c_r[nz]) <= 1e-14 * np.abs(c_r[nz]))
        assert np.array_equal(c_o[~nz], c_r[~nz])
