"""The CUDA photon kernel against the CPU oracle, through the C-ABI.

Bit-exact: every packet's event sequence (tet and event kind per step), its
generator states at the end, its step/hit/scatter/restore/detection counts,
its optical path and summed contribution, in each precision; every tally
count.  Tally sums agree to summation order only (device atomics): 1e-12
relative in FP64 accumulation, 1e-5 in the all-FP32 form.
"""
import os
import subprocess

import numpy as np
import pytest

from conftest import GOLDEN, ROOT, three_sigma_ok

import oracle_py

pytestmark = pytest.mark.gpu

REC_BYTES = oracle_py.PACKET_DTYPE.itemsize
SUM_RTOL = {0: 1e-12, 1: 1e-5, 2: 1e-12}
# The all-FP32 form accumulates with float atomics, which flush subnormal
# results to zero (squares of contributions below ~1e-19 vanish on the
# device, not in the oracle).
SUM_ATOL = {0: 0.0, 1: 1e-37, 2: 0.0}


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


def run_gpu(ctx, torch, deck, n_photons, lanes, seed, precision, record=True):
    mid = ctx.upload_mesh(deck["mesh"])
    sim = deck["sim"]
    buf = torch.zeros(lanes * REC_BYTES, dtype=torch.uint8, device="cuda") if record else None
    jid = ctx.submit(mid, sim, sim.start_x, deck["root"], n_photons=n_photons, seed=seed,
                     n_lanes=lanes, precision=precision)
    if record:
        ctx.record_next_launch(buf.data_ptr())
    ctx.flush()
    t = ctx.fetch(jid, sim.num_optical_depth_length_steps)
    st = ctx.stats(jid)
    ctx.release(jid)
    ctx.release_mesh(mid)
    rec = np.frombuffer(buf.cpu().numpy().tobytes(), dtype=oracle_py.PACKET_DTYPE) if record else None
    return t, st, rec


def run_oracle(oracle, octmps, deck, n_photons, lanes, seed, precision, multipliers):
    rng = octmps.rng_init(multipliers[: 3 + 3 * lanes], lanes, seed)
    p = oracle_py.params_from_sim(deck["sim"])
    return oracle.run(p, deck["mesh"], (deck["sim"].start_x, 0, 0), deck["root"], n_photons,
                      lanes, rng, precision, record=True)


def assert_tallies_equal(t_gpu, t_orc, precision, nbins):
    for k in ("num_filtered", "num_filtered_class1", "num_filtered_class2"):
        assert t_gpu[k] == t_orc[k], k
    for k in ("count1", "count2"):
        np.testing.assert_array_equal(t_gpu[k], t_orc[k], err_msg=k)
    for k in ("sum1", "sumsq1", "sum2", "sumsq2"):
        np.testing.assert_allclose(t_gpu[k][:nbins], t_orc[k][:nbins], rtol=SUM_RTOL[precision],
                                   atol=SUM_ATOL[precision], err_msg=k)
    for k in ("max1", "max2"):
        np.testing.assert_array_equal(t_gpu[k][:nbins], t_orc[k][:nbins], err_msg=k)


def assert_records_equal(r_gpu, r_orc):
    for f in r_orc.dtype.names:
        bad = np.where(r_gpu[f] != r_orc[f])[0]
        assert len(bad) == 0, (f, bad[:5], r_gpu[f][bad[:3]], r_orc[f][bad[:3]])


@pytest.mark.parametrize("form", [0, 1])
@pytest.mark.parametrize("precision", [0, 1, 2])
@pytest.mark.parametrize("deckname", ["small_deck", "small_matched_deck"])
def test_first_packets_and_tallies_bit_exact(request, ctx, torch_cuda, octmps, oracle,
                                             multipliers, precision, deckname, form):
    """Both kernel forms (0 per-lane, 1 pooled) against the oracle."""
    deck = request.getfixturevalue(deckname)
    lanes, n = 3000, 3000  # one packet per lane
    ctx.configure(kernel_form=form, block_size=0, blocks_per_sm=0)
    try:
        t_g, st, r_g = run_gpu(ctx, torch_cuda, deck, n, lanes, 985456376, precision)
    finally:
        ctx.configure(kernel_form=0, block_size=0, blocks_per_sm=0)
    t_o, r_o = run_oracle(oracle, octmps, deck, n, lanes, 985456376, precision, multipliers)
    assert st["packets"] == n
    assert st["steps"] == t_o["steps"] and st["restores"] == t_o["restores"]
    assert_records_equal(r_g, r_o)
    assert_tallies_equal(t_g, t_o, precision, deck["sim"].num_optical_depth_length_steps)


@pytest.mark.parametrize("form", [0, 1])
@pytest.mark.parametrize("precision", [0, 2])
def test_many_packets_per_lane_bit_exact(ctx, torch_cuda, octmps, oracle, multipliers, small_deck,
                                         precision, form):
    """Lanes run several packets in a row from the same streams (N % lanes != 0)."""
    lanes, n = 997, 20000
    ctx.configure(kernel_form=form, block_size=0, blocks_per_sm=0)
    try:
        t_g, st, r_g = run_gpu(ctx, torch_cuda, small_deck, n, lanes, 5, precision)
    finally:
        ctx.configure(kernel_form=0, block_size=0, blocks_per_sm=0)
    t_o, r_o = run_oracle(oracle, octmps, small_deck, n, lanes, 5, precision, multipliers)
    assert st["packets"] == n and st["steps"] == t_o["steps"]
    assert_records_equal(r_g, r_o)
    assert_tallies_equal(t_g, t_o, precision, small_deck["sim"].num_optical_depth_length_steps)


def test_batch_equals_alone(ctx, torch_cuda, octmps, small_deck, small_matched_deck):
    """Jobs of two meshes, several probes, seeds and sizes in one persistent
    launch give the same counts as each job alone (sums to summation order)."""
    specs = [(small_deck, 0.0, 1, 5000, 1000), (small_matched_deck, 0.0, 2, 3000, 3000),
             (small_deck, 0.0, 3, 8000, 777), (small_matched_deck, 0.0, 4, 100, 100)]
    meshes = {id(d): ctx.upload_mesh(d["mesh"]) for d, *_ in specs}
    nb = small_deck["sim"].num_optical_depth_length_steps
    alone = []
    for d, x, seed, n, lanes in specs:
        j = ctx.submit(meshes[id(d)], d["sim"], x, d["root"], n_photons=n, seed=seed, n_lanes=lanes)
        alone.append(ctx.fetch(j, nb))
        ctx.release(j)
    ids = [ctx.submit(meshes[id(d)], d["sim"], x, d["root"], n_photons=n, seed=seed, n_lanes=lanes)
           for d, x, seed, n, lanes in specs]
    ctx.flush()
    for j, a, s in zip(ids, alone, specs):
        b = ctx.fetch(j, nb)
        assert ctx.stats(j)["packets"] == s[3]
        assert_tallies_equal(b, a, 0, nb)
        ctx.release(j)
    for mid in meshes.values():
        ctx.release_mesh(mid)


def test_product_form_within_3_sigma_of_reference(ctx, octmps, small_deck):
    """The default (mixed FP32/FP64) kernel against four reference A-scans."""
    ref = np.load(os.path.join(GOLDEN, "small_ref_tallies.npz"))
    sim = small_deck["sim"]
    nb = sim.num_optical_depth_length_steps
    n = sim.number_of_photons
    mid = ctx.upload_mesh(small_deck["mesh"])
    ids = [ctx.submit(mid, sim, sim.start_x, small_deck["root"], seed=s, n_lanes=2400)
           for s in (21, 22, 23, 24)]
    ts = [ctx.fetch(j, nb) for j in ids]
    for j in ids:
        ctx.release(j)
    ctx.release_mesh(mid)
    g = {k: sum(t[k] for t in ts) for k in ("sum1", "sumsq1", "sum2", "sumsq2")}
    r = {k: sum(ref[f"run{i}_{k}"] for i in range(4)) for k in g}
    for c in ("1", "2"):
        frac, worst = three_sigma_ok(g["sum" + c][:nb], g["sumsq" + c][:nb], 4 * n,
                                     r["sum" + c][:nb], r["sumsq" + c][:nb], 4 * n)
        assert frac >= 0.98 and worst < 6.0, (c, frac, worst)


def test_full_size_plain_ascan(ctx, torch_cuda, octmps, oracle, meshgen, multipliers, workdir):
    """Config 1 at full size (288,000 tets, 1e5 packets, one A-scan): the first
    packets of 2000 lanes bit-exact against the oracle; whole-run invariants."""
    p = meshgen.config_plain_ascan(os.path.join(workdir, "plain"))
    sim = octmps.read_deck(p["opt"], p["mci"])
    deck = {"sim": sim, "mesh": octmps.build_mesh(p["mesh"]), "root": None}
    deck["root"] = deck["mesh"].find_root(sim.start_x)
    t_g, st, r_g = run_gpu(ctx, torch_cuda, deck, 2000, 2000, 1, 0)
    t_o, r_o = run_oracle(oracle, octmps, deck, 2000, 2000, 1, 0, multipliers)
    assert_records_equal(r_g, r_o)
    assert_tallies_equal(t_g, t_o, 0, sim.num_optical_depth_length_steps)
    mid = ctx.upload_mesh(deck["mesh"])
    j = ctx.submit(mid, sim, sim.start_x, deck["root"], seed=1)
    t = ctx.fetch(j, sim.num_optical_depth_length_steps)
    s = ctx.stats(j)
    ctx.release(j)
    ctx.release_mesh(mid)
    assert s["packets"] == 100000
    assert t["num_filtered"] > 0
    # every detection adds one count to each in-range bin of its window of 6
    assert t["count1"].sum() + t["count2"].sum() <= 6 * t["num_filtered"]
    assert t["num_filtered_class1"] + t["num_filtered_class2"] <= t["num_filtered"]
    assert np.all(t["max1"] <= t["sum1"] + 1e-300) and np.all(t["sumsq1"] >= 0)


def test_error_paths(ctx, octmps, small_deck):
    sim = small_deck["sim"]
    mid = ctx.upload_mesh(small_deck["mesh"])
    with pytest.raises(octmps.OctmpsError) as e:
        ctx.submit(mid, sim, 0.0, -1)
    assert e.value.status == 1
    with pytest.raises(octmps.OctmpsError) as e:
        ctx.submit(mid + 1000, sim, 0.0, small_deck["root"])
    assert e.value.status == 5
    with pytest.raises(octmps.OctmpsError) as e:
        ctx.submit(mid, sim, 0.0, small_deck["root"], precision=7)
    assert e.value.status == 1
    with pytest.raises(octmps.OctmpsError) as e:
        ctx.submit(mid, sim, 0.0, small_deck["root"], n_photons=10 ** 6, n_lanes=10 ** 6)
    assert e.value.status == 1
    # a wait that times out leaves the job running; a later wait completes it
    j = ctx.submit(mid, sim, 0.0, small_deck["root"], n_photons=400000, n_lanes=4000)
    ctx.flush()
    st = ctx.wait(j, 0)
    assert st in (0, 4)
    assert ctx.wait(j, -1) == 0
    ctx.release(j)
    ctx.release_mesh(mid)
    with pytest.raises(octmps.OctmpsError):
        ctx.release_mesh(mid)


def test_cli_end_to_end(octmps, oracle, small_deck, multipliers, tmp_path):
    """The drop-in CLI writes the reference's four .out files; its counts equal
    the oracle's for the same lanes and seed, its means to print precision."""
    p = small_deck["paths"]
    np.savetxt(tmp_path / "safeprimes_base32.txt",
               np.stack([multipliers, multipliers - 1, np.full_like(multipliers, 2 ** 32 - 1)], 1),
               fmt="%d")
    exe = os.path.join(ROOT, "oct-mps_b200", "octmps")
    r = subprocess.run([exe, "-S7", "-L2400", p["opt"], p["mesh"], p["mci"]], cwd=tmp_path,
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    sim = small_deck["sim"]
    rng = octmps.rng_init(multipliers[: 3 + 3 * 2400], 2400, 7)
    t = oracle.run(oracle_py.params_from_sim(sim), small_deck["mesh"], (sim.start_x, 0, 0),
                   small_deck["root"], sim.number_of_photons, 2400, rng, 0)
    d = tmp_path / "want"
    d.mkdir()
    octmps.write_result(str(d), sim, sim.start_x, t)
    for fn in ("ClassI_Scatt.out", "ClassII_Scatt.out", "ClassI_ScattFilt.out",
               "ClassII_ScattFilt.out"):
        got = np.loadtxt(tmp_path / fn, delimiter=",")
        want = np.loadtxt(d / fn, delimiter=",")
        np.testing.assert_array_equal(got[:, [0, 1, 4]], want[:, [0, 1, 4]])
        np.testing.assert_allclose(got[:, 2:4], want[:, 2:4], rtol=2e-5, atol=0)
    assert (tmp_path / "BiasParam.mco").read_text() == (d / "BiasParam.mco").read_text()


def test_jobs_join_a_running_launch_and_match_alone(ctx, octmps, small_deck, small_matched_deck):
    """Continuous batching: jobs submitted while a long job runs are taken up
    at once (they finish while it still runs, by the running launch's threads
    or by a launch started beside it) and give the same counts as each job
    run alone."""
    nb = small_deck["sim"].num_optical_depth_length_steps
    m1 = ctx.upload_mesh(small_deck["mesh"])
    m2 = ctx.upload_mesh(small_matched_deck["mesh"])
    late = [(small_matched_deck, m2, 7, 4000, 500), (small_deck, m1, 8, 3000, 300),
            (small_deck, m1, 9, 2000, 2000)]
    alone = []
    for d, mid, seed, n, lanes in late:
        j = ctx.submit(mid, d["sim"], 0.0, d["root"], n_photons=n, seed=seed, n_lanes=lanes)
        alone.append(ctx.fetch(j, nb))
        ctx.release(j)
    # a long job first (500 packets in a row on each of its 2000 lanes, a
    # few seconds), then the others while it runs
    big = ctx.submit(m1, small_deck["sim"], 0.0, small_deck["root"], n_photons=1_000_000,
                     seed=1, n_lanes=2000)
    ctx.flush()
    ids = [ctx.submit(mid, d["sim"], 0.0, d["root"], n_photons=n, seed=seed, n_lanes=lanes)
           for d, mid, seed, n, lanes in late]
    ctx.flush()
    for j, a in zip(ids, alone):
        b = ctx.fetch(j, nb)
        assert_tallies_equal(b, a, 0, nb)
    assert ctx.wait(big, 0) == 4  # the long job still runs (OCTMPS_ERR_TIMEOUT)
    ctx.fetch(big, nb)
    assert ctx.stats(big)["packets"] == 1_000_000
    ctx.synchronize()
    for j in ids + [big]:
        s = ctx.stats(j)
        assert s["launch_id"] >= 1 and s["device_ms"] > 0
    for j in ids + [big]:
        ctx.release(j)
    ctx.release_mesh(m1)
    ctx.release_mesh(m2)


def test_completion_queue_reports_each_job_once(ctx, octmps, small_deck):
    sim = small_deck["sim"]
    mid = ctx.upload_mesh(small_deck["mesh"])
    ids = [ctx.submit(mid, sim, 0.0, small_deck["root"], n_photons=3000 + 100 * k, seed=20 + k,
                      n_lanes=300) for k in range(5)]
    ctx.flush()
    seen = []
    for _ in range(200000):
        seen += ctx.poll()
        if len(seen) >= len(ids):
            break
    assert sorted(seen) == sorted(ids)
    assert ctx.poll() == []
    for j in ids:
        assert ctx.wait(j, 0) == 0
        ctx.release(j)
    ctx.release_mesh(mid)


def test_admission_by_hbm_budget(octmps, multipliers, small_deck, torch_cuda):
    """Jobs beyond the HBM budget are refused (OCTMPS_ERR_BUDGET) until
    finished jobs are released."""
    sim = small_deck["sim"]
    with octmps.Context(0, multipliers) as c:
        lanes = 1000
        nb = sim.num_optical_depth_length_steps
        # tally block (as laid out on the device) + statistics words, FP64 sums
        per_job = 32 + 2 * (((nb + 1) * 8 + 15) // 16 * 16) + \
            6 * (((nb + 2) * 8 + 15) // 16 * 16) + 32
        c.configure(hbm_budget_bytes=lanes * 36 + 2 * per_job + per_job // 2)
        mid = c.upload_mesh(small_deck["mesh"])
        a = c.submit(mid, sim, 0.0, small_deck["root"], n_photons=2000, seed=3, n_lanes=lanes)
        b = c.submit(mid, sim, 0.0, small_deck["root"], n_photons=2000, seed=3, n_lanes=lanes)
        with pytest.raises(octmps.OctmpsError) as e:
            c.submit(mid, sim, 0.0, small_deck["root"], n_photons=2000, seed=3, n_lanes=lanes)
        assert e.value.status == 8
        c.flush()
        c.fetch(a, nb)
        c.release(a)
        c.synchronize()  # released memory counts until no launch runs
        d = c.submit(mid, sim, 0.0, small_deck["root"], n_photons=2000, seed=3, n_lanes=lanes)
        c.flush()
        for j in (b, d):
            c.fetch(j, nb)
            c.release(j)
        c.release_mesh(mid)


def test_stopped_packet_bit_exact_on_2m_tet_mesh(ctx, torch_cuda, octmps, oracle, multipliers,
                                                  plain_2m_deck):
    """First packets of 5619 lanes on the 1,999,200-tet mesh, the last of them
    a packet that makes no progress: the kernel stops it at the same step as
    the oracle (one stopped packet), and every record and count agrees."""
    from conftest import STUCK_CASE as S
    d = dict(plain_2m_deck)
    d["root"] = d["mesh"].find_root(S["x"])
    d["sim"] = type(d["sim"]).from_buffer_copy(d["sim"])  # probe at the case's x
    d["sim"].start_x = S["x"]
    lanes = S["lane"] + 1
    t_g, st, r_g = run_gpu(ctx, torch_cuda, d, lanes, lanes, S["seed"], 0)
    t_o, r_o = run_oracle(oracle, octmps, d, lanes, lanes, S["seed"], 0, multipliers)
    assert st["stopped"] == 1 and t_o["capped"] == 1
    assert r_g["steps"][S["lane"]] == S["steps"]
    assert st["steps"] == t_o["steps"]
    assert_records_equal(r_g, r_o)
    assert_tallies_equal(t_g, t_o, 0, d["sim"].num_optical_depth_length_steps)


@pytest.mark.parametrize("precision", [0, 1])
def test_fp32_forms_keep_the_likelihood_finite(ctx, octmps, layers_deck, precision):
    """37 packets on each of 36,486 lanes of the four-layer slab, the last lane
    being the one whose 37th packet had a NaN likelihood before cosines were
    clamped: no NaN or infinite contribution, every sum finite."""
    from conftest import NAN_CASE as S
    d = layers_deck
    nb = d["sim"].num_optical_depth_length_steps
    lanes = S["lane"] + 1
    mid = ctx.upload_mesh(d["mesh"])
    j = ctx.submit(mid, d["sim"], d["x"], d["root"], n_photons=S["packets"] * lanes,
                   seed=S["seed"], n_lanes=lanes, precision=precision)
    t = ctx.fetch(j, nb)
    ctx.release(j)
    ctx.release_mesh(mid)
    assert t["num_nonfinite"] == 0
    for k in ("sum1", "sumsq1", "sum2", "sumsq2"):
        assert np.all(np.isfinite(t[k][:nb])), k


def test_autotune_picks_a_variant_and_keeps_results(ctx, octmps, small_deck):
    """The autotuner times each launch variant (kernel form, block size,
    blocks per SM, scatter share, optionally lanes) on a sample and keeps the
    fastest; the launch variants change timing only, never the counts."""
    sim = small_deck["sim"]
    nb = sim.num_optical_depth_length_steps
    mid = ctx.upload_mesh(small_deck["mesh"])
    variants = [(0, 256, 2, 12), (0, 128, 7, 16), (0, 512, 2, 12), (1, 128, 4, 12),
                (0, 256, 3, 12, 10_000)]
    best, table = ctx.autotune(mid, sim, 0.0, small_deck["root"], n_photons=100_000,
                               n_jobs=2, n_lanes=20_000, variants=variants)
    assert len(table) == 5 and best in table and all(r[5] > 0 for r in table)
    assert [r[4] for r in table] == [20_000] * 4 + [10_000]
    runs = []
    for form, bs, b, sh in ((0, 256, 2, 8), (0, 256, 3, 24), (0, 128, 6, 12), (0, 128, 8, 4),
                            (0, 512, 2, 20), (1, 128, 5, 8), (1, 128, 6, 24)):
        ctx.configure(kernel_form=form, block_size=bs, blocks_per_sm=b, scatter_share=sh)
        j = ctx.submit(mid, sim, 0.0, small_deck["root"], n_photons=30_000, seed=3, n_lanes=3000)
        runs.append(ctx.fetch(j, nb))
        ctx.release(j)
    ctx.configure(kernel_form=0, block_size=0, blocks_per_sm=0, scatter_share=0)
    for r in runs[1:]:
        assert_tallies_equal(r, runs[0], 0, nb)
    ctx.release_mesh(mid)


def test_configure_rejects_launch_variants_that_do_not_exist(ctx, octmps):
    """Per-lane blocks: 256 x 2..4, 128 x 6..8, 512 x 2; pooled: 128 x 2..6."""
    for bad in ({"block_size": 128, "blocks_per_sm": 3}, {"block_size": 512, "blocks_per_sm": 3},
                {"block_size": 64}, {"block_size": 256, "blocks_per_sm": 5},
                {"kernel_form": 1, "block_size": 256}, {"kernel_form": 1, "blocks_per_sm": 7}):
        with pytest.raises(octmps.OctmpsError):
            ctx.configure(**bad)
    for good in ({"block_size": 128, "blocks_per_sm": 7}, {"block_size": 512},
                 {"block_size": 128}, {"kernel_form": 1, "blocks_per_sm": 5}):
        ctx.configure(**good)
        ctx.configure(kernel_form=0, block_size=0, blocks_per_sm=0)
