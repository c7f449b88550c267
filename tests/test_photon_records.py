"""RecordPhotonsFlag: per-detection records (the FilteredPhotons.mco fields
that BiasParam.mco describes, src/octmps_io.cpp:259-270).  The reference
creates the file but writes no record; the records here are the values its
tally uses at each detection (src/octmps_kernel.cuh:684-744): the weight that
leaves, w (1 - R), the likelihood ratio, the radius and cosine at the exit,
the optical path and the maximum depth.

CPU: the oracle's records against its own tally, and the file writer.  GPU:
the kernel's records against the oracle's, as sets, bit for bit, in the three
forms, the capacity limit, and the CLI's file.
"""
import ctypes as C
import math
import os

import numpy as np
import pytest

import oracle_py


def oracle_records(oracle, octmps, deck, n, lanes, seed, precision, multipliers, cap):
    rng = octmps.rng_init(multipliers[: 3 + 3 * lanes], lanes, seed)
    p = oracle_py.params_from_sim(deck["sim"])
    t, recs, n_det = oracle.run(p, deck["mesh"], (deck["sim"].start_x, 0, 0), deck["root"], n,
                                lanes, rng, precision, photon_records=cap)
    return t, recs, n_det


def sorted_records(r):
    return np.sort(np.asarray(r, dtype=oracle_py.RECORD_DTYPE), order=list(oracle_py.RECORD_DTYPE.names))


@pytest.mark.parametrize("precision", [0, 2])
def test_oracle_records_match_its_tally(oracle, octmps, multipliers, small_deck, precision):
    """One record per detection; each record's class and bin give the tally's
    Class I/II totals; the fields respect the collection criteria."""
    sim = small_deck["sim"]
    t, recs, n_det = oracle_records(oracle, octmps, small_deck, 20_000, 2000, 7, precision,
                                    multipliers, 100_000)
    assert n_det == t["num_filtered"] == len(recs) > 100
    assert np.all(recs["radius"] < sim.max_collecting_radius)
    assert np.all(recs["cos_angle"] > math.cos(sim.max_collecting_angle_deg * 3.14159265359 / 180) - 1e-6)
    # a likelihood ratio can underflow to 0 in FP32
    assert np.all(recs["weight"] > 0) and np.all(recs["likelihood"] >= 0)
    # class and bin as the tally takes them: depth = path / 2, class I when the
    # maximum depth passes depth - Lc/2, counted when the bin is in range
    depth = recs["optical_path"] / 2
    vp = np.floor((depth - sim.optical_depth_shift) / (sim.coherence_length_source / 6))
    inside = (vp >= 0) & (vp < sim.num_optical_depth_length_steps)
    class1 = recs["max_depth"] > depth - sim.coherence_length_source / 2
    n1, n2 = int(np.sum(inside & class1)), int(np.sum(inside & ~class1))
    # bin edges may fall either side by one rounding: allow a handful
    assert abs(n1 - t["num_filtered_class1"]) <= 3 and abs(n2 - t["num_filtered_class2"]) <= 3


def test_oracle_record_capacity_counts_every_detection(oracle, octmps, multipliers, small_deck):
    t, recs, n_det = oracle_records(oracle, octmps, small_deck, 20_000, 2000, 7, 0, multipliers, 10)
    assert len(recs) == 10 and n_det == t["num_filtered"] > 10


def test_writer_appends_records_and_keeps_them_with_the_flag(octmps, small_deck, tmp_path):
    """FilteredPhotons.mco: probe position, Weight, LikelihoodRatio, Radius,
    AngleRad (acos of the cosine), OpticalPath, MaxDepth per line; without the
    flag the bias writer creates it empty as the reference does, with it the
    records stay."""
    d = str(tmp_path)
    r = np.zeros(3, dtype=octmps.RECORD_DTYPE)
    r["weight"] = [0.5, 0.25, 0.125]
    r["likelihood"] = [1.0, 2.0, 3.0]
    r["radius"] = [1e-3, 2e-3, 3e-3]
    r["cos_angle"] = [1.0, 0.5, 0.0]
    r["optical_path"] = [0.1, 0.2, 0.3]
    r["max_depth"] = [0.01, 0.02, 0.03]
    octmps.write_filtered_photons(d, -0.004, r[:2])
    octmps.write_filtered_photons(d, 0.004, r[2:])
    rows = [list(map(float, line.split("\t"))) for line in
            open(os.path.join(d, "FilteredPhotons.mco")).read().splitlines()]
    assert len(rows) == 3
    np.testing.assert_allclose([row[0] for row in rows], [-0.004, -0.004, 0.004])
    np.testing.assert_allclose([row[4] for row in rows], [0.0, math.acos(0.5), math.pi / 2],
                               rtol=1e-5)
    np.testing.assert_allclose([row[1] for row in rows], r["weight"])
    sim = type(small_deck["sim"]).from_buffer_copy(small_deck["sim"])
    nb = sim.num_optical_depth_length_steps
    t = octmps.empty_tally(nb)
    sim.record_photons_flag = 1
    octmps.write_result(d, sim, 0.0, t)
    assert len(open(os.path.join(d, "FilteredPhotons.mco")).read().splitlines()) == 3
    sim.record_photons_flag = 0
    octmps.write_result(d, sim, 0.0, t)
    assert open(os.path.join(d, "FilteredPhotons.mco")).read() == ""


@pytest.fixture(scope="module")
def gpu_ctx(octmps, multipliers):
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.fail("a GPU test ran without a CUDA device")
    c = octmps.Context(0, multipliers)
    yield c
    c.close()


def gpu_records(ctx, deck, n, lanes, seed, precision):
    sim = type(deck["sim"]).from_buffer_copy(deck["sim"])
    sim.record_photons_flag = 1
    mid = ctx.upload_mesh(deck["mesh"])
    j = ctx.submit(mid, sim, sim.start_x, deck["root"], n_photons=n, seed=seed, n_lanes=lanes,
                   precision=precision)
    ctx.flush()
    t = ctx.fetch(j, sim.num_optical_depth_length_steps)
    recs, n_det = ctx.photon_records(j)
    ctx.release(j)
    ctx.release_mesh(mid)
    return t, recs, n_det


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [0, 1, 2])
def test_gpu_records_equal_oracle_records(gpu_ctx, octmps, oracle, multipliers, small_deck,
                                          precision):
    """The kernel's detected-packet records equal the oracle's as a set, bit
    for bit (their order follows the threads' timing)."""
    t_g, r_g, n_g = gpu_records(gpu_ctx, small_deck, 20_000, 2000, 7, precision)
    t_o, r_o, n_o = oracle_records(oracle, octmps, small_deck, 20_000, 2000, 7, precision,
                                   multipliers, 100_000)
    assert n_g == n_o == t_g["num_filtered"] == len(r_g) > 100
    a, b = sorted_records(r_g), sorted_records(r_o)
    for f in oracle_py.RECORD_DTYPE.names:
        np.testing.assert_array_equal(a[f], b[f], err_msg=f)


@pytest.mark.gpu
def test_pooled_form_records_equal_oracle_records(gpu_ctx, octmps, oracle, multipliers,
                                                  small_deck):
    """The pooled kernel form keeps the same records (it shares the tally)."""
    gpu_ctx.configure(kernel_form=1, block_size=0, blocks_per_sm=0)
    try:
        t_g, r_g, n_g = gpu_records(gpu_ctx, small_deck, 20_000, 2000, 7, 0)
    finally:
        gpu_ctx.configure(kernel_form=0, block_size=0, blocks_per_sm=0)
    _, r_o, n_o = oracle_records(oracle, octmps, small_deck, 20_000, 2000, 7, 0, multipliers,
                                 100_000)
    assert n_g == n_o == len(r_g) > 100
    a, b = sorted_records(r_g), sorted_records(r_o)
    for f in oracle_py.RECORD_DTYPE.names:
        np.testing.assert_array_equal(a[f], b[f], err_msg=f)


@pytest.mark.gpu
def test_gpu_record_capacity_and_jobs_without_the_flag(gpu_ctx, octmps, small_deck):
    gpu_ctx.set_photon_record_capacity(10)
    try:
        t, recs, n_det = gpu_records(gpu_ctx, small_deck, 20_000, 2000, 7, 0)
    finally:
        gpu_ctx.set_photon_record_capacity(0)
    assert len(recs) == 10 and n_det == t["num_filtered"] > 10
    mid = gpu_ctx.upload_mesh(small_deck["mesh"])
    sim = small_deck["sim"]
    j = gpu_ctx.submit(mid, sim, sim.start_x, small_deck["root"], n_photons=5000, seed=3,
                       n_lanes=1000)
    gpu_ctx.flush()
    gpu_ctx.fetch(j, sim.num_optical_depth_length_steps)
    recs, n_det = gpu_ctx.photon_records(j)
    assert len(recs) == 0 and n_det == 0
    gpu_ctx.release(j)
    gpu_ctx.release_mesh(mid)


@pytest.mark.gpu
def test_cli_writes_the_records_of_every_detection(gpu_ctx, octmps, oracle, meshgen, multipliers,
                                                   small_deck, tmp_path):
    """The drop-in CLI with RecordPhotonsFlag set writes FilteredPhotons.mco:
    one line per detection, the same lines as the oracle's records printed the
    same way (as sets: the kernel's order follows its threads)."""
    import subprocess
    from conftest import ROOT
    p = small_deck["paths"]
    mci = str(tmp_path / "record.mci")
    meshgen.write_mci(mci, record=1)
    np.savetxt(tmp_path / "safeprimes_base32.txt",
               np.stack([multipliers, multipliers - 1, np.full_like(multipliers, 2 ** 32 - 1)], 1),
               fmt="%d")
    exe = os.path.join(ROOT, "oct-mps_b200", "octmps")
    r = subprocess.run([exe, "-S7", "-L2400", p["opt"], p["mesh"], mci], cwd=tmp_path,
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    got = (tmp_path / "FilteredPhotons.mco").read_text().splitlines()
    sim = small_deck["sim"]
    _, recs, n_det = oracle_records(oracle, octmps, small_deck, sim.number_of_photons, 2400, 7, 0,
                                    multipliers, 10 * sim.number_of_photons)
    want = ["\t".join("%G" % v for v in (sim.start_x, q["weight"], q["likelihood"], q["radius"],
                                          math.acos(q["cos_angle"]), q["optical_path"],
                                          q["max_depth"])) for q in recs]
    assert len(got) == n_det > 100
    assert sorted(got) == sorted(want)
    assert "Description of fields in file FilteredPhotons.mco" in (tmp_path / "BiasParam.mco").read_text()
