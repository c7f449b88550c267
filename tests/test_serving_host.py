"""Host logic of the serving loop and of the synthetic configurations (no GPU):
request streams, lane policy, latency statistics, request overlap, and the
layered and random-inclusion meshes."""
import os

import numpy as np
import pytest


@pytest.fixture(scope="module")
def serve():
    import serve as m
    return m


def fake_meshes():
    return {k: {} for k in ("m50k", "m400k", "m1M", "m2M")}


def test_stream_mix_and_sizes(serve):
    reqs = serve.make_stream(fake_meshes(), 400, 2.0, np.random.default_rng(5), 1.0)
    kinds = [r.kind for _, r in reqs]
    assert 0.65 < kinds.count("ascan") / len(kinds) < 0.85  # A-scan : B-scan = 3 : 1
    times = [t for t, _ in reqs]
    assert all(b > a for a, b in zip(times, times[1:]))
    gaps = np.diff([0.0] + times)
    assert 0.35 < gaps.mean() < 0.65  # Poisson arrivals at 2 per second
    for _, r in reqs:
        if r.kind == "ascan":
            assert len(r.xs) == 1 and 1e5 <= r.photons <= 1e7
        else:
            assert 32 <= len(r.xs) <= 128 and r.photons == 100_000
            assert np.allclose(np.diff(r.xs), 1e-4)


def test_stream_requests_do_not_depend_on_the_rate(serve):
    a = serve.make_stream(fake_meshes(), 50, 1e9, np.random.default_rng(55), 1.0)
    b = serve.make_stream(fake_meshes(), 50, 0.3, np.random.default_rng(55), 1.0)
    for (_, ra), (_, rb) in zip(a, b):
        assert (ra.kind, ra.mesh_key, ra.xs, ra.photons, ra.seed) == \
            (rb.kind, rb.mesh_key, rb.xs, rb.photons, rb.seed)


def test_lane_policy(serve):
    R = serve.Request
    assert serve.lanes_for(R(0, "ascan", "m", [0.0], 10_000_000, 1)) == 88_800
    assert serve.lanes_for(R(0, "ascan", "m", [0.0], 10_000_000, 1), 1 << 18) == 1 << 18
    assert serve.lanes_for(R(0, "ascan", "m", [0.0], 100_000, 1)) == 12_500
    assert serve.lanes_for(R(0, "ascan", "m", [0.0], 5, 1)) == 1
    assert serve.lanes_for(R(0, "ascan", "m", [0.0], 100_000, 1, lanes=777)) == 777


def test_latency_stats_and_overlap(serve):
    R = serve.Request
    reqs = []
    for i, (arr, adm, done, kind) in enumerate([(0, 0, 1, "ascan"), (0.5, 0.5, 2, "ascan"),
                                                (5, 5, 6, "bscan"), (3, 3, 4, "ascan")]):
        r = R(i, kind, "m", [0.0], 1000, 1)
        r.t_arrival, r.t_admitted, r.t_done = arr, adm, done
        reqs.append(r)
    st = serve.latency_stats(reqs)
    assert st["ascan"]["n"] == 3 and st["bscan"]["n"] == 1
    assert st["ascan"]["p50_ms"] == pytest.approx(1000.0)
    assert st["bscan"]["p99_ms"] == pytest.approx(1000.0)
    assert serve.overlapping(reqs) == 2  # the first two overlap; the others stand alone


def test_layered_slab_geometry(octmps, meshgen, tmp_path):
    """The four-layer slab: tilted interfaces lie on grid faces, so every tet
    sits in one layer, layers stack in order, and the mesh is conforming."""
    p = meshgen.config_layers(str(tmp_path / "lay"), nx=12, ny=12, nz=10)
    mesh = octmps.build_mesh(p["mesh"])
    sim = octmps.read_deck(p["opt"], p["mci"])
    assert sim.n_regions == 5 and sim.num_optical_depth_length_steps == 1499
    n = np.loadtxt(p["mesh"], max_rows=2).astype(int)
    verts = np.loadtxt(p["mesh"], skiprows=2, max_rows=n[0])
    tets = np.loadtxt(p["mesh"], skiprows=2 + n[0], dtype=int)
    cz = verts[tets[:, :4] - 1, 2].mean(axis=1)
    cx = verts[tets[:, :4] - 1, 0].mean(axis=1)
    tilt = np.tan(np.radians(5.0))
    bounds = [lambda x: 0.0 * x, lambda x: 0.01 + 0.0 * x, lambda x: 0.03 + tilt * x,
              lambda x: 0.07 + tilt * x, lambda x: 0.15 + 0.0 * x]
    for region in range(1, 5):
        sel = tets[:, 4] == region
        assert sel.any()
        assert np.all(cz[sel] > bounds[region - 1](cx[sel]))
        assert np.all(cz[sel] < bounds[region](cx[sel]))
    # conforming: every interior face is shared by exactly two tets
    faces = np.sort(np.concatenate([tets[:, [0, 1, 2]], tets[:, [0, 1, 3]], tets[:, [0, 2, 3]],
                                    tets[:, [1, 2, 3]]]), axis=1)
    _, counts = np.unique(faces, axis=0, return_counts=True)
    assert counts.max() == 2
    assert mesh.find_root(0.0) >= 0


def test_random_jobs_are_reproducible(meshgen, tmp_path):
    a = [meshgen.config_random_job(str(tmp_path / f"a{i}"), r, i, target_tets=60_000,
                                   n_photons=1000)
         for r in [np.random.default_rng(4)] for i in range(2)]
    b = [meshgen.config_random_job(str(tmp_path / f"b{i}"), r, i, target_tets=60_000,
                                   n_photons=1000)
         for r in [np.random.default_rng(4)] for i in range(2)]
    for pa, pb in zip(a, b):
        assert pa["n_tets"] == pb["n_tets"]
        for k in ("mesh", "opt"):
            assert open(pa[k]).read() == open(pb[k]).read()
