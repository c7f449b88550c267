"""Host-side pieces of the drop-in (no GPU): C-ABI exports, multiplier table,
RNG seeding, parsers, mesh builder, root finding and writers, each against
known answers produced by the reference's own code (tests/golden/)."""
import json
import os
import re

import numpy as np
import pytest

from conftest import GOLDEN, ROOT, ref_deck_paths


def header_functions():
    src = open(os.path.join(ROOT, "include", "octmps_capi.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(octmps_\w+)\s*\(", src)))


def test_library_exports_every_declared_symbol(octmps):
    L = octmps.lib()
    declared = header_functions()
    assert len(declared) >= 20
    missing = [n for n in declared if not hasattr(L, n)]
    assert not missing, missing
    assert sorted(octmps.EXPORTED) == declared


def test_status_strings(octmps):
    L = octmps.lib()
    for st in range(10):
        assert L.octmps_status_string(st).decode() == octmps.STATUS[st]


def is_prime(n):
    if n < 2:
        return False
    for p in (2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37):
        if n % p == 0:
            return n == p
    d, s = n - 1, 0
    while d % 2 == 0:
        d //= 2
        s += 1
    for a in (2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37):
        x = pow(a, d, n)
        if x in (1, n - 1):
            continue
        for _ in range(s - 1):
            x = x * x % n
            if x == n - 1:
                break
        else:
            return False
    return True


def test_safeprimes_are_valid_mwc_multipliers(octmps):
    a = octmps.safeprimes(400)
    assert np.all(np.diff(a.astype(np.int64)) < 0), "descending, no repeats"
    for v in a[:: 7]:
        v = int(v)
        assert is_prime(v * 2 ** 32 - 1) and is_prime(v * 2 ** 31 - 1)
    # nothing skipped between the first two entries
    first, second = int(a[0]), int(a[1])
    for v in range(second + 1, first):
        assert not (is_prime(v * 2 ** 32 - 1) and is_prime(v * 2 ** 31 - 1))
    for v in range(first + 1, 2 ** 32):
        assert not (is_prime(v * 2 ** 32 - 1) and is_prime(v * 2 ** 31 - 1))


def test_safeprimes_file_roundtrip(octmps, tmp_path):
    p = str(tmp_path / "safeprimes_base32.txt")
    octmps.write_safeprimes(p, 1000)
    a = octmps.read_safeprimes(p, 5000)
    assert len(a) == 1000
    np.testing.assert_array_equal(a, octmps.safeprimes(1000))


def test_rng_init_matches_reference_init_rng(octmps):
    kat = np.load(os.path.join(GOLDEN, "rng_kat.npz"))
    mult = kat["multipliers_head"]
    np.testing.assert_array_equal(mult, octmps.safeprimes(len(mult)))
    lanes = (len(mult) - 3) // 3
    for seed in (985456376, 1, 123456789):
        got = octmps.rng_init(mult, lanes, seed)
        for k in ("x", "a", "xR", "aR", "xS", "aS"):
            np.testing.assert_array_equal(got[k], kat[f"seed{seed}_{k}"], err_msg=f"{seed} {k}")


def test_rng_init_rejects_bad_seed_and_short_table(octmps):
    mult = octmps.safeprimes(3 + 3 * 4)
    with pytest.raises(octmps.OctmpsError):
        octmps.rng_init(mult, 4, 0)  # "not a valid seed" in init_RNG
    with pytest.raises(octmps.OctmpsError):
        octmps.rng_init(mult, 5, 1)


def decks():
    return json.load(open(os.path.join(GOLDEN, "decks.json")))


@pytest.mark.parametrize("name", ["Sphere", "FourLayers", "WangBump", "Ellipsoidand2Spheres"])
def test_parsers_match_reference(octmps, name):
    opt, _, mci = ref_deck_paths(name)
    want = decks()[name]["sim"]
    s = octmps.read_deck(opt, mci)
    for k, v in want.items():
        if k == "regions":
            got = [[s.regions[i].n, s.regions[i].mua, s.regions[i].mus, s.regions[i].g]
                   for i in range(1, s.n_regions)]
            assert [[x.hex() for x in r] for r in got] == v
        elif k == "ambient_n":
            assert s.regions[0].n.hex() == v
        else:
            g = getattr(s, k)
            assert (g.hex() if isinstance(g, float) else g) == v, k


@pytest.mark.parametrize("name", ["Sphere", "FourLayers", "WangBump", "Ellipsoidand2Spheres"])
def test_mesh_builder_matches_reference(octmps, name):
    import hashlib
    _, mesh_path, _ = ref_deck_paths(name)
    want = decks()[name]
    m = octmps.build_mesh(mesh_path)
    assert m.n_tets == want["n_tets"]
    assert m.n_distinct == want["n_distinct_faces"]
    h = hashlib.sha256()
    for a in (m.region, m.faces, m.signs, m.adj):
        h.update(np.ascontiguousarray(a).tobytes())
    assert h.hexdigest() == want["sha256_region_faces_signs_adj"]
    assert hashlib.sha256(m.planes[: m.n_distinct].tobytes()).hexdigest() == want["sha256_planes"]
    sim_start = float.fromhex(want["sim"]["start_x"])
    assert m.find_root(sim_start) == want["root_at_start_x"]


def test_mesh_builder_matches_reference_live(octmps, reference, small_deck):
    """Same check against the reference builder run now, on a generated mesh."""
    rm = reference.build_mesh(small_deck["paths"]["mesh"], (small_deck["sim"].start_x, 0, 0))
    m = small_deck["mesh"]
    for k in ("region", "faces", "signs", "adj"):
        np.testing.assert_array_equal(rm[k], getattr(m, k))
    np.testing.assert_array_equal(rm["planes"][: m.n_distinct], m.planes[: m.n_distinct])
    assert rm["root"] == small_deck["root"]


def test_root_finding_rejects_probe_off_surface(octmps, small_deck):
    with pytest.raises(octmps.OctmpsError):
        small_deck["mesh"].find_root(5.0)  # outside the box


def test_mesh_builder_errors(octmps, tmp_path):
    with pytest.raises(octmps.OctmpsError):
        octmps.build_mesh(str(tmp_path / "missing.mesh"))
    bad = tmp_path / "bad.mesh"
    bad.write_text("4\n1\n0 0 0\n1 0 0\n0 1 0\n0 0 1\n1 2 3 9 1\n")  # vertex 9 does not exist
    with pytest.raises(octmps.OctmpsError):
        octmps.build_mesh(str(bad))


def test_writers_match_reference_bytes(octmps, small_deck, tmp_path):
    ref = np.load(os.path.join(GOLDEN, "small_ref_tallies.npz"))
    t = {k[5:]: ref[k] for k in ref.files if k.startswith("run0_")}
    d = str(tmp_path)
    octmps.write_result(d, small_deck["sim"], 0.0, t)
    octmps.write_result(d, small_deck["sim"], 0.001, t)
    want = json.load(open(os.path.join(GOLDEN, "small_writer_output.json")))
    got = {fn: open(os.path.join(d, fn)).read() for fn in sorted(os.listdir(d))}
    assert sorted(got) == sorted(want)
    for fn in want:
        assert got[fn] == want[fn], fn


def test_parser_error_paths(octmps, tmp_path):
    with pytest.raises(octmps.OctmpsError):
        octmps.read_opt(str(tmp_path / "none.opt"))
    p = tmp_path / "trunc.opt"
    p.write_text("1.0\n1\nname A\n100\n")  # ends before the regions
    with pytest.raises(octmps.OctmpsError):
        octmps.read_opt(str(p))


def test_probe_positions_follow_reference_loop(octmps, small_deck):
    s = small_deck["sim"]
    s2 = type(s).from_buffer_copy(s)
    s2.start_x, s2.step_x, s2.end_x = -0.01, 0.0002, 0.01
    xs = octmps.probe_positions(s2)
    x, want = -0.01, []
    while x < 0.01:
        want.append(x)
        x += 0.0002
    assert xs == want and len(xs) in (100, 101)


def test_cli_usage_without_arguments():
    import subprocess
    exe = os.path.join(ROOT, "oct-mps_b200", "octmps")
    r = subprocess.run([exe], capture_output=True, text=True)
    assert r.returncode == 1
    assert "Usage:" in r.stdout and "-S<seed>" in r.stdout


def test_mesh_builder_matches_reference_on_the_bscan_mesh(octmps, meshgen, workdir):
    """The product's O(T) builder against the reference's own MeshGraph +
    SerializeGraph + FindRootofGraph on the benchmark's 380,928-tet B-scan
    mesh (their output cached by oracle/ref_mesh_cache.py, about two hours of
    the reference's O(T^2) face matching): every tet's region, faces, signs
    and neighbours, every distinct face plane and the root of every one of
    the 256 probe positions identical."""
    import sys
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import ref_mesh_cache
    p = meshgen.config_bscan(os.path.join(workdir, "bscan_refmesh"))
    try:
        c = ref_mesh_cache.load(p["mesh"])
    except FileNotFoundError as e:
        pytest.skip(str(e))
    m = octmps.build_mesh(p["mesh"])
    np.testing.assert_array_equal(m.region, c["tet"][:, 1])
    np.testing.assert_array_equal(m.faces, c["tet"][:, 2:6])
    np.testing.assert_array_equal(m.signs, c["tet"][:, 6:10])
    np.testing.assert_array_equal(m.adj, c["tet"][:, 10:14])
    assert m.n_distinct == len(c["planes"])
    np.testing.assert_array_equal(m.planes[: len(c["planes"])], c["planes"])
    xs = octmps.probe_positions(octmps.read_deck(p["opt"], p["mci"]))
    np.testing.assert_array_equal(np.asarray(xs), c["xs"])
    assert [m.find_root(x) for x in xs] == [int(r) for r in c["roots"]]
