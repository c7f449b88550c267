"""The allocation-free A-scan entry point against the regular job API.

octmps_ascan_run_noalloc is for callers that may not allocate device memory
(a fixed device arena, a caching allocator that owns the GPU, code where an
allocation could stall).  The caller owns every buffer; the library's
scratch lives in a fixed device array.  This file is collected last so that a
run stopping at its first failure has already run every other test; it also
passes alone in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


class NoallocAscan(C.Structure):
    _fields_ = [
        ("sim", C.c_void_p), ("planes", C.c_void_p), ("adj", C.c_void_p),
        ("n_tets", C.c_int32), ("root_tet", C.c_int32), ("root_region", C.c_int32),
        ("probe_x", C.c_double), ("probe_y", C.c_double), ("probe_z", C.c_double),
        ("n_photons", C.c_uint64), ("n_lanes", C.c_uint32),
        ("rng_x", C.c_void_p), ("rng_a", C.c_void_p), ("rng_xR", C.c_void_p),
        ("rng_aR", C.c_void_p), ("rng_xS", C.c_void_p), ("rng_aS", C.c_void_p),
        ("tally", C.c_void_p),
    ]


def r16(n):
    return (n + 15) // 16 * 16


def parse_tally(raw, nb):
    """The documented device layout of the tally block."""
    out = {}
    tot = np.frombuffer(raw[:32], np.uint64)
    out["num_filtered"], out["num_filtered_class1"], out["num_filtered_class2"] = (int(v) for v in tot[:3])
    off = 32
    for k in ("count1", "count2"):
        out[k] = np.frombuffer(raw[off:off + (nb + 1) * 8], np.uint64)
        off += r16((nb + 1) * 8)
    for k in ("sum1", "sumsq1", "sum2", "sumsq2", "max1", "max2"):
        out[k] = np.frombuffer(raw[off:off + (nb + 2) * 8], np.float64)
        off += r16((nb + 2) * 8)
    assert off == len(raw)
    return out


def noalloc_call(octmps, torch, sim, mesh, root, lanes, n, seed, mult, adj_override=None):
    """Caller-owned device buffers in the documented layouts, the argument
    block and the bound entry point.  Returns (args, buffers, function, stream)."""
    nb = sim.num_optical_depth_length_steps
    planes = (mesh.planes[mesh.faces] * mesh.signs[:, :, None]).astype(np.float32)
    adj = mesh.adj.astype(np.int64)
    adj = np.where(adj < 0, -1, adj | (mesh.region[np.maximum(adj, 0)].astype(np.int64) << 24))
    if adj_override is not None:
        adj = adj_override(adj)
    adj = adj.astype(np.uint32).view(np.int32)
    rng = octmps.rng_init(mult, lanes, seed)
    dev = {
        "planes": torch.from_numpy(np.ascontiguousarray(planes).reshape(-1)).cuda(),
        "adj": torch.from_numpy(np.ascontiguousarray(adj).reshape(-1)).cuda(),
    }
    for k in ("x", "xR", "xS"):
        dev[k] = torch.from_numpy(rng[k].view(np.int64)).cuda()
    for k in ("a", "aR", "aS"):
        dev[k] = torch.from_numpy(rng[k].view(np.int32)).cuda()
    tally_bytes = 32 + 2 * r16((nb + 1) * 8) + 6 * r16((nb + 2) * 8)
    dev["tally"] = torch.full((tally_bytes,), 0xAB, dtype=torch.uint8, device="cuda")
    torch.cuda.synchronize()

    a = NoallocAscan()
    a.sim = C.cast(C.pointer(sim), C.c_void_p)
    a.planes, a.adj = dev["planes"].data_ptr(), dev["adj"].data_ptr()
    a.n_tets, a.root_tet, a.root_region = mesh.n_tets, root, int(mesh.region[root])
    a.probe_x, a.probe_y, a.probe_z = sim.start_x, 0.0, 0.0
    a.n_photons, a.n_lanes = n, lanes
    a.rng_x, a.rng_a = dev["x"].data_ptr(), dev["a"].data_ptr()
    a.rng_xR, a.rng_aR = dev["xR"].data_ptr(), dev["aR"].data_ptr()
    a.rng_xS, a.rng_aS = dev["xS"].data_ptr(), dev["aS"].data_ptr()
    a.tally = dev["tally"].data_ptr()

    f = octmps.lib().octmps_ascan_run_noalloc
    f.restype = C.c_int
    f.argtypes = [C.POINTER(NoallocAscan), C.c_void_p]
    return a, dev, f, torch.cuda.current_stream().cuda_stream


def test_noalloc_entry_point_matches_job_api(octmps, small_deck):
    torch = pytest.importorskip("torch")
    assert torch.cuda.is_available()
    sim, mesh, root = small_deck["sim"], small_deck["mesh"], small_deck["root"]
    nb = sim.num_optical_depth_length_steps
    lanes, n, seed = 2000, 20000, 5
    mult = octmps.safeprimes(3 + 3 * lanes)

    # the existing entry point
    with octmps.Context(0, mult) as ctx:
        mid = ctx.upload_mesh(mesh)
        jid = ctx.submit(mid, sim, sim.start_x, root, n_photons=n, seed=seed, n_lanes=lanes)
        want = ctx.fetch(jid, nb)
        ctx.release(jid)

    a, dev, f, stream = noalloc_call(octmps, torch, sim, mesh, root, lanes, n, seed, mult)
    for call in range(2):  # the scratch keeps the previous call's contents
        st = f(C.byref(a), C.c_void_p(stream))
        assert st == 0, (st, octmps.STATUS.get(st))
        torch.cuda.synchronize()
        got = parse_tally(dev["tally"].cpu().numpy().tobytes(), nb)
        for k in ("num_filtered", "num_filtered_class1", "num_filtered_class2"):
            assert got[k] == want[k], (call, k)
        for k in ("count1", "count2"):
            np.testing.assert_array_equal(got[k], want[k], err_msg=f"call {call} {k}")
        for k in ("sum1", "sumsq1", "sum2", "sumsq2"):
            np.testing.assert_allclose(got[k][:nb], want[k][:nb], rtol=1e-12, atol=0,
                                       err_msg=f"call {call} {k}")
        for k in ("max1", "max2"):
            np.testing.assert_array_equal(got[k][:nb], want[k][:nb], err_msg=f"call {call} {k}")

    # more regions than the fixed scratch holds: rejected, nothing launched
    big = type(sim).from_buffer_copy(sim)
    big.n_regions = 101
    a.sim = C.cast(C.pointer(big), C.c_void_p)
    assert f(C.byref(a), C.c_void_p(stream)) == 1


def test_noalloc_bad_neighbour_entries_are_reported(octmps, small_deck):
    """The caller's neighbour array is checked on the device before any
    photon follows it.  Both cases keep every access in bounds even without
    the check (a region below the fixed table's 100 entries; arrays allocated
    for the whole mesh while n_tets claims half of it), so the test shows the
    report, not a fault."""
    torch = pytest.importorskip("torch")
    assert torch.cuda.is_available()
    sim, mesh, root = small_deck["sim"], small_deck["mesh"], small_deck["root"]
    lanes, n, seed = 500, 1000, 9
    mult = octmps.safeprimes(3 + 3 * lanes)
    bad_region = sim.n_regions  # one past the job's regions
    a, dev, f, stream = noalloc_call(
        octmps, torch, sim, mesh, root, lanes, n, seed, mult,
        adj_override=lambda adj: np.where(adj < 0, -1, (adj & 0xFFFFFF) | (bad_region << 24)))
    assert f(C.byref(a), C.c_void_p(stream)) == 1  # OCTMPS_ERR_INVALID_ARG
    a, dev, f, stream = noalloc_call(octmps, torch, sim, mesh, root, lanes, n, seed, mult)
    assert root < mesh.n_tets // 2
    a.n_tets = mesh.n_tets // 2  # neighbours in the second half are out of range
    assert f(C.byref(a), C.c_void_p(stream)) == 1
    a.n_tets = mesh.n_tets  # the next call starts clean
    assert f(C.byref(a), C.c_void_p(stream)) == 0
