"""The serving loop: A-scan and B-scan requests that arrive while others run
(continuous batching into running launches, two meshes resident) give the
same tallies as each of their A-scans run alone."""
import time

import pytest

from test_gpu_kernel import assert_tallies_equal

pytestmark = pytest.mark.gpu


def test_served_requests_match_alone(octmps, multipliers, small_deck, small_matched_deck):
    import serve

    nb = small_deck["sim"].num_optical_depth_length_steps
    assert small_matched_deck["sim"].num_optical_depth_length_steps == nb
    with octmps.Context(0, multipliers) as ctx:
        meshes = {}
        for key, d in (("plain", small_deck), ("matched", small_matched_deck)):
            meshes[key] = {"sim": d["sim"], "mesh": d["mesh"], "roots": {},
                           "id": ctx.upload_mesh(d["mesh"])}
        reqs = [
            # 400 packets in a row on each of 1000 lanes: runs a few seconds
            serve.Request(0, "ascan", "plain", [0.0], 400_000, 11, lanes=1000),
            serve.Request(1, "bscan", "matched", [-0.0004, -0.0002, 0.0, 0.0002], 20_000, 21),
            serve.Request(2, "ascan", "matched", [0.0001], 5_000, 31),
            serve.Request(3, "bscan", "plain", [-0.0003, 0.0003], 40_000, 41),
            serve.Request(4, "ascan", "plain", [0.0002], 1_000, 51),
        ]
        alone = {}
        for r in reqs:
            m = meshes[r.mesh_key]
            for k, x in enumerate(r.xs):
                root = m["mesh"].find_root(x)
                j = ctx.submit(m["id"], m["sim"], x, root, n_photons=r.photons, seed=r.seed + k,
                               n_lanes=serve.lanes_for(r))
                alone[(r.rid, k)] = ctx.fetch(j, nb)
                ctx.release(j)
        srv = serve.Server(ctx, meshes)
        for r in reqs:  # the first request is still running when the others arrive
            srv.submit(r)
            time.sleep(0.003)
        assert srv.drain(300)
        srv.close()
        assert not srv.errors, srv.errors
        for r in reqs:
            assert r.t_done is not None
            for k in range(len(r.xs)):
                assert_tallies_equal(r.results[k], alone[(r.rid, k)], 0, nb)
        # a later request finished before the first, long one did
        assert min(r.t_done for r in reqs[1:]) < reqs[0].t_done
