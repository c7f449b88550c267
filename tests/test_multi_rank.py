"""Multi-GPU B-scan host logic with two gloo ranks on CPU.

Each rank runs its share of the A-scans (here through the CPU oracle standing
in for a GPU) and rank 0 gathers and writes the output files; the files must be
byte-identical to a single-rank run, every A-scan present exactly once."""
import os
import socket
import sys

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from conftest import ROOT


def free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def oracle_runner(sim, mesh, seeds_used):
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import octmps
    import oracle_py
    O = oracle_py.Oracle()
    p = oracle_py.params_from_sim(sim)
    lanes = 200
    mult = octmps.safeprimes(3 + 3 * lanes)

    def run(items):
        out = {}
        for k, x, root in items:
            rng = octmps.rng_init(mult, lanes, 1000 + k)
            t = O.run(p, mesh, (x, 0.0, 0.0), root, 1000, lanes, rng, 0, n_threads=1)
            out[k] = {key: t[key] for key in t}
            seeds_used.append(k)
        return out

    return run


def scan_deck(tmp, octmps, meshgen):
    p = meshgen.config_small(tmp, n_photons=1000)
    sim = octmps.read_deck(p["opt"], p["mci"])
    sim.start_x, sim.step_x, sim.end_x = -0.02, 0.005, 0.0205  # 9 A-scans
    return sim, octmps.build_mesh(p["mesh"])


def worker(rank, world, port, tmp, result_dir):
    sys.path.insert(0, os.path.join(ROOT, "oct-mps_b200"))
    import bscan
    import meshgen
    import octmps
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        sim, mesh = scan_deck(os.path.join(tmp, f"deck{rank}"), octmps, meshgen)
        done = []
        bscan.run_bscan(sim, mesh, oracle_runner(sim, mesh, done), world, rank, dist,
                        out_dir=result_dir if rank == 0 else None)
        with open(os.path.join(tmp, f"done{rank}.txt"), "w") as f:
            f.write(",".join(map(str, done)))
    finally:
        dist.barrier()
        dist.destroy_process_group()


def test_two_rank_bscan_equals_single_rank(tmp_path, octmps, meshgen):
    sys.path.insert(0, os.path.join(ROOT, "oct-mps_b200"))
    import bscan
    single = tmp_path / "single"
    sim, mesh = scan_deck(str(tmp_path / "deck"), octmps, meshgen)
    done = []
    bscan.run_bscan(sim, mesh, oracle_runner(sim, mesh, done), out_dir=str(single))
    assert sorted(done) == list(range(9))

    multi = tmp_path / "multi"
    mp.spawn(worker, args=(2, free_port(), str(tmp_path), str(multi)), nprocs=2, join=True)
    d0 = [int(v) for v in open(tmp_path / "done0.txt").read().split(",")]
    d1 = [int(v) for v in open(tmp_path / "done1.txt").read().split(",")]
    assert d0 == [0, 2, 4, 6, 8] and d1 == [1, 3, 5, 7]
    for fn in sorted(os.listdir(single)):
        assert (multi / fn).read_bytes() == (single / fn).read_bytes(), fn


def test_partition_covers_every_ascan_once():
    sys.path.insert(0, os.path.join(ROOT, "oct-mps_b200"))
    import bscan
    for n in (1, 7, 256):
        for world in (1, 2, 3, 8):
            parts = [bscan.my_ascans(n, world, r) for r in range(world)]
            flat = sorted(k for p in parts for k in p)
            assert flat == list(range(n))
            assert max(map(len, parts)) - min(map(len, parts)) <= 1


def test_cli_gpu_split_matches_the_rank_split(octmps):
    """The CLI's -G split of A-scans over GPUs (octmps_ascans_of_gpu, which
    csrc/main.cpp calls per GPU thread) is the multi-rank driver's split:
    every A-scan exactly once, round robin, sizes within one."""
    sys.path.insert(0, os.path.join(ROOT, "oct-mps_b200"))
    import bscan
    for n in (0, 1, 5, 256, 1000):
        for g in (1, 2, 3, 4, 8):
            parts = [octmps.ascans_of_gpu(n, g, r) for r in range(g)]
            assert parts == [bscan.my_ascans(n, g, r) for r in range(g)]
            assert sorted(k for p in parts for k in p) == list(range(n))
    for bad in ((10, 0, 0), (10, 2, 2)):
        with pytest.raises(octmps.OctmpsError):
            octmps.ascans_of_gpu(*bad)

