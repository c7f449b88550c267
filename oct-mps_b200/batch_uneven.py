"""Batched uneven jobs: many different meshes and job sizes in one launch.

64 jobs drawn from numpy.random.default_rng(4): the 2 x 2 x 1.5 mm box with
1-4 ellipsoid inclusions, each job its own mesh of 50k-800k tets, packets
log-uniform in 1e4-1e7, seed = job index + 1.  Every mesh is uploaded once;
the jobs then run (a) all submitted together into one job table (batched),
and (b) one at a time, each its own launch (plain).  Both report device time
(CUDA events around the launches) and packets/s; the tallies of the two runs
are checked to be the same job by job (counts exact, sums to summation
order).

    python batch_uneven.py [--jobs 64] [--precision 0]
"""
import argparse
import json
import os
import tempfile
import time

import numpy as np

import octmps


def build_jobs(n_jobs, workdir):
    import meshgen
    rng = np.random.default_rng(4)
    jobs = []
    for i in range(n_jobs):
        p = meshgen.config_random_job(os.path.join(workdir, f"job{i}"), rng, i)
        sim = octmps.read_deck(p["opt"], p["mci"])
        mesh = octmps.build_mesh(p["mesh"])
        x = octmps.probe_positions(sim)[0]
        jobs.append({"sim": sim, "mesh": mesh, "x": x, "root": mesh.find_root(x),
                     "photons": sim.number_of_photons, "seed": i + 1, "tets": p["n_tets"]})
    return jobs


def run(ctx, jobs, precision=0):
    """Uploads every job's mesh, runs the jobs (a) batched into one job table
    and (b) one launch per job, checks the tallies agree job by job, and
    returns the figures (device time by CUDA events around the launches)."""
    total = sum(j["photons"] for j in jobs)
    for j in jobs:
        j["mid"] = ctx.upload_mesh(j["mesh"])

    def submit(j):
        return ctx.submit(j["mid"], j["sim"], j["x"], j["root"], n_photons=j["photons"],
                          seed=j["seed"], precision=precision)

    def fetch(j, jid):
        return ctx.fetch(jid, j["sim"].num_optical_depth_length_steps)

    # batched: one table, launches overlap every job
    t0 = time.perf_counter()
    ids = [submit(j) for j in jobs]
    ctx.flush()
    batched = [fetch(j, jid) for j, jid in zip(jobs, ids)]
    ctx.synchronize()
    wall_b = time.perf_counter() - t0
    launches = {}
    steps_b = stopped = 0
    for jid in ids:
        s = ctx.stats(jid)
        launches[s["launch_id"]] = s["device_ms"]
        steps_b += s["steps"]
        stopped += s["stopped"]
        ctx.release(jid)
    dev_b = sum(launches.values()) / 1e3
    # plain: one job per launch
    dev_p = 0.0
    t0 = time.perf_counter()
    same = True
    for j, tb in zip(jobs, batched):
        jid = submit(j)
        ctx.flush()
        tp = fetch(j, jid)
        ctx.synchronize()
        dev_p += ctx.stats(jid)["device_ms"] / 1e3
        ctx.release(jid)
        nb = j["sim"].num_optical_depth_length_steps
        same &= all(tp[k] == tb[k] for k in ("num_filtered", "num_filtered_class1",
                                             "num_filtered_class2"))
        same &= bool(np.array_equal(tp["count1"], tb["count1"]))
        same &= bool(np.allclose(tp["sum1"][:nb], tb["sum1"][:nb], rtol=1e-12, atol=0))
    wall_p = time.perf_counter() - t0
    for j in jobs:
        ctx.release_mesh(j["mid"])
    return {
        "workload": f"{len(jobs)} jobs, {min(j['tets'] for j in jobs)}-"
                    f"{max(j['tets'] for j in jobs)} tets, {min(j['photons'] for j in jobs)}-"
                    f"{max(j['photons'] for j in jobs)} packets each, {total} packets in all",
        "batched": {"device_s": dev_b, "wall_s": wall_b, "launches": len(launches),
                    "packets_per_s": total / dev_b, "steps": steps_b, "stopped": stopped},
        "plain": {"device_s": dev_p, "wall_s": wall_p, "packets_per_s": total / dev_p},
        "batched_over_plain": dev_p / dev_b,
        "tallies_equal_job_by_job": bool(same),
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--jobs", type=int, default=64)
    ap.add_argument("--precision", type=int, default=0)
    ap.add_argument("--device", type=int, default=0)
    args = ap.parse_args()
    work = tempfile.mkdtemp(prefix="octmps_uneven_")
    t0 = time.perf_counter()
    jobs = build_jobs(args.jobs, work)
    t_build = time.perf_counter() - t0
    mult = octmps.safeprimes(3 + 3 * 88800)
    with octmps.Context(args.device, mult) as ctx:
        out = run(ctx, jobs, args.precision)
    out["host_mesh_build_s"] = t_build
    print(json.dumps(out, indent=1))


if __name__ == "__main__":
    main()
