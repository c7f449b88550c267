"""B-scans over several GPUs: one rank per GPU, A-scans partitioned, no data exchange.

The reference splits the photons of every A-scan over its GPUs and sums the
per-GPU tallies on the host (src/main.cu:692-793), relaunching the whole
set-up for each A-scan (src/main.cu:948-1051).  Here each rank takes every
world-th A-scan of the scan (k = rank, rank + world, ...), runs all of them in
one persistent launch on its GPU, and rank 0 gathers the finished tallies and
writes the reference's output files in scan order.  The only communication is
the final gather of a few tens of KB per A-scan; there is no collective on the
data path.

Launch with torchrun (one process per GPU, MASTER_ADDR=127.0.0.1) or call
run_bscan() directly with world=1.
"""
import os

import octmps


def my_ascans(n_ascans, world, rank):
    """A-scan indices owned by `rank`: round robin, so neighbouring probe
    positions (similar cost) spread over the GPUs."""
    return list(range(rank, n_ascans, world))


def gpu_runner(ctx, mesh_id, sim, seed=985456376, seed_per_ascan=False, n_lanes=0,
               precision=octmps.PREC_MIXED):
    """A runner for run_bscan: submits a rank's A-scans to one context, runs
    them in one launch, returns {k: tally}."""
    nb = sim.num_optical_depth_length_steps

    def run(items):
        ids = {k: ctx.submit(mesh_id, sim, x, root, seed=seed + (k if seed_per_ascan else 0),
                             n_lanes=n_lanes, precision=precision)
               for k, x, root in items}
        ctx.flush()
        out = {}
        for k, j in ids.items():
            out[k] = ctx.fetch(j, nb)
            ctx.release(j)
        return out

    return run


def run_bscan(sim, mesh, runner, world=1, rank=0, dist=None, out_dir=None):
    """Runs the scan's A-scans owned by this rank with `runner` (a function
    taking [(k, x, root_tet)] and returning {k: tally dict}), gathers all
    tallies on rank 0 and, if out_dir is given, writes the reference's output
    files there in scan order.  Returns the list of tallies in scan order on
    rank 0 (None on other ranks)."""
    xs = octmps.probe_positions(sim)
    mine = [(k, xs[k], mesh.find_root(xs[k])) for k in my_ascans(len(xs), world, rank)]
    results = runner(mine) if mine else {}
    if dist is not None and world > 1:
        gathered = [None] * world if rank == 0 else None
        dist.gather_object(results, gathered, dst=0)
    else:
        gathered = [results]
    if rank != 0:
        return None
    merged = {}
    for part in gathered:
        merged.update(part)
    missing = [k for k in range(len(xs)) if k not in merged]
    if missing:
        raise RuntimeError(f"A-scans missing after the gather: {missing[:8]}")
    ordered = [merged[k] for k in range(len(xs))]
    if out_dir is not None:
        os.makedirs(out_dir, exist_ok=True)
        for k, t in enumerate(ordered):
            octmps.write_result(out_dir, sim, xs[k], t)
    return ordered
