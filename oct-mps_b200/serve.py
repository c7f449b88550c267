"""Serving loop: A-scan and B-scan requests against resident meshes.

Requests (an A-scan: one probe position; a B-scan: several) arrive while
others run.  The admitter submits each request's jobs to the context as soon
as the HBM budget allows (a refused submit waits for finished requests to
release memory); the context appends them to the running persistent launch,
whose threads take them up as they free up, so their work overlaps the work
already on the GPU (continuous batching).  A collector thread takes finished
jobs off the context's completion queue, fetches and releases them, and
records each request's latency (arrival to last A-scan fetched).  Throughput
(packets/s) and p50/p99 latency per request type are reported.

    python serve.py [--loads 0.5,0.9,1.2] [--requests 24] [--scale small|full]
    python bench.py --serve          (the full study, recorded as a bench line)
"""
import argparse
import json
import os
import queue
import tempfile
import threading
import time

import numpy as np

import octmps


class Request:
    def __init__(self, rid, kind, mesh_key, xs, photons, seed, lanes=0):
        self.rid, self.kind, self.mesh_key = rid, kind, mesh_key
        self.xs, self.photons, self.seed = xs, photons, seed
        self.lanes = lanes    # RNG lanes per A-scan (0: Server.lanes_for's choice)
        self.t_arrival = None
        self.t_admitted = None
        self.t_done = None
        self.jobs = []        # (job id, k)
        self.results = {}     # k -> tally
        self.launch_ids = set()


def lanes_for(req, max_lanes=88800):
    """RNG lanes of each of a request's A-scans: about 8 packets per lane.
    A lane runs its packets one after another, so a job's latency on an
    otherwise idle GPU grows with its packets per lane; many short lanes also
    spread one large job over every SM."""
    return req.lanes or int(min(max_lanes, max(1, req.photons // 8)))


class Server:
    """Admission + completion around one context (one GPU)."""

    def __init__(self, ctx, meshes, poll_s=0.0005, max_lanes=88800):
        self.ctx = ctx
        self.max_lanes = max_lanes  # the context's multiplier table covers this many lanes
        self.meshes = meshes  # key -> dict(id=mesh id, sim=Sim, mesh=Mesh, roots=dict x->root)
        self.incoming = queue.Queue()
        self.inflight = 0
        self.owner = {}       # job id -> (request, k)
        self.done = []
        self.lock = threading.Lock()
        self.stop = False
        self.poll_s = poll_s
        self.packets_done = 0
        self.errors = []
        self.t_admit = threading.Thread(target=self._admit, daemon=True)
        self.t_collect = threading.Thread(target=self._collect, daemon=True)
        self.t_admit.start()
        self.t_collect.start()

    def root(self, key, x):
        m = self.meshes[key]
        if x not in m["roots"]:
            m["roots"][x] = m["mesh"].find_root(x)
        return m["roots"][x]

    def lanes_for(self, req):
        return lanes_for(req, self.max_lanes)

    def submit(self, req):
        req.t_arrival = time.perf_counter()
        with self.lock:
            self.inflight += 1
        self.incoming.put(req)

    def _admit(self):
        pending = None
        while not self.stop:
            if pending is None:
                try:
                    pending = self.incoming.get(timeout=0.01)
                except queue.Empty:
                    continue
            m = self.meshes[pending.mesh_key]
            try:
                while len(pending.jobs) < len(pending.xs):
                    k = len(pending.jobs)
                    x = pending.xs[k]
                    j = self.ctx.submit(m["id"], m["sim"], x, self.root(pending.mesh_key, x),
                                        n_photons=pending.photons, seed=pending.seed + k,
                                        n_lanes=self.lanes_for(pending))
                    pending.jobs.append((j, k))
                    with self.lock:
                        self.owner[j] = (pending, k)
                self.ctx.flush()
                pending.t_admitted = time.perf_counter()
                pending = None
            except octmps.OctmpsError as e:
                if e.status == 8:  # HBM budget: wait for finished requests
                    time.sleep(0.002)
                else:  # the request fails; its jobs already submitted still drain
                    self.errors.append(str(e))
                    pending.t_done = time.perf_counter()
                    with self.lock:
                        self.inflight -= 1
                    pending = None

    def _collect(self):
        """Takes finished jobs off the context's completion queue, fetches and
        releases them; a request is done when all of its A-scans are."""
        unowned = []
        while not self.stop:
            try:
                ids = unowned + self.ctx.poll()
            except octmps.OctmpsError as e:
                self.errors.append(str(e))
                time.sleep(0.01)
                continue
            unowned = []
            for j in ids:
                with self.lock:
                    own = self.owner.pop(j, None)
                if own is None:  # finished before its submitter recorded it
                    unowned.append(j)
                    continue
                req, k = own
                nb = self.meshes[req.mesh_key]["sim"].num_optical_depth_length_steps
                st = self.ctx.wait(j, 0)
                if st != 0:
                    self.errors.append(f"job {j}: status {st}: {self.ctx.last_error()}")
                try:
                    req.results[k] = self.ctx.fetch(j, nb) if st == 0 else None
                    s = self.ctx.stats(j)
                    req.launch_ids.add(s["launch_id"])
                    self.packets_done += s["packets"]
                except octmps.OctmpsError as e:
                    self.errors.append(str(e))
                    req.results[k] = None
                self.ctx.release(j)
                if len(req.results) == len(req.xs) and req.t_done is None:
                    req.t_done = time.perf_counter()
                    with self.lock:
                        self.inflight -= 1
                        self.done.append(req)
            if not ids:
                time.sleep(self.poll_s)

    def drain(self, timeout_s=3600):
        t0 = time.perf_counter()
        while time.perf_counter() - t0 < timeout_s:
            with self.lock:
                busy = self.inflight > 0
            if not busy:
                return True
            time.sleep(0.01)
        return False

    def close(self):
        self.stop = True
        self.t_admit.join(5)
        self.t_collect.join(5)


def latency_stats(reqs):
    out = {}
    for kind in sorted({r.kind for r in reqs}):
        lat = np.array([(r.t_done - r.t_arrival) * 1e3 for r in reqs if r.kind == kind])
        out[kind] = {"n": int(len(lat)), "p50_ms": float(np.percentile(lat, 50)),
                     "p99_ms": float(np.percentile(lat, 99)), "mean_ms": float(lat.mean())}
    return out


def overlapping(reqs):
    """Requests whose time on the GPU (admission to completion) overlapped
    another request's."""
    n = 0
    for r in reqs:
        n += any(o is not r and o.t_admitted < r.t_done and r.t_admitted < o.t_done for o in reqs)
    return n


def build_meshes(scale, workdir):
    """The four resident meshes of the served-stream configuration: a small
    one (~50k tets), the B-scan mesh (~381k), a four-layer slab (~1M) and the
    plain-A-scan geometry on a finer grid (~2M).  scale='small' shrinks every
    grid for a quick run."""
    import meshgen
    f = 1.0 if scale == "full" else 0.35
    g = lambda n: max(4, int(round(n * f)))  # noqa: E731
    specs = {
        "m50k": lambda d: meshgen.config_plain_ascan(d, nx=g(21), ny=g(21), nz=g(19)),
        "m400k": lambda d: meshgen.config_bscan(d, nx=g(64), ny=g(32), nz=g(31)),
        "m1M": lambda d: meshgen.config_layers(d, nx=g(60), ny=g(60), nz=g(46)),
        "m2M": lambda d: meshgen.config_plain_ascan(d, nx=g(70), ny=g(70), nz=g(68)),
    }
    out = {}
    for key, make in specs.items():
        p = make(os.path.join(workdir, key))
        sim = octmps.read_deck(p["opt"], p["mci"])
        out[key] = {"sim": sim, "mesh": octmps.build_mesh(p["mesh"]), "roots": {},
                    "n_tets": p["n_tets"]}
    return out


def make_stream(meshes, n_req, rate_hz, rng, photon_scale=1.0):
    """Poisson arrivals; A-scan : B-scan = 3 : 1; A-scans 1e5-1e7 packets
    (log-uniform), B-scans 32-128 A-scans x 1e5 packets (times photon_scale)."""
    keys = sorted(meshes)
    t, reqs = 0.0, []
    for rid in range(n_req):
        t += rng.exponential(1.0 / rate_hz)
        key = keys[rng.integers(len(keys))]
        span = 0.002
        if rng.random() < 0.75:
            x = float(rng.uniform(-span, span))
            n = int(10 ** rng.uniform(5, 7) * photon_scale)
            reqs.append((t, Request(rid, "ascan", key, [x], max(1000, n), 1 + 1000 * rid)))
        else:
            na = int(rng.integers(32, 129))
            x0 = float(rng.uniform(-span, span))
            xs = [x0 + 1e-4 * (k - na / 2) for k in range(na)]
            reqs.append((t, Request(rid, "bscan", key, xs, max(1000, int(1e5 * photon_scale)),
                                    1 + 1000 * rid)))
    return reqs


def run_stream(server, reqs, speed=1.0):
    t0 = time.perf_counter()
    for t, req in reqs:
        delay = t / speed - (time.perf_counter() - t0)
        if delay > 0:
            time.sleep(delay)
        server.submit(req)
    server.drain()
    return time.perf_counter() - t0


def serve_levels(ctx, meshes, loads, n_requests, photon_scale=1.0, max_lanes=1 << 18,
                 n_calibration=None, log=None):
    """The served-stream study: capacity, then each offered load.

    Capacity is measured on a Poisson stream, not with every request queued
    at once: a first estimate c0 comes from a queued batch of
    n_calibration requests; a Poisson stream offered at 1.5 x c0 then runs
    n_requests requests, and its sustained throughput (packets completed /
    time from the first arrival to the last completion) is the capacity.
    Each load level then offers load x capacity in Poisson arrivals
    (seeded streams) of n_requests requests; throughput, p50/p99 latency per
    request type and how many requests overlapped another on the GPU are
    reported."""
    n_cal = n_calibration or max(8, n_requests // 8)
    cal = make_stream(meshes, n_cal, 1e9, np.random.default_rng(55), photon_scale)
    srv = Server(ctx, meshes, max_lanes=max_lanes)
    wall = run_stream(srv, cal)
    c0 = srv.packets_done / wall
    per_req0 = srv.packets_done / len(cal)
    srv.close()
    sat = make_stream(meshes, n_requests, 1.5 * c0 / per_req0, np.random.default_rng(56),
                      photon_scale)
    srv = Server(ctx, meshes, max_lanes=max_lanes)
    wall = run_stream(srv, sat)
    srv.close()
    capacity = srv.packets_done / wall
    work_per_req = srv.packets_done / len(sat)
    out = {"queued_estimate_packets_per_s": c0, "capacity_packets_per_s": capacity,
           "capacity_stream": {"requests": len(sat), "offered_packets_per_s": 1.5 * c0,
                               "wall_s": wall, "latency": latency_stats([r for _, r in sat])},
           "mean_packets_per_request": work_per_req, "levels": [], "errors": srv.errors[:3]}
    if log:
        log(out)
    rng = np.random.default_rng(5)
    for load in loads:
        rate = load * capacity / work_per_req
        reqs = make_stream(meshes, n_requests, rate, rng, photon_scale)
        srv = Server(ctx, meshes, max_lanes=max_lanes)
        wall = run_stream(srv, reqs)
        srv.close()
        done = [r for _, r in reqs]
        lvl = {"offered_load": load, "arrival_rate_hz": rate, "requests": len(done),
               "wall_s": wall, "throughput_packets_per_s": srv.packets_done / wall,
               "offered_packets_per_s": rate * work_per_req, "latency": latency_stats(done),
               "errors": srv.errors[:3], "requests_overlapping_another": overlapping(done)}
        out["levels"].append(lvl)
        if log:
            log(lvl)
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--loads", default="0.5,0.9,1.2")
    ap.add_argument("--requests", type=int, default=24)
    ap.add_argument("--scale", default="small", choices=["small", "full"])
    ap.add_argument("--photon-scale", type=float, default=0.1)
    ap.add_argument("--device", type=int, default=0)
    args = ap.parse_args()
    work = tempfile.mkdtemp(prefix="octmps_serve_")
    meshes = build_meshes(args.scale, work)
    max_lanes = 1 << 18
    mult = octmps.safeprimes(3 + 3 * max_lanes)
    rng = np.random.default_rng(5)
    with octmps.Context(args.device, mult) as ctx:
        for m in meshes.values():
            m["id"] = ctx.upload_mesh(m["mesh"])
        serve_levels(ctx, meshes, [float(v) for v in args.loads.split(",")], args.requests,
                     args.photon_scale, max_lanes,
                     log=lambda d: print(json.dumps(d), flush=True))

if __name__ == "__main__":
    main()
