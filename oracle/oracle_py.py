"""ctypes wrapper of the CPU oracle and of the reference's host build.

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline leg, never by the product.

* ``Oracle`` wraps _build/liboctmps_oracle.so, the restatement of the
  per-photon method in oracle.cpp (three precisions).
* ``Reference`` wraps _ref/libocref.so, the reference's own routine
  (src/octmps_kernel.cuh), parsers, mesh builder and writers, compiled for
  the host by oracle/Makefile through the shim in ref_host/.
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "_build", "liboctmps_oracle.so")
CENSUS_SO = os.path.join(HERE, "_build", "liboctmps_census.so")
CENSUS_FIELDS = ("add", "mul", "div", "sqrt", "fma", "trans")
REF_SO = os.path.join(HERE, "_ref", "libocref.so")
# the same sources built -O3 -march=x86-64-v4 with contraction: the timed CPU baseline
REF_FAST_SO = os.path.join(HERE, "_ref", "libocref_fast.so")
# the same sources with log and sincos routed to the oracle's series
REF_METHOD_SO = os.path.join(HERE, "_ref", "libocref_method.so")
MAX_REGIONS = 100

P = C.POINTER


class OracleParams(C.Structure):
    _fields_ = [
        ("n_regions", C.c_int32),
        ("region_n", C.c_double * MAX_REGIONS), ("region_mua", C.c_double * MAX_REGIONS),
        ("region_mus", C.c_double * MAX_REGIONS), ("region_g", C.c_double * MAX_REGIONS),
        ("type_bias", C.c_int32), ("nbins", C.c_int32),
        ("target_depth_min", C.c_double), ("target_depth_max", C.c_double),
        ("backward_bias_coefficient", C.c_double),
        ("max_collecting_angle_deg", C.c_double), ("max_collecting_radius", C.c_double),
        ("probability_additional_bias", C.c_double),
        ("optical_depth_shift", C.c_double), ("coherence_length_source", C.c_double),
        ("rnd_step_size_in_tissue", C.c_double),
    ]


class OracleMesh(C.Structure):
    _fields_ = [
        ("n_tets", C.c_int32), ("n_faces", C.c_int32),
        ("region", P(C.c_int32)), ("faces", P(C.c_int32)), ("signs", P(C.c_int32)),
        ("adj", P(C.c_int32)), ("planes", P(C.c_double)),
    ]


class OracleTally(C.Structure):
    _fields_ = [
        ("num_filtered", C.c_uint64), ("num_filtered_class1", C.c_uint64),
        ("num_filtered_class2", C.c_uint64),
        ("count1", P(C.c_uint64)), ("count2", P(C.c_uint64)),
        ("sum1", P(C.c_double)), ("max1", P(C.c_double)), ("sumsq1", P(C.c_double)),
        ("sum2", P(C.c_double)), ("max2", P(C.c_double)), ("sumsq2", P(C.c_double)),
        ("steps", C.c_uint64), ("restores", C.c_uint64), ("packets", C.c_uint64),
        ("capped", C.c_uint64),
    ]


# One detected packet (RecordPhotonsFlag), as OraclePhotonRecord and the
# library's octmps_photon_record.
RECORD_DTYPE = np.dtype([
    ("weight", np.float64), ("likelihood", np.float64), ("radius", np.float64),
    ("cos_angle", np.float64), ("optical_path", np.float64), ("max_depth", np.float64),
])

PACKET_DTYPE = np.dtype([
    ("hash", np.uint64), ("x", np.uint64), ("xR", np.uint64), ("xS", np.uint64),
    ("steps", np.uint32), ("hits", np.uint32), ("scatters", np.uint32),
    ("restores", np.uint32), ("detections", np.uint32), ("survivals", np.uint32),
    ("contribution", np.float64), ("optical_path", np.float64),
])
assert PACKET_DTYPE.itemsize == 72


class RefSim(C.Structure):
    _fields_ = [
        ("start_x", C.c_double), ("step_x", C.c_double), ("end_x", C.c_double),
        ("number_of_photons", C.c_uint32), ("n_regions", C.c_int32),
        ("region_n", C.c_double * MAX_REGIONS), ("region_mua", C.c_double * MAX_REGIONS),
        ("region_mus", C.c_double * MAX_REGIONS), ("region_g", C.c_double * MAX_REGIONS),
        ("region_mutr", C.c_double * MAX_REGIONS),
        ("type_simulation", C.c_int32), ("type_bias", C.c_int32),
        ("record_photons_flag", C.c_int32), ("num_optical_depth_length_steps", C.c_int32),
        ("backward_bias_coefficient", C.c_double), ("target_depth_min", C.c_double),
        ("target_depth_max", C.c_double), ("coherence_length_source", C.c_double),
        ("max_collecting_radius", C.c_double), ("max_collecting_angle_deg", C.c_double),
        ("probability_additional_bias", C.c_double), ("max_relative_contribution", C.c_double),
        ("max_filtered_optical_depth", C.c_double), ("optical_depth_shift", C.c_double),
        ("rnd_step_size_in_tissue", C.c_double),
    ]


class RefMesh(C.Structure):
    _fields_ = [("n_tets", C.c_int32), ("n_faces", C.c_int32), ("root", C.c_int32),
                ("tet", P(C.c_int32)), ("face", P(C.c_double))]


class RefTally(C.Structure):
    _fields_ = [
        ("num_filtered", C.c_uint64), ("num_filtered_class1", C.c_uint64),
        ("num_filtered_class2", C.c_uint64),
        ("count1", P(C.c_uint64)), ("count2", P(C.c_uint64)),
        ("sum1", P(C.c_double)), ("max1", P(C.c_double)), ("sumsq1", P(C.c_double)),
        ("sum2", P(C.c_double)), ("max2", P(C.c_double)), ("sumsq2", P(C.c_double)),
    ]


def _ptr(a, ct):
    return a.ctypes.data_as(P(ct))


def empty_tally(nbins):
    t = {"count1": np.zeros(nbins + 1, np.uint64), "count2": np.zeros(nbins + 1, np.uint64)}
    for k in ("sum1", "max1", "sumsq1", "sum2", "max2", "sumsq2"):
        t[k] = np.zeros(nbins + 2, np.float64)
    return t


def _fill_tally_struct(cls, t):
    s = cls()
    for k in ("count1", "count2"):
        setattr(s, k, _ptr(t[k], C.c_uint64))
    for k in ("sum1", "max1", "sumsq1", "sum2", "max2", "sumsq2"):
        setattr(s, k, _ptr(t[k], C.c_double))
    return s


def params_from_sim(sim):
    """OracleParams from a product octmps.Sim (or any object with its fields)."""
    p = OracleParams()
    p.n_regions = sim.n_regions
    for i in range(sim.n_regions):
        r = sim.regions[i]
        p.region_n[i], p.region_mua[i], p.region_mus[i], p.region_g[i] = r.n, r.mua, r.mus, r.g
    p.type_bias = sim.type_bias
    p.nbins = sim.num_optical_depth_length_steps
    for k in ("target_depth_min", "target_depth_max", "backward_bias_coefficient",
              "max_collecting_angle_deg", "max_collecting_radius", "probability_additional_bias",
              "optical_depth_shift", "coherence_length_source", "rnd_step_size_in_tissue"):
        setattr(p, k, getattr(sim, k))
    return p


class Oracle:
    def __init__(self, path=ORACLE_SO):
        if not os.path.exists(path):
            raise ImportError(f"{path} not built; run make in {HERE}")
        L = C.CDLL(path)
        L.oracle_run.restype = C.c_int
        L.oracle_run.argtypes = [P(OracleParams), P(OracleMesh), C.c_double, C.c_double,
                                 C.c_double, C.c_int32, C.c_uint64, C.c_uint32,
                                 P(C.c_uint64), P(C.c_uint32), P(C.c_uint64), P(C.c_uint32),
                                 P(C.c_uint64), P(C.c_uint32), C.c_int, C.c_int,
                                 P(OracleTally), C.c_void_p]
        L.oracle_dump_lane.restype = C.c_int
        L.oracle_dump_lane.argtypes = [P(OracleParams), P(OracleMesh), C.c_double, C.c_double,
                                       C.c_double, C.c_int32, C.c_uint64, C.c_uint32,
                                       C.c_uint64, C.c_uint32, C.c_uint64, C.c_uint32, C.c_int,
                                       P(C.c_double), C.c_uint32, C.c_uint64]
        L.oracle_logf.restype = C.c_float
        L.oracle_logf.argtypes = [C.c_float]
        L.oracle_log.restype = C.c_double
        L.oracle_log.argtypes = [C.c_double]
        L.oracle_sincos_turn_f.argtypes = [C.c_float, P(C.c_float), P(C.c_float)]
        L.oracle_sincos_d.argtypes = [C.c_double, P(C.c_double), P(C.c_double)]
        L.oracle_div_rd.restype = C.c_double
        L.oracle_div_rd.argtypes = [C.c_double, C.c_double]
        L.oracle_safeprimes.restype = C.c_int
        L.oracle_safeprimes.argtypes = [P(C.c_uint32), C.c_uint64]
        L.oracle_uint2float_rz.restype = C.c_float
        L.oracle_uint2float_rz.argtypes = [C.c_uint32]
        L.oracle_set_photon_records.restype = C.c_uint64
        L.oracle_set_photon_records.argtypes = [C.c_void_p, C.c_uint64]
        self.L = L

    def safeprimes(self, count):
        """The MWC multiplier list (first column of safeprimes_base32.txt)."""
        out = np.zeros(count, np.uint32)
        if self.L.oracle_safeprimes(_ptr(out, C.c_uint32), count) != 0:
            raise RuntimeError("multiplier list too short")
        return out

    def write_safeprimes(self, path, count):
        """safeprimes_base32.txt with `count` rows: a, then the high and low
        32-bit words of a*2^32 - 1 (the reference reads the first column)."""
        a = self.safeprimes(count)
        with open(path, "w") as f:
            for v in a.tolist():
                f.write(f"{v} {v - 1} {0xffffffff}\n")

    @staticmethod
    def _mesh(mesh):
        m = OracleMesh()
        m.n_tets = len(mesh.region)
        m.n_faces = len(mesh.planes)
        m.region = _ptr(mesh.region, C.c_int32)
        m.faces = _ptr(mesh.faces, C.c_int32)
        m.signs = _ptr(mesh.signs, C.c_int32)
        m.adj = _ptr(mesh.adj, C.c_int32)
        m.planes = _ptr(mesh.planes, C.c_double)
        return m

    def dump_lane(self, params, mesh, probe, root, rng, lane, precision, max_steps=100000,
                  packet=0):
        """Per-step state (tet, event, x, y, z, ux, uy, uz, w, s, path, LR) of a lane's
        packet number `packet` (0 = first)."""
        out = np.zeros((max_steps, 12))
        n = self.L.oracle_dump_lane(C.byref(params), C.byref(self._mesh(mesh)), probe[0], probe[1],
                                    probe[2], root, int(rng["x"][lane]), int(rng["a"][lane]),
                                    int(rng["xR"][lane]), int(rng["aR"][lane]),
                                    int(rng["xS"][lane]), int(rng["aS"][lane]), precision,
                                    _ptr(out, C.c_double), max_steps, packet)
        return out[:min(n, max_steps)]

    def run(self, params, mesh, probe, root, n_photons, n_lanes, rng, precision, n_threads=0,
            record=False, photon_records=0):
        """One A-scan.  mesh: object with region/faces/signs/adj/planes arrays.
        record: also return the first packet of every lane.  photon_records: keep
        up to this many detected-packet records (RECORD_DTYPE, detection order)
        and return them with the number of detections, (..., records, n)."""
        m = OracleMesh()
        m.n_tets = len(mesh.region)
        m.n_faces = len(mesh.planes)
        m.region = _ptr(mesh.region, C.c_int32)
        m.faces = _ptr(mesh.faces, C.c_int32)
        m.signs = _ptr(mesh.signs, C.c_int32)
        m.adj = _ptr(mesh.adj, C.c_int32)
        m.planes = _ptr(mesh.planes, C.c_double)
        t = empty_tally(params.nbins)
        ts = _fill_tally_struct(OracleTally, t)
        rec = np.zeros(n_lanes, dtype=PACKET_DTYPE) if record else None
        precs = np.zeros(photon_records, dtype=RECORD_DTYPE) if photon_records else None
        self.L.oracle_set_photon_records(precs.ctypes.data if photon_records else None,
                                         photon_records)
        st = self.L.oracle_run(C.byref(params), C.byref(m), probe[0], probe[1], probe[2], root,
                               n_photons, n_lanes,
                               _ptr(rng["x"], C.c_uint64), _ptr(rng["a"], C.c_uint32),
                               _ptr(rng["xR"], C.c_uint64), _ptr(rng["aR"], C.c_uint32),
                               _ptr(rng["xS"], C.c_uint64), _ptr(rng["aS"], C.c_uint32),
                               precision, n_threads, C.byref(ts),
                               rec.ctypes.data if record else None)
        n_det = self.L.oracle_set_photon_records(None, 0)
        if st != 0:
            raise RuntimeError(f"oracle_run failed: {st}")
        for k in ("num_filtered", "num_filtered_class1", "num_filtered_class2", "steps",
                  "restores", "packets", "capped"):
            t[k] = getattr(ts, k)
        out = (t, rec) if record else (t,)
        if photon_records:
            out += (precs[:min(n_det, photon_records)], n_det)
        return out if len(out) > 1 else t


class Reference:
    def __init__(self, path=REF_SO):
        if not os.path.exists(path):
            raise ImportError(f"{path} not built (needs the reference tree); see {HERE}/Makefile")
        L = C.CDLL(path)
        L.ref_init_rng.restype = C.c_int
        L.ref_init_rng.argtypes = [P(C.c_uint64), P(C.c_uint32), P(C.c_uint64), P(C.c_uint32),
                                   P(C.c_uint64), P(C.c_uint32), C.c_uint32, C.c_char_p,
                                   C.c_uint64]
        L.ref_parse.restype = C.c_int
        L.ref_parse.argtypes = [C.c_char_p, C.c_char_p, P(RefSim)]
        L.ref_mesh_counts.argtypes = [C.c_char_p, P(C.c_int32), P(C.c_int32)]
        L.ref_mesh_build.argtypes = [C.c_char_p, C.c_double, C.c_double, C.c_double,
                                     P(C.c_int32), P(C.c_double), P(C.c_int32)]
        L.ref_mesh_build_roots.restype = C.c_int
        L.ref_mesh_build_roots.argtypes = [C.c_char_p, C.c_int32, P(C.c_double), P(C.c_int32),
                                           P(C.c_double), P(C.c_int32)]
        L.ref_run.restype = C.c_int
        L.ref_run.argtypes = [P(RefSim), P(RefMesh), C.c_double, C.c_double, C.c_double,
                              C.c_uint32, P(C.c_uint64), P(C.c_uint32), P(C.c_uint64),
                              P(C.c_uint32), P(C.c_uint64), P(C.c_uint32), C.c_int,
                              P(RefTally), P(C.c_double), P(C.c_uint32)]
        L.ref_trace_first_packets.argtypes = [P(RefSim), P(RefMesh), C.c_double, C.c_double,
                                              C.c_double, C.c_uint32, P(C.c_uint64),
                                              P(C.c_uint32), P(C.c_uint64), P(C.c_uint32),
                                              P(C.c_uint64), P(C.c_uint32), C.c_uint32,
                                              C.c_void_p, C.c_int64, P(C.c_double), C.c_uint32]
        L.ref_write_result.argtypes = [P(RefSim), C.c_double, P(RefTally)]
        self.L = L
        self.threads_per_block = L.ref_num_threads_per_block()

    def init_rng(self, n_lanes, safeprimes_path, seed):
        out = {k: np.zeros(n_lanes, dtype=np.uint64 if k.startswith("x") else np.uint32)
               for k in ("x", "a", "xR", "aR", "xS", "aS")}
        st = self.L.ref_init_rng(_ptr(out["x"], C.c_uint64), _ptr(out["a"], C.c_uint32),
                                 _ptr(out["xR"], C.c_uint64), _ptr(out["aR"], C.c_uint32),
                                 _ptr(out["xS"], C.c_uint64), _ptr(out["aS"], C.c_uint32),
                                 n_lanes, os.fsencode(safeprimes_path), seed)
        if st != 0:
            raise RuntimeError("init_RNG failed")
        return out

    def parse(self, opt_path, mci_path):
        s = RefSim()
        st = self.L.ref_parse(os.fsencode(opt_path), os.fsencode(mci_path), C.byref(s))
        if st != 0:
            raise RuntimeError(f"reference parse failed: {st}")
        return s

    def build_mesh(self, mesh_path, probe):
        nv, nt = C.c_int32(), C.c_int32()
        self.L.ref_mesh_counts(os.fsencode(mesh_path), C.byref(nv), C.byref(nt))
        T = nt.value
        tet = np.zeros(T * 14, np.int32)
        face = np.zeros(4 * T * 4, np.float64)
        root = C.c_int32(-1)
        st = self.L.ref_mesh_build(os.fsencode(mesh_path), probe[0], probe[1], probe[2],
                                   _ptr(tet, C.c_int32), _ptr(face, C.c_double), C.byref(root))
        if st != 0:
            raise RuntimeError(f"reference mesh build failed: {st}")
        tet = tet.reshape(T, 14)
        return {"idx": tet[:, 0].copy(), "region": tet[:, 1].copy(),
                "faces": tet[:, 2:6].copy(), "signs": tet[:, 6:10].copy(),
                "adj": tet[:, 10:14].copy(), "planes": face.reshape(-1, 4), "root": root.value,
                "n_vertices": nv.value}

    def build_mesh_roots(self, mesh_path, probe_xs):
        """MeshGraph + SerializeGraph once and the root tet of each probe position
        (x, 0, 0), with the reference's own functions (O(T^2) in the tet count:
        about an hour at 381k tets).  Returns the serialised arrays, the faces
        trimmed to the distinct ones, and the roots (-1 where none is found)."""
        nv, nt = C.c_int32(), C.c_int32()
        self.L.ref_mesh_counts(os.fsencode(mesh_path), C.byref(nv), C.byref(nt))
        T = nt.value
        tet = np.zeros(T * 14, np.int32)
        face = np.zeros(4 * T * 4, np.float64)
        xs = np.ascontiguousarray(probe_xs, np.float64)
        roots = np.full(len(xs), -1, np.int32)
        st = self.L.ref_mesh_build_roots(os.fsencode(mesh_path), len(xs), _ptr(xs, C.c_double),
                                         _ptr(tet, C.c_int32), _ptr(face, C.c_double),
                                         _ptr(roots, C.c_int32))
        if st != 0:
            raise RuntimeError(f"reference mesh build failed: {st}")
        tet = tet.reshape(T, 14)
        n_faces = int(tet[:, 2:6].max()) + 1
        return {"tet": tet, "planes": face.reshape(-1, 4)[:n_faces].copy(), "roots": roots,
                "n_vertices": nv.value}

    @staticmethod
    def mesh_struct(mesh, root):
        """RefMesh of a mesh: an object with region/faces/signs/adj/planes
        arrays, or a dict {"tet": (T, 14) serialised tets, "planes": (F, 4)}
        as SerializeGraph writes them."""
        if isinstance(mesh, dict):
            tet = np.ascontiguousarray(mesh["tet"], np.int32)
            planes = np.ascontiguousarray(mesh["planes"], np.float64)
            m = RefMesh(len(tet), len(planes), root, _ptr(tet, C.c_int32),
                        _ptr(planes, C.c_double))
            m._keep = (tet, planes)
            return m
        T = len(mesh.region)
        tet = np.zeros((T, 14), np.int32)
        tet[:, 0] = np.arange(T)
        tet[:, 1] = mesh.region
        tet[:, 2:6] = mesh.faces
        tet[:, 6:10] = mesh.signs
        tet[:, 10:14] = mesh.adj
        tet = np.ascontiguousarray(tet)
        planes = np.ascontiguousarray(mesh.planes, np.float64)
        m = RefMesh(T, len(planes), root, _ptr(tet, C.c_int32), _ptr(planes, C.c_double))
        m._keep = (tet, planes)
        return m

    def run(self, sim, mesh, root, probe, n_blocks, rng, n_threads=0):
        """One A-scan through OCTMPSKernel with n_blocks*600 lanes; rng is
        modified in place (it is the lanes' state).  mesh: see mesh_struct."""
        m = self.mesh_struct(mesh, root)
        nb = sim.num_optical_depth_length_steps
        t = empty_tally(nb)
        ts = _fill_tally_struct(RefTally, t)
        secs = C.c_double()
        launches = C.c_uint32()
        st = self.L.ref_run(C.byref(sim), C.byref(m), probe[0], probe[1], probe[2], n_blocks,
                            _ptr(rng["x"], C.c_uint64), _ptr(rng["a"], C.c_uint32),
                            _ptr(rng["xR"], C.c_uint64), _ptr(rng["aR"], C.c_uint32),
                            _ptr(rng["xS"], C.c_uint64), _ptr(rng["aS"], C.c_uint32),
                            n_threads, C.byref(ts), C.byref(secs), C.byref(launches))
        if st != 0:
            raise RuntimeError(f"ref_run failed: {st}")
        t["num_filtered"] = ts.num_filtered
        t["num_filtered_class1"] = ts.num_filtered_class1
        t["num_filtered_class2"] = ts.num_filtered_class2
        t["seconds"] = secs.value
        t["launches"] = launches.value
        return t

    def trace(self, sim, mesh, root, probe, rng, n_lanes, max_steps=10_000_000, dump_lane=-1,
              dump_max=100000):
        m = self.mesh_struct(mesh, root)
        rec = np.zeros(n_lanes, dtype=PACKET_DTYPE)
        dump = np.zeros((dump_max, 12)) if dump_lane >= 0 else None
        self.L.ref_trace_first_packets(C.byref(sim), C.byref(m), probe[0], probe[1], probe[2],
                                       n_lanes,
                                       _ptr(rng["x"], C.c_uint64), _ptr(rng["a"], C.c_uint32),
                                       _ptr(rng["xR"], C.c_uint64), _ptr(rng["aR"], C.c_uint32),
                                       _ptr(rng["xS"], C.c_uint64), _ptr(rng["aS"], C.c_uint32),
                                       max_steps, rec.ctypes.data, dump_lane,
                                       _ptr(dump, C.c_double) if dump is not None else None,
                                       dump_max)
        if dump is not None:
            return rec, dump[:min(int(rec["steps"][dump_lane]), dump_max)]
        return rec

    def write_result(self, sim, probe_x, t):
        ts = _fill_tally_struct(RefTally, t)
        ts.num_filtered = int(t["num_filtered"])
        ts.num_filtered_class1 = int(t["num_filtered_class1"])
        ts.num_filtered_class2 = int(t["num_filtered_class2"])
        self.L.ref_write_result(C.byref(sim), probe_x, C.byref(ts))


def census(params, mesh, probe, root, n_photons, n_lanes, rng, precision=0):
    """Floating-point operations of one A-scan of the oracle's method, counted
    as they execute (census.cpp), on one thread.  Returns (tally, counts) with
    counts {"fp32": {...}, "fp64": {...}, "flops": ..., "flops_per_step": ...}:
    + - x / sqrt 1 each, fused multiply-add 2, transcendental 1."""
    if not os.path.exists(CENSUS_SO):
        raise ImportError(f"{CENSUS_SO} not built; run make in {HERE}")
    L = C.CDLL(CENSUS_SO)
    L.census_run.restype = C.c_int
    L.census_run.argtypes = [P(OracleParams), P(OracleMesh), C.c_double, C.c_double, C.c_double,
                             C.c_int32, C.c_uint64, C.c_uint32, P(C.c_uint64), P(C.c_uint32),
                             P(C.c_uint64), P(C.c_uint32), P(C.c_uint64), P(C.c_uint32), C.c_int,
                             P(OracleTally), P(C.c_uint64)]
    t = empty_tally(params.nbins)
    ts = _fill_tally_struct(OracleTally, t)
    out = np.zeros(12, np.uint64)
    st = L.census_run(C.byref(params), C.byref(Oracle._mesh(mesh)), probe[0], probe[1], probe[2],
                      root, n_photons, n_lanes, _ptr(rng["x"], C.c_uint64),
                      _ptr(rng["a"], C.c_uint32), _ptr(rng["xR"], C.c_uint64),
                      _ptr(rng["aR"], C.c_uint32), _ptr(rng["xS"], C.c_uint64),
                      _ptr(rng["aS"], C.c_uint32), precision, C.byref(ts), _ptr(out, C.c_uint64))
    if st != 0:
        raise RuntimeError(f"census_run failed: {st}")
    for k in ("num_filtered", "num_filtered_class1", "num_filtered_class2", "steps",
              "restores", "packets", "capped"):
        t[k] = getattr(ts, k)
    counts = {"fp32": dict(zip(CENSUS_FIELDS, (int(v) for v in out[:6]))),
              "fp64": dict(zip(CENSUS_FIELDS, (int(v) for v in out[6:])))}
    flops = sum(c["add"] + c["mul"] + c["div"] + c["sqrt"] + 2 * c["fma"] + c["trans"]
                for c in counts.values())
    counts["flops"] = flops
    counts["flops_per_step"] = flops / max(t["steps"], 1)
    for k in ("fp32", "fp64"):
        c = counts[k]
        counts[k + "_flops_per_step"] = (c["add"] + c["mul"] + c["div"] + c["sqrt"] +
                                         2 * c["fma"] + c["trans"]) / max(t["steps"], 1)
    return t, counts
