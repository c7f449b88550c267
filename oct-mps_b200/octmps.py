"""Python binding of the OCT-MPS B200 library (liboctmps_b200.so), via ctypes.

The library is C-ABI only (include/octmps_capi.h); this module mirrors it
for the tests and the benchmark.  Names follow the reference's host API:
``read_opt``/``read_mci`` are read_simulation_data and Bias_Read
(src/octmps_io.cpp:504-645, src/bias.cpp:9-110), ``build_mesh`` is
MeshGraph + SerializeGraph (src/mesh.cpp), ``Context.submit`` / ``fetch``
stand where RunGPUi (src/main.cu:43-660) stood.

There is no CPU fallback: if the shared library is missing the import
fails, and if no sm_100 GPU is present ``Context`` raises.
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboctmps_b200.so")

MAX_REGIONS = 100
PREC_MIXED, PREC_FP32, PREC_FP64 = 0, 1, 2
STATUS = {
    0: "ok", 1: "invalid argument", 2: "out of memory", 3: "CUDA device error",
    4: "timeout", 5: "not found", 6: "file I/O error", 7: "no usable CUDA device",
    8: "HBM budget exceeded", 9: "kernel reported an error",
}


class OctmpsError(RuntimeError):
    def __init__(self, status, message=""):
        super().__init__(f"{STATUS.get(status, status)}: {message}")
        self.status = status


class Region(C.Structure):
    _fields_ = [("n", C.c_double), ("mua", C.c_double), ("mus", C.c_double), ("g", C.c_double)]


class Sim(C.Structure):
    _fields_ = [
        ("start_x", C.c_double), ("step_x", C.c_double), ("end_x", C.c_double),
        ("number_of_photons", C.c_uint32), ("n_regions", C.c_int32),
        ("regions", Region * MAX_REGIONS),
        ("type_simulation", C.c_int32), ("type_bias", C.c_int32),
        ("record_photons_flag", C.c_int32), ("num_optical_depth_length_steps", C.c_int32),
        ("backward_bias_coefficient", C.c_double),
        ("target_depth_min", C.c_double), ("target_depth_max", C.c_double),
        ("coherence_length_source", C.c_double), ("max_collecting_radius", C.c_double),
        ("max_collecting_angle_deg", C.c_double), ("probability_additional_bias", C.c_double),
        ("max_relative_contribution", C.c_double), ("max_filtered_optical_depth", C.c_double),
        ("optical_depth_shift", C.c_double), ("rnd_step_size_in_tissue", C.c_double),
    ]


class MeshDesc(C.Structure):
    _fields_ = [
        ("n_tets", C.c_int32), ("n_faces", C.c_int32),
        ("tet_region", C.POINTER(C.c_int32)), ("tet_faces", C.POINTER(C.c_int32)),
        ("tet_signs", C.POINTER(C.c_int32)), ("tet_adj", C.POINTER(C.c_int32)),
        ("face_plane", C.POINTER(C.c_double)),
    ]


class HostMesh(C.Structure):
    _fields_ = [
        ("n_vertices", C.c_int32), ("n_tets", C.c_int32), ("n_faces", C.c_int32),
        ("n_distinct", C.c_int32),
        ("tet_region", C.POINTER(C.c_int32)), ("tet_faces", C.POINTER(C.c_int32)),
        ("tet_signs", C.POINTER(C.c_int32)), ("tet_adj", C.POINTER(C.c_int32)),
        ("face_plane", C.POINTER(C.c_double)),
    ]


class RngLanes(C.Structure):
    _fields_ = [
        ("x", C.POINTER(C.c_uint64)), ("a", C.POINTER(C.c_uint32)),
        ("xR", C.POINTER(C.c_uint64)), ("aR", C.POINTER(C.c_uint32)),
        ("xS", C.POINTER(C.c_uint64)), ("aS", C.POINTER(C.c_uint32)),
    ]


class Job(C.Structure):
    _fields_ = [
        ("mesh", C.c_int32), ("sim", C.POINTER(Sim)),
        ("probe_x", C.c_double), ("probe_y", C.c_double), ("probe_z", C.c_double),
        ("root_tet", C.c_int32), ("n_photons", C.c_uint64), ("seed", C.c_uint64),
        ("n_lanes", C.c_uint32), ("precision", C.c_int32),
    ]


class Tally(C.Structure):
    _fields_ = [
        ("num_filtered", C.c_uint64), ("num_filtered_class1", C.c_uint64),
        ("num_filtered_class2", C.c_uint64),
        ("count1", C.POINTER(C.c_uint64)), ("count2", C.POINTER(C.c_uint64)),
        ("sum1", C.POINTER(C.c_double)), ("max1", C.POINTER(C.c_double)),
        ("sumsq1", C.POINTER(C.c_double)),
        ("sum2", C.POINTER(C.c_double)), ("max2", C.POINTER(C.c_double)),
        ("sumsq2", C.POINTER(C.c_double)), ("num_nonfinite", C.c_uint64),
    ]


class JobStats(C.Structure):
    _fields_ = [
        ("packets", C.c_uint64), ("steps", C.c_uint64), ("restores", C.c_uint64),
        ("device_ms", C.c_double), ("submit_to_done_ms", C.c_double),
        ("launch_id", C.c_int64), ("stopped", C.c_uint64),
    ]


class LaunchConfig(C.Structure):
    _fields_ = [
        ("block_size", C.c_int32), ("blocks_per_sm", C.c_int32), ("default_lanes", C.c_int32),
        ("use_graphs", C.c_int32), ("hbm_budget_bytes", C.c_uint64),
        ("scatter_share", C.c_int32), ("linger_us", C.c_int32), ("kernel_form", C.c_int32),
    ]


class Incident(C.Structure):
    _fields_ = [
        ("stopped", C.c_int32), ("tet", C.c_int32), ("job", C.c_int64), ("seed", C.c_uint64),
        ("n_lanes", C.c_uint64), ("n_photons", C.c_uint64), ("lane", C.c_uint64),
        ("packets_left", C.c_uint64), ("steps", C.c_uint64), ("pos", C.c_double * 3),
        ("dir", C.c_double * 3), ("weight", C.c_double), ("step_left", C.c_double),
    ]


# Symbols include/octmps_capi.h declares (checked by the CPU tests).
EXPORTED = [
    "octmps_ctx_create", "octmps_ctx_destroy", "octmps_last_error", "octmps_status_string",
    "octmps_ctx_set_multipliers", "octmps_ctx_configure", "octmps_mesh_build_file",
    "octmps_mesh_host_free", "octmps_mesh_find_root", "octmps_mesh_upload", "octmps_mesh_release",
    "octmps_rng_init", "octmps_job_submit", "octmps_ctx_flush", "octmps_ctx_synchronize",
    "octmps_ctx_poll", "octmps_debug_incident", "octmps_job_wait",
    "octmps_job_fetch", "octmps_job_fetch_stats", "octmps_job_release", "octmps_read_opt",
    "octmps_read_mci", "octmps_write_result", "octmps_safeprimes_generate",
    "octmps_safeprimes_write", "octmps_safeprimes_read", "octmps_ascan_run_noalloc",
    "octmps_probe_positions", "octmps_ascans_of_gpu", "octmps_ctx_set_photon_record_capacity",
    "octmps_job_photon_records", "octmps_write_filtered_photons",
]

# One detected packet (RecordPhotonsFlag), as octmps_photon_record.
RECORD_DTYPE = np.dtype([
    ("weight", np.float64), ("likelihood", np.float64), ("radius", np.float64),
    ("cos_angle", np.float64), ("optical_path", np.float64), ("max_depth", np.float64),
])

_lib = None


def lib():
    """Loads liboctmps_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} not built; run make in {HERE}")
        L = C.CDLL(LIB_PATH)
        P = C.POINTER
        sig = {
            "octmps_ctx_create": (C.c_int, [C.c_int, P(C.c_void_p)]),
            "octmps_ctx_destroy": (C.c_int, [C.c_void_p]),
            "octmps_last_error": (C.c_char_p, [C.c_void_p]),
            "octmps_status_string": (C.c_char_p, [C.c_int]),
            "octmps_ctx_set_multipliers": (C.c_int, [C.c_void_p, P(C.c_uint32), C.c_uint64]),
            "octmps_ctx_configure": (C.c_int, [C.c_void_p, P(LaunchConfig)]),
            "octmps_mesh_build_file": (C.c_int, [C.c_char_p, P(HostMesh)]),
            "octmps_mesh_host_free": (None, [P(HostMesh)]),
            "octmps_mesh_find_root": (C.c_int, [P(MeshDesc), C.c_double, C.c_double, C.c_double,
                                                P(C.c_int32)]),
            "octmps_mesh_upload": (C.c_int, [C.c_void_p, P(MeshDesc), P(C.c_int32)]),
            "octmps_mesh_release": (C.c_int, [C.c_void_p, C.c_int32]),
            "octmps_rng_init": (C.c_int, [P(C.c_uint32), C.c_uint64, C.c_uint32, C.c_uint64,
                                          P(RngLanes)]),
            "octmps_job_submit": (C.c_int, [C.c_void_p, P(Job), P(C.c_int64)]),
            "octmps_ctx_flush": (C.c_int, [C.c_void_p]),
            "octmps_ctx_synchronize": (C.c_int, [C.c_void_p]),
            "octmps_ctx_poll": (C.c_int, [C.c_void_p, P(C.c_int64), C.c_int32, P(C.c_int32)]),
            "octmps_debug_incident": (C.c_int, [C.c_void_p, C.c_int32, P(Incident)]),
            "octmps_job_wait": (C.c_int, [C.c_void_p, C.c_int64, C.c_int32]),
            "octmps_job_fetch": (C.c_int, [C.c_void_p, C.c_int64, P(Tally)]),
            "octmps_job_fetch_stats": (C.c_int, [C.c_void_p, C.c_int64, P(JobStats)]),
            "octmps_job_release": (C.c_int, [C.c_void_p, C.c_int64]),
            "octmps_read_opt": (C.c_int, [C.c_char_p, P(Sim)]),
            "octmps_read_mci": (C.c_int, [C.c_char_p, P(Sim)]),
            "octmps_write_result": (C.c_int, [C.c_char_p, P(Sim), C.c_double, P(Tally)]),
            "octmps_safeprimes_generate": (C.c_int, [P(C.c_uint32), C.c_uint64]),
            "octmps_safeprimes_write": (C.c_int, [C.c_char_p, C.c_uint64]),
            "octmps_safeprimes_read": (C.c_int64, [C.c_char_p, P(C.c_uint32), C.c_uint64]),
            "octmps_debug_record_next_launch": (C.c_int, [C.c_void_p, C.c_void_p]),
            "octmps_probe_positions": (C.c_int64, [P(Sim), P(C.c_double), C.c_uint64]),
            "octmps_ascans_of_gpu": (C.c_int64, [C.c_uint64, C.c_uint32, C.c_uint32,
                                                 P(C.c_uint64), C.c_uint64]),
            "octmps_ctx_set_photon_record_capacity": (C.c_int, [C.c_void_p, C.c_uint64]),
            "octmps_job_photon_records": (C.c_int, [C.c_void_p, C.c_int64, C.c_void_p,
                                                    C.c_uint64, P(C.c_uint64), P(C.c_uint64)]),
            "octmps_write_filtered_photons": (C.c_int, [C.c_char_p, C.c_double, C.c_void_p,
                                                        C.c_uint64]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def _ptr(arr, ctype):
    return arr.ctypes.data_as(C.POINTER(ctype))


def _check(st, ctx=None):
    if st != 0:
        msg = lib().octmps_last_error(ctx).decode() if ctx else ""
        raise OctmpsError(st, msg)


# ------------------------------------------------------------------ files --

def read_opt(path):
    s = Sim()
    _check(lib().octmps_read_opt(os.fsencode(path), C.byref(s)))
    return s


def read_mci(path, sim):
    _check(lib().octmps_read_mci(os.fsencode(path), C.byref(sim)))
    return sim


def read_deck(opt_path, mci_path):
    return read_mci(mci_path, read_opt(opt_path))


def probe_positions(sim):
    """The A-scan loop of main (src/main.cu:948-950), in the same double steps."""
    n = lib().octmps_probe_positions(C.byref(sim), None, 0)
    if n < 0:
        raise OctmpsError(1, "probe scan never ends (step_x <= 0)")
    out = np.zeros(n, np.float64)
    lib().octmps_probe_positions(C.byref(sim), _ptr(out, C.c_double), n)
    return out.tolist()


def ascans_of_gpu(n_ascans, n_gpus, gpu):
    """A-scans GPU `gpu` of `n_gpus` runs under the CLI's -G (round robin)."""
    n = lib().octmps_ascans_of_gpu(n_ascans, n_gpus, gpu, None, 0)
    if n < 0:
        raise OctmpsError(1, f"invalid split: gpu {gpu} of {n_gpus}")
    out = np.zeros(n, np.uint64)
    lib().octmps_ascans_of_gpu(n_ascans, n_gpus, gpu, _ptr(out, C.c_uint64), n)
    return [int(k) for k in out]


class Mesh:
    """A mesh in SerializeGraph's layout (numpy arrays owned by Python)."""

    def __init__(self, region, faces, signs, adj, planes, n_vertices=0, n_distinct=0):
        self.region = np.ascontiguousarray(region, dtype=np.int32)
        self.faces = np.ascontiguousarray(faces, dtype=np.int32).reshape(-1, 4)
        self.signs = np.ascontiguousarray(signs, dtype=np.int32).reshape(-1, 4)
        self.adj = np.ascontiguousarray(adj, dtype=np.int32).reshape(-1, 4)
        self.planes = np.ascontiguousarray(planes, dtype=np.float64).reshape(-1, 4)
        self.n_vertices = n_vertices
        self.n_distinct = n_distinct

    @property
    def n_tets(self):
        return len(self.region)

    def desc(self):
        d = MeshDesc()
        d.n_tets = self.n_tets
        d.n_faces = len(self.planes)
        d.tet_region = _ptr(self.region, C.c_int32)
        d.tet_faces = _ptr(self.faces, C.c_int32)
        d.tet_signs = _ptr(self.signs, C.c_int32)
        d.tet_adj = _ptr(self.adj, C.c_int32)
        d.face_plane = _ptr(self.planes, C.c_double)
        d._keep = self
        return d

    def find_root(self, px, py=0.0, pz=0.0):
        r = C.c_int32(-1)
        st = lib().octmps_mesh_find_root(C.byref(self.desc()), px, py, pz, C.byref(r))
        if st != 0:
            raise OctmpsError(st, f"probe ({px}, {py}, {pz}) is not on a boundary face")
        return r.value


def build_mesh(path):
    """MeshGraph + SerializeGraph of a .mesh file (O(T) hash-based)."""
    hm = HostMesh()
    _check(lib().octmps_mesh_build_file(os.fsencode(path), C.byref(hm)))
    try:
        T, F = hm.n_tets, hm.n_faces
        m = Mesh(np.ctypeslib.as_array(hm.tet_region, (T,)).copy(),
                 np.ctypeslib.as_array(hm.tet_faces, (4 * T,)).copy(),
                 np.ctypeslib.as_array(hm.tet_signs, (4 * T,)).copy(),
                 np.ctypeslib.as_array(hm.tet_adj, (4 * T,)).copy(),
                 np.ctypeslib.as_array(hm.face_plane, (4 * F,)).copy(),
                 n_vertices=hm.n_vertices, n_distinct=hm.n_distinct)
    finally:
        lib().octmps_mesh_host_free(C.byref(hm))
    return m


# ------------------------------------------------------------------- RNG --

def safeprimes(count):
    a = np.zeros(count, dtype=np.uint32)
    _check(lib().octmps_safeprimes_generate(_ptr(a, C.c_uint32), count))
    return a


def write_safeprimes(path, count):
    _check(lib().octmps_safeprimes_write(os.fsencode(path), count))


def read_safeprimes(path, max_count):
    a = np.zeros(max_count, dtype=np.uint32)
    n = lib().octmps_safeprimes_read(os.fsencode(path), _ptr(a, C.c_uint32), max_count)
    if n < 0:
        raise OctmpsError(6, f"cannot read {path}")
    return a[:n]


def rng_init(multipliers, n_lanes, seed):
    """init_RNG (src/octmps_kernel.cuh:52-172) from an in-memory multiplier table."""
    out = {k: np.zeros(n_lanes, dtype=np.uint64 if k.startswith("x") else np.uint32)
           for k in ("x", "a", "xR", "aR", "xS", "aS")}
    rl = RngLanes(*[_ptr(out[k], C.c_uint64 if k.startswith("x") else C.c_uint32)
                    for k in ("x", "a", "xR", "aR", "xS", "aS")])
    m = np.ascontiguousarray(multipliers, dtype=np.uint32)
    _check(lib().octmps_rng_init(_ptr(m, C.c_uint32), len(m), n_lanes, seed, C.byref(rl)))
    return out


# ----------------------------------------------------------------- tallies --

def empty_tally(nbins):
    t = {"count1": np.zeros(nbins + 1, np.uint64), "count2": np.zeros(nbins + 1, np.uint64)}
    for k in ("sum1", "max1", "sumsq1", "sum2", "max2", "sumsq2"):
        t[k] = np.zeros(nbins + 2, np.float64)
    return t


def tally_struct(t):
    s = Tally()
    for k in ("count1", "count2"):
        setattr(s, k, _ptr(t[k], C.c_uint64))
    for k in ("sum1", "max1", "sumsq1", "sum2", "max2", "sumsq2"):
        setattr(s, k, _ptr(t[k], C.c_double))
    s.num_filtered = int(t.get("num_filtered", 0))
    s.num_filtered_class1 = int(t.get("num_filtered_class1", 0))
    s.num_filtered_class2 = int(t.get("num_filtered_class2", 0))
    return s


def write_result(directory, sim, probe_x, t):
    _check(lib().octmps_write_result(os.fsencode(directory), C.byref(sim), probe_x,
                                     C.byref(tally_struct(t))))


def write_filtered_photons(directory, probe_x, records):
    """Appends RECORD_DTYPE records to FilteredPhotons.mco in `directory`."""
    r = np.ascontiguousarray(records, dtype=RECORD_DTYPE)
    _check(lib().octmps_write_filtered_photons(os.fsencode(directory), probe_x,
                                               r.ctypes.data if len(r) else None, len(r)))


# ---------------------------------------------------------------- context --

class Context:
    """One GPU: resident meshes, queued jobs, persistent launches."""

    def __init__(self, device=0, multipliers=None):
        self.h = C.c_void_p()
        _check(lib().octmps_ctx_create(device, C.byref(self.h)))
        self._keep = []
        self._cfg = {"block_size": 0, "blocks_per_sm": 0, "default_lanes": 0,
                     "hbm_budget_bytes": 0, "scatter_share": 0, "linger_us": 0,
                     "kernel_form": 0}
        if multipliers is not None:
            self.set_multipliers(multipliers)

    def close(self):
        if self.h:
            lib().octmps_ctx_destroy(self.h)
            self.h = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def last_error(self):
        return lib().octmps_last_error(self.h).decode()

    def set_multipliers(self, a):
        a = np.ascontiguousarray(a, dtype=np.uint32)
        _check(lib().octmps_ctx_set_multipliers(self.h, _ptr(a, C.c_uint32), len(a)), self.h)

    def configure(self, **settings):
        """Launch configuration (octmps_launch_config): block_size,
        blocks_per_sm, default_lanes, hbm_budget_bytes, scatter_share,
        linger_us, kernel_form (0 per-lane, 1 pooled); settings not given keep
        their current values (0 = default)."""
        unknown = set(settings) - set(self._cfg)
        if unknown:
            raise TypeError(f"unknown launch settings: {sorted(unknown)}")
        cfg = dict(self._cfg, **settings)
        c = LaunchConfig(cfg["block_size"], cfg["blocks_per_sm"], cfg["default_lanes"], 0,
                         cfg["hbm_budget_bytes"], cfg["scatter_share"], cfg["linger_us"],
                         cfg["kernel_form"])
        _check(lib().octmps_ctx_configure(self.h, C.byref(c)), self.h)
        self._cfg = cfg

    # Default launch variants of autotune(): (kernel_form, block_size,
    # blocks_per_sm, scatter_share).  Per-lane kernel: 256-thread blocks at
    # 2-4 per SM and a few scatter shares, 128-thread blocks at 6-8 and
    # 512-thread blocks at 2 (the register cap follows from block size x
    # blocks); pooled kernel at 4-5 blocks.
    AUTOTUNE_VARIANTS = ([(0, 256, 2, 12)] + [(0, 256, 3, sh) for sh in (10, 12, 14)] +
                         [(0, 256, 4, 12)] + [(0, 128, b, 12) for b in (6, 7, 8)] +
                         [(0, 512, 2, 12)] + [(1, 128, b, 12) for b in (4, 5)])

    def autotune(self, mesh_id, sim, probe_x, root, precision=PREC_MIXED, n_photons=1_000_000,
                 n_jobs=4, n_lanes=0, variants=None, seed=1):
        """Times a sample of the workload (n_jobs jobs of n_photons packets,
        seeds seed..seed+n_jobs-1, in one launch) under each launch variant
        and keeps the fastest, by propagation steps per second of device
        time.  The sample should keep the whole GPU busy for most of its
        launch, or the launch's tail decides the ranking.

        `variants`: tuples (kernel_form, block_size, blocks_per_sm,
        scatter_share[, n_lanes]); default AUTOTUNE_VARIANTS.  An n_lanes
        entry (photons per lane = n_photons / n_lanes) overrides the sample's
        lane count for that variant: the lane count decides which random
        numbers each packet draws, so a job's results equal the reference's
        only at the reference's own lane count, and callers that need that
        leave it out.  The scatter share is the point at which a warp turns
        to its waiting scattering halves (the regeneration of its lanes'
        boundary work), linger_us the point at which idle threads give up.
        Returns (best, [(kernel_form, block_size, blocks_per_sm, scatter_share,
        n_lanes, steps_per_s), ...]) and leaves the best variant configured."""
        if variants is None:
            variants = self.AUTOTUNE_VARIANTS
        nb = sim.num_optical_depth_length_steps
        table = []
        for v in variants:
            form, block, b, sh = v[:4]
            lanes = v[4] if len(v) > 4 else n_lanes
            self.configure(kernel_form=form, block_size=block, blocks_per_sm=b, scatter_share=sh)
            ids = [self.submit(mesh_id, sim, probe_x, root, n_photons=n_photons,
                               seed=seed + k, n_lanes=lanes, precision=precision)
                   for k in range(n_jobs)]
            self.flush()
            for j in ids:
                self.fetch(j, nb)
            self.synchronize()
            sts = [self.stats(j) for j in ids]
            for j in ids:
                self.release(j)
            ms = {s["launch_id"]: s["device_ms"] for s in sts}
            table.append((form, block, b, sh, lanes,
                          sum(s["steps"] for s in sts) / (sum(ms.values()) / 1e3)))
        best = max(table, key=lambda r: r[5])
        self.configure(kernel_form=best[0], block_size=best[1], blocks_per_sm=best[2],
                       scatter_share=best[3])
        return best, table

    def upload_mesh(self, mesh):
        mid = C.c_int32()
        _check(lib().octmps_mesh_upload(self.h, C.byref(mesh.desc()), C.byref(mid)), self.h)
        return mid.value

    def release_mesh(self, mid):
        _check(lib().octmps_mesh_release(self.h, mid), self.h)

    def submit(self, mesh_id, sim, probe_x, root, n_photons=0, seed=0, n_lanes=0,
               precision=PREC_MIXED, probe_y=0.0, probe_z=0.0):
        j = Job()
        j.mesh = mesh_id
        j.sim = C.pointer(sim)
        j.probe_x, j.probe_y, j.probe_z = probe_x, probe_y, probe_z
        j.root_tet = root
        j.n_photons = n_photons
        j.seed = seed
        j.n_lanes = n_lanes
        j.precision = precision
        jid = C.c_int64()
        _check(lib().octmps_job_submit(self.h, C.byref(j), C.byref(jid)), self.h)
        return jid.value

    def flush(self):
        _check(lib().octmps_ctx_flush(self.h), self.h)

    def last_error(self):
        return lib().octmps_last_error(self.h).decode()

    def synchronize(self):
        """Waits until every launch of the context has ended."""
        _check(lib().octmps_ctx_synchronize(self.h), self.h)

    def poll(self, max_ids=1024):
        """Ids of jobs finished since the last poll (never waits)."""
        buf = (C.c_int64 * max_ids)()
        n = C.c_int32()
        _check(lib().octmps_ctx_poll(self.h, buf, max_ids, C.byref(n)), self.h)
        return list(buf[: n.value])

    def incident(self, precision=PREC_MIXED):
        """The first packet of the precision's job table stopped at the step
        cap (None if none), as a dict."""
        inc = Incident()
        _check(lib().octmps_debug_incident(self.h, precision, C.byref(inc)), self.h)
        if not inc.stopped:
            return None
        return {f: (list(getattr(inc, f)) if f in ("pos", "dir") else getattr(inc, f))
                for f, _ in Incident._fields_}

    def wait(self, jid, timeout_ms=-1):
        return lib().octmps_job_wait(self.h, jid, timeout_ms)

    def fetch(self, jid, nbins):
        t = empty_tally(nbins)
        s = tally_struct(t)
        _check(lib().octmps_job_fetch(self.h, jid, C.byref(s)), self.h)
        t["num_filtered"] = s.num_filtered
        t["num_filtered_class1"] = s.num_filtered_class1
        t["num_filtered_class2"] = s.num_filtered_class2
        t["num_nonfinite"] = s.num_nonfinite
        return t

    def stats(self, jid):
        s = JobStats()
        st = lib().octmps_job_fetch_stats(self.h, jid, C.byref(s))
        if st not in (0, 9):
            _check(st, self.h)
        return {"packets": s.packets, "steps": s.steps, "restores": s.restores,
                "device_ms": s.device_ms, "submit_to_done_ms": s.submit_to_done_ms,
                "launch_id": s.launch_id, "stopped": s.stopped}

    def release(self, jid):
        _check(lib().octmps_job_release(self.h, jid), self.h)

    def set_photon_record_capacity(self, capacity):
        """Records kept per job with RecordPhotonsFlag (0 = the job's packets)."""
        _check(lib().octmps_ctx_set_photon_record_capacity(self.h, capacity), self.h)

    def photon_records(self, jid):
        """(records as RECORD_DTYPE in detection order, detections in all) of a
        finished job whose sim sets record_photons_flag."""
        kept, det = C.c_uint64(), C.c_uint64()
        _check(lib().octmps_job_photon_records(self.h, jid, None, 0, C.byref(kept),
                                               C.byref(det)), self.h)
        out = np.zeros(kept.value, dtype=RECORD_DTYPE)
        if kept.value:
            _check(lib().octmps_job_photon_records(self.h, jid, out.ctypes.data, kept.value,
                                                   C.byref(kept), C.byref(det)), self.h)
        return out, det.value

    def record_next_launch(self, device_ptr):
        _check(lib().octmps_debug_record_next_launch(self.h, C.c_void_p(device_ptr)), self.h)
