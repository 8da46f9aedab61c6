"""nebula_b200: B200-native electron transport for Nebula-format SEM simulations.

The product is the C-ABI library ``libnbx.so`` (``include/nbx.h``) with its
sm_100a kernels, and the ``nebula_b200`` command-line program that mirrors
Nebula's ``nebula_gpu``.  This module is a thin ctypes binding over that
C ABI for Python callers (tests, benchmarks, notebooks).  It does not compute
anything itself: when the library is missing, loading fails loudly.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libnbx.so")

NBX_OK = 0
ERRORS = {-1: "invalid argument", -2: "out of memory", -3: "CUDA error", -4: "device wait timed out",
          -5: "malformed input", -6: "call out of order", -7: "no CUDA device", -8: "device queue overflow"}


class NbxError(RuntimeError):
    def __init__(self, code, msg=""):
        super().__init__("%s (%d)%s" % (ERRORS.get(code, "error"), code, (": " + msg) if msg else ""))
        self.code = code


# ---------------------------------------------------------------------------
# ctypes mirrors of include/nbx.h
# ---------------------------------------------------------------------------
class Triangle(C.Structure):
    _fields_ = [("r0", C.c_float * 3), ("e1", C.c_float * 3), ("e2", C.c_float * 3), ("mat_in", C.c_int32),
                ("mat_out", C.c_int32)]


class Octree(C.Structure):
    _fields_ = [("octree_data", C.POINTER(C.c_int32)), ("n_octree", C.c_uint64),
                ("triangles", C.POINTER(Triangle)), ("n_triangles", C.c_uint64), ("center", C.c_float * 3),
                ("halfsize", C.c_float * 3), ("duplicates_dropped", C.c_uint64), ("max_depth", C.c_int32)]


class Table1D(C.Structure):
    _fields_ = [("n", C.c_int32), ("x_min", C.c_float), ("x_step", C.c_float), ("data", C.POINTER(C.c_float))]


class Table2D(C.Structure):
    _fields_ = [("width", C.c_int32), ("height", C.c_int32), ("x_min", C.c_float), ("x_step", C.c_float),
                ("y_min", C.c_float), ("y_step", C.c_float), ("data", C.POINTER(C.c_float))]


class Table3D(C.Structure):
    _fields_ = [("width", C.c_int32), ("height", C.c_int32), ("depth", C.c_int32), ("x_min", C.c_float),
                ("x_step", C.c_float), ("y_min", C.c_float), ("y_step", C.c_float), ("z_min", C.c_float),
                ("z_step", C.c_float), ("data", C.POINTER(C.c_float))]


class Material(C.Structure):
    _fields_ = [("barrier", C.c_float), ("elastic_imfp", Table1D), ("elastic_icdf", Table2D),
                ("phonon_loss", C.c_float), ("recoil_const", C.c_float), ("inelastic_imfp", Table1D),
                ("inelastic_icdf", Table2D), ("ionisation", Table2D), ("fermi", C.c_float),
                ("band_gap", C.c_float), ("max_energy", C.c_float), ("name", C.c_char * 64),
                ("has_kieft_inelastic", C.c_int32), ("has_full_penn", C.c_int32), ("penn_imfp", Table1D),
                ("penn_omega_icdf", Table2D), ("penn_q_icdf", Table3D), ("penn_ionisation", Table3D),
                ("penn_max_energy", C.c_float)]


INELASTIC_MODELS = {"kieft": 0, "penn": 1, "full_penn": 1}


class Config(C.Structure):
    _fields_ = [("device", C.c_int32), ("seed", C.c_uint32), ("energy_threshold", C.c_float),
                ("capacity", C.c_uint64), ("record_detected", C.c_int32), ("record_capacity", C.c_uint64),
                ("block_size", C.c_int32), ("blocks_per_sm", C.c_int32), ("inelastic_model", C.c_int32),
                ("record_deposits", C.c_int32), ("deposit_capacity", C.c_uint64), ("shared_pop", C.c_int32)]


class Tuning(C.Structure):
    _fields_ = [("blocks_per_sm", C.c_int32), ("block_size", C.c_int32), ("stack_depth", C.c_int32),
                ("chunk", C.c_int32), ("queue_capacity", C.c_uint64), ("sample_ms", C.c_double)]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


class Stats(C.Structure):
    _fields_ = [(n, C.c_uint64) for n in (
        "primaries_pushed", "primaries_done", "steps", "events_elastic", "events_inelastic", "events_boundary",
        "secondaries", "detected", "detected_se", "detected_bse", "terminated", "records_dropped", "generations",
        "queue_overflow", "inferences", "roulette_killed", "splits", "samples")] + [
        ("last_run_ms", C.c_double), ("last_kernel_ms", C.c_double), ("deposits", C.c_uint64),
        ("deposits_dropped", C.c_uint64)]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


DETECTED_DTYPE = np.dtype([("pos", "<f4", (3,)), ("dir", "<f4", (3,)), ("E", "<f4"), ("tag", "<u4")])
DEPOSIT_DTYPE = np.dtype([("pos", "<f4", (3,)), ("E", "<f4"), ("dE", "<f4"), ("tag", "<u4")])
ELECTRON_DTYPE = np.dtype([("pos", "<f4", (3,)), ("dir", "<f4", (3,)), ("E", "<f4"), ("mat", "<i4"),
                           ("last_tri", "<i4"), ("tag", "<u4"), ("uid", "<u8"), ("step", "<u4"), ("pad", "<u4")])
assert ELECTRON_DTYPE.itemsize == 56
TABLE_IDS = {"el_imfp": 0, "el_icdf": 1, "in_imfp": 2, "in_icdf": 3, "ion": 4}

_lib = None
_vp = C.c_void_p


def _ptr(a):
    return a.ctypes.data_as(_vp) if a is not None else None


def lib():
    """Load libnbx.so; raises ImportError if the extension has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError("nebula_b200: %s is missing; run `python -m nebula_b200.build`" % LIB_PATH)
    L = C.CDLL(LIB_PATH)
    sig = {
        "nbx_version": (C.c_int, [C.POINTER(C.c_int)] * 3),
        "nbx_error_string": (C.c_char_p, [C.c_int]),
        "nbx_free": (None, [_vp]),
        "nbx_load_tri": (C.c_int, [C.c_char_p, C.POINTER(C.POINTER(Triangle)), C.POINTER(C.c_uint64)]),
        "nbx_load_pri": (C.c_int, [C.c_char_p, C.POINTER(_vp), C.POINTER(C.c_uint64)]),
        "nbx_octree_build": (C.c_int, [_vp, C.c_uint64, C.POINTER(C.POINTER(Octree))]),
        "nbx_octree_free": (None, [C.POINTER(Octree)]),
        "nbx_material_load": (C.c_int, [C.c_char_p, C.POINTER(C.POINTER(Material))]),
        "nbx_material_free": (None, [C.POINTER(Material)]),
        "nbx_device_count": (C.c_int, [C.POINTER(C.c_int)]),
        "nbx_config_default": (None, [C.POINTER(Config)]),
        "nbx_create": (C.c_int, [C.POINTER(_vp), C.POINTER(Config)]),
        "nbx_destroy": (None, [_vp]),
        "nbx_last_error": (C.c_char_p, [_vp]),
        "nbx_set_geometry": (C.c_int, [_vp, C.POINTER(Octree)]),
        "nbx_add_material": (C.c_int, [_vp, C.POINTER(Material)]),
        "nbx_set_tag_range": (C.c_int, [_vp, C.c_uint64]),
        "nbx_push": (C.c_int, [_vp, _vp, _vp, C.c_uint64, C.POINTER(C.c_uint64)]),
        "nbx_run": (C.c_int, [_vp]),
        "nbx_host_alloc": (C.c_int, [C.c_uint64, C.POINTER(_vp)]),
        "nbx_host_free": (None, [_vp]),
        "nbx_get_running_count": (C.c_int, [_vp, C.POINTER(C.c_uint64)]),
        "nbx_get_stats": (C.c_int, [_vp, C.POINTER(Stats)]),
        "nbx_flush_detected": (C.c_int, [_vp, _vp, C.c_uint64, C.POINTER(C.c_uint64)]),
        "nbx_flush_deposits": (C.c_int, [_vp, _vp, C.c_uint64, C.POINTER(C.c_uint64)]),
        "nbx_get_tag_counts": (C.c_int, [_vp, C.c_uint64, C.c_uint64, _vp, _vp]),
        "nbx_pixel_yields": (C.c_int, [_vp, _vp, C.c_uint64, C.c_uint64, _vp]),
        "nbx_set_pixel_map": (C.c_int, [_vp, _vp, C.c_uint64]),
        "nbx_enable_pixel_spectra": (C.c_int, [_vp, C.c_uint64, C.c_int32, C.c_float]),
        "nbx_get_pixel_spectra": (C.c_int, [_vp, _vp]),
        "nbx_get_spectrum": (C.c_int, [_vp, _vp, C.c_uint32, C.POINTER(C.c_float)]),
        "nbx_reset_tallies": (C.c_int, [_vp]),
        "nbx_ray_query": (C.c_int, [_vp, _vp, _vp, _vp, _vp, _vp, C.c_uint64, _vp, _vp]),
        "nbx_table_query": (C.c_int, [_vp, C.c_int32, C.c_int32, _vp, _vp, C.c_uint64, _vp]),
        "nbx_table3_query": (C.c_int, [_vp, C.c_int32, C.c_int32, _vp, _vp, _vp, C.c_uint64, _vp]),
        "nbx_philox": (C.c_int, [_vp, _vp, _vp, C.c_uint64, _vp]),
        "nbx_step_query": (C.c_int, [_vp, _vp, C.c_uint64, _vp, _vp, _vp, _vp]),
        "nbx_set_uid_base": (C.c_int, [_vp, C.c_uint64]),
        "nbx_set_mode": (C.c_int, [_vp, C.c_int32, C.c_float, C.c_float, C.c_int32]),
        "nbx_set_birth_roulette": (C.c_int, [_vp, C.c_float, C.c_float, C.c_float]),
        "nbx_build_surface_map": (C.c_int, [_vp, _vp, _vp, C.c_float, C.c_float]),
        "nbx_set_sample_capacity": (C.c_int, [_vp, C.c_uint64]),
        "nbx_get_samples": (C.c_int, [_vp, _vp, _vp, _vp, C.c_uint64, C.POINTER(C.c_uint64)]),
        "nbx_get_tag_weights": (C.c_int, [_vp, C.c_uint64, C.c_uint64, _vp, _vp]),
        "nbx_features_query": (C.c_int, [_vp, _vp, C.c_uint64, _vp]),
        "nbx_mlp_set_params": (C.c_int, [_vp, _vp]),
        "nbx_mlp_get_params": (C.c_int, [_vp, _vp]),
        "nbx_mlp_grad": (C.c_int, [_vp, _vp, _vp, C.c_uint64, _vp, C.POINTER(C.c_float)]),
        "nbx_mlp_train": (C.c_int, [_vp, _vp, _vp, C.c_uint64, C.c_int32, C.c_int32, C.c_float, C.c_uint32, _vp]),
        "nbx_mlp_predict": (C.c_int, [_vp, _vp, C.c_uint64, _vp]),
        "nbx_autotune": (C.c_int, [_vp, _vp, _vp, C.c_uint64, C.POINTER(Tuning)]),
        "nbx_set_tuning": (C.c_int, [_vp, C.POINTER(Tuning)]),
        "nbx_stage": (C.c_int, [_vp, _vp, _vp, C.c_uint64]),
        "nbx_push_staged": (C.c_int, [_vp, C.POINTER(C.c_uint64)]),
        "nbx_set_learned_cost": (C.c_int, [_vp, _vp, C.c_int32, C.c_int32, C.c_float, C.c_float, C.c_float]),
        "nbx_set_importance_table": (C.c_int, [_vp, C.c_int32, C.c_int32, C.c_int32]),
        "nbx_get_tuning": (C.c_int, [_vp, C.POINTER(Tuning)]),
        "nbx_run_noalloc": (C.c_int, [_vp, _vp, _vp, C.c_uint32, C.c_uint64, _vp, _vp, C.c_uint64,
                                      C.POINTER(C.c_uint64)]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _lib = L
    return L


def _check(rc, ctx=None):
    if rc != NBX_OK:
        msg = lib().nbx_last_error(ctx).decode()
        raise NbxError(rc, msg)


def device_count():
    n = C.c_int(0)
    lib().nbx_device_count(C.byref(n))
    return n.value


class _HostBlock:
    """Page-locked host memory from nbx_host_alloc, freed with the object."""

    def __init__(self, nbytes):
        self._L = lib()     # kept, so the free also works while the interpreter shuts down
        self.p = C.c_void_p()
        _check(self._L.nbx_host_alloc(C.c_uint64(nbytes), C.byref(self.p)))

    def __del__(self):
        if getattr(self, "p", None) and self.p.value:
            self._L.nbx_host_free(self.p)
            self.p = None


def host_empty(shape, dtype=np.float32) -> np.ndarray:
    """An uninitialised numpy array in page-locked host memory
    (nbx_host_alloc), freed when the last view of it goes away.
    Context.stage copies from such arrays asynchronously, so the copy
    overlaps a run; from ordinary (pageable) arrays it works too, but the
    call then waits for the copy.  Needs a CUDA device."""
    dtype = np.dtype(dtype)
    n = int(np.prod(shape, dtype=np.int64))
    nbytes = max(n * dtype.itemsize, 1)
    block = _HostBlock(nbytes)
    raw = (C.c_char * nbytes).from_address(block.p.value)
    raw._nbx_block = block          # the array's base keeps the allocation alive
    return np.frombuffer(raw, dtype=dtype, count=n).reshape(shape)


# ---------------------------------------------------------------------------
# Host-side helpers
# ---------------------------------------------------------------------------
def triangles_from_tri_array(tris) -> np.ndarray:
    """TRI_DTYPE (vertices) -> nbx_triangle records (r0, e1 = r1 - r0, e2 = r2 - r0) in float32."""
    v = np.asarray(tris["v"], np.float32)
    out = np.zeros(len(tris), np.dtype([("r0", "<f4", 3), ("e1", "<f4", 3), ("e2", "<f4", 3),
                                        ("mat_in", "<i4"), ("mat_out", "<i4")]))
    out["r0"] = v[:, 0]
    out["e1"] = (v[:, 1] - v[:, 0]).astype(np.float32)
    out["e2"] = (v[:, 2] - v[:, 0]).astype(np.float32)
    out["mat_in"] = tris["mat_in"]
    out["mat_out"] = tris["mat_out"]
    return out


def load_tri(path) -> np.ndarray:
    p = C.POINTER(Triangle)()
    n = C.c_uint64()
    _check(lib().nbx_load_tri(str(path).encode(), C.byref(p), C.byref(n)))
    raw = C.string_at(p, 44 * n.value)
    lib().nbx_free(C.cast(p, _vp))
    return np.frombuffer(raw, triangles_from_tri_array(np.zeros(0, [("v", "<f4", (3, 3)), ("mat_in", "<i4"),
                                                                        ("mat_out", "<i4")])).dtype).copy()


class HostOctree:
    """Linearized octree built by the library's host builder."""

    def __init__(self, triangles: np.ndarray):
        tri = np.ascontiguousarray(triangles)
        assert tri.dtype.itemsize == 44
        self._L = lib()     # kept, so the free also works while the interpreter shuts down
        self._p = C.POINTER(Octree)()
        _check(self._L.nbx_octree_build(_ptr(tri), len(tri), C.byref(self._p)))
        o = self._p.contents
        self.octree_data = np.ctypeslib.as_array(o.octree_data, (o.n_octree,)).copy()
        raw = C.string_at(o.triangles, 44 * o.n_triangles)
        self.triangles = np.frombuffer(raw, tri.dtype).copy()
        self.center = np.array(o.center, np.float32)
        self.halfsize = np.array(o.halfsize, np.float32)
        self.duplicates_dropped = o.duplicates_dropped
        self.max_depth = o.max_depth

    def __del__(self):
        if getattr(self, "_p", None):
            self._L.nbx_octree_free(self._p)
            self._p = None


class HostMaterial:
    """A .mat file loaded and transformed by the library's host loader."""

    def __init__(self, path):
        self._L = lib()     # kept, so the free also works while the interpreter shuts down
        self._p = C.POINTER(Material)()
        _check(self._L.nbx_material_load(str(path).encode(), C.byref(self._p)))
        m = self._p.contents
        self.barrier, self.fermi, self.band_gap = m.barrier, m.fermi, m.band_gap
        self.phonon_loss, self.recoil_const, self.max_energy = m.phonon_loss, m.recoil_const, m.max_energy
        self.name = m.name.decode()

        def t1(t):
            return np.ctypeslib.as_array(t.data, (t.n,)).copy(), (t.x_min, t.x_step, 0.0, 0.0)

        def t2(t):
            a = np.ctypeslib.as_array(t.data, (t.width * t.height,)).copy().reshape(t.width, t.height)
            return a, (t.x_min, t.x_step, t.y_min, t.y_step)

        def t3(t):
            a = np.ctypeslib.as_array(t.data, (t.width * t.height * t.depth,)).copy()
            return a.reshape(t.width, t.height, t.depth), (t.x_min, t.x_step, t.y_min, t.y_step, t.z_min, t.z_step)

        self.has_kieft_inelastic, self.has_penn = bool(m.has_kieft_inelastic), bool(m.has_full_penn)
        self.penn_max_energy = m.penn_max_energy
        self.tables = {"el_imfp": t1(m.elastic_imfp), "el_icdf": t2(m.elastic_icdf)}
        if self.has_kieft_inelastic:
            self.tables.update({"in_imfp": t1(m.inelastic_imfp), "in_icdf": t2(m.inelastic_icdf),
                                "ion": t2(m.ionisation)})
        if self.has_penn:
            self.tables.update({"penn_imfp": t1(m.penn_imfp), "penn_omega_icdf": t2(m.penn_omega_icdf),
                                "penn_q_icdf": t3(m.penn_q_icdf), "penn_ion": t3(m.penn_ionisation)})

    def __del__(self):
        if getattr(self, "_p", None):
            self._L.nbx_material_free(self._p)
            self._p = None


# ---------------------------------------------------------------------------
# Device context
# ---------------------------------------------------------------------------
class Context:
    """One simulation context on one GPU (the reference's gpu_driver)."""

    def __init__(self, device=0, seed=0x78C7E39B, energy_threshold=0.0, record_detected=False,
                 record_capacity=0, capacity=0, block_size=0, blocks_per_sm=0, inelastic="kieft",
                 record_deposits=False, deposit_capacity=0, shared_pop=False):
        L = lib()
        cfg = Config()
        L.nbx_config_default(C.byref(cfg))
        cfg.device, cfg.seed, cfg.energy_threshold = device, seed, energy_threshold
        cfg.record_detected, cfg.record_capacity, cfg.capacity = int(record_detected), record_capacity, capacity
        cfg.block_size, cfg.blocks_per_sm = block_size, blocks_per_sm
        cfg.inelastic_model = INELASTIC_MODELS.get(inelastic, inelastic)
        cfg.record_deposits, cfg.deposit_capacity = int(record_deposits), deposit_capacity
        cfg.shared_pop = int(shared_pop)
        self.h = _vp()
        self._pixel_map_len = 0
        _check(L.nbx_create(C.byref(self.h), C.byref(cfg)))
        self.L = L
        self._keep = []

    def close(self):
        if getattr(self, "h", None):
            self.L.nbx_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def _ck(self, rc):
        _check(rc, self.h)

    def set_geometry(self, octree: HostOctree):
        self._ck(self.L.nbx_set_geometry(self.h, octree._p))
        self.octree = octree

    def add_material(self, mat: HostMaterial):
        self._ck(self.L.nbx_add_material(self.h, mat._p))
        self._keep.append(mat)

    def set_tag_range(self, n):
        self._ck(self.L.nbx_set_tag_range(self.h, n))

    def push(self, particles: np.ndarray, tags: np.ndarray) -> int:
        p = np.ascontiguousarray(particles, np.float32).reshape(-1, 7)
        t = np.ascontiguousarray(tags, np.uint32)
        acc = C.c_uint64()
        self._ck(self.L.nbx_push(self.h, _ptr(p), _ptr(t), len(t), C.byref(acc)))
        return acc.value

    def stage(self, particles: np.ndarray, tags: np.ndarray):
        """Start copying a batch to the device (nbx_stage); keep the arrays
        alive and unchanged until push_staged() returns."""
        p = np.ascontiguousarray(particles, np.float32).reshape(-1, 7)
        t = np.ascontiguousarray(tags, np.uint32)
        self._staged = (p, t)
        self._ck(self.L.nbx_stage(self.h, _ptr(p), _ptr(t), len(t)))

    def push_staged(self) -> int:
        acc = C.c_uint64()
        self._ck(self.L.nbx_push_staged(self.h, C.byref(acc)))
        self._staged = None
        return acc.value

    def push_records(self, recs: np.ndarray, first_tag=0) -> int:
        """Push .pri records; tag i is the record's index (+first_tag)."""
        p = np.zeros((len(recs), 7), np.float32)
        p[:, 0:3] = recs["pos"]
        p[:, 3:6] = recs["dir"]
        p[:, 6] = recs["E"]
        return self.push(p, np.arange(first_tag, first_tag + len(recs), dtype=np.uint32))

    def run(self):
        self._ck(self.L.nbx_run(self.h))

    def set_uid_base(self, base):
        self._ck(self.L.nbx_set_uid_base(self.h, base))

    def autotune(self, particles: np.ndarray, tags: np.ndarray) -> dict:
        """Pick the fastest launch shape, stack depth and chunk size on a
        sample, in the context's current mode; returns the chosen settings."""
        p = np.ascontiguousarray(particles, np.float32).reshape(-1, 7)
        t = np.ascontiguousarray(tags, np.uint32)
        out = Tuning()
        self._ck(self.L.nbx_autotune(self.h, _ptr(p), _ptr(t), len(t), C.byref(out)))
        return out.as_dict()

    def set_tuning(self, blocks_per_sm, block_size, stack_depth=16, chunk=8):
        tu = Tuning(blocks_per_sm, block_size, stack_depth, chunk, 0, 0.0)
        self._ck(self.L.nbx_set_tuning(self.h, C.byref(tu)))

    def tuning(self) -> dict:
        out = Tuning()
        self._ck(self.L.nbx_get_tuning(self.h, C.byref(out)))
        return out.as_dict()

    def stats(self) -> dict:
        s = Stats()
        self._ck(self.L.nbx_get_stats(self.h, C.byref(s)))
        return s.as_dict()

    def flush_detected(self, cap=None) -> np.ndarray:
        st = self.stats()
        cap = cap if cap is not None else int(st["detected"]) + 16
        out = np.zeros(cap, DETECTED_DTYPE)
        n = C.c_uint64()
        self._ck(self.L.nbx_flush_detected(self.h, _ptr(out), cap, C.byref(n)))
        return out[: n.value]

    def flush_deposits(self, chunk=1 << 22) -> np.ndarray:
        """All energy-deposit records pending on the device (DEPOSIT_DTYPE)."""
        parts = []
        while True:
            out = np.zeros(chunk, DEPOSIT_DTYPE)
            n = C.c_uint64()
            self._ck(self.L.nbx_flush_deposits(self.h, _ptr(out), chunk, C.byref(n)))
            if n.value == 0:
                break
            parts.append(out[: n.value])
        return np.concatenate(parts) if parts else np.zeros(0, DEPOSIT_DTYPE)

    def tag_counts(self, first, n):
        se = np.zeros(n, np.uint32)
        bse = np.zeros(n, np.uint32)
        self._ck(self.L.nbx_get_tag_counts(self.h, first, n, _ptr(se), _ptr(bse)))
        return se, bse

    def set_pixel_map(self, pixel_of_tag: np.ndarray):
        m = np.ascontiguousarray(pixel_of_tag, np.uint32)
        self._ck(self.L.nbx_set_pixel_map(self.h, _ptr(m), len(m)))
        self._pixel_map_len = len(m)

    def enable_pixel_spectra(self, n_pixels, n_bins=200, bin_width=0.5):
        self._ck(self.L.nbx_enable_pixel_spectra(self.h, n_pixels, n_bins, bin_width))
        self._spec_shape = (n_pixels, n_bins)

    def pixel_spectra(self) -> np.ndarray:
        out = np.zeros(self._spec_shape, np.float32)
        self._ck(self.L.nbx_get_pixel_spectra(self.h, _ptr(out)))
        return out

    def pixel_yields(self, pixel_of_tag, n_pixels: int, out=None) -> np.ndarray:
        """Per-pixel sums; pixel_of_tag=None uses the map of set_pixel_map.
        `out` (n_pixels x 5 float64, e.g. in pinned memory) is filled in place."""
        if out is None:
            out = np.zeros((n_pixels, 5), np.float64)
        if pixel_of_tag is None:
            self._ck(self.L.nbx_pixel_yields(self.h, None, self._pixel_map_len, n_pixels, _ptr(out)))
        else:
            m = np.ascontiguousarray(pixel_of_tag, np.uint32)
            self._ck(self.L.nbx_pixel_yields(self.h, _ptr(m), len(m), n_pixels, _ptr(out)))
            self._pixel_map_len = 0
        return out

    def spectrum(self, n_bins=20000):
        out = np.zeros(n_bins, np.uint64)
        w = C.c_float()
        self._ck(self.L.nbx_get_spectrum(self.h, _ptr(out), n_bins, C.byref(w)))
        return out, w.value

    def reset_tallies(self):
        self._ck(self.L.nbx_reset_tallies(self.h))

    def ray_query(self, pos, dirs, dist, ignore_tri, ignore_mat):
        pos = np.ascontiguousarray(pos, np.float32)
        dirs = np.ascontiguousarray(dirs, np.float32)
        dist = np.ascontiguousarray(dist, np.float32)
        it = np.ascontiguousarray(ignore_tri, np.int32)
        im = np.ascontiguousarray(ignore_mat, np.int32)
        n = len(dist)
        od = np.zeros(n, np.float32)
        ot = np.zeros(n, np.int32)
        self._ck(self.L.nbx_ray_query(self.h, _ptr(pos), _ptr(dirs), _ptr(dist), _ptr(it), _ptr(im), n, _ptr(od),
                                      _ptr(ot)))
        return od, ot

    def table_query(self, material, table, x, y=None):
        x = np.ascontiguousarray(x, np.float32)
        y = None if y is None else np.ascontiguousarray(y, np.float32)
        out = np.zeros_like(x)
        self._ck(self.L.nbx_table_query(self.h, material, TABLE_IDS.get(table, table), _ptr(x), _ptr(y), len(x),
                                        _ptr(out)))
        return out

    def table3_query(self, material, table, x, y, z):
        """Full Penn 3-D tables: table "q" (or 0) / "ion3" (or 1)."""
        x = np.ascontiguousarray(x, np.float32)
        y = np.ascontiguousarray(y, np.float32)
        z = np.ascontiguousarray(z, np.float32)
        out = np.zeros_like(x)
        t = {"q": 0, "ion3": 1}.get(table, table)
        self._ck(self.L.nbx_table3_query(self.h, material, t, _ptr(x), _ptr(y), _ptr(z), len(x), _ptr(out)))
        return out

    def philox(self, ctr, key):
        ctr = np.ascontiguousarray(ctr, np.uint32).reshape(-1, 4)
        key = np.ascontiguousarray(key, np.uint32).reshape(-1, 2)
        out = np.zeros_like(ctr)
        self._ck(self.L.nbx_philox(self.h, _ptr(ctr), _ptr(key), len(ctr), _ptr(out)))
        return out

    # ---- learned roulette -------------------------------------------------
    MODES = {"plain": 0, "sample": 1, "learned": 2}

    def set_mode(self, mode, rr_threshold=0.05, split_threshold=0.5, max_roulette_exp=6):
        """plain / sample / learned (see include/nbx.h); in learned mode a
        newborn secondary of importance p < rr_threshold plays roulette with
        survival p / rr_threshold rounded to a power of two (at least
        2^-max_roulette_exp) and one with p > split_threshold splits in two."""
        self._ck(self.L.nbx_set_mode(self.h, self.MODES.get(mode, mode), rr_threshold, split_threshold,
                                     max_roulette_exp))

    def set_birth_roulette(self, min_distance, max_energy, survival):
        """Learned mode: roulette at a secondary's birth (see include/nbx.h)."""
        self._ck(self.L.nbx_set_birth_roulette(self.h, min_distance, max_energy, survival))

    def set_learned_cost(self, mean_cost, log_e_min, log_e_max, value_per_cost):
        """Cost-aware survival of the learned mode (see include/nbx.h):
        mean_cost is n_materials x n_bins steps; None turns it off."""
        if mean_cost is None:
            self._ck(self.L.nbx_set_learned_cost(self.h, None, 0, 0, 0.0, 1.0, 1.0))
            return
        t = np.ascontiguousarray(mean_cost, np.float32)
        if t.ndim == 1:
            t = t[None, :]
        self._ck(self.L.nbx_set_learned_cost(self.h, _ptr(t), t.shape[0], t.shape[1], log_e_min, log_e_max,
                                             value_per_cost))

    def set_importance_table(self, n_energy=48, n_distance=32, n_cosine=16):
        """Learned mode: birth decisions from the network tabulated on a grid
        over its inputs (see include/nbx.h); set_importance_table(0, 0, 0)
        returns to the network evaluated for every newborn."""
        self._ck(self.L.nbx_set_importance_table(self.h, n_energy, n_distance, n_cosine))

    def build_surface_map(self, lo, hi, cell=1.0, d_max=20.0):
        lo = np.ascontiguousarray(lo, np.float32)
        hi = np.ascontiguousarray(hi, np.float32)
        self._ck(self.L.nbx_build_surface_map(self.h, _ptr(lo), _ptr(hi), cell, d_max))

    def set_sample_capacity(self, n):
        self._ck(self.L.nbx_set_sample_capacity(self.h, n))

    def get_samples(self, cap, with_cost=False):
        """Recorded training samples (and clears them): features n x 6 at
        birth, labels n, and with `with_cost` the steps of each sample's
        sub-cascade."""
        f = np.zeros((cap, 6), np.float32)
        y = np.zeros(cap, np.float32)
        c = np.zeros(cap, np.float32)
        n = C.c_uint64()
        self._ck(self.L.nbx_get_samples(self.h, _ptr(f), _ptr(y), _ptr(c), cap, C.byref(n)))
        if with_cost:
            return f[: n.value], y[: n.value], c[: n.value]
        return f[: n.value], y[: n.value]

    def tag_weights(self, first, n):
        se = np.zeros(n, np.float32)
        bse = np.zeros(n, np.float32)
        self._ck(self.L.nbx_get_tag_weights(self.h, first, n, _ptr(se), _ptr(bse)))
        return se, bse

    def features(self, electrons):
        e = np.ascontiguousarray(electrons, ELECTRON_DTYPE)
        out = np.zeros((len(e), 6), np.float32)
        self._ck(self.L.nbx_features_query(self.h, _ptr(e), len(e), _ptr(out)))
        return out

    def mlp_set_params(self, params):
        p = np.ascontiguousarray(params, np.float32)
        assert p.size == 5768
        self._ck(self.L.nbx_mlp_set_params(self.h, _ptr(p)))

    def mlp_get_params(self):
        p = np.zeros(5768, np.float32)
        self._ck(self.L.nbx_mlp_get_params(self.h, _ptr(p)))
        return p

    def mlp_grad(self, features, labels):
        f = np.ascontiguousarray(features, np.float32)
        y = np.ascontiguousarray(labels, np.float32)
        g = np.zeros(5768, np.float32)
        loss = C.c_float()
        self._ck(self.L.nbx_mlp_grad(self.h, _ptr(f), _ptr(y), len(y), _ptr(g), C.byref(loss)))
        return loss.value, g

    def mlp_train(self, features, labels, epochs=5, batch=8192, lr=1e-3, seed=0):
        f = np.ascontiguousarray(features, np.float32)
        y = np.ascontiguousarray(labels, np.float32)
        losses = np.zeros(epochs, np.float32)
        self._ck(self.L.nbx_mlp_train(self.h, _ptr(f), _ptr(y), len(y), epochs, batch, lr, seed, _ptr(losses)))
        return losses

    def mlp_predict(self, features):
        f = np.ascontiguousarray(features, np.float32)
        out = np.zeros(len(f), np.float32)
        self._ck(self.L.nbx_mlp_predict(self.h, _ptr(f), len(f), _ptr(out)))
        return out

    def step_query(self, electrons: np.ndarray):
        e = np.ascontiguousarray(electrons.copy(), ELECTRON_DTYPE)
        n = len(e)
        st = np.zeros(n, np.int32)
        ev = np.zeros(n, np.int32)
        se = np.zeros(n, ELECTRON_DTYPE)
        hs = np.zeros(n, np.int32)
        self._ck(self.L.nbx_step_query(self.h, _ptr(e), n, _ptr(st), _ptr(ev), _ptr(se), _ptr(hs)))
        return e, st, ev, se, hs


def run_noalloc(ctx: Context, d_particles: int, d_tags: int, n: int, uid_base: int, d_se: int, d_bse: int,
                n_tags: int):
    """nbx_run_noalloc on device pointers (ints); returns {elastic, inelastic,
    boundary, detected} of the call."""
    counts = (C.c_uint64 * 4)()
    rc = ctx.L.nbx_run_noalloc(ctx.h, _vp(d_particles), _vp(d_tags), n, uid_base, _vp(d_se), _vp(d_bse), n_tags,
                               counts)
    ctx._ck(rc)
    return dict(zip(("elastic", "inelastic", "boundary", "detected"), [int(c) for c in counts]))


def setup(tri_path_or_array, mat_paths, **ctx_kwargs):
    """Load geometry (.tri path or TRI_DTYPE array) and materials into a new Context."""
    if isinstance(tri_path_or_array, (str, os.PathLike)):
        tris = load_tri(tri_path_or_array)
    else:
        tris = triangles_from_tri_array(tri_path_or_array)
    oct_ = HostOctree(tris)
    ctx = Context(**ctx_kwargs)
    ctx.set_geometry(oct_)
    for p in mat_paths:
        ctx.add_material(HostMaterial(p))
    return ctx


def fit_cost_table(features, costs, n_materials=1, n_bins=32):
    """Mean sub-cascade cost per (material, log-energy bin) from sample-mode
    records (features as recorded: f[0] = (log E - 2.5) / 6.5, material
    one-hot in f[3:6]), for nbx_set_learned_cost: returns (table
    n_materials x n_bins, log_e_min, log_e_max).  Empty bins take the
    nearest filled bin of the same material (1 step if the material has
    none)."""
    f = np.asarray(features, np.float64)
    c = np.asarray(costs, np.float64)
    log_e = f[:, 0] * 6.5 + 2.5
    lo, hi = 2.5, 9.0
    b = np.clip(((log_e - lo) / (hi - lo) * n_bins).astype(np.int64), 0, n_bins - 1)
    mat = np.argmax(f[:, 3:6], axis=1) if f.shape[1] >= 6 else np.zeros(len(f), np.int64)
    table = np.ones((n_materials, n_bins), np.float64)
    for m in range(n_materials):
        sel = mat == m
        s = np.bincount(b[sel], weights=c[sel], minlength=n_bins)
        k = np.bincount(b[sel], minlength=n_bins)
        filled = np.flatnonzero(k)
        if len(filled) == 0:
            continue
        mean = np.where(k > 0, s / np.maximum(k, 1), 0.0)
        nearest = filled[np.abs(np.arange(n_bins)[:, None] - filled[None, :]).argmin(axis=1)]
        table[m] = np.maximum(mean[nearest], 1.0)
    return table.astype(np.float32), lo, hi


def mlp_init_params(seed=0) -> np.ndarray:
    """Seeded Glorot-uniform parameters for the escape-probability network in
    the include/nbx.h layout (W1[64][16] b1[64] W2[64][64] b2[64] W3[8][64]
    b3[8]); biases and the padding columns/rows are zero."""
    rng = np.random.default_rng(seed)
    f, h, pin, pout = 6, 64, 16, 8
    p = np.zeros(h * pin + h + h * h + h + pout * h + pout, np.float64)
    w1 = np.zeros((h, pin))
    lim1 = np.sqrt(6.0 / (f + h))
    w1[:, :f] = rng.uniform(-lim1, lim1, (h, f))
    p[0:h * pin] = w1.ravel()
    o_w2 = h * pin + h
    lim2 = np.sqrt(6.0 / (h + h))
    p[o_w2:o_w2 + h * h] = rng.uniform(-lim2, lim2, h * h)
    o_w3 = o_w2 + h * h + h
    lim3 = np.sqrt(6.0 / (h + 1))
    p[o_w3:o_w3 + h] = rng.uniform(-lim3, lim3, h)
    return p.astype(np.float32)
