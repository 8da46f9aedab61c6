"""Checkers for the nebula_b200 transport path (TEST INFRASTRUCTURE ONLY).

Two CPU implementations the CUDA kernels are compared against:

* ``ref``  -- the reference's own CPU code compiled from its source tree by
  ``oracle/Makefile`` into ``oracle/_ref/libnbref.so`` (octree builder,
  ``octree<false>::propagate``, Kieft material loaders and table lookups, and
  a cpu_mt_main-style multi-threaded run) and, on the reference's stock
  physics configuration (full Penn inelastic model), into
  ``oracle/_ref/libnbref_penn.so``.
* ``port`` -- the plain-C restatement ``oracle/nbx_oracle.c``
  (``oracle/libnbx_oracle.so``), which shares the product's per-electron
  Philox random-number scheme so single events can be compared directly.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg use
this package; the product never imports it.
"""
from __future__ import annotations

import ctypes as C
import os
import shutil
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_SO = os.path.join(HERE, "_ref", "libnbref.so")
REF_PENN_SO = os.path.join(HERE, "_ref", "libnbref_penn.so")
PORT_SO = os.path.join(HERE, "libnbx_oracle.so")
REF_BIN = os.path.join(HERE, "_ref", "nebula_cpu_mt_kieft")
REF_BIN_PENN = os.path.join(HERE, "_ref", "nebula_cpu_mt")

_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
_u32p = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")

_ref = {}
_port = None


def reference_source_dir():
    """The reference's source tree: $NEBULA_REFERENCE_SOURCE, else a
    checkout named `reference` beside this repository (reference/source)."""
    env = os.environ.get("NEBULA_REFERENCE_SOURCE")
    if env:
        return env
    return os.path.normpath(os.path.join(HERE, "..", "..", "reference", "source"))


def build(reference_dir=None):
    """Compile the checkers (port always; ref when the reference tree exists)."""
    import subprocess
    reference_dir = reference_dir or reference_source_dir()
    subprocess.run(["make", "-s", "-C", HERE, "port"], check=True)
    if os.path.isdir(reference_dir):
        subprocess.run(["make", "-s", "-C", HERE, "ref", "REF=" + reference_dir], check=True)
        # the reference's GPU program, when nvcc is present
        if shutil.which(os.environ.get("NVCC", "nvcc")) or os.path.exists("/usr/local/cuda/bin/nvcc"):
            env = dict(os.environ)
            if not shutil.which(env.get("NVCC", "nvcc")):
                env["NVCC"] = "/usr/local/cuda/bin/nvcc"
            # optional: the GPU-to-GPU comparison only; a failed build leaves it out
            r = subprocess.run(["make", "-s", "-C", HERE, "gpu", "REF=" + reference_dir], check=False, env=env)
            if r.returncode != 0:
                print("oracle: the reference's GPU program did not build; it is left out", file=sys.stderr)


def have_ref(penn=False):
    return os.path.exists(REF_PENN_SO if penn else REF_SO)


def ref(penn=False):
    """The compiled reference: Kieft inelastic model, or with ``penn`` the
    stock full Penn model."""
    if penn not in _ref:
        lib = C.CDLL(REF_PENN_SO if penn else REF_SO)
        lib.nbref_build_octree.restype = C.c_int
        lib.nbref_build_octree.argtypes = [_f32p, _i32p, C.c_int64, C.POINTER(C.POINTER(C.c_int32)),
                                           C.POINTER(C.c_int64), C.POINTER(C.POINTER(C.c_float)),
                                           C.POINTER(C.POINTER(C.c_int32)), C.POINTER(C.c_int64),
                                           _f32p, _f32p]
        lib.nbref_free.argtypes = [C.c_void_p]
        lib.nbref_geometry_create.restype = C.c_void_p
        lib.nbref_geometry_create.argtypes = [_f32p, _i32p, C.c_int64]
        lib.nbref_geometry_destroy.argtypes = [C.c_void_p]
        lib.nbref_geometry_info.argtypes = [C.c_void_p, _f32p, _f32p, C.POINTER(C.c_float)]
        lib.nbref_propagate.argtypes = [C.c_void_p, _f32p, _f32p, _f32p, _i32p, _i32p, C.c_int64, _f32p, _i32p]
        lib.nbref_in_domain.argtypes = [C.c_void_p, _f32p, C.c_int64, _i32p]
        lib.nbref_material_load.restype = C.c_void_p
        lib.nbref_material_load.argtypes = [C.c_char_p]
        lib.nbref_material_destroy.argtypes = [C.c_void_p]
        lib.nbref_material_info.argtypes = [C.c_void_p, _f32p]
        lib.nbref_material_eval.argtypes = [C.c_void_p, C.c_int, _f32p, _f32p, C.c_int64, _f32p]
        lib.nbref_material_table.argtypes = [C.c_void_p, C.c_int, C.c_void_p, _i32p, _f32p]
        lib.nbref_material_eval3.restype = C.c_int
        lib.nbref_material_eval3.argtypes = [C.c_void_p, C.c_int, _f32p, _f32p, _f32p, C.c_int64, _f32p]
        lib.nbref_material_table3.restype = C.c_int
        lib.nbref_material_table3.argtypes = [C.c_void_p, C.c_int, C.c_void_p, _i32p, _f32p]
        lib.nbref_run.restype = C.c_int
        lib.nbref_run.argtypes = [C.c_char_p, C.c_char_p, C.POINTER(C.c_char_p), C.c_int, C.c_uint32, C.c_float,
                                  C.c_int, C.c_int, C.c_int64, C.POINTER(C.c_void_p), C.POINTER(C.c_int64),
                                  np.ctypeslib.ndpointer(np.uint64, flags="C_CONTIGUOUS"),
                                  C.POINTER(C.c_double)]
        _ref[penn] = lib
    return _ref[penn]


def port():
    global _port
    if _port is None:
        lib = C.CDLL(PORT_SO)
        lib.nbo_philox4x32_10.argtypes = [_u32p, _u32p, _u32p]
        lib.nbo_u01.restype = C.c_float
        lib.nbo_u01.argtypes = [C.c_uint32]
        lib.nbo_secondary_uid.restype = C.c_uint64
        lib.nbo_secondary_uid.argtypes = [C.c_uint64, C.c_uint32]
        lib.nbo_triangle_intersect.restype = C.c_float
        lib.nbo_triangle_intersect.argtypes = [_f32p, _f32p, _f32p]
        lib.nbo_propagate_batch.argtypes = [C.c_void_p, _f32p, _f32p, _f32p, _i32p, _i32p, C.c_int64, _f32p, _i32p]
        lib.nbo_table1d_get.restype = C.c_float
        lib.nbo_table1d_get.argtypes = [C.c_void_p, C.c_float]
        lib.nbo_table2d_get.restype = C.c_float
        lib.nbo_table2d_get.argtypes = [C.c_void_p, C.c_float, C.c_float]
        lib.nbo_table2d_get_rounddown.restype = C.c_float
        lib.nbo_table2d_get_rounddown.argtypes = [C.c_void_p, C.c_float, C.c_float]
        lib.nbo_elastic.argtypes = [C.c_void_p, C.c_void_p, C.c_float, C.c_float]
        lib.nbo_inelastic.restype = C.c_int
        lib.nbo_inelastic.argtypes = [C.c_void_p, C.c_void_p, _f32p, C.c_void_p]
        lib.nbo_boundary.restype = C.c_int
        lib.nbo_boundary.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_float]
        lib.nbo_step.restype = C.c_int
        lib.nbo_step.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(C.c_int), C.c_void_p,
                                 C.POINTER(C.c_int)]
        lib.nbo_geom_counters.argtypes = [np.ctypeslib.ndpointer(np.uint64, flags="C_CONTIGUOUS")]
        lib.nbo_geom_counters_reset.argtypes = []
        lib.nbo_run.restype = C.c_int
        lib.nbo_run.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, _f32p, _u32p, C.c_uint64, C.c_uint64,
                                C.c_void_p, C.c_uint64, C.c_void_p, C.c_void_p, C.c_void_p]
        _port = lib
    return _port


# ---------------------------------------------------------------------------
# ctypes mirrors of nbx_oracle.h
# ---------------------------------------------------------------------------
class Geometry(C.Structure):
    _fields_ = [("octree_data", C.c_void_p), ("tri", C.c_void_p), ("tri_mat", C.c_void_p),
                ("center", C.c_float * 3), ("half", C.c_float * 3), ("max_extent", C.c_float)]


class Table1D(C.Structure):
    _fields_ = [("n", C.c_int), ("x_min", C.c_float), ("x_step", C.c_float), ("data", C.c_void_p)]


class Table2D(C.Structure):
    _fields_ = [("w", C.c_int), ("h", C.c_int), ("x_min", C.c_float), ("x_step", C.c_float),
                ("y_min", C.c_float), ("y_step", C.c_float), ("data", C.c_void_p)]


class Table3D(C.Structure):
    _fields_ = [("w", C.c_int), ("h", C.c_int), ("d", C.c_int), ("x_min", C.c_float), ("x_step", C.c_float),
                ("y_min", C.c_float), ("y_step", C.c_float), ("z_min", C.c_float), ("z_step", C.c_float),
                ("data", C.c_void_p)]


class Material(C.Structure):
    _fields_ = [("barrier", C.c_float), ("el_imfp", Table1D), ("el_icdf", Table2D), ("phonon_loss", C.c_float),
                ("recoil_const", C.c_float), ("in_imfp", Table1D), ("in_icdf", Table2D), ("ion", Table2D),
                ("fermi", C.c_float), ("band_gap", C.c_float), ("q", Table3D), ("ion3", Table3D)]


class Electron(C.Structure):
    _fields_ = [("pos", C.c_float * 3), ("dir", C.c_float * 3), ("E", C.c_float), ("mat", C.c_int32),
                ("last_tri", C.c_int32), ("tag", C.c_uint32), ("uid", C.c_uint64), ("step", C.c_uint32)]


class Params(C.Structure):
    _fields_ = [("seed", C.c_uint32), ("min_energy", C.c_float), ("max_energy", C.c_float), ("penn", C.c_int)]


class Counts(C.Structure):
    _fields_ = [("n_primaries", C.c_uint64), ("n_detected", C.c_uint64), ("n_dropped_records", C.c_uint64),
                ("n_elastic", C.c_uint64), ("n_inelastic", C.c_uint64), ("n_boundary", C.c_uint64),
                ("n_secondaries", C.c_uint64), ("n_steps", C.c_uint64)]


# ---------------------------------------------------------------------------
# Reference-side helpers
# ---------------------------------------------------------------------------
def _split_tris(tris):
    v = np.ascontiguousarray(tris["v"].reshape(-1, 9), np.float32)
    m = np.ascontiguousarray(np.stack([tris["mat_in"], tris["mat_out"]], 1), np.int32)
    return v, m


def ref_build_octree(tris):
    """Reference linearized octree: (octree_data, tri_geom[n,9], tri_mats[n,2], center, half)."""
    lib = ref()
    v, m = _split_tris(tris)
    data = C.POINTER(C.c_int32)()
    nd = C.c_int64()
    tg = C.POINTER(C.c_float)()
    tm = C.POINTER(C.c_int32)()
    nt = C.c_int64()
    c = np.zeros(3, np.float32)
    h = np.zeros(3, np.float32)
    rc = lib.nbref_build_octree(v, m, len(tris), C.byref(data), C.byref(nd), C.byref(tg), C.byref(tm),
                                C.byref(nt), c, h)
    if rc != 0:
        raise RuntimeError("reference octree build failed")
    od = np.ctypeslib.as_array(data, (nd.value,)).copy()
    geom = np.ctypeslib.as_array(tg, (nt.value * 9,)).copy().reshape(-1, 9) if nt.value else np.zeros((0, 9), np.float32)
    mats = np.ctypeslib.as_array(tm, (nt.value * 2,)).copy().reshape(-1, 2) if nt.value else np.zeros((0, 2), np.int32)
    for p in (data, tg, tm):
        lib.nbref_free(C.cast(p, C.c_void_p))
    return od, geom, mats, c, h


class RefGeometry:
    def __init__(self, tris):
        self.lib = ref()
        v, m = _split_tris(tris)
        self.h = self.lib.nbref_geometry_create(v, m, len(tris))
        if not self.h:
            raise RuntimeError("reference geometry creation failed")
        mn = np.zeros(3, np.float32)
        mx = np.zeros(3, np.float32)
        me = C.c_float()
        self.lib.nbref_geometry_info(self.h, mn, mx, C.byref(me))
        self.aabb_min, self.aabb_max, self.max_extent = mn, mx, me.value

    def propagate(self, pos, dirs, dist, ignore_tri, ignore_mat):
        n = len(dist)
        od = np.zeros(n, np.float32)
        ot = np.zeros(n, np.int32)
        self.lib.nbref_propagate(self.h, np.ascontiguousarray(pos, np.float32), np.ascontiguousarray(dirs, np.float32),
                                 np.ascontiguousarray(dist, np.float32), np.ascontiguousarray(ignore_tri, np.int32),
                                 np.ascontiguousarray(ignore_mat, np.int32), n, od, ot)
        return od, ot

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.nbref_geometry_destroy(self.h)
            self.h = None


class RefMaterial:
    """A .mat file loaded by the reference's own loaders: Kieft elastic with
    the Kieft inelastic model, or with ``penn`` the full Penn model (whose
    ``in_imfp`` / ``in_icdf`` are the Penn log-IMFP and log-omega ICDF, and
    whose 3-D tables are read with ``table3`` / ``eval3``)."""

    TABLES = {"el_imfp": 0, "el_icdf": 1, "in_imfp": 2, "in_icdf": 3, "ion": 4}
    TABLES3 = {"q": 0, "ion3": 1}

    def __init__(self, path, penn=False):
        self.penn = penn
        self.lib = ref(penn)
        self.h = self.lib.nbref_material_load(str(path).encode())
        if not self.h:
            raise RuntimeError("reference material load failed: %s" % path)
        info = np.zeros(6, np.float32)
        self.lib.nbref_material_info(self.h, info)
        (self.barrier, self.fermi, self.band_gap, self.phonon_loss, self.recoil_const, self.max_energy) = [
            float(x) for x in info]
        self.info = info

    def eval(self, which, x, y=None):
        x = np.ascontiguousarray(x, np.float32)
        y = np.ascontiguousarray(np.zeros_like(x) if y is None else y, np.float32)
        out = np.zeros_like(x)
        self.lib.nbref_material_eval(self.h, self.TABLES[which], x, y, len(x), out)
        return out

    def table(self, which):
        """(values, (x_min, x_step, y_min, y_step)) of one reference table."""
        dims = np.zeros(2, np.int32)
        sc = np.zeros(4, np.float32)
        self.lib.nbref_material_table(self.h, self.TABLES[which], None, dims, sc)
        out = np.zeros(int(dims[0]) * int(dims[1]), np.float32)
        self.lib.nbref_material_table(self.h, self.TABLES[which], out.ctypes.data, dims, sc)
        vals = out.reshape(int(dims[0]), int(dims[1])) if which not in ("el_imfp", "in_imfp") else out
        return vals, tuple(float(v) for v in sc)

    def eval3(self, which, x, y, z):
        x = np.ascontiguousarray(x, np.float32)
        y = np.ascontiguousarray(y, np.float32)
        z = np.ascontiguousarray(z, np.float32)
        out = np.zeros_like(x)
        if self.lib.nbref_material_eval3(self.h, self.TABLES3[which], x, y, z, len(x), out) != 0:
            raise RuntimeError("3-D tables exist only in the full Penn build")
        return out

    def table3(self, which):
        """(values[w][h][d], (x_min, x_step, y_min, y_step, z_min, z_step))."""
        dims = np.zeros(3, np.int32)
        sc = np.zeros(6, np.float32)
        if self.lib.nbref_material_table3(self.h, self.TABLES3[which], None, dims, sc) != 0:
            raise RuntimeError("3-D tables exist only in the full Penn build")
        out = np.zeros(int(np.prod(dims.astype(np.int64))), np.float32)
        self.lib.nbref_material_table3(self.h, self.TABLES3[which], out.ctypes.data, dims, sc)
        return out.reshape(tuple(int(d) for d in dims)), tuple(float(v) for v in sc)

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.nbref_material_destroy(self.h)
            self.h = None


def ref_run(tri_path, pri_path, mat_paths, seed=0x78C7E39B, energy_threshold=0.0, threads=0, count_events=False,
            max_primaries=-1, penn=False):
    """cpu_mt_main-style run of the reference CPU path (Kieft build, or the
    stock full Penn build with ``penn``).  Returns (records[RECORD_DTYPE],
    stats dict, seconds)."""
    from nebula_b200 import formats
    lib = ref(penn)
    arr = (C.c_char_p * len(mat_paths))(*[str(p).encode() for p in mat_paths])
    recs = C.c_void_p()
    nrec = C.c_int64()
    stats = np.zeros(5, np.uint64)
    secs = C.c_double()
    rc = lib.nbref_run(str(tri_path).encode(), str(pri_path).encode(), arr, len(mat_paths), seed, energy_threshold,
                       threads, 1 if count_events else 0, max_primaries, C.byref(recs), C.byref(nrec), stats,
                       C.byref(secs))
    if rc != 0:
        raise RuntimeError("reference run failed (%d)" % rc)
    buf = C.string_at(recs, nrec.value * 36) if nrec.value else b""
    lib.nbref_free(recs)
    records = np.frombuffer(buf, np.uint8).view(formats.RECORD_DTYPE).copy() if buf else np.zeros(0, formats.RECORD_DTYPE)
    keys = ["n_primaries", "n_detected", "n_intersect", "n_elastic", "n_inelastic"]
    return records, dict(zip(keys, [int(s) for s in stats])), secs.value


# ---------------------------------------------------------------------------
# Port-side helpers (C restatement), fed with the reference's own octree and
# material tables so it checks the product's kernels independently of the
# product's host-side builders.
# ---------------------------------------------------------------------------
class PortGeometry:
    def __init__(self, tris):
        od, geom, mats, c, h = ref_build_octree(tris)
        self.octree_data = np.ascontiguousarray(od, np.int32)
        self.tri = np.ascontiguousarray(geom, np.float32)
        self.tri_mat = np.ascontiguousarray(mats, np.int32)
        self.center, self.half = c, h
        # octree factory: max_extent = 2 * magnitude(halfsize) (geometry/octree.inl:247-253)
        hh = h.astype(np.float32)
        mag = np.float32(np.sqrt(np.float32(hh[0] * hh[0] + hh[1] * hh[1]) + np.float32(hh[2] * hh[2])))
        self.max_extent = np.float32(2) * mag
        self.s = Geometry(self.octree_data.ctypes.data, self.tri.ctypes.data, self.tri_mat.ctypes.data,
                          (C.c_float * 3)(*c), (C.c_float * 3)(*h), float(self.max_extent))

    def propagate(self, pos, dirs, dist, ignore_tri, ignore_mat):
        n = len(dist)
        od = np.zeros(n, np.float32)
        ot = np.zeros(n, np.int32)
        port().nbo_propagate_batch(C.byref(self.s), np.ascontiguousarray(pos, np.float32),
                                   np.ascontiguousarray(dirs, np.float32), np.ascontiguousarray(dist, np.float32),
                                   np.ascontiguousarray(ignore_tri, np.int32), np.ascontiguousarray(ignore_mat, np.int32),
                                   n, od, ot)
        return od, ot


class PortMaterial:
    """Material for the C restatement, built from the reference loader's own
    tables and axis parameters."""

    def __init__(self, ref_mat: RefMaterial):
        self.ref = ref_mat
        self.arrays = {}
        t = {}
        for name in ("el_imfp", "in_imfp"):
            a, (xm, xs, _, _) = ref_mat.table(name)
            a = np.ascontiguousarray(a, np.float32)
            self.arrays[name] = a
            t[name] = Table1D(len(a), xm, xs, a.ctypes.data)
        for name in ("el_icdf", "in_icdf") + (() if ref_mat.penn else ("ion",)):
            a, (xm, xs, ym, ys) = ref_mat.table(name)
            a = np.ascontiguousarray(a, np.float32)
            self.arrays[name] = a
            t[name] = Table2D(a.shape[0], a.shape[1], xm, xs, ym, ys, a.ctypes.data)
        if ref_mat.penn:
            # full Penn build: in_imfp / in_icdf above are the Penn tables
            t["ion"] = Table2D()
            for name in ("q", "ion3"):
                a, (xm, xs, ym, ys, zm, zs) = ref_mat.table3(name)
                a = np.ascontiguousarray(a, np.float32)
                self.arrays[name] = a
                t[name] = Table3D(a.shape[0], a.shape[1], a.shape[2], xm, xs, ym, ys, zm, zs, a.ctypes.data)
        else:
            t["q"] = Table3D()
            t["ion3"] = Table3D()
        self.s = Material(ref_mat.barrier, t["el_imfp"], t["el_icdf"], ref_mat.phonon_loss, ref_mat.recoil_const,
                          t["in_imfp"], t["in_icdf"], t["ion"], ref_mat.fermi, ref_mat.band_gap, t["q"], t["ion3"])


def port_materials(ref_mats):
    """Contiguous nbo_material array for the C restatement."""
    pms = [PortMaterial(m) for m in ref_mats]
    arr = (Material * len(pms))(*[p.s for p in pms])
    return pms, arr


def philox(ctr, key):
    out = np.zeros(4, np.uint32)
    port().nbo_philox4x32_10(np.ascontiguousarray(ctr, np.uint32), np.ascontiguousarray(key, np.uint32), out)
    return out


def port_run(pg: "PortGeometry", mats_arr, primaries_7f, tags, seed, max_energy, min_energy=0.0,
             uid_base=0, records_cap=0, per_primary=True, penn=False):
    """Run the C restatement; returns (counts dict, se_count, bse_count, records, geom_counters)."""
    from nebula_b200 import formats
    P = port()
    n = len(tags)
    prm = Params(seed, min_energy, max_energy, 1 if penn else 0)
    se = np.zeros(n, np.uint32) if per_primary else None
    bse = np.zeros(n, np.uint32) if per_primary else None
    recs = np.zeros(max(records_cap, 1), formats.RECORD_DTYPE)
    c = Counts()
    P.nbo_geom_counters_reset()
    rc = P.nbo_run(C.byref(pg.s), mats_arr, C.byref(prm), np.ascontiguousarray(primaries_7f, np.float32).reshape(-1),
                   np.ascontiguousarray(tags, np.uint32), uid_base, n, recs.ctypes.data if records_cap else None,
                   records_cap, se.ctypes.data if se is not None else None,
                   bse.ctypes.data if bse is not None else None, C.byref(c))
    if rc != 0:
        raise RuntimeError("oracle run failed")
    gc = np.zeros(2, np.uint64)
    P.nbo_geom_counters(gc)
    counts = {f: getattr(c, f) for f, _ in Counts._fields_}
    nrec = min(records_cap, counts["n_detected"] - counts["n_dropped_records"])
    return counts, se, bse, recs[:nrec], gc
