"""Nebula file formats: ``.tri`` geometry, ``.pri`` primaries, detected records.

* ``.tri``: text, one triangle per line, 11 columns
  ``material_in material_out x0 y0 z0 x1 y1 z1 x2 y2 z2`` (nm), ``#`` comments
  (``source/io/load_tri_file.cpp:8-60``).
* ``.pri``: binary, 36-byte records ``float pos[3], dir[3], E; int32 px, py``
  (``source/io/load_pri_file.cpp:134-246``).
* detected electrons: binary, the same 36-byte record layout, written by the
  simulators to stdout (``source/cpu_mt_main.cpp:183-190``,
  ``source/gpu_main.cu:199-206``).
"""
from __future__ import annotations

import numpy as np

# Special material indices (source/core/cpu_material_manager.h:82-91).
NOP = -128
TERMINATOR = -127
DETECTOR = -126
DETECTOR_LT50 = -125
DETECTOR_GE50 = -124
VACUUM = -123
MIRROR = -122

RECORD_DTYPE = np.dtype([
    ("pos", "<f4", (3,)),
    ("dir", "<f4", (3,)),
    ("E", "<f4"),
    ("px", "<i4"),
    ("py", "<i4"),
])
assert RECORD_DTYPE.itemsize == 36

# Triangle table: vertices as float32 (3 vertices x 3 coordinates) + materials.
TRI_DTYPE = np.dtype([
    ("mat_in", "<i4"),
    ("mat_out", "<i4"),
    ("v", "<f4", (3, 3)),
])


def write_tri(path, tris: np.ndarray) -> None:
    """Write a TRI_DTYPE array as a ``.tri`` text file (float32-exact)."""
    with open(path, "w") as f:
        f.write("# in out x0 y0 z0 x1 y1 z1 x2 y2 z2 (nm)\n")
        v = tris["v"].reshape(-1, 9).astype(np.float32)
        for mi, mo, row in zip(tris["mat_in"], tris["mat_out"], v):
            f.write("%d %d %s\n" % (mi, mo, " ".join("%.9g" % float(c) for c in row)))


def read_tri(path) -> np.ndarray:
    """Read a ``.tri`` file with the reference's rules (11 columns, ``#`` comments)."""
    rows = []
    with open(path) as f:
        for line_num, line in enumerate(f, start=2):
            s = line.strip()
            if not s or s.startswith("#"):
                continue
            cols = s.split()
            if len(cols) != 11:
                raise ValueError("invalid number of columns in line '%d'" % line_num)
            rows.append((int(cols[0]), int(cols[1]), [float(c) for c in cols[2:]]))
    out = np.zeros(len(rows), TRI_DTYPE)
    for i, (a, b, c) in enumerate(rows):
        out[i]["mat_in"] = a
        out[i]["mat_out"] = b
        out[i]["v"] = np.asarray(c, np.float64).astype(np.float32).reshape(3, 3)
    return out


def write_pri(path, recs: np.ndarray) -> None:
    np.ascontiguousarray(recs, RECORD_DTYPE).tofile(path)


def read_pri(path) -> np.ndarray:
    raw = np.fromfile(path, np.uint8)
    if raw.size % 36:
        raise ValueError("Unexpected end of primaries file")
    return raw.view(RECORD_DTYPE)


def read_detected(path_or_bytes) -> np.ndarray:
    if isinstance(path_or_bytes, (bytes, bytearray)):
        raw = np.frombuffer(path_or_bytes, np.uint8)
    else:
        raw = np.fromfile(path_or_bytes, np.uint8)
    n = raw.size // 36
    return raw[: n * 36].view(RECORD_DTYPE)


def make_records(pos, dirs, energy, px, py) -> np.ndarray:
    n = len(energy)
    r = np.zeros(n, RECORD_DTYPE)
    r["pos"] = pos
    r["dir"] = dirs
    r["E"] = energy
    r["px"] = px
    r["py"] = py
    return r
