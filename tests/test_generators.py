"""The seeded geometry generators produce closed, consistently oriented
meshes: a ray from any point of a known region leaves it through a triangle
whose material on the ray's side is that region's material (the normal
points to the `mat_out` side, geometry/trimesh conventions of the .tri
format), and the contact-hole cells share their boundary vertices."""
from collections import Counter

import numpy as np

from nebula_b200 import formats, generators as g


def _first_hit(v, p, d):
    v0, e1, e2 = v[:, 0], v[:, 1] - v[:, 0], v[:, 2] - v[:, 0]
    pv = np.cross(d, e2)
    det = (e1 * pv).sum(1)
    with np.errstate(divide="ignore", invalid="ignore"):
        inv = 1.0 / det
        tv = p - v0
        u = (tv * pv).sum(1) * inv
        qv = np.cross(tv, e1)
        w = (qv @ d) * inv
        t = (qv * e2).sum(1) * inv
    hit = (np.abs(det) > 1e-12) & (u >= 0) & (w >= 0) & (u + w <= 1) & (t > 1e-9)
    if not hit.any():
        return -1
    return int(np.argmin(np.where(hit, t, np.inf)))


def _holes_region(p, n, pitch, radius, rough, depth, plug_depth, substrate):
    """Material at point p of the contact-hole geometry, None within the
    edge-roughness band of a hole wall."""
    half = n * pitch / 2
    x, y, z = p
    if abs(x) > half or abs(y) > half or z > 0 or z < -depth - substrate:
        return formats.VACUUM
    cx = -half + pitch * (np.clip(np.floor((x + half) / pitch), 0, n - 1) + 0.5)
    cy = -half + pitch * (np.clip(np.floor((y + half) / pitch), 0, n - 1) + 0.5)
    r = np.hypot(x - cx, y - cy)
    inside, outside = r < radius - rough - 0.5, r > radius + rough + 0.5
    if z > -depth:
        return formats.VACUUM if inside else (0 if outside else None)
    if z > -depth - plug_depth:
        return 1 if inside else (2 if outside else None)
    return 2


def test_contact_holes_closed_and_oriented():
    n = 2
    tris = g.contact_hole_geometry(n_holes=n, seed=3)
    keep = tris["mat_in"] != formats.DETECTOR
    t = tris[keep]
    v = t["v"].reshape(-1, 3, 3).astype(np.float64)
    nrm = np.cross(v[:, 1] - v[:, 0], v[:, 2] - v[:, 0])
    rng = np.random.default_rng(7)
    checked = 0
    for _ in range(1500):
        p = rng.uniform([-100, -100, -640], [100, 100, 10])
        reg = _holes_region(p, n, 80.0, 20.0, 2.0, 100.0, 50.0, 500.0)
        if reg is None:
            continue
        d = rng.normal(size=3)
        d /= np.linalg.norm(d)
        k = _first_hit(v, p, d)
        if k < 0:
            assert reg == formats.VACUUM, p
            continue
        side = t["mat_in"][k] if d @ nrm[k] > 0 else t["mat_out"][k]
        assert side == reg, (p, d, k)
        checked += 1
    assert checked > 800


def test_contact_hole_cells_share_vertices():
    """Inside the array every edge is shared by two triangles, or by four
    on the rings where the hole wall, the hole floor, the film/substrate
    interface and the plug wall meet; single edges lie only on the outer
    box, where the box faces meet the cells' boundary points."""
    n, n_theta = 2, 48
    tris = g.contact_hole_geometry(n_holes=n, n_theta=n_theta, seed=1)
    t = tris[tris["mat_in"] != formats.DETECTOR]
    pts = t["v"].reshape(-1, 3)
    _, vid = np.unique(pts, axis=0, return_inverse=True)
    vid = vid.reshape(-1, 3)
    edges = Counter()
    for a, b, c in vid:
        for e in ((a, b), (b, c), (c, a)):
            edges[(min(e), max(e))] += 1
    counts = Counter(edges.values())
    assert set(counts) <= {1, 2, 4}
    assert counts[4] == n * n * n_theta
    uniq = np.unique(pts, axis=0)
    half = n * 80.0 / 2
    for (a, b), c in edges.items():
        if c == 1:
            for q in (uniq[a], uniq[b]):
                assert abs(abs(q[0]) - half) < 1e-9 or abs(abs(q[1]) - half) < 1e-9


def test_streamed_scan_matches_blocks(tmp_path):
    """write_scan_pri streams the scan block by block: the file holds every
    pixel's primaries, in row-major order, and equals the concatenation of
    the per-block scans."""
    p = str(tmp_path / "s.pri")
    n = g.write_scan_pri(p, 24, 21, 3, 800.0, rows_per_block=8, seed=5, spacing=2.0, origin=(-24.0, -21.0))
    r = formats.read_pri(p)
    assert n == len(r) == 24 * 21 * 3
    assert np.array_equal(r["py"], np.repeat(np.arange(21), 24 * 3))
    blocks = [g.scan_beam(24, 21, 3, 800.0, seed=[5, k], rows=range(8 * k, min(21, 8 * k + 8)), spacing=2.0,
                          origin=(-24.0, -21.0)) for k in range(3)]
    assert np.array_equal(np.concatenate(blocks).view(np.uint8), r.view(np.uint8))


def test_workload_writer(tmp_path):
    out = g.write_workload("grating", str(tmp_path), rows=2)
    assert len(out["mats"]) == 1
    r = formats.read_pri(out["pri"])
    assert len(r) == 2 * 256 * 100 and set(np.unique(r["py"])) == {0, 1}
    assert len(formats.read_tri(out["tri"])) == len(g.grating_geometry())


def _side_material(v, nrm, t, p, d):
    k = _first_hit(v, p, d)
    if k < 0:
        return None
    return t["mat_in"][k] if d @ nrm[k] > 0 else t["mat_out"][k]


def test_grating_and_rough_consistently_oriented():
    """Any point seen from two random directions lies in the same material,
    and points above the top surface lie in vacuum: the grating and rough
    slab meshes are closed and their normals point to the mat_out side."""
    geoms = {"grating": (g.grating_geometry(n_lines=3, length=200.0), 60.0),
             "rough": (g.rough_geometry(n=24, size=100.0, seed=3), 20.0)}
    rng = np.random.default_rng(11)
    for name, (tris, z_top) in geoms.items():
        t = tris[tris["mat_in"] != formats.DETECTOR]
        v = t["v"].reshape(-1, 3, 3).astype(np.float64)
        nrm = np.cross(v[:, 1] - v[:, 0], v[:, 2] - v[:, 0])
        lo, hi = v.reshape(-1, 3).min(0), v.reshape(-1, 3).max(0)
        agree = 0
        for _ in range(400):
            p = rng.uniform(lo + 1.0, hi - 1.0)
            d1, d2 = rng.normal(size=3), rng.normal(size=3)
            m1 = _side_material(v, nrm, t, p, d1 / np.linalg.norm(d1))
            m2 = _side_material(v, nrm, t, p, d2 / np.linalg.norm(d2))
            if m1 is None or m2 is None:
                continue
            assert m1 == m2, (name, p, m1, m2)
            agree += 1
        assert agree > 300, (name, agree)
        # above the highest surface point: vacuum from any direction
        for _ in range(50):
            p = np.array([rng.uniform(lo[0] + 1, hi[0] - 1), rng.uniform(lo[1] + 1, hi[1] - 1), z_top])
            d = rng.normal(size=3)
            d[2] = -abs(d[2]) - 0.5
            m = _side_material(v, nrm, t, p, d / np.linalg.norm(d))
            assert m in (None, formats.VACUUM), (name, p, m)


def test_banded_disc_tiles_the_polygon():
    """The hole-floor disc (bands to inner rings, then a small fan) covers the
    rough polygon exactly once: its triangles' signed areas sum to the
    polygon's area, all with the orientation of the ring, and no vertex is
    shared by more than 12 triangles (below the octree's split count)."""
    rng = np.random.default_rng(4)
    n = 48
    th = 2 * np.pi * np.arange(n) / n
    r = 20.0 + rng.uniform(-2, 2, n)
    ring = np.stack([r * np.cos(th), r * np.sin(th), np.full(n, -100.0)], -1)[None]
    ctr = np.array([[0.0, 0.0, -100.0]])
    tris = g._disc(ctr, ring, 1, formats.VACUUM)
    v = tris["v"].astype(np.float64)
    area = 0.5 * ((v[:, 1, 0] - v[:, 0, 0]) * (v[:, 2, 1] - v[:, 0, 1]) -
                  (v[:, 1, 1] - v[:, 0, 1]) * (v[:, 2, 0] - v[:, 0, 0]))
    x, y = ring[0, :, 0], ring[0, :, 1]
    poly = 0.5 * np.sum(x * np.roll(y, -1) - np.roll(x, -1) * y)
    assert np.all(area > 0)
    assert abs(area.sum() - poly) < 1e-3 * poly
    assert len(tris) == 72 + 36 + 12
    _, vid = np.unique(v.reshape(-1, 3).astype(np.float32), axis=0, return_inverse=True)
    assert np.bincount(vid.ravel()).max() <= 12
