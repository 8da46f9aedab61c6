"""Generate tests/golden/golden.json from the reference's own CPU code.

Run in an environment where oracle/_ref/libnbref.so has been built from the
reference source tree (oracle/Makefile).  The vectors are outputs of the
reference's octree<false>::propagate on two synthetic geometries of
nebula_b200.generators: the cube of cube_geometry() and a 2 x 2
contact-hole array (contact_hole_geometry(n_holes=2, seed=3)), so tests can
check the oracle and the kernels against them where the reference is not
available."""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import oracle  # noqa: E402
from nebula_b200 import generators as g  # noqa: E402


def rays(rng, tris, n, z_sigma, mean_dist, mats):
    """n rays through the geometry's box (half of them near z = 0), the
    current material drawn from `mats`, and the reference's answers."""
    rg = oracle.RefGeometry(tris)
    pos = (rg.aabb_min + (rg.aabb_max - rg.aabb_min) * rng.random((n, 3))).astype(np.float32)
    pos[: n // 2, 2] = rng.normal(0, z_sigma, n // 2).astype(np.float32)
    d = rng.normal(size=(n, 3)).astype(np.float32)
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    d = d.astype(np.float32)
    dist = rng.exponential(mean_dist, n).astype(np.float32)
    ign = np.full(n, -1, np.int32)
    imat = rng.choice(np.array(mats, np.int32), n)
    od, ot = rg.propagate(pos, d, dist, ign, imat)
    return {"pos": pos.tolist(), "dir": d.tolist(), "dist": dist.tolist(), "ignore_tri": ign.tolist(),
            "ignore_mat": imat.tolist(), "tri": ot.tolist(), "dist_bits": od.view(np.uint32).tolist()}


def main():
    rng = np.random.default_rng(2024)
    out = {"cube_rays": rays(rng, g.cube_geometry(), 256, 20.0, 200.0, [-123, 0])}
    # 2 x 2 contact holes: three materials, conforming curved walls
    out["holes_rays"] = rays(np.random.default_rng(2025), g.contact_hole_geometry(n_holes=2, seed=3), 256, 60.0, 40.0,
                             [-123, 0, 1, 2])
    with open(os.path.join(HERE, "golden.json"), "w") as f:
        json.dump(out, f)


if __name__ == "__main__":
    main()
