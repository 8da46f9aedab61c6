"""Host-side builders against the reference's own code (oracle/_ref):
the linearized octree must be word-for-word identical (it fixes the
traversal order, hence bit-exact ray results), and the material tables
bit-identical to the reference loaders' output."""
import numpy as np
import pytest

import nebula_b200 as nb
from nebula_b200 import formats, generators as g


def _compare_octree(oracle, tris):
    od, geom, mats, c, h = oracle.ref_build_octree(tris)
    ho = nb.HostOctree(nb.triangles_from_tri_array(tris))
    t = ho.triangles
    mine = np.concatenate([t["r0"], t["e1"], t["e2"]], 1)
    assert np.array_equal(od, ho.octree_data)
    assert np.array_equal(geom.view(np.uint32), mine.view(np.uint32))
    assert np.array_equal(mats, np.stack([t["mat_in"], t["mat_out"]], 1))
    assert np.array_equal(c.view(np.uint32), ho.center.view(np.uint32))
    assert np.array_equal(h.view(np.uint32), ho.halfsize.view(np.uint32))
    return ho


@pytest.mark.parametrize("name", ["cube", "grating", "rough", "holes"])
def test_octree_layout_identical(oracle_built, inputs, name):
    ho = _compare_octree(oracle_built, inputs[name])
    assert len(ho.octree_data) >= 8


def test_octree_duplicates_and_soup(oracle_built):
    rng = np.random.default_rng(5)
    n = 3000
    v = rng.normal(0, 50, (n, 3, 3)).astype(np.float32)
    v[100:110] = v[0:10]                      # exact duplicates
    v[200:205] = v[20:25][:, [1, 2, 0]]       # cyclic permutations
    tris = np.zeros(n, formats.TRI_DTYPE)
    tris["v"] = v
    tris["mat_in"] = 0
    tris["mat_out"] = -123
    ho = _compare_octree(oracle_built, tris)
    assert ho.duplicates_dropped > 0


def test_octree_deep_split(oracle_built):
    # many tiny triangles clustered at one point force splits to max depth
    rng = np.random.default_rng(9)
    n = 400
    base = rng.normal(0, 1e-3, (n, 1, 3))
    v = (base + rng.normal(0, 1e-4, (n, 3, 3))).astype(np.float32)
    far = np.array([[[-100, -100, -100], [100, -100, -100], [0, 100, 100]]], np.float32)
    v = np.concatenate([v, far])
    tris = np.zeros(len(v), formats.TRI_DTYPE)
    tris["v"] = v
    tris["mat_in"] = 0
    tris["mat_out"] = -123
    ho = _compare_octree(oracle_built, tris)
    assert ho.max_depth >= 10


@pytest.mark.parametrize("mat", ["si", "sio2", "w"])
def test_material_tables_identical(oracle_built, inputs, mat):
    rm = oracle_built.RefMaterial(inputs[mat])
    hm = nb.HostMaterial(inputs[mat])
    for name in ("el_imfp", "in_imfp", "el_icdf", "in_icdf", "ion"):
        a, sa = rm.table(name)
        b, sb = hm.tables[name]
        assert a.shape == b.shape, name
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32)), name
        assert np.array_equal(np.float32(sa), np.float32(sb)), name
    for k, v in zip(("barrier", "fermi", "band_gap", "phonon_loss", "recoil_const", "max_energy"), rm.info):
        assert np.float32(getattr(hm, k)) == np.float32(v), k


@pytest.mark.parametrize("mat", ["si", "sio2", "w"])
def test_penn_tables_identical(oracle_built, inputs, mat):
    """Full Penn tables of the host loader against the stock reference build's
    full_penn::create (physics/full_penn.h:296-392): bit-identical values and
    axis parameters, including the 3-D q ICDF and ionisation tables."""
    if not oracle_built.have_ref(penn=True):
        pytest.skip("reference full Penn build unavailable")
    rm = oracle_built.RefMaterial(inputs[mat], penn=True)
    hm = nb.HostMaterial(inputs[mat])
    assert hm.has_penn and hm.has_kieft_inelastic
    for ref_name, host_name in (("in_imfp", "penn_imfp"), ("in_icdf", "penn_omega_icdf")):
        a, sa = rm.table(ref_name)
        b, sb = hm.tables[host_name]
        assert a.shape == b.shape, host_name
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32)), host_name
        assert np.array_equal(np.float32(sa), np.float32(sb)), host_name
    for ref_name, host_name in (("q", "penn_q_icdf"), ("ion3", "penn_ion")):
        a, sa = rm.table3(ref_name)
        b, sb = hm.tables[host_name]
        assert a.shape == b.shape, host_name
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32)), host_name
        assert np.array_equal(np.float32(sa), np.float32(sb)), host_name
    # the reference's max energy is the minimum over the stock mechanisms
    assert np.float32(hm.penn_max_energy) == np.float32(rm.max_energy)
    assert np.float32(hm.fermi) == np.float32(rm.fermi) and np.float32(hm.band_gap) == np.float32(rm.band_gap)
