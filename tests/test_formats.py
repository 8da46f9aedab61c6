"""File formats: the HDF5-subset writer/reader pair, .tri and .pri I/O, and
input validation (malformed files are rejected on the host)."""
import os

import numpy as np
import pytest

import nebula_b200 as nb
from nebula_b200 import formats, generators as g
from nebula_b200.h5mat import MatFile


def test_mat_roundtrip_values(inputs):
    m = nb.HostMaterial(inputs["si"])
    assert m.name == "Si-like"
    assert m.barrier == np.float32(12.6)
    assert m.fermi == np.float32(7.8)
    assert m.band_gap == np.float32(1.12)
    assert m.phonon_loss == np.float32(0.063)
    # elastic IMFP written in m^-1 must come back as log(imfp / nm^-1)
    K = g._geomspace(1.0, 1e4, 128)
    expect = np.log(g.elastic_imfp(K, 14, 49.94, 1.0))
    got, (xmin, xstep, _, _) = m.tables["el_imfp"]
    assert np.allclose(got, expect, rtol=1e-5, atol=1e-5)
    assert xmin == 0.0
    assert np.isclose(xstep, 127 / np.log(1e4), rtol=1e-6)
    icdf, (_, _, ymin, ystep) = m.tables["el_icdf"]
    assert icdf.shape == (128, 256) and icdf.min() >= -1 and icdf.max() <= 1
    assert ymin == 0.0 and ystep == 255.0
    ion, _ = m.tables["ion"]
    assert set(np.unique(ion)) <= {-1.0, np.float32(99.8)}


def test_mat_missing_band_gap_and_units(tmp_path):
    """W-like has no band_gap attribute: the loader falls back to -1 eV."""
    p = g.make_material(str(tmp_path / "w.mat"), "w")
    m = nb.HostMaterial(p)
    assert m.band_gap == -1.0


def test_mat_rejects_corrupt_files(tmp_path, inputs):
    raw = open(inputs["si"], "rb").read()
    bad = tmp_path / "trunc.mat"
    bad.write_bytes(raw[: len(raw) // 3])
    with pytest.raises(nb.NbxError):
        nb.HostMaterial(str(bad))
    notmat = tmp_path / "x.mat"
    notmat.write_bytes(b"not an hdf5 file at all" * 10)
    with pytest.raises(nb.NbxError):
        nb.HostMaterial(str(notmat))
    with pytest.raises(nb.NbxError):
        nb.HostMaterial(str(tmp_path / "missing.mat"))
    # a valid HDF5 file without the Kieft groups
    f = MatFile()
    f.set_property_quantity("barrier", 1.0, "eV")
    f.write(str(tmp_path / "empty.mat"))
    with pytest.raises(nb.NbxError):
        nb.HostMaterial(str(tmp_path / "empty.mat"))


def test_mat_unknown_unit_rejected(tmp_path):
    f = MatFile()
    f.set_property_quantity("barrier", 1.0, "furlong")
    f.group("/kieft/elastic")
    f.write(str(tmp_path / "u.mat"))
    with pytest.raises(nb.NbxError):
        nb.HostMaterial(str(tmp_path / "u.mat"))


def test_tri_roundtrip(tmp_path):
    tris = g.grating_geometry(n_lines=3, length=200.0)
    p = str(tmp_path / "g.tri")
    formats.write_tri(p, tris)
    back = formats.read_tri(p)
    assert np.array_equal(back["v"].view(np.uint32), tris["v"].view(np.uint32))
    lib_tris = nb.load_tri(p)
    expect = nb.triangles_from_tri_array(tris)
    assert np.array_equal(lib_tris.view(np.uint8), expect.view(np.uint8))


def test_tri_bad_columns(tmp_path):
    p = tmp_path / "bad.tri"
    p.write_text("# comment\n0 -123 0 0 0 1 0 0 0 1\n")
    with pytest.raises(ValueError):
        formats.read_tri(str(p))
    with pytest.raises(nb.NbxError):
        nb.load_tri(str(p))


def test_pri_roundtrip_and_truncation(tmp_path):
    recs = g.scan_beam(4, 4, 3, 500.0, seed=2)
    p = str(tmp_path / "a.pri")
    formats.write_pri(p, recs)
    assert os.path.getsize(p) == 36 * len(recs)
    back = formats.read_pri(p)
    assert np.array_equal(back.view(np.uint8), recs.view(np.uint8))
    open(p, "ab").write(b"\0" * 5)
    with pytest.raises(ValueError):
        formats.read_pri(p)


def test_record_dtype():
    assert formats.RECORD_DTYPE.itemsize == 36
    assert nb.DETECTED_DTYPE.itemsize == 32
    assert nb.ELECTRON_DTYPE.itemsize == 56
