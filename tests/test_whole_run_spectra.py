"""Whole-run parity of the GPU path against the reference CPU path
(cpu_mt_main-style driver, cpu_mt_main.cpp:158-203) on subsamples of the
benchmark scans: per-pixel SE and BSE yields, the exit-energy spectrum and
the exit polar-angle spectrum of the detected electrons.

* Grating line scan (500 eV, 8 of the 256 pixel rows = 204,800 primaries),
  Kieft inelastic model and the stock full Penn model.
* Rough slab (526,334 triangles) with the mixed {0.3, 1, 3, 5} keV beam: a
  32 x 32-pixel subsample of the 512 x 512 scan (20,480 primaries), checked
  per beam energy, Kieft and full Penn.
* Contact holes (three materials): a 16 x 16-pixel patch over the middle
  hole of the 3 x 3 array at 1 keV (20,480 primaries), Kieft and full Penn.

Each detected record carries the electron's position, direction and energy
(cpu_mt_main.cpp:182-189 on the CPU; the GPU's nbx_flush_detected); the
polar angle is that of the direction, cos(theta) = dz / |d|.  The reference
runs on one thread, so for the fixed seeds both sides are deterministic and
the outcome of every check is reproducible.

Acceptance (3 sigma): per-pixel chi-square of the mean yields with sigma from
each side's per-primary sample variance (about the per-energy means for the
mixed beam), |chi2 - dof| <= 3 sqrt(2 dof); the
total yields by a two-sample z < 3; two-sample chi-square of the spectra on
bins merged to at least 20 pooled counts, |chi2 - dof| <= 3 sqrt(2 dof);
events per primary within 5 %."""
import numpy as np
import pytest

import oracle
import nebula_b200 as nb
from nebula_b200 import formats, generators as g

pytestmark = pytest.mark.gpu


def _chi2_ok(chi2, dof):
    return abs(chi2 - dof) <= 3 * np.sqrt(2 * dof)


def _pixel_chi2(c1, c2, pix, n_pix, strata=None):
    """Chi-square of per-pixel mean yields; each side's per-pixel sample
    variance (the side's pooled variance where a pixel's own is zero).

    strata (optional, one label per primary, the same on both sides, e.g.
    the beam energy): both sides simulate the same primaries, so the spread
    of the stratum means inside a pixel cancels in the difference of the
    pixel means; the variances are then taken of each side's residuals about
    its own stratum means."""
    def moments(c):
        r = c
        if strata is not None:
            _, k = np.unique(strata, return_inverse=True)
            r = c - (np.bincount(k, weights=c) / np.bincount(k))[k]
        n = np.bincount(pix, minlength=n_pix).astype(np.float64)
        mean = np.bincount(pix, weights=c, minlength=n_pix) / n
        rm = np.bincount(pix, weights=r, minlength=n_pix) / n
        r2 = np.bincount(pix, weights=r * r, minlength=n_pix)
        var = (r2 - n * rm * rm) / np.maximum(n - 1, 1)
        return n, mean, np.where(var > 0, var, max(r.var(), 1e-12))
    n1, m1, v1 = moments(c1)
    n2, m2, v2 = moments(c2)
    return float(((m1 - m2) ** 2 / (v1 / n1 + v2 / n2)).sum()), n_pix


def _z(a, b):
    return (a.mean() - b.mean()) / np.sqrt(a.var() / len(a) + b.var() / len(b))


def _merged_edges(pooled, fine_edges, min_count=20):
    """Fine bins merged left to right until each holds min_count pooled values
    (a leftover tail joins the last bin)."""
    h, _ = np.histogram(pooled, fine_edges)
    edges, acc = [fine_edges[0]], 0
    for i, c in enumerate(h):
        acc += c
        if acc >= min_count:
            edges.append(fine_edges[i + 1])
            acc = 0
    if acc and len(edges) > 1:
        edges[-1] = fine_edges[-1]
    return np.asarray(edges)


def _spectrum_chi2(x1, x2, fine_edges):
    """Two-sample chi-square of two samples' histograms (unequal totals)."""
    edges = _merged_edges(np.concatenate([x1, x2]), fine_edges)
    h1, _ = np.histogram(x1, edges)
    h2, _ = np.histogram(x2, edges)
    h1, h2 = h1.astype(np.float64), h2.astype(np.float64)
    n1, n2 = h1.sum(), h2.sum()
    m = (h1 + h2) > 0
    k1, k2 = np.sqrt(n2 / n1), np.sqrt(n1 / n2)
    chi2 = float((((k1 * h1 - k2 * h2) ** 2) / (h1 + h2))[m].sum())
    return chi2, int(m.sum()) - 1


def _energy_edges(e_max):
    """0.5 eV bins below 50 eV, 10 eV bins above."""
    return np.concatenate([np.arange(0.0, 50.0, 0.5), np.arange(50.0, e_max + 20.0, 10.0)])


ANGLE_EDGES = np.linspace(-1.0, 1.0, 81)


def _cos_polar(d):
    d = np.asarray(d, np.float64)
    return d[:, 2] / np.linalg.norm(d, axis=1)


def _tagged(recs):
    """The same primaries with the primary index as pixel x, so per-primary
    counts of the reference run can be recovered from its detected records."""
    t = recs.copy()
    t["px"] = np.arange(len(recs))
    t["py"] = 0
    return t


def _run_both(tri_array, tri_path, mats, recs, tmp_path, gpu_seed, ref_seed, penn=False):
    n = len(recs)
    pri = str(tmp_path / "scan.pri")
    formats.write_pri(pri, _tagged(recs))
    ref_recs, st, _ = oracle.ref_run(tri_path, pri, mats, seed=ref_seed, threads=1, count_events=True, penn=penn)
    ref_se = np.bincount(ref_recs["px"][ref_recs["E"] < 50], minlength=n).astype(np.float64)
    ref_bse = np.bincount(ref_recs["px"][ref_recs["E"] >= 50], minlength=n).astype(np.float64)
    ctx = nb.setup(tri_array, mats, device=0, seed=gpu_seed, record_detected=True,
                   inelastic="penn" if penn else "kieft")
    try:
        ctx.set_tag_range(n)
        ctx.push_records(recs)
        ctx.run()
        s = ctx.stats()
        se, bse = ctx.tag_counts(0, n)
        det = ctx.flush_detected()
    finally:
        ctx.close()
    assert s["records_dropped"] == 0 and s["queue_overflow"] == 0
    assert len(det) == s["detected"]
    ev_g = (s["events_elastic"] + s["events_inelastic"] + s["events_boundary"]) / n
    ev_r = (st["n_intersect"] + st["n_elastic"] + st["n_inelastic"]) / n
    return dict(se=se.astype(np.float64), bse=bse.astype(np.float64), det=det, ev=ev_g), \
        dict(se=ref_se, bse=ref_bse, det=ref_recs, ev=ev_r)


def _check_spectra(gpu_det, ref_det, e_max, what):
    chi2, dof = _spectrum_chi2(gpu_det["E"], ref_det["E"], _energy_edges(e_max))
    assert _chi2_ok(chi2, dof), ("exit-energy spectrum", what, chi2, dof)
    chi2, dof = _spectrum_chi2(_cos_polar(gpu_det["dir"]), _cos_polar(ref_det["dir"]), ANGLE_EDGES)
    assert _chi2_ok(chi2, dof), ("exit-angle spectrum", what, chi2, dof)
    # the low-energy (SE) part of the spectrum on its own, 0.5 eV bins
    lo_g, lo_r = gpu_det["E"][gpu_det["E"] < 50], ref_det["E"][ref_det["E"] < 50]
    chi2, dof = _spectrum_chi2(lo_g, lo_r, np.arange(0.0, 50.5, 0.5))
    assert _chi2_ok(chi2, dof), ("SE spectrum", what, chi2, dof)


def _grating_rows():
    w = g.SCANS["grating"]
    return g.scan_beam(w["nx"], w["ny"], w["per_pixel"], w["energy"], spacing=w["spacing"], origin=w["origin"],
                       z_start=w["z_start"], seed=41, rows=range(0, w["ny"], 32))


@pytest.mark.parametrize("model", ["kieft", "penn"])
def test_grating_8_rows_yields_and_spectra(inputs, oracle_built, tmp_path, model):
    """Grating scan, 8 pixel rows evenly spread over the 256 (204,800
    primaries at 500 eV): per-pixel SE/BSE chi-square over 2,048 pixels,
    cross-line profiles (the 8 rows averaged, 256 columns), total yields,
    exit-energy and exit-angle spectra, events per primary."""
    penn = model == "penn"
    if penn and not oracle.have_ref(penn=True):
        pytest.skip("reference full Penn build unavailable")
    recs = _grating_rows()
    n = len(recs)
    assert n == 204800
    gpu, ref = _run_both(inputs["grating"], inputs["grating_tri"], [inputs["si"]], recs, tmp_path,
                         gpu_seed=101, ref_seed=7, penn=penn)
    pixel = recs["py"].astype(np.int64) * 256 + recs["px"]
    _, pixel = np.unique(pixel, return_inverse=True)
    column = recs["px"].astype(np.int64)
    for key in ("se", "bse"):
        chi2, dof = _pixel_chi2(gpu[key], ref[key], pixel, 2048)
        assert _chi2_ok(chi2, dof), (model, key, "pixels", chi2, dof)
        chi2, dof = _pixel_chi2(gpu[key], ref[key], column, 256)
        assert _chi2_ok(chi2, dof), (model, key, "cross-line profile", chi2, dof)
        assert abs(_z(gpu[key], ref[key])) < 3, (model, key, gpu[key].mean(), ref[key].mean())
    _check_spectra(gpu["det"], ref["det"], 500.0, model)
    assert abs(gpu["ev"] - ref["ev"]) / ref["ev"] < 0.05, (gpu["ev"], ref["ev"])


@pytest.fixture(scope="module")
def rough_full(tmp_path_factory):
    """The benchmark's rough slab: 512 x 512 Gaussian height field (RMS 3 nm,
    correlation 10 nm) over 1 um, 526,334 triangles."""
    d = tmp_path_factory.mktemp("rough_full")
    tris = g.SCANS["rough"]["geometry"]()
    p = str(d / "rough.tri")
    formats.write_tri(p, tris)
    return tris, p


@pytest.mark.parametrize("model", ["kieft", "penn"])
def test_rough_slab_mixed_beam_per_energy(inputs, oracle_built, tmp_path, rough_full, model):
    """Rough slab with the mixed-energy beam: every 16th pixel row and column
    of the 512 x 512 scan (32 x 32 pixels x 20 primaries, energies drawn from
    {300, 1000, 3000, 5000} eV), Kieft model and the stock full Penn model.
    Per-pixel SE/BSE chi-square over the 1,024 pixels, and for each beam
    energy: SE and BSE yields, exit-energy and exit-angle spectra; events per
    primary over the whole sample."""
    penn = model == "penn"
    if penn and not oracle.have_ref(penn=True):
        pytest.skip("reference full Penn build unavailable")
    tris, tri_path = rough_full
    w = g.SCANS["rough"]
    recs = g.scan_beam(w["nx"], w["ny"], w["per_pixel"], w["energy"], spacing=w["spacing"], origin=w["origin"],
                       z_start=w["z_start"], seed=43, energies=w["energies"], rows=range(0, w["ny"], 16))
    recs = recs[recs["px"] % 16 == 0]
    n = len(recs)
    assert n == 32 * 32 * 20
    gpu, ref = _run_both(tris, tri_path, [inputs["si"]], recs, tmp_path, gpu_seed=103, ref_seed=11, penn=penn)
    pixel = (recs["py"].astype(np.int64) // 16) * 32 + recs["px"] // 16
    energy = recs["E"]
    for key in ("se", "bse"):
        chi2, dof = _pixel_chi2(gpu[key], ref[key], pixel, 1024, strata=energy)
        assert _chi2_ok(chi2, dof), (model, key, "pixels", chi2, dof)
    gpu_tag_E = energy[gpu["det"]["tag"]]
    ref_tag_E = energy[ref["det"]["px"]]
    for e0 in w["energies"]:
        sel = energy == np.float32(e0)
        assert sel.sum() > 4000
        for key in ("se", "bse"):
            assert abs(_z(gpu[key][sel], ref[key][sel])) < 3, (model, e0, key, gpu[key][sel].mean(),
                                                               ref[key][sel].mean())
        _check_spectra(gpu["det"][gpu_tag_E == np.float32(e0)], ref["det"][ref_tag_E == np.float32(e0)], e0,
                       "%s %g eV" % (model, e0))
    assert abs(gpu["ev"] - ref["ev"]) / ref["ev"] < 0.05, (gpu["ev"], ref["ev"])


@pytest.mark.parametrize("model", ["kieft", "penn"])
def test_contact_holes_patch_yields_and_spectra(inputs, oracle_built, tmp_path, model):
    """Three materials (SiO2-like film, W-like plugs, Si-like substrate) on
    the 3 x 3 contact-hole array: a 16 x 16-pixel patch at 5 nm spacing over
    the middle hole (walls, floor and the film around it), 80 primaries per
    pixel at 1 keV, Kieft and full Penn.  Per-pixel SE/BSE chi-square over
    the 256 pixels, total yields, exit-energy and exit-angle spectra, events
    per primary."""
    penn = model == "penn"
    if penn and not oracle.have_ref(penn=True):
        pytest.skip("reference full Penn build unavailable")
    recs = g.scan_beam(16, 16, 80, 1000.0, spacing=5.0, origin=(-37.5, -37.5), z_start=10.0, seed=47)
    n = len(recs)
    assert n == 16 * 16 * 80
    mats = [inputs["sio2"], inputs["w"], inputs["si"]]
    gpu, ref = _run_both(inputs["holes"], inputs["holes_tri"], mats, recs, tmp_path, gpu_seed=107, ref_seed=13,
                         penn=penn)
    pixel = recs["py"].astype(np.int64) * 16 + recs["px"]
    for key in ("se", "bse"):
        chi2, dof = _pixel_chi2(gpu[key], ref[key], pixel, 256)
        assert _chi2_ok(chi2, dof), (model, key, "pixels", chi2, dof)
        assert abs(_z(gpu[key], ref[key])) < 3, (model, key, gpu[key].mean(), ref[key].mean())
    _check_spectra(gpu["det"], ref["det"], 1000.0, "contact holes " + model)
    assert abs(gpu["ev"] - ref["ev"]) / ref["ev"] < 0.05, (gpu["ev"], ref["ev"])
