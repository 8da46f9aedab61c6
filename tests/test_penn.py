"""Full Penn inelastic model on the GPU (the reference's stock physics,
physics_config.h:21-24 with physics/full_penn.h), through the C ABI.

* Table lookups: the Penn log-IMFP (1-D), log-omega ICDF (2-D), q ICDF
  (3-D, trilinear) and ionisation table (3-D, rounddown) bit-exact against
  the reference's stock build (oracle/_ref/libnbref_penn.so), including
  extrapolation beyond every axis.
* Single steps: against the C restatement fed the same Philox uniforms,
  within the tolerance of the Kieft step test.
* Whole runs: SE/BSE yields, exit spectra and events per primary against the
  stock reference CPU path (cpu_mt_main-style driver).
"""
import ctypes as C

import numpy as np
import pytest

import oracle
import nebula_b200 as nb
from nebula_b200 import formats, generators as g

pytestmark = pytest.mark.gpu


def _bits(a):
    a = np.ascontiguousarray(a, np.float32).copy()
    b = a.view(np.uint32)
    b[np.isnan(a)] = 0x7FC00000
    return b


def _need_penn_ref():
    if not oracle.have_ref(penn=True):
        pytest.skip("reference full Penn build unavailable")


@pytest.mark.parametrize("mat", ["si", "w"])
def test_penn_tables_bit_exact_vs_reference(inputs, oracle_built, mat):
    _need_penn_ref()
    ctx = nb.setup(inputs["cube"], [inputs[mat]], device=0, inelastic="penn")
    rm = oracle.RefMaterial(inputs[mat], penn=True)
    rng = np.random.default_rng(9)
    n = 100000
    x = rng.uniform(-1.0, 10.5, n).astype(np.float32)
    w = rng.uniform(-0.2, 1.2, n).astype(np.float32)
    wl = rng.uniform(-11.0, 0.5, n).astype(np.float32)
    ctr = np.stack([np.arange(n), np.ones(n), np.full(n, 3), np.zeros(n)], 1).astype(np.uint32)
    bits = ctx.philox(ctr, np.tile(np.array([[77, 0]], np.uint32), (n, 1)))[:, 0]
    u = ((bits >> 9).astype(np.float32) * np.float32(1.1920928955078125e-07)
         + np.float32(5.9604644775390625e-08)).astype(np.float32)
    for name in ("in_imfp", "in_icdf"):   # Penn log-IMFP and log-omega ICDF
        assert np.array_equal(_bits(ctx.table_query(0, name, x, u)), _bits(rm.eval(name, x, u))), name
    assert np.array_equal(_bits(ctx.table3_query(0, "q", x, w, u)), _bits(rm.eval3("q", x, w, u)))
    assert np.array_equal(_bits(ctx.table3_query(0, "ion3", x, wl, u)), _bits(rm.eval3("ion3", x, wl, u)))
    with pytest.raises(nb.NbxError):
        ctx.table_query(0, "ion", x[:4], u[:4])   # no Kieft ionisation table under full Penn
    ctx.close()


def test_penn_model_needs_penn_tables(inputs, tmp_path):
    path = g.make_material(str(tmp_path / "kieft_only.mat"), "si", penn=False)
    ctx = nb.Context(device=0, inelastic="penn")
    with pytest.raises(nb.NbxError):
        ctx.add_material(nb.HostMaterial(path))
    ctx.close()
    ctx = nb.Context(device=0)
    with pytest.raises(nb.NbxError):
        ctx.table3_query(0, "q", [0.0], [0.0], [0.0])
    ctx.close()


def test_penn_step_vs_restatement(inputs, oracle_built):
    """One step per electron on the GPU and in the C restatement (stock
    tables, same Philox uniforms): vacuum steps bit-exact, material steps
    within 1e-4 for at least 99.9 %."""
    _need_penn_ref()
    tris = inputs["grating"]
    ctx = nb.setup(tris, [inputs["si"]], device=0, seed=41, inelastic="penn")
    pg = oracle.PortGeometry(tris)
    rm = oracle.RefMaterial(inputs["si"], penn=True)
    pms, arr = oracle.port_materials([rm])
    prm = oracle.Params(41, 0.0, rm.max_energy, 1)
    rng = np.random.default_rng(12)
    n = 20000
    e0 = np.zeros(n, nb.ELECTRON_DTYPE)
    e0["pos"] = np.array([-200, -200, -50], np.float32) + np.array([400, 400, 130], np.float32) * rng.random((n, 3))
    d = rng.normal(size=(n, 3))
    e0["dir"] = d / np.linalg.norm(d, axis=1, keepdims=True)
    e0["E"] = np.exp(rng.uniform(np.log(13.0), np.log(1500.0), n))
    e0["mat"] = rng.choice(np.array([-123, 0], np.int32), n)
    e0["last_tri"] = -1
    e0["tag"] = np.arange(n)
    e0["uid"] = rng.integers(0, 2 ** 62, n, dtype=np.uint64)
    e0["step"] = rng.integers(0, 1000, n)
    ge, gst, gev, gse, ghs = ctx.step_query(e0)
    P = oracle.port()
    close = material_steps = inelastic = with_se = 0
    for i in range(n):
        el = oracle.Electron()
        C.memmove(C.byref(el), e0[i:i + 1].ctypes.data, 52)
        el.uid = int(e0["uid"][i])
        el.step = int(e0["step"][i])
        ev = C.c_int()
        hs = C.c_int()
        se = oracle.Electron()
        st = P.nbo_step(C.byref(pg.s), arr, C.byref(prm), C.byref(el), C.byref(ev), C.byref(se), C.byref(hs))
        if e0["mat"][i] < 0:
            assert st == gst[i] and ev.value == gev[i], i
            continue
        material_steps += 1
        inelastic += ev.value == 1
        ok = (st == gst[i] and ev.value == gev[i] and hs.value == ghs[i]
              and np.allclose(np.array(el.pos), ge["pos"][i], rtol=1e-4, atol=1e-4)
              and np.allclose(np.array(el.dir), ge["dir"][i], rtol=1e-3, atol=1e-4)
              and abs(el.E - ge["E"][i]) <= 1e-4 * max(1.0, abs(el.E)))
        if ok and hs.value:
            with_se += 1
            ok = (abs(se.E - gse["E"][i]) <= 1e-3 * max(1.0, abs(se.E))
                  and np.allclose(np.array(se.dir), gse["dir"][i], rtol=1e-3, atol=1e-3))
        close += ok
    assert material_steps > n // 3 and inelastic > 200 and with_se > 50
    assert close >= 0.999 * material_steps, (close, material_steps)
    ctx.close()


def test_penn_whole_run_vs_reference_cpu(inputs, oracle_built, tmp_path):
    """Cube, 3 x 10^4 primaries at 1 keV with the full Penn model: per-primary
    SE/BSE yields within 3 sigma of the stock reference CPU path, exit
    spectrum chi-square within 3 sqrt(2 dof), events per primary within 5 %."""
    _need_penn_ref()
    n = 30000
    recs = g.point_beam(n, 1000.0, pos=(0.0, 0.0, 1.0))
    recs["px"] = np.arange(n)
    pri = str(tmp_path / "penn.pri")
    formats.write_pri(pri, recs)
    ref_recs, st, _ = oracle.ref_run(inputs["cube_tri"], pri, [inputs["si"]], seed=2, threads=1, count_events=True,
                                     penn=True)
    ctx = nb.setup(inputs["cube"], [inputs["si"]], device=0, seed=6, record_detected=True, inelastic="penn")
    ctx.reset_tallies()
    ctx.push_records(recs)
    ctx.run()
    s = ctx.stats()
    se, bse = (a.astype(np.float64) for a in ctx.tag_counts(0, n))
    det = ctx.flush_detected()
    px = ref_recs["px"].astype(np.int64)
    se_r = np.bincount(px[ref_recs["E"] < 50], minlength=n).astype(np.float64)
    bse_r = np.bincount(px[ref_recs["E"] >= 50], minlength=n).astype(np.float64)
    for a, b in ((se, se_r), (bse, bse_r)):
        z = (a.mean() - b.mean()) / np.sqrt(a.var() / n + b.var() / n)
        assert abs(z) < 3, (a.mean(), b.mean(), z)
    bins = np.concatenate([np.arange(0, 50, 2.0), np.arange(50, 1001, 50.0)])
    h_g = np.histogram(det["E"], bins)[0].astype(float)
    h_r = np.histogram(ref_recs["E"], bins)[0].astype(float)
    m = (h_g + h_r) > 0
    k1, k2 = np.sqrt(h_r.sum() / h_g.sum()), np.sqrt(h_g.sum() / h_r.sum())
    chi2 = (((k1 * h_g - k2 * h_r) ** 2) / (h_g + h_r))[m].sum()
    dof = m.sum() - 1
    assert abs(chi2 - dof) <= 3 * np.sqrt(2 * dof), (chi2, dof)
    ev_g = (s["events_elastic"] + s["events_inelastic"] + s["events_boundary"]) / n
    ev_r = (st["n_intersect"] + st["n_elastic"] + st["n_inelastic"]) / n
    assert abs(ev_g - ev_r) / ev_r < 0.05, (ev_g, ev_r)
    ctx.close()
