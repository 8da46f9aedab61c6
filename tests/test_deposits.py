"""Energy-deposit recording (the reference's energydeposit_cpu_driver and
cpu_energydep.cpp), on the GPU through the C ABI and the CLI.

* Recording deposits leaves the transport unchanged: same tallies and steps
  as a plain run with the same seed.
* Every record is a scattering event that changed the energy: one per such
  event, with a positive energy loss and the primary's tag.
* Against the reference's own nebula_cpu_energydep (Kieft and stock full
  Penn builds): deposits per primary, energy deposited per primary and its
  depth (dE-weighted mean z and a coarse depth profile) agree within a few
  sigma of the per-primary spread.
"""
import os
import subprocess

import numpy as np
import pytest

import oracle
import nebula_b200 as nb
from nebula_b200 import formats, generators as g

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DEP28 = np.dtype([("pos", "<f4", (3,)), ("E", "<f4"), ("dE", "<f4"), ("px", "<i4"), ("py", "<i4")])


def _run(ctx, recs):
    ctx.reset_tallies()
    ctx.push_records(recs)
    ctx.run()
    return ctx.stats(), ctx.tag_counts(0, len(recs))


def _beam(n, energy):
    recs = g.point_beam(n, energy, pos=(0.0, 0.0, 1.0))
    recs["px"] = np.arange(n)
    return recs


def test_deposits_leave_transport_unchanged(inputs):
    recs = _beam(3000, 1000.0)
    plain = nb.setup(inputs["cube"], [inputs["si"]], device=0, seed=21)
    dep = nb.setup(inputs["cube"], [inputs["si"]], device=0, seed=21, record_deposits=True)
    sp, (sep, bsep) = _run(plain, recs)
    sd, (sed, bsed) = _run(dep, recs)
    assert sp["steps"] == sd["steps"]
    assert np.array_equal(sep, sed) and np.array_equal(bsep, bsed)
    d = dep.flush_deposits()
    assert len(d) == sd["deposits"] > 0 and sd["deposits_dropped"] == 0
    assert len(d) <= sd["events_elastic"] + sd["events_inelastic"]
    assert len(d) >= 0.9 * (sd["events_elastic"] + sd["events_inelastic"])
    assert np.all(d["dE"] > 0) and np.all(d["tag"] < len(recs))
    assert len(dep.flush_deposits()) == 0           # flushed records are gone
    # a second run appends from an empty buffer again
    _run(dep, recs[:500])
    assert len(dep.flush_deposits()) == dep.stats()["deposits"]
    plain.close()
    dep.close()


def test_deposit_buffer_overflow_is_counted(inputs):
    recs = _beam(200, 1000.0)
    ctx = nb.setup(inputs["cube"], [inputs["si"]], device=0, seed=3, record_deposits=True,
                   deposit_capacity=1 << 12)
    s, _ = _run(ctx, recs)
    d = ctx.flush_deposits()
    assert s["deposits_dropped"] > 0 and len(d) == s["deposits"] <= (1 << 12)
    ctx.close()


def _per_primary(pos_z, dE, px, n, edges):
    cnt = np.bincount(px, minlength=n).astype(float)
    tot = np.bincount(px, weights=dE, minlength=n)
    zsum = np.bincount(px, weights=dE * pos_z, minlength=n)
    prof = np.stack([np.bincount(px, weights=dE * ((pos_z >= lo) & (pos_z < hi)), minlength=n)
                     for lo, hi in zip(edges[:-1], edges[1:])], 1)
    return cnt, tot, zsum, prof


@pytest.mark.parametrize("model", ["kieft", "penn"])
def test_deposits_vs_reference_cpu_energydep(inputs, oracle_built, tmp_path, model):
    binary = os.path.join(ROOT, "oracle", "_ref",
                          "nebula_cpu_energydep" + ("_kieft" if model == "kieft" else ""))
    if not os.path.exists(binary):
        pytest.skip("reference energy-deposit program unavailable")
    n = 4000
    recs = _beam(n, 1000.0)
    pri = str(tmp_path / "p.pri")
    formats.write_pri(pri, recs)
    dep_file = str(tmp_path / "dep.bin")
    r = subprocess.run([binary, "--seed=9", "--detect-filename=" + str(tmp_path / "det.bin"),
                        "--deposit-filename=" + dep_file, inputs["cube_tri"], pri, inputs["si"]],
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-500:]
    ref = np.fromfile(dep_file, DEP28)
    ctx = nb.setup(inputs["cube"], [inputs["si"]], device=0, seed=17, record_deposits=True, inelastic=model)
    _run(ctx, recs)
    mine = ctx.flush_deposits()
    ctx.close()
    edges = np.array([-1e9, -40.0, -20.0, -10.0, -5.0, -2.0, 0.0, 1e9])
    a = _per_primary(mine["pos"][:, 2].astype(float), mine["dE"].astype(float), mine["tag"].astype(np.int64), n,
                     edges)
    b = _per_primary(ref["pos"][:, 2].astype(float), ref["dE"].astype(float), ref["px"].astype(np.int64), n, edges)
    for qa, qb, what in ((a[0], b[0], "deposits"), (a[1], b[1], "energy"), (a[2], b[2], "z moment")):
        z = (qa.mean() - qb.mean()) / np.sqrt(qa.var() / n + qb.var() / n)
        assert abs(z) < 3.5, (what, qa.mean(), qb.mean(), z)
    for k in range(len(edges) - 1):
        qa, qb = a[3][:, k], b[3][:, k]
        if qa.var() + qb.var() == 0:
            continue
        z = (qa.mean() - qb.mean()) / np.sqrt(qa.var() / n + qb.var() / n)
        assert abs(z) < 4, ("depth bin", k, qa.mean(), qb.mean(), z)


def test_cli_energy_deposit_mode(inputs, tmp_path):
    cli = os.path.join(ROOT, "nebula_b200", "nebula_b200")
    if not os.path.exists(cli):
        pytest.skip("CLI not built")
    recs = _beam(1500, 1000.0)
    pri = str(tmp_path / "p.pri")
    formats.write_pri(pri, recs)
    det, dep = str(tmp_path / "det.bin"), str(tmp_path / "dep.bin")
    r = subprocess.run([cli, "--energy-deposit", "1", "--prescan-size", "200", "--detect-filename", det,
                        "--deposit-filename", dep, inputs["cube_tri"], pri, inputs["si"]],
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-500:]
    d = np.fromfile(dep, DEP28)
    e = np.fromfile(det, formats.RECORD_DTYPE)
    assert len(d) > 100 * len(recs) and len(e) > 0
    assert np.all(d["dE"] > 0) and set(np.unique(d["px"])) <= set(range(len(recs)))
    assert np.all(d["py"] == 0)
