"""bench.py's host-side helpers, without a GPU: workload definitions,
per-workload defaults and the CPU samples."""
import argparse
import importlib.util
import os

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _bench():
    spec = importlib.util.spec_from_file_location("bench_under_test", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def test_workloads_merge_scan_definitions():
    b = _bench()
    from nebula_b200 import generators as g
    for name in ("grating", "rough", "holes"):
        w = b.workload(name)
        for k in ("nx", "ny", "per_pixel", "energy", "materials", "rows", "cpu_sample", "ref_sample"):
            assert k in w, (name, k)
        assert w["nx"] == g.SCANS[name]["nx"]
    assert b.workload("holes")["materials"] == ("sio2", "w", "si")


def test_configure_defaults_and_description():
    b = _bench()
    for name, rows in (("grating", 256), ("rough", 512), ("holes", 64)):
        args = argparse.Namespace(workload=name, rows=0)
        b.configure(args)
        assert args.rows == rows
        assert b.NX == b.workload(name)["nx"]
    args = argparse.Namespace(workload="holes", rows=16)
    b.configure(args)
    assert "16 pixel rows (3276800 primaries)" in b.WORKLOAD
    args = argparse.Namespace(workload="grating", rows=10**6)
    b.configure(args)
    assert args.rows == 256


def test_strided_sample_spans_the_scan():
    b = _bench()
    from nebula_b200 import generators as g
    recs = g.scan_beam(16, 8, 10, 500.0, seed=1)
    sub = b.strided_sample(recs, 64)
    assert len(sub) == 64
    assert set(np.unique(sub["py"])) == set(range(8))      # every row represented
    assert b.strided_sample(recs, 10**6) is recs


def test_simulation_time_parsing():
    b = _bench()
    log = "Loading...\n\rProgress 100%\n\nSimulation successful!\n\n                     Simulation: 13.001\n"
    assert b._simulation_seconds(log) == 13.001
    assert b._simulation_seconds("no timing here") is None


def test_fom_does_not_grow_with_the_number_of_steps():
    """The plain figure of merit uses each step's own per-primary variance.
    On synthetic per-tag counts whose per-pixel means differ strongly (every
    step repeats the same pixels), the estimate is the same for 1, 3 and 20
    steps and matches the analytic per-primary variance; the variance of the
    counts summed over K steps (divided by K) instead grows like K times the
    spread of the pixel means."""
    b = _bench()
    rng = np.random.default_rng(3)
    n_pix, per = 400, 50
    mu = np.repeat(rng.uniform(0.1, 2.0, n_pix), per)      # per-primary mean, fixed by its pixel
    n = len(mu)
    true_var = float(np.mean(mu) + np.var(mu))               # Poisson counts: E[Var] + Var[E]
    t = 0.35
    foms, old = {}, {}
    for k in (1, 3, 20):
        steps = [rng.poisson(mu) for _ in range(k)]
        foms[k] = b.plain_fom([b.step_moments(c)[1] for c in steps], n, [t] * k)
        summed = np.sum(steps, axis=0).astype(np.float64)
        old[k] = 1.0 / (np.var(summed) / k / (n * k) * (t * k))
    expected = 1.0 / (true_var / n * t)
    for k, f in foms.items():
        assert abs(f / expected - 1) < 0.03, (k, f, expected)
    assert abs(foms[20] / foms[1] - 1) < 0.03
    assert old[20] / old[1] < 0.5          # the summed-count estimator drifts with K
    assert b.fom(0.0, n, t) is None and b.fom(1.0, n, 0.0) is None


def test_reference_gpu_program_refused_on_contact_holes(tmp_path):
    """The reference's GPU program stops making progress on the contact-hole
    scan: bench.py refuses to run it there and says why, without running
    anything."""
    b = _bench()
    out = b.reference_gpu("/nonexistent.tri", [], np.zeros(0), str(tmp_path), workload="holes")
    assert "unavailable" in out and "stalls" in out["unavailable"]
    assert "holes" in b.REFERENCE_GPU_STALLS
