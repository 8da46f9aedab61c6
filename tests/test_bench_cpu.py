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
