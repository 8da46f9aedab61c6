#!/usr/bin/env python
"""Benchmark: scattering events/s of the electron-transport hot path.

Workload (the reference's line-space grating SEM scan): Si-like lines 32 nm
wide at 64 nm pitch, 50 nm tall, 2 um long on a substrate (5,136 triangles);
256 x 256 pixels at 1 nm, 100 primaries per pixel at 500 eV (6,553,600
primaries), Gaussian spot sigma 1 nm with 0.5 deg divergence; synthetic
Si-like Kieft tables.  One step = one pass of the transport over the whole
scan (every primary and its full secondary cascade).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl nbx|reference]
                  [--workload grating|rough|holes] [--inelastic kieft|penn]

The other workloads are the rough slab with mixed beam energies and the
three-material contact-hole array (64 of its 1024 pixel rows per step).

Under torchrun the job is one frame of the scan per rank (fixed work per GPU:
weak scaling), sharded over the ranks by global primary index with
nebula_b200.replicas (each rank's random streams start at its shard's global
index), and the per-pixel FP64 sums are added up over the ranks with
replicas.reduce_pixel_yields once, after timing; no data-path collective.  Rank 0
prints one JSON line.  value = events/s over all ranks with the primaries
already resident in HBM (device time of nbx_run, CUDA events on the library's
stream, max over ranks); e2e = the same through the C ABI from pinned host
buffers, wall clock, max over ranks: every step stages the next step's
primaries (host-to-device copy on the library's copy stream, overlapping the
run), runs its own, reads the per-pixel yields back and queues the staged
primaries on the device.
"""
from __future__ import annotations

import argparse
import csv
import io
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "scattering events/s & SE-yield FOM 1/(σ²t): learned-RR vs plain, 1×B200 vs CPU"
NX = NY = 256
PER_PIXEL = 100
ENERGY = 500.0
WORKLOAD = "grating 256x256 px x 100 primaries @ 500 eV (6,553,600 primaries), 5,136 triangles, Si-like Kieft tables"

# Scans the bench can run (geometry, materials and raster scan in
# nebula_b200.generators.SCANS): the grating line scan (the headline
# workload), the rough-slab scan with mixed beam energies and the
# multi-material contact-hole array.  `rows` is the default pixel-row subset
# of one step, `cpu_sample` / `ref_sample` the primaries (evenly strided over
# the step's scan) of the CPU-baseline run and of each reference-arm step,
# `learned` the nearest-surface map and training scan of the learned leg
# (single-material workloads).
WORKLOADS = {
    "grating": dict(rows=256, cpu_sample=409600, ref_sample=102400, desc=WORKLOAD,
                    # config 4 as written: weight window 0.05, splitting above 0.5
                    learned=dict(map_lo=(-180, -180, -60), map_hi=(180, 180, 60), cell=1.0, d_max=20.0,
                                 train_per_pixel=2, train_on=("grating", "rough"), policy="window",
                                 # survival floor 2^-3 (config 4 leaves it open): fewer heavy weights
                                 max_roulette_exp=3)),
    "rough": dict(rows=512, cpu_sample=163840, ref_sample=40960,
                  learned=dict(map_lo=(-500, -500, -40), map_hi=(500, 500, 30), cell=2.0, d_max=10.0,
                               train_per_pixel=1, train_on=("grating", "rough"), policy="cost"),
                  desc="rough slab: 512x512 Gaussian height field (RMS 3 nm, correlation 10 nm) over 1 um, "
                       "526,334 triangles; 512x512 px x 20 primaries (5,242,880) at E uniform over "
                       "{300, 1000, 3000, 5000} eV, Si-like Kieft tables"),
    "holes": dict(rows=64, tune_row=8, cpu_sample=204800, ref_sample=102400,
                  # the map covers the default 64 pixel rows (y up to -1121 nm)
                  learned=dict(map_lo=(-1290, -1290, -170), map_hi=(1290, -1100, 25), cell=2.0, d_max=10.0,
                               train_per_pixel=8, train_rows=64, train_on=("holes",), policy="cost"),
                  desc="contact holes: 32x32 holes (40 nm diameter, 100 nm deep, +-2 nm edge roughness) in a "
                       "SiO2-like film over W-like plugs on a Si-like substrate, 2,506,772 triangles over "
                       "2.56 um; 1024x1024 px at 2.5 nm x 200 primaries at 1 keV, one step = %d pixel rows "
                       "(%d primaries); SiO2/W/Si-like Kieft tables"),
}


def workload(name):
    """Bench settings of a workload merged with its scan definition."""
    from nebula_b200 import generators as g
    return dict(g.SCANS[name], **WORKLOADS[name])


def configure(args):
    """Point the module's scan constants at the chosen workload."""
    global NX, NY, PER_PIXEL, ENERGY, WORKLOAD
    w = workload(args.workload)
    NX, NY, PER_PIXEL, ENERGY = w["nx"], w["ny"], w["per_pixel"], w["energy"]
    if args.rows <= 0:
        args.rows = w["rows"]
    args.rows = min(args.rows, NY)
    WORKLOAD = w["desc"] % (args.rows, args.rows * NX * PER_PIXEL) if "%d" in w["desc"] else w["desc"]


def workload_name(args):
    if args.inelastic == "penn":
        return WORKLOAD.replace("Kieft tables", "full Penn inelastic + Kieft elastic tables")
    return WORKLOAD


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def init_dist(world):
    if world <= 1:
        return None
    import datetime

    import torch.distributed as dist
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=120))
    return dist


def allreduce_max(dist, x):
    if dist is None:
        return x
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def allreduce_sum(dist, x):
    if dist is None:
        return x
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def barrier(dist):
    if dist is not None:
        dist.barrier()


def make_workload(tmp, rank=0, rows=None, workload="grating"):
    """Material files (in geometry order), triangles, .tri path and the
    scan's primaries (pixel rows `rows`, all if None)."""
    from nebula_b200 import formats, generators as g
    w = g.SCANS[workload]
    mats = [g.make_material(os.path.join(tmp, k + ".mat"), kind=k) for k in w["materials"]]
    tris = w["geometry"]()
    tri_path = os.path.join(tmp, workload + ".tri")
    formats.write_tri(tri_path, tris)
    recs = g.scan_beam(w["nx"], w["ny"], w["per_pixel"], w["energy"], spacing=w["spacing"], origin=w["origin"],
                       z_start=w["z_start"], seed=1000 + rank, energies=w["energies"], rows=rows)
    return mats, tris, tri_path, recs


def strided_sample(recs, count):
    """`count` primaries evenly strided over the scan (every pixel row of
    the step is represented)."""
    if count >= len(recs):
        return recs
    return recs[np.linspace(0, len(recs) - 1, count).astype(np.int64)]


def step_moments(counts):
    """(mean, variance) of one run's per-primary counts or weights."""
    c = np.asarray(counts, np.float64)
    return float(c.mean()), float(c.var())


def fom(var_per_primary, n, seconds):
    """Figure of merit 1 / (sigma^2 t) of a mean yield estimated from n
    primaries in `seconds` of device time, sigma^2 = var_per_primary / n.
    var_per_primary must be the variance of ONE run's per-primary values:
    summing the counts of K repeated runs of the same scan before taking the
    variance adds K times the spread of the per-pixel means, and the result
    would grow with K."""
    if not (var_per_primary > 0) or not (seconds > 0) or n <= 0:
        return None
    return 1.0 / (var_per_primary / n * seconds)


def plain_fom(step_vars, n, step_seconds):
    """FOM of K timed plain steps, each one independent run over the same n
    primaries: per-step variances and device times averaged."""
    return fom(sum(step_vars) / len(step_vars), n, sum(step_seconds) / len(step_seconds))


class ClockSampler:
    """nvidia-smi clock/throttle sampling during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.out = tempfile.TemporaryFile(mode="w+")

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.Q,
                                          "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.out,
                                         stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.out.seek(0)
        rows = [r for r in csv.reader(io.StringIO(self.out.read())) if len(r) >= 9]
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[1]))
                mx = float(r[2])
            except ValueError:
                continue
            for nm, v in zip(names, r[5:9]):
                if v.strip().lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def algorithmic_bytes_per_event(tris, mat_paths, recs, seed, penn=False):
    """Section-8(d) algorithmic bytes per event, counted by the instrumented
    CPU restatement on a fixed sample of the workload.  An inelastic event
    reads a 2-D ICDF (16 B) and a rounddown value (4 B) under Kieft, and the
    2-D ICDF, a trilinear 3-D q lookup (32 B) and a 3-D rounddown (4 B) under
    full Penn."""
    import oracle
    pg = oracle.PortGeometry(tris)
    rms = [oracle.RefMaterial(p, penn=penn) for p in mat_paths]
    pms, arr = oracle.port_materials(rms)
    sample = strided_sample(recs, 2000)
    prim = np.zeros((len(sample), 7), np.float32)
    prim[:, 0:3] = sample["pos"]
    prim[:, 3:6] = sample["dir"]
    prim[:, 6] = sample["E"]
    c, _, _, _, gc = oracle.port_run(pg, arr, prim, np.arange(len(sample), dtype=np.uint32), seed,
                                     max_energy=min(m.max_energy for m in rms), penn=penn)
    ev = c["n_elastic"] + c["n_inelastic"] + c["n_boundary"]
    b_state = 88.0
    b_inel = 52.0 if penn else 20.0
    b_tables = 16.0 + (16.0 * c["n_elastic"] + b_inel * c["n_inelastic"] + 52.0 * c["n_boundary"]) / ev
    b_geom = (4.0 * float(gc[0]) + 44.0 * float(gc[1])) / ev
    return b_state + b_tables + b_geom, {"state": b_state, "tables": round(b_tables, 2), "geom": round(b_geom, 2),
                                         "octree_words_per_event": round(float(gc[0]) / ev, 2),
                                         "triangles_per_event": round(float(gc[1]) / ev, 3),
                                         "sample_primaries": len(sample), "sample_events": ev}


def cpu_baseline(tri_path, mat_paths, recs, tmp, count, penn=False):
    """The reference's own CPU path (oracle/_ref, cpu_mt_main-style driver;
    the stock full Penn build with `penn`) on `count` primaries evenly
    strided over the step's scan, all host cores."""
    import oracle
    from nebula_b200 import formats
    if not oracle.have_ref(penn):
        return None
    sub = strided_sample(recs, count)
    pri = os.path.join(tmp, "cpu_sample.pri")
    formats.write_pri(pri, sub)
    cores = os.cpu_count() or 1
    _, st, secs = oracle.ref_run(tri_path, pri, mat_paths, threads=cores, count_events=True, penn=penn)
    ev = st["n_intersect"] + st["n_elastic"] + st["n_inelastic"]
    return {"value": ev / secs, "unit": "events/s", "cores": cores, "kind": "reference",
            "sample": "%d primaries evenly strided over the step's scan (%d events) in %.2f s"
                      % (len(sub), ev, secs),
            "primaries_per_s": st["n_primaries"] / secs}


def _simulation_seconds(log):
    """The `Simulation: <seconds>` line both programs print on stderr."""
    for line in log.splitlines()[::-1]:
        if "Simulation:" in line:
            try:
                return float(line.split(":")[-1])
            except ValueError:
                return None
    return None


# Workloads on which the reference's own GPU program is not run: on the
# contact-hole scan it stops making progress (every slot holds a running
# electron whose secondary waits for a free slot, drivers/gpu/
# gpu_driver.inl:523-528 and gpu_particle_manager.inl:355-376), so it would
# only run into the timeout.
REFERENCE_GPU_STALLS = {
    "holes": "reference program stalls on this workload (see profiles/reference_gpu_program.md)",
}


def reference_gpu(tri_path, mat_paths, recs, tmp, penn=False, timeout=120, workload="grating"):
    """The reference's own GPU program (gpu_main.cu built for sm_100a by
    `make -C oracle gpu`) and the nbx CLI on the same .tri/.pri/.mat files,
    one after the other on this GPU; each program's own `Simulation:` time.
    The reference checks for completion once a second (gpu_main.cu:410-426),
    so its time is a whole number of seconds, an upper bound.  Test
    infrastructure: opt-in (--reference-gpu), not part of the default run,
    and refused on the workloads of REFERENCE_GPU_STALLS."""
    if workload in REFERENCE_GPU_STALLS:
        return {"unavailable": REFERENCE_GPU_STALLS[workload]}
    from nebula_b200 import formats
    binary = os.path.join(ROOT, "oracle", "_ref", "nebula_gpu" if penn else "nebula_gpu_kieft")
    cli = os.path.join(ROOT, "nebula_b200", "nebula_b200")
    if not (os.path.exists(binary) and os.path.exists(cli)):
        return {"unavailable": "reference GPU program or nbx CLI not built"}
    pri = os.path.join(tmp, "refgpu.pri")
    formats.write_pri(pri, recs)
    out = {"primaries": len(recs), "resolution_s": 1.0}
    runs = (("reference", [binary]), ("nbx_cli", [cli] + (["--inelastic", "penn"] if penn else [])))
    for name, cmd in runs:
        try:
            r = subprocess.run(cmd + [tri_path, pri] + list(mat_paths), stdout=subprocess.DEVNULL,
                               stderr=subprocess.PIPE, timeout=timeout, text=True)
        except subprocess.TimeoutExpired:
            out[name] = {"status": "timed out after %d s" % timeout}
            continue
        secs = _simulation_seconds(r.stderr)
        out[name] = {"status": r.returncode, "simulation_s": secs,
                     "primaries_per_s": len(recs) / secs if secs else None}
    ref_s = out.get("reference", {}).get("simulation_s")
    nbx_s = out.get("nbx_cli", {}).get("simulation_s")
    out["nbx_speedup_at_least"] = (ref_s - 1.0) / nbx_s if ref_s and nbx_s else None
    return out


def run_reference(args):
    rank, world, local = dist_env()
    if rank != 0:
        return 0
    import oracle
    penn = args.inelastic == "penn"
    with tempfile.TemporaryDirectory() as tmp:
        if not oracle.have_ref(penn):
            print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref reference library not built"}))
            return 0
        from nebula_b200 import formats
        mats, tris, tri_path, recs = make_workload(tmp, rows=range(args.rows), workload=args.workload)
        sub = strided_sample(recs, WORKLOADS[args.workload]["ref_sample"])
        pri = os.path.join(tmp, "ref_step.pri")
        formats.write_pri(pri, sub)
        cores = os.cpu_count() or 1
        total_ev, total_s, total_p = 0, 0.0, 0
        for i in range(args.warmup + args.steps):
            _, st, secs = oracle.ref_run(tri_path, pri, mats, seed=0x78C7E39B + i, threads=cores, count_events=True,
                                         penn=penn)
            if i >= args.warmup:
                total_ev += st["n_intersect"] + st["n_elastic"] + st["n_inelastic"]
                total_s += secs
                total_p += st["n_primaries"]
        v = total_ev / total_s
        line = {"metric": METRIC, "value": v, "unit": "events/s", "impl": "reference", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000 * total_s / args.steps,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                "data": "synthetic", "primaries_per_s": total_p / total_s,
                "config": {"workload": workload_name(args), "inelastic": args.inelastic,
                           "step_sample": "%d primaries per step, evenly strided over the scan" % len(sub)},
                "cpu_baseline": {"value": v, "unit": "events/s", "cores": cores, "kind": "reference",
                                 "sample": "%d primaries per step, %d steps" % (len(sub), args.steps)},
                "e2e": {"value": v, "unit": "events/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
    return 0


# Grid of the network's importance table (scaled log energy x distance to
# the surface x cosine toward its normal).
IMPORTANCE_GRID = (48, 32, 16)

# Training records per scan of the learned leg (about 4 M in all, the
# records of the grating and the rough-slab scans for those two workloads).
TRAIN_RECORDS = 2_000_000


def sample_records(name, tmp, local, rank, penn):
    """Sample-mode run over the training scan of workload `name` (its own
    seed): (features, labels, costs) of up to TRAIN_RECORDS newborn
    electrons, recorded at birth."""
    import nebula_b200 as nb
    from nebula_b200 import generators as g
    w = workload(name)
    L = w["learned"]
    mats = [g.make_material(os.path.join(tmp, "train_%s_%s.mat" % (name, k)), kind=k) for k in w["materials"]]
    ctx = nb.setup(w["geometry"](), mats, device=local, seed=0x3C6EF372 + rank, inelastic=penn and "penn" or "kieft")
    try:
        ctx.build_surface_map(list(L["map_lo"]), list(L["map_hi"]), L["cell"], L["d_max"])
        rows = range(L["train_rows"]) if "train_rows" in L else None
        train = g.scan_beam(w["nx"], w["ny"], L["train_per_pixel"], w["energy"], spacing=w["spacing"],
                            origin=w["origin"], z_start=w["z_start"], seed=0x51ED + rank, energies=w["energies"],
                            rows=rows)
        ctx.set_sample_capacity(1 << 23)
        ctx.set_mode("sample")
        ctx.set_tag_range(len(train))
        ctx.reset_tallies()
        ctx.push_records(train)
        ctx.run()
        f, y, c = ctx.get_samples(1 << 23, with_cost=True)
    finally:
        ctx.close()
    if len(y) > TRAIN_RECORDS:
        keep = np.random.default_rng(rank).choice(len(y), TRAIN_RECORDS, replace=False)
        f, y, c = f[keep], y[keep], c[keep]
    return f, y, c


def learned_fom(args, tris, mats, local, rank, prim, tags, plain, tmp, tune_sample):
    """SE-yield figure of merit of the learned roulette on the same scan.

    Training data: sample-mode runs of the workload's training scans (for the
    grating and the rough slab: both of them, about 4 M records recorded at
    the birth of newborn electrons).  The network (6 -> 64 -> 64 -> 1) is
    trained on them on the GPU (8 epochs, batch 8192, Adam lr 1e-3).  Then the
    whole scan runs once in learned mode with one tag per primary: every
    newborn secondary is scored at birth, plays roulette below rr_threshold
    (default 0.05) and splits above split_threshold (default 0.5).
    FOM = 1 / (sigma^2 t): sigma^2 = per-primary variance of the weighted SE
    count of that one run / n, t = its device time -- the same estimator as
    the plain FOM of one timed step.  `z` compares the weighted SE and BSE
    yields with the plain yields of the timed steps (unbiasedness).  `plain`:
    the plain steps' means, per-step variances, step count and FOM."""
    import nebula_b200 as nb
    n = len(tags)
    w = workload(args.workload)
    L = w["learned"]
    penn = args.inelastic == "penn"
    t0 = time.perf_counter()
    parts = [sample_records(name, tmp, local, rank, penn) for name in L["train_on"]]
    f = np.concatenate([p[0] for p in parts])
    y = np.concatenate([p[1] for p in parts])
    cost = np.concatenate([p[2] for p in parts])
    t_sample = time.perf_counter() - t0
    ctx = nb.setup(tris, mats, device=local, seed=0x2545F491 + rank, blocks_per_sm=args.learned_variant or 4,
                   block_size=args.learned_block, inelastic=args.inelastic)
    try:
        ctx.build_surface_map(list(L["map_lo"]), list(L["map_hi"]), L["cell"], L["d_max"])
        ctx.mlp_set_params(nb.mlp_init_params(0))
        t0 = time.perf_counter()
        losses = ctx.mlp_train(f, y, epochs=8, batch=8192, lr=1e-3, seed=1)
        t_train = time.perf_counter() - t0
        ctx.set_tag_range(n)
        policy = args.learned_policy or L["policy"]
        # the cost-aware survival runs without splitting: a split adds
        # near-surface work, the most expensive steps of the scan
        split = 2.0 if policy == "cost" else args.split_threshold
        # roulette floor (a deeper floor lets the rare heavy survivors dominate
        # the variance): the flag, else the workload's own for its own policy,
        # else 2^-4 for the cost-aware survival and 2^-6 for the window
        max_k = args.max_roulette_exp or (L.get("max_roulette_exp") if policy == L["policy"] else None) or \
            (4 if policy == "cost" else 6)
        ctx.set_mode("learned", rr_threshold=args.rr_threshold, split_threshold=split, max_roulette_exp=max_k)
        if args.birth_rr:
            ctx.set_birth_roulette(*[float(v) for v in args.birth_rr.split(",")])
        cost_info = None
        if policy == "cost" and not args.birth_rr:
            # cost-aware survival: mean sub-cascade cost per (material, log E)
            # from the training records; K = steps / variance per primary of
            # the plain timed steps
            table, lo, hi = nb.fit_cost_table(f, cost, n_materials=len(mats))
            value_per_cost = plain["steps_per_primary"] / plain["var_se"]
            ctx.set_learned_cost(table, lo, hi, value_per_cost)
            cost_info = {"value_per_cost": value_per_cost, "bins": int(table.shape[1])}
        if args.learned_eval == "table" and not args.birth_rr:
            ctx.set_importance_table(*IMPORTANCE_GRID)
        # launch shape, stack depth and chunk tuned in learned mode on the
        # plain leg's tuning sample (unless --learned-variant fixes the shape)
        tuned = ctx.autotune(prim[tune_sample], tags[tune_sample]) if not args.learned_variant else ctx.tuning()
        ctx.reset_tallies()
        ctx.push(prim, tags)
        ctx.run()
        s = ctx.stats()
        sw, bw = ctx.tag_weights(0, n)
        # the learned kernel's own cost: the same scan with every decision
        # off (the network still scores every newborn)
        ctx.set_birth_roulette(0.0, 0.0, 0.0)
        ctx.set_learned_cost(None, 0.0, 1.0, 1.0)
        # decisions off, network (or table) still consulted for every newborn
        ctx.set_mode("learned", rr_threshold=1e-30, split_threshold=0.99999, max_roulette_exp=max_k)
        ctx.reset_tallies()
        ctx.push(prim, tags)
        ctx.run()
        s_off = ctx.stats()
        t = s["last_run_ms"] / 1000.0
        m_se, v_se = step_moments(sw)
        m_bse, v_bse = step_moments(bw)
        fom_l = fom(v_se, n, t)
        k = plain["steps"]
        z_se = (m_se - plain["mean_se"]) / math.sqrt(v_se / n + plain["var_se"] / (n * k))
        z_bse = (m_bse - plain["mean_bse"]) / math.sqrt(v_bse / n + plain["var_bse"] / (n * k))
        return {"fom_se": fom_l, "fom_se_plain": plain["fom"], "plain_ns_per_step": plain["ns_per_step"],
                "gain": fom_l / plain["fom"] if (fom_l and plain["fom"]) else None,
                "se_yield": m_se, "bse_yield": m_bse, "z_vs_plain": z_se, "z_bse_vs_plain": z_bse,
                "run_ms": s["last_run_ms"], "var_ratio": v_se / plain["var_se"],
                "policy": ("fixed rule at birth " + args.birth_rr) if args.birth_rr else
                          ("network at birth (%s), %s" % (
                              "importance table %dx%dx%d" % IMPORTANCE_GRID if args.learned_eval == "table"
                              else "tensor cores per newborn",
                              "cost-aware survival" if cost_info else "weight window")),
                "cost_aware": cost_info,
                "decisions_off": {"run_ms": s_off["last_run_ms"], "steps": s_off["steps"],
                                  "ns_per_step": 1e6 * s_off["last_run_ms"] / max(s_off["steps"], 1),
                                  "inferences": s_off["inferences"]},
                "rr_threshold": args.rr_threshold, "split_threshold": split,
                "max_roulette_exp": max_k,
                "autotuned": tuned,
                "inferences": s["inferences"], "roulette_killed": s["roulette_killed"], "splits": s["splits"],
                "steps": s["steps"], "train_on": list(L["train_on"]), "train_samples": int(len(y)),
                "train_positive_rate": float(y.mean()) if len(y) else None,
                "train_mean_cost": float(cost.mean()) if len(cost) else None,
                "sample_s": round(t_sample, 3), "train_s": round(t_train, 3),
                "train_loss": [round(float(v), 5) for v in losses]}
    finally:
        ctx.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1, help="GPUs of the run (ranks come from torchrun)")
    ap.add_argument("--steps", type=int, default=5, help="timed steps")
    ap.add_argument("--warmup", type=int, default=3, help="untimed warm-up steps")
    ap.add_argument("--impl", default="nbx", choices=["nbx", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--workload", default="grating", choices=sorted(WORKLOADS),
                    help="grating line scan (headline), rough slab with mixed energies, or the "
                         "three-material contact-hole array")
    ap.add_argument("--rows", type=int, default=0,
                    help="pixel rows of one step (0: the workload's default, all rows but for the contact holes)")
    ap.add_argument("--variant", type=int, default=0, help="transport variant 2/3/4/7 (0: autotune)")
    ap.add_argument("--block", type=int, default=0, help="threads per block with --variant (0: 128)")
    ap.add_argument("--no-learned", action="store_true", help="skip the learned-roulette FOM comparison")
    ap.add_argument("--reference-gpu", action="store_true",
                    help="also time the reference's own GPU program and the nbx CLI on the step's primaries")
    ap.add_argument("--shared-pop", action="store_true",
                    help="all transport blocks pop primaries from one cursor (default: per-SM ranges)")
    ap.add_argument("--learned-variant", type=int, default=0,
                    help="transport variant of the learned leg (0: autotuned in learned mode)")
    ap.add_argument("--learned-block", type=int, default=256, help="threads per block of the learned leg")
    ap.add_argument("--birth-rr", default="",
                    help="learned leg: a fixed rule at birth instead of the network, "
                         "'min_distance_nm,max_energy_eV,survival' (default off)")
    ap.add_argument("--rr-threshold", type=float, default=0.05,
                    help="learned leg: importance below which a newborn secondary plays roulette")
    ap.add_argument("--split-threshold", type=float, default=0.5,
                    help="learned leg: importance above which a newborn secondary splits in two")
    ap.add_argument("--max-roulette-exp", type=int, default=0,
                    help="learned leg: lowest roulette survival is 2^-this (0: the workload's default for its "
                         "policy, else 4 for the cost-aware survival and 6 for the weight window)")
    ap.add_argument("--learned-eval", default="table", choices=["table", "fused"],
                    help="learned leg: network tabulated once over its inputs (table) or evaluated on the tensor "
                         "cores for every newborn (fused)")
    ap.add_argument("--learned-policy", default="", choices=["", "window", "cost"],
                    help="learned leg: weight window on the network's importance (rr/split thresholds; the "
                         "grating's default, BASELINE's learned config), or cost-aware survival w sqrt(p K / c) "
                         "without splitting (the rough slab's and the contact holes' default)")
    ap.add_argument("--inelastic", default="kieft", choices=["kieft", "penn"],
                    help="inelastic model: Kieft & Bosch (the headline workload) or full Penn (the reference's stock build)")
    args = ap.parse_args()
    configure(args)
    if args.impl == "reference":
        return run_reference(args)

    rank, world, local = dist_env()
    dist = init_dist(world)
    import nebula_b200 as nb

    tmp = tempfile.mkdtemp(prefix="nbx_bench_")
    from nebula_b200 import replicas
    mats, tris, tri_path, recs = make_workload(tmp, rows=range(args.rows), workload=args.workload)
    ctx = nb.setup(tris, mats, device=local, seed=0x78C7E39B, inelastic=args.inelastic,
                   shared_pop=args.shared_pop)
    n = len(recs)
    prim = np.zeros((n, 7), np.float32)
    prim[:, 0:3] = recs["pos"]
    prim[:, 3:6] = recs["dir"]
    prim[:, 6] = recs["E"]
    tags = np.arange(n, dtype=np.uint32)
    pixel_of_tag = (recs["py"].astype(np.uint32) * NX + recs["px"].astype(np.uint32))
    # the library's own page-locked host buffers (nbx_host_alloc)
    pin_p = nb.host_empty((n, 7), np.float32)
    pin_t = nb.host_empty(n, np.uint32)
    pinned = True
    pin_p[:] = prim
    pin_t[:] = tags
    ctx.set_tag_range(n)
    # Autotune the transport launch shape on a 16-row sample of the scan.
    tune_n = 0
    # the autotuner's sample: at least 16 pixel rows and about 1.6 M primaries
    # (records are row-major; short runs rank the launch shapes by their
    # tails) from `tune_row` (the contact holes' first band of holes; the
    # grating and the slab are uniform)
    tune_rows = min(args.rows, max(16, -(-1600000 // (NX * PER_PIXEL))))
    r0 = min(WORKLOADS[args.workload].get("tune_row", 0), max(0, args.rows - tune_rows))
    tune_sample = np.arange(r0 * NX * PER_PIXEL, min(n, (r0 + tune_rows) * NX * PER_PIXEL))
    if args.variant:
        ctx.close()
        ctx = nb.setup(tris, mats, device=local, seed=0x78C7E39B, blocks_per_sm=args.variant,
                       block_size=args.block or 128, inelastic=args.inelastic, shared_pop=args.shared_pop)
        ctx.set_tag_range(n)
        tuned = ctx.tuning()
    else:
        tuned = ctx.autotune(prim[tune_sample], tags[tune_sample])
        tune_n = len(tune_sample)

    # One job of `world` frames of the scan, sharded by global primary index:
    # this rank's shard is [g_start, g_stop) of every step's world * n
    # primaries (one frame), simulated with the global index as its random-
    # stream base, so the combined result does not depend on the rank count.
    g_start, g_stop = replicas.shard_range(world * n, rank, world)
    assert g_stop - g_start == n
    step_no = [0]

    def push_step():
        ctx.set_uid_base(step_no[0] * world * n + g_start)
        step_no[0] += 1
        ctx.push(pin_p, pin_t)

    for _ in range(args.warmup):
        ctx.reset_tallies()
        push_step()
        barrier(dist)
        ctx.run()

    # Device-resident timing: primaries pushed before the timed run.  Each
    # timed step is one independent run over the scan; its per-primary counts
    # are read back after the run (outside the device-timed region) for the
    # per-step variance of the figure of merit.
    dev_ms, events, gens, launches, plain_steps = [], 0, 0, 0, 0
    se_mom, bse_mom = [], []
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            ctx.reset_tallies()
            push_step()
            barrier(dist)
            ctx.run()
            s1 = ctx.stats()
            dev_ms.append(s1["last_run_ms"])
            events += s1["events_elastic"] + s1["events_inelastic"] + s1["events_boundary"]
            plain_steps += s1["steps"]
            gens = s1["generations"]
            launches += s1["generations"]
            se_k, bse_k = ctx.tag_counts(0, n)
            se_mom.append(step_moments(se_k))
            bse_mom.append(step_moments(bse_k))
    clocks = clk.summary()
    t_dev = allreduce_max(dist, sum(dev_ms) / 1000.0)
    ev_all = allreduce_sum(dist, events)
    value = ev_all / t_dev
    prim_all = allreduce_sum(dist, n * args.steps)

    # SE-yield figure of merit of one timed step: per-primary variance of
    # that step's SE counts, sigma^2 of its mean yield, t = its device time.
    plain = {"steps": args.steps,
             "mean_se": sum(m for m, _ in se_mom) / args.steps, "var_se": sum(v for _, v in se_mom) / args.steps,
             "mean_bse": sum(m for m, _ in bse_mom) / args.steps,
             "var_bse": sum(v for _, v in bse_mom) / args.steps,
             "steps_per_primary": plain_steps / (n * args.steps),
             "ns_per_step": 1e6 * sum(dev_ms) / max(plain_steps, 1)}
    plain["fom"] = plain_fom([v for _, v in se_mom], n, [ms / 1000.0 for ms in dev_ms])
    mean_se = plain["mean_se"]

    # End-to-end through the C ABI from pinned host buffers.  The scan's
    # tag -> pixel map is given once, like the geometry (setup, untimed).
    ctx.set_pixel_map(pixel_of_tag)
    n_pix = args.rows * NX
    pin_y = nb.host_empty((n_pix, 5), np.float64)
    # Pipelined like a scan that streams its frames: each step starts the copy
    # of the next step's primaries (nbx_stage, on the library's copy stream)
    # and runs its own while that copy is in flight, reads its per-pixel
    # yields back, then queues the next step's primaries on the device
    # (nbx_push_staged).  Every step holds one host-to-device copy of a
    # step's inputs and one device-to-host read of a step's result.
    e2e_s = []
    parts = {"stage_ms": 0.0, "run_ms": 0.0, "yields_ms": 0.0, "push_staged_ms": 0.0}

    def step_base():
        return step_no[0] * world * n + g_start

    # one untimed pass of the end-to-end calls first (the yields kernel's
    # first launch loads its module), leaving the first timed step's
    # primaries queued
    ctx.reset_tallies()
    ctx.set_uid_base(step_base())
    step_no[0] += 1
    ctx.push(pin_p, pin_t)
    ctx.run()
    ctx.pixel_yields(None, n_pix, out=pin_y)
    ctx.set_uid_base(step_base())
    step_no[0] += 1
    ctx.stage(pin_p, pin_t)        # the staging buffers and copy stream are made here
    ctx.push_staged()
    for _ in range(args.steps):
        ctx.reset_tallies()
        barrier(dist)
        t0 = time.perf_counter()
        ctx.stage(pin_p, pin_t)
        t1 = time.perf_counter()
        ctx.run()
        t2 = time.perf_counter()
        out = ctx.pixel_yields(None, n_pix, out=pin_y)
        t3 = time.perf_counter()
        ctx.set_uid_base(step_base())
        step_no[0] += 1
        ctx.push_staged()
        t4 = time.perf_counter()
        e2e_s.append(t4 - t0)
        parts["stage_ms"] += 1000 * (t1 - t0) / args.steps
        parts["run_ms"] += 1000 * (t2 - t1) / args.steps
        parts["yields_ms"] += 1000 * (t3 - t2) / args.steps
        parts["push_staged_ms"] += 1000 * (t4 - t3) / args.steps
    t_e2e = allreduce_max(dist, sum(e2e_s))
    e2e_val = ev_all / t_e2e
    # the job's image: the last step's per-pixel sums added up over the ranks
    # (one collective, after timing)
    image = replicas.reduce_pixel_yields(dist, out)
    image_yield = {"frames": world, "primaries": float(image[:, 0].sum()),
                   "se_yield": float(image[:, 1].sum() / max(image[:, 0].sum(), 1.0)),
                   "bse_yield": float(image[:, 3].sum() / max(image[:, 0].sum(), 1.0))}
    h2d = n * 7 * 4 + n * 4
    d2h = n_pix * 5 * 8

    # every workload defines the learned leg's surface map and training scans
    learned = None if (args.no_learned or "learned" not in WORKLOADS[args.workload]) else \
        learned_fom(args, tris, mats, local, rank, prim, tags, plain, tmp, tune_sample)

    line = None
    if rank == 0:
        peak, peak_kind = measured_peaks()
        b_event, b_parts = algorithmic_bytes_per_event(tris, mats, recs, 0x78C7E39B, penn=args.inelastic == "penn")
        achieved = events * b_event / (sum(dev_ms) / 1000.0) / 1e9
        # DRAM bytes per launch: the ncu capture's bytes per event (Kieft
        # model, this workload) times the events of one step, whose first
        # generation's launch carries the whole scan
        traffic, dram_frac, ncu = None, None, None
        tp = os.path.join(ROOT, "profiles", "transport_kernel_traffic_%s.json" % args.workload)
        if os.path.exists(tp) and args.inelastic == "kieft":
            with open(tp) as f:
                prof = json.load(f)
            traffic = prof["dram_bytes_per_event"] * events / args.steps
            # measured DRAM bytes at this run's event rate, against the HBM peak
            dram_frac = prof["dram_bytes_per_event"] * (events / (sum(dev_ms) / 1000.0)) / 1e9 / peak
            ncu = {k: prof[k] for k in ("issue_active", "simt_lanes_per_instruction", "l1_hit", "l2_hit",
                                        "source") if k in prof}
        cpu = None if args.no_cpu_baseline else cpu_baseline(tri_path, mats, recs, tmp,
                                                              WORKLOADS[args.workload]["cpu_sample"],
                                                              penn=args.inelastic == "penn")
        ref_gpu = reference_gpu(tri_path, mats, recs, tmp, penn=args.inelastic == "penn",
                                workload=args.workload) if args.reference_gpu else None
        line = {
            "metric": METRIC, "value": value, "unit": "events/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1000.0 * t_dev / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": workload_name(args), "inelastic": args.inelastic,
                       "parallelism": "replicas x%d (one scan frame per rank, sharded by global primary index)"
                                      % world,
                       "l2": "inputs larger than L2 (primary queue %.0f MB per step)" % (n * 48 / 1e6),
                       "autotuned": dict(tuned, tuned_on="%d primaries of the scan" % tune_n if tune_n else
                                         "not tuned (--variant given)"),
                       "pop": "shared cursor" if args.shared_pop else "per-SM ranges"},
            "primaries_per_s": prim_all / t_dev,
            "events_per_primary": events / (n * args.steps),
            "se_yield": mean_se, "bse_yield": plain["mean_bse"],
            "fom_se_plain": plain["fom"],
            "learned_rr": learned,
            "image": image_yield,
            "generations_per_step": gens,
            "gpu_launches": int(launches),
            "e2e": {"value": e2e_val, "unit": "events/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "pinned_host": pinned, "breakdown_ms_per_step": {k: round(v, 2) for k, v in parts.items()}},
            # achieved/frac: the algorithmic bytes per event (octree, triangle,
            # table and state gathers) at the measured event rate against the
            # HBM peak.  L1 and L2 serve nearly all of those gathers (dram_frac
            # is the DRAM traffic actually measured), and the kernel is bound
            # by instruction issue under warp divergence (ncu figures).
            "roofline": {"bound": "issue/L1-L2 latency", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic, "dram_frac": dram_frac, "ncu": ncu,
                         "peak_kind": peak_kind, "bytes_per_event": round(b_event, 2), "bytes_breakdown": b_parts,
                         "kernel": "transport_kernel"},
            "clocks": clocks,
            "cpu_baseline": cpu,
            "reference_gpu_program": ref_gpu,
        }
        print(json.dumps(line), flush=True)
    ctx.close()
    if dist is not None:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
