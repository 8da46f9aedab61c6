"""Multi-GPU replica logic on CPU: two gloo ranks each simulate a contiguous
share of a scan (here with the C restatement standing in for the GPU
simulator) using global primary indices as random-stream bases, then sum the
per-pixel accumulators.  The result must equal the single-process run bit
for bit: sharding changes nothing."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from nebula_b200 import generators as g
from nebula_b200.replicas import reduce_pixel_yields, shard_range

NX, NY, PER = 6, 4, 5


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


class OracleCtx:
    """Minimal stand-in with the Context methods run_shard needs, simulating
    with the C restatement."""

    def __init__(self, tris, mat_path, seed):
        import oracle
        self.pg = oracle.PortGeometry(tris)
        self.rm = oracle.RefMaterial(mat_path)
        self.pms, self.arr = oracle.port_materials([self.rm])
        self.seed = seed
        self.uid = 0

    def simulate(self, recs):
        import oracle
        prim = np.zeros((len(recs), 7), np.float32)
        prim[:, 0:3] = recs["pos"]
        prim[:, 3:6] = recs["dir"]
        prim[:, 6] = recs["E"]
        c, se, bse, _, _ = oracle.port_run(self.pg, self.arr, prim, np.arange(len(recs), dtype=np.uint32), self.seed,
                                           max_energy=self.rm.max_energy, uid_base=self.uid)
        out = np.zeros((NX * NY, 5))
        pix = recs["py"] * NX + recs["px"]
        np.add.at(out[:, 0], pix, 1.0)
        np.add.at(out[:, 1], pix, se)
        np.add.at(out[:, 2], pix, se.astype(float) ** 2)
        np.add.at(out[:, 3], pix, bse)
        np.add.at(out[:, 4], pix, bse.astype(float) ** 2)
        return out


def _worker(rank, world, port, mat, out_dir):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    recs = g.scan_beam(NX, NY, PER, 500.0, origin=(-3.0, -2.0), seed=3)
    ctx = OracleCtx(g.grating_geometry(n_lines=5, length=200.0), mat, 31)
    start, stop = shard_range(len(recs), rank, world)
    ctx.uid = start
    part = ctx.simulate(recs[start:stop])
    total = reduce_pixel_yields(dist, part)
    if rank == 0:
        np.save(os.path.join(out_dir, "total.npy"), total)
    dist.barrier()
    dist.destroy_process_group()


def test_shard_range():
    assert [shard_range(10, r, 3) for r in range(3)] == [(0, 4), (4, 7), (7, 10)]
    assert [shard_range(2, r, 4) for r in range(4)] == [(0, 1), (1, 2), (2, 2), (2, 2)]


def test_two_gloo_ranks_equal_single_process(tmp_path, inputs, oracle_built):
    mat = inputs["si"]
    ctx = mp.get_context("spawn")
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, mat, str(tmp_path))) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=300)
        assert p.exitcode == 0
    total = np.load(tmp_path / "total.npy")
    recs = g.scan_beam(NX, NY, PER, 500.0, origin=(-3.0, -2.0), seed=3)
    single = OracleCtx(g.grating_geometry(n_lines=5, length=200.0), mat, 31).simulate(recs)
    assert np.array_equal(total, single)
    assert total[:, 0].sum() == len(recs)
