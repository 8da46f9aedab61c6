"""Multi-GPU replica logic on CPU, through the product's replica code.

Two gloo ranks each run ``nebula_b200.replicas.run_shard`` -- the function a
multi-GPU job calls -- on a contiguous share of one scan and sum the per-pixel
accumulators with ``replicas.reduce_pixel_yields``.  The simulator behind it
is a stand-in context with the nbx Context methods run_shard calls
(set_uid_base, reset_tallies, set_tag_range, push_records, run,
pixel_yields), which simulates with the C restatement instead of the GPU and
keeps the library's random-stream numbering: a pushed primary's stream index
is the uid base plus its running index.  The summed result must equal the
single-process run bit for bit: sharding changes nothing."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from nebula_b200 import generators as g
from nebula_b200 import replicas
from nebula_b200.replicas import reduce_pixel_yields, run_shard, shard_range

NX, NY, PER = 6, 4, 5


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


class OracleCtx:
    """Stand-in for nebula_b200.Context over the C restatement: the calls and
    the tag / uid semantics run_shard relies on (tag i = the i-th pushed
    record since the last reset; uid = uid base + running push index)."""

    def __init__(self, tris, mat_path, seed):
        import oracle
        self.pg = oracle.PortGeometry(tris)
        self.rm = oracle.RefMaterial(mat_path)
        self.pms, self.arr = oracle.port_materials([self.rm])
        self.seed = seed
        self.uid_next = 0
        self.calls = []
        self.reset_tallies()

    def set_uid_base(self, base):
        assert 0 <= base < 2 ** 63
        self.uid_next = base
        self.calls.append("set_uid_base")

    def reset_tallies(self):
        self.se = np.zeros(0, np.uint32)
        self.bse = np.zeros(0, np.uint32)
        self.queued = []
        self.calls = getattr(self, "calls", []) + ["reset_tallies"]

    def set_tag_range(self, n):
        self.n_tags = n
        self.se = np.zeros(n, np.uint32)
        self.bse = np.zeros(n, np.uint32)
        self.calls.append("set_tag_range")

    def push_records(self, recs, first_tag=0):
        prim = np.zeros((len(recs), 7), np.float32)
        prim[:, 0:3] = recs["pos"]
        prim[:, 3:6] = recs["dir"]
        prim[:, 6] = recs["E"]
        self.queued.append((prim, np.arange(first_tag, first_tag + len(recs), dtype=np.uint32), self.uid_next))
        self.uid_next += len(recs)
        self.calls.append("push_records")
        return len(recs)

    def run(self):
        import oracle
        for prim, tags, uid in self.queued:
            _, se, bse, _, _ = oracle.port_run(self.pg, self.arr, prim, tags, self.seed,
                                               max_energy=self.rm.max_energy, uid_base=uid)
            self.se[tags] += se
            self.bse[tags] += bse
        self.queued = []
        self.calls.append("run")

    def pixel_yields(self, pixel_of_tag, n_pixels, out=None):
        out = np.zeros((n_pixels, 5)) if out is None else out
        pix = np.asarray(pixel_of_tag, np.int64)
        se = self.se[: len(pix)].astype(np.float64)
        bse = self.bse[: len(pix)].astype(np.float64)
        np.add.at(out[:, 0], pix, 1.0)
        np.add.at(out[:, 1], pix, se)
        np.add.at(out[:, 2], pix, se ** 2)
        np.add.at(out[:, 3], pix, bse)
        np.add.at(out[:, 4], pix, bse ** 2)
        self.calls.append("pixel_yields")
        return out


def _scan():
    return g.scan_beam(NX, NY, PER, 500.0, origin=(-3.0, -2.0), seed=3)


def _ctx(mat):
    return OracleCtx(g.grating_geometry(n_lines=5, length=200.0), mat, 31)


def _worker(rank, world, port, mat, out_dir):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    ctx = _ctx(mat)
    part = run_shard(ctx, _scan(), rank, world, NX * NY, NX)
    total = reduce_pixel_yields(dist, part)
    np.save(os.path.join(out_dir, "part%d.npy" % rank), part)
    if rank == 0:
        np.save(os.path.join(out_dir, "total.npy"), total)
    dist.barrier()
    dist.destroy_process_group()


def test_shard_range():
    assert [shard_range(10, r, 3) for r in range(3)] == [(0, 4), (4, 7), (7, 10)]
    assert [shard_range(2, r, 4) for r in range(4)] == [(0, 1), (1, 2), (2, 2), (2, 2)]


def test_run_shard_call_sequence_and_empty_shard(inputs, oracle_built):
    """run_shard sets the shard's global uid base before pushing, resets the
    tallies, and returns zeros for a rank whose share is empty."""
    ctx = _ctx(inputs["si"])
    recs = _scan()[:2]
    out = run_shard(ctx, recs, 3, 4, NX * NY, NX)      # ranks 2 and 3 get nothing
    assert out.shape == (NX * NY, 5) and not out.any()
    ctx = _ctx(inputs["si"])
    out = run_shard(ctx, _scan(), 1, 2, NX * NY, NX)
    start, stop = shard_range(NX * NY * PER, 1, 2)
    assert ctx.calls.index("set_uid_base") < ctx.calls.index("push_records") < ctx.calls.index("run")
    assert ctx.uid_next == stop                        # pushed with global indices start..stop-1
    assert out[:, 0].sum() == stop - start


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
    single = run_shard(_ctx(mat), _scan(), 0, 1, NX * NY, NX)
    assert np.array_equal(total, single)
    assert total[:, 0].sum() == NX * NY * PER
    # both ranks did work, and neither alone gives the whole image
    parts = [np.load(tmp_path / ("part%d.npy" % r)) for r in range(2)]
    assert all(p[:, 0].sum() > 0 for p in parts)
    assert np.array_equal(parts[0] + parts[1], total)
    assert replicas.reduce_pixel_yields(None, single) is single
