"""The allocation-free transport entry point (nbx_run_noalloc).

Some callers cannot allocate device memory themselves (their own caching
allocator owns the GPU, or an allocation's implicit synchronisation would
stall their streams); nbx_run_noalloc serves them from a fixed scratch array
inside the library.  This test runs two batches in a row through it, from
device buffers, and compares the per-primary SE/BSE tallies and event counts
with the existing nbx_push + nbx_run path on the same primaries and random
streams: the transport is deterministic per electron, so the tallies must be
identical (the exact-match tolerance of the other integer-tally tests).  It
also checks that an oversized request, a random-stream index past 2^63 and a
context that is not in plain mode are refused.  The file is named to be
collected last."""
import numpy as np
import pytest

import nebula_b200 as nb
from nebula_b200 import generators as g

pytestmark = pytest.mark.gpu


def _prims(recs):
    p = np.zeros((len(recs), 7), np.float32)
    p[:, 0:3] = recs["pos"]
    p[:, 3:6] = recs["dir"]
    p[:, 6] = recs["E"]
    return p


def test_noalloc_matches_push_run(tmp_path):
    import torch
    mat = g.make_material(str(tmp_path / "si.mat"))
    tris = g.grating_geometry(n_lines=7, length=400.0)
    batches = [g.scan_beam(32, 16, 8, 500.0, origin=(-16.0, -8.0), seed=s) for s in (31, 32)]
    n = len(batches[0])
    assert n == len(batches[1]) and n <= 65536

    # Existing entry point: push + run, one batch after the other.
    ref = nb.setup(tris, [mat], device=0, seed=1234)
    ref.set_tag_range(n)
    expected = []
    for recs in batches:
        ref.reset_tallies()
        ref.push(_prims(recs), np.arange(n, dtype=np.uint32))
        ref.run()
        se, bse = ref.tag_counts(0, n)
        st = ref.stats()
        expected.append((se, bse, (st["events_elastic"], st["events_inelastic"], st["events_boundary"], st["detected"])))
    ref.close()

    # Allocation-free entry point on a fresh context, same seed, same uids.
    ctx = nb.setup(tris, [mat], device=0, seed=1234)
    dev = torch.device("cuda:0")
    uid = 0
    for recs, (e_se, e_bse, e_counts) in zip(batches, expected):
        d_p = torch.from_numpy(_prims(recs)).to(dev)
        d_t = torch.arange(n, dtype=torch.int32, device=dev)
        d_se = torch.zeros(n, dtype=torch.int32, device=dev)
        d_bse = torch.zeros(n, dtype=torch.int32, device=dev)
        torch.cuda.synchronize()
        counts = nb.run_noalloc(ctx, d_p.data_ptr(), d_t.data_ptr(), n, uid, d_se.data_ptr(), d_bse.data_ptr(), n)
        uid += n
        se = d_se.cpu().numpy().view(np.uint32)
        bse = d_bse.cpu().numpy().view(np.uint32)
        assert np.array_equal(se, e_se)
        assert np.array_equal(bse, e_bse)
        assert (counts["elastic"], counts["inelastic"], counts["boundary"], counts["detected"]) == e_counts
        assert counts["detected"] > 0

    with pytest.raises(nb.NbxError) as e:
        nb.run_noalloc(ctx, d_p.data_ptr(), d_t.data_ptr(), 65537, 0, d_se.data_ptr(), d_bse.data_ptr(), n)
    assert e.value.code == -1
    ctx.close()


def test_noalloc_refuses_non_plain_modes_and_uid_overflow(tmp_path):
    """The entry point runs plain transport only: a context in sample or
    learned mode gets NBX_ERR_STATE instead of silently unweighted tallies.
    uid_base + n past 2^63 would reuse random streams and gets NBX_ERR_ARG.
    Nothing is added to the tallies by a refused call, and a plain call on
    the same context still works afterwards."""
    import torch
    mat = g.make_material(str(tmp_path / "si.mat"))
    tris = g.grating_geometry(n_lines=7, length=400.0)
    recs = g.scan_beam(8, 8, 4, 500.0, origin=(-4.0, -4.0), seed=5)
    n = len(recs)
    ctx = nb.setup(tris, [mat], device=0, seed=99)
    dev = torch.device("cuda:0")
    d_p = torch.from_numpy(_prims(recs)).to(dev)
    d_t = torch.arange(n, dtype=torch.int32, device=dev)
    d_se = torch.zeros(n, dtype=torch.int32, device=dev)
    d_bse = torch.zeros(n, dtype=torch.int32, device=dev)
    torch.cuda.synchronize()
    for mode in ("sample", "learned"):
        ctx.set_mode(mode)
        with pytest.raises(nb.NbxError) as e:
            nb.run_noalloc(ctx, d_p.data_ptr(), d_t.data_ptr(), n, 0, d_se.data_ptr(), d_bse.data_ptr(), n)
        assert e.value.code == -6
    ctx.set_mode("plain")
    with pytest.raises(nb.NbxError) as e:
        nb.run_noalloc(ctx, d_p.data_ptr(), d_t.data_ptr(), n, 2 ** 63 - n + 1, d_se.data_ptr(), d_bse.data_ptr(), n)
    assert e.value.code == -1
    assert int(d_se.sum().item()) == 0 and int(d_bse.sum().item()) == 0
    counts = nb.run_noalloc(ctx, d_p.data_ptr(), d_t.data_ptr(), n, 2 ** 63 - n, d_se.data_ptr(), d_bse.data_ptr(), n)
    assert counts["detected"] == int(d_se.sum().item()) + int(d_bse.sum().item()) > 0
    ctx.close()
