"""Sparse footprint slices on the device (glide_footprint_compact through
glide_b200.sparse) against the oracle's compaction, bit for bit: offsets, cells in
ascending order, values unchanged (-0.0, NaN, inf and subnormals kept), the ring rows
cleared; a row outside the ring and a short capacity reported in the status word; and
the ring footprint of a whole run streamed through SparseSliceStream, rebuilt on the
host bit-identical to the slices it compacted."""

from __future__ import annotations

import numpy as np
import pytest
import torch

from oracle import sparse_slices as osp

pytestmark = pytest.mark.gpu


def _rows(rng, n_rows, cells, density=0.03):
    x = np.zeros((n_rows, cells), dtype=np.float32)
    mask = rng.random(x.shape) < density
    x[mask] = rng.gamma(0.5, 2e-3, int(mask.sum())).astype(np.float32)
    x[1] = 0.0  # an empty slice
    x[2] = rng.normal(size=cells).astype(np.float32)  # every cell non-zero
    x[2][x[2] == 0.0] = 1.0
    sp = np.array([-0.0, np.nan, np.inf, 1e-45, -3.5], dtype=np.float32)[: min(5, cells)]
    x[3, : sp.size] = sp
    x[4, -1] = 7.0  # the last cell of a slice
    return x


def _bits(a):
    return np.ascontiguousarray(a).view(np.uint32)


@pytest.mark.parametrize("cells", [1, 2047, 2048, 2049, 3922, 112681])
def test_compact_matches_oracle(cuda_device, cells):
    from glide_b200.sparse import compact_rows

    rng = np.random.default_rng(cells)
    n_rows, k = 9, 6
    x = _rows(rng, n_rows, cells)
    # distinct rows (clear), starting with the dense, the empty and the special-value slice
    sel = np.array([2, 1, 3] + [i for i in rng.permutation(n_rows).tolist() if i not in (1, 2, 3)])[:k]
    rows = torch.from_numpy(x).to(cuda_device)
    idx = torch.from_numpy(sel.astype(np.int64)).to(cuda_device)
    status = torch.zeros(1, dtype=torch.int32, device=cuda_device)
    off, cell, val = compact_rows(rows, idx, clear=True, status=status)
    torch.cuda.synchronize()
    o_off, o_cell, o_val = osp.compact(x[sel])
    off = off.cpu().numpy()
    np.testing.assert_array_equal(off, o_off)
    total = int(off[-1])
    np.testing.assert_array_equal(cell[:total].cpu().numpy(), o_cell)
    np.testing.assert_array_equal(_bits(val[:total].cpu().numpy()), _bits(o_val))
    after = rows.cpu().numpy()
    assert not _bits(after[sel]).any()  # compacted rows cleared
    rest = np.setdiff1d(np.arange(n_rows), sel)
    np.testing.assert_array_equal(_bits(after[rest]), _bits(x[rest]))
    assert int(status.item()) == 0


def test_bad_rows_are_reported_and_empty(cuda_device):
    from glide_b200 import _abi
    from glide_b200.sparse import compact_rows

    rng = np.random.default_rng(5)
    x = _rows(rng, 6, 5000)
    rows = torch.from_numpy(x).to(cuda_device)
    sel = np.array([0, 6, 2, -1, 4], dtype=np.int64)
    status = torch.zeros(1, dtype=torch.int32, device=cuda_device)
    off, cell, val = compact_rows(rows, torch.from_numpy(sel).to(cuda_device), clear=True, status=status)
    torch.cuda.synchronize()
    assert int(status.item()) == _abi.GLIDE_STATUS_BAD_ROW
    good = x[[0, 0, 2, 0, 4]].copy()
    good[[1, 3]] = 0.0  # the bad rows come back as empty slices
    o_off, o_cell, o_val = osp.compact(good)
    off = off.cpu().numpy()
    np.testing.assert_array_equal(off, o_off)
    np.testing.assert_array_equal(cell[: off[-1]].cpu().numpy(), o_cell)
    np.testing.assert_array_equal(_bits(val[: off[-1]].cpu().numpy()), _bits(o_val))
    after = rows.cpu().numpy()
    assert not _bits(after[[0, 2, 4]]).any()
    np.testing.assert_array_equal(_bits(after[[1, 3, 5]]), _bits(x[[1, 3, 5]]))


def test_short_capacity_writes_nothing(cuda_device):
    from glide_b200 import _abi
    from glide_b200.sparse import compact_rows

    rng = np.random.default_rng(6)
    x = _rows(rng, 5, 3000)
    rows = torch.from_numpy(x).to(cuda_device)
    idx = torch.arange(5, dtype=torch.int64, device=cuda_device)
    total = int(osp.compact(x)[0][-1])
    cap = total - 1
    out = (torch.full((6,), -7, dtype=torch.int64, device=cuda_device),
           torch.full((cap,), -7, dtype=torch.int32, device=cuda_device),
           torch.full((cap,), -7.0, dtype=torch.float32, device=cuda_device))
    status = torch.zeros(1, dtype=torch.int32, device=cuda_device)
    off, cell, val = compact_rows(rows, idx, clear=True, capacity=cap, status=status, out=out)
    torch.cuda.synchronize()
    assert int(status.item()) == _abi.GLIDE_STATUS_COMPACT_OVERFLOW
    np.testing.assert_array_equal(off.cpu().numpy(), osp.compact(x)[0])  # the offsets say what was needed
    assert (cell.cpu().numpy() == -7).all() and (val.cpu().numpy() == -7.0).all()
    np.testing.assert_array_equal(_bits(rows.cpu().numpy()), _bits(x))  # nothing cleared


def test_no_slices(cuda_device):
    from glide_b200.sparse import compact_rows

    rows = torch.ones((3, 100), dtype=torch.float32, device=cuda_device)
    off, _, _ = compact_rows(rows, torch.zeros(0, dtype=torch.int64, device=cuda_device), clear=True)
    torch.cuda.synchronize()
    assert off.cpu().tolist() == [0]
    assert bool((rows == 1.0).all())


def test_stream_dense_protocol(cuda_device):
    """SparseSliceStream called with dense slices (the HostSliceStream protocol) leaves
    them unchanged and delivers their sparse form."""
    from glide_b200.sparse import SparseSliceStream, densify

    rng = np.random.default_rng(7)
    shape = (1, 37, 53)
    got = []
    def on_host(r, b, o, c, v):
        got.append((r, b, densify(o, c, v, shape)))

    sink = SparseSliceStream(cuda_device, shape, on_host=on_host, buffers=2, initial_density=0.0)
    calls = []
    for j in range(4):
        x = _rows(rng, 6, int(np.prod(shape))).reshape((6,) + shape)
        d = torch.from_numpy(x).to(cuda_device)
        r = torch.arange(6, dtype=torch.int64, device=cuda_device) + 10 * j
        sink(r, torch.full((6,), j, dtype=torch.int64, device=cuda_device), d)
        calls.append((x, d))
    sink.drain()
    assert len(got) == 4 and sink.short_copies >= 1
    for j, (x, d) in enumerate(calls):
        r, b, dense = got[j]
        assert r.tolist() == list(range(10 * j, 10 * j + 6)) and (b == j).all()
        np.testing.assert_array_equal(_bits(dense), _bits(x))
        np.testing.assert_array_equal(_bits(d.cpu().numpy()), _bits(x))


@pytest.mark.parametrize("buffers,initial_density", [(2, 1.0 / 32.0), (1, 0.0)])
def test_ring_footprint_streamed_sparse(cuda_device, buffers, initial_density):
    """A whole run's ring footprint through SparseSliceStream: every delivered slice is
    bit-identical to the dense slice it was compacted from, the ring slots are cleared
    for later bins, and the releases assemble into the dense footprint."""
    import dataclasses

    from fixtures import load_run
    from gpu_cases import run_gpu, runner_for, state_from

    from glide_b200.sparse import ReleaseAssembler, SparseSliceStream, densify

    run = load_run("run_small")
    dense_run = run_gpu(run, cuda_device).footprint.cpu().numpy()
    r = runner_for(run, cuda_device)
    r.footprint = dataclasses.replace(r.footprint, ring=2)
    fp = r.footprint
    shape = (len(fp.z_edges) - 1, fp.n_y, fp.n_x)
    delivered = {}
    blocks = {}
    asm = ReleaseAssembler(fp.n_time_bins, shape, lambda rel, block: blocks.__setitem__(rel, block))

    def on_host(r_idx, b_idx, off, cell, val):
        for key, sl in zip(zip(r_idx.tolist(), b_idx.tolist()), densify(off, cell, val, shape)):
            delivered[key] = sl
        asm(r_idx, b_idx, off, cell, val)

    sparse = SparseSliceStream(cuda_device, shape, on_host=on_host, buffers=buffers, initial_density=initial_density)
    snapshots = {}

    class Recorder:
        """Takes a dense copy of each slice (stream-ordered) before the sparse sink clears it."""

        def from_rows(self, rows, flat, ri, bi):
            dense = rows.index_select(0, flat).clone()
            snapshots[len(snapshots)] = (ri.clone(), bi.clone(), dense)
            sparse.from_rows(rows, flat, ri, bi)

    r.footprint_sink = Recorder()
    z = run.z
    st = state_from(z["particles0"], z["rel_off"], z["win_end_off"], z["release_idx"], cuda_device)
    out = r.start(st, batch_start=run.dt_("batch_start"), cursor_start=run.dt_("cursor_start"),
                  cursor_terminus=run.dt_("cursor_terminus"), sim_length_s=float(z["sim_length_s"]),
                  dt_seconds=float(z["dt_s"])).run()
    sparse.drain()
    asm.finish()
    assert out.status == 0 and len(snapshots) > 0
    n = 0
    for ri, bi, dense in snapshots.values():
        for rr, bb, sl in zip(ri.tolist(), bi.tolist(), dense.cpu().numpy()):
            np.testing.assert_array_equal(_bits(delivered[(rr, bb)].reshape(-1)), _bits(sl))
            n += 1
    assert n == len(delivered)
    # every entry crossed once (plus the slice offsets), however short the speculation was
    n_calls = len(snapshots)
    assert sparse.entries == sum(int((_bits(d.cpu().numpy()) != 0).sum()) for _, _, d in snapshots.values())
    assert sparse.entries * 8 <= sparse.bytes_moved <= 8 * (sparse.entries + sparse.speculated) + 8 * (n + n_calls)
    host = np.stack([blocks.get(i, np.zeros_like(dense_run[0])) for i in range(fp.n_releases)])
    np.testing.assert_allclose(host, dense_run, rtol=1e-5, atol=1e-7)
