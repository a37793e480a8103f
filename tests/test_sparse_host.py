"""Host side of the sparse footprint slices, without a GPU: the oracle's compaction
round-trips dense slices bit-exactly (-0.0, NaN, inf, subnormals included), the
package's ``densify`` agrees with it, and ``ReleaseAssembler`` hands each release to a
writer with the reference's ``write_footprint_region`` signature as the dense
``(1, T, Z, Y, X)`` block."""

from __future__ import annotations

import numpy as np

from oracle import sparse_slices as osp


def _slices(rng, k, shape, density=0.03):
    x = np.zeros((k,) + shape, dtype=np.float32)
    mask = rng.random(x.shape) < density
    x[mask] = rng.gamma(0.5, 2e-3, mask.sum()).astype(np.float32)
    flat = x.reshape(k, -1)
    if k > 3:
        flat[1] = 0.0  # an empty slice
        flat[2] = rng.normal(size=flat.shape[1]).astype(np.float32)  # every cell non-zero
        flat[3, :5] = np.array([-0.0, np.nan, np.inf, 1e-45, -3.5], dtype=np.float32)
    return x


def test_oracle_round_trip_is_bit_exact():
    rng = np.random.default_rng(1)
    x = _slices(rng, 6, (2, 9, 13))
    off, cell, val = osp.compact(x)
    assert off[0] == 0 and off[-1] == cell.size == val.size
    assert off[2] - off[1] == 0 and off[3] - off[2] == 2 * 9 * 13
    back = osp.densify(off, cell, val, (2, 9, 13))
    np.testing.assert_array_equal(back.view(np.uint32), x.view(np.uint32))
    for s in range(6):  # ascending cells within each slice
        assert np.all(np.diff(cell[off[s]:off[s + 1]]) > 0)
    off0, cell0, val0 = osp.compact(np.zeros((0, 5), np.float32))
    assert off0.tolist() == [0] and cell0.size == 0 and val0.size == 0


def test_package_densify_matches_oracle():
    from glide_b200.sparse import densify

    rng = np.random.default_rng(2)
    x = _slices(rng, 9, (1, 17, 23))
    off, cell, val = osp.compact(x)
    a = densify(off, cell, val, (1, 17, 23))
    np.testing.assert_array_equal(a.view(np.uint32), osp.densify(off, cell, val, (1, 17, 23)).view(np.uint32))
    # buffers longer than the total (the stream's pinned buffers) are cut at the total
    pad_c = np.concatenate([cell, np.full(7, 10**6, np.int32)])
    pad_v = np.concatenate([val, np.ones(7, np.float32)])
    np.testing.assert_array_equal(densify(off, pad_c, pad_v, (1, 17, 23)).view(np.uint32), x.view(np.uint32))


class _FakeWriter:
    """Records ``write_footprint_region`` calls with the reference's checks of the region."""

    def __init__(self):
        self.calls = []

    def write_footprint_region(self, path, footprint, *, release_start, release_stop, dims=None):
        arr = footprint.detach().to(device="cpu").numpy()
        if arr.ndim != 5:
            raise ValueError("footprint must have shape (R, T, Z, Y, X)")
        if arr.shape[0] != release_stop - release_start:
            raise ValueError("footprint leading dim != region size")
        self.calls.append((path, release_start, release_stop, arr.copy()))


def test_release_assembler_writes_dense_regions():
    from glide_b200.sparse import ReleaseAssembler, region_writer

    rng = np.random.default_rng(3)
    n_rel, n_t, shape = 5, 4, (1, 11, 7)
    dense = _slices(rng, n_rel * n_t, shape).reshape((n_rel, n_t) + shape)
    w = _FakeWriter()
    asm = ReleaseAssembler(n_t, shape, region_writer(w, "fp.zarr"))
    # windows deliver the releases' bins in time order, releases interleaved; release 4 never
    # completes its last bin
    for b in range(n_t):
        rel = [r for r in (3, 0, 4, 2, 1) if not (r == 4 and b == n_t - 1)]
        off, cell, val = osp.compact(dense[rel, b])
        # pinned buffers are reused after the call: hand in arrays that get overwritten
        cell_buf, val_buf = cell.copy(), val.copy()
        asm(np.array(rel), np.full(len(rel), b), off, cell_buf, val_buf)
        cell_buf[:] = -1
        val_buf[:] = np.nan
    assert sorted(c[1] for c in w.calls) == [0, 1, 2, 3] and asm.written == 4
    asm.finish()
    assert asm.written == 5 and not asm.open
    for path, r0, r1, arr in w.calls:
        assert path == "fp.zarr" and r1 == r0 + 1 and arr.shape == (1, n_t) + shape
        want = dense[r0].copy()
        if r0 == 4:
            want[n_t - 1] = 0.0
        np.testing.assert_array_equal(arr[0].view(np.uint32), want.view(np.uint32))


def test_release_assembler_sums_a_bin_delivered_twice():
    from glide_b200.sparse import ReleaseAssembler

    got = {}
    asm = ReleaseAssembler(1, (3,), lambda r, block: got.__setitem__(r, block))
    asm(np.array([0]), np.array([0]), np.array([0, 2]), np.array([0, 2], np.int32), np.array([1.0, 2.0], np.float32))
    np.testing.assert_array_equal(got.pop(0), np.array([[1.0, 0.0, 2.0]], np.float32))  # one bin: complete at once
    asm2 = ReleaseAssembler(2, (3,), lambda r, block: got.__setitem__(r, block))
    for part in ((0, [0, 2], [1.0, 2.0]), (0, [2], [0.5]), (1, [1], [4.0])):
        b, c, v = part
        asm2(np.array([7]), np.array([b]), np.array([0, len(c)]), np.array(c, np.int32), np.array(v, np.float32))
    np.testing.assert_array_equal(got[7], np.array([[1.0, 0.0, 2.5], [0.0, 4.0, 0.0]], np.float32))


def test_float64_slices_round_trip_and_assemble():
    """FP64 footprints (``value_f64``): the oracle's compaction keeps float64 values
    bit-exactly, the package's ``densify`` rebuilds them in float64, and the assembler
    hands float64 blocks to the writer when built with ``dtype=np.float64``."""
    from glide_b200.sparse import ReleaseAssembler, densify

    rng = np.random.default_rng(9)
    shape = (1, 7, 11)
    x = _slices(rng, 4, shape).astype(np.float64)
    x.reshape(4, -1)[0, :3] = np.array([5e-324, -0.0, 1.0 + 2.0**-40])  # not representable in float32
    off, cell, val = osp.compact(x)
    assert val.dtype == np.float64
    np.testing.assert_array_equal(osp.densify(off, cell, val, shape).view(np.uint64), x.view(np.uint64))
    np.testing.assert_array_equal(densify(off, cell, val, shape).view(np.uint64), x.view(np.uint64))
    got = {}
    asm = ReleaseAssembler(2, shape, lambda r, block: got.__setitem__(r, block), dtype=np.float64)
    asm(np.array([3, 3]), np.array([0, 1]), off[:3], cell, val)
    assert got[3].dtype == np.float64
    np.testing.assert_array_equal(got[3].reshape(2, -1).view(np.uint64), x[:2].reshape(2, -1).view(np.uint64))
