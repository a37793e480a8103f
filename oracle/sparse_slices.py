"""Oracle of the sparse footprint-slice form (test infrastructure: the CUDA
compaction is checked against it, nothing in the package imports it).

The reference hands dense ``(release, T, Z, Y, X)`` float32 blocks to
``OutputWriter.write_footprint_region`` (src/lpdm/output_writer.py:215-243). The
sparse form keeps, per slice (one ``[Z, Y, X]`` block), the cells whose float32 (or,
for an FP64 footprint, float64) bit pattern is not zero, in ascending cell order, with the value unchanged; the dense
slice is rebuilt exactly by writing those values into zeros. So the reference's own
dense slice is the golden value of every round trip.
"""

from __future__ import annotations

import numpy as np


def compact(slices: np.ndarray):
    """``slices`` [k, ...] float32 (or float64) -> (slice_offset int64 [k + 1], cell int32
    [total], value [total] of the slices' dtype)."""
    dt = np.float64 if np.asarray(slices).dtype == np.float64 else np.float32
    x = np.ascontiguousarray(slices, dtype=dt).reshape(slices.shape[0], int(np.prod(slices.shape[1:])))
    bits = x.view(np.uint64 if dt == np.float64 else np.uint32)
    cells, values, counts = [], [], []
    for s in range(x.shape[0]):
        nz = np.flatnonzero(bits[s] != 0)
        cells.append(nz.astype(np.int32))
        values.append(x[s, nz])
        counts.append(nz.size)
    offset = np.zeros(x.shape[0] + 1, dtype=np.int64)
    offset[1:] = np.cumsum(counts)
    cat = (lambda parts, t: np.concatenate(parts).astype(t) if parts else np.zeros(0, t))
    return offset, cat(cells, np.int32), cat(values, dt)


def densify(slice_offset: np.ndarray, cell: np.ndarray, value: np.ndarray, slice_shape: tuple) -> np.ndarray:
    """The inverse of ``compact``: [k, *slice_shape] of the values' dtype."""
    k = slice_offset.size - 1
    out = np.zeros((k, int(np.prod(slice_shape))), dtype=np.asarray(value).dtype)
    for s in range(k):
        a, b = int(slice_offset[s]), int(slice_offset[s + 1])
        out[s, cell[a:b]] = value[a:b]
    return out.reshape((k,) + tuple(slice_shape))
