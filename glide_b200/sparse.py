"""Completed footprint slices leave the device as (cell, value) lists.

The reference copies each batch's dense ``(release, T, Z, Y, X)`` footprint to the
host and hands it to ``OutputWriter.write_footprint_region``
(src/lpdm/output_writer.py:215-243). A slice of one release and one time_ago bin is
mostly zeros (a plume covers a few thousand of the 1.1e5 cells of the EUROPE grid
in an hour), so here the ring footprint's completed slices are compacted on the
device (``glide_footprint_compact``) and only the non-zero cells cross PCIe:

* ``compact_rows`` — one compaction of rows of a ``[n_rows, cells]`` float32 (or
  float64) tensor;
* ``SparseSliceStream`` — a ring-footprint sink (``BatchRunner(footprint_sink=...)``):
  compacts the window's completed slices on the step stream (and clears their ring
  slots), copies the lists to pinned host memory on a copy stream and hands them
  to ``on_host`` once they have landed;
* ``densify`` / ``ReleaseAssembler`` — the host side: slices back to dense blocks,
  gathered per release into the ``(1, T, Z, Y, X)`` regions the reference's writer
  takes (``region_writer``).

A cell is kept when its value's bit pattern is not zero, so ``densify`` rebuilds the
dense slice bit-exactly.
"""

from __future__ import annotations

import ctypes as C
from typing import Callable

import numpy as np
import torch

from glide_b200 import _abi
from glide_b200.window import stream_handle


def _scratch_bytes(k: int, cells: int) -> int:
    nb = C.c_size_t()
    _abi.check(_abi.lib.glide_footprint_compact_scratch_bytes(int(k), int(cells), C.byref(nb)),
               "glide_footprint_compact_scratch_bytes")
    return int(nb.value)


def compact_rows(rows: torch.Tensor, row_index: torch.Tensor, *, clear: bool = False, capacity: int | None = None,
                 status: torch.Tensor | None = None, out: tuple | None = None, scratch: torch.Tensor | None = None,
                 stream: torch.cuda.Stream | None = None):
    """Compacts ``rows[row_index[s]]`` for s in [0, k) on ``stream`` (default: the current
    stream), without synchronising. Returns device tensors ``(slice_offset [k + 1] int64,
    cell [capacity] int32, value [capacity] of the rows' dtype)``; slice s holds entries
    ``[slice_offset[s], slice_offset[s + 1])``. ``capacity`` defaults to ``k * cells``
    (every cell non-zero), which cannot overflow. ``clear`` sets the compacted rows to zero.
    ``out`` reuses ``(slice_offset, cell, value)`` tensors, ``scratch`` a uint8 tensor."""
    if (rows.device.type != "cuda" or rows.dtype not in (torch.float32, torch.float64) or rows.dim() != 2
            or not rows.is_contiguous()):
        raise ValueError("rows must be a contiguous 2-D float32 or float64 CUDA tensor")
    if row_index.dtype != torch.int64 or row_index.device != rows.device or not row_index.is_contiguous():
        raise ValueError("row_index must be a contiguous int64 tensor on the rows' device")
    n_rows, cells = rows.shape
    k = int(row_index.numel())
    cap = k * cells if capacity is None else int(capacity)
    dev = rows.device
    if out is None:
        out = (torch.empty(k + 1, dtype=torch.int64, device=dev),
               torch.empty(max(cap, 1), dtype=torch.int32, device=dev),
               torch.empty(max(cap, 1), dtype=rows.dtype, device=dev))
    off, cell, value = out
    if off.numel() < k + 1 or cell.numel() < cap or value.numel() < cap:
        raise ValueError("output tensors smaller than k + 1 offsets / capacity entries")
    if value.dtype != rows.dtype:
        raise ValueError("the value output must have the rows' dtype")
    need = _scratch_bytes(k, cells)
    if scratch is None or scratch.numel() < need:
        scratch = torch.empty(max(need, 8), dtype=torch.uint8, device=dev)
    a = _abi.CompactArgs()
    a.rows, a.n_rows, a.cells = rows.data_ptr(), n_rows, cells
    a.row_index, a.k, a.clear = row_index.data_ptr(), k, 1 if clear else 0
    a.slice_offset, a.out_cell, a.out_value, a.capacity = off.data_ptr(), cell.data_ptr(), value.data_ptr(), cap
    a.status = None if status is None else status.data_ptr()
    a.scratch, a.scratch_bytes = scratch.data_ptr(), scratch.numel()
    a.value_f64 = 1 if rows.dtype == torch.float64 else 0
    _abi.check(_abi.lib.glide_footprint_compact(C.byref(a), stream_handle(stream)), "glide_footprint_compact")
    return off, cell, value


def densify(slice_offset: np.ndarray, cell: np.ndarray, value: np.ndarray, slice_shape: tuple) -> np.ndarray:
    """(slice_offset [k + 1], cell, value) -> dense slices [k, *slice_shape] of the values' dtype."""
    slice_offset = np.asarray(slice_offset, dtype=np.int64)
    k = slice_offset.size - 1
    n = int(np.prod(slice_shape))
    out = np.zeros((k, n), dtype=np.asarray(value).dtype)
    total = int(slice_offset[-1])
    owner = np.repeat(np.arange(k), np.diff(slice_offset))
    out[owner, np.asarray(cell[:total], dtype=np.int64)] = value[:total]
    return out.reshape((k,) + tuple(slice_shape))


class SparseSliceStream:
    """A ring-footprint sink that moves completed slices to the host as (cell, value) lists.

    Per call (one window's completed (release, bin) slices): ``glide_footprint_compact`` on
    the step stream reads the slices straight from the ring rows and clears them (the
    ring slot is free for a later bin in stream order); on ``copy_stream`` the slice
    offsets and a speculative prefix of the entries (``headroom`` x the call's slices x
    the expected entries per slice: a maximum of the recent calls' mean entries per slice
    that decays by ``decay`` per call) go to pinned host memory. When the call's buffer is needed
    again (or at ``drain()``) the host waits for those copies, copies whatever the
    speculation missed, and calls ``on_host(r_idx, b_idx, slice_offset, cell, value)``
    (numpy arrays, valid during the call). The device buffers are sized for every
    cell of every slice non-zero (8 bytes per cell and slice of a call, per buffer), so
    the compaction never overflows; ``capacity`` sizes them for that many slices up
    front.

    ``bytes_moved`` counts the bytes copied to the host (``speculated`` the entries of the
    speculative copies, ``short_copies`` the calls whose speculation was short and took a
    second copy); ``dense_bytes`` what the dense slices would have been. ``dtype`` is the
    footprint's value type (float32 or float64)."""

    def __init__(self, device, slice_shape: tuple, on_host: Callable | None = None, buffers: int = 2,
                 headroom: float = 1.25, initial_density: float = 1.0 / 32.0, capacity: int = 0,
                 dtype: torch.dtype = torch.float32, decay: float = 0.95) -> None:
        self.device = torch.device(device)
        self.dtype = dtype
        self.value_bytes = torch.empty((), dtype=dtype).element_size()
        self.slice_shape = tuple(int(s) for s in slice_shape)
        self.cells = int(np.prod(self.slice_shape))
        self.on_host = on_host
        self.headroom = float(headroom)
        self.per_slice = float(initial_density) * self.cells  # speculation: entries per slice
        self.decay = float(decay)
        self.speculated = 0
        self.copy_stream = torch.cuda.Stream(device=self.device)
        self.status = torch.zeros(1, dtype=torch.int32, device=self.device)
        self.slots = [{"k": 0, "h": 0} for _ in range(max(1, int(buffers)))]
        self.pending: list = [None] * len(self.slots)
        self.next = 0
        self.bytes_moved = 0
        self.dense_bytes = 0
        self.entries = 0
        self.short_copies = 0  # calls whose speculative copy was too short
        for slot in self.slots:  # `capacity` slices per call allocated up front (more grow the buffers)
            if capacity > 0:
                self._device_buffers(slot, int(capacity))

    def _device_buffers(self, slot: dict, k: int) -> None:
        if "off" in slot and k <= slot["k"]:
            return
        kk = max(k, 1, 2 * slot["k"])
        d = self.device
        slot["k"] = kk
        slot["off"] = torch.empty(kk + 1, dtype=torch.int64, device=d)
        slot["cell"] = torch.empty(kk * self.cells, dtype=torch.int32, device=d)
        slot["value"] = torch.empty(kk * self.cells, dtype=self.dtype, device=d)
        slot["scratch"] = torch.empty(_scratch_bytes(kk, self.cells), dtype=torch.uint8, device=d)
        slot["h_off"] = torch.empty(kk + 1, dtype=torch.int64).pin_memory()
        slot["h_idx"] = torch.empty((2, kk), dtype=torch.int64).pin_memory()

    def _host_entries(self, slot: dict, n: int) -> None:
        if "h_cell" in slot and n <= slot["h"]:
            return
        nn = max(n, 1, int(slot["h"] * 1.5) + 1)
        slot["h"] = nn
        slot["h_cell"] = torch.empty(nn, dtype=torch.int32).pin_memory()
        slot["h_value"] = torch.empty(nn, dtype=self.dtype).pin_memory()

    def _deliver(self, i: int) -> None:
        p = self.pending[i]
        if p is None:
            return
        done, k, spec = p
        done.synchronize()
        self.pending[i] = None
        slot = self.slots[i]
        off = slot["h_off"][: k + 1].numpy()
        total = int(off[k])
        if total > spec:  # the speculation was short: copy the rest now
            self.short_copies += 1
            if total > slot["h"]:  # larger host buffers, keeping the entries that have landed
                old_cell, old_value = slot["h_cell"], slot["h_value"]
                self._host_entries(slot, total)
                slot["h_cell"][:spec].copy_(old_cell[:spec])
                slot["h_value"][:spec].copy_(old_value[:spec])
            with torch.cuda.stream(self.copy_stream):
                slot["h_cell"][spec:total].copy_(slot["cell"][spec:total], non_blocking=True)
                slot["h_value"][spec:total].copy_(slot["value"][spec:total], non_blocking=True)
                ev = self.copy_stream.record_event()
            ev.synchronize()
            self.bytes_moved += (total - spec) * (4 + self.value_bytes)
        if k > 0:  # a call's slices average out: follow their mean density, forget old peaks slowly
            self.per_slice = max(self.per_slice * self.decay, total / k)
        self.entries += total
        if self.on_host is not None:
            idx = slot["h_idx"][:, :k].numpy()
            self.on_host(idx[0].copy(), idx[1].copy(), off.copy(), slot["h_cell"][:total].numpy(),
                         slot["h_value"][:total].numpy())

    def from_rows(self, rows: torch.Tensor, flat: torch.Tensor, r_idx: torch.Tensor, b_idx: torch.Tensor,
                  clear: bool = True) -> None:
        """Slices ``rows[flat[s]]`` ([n_rows, cells] of the stream's dtype, on the current stream's device)
        for (release r_idx[s], bin b_idx[s]); ``clear`` zeroes those rows after reading them
        (``flat`` must then be distinct)."""
        k = int(flat.numel())
        i = self.next
        self.next = (self.next + 1) % len(self.slots)
        self._deliver(i)
        slot = self.slots[i]
        self._device_buffers(slot, k)
        cur = torch.cuda.current_stream(self.device)
        compact_rows(rows, flat, clear=clear, capacity=k * self.cells, status=self.status,
                     out=(slot["off"], slot["cell"], slot["value"]), scratch=slot["scratch"], stream=cur)
        spec = min(k * self.cells, int(np.ceil(self.headroom * self.per_slice * k)))
        self.speculated += spec
        self._host_entries(slot, spec)
        ready = cur.record_event()
        with torch.cuda.stream(self.copy_stream):
            self.copy_stream.wait_event(ready)
            slot["h_off"][: k + 1].copy_(slot["off"][: k + 1], non_blocking=True)
            slot["h_idx"][0, :k].copy_(r_idx, non_blocking=True)
            slot["h_idx"][1, :k].copy_(b_idx, non_blocking=True)
            if spec > 0:
                slot["h_cell"][:spec].copy_(slot["cell"][:spec], non_blocking=True)
                slot["h_value"][:spec].copy_(slot["value"][:spec], non_blocking=True)
            for t in (r_idx, b_idx):  # keep their memory until the copies have run
                t.record_stream(self.copy_stream)
            done = self.copy_stream.record_event()
        self.pending[i] = (done, k, spec)
        self.bytes_moved += spec * (4 + self.value_bytes) + (k + 1) * 8  # footprint data only
        self.dense_bytes += k * self.cells * self.value_bytes

    def __call__(self, r_idx: torch.Tensor, b_idx: torch.Tensor, slices: torch.Tensor) -> None:
        """The dense-slice sink protocol: slices [k, *slice_shape] (left unchanged)."""
        k = int(slices.shape[0])
        rows = slices.reshape(k, self.cells)
        if not rows.is_contiguous():
            rows = rows.contiguous()
        self.from_rows(rows, torch.arange(k, dtype=torch.int64, device=rows.device), r_idx, b_idx, clear=False)

    def drain(self) -> None:
        """Waits for every copy in flight and hands it to ``on_host``; raises if the device
        reported a row outside the ring."""
        for j in range(len(self.slots)):
            self._deliver((self.next + j) % len(self.slots))
        st = int(self.status.item())
        if st:
            self.status.zero_()  # reported once: later drains of good windows succeed
            raise RuntimeError(f"glide_footprint_compact reported status {st:#x}")


class ReleaseAssembler:
    """An ``on_host`` consumer of ``SparseSliceStream``: keeps each release's sparse slices
    until all ``n_time_bins`` of them have arrived, then calls ``write_release(r, block)``
    with the dense ``[T, *slice_shape]`` block (float32, or ``dtype``). ``finish()`` writes
    the releases still open (bins that never arrived are zero)."""

    def __init__(self, n_time_bins: int, slice_shape: tuple, write_release: Callable[[int, np.ndarray], None],
                 dtype=np.float32) -> None:
        self.dtype = np.dtype(dtype)
        self.n_time_bins = int(n_time_bins)
        self.slice_shape = tuple(int(s) for s in slice_shape)
        self.write_release = write_release
        self.open: dict[int, dict[int, tuple]] = {}
        self.written = 0

    def __call__(self, r_idx, b_idx, slice_offset, cell, value) -> None:
        for s, (r, b) in enumerate(zip(r_idx.tolist(), b_idx.tolist())):
            a, e = int(slice_offset[s]), int(slice_offset[s + 1])
            bins = self.open.setdefault(int(r), {})
            # copies: the arrays handed in are only valid during the call
            bins.setdefault(int(b), []).append((np.array(cell[a:e], dtype=np.int64),
                                                np.array(value[a:e], dtype=self.dtype)))
            if len(bins) == self.n_time_bins:
                self._write(int(r))

    def _write(self, r: int) -> None:
        bins = self.open.pop(r)
        block = np.zeros((self.n_time_bins, int(np.prod(self.slice_shape))), dtype=self.dtype)
        for b, parts in bins.items():
            (c, v), rest = parts[0], parts[1:]
            block[b, c] = v  # assigned, not added: the values land bit-unchanged
            for c, v in rest:  # a bin delivered in several parts sums them
                block[b, c] += v
        self.write_release(r, block.reshape((self.n_time_bins,) + self.slice_shape))
        self.written += 1

    def finish(self) -> None:
        for r in sorted(self.open):
            self._write(r)


def region_writer(writer, path: str) -> Callable[[int, np.ndarray], None]:
    """``write_release`` for ``ReleaseAssembler`` that hands each release to a writer with the
    reference's ``write_footprint_region(path, footprint, *, release_start, release_stop)``
    (footprint ``(1, T, Z, Y, X)``, a CPU tensor)."""

    def write(r: int, block: np.ndarray) -> None:
        writer.write_footprint_region(path, torch.from_numpy(block[None]), release_start=r, release_stop=r + 1)

    return write
