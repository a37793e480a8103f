"""Device-side met windows: raw snapshot fields on the GPU and their packed bricks.

``WindowFields`` holds the raw float32 fields of a window's two snapshots on the
device (the reference copies the window to the device once per window,
``HannaScheme._cached_raw_device_met``, src/lpdm/turbulence/hanna.py:747-796);
``PackedWindow`` owns the three bricks the step kernel reads and fills them
with ``glide_window_pack``; ``HostMetStreamer`` serves windows from host memory
with prefetch.
"""

from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from datetime import datetime

import numpy as np
import torch

from glide_b200 import _abi

MET_DTYPES = {"f32": _abi.GLIDE_MET_F32, "bf16": _abi.GLIDE_MET_BF16, "f16": _abi.GLIDE_MET_F16}
THREE_D = ("u", "v", "w", "t", "q")
TWO_D = ("blh", "sp", "ustar", "shf")


def _ptr(t: torch.Tensor | None) -> int | None:
    return None if t is None else t.data_ptr()


def stream_handle(stream: torch.cuda.Stream | None = None) -> int:
    s = stream if stream is not None else torch.cuda.current_stream()
    return s.cuda_stream


@dataclass
class GridInfo:
    """Geometry of a met grid (the reference's ``GridInterpolationBounds``)."""

    lon: np.ndarray
    lat: np.ndarray
    level: np.ndarray
    pressure_level_hpa: np.ndarray
    level_sorted_dev: torch.Tensor = field(repr=False, default=None)
    p_hpa_dev: torch.Tensor = field(repr=False, default=None)
    height_level_dev: torch.Tensor = field(repr=False, default=None)
    level_lut_dev: torch.Tensor = field(repr=False, default=None)
    lut_inv_dz: float = 0.0

    @property
    def shape(self) -> tuple[int, int, int]:
        return (len(self.level), len(self.lat), len(self.lon))

    @property
    def ascending(self) -> bool:
        return bool(self.level[-1] > self.level[0])

    def level_lut(self, max_entries: int = 4096) -> tuple[np.ndarray, float]:
        """Bucket table of the level search: ``lut[b] = searchsorted(level, b / inv_dz)``
        (float32 levels, left insertion), buckets no wider than the thinnest layer."""
        lv = np.sort(np.asarray(self.level, dtype=np.float32))
        thinnest = float(np.min(np.diff(lv.astype(np.float64)))) if lv.size > 1 else 1.0
        top = float(lv[-1]) if float(lv[-1]) > 0 else 1.0
        n = int(min(max_entries, max(2, np.ceil(top / max(thinnest, 1e-3)) + 1)))
        inv_dz = np.float32((n - 1) / top)
        edges = (np.arange(n, dtype=np.float64) / np.float64(inv_dz)).astype(np.float32)
        lut = np.searchsorted(lv, edges, side="left").astype(np.int32)
        return lut, float(inv_dz)

    def to_device(self, device) -> GridInfo:
        lut, inv = self.level_lut()
        self.level_lut_dev = torch.as_tensor(lut, device=device)
        self.lut_inv_dz = inv
        self.level_sorted_dev = torch.as_tensor(np.sort(np.asarray(self.level, dtype=np.float32)), device=device)
        self.p_hpa_dev = torch.as_tensor(np.asarray(self.pressure_level_hpa, dtype=np.float32), device=device)
        self.height_level_dev = torch.as_tensor(np.asarray(self.level, dtype=np.float32), device=device)
        return self

    def c_grid(self) -> _abi.Grid:
        nz, ny, nx = self.shape
        lut = self.level_lut_dev
        return _abi.Grid(nz, ny, nx, 1 if self.ascending else 0, float(self.lon[0]), float(self.lon[-1]),
                         float(self.lat[0]), float(self.lat[-1]), self.level_sorted_dev.data_ptr(),
                         None if lut is None else lut.data_ptr(), 0 if lut is None else lut.numel(),
                         self.lut_inv_dz)


@dataclass
class Snapshot:
    """Raw float32 device fields of one hourly snapshot: 3-D ``[Z, Y, X]`` (t, u, v, w, q)
    and 2-D ``[Y, X]`` (blh, sp, ustar, shf, t_lowest)."""

    time: datetime
    fields: dict

    def __getitem__(self, k):
        return self.fields[k]


@dataclass
class WindowFields:
    """The two snapshots of one window plus the per-column heights."""

    start: Snapshot
    end: Snapshot
    grid: GridInfo
    height3d: torch.Tensor | None = None  # [Z, Y, X] or None (level broadcast)

    @property
    def time_start(self) -> datetime:
        return self.start.time

    @property
    def time_end(self) -> datetime:
        return self.end.time


def _contig_plane(t: torch.Tensor, device) -> torch.Tensor:
    t = t.to(device=device, dtype=torch.float32, non_blocking=True)
    return t if t.is_contiguous() else t.contiguous()


def window_from_hourly(win, grid: GridInfo, device, lowest: int | None = None) -> WindowFields:
    """Device ``WindowFields`` from a reference-format ``HourlyMetTensors`` window."""
    names = win.channel_names
    lowest = int(np.argmin(np.asarray(win.metadata.level))) if lowest is None else lowest
    snaps = []
    for s, tt in ((0, win.metadata.time_start), (1, win.metadata.time_end)):
        src = win.hour_start if s == 0 else win.hour_end
        f = {}
        for name in THREE_D:
            if name in names:
                f[name] = _contig_plane(src[names.index(name)], device)
        for name in TWO_D:
            f[name] = _contig_plane(src[names.index(name)][0], device)
        f["t_lowest"] = f["t"][lowest] if f["t"][lowest].is_contiguous() else f["t"][lowest].contiguous()
        snaps.append(Snapshot(tt, f))
    h3 = None
    if win.height_agl_m is not None:
        h = win.height_agl_m
        lev = torch.as_tensor(np.asarray(win.metadata.level, dtype=np.float32)).view(-1, 1, 1)
        if not (h.stride(1) == 0 and h.stride(2) == 0 and torch.equal(h[:, :1, :1].cpu().float(), lev)):
            h3 = _contig_plane(h, device)
    return WindowFields(snaps[0], snaps[1], grid, h3)


class PackedWindow:
    """Packed bricks of one window (wind, surface, support) in device memory."""

    def __init__(self, grid: GridInfo, met_dtype: str, device) -> None:
        nz, ny, nx = grid.shape
        self.grid = grid
        self.met_dtype = met_dtype
        self.code = MET_DTYPES[met_dtype]
        wb, sb, pb = C.c_size_t(), C.c_size_t(), C.c_size_t()
        _abi.check(_abi.lib.glide_window_packed_bytes(nz, ny, nx, self.code, C.byref(wb), C.byref(sb), C.byref(pb)),
                   "glide_window_packed_bytes")
        # 16-byte aligned storage (torch allocations are 512-byte aligned)
        self.wind = torch.empty(wb.value, dtype=torch.uint8, device=device)
        self.surf = torch.empty(sb.value, dtype=torch.uint8, device=device)
        self.support = torch.empty(pb.value, dtype=torch.uint8, device=device)
        # sums of u, v, w of the start and end snapshots over all cells (the grid means of the
        # runtime's wind diagnostic), written by pack()
        self.wind_sum = torch.zeros(6, dtype=torch.float64, device=device)
        self.key = None

    @property
    def nbytes(self) -> int:
        return self.wind.numel() + self.surf.numel() + self.support.numel()

    def pack(self, wf: WindowFields, *, meander_coefficient: float = 0.16, meander_radius: int = 1,
             build_meander: bool = True, stream=None) -> None:
        d = _abi.WindowDesc()
        d.grid = wf.grid.c_grid()
        for s, snap in enumerate((wf.start, wf.end)):
            d.u[s] = snap["u"].data_ptr()
            d.v[s] = snap["v"].data_ptr()
            d.w[s] = snap["w"].data_ptr()
            d.t[s] = snap["t"].data_ptr()
            d.t_lowest[s] = snap["t_lowest"].data_ptr()
            d.blh[s] = snap["blh"].data_ptr()
            d.sp[s] = snap["sp"].data_ptr()
            d.ustar[s] = snap["ustar"].data_ptr()
            d.shf[s] = snap["shf"].data_ptr()
        d.height3d = _ptr(wf.height3d)
        d.height_level = wf.grid.height_level_dev.data_ptr()
        d.pressure_hpa = wf.grid.p_hpa_dev.data_ptr()
        d.meander_coefficient = float(meander_coefficient)
        d.meander_radius = int(meander_radius)
        d.build_meander = 1 if build_meander else 0
        d.met_dtype = self.code
        d.wind_packed = self.wind.data_ptr()
        d.surf_packed = self.surf.data_ptr()
        d.support_packed = self.support.data_ptr()
        d.wind_sum = self.wind_sum.data_ptr()
        with torch.cuda.stream(stream if stream is not None else torch.cuda.current_stream()):
            self.wind_sum.zero_()
        _abi.check(_abi.lib.glide_window_pack(C.byref(d), stream_handle(stream)), "glide_window_pack")
        self.key = wf.time_start

    def typed(self, which: str) -> torch.Tensor:
        """A brick viewed as float32 [.., 8|16] (float32 storage only; for tests)."""
        buf = getattr(self, which)
        if self.met_dtype == "f32":
            v = buf.view(torch.float32)
        elif self.met_dtype == "bf16":
            v = buf.view(torch.bfloat16).float()
        else:
            v = buf.view(torch.float16).float()
        nz, ny, nx = self.grid.shape
        return v.view(ny, nx, 16) if which == "surf" else v.view(nz, ny, nx, 8)


def grid_from_synthetic(syn) -> GridInfo:
    return GridInfo(np.asarray(syn.lon), np.asarray(syn.lat), np.asarray(syn.levels),
                    np.asarray(syn.pressure_level_hpa))


def window_from_synthetic(syn, h: int, grid: GridInfo) -> WindowFields:
    """Device ``WindowFields`` of bracket ``[h, h+1]`` of a ``SyntheticMet`` whose fields
    already live on the device (no copy)."""
    lowest = int(np.argmin(syn.levels))
    snaps = []
    for k in (h, h + 1):
        f = dict(syn.fields[k])
        f["t_lowest"] = f["t"][lowest]
        snaps.append(Snapshot(syn.times[k], f))
    return WindowFields(snaps[0], snaps[1], grid, None)


def window_from_arrays(fields: dict, h: int, times: list, grid: GridInfo, device, lowest: int = 0) -> WindowFields:
    """Device ``WindowFields`` from stacked host arrays ``fields[name][snapshot]``."""
    snaps = []
    for k in (h, h + 1):
        f = {n: torch.as_tensor(np.ascontiguousarray(fields[n][k]), dtype=torch.float32, device=device)
             for n in fields}
        f["t_lowest"] = f["t"][lowest]
        snaps.append(Snapshot(times[k], f))
    return WindowFields(snaps[0], snaps[1], grid, None)


class HostMetStreamer:
    """Streams hourly snapshots from (pinned) host memory to the device.

    The device holds ``slots`` snapshot buffers. A window ``[h, h+1]`` needs two;
    walking backward, the next window needs one new snapshot, which
    ``prefetch(hour)`` copies on a side stream while the current window computes
    (the device-side counterpart of the reference's ``MetPrefetcher``,
    src/lpdm/main.py:791-889). A slot is overwritten only after the compute stream
    has passed the point where its previous snapshot was last used.

    ``host_snapshot(k)`` returns snapshot ``k`` as a dict of host tensors (3-D
    ``[Z, Y, X]``: u, v, w, t, q; 2-D ``[Y, X]``: blh, sp, ustar, shf); ``times[k]``
    is its time.
    """

    NAMES = ("u", "v", "w", "t", "q", "blh", "sp", "ustar", "shf")

    def __init__(self, host_snapshot, times: list, grid: GridInfo, device, lowest: int = 0, slots: int = 3) -> None:
        if slots < 3:
            raise ValueError("need at least 3 snapshot slots (two in use, one being filled)")
        self.host_snapshot = host_snapshot
        self.times = list(times)
        self.grid = grid
        self.device = torch.device(device)
        self.lowest = lowest
        self.copy_stream = torch.cuda.Stream(device=self.device)
        self.slots: list[dict] = []
        self.slot_of: dict[int, int] = {}
        self.ready: dict[int, torch.cuda.Event] = {}
        self.free_after: list[torch.cuda.Event | None] = [None] * slots
        self.n_slots = slots
        self.bytes_copied = 0
        self.t0 = self.times[0]

    def _index(self, hour: datetime) -> int:
        return int(round((hour - self.t0).total_seconds() / 3600.0))

    def _alloc(self, like: dict) -> dict:
        return {k: torch.empty(v.shape, dtype=torch.float32, device=self.device) for k, v in like.items()}

    def _load(self, k: int, keep: set) -> None:
        """Start copying snapshot k into a free slot (on the copy stream)."""
        if k in self.slot_of or k < 0 or k >= len(self.times):
            return
        host = self.host_snapshot(k)
        used = set(self.slot_of.values())
        if len(self.slots) < self.n_slots:
            self.slots.append(self._alloc(host))
            slot = len(self.slots) - 1
        else:
            victims = [(s, kk) for kk, s in self.slot_of.items() if kk not in keep]
            if not victims:
                raise RuntimeError("no free snapshot slot")
            slot, kk = max(victims, key=lambda v: v[1])  # the cursor walks backward: drop the latest
            del self.slot_of[kk]
            self.ready.pop(kk, None)
        del used
        ev_free = self.free_after[slot]
        with torch.cuda.stream(self.copy_stream):
            if ev_free is not None:
                self.copy_stream.wait_event(ev_free)
            for name, src in host.items():
                self.slots[slot][name].copy_(src, non_blocking=True)
                self.bytes_copied += src.numel() * src.element_size()
            ev = torch.cuda.Event()
            ev.record(self.copy_stream)
        self.slot_of[k] = slot
        self.ready[k] = ev

    def _snapshot(self, k: int) -> Snapshot:
        slot = self.slots[self.slot_of[k]]
        torch.cuda.current_stream(self.device).wait_event(self.ready[k])
        f = dict(slot)
        f["t_lowest"] = f["t"][self.lowest]
        return Snapshot(self.times[k], f)

    def __call__(self, hour: datetime) -> WindowFields:
        h = self._index(hour)
        self._load(h + 1, {h, h + 1})
        self._load(h, {h, h + 1})
        return WindowFields(self._snapshot(h), self._snapshot(h + 1), self.grid, None)

    def window_done(self, hour: datetime) -> None:
        """Marks the point of the compute stream after which the window's snapshots
        may be overwritten (called once the window's launches are issued)."""
        h = self._index(hour)
        ev = torch.cuda.Event()
        ev.record(torch.cuda.current_stream(self.device))
        for k in (h, h + 1):
            if k in self.slot_of:
                self.free_after[self.slot_of[k]] = ev

    def prefetch(self, hour: datetime) -> None:
        """Starts the copy of the snapshots window ``hour`` needs, keeping the
        current window's (the one after it in time) resident."""
        h = self._index(hour)
        self._load(h, {h, h + 1, h + 2})
        self._load(h + 1, {h, h + 1, h + 2})
