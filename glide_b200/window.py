"""Device-side met windows: raw snapshot fields on the GPU and their packed bricks.

``DeviceMet`` holds the raw float32 fields of the met snapshots on the device
(the reference copies the window to the device once per window,
``HannaScheme._cached_raw_device_met``, src/lpdm/turbulence/hanna.py:747-796);
``PackedWindow`` owns the three bricks the step kernel reads and fills them
with ``glide_window_pack``.
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
