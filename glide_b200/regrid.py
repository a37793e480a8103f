"""Pressure-level -> terrain-following (AGL) regrid of met hours on the device.

The reference's met reader resamples every hour from pressure (or model) levels
onto a fixed above-ground-level grid on its host prefetch thread
(``MetReader._resample_hour_to_agl``, src/lpdm/met_reader.py:641-693, using
src/lpdm/vertical_grid.py:166-318): per-column bracketing that skips sub-surface
levels, linear interpolation of every channel, a slope correction of ``w`` into
the terrain-following frame, and the per-level bbox-mean pressure.
``regrid_hour_to_agl`` does the same with one ``glide_agl_regrid`` call and
returns what that method returns. The terrain slopes (``np.gradient`` of the
surface height, the reference's ``terrain_gradient``) are computed once per
terrain on the host.
"""

from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from glide_b200 import _abi
from glide_b200.window import stream_handle

GRAVITY = 9.80665
M_PER_DEG_LAT = 110540.0
M_PER_DEG_LON_EQ = 111320.0


def terrain_gradient(terrain_m: np.ndarray, lat_deg: np.ndarray, lon_deg: np.ndarray):
    """(dh/dx east, dh/dy north) in m/m, [Y, X], with numpy's dtypes: dh/dx float64 and, for a
    float32 terrain, dh/dy float32 (vertical_grid.py:277-293)."""
    dh_dlat, dh_dlon = np.gradient(terrain_m, lat_deg, lon_deg)
    m_lon = np.clip(M_PER_DEG_LON_EQ * np.cos(np.deg2rad(lat_deg)), 1.0, None)
    return dh_dlon / m_lon[:, None], dh_dlat / M_PER_DEG_LAT


def _dev(x, dtype, device) -> torch.Tensor:
    t = torch.as_tensor(x)
    if t.device.type != "cuda":
        t = t.to(dtype=dtype).contiguous().pin_memory().to(device, non_blocking=True)
    return t.to(device=device, dtype=dtype).contiguous()


def regrid_hour_to_agl(tensor_p, height_agl_p, agl_levels, channel_names, *, z_sfc=None, lat=None, lon=None,
                       pressure_p_hpa=None, device="cuda", stream=None):
    """Regrid one hour's ``[C, Zp, Y, X]`` channels onto ``agl_levels``.

    ``height_agl_p`` [Zp, Y, X]: AGL height of each stored level (negative below
    ground). With ``u``, ``v``, ``w`` among ``channel_names`` and the surface
    geopotential ``z_sfc`` [Y, X] (m^2/s^2) and ``lat`` / ``lon``, ``w`` is
    slope-corrected. Returns ``(tensor_agl [C, Za, Y, X] float32 on the device,
    agl_levels float64, pressure_level_hpa [Za] float64 or None)``."""
    device = torch.device(device)
    stream = stream if stream is not None else torch.cuda.current_stream(device)
    agl = np.ascontiguousarray(np.asarray(agl_levels, dtype=np.float64))
    with torch.cuda.stream(stream):
        f = _dev(tensor_p, torch.float32, device)
        h = _dev(height_agl_p, torch.float32, device)
        nc, zp, ny, nx = f.shape
        if tuple(h.shape) != (zp, ny, nx):
            raise ValueError(f"height_agl_p {tuple(h.shape)} must match the channels' {(zp, ny, nx)}")
        out = torch.empty((nc, agl.size, ny, nx), dtype=torch.float32, device=device)
        nb = C.c_size_t()
        _abi.check(_abi.lib.glide_agl_regrid_scratch_bytes(agl.size, ny, nx, C.byref(nb)),
                   "glide_agl_regrid_scratch_bytes")
        scratch = torch.empty(nb.value, dtype=torch.uint8, device=device)
        a = _abi.RegridArgs()
        a.n_channels, a.zp, a.za, a.ny, a.nx = nc, zp, agl.size, ny, nx
        a.height_agl_p, a.fields_p, a.fields_agl = h.data_ptr(), f.data_ptr(), out.data_ptr()
        a.agl_levels = agl.ctypes.data
        a.u_channel = a.v_channel = a.w_channel = -1
        keep = []
        names = list(channel_names)
        if z_sfc is not None and all(k in names for k in ("u", "v", "w")):
            z = np.asarray(z_sfc.cpu() if isinstance(z_sfc, torch.Tensor) else z_sfc)
            if z.ndim == 3:
                z = z[0]
            dhdx, dhdy = terrain_gradient(z / GRAVITY, np.asarray(lat), np.asarray(lon))
            dx, dy = _dev(dhdx, torch.float64, device), _dev(dhdy, torch.float64, device)
            keep += [dx, dy]
            a.u_channel, a.v_channel, a.w_channel = names.index("u"), names.index("v"), names.index("w")
            a.dhdx, a.dhdy = dx.data_ptr(), dy.data_ptr()
            # the slopes keep numpy's dtypes' arithmetic: a float32 slope multiplies in float32
            a.slope_f32 = (1 if np.asarray(dhdx).dtype == np.float32 else 0) | \
                (2 if np.asarray(dhdy).dtype == np.float32 else 0)
            a.z_top_m = float(agl[-1])
        p_level = None
        if pressure_p_hpa is not None:
            p = _dev(pressure_p_hpa, torch.float64, device)
            p_level = torch.empty(agl.size, dtype=torch.float64, device=device)
            keep += [p]
            a.pressure_p_hpa, a.pressure_level_hpa = p.data_ptr(), p_level.data_ptr()
        a.scratch, a.scratch_bytes = scratch.data_ptr(), nb.value
        _abi.check(_abi.lib.glide_agl_regrid(C.byref(a), stream_handle(stream)), "glide_agl_regrid")
    return out, agl, (None if p_level is None else p_level.cpu().numpy())
