"""Oracle of the pressure-level -> terrain-following (AGL) regrid (test infrastructure:
the CUDA path is checked against it, nothing in the package imports it).

numpy restatement of ``lpdm.vertical_grid`` as ``MetReader._resample_hour_to_agl``
uses it (src/lpdm/met_reader.py:641-693):

* ``weights`` — ``compute_agl_regrid_weights`` (vertical_grid.py:166-219): per
  column, levels put surface-first (flipped when the bbox-mean profile is
  top-of-atmosphere first), the insertion index of each target height, the lower
  bracket clamped to the column's first above-ground level and to Zp - 2, the
  fraction (t - h_lo) / max(h_hi - h_lo, 1e-6) clamped to [0, 1], in float64;
* ``apply`` — ``apply_agl_regrid`` (vertical_grid.py:222-258): gather of the two
  bracketing levels in the stored orientation and ``torch.lerp`` with the fraction
  cast to the field's dtype (FMA form of the CPU kernel);
* ``slope_correct_w`` (vertical_grid.py:296-318) in float64, rounded to the field
  dtype; ``terrain_gradient`` (vertical_grid.py:277-293) is ``np.gradient`` as in
  the reference.
"""

from __future__ import annotations

import numpy as np

M_PER_DEG_LAT = 110540.0
M_PER_DEG_LON_EQ = 111320.0


def weights(height_agl_p: np.ndarray, agl_levels: np.ndarray):
    """(lower [Za, Y, X] int, frac [Za, Y, X] float64, flipped)."""
    zp = height_agl_p.shape[0]
    agl = np.asarray(agl_levels, dtype=np.float64)
    mean_profile = np.nanmean(height_agl_p, axis=(1, 2))
    flipped = bool(mean_profile[0] > mean_profile[-1])
    h = np.asarray(height_agl_p, dtype=np.float64)
    if flipped:
        h = h[::-1]
    rows = h.reshape(zp, -1).T  # [cols, Zp], ascending
    idx = np.array([np.searchsorted(r, agl, side="left") for r in rows])  # [cols, Za]
    k0 = (rows < 0.0).sum(axis=1, keepdims=True)
    lower = np.minimum(np.maximum(np.maximum(idx - 1, 0), k0), zp - 2)
    h_lo = np.take_along_axis(rows, lower, axis=1)
    h_hi = np.take_along_axis(rows, lower + 1, axis=1)
    frac = np.clip((agl[None, :] - h_lo) / np.maximum(h_hi - h_lo, 1e-6), 0.0, 1.0)
    shape = (agl.size,) + height_agl_p.shape[1:]
    return lower.T.reshape(shape), frac.T.reshape(shape), flipped


def torch_lerp(s, e, w):
    """torch.lerp(s, e, w) elementwise, the FMA form of the CPU kernel, in s's dtype."""
    dt = s.dtype
    w = w.astype(dt)
    d = (e - s).astype(dt)
    lo = np.abs(w) < 0.5
    # a fused multiply-add rounds once: evaluate in float64 (exact product for float32) and round
    if dt == np.float32:
        a = (w.astype(np.float64) * d.astype(np.float64) + s.astype(np.float64)).astype(np.float32)
        b = ((w - np.float32(1.0)).astype(np.float64) * d.astype(np.float64) + e.astype(np.float64)).astype(np.float32)
    else:
        a = w * d + s
        b = (w - 1.0) * d + e
    return np.where(lo, a, b).astype(dt)


def apply(field_p: np.ndarray, lower: np.ndarray, frac: np.ndarray, flipped: bool) -> np.ndarray:
    """[C, Zp, Y, X] -> [C, Za, Y, X]."""
    zp = field_p.shape[1]
    if flipped:
        lo_idx, hi_idx = (zp - 1) - lower, (zp - 2) - lower
    else:
        lo_idx, hi_idx = lower, lower + 1
    f_lo = np.take_along_axis(field_p, np.broadcast_to(lo_idx, (field_p.shape[0],) + lo_idx.shape), axis=1)
    f_hi = np.take_along_axis(field_p, np.broadcast_to(hi_idx, (field_p.shape[0],) + hi_idx.shape), axis=1)
    return torch_lerp(f_lo, f_hi, np.broadcast_to(frac, f_lo.shape))


def terrain_gradient(terrain_m: np.ndarray, lat: np.ndarray, lon: np.ndarray):
    dh_dlat, dh_dlon = np.gradient(terrain_m, lat, lon)
    m_lon = np.clip(M_PER_DEG_LON_EQ * np.cos(np.deg2rad(lat)), 1.0, None)
    return dh_dlon / m_lon[:, None], dh_dlat / M_PER_DEG_LAT


def slope_correct_w(w, u, v, dhdx, dhdy, agl_levels, z_top_m: float):
    taper = np.clip(1.0 - np.asarray(agl_levels, np.float64) / max(float(z_top_m), 1.0), 0.0, 1.0)
    return (w - taper[:, None, None] * (u * dhdx[None] + v * dhdy[None])).astype(w.dtype)
