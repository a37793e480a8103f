"""Generate ``regrid.npz``: golden outputs of the reference's pressure-level ->
terrain-following (AGL) regrid, run on seeded synthetic columns.

Run in a container that holds the reference source (mrghg/glide) read-only:

    python tests/golden/make_regrid_golden.py --reference /path/to/glide

It imports ``lpdm.vertical_grid`` and reproduces the sequence of
``MetReader._resample_hour_to_agl`` (src/lpdm/met_reader.py:641-693):
``compute_agl_regrid_weights`` -> ``apply_agl_regrid`` of the float32 channels
-> ``terrain_gradient`` + ``slope_correct_w`` of ``w`` -> ``apply_agl_regrid`` of
the float64 pressure and its per-level mean. Two cases: levels stored
top-of-atmosphere first with sub-surface (negative AGL) levels under high terrain
and a descending latitude axis, and levels stored surface first.
"""

from __future__ import annotations

import argparse
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
GRAVITY = 9.80665  # met_reader.GRAVITY_M_S2


def _case(rng, zp: int, ny: int, nx: int, toa_first: bool, lat_descending: bool):
    lat = np.linspace(60.0, 40.0, ny) if lat_descending else np.linspace(40.0, 60.0, ny)
    lon = np.linspace(-10.0, 15.0, nx)
    terrain = np.clip(rng.normal(600.0, 500.0, (ny, nx)), 0.0, 2500.0)
    # pressure-level geometric heights (MSL), plus per-column noise, then AGL
    msl = np.sort(rng.uniform(50.0, 16000.0, zp))
    msl[0] = 100.0
    h_msl = msl[:, None, None] + rng.normal(0.0, 30.0, (zp, ny, nx))
    h_msl = np.sort(h_msl, axis=0)
    height_agl = (h_msl - terrain[None]).astype(np.float32)  # sub-surface levels negative
    p_hpa = 1013.25 * np.exp(-h_msl / 8000.0)
    fields = np.stack([rng.normal(5.0, 8.0, (zp, ny, nx)), rng.normal(0.0, 6.0, (zp, ny, nx)),
                       rng.normal(0.0, 0.1, (zp, ny, nx)), 288.0 - 6.5e-3 * h_msl]).astype(np.float32)
    if toa_first:
        height_agl = height_agl[::-1].copy()
        p_hpa = p_hpa[::-1].copy()
        fields = fields[:, ::-1].copy()
    z_sfc = (terrain * GRAVITY).astype(np.float32)
    return lat, lon, height_agl, p_hpa, fields, z_sfc


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", required=True, help="root of the reference source tree (holds src/lpdm)")
    args = ap.parse_args()
    sys.path.insert(0, str(Path(args.reference) / "src"))
    import torch

    torch.set_num_threads(1)
    from lpdm.vertical_grid import (apply_agl_regrid, compute_agl_regrid_weights, slope_correct_w,
                                    stretched_agl_levels, terrain_gradient)

    rng = np.random.default_rng(20261208)
    out = {}
    for name, (zp, ny, nx, toa, latd) in {"toa": (14, 9, 11, True, True), "sfc": (10, 7, 8, False, False)}.items():
        lat, lon, h, p, f, z_sfc = _case(rng, zp, ny, nx, toa, latd)
        agl = stretched_agl_levels(12, 15000.0, first_layer_m=20.0)
        w = compute_agl_regrid_weights(h, agl)
        arr = apply_agl_regrid(f, w)
        dhdx, dhdy = terrain_gradient(z_sfc / GRAVITY, lat, lon)
        arr[2] = slope_correct_w(arr[2], arr[0], arr[1], dhdx, dhdy, agl, float(agl[-1]))
        p_agl = apply_agl_regrid(np.ascontiguousarray(p)[None], w)[0]
        out.update({f"{name}_lat": lat, f"{name}_lon": lon, f"{name}_height_agl": h, f"{name}_p_hpa": p,
                    f"{name}_fields": f, f"{name}_z_sfc": z_sfc, f"{name}_agl": agl,
                    f"{name}_lower": w.lower.astype(np.int32), f"{name}_frac": w.frac,
                    f"{name}_flipped": np.array(w.flipped), f"{name}_out": arr.astype(np.float32),
                    f"{name}_p_level": p_agl.mean(axis=(1, 2)), f"{name}_dhdx": dhdx, f"{name}_dhdy": dhdy})
    np.savez_compressed(HERE / "regrid.npz", **out)
    print("wrote", HERE / "regrid.npz", sorted(out))


if __name__ == "__main__":
    main()
