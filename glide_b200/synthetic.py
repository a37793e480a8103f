"""Seeded synthetic meteorology and releases.

There is no ERA5 data here, so every workload runs on synthetic met with the
shapes and value distributions of the reference's EUROPE-box runs
(``configs/example_multisite_january.yaml``):

* levels: a geometrically stretched terrain-following AGL ladder from 0 to
  20 km whose first layer is 10 m thick (the reference's
  ``vertical_grid.stretched_agl_levels``, ``src/lpdm/vertical_grid.py:70-144``:
  layer k is ``first * r**k`` thick, ``r`` solved so the layers span the top);
* horizontal grid: 0.25 deg cell centres ``lon0 + 0.25 i``, ``lat0 + 0.25 j``;
* winds: ``U_ref ln(max(z, z0)/z0)/ln(10/z0) (cos th, sin th)`` plus a Gaussian
  random field (GRF: white noise filtered by a Gaussian of 4 cells, unit
  variance after rescaling, correlated over 2 levels vertically) of 5 m/s;
* ``w``: GRF of 0.05 m/s, then the terrain-following correction
  ``w - (1 - z/z_top) (u dh/dx + v dh/dy)`` (``vertical_grid.py:296-316``);
* terrain GRF mapped to 0-500 m; ``sp = 101325 exp(-terrain/8000)``;
* boundary layer: ``blh ~ U(300, 1500)`` m and ``ustar ~ U(0.1, 0.6)`` m/s
  (GRF mapped through the normal CDF); a stability regime per column
  (stable ``L ~ U(10, 500)``, neutral ``|L| = 1e5``, unstable
  ``L ~ U(-500, -10)``) turned into ``shf = -u*^3 T rho c_p / (kappa g L)``,
  clipped to +-200 W/m2;
* ``t``: a dry-adiabatic mixed layer to 1.2 km, 6.5 K/km above (>= 216.65 K),
  plus GRF(1 K); the surface level is 0.8 K warmer (6.8 K in moist columns);
* ``q = q_sfc exp(-z/2500)``; a seeded fraction of columns (20 % by default)
  is moist-unstable (``q_sfc`` 10 g/kg, warm surface), the rest 7.5 g/kg;
* time: each hourly snapshot's random parts follow an AR(1) with correlation
  0.7 to the previous hour.

Everything is generated with torch (CPU or CUDA) from one integer seed.
"""

from __future__ import annotations

import math
from dataclasses import dataclass, field
from datetime import UTC, datetime, timedelta

import numpy as np
import torch

from glide_b200.met import HourlyMetTensors, MetFieldMetadata

KARMAN = 0.4
GRAVITY = 9.80665
R_DRY = 287.05
C_P = 1005.0

THREE_D = ("u", "v", "w", "t", "q")
TWO_D = ("blh", "sp", "ustar", "shf")


def stretched_agl_levels(n_levels: int, alt_max_m: float, first_layer_m: float = 10.0) -> np.ndarray:
    """Ascending AGL heights ``[n_levels]`` from 0 to ``alt_max_m``; the first layer is
    ``first_layer_m`` thick and each higher layer a constant ratio thicker.

    The benchmark levels are defined as the reference's ``stretched_agl_levels``
    (src/lpdm/vertical_grid.py:70-144), so this follows its steps: the geometric-series
    span in closed form, the ratio bracketed by doubling from [1, 2] and bisected 200
    times, the cumulative sum of the layer thicknesses with the top pinned to
    ``alt_max_m``."""
    if n_levels < 2:
        raise ValueError("n_levels must be >= 2")
    n_layers = n_levels - 1
    if n_layers == 1:
        return np.array([0.0, float(alt_max_m)])
    if first_layer_m * n_layers >= alt_max_m:
        raise ValueError("first layer too thick for the requested ladder")

    def span(r: float) -> float:
        return first_layer_m * n_layers if abs(r - 1.0) < 1e-12 else first_layer_m * (r**n_layers - 1.0) / (r - 1.0)

    lo, hi = 1.0, 2.0
    while span(hi) < alt_max_m:
        hi *= 2.0
    for _ in range(200):
        mid = 0.5 * (lo + hi)
        if span(mid) < alt_max_m:
            lo = mid
        else:
            hi = mid
    r = 0.5 * (lo + hi)
    levels = np.concatenate(([0.0], np.cumsum(first_layer_m * r ** np.arange(n_layers, dtype=np.float64))))
    levels[-1] = float(alt_max_m)
    return levels


@dataclass
class SyntheticMetSpec:
    nz: int = 40
    ny: int = 64
    nx: int = 64
    lon0: float = 0.0
    lat0: float = 40.0
    dlon: float = 0.25
    dlat: float = 0.25
    n_snapshots: int = 4
    alt_max_m: float = 20000.0
    first_layer_m: float = 10.0
    seed: int = 20261203
    moist_fraction: float = 0.2
    start_time: datetime = field(default_factory=lambda: datetime(2026, 1, 15, 0, tzinfo=UTC))
    wind_pert_m_s: float = 5.0
    u_ref_m_s: float = 5.0


def config_met_spec(index: int, n_snapshots: int | None = None) -> SyntheticMetSpec:
    """Met spec of the named workloads: 0 = 64x64x40 CPU smoke case,
    1 = 281x401x60 EUROPE box (25 hourly snapshots)."""
    if index == 0:
        return SyntheticMetSpec(nz=40, ny=64, nx=64, lon0=0.0, lat0=40.0, n_snapshots=n_snapshots or 4,
                                seed=20261203, moist_fraction=0.0)
    if index == 1:
        return SyntheticMetSpec(nz=60, ny=281, nx=401, lon0=-60.0, lat0=10.0, n_snapshots=n_snapshots or 25,
                                seed=20261204)
    raise ValueError(f"no met spec for workload {index}")


def _gaussian_filter_1d(x: torch.Tensor, sigma: float, dim: int) -> torch.Tensor:
    radius = max(1, int(math.ceil(3 * sigma)))
    k = torch.arange(-radius, radius + 1, device=x.device, dtype=x.dtype)
    kern = torch.exp(-0.5 * (k / sigma) ** 2)
    kern = kern / kern.sum()
    x = x.movedim(dim, -1)
    shp = x.shape
    flat = x.reshape(-1, 1, shp[-1])
    padded = torch.nn.functional.pad(flat, (radius, radius), mode="replicate")
    out = torch.nn.functional.conv1d(padded, kern.view(1, 1, -1)).reshape(shp)
    return out.movedim(-1, dim)


def gaussian_random_field(gen: torch.Generator, shape: tuple[int, ...], sigma_cells: float,
                          device, z_sigma: float | None = None) -> torch.Tensor:
    """Unit-variance GRF over the last two axes (FFT Gaussian filter of white noise),
    optionally correlated along axis -3 by a Gaussian of ``z_sigma`` levels."""
    noise = torch.randn(shape, generator=gen, device=device, dtype=torch.float32)
    ny, nx = shape[-2], shape[-1]
    ky = torch.fft.fftfreq(ny, device=device).view(-1, 1)
    kx = torch.fft.rfftfreq(nx, device=device).view(1, -1)
    filt = torch.exp(-2.0 * math.pi**2 * sigma_cells**2 * (ky**2 + kx**2))
    f = torch.fft.irfft2(torch.fft.rfft2(noise) * filt, s=(ny, nx))
    if z_sigma is not None and len(shape) >= 3 and shape[-3] > 1:
        f = _gaussian_filter_1d(f, z_sigma, dim=len(shape) - 3)
    f = f - f.mean()
    return f / f.std().clamp(min=1e-12)


class SyntheticMet:
    """Hourly synthetic snapshots for one workload.

    ``fields[h][name]`` holds snapshot ``h``: 3-D fields ``[Z, Y, X]`` and 2-D
    fields ``[Y, X]`` (float32, on ``device``). ``window(h)`` returns the
    ``[h, h+1]`` bracket in the reference's ``HourlyMetTensors`` layout.
    """

    def __init__(self, spec: SyntheticMetSpec, device: str | torch.device = "cpu") -> None:
        self.spec = spec
        self.device = torch.device(device)
        s = spec
        self.levels = stretched_agl_levels(s.nz, s.alt_max_m, s.first_layer_m)
        self.lon = s.lon0 + s.dlon * np.arange(s.nx, dtype=np.float64)
        self.lat = s.lat0 + s.dlat * np.arange(s.ny, dtype=np.float64)
        self.times = [s.start_time + timedelta(hours=h) for h in range(s.n_snapshots)]
        gen = torch.Generator(device=self.device)
        gen.manual_seed(int(s.seed))
        dev = self.device
        z = torch.as_tensor(self.levels, dtype=torch.float32, device=dev).view(-1, 1, 1)
        shape3 = (s.nz, s.ny, s.nx)
        shape2 = (s.ny, s.nx)
        ndtr = torch.special.ndtr

        terrain = 500.0 * ndtr(gaussian_random_field(gen, shape2, 4.0, dev))
        sp = 101325.0 * torch.exp(-terrain / 8000.0)
        lat_rad = torch.deg2rad(torch.as_tensor(self.lat, dtype=torch.float32, device=dev))
        dh_dlat, dh_dlon = torch.gradient(terrain, spacing=(s.dlat, s.dlon))
        dhdx = dh_dlon / (111320.0 * torch.cos(lat_rad).clamp(min=1e-3)).view(-1, 1)
        dhdy = dh_dlat / 110540.0
        taper = (1.0 - z / max(s.alt_max_m, 1.0)).clamp(0.0, 1.0)
        moist = ndtr(gaussian_random_field(gen, shape2, 3.0, dev)) < s.moist_fraction
        self.terrain = terrain
        self.moist_mask = moist

        z0 = 0.1
        profile = torch.log(torch.clamp(z, min=z0) / z0) / math.log(10.0 / z0)
        # dry-adiabatic mixed layer to 1.2 km, 6.5 K/km above (floored at 216.65 K)
        t_base = torch.clamp(288.0 - 9.8e-3 * torch.clamp(z, max=1200.0)
                             - 6.5e-3 * torch.clamp(z - 1200.0, min=0.0), min=216.65)
        # surface-level excess (0.8 K everywhere, +6 K in moist-unstable columns) and a
        # humid boundary layer there: the parcel lift of those columns triggers deep convection
        excess = (0.8 + torch.where(moist, 6.0, 0.0)).unsqueeze(0) * (z == 0.0).float()
        t_base_col = t_base + excess
        q_sfc = torch.where(moist, 0.010, 0.0075)
        q_base = q_sfc * torch.exp(-z / 2500.0)

        rho_ar = 0.7
        keep = math.sqrt(1.0 - rho_ar**2)
        state: dict[str, torch.Tensor] = {}

        def ar(key: str, fresh: torch.Tensor) -> torch.Tensor:
            prev = state.get(key)
            nxt = fresh if prev is None else rho_ar * prev + keep * fresh
            state[key] = nxt
            return nxt

        theta0 = float(torch.rand((), generator=gen, device=dev)) * 2.0 * math.pi
        self.fields: list[dict[str, torch.Tensor]] = []
        for h in range(s.n_snapshots):
            th = theta0 + 0.15 * h
            gu = ar("u", gaussian_random_field(gen, shape3, 4.0, dev, z_sigma=2.0))
            gv = ar("v", gaussian_random_field(gen, shape3, 4.0, dev, z_sigma=2.0))
            gw = ar("w", gaussian_random_field(gen, shape3, 4.0, dev, z_sigma=2.0))
            gt = ar("t", gaussian_random_field(gen, shape3, 4.0, dev, z_sigma=2.0))
            gq = ar("q", gaussian_random_field(gen, shape3, 4.0, dev, z_sigma=2.0))
            gb = ar("blh", gaussian_random_field(gen, shape2, 4.0, dev))
            gs = ar("ustar", gaussian_random_field(gen, shape2, 4.0, dev))
            gr = ar("regime", gaussian_random_field(gen, shape2, 3.0, dev))
            gl = ar("lmag", gaussian_random_field(gen, shape2, 3.0, dev))

            u = s.u_ref_m_s * profile * math.cos(th) + s.wind_pert_m_s * gu
            v = s.u_ref_m_s * profile * math.sin(th) + s.wind_pert_m_s * gv
            w = 0.05 * gw - taper * (u * dhdx + v * dhdy)
            t = t_base_col + 1.0 * gt
            q = torch.clamp(q_base * (1.0 + 0.1 * gq), min=0.0)
            blh = 300.0 + 1200.0 * ndtr(gb)
            ustar = 0.1 + 0.5 * ndtr(gs)
            r = ndtr(gr)
            lm = ndtr(gl)
            L = torch.where(r < 1.0 / 3.0, 10.0 + 490.0 * lm,
                            torch.where(r < 2.0 / 3.0, torch.full_like(lm, 1e5), -(10.0 + 490.0 * lm)))
            t_sfc = t[0]
            rho = sp / (R_DRY * t_sfc)
            shf = torch.clamp(-(ustar**3) * t_sfc * rho * C_P / (KARMAN * GRAVITY * L), -200.0, 200.0)
            self.fields.append({
                "u": u.contiguous(), "v": v.contiguous(), "w": w.contiguous(),
                "t": t.contiguous(), "q": q.contiguous(),
                "blh": blh.contiguous(), "sp": sp.clone(), "ustar": ustar.contiguous(),
                "shf": shf.contiguous(),
            })
        p_col = (sp.view(1, s.ny, s.nx) * torch.exp(-z / 8000.0)).mean(dim=(1, 2)) / 100.0
        self.pressure_level_hpa = p_col.double().cpu().numpy()
        self.height_agl = z.expand(shape3).contiguous()

    @property
    def shape(self) -> tuple[int, int, int]:
        return (self.spec.nz, self.spec.ny, self.spec.nx)

    def metadata(self, h: int) -> MetFieldMetadata:
        return MetFieldMetadata(
            lon=self.lon.copy(), lat=self.lat.copy(), level=self.levels.copy(),
            pressure_level_hpa=self.pressure_level_hpa.copy(),
            time_start=self.times[h], time_end=self.times[h + 1],
            variable_units={"u": "m/s", "v": "m/s", "w": "m/s", "t": "K", "q": "kg/kg",
                            "blh": "m", "sp": "Pa", "ustar": "m/s", "shf": "W m**-2"},
        )

    def window(self, h: int, channel_names: tuple[str, ...] = ("u", "v", "w", "blh", "sp", "t", "ustar", "shf", "q"),
               device: str | torch.device | None = None) -> HourlyMetTensors:
        """The ``[h, h+1]`` bracket as ``HourlyMetTensors`` (2-D fields broadcast over Z)."""
        dev = torch.device(device) if device is not None else self.device
        nz = self.spec.nz

        def stack(snap: dict[str, torch.Tensor]) -> torch.Tensor:
            chans = []
            for name in channel_names:
                f = snap[name]
                if f.dim() == 2:
                    f = f.unsqueeze(0).expand(nz, -1, -1)
                chans.append(f.to(dev))
            return torch.stack(chans, dim=0)

        return HourlyMetTensors(
            hour_start=stack(self.fields[h]),
            hour_end=stack(self.fields[h + 1]),
            metadata=self.metadata(h),
            channel_names=tuple(channel_names),
            height_agl_m=self.height_agl.to(dev),
        )

    def window_index(self, t: datetime) -> int:
        """Index ``h`` of the bracket containing ``t`` (floor to the hour)."""
        t0 = self.times[0]
        return int((t - t0).total_seconds() // 3600)
