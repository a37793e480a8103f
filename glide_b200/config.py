"""Run configuration of a batch: the reference's scheme knobs, output grid and met
domain (``src/lpdm/config.py``), as plain dataclasses. No CUDA library is loaded by
this module, so configurations can be built (and the CPU baselines run) without it.
"""

from __future__ import annotations

from dataclasses import dataclass

import torch


@dataclass(frozen=True)
class HannaConfig:
    """``HannaScheme`` knobs (src/lpdm/turbulence/hanna.py:440-520)."""

    meander_enabled: bool = False
    meander_coefficient: float = 0.16
    meander_stencil_radius: int = 1
    meander_timescale_seconds: float = 1800.0
    substep_c: float = 0.5
    max_substeps: int = 50
    z_ubl_m: float = 2.0
    flexpart_tl_floors: bool = True
    surface_layer_override: bool = False


@dataclass(frozen=True)
class EmanuelConfig:
    """``EmanuelReducedConvection`` knobs (src/lpdm/convection/emanuel.py:531-565)."""

    closure_c: float = 0.03
    trigger_dtv_k: float = 0.9
    min_cape_j_kg: float = 50.0
    min_cloud_depth_m: float = 500.0


@dataclass(frozen=True)
class FootprintSpec:
    """``OutputGridConfig`` and the gridder's release count (src/lpdm/config.py:360-382)."""

    lon_bounds: tuple[float, float]
    lat_bounds: tuple[float, float]
    n_x: int
    n_y: int
    z_edges: tuple[float, ...]
    n_time_bins: int
    n_releases: int = 1
    ring: int = 0  # > 0: keep only `ring` live time-ago slices per release, flushed as bins complete
    # "f32": float32 values (FootprintGridder's default dtype); "f64": float64 values, each
    # weight * dt formed and summed in FP64 (FootprintGridder(dtype=torch.float64))
    value_dtype: str = "f32"

    def __post_init__(self) -> None:
        if self.value_dtype not in ("f32", "f64"):
            raise ValueError(f"value_dtype must be 'f32' or 'f64', got {self.value_dtype!r}")

    @property
    def torch_dtype(self) -> torch.dtype:
        return torch.float64 if self.value_dtype == "f64" else torch.float32

    @property
    def shape(self) -> tuple[int, int, int, int, int]:
        return (self.n_releases, self.n_time_bins, len(self.z_edges) - 1, self.n_y, self.n_x)

    @property
    def device_shape(self) -> tuple[int, int, int, int, int]:
        t = self.ring if self.ring > 0 else self.n_time_bins
        return (self.n_releases, t, len(self.z_edges) - 1, self.n_y, self.n_x)


@dataclass(frozen=True)
class DomainSpec:
    """``MetDomainConfig`` bounds of the escape kill (src/lpdm/main.py:690-711)."""

    lon_bounds: tuple[float, float]
    lat_bounds: tuple[float, float]
    alt_max_m: float
