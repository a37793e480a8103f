"""The reference's plug-in interface, backed by the CUDA library.

Mirrors ``src/lpdm/turbulence/base.py:26-122`` (``TurbulenceScheme`` and its
name registry), ``src/lpdm/convection/base.py:32-128`` (``ConvectionScheme``)
and ``src/lpdm/footprint_gridder.py:27-197`` (``FootprintGridder``) with the
same method names, argument meaning and error behaviour, so the reference's
per-step runtime (``main.py:1382-1477``) can call them unchanged:

* ``HannaB200Scheme`` (``"hanna_1982_b200"``): ``step()`` is one ``glide_step``
  launch (``n_steps = 1``, the caller's ``active_mask``, no footprint) on the
  reference's ``(N, 4)`` particle tensor in place; ``step_includes_advection``
  is True (RK2 advection is fused, as on the reference's static path).
* ``EmanuelB200Convection`` (``"emanuel_reduced_b200"``): ``maybe_convect()`` is
  one ``glide_convect`` (no host synchronisation).
* ``FootprintGridderB200``: ``accumulate()`` is ``glide_footprint_accumulate``.

Inputs must be CUDA tensors; there is no CPU fallback.
"""

from __future__ import annotations

import ctypes as C
import os
from abc import ABC, abstractmethod
from collections.abc import Callable, Sequence
from typing import ClassVar

import numpy as np
import torch

from glide_b200 import _abi
from glide_b200.window import GridInfo, PackedWindow, stream_handle, window_from_hourly

TurbulenceState = dict
ConvectionState = dict


def _require_cuda(t: torch.Tensor, what: str) -> None:
    if not t.is_cuda:
        raise ValueError(f"{what} must be a CUDA tensor (glide_b200 has no CPU path)")


# ---------------------------------------------------------------------------
# ABCs and registries (turbulence/base.py:26-122, convection/base.py:32-128)
# ---------------------------------------------------------------------------


class TurbulenceScheme(ABC):
    name: ClassVar[str]

    @abstractmethod
    def required_met_keys(self) -> tuple[str, ...]:
        """Met keys read from ``HourlyMetTensors`` beyond u, v, w, blh, sp."""

    @abstractmethod
    def initialize_state(self, n_particles: int, *, device: torch.device, dtype: torch.dtype) -> TurbulenceState:
        """Per-particle state tensors."""

    @abstractmethod
    def step(self, particles: torch.Tensor, state: TurbulenceState, met_window, t_alpha: float, dt_seconds: float,
             active_mask: torch.Tensor, engine) -> tuple[torch.Tensor, TurbulenceState]:
        """One turbulence step; inactive particles are left unmodified."""

    def step_includes_advection(self, engine) -> bool:
        del engine
        return False


class ConvectionScheme(ABC):
    name: ClassVar[str]

    @abstractmethod
    def required_met_keys(self) -> tuple[str, ...]:
        """Met keys read from ``HourlyMetTensors``."""

    def initialize_state(self, n_particles: int, *, device: torch.device, dtype: torch.dtype) -> ConvectionState:
        del n_particles, device, dtype
        return {}

    @abstractmethod
    def maybe_convect(self, particles: torch.Tensor, state: ConvectionState, met_window, *, t_alpha: float,
                      dt_seconds: float, active_mask: torch.Tensor, engine, generator=None):
        """Redistribute particles vertically once per met window."""


_TURB: dict[str, type[TurbulenceScheme]] = {}
_CONV: dict[str, type[ConvectionScheme]] = {}


def _register(reg: dict, cls):
    if not getattr(cls, "name", ""):
        raise TypeError(f"{cls.__name__} must define a non-empty class-level `name` attribute")
    existing = reg.get(cls.name)
    if existing is not None and existing is not cls:
        raise ValueError(f"scheme name {cls.name!r} already registered to {existing.__name__}")
    reg[cls.name] = cls
    return cls


def register_scheme(cls: type[TurbulenceScheme]) -> type[TurbulenceScheme]:
    return _register(_TURB, cls)


def register_convection_scheme(cls: type[ConvectionScheme]) -> type[ConvectionScheme]:
    return _register(_CONV, cls)


def get_scheme(name: str, **kwargs) -> TurbulenceScheme:
    if name not in _TURB:
        available = ", ".join(sorted(_TURB)) or "<none>"
        raise KeyError(f"Unknown turbulence scheme {name!r}. Registered schemes: {available}")
    return _TURB[name](**kwargs)


def get_convection_scheme(name: str, **kwargs) -> ConvectionScheme:
    if name not in _CONV:
        available = ", ".join(sorted(_CONV)) or "<none>"
        raise KeyError(f"Unknown convection scheme {name!r}. Registered: {available}")
    return _CONV[name](**kwargs)


def register_with_reference(turbulence_base, convection_base) -> None:
    """Registers ``hanna_1982_b200`` and ``emanuel_reduced_b200`` in the reference's own
    scheme registries, given its ``lpdm.turbulence.base`` and ``lpdm.convection.base``
    modules (``register_scheme``, turbulence/base.py:96-107, convection/base.py:102-113),
    so its ``get_scheme`` / ``get_convection_scheme`` build them by name and its runtime
    (``lpdm.main._run``) runs them. The registries check only the ``name`` attribute,
    which these classes share with their registrations here."""
    turbulence_base.register_scheme(HannaB200Scheme)
    convection_base.register_scheme(EmanuelB200Convection)


def list_schemes() -> tuple[str, ...]:
    return tuple(sorted(_TURB))


def list_convection_schemes() -> tuple[str, ...]:
    return tuple(sorted(_CONV))


class _WindowCache:
    """Per-window device staging shared by the schemes: the grid (with its level
    lookup table) and the raw device fields of the current window."""

    def __init__(self) -> None:
        self.grid: GridInfo | None = None
        self.grid_key = None
        self.key = None
        self.fields = None

    def get(self, met_window, device):
        md = met_window.metadata
        gkey = (tuple(np.asarray(md.level).tolist()), float(md.lon[0]), float(md.lon[-1]), len(md.lon),
                float(md.lat[0]), float(md.lat[-1]), len(md.lat), tuple(np.asarray(md.pressure_level_hpa).tolist()))
        if self.grid is None or self.grid_key != gkey:
            self.grid = GridInfo(np.asarray(md.lon), np.asarray(md.lat), np.asarray(md.level),
                                 np.asarray(md.pressure_level_hpa)).to_device(device)
            self.grid_key = gkey
            self.key = None
        if self.key != md.time_start:
            self.fields = window_from_hourly(met_window, self.grid, device)
            self.key = md.time_start
        return self.grid, self.fields


# ---------------------------------------------------------------------------
# Hanna (hanna.py:434-1978) on the CUDA path
# ---------------------------------------------------------------------------


@register_scheme
class HannaB200Scheme(TurbulenceScheme):
    """``HannaScheme`` (``hanna_1982``) with the whole static step core in one kernel.

    Constructor arguments are ``HannaScheme``'s (hanna.py:440-520) plus
    ``met_dtype`` (packed met storage: ``"f32"``, ``"bf16"``, ``"f16"``), ``seed``
    (Philox-4x32-10 key of the turbulence noise) and ``noise_provider``: a callable
    ``step_number -> (substep [max_substeps, 3, N], meander [2, N])`` of CUDA
    float32 normals that replaces the generated noise (reproducible comparisons).
    """

    name: ClassVar[str] = "hanna_1982_b200"

    def __init__(self, *, meander_enabled: bool = False, meander_coefficient: float = 0.16,
                 meander_stencil_radius: int = 1, meander_timescale_seconds: float = 1800.0,
                 substep_c: float = 0.5, max_substeps: int = 50, z_ubl_m: float = 2.0,
                 static_substeps: bool | None = None, flexpart_tl_floors: bool = True,
                 surface_layer_override: bool = False, met_dtype: str = "f32", seed: int = 0,
                 noise_provider: Callable | None = None) -> None:
        if meander_coefficient <= 0:
            raise ValueError("meander_coefficient must be > 0")
        if meander_stencil_radius < 1:
            raise ValueError("meander_stencil_radius must be >= 1")
        if meander_timescale_seconds <= 0:
            raise ValueError("meander_timescale_seconds must be > 0")
        if substep_c <= 0:
            raise ValueError("substep_c must be > 0")
        if max_substeps < 1:
            raise ValueError("max_substeps must be >= 1")
        if z_ubl_m < 0:
            raise ValueError("z_ubl_m must be >= 0")
        del static_substeps  # the kernel always runs the static (full-set, mask-gated) step
        self.meander_enabled = bool(meander_enabled)
        self.meander_coefficient = float(meander_coefficient)
        self.meander_stencil_radius = int(meander_stencil_radius)
        self.meander_timescale_seconds = float(meander_timescale_seconds)
        self.substep_c = float(substep_c)
        self.max_substeps = int(max_substeps)
        self.z_ubl_m = float(z_ubl_m)
        self.flexpart_tl_floors = bool(flexpart_tl_floors)
        self.surface_layer_override = bool(surface_layer_override)
        self.met_dtype = met_dtype
        self.seed = int(seed)
        self.noise_provider = noise_provider
        self.step_count = 0
        self._cache = _WindowCache()
        self._packed: PackedWindow | None = None
        self._status = None

    def required_met_keys(self) -> tuple[str, ...]:
        return ("t", "ustar", "shf")

    def initialize_state(self, n_particles: int, *, device: torch.device, dtype: torch.dtype) -> TurbulenceState:
        if dtype != torch.float32:
            raise ValueError("HannaB200Scheme integrates in float32")
        names = ["u_prime", "v_prime", "w_prime"] + (["u_meander", "v_meander"] if self.meander_enabled else [])
        return {k: torch.zeros(n_particles, device=device, dtype=dtype) for k in names}

    def step_includes_advection(self, engine) -> bool:
        del engine
        return True

    def _packed_window(self, met_window, device) -> PackedWindow:
        grid, fields = self._cache.get(met_window, device)
        if self._packed is None or self._packed.grid is not grid:
            self._packed = PackedWindow(grid, self.met_dtype, device)
        if self._packed.key != fields.time_start:
            self._packed.pack(fields, meander_coefficient=self.meander_coefficient,
                              meander_radius=self.meander_stencil_radius, build_meander=self.meander_enabled)
        return self._packed

    @property
    def device_status(self) -> int:
        """The device status word (``GLIDE_STATUS_*`` bits); reading it synchronises."""
        return 0 if self._status is None else int(self._status.item())

    def step(self, particles, state, met_window, t_alpha, dt_seconds, active_mask, engine=None):
        _require_cuda(particles, "particles")
        if particles.dim() != 2 or particles.shape[1] != 4 or particles.dtype != torch.float32:
            raise ValueError("particles must be a float32 (N, 4) tensor")
        if not particles.is_contiguous():
            raise ValueError("particles must be contiguous")
        n = particles.shape[0]
        dev = particles.device
        if active_mask.shape != (n,):
            raise ValueError("active_mask must have shape (N,)")
        mask = active_mask.to(device=dev, dtype=torch.uint8).contiguous()
        for k in ("u_prime", "v_prime", "w_prime") + (("u_meander", "v_meander") if self.meander_enabled else ()):
            t = state[k]
            if t.shape != (n,) or t.dtype != torch.float32 or not t.is_cuda or not t.is_contiguous():
                raise ValueError(f"state[{k!r}] must be a contiguous float32 CUDA tensor of shape (N,)")
        packed = self._packed_window(met_window, dev)
        if self._status is None:
            self._status = torch.zeros(1, dtype=torch.int32, device=dev)
        a = _abi.StepArgs()
        a.n = n
        base = particles.data_ptr()
        a.lon, a.lat, a.z, a.weight, a.pos_stride = base, base + 4, base + 8, base + 12, 4
        a.u_prime, a.v_prime, a.w_prime = (state["u_prime"].data_ptr(), state["v_prime"].data_ptr(),
                                           state["w_prime"].data_ptr())
        if self.meander_enabled:
            a.u_meander, a.v_meander = state["u_meander"].data_ptr(), state["v_meander"].data_ptr()
        a.active_mask = mask.data_ptr()
        a.wind_packed, a.surf_packed, a.support_packed = (packed.wind.data_ptr(), packed.surf.data_ptr(),
                                                          packed.support.data_ptr())
        a.met_dtype = packed.code
        a.grid = packed.grid.c_grid()
        a.substep_c, a.max_substeps, a.z_ubl_m = self.substep_c, self.max_substeps, self.z_ubl_m
        a.flexpart_tl_floors, a.surface_layer_override = int(self.flexpart_tl_floors), int(self.surface_layer_override)
        a.meander_enabled, a.meander_timescale_s = int(self.meander_enabled), self.meander_timescale_seconds
        a.sched = None
        a.sched0 = _abi.StepSched(0.0, float(dt_seconds), float(t_alpha), self.step_count)
        a.n_steps, a.phys_begin, a.post_begin = 1, 0, 1
        keep = None
        if self.noise_provider is not None:
            sub, mea = self.noise_provider(self.step_count)
            if tuple(sub.shape) != (self.max_substeps, 3, n) or not sub.is_contiguous() or sub.dtype != torch.float32:
                raise ValueError(f"noise_provider substep noise must be contiguous float32 ({self.max_substeps}, 3, {n})")
            if self.meander_enabled and (mea is None or tuple(mea.shape) != (2, n) or not mea.is_contiguous()):
                raise ValueError(f"noise_provider meander noise must be contiguous float32 (2, {n})")
            a.noise_substep = sub.data_ptr()
            a.noise_meander = None if mea is None else mea.data_ptr()
            keep = (sub, mea)
        a.seed = self.seed
        a.status = self._status.data_ptr()
        _abi.check(_abi.lib.glide_step(C.byref(a), stream_handle()), "glide_step")
        del keep
        self.step_count += 1
        return particles, state


# ---------------------------------------------------------------------------
# Emanuel convection (emanuel.py:510-805) on the CUDA path
# ---------------------------------------------------------------------------


@register_convection_scheme
class EmanuelB200Convection(ConvectionScheme):
    """``EmanuelReducedConvection`` (``emanuel_reduced``), column build in FP64 on the
    device. ``uniform_provider(call_number) -> [2, N]`` CUDA float32 uniforms replaces
    the generated draws (reproducible comparisons)."""

    name: ClassVar[str] = "emanuel_reduced_b200"

    def __init__(self, *, closure_c: float = 0.03, trigger_dtv_k: float = 0.9, min_cape_j_kg: float = 50.0,
                 min_cloud_depth_m: float = 500.0, seed: int = 0, uniform_provider: Callable | None = None) -> None:
        if closure_c <= 0:
            raise ValueError("closure_c must be > 0")
        if trigger_dtv_k < 0:
            raise ValueError("trigger_dtv_k must be >= 0")
        if min_cape_j_kg < 0:
            raise ValueError("min_cape_j_kg must be >= 0")
        if min_cloud_depth_m < 0:
            raise ValueError("min_cloud_depth_m must be >= 0")
        self.closure_c = float(closure_c)
        self.trigger_dtv_k = float(trigger_dtv_k)
        self.min_cape_j_kg = float(min_cape_j_kg)
        self.min_cloud_depth_m = float(min_cloud_depth_m)
        self.seed = int(seed)
        self.uniform_provider = uniform_provider
        self.calls = 0
        self._cache = _WindowCache()
        self._scratch = None
        self.n_moved = None

    def required_met_keys(self) -> tuple[str, ...]:
        return ("t", "q")

    def maybe_convect(self, particles, state, met_window, *, t_alpha, dt_seconds, active_mask, engine=None,
                      generator=None):
        del dt_seconds, generator
        _require_cuda(particles, "particles")
        if met_window.height_agl_m is None:
            raise ValueError("EmanuelB200Convection requires HourlyMetTensors.height_agl_m")
        n = particles.shape[0]
        dev = particles.device
        grid, fields = self._cache.get(met_window, dev)
        nz, ny, nx = grid.shape
        if self._scratch is None or self._scratch.device != dev:
            nb = C.c_size_t()
            _abi.check(_abi.lib.glide_convect_scratch_bytes(nz, C.byref(nb)), "glide_convect_scratch_bytes")
            self._scratch = torch.zeros(nb.value // 8, dtype=torch.float64, device=dev)
        mask = active_mask.to(device=dev, dtype=torch.uint8).contiguous()
        self.n_moved = torch.zeros(1, dtype=torch.int32, device=dev)
        a = _abi.ConvectArgs()
        a.n = n
        a.z, a.z_stride = particles.data_ptr() + 8, 4
        a.active_mask = mask.data_ptr()
        a.sched = _abi.StepSched(0.0, 0.0, float(t_alpha), self.calls)
        a.nz, a.ny, a.nx = nz, ny, nx
        for k, snap in enumerate((fields.start, fields.end)):
            a.t[k], a.q[k] = snap["t"].data_ptr(), snap["q"].data_ptr()
        a.height3d = None if fields.height3d is None else fields.height3d.data_ptr()
        a.height_level = grid.height_level_dev.data_ptr()
        a.pressure_hpa = grid.p_hpa_dev.data_ptr()
        a.alpha = float(t_alpha)
        a.closure_c, a.trigger_dtv_k = self.closure_c, self.trigger_dtv_k
        a.min_cape_j_kg, a.min_cloud_depth_m = self.min_cape_j_kg, self.min_cloud_depth_m
        keep = None
        if self.uniform_provider is not None:
            u = self.uniform_provider(self.calls)
            if tuple(u.shape) != (2, n) or u.dtype != torch.float32 or not u.is_contiguous():
                raise ValueError(f"uniform_provider must return contiguous float32 (2, {n})")
            a.uniforms = u.data_ptr()
            keep = u
        a.seed = self.seed
        a.scratch = self._scratch.data_ptr()
        a.n_moved = self.n_moved.data_ptr()
        _abi.check(_abi.lib.glide_convect(C.byref(a), stream_handle()), "glide_convect")
        del keep
        self.calls += 1
        return particles, state


# ---------------------------------------------------------------------------
# FootprintGridder (footprint_gridder.py:27-197) on the CUDA path
# ---------------------------------------------------------------------------


class FootprintGridderB200:
    """5-D ``(release, time_ago, z, lat, lon)`` residence-time footprint on the device."""

    MAX_FOOTPRINT_GIB: float = 32.0

    def __init__(self, lon_bounds: tuple[float, float], lat_bounds: tuple[float, float], z_edges_m: Sequence[float],
                 n_time_bins: int, n_y: int, n_x: int, *, n_releases: int = 1, device="cuda",
                 dtype: torch.dtype = torch.float32) -> None:
        z_edges = np.asarray(list(z_edges_m), dtype=float)
        if z_edges.ndim != 1 or z_edges.size < 2:
            raise ValueError("z_edges_m must be a 1D sequence with at least 2 values")
        if not np.all(np.diff(z_edges) > 0):
            raise ValueError("z_edges_m must be strictly ascending")
        n_z = int(z_edges.size - 1)
        if min(n_time_bins, n_y, n_x, n_releases) <= 0 or n_z <= 0:
            raise ValueError("All footprint dimensions must be > 0")
        if dtype not in (torch.float32, torch.float64):
            raise ValueError("FootprintGridderB200 accumulates in float32 or float64")
        self.device = torch.device(device)
        self.dtype = dtype
        n_elements = int(n_releases) * int(n_time_bins) * n_z * int(n_y) * int(n_x)
        env_cap = os.environ.get("LPDM_FOOTPRINT_MAX_GIB")
        cap_gib = float(env_cap) if env_cap else self.MAX_FOOTPRINT_GIB
        elem = torch.empty((), dtype=dtype).element_size()
        if n_elements * elem > int(cap_gib * 1024**3):
            raise MemoryError(f"Footprint tensor would require {n_elements * elem / 1024**3:.2f} GiB; cap is "
                              f"{cap_gib:.2f} GiB (raise it via LPDM_FOOTPRINT_MAX_GIB)")
        self.tensor = torch.zeros((n_releases, n_time_bins, n_z, n_y, n_x), device=self.device, dtype=dtype)
        self.lon_min, self.lon_max = lon_bounds
        self.lat_min, self.lat_max = lat_bounds
        self.z_edges = torch.tensor(z_edges, dtype=torch.float32, device=self.device)
        self.z_min, self.z_max = float(z_edges[0]), float(z_edges[-1])
        self.n_releases, self.n_t, self.n_z, self.n_y, self.n_x = int(n_releases), n_time_bins, n_z, n_y, n_x

    def accumulate(self, particles: torch.Tensor, active_mask: torch.Tensor, weights: torch.Tensor,
                   t_idx: torch.Tensor, release_idx: torch.Tensor, dt_seconds: float) -> None:
        """Adds ``weights * dt_seconds`` of every active in-range particle to its cell
        (formed and summed in FP64 when the gridder is float64)."""
        _require_cuda(particles, "particles")
        n = particles.shape[0]
        if particles.dim() != 2 or particles.shape[1] < 3 or particles.dtype != torch.float32:
            raise ValueError("particles must be a float32 (N, >=3) tensor")
        if particles.stride(1) != 1:
            raise ValueError("particles columns must be adjacent (stride 1)")
        if weights.dim() != 1 or weights.dtype != torch.float32:
            raise ValueError("weights must be a float32 (N,) tensor")
        g = _abi.FootprintGrid(self.lon_min, self.lon_max, self.lat_min, self.lat_max, self.n_releases, self.n_t,
                               self.n_z, self.n_y, self.n_x, self.z_edges.data_ptr(), 0,
                               1 if self.dtype == torch.float64 else 0)
        act = active_mask.to(dtype=torch.uint8).contiguous()
        t32 = t_idx.to(dtype=torch.int32).contiguous()
        r32 = release_idx.to(dtype=torch.int32).contiguous()
        base = particles.data_ptr()
        ps = particles.stride(0)
        _abi.check(_abi.lib.glide_footprint_accumulate(n, base, base + 4, base + 8, ps, act.data_ptr(),
                                                       weights.data_ptr(), weights.stride(0), t32.data_ptr(),
                                                       r32.data_ptr(), float(dt_seconds), C.byref(g),
                                                       self.tensor.data_ptr(), stream_handle()),
                   "glide_footprint_accumulate")
