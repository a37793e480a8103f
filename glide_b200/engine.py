"""``GPUEngine``'s particle primitives on the CUDA library.

``GPUEngineB200`` has the method names, arguments, shapes and return
conventions of the reference's ``lpdm.gpu_engine.GPUEngine`` for the per-substep
particle updates (src/lpdm/gpu_engine.py:308-507):

* ``update_langevin_velocity`` — exact Ornstein-Uhlenbeck step with an optional
  deterministic drift (``_ou_step_kernel`` :26-42);
* ``apply_vertical_turbulence`` / ``apply_horizontal_turbulence`` —
  displacement by the turbulent velocity, backward by default;
* ``reflect_surface`` — smooth-wall reflection of (z, w);
* ``rk2_advect_backward`` — the midpoint RK2 of a wind callable.

Each is one launch of a kernel built from the same device functions as the fused
step kernel's substep loop, so engine-level checks (OU statistics, Taylor
dispersion, the diffusion limit) test the fused path's arithmetic. Arithmetic is
float32 on a CUDA device; inputs are copied, results returned as new tensors, as
the reference does. Without ``noise=`` the normals come from the library's
counter-based generator, keyed by ``seed`` and a per-call counter.
"""

from __future__ import annotations

import ctypes as C
from typing import Callable

import torch

from glide_b200 import _abi


def _stream(device) -> int:
    return torch.cuda.current_stream(device).cuda_stream


class GPUEngineB200:
    def __init__(self, device="cuda", dtype=torch.float32, seed: int = 0) -> None:
        self.device = torch.device(device)
        if self.device.type != "cuda":
            raise ValueError("GPUEngineB200 runs on a CUDA device")
        if dtype != torch.float32:
            raise ValueError("GPUEngineB200 computes in float32")
        self.dtype = dtype
        self.seed = int(seed)
        self._counter = 0

    # -- helpers -------------------------------------------------------------------
    def _tensor(self, x: torch.Tensor) -> torch.Tensor:
        return x.to(device=self.device, dtype=self.dtype).contiguous()

    def _per_particle(self, x, n: int, name: str):
        """(device pointer or None, scalar, keep-alive tensor) of a scalar or per-particle input."""
        if isinstance(x, torch.Tensor) and x.numel() != 1:
            if x.numel() != n:
                raise ValueError(f"{name} must be a scalar or have {n} elements")
            t = self._tensor(x.reshape(-1))
            return t.data_ptr(), 0.0, t
        return None, float(x), None

    @staticmethod
    def _check_particles(particles: torch.Tensor) -> None:
        if particles.ndim != 2 or particles.shape[1] != 4:
            raise ValueError("particles must have shape (N, 4)")

    def _check_vector(self, v: torch.Tensor, n: int, name: str) -> torch.Tensor:
        if v.ndim != 1 or v.shape[0] != n:
            raise ValueError(f"{name} must have shape (N,)")
        return self._tensor(v)

    # -- primitives ------------------------------------------------------------------
    def rk2_advect_backward(self, particles: torch.Tensor, dt_seconds: float,
                            wind_fn: Callable[[torch.Tensor], torch.Tensor]) -> torch.Tensor:
        """x* = x - dt/2 U(x), x' = x - dt U(x*) on the [x, y, z] columns; weight kept."""
        self._check_particles(particles)
        if dt_seconds <= 0:
            raise ValueError("dt_seconds must be > 0")
        state = self._tensor(particles)
        n = state.shape[0]
        v1 = wind_fn(state[:, :3])
        if tuple(v1.shape) != (n, 3):
            raise ValueError("wind_fn must return velocity tensor shaped (N, 3)")
        v1 = self._tensor(v1)
        x_mid = torch.empty((n, 3), device=self.device, dtype=self.dtype)
        s = _stream(self.device)
        _abi.check(_abi.lib.glide_rk2_stage(n, state.data_ptr(), 4, v1.data_ptr(), 3, 0.5 * float(dt_seconds),
                                            x_mid.data_ptr(), 3, s), "glide_rk2_stage")
        v2 = wind_fn(x_mid)
        if tuple(v2.shape) != (n, 3):
            raise ValueError("wind_fn must return velocity tensor shaped (N, 3)")
        v2 = self._tensor(v2)
        out = state.clone()
        _abi.check(_abi.lib.glide_rk2_stage(n, state.data_ptr(), 4, v2.data_ptr(), 3, float(dt_seconds),
                                            out.data_ptr(), 4, s), "glide_rk2_stage")
        return out

    def update_langevin_velocity(self, w_prime: torch.Tensor, t_lagrangian, sigma_w2, dt_seconds,
                                 noise: torch.Tensor | None = None, drift=0.0) -> torch.Tensor:
        """a w + drift dt + sqrt(max(sigma^2 (1 - a^2), 0)) eta with a = exp(-dt / T_L)."""
        w = self._tensor(w_prime).clone()
        n = w.numel()
        a = _abi.OuArgs()
        a.n, a.w = n, w.data_ptr()
        keep = []
        for field, value, name in (("t_l", t_lagrangian, "t_lagrangian"), ("sigma2", sigma_w2, "sigma_w2"),
                                   ("dt", dt_seconds, "dt_seconds"), ("drift", drift, "drift")):
            ptr, scalar, t = self._per_particle(value, n, name)
            setattr(a, field, ptr)
            setattr(a, field + "_scalar", scalar)
            keep.append(t)
        if noise is not None:
            if tuple(noise.shape) != tuple(w_prime.shape):
                raise ValueError("noise must have same shape as w_prime")
            eta = self._tensor(noise.reshape(-1))
            keep.append(eta)
            a.noise = eta.data_ptr()
        a.seed, a.counter = self.seed, self._counter
        self._counter += 1
        _abi.check(_abi.lib.glide_ou_update(C.byref(a), _stream(self.device)), "glide_ou_update")
        return w.reshape(w_prime.shape)

    def apply_vertical_turbulence(self, particles: torch.Tensor, w_prime: torch.Tensor, dt_seconds, *,
                                  backward: bool = True) -> torch.Tensor:
        self._check_particles(particles)
        out = self._tensor(particles).clone()
        n = out.shape[0]
        wp = self._check_vector(w_prime, n, "w_prime")
        dptr, dsc, dkeep = self._per_particle(dt_seconds, n, "dt_seconds")
        _abi.check(_abi.lib.glide_displace_vertical(n, out.data_ptr() + 8, 4, wp.data_ptr(), dptr, dsc,
                                                    int(backward), _stream(self.device)), "glide_displace_vertical")
        return out

    def apply_horizontal_turbulence(self, particles: torch.Tensor, u_prime: torch.Tensor, v_prime: torch.Tensor,
                                    dt_seconds, *, backward: bool = True) -> torch.Tensor:
        self._check_particles(particles)
        out = self._tensor(particles).clone()
        n = out.shape[0]
        up = self._check_vector(u_prime, n, "u_prime")
        vp = self._check_vector(v_prime, n, "v_prime")
        dptr, dsc, dkeep = self._per_particle(dt_seconds, n, "dt_seconds")
        _abi.check(_abi.lib.glide_displace_horizontal(n, out.data_ptr(), out.data_ptr() + 4, 4, up.data_ptr(),
                                                      vp.data_ptr(), dptr, dsc, int(backward), _stream(self.device)),
                   "glide_displace_horizontal")
        return out

    def reflect_surface(self, particles: torch.Tensor, w_prime: torch.Tensor, *,
                        z_surface: float = 0.0) -> tuple[torch.Tensor, torch.Tensor]:
        self._check_particles(particles)
        out = self._tensor(particles).clone()
        n = out.shape[0]
        if w_prime.ndim != 1 or w_prime.shape[0] != n:
            raise ValueError("w_prime must have shape (N,) matching particles")
        wp = self._tensor(w_prime).clone()
        _abi.check(_abi.lib.glide_reflect_surface(n, out.data_ptr() + 8, 4, wp.data_ptr(), float(z_surface),
                                                  _stream(self.device)), "glide_reflect_surface")
        return out, wp
