"""Analytic dispersion and diffusion-limit checks of the engine primitives.

The reference pins its stochastic transport against closed forms at the engine
level (tests/test_dispersion_analytic.py, tests/test_diffusion_pde.py), with a
prescribed constant (sigma_w, T_L), because the assembled Hanna scheme has no
homogeneous regime. The same checks run here through ``GPUEngineB200``, whose
kernels share their arithmetic with the fused step kernel's substep loop:

* the OU velocity is stationary at sigma_w^2 with autocorrelation exp(-tau / T_L);
* midpoint RK2 closes a solid-body rotation to second order in dt;
* the vertical spread follows Taylor (1921) from the ballistic to the diffusive
  limit, and the forward-Euler position bias grows with dt / T_L as documented;
* with the Thomson well-mixed drift and reflections, the binned particle density
  follows a conservative Crank-Nicolson solution of dc/dt = d/dz(K dc/dz), and is
  far from solutions whose near-surface K is halved or quartered.

Arithmetic is float32 on the device (the reference runs these in float64); the
tolerances are the reference's.
"""

from __future__ import annotations

import math

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _engine(device, seed):
    from glide_b200.engine import GPUEngineB200

    return GPUEngineB200(device=device, seed=seed)


def _randn(n, device, seed):
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    return torch.randn(n, device=device, dtype=torch.float32, generator=g)


def _taylor_var(sigma_w2: float, t_l: float, t: float) -> float:
    return 2.0 * sigma_w2 * t_l * (t - t_l * (1.0 - math.exp(-t / t_l)))


def test_ou_stationary_variance_and_autocorrelation(cuda_device):
    eng = _engine(cuda_device, 4111)
    n, sigma_w2, t_l, dt = 100_000, 0.7, 100.0, 5.0
    w = _randn(n, cuda_device, 1) * math.sqrt(sigma_w2)
    for _ in range(int(2 * t_l / dt)):  # burn-in
        w = eng.update_langevin_velocity(w, t_lagrangian=t_l, sigma_w2=sigma_w2, dt_seconds=dt)
    frames = []
    for _ in range(int(3 * t_l / dt) + 1):
        frames.append(w)
        w = eng.update_langevin_velocity(w, t_lagrangian=t_l, sigma_w2=sigma_w2, dt_seconds=dt)
    f = torch.stack(frames).double()
    var = f.var(unbiased=True).item()
    assert 0.97 * sigma_w2 <= var <= 1.03 * sigma_w2, var
    c = f - f.mean()
    for tau in (0.5, 1.0, 2.0):
        lag = int(round(tau * t_l / dt))
        r = (c[:-lag] * c[lag:]).mean().item() / var
        assert abs(r - math.exp(-tau)) < 0.02, (tau, r)


def _rotate(eng, start, omega, dt, period):
    def wind(xyz):
        out = torch.zeros_like(xyz)
        out[:, 0] = -omega * xyz[:, 1]
        out[:, 1] = omega * xyz[:, 0]
        return out

    p = start.clone()
    for _ in range(int(round(period / dt))):
        p = eng.rk2_advect_backward(p, dt_seconds=dt, wind_fn=wind)
    return p


def test_solid_body_rotation_closes_to_second_order(cuda_device):
    eng = _engine(cuda_device, 0)
    omega, period = 2.0 * math.pi / 3600.0, 3600.0
    start = torch.tensor([[100_000.0, 0.0, 500.0, 0.25], [0.0, 50_000.0, 500.0, 0.25],
                          [-70_000.0, 40_000.0, 500.0, 0.25], [30_000.0, -80_000.0, 500.0, 0.25]],
                         device=cuda_device)
    dts = [60.0, 30.0, 15.0]
    errs = []
    for dt in dts:
        fin = _rotate(eng, start, omega, dt, period)
        errs.append(torch.linalg.norm((fin[:, :2] - start[:, :2]).double(), dim=1).max().item())
    for a, b in zip(errs[:-1], errs[1:]):
        assert a / max(b, 1e-12) > 3.5, errs
    r_max = torch.linalg.norm(start[:, :2], dim=1).max().item()
    assert errs[-1] < 1e-3 * r_max, errs
    fin = _rotate(eng, start, omega, dts[-1], period)
    assert torch.equal(fin[:, 2], start[:, 2]) and torch.equal(fin[:, 3], start[:, 3])


def test_taylor_dispersion_ballistic_to_diffusive(cuda_device):
    eng = _engine(cuda_device, 2201)
    n, sigma_w2, t_l, dt = 100_000, 1.0, 100.0, 1.0
    p = torch.zeros((n, 4), device=cuda_device)
    p[:, 3] = 1.0 / n
    w = _randn(n, cuda_device, 2) * math.sqrt(sigma_w2)
    checkpoints = [0.1, 0.3, 1.0, 3.0, 10.0, 30.0]
    sz = {}
    step = 0
    for c in checkpoints:
        while step < int(round(c * t_l / dt)):
            w = eng.update_langevin_velocity(w, t_lagrangian=t_l, sigma_w2=sigma_w2, dt_seconds=dt)
            p = eng.apply_vertical_turbulence(p, w, dt_seconds=dt, backward=False)
            step += 1
        sz[c] = p[:, 2].double().std(unbiased=True).item()
    for c in checkpoints:
        want = math.sqrt(_taylor_var(sigma_w2, t_l, c * t_l))
        assert abs(sz[c] - want) / want < 0.05, (c, sz[c], want)
    assert abs(sz[0.1] - 0.1 * t_l) / (0.1 * t_l) < 0.05  # ballistic: sigma_w t
    k, t_dif = sigma_w2 * t_l, 30.0 * t_l
    assert abs(sz[30.0] ** 2 - 2.0 * k * t_dif) / (2.0 * k * t_dif) < 0.08  # diffusive: 2 K t
    assert abs(p[:, 3].double().sum().item() - 1.0) < 1e-5


def test_taylor_position_bias_grows_with_dt(cuda_device):
    t_l, sigma_w2 = 100.0, 1.0
    total = 5.0 * t_l
    want = math.sqrt(_taylor_var(sigma_w2, t_l, total))

    def spread(dt):
        eng = _engine(cuda_device, 71)
        n = 100_000
        p = torch.zeros((n, 4), device=cuda_device)
        w = _randn(n, cuda_device, 3) * math.sqrt(sigma_w2)
        for _ in range(int(round(total / dt))):
            w = eng.update_langevin_velocity(w, t_lagrangian=t_l, sigma_w2=sigma_w2, dt_seconds=dt)
            p = eng.apply_vertical_turbulence(p, w, dt_seconds=dt, backward=False)
        return p[:, 2].double().std(unbiased=True).item()

    assert abs(spread(1.0) - want) / want < 0.02
    assert abs(spread(20.0) - want) / want < 0.15


def test_horizontal_and_backward_displacement_and_reflection(cuda_device):
    """The displacement and reflection primitives against their closed forms."""
    eng = _engine(cuda_device, 5)
    p = torch.tensor([[10.0, 60.0, 5.0, 1.0], [-3.0, 0.0, 50.0, 1.0], [0.0, 89.9, 1.0, 1.0]], device=cuda_device)
    u = torch.tensor([10.0, -5.0, 1.0], device=cuda_device)
    v = torch.tensor([2.0, 3.0, 0.0], device=cuda_device)
    w = torch.tensor([1.0, -2.0, 4.0], device=cuda_device)
    q = eng.apply_horizontal_turbulence(p, u, v, 30.0)  # backward
    m_lon = 111320.0 * np.maximum(np.abs(np.cos(np.deg2rad(p[:, 1].cpu().numpy().astype(np.float64)))), 0.05)
    np.testing.assert_allclose(q[:, 0].cpu().numpy(), p[:, 0].cpu().numpy() - 30.0 * u.cpu().numpy() / m_lon,
                               rtol=1e-6, atol=1e-6)
    np.testing.assert_allclose(q[:, 1].cpu().numpy(), p[:, 1].cpu().numpy() - 30.0 * v.cpu().numpy() / 110540.0,
                               rtol=1e-6, atol=1e-6)
    zq = eng.apply_vertical_turbulence(p, w, 10.0)  # backward: z - w dt
    np.testing.assert_allclose(zq[:, 2].cpu().numpy(), [-5.0, 70.0, -39.0])
    r, wr = eng.reflect_surface(zq, w)
    np.testing.assert_allclose(r[:, 2].cpu().numpy(), [5.0, 70.0, 39.0])
    np.testing.assert_allclose(wr.cpu().numpy(), [-1.0, -2.0, -4.0])
    # injected noise gives the exact OU formula
    eta = torch.tensor([0.5, -1.0, 2.0], device=cuda_device)
    out = eng.update_langevin_velocity(w, t_lagrangian=50.0, sigma_w2=0.8, dt_seconds=10.0, noise=eta, drift=0.1)
    a = math.exp(-10.0 / 50.0)
    want = a * w.cpu().numpy() + 0.1 * 10.0 + math.sqrt(0.8 * (1 - a * a)) * eta.cpu().numpy()
    np.testing.assert_allclose(out.cpu().numpy(), want, rtol=2e-6, atol=1e-6)


# --------------------------------------------------------------------------- diffusion limit

K0, A_KZ, Z_CAP, H_TOP, T_L = 0.02, 0.12, 200.0, 400.0, 10.0
DT, N_PART, Z0_LO, Z0_HI = 1.0, 100_000, 5.0, 15.0
CHECKPOINTS, BIN_W, PDE_DZ = (300.0, 900.0, 1800.0), 20.0, 2.0


def _cn_stepper(k_faces: np.ndarray, n_nodes: int):
    """Conservative flux-form Crank-Nicolson step with zero-flux boundaries."""
    from scipy.linalg import solve_banded

    main = np.zeros(n_nodes)
    main[0] = k_faces[0]
    main[1:-1] = k_faces[:-1] + k_faces[1:]
    main[-1] = k_faces[-1]
    lam = DT / PDE_DZ ** 2
    ab = np.zeros((3, n_nodes))
    ab[0, 1:] = -0.5 * lam * k_faces
    ab[1, :] = 1.0 + 0.5 * lam * main
    ab[2, :-1] = -0.5 * lam * k_faces

    def step(c):
        rhs = c - 0.5 * lam * (main * c - np.r_[0.0, k_faces * c[:-1]] - np.r_[k_faces * c[1:], 0.0])
        return solve_banded((1, 1), ab, rhs)

    return step


@pytest.fixture(scope="module")
def diffusion(cuda_device):
    eng = _engine(cuda_device, 3301)

    def sigma2(z):
        return (K0 + A_KZ * torch.clamp(z, max=Z_CAP)) / T_L

    g = torch.Generator(device=cuda_device)
    g.manual_seed(4)
    z = torch.rand(N_PART, device=cuda_device, generator=g) * (Z0_HI - Z0_LO) + Z0_LO
    w = torch.randn(N_PART, device=cuda_device, generator=g) * torch.sqrt(sigma2(z))
    p = torch.zeros((N_PART, 4), device=cuda_device)
    p[:, 2] = z
    p[:, 3] = 1.0 / N_PART

    z_nodes = np.arange(0.0, H_TOP + PDE_DZ / 2, PDE_DZ)
    z_faces = (z_nodes[:-1] + z_nodes[1:]) / 2
    steppers = {}
    for name, f in (("true", 1.0), ("half", 0.5), ("quarter", 0.25)):
        k = K0 + A_KZ * np.minimum(z_faces, Z_CAP)
        k[z_faces < 50.0] *= f
        steppers[name] = _cn_stepper(k, len(z_nodes))
    c0 = np.where((z_nodes >= Z0_LO) & (z_nodes <= Z0_HI), 1.0, 0.0)
    pde = {name: c0 / c0.sum() for name in steppers}
    edges = np.arange(0.0, H_TOP + BIN_W / 2, BIN_W)
    node_bin = np.minimum((z_nodes // BIN_W).astype(int), len(edges) - 2)

    def binned(c):
        h = np.bincount(node_bin, weights=c, minlength=len(edges) - 1)
        return h / h.sum()

    out = {}
    t = 0.0
    dsig2 = A_KZ / T_L
    for t_check in CHECKPOINTS:
        for _ in range(int(round((t_check - t) / DT))):
            zc = p[:, 2]
            s2 = sigma2(zc)
            drift = 0.5 * (1.0 + w * w / s2) * torch.where(zc < Z_CAP, dsig2, 0.0)  # Thomson well-mixed drift
            w = eng.update_langevin_velocity(w, t_lagrangian=T_L, sigma_w2=s2, dt_seconds=DT, drift=drift)
            p = eng.apply_vertical_turbulence(p, w, dt_seconds=DT, backward=False)
            p, w = eng.reflect_surface(p, w, z_surface=0.0)
            above = p[:, 2] > H_TOP  # reflecting lid
            p[:, 2] = torch.where(above, 2.0 * H_TOP - p[:, 2], p[:, 2])
            w = torch.where(above, -w, w)
            for name in pde:
                pde[name] = steppers[name](pde[name])
        t = t_check
        hist, _ = np.histogram(p[:, 2].cpu().numpy(), bins=edges)
        out[t_check] = dict(particles=hist / hist.sum(), **{k: binned(c) for k, c in pde.items()})
    assert abs(p[:, 3].double().sum().item() - 1.0) < 1e-5
    return out


def test_langevin_diffusion_limit_matches_pde(diffusion):
    for t_check in CHECKPOINTS:
        got, want = diffusion[t_check]["particles"], diffusion[t_check]["true"]
        assert np.abs(got - want).sum() < 0.08, t_check
        ns_got, ns_want = got[:3].sum(), want[:3].sum()  # 0-60 m
        assert abs(ns_got - ns_want) / ns_want < 0.12, (t_check, ns_got, ns_want)


def test_diffusion_limit_rejects_wrong_near_surface_k(diffusion):
    for t_check, min_half, min_quarter in ((300.0, 0.25, 0.45), (900.0, 0.20, 0.45), (1800.0, 0.12, 0.30)):
        got = diffusion[t_check]["particles"]
        assert np.abs(got - diffusion[t_check]["half"]).sum() > min_half, t_check
        assert np.abs(got - diffusion[t_check]["quarter"]).sum() > min_quarter, t_check


def test_latitude_displacement_division_is_exact_for_every_float(cuda_device):
    """The latitude displacement divides by 110540 m per degree through a reciprocal
    and one fused correction step; over all 2^32 float32 inputs its quotient equals
    the IEEE division (torch's elementwise tensor division) bit for bit (NaN as NaN)."""
    eng = _engine(cuda_device, 0)
    chunk = 1 << 27
    c = None
    for start in range(0, 1 << 32, chunk):
        bits = torch.arange(start, start + chunk, dtype=torch.int64, device=cuda_device)
        x = bits.to(torch.int32).view(torch.float32)  # every bit pattern once
        p = torch.zeros((chunk, 4), device=cuda_device)
        zero = torch.zeros(chunk, device=cuda_device)
        got = eng.apply_horizontal_turbulence(p, zero, x, 1.0, backward=False)[:, 1]
        if c is None:
            c = torch.full((chunk,), 110540.0, device=cuda_device)
        want = 0.0 + x / c
        same = (got.view(torch.int32) == want.view(torch.int32)) | (torch.isnan(got) & torch.isnan(want))
        assert bool(same.all()), (start, int((~same).sum()))
        del bits, x, p, got, want, same
