"""Physics checks of the CUDA path that need no oracle:

* the well-mixed criterion (Thomson 1987) through the Hanna backward step, set up
  as the reference's V1 test (tests/test_main_runtime.py:575-732 of the reference:
  neutral BL, uniform fields, particles uniform in [0, blh], reflection at the
  BL top added by the harness) with 100,000 particles instead of 6,000;
* inactive particles come back bit-unchanged (turbulence/base.py:51-76);
* with zero turbulent noise and zero initial perturbation velocities in a uniform
  wind, the horizontal step is exactly the RK2 midpoint formula.
"""

from __future__ import annotations

from datetime import UTC, datetime, timedelta

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def uniform_window(*, blh=3000.0, ustar=0.4, u=0.0, v=0.0, n_lev=6, n_lat=4, n_lon=4, shf=0.0):
    from glide_b200.met import HourlyMetTensors, MetFieldMetadata

    shape = (n_lev, n_lat, n_lon)
    vals = {"u": u, "v": v, "w": 0.0, "blh": blh, "sp": 101325.0, "t": 280.0, "ustar": ustar, "shf": shf, "q": 0.0}
    names = tuple(vals)
    fields = torch.stack([torch.full(shape, float(vals[k])) for k in names])
    t0 = datetime(2024, 1, 1, 12, 0, 0, tzinfo=UTC)
    level = np.linspace(0.0, max(4000.0, 1.5 * blh), n_lev)
    md = MetFieldMetadata(lon=np.linspace(-2.0, 2.0, n_lon), lat=np.linspace(40.0, 50.0, n_lat), level=level,
                          pressure_level_hpa=np.linspace(1000.0, 600.0, n_lev), time_start=t0,
                          time_end=t0 + timedelta(hours=1))
    height = torch.as_tensor(level, dtype=torch.float32).view(n_lev, 1, 1).expand(shape).contiguous()
    return HourlyMetTensors(fields, fields.clone(), md, names, height)


def test_well_mixed_criterion_hanna_backward(cuda_device):
    from glide_b200.schemes import HannaB200Scheme

    torch.manual_seed(202605301)
    blh = 3000.0
    scheme = HannaB200Scheme(meander_enabled=False, seed=7)
    met = uniform_window(blh=blh, ustar=0.4)
    n = 100_000
    p = torch.zeros(n, 4, dtype=torch.float32, device=cuda_device)
    p[:, 1] = 45.0
    p[:, 2] = torch.rand(n, device=cuda_device) * blh
    p[:, 3] = 1.0 / n
    state = scheme.initialize_state(n, device=cuda_device, dtype=torch.float32)
    active = torch.ones(n, dtype=torch.bool, device=cuda_device)
    for _ in range(1500):  # dt 15 s, ~100 T_L
        p, state = scheme.step(p, state, met, 0.5, 15.0, active, None)
        above = p[:, 2] > blh  # harness reflection at the BL top, as in the reference test
        p[:, 2] = torch.where(above, 2.0 * blh - p[:, 2], p[:, 2])
        state["w_prime"] = torch.where(above, -state["w_prime"], state["w_prime"])
    z = p[:, 2].cpu().numpy()
    assert scheme.device_status == 0
    in_bl = (z >= 0.0) & (z <= blh)
    assert in_bl.mean() > 0.99
    counts, _ = np.histogram(z[in_bl], bins=np.linspace(0.0, blh, 11))
    interior = counts[2:8]
    rel_rms = float(np.sqrt(np.mean(((interior - interior.mean()) / interior.mean()) ** 2)))
    assert rel_rms < 0.15, (rel_rms, counts.tolist())


def test_inactive_particles_are_unchanged(cuda_device):
    from glide_b200.schemes import HannaB200Scheme

    scheme = HannaB200Scheme(meander_enabled=True, seed=3)
    met = uniform_window(u=5.0, v=-3.0)
    n = 4096
    g = torch.Generator(device=cuda_device).manual_seed(1)
    p = torch.stack([torch.rand(n, device=cuda_device, generator=g) * 3 - 1.5,
                     41 + torch.rand(n, device=cuda_device, generator=g) * 8,
                     torch.rand(n, device=cuda_device, generator=g) * 2000,
                     torch.full((n,), 1.0 / n, device=cuda_device)], dim=1).contiguous()
    state = scheme.initialize_state(n, device=cuda_device, dtype=torch.float32)
    for k in state:
        state[k].normal_(generator=g)
    active = torch.rand(n, device=cuda_device, generator=g) < 0.5
    p0 = p.clone()
    s0 = {k: v.clone() for k, v in state.items()}
    p, state = scheme.step(p, state, met, 0.3, 30.0, active, None)
    torch.cuda.synchronize()
    inact = ~active
    assert torch.equal(p[inact], p0[inact])
    for k in state:
        assert torch.equal(state[k][inact], s0[k][inact]), k
    assert not torch.equal(p[active], p0[active])


def test_uniform_wind_step_is_rk2_midpoint(cuda_device):
    from glide_b200.schemes import HannaB200Scheme

    n = 2048
    ms = 6
    zeros = (torch.zeros(ms, 3, n, device=cuda_device), torch.zeros(2, n, device=cuda_device))
    scheme = HannaB200Scheme(meander_enabled=False, max_substeps=ms, noise_provider=lambda k: zeros)
    u, v = 12.0, -7.0
    met = uniform_window(u=u, v=v, ustar=0.3)
    lat0 = torch.linspace(41.0, 49.0, n, device=cuda_device)
    p = torch.stack([torch.zeros(n, device=cuda_device), lat0, torch.full((n,), 500.0, device=cuda_device),
                     torch.full((n,), 1.0 / n, device=cuda_device)], dim=1).contiguous()
    state = scheme.initialize_state(n, device=cuda_device, dtype=torch.float32)
    active = torch.ones(n, dtype=torch.bool, device=cuda_device)
    dt = 60.0
    p, state = scheme.step(p, state, met, 0.5, dt, active, None)
    lat = lat0.double().cpu().numpy()
    lat_mid = lat - 0.5 * dt * v / 110540.0
    exp_lon = -dt * u / (111320.0 * np.abs(np.cos(np.deg2rad(lat_mid))))
    exp_lat = lat - dt * v / 110540.0
    got = p.double().cpu().numpy()
    np.testing.assert_allclose(got[:, 0], exp_lon, rtol=2e-5, atol=1e-9)
    np.testing.assert_allclose(got[:, 1], exp_lat, rtol=1e-6)
    assert torch.all(state["u_prime"] == 0) and torch.all(state["v_prime"] == 0)
