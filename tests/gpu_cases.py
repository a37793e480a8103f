"""Builders shared by the GPU tests: run the golden batches through the CUDA path."""

from __future__ import annotations

from datetime import UTC, datetime

import numpy as np
import torch

from fixtures import GoldenRun, conv_uniforms, noise_block, oracle_kwargs
from glide_b200.runtime import (BatchRunner, DomainSpec, EmanuelConfig, FootprintSpec, HannaConfig, ParticleState,
                                plan_steps)
from glide_b200.window import GridInfo, window_from_arrays


def grid_of(run: GoldenRun) -> GridInfo:
    m = run.met
    return GridInfo(np.asarray(m.lon), np.asarray(m.lat), np.asarray(m.levels), np.asarray(m.p_hpa))


def runner_for(run: GoldenRun, device, *, step_offset: int = 0, injected: bool = True, met_dtype: str = "f32",
               seed: int = 1234) -> BatchRunner:
    z = run.z
    m = run.met
    grid = grid_of(run).to_device(device)
    times = [m.time(h) for h in range(m.n_snapshots)]
    cache: dict = {}

    def window_provider(hour: datetime):
        h = m.index(hour)
        if h not in cache:
            cache.clear()
            cache[h] = window_from_arrays(m.fields, h, times, grid, device, lowest=int(np.argmin(m.levels)))
        return cache[h]

    n = run.n
    ms = int(z["max_substeps"])
    seed_n = int(z["noise_seed"])
    cseed = int(z["conv_seed"])

    def noise_provider(steps):
        sub, mea = noise_block(seed_n, [s + step_offset for s in steps], ms, n)
        return torch.from_numpy(sub).to(device), torch.from_numpy(mea).to(device)

    def conv_provider(step):
        u1, u2 = conv_uniforms(cseed, step + step_offset, n)
        return torch.from_numpy(np.stack([u1, u2])).to(device)

    nxy = z["grid_nxy"]
    n_rel = int(z["release_idx"].max()) + 1
    return BatchRunner(
        grid=grid, window_provider=window_provider,
        hanna=HannaConfig(meander_enabled=bool(z["meander"]), max_substeps=ms),
        footprint=FootprintSpec(tuple(z["grid_lon"]), tuple(z["grid_lat"]), int(nxy[0]), int(nxy[1]),
                                tuple(float(e) for e in z["grid_z"]), int(nxy[2]), n_rel),
        domain=DomainSpec(tuple(z["dom_lon"]), tuple(z["dom_lat"]), float(z["dom_alt"])),
        emanuel=EmanuelConfig() if bool(z["convection"]) else None,
        met_dtype=met_dtype, device=device, seed=seed,
        noise_provider=noise_provider if injected else None,
        conv_uniform_provider=conv_provider if injected else None,
    )


def state_from(particles, rel_off, win_end, ridx, device, state: dict | None = None, alive=None) -> ParticleState:
    st = ParticleState.from_particles(np.asarray(particles).T.copy(), rel_off, win_end, ridx, device)
    if state is not None:
        for k, v in state.items():
            getattr(st, k).copy_(torch.as_tensor(np.asarray(v, dtype=np.float32)))
    if alive is not None:
        st.alive.copy_(torch.as_tensor(np.asarray(alive, dtype=np.uint8)))
    return st


def cursor_of(run: GoldenRun, step: int) -> datetime:
    z = run.z
    steps = plan_steps(run.dt_("batch_start"), run.dt_("cursor_start"), run.dt_("cursor_terminus"), float(z["dt_s"]))
    return steps[step].cursor


def run_gpu(run: GoldenRun, device, *, max_steps=None, **kw):
    z = run.z
    r = runner_for(run, device, **kw)
    st = state_from(z["particles0"], z["rel_off"], z["win_end_off"], z["release_idx"], device)
    out = r.start(st, batch_start=run.dt_("batch_start"), cursor_start=run.dt_("cursor_start"),
                  cursor_terminus=run.dt_("cursor_terminus"), sim_length_s=float(z["sim_length_s"]),
                  dt_seconds=float(z["dt_s"]), max_steps=max_steps).run()
    torch.cuda.synchronize()
    return out


def as_numpy(out):
    s = out.state
    parts = np.stack([s.lon.cpu().numpy(), s.lat.cpu().numpy(), s.z.cpu().numpy(), s.weight.cpu().numpy()])
    state = {k: getattr(s, k).cpu().numpy() for k in ("u_prime", "v_prime", "w_prime", "u_meander", "v_meander")}
    return parts, state, s.alive.cpu().numpy().astype(bool), out.footprint.cpu().numpy()


def oracle_from(run: GoldenRun, **kw):
    from oracle.runtime import run_batch

    return run_batch(**oracle_kwargs(run), **kw)


UTC_ = UTC
