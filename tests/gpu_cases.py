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
               seed: int = 1234, hanna_kw: dict | None = None, launch_variant: int = 0,
               reorder: bool = True, steps_per_launch: int | None = None,
               fuse_convection: bool = True, fp_dtype: str = "f32") -> BatchRunner:
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
    runner = BatchRunner(
        grid=grid, window_provider=window_provider,
        hanna=HannaConfig(meander_enabled=bool(z["meander"]), max_substeps=ms, **(hanna_kw or {})),
        footprint=FootprintSpec(tuple(z["grid_lon"]), tuple(z["grid_lat"]), int(nxy[0]), int(nxy[1]),
                                tuple(float(e) for e in z["grid_z"]), int(nxy[2]), n_rel, value_dtype=fp_dtype),
        domain=DomainSpec(tuple(z["dom_lon"]), tuple(z["dom_lat"]), float(z["dom_alt"])),
        emanuel=EmanuelConfig() if bool(z["convection"]) else None,
        met_dtype=met_dtype, device=device, seed=seed,
        noise_provider=noise_provider if injected else None,
        conv_uniform_provider=conv_provider if injected else None,
    )
    runner.launch_variant = launch_variant
    runner.reorder = reorder
    runner.steps_per_launch = steps_per_launch
    runner.fuse_convection = fuse_convection
    return runner


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


def hourly_window(run: GoldenRun, h: int):
    """The reference-format ``HourlyMetTensors`` of bracket ``[h, h+1]`` (host tensors,
    2-D fields broadcast over Z)."""
    from glide_b200.met import HourlyMetTensors, MetFieldMetadata

    m = run.met
    names = ("u", "v", "w", "blh", "sp", "t", "ustar", "shf", "q")
    nz = m.fields["u"].shape[1]

    def stack(k):
        chans = []
        for name in names:
            f = torch.as_tensor(m.fields[name][k])
            chans.append(f.unsqueeze(0).expand(nz, -1, -1) if f.dim() == 2 else f)
        return torch.stack(chans)

    md = MetFieldMetadata(lon=np.asarray(m.lon), lat=np.asarray(m.lat), level=np.asarray(m.levels),
                          pressure_level_hpa=np.asarray(m.p_hpa), time_start=m.time(h), time_end=m.time(h + 1))
    lev = torch.as_tensor(np.asarray(m.levels, dtype=np.float32)).view(-1, 1, 1)
    return HourlyMetTensors(stack(h), stack(h + 1), md, names, lev.expand(nz, *m.fields["u"].shape[2:]))


def run_plugin_loop(run: GoldenRun, device):
    """The reference's static per-step runtime body (main.py:1382-1477) driving the
    B200 plug-ins: HannaB200Scheme.step, EmanuelB200Convection.maybe_convect,
    FootprintGridderB200.accumulate and the escape kill, with injected noise."""
    from glide_b200.runtime import plan_steps
    from glide_b200.schemes import FootprintGridderB200, get_convection_scheme, get_scheme

    z = run.z
    n = run.n
    ms = int(z["max_substeps"])
    seed, cseed = int(z["noise_seed"]), int(z["conv_seed"])

    def noise(step):
        from fixtures import step_noise

        sub, mea = step_noise(seed, step, ms, n)
        return torch.from_numpy(sub).to(device), torch.from_numpy(mea).to(device)

    cur_step = {"k": 0}

    def uniforms(_call):
        u1, u2 = conv_uniforms(cseed, cur_step["k"], n)
        return torch.from_numpy(np.stack([u1, u2])).to(device)

    scheme = get_scheme("hanna_1982_b200", meander_enabled=bool(z["meander"]), max_substeps=ms,
                        noise_provider=noise)
    conv = (get_convection_scheme("emanuel_reduced_b200", uniform_provider=uniforms)
            if bool(z["convection"]) else None)
    nxy = z["grid_nxy"]
    gridder = FootprintGridderB200(tuple(z["grid_lon"]), tuple(z["grid_lat"]), tuple(z["grid_z"]), int(nxy[2]),
                                   int(nxy[1]), int(nxy[0]), n_releases=int(z["release_idx"].max()) + 1,
                                   device=device)
    particles = torch.as_tensor(z["particles0"].T.copy(), device=device)
    state = scheme.initialize_state(n, device=device, dtype=torch.float32)
    rel = torch.as_tensor(z["rel_off"], device=device)
    wend = torch.as_tensor(z["win_end_off"], device=device)
    ridx = torch.as_tensor(z["release_idx"], device=device)
    alive = torch.ones(n, dtype=torch.bool, device=device)
    L = float(z["sim_length_s"])
    dl0, dl1 = (float(v) for v in z["dom_lon"])
    da0, da1 = (float(v) for v in z["dom_lat"])
    alt = float(z["dom_alt"])
    esc, act = [], []
    last_bracket = None
    windows: dict = {}
    steps = plan_steps(run.dt_("batch_start"), run.dt_("cursor_start"), run.dt_("cursor_terminus"), float(z["dt_s"]))
    for k, st in enumerate(steps):
        cur = st.cursor_off
        active = (rel >= cur) & (rel - L <= cur) & alive
        h = run.met.index(st.hour)
        if h not in windows:
            windows.clear()
            windows[h] = hourly_window(run, h)
        win = windows[h]
        particles, state = scheme.step(particles, state, win, st.alpha, st.delta, active, None)
        if win.metadata.time_start != last_bracket:
            if conv is not None:
                cur_step["k"] = k
                particles, _ = conv.maybe_convect(particles, {}, win, t_alpha=st.alpha, dt_seconds=st.delta,
                                                  active_mask=active, engine=None)
            last_bracket = win.metadata.time_start
        t_idx = ((wend - cur).clamp_(min=0.0) / 3600.0).floor().to(torch.int64)
        if gridder.n_t == 1:
            t_idx.clamp_(max=0)
        gridder.accumulate(particles[:, :3], active, particles[:, 3], t_idx, ridx, st.delta)
        lon, lat, zz = particles[:, 0], particles[:, 1], particles[:, 2]
        within = (lon >= dl0) & (lon <= dl1) & (lat >= da0) & (lat <= da1) & (zz <= alt)
        newly = active & ~within
        alive = alive & ~newly
        esc.append(int(newly.sum()))
        act.append(int(active.sum()))
    torch.cuda.synchronize()
    return particles.T.cpu().numpy(), alive.cpu().numpy(), gridder.tensor.cpu().numpy(), np.array(esc), \
        np.array(act), scheme.device_status
