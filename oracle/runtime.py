"""Oracle: the per-step runtime body around the scheme (test infrastructure only).

Restates the static branch of the reference's cursor loop
(``src/lpdm/main.py:1382-1477``): active mask, met window and RK2 time weight,
the scheme step, once-per-window convection, time-ago bin, footprint
scatter-add (``src/lpdm/footprint_gridder.py:117-197``) and the escape kill
(``main.py:690-711``).
"""

from __future__ import annotations

from collections.abc import Callable
from dataclasses import dataclass, field
from datetime import UTC, datetime, timedelta

import numpy as np

from oracle import convection as conv
from oracle.hanna import HannaParams, StepNoise, build_step_inputs, step_core


@dataclass(frozen=True)
class GridSpec:
    """``OutputGridConfig`` + gridder shape (config.py:360-382, footprint_gridder.py:50-115)."""

    lon_bounds: tuple[float, float]
    lat_bounds: tuple[float, float]
    n_x: int
    n_y: int
    z_edges: tuple[float, ...]
    n_time_bins: int
    n_releases: int = 1

    @property
    def shape(self) -> tuple[int, int, int, int, int]:
        return (self.n_releases, self.n_time_bins, len(self.z_edges) - 1, self.n_y, self.n_x)


@dataclass(frozen=True)
class DomainSpec:
    """``MetDomainConfig`` bounds used by the escape test (config.py:385-455)."""

    lon_bounds: tuple[float, float]
    lat_bounds: tuple[float, float]
    alt_max_m: float


def hour_floor(t: datetime) -> datetime:
    """main.py:380-381"""
    return t.astimezone(UTC).replace(minute=0, second=0, microsecond=0)


def advection_alpha(time_start: datetime, time_end: datetime, t_cursor: datetime, delta_s: float) -> float:
    """``_advection_alpha_wind_mean`` alpha (main.py:892-919)."""
    ts, te = time_start.timestamp(), time_end.timestamp()
    t_eval = t_cursor.timestamp() - 0.5 * delta_s
    return max(0.0, min(1.0, (t_eval - ts) / max(1.0, float(te - ts))))


def footprint_indices(xyz, active, t_idx, release_idx, g: GridSpec, dt):
    """Flat cell index and validity of ``FootprintGridder.accumulate`` (footprint_gridder.py:154-193)."""
    lon, lat, z = xyz[0].astype(dt), xyz[1].astype(dt), xyz[2].astype(dt)
    x_idx = np.floor((lon - dt(g.lon_bounds[0])) / dt(max(1e-6, g.lon_bounds[1] - g.lon_bounds[0])) * dt(g.n_x))
    y_idx = np.floor((lat - dt(g.lat_bounds[0])) / dt(max(1e-6, g.lat_bounds[1] - g.lat_bounds[0])) * dt(g.n_y))
    with np.errstate(invalid="ignore"):
        x_idx = np.nan_to_num(x_idx, nan=-1.0, posinf=-1.0, neginf=-1.0).astype(np.int64)
        y_idx = np.nan_to_num(y_idx, nan=-1.0, posinf=-1.0, neginf=-1.0).astype(np.int64)
    edges = np.asarray(g.z_edges, dtype=dt)
    n_z = edges.size - 1
    z_idx = np.searchsorted(edges, z, side="left") - 1
    valid = (active & (release_idx >= 0) & (release_idx < g.n_releases) & (x_idx >= 0) & (x_idx < g.n_x)
             & (y_idx >= 0) & (y_idx < g.n_y) & (z_idx >= 0) & (z_idx < n_z) & (t_idx >= 0)
             & (t_idx < g.n_time_bins))
    r = np.clip(release_idx, 0, g.n_releases - 1)
    t = np.clip(t_idx, 0, g.n_time_bins - 1)
    zc = np.clip(z_idx, 0, n_z - 1)
    yc = np.clip(y_idx, 0, g.n_y - 1)
    xc = np.clip(x_idx, 0, g.n_x - 1)
    st = n_z * g.n_y * g.n_x
    flat = r * (g.n_time_bins * st) + t * st + zc * (g.n_y * g.n_x) + yc * g.n_x + xc
    return flat, valid


def accumulate(fp_flat, xyz, active, weights, t_idx, release_idx, g: GridSpec, delta: float, dt, fdt=None):
    """``FootprintGridder.accumulate``: scatter-add ``weight * valid * dt`` in particle order;
    the cell indices in ``dt``, the contributions formed and added in ``fdt`` (default ``dt``)."""
    fdt = fdt or dt
    flat, valid = footprint_indices(xyz, active, t_idx, release_idx, g, dt)
    w_eff = weights.astype(fdt) * valid.astype(fdt) * fdt(delta)
    np.add.at(fp_flat, flat, w_eff)


def within_met_domain(xyz, d: DomainSpec, dt):
    """main.py:690-711"""
    lon, lat, z = xyz[0].astype(dt), xyz[1].astype(dt), xyz[2].astype(dt)
    return ((lon >= dt(d.lon_bounds[0])) & (lon <= dt(d.lon_bounds[1])) & (lat >= dt(d.lat_bounds[0]))
            & (lat <= dt(d.lat_bounds[1])) & (z <= dt(d.alt_max_m)))


def time_ago_index(win_end_off, cursor_off: float, n_time_bins: int, dt):
    """main.py:1459-1465"""
    el = np.maximum(win_end_off.astype(dt) - dt(cursor_off), dt(0))
    t_idx = np.floor(el / dt(3600.0)).astype(np.int64)
    if n_time_bins == 1:
        t_idx = np.minimum(t_idx, 0)
    return t_idx


def window_from_met(hmt) -> dict:
    """Oracle window dict from an ``HourlyMetTensors`` (reference's or glide_b200's)."""
    names = hmt.channel_names
    w: dict = {}
    for n in ("u", "v", "w", "t", "q"):
        if n in names:
            s, e = hmt.channel(n)
            w[n] = np.stack([np.asarray(s.detach().cpu().float()), np.asarray(e.detach().cpu().float())])
    for n in ("blh", "sp", "ustar", "shf"):
        if n in names:
            s, e = hmt.channel(n)
            w[n] = np.stack([np.asarray(s[0].detach().cpu().float()), np.asarray(e[0].detach().cpu().float())])
    md = hmt.metadata
    w["height"] = np.asarray(hmt.height_agl_m.detach().cpu().float())
    w["level"] = np.asarray(md.level, dtype=np.float64)
    w["p_hpa"] = np.asarray(md.pressure_level_hpa, dtype=np.float64)
    w["lon"] = np.asarray(md.lon, dtype=np.float64)
    w["lat"] = np.asarray(md.lat, dtype=np.float64)
    w["time_start"] = md.time_start
    w["time_end"] = md.time_end
    return w


@dataclass
class BatchResult:
    particles: np.ndarray  # [4, N]
    state: dict
    alive: np.ndarray
    footprint: np.ndarray  # [R, T, Zb, Y, X]
    escaped_per_step: list = field(default_factory=list)
    active_per_step: list = field(default_factory=list)
    convection: list = field(default_factory=list)  # (window start, fires, n_moved)
    n_steps: int = 0
    snapshots: dict = field(default_factory=dict)
    # per-step diagnostics (main.py:1565-1566): mean (lon, lat, z) of all particles after the
    # step, and the grid-mean (u, v, w) of the window lerped by the step's RK2 weight
    diag_pos: list = field(default_factory=list)
    diag_wind: list = field(default_factory=list)


def wind_mean(win: dict, alpha: float) -> np.ndarray:
    """``_advection_alpha_wind_mean``'s wind (main.py:892-938): float32 grid means of u, v, w of
    the two snapshots, lerped as ``mean_start * (1 - alpha) + mean_end * alpha`` in float32."""
    m = [np.array([np.mean(win[c][s], dtype=np.float64) for c in ("u", "v", "w")]).astype(np.float32)
         for s in (0, 1)]
    return m[0] * np.float32(1.0 - alpha) + m[1] * np.float32(alpha)


def run_batch(*, get_window: Callable[[datetime], dict], particles, rel_off, win_end_off, release_idx,
              batch_start: datetime, cursor_start: datetime, cursor_terminus: datetime, sim_length_s: float,
              dt_seconds: float, params: HannaParams, grid: GridSpec, domain: DomainSpec,
              noise_fn: Callable[[int], StepNoise], emanuel: conv.EmanuelParams | None = None,
              conv_uniforms_fn: Callable[[int], tuple[np.ndarray, np.ndarray]] | None = None,
              dtype=np.float32, conv_dtype=None, max_steps: int | None = None,
              init_state: dict | None = None, init_alive=None, step_offset: int = 0,
              inputs_cache: dict | None = None, convect_first: bool = True,
              snapshot_steps: tuple = (), fp_dtype=None) -> BatchResult:
    """The static cursor loop of ``main._run`` for one batch (main.py:1382-1477).

    ``init_state`` / ``init_alive`` / ``step_offset`` resume a batch mid-way: the
    loop starts at ``cursor_start`` from that state and numbers its steps from
    ``step_offset`` (the noise rows). ``inputs_cache`` keeps the per-window support
    stacks across calls; ``convect_first=False`` treats the first window as already
    convected (a resumed mid-window start). ``snapshot_steps``: step counts after
    which the particles are recorded in ``BatchResult.snapshots``. ``fp_dtype`` is the
    footprint's value type (default: ``dtype``): float64 with float32 particles is the
    FP64 gridder fed float32 positions and weights."""
    dt = dtype
    conv_dt = conv_dtype or dtype
    fdt = fp_dtype or dtype
    n = particles.shape[1]
    p = particles.astype(dt).copy()
    state = {k: np.zeros(n, dtype=dt) for k in ("u_prime", "v_prime", "w_prime")}
    if params.meander_enabled:
        state["u_meander"] = np.zeros(n, dtype=dt)
        state["v_meander"] = np.zeros(n, dtype=dt)
    if init_state is not None:
        state = {k: np.asarray(init_state[k], dtype=dt).copy() for k in state}
    alive = np.ones(n, dtype=bool) if init_alive is None else np.asarray(init_alive, dtype=bool).copy()
    fp = np.zeros(int(np.prod(grid.shape)), dtype=fdt)
    rel_off = rel_off.astype(dt)
    win_end_off = win_end_off.astype(dt)
    res = BatchResult(p, state, alive, fp.reshape(grid.shape))
    bstart = batch_start.timestamp()
    cache: dict = inputs_cache if inputs_cache is not None else {}
    last_bracket = None if convect_first else hour_floor(cursor_start)
    t_cursor = cursor_start
    step = 0
    while t_cursor > cursor_terminus:
        if max_steps is not None and step >= max_steps:
            break
        gstep = step + step_offset
        delta = min(float(dt_seconds), (t_cursor - cursor_terminus).total_seconds())
        cur = t_cursor.timestamp() - bstart
        active = (rel_off >= dt(cur)) & ((rel_off - dt(sim_length_s)) <= dt(cur)) & alive
        hk = hour_floor(t_cursor)
        if cache.get("key") != hk:
            win = get_window(hk)
            cache.clear()
            cache.update(key=hk, win=win, inp=build_step_inputs(win, params, dt))
        win, inp = cache["win"], cache["inp"]
        alpha = advection_alpha(win["time_start"], win["time_end"], t_cursor, delta)
        p, state = step_core(p, state, active, inp, alpha, delta, params, noise_fn(gstep), dt)
        if win["time_start"] != last_bracket:
            if emanuel is not None and bool(np.any(active)):
                col = conv.build_column(win["t"][0], win["t"][1], win["q"][0], win["q"][1], win["height"],
                                        win["p_hpa"], alpha, emanuel, conv_dt)
                u1, u2 = conv_uniforms_fn(gstep)
                z_new, n_moved = conv.redistribute(p[2], active, col, u1, u2, conv_dt)
                p[2] = z_new.astype(dt)
                res.convection.append((win["time_start"], col.fires, n_moved))
            last_bracket = win["time_start"]
        t_idx = time_ago_index(win_end_off, cur, grid.n_time_bins, dt)
        accumulate(fp, p[:3], active, p[3], t_idx, release_idx, grid, delta, dt, fdt)
        escaped = active & ~within_met_domain(p[:3], domain, dt)
        alive = alive & ~escaped
        res.escaped_per_step.append(int(escaped.sum()))
        res.active_per_step.append(int(active.sum()))
        res.diag_pos.append(np.mean(p[:3].astype(np.float64), axis=1).astype(dt))
        res.diag_wind.append(wind_mean(win, alpha))
        t_cursor = t_cursor - timedelta(seconds=delta)
        step += 1
        if step in snapshot_steps:
            res.snapshots[step] = p.copy()
    res.particles, res.state, res.alive = p, state, alive
    res.footprint = fp.reshape(grid.shape)
    res.n_steps = step
    return res
