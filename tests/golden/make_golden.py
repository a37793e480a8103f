"""Generate the golden fixtures by running the reference implementation itself.

Run in a container that holds the reference source (mrghg/glide) read-only:

    python tests/golden/make_golden.py --reference /path/to/glide

It imports the reference's ``src/lpdm`` (an ``xarray`` stand-in module is put
on the path: the hot path only uses xarray for type annotations), builds small
synthetic met windows with ``glide_b200.synthetic``, and records:

* ``units.npz`` — reference outputs of the free physics functions, the grid
  samplers, the per-window support stacks and the Emanuel column build;
* ``run_small.npz`` — a whole batch through the reference's static step path
  (``HannaScheme`` with ``static_substeps=True``, meander on,
  ``EmanuelReducedConvection``, ``FootprintGridder``, the escape kill), driven
  by a replica of the cursor loop ``main.py:1382-1477`` with injected noise.
* ``run_c0.npz`` — a 3 h batch on the 64x64x40 smoke-case met with meander
  and convection off (the met is regenerated from its seed; a checksum of it
  is stored);
* ``run_c1.npz`` — the single-site EUROPE-box workload (60x281x401 met, dt
  30 s, meander and hourly convection on) for 20,000 particles of its release,
  2 h backward from the release end (met regenerated from its seed).

Every batch also records the runtime's per-step diagnostics (mean particle
position, grid-mean wind; ``main.py:1565-1566``) and the footprint of the same
trajectories accumulated by the reference's gridder in float64
(``out_footprint_f64``): the float32 gridder adds ~1e5 contributions per cell at the
EUROPE-box case, and its round-off (1.7e-3 relative L1 there) is larger than the
trajectories' differences.

Noise is not stored: it is regenerated from the recorded seed by
``tests/golden/noise.py``.
"""

from __future__ import annotations

import argparse
import math
import sys
import tempfile
import types
from datetime import UTC, datetime, timedelta
from pathlib import Path
from types import SimpleNamespace

import numpy as np

HERE = Path(__file__).resolve().parent
REPO = HERE.parents[1]
sys.path.insert(0, str(REPO))
sys.path.insert(0, str(HERE))

from noise import conv_uniforms, step_noise  # noqa: E402

from glide_b200.synthetic import SyntheticMet, SyntheticMetSpec, config_met_spec  # noqa: E402


def _import_reference(ref_root: Path):
    stub_dir = Path(tempfile.mkdtemp(prefix="glide_xr_"))
    (stub_dir / "xarray").mkdir()
    (stub_dir / "xarray" / "__init__.py").write_text(
        "class Dataset:\n    pass\n\n\nclass DataArray:\n    pass\n"
    )
    # a source tree (src/lpdm) or an installed package directory (lpdm)
    sys.path.insert(0, str(ref_root / "src") if (ref_root / "src" / "lpdm").is_dir() else str(ref_root))
    sys.path.insert(0, str(stub_dir))
    import os

    os.environ["GLIDE_STATIC_SUBSTEPS"] = "1"
    os.environ["GLIDE_COMPILE"] = "0"
    import lpdm.convection.emanuel as em
    import lpdm.footprint_gridder as fg
    import lpdm.gpu_engine as ge
    import lpdm.main as lmain
    import lpdm.met_reader as mr
    import lpdm.turbulence.hanna as hn

    return SimpleNamespace(em=em, fg=fg, ge=ge, main=lmain, mr=mr, hn=hn)


def _ref_window(ref, syn: SyntheticMet, h: int):
    """A reference ``HourlyMetTensors`` for bracket ``[h, h+1]``."""
    win = syn.window(h)
    md = win.metadata
    return ref.mr.HourlyMetTensors(
        hour_start=win.hour_start.contiguous(),
        hour_end=win.hour_end.contiguous(),
        metadata=ref.mr.MetFieldMetadata(
            lon=md.lon, lat=md.lat, level=md.level, pressure_level_hpa=md.pressure_level_hpa,
            time_start=md.time_start, time_end=md.time_end, variable_units=dict(md.variable_units)),
        channel_names=win.channel_names,
        height_agl_m=win.height_agl_m.contiguous(),
    )


def _met_arrays(syn: SyntheticMet) -> dict:
    out = {}
    for name in ("u", "v", "w", "t", "q", "blh", "sp", "ustar", "shf"):
        out[f"met_{name}"] = np.stack([f[name].numpy() for f in syn.fields]).astype(np.float32)
    out["met_levels"] = syn.levels
    out["met_p_hpa"] = syn.pressure_level_hpa
    out["met_lon"] = syn.lon
    out["met_lat"] = syn.lat
    out["met_t0"] = np.array(syn.times[0].timestamp())
    return out


# ---------------------------------------------------------------------------
# unit goldens
# ---------------------------------------------------------------------------


def make_units(ref, out_path: Path) -> None:
    import torch

    hn, em, ge = ref.hn, ref.em, ref.ge
    rng = np.random.default_rng(7)
    n = 2000
    z = np.concatenate([rng.uniform(0.0, 2500.0, n - 8), [0.0, 1.0, 2.0, 5.0, 1000.0, 1500.0, 3000.0, 50.0]])
    blh = rng.uniform(50.0, 2000.0, n)
    ustar = rng.uniform(1e-3, 0.8, n)
    w_star = np.where(rng.uniform(size=n) < 0.5, 0.0, rng.uniform(0.1, 3.0, n))
    hol = rng.choice([-50.0, -5.0, -1.0001, -0.5, 0.0, 0.5, 1.0001, 5.0, 50.0], n) * rng.uniform(0.5, 2.0, n)
    lat = rng.uniform(-80.0, 80.0, n)
    shf = rng.uniform(-200.0, 200.0, n)
    shf[:20] = 0.0
    tsfc = rng.uniform(260.0, 305.0, n)
    sp = rng.uniform(70000.0, 104000.0, n)
    f32 = lambda a: torch.as_tensor(np.asarray(a, dtype=np.float32))  # noqa: E731
    res = dict(z=z.astype(np.float32), blh=blh.astype(np.float32), ustar=ustar.astype(np.float32),
               w_star=w_star.astype(np.float32), hol=hol.astype(np.float32), lat=lat.astype(np.float32),
               shf=shf.astype(np.float32), tsfc=tsfc.astype(np.float32), sp=sp.astype(np.float32))
    outs = hn.in_bl_sigma_TL(f32(z), f32(blh), f32(ustar), f32(w_star), f32(hol), f32(lat))
    res["in_bl"] = np.stack([o.numpy() for o in outs])
    res["obukhov"] = hn.obukhov_length(f32(ustar), f32(shf), f32(tsfc), f32(sp)).numpy()
    res["wstar"] = hn.convective_velocity(f32(blh), f32(shf), f32(tsfc), f32(sp)).numpy()
    res["coriolis"] = hn.coriolis_parameter(f32(lat)).numpy()
    res["sl_sigma_w"] = hn.surface_layer_sigma_w(f32(z), f32(ustar), hn.obukhov_length(f32(ustar), f32(shf), f32(tsfc), f32(sp))).numpy()
    ri = rng.uniform(-1.0, 1.0, n).astype(np.float32)
    shear = rng.uniform(0.0, 0.05, n).astype(np.float32)
    n2 = rng.uniform(-1e-4, 4e-4, n).astype(np.float32)
    res.update(ri=ri, shear=shear, n2=n2)
    kz = hn.free_trop_diffusivity(f32(np.maximum(z, 1.0)), f32(shear), f32(ri))
    res["kz"] = kz.numpy()
    sw, tl = hn.free_trop_sigma_TL(kz, f32(n2))
    res["ft_sw"], res["ft_tl"] = sw.numpy(), tl.numpy()

    # grid sampling + support stacks on a small synthetic window
    syn = SyntheticMet(SyntheticMetSpec(nz=12, ny=20, nx=24, n_snapshots=2, moist_fraction=0.5, seed=101))
    res.update({f"u_{k}": v for k, v in _met_arrays(syn).items()})
    win = _ref_window(ref, syn, 0)
    scheme = hn.HannaScheme(meander_enabled=True, static_substeps=True, max_substeps=6)
    engine = ge.GPUEngine(device="cpu")
    ft, gb = scheme._free_trop_fields(win, torch.device("cpu"), torch.float32)
    res["stack_ft"] = ft.numpy()
    res["stack_density"] = scheme._density_fields(win, torch.device("cpu"), torch.float32).numpy()
    res["stack_meander"] = scheme._meander_sigma_fields(win, torch.device("cpu"), torch.float32)[0].numpy()
    m = 2000
    plon = rng.uniform(syn.lon[0] - 0.3, syn.lon[-1] + 0.3, m).astype(np.float32)
    plat = rng.uniform(syn.lat[0] - 0.3, syn.lat[-1] + 0.3, m).astype(np.float32)
    pz = np.concatenate([rng.uniform(-5.0, 21000.0, m - 6), syn.levels[:6]]).astype(np.float32)
    res.update(s_lon=plon, s_lat=plat, s_z=pz)
    res["sample_tri"] = hn.HannaScheme._interp_3d_field(ft, gb, f32(plon), f32(plat), f32(pz), engine).numpy()
    blh_s, blh_e = win.channel("blh")
    res["sample_bil"] = hn.HannaScheme._bilinear_at(blh_s[0], gb.lon_first, gb.lon_last, gb.lat_first, gb.lat_last,
                                                    f32(plon), f32(plat)).numpy()
    lerped = torch.empty_like(blh_s[0])
    torch.lerp(blh_s[0], blh_e[0], 0.3333, out=lerped)
    res["lerp_blh"] = lerped.numpy()

    # Emanuel column build on the window's bbox-mean column
    t_s, t_e = win.channel("t")
    q_s, q_e = win.channel("q")
    alpha = 0.37
    t_col = (t_s * (1.0 - alpha) + t_e * alpha).mean(dim=(1, 2))
    q_col = (q_s * (1.0 - alpha) + q_e * alpha).mean(dim=(1, 2)).clamp(min=0.0)
    p = torch.as_tensor(np.array(syn.pressure_level_hpa), dtype=torch.float32) * 100.0
    i_lcl, i_lnb, cape, dtv = em.compute_lcl_lnb_cape(t_col, q_col, p)
    res.update(c_t=t_col.numpy(), c_q=q_col.numpy(), c_p=p.numpy(),
               c_out=np.array([int(i_lcl), int(i_lnb), float(cape), float(dtv)], dtype=np.float64))
    fm = em.compute_mass_flux_matrix(t_col, q_col, p, i_lcl=int(i_lcl), i_lnb=int(i_lnb), m_b=0.05 * 3600.0)
    res["c_fmass"] = fm.numpy()
    res["c_layer_mass"] = em._layer_masses_per_area(p).numpy()
    np.savez_compressed(out_path, **res)
    print("wrote", out_path)


# ---------------------------------------------------------------------------
# whole-batch golden
# ---------------------------------------------------------------------------


class _NoiseShim:
    """Supplies injected noise to ``GPUEngine.update_langevin_velocity``: substep
    calls come in (u, v, w) triples per substep; meander calls carry a float
    ``t_lagrangian``."""

    def __init__(self, ref, seed: int, n: int, max_substeps: int) -> None:
        self.ref, self.seed, self.n, self.max_substeps = ref, seed, n, max_substeps
        self.step = 0
        self.calls = 0
        self.meander_calls = 0
        self.cached_step, self.cached = None, None
        self.orig = ref.ge.GPUEngine.update_langevin_velocity
        shim = self

        def patched(engine, w_prime, t_lagrangian, sigma_w2, dt_seconds, noise=None, drift=0.0):
            import torch

            if noise is None:
                if shim.cached_step != shim.step:  # one draw of the step's noise serves all its calls
                    shim.cached = step_noise(shim.seed, shim.step, shim.max_substeps, shim.n)
                    shim.cached_step = shim.step
                sub, mea = shim.cached
                if isinstance(t_lagrangian, float):
                    noise = torch.from_numpy(mea[shim.meander_calls].copy()).to(w_prime.device)
                    shim.meander_calls += 1
                else:
                    i, c = divmod(shim.calls, 3)
                    noise = torch.from_numpy(sub[i, c].copy()).to(w_prime.device)
                    shim.calls += 1
            return shim.orig(engine, w_prime, t_lagrangian, sigma_w2, dt_seconds, noise=noise, drift=drift)

        ref.ge.GPUEngine.update_langevin_velocity = patched

    def begin_step(self, step: int) -> None:
        self.step, self.calls, self.meander_calls = step, 0, 0

    def restore(self) -> None:
        self.ref.ge.GPUEngine.update_langevin_velocity = self.orig


class _RandShim:
    """Replaces ``torch.rand`` inside ``emanuel`` with the injected uniforms."""

    def __init__(self, ref, seed: int) -> None:
        self.ref, self.seed = ref, seed
        self.step = 0
        self.k = 0
        self.orig = ref.em.torch.rand
        shim = self
        real_torch = ref.em.torch

        def rand(n, generator=None, device=None, dtype=None):
            import torch

            u1, u2 = conv_uniforms(shim.seed, shim.step, int(n))
            arr = (u1, u2)[shim.k]
            shim.k += 1
            return torch.from_numpy(arr.copy()).to(device if device is not None else "cpu")

        proxy = types.ModuleType("torch_proxy")
        proxy.__dict__.update({k: getattr(real_torch, k) for k in dir(real_torch) if not k.startswith("__")})
        proxy.rand = rand
        ref.em.torch = proxy
        self.real_torch = real_torch

    def begin(self, step: int) -> None:
        self.step, self.k = step, 0

    def restore(self) -> None:
        self.ref.em.torch = self.real_torch


def _batch_setup(case: str):
    if case == "small":
        spec = SyntheticMetSpec(nz=12, ny=20, nx=24, n_snapshots=4, moist_fraction=0.5, seed=202,
                                start_time=datetime(2026, 1, 15, 0, tzinfo=UTC), wind_pert_m_s=6.0)
        rel = [  # (lon, lat, z, n, release time, duration)
            (2.9, 42.4, 50.0, 256, datetime(2026, 1, 15, 2, 10, tzinfo=UTC), 1800.0),
            (None, None, None, 512, datetime(2026, 1, 15, 2, 30, tzinfo=UTC), 1200.0),
        ]
        sim_length_s = 7170.0
        dt_s = 60.0
        meander, convection = True, True
        grid = dict(lon_bounds=(0.0, 5.75), lat_bounds=(40.0, 44.75), n_x=23, n_y=19, z_edges=(0.0, 100.0, 500.0),
                    n_time_bins=3)
        domain = dict(lon_bounds=(0.5, 5.25), lat_bounds=(40.5, 44.25), alt_max_m=6000.0)
    elif case == "c1":
        # the single-site EUROPE-box workload (60 x 281 x 401 met, dt 30 s, meander and hourly
        # convection on): 20,000 particles of its 100 m release at (-5, 52) over a 1 h release
        # window, run 2 h backward from the release end (every particle is 1-2 h old at the end)
        spec = config_met_spec(1, n_snapshots=4)
        t0 = spec.start_time
        rel = [(-5.0, 52.0, 100.0, 20000, t0 + timedelta(hours=1), 3600.0)]
        sim_length_s = 24 * 3600.0
        dt_s = 30.0
        meander, convection = True, True
        grid = dict(lon_bounds=(-60.125, 40.125), lat_bounds=(9.875, 80.125), n_x=401, n_y=281,
                    z_edges=(0.0, 100.0), n_time_bins=24)
        domain = dict(lon_bounds=(-60.0, 40.0), lat_bounds=(10.0, 80.0), alt_max_m=20000.0)
        return spec, rel, sim_length_s, dt_s, meander, convection, grid, domain, 2 * 3600.0
    else:
        spec = SyntheticMetSpec(nz=40, ny=64, nx=64, lon0=0.0, lat0=40.0, n_snapshots=5, moist_fraction=0.0,
                                seed=20261203, start_time=datetime(2026, 1, 14, 23, tzinfo=UTC))
        rel = [(8.0, 48.0, 50.0, 2000, datetime(2026, 1, 15, 1, 0, tzinfo=UTC), 3600.0)]
        sim_length_s = 3 * 3600.0
        dt_s = 60.0
        meander, convection = False, False
        grid = dict(lon_bounds=(0.0, 16.0), lat_bounds=(40.0, 56.0), n_x=64, n_y=64, z_edges=(0.0, 100.0),
                    n_time_bins=3)
        domain = dict(lon_bounds=(0.0, 15.75), lat_bounds=(40.0, 55.75), alt_max_m=20000.0)
    return spec, rel, sim_length_s, dt_s, meander, convection, grid, domain, None


def _particles(spec: SyntheticMetSpec, rel, seed: int):
    rng = np.random.default_rng(seed)
    batch_start = min(r[4] for r in rel)
    cols, offs, ends, ridx = [], [], [], []
    for k, (lon, lat, z, n, t_rel, dur) in enumerate(rel):
        if lon is None:  # a spread cloud over the domain: exercises every regime and edge
            lo = rng.uniform(spec.lon0 + 0.1, spec.lon0 + spec.dlon * (spec.nx - 1) - 0.1, n)
            la = rng.uniform(spec.lat0 + 0.1, spec.lat0 + spec.dlat * (spec.ny - 1) - 0.1, n)
            zz = np.exp(rng.uniform(np.log(1.0), np.log(8000.0), n))
        else:
            lo, la, zz = np.full(n, lon), np.full(n, lat), np.full(n, z)
        cols.append(np.stack([lo, la, zz, np.full(n, 1.0 / n)]))
        rel_off = (t_rel - batch_start).total_seconds()
        offs.append(rng.uniform(0.0, dur, n) + rel_off)
        ends.append(np.full(n, rel_off + dur))
        ridx.append(np.full(n, k))
    return (np.concatenate(cols, axis=1).astype(np.float32), np.concatenate(offs).astype(np.float32),
            np.concatenate(ends).astype(np.float32), np.concatenate(ridx).astype(np.int64), batch_start)


def drive_batch(ref, case: str, noise_seed: int, device: str = "cpu", snap_every: int = 20) -> dict:
    """Runs golden case ``case`` through the reference's static step path on ``device``
    (its eager torch ops on the CPU or on CUDA), with the injected noise of ``noise_seed``,
    driven by a replica of the cursor loop ``main.py:1382-1477``; returns the fixture's
    arrays (inputs, run configuration and outputs)."""
    import torch

    dev = torch.device(device)
    spec, rel, sim_length_s, dt_s, meander, convection, grid, domain, run_s = _batch_setup(case)
    syn = SyntheticMet(spec)
    particles, rel_off, win_end, ridx, batch_start = _particles(spec, rel, noise_seed + 1)
    n = particles.shape[1]
    max_substeps = 6
    window_ends = [r[4] + timedelta(seconds=r[5]) for r in rel]
    cursor_start = max(window_ends)
    terminus = min(window_ends) - timedelta(seconds=sim_length_s if run_s is None else run_s)

    scheme = ref.hn.HannaScheme(meander_enabled=meander, static_substeps=True, max_substeps=max_substeps)
    conv_scheme = ref.em.EmanuelReducedConvection() if convection else None
    engine = ref.ge.GPUEngine(device=str(dev))
    gridder = ref.fg.FootprintGridder(lon_bounds=grid["lon_bounds"], lat_bounds=grid["lat_bounds"],
                                      z_edges_m=grid["z_edges"], n_time_bins=grid["n_time_bins"],
                                      n_y=grid["n_y"], n_x=grid["n_x"], n_releases=len(rel), device=dev)
    # the same gridder in float64 fed the same (float32) trajectories: the footprint without
    # the float32 round-off of ~1e5 small additions per cell
    gridder64 = ref.fg.FootprintGridder(lon_bounds=grid["lon_bounds"], lat_bounds=grid["lat_bounds"],
                                        z_edges_m=grid["z_edges"], n_time_bins=grid["n_time_bins"],
                                        n_y=grid["n_y"], n_x=grid["n_x"], n_releases=len(rel), device=dev,
                                        dtype=torch.float64)
    cfg = SimpleNamespace(met_domain=SimpleNamespace(**domain))
    shim = _NoiseShim(ref, noise_seed, n, max_substeps)
    rshim = _RandShim(ref, noise_seed + 7) if convection else None
    p = torch.from_numpy(particles.T.copy()).to(dev)
    rel_t = torch.from_numpy(rel_off).to(dev)
    end_t = torch.from_numpy(win_end).to(dev)
    ridx_t = torch.from_numpy(ridx).to(dev)
    state = scheme.initialize_state(n, device=dev, dtype=torch.float32)
    alive = torch.ones(n, dtype=torch.bool, device=dev)
    windows: dict = {}
    last_bracket = None
    wind_cache: dict = {}
    esc, act, conv_log, snaps, diag_pos, diag_wind = [], [], [], [], [], []
    t_cursor = cursor_start
    step = 0
    bstart = batch_start.timestamp()
    host = lambda t: t.detach().cpu().numpy()  # noqa: E731
    try:
        while t_cursor > terminus:
            delta = min(dt_s, (t_cursor - terminus).total_seconds())
            cur = t_cursor.timestamp() - bstart
            active = (rel_t >= cur) & (rel_t - sim_length_s <= cur) & alive
            h = syn.window_index(ref.main._hour_floor(t_cursor))
            if h not in windows:
                windows[h] = _ref_window(ref, syn, h)
            win = windows[h]
            alpha, wind_mean = ref.main._advection_alpha_wind_mean(win, t_cursor, delta, dev, torch.float32,
                                                                   wind_cache)
            shim.begin_step(step)
            p, state = scheme.step(particles=p, state=state, met_window=win, t_alpha=alpha, dt_seconds=delta,
                                   active_mask=active, engine=engine)
            if win.metadata.time_start != last_bracket:
                if conv_scheme is not None:
                    rshim.begin(step)
                    before = p[:, 2].clone()
                    p, _ = conv_scheme.maybe_convect(particles=p, state={}, met_window=win, t_alpha=alpha,
                                                     dt_seconds=delta, active_mask=active, engine=engine)
                    conv_log.append((step, int((p[:, 2] != before).sum())))
                last_bracket = win.metadata.time_start
            el = (end_t - cur).clamp_(min=0.0)
            t_idx = (el / 3600.0).floor().to(torch.int64)
            if gridder.n_t == 1:
                t_idx.clamp_(max=0)
            gridder.accumulate(particles=p[:, :3], active_mask=active, weights=p[:, 3], t_idx=t_idx,
                               release_idx=ridx_t, dt_seconds=delta)
            gridder64.accumulate(particles=p[:, :3].double(), active_mask=active, weights=p[:, 3].double(),
                                 t_idx=t_idx, release_idx=ridx_t, dt_seconds=delta)
            newly = active & ~ref.main._within_met_domain(p, cfg)
            alive = alive & ~newly
            esc.append(int(newly.sum()))
            act.append(int(active.sum()))
            # the per-step diagnostics of main.py:1565-1566
            diag_pos.append(host(p[:, :3].mean(dim=0)).copy())
            diag_wind.append(host(wind_mean).copy())
            if step % snap_every == 0:
                snaps.append((step, host(p).T.copy()))
            t_cursor = t_cursor - timedelta(seconds=delta)
            step += 1
    finally:
        shim.restore()
        if rshim is not None:
            rshim.restore()

    out = dict(particles0=particles, rel_off=rel_off, win_end_off=win_end, release_idx=ridx,
               batch_start=np.array(batch_start.timestamp()), cursor_start=np.array(cursor_start.timestamp()),
               cursor_terminus=np.array(terminus.timestamp()), sim_length_s=np.array(sim_length_s),
               dt_s=np.array(dt_s), max_substeps=np.array(max_substeps), meander=np.array(meander),
               convection=np.array(convection), noise_seed=np.array(noise_seed), conv_seed=np.array(noise_seed + 7),
               grid_lon=np.array(grid["lon_bounds"]), grid_lat=np.array(grid["lat_bounds"]),
               grid_nxy=np.array([grid["n_x"], grid["n_y"], grid["n_time_bins"]]), grid_z=np.array(grid["z_edges"]),
               dom_lon=np.array(domain["lon_bounds"]), dom_lat=np.array(domain["lat_bounds"]),
               dom_alt=np.array(domain["alt_max_m"]),
               out_particles=host(p).T.copy(), out_alive=host(alive), out_footprint=host(gridder.tensor),
               out_footprint_f64=host(gridder64.tensor),
               out_escaped=np.array(esc), out_active=np.array(act), out_conv=np.array(conv_log).reshape(-1, 2),
               snap_steps=np.array([s for s, _ in snaps]), snap_particles=np.stack([a for _, a in snaps]),
               out_diag_pos=np.stack(diag_pos).astype(np.float32), out_diag_wind=np.stack(diag_wind).astype(np.float32),
               n_steps=np.array(step))
    for k, v in state.items():
        out[f"out_{k}"] = host(v)
    met = _met_arrays(syn)
    if case == "small":
        out.update(met)
    else:  # large met is regenerated from its seed; store a checksum of it instead
        out["met_checksum"] = np.array([float(np.sum(met[f"met_{k}"], dtype=np.float64))
                                        for k in ("u", "v", "w", "t", "q", "blh", "sp", "ustar", "shf")])
        out["met_seed"] = np.array(spec.seed)
        out["met_case"] = np.array(case)
    return out


# noise seed of each golden batch
NOISE_SEEDS = {"small": 4242, "c0": 777, "c1": 9001}
# snapshot interval (outer steps) of each golden batch
SNAP_EVERY = {"small": 20, "c0": 20, "c1": 60}


def make_run(ref, case: str, out_path: Path) -> None:
    out = drive_batch(ref, case, NOISE_SEEDS[case], snap_every=SNAP_EVERY[case])
    np.savez_compressed(out_path, **out)
    print("wrote", out_path, "steps", int(out["n_steps"]), "escaped", int(out["out_escaped"].sum()),
          "conv", out["out_conv"].tolist())


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", required=True, help="root of the reference source tree (holds src/lpdm)")
    ap.add_argument("--only", nargs="*", choices=["units", "small", "c0", "c1"],
                    help="fixtures to (re)generate (default: all)")
    args = ap.parse_args()
    ref = _import_reference(Path(args.reference))
    want = set(args.only or ["units", "small", "c0", "c1"])
    if "units" in want:
        make_units(ref, HERE / "units.npz")
    if "small" in want:
        make_run(ref, "small", HERE / "run_small.npz")
    if "c0" in want:
        make_run(ref, "c0", HERE / "run_c0.npz")
    if "c1" in want:
        make_run(ref, "c1", HERE / "run_c1.npz")


if __name__ == "__main__":
    main()
