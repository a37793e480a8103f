"""Loaders that turn the golden batch fixtures into runnable cases.

A case carries the met (from the fixture or regenerated from its seed), the
particle inputs, the run configuration, and the injected-noise generators of
``tests/golden/noise.py``.
"""

from __future__ import annotations

import sys
from dataclasses import dataclass
from datetime import UTC, datetime
from pathlib import Path

import numpy as np

GOLDEN = Path(__file__).resolve().parent / "golden"
if str(GOLDEN) not in sys.path:
    sys.path.insert(0, str(GOLDEN))

from noise import conv_uniforms, noise_block, step_noise  # noqa: E402,F401

from glide_b200.synthetic import SyntheticMet, SyntheticMetSpec, config_met_spec  # noqa: E402

FIELDS = ("u", "v", "w", "t", "q", "blh", "sp", "ustar", "shf")


@dataclass
class MetArrays:
    fields: dict  # name -> [S, Z, Y, X] or [S, Y, X] float32
    levels: np.ndarray
    p_hpa: np.ndarray
    lon: np.ndarray
    lat: np.ndarray
    t0: float

    @property
    def n_snapshots(self) -> int:
        return self.fields["u"].shape[0]

    def time(self, h: int) -> datetime:
        return datetime.fromtimestamp(self.t0 + 3600.0 * h, tz=UTC)

    def index(self, t: datetime) -> int:
        return int(round((t.timestamp() - self.t0) / 3600.0))

    def oracle_window(self, h: int) -> dict:
        f = self.fields
        w = {n: f[n][h:h + 2] for n in FIELDS}
        nz = f["u"].shape[1]
        w["height"] = np.broadcast_to(self.levels.astype(np.float32).reshape(-1, 1, 1),
                                      (nz,) + f["u"].shape[2:]).copy()
        w.update(level=self.levels, p_hpa=self.p_hpa, lon=self.lon, lat=self.lat,
                 time_start=self.time(h), time_end=self.time(h + 1))
        return w


def met_from_synthetic(syn: SyntheticMet) -> MetArrays:
    fields = {n: np.stack([fs[n].cpu().numpy() for fs in syn.fields]).astype(np.float32) for n in FIELDS}
    return MetArrays(fields, syn.levels, syn.pressure_level_hpa, syn.lon, syn.lat, syn.times[0].timestamp())


@dataclass
class GoldenRun:
    name: str
    z: dict
    met: MetArrays

    def __getitem__(self, k):
        return self.z[k]

    @property
    def n(self) -> int:
        return int(self.z["particles0"].shape[1])

    def dt_(self, key) -> datetime:
        return datetime.fromtimestamp(float(self.z[key]), tz=UTC)


def load_run(name: str) -> GoldenRun:
    z = dict(np.load(GOLDEN / f"{name}.npz"))
    if "met_u" in z:
        met = MetArrays({n: z[f"met_{n}"] for n in FIELDS}, z["met_levels"], z["met_p_hpa"], z["met_lon"],
                        z["met_lat"], float(z["met_t0"]))
    else:
        case = str(z["met_case"]) if "met_case" in z else "c0"
        spec = config_met_spec(1, n_snapshots=4) if case == "c1" else _c0_spec(int(z["met_seed"]))
        if spec.seed != int(z["met_seed"]):
            raise RuntimeError(f"{name}: met seed {int(z['met_seed'])} does not match the {case} spec")
        met = met_from_synthetic(SyntheticMet(spec))
        chk = np.array([float(np.sum(met.fields[k], dtype=np.float64)) for k in FIELDS])
        if not np.allclose(chk, z["met_checksum"], rtol=1e-6, atol=1e-3):
            raise RuntimeError(f"regenerated met of {name} does not match its checksum")
    return GoldenRun(name, z, met)


def _c0_spec(seed: int) -> SyntheticMetSpec:
    return SyntheticMetSpec(nz=40, ny=64, nx=64, lon0=0.0, lat0=40.0, n_snapshots=5, moist_fraction=0.0,
                            seed=seed, start_time=datetime(2026, 1, 14, 23, tzinfo=UTC))


def flipped_levels(run: GoldenRun) -> GoldenRun:
    """The same case with the met stored top-down (descending level order), as a
    pressure-level reader would deliver it."""
    m = run.met
    fields = {k: (v[:, ::-1].copy() if v.ndim == 4 else v) for k, v in m.fields.items()}
    met = MetArrays(fields, np.asarray(m.levels)[::-1].copy(), np.asarray(m.p_hpa)[::-1].copy(), m.lon, m.lat, m.t0)
    return GoldenRun(run.name + "_desc", run.z, met)


def oracle_kwargs(run: GoldenRun, dtype=np.float32, conv_dtype=None, hanna_kw: dict | None = None):
    """Keyword arguments of ``oracle.run_batch`` reproducing the golden batch."""
    from oracle.convection import EmanuelParams
    from oracle.hanna import HannaParams, StepNoise
    from oracle.runtime import DomainSpec, GridSpec

    z = run.z
    n = run.n
    ms = int(z["max_substeps"])
    seed = int(z["noise_seed"])
    cseed = int(z["conv_seed"])
    nxy = z["grid_nxy"]

    def noise_fn(step):
        sub, mea = step_noise(seed, step, ms, n)
        return StepNoise(sub, mea)

    n_rel = int(z["release_idx"].max()) + 1
    return dict(
        get_window=lambda hk: run.met.oracle_window(run.met.index(hk)),
        particles=z["particles0"], rel_off=z["rel_off"], win_end_off=z["win_end_off"], release_idx=z["release_idx"],
        batch_start=run.dt_("batch_start"), cursor_start=run.dt_("cursor_start"),
        cursor_terminus=run.dt_("cursor_terminus"), sim_length_s=float(z["sim_length_s"]), dt_seconds=float(z["dt_s"]),
        params=HannaParams(meander_enabled=bool(z["meander"]), max_substeps=ms, **(hanna_kw or {})),
        grid=GridSpec(tuple(z["grid_lon"]), tuple(z["grid_lat"]), int(nxy[0]), int(nxy[1]), tuple(z["grid_z"]),
                      int(nxy[2]), n_rel),
        domain=DomainSpec(tuple(z["dom_lon"]), tuple(z["dom_lat"]), float(z["dom_alt"])),
        noise_fn=noise_fn,
        emanuel=EmanuelParams() if bool(z["convection"]) else None,
        conv_uniforms_fn=lambda step: conv_uniforms(cseed, step, n),
        dtype=dtype, conv_dtype=conv_dtype,
    )
