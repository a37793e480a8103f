"""The drop-in inside the reference's own runtime: ``lpdm.main._run`` (the reference's
whole cursor loop, release generation, met fetch and prefetch, footprint gridder,
escape kill, diagnostics and output writing) run twice on the same synthetic met
reader and configuration:

* ``stock`` — its own schemes, ``HannaScheme`` (``hanna_1982``, eager static path on
  CUDA) and ``EmanuelReducedConvection`` (``emanuel_reduced``);
* ``b200``  — this library's ``hanna_1982_b200`` and ``emanuel_reduced_b200``,
  registered in the reference's registries (``glide_b200.schemes.register_with_reference``)
  and built by the reference's ``get_scheme`` / ``get_convection_scheme``.

Both are fed the same injected turbulence noise and convection uniforms (numbered by
step and by convection call), so their outputs are comparable particle by particle.
The reference's ``OutputWriter`` is replaced by an in-memory writer (its Zarr and
Parquet backends are outside the hot path); everything else is the reference's code.

Prints a JSON report: per-step active and escaped counts equal, the fraction of
endpoint particles within 1e-5 / 1e-4 relative, the footprint's relative L1, and the
diagnostic rows' agreement. Needs a CUDA device and the reference installed as a
package directory (``pip install --no-deps --target <dir> <reference>``) or a source tree:

    python tests/golden/reference_runtime_dropin.py --reference baseline/_ref
"""

from __future__ import annotations

import argparse
import json
import sys
import time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent.parent))
sys.path.insert(0, str(HERE))

import make_golden  # noqa: E402
from noise import conv_uniforms, step_noise  # noqa: E402

NOISE_SEED, CONV_SEED = 31337, 31344
N_PARTICLES = 20_000
MAX_SUBSTEPS = 6


class MemoryWriter:
    """The reference's ``OutputWriter`` interface (src/lpdm/output_writer.py:50-243),
    keeping everything in memory."""

    def __init__(self) -> None:
        self.footprint = None
        self.particles = None
        self.rows = None
        self.metadata = {}

    def write_particles_parquet(self, path, particles, *, release_idx=None):
        self.particles = particles.detach().cpu().numpy().copy()

    def write_trajectory_parquet(self, path, step_seconds, rows):
        self.rows = [dict(r) for r in rows]

    def write_metadata_json(self, path, payload):
        self.metadata[path] = payload

    def create_footprint_store(self, path, *, shape, dims=None, coords=None, attrs=None):
        self.footprint = np.zeros(shape, dtype=np.float32)

    def write_footprint_region(self, path, footprint, *, release_start, release_stop, dims=None):
        self.footprint[release_start:release_stop] = footprint.detach().cpu().numpy()


def _reader(ref, syn):
    """A ``MetReader`` serving the synthetic met's hourly brackets as the reference's
    ``HourlyMetTensors`` on the host (as ``met_cache_on_host`` keeps them)."""

    class SyntheticReader(ref.mr.MetReader):
        def get_time_coverage(self):
            return syn.times[0], syn.times[-1]

        def fetch_hourly_window(self, request):
            return make_golden._ref_window(ref, syn, syn.window_index(request.time.start))

    return SyntheticReader()


def _config(ref, syn, output_uri: str, scheme: str, convection: str):
    t_rel = syn.times[2]  # release hour [2, 3]; the cursor walks back from hour 3 to hour 1
    return ref.cfg.RunConfig.model_validate({
        "io": {"zarr_store": "synthetic://europe-box", "output_uri": output_uri},
        "simulation": {"start_time": t_rel, "length_seconds": 7200, "dt_seconds": 30, "device": "cuda"},
        "release": {"kind": "point", "lon": -5.0, "lat": 52.0, "alt_agl_m": 100.0, "duration_seconds": 3600,
                    "n_particles": N_PARTICLES, "seed": 42},
        "turbulence": {"scheme": scheme, "max_substeps": MAX_SUBSTEPS, "meander": {"enabled": True}},
        "convection": {"scheme": convection},
        "output_grid": {"lon_bounds": (-60.125, 40.125), "lat_bounds": (9.875, 80.125), "n_x": 401, "n_y": 281,
                        "z_edges_m": (0.0, 100.0), "n_time_bins": 3},
        "met_domain": {"lon_bounds": (-60.0, 40.0), "lat_bounds": (10.0, 80.0), "alt_max_m": 20000.0},
        "memory": {"met_cache_max_hours": 2, "met_cache_on_host": True, "met_prefetch": True,
                   "log_every_steps": 0, "gc_every_steps": 0, "guard_check_every_steps": 1},
    })


def _run_stock(ref, syn):
    """``_run`` with the reference's own schemes (built from the config by its runtime's
    kwargs helpers), injected noise through ``GPUEngine.update_langevin_velocity``'s
    ``noise=`` argument and uniforms through ``torch.rand`` in ``emanuel``."""
    cfg = _config(ref, syn, "memory://stock", "hanna_1982", "emanuel_reduced")
    scheme = ref.hn.HannaScheme(static_substeps=True, **ref.main._scheme_kwargs(cfg))
    conv = ref.em.EmanuelReducedConvection(**ref.main._convection_scheme_kwargs(cfg))
    shim = make_golden._NoiseShim(ref, NOISE_SEED, N_PARTICLES, MAX_SUBSTEPS)
    rshim = make_golden._RandShim(ref, CONV_SEED)
    counter = {"step": 0, "conv": 0}
    step0, conv0 = scheme.step, conv.maybe_convect

    def step(*a, **kw):
        shim.begin_step(counter["step"])
        counter["step"] += 1
        return step0(*a, **kw)

    def maybe_convect(*a, **kw):
        rshim.begin(counter["conv"])
        counter["conv"] += 1
        return conv0(*a, **kw)

    scheme.step, conv.maybe_convect = step, maybe_convect
    try:
        ref.main._run(cfg, reader=_reader(ref, syn), scheme=scheme, convection_scheme=conv)
    finally:
        shim.restore()
        rshim.restore()
    return counter


def _run_b200(ref, syn):
    """``_run`` with this library's schemes, registered in the reference's registries and
    built there by name, fed the same noise and uniforms."""
    import torch

    import lpdm.convection.base as cb
    import lpdm.turbulence.base as tb

    from glide_b200.schemes import register_with_reference

    register_with_reference(tb, cb)
    dev = torch.device("cuda")

    def noise(step):
        sub, mea = step_noise(NOISE_SEED, step, MAX_SUBSTEPS, N_PARTICLES)
        return torch.from_numpy(sub).to(dev), torch.from_numpy(mea).to(dev)

    def uniforms(call):
        return torch.from_numpy(np.stack(conv_uniforms(CONV_SEED, call, N_PARTICLES))).to(dev)

    cfg = _config(ref, syn, "memory://b200", "hanna_1982_b200", "emanuel_reduced_b200")
    scheme = tb.get_scheme("hanna_1982_b200", meander_enabled=True, max_substeps=MAX_SUBSTEPS, noise_provider=noise)
    conv = cb.get_scheme("emanuel_reduced_b200", uniform_provider=uniforms)
    ref.main._run(cfg, reader=_reader(ref, syn), scheme=scheme, convection_scheme=conv)
    return {"step": scheme.step_count, "conv": conv.calls, "device_status": scheme.device_status}


def _scaled_err(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    scale = np.maximum(np.abs(b[:, :3]), np.array([[1.0, 1.0, 10.0]]))
    return (np.abs(a[:, :3] - b[:, :3]) / scale).max(axis=1)


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", required=True, help="reference package directory or source tree")
    args = ap.parse_args()
    import torch

    if not torch.cuda.is_available():
        raise SystemExit("needs a CUDA device")
    ref = make_golden._import_reference(Path(args.reference).resolve())
    import lpdm.config as lcfg

    ref.cfg = lcfg
    from glide_b200.synthetic import SyntheticMet, config_met_spec

    syn = SyntheticMet(config_met_spec(1, n_snapshots=5))
    writers, counters, walls = {}, {}, {}
    for name, fn in (("stock", _run_stock), ("b200", _run_b200)):
        w = MemoryWriter()
        ref.main.OutputWriter = lambda w=w: w
        t = time.perf_counter()
        counters[name] = fn(ref, syn)
        torch.cuda.synchronize()
        walls[name] = time.perf_counter() - t
        writers[name] = w
        print(f"{name}: _run done in {walls[name]:.1f} s", file=sys.stderr, flush=True)
    a, b = writers["b200"], writers["stock"]
    ra, rb = a.rows, b.rows
    err = _scaled_err(a.particles, b.particles)
    fa, fb = a.footprint.astype(np.float64), b.footprint.astype(np.float64)
    col = lambda rows, k: np.array([r[k] for r in rows], dtype=np.float64)  # noqa: E731
    pos = max(float(np.max(np.abs(col(ra, k) - col(rb, k)) / np.maximum(np.abs(col(rb, k)), 1.0)))
              for k in ("mean_lon", "mean_lat", "mean_alt_agl_m"))
    wind = max(float(np.max(np.abs(col(ra, k) - col(rb, k)))) for k in ("u_mean_m_s", "v_mean_m_s", "w_mean_m_s"))
    report = {
        "case": f"lpdm.main._run: point release of {N_PARTICLES} particles at (-5, 52) 100 m over 1 h, 2 h "
                "backward, dt 30 s, meander and emanuel_reduced on, 60x281x401 synthetic met, 3 time_ago bins",
        "steps": [len(ra), len(rb)],
        "scheme_calls": counters,
        "active_equal": bool(np.array_equal(col(ra, "active_particles"), col(rb, "active_particles"))),
        "escaped_equal": bool(np.array_equal(col(ra, "escaped_this_step"), col(rb, "escaped_this_step"))),
        "within_1e-5": float(np.mean(err < 1e-5)), "within_1e-4": float(np.mean(err < 1e-4)),
        "median_rel_err": float(np.median(err)), "max_rel_err": float(err.max()),
        "footprint_rel_l1": float(np.abs(fa - fb).sum() / max(np.abs(fb).sum(), 1e-300)),
        "footprint_total": [float(fa.sum()), float(fb.sum())],
        "diag_pos_max_rel": pos, "diag_wind_max_abs": wind,
        "wall_s": walls,
    }
    print(json.dumps(report), flush=True)


if __name__ == "__main__":
    main()
