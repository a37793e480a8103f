"""Precision sweep of the met storage type on the single-site EUROPE-box workload.

The CUDA path with the packed met stored float32, bf16 and fp16 (interpolation,
particle state and integration in float32; the convective column in FP64) is run
beside the numpy oracle run entirely in FP64 (``oracle.runtime.run_batch`` with
``dtype=np.float64``), all on the same met, the same injected noise and the same
convection uniforms, for N particles of the 100 m release over 24 h backward at
dt 30 s (meander and hourly convection on). For every N and storage type it
reports:

* the footprint's relative L1 against the FP64 oracle, in total and per time_ago
  bin, and the relative error of the peak cell;
* the same L1 minus the float32 run's (what the storage type costs beyond the
  float32-versus-FP64 floor);
* the RMS horizontal and vertical position drift after 1, 6 and 24 h;
* escaped-particle counts (GPU modes and oracle).

Noise and uniforms are drawn per (step, chunk of particles) from numpy PCG64
streams, so the oracle runs chunk by chunk in worker processes (particles are
independent given the met) and the GPU runs see the concatenated chunks. The met is
generated once on the device; the oracle workers read a host copy of it through
memory-mapped files.

    python tests/golden/precision_sweep.py --particles 2000 20000 200000
"""

from __future__ import annotations

import argparse
import json
import os
import sys
import tempfile
import time
from datetime import timedelta
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path.insert(0, str(ROOT))

DT_S = 30.0
SIM_LENGTH_S = 24 * 3600.0
MAX_SUBSTEPS = 6
CHUNK = 12_500  # particles per noise chunk (and per oracle task)
NOISE_SEED, CONV_SEED = 424242, 515151
FIELDS = ("u", "v", "w", "t", "q", "blh", "sp", "ustar", "shf")
MARKS = {"1h": 1 + 120, "6h": 1 + 6 * 120, "24h": 2880}


def chunk_edges(n: int) -> np.ndarray:
    return np.unique(np.concatenate([np.arange(0, n, CHUNK), [n]]))


def chunk_noise(step: int, c: int, m: int):
    rng = np.random.default_rng([NOISE_SEED, int(step), int(c)])
    return (rng.standard_normal((MAX_SUBSTEPS, 3, m), dtype=np.float32),
            rng.standard_normal((2, m), dtype=np.float32))


def chunk_uniforms(step: int, c: int, m: int):
    rng = np.random.default_rng([CONV_SEED, int(step), int(c)])
    return rng.random(m, dtype=np.float32), rng.random(m, dtype=np.float32)


def workload(n: int):
    """The single-site workload's release (bench.py's), first n particles."""
    from glide_b200.config import DomainSpec, EmanuelConfig, FootprintSpec, HannaConfig
    from glide_b200.synthetic import config_met_spec

    spec = config_met_spec(1, n_snapshots=26)
    release_time = spec.start_time + timedelta(hours=23)
    rel_end = release_time + timedelta(hours=1)
    rng = np.random.default_rng(20261204)
    particles = np.stack([np.full(n, -5.0), np.full(n, 52.0), np.full(n, 100.0), np.full(n, 1.0 / n)],
                         axis=1).astype(np.float32)
    return dict(spec=spec, particles=particles, rel_off=rng.uniform(0.0, 3600.0, n).astype(np.float32),
                win_end=np.full(n, 3600.0, dtype=np.float32), ridx=np.zeros(n, dtype=np.int32),
                batch_start=release_time, cursor_start=rel_end, terminus=rel_end - timedelta(seconds=SIM_LENGTH_S),
                hanna=HannaConfig(meander_enabled=True, max_substeps=MAX_SUBSTEPS), emanuel=EmanuelConfig(),
                footprint=FootprintSpec((-60.125, 40.125), (9.875, 80.125), 401, 281, (0.0, 100.0), 24, 1),
                domain=DomainSpec((-60.0, 40.0), (10.0, 80.0), 20000.0))


# ---------------------------------------------------------------------------
# the FP64 oracle, one chunk of particles per task
# ---------------------------------------------------------------------------

_MET: dict = {}


def _met_window(path: str, meta: dict, h: int) -> dict:
    if not _MET:
        _MET.update({k: np.load(os.path.join(path, f"{k}.npy"), mmap_mode="r") for k in FIELDS})
    from datetime import UTC, datetime

    w = {k: np.array(_MET[k][h:h + 2]) for k in FIELDS}
    nz = w["u"].shape[1]
    w["height"] = np.broadcast_to(np.asarray(meta["levels"], dtype=np.float32).reshape(-1, 1, 1),
                                  (nz,) + w["u"].shape[2:]).copy()
    t0 = datetime.fromtimestamp(meta["t0"], tz=UTC)
    w.update(level=np.asarray(meta["levels"]), p_hpa=np.asarray(meta["p_hpa"]), lon=np.asarray(meta["lon"]),
             lat=np.asarray(meta["lat"]), time_start=t0 + timedelta(hours=h), time_end=t0 + timedelta(hours=h + 1))
    return w


def _oracle_chunk(task):
    path, meta, n, c, lo, hi = task
    from datetime import UTC, datetime

    from oracle.convection import EmanuelParams
    from oracle.hanna import HannaParams, StepNoise
    from oracle.runtime import DomainSpec, GridSpec, run_batch

    cfg = workload(n)
    m = hi - lo
    t0 = datetime.fromtimestamp(meta["t0"], tz=UTC)
    t = time.perf_counter()
    res = run_batch(
        get_window=lambda hk: _met_window(path, meta, int(round((hk - t0).total_seconds() / 3600.0))),
        particles=cfg["particles"][lo:hi].T.copy(), rel_off=cfg["rel_off"][lo:hi], win_end_off=cfg["win_end"][lo:hi],
        release_idx=np.zeros(m, dtype=np.int64), batch_start=cfg["batch_start"], cursor_start=cfg["cursor_start"],
        cursor_terminus=cfg["terminus"], sim_length_s=SIM_LENGTH_S, dt_seconds=DT_S,
        params=HannaParams(meander_enabled=True, max_substeps=MAX_SUBSTEPS),
        grid=GridSpec((-60.125, 40.125), (9.875, 80.125), 401, 281, (0.0, 100.0), 24, 1),
        domain=DomainSpec((-60.0, 40.0), (10.0, 80.0), 20000.0),
        noise_fn=lambda k: StepNoise(*chunk_noise(k, c, m)), emanuel=EmanuelParams(),
        conv_uniforms_fn=lambda k: chunk_uniforms(k, c, m), dtype=np.float64, conv_dtype=np.float64,
        snapshot_steps=tuple(MARKS.values()))
    return (c, res.footprint, {k: res.snapshots[k][:3] for k in MARKS.values()}, int(sum(res.escaped_per_step)),
            time.perf_counter() - t)


def run_oracle(path: str, meta: dict, n: int, workers: int) -> dict:
    import multiprocessing as mp

    edges = chunk_edges(n)
    tasks = [(path, meta, n, c, int(edges[c]), int(edges[c + 1])) for c in range(len(edges) - 1)]
    with mp.get_context("spawn").Pool(min(workers, len(tasks))) as pool:
        parts = sorted(pool.map(_oracle_chunk, tasks, chunksize=1), key=lambda r: r[0])
    fp = sum(p[1] for p in parts)
    snaps = {k: np.concatenate([p[2][k] for p in parts], axis=1) for k in MARKS.values()}
    return {"footprint": fp, "snapshots": snaps, "escaped": sum(p[3] for p in parts),
            "cpu_s": sum(p[4] for p in parts)}


# ---------------------------------------------------------------------------
# the CUDA path, the three storage types in lockstep (one noise draw per window)
# ---------------------------------------------------------------------------


def run_gpu(syn, grid, n: int, modes: tuple) -> dict:
    import torch

    from glide_b200.runtime import BatchRunner, ParticleState
    from glide_b200.window import window_from_synthetic

    dev = torch.device("cuda", 0)
    cfg = workload(n)
    edges = chunk_edges(n)
    cache: dict = {}

    def noise_provider(steps):
        key = (steps[0], steps[-1])
        if cache.get("key") != key:
            sub = np.empty((len(steps), MAX_SUBSTEPS, 3, n), dtype=np.float32)
            mea = np.empty((len(steps), 2, n), dtype=np.float32)
            for i, k in enumerate(steps):
                for c in range(len(edges) - 1):
                    lo, hi = int(edges[c]), int(edges[c + 1])
                    sub[i, :, :, lo:hi], mea[i, :, lo:hi] = chunk_noise(k, c, hi - lo)
            cache.update(key=key, val=(torch.from_numpy(sub).to(dev), torch.from_numpy(mea).to(dev)))
        return cache["val"]

    def conv_provider(k):
        u = np.empty((2, n), dtype=np.float32)
        for c in range(len(edges) - 1):
            lo, hi = int(edges[c]), int(edges[c + 1])
            u[0, lo:hi], u[1, lo:hi] = chunk_uniforms(k, c, hi - lo)
        return torch.from_numpy(u).to(dev)

    runs = {}
    for mode in modes:
        r = BatchRunner(grid=grid, window_provider=lambda hk: window_from_synthetic(syn, syn.window_index(hk), grid),
                        hanna=cfg["hanna"], footprint=cfg["footprint"], domain=cfg["domain"], emanuel=cfg["emanuel"],
                        met_dtype=mode, device=dev, noise_provider=noise_provider, conv_uniform_provider=conv_provider,
                        pipeline=False)
        st = ParticleState.from_particles(cfg["particles"], cfg["rel_off"], cfg["win_end"], cfg["ridx"], dev)
        runs[mode] = r.start(st, batch_start=cfg["batch_start"], cursor_start=cfg["cursor_start"],
                             cursor_terminus=cfg["terminus"], sim_length_s=SIM_LENGTH_S, dt_seconds=DT_S)
    snaps = {m: {} for m in modes}
    first = runs[modes[0]]
    while not first.done:
        for mode, run in runs.items():
            run.step_window()
            done = run.windows[run.next_window - 1][1]
            if done in MARKS.values():
                s = run.state
                snaps[mode][done] = np.stack([s.lon.cpu().numpy(), s.lat.cpu().numpy(), s.z.cpu().numpy()])
    out = {}
    for mode, run in runs.items():
        o = run.finish()
        out[mode] = {"footprint": o.footprint.cpu().numpy().astype(np.float64), "snapshots": snaps[mode],
                     "escaped": int(o.escaped_per_step.sum()), "status": o.status}
    return out


def _metrics(res: dict, ora: dict) -> dict:
    fa, fb = res["footprint"], ora["footprint"]
    d = {"escaped": res["escaped"], "status": res.get("status", 0)}
    d["footprint_rel_l1"] = float(np.abs(fa - fb).sum() / np.abs(fb).sum())
    per_bin = []
    for t in range(fb.shape[1]):
        den = np.abs(fb[:, t]).sum()
        per_bin.append(float(np.abs(fa[:, t] - fb[:, t]).sum() / den) if den > 0 else None)
    d["footprint_rel_l1_per_time_ago_bin"] = per_bin
    d["footprint_peak_rel_err"] = float(abs(fa.max() - fb.max()) / fb.max())
    for name, k in MARKS.items():
        a, b = res["snapshots"][k], ora["snapshots"][k]
        dx = (a[0] - b[0]) * 111320.0 * np.cos(np.deg2rad(b[1]))
        dy = (a[1] - b[1]) * 110540.0
        d[f"rms_horizontal_m_{name}"] = float(np.sqrt(np.mean(dx * dx + dy * dy)))
        d[f"rms_vertical_m_{name}"] = float(np.sqrt(np.mean((a[2] - b[2]) ** 2)))
    return d


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--particles", type=int, nargs="*", default=[2000, 20000, 200000])
    ap.add_argument("--modes", nargs="*", default=["f32", "bf16", "f16"])
    ap.add_argument("--workers", type=int, default=0, help="oracle processes (default: by cores and free memory)")
    args = ap.parse_args()
    import psutil
    import torch

    from glide_b200.synthetic import SyntheticMet
    from glide_b200.window import grid_from_synthetic

    dev = torch.device("cuda", 0)
    cfg = workload(max(args.particles))
    syn = SyntheticMet(cfg["spec"], device=dev)
    grid = grid_from_synthetic(syn).to_device(dev)
    path = tempfile.mkdtemp(prefix="glide_met_")
    for k in FIELDS:  # one .npy per field, memory-mapped by the oracle workers
        np.save(os.path.join(path, f"{k}.npy"), np.stack([f[k].cpu().numpy() for f in syn.fields]))
    meta = {"levels": np.asarray(syn.levels).tolist(), "p_hpa": np.asarray(syn.pressure_level_hpa).tolist(),
            "lon": np.asarray(syn.lon).tolist(), "lat": np.asarray(syn.lat).tolist(),
            "t0": syn.times[0].timestamp()}
    workers = args.workers or max(1, min(os.cpu_count() or 1, int(psutil.virtual_memory().available / 4e9)))
    try:
        for n in args.particles:
            t = time.perf_counter()
            gpu = run_gpu(syn, grid, n, tuple(args.modes))
            t_gpu = time.perf_counter() - t
            t = time.perf_counter()
            ora = run_oracle(path, meta, n, workers)
            t_ora = time.perf_counter() - t
            line = {"workload": "precision", "particles": n, "hours": 24, "oracle": "FP64 numpy oracle",
                    "oracle_escaped": ora["escaped"], "oracle_wall_s": t_ora, "oracle_workers": workers,
                    "gpu_wall_s": t_gpu, "modes": {}}
            for mode in args.modes:
                line["modes"][mode] = _metrics(gpu[mode], ora)
            if "f32" in line["modes"]:
                floor = line["modes"]["f32"]["footprint_rel_l1"]
                for mode, d in line["modes"].items():
                    d["footprint_rel_l1_minus_f32"] = d["footprint_rel_l1"] - floor
            print(json.dumps(line), flush=True)
    finally:
        import shutil

        shutil.rmtree(path, ignore_errors=True)


if __name__ == "__main__":
    main()
