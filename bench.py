"""Benchmark of the B200 particle-step engine on the single-site EUROPE-box workload.

Workload (one B200): one release at 100 m AGL of 200,000 particles over a 1 h
release window, integrated 24 h backward at dt = 30 s (2,880 outer steps) with
the Hanna scheme (max_substeps 6), meander on, Emanuel convection once per
met window, a 24 x 281 x 401 time_ago x lat x lon footprint (0-100 m layer),
on seeded synthetic met of 60 x 281 x 401 cells (0.25 deg, 26 hourly
snapshots, float32). A bench step is one met window: 120 outer steps of the
whole particle set, including the window's met packing and convection.

``value``: particle-steps/s (particles x outer steps / device time), met
resident in HBM. ``e2e``: the same job through the public runtime with the met
snapshots in pinned host memory: every step copies its new snapshot to the
device and reads back the window's diagnostics and footprint slice.

``--impl reference``: the reference algorithm's CPU implementation (the numpy
oracle port, all host cores, particle-parallel) on the same workload, timed on
a bounded sample per step.

Multi-GPU (torchrun): every rank runs its own release (replicas, weak scaling).
"""

from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import time
from datetime import UTC, datetime, timedelta
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

N_PARTICLES = 200_000
DT_S = 30.0
SIM_LENGTH_S = 24 * 3600.0
RELEASE_HEIGHT_M = 100.0
SITE = (-5.0, 52.0)
# algorithmic bytes per particle-step (met gathers 200 values x b + 86 B of state, footprint, flags)
B_ALG = {"f32": 200 * 4 + 86, "bf16": 200 * 2 + 86, "f16": 200 * 2 + 86}
METRIC = "particle-steps/s"
# From one ncu capture of the step kernel on this workload (float32 met, a window 7 h after
# the release, 200,000 particles x 120 steps; profiles/step_kernel_single_site_f32.md):
# DRAM bytes per launch and warp instructions issued per particle-step. The plume's met
# is served from L1, so the kernel is bound by instruction issue, not by HBM.
STEP_KERNEL_NCU = {"dram_bytes_per_launch": 10.998e6, "warp_inst_per_particle_step": 2.599e9 / 2.4e7,
                   "particle_steps_per_launch": 2.4e7}
SM_COUNT, SMSP_PER_SM = 148, 4
CPU_SAMPLE_STEPS = 40  # outer steps of all particles per step of the reference arm (~5 s on 16 cores)
CPU_BASELINE_STEPS = 120  # outer steps of all particles in the B200 arm's cpu_baseline sample (one met hour)
CPU_BASELINE_REPEATS = 3  # the hour stepped this many times (~15 s on 16 cores)


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference", "reference-gpu"],
                    help="reference: the reference algorithm on the host cores (oracle port); reference-gpu: "
                         "the reference's own torch.compile CUDA-graph step path installed in baseline/_ref")
    ap.add_argument("--met", default="f32", choices=["f32", "bf16", "f16"])
    ap.add_argument("--particles", type=int, default=N_PARTICLES)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-graph", action="store_true", help="skip the CUDA-graph replay of the whole job")
    ap.add_argument("--snapshots", type=int, default=26,
                    help="generate only the last N hourly snapshots (small profiling cases)")
    ap.add_argument("--workload", default="single-site",
                    choices=["single-site", "multisite", "serving", "regrid", "periodic"],
                    help="multisite: 56 sites x 48 hourly releases, 5 days backward, ring footprints; "
                         "serving: Poisson stream of footprint requests through FootprintServer")
    ap.add_argument("--requests", type=int, default=2000)
    ap.add_argument("--rate", type=float, default=5.0)
    ap.add_argument("--max-active", type=int, default=64)
    ap.add_argument("--no-sequential", action="store_true")
    ap.add_argument("--no-autotune", action="store_true", help="use launch variant 0 instead of tuning")
    ap.add_argument("--no-reorder", action="store_true", help="step particles in index order (no work-class sort)")
    ap.add_argument("--no-pipeline", action="store_true", help="prepare each window inline (no side stream)")
    ap.add_argument("--separate-convection", action="store_true",
                    help="convection in its own kernel between two step launches (not fused)")
    ap.add_argument("--steps-per-launch", type=int, default=None,
                    help="outer steps per step-kernel launch with --no-autotune (default: a whole window)")
    ap.add_argument("--sites", type=int, default=56)
    ap.add_argument("--release-times", type=int, default=48)
    ap.add_argument("--days", type=float, default=5.0)
    ap.add_argument("--periodic-releases", type=int, default=720,
                    help="periodic: hourly releases of 20,000 particles (the reference's example has 720)")
    ap.add_argument("--no-diagnostics", action="store_true",
                    help="skip the per-step mean-position / mean-wind diagnostics (BatchRunner.diagnostics)")
    ap.add_argument("--no-extras", action="store_true",
                    help="default workload: skip the extra jobs (reference GPU path, multisite, periodic)")
    ap.add_argument("--dense-footprints", action="store_true",
                    help="multisite: move completed slices to the host dense (default: as (cell, value) lists)")
    return ap.parse_args()


def workload(n_particles: int, rank: int = 0, n_snapshots: int = 26):
    import dataclasses

    from glide_b200.config import DomainSpec, EmanuelConfig, FootprintSpec, HannaConfig
    from glide_b200.synthetic import config_met_spec

    spec = config_met_spec(1, n_snapshots=26)
    t0 = spec.start_time
    if n_snapshots < 26:  # same hours at the end of the job, fewer generated before them
        spec = dataclasses.replace(spec, n_snapshots=n_snapshots, start_time=t0 + timedelta(hours=26 - n_snapshots))
    release_time = t0 + timedelta(hours=23)
    rel_end = release_time + timedelta(hours=1)
    rng = np.random.default_rng(20261204 + rank)
    lon, lat = SITE[0] + 2.0 * rank, SITE[1] - 1.0 * rank
    particles = np.stack([np.full(n_particles, lon), np.full(n_particles, lat), np.full(n_particles, RELEASE_HEIGHT_M),
                          np.full(n_particles, 1.0 / n_particles)], axis=1).astype(np.float32)
    rel_off = rng.uniform(0.0, 3600.0, n_particles).astype(np.float32)
    win_end = np.full(n_particles, 3600.0, dtype=np.float32)
    ridx = np.zeros(n_particles, dtype=np.int32)
    cfg = dict(
        spec=spec, particles=particles, rel_off=rel_off, win_end=win_end, ridx=ridx,
        batch_start=release_time, cursor_start=rel_end, terminus=rel_end - timedelta(seconds=SIM_LENGTH_S),
        hanna=HannaConfig(meander_enabled=True, max_substeps=6),
        emanuel=EmanuelConfig(),
        footprint=FootprintSpec((-60.125, 40.125), (9.875, 80.125), 401, 281, (0.0, 100.0), 24, 1),
        domain=DomainSpec((-60.0, 40.0), (10.0, 80.0), 20000.0),
    )
    return cfg


class ClockSampler:
    """nvidia-smi clock / throttle-reason sampling during the timed region (samples go to a
    CSV in the system temp directory, or in GLIDE_BENCH_CLOCKS_DIR when set)."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int) -> None:
        import tempfile

        self.gpu = gpu_index
        self.proc = None
        out = os.environ.get("GLIDE_BENCH_CLOCKS_DIR") or tempfile.gettempdir()
        self.path = Path(out) / f"glide_bench_clocks_gpu{gpu_index}_{os.getpid()}.csv"

    def __enter__(self):
        try:
            self.path.parent.mkdir(parents=True, exist_ok=True)
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                          "-i", str(self.gpu), "-lms", "20"], stdout=self.f,
                                         stderr=subprocess.DEVNULL)
            # nvidia-smi takes a moment to start: the timed region begins once it samples
            t_end = time.monotonic() + 3.0
            while time.monotonic() < t_end and self.proc.poll() is None:
                self.f.flush()
                if self.path.stat().st_size > 0:
                    break
                time.sleep(0.01)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            self.proc.wait(timeout=5)
            self.f.close()

    def summary(self) -> dict:
        if self.proc is None or not self.path.exists():
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.path.read_text().splitlines():
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_peak_hbm() -> tuple[float, str]:
    p = ROOT / "MEASURED_PEAKS.json"
    try:
        return float(json.loads(p.read_text())["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


# ---------------------------------------------------------------------------
# reference arm / CPU baseline: the oracle port, particle-parallel over processes
# ---------------------------------------------------------------------------


def prepare_cpu_sample(syn, cfg, n_particles: int) -> str:
    """Saves the met window and particles the CPU sample needs to an .npz in shared
    memory for the worker processes. The sample starts one outer step into the first
    hour after the release hour, when every particle is released and active, so each
    counted particle-step is computed; per-window work (support stacks, convection)
    is excluded from the CPU timing."""
    import tempfile

    h = syn.window_index(cfg["batch_start"] - timedelta(seconds=DT_S))
    f0, f1 = syn.fields[h], syn.fields[h + 1]
    arrs = {f"w_{k}": np.stack([f0[k].cpu().numpy(), f1[k].cpu().numpy()]) for k in f0}
    arrs.update(height=syn.height_agl.cpu().numpy(), level=syn.levels, p_hpa=syn.pressure_level_hpa, lon=syn.lon,
                lat=syn.lat, t_start=np.array(syn.times[h].timestamp()), t_end=np.array(syn.times[h + 1].timestamp()),
                particles=cfg["particles"][:n_particles], rel_off=cfg["rel_off"][:n_particles],
                win_end=cfg["win_end"][:n_particles],
                batch_start=np.array(cfg["batch_start"].timestamp()),
                cursor=np.array((cfg["batch_start"] - timedelta(seconds=DT_S)).timestamp()),
                terminus=np.array(cfg["terminus"].timestamp()))
    d = "/dev/shm" if os.path.isdir("/dev/shm") else None
    fd, path = tempfile.mkstemp(suffix=".npz", prefix="glide_cpu_", dir=d)
    os.close(fd)
    np.savez(path, **arrs)
    return path


_CPU_CACHE: dict = {}


def _cpu_chunk(args):
    path, lo, hi, n_steps, seed = args
    from oracle.convection import EmanuelParams
    from oracle.hanna import HannaParams, StepNoise
    from oracle.runtime import DomainSpec, GridSpec, run_batch

    z = np.load(path)
    ts = lambda v: datetime.fromtimestamp(float(v), tz=UTC)  # noqa: E731
    w = {k[2:]: z[k] for k in z.files if k.startswith("w_")}
    w.update(height=z["height"], level=z["level"], p_hpa=z["p_hpa"], lon=z["lon"], lat=z["lat"],
             time_start=ts(z["t_start"]), time_end=ts(z["t_end"]))
    n = hi - lo
    rng = np.random.default_rng(seed)

    def noise_fn(step):
        return StepNoise(rng.standard_normal((6, 3, n), dtype=np.float32), rng.standard_normal((2, n), dtype=np.float32))

    kw = {}
    cache = _CPU_CACHE.setdefault(path, {})
    if not cache:  # per-window support stacks, built once per process (not timed)
        from oracle.hanna import build_step_inputs

        cache.update(key=datetime.fromtimestamp(float(z["t_start"]), tz=UTC), win=w,
                     inp=build_step_inputs(w, HannaParams(meander_enabled=True, max_substeps=6), np.float32))
    t = time.perf_counter()
    run_batch(get_window=lambda hk: w, particles=z["particles"][lo:hi].T.copy(), rel_off=z["rel_off"][lo:hi],
              win_end_off=z["win_end"][lo:hi], release_idx=np.zeros(n, dtype=np.int64),
              batch_start=ts(z["batch_start"]), cursor_start=ts(z["cursor"]), cursor_terminus=ts(z["terminus"]),
              sim_length_s=SIM_LENGTH_S, dt_seconds=DT_S, params=HannaParams(meander_enabled=True, max_substeps=6),
              grid=GridSpec((-60.125, 40.125), (9.875, 80.125), 401, 281, (0.0, 100.0), 24, 1),
              domain=DomainSpec((-60.0, 40.0), (10.0, 80.0), 20000.0), noise_fn=noise_fn,
              emanuel=EmanuelParams(), conv_uniforms_fn=lambda s: (rng.random(n, dtype=np.float32),
                                                                   rng.random(n, dtype=np.float32)),
              max_steps=n_steps, inputs_cache=cache, convect_first=False, **kw)
    return time.perf_counter() - t


def cpu_oracle_rate(path: str, n_particles: int, n_steps: int, workers: int, repeats: int = 1) -> tuple[float, float]:
    """(particle-steps/s, seconds) of the oracle on ``workers`` spawned processes, each
    stepping its share of the particles; a repeat's time is its slowest worker's
    stepping time (the per-window support stacks are built once per process, untimed),
    and ``repeats`` runs of the same sample add up."""
    import multiprocessing as mp

    edges = np.linspace(0, n_particles, workers + 1).astype(int)
    tasks = [(path, int(edges[i]), int(edges[i + 1]), n_steps, 1000 + i) for i in range(workers)]
    ctx = mp.get_context("spawn")
    wall = 0.0
    with ctx.Pool(workers) as pool:
        pool.map(_cpu_chunk, [(path, 0, 64, 1, 7)] * (4 * workers), chunksize=1)  # imports + per-process stacks
        for _ in range(max(1, repeats)):
            wall += max(pool.map(_cpu_chunk, tasks, chunksize=1))
    return n_particles * n_steps * max(1, repeats) / wall, wall


def _cpu_met(cfg):
    import torch

    from glide_b200.synthetic import SyntheticMet

    return SyntheticMet(cfg["spec"], device="cuda" if torch.cuda.is_available() else "cpu")


def run_reference(args) -> None:
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    workers = os.cpu_count() or 1
    n_sample_steps = CPU_SAMPLE_STEPS
    cfg = workload(args.particles)
    path = prepare_cpu_sample(_cpu_met(cfg), cfg, args.particles)
    try:
        rates = []
        for _ in range(min(args.warmup, 1)):
            cpu_oracle_rate(path, args.particles, 1, workers)
        for _ in range(args.steps):
            rates.append(cpu_oracle_rate(path, args.particles, n_sample_steps, workers)[0])
    finally:
        os.unlink(path)
    value = float(statistics.median(rates))
    sample = f"{args.particles} particles x {n_sample_steps} outer steps per step, oracle port on {workers} processes"
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * args.particles * n_sample_steps / value,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "single-site 24 h backward, 200k particles, 60x281x401 met, dt 30 s"},
            "cpu_baseline": {"value": value, "unit": METRIC, "cores": workers, "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# B200 arm
# ---------------------------------------------------------------------------


def multisite_workload(args, rank: int = 0):
    """56 sites x 48 hourly 1 h releases, particle counts log-uniform in [2e3, 2e4]
    (~2e7 in all), heights U(10, 300) m, 5 days backward at dt = 30 s, a 120-bin
    time_ago footprint per release kept as two live slices (ring)."""
    import dataclasses

    from glide_b200.config import DomainSpec, EmanuelConfig, FootprintSpec, HannaConfig
    from glide_b200.synthetic import config_met_spec

    rng = np.random.default_rng(20261206 + rank)
    n_sites, n_times = args.sites, args.release_times
    length_s = args.days * 86400.0
    base = config_met_spec(1)
    t_rel0 = base.start_time + timedelta(hours=int(np.ceil(length_s / 3600.0)) + 1)
    n_snap = int(np.ceil(length_s / 3600.0)) + n_times + 3
    spec = dataclasses.replace(base, n_snapshots=n_snap, seed=20261206 + rank)
    sites = np.stack([rng.uniform(-50.0, 30.0, n_sites), rng.uniform(20.0, 70.0, n_sites)], axis=1)
    counts, heights, parts, rel_off, win_end, ridx = [], [], [], [], [], []
    r = 0
    for k in range(n_times - 1, -1, -1):  # latest releases first: they activate first walking backward
        for s_i in range(n_sites):
            n = int(np.exp(rng.uniform(np.log(2000.0), np.log(20000.0))))
            h = rng.uniform(10.0, 300.0)
            off = k * 3600.0
            parts.append(np.stack([np.full(n, sites[s_i, 0]), np.full(n, sites[s_i, 1]), np.full(n, h),
                                   np.full(n, 1.0 / n)], axis=1))
            rel_off.append(off + rng.uniform(0.0, 3600.0, n))
            win_end.append(np.full(n, off + 3600.0))
            ridx.append(np.full(n, r))
            counts.append(n)
            r += 1
    cfg = dict(
        spec=spec, particles=np.concatenate(parts).astype(np.float32),
        rel_off=np.concatenate(rel_off).astype(np.float32), win_end=np.concatenate(win_end).astype(np.float32),
        ridx=np.concatenate(ridx).astype(np.int32), counts=np.array(counts), n_releases=r,
        batch_start=t_rel0, cursor_start=t_rel0 + timedelta(hours=n_times),
        terminus=t_rel0 + timedelta(hours=1) - timedelta(seconds=length_s), length_s=length_s,
        hanna=HannaConfig(meander_enabled=True, max_substeps=6), emanuel=EmanuelConfig(),
        footprint=FootprintSpec((-60.125, 40.125), (9.875, 80.125), 401, 281, (0.0, 100.0),
                                int(np.ceil(length_s / 3600.0)), r, ring=2),
        domain=DomainSpec((-60.0, 40.0), (10.0, 80.0), 20000.0),
    )
    return cfg


def run_multisite(args, emit: bool = True) -> dict:
    """The batched multi-release job: every release in one particle batch, one fused
    launch per met window, completed time_ago slices streamed to pinned host memory
    (compacted to (cell, value) lists on the device unless --dense-footprints)."""
    import torch

    from glide_b200.runtime import BatchRunner, ParticleState
    from glide_b200.synthetic import SyntheticMet
    from glide_b200.window import grid_from_synthetic, window_from_synthetic

    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    cfg = multisite_workload(args)
    syn = SyntheticMet(cfg["spec"], device=dev)
    grid = grid_from_synthetic(syn).to_device(dev)
    from glide_b200.runtime import HostSliceStream
    from glide_b200.sparse import SparseSliceStream

    stream = torch.cuda.current_stream()
    fp = cfg["footprint"]
    totals = torch.zeros(fp.n_releases, fp.n_time_bins, dtype=torch.float64, device=dev)
    slice_shape = (len(fp.z_edges) - 1, fp.n_y, fp.n_x)
    host_total = [0.0]
    # completed slices go to pinned host memory on a copy stream (a writer would take them from on_host):
    # as (cell, value) lists compacted on the device, or dense
    if args.dense_footprints:
        to_host = HostSliceStream(dev, slice_shape, capacity=fp.n_releases)

        def sink(r_idx, b_idx, slices):
            k = slices.shape[0]
            totals.view(-1).index_add_(0, r_idx * fp.n_time_bins + b_idx,
                                       slices.view(k, -1).sum(dim=1, dtype=torch.float64))
            to_host(r_idx, b_idx, slices)
    else:
        def on_host(r_idx, b_idx, off, cell, value):
            host_total[0] += float(value.sum(dtype=np.float64))  # the host's view of what arrived

        to_host = SparseSliceStream(dev, slice_shape, on_host=on_host, capacity=fp.n_releases)

        class SparseSink:
            def from_rows(self, rows, flat, r_idx, b_idx):
                totals.view(-1).index_add_(0, r_idx * fp.n_time_bins + b_idx,
                                           rows.index_select(0, flat).sum(dim=1, dtype=torch.float64))
                to_host.from_rows(rows, flat, r_idx, b_idx)

        sink = SparseSink()

    runner = BatchRunner(grid=grid, window_provider=lambda hk: window_from_synthetic(syn, syn.window_index(hk), grid),
                         hanna=cfg["hanna"], footprint=fp, domain=cfg["domain"], emanuel=cfg["emanuel"],
                         met_dtype=args.met, device=dev, seed=77, footprint_sink=sink)
    state = ParticleState.from_particles(cfg["particles"], cfg["rel_off"], cfg["win_end"], cfg["ridx"], dev)
    run = runner.start(state, batch_start=cfg["batch_start"], cursor_start=cfg["cursor_start"],
                       cursor_terminus=cfg["terminus"], sim_length_s=cfg["length_s"], dt_seconds=DT_S)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    t_wall = time.perf_counter()
    with ClockSampler(0) as clocks:
        e0.record(stream)
        run.run()
        to_host.drain()
        stream.wait_stream(to_host.copy_stream)  # the last slices are on the host inside the timed region
        e1.record(stream)
        torch.cuda.synchronize()
    wall = time.perf_counter() - t_wall
    t = e0.elapsed_time(e1) / 1e3
    act = run.act[: len(run.steps)].cpu().numpy().astype(np.int64)
    active_ps = int(act.sum())
    n_total = int(cfg["particles"].shape[0])
    line = {"metric": "active particle-steps/s", "value": active_ps / t, "unit": "particle-steps/s",
            "footprints_per_s": cfg["n_releases"] / t, "n_gpus": 1, "workload": "multisite",
            "releases": cfg["n_releases"], "particles": n_total, "outer_steps": len(run.steps),
            "windows": len(run.windows), "active_particle_steps": active_ps,
            "buffer_particle_steps_per_s": n_total * len(run.steps) / t, "device_s": t, "wall_s": wall,
            "dtype": args.met, "footprint_form": "dense" if args.dense_footprints else "sparse",
            "footprint_d2h_bytes": to_host.bytes_moved, "status": int(run.status.item()),
            "footprint_total": float(totals.sum().item()), "clocks": clocks.summary()}
    if not args.dense_footprints:
        line.update({"footprint_dense_bytes": to_host.dense_bytes, "footprint_entries": to_host.entries,
                     "footprint_total_host": host_total[0], "short_copies": to_host.short_copies})
    if emit:
        print(json.dumps(line), flush=True)
    return line


PERIODIC_SITE = (-9.9046, 53.3267)  # Mace Head, the reference's periodic example
PERIODIC_MET_PERIOD_H = 168


def periodic_workload(args, rank: int = 0):
    """The reference's periodic single-site job (configs/example_mhd_january_periodic.yaml):
    720 hourly 1 h releases of 20,000 particles at 10 m AGL at one site, each integrated
    5 days backward at dt = 60 s with meander and Emanuel convection, a time-integrated
    footprint (n_time_bins 1) in three layers (0-40 m, 40 m-1 km, 1-5 km) on the
    EUROPE-box grid. The synthetic met (60 x 281 x 401) has 169 hourly snapshots; the
    job's 840 hours use them cyclically (hour h reads window h mod 168)."""
    import dataclasses

    from glide_b200.config import DomainSpec, EmanuelConfig, FootprintSpec, HannaConfig
    from glide_b200.synthetic import config_met_spec

    rng = np.random.default_rng(20261207 + rank)
    n_rel, per = args.periodic_releases, 20_000
    length_s = 5 * 86400.0
    base = config_met_spec(1)
    spec = dataclasses.replace(base, n_snapshots=PERIODIC_MET_PERIOD_H + 1, seed=20261207 + rank)
    t_rel0 = base.start_time + timedelta(hours=121)
    n = n_rel * per
    parts = np.empty((n, 4), dtype=np.float32)
    parts[:, 0], parts[:, 1], parts[:, 2], parts[:, 3] = PERIODIC_SITE[0], PERIODIC_SITE[1], 10.0, 1.0 / per
    k = np.repeat(np.arange(n_rel - 1, -1, -1), per)  # latest releases first: they activate first walking backward
    rel_off = (k * 3600.0 + rng.uniform(0.0, 3600.0, n)).astype(np.float32)
    cfg = dict(
        spec=spec, particles=parts, rel_off=rel_off, win_end=(k * 3600.0 + 3600.0).astype(np.float32),
        ridx=k.astype(np.int32), n_releases=n_rel, per_release=per,
        batch_start=t_rel0, cursor_start=t_rel0 + timedelta(hours=n_rel),
        terminus=t_rel0 + timedelta(hours=1) - timedelta(seconds=length_s), length_s=length_s, dt_s=60.0,
        hanna=HannaConfig(meander_enabled=True, max_substeps=6), emanuel=EmanuelConfig(),
        footprint=FootprintSpec((-60.125, 40.125), (9.875, 80.125), 401, 281, (0.0, 40.0, 1000.0, 5000.0), 1, n_rel),
        domain=DomainSpec((-60.0, 40.0), (10.0, 80.0), 15000.0),
    )
    return cfg


def _cyclic_index(syn):
    def index_of(hour):
        return syn.window_index(hour) % PERIODIC_MET_PERIOD_H

    return index_of


def _cyclic_provider(syn, grid):
    """Window provider of the periodic job: window h of the synthetic met (h = the hour's
    index mod the period) stamped with the requested hour."""
    from glide_b200.window import Snapshot, WindowFields

    lowest = int(np.argmin(syn.levels))
    index_of = _cyclic_index(syn)

    def provider(hour):
        h = index_of(hour)
        snaps = []
        for kk, t in ((h, hour), (h + 1, hour + timedelta(hours=1))):
            f = dict(syn.fields[kk])
            f["t_lowest"] = f["t"][lowest]
            snaps.append(Snapshot(t, f))
        return WindowFields(snaps[0], snaps[1], grid, None)

    return provider


def run_periodic(args, emit: bool = True, with_reference: bool = True) -> dict:
    """The 720-release, 5-day job in one batch (one fused launch per met window, bf16
    met by default), timed whole with CUDA events: footprints/s and active
    particle-steps/s. Beside it, the reference's CUDA-graph path on one of the batches
    its runtime would run (24 releases, one calendar day: 480,000 particles), timed on 240
    steps once all of them are released."""
    import torch

    from glide_b200.runtime import BatchRunner, ParticleState
    from glide_b200.synthetic import SyntheticMet
    from glide_b200.window import grid_from_synthetic

    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    cfg = periodic_workload(args)
    t_gen = time.perf_counter()
    syn = SyntheticMet(cfg["spec"], device=dev)
    t_gen = time.perf_counter() - t_gen
    grid = grid_from_synthetic(syn).to_device(dev)
    met = args.met if args.met != "f32" else "bf16"
    runner = BatchRunner(grid=grid, window_provider=_cyclic_provider(syn, grid), hanna=cfg["hanna"],
                         footprint=cfg["footprint"], domain=cfg["domain"], emanuel=cfg["emanuel"], met_dtype=met,
                         device=dev, seed=91)
    state = ParticleState.from_particles(cfg["particles"], cfg["rel_off"], cfg["win_end"], cfg["ridx"], dev)
    run = runner.start(state, batch_start=cfg["batch_start"], cursor_start=cfg["cursor_start"],
                       cursor_terminus=cfg["terminus"], sim_length_s=cfg["length_s"], dt_seconds=cfg["dt_s"])
    stream = torch.cuda.current_stream()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    t_wall = time.perf_counter()
    with ClockSampler(0) as clocks:
        e0.record(stream)
        out = run.run()
        e1.record(stream)
        torch.cuda.synchronize()
    wall = time.perf_counter() - t_wall
    t = e0.elapsed_time(e1) / 1e3
    act = out.active_per_step.astype(np.int64)
    active_ps = int(act.sum())
    fp_total = float(out.footprint.sum(dtype=torch.float64).item())
    line = {"workload": "periodic", "metric": "footprints/s", "value": cfg["n_releases"] / t, "unit": "footprints/s",
            "active_particle_steps_per_s": active_ps / t, "releases": cfg["n_releases"],
            "particles": int(cfg["particles"].shape[0]), "outer_steps": out.n_steps, "windows": len(run.windows),
            "active_particle_steps": active_ps, "device_s": t, "wall_s": wall, "met_generation_s": t_gen,
            "met": met, "dt_s": cfg["dt_s"], "status": out.status, "escaped": int(out.escaped_per_step.sum()),
            "footprint_total": fp_total, "clocks": clocks.summary(),
            "config": "720 hourly releases x 20,000 particles at (-9.9046, 53.3267) 10 m, 5 days backward, dt 60 s, "
                      "meander + convection, time-integrated 3-layer footprint, 60x281x401 synthetic met "
                      f"({PERIODIC_MET_PERIOD_H + 1} snapshots used cyclically)"}
    del out, run, state, runner
    torch.cuda.empty_cache()
    if with_reference and _reference_modules() is not None:
        day = 24
        sel = cfg["ridx"] < day  # the first calendar day's releases: one batch of the reference's runtime
        rcfg = dict(cfg, particles=cfg["particles"][sel], rel_off=cfg["rel_off"][sel], win_end=cfg["win_end"][sel],
                    ridx=cfg["ridx"][sel])
        res = reference_cuda_graph_rate(rcfg, _reference_window_fn(syn, _cyclic_index(syn)),
                                        cursor_start=cfg["batch_start"], n_warm=130, n_time=240, dt_s=cfg["dt_s"],
                                        sim_length_s=cfg["length_s"])
        res["slice"] = ("one day's batch (24 releases x 20,000 particles, all released), 240 steps from the "
                        "batch's first release hour backward after 130 untimed; f32 met (the reference's)")
        line["reference_gpu"] = res
        if "value" in res:
            line["vs_reference_gpu"] = line["active_particle_steps_per_s"] / res["value"]
    if emit:
        print(json.dumps(line), flush=True)
    return line


def run_regrid(args) -> None:
    """One met hour regridded from 37 pressure levels onto 60 AGL levels over the
    EUROPE box (281 x 401), 9 channels with slope-corrected w and the per-level
    pressure: ``glide_agl_regrid`` with the inputs in HBM (CUDA events, median of
    ``--steps``), beside the reference's own ``lpdm.vertical_grid`` functions on the
    host as ``MetReader._resample_hour_to_agl`` calls them (from the installed
    reference in baseline/_ref, when present)."""
    import torch

    from glide_b200.regrid import regrid_hour_to_agl
    from glide_b200.synthetic import stretched_agl_levels

    dev = torch.device("cuda", 0)
    rng = np.random.default_rng(20261209)
    zp, ny, nx, nc = 37, 281, 401, 9
    names = ["u", "v", "w", "t", "q", "blh", "sp", "ustar", "shf"]
    lat, lon = np.linspace(10.0, 80.0, ny), np.linspace(-60.0, 40.0, nx)
    terrain = np.clip(rng.normal(400.0, 400.0, (ny, nx)), 0.0, 3000.0)
    msl = np.sort(np.concatenate([[100.0], rng.uniform(200.0, 20000.0, zp - 1)]))[::-1]  # top-of-atmosphere first
    h_agl = (msl[:, None, None] + rng.normal(0.0, 20.0, (zp, ny, nx)) - terrain[None]).astype(np.float32)
    fields = rng.normal(0.0, 5.0, (nc, zp, ny, nx)).astype(np.float32)
    p_hpa = 1013.25 * np.exp(-(h_agl.astype(np.float64) + terrain[None]) / 8000.0)
    z_sfc = (terrain * 9.80665).astype(np.float32)
    agl = stretched_agl_levels(60, 20000.0, 10.0)
    f_dev = torch.from_numpy(fields).to(dev)
    h_dev = torch.from_numpy(h_agl).to(dev)
    p_dev = torch.from_numpy(p_hpa).to(dev)
    kw = dict(z_sfc=z_sfc, lat=lat, lon=lon, pressure_p_hpa=p_dev, device=dev)
    for _ in range(max(args.warmup, 1)):
        regrid_hour_to_agl(f_dev, h_dev, agl, names, **kw)
    times = []
    for _ in range(args.steps):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        regrid_hour_to_agl(f_dev, h_dev, agl, names, **kw)
        e1.record()
        torch.cuda.synchronize()
        times.append(e0.elapsed_time(e1) / 1e3)
    gpu_s = float(np.median(times))
    line = {"metric": "regrid s per met hour", "value": gpu_s, "unit": "s", "higher_is_better": False,
            "workload": "regrid", "shape": {"channels": nc, "pressure_levels": zp, "agl_levels": int(agl.size),
                                            "ny": ny, "nx": nx},
            "note": "device time incl. the host terrain gradient and the pressure-level readback"}
    ref = ROOT / "baseline" / "_ref"
    if ref.is_dir():
        sys.path.insert(0, str(ref))
        try:
            from lpdm.vertical_grid import (apply_agl_regrid, compute_agl_regrid_weights, slope_correct_w,
                                            terrain_gradient)

            t = time.perf_counter()
            w = compute_agl_regrid_weights(h_agl, agl)
            arr = apply_agl_regrid(fields, w)
            dhdx, dhdy = terrain_gradient(z_sfc / 9.80665, lat, lon)
            arr[2] = slope_correct_w(arr[2], arr[0], arr[1], dhdx, dhdy, agl, float(agl[-1]))
            apply_agl_regrid(np.ascontiguousarray(p_hpa)[None], w)[0].mean(axis=(1, 2))
            cpu_s = time.perf_counter() - t
            line["reference_cpu"] = {"value": cpu_s, "unit": "s", "cores": torch.get_num_threads(),
                                     "kind": "reference", "sample": "the same hour through lpdm.vertical_grid"}
        except Exception as exc:  # the reference install is optional here
            line["reference_cpu"] = {"unavailable": f"{type(exc).__name__}: {exc}"}
    print(json.dumps(line), flush=True)


def run_serving(args) -> None:
    """Poisson stream (default 5 requests/s, 2,000 requests) of footprint requests:
    site among 56, release time uniform in 48 h, particles log-uniform in
    [1e3, 5e4], backward duration uniform in [6, 120] h, dt 30 s, BF16 met with all
    169 windows resident; 60 GB budget for particle state and footprints. Reports
    throughput and p50/p90/p99 end-to-end latency; then the capacity with the same
    requests submitted at once, and the same requests run one at a time (no overlap)
    for comparison."""
    import dataclasses

    import torch

    from glide_b200.runtime import DomainSpec, EmanuelConfig, FootprintSpec, HannaConfig
    from glide_b200.serving import FootprintServer, poisson_requests
    from glide_b200.synthetic import SyntheticMet, config_met_spec
    from glide_b200.window import grid_from_synthetic, window_from_synthetic

    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    base = config_met_spec(1)
    spec = dataclasses.replace(base, n_snapshots=171, seed=20261207)
    syn = SyntheticMet(spec, device=dev)
    grid = grid_from_synthetic(syn).to_device(dev)
    t_rel0 = syn.times[0] + timedelta(hours=121)
    rng = np.random.default_rng(20261207)
    sites = np.stack([rng.uniform(-50.0, 30.0, 56), rng.uniform(20.0, 70.0, 56)], axis=1)
    reqs = poisson_requests(args.requests, args.rate, sites, t_rel0, 48.0, seed=20261207)
    kw = dict(grid=grid, met_provider=lambda hk: window_from_synthetic(syn, syn.window_index(hk), grid),
              horizon_start=syn.times[0], horizon_end=syn.times[-1],
              hanna=HannaConfig(meander_enabled=True, max_substeps=6), emanuel=EmanuelConfig(),
              footprint=FootprintSpec((-60.125, 40.125), (9.875, 80.125), 401, 281, (0.0, 100.0), 1),
              domain=DomainSpec((-60.0, 40.0), (10.0, 80.0), 20000.0), met_dtype=args.met if args.met != "f32"
              else "bf16", device=dev, hbm_budget_bytes=60e9)
    t_pack = time.perf_counter()
    server = FootprintServer(max_active=args.max_active, n_streams=16, **kw)
    t_pack = time.perf_counter() - t_pack
    with ClockSampler(0) as clocks:
        t = time.perf_counter()
        res = server.serve(reqs, realtime=True)
        wall = time.perf_counter() - t
    lat = np.array([r.latency_s for r in res])
    aps = sum(r.active_particle_steps for r in res)
    line = {"metric": "footprints/s", "value": len(res) / wall, "unit": "footprints/s", "workload": "serving",
            "requests": len(res), "rate_per_s": args.rate, "wall_s": wall,
            "latency_s": {"p50": float(np.percentile(lat, 50)), "p90": float(np.percentile(lat, 90)),
                          "p99": float(np.percentile(lat, 99)), "max": float(lat.max())},
            "active_particle_steps_per_s": aps / wall, "peak_active": server.stats.peak_active,
            "peak_state_bytes": server.stats.peak_bytes, "resident_packed_bytes": server.resident.nbytes,
            "pack_s": t_pack, "dtype": kw["met_dtype"], "clocks": clocks.summary()}
    # capacity: the same requests all submitted at once
    sat = FootprintServer(max_active=args.max_active, n_streams=16, **kw)
    t = time.perf_counter()
    sat_res = sat.serve([dataclasses.replace(r) for r in reqs], realtime=False)
    sat_wall = time.perf_counter() - t
    line["saturated"] = {"footprints_per_s": len(sat_res) / sat_wall, "wall_s": sat_wall,
                         "active_particle_steps_per_s": sum(r.active_particle_steps for r in sat_res) / sat_wall,
                         "peak_active": sat.stats.peak_active}
    if not args.no_sequential:
        seq = FootprintServer(max_active=1, n_streams=1, **kw)
        t = time.perf_counter()
        sres = seq.serve([dataclasses.replace(r) for r in reqs], realtime=False)
        swall = time.perf_counter() - t
        service = np.array([r.finished_s - r.admitted_s for r in sres])
        line["one_at_a_time"] = {"footprints_per_s": len(sres) / swall, "wall_s": swall,
                                 "service_s_p50": float(np.percentile(service, 50)),
                                 "service_s_p99": float(np.percentile(service, 99)),
                                 "active_particle_steps_per_s": sum(r.active_particle_steps for r in sres) / swall}
    print(json.dumps(line), flush=True)


_REF_MODULES = None


def _reference_modules():
    """The reference's modules from the pip-installed copy in baseline/_ref (its hot path
    imports xarray only for annotations; a two-class stand-in module is supplied), or
    None when it is not installed."""
    global _REF_MODULES
    if _REF_MODULES is not None:
        return _REF_MODULES
    import tempfile
    from types import SimpleNamespace

    ref = ROOT / "baseline" / "_ref"
    if not (ref / "lpdm").is_dir():
        return None
    stub = Path(tempfile.mkdtemp(prefix="glide_xr_"))
    (stub / "xarray").mkdir()
    (stub / "xarray" / "__init__.py").write_text("class Dataset:\n    pass\n\n\nclass DataArray:\n    pass\n")
    sys.path.insert(0, str(ref))
    sys.path.insert(0, str(stub))
    import lpdm.convection.emanuel as em
    import lpdm.footprint_gridder as fg
    import lpdm.gpu_engine as ge
    import lpdm.main as lm
    import lpdm.met_reader as mr
    import lpdm.turbulence.hanna as hn

    _REF_MODULES = SimpleNamespace(em=em, fg=fg, ge=ge, lm=lm, mr=mr, hn=hn)
    return _REF_MODULES


def reference_cuda_graph_rate(cfg, window_fn, *, cursor_start, n_warm: int, n_time: int, dt_s: float,
                              sim_length_s: float) -> dict:
    """The reference's own GPU path on a workload: its HannaScheme static step core compiled
    with torch.compile(mode="reduce-overhead") (the CUDA-graph path of GLIDE_COMPILE=1),
    its Emanuel convection once per window, FootprintGridder and the escape kill, driven
    step by step as its cursor loop does (main.py:1382-1477) with its own RNG, on all of
    ``cfg``'s particles from ``cursor_start``. ``window_fn(hour)`` gives the reference's
    ``HourlyMetTensors`` (host tensors) of the window starting at ``hour``. Times ``n_time``
    steps after ``n_warm`` (the compile, the first window) with CUDA events; the value is
    active particle-steps per second."""
    import torch

    ref = _reference_modules()
    if ref is None:
        return {"unavailable": "reference not installed in baseline/_ref"}
    dev = torch.device("cuda")
    n = int(cfg["particles"].shape[0])
    hc = cfg["hanna"]
    scheme = ref.hn.HannaScheme(meander_enabled=hc.meander_enabled, max_substeps=hc.max_substeps)
    conv = ref.em.EmanuelReducedConvection() if cfg.get("emanuel") is not None else None
    engine = ref.ge.GPUEngine(device="cuda", compile_hot_paths=True)
    fp = cfg["footprint"]
    gridder = ref.fg.FootprintGridder(lon_bounds=fp.lon_bounds, lat_bounds=fp.lat_bounds, z_edges_m=fp.z_edges,
                                      n_time_bins=fp.n_time_bins, n_y=fp.n_y, n_x=fp.n_x,
                                      n_releases=int(cfg["ridx"].max()) + 1, device=dev)
    dom = cfg["domain"]
    from types import SimpleNamespace

    mcfg = SimpleNamespace(met_domain=SimpleNamespace(lon_bounds=dom.lon_bounds, lat_bounds=dom.lat_bounds,
                                                      alt_max_m=dom.alt_max_m))
    p = torch.as_tensor(cfg["particles"], device=dev)
    rel = torch.as_tensor(cfg["rel_off"], device=dev)
    wend = torch.as_tensor(cfg["win_end"], device=dev)
    ridx = torch.as_tensor(cfg["ridx"], device=dev).to(torch.int64)
    state = scheme.initialize_state(n, device=dev, dtype=torch.float32)
    alive = torch.ones(n, dtype=torch.bool, device=dev)
    t_cursor, term = cursor_start, cfg["terminus"]
    bstart = cfg["batch_start"].timestamp()
    windows: dict = {}
    last = None
    wcache: dict = {}
    active_steps = torch.zeros((), dtype=torch.int64, device=dev)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    t_wall = time.perf_counter()
    for k in range(n_warm + n_time):
        if k == n_warm:
            torch.cuda.synchronize()
            active_steps.zero_()
            e0.record()
        delta = min(dt_s, (t_cursor - term).total_seconds())
        cur = t_cursor.timestamp() - bstart
        active = (rel >= cur) & (rel - sim_length_s <= cur) & alive
        hour = ref.lm._hour_floor(t_cursor)
        if hour not in windows:
            windows.clear()
            windows[hour] = window_fn(hour)
        win = windows[hour]
        alpha, _ = ref.lm._advection_alpha_wind_mean(win, t_cursor, delta, dev, torch.float32, wcache)
        p, state = scheme.step(particles=p, state=state, met_window=win, t_alpha=alpha, dt_seconds=delta,
                               active_mask=active, engine=engine)
        if win.metadata.time_start != last:
            if conv is not None:
                p, _ = conv.maybe_convect(particles=p, state={}, met_window=win, t_alpha=alpha, dt_seconds=delta,
                                          active_mask=active, engine=engine)
            last = win.metadata.time_start
        t_idx = ((wend - cur).clamp_(min=0.0) / 3600.0).floor().to(torch.int64)
        if gridder.n_t == 1:
            t_idx.clamp_(max=0)
        gridder.accumulate(particles=p[:, :3], active_mask=active, weights=p[:, 3], t_idx=t_idx, release_idx=ridx,
                           dt_seconds=delta)
        alive = alive & ~(active & ~ref.lm._within_met_domain(p, mcfg))
        active_steps += active.sum()
        t_cursor = t_cursor - timedelta(seconds=delta)
    e1.record()
    torch.cuda.synchronize()
    t = e0.elapsed_time(e1) / 1e3
    act = int(active_steps.item())
    return {"value": act / t, "unit": "active particle-steps/s", "particles": n, "steps": n_time,
            "warmup": n_warm, "ms_per_step": 1e3 * t / n_time, "active_particle_steps": act,
            "graph_state": scheme._graph_compile_state, "wall_s": time.perf_counter() - t_wall}


def _reference_window_fn(syn, index_of=None):
    """``window_fn`` of reference_cuda_graph_rate from a SyntheticMet: the window starting
    at an hour as the reference's ``HourlyMetTensors`` on the host; ``index_of(hour)`` maps
    the hour to the synthetic window index (default: ``syn.window_index``)."""
    def window_fn(hour):
        ref = _reference_modules()
        h = syn.window_index(hour) if index_of is None else index_of(hour)
        w = syn.window(h, device="cpu")
        md = w.metadata
        return ref.mr.HourlyMetTensors(
            hour_start=w.hour_start.contiguous(), hour_end=w.hour_end.contiguous(),
            metadata=ref.mr.MetFieldMetadata(lon=md.lon, lat=md.lat, level=md.level,
                                             pressure_level_hpa=md.pressure_level_hpa, time_start=hour,
                                             time_end=hour + timedelta(hours=1),
                                             variable_units=dict(md.variable_units)),
            channel_names=w.channel_names, height_agl_m=w.height_agl_m.contiguous())

    return window_fn


def single_site_reference_gpu(syn, cfg, n_warm: int = 130, n_time: int = 240) -> dict:
    """The reference's CUDA-graph path on the single-site workload, from the release end:
    the first 130 steps (the compile, the one-step first window and a full window) untimed,
    the next 240 timed, when every particle of the 1 h release is active."""
    res = reference_cuda_graph_rate(cfg, _reference_window_fn(syn), cursor_start=cfg["cursor_start"],
                                    n_warm=n_warm, n_time=n_time, dt_s=DT_S, sim_length_s=SIM_LENGTH_S)
    if "value" in res:
        res["particle_steps_per_s"] = int(cfg["particles"].shape[0]) * n_time / (res["ms_per_step"] * n_time / 1e3)
    return res


def run_reference_gpu(args) -> None:
    """``--impl reference-gpu``: the reference's own torch.compile CUDA-graph step path
    (installed in baseline/_ref) on the single-site workload."""
    import torch

    from glide_b200.synthetic import SyntheticMet

    n = args.particles
    cfg = workload(n, 0, n_snapshots=max(5, args.snapshots if args.snapshots < 26 else 5))
    syn = SyntheticMet(cfg["spec"], device=torch.device("cuda"))
    res = single_site_reference_gpu(syn, cfg)
    if "unavailable" in res:
        print(json.dumps({"impl": "reference-gpu", **res}))
        return
    value = res["particle_steps_per_s"]
    print(json.dumps({"impl": "reference-gpu", "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": 1,
                      "steps": res["steps"], "warmup": res["warmup"], "ms_per_step": res["ms_per_step"],
                      "higher_is_better": True, "dtype": "f32", "data": "synthetic", "graph_state": res["graph_state"],
                      "config": {"workload": "single-site 24 h backward, 200k particles, 60x281x401 met, dt 30 s",
                                 "step": "one outer step (the reference's graph replay + convection + gridder)"}}),
          flush=True)


def main() -> None:
    args = parse()
    if args.impl == "reference-gpu":
        run_reference_gpu(args)
        return
    if args.workload == "regrid":
        run_regrid(args)
        return
    if args.workload == "multisite":
        run_multisite(args)
        return
    if args.workload == "periodic":
        run_periodic(args)
        return
    if args.workload == "serving":
        run_serving(args)
        return
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args)
        return
    import torch
    import torch.distributed as dist

    from glide_b200.runtime import BatchRunner, ParticleState
    from glide_b200.synthetic import SyntheticMet
    from glide_b200.window import grid_from_synthetic, window_from_synthetic

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=dev)
    cfg = workload(args.particles, rank, args.snapshots)
    syn = SyntheticMet(cfg["spec"], device=dev)
    grid = grid_from_synthetic(syn).to_device(dev)
    n_windows_total = args.snapshots - 1
    if args.warmup + args.steps > n_windows_total:
        raise SystemExit(f"warmup + steps must be <= {n_windows_total} windows (the 24 h job)")

    tuned = {"variant": 0, "steps_per_launch": args.steps_per_launch, "times_ms": {}}

    def make_runner(provider):
        r = BatchRunner(grid=grid, window_provider=provider, hanna=cfg["hanna"], footprint=cfg["footprint"],
                        domain=cfg["domain"], emanuel=cfg["emanuel"], met_dtype=args.met, device=dev,
                        seed=1234 + rank, pipeline=not args.no_pipeline)
        r.launch_variant = tuned["variant"]
        r.steps_per_launch = tuned["steps_per_launch"]
        r.fuse_convection = not args.separate_convection
        r.reorder = not args.no_reorder
        r.diagnostics = not args.no_diagnostics
        return r

    def fresh_state():
        return ParticleState.from_particles(cfg["particles"], cfg["rel_off"], cfg["win_end"], cfg["ridx"], dev)

    runner = make_runner(lambda hk: window_from_synthetic(syn, syn.window_index(hk), grid))
    kw = dict(batch_start=cfg["batch_start"], cursor_start=cfg["cursor_start"], cursor_terminus=cfg["terminus"],
              sim_length_s=SIM_LENGTH_S, dt_seconds=DT_S)
    if not args.no_autotune:  # launch shape picked by the autotuner, before and outside the timed region
        from glide_b200.autotune import tune

        tuned.update(tune(runner, fresh_state(), **kw))
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device=dev)

    # instrument the step-kernel launches with events on the launching stream
    import glide_b200._abi as abi

    stream = torch.cuda.current_stream()
    kernel_events: list = []
    real_step = abi.lib.glide_step

    def timed_step(a, s):  # events on the stream the kernel is launched on
        ls = torch.cuda.ExternalStream(s, device=dev) if s else stream
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(ls)
        rc = real_step(a, s)
        e1.record(ls)
        if record_kernels:
            kernel_events.append((e0, e1))
        return rc

    abi.lib.glide_step = timed_step
    real_reorder = abi.lib.glide_reorder_by_key
    reorders = [0]

    def counted_reorder(*a):  # three kernels per call
        if record_kernels:
            reorders[0] += 1
        return real_reorder(*a)

    abi.lib.glide_reorder_by_key = counted_reorder
    record_kernels = False
    run = runner.start(fresh_state(), **kw)
    for _ in range(args.warmup):
        run.step_window()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    steps_per_window = []
    win_events = []
    with ClockSampler(local) as clocks:
        record_kernels = True
        for _ in range(args.steps):
            flush.fill_(1)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            j0, j1 = run.windows[run.next_window]
            e0.record(stream)
            run.step_window()
            e1.record(stream)
            win_events.append((e0, e1))
            steps_per_window.append(j1 - j0)
        torch.cuda.synchronize()
        record_kernels = False
        if world > 1:
            dist.barrier()
        t_dev = sum(a.elapsed_time(b) for a, b in win_events) / 1e3
        # ---- end to end (met in pinned host memory, copies inside the timed region), sampled too
        e2e = None
        if not args.no_e2e:
            e2e = run_e2e(args, cfg, syn, grid, make_runner, fresh_state, kw, dev, stream, world)
    t_kernel = sum(a.elapsed_time(b) for a, b in kernel_events) / 1e3
    n_kernel_launches = len(kernel_events)
    out = run.finish() if run.done else None
    status = int(run.status.item())
    t_max = t_dev
    if world > 1:
        tt = torch.tensor([t_dev], device=dev)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        t_max = float(tt.item())
    n_outer = sum(steps_per_window)
    p_steps = args.particles * n_outer
    value = world * p_steps / t_max
    ms_per_step = 1e3 * t_max / args.steps


    # ---- the whole job captured into one CUDA graph, replayed once
    graph = None
    if not args.no_graph:
        abi.lib.glide_step = real_step
        abi.lib.glide_reorder_by_key = real_reorder
        graph = run_graph(cfg, syn, grid, make_runner, fresh_state, kw, dev, stream)

    if rank == 0:
        peak, peak_kind = measured_peak_hbm()
        achieved = B_ALG[args.met] * p_steps / t_kernel / 1e9
        clk = clocks.summary()
        line = {
            "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": args.met, "data": "synthetic",
            "config": {"workload": "single-site 24 h backward, 200k particles, 60x281x401 met, dt 30 s",
                       "particles": args.particles, "outer_steps_per_step": n_outer / args.steps,
                       "met_storage": args.met, "meander": True, "convection": "emanuel_reduced",
                       "max_substeps": 6, "step": "one met window (pack + convection + fused steps)",
                       "l2": "flushed (256 MB write) before every timed step; met bricks 440 MB > L2",
                       "parallelism": f"replicas x{world}", "launch_variant": tuned["variant"],
                       "steps_per_launch": tuned["steps_per_launch"] or "window",
                       "particle_order": "identity" if args.no_reorder else "work class, rebuilt before every launch",
                       "autotune_ms_per_window": {str(k): round(v, 3) for k, v in tuned["times_ms"].items()},
                       "autotune_steps_per_launch_ms": {str(k or "window"): round(v, 3)
                                                        for k, v in tuned.get("steps_times_ms", {}).items()}},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_kind": peak_kind,
                         # ncu DRAM bytes of one window's launch (the same workload's launch)
                         "traffic": STEP_KERNEL_NCU["dram_bytes_per_launch"] if args.met == "f32" else None,
                         "kernel": "step_kernel", "bytes_per_particle_step": B_ALG[args.met],
                         "kernel_time_share": t_kernel / t_dev,
                         "limiter": "instruction issue: the plume's met gathers hit L1 (DRAM traffic ~1/2000 of "
                                    "the algorithmic bytes), so the HBM frac is nominal",
                         "issue": issue_fraction(p_steps / t_kernel, clk)},
            "clocks": clk,
            # step launches (the convection fused in) + 3 per particle-order rebuild + per window: 3 packing
            # (surface, cells, wind sums) and 2 for the convection column
            "gpu_launches": n_kernel_launches + 3 * reorders[0] + 5 * args.steps,
            "status": status,
        }
        if e2e is not None:
            line["e2e"] = e2e
        if graph is not None:
            line["graph"] = graph
        if not args.no_cpu_baseline and world == 1:
            workers = os.cpu_count() or 1
            path = prepare_cpu_sample(syn, cfg, args.particles)
            try:
                rate, wall = cpu_oracle_rate(path, args.particles, CPU_BASELINE_STEPS, workers,
                                             repeats=CPU_BASELINE_REPEATS)
            finally:
                os.unlink(path)
            line["cpu_baseline"] = {"value": rate, "unit": METRIC, "cores": workers, "kind": "port",
                                    "sample": f"{CPU_BASELINE_REPEATS} x {args.particles} particles x "
                                              f"{CPU_BASELINE_STEPS} outer steps, all "
                                              f"released (oracle port, {workers} processes, {wall:.1f} s)"}
        if world == 1 and not args.no_extras:
            line.update(run_extras(args, syn, cfg, value, line))
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def issue_fraction(kernel_particle_steps_per_s: float, clk: dict) -> dict:
    """The step kernel's instruction-issue rate against the issue ceiling (one warp
    instruction per SM sub-partition per clock): warp instructions per particle-step from
    the ncu capture x the live particle-steps/s, over 148 x 4 x the median SM clock
    sampled during the timed region."""
    mhz = clk.get("sm_mhz") or clk.get("sm_max_mhz") or 1965.0
    achieved = STEP_KERNEL_NCU["warp_inst_per_particle_step"] * kernel_particle_steps_per_s
    peak = SM_COUNT * SMSP_PER_SM * mhz * 1e6
    return {"achieved_warp_inst_per_s": achieved, "peak_warp_inst_per_s": peak, "frac": achieved / peak,
            "warp_inst_per_particle_step": STEP_KERNEL_NCU["warp_inst_per_particle_step"], "sm_mhz": mhz}


def run_extras(args, syn, cfg, value: float, line: dict) -> dict:
    """Extra jobs of the default run, beside the headline (each one's failure is recorded,
    not raised): the reference's own CUDA-graph path on the same single-site workload and
    B200, the 2,688-release multisite job and the 720-release periodic job (bf16 met)."""
    import argparse

    import torch

    extras: dict = {}
    t = time.perf_counter()
    try:
        ref = single_site_reference_gpu(syn, cfg)
        if "particle_steps_per_s" in ref:
            ref["vs_reference_gpu"] = value / ref["particle_steps_per_s"]
            if "e2e" in line:
                ref["e2e_vs_reference_gpu"] = line["e2e"]["value"] / ref["particle_steps_per_s"]
        extras["reference_gpu"] = ref
    except Exception as exc:  # noqa: BLE001 - an extra never costs the headline line
        extras["reference_gpu"] = {"error": f"{type(exc).__name__}: {exc}"}
    extras["reference_gpu"]["extra_wall_s"] = time.perf_counter() - t
    torch.cuda.empty_cache()
    for name, fn in (("multisite", run_multisite), ("periodic", run_periodic)):
        t = time.perf_counter()
        try:
            extras[name] = fn(argparse.Namespace(**{**vars(args), "met": "bf16"}), emit=False)
        except Exception as exc:  # noqa: BLE001
            extras[name] = {"error": f"{type(exc).__name__}: {exc}"}
        extras[name]["extra_wall_s"] = time.perf_counter() - t
        torch.cuda.empty_cache()
    return extras


def run_graph(cfg, syn, grid, make_runner, fresh_state, kw, dev, stream) -> dict:
    """The full 24 h job (every window: particle order, packing, convection column, the
    step launch with fused convection) captured into one CUDA graph and replayed once,
    timed with CUDA events: the met is device-resident, one stream, no host work during
    the replay."""
    import torch

    from glide_b200.window import window_from_synthetic

    runner = make_runner(lambda hk: window_from_synthetic(syn, syn.window_index(hk), grid))
    runner.pipeline = False
    run = runner.start(fresh_state(), **kw)
    windows = len(run.windows)
    t = time.perf_counter()
    g = run.capture()
    capture_s = time.perf_counter() - t
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    g.replay()
    e1.record(stream)
    torch.cuda.synchronize()
    sec = e0.elapsed_time(e1) / 1e3
    out = run.finish()
    p_steps = int(cfg["particles"].shape[0]) * len(run.steps)
    return {"value": p_steps / sec, "unit": METRIC, "windows": windows, "outer_steps": len(run.steps),
            "replay_s": sec, "capture_s": capture_s, "status": out.status,
            "note": "whole 24 h job as one graph replay (first windows include the release hour)"}


def run_e2e(args, cfg, syn, grid, make_runner, fresh_state, kw, dev, stream, world) -> dict:
    """The job through the public runtime with the met in pinned host memory: each
    window's new snapshot is copied to the device by ``HostMetStreamer`` (prefetched
    on a copy stream during the previous window); each step reads back the window's
    diagnostics and the footprint slice of its time-ago bin."""
    import torch

    from glide_b200.window import HostMetStreamer

    names = HostMetStreamer.NAMES
    host = [{k: f[k].to("cpu").pin_memory() for k in names} for f in syn.fields]
    streamer = HostMetStreamer(lambda k: host[k], syn.times, grid, dev, lowest=int(np.argmin(syn.levels)))
    runner = make_runner(streamer)
    run = runner.start(fresh_state(), **kw)
    for _ in range(args.warmup):
        run.step_window()
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    b0 = streamer.bytes_copied
    d2h = 0
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    n_outer = 0
    for _ in range(args.steps):
        j0, j1 = run.windows[run.next_window]
        run.step_window()
        esc = run.esc[j0:j1].to("cpu", non_blocking=True)
        act = run.act[j0:j1].to("cpu", non_blocking=True)
        tbin = min(int((3600.0 - run.steps[j1 - 1].cursor_off) // 3600.0), run.footprint.shape[1] - 1)
        fp_slice = run.footprint[:, max(tbin, 0)].to("cpu", non_blocking=True)
        d2h += esc.numel() * 4 + act.numel() * 4 + fp_slice.numel() * 4
        n_outer += j1 - j0
    e1.record(stream)
    torch.cuda.synchronize()
    t = e0.elapsed_time(e1) / 1e3
    if world > 1:
        tt = torch.tensor([t], device=dev)
        torch.distributed.all_reduce(tt, op=torch.distributed.ReduceOp.MAX)
        t = float(tt.item())
    h2d = streamer.bytes_copied - b0
    return {"value": world * args.particles * n_outer / t, "unit": METRIC,
            "h2d_bytes_per_step": h2d / args.steps, "d2h_bytes_per_step": d2h / args.steps}


if __name__ == "__main__":
    main()
