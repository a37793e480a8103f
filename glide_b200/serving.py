"""Footprint serving: continuous batching of backward-footprint requests on one GPU.

A request is one release (site, release time, particle count, backward duration).
The server keeps every met window of its horizon packed and resident in HBM
(read-only, shared by all requests), admits requests while their particle state
and footprint fit an HBM budget and a concurrency cap, and advances every
admitted request one met window per scheduling tick. By default (``grouped``)
a tick packs the next window of every admitted request — requests of different
particle counts, release times and cursor positions, each with its own met
window, schedule and footprint — into grouped launches (``glide_step_batched``,
up to 32 requests each) on one stream: one launch per tick fills the GPU with
many small requests. Otherwise each request runs its own launches on a stream of
a pool. A request that arrives while others run is admitted as soon as the
concurrency cap and the HBM budget allow. Each request's noise is keyed by its
own seed and its own particle and step numbers, so its result does not depend on
what else runs.

The per-request work is exactly the batch runtime's (``glide_b200.runtime``):
per window one fused step launch with the window's convection inside it; the
convection columns of the resident windows are built once and shared.
"""

from __future__ import annotations

import time
from collections import deque
from dataclasses import dataclass, field
from datetime import datetime, timedelta

import numpy as np
import torch

from glide_b200.runtime import (BatchRun, BatchRunner, DomainSpec, EmanuelConfig, FootprintSpec, HannaConfig,
                                ParticleState, hour_floor, launch_grouped)
from glide_b200.window import GridInfo, PackedWindow, WindowFields


@dataclass
class FootprintRequest:
    """One backward footprint: ``n_particles`` released at (lon, lat, height) over
    ``release_s`` seconds from ``release_time``, integrated ``duration_h`` hours
    backward from the release end, binned hourly (time_ago) on the server's grid."""

    request_id: int
    lon: float
    lat: float
    height_m: float
    release_time: datetime
    n_particles: int
    duration_h: float
    seed: int = 0
    release_s: float = 3600.0
    arrival_s: float = 0.0  # offset of the arrival from the start of the stream


@dataclass
class FootprintResult:
    request_id: int
    footprint: torch.Tensor | None  # [time_ago, Zb, Y, X] on the host when kept
    bin_totals: np.ndarray  # per time_ago bin sum
    escaped: int
    n_steps: int
    active_particle_steps: int
    arrival_s: float
    admitted_s: float
    finished_s: float

    @property
    def latency_s(self) -> float:
        return self.finished_s - self.arrival_s


class _Resident:
    """Packed windows of the whole horizon, built once and shared read-only."""

    def __init__(self, grid: GridInfo, provider, hours: list[datetime], hanna: HannaConfig, met_dtype: str,
                 device) -> None:
        self.windows: dict[datetime, tuple[WindowFields, PackedWindow]] = {}
        for h in hours:
            wf = provider(h)
            pw = PackedWindow(grid, met_dtype, device)
            pw.pack(wf, meander_coefficient=hanna.meander_coefficient, meander_radius=hanna.meander_stencil_radius,
                    build_meander=hanna.meander_enabled)
            self.windows[h] = (wf, pw)

    @property
    def nbytes(self) -> int:
        return sum(pw.nbytes for _, pw in self.windows.values())


@dataclass
class _Active:
    req: FootprintRequest
    run: BatchRun
    stream: torch.cuda.Stream
    nbytes: int
    admitted_s: float
    done_event: torch.cuda.Event | None = None
    issued_all: bool = False
    host: dict | None = None  # pinned copies of the results, valid once done_event has completed


@dataclass
class ServerStats:
    admitted: int = 0
    completed: int = 0
    ticks: int = 0
    windows_issued: int = 0
    launches: int = 0  # step launches (grouped launches count once)
    peak_active: int = 0
    peak_bytes: int = 0
    results: list = field(default_factory=list)


class FootprintServer:
    """Continuous-batching footprint server on one GPU.

    ``met_provider(hour) -> WindowFields`` serves the device-resident raw met; all
    windows between ``horizon_start`` and ``horizon_end`` are packed at start-up.
    ``hbm_budget_bytes`` bounds the particle state + footprints of admitted requests,
    ``max_active`` the number of requests in flight (one CUDA stream each, from a
    pool of ``n_streams``). With ``order_particles`` each request's particles are
    regrouped by work class before every window, as the batch runtime does (results
    do not depend on it).
    """

    def __init__(self, *, grid: GridInfo, met_provider, horizon_start: datetime, horizon_end: datetime,
                 hanna: HannaConfig, emanuel: EmanuelConfig | None, footprint: FootprintSpec, domain: DomainSpec,
                 hbm_budget_bytes: float = 60e9, max_active: int = 64, n_streams: int = 16, met_dtype: str = "bf16",
                 dt_seconds: float = 30.0, device="cuda", keep_footprints: bool = False,
                 grouped: bool = True, order_particles: bool = True) -> None:
        self.device = torch.device(device)
        self.order_particles = bool(order_particles)
        self.grid = grid if grid.level_sorted_dev is not None else grid.to_device(self.device)
        self.hanna, self.emanuel, self.domain = hanna, emanuel, domain
        self.fp_template = footprint
        self.budget = float(hbm_budget_bytes)
        self.max_active = int(max_active)
        self.dt = float(dt_seconds)
        self.met_dtype = met_dtype
        self.keep = keep_footprints
        hours = []
        h = hour_floor(horizon_start)
        while h < horizon_end:
            hours.append(h)
            h = h + timedelta(hours=1)
        self.resident = _Resident(self.grid, met_provider, hours, hanna, met_dtype, self.device)
        torch.cuda.synchronize(self.device)
        self.grouped = bool(grouped)
        self.column_cache: dict = {}  # (hour, alpha) -> convection column, shared by all requests
        if self.grouped:
            self.streams = [torch.cuda.Stream(device=self.device)]
        else:
            self.streams = [torch.cuda.Stream(device=self.device) for _ in range(max(1, n_streams))]
        self.pending: deque[FootprintRequest] = deque()
        self.active: list[_Active] = []
        self.bytes_in_use = 0
        self.stats = ServerStats()
        self.t0 = None

    # -- request bookkeeping ------------------------------------------------------

    def request_bytes(self, req: FootprintRequest) -> int:
        n_bins = int(np.ceil(req.duration_h))
        fp = self.fp_template
        per_bin = (len(fp.z_edges) - 1) * fp.n_y * fp.n_x * 4
        return int(req.n_particles) * 64 + n_bins * per_bin

    def _runner_for(self, req: FootprintRequest, stream) -> BatchRunner:
        res = self.resident.windows

        def provider(hour):
            return res[hour][0]

        fp = FootprintSpec(self.fp_template.lon_bounds, self.fp_template.lat_bounds, self.fp_template.n_x,
                           self.fp_template.n_y, self.fp_template.z_edges, int(np.ceil(req.duration_h)), 1)
        r = BatchRunner(grid=self.grid, window_provider=provider, hanna=self.hanna, footprint=fp,
                        domain=self.domain, emanuel=self.emanuel, met_dtype=self.met_dtype, device=self.device,
                        seed=req.seed, packed_provider=lambda hour: res[hour][1])
        r.column_cache = self.column_cache
        r.reorder = self.order_particles  # each request's particles regrouped by work class per window
        return r

    def _admit(self, req: FootprintRequest, now_s: float) -> None:
        stream = self.streams[self.stats.admitted % len(self.streams)]
        n = int(req.n_particles)
        rng = np.random.default_rng(req.seed)
        parts = np.stack([np.full(n, req.lon), np.full(n, req.lat), np.full(n, req.height_m), np.full(n, 1.0 / n)],
                         axis=1).astype(np.float32)
        rel_off = rng.uniform(0.0, req.release_s, n).astype(np.float32)
        win_end = np.full(n, req.release_s, dtype=np.float32)
        with torch.cuda.stream(stream):
            runner = self._runner_for(req, stream)
            state = ParticleState.from_particles(parts, rel_off, win_end, np.zeros(n, dtype=np.int32), self.device)
            end = req.release_time + timedelta(seconds=req.release_s)
            run = runner.start(state, batch_start=req.release_time, cursor_start=end,
                               cursor_terminus=end - timedelta(hours=req.duration_h),
                               sim_length_s=req.duration_h * 3600.0, dt_seconds=self.dt)
        nb = self.request_bytes(req)
        self.active.append(_Active(req, run, stream, nb, now_s))
        self.bytes_in_use += nb
        self.stats.admitted += 1

    def _collect(self, a: _Active) -> None:
        """Queue the request's reductions and their copies to pinned host memory behind
        its last window, then its done event: nothing here waits for the device."""
        run = a.run
        n = len(run.steps)
        with torch.cuda.stream(a.stream):
            fp = run.footprint[0]
            counts = torch.stack([run.esc[:n].to(torch.int64).sum(), run.act[:n].to(torch.int64).sum()])
            host = {"totals": torch.empty(fp.shape[0], dtype=torch.float64).pin_memory(),
                    "counts": torch.empty(2, dtype=torch.int64).pin_memory()}
            host["totals"].copy_(fp.sum(dim=(1, 2, 3), dtype=torch.float64), non_blocking=True)
            host["counts"].copy_(counts, non_blocking=True)
            if self.keep:
                host["footprint"] = torch.empty(fp.shape, dtype=fp.dtype).pin_memory()
                host["footprint"].copy_(fp, non_blocking=True)
            a.done_event = torch.cuda.Event()
            a.done_event.record(a.stream)
        a.host = host

    def _finish(self, a: _Active, now_s: float) -> FootprintResult:
        h = a.host  # the done event has completed: the pinned copies are final
        esc, act = (int(v) for v in h["counts"].tolist())
        return FootprintResult(a.req.request_id, h.get("footprint"), h["totals"].numpy(), esc, len(a.run.steps), act,
                               a.req.arrival_s, a.admitted_s, now_s)

    # -- the scheduling loop ------------------------------------------------------

    def now(self) -> float:
        return time.perf_counter() - self.t0

    def tick(self) -> list[FootprintResult]:
        """Admit what fits, advance every in-flight request by one window, collect
        finished requests."""
        now = self.now()
        while self.pending and len(self.active) < self.max_active:
            req = self.pending[0]
            if req.arrival_s > now:
                break
            if self.bytes_in_use + self.request_bytes(req) > self.budget and self.active:
                break
            self._admit(self.pending.popleft(), now)
        self.stats.peak_active = max(self.stats.peak_active, len(self.active))
        self.stats.peak_bytes = max(self.stats.peak_bytes, self.bytes_in_use)
        if self.grouped:
            stream = self.streams[0]
            args, keep, ending = [], [], []
            for a in self.active:
                if a.issued_all:
                    continue
                arg, k = a.run.next_window_args(stream)
                args.append(arg)
                keep.append(k)
                if a.run.done:
                    ending.append(a)
            if args:
                launch_grouped(args, stream)
                self.stats.windows_issued += len(args)
                self.stats.launches += (len(args) + 31) // 32
            for a in ending:
                a.issued_all = True
                self._collect(a)
            del keep  # the launches are queued behind everything they read
        else:
            for a in self.active:
                if a.issued_all:
                    continue
                with torch.cuda.stream(a.stream):
                    a.run.step_window(a.stream)
                    self.stats.windows_issued += 1
                    self.stats.launches += 1
                    if a.run.done:
                        a.issued_all = True
                        self._collect(a)
        finished = []
        keep = []
        for a in self.active:
            if a.issued_all and a.done_event.query():
                res = self._finish(a, self.now())
                self.bytes_in_use -= a.nbytes
                self.stats.completed += 1
                finished.append(res)
            else:
                keep.append(a)
        self.active = keep
        self.stats.ticks += 1
        return finished

    def serve(self, requests: list[FootprintRequest], *, realtime: bool = True) -> list[FootprintResult]:
        """Feed ``requests`` at their arrival offsets (wall clock when ``realtime``,
        all at once otherwise) and run until every one has finished."""
        self.pending = deque(sorted(requests, key=lambda r: r.arrival_s))
        if not realtime:
            for r in self.pending:
                r.arrival_s = 0.0
        self.t0 = time.perf_counter()
        results: list[FootprintResult] = []
        while self.pending or self.active:
            if not self.active and self.pending and self.pending[0].arrival_s > self.now():
                time.sleep(min(0.005, max(0.0, self.pending[0].arrival_s - self.now())))
                continue
            results.extend(self.tick())
        self.stats.results = results
        return results


def poisson_requests(n: int, rate_per_s: float, sites: np.ndarray, t_release0: datetime, window_h: float,
                     n_range=(1000, 50000), duration_range_h=(6.0, 120.0), seed: int = 0) -> list[FootprintRequest]:
    """A seeded Poisson request stream: site among ``sites`` (lon, lat), release time
    uniform (whole minutes) in ``window_h`` hours after ``t_release0``, particle count
    log-uniform in ``n_range``, backward duration uniform in ``duration_range_h``."""
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0 / rate_per_s, n))
    out = []
    for i in range(n):
        s = int(rng.integers(len(sites)))
        rel = t_release0 + timedelta(minutes=int(rng.integers(int(window_h * 60))))
        n_p = int(np.exp(rng.uniform(np.log(n_range[0]), np.log(n_range[1]))))
        dur = float(rng.uniform(*duration_range_h))
        out.append(FootprintRequest(i, float(sites[s, 0]), float(sites[s, 1]), float(rng.uniform(10.0, 300.0)), rel,
                                    n_p, dur, seed=int(rng.integers(1 << 31)), arrival_s=float(t[i])))
    return out
