"""Fused batch runtime: the reference's per-step cursor loop, one met window per launch.

Replaces the static branch of the reference's cursor loop
(``src/lpdm/main.py:1382-1477``: active mask, met window and RK2 weight, the
scheme step, once-per-window convection, time-ago bin, footprint scatter-add,
escape kill) for one batch. The host computes the step schedule exactly as the
reference does (cursor arithmetic in ``datetime``, float32 rounding of the
cursor offset) and then issues, per met window,

* without convection: ONE ``glide_step`` launch covering every outer step of
  the window (physics + footprint + escape fused, state in registers);
* with convection: ``glide_step`` for the physics of the window's first step,
  ``glide_convect_redistribute`` against the window's column, then one
  ``glide_step`` that does the first step's footprint/escape and all remaining
  steps — the reference's step -> convection -> footprint -> kill order.

The work that depends only on met (packing the bricks, building the convection
column) is done for window k+1 on a side stream while window k's steps run,
into the second of two brick / column slots.

No launch synchronises with the host; per-step diagnostics (escaped and
active counts) accumulate in device arrays read once per batch.
"""

from __future__ import annotations

import ctypes as C
from collections.abc import Callable
from dataclasses import dataclass, field
from datetime import UTC, datetime, timedelta

import numpy as np
import torch

from glide_b200 import _abi
from glide_b200.config import DomainSpec, EmanuelConfig, FootprintSpec, HannaConfig  # noqa: F401 (re-exported)
from glide_b200.window import GridInfo, PackedWindow, WindowFields, stream_handle


@dataclass
class ParticleState:
    """Structure-of-arrays particle state on the device."""

    lon: torch.Tensor
    lat: torch.Tensor
    z: torch.Tensor
    weight: torch.Tensor
    u_prime: torch.Tensor
    v_prime: torch.Tensor
    w_prime: torch.Tensor
    u_meander: torch.Tensor
    v_meander: torch.Tensor
    rel_off: torch.Tensor
    win_end_off: torch.Tensor
    release_idx: torch.Tensor  # int32
    alive: torch.Tensor  # uint8

    @property
    def n(self) -> int:
        return self.lon.numel()

    @classmethod
    def from_particles(cls, particles, rel_off, win_end_off, release_idx, device) -> ParticleState:
        """From the reference's ``(N, 4)`` [lon, lat, z, weight] layout and sidecars
        (``ParticleBatch``, src/lpdm/release_generator.py:202-237)."""
        p = torch.as_tensor(particles, dtype=torch.float32)
        if p.dim() != 2 or p.shape[1] != 4:
            raise ValueError("particles must have shape (N, 4)")
        n = p.shape[0]
        p = _upload(p, device)
        z = torch.zeros(n, dtype=torch.float32, device=device)
        return cls(p[:, 0].contiguous(), p[:, 1].contiguous(), p[:, 2].contiguous(), p[:, 3].contiguous(),
                   z.clone(), z.clone(), z.clone(), z.clone(), z.clone(),
                   _upload(torch.as_tensor(rel_off, dtype=torch.float32), device),
                   _upload(torch.as_tensor(win_end_off, dtype=torch.float32), device),
                   _upload(torch.as_tensor(release_idx), device).to(dtype=torch.int32),
                   torch.ones(n, dtype=torch.uint8, device=device))

    def particles(self) -> torch.Tensor:
        return torch.stack([self.lon, self.lat, self.z, self.weight], dim=1)


def _upload(t: torch.Tensor, device) -> torch.Tensor:
    """Host tensor -> device through pinned memory, asynchronous on the current stream
    (a pageable copy would wait for the stream's earlier work); device tensors pass."""
    device = torch.device(device)
    if t.device == device or device.type != "cuda":
        return t.to(device)
    return t.contiguous().pin_memory().to(device, non_blocking=True)


@dataclass
class StepPlan:
    cursor: datetime
    cursor_off: float
    delta: float
    hour: datetime
    alpha: float = 0.0


# The step kernel's launch shape when the runner sets none: one 768-thread block per SM
# once a batch gives every SM such a block, 128-thread blocks (six per SM) below that,
# where the smaller blocks spread a small batch over more SMs. Measured on one B200
# against 128 x 6: 7 % faster on the 200,000-particle single-site window, 7 % on the
# 720-release periodic job, 6 % on the 2,688-release multisite job.
_WIDE_SHAPE = (768, 1)
_NARROW_SHAPE = (128, 6)


def default_launch_variant(n_particles: int, device) -> int:
    """Launch variant of the default shape for a batch of ``n_particles`` on ``device``."""
    shapes = {}
    nv = C.c_int32()
    _abi.check(_abi.lib.glide_step_launch_variants(C.byref(nv)), "glide_step_launch_variants")
    for v in range(nv.value - 1):  # the last variant is the general kernel at shape 0
        t, b = C.c_int32(), C.c_int32()
        _abi.check(_abi.lib.glide_step_launch_variant_info(v, C.byref(t), C.byref(b)), "glide_step_launch_variant_info")
        shapes.setdefault((t.value, b.value), v)
    sms = torch.cuda.get_device_properties(torch.device(device)).multi_processor_count
    wide = n_particles >= sms * _WIDE_SHAPE[0] * _WIDE_SHAPE[1]
    return shapes.get(_WIDE_SHAPE if wide else _NARROW_SHAPE, 0)


def hour_floor(t: datetime) -> datetime:
    """main.py:380-381"""
    return t.astimezone(UTC).replace(minute=0, second=0, microsecond=0)


_EPOCH = datetime(1970, 1, 1, tzinfo=UTC)
_US = timedelta(microseconds=1)
_HOUR_US = 3_600_000_000


class StepPlans:
    """The cursor walk as arrays — cursor and hour instants in integer microseconds
    since the epoch, float64 cursor offsets, step lengths and RK2 weights — so a
    batch of thousands of steps is planned without a Python loop. Indexing gives
    ``StepPlan`` records; slicing gives a shorter ``StepPlans``."""

    def __init__(self, cursor_us: np.ndarray, cursor_off: np.ndarray, delta: np.ndarray, hour_us: np.ndarray,
                 alpha: np.ndarray, tz) -> None:
        self.cursor_us, self.cursor_off, self.delta = cursor_us, cursor_off, delta
        self.hour_us, self.alpha, self.tz = hour_us, alpha, tz

    def __len__(self) -> int:
        return int(self.cursor_us.shape[0])

    def __getitem__(self, k):
        if isinstance(k, slice):
            return StepPlans(self.cursor_us[k], self.cursor_off[k], self.delta[k], self.hour_us[k], self.alpha[k],
                             self.tz)
        cursor = (_EPOCH + int(self.cursor_us[k]) * _US).astimezone(self.tz)
        return StepPlan(cursor, float(self.cursor_off[k]), float(self.delta[k]), _EPOCH + int(self.hour_us[k]) * _US,
                        float(self.alpha[k]))

    def __iter__(self):
        return (self[k] for k in range(len(self)))


def plan_steps(batch_start: datetime, cursor_start: datetime, cursor_terminus: datetime,
               dt_seconds: float) -> StepPlans | list[StepPlan]:
    """The cursor walk of main.py:1383-1389, 1610 with the alpha of main.py:916-919
    for hourly windows [hour, hour + 1 h]: steps of ``dt_seconds`` back from
    ``cursor_start`` while the cursor is after ``cursor_terminus``, the last one cut
    to end on it. Timezone-aware instants are planned with numpy in exact integer
    microseconds, reproducing ``datetime`` arithmetic (step lengths rounded to the
    microsecond as ``timedelta`` rounds them); naive ones step by step."""
    if cursor_start.tzinfo is None or cursor_terminus.tzinfo is None or batch_start.tzinfo is None:
        return _plan_steps_loop(batch_start, cursor_start, cursor_terminus, dt_seconds)
    dt = float(dt_seconds)
    dt_us = timedelta(seconds=dt) // _US
    if dt_us <= 0:
        raise ValueError("dt_seconds must be positive")
    t0 = (cursor_start - _EPOCH) // _US
    term = (cursor_terminus - _EPOCH) // _US
    b = batch_start.timestamp()
    if t0 <= term:
        z = np.zeros(0)
        return StepPlans(np.zeros(0, np.int64), z, z, np.zeros(0, np.int64), z, cursor_start.tzinfo)
    # full steps while the remaining span exceeds dt (as the float comparison of min() sees it)
    n_max = (t0 - term) // dt_us + 2
    j = np.arange(n_max, dtype=np.int64)
    remain_s = (t0 - term - j * dt_us) / 1e6
    full = remain_s > dt
    n_full = int(np.argmin(full)) if not full.all() else n_max
    cursor_us = t0 - np.arange(n_full + 1, dtype=np.int64) * dt_us
    delta = np.full(n_full + 1, dt)
    delta[n_full] = remain_s[n_full]
    t_s = cursor_us / 1e6
    hour_us = cursor_us - np.mod(cursor_us, _HOUR_US)
    ts = hour_us / 1e6
    te = (hour_us + _HOUR_US) / 1e6
    alpha = np.clip((t_s - 0.5 * delta - ts) / np.maximum(1.0, te - ts), 0.0, 1.0)
    return StepPlans(cursor_us, t_s - b, delta, hour_us, alpha, cursor_start.tzinfo)


def _plan_steps_loop(batch_start: datetime, cursor_start: datetime, cursor_terminus: datetime,
                     dt_seconds: float) -> list[StepPlan]:
    steps = []
    t = cursor_start
    b = batch_start.timestamp()
    while t > cursor_terminus:
        delta = min(float(dt_seconds), (t - cursor_terminus).total_seconds())
        hk = hour_floor(t)
        ts, te = hk.timestamp(), (hk + timedelta(hours=1)).timestamp()
        alpha = max(0.0, min(1.0, (t.timestamp() - 0.5 * delta - ts) / max(1.0, te - ts)))
        steps.append(StepPlan(t, t.timestamp() - b, delta, hk, alpha))
        t = t - timedelta(seconds=delta)
    return steps


def schedule_array(steps) -> np.ndarray:
    """``glide_step_sched`` records (float32 cursor offset, delta, alpha; int32 index)."""
    rec = np.zeros(len(steps), dtype=np.dtype([("c", "<f4"), ("d", "<f4"), ("a", "<f4"), ("i", "<i4")]))
    if isinstance(steps, StepPlans):
        rec["c"], rec["d"], rec["a"] = steps.cursor_off, steps.delta, steps.alpha
        rec["i"] = np.arange(len(steps), dtype=np.int32)
        return rec
    for k, s in enumerate(steps):
        rec[k] = (np.float32(s.cursor_off), np.float32(s.delta), np.float32(s.alpha), k)
    return rec


def window_ranges(steps) -> list[tuple[int, int]]:
    """Runs [k, e) of consecutive steps in the same hourly window."""
    if isinstance(steps, StepPlans):
        h = steps.hour_us
        if h.size == 0:
            return []
        cuts = np.flatnonzero(h[1:] != h[:-1]) + 1
        edges = [0, *cuts.tolist(), int(h.size)]
        return list(zip(edges[:-1], edges[1:]))
    out = []
    k = 0
    while k < len(steps):
        e = k
        while e < len(steps) and steps[e].hour == steps[k].hour:
            e += 1
        out.append((k, e))
        k = e
    return out


@dataclass
class BatchOutput:
    state: ParticleState
    footprint: torch.Tensor
    escaped_per_step: np.ndarray
    active_per_step: np.ndarray
    n_steps: int
    convection: list = field(default_factory=list)  # (window start, n_moved device tensor)
    status: int = 0
    # per-step diagnostics of the reference runtime (main.py:1565-1566, 1612-1643), float32
    # [n_steps, 3]: mean (lon, lat, z) of all particles after the step, and the grid-mean
    # (u, v, w) of the step's window lerped by its RK2 weight; None when not computed
    diag_pos: np.ndarray | None = None
    diag_wind: np.ndarray | None = None

    def diagnostic_rows(self) -> list[dict]:
        """The per-step rows the reference's runtime writes (main.py:1612-1643) for this
        batch: step number within the batch, mean position, mean wind, active, escaped and
        alive counts."""
        if self.diag_pos is None:
            raise ValueError("the batch ran without diagnostics")
        n = int(self.state.n)
        alive = n - np.cumsum(self.escaped_per_step)
        return [{"step": k + 1, "mean_lon": float(p[0]), "mean_lat": float(p[1]), "mean_alt_agl_m": float(p[2]),
                 "u_mean_m_s": float(w[0]), "v_mean_m_s": float(w[1]), "w_mean_m_s": float(w[2]),
                 "active_particles": int(a), "escaped_this_step": int(e), "alive_particles": int(al)}
                for k, (p, w, a, e, al) in enumerate(zip(self.diag_pos, self.diag_wind, self.active_per_step,
                                                         self.escaped_per_step, alive))]


class BatchRun:
    """One batch in flight. ``step_window()`` issues the launches of the next window."""

    def __init__(self, runner: BatchRunner, state: ParticleState, steps: list[StepPlan], sim_length_s: float) -> None:
        self.r = runner
        self.state = state
        self.steps = steps
        self.sim_length_s = float(sim_length_s)
        dev = runner.device
        self._default_variant: int | None = None
        self.sched_dev = _upload(torch.from_numpy(schedule_array(steps).view(np.uint8).copy()), dev)
        self.esc = torch.zeros(max(1, len(steps)), dtype=torch.int32, device=dev)
        self.act = torch.zeros(max(1, len(steps)), dtype=torch.int32, device=dev)
        self.status = torch.zeros(1, dtype=torch.int32, device=dev)
        # per-step diagnostics: fixed-point position sums [n_steps][3] (the step kernel adds to
        # them) and each window's wind sums [n_windows][6] (copied from its packed window)
        self.diagnostics = runner.diagnostics
        self.diag_sum = torch.zeros((max(1, len(steps)), 3), dtype=torch.int64, device=dev) \
            if self.diagnostics else None
        fp = runner.footprint
        self.footprint = torch.zeros(fp.device_shape, dtype=fp.torch_dtype, device=dev)
        self.footprint_out = None
        self.sink = runner.footprint_sink
        if fp.ring > 0:
            if fp.n_time_bins == 1:
                raise ValueError("ring footprints need n_time_bins > 1 (a single bin is already one slice)")
            # each release's particles share one window end (release_generator.py:312-314): one bin per step
            ends = np.full(fp.n_releases, np.nan, dtype=np.float32)
            r_host = state.release_idx.cpu().numpy()
            w_host = state.win_end_off.cpu().numpy()
            for r in np.unique(r_host):
                vals = np.unique(w_host[r_host == r])
                if vals.size != 1:
                    raise ValueError(f"ring footprints need one window end per release (release {r} has {vals.size})")
                if 0 <= r < fp.n_releases:
                    ends[r] = vals[0]
            self.release_end = ends
            if self.sink is None:
                self.footprint_out = torch.zeros(fp.shape, dtype=fp.torch_dtype, device=dev)
                out = self.footprint_out

                rows_out = out.view(fp.n_releases * fp.n_time_bins, -1)

                def sink(r_idx, b_idx, slices):
                    rows_out.index_add_(0, r_idx * fp.n_time_bins + b_idx, slices.reshape(slices.shape[0], -1))

                self.sink = sink
        self.z_edges = _upload(torch.as_tensor(np.asarray(runner.footprint.z_edges, dtype=np.float32)), dev)
        # windows = runs of consecutive steps with the same hour
        self.windows: list[tuple[int, int]] = window_ranges(steps)
        self.wind_sum = torch.zeros((max(1, len(self.windows)), 6), dtype=torch.float64, device=dev) \
            if self.diagnostics else None
        self.next_window = 0
        self.conv_log: list = []
        # per-window preparation, double-buffered when pipelined (bricks and column of
        # window k+1 built on a side stream while window k's steps run)
        self.pipelined = runner.pipeline and runner.packed_provider is None
        self.prep_stream = torch.cuda.Stream(device=dev) if self.pipelined else None
        self.prepared: dict = {}
        self.slot_free: list = [None, None]
        self.conv_scratch = []
        if runner.emanuel is not None:
            nb = C.c_size_t()
            _abi.check(_abi.lib.glide_convect_scratch_bytes(runner.grid.shape[0], C.byref(nb)),
                       "glide_convect_scratch_bytes")
            self.conv_scratch = [torch.zeros(nb.value // 8, dtype=torch.float64, device=dev) for _ in range(2)]
        # particle ordering by work class (glide_reorder_by_key): each window's launches step
        # the particles in the order built from the work keys of the previous window
        self.order = self.work_key = self.reorder_scratch = None
        self.keys_valid = False  # work_key holds the keys of a launch
        self.order_valid = False  # order holds a permutation built from such keys
        if runner.reorder and state.n > 0:
            nb = C.c_size_t()
            _abi.check(_abi.lib.glide_reorder_scratch_bytes(state.n, C.byref(nb)), "glide_reorder_scratch_bytes")
            self.order = torch.empty(state.n, dtype=torch.int32, device=dev)
            self.work_key = torch.zeros(state.n, dtype=torch.uint8, device=dev)
            self.reorder_scratch = torch.empty(nb.value, dtype=torch.uint8, device=dev)

    @property
    def done(self) -> bool:
        return self.next_window >= len(self.windows)

    def _step_args(self, packed: PackedWindow, j0: int, n_steps: int, phys_begin: int, post_begin: int,
                   noise, noise_row: int = 0) -> _abi.StepArgs:
        """Arguments of one ``glide_step`` launch of steps [j0, j0 + n_steps); ``noise_row``
        is j0's row in the window's injected noise buffers."""
        r, s = self.r, self.state
        h = r.hanna
        a = _abi.StepArgs()
        a.n = s.n
        a.lon, a.lat, a.z, a.weight = s.lon.data_ptr(), s.lat.data_ptr(), s.z.data_ptr(), s.weight.data_ptr()
        a.pos_stride = 1
        a.u_prime, a.v_prime, a.w_prime = s.u_prime.data_ptr(), s.v_prime.data_ptr(), s.w_prime.data_ptr()
        a.u_meander, a.v_meander = s.u_meander.data_ptr(), s.v_meander.data_ptr()
        a.rel_off, a.win_end_off = s.rel_off.data_ptr(), s.win_end_off.data_ptr()
        a.release_idx, a.alive, a.active_mask = s.release_idx.data_ptr(), s.alive.data_ptr(), None
        a.sim_length_s = self.sim_length_s
        a.wind_packed, a.surf_packed, a.support_packed = (packed.wind.data_ptr(), packed.surf.data_ptr(),
                                                          packed.support.data_ptr())
        a.met_dtype = packed.code
        a.grid = r.grid.c_grid()
        a.substep_c, a.max_substeps, a.z_ubl_m = h.substep_c, h.max_substeps, h.z_ubl_m
        a.flexpart_tl_floors, a.surface_layer_override = int(h.flexpart_tl_floors), int(h.surface_layer_override)
        a.meander_enabled, a.meander_timescale_s = int(h.meander_enabled), h.meander_timescale_seconds
        a.sched = self.sched_dev.data_ptr() + 16 * j0
        a.n_steps, a.phys_begin, a.post_begin = n_steps, phys_begin, post_begin
        if noise is not None:
            sub, mea = noise
            a.noise_substep = sub[noise_row].data_ptr()
            a.noise_meander = None if mea is None else mea[noise_row].data_ptr()
        a.seed = r.seed
        a.footprint = self.footprint.data_ptr()
        fp = r.footprint
        a.fp = _abi.FootprintGrid(fp.lon_bounds[0], fp.lon_bounds[1], fp.lat_bounds[0], fp.lat_bounds[1],
                                  fp.n_releases, fp.n_time_bins, len(fp.z_edges) - 1, fp.n_y, fp.n_x,
                                  self.z_edges.data_ptr(), fp.ring, 1 if fp.value_dtype == "f64" else 0)
        d = r.domain
        a.dom_lon_min, a.dom_lon_max = d.lon_bounds
        a.dom_lat_min, a.dom_lat_max = d.lat_bounds
        a.dom_alt_max = d.alt_max_m
        a.escaped_per_step = self.esc.data_ptr() + 4 * j0
        a.active_per_step = self.act.data_ptr() + 4 * j0
        a.status = self.status.data_ptr()
        a.diag_pos_fixed = None if self.diag_sum is None else self.diag_sum.data_ptr() + 24 * j0
        if r.launch_variant is not None:
            a.launch_variant = r.launch_variant
        else:
            if self._default_variant is None:
                self._default_variant = default_launch_variant(self.state.n, r.device)
            a.launch_variant = self._default_variant
        if self.work_key is not None:
            a.order = self.order.data_ptr() if self.order_valid else None
            a.work_key = self.work_key.data_ptr()
        return a

    def _noise(self, j0: int, j1: int):
        """Injected normals of steps [j0, j1), checked against the extents the kernel indexes."""
        r = self.r
        noise = r.noise_provider(list(range(j0, j1))) if r.noise_provider is not None else None
        if noise is not None:
            sub, mea = noise
            want = (j1 - j0, r.hanna.max_substeps, 3, self.state.n)
            if tuple(sub.shape) != want or sub.dtype != torch.float32 or not sub.is_contiguous():
                raise ValueError(f"injected substep noise must be contiguous float32 {want}, got {tuple(sub.shape)}")
            if r.hanna.meander_enabled and (mea is None or tuple(mea.shape) != (j1 - j0, 2, self.state.n)
                                            or mea.dtype != torch.float32 or not mea.is_contiguous()):
                raise ValueError("injected meander noise must be contiguous float32 (steps, 2, n)")
        return noise

    def _column_for(self, j: int, stream) -> torch.Tensor:
        """The convection column of the window at step j (its first step), from the
        runner's ``column_cache`` (keyed by hour and float32 RK2 weight) or built here
        with ``glide_convect`` and no particles."""
        r = self.r
        st = self.steps[j]
        key = (st.hour, float(np.float32(st.alpha)))
        cache = r.column_cache
        if cache is not None and key in cache:
            return cache[key]
        nb = C.c_size_t()
        _abi.check(_abi.lib.glide_convect_scratch_bytes(r.grid.shape[0], C.byref(nb)), "glide_convect_scratch_bytes")
        with torch.cuda.stream(stream):
            col = torch.zeros(nb.value // 8, dtype=torch.float64, device=r.device)
            a = self._convect_args(r.window_provider(st.hour), j, col, n_particles=0)
            _abi.check(_abi.lib.glide_convect(C.byref(a), stream_handle(stream)), "glide_convect")
        if cache is not None:
            cache[key] = col
        return col

    def next_window_args(self, stream) -> tuple:
        """For grouped launches (``glide_step_batched``): the next window as one launch
        with its convection fused in, from prebuilt met (``packed_provider``) and cached
        columns; nothing is launched but a missing column build. Returns the launch's
        arguments and the objects they point into (keep them until the launch has run).
        With the runner's particle order on, the batch's particles are regrouped by the
        work classes of its previous window (on ``stream``, before the launch)."""
        r = self.r
        if self.done:
            raise RuntimeError("the batch has no window left")
        if r.packed_provider is None or r.footprint.ring > 0:
            raise ValueError("grouped launches need a packed_provider and a dense footprint")
        k = self.next_window
        j0, j1 = self.windows[k]
        self.next_window += 1
        first = self.steps[j0]
        packed = r.packed_provider(first.hour)
        self._record_wind_sum(k, packed, stream)
        noise = self._noise(j0, j1)
        keep = [packed, noise]
        if self.work_key is not None:
            self._reorder(stream_handle(stream))
        a = self._step_args(packed, j0, j1 - j0, 0, 0, noise)  # with the order and work keys, if any
        self.keys_valid = self.work_key is not None  # once the caller's launch has run
        if r.emanuel is not None:
            col = self._column_for(j0, stream)
            with torch.cuda.stream(stream):
                conv = self._fused_convection(first.hour, j0, col)
            a.conv_column, a.conv_step, a.conv_nz = conv["conv_column"], 0, conv["conv_nz"]
            a.conv_uniforms, a.conv_moved = conv["conv_uniforms"], conv["conv_moved"]
            keep += [col, conv["keep"]]
        return a, keep

    def _record_wind_sum(self, k: int, packed: PackedWindow, stream) -> None:
        """Window k's wind sums (computed when its bricks were packed) into the batch's
        per-window table, on ``stream`` after the packing."""
        if self.wind_sum is None:
            return
        if packed.wind_sum is None:
            raise ValueError("diagnostics need packed windows with wind sums (PackedWindow.pack)")
        with torch.cuda.stream(stream):
            self.wind_sum[k].copy_(packed.wind_sum, non_blocking=True)

    def _reorder(self, sh) -> None:
        """Rebuild the particle order from the work keys of the last launch."""
        if self.keys_valid:
            _abi.check(_abi.lib.glide_reorder_by_key(self.state.n, self.work_key.data_ptr(), self.order.data_ptr(),
                                                     self.reorder_scratch.data_ptr(), self.reorder_scratch.numel(),
                                                     sh), "glide_reorder_by_key")
            self.order_valid = True

    def _fused_convection(self, hour: datetime, j: int, scratch: torch.Tensor) -> dict:
        """Fields of the window's convection fused into its first launch (at its first
        step) against a prebuilt column."""
        r, s = self.r, self.state
        moved = torch.zeros(1, dtype=torch.int32, device=r.device)
        u = r.conv_uniform_provider(j) if r.conv_uniform_provider is not None else None
        if u is not None and (tuple(u.shape) != (2, s.n) or u.dtype != torch.float32 or not u.is_contiguous()):
            raise ValueError(f"injected convection uniforms must be contiguous float32 (2, {s.n})")
        self.conv_log.append((hour, moved))
        return {"conv_column": scratch.data_ptr(), "conv_nz": r.grid.shape[0], "conv_moved": moved.data_ptr(),
                "conv_uniforms": None if u is None else u.data_ptr(), "keep": u}

    def _launch_range(self, packed: PackedWindow, j0: int, j1: int, phys_skip: int, noise, sh,
                      conv: dict | None = None) -> None:
        """The window's steps [j0, j1) in launches of ``steps_per_launch`` steps (all in one
        when unset), the particle order rebuilt between launches; the first launch leaves
        out the physics of its first ``phys_skip`` steps (already run before convection),
        and applies ``conv`` (fused convection) at its first step."""
        per = self.r.steps_per_launch or (j1 - j0)
        j = j0
        while j < j1:
            c = min(per, j1 - j)
            if j > j0:
                self._reorder(sh)
            a = self._step_args(packed, j, c, phys_skip if j == j0 else 0, 0, noise, noise_row=j - j0)
            if conv is not None and j == j0:
                a.conv_column, a.conv_step, a.conv_nz = conv["conv_column"], 0, conv["conv_nz"]
                a.conv_uniforms, a.conv_moved = conv["conv_uniforms"], conv["conv_moved"]
            _abi.check(_abi.lib.glide_step(C.byref(a), sh), "glide_step")
            self.keys_valid = self.work_key is not None
            j += c

    def _prepare(self, k: int) -> None:
        """Per-window work that depends only on met: fetch the window, pack its bricks
        and build its convection column (``glide_convect`` with no particles), on the
        prep stream (pipelined: overlapping the previous window's steps) or inline."""
        r = self.r
        j0 = self.windows[k][0]
        first = self.steps[j0]
        slot = k % 2 if self.pipelined else 0
        prep_stream = self.prep_stream if self.pipelined else torch.cuda.current_stream(r.device)
        with torch.cuda.stream(prep_stream):
            if self.slot_free[slot] is not None:
                prep_stream.wait_event(self.slot_free[slot])
            wf = r.window_provider(first.hour)
            if wf.time_start != first.hour:
                raise ValueError(f"window provider returned {wf.time_start} for hour {first.hour}")
            packed = r.packed_for(wf, prep_stream, slot=slot)
            scratch = None
            if r.emanuel is not None:
                scratch = self.conv_scratch[slot]
                a = self._convect_args(wf, j0, scratch, n_particles=0)
                _abi.check(_abi.lib.glide_convect(C.byref(a), stream_handle(prep_stream)), "glide_convect")
            ev = torch.cuda.Event()
            ev.record(prep_stream)
        self.prepared[k] = (wf, packed, scratch, ev)

    def release(self) -> None:
        """Per-batch reclaim (the reference's end-of-batch ``del`` + ``empty_cache``,
        main.py:1656-1673): drop this batch's device working buffers — schedule, per-step
        counters and diagnostic sums, particle order and work keys, convection scratch,
        the windows prepared ahead — so that a long run's device memory stays one batch's
        worth. What ``finish()`` handed out (the particle state, the footprint) stays
        with its holder; ``BatchRunner.release()`` also frees the runner's packed-window
        slots and returns the cached blocks to the driver. The batch can neither step nor
        finish after it. The device is synchronised first: a window prepared ahead on the
        side stream, or a launch still queued, may be using the buffers."""
        torch.cuda.synchronize(self.r.device)
        self.released = True
        self.sched_dev = self.esc = self.act = self.diag_sum = self.wind_sum = None
        self.order = self.work_key = self.reorder_scratch = None
        self.keys_valid = self.order_valid = False
        self.conv_scratch = []
        self.prepared = {}
        self.slot_free = [None, None]
        self.z_edges = None
        self.footprint = self.footprint_out = None

    def step_window(self, stream=None) -> bool:
        """Issue the launches of the next met window; False when the batch is done.
        Each window is an NVTX range named after its hour (for NVIDIA's profilers)."""
        if getattr(self, "released", False):
            raise RuntimeError("this batch was released")
        if self.done:
            return False
        torch.cuda.nvtx.range_push(f"glide window {self.steps[self.windows[self.next_window][0]].hour:%Y-%m-%dT%H}")
        try:
            return self._step_window(stream)
        finally:
            torch.cuda.nvtx.range_pop()

    def _step_window(self, stream) -> bool:
        r = self.r
        k = self.next_window
        j0, j1 = self.windows[k]
        self.next_window += 1
        first = self.steps[j0]
        caller = stream if stream is not None else torch.cuda.current_stream(r.device)
        main = stream if stream is not None else r.step_stream
        if k not in self.prepared:
            self._prepare(k)
        wf, packed, scratch, ready = self.prepared.pop(k)
        main.wait_event(ready)
        self._record_wind_sum(k, packed, main)
        noise = self._noise(j0, j1)
        if main is not caller:  # the caller's work so far (state, noise) comes first
            main.wait_stream(caller)
        sh = stream_handle(main)
        n = j1 - j0
        with torch.cuda.stream(main):
            self._reorder(sh)
            if r.emanuel is not None and r.fuse_convection:
                conv = self._fused_convection(wf.time_start, j0, scratch)
                self._launch_range(packed, j0, j1, 0, noise, sh, conv=conv)
            elif r.emanuel is not None:
                a = self._step_args(packed, j0, 1, 0, 1, noise)
                _abi.check(_abi.lib.glide_step(C.byref(a), sh), "glide_step")
                self.keys_valid = self.work_key is not None
                self._redistribute(wf, j0, scratch, main)
                self._launch_range(packed, j0, j1, 1, noise, sh)
            else:
                self._launch_range(packed, j0, j1, 0, noise, sh)
            done = torch.cuda.Event()
            done.record(main)
            self.slot_free[k % 2 if self.pipelined else 0] = done
            if r.footprint.ring > 0:
                self._flush_completed_bins(j0, j1)
            prov = r.window_provider
            if hasattr(prov, "window_done"):  # streaming provider: release this window, prefetch the next
                prov.window_done(first.hour)
                if not self.done:
                    prov.prefetch(self.steps[self.windows[self.next_window][0]].hour)
        if main is not caller:  # later work on the caller's stream sees this window's results
            caller.wait_stream(main)
        if self.pipelined and not self.done:
            self._prepare(self.next_window)  # overlaps this window's steps
        return True

    def _bins(self, j: int) -> np.ndarray:
        """Time-ago bin of every release at step j (main.py:1459-1465, float32)."""
        el = np.maximum(self.release_end - np.float32(self.steps[j].cursor_off), np.float32(0.0))
        with np.errstate(invalid="ignore"):
            return np.floor(el / np.float32(3600.0))

    def _flush_completed_bins(self, j0: int, j1: int) -> None:
        """After window [j0, j1): hand every bin no later step can reach to the sink and
        clear its ring slot. Bins advance with the cursor, so a bin is complete once the
        next step's bin is past it (or the batch ends)."""
        fp = self.r.footprint
        lo = self._bins(j0)
        hi = self._bins(j1 - 1)
        nxt = self._bins(j1) if j1 < len(self.steps) else np.full_like(hi, np.inf)
        rel = np.nonzero(np.isfinite(lo))[0]
        if rel.size == 0:
            return
        first, last = lo[rel].astype(np.int64), hi[rel].astype(np.int64)
        span = np.maximum(last - first + 1, 0)
        rep = np.repeat(np.arange(rel.size), span)  # (release, bin) pairs in release-major order
        b_all = first[rep] + (np.arange(rep.size) - np.repeat(np.cumsum(span) - span, span))
        keep = (b_all < nxt[rel][rep]) & (b_all >= 0) & (b_all < fp.n_time_bins)
        if not keep.any():
            return
        idx = np.stack([rel[rep][keep], b_all[keep]]).astype(np.int64)
        # through pinned memory: an asynchronous copy, so the host does not wait for the window
        dev_idx = torch.from_numpy(idx).pin_memory().to(self.footprint.device, non_blocking=True)
        ri, bi = dev_idx[0], dev_idx[1]
        # the ring as rows of (release, slot) slices: index_select / index_fill_ enqueue
        # without waiting for the device (a scalar index_put_ through advanced indexing does not)
        rows = self.footprint.view(fp.n_releases * fp.ring, -1)
        flat = ri * fp.ring + bi % fp.ring
        from_rows = getattr(self.sink, "from_rows", None)
        if from_rows is not None:  # the sink reads the slices from the ring and clears their slots
            flat_host = idx[0] * fp.ring + idx[1] % fp.ring
            if np.unique(flat_host).size != flat_host.size:
                raise RuntimeError("ring flush names a ring slot twice")
            from_rows(rows, flat, ri, bi)
            return
        slices = rows.index_select(0, flat).view((-1,) + tuple(self.footprint.shape[2:]))
        self.sink(ri, bi, slices)
        rows.index_fill_(0, flat, 0.0)

    def _convect_args(self, wf: WindowFields, j: int, scratch: torch.Tensor, n_particles: int) -> _abi.ConvectArgs:
        r, s, e = self.r, self.state, self.r.emanuel
        nz, ny, nx = r.grid.shape
        st = self.steps[j]
        a = _abi.ConvectArgs()
        a.n = n_particles
        a.z, a.z_stride = s.z.data_ptr(), 1
        a.rel_off, a.alive, a.active_mask = s.rel_off.data_ptr(), s.alive.data_ptr(), None
        a.sim_length_s = self.sim_length_s
        a.sched = _abi.StepSched(np.float32(st.cursor_off), st.delta, st.alpha, j)
        a.nz, a.ny, a.nx = nz, ny, nx
        for k, snap in enumerate((wf.start, wf.end)):
            a.t[k] = snap["t"].data_ptr()
            a.q[k] = snap["q"].data_ptr()
        a.height3d = None if wf.height3d is None else wf.height3d.data_ptr()
        a.height_level = r.grid.height_level_dev.data_ptr()
        a.pressure_hpa = r.grid.p_hpa_dev.data_ptr()
        a.alpha = st.alpha
        a.closure_c, a.trigger_dtv_k = e.closure_c, e.trigger_dtv_k
        a.min_cape_j_kg, a.min_cloud_depth_m = e.min_cape_j_kg, e.min_cloud_depth_m
        a.seed = r.seed
        a.scratch = scratch.data_ptr()
        return a

    def _redistribute(self, wf: WindowFields, j: int, scratch: torch.Tensor, stream) -> None:
        """The window's convective redistribution against its prebuilt column
        (emanuel.py:720-805)."""
        r, s = self.r, self.state
        moved = torch.zeros(1, dtype=torch.int32, device=r.device)
        a = self._convect_args(wf, j, scratch, n_particles=s.n)
        u = r.conv_uniform_provider(j) if r.conv_uniform_provider is not None else None
        if u is not None and (tuple(u.shape) != (2, s.n) or u.dtype != torch.float32 or not u.is_contiguous()):
            raise ValueError(f"injected convection uniforms must be contiguous float32 (2, {s.n})")
        a.uniforms = None if u is None else u.data_ptr()
        a.n_moved = moved.data_ptr()
        _abi.check(_abi.lib.glide_convect_redistribute(C.byref(a), stream_handle(stream)), "glide_convect_redistribute")
        self.conv_log.append((wf.time_start, moved))

    def capture(self) -> torch.cuda.CUDAGraph:
        """Record every remaining window of the batch — particle order, step launches with
        their fused convection, per-window packing and convection columns — into one CUDA
        graph; ``graph.replay()`` then runs the batch with no host work, and ``finish()``
        reads the results. The met the windows need must already be on the device
        (device-resident window provider or ``packed_provider``), the footprint dense,
        the noise generated, and the runner not pipelined (one stream). Replaying again
        continues from whatever the state tensors hold (new particles can be copied in)."""
        r = self.r
        if r.footprint.ring > 0 or r.noise_provider is not None or r.conv_uniform_provider is not None:
            raise ValueError("capture needs a dense footprint and generated noise")
        if self.pipelined:
            raise ValueError("capture needs BatchRunner(pipeline=False)")
        g = torch.cuda.CUDAGraph()
        s = torch.cuda.Stream(device=r.device)
        s.wait_stream(torch.cuda.current_stream(r.device))
        with torch.cuda.graph(g, stream=s):
            while self.step_window(s):
                pass
        torch.cuda.current_stream(r.device).wait_stream(s)
        return g

    def run(self, stream=None) -> BatchOutput:
        while self.step_window(stream):
            pass
        return self.finish()

    def finish(self) -> BatchOutput:
        if getattr(self, "released", False):
            raise RuntimeError("this batch was released: finish() before release()")
        n = len(self.steps)
        status = int(self.status.item())
        fp = self.footprint if self.r.footprint.ring == 0 else self.footprint_out
        out = BatchOutput(self.state, fp, self.esc[:n].cpu().numpy(), self.act[:n].cpu().numpy(), n,
                          self.conv_log, status)
        if self.diag_sum is not None and n > 0:
            scale = np.array([_abi.GLIDE_DIAG_DEG_SCALE, _abi.GLIDE_DIAG_DEG_SCALE, _abi.GLIDE_DIAG_M_SCALE],
                             dtype=np.float64)
            sums = self.diag_sum[:n].cpu().numpy().astype(np.float64) / scale
            out.diag_pos = (sums / max(1, self.state.n)).astype(np.float32)
            out.diag_wind = self._diag_wind(self.wind_sum.cpu().numpy())
        return out

    def _diag_wind(self, sums: np.ndarray) -> np.ndarray:
        """Per-step grid-mean wind from the windows' sums: the float32 means of the two
        snapshots lerped by the step's RK2 weight as _advection_alpha_wind_mean does
        (main.py:892-938: ``mean_start * (1 - alpha) + mean_end * alpha`` in float32)."""
        ncell = float(np.prod(self.r.grid.shape))
        out = np.zeros((len(self.steps), 3), dtype=np.float32)
        for k, (j0, j1) in enumerate(self.windows):
            m0 = (sums[k, :3] / ncell).astype(np.float32)
            m1 = (sums[k, 3:] / ncell).astype(np.float32)
            alpha = np.asarray([self.steps[j].alpha for j in range(j0, j1)], dtype=np.float64)
            om = (1.0 - alpha).astype(np.float32)[:, None]
            out[j0:j1] = m0[None, :] * om + m1[None, :] * alpha.astype(np.float32)[:, None]
        return out


def launch_grouped(args: list, stream) -> None:
    """Launch ``glide_step`` argument sets (``BatchRun.next_window_args``) as grouped
    launches of up to ``GLIDE_STEP_BATCH_MAX`` batches on ``stream``."""
    cap = _abi.GLIDE_STEP_BATCH_MAX
    for i in range(0, len(args), cap):
        chunk = args[i:i + cap]
        arr = (_abi.StepArgs * len(chunk))(*chunk)
        _abi.check(_abi.lib.glide_step_batched(arr, len(chunk), stream_handle(stream)), "glide_step_batched")


class HostSliceStream:
    """A ring-footprint sink (``BatchRunner(footprint_sink=...)``) that moves the
    completed time-ago slices to pinned host memory on its own copy stream, so the
    device-to-host traffic overlaps the following windows' steps instead of
    delaying them. Each call copies the window's slices and their (release, bin)
    indices into one of ``buffers`` alternating pinned buffers; ``on_host(r_idx,
    b_idx, slices)`` (int64 numpy arrays and a pinned CPU tensor ``[k, Zb, Y, X]``,
    valid during the call) runs on the host once a copy has landed: when its buffer
    is needed again, or at ``drain()``. ``bytes_moved`` counts the slice bytes.
    ``dtype`` is the footprint's value type (float32 or float64)."""

    def __init__(self, device, slice_shape: tuple, capacity: int, on_host: Callable | None = None,
                 buffers: int = 2, dtype: torch.dtype = torch.float32) -> None:
        self.device = torch.device(device)
        self.dtype = dtype
        self.slice_shape = tuple(slice_shape)
        self.on_host = on_host
        self.copy_stream = torch.cuda.Stream(device=self.device)
        self.bufs = [self._alloc(max(1, int(capacity))) for _ in range(max(1, buffers))]
        self.pending: list = [None] * len(self.bufs)
        self.next = 0
        self.bytes_moved = 0

    def _alloc(self, k: int) -> dict:
        return {"slices": torch.empty((k,) + self.slice_shape, dtype=self.dtype).pin_memory(),
                "idx": torch.empty((2, k), dtype=torch.int64).pin_memory()}

    def _deliver(self, slot: int) -> None:
        p = self.pending[slot]
        if p is None:
            return
        done, k = p
        done.synchronize()
        self.pending[slot] = None
        if self.on_host is not None:
            buf = self.bufs[slot]
            idx = buf["idx"][:, :k].numpy()
            self.on_host(idx[0].copy(), idx[1].copy(), buf["slices"][:k])

    def __call__(self, r_idx: torch.Tensor, b_idx: torch.Tensor, slices: torch.Tensor) -> None:
        if slices.dtype != self.dtype:
            raise ValueError(f"HostSliceStream holds {self.dtype} slices, got {slices.dtype} "
                             "(pass dtype= to match the footprint's value type)")
        k = int(slices.shape[0])
        slot = self.next
        self.next = (self.next + 1) % len(self.bufs)
        self._deliver(slot)
        if k > self.bufs[slot]["slices"].shape[0]:
            self.bufs[slot] = self._alloc(k)
        buf = self.bufs[slot]
        ready = torch.cuda.current_stream(self.device).record_event()
        with torch.cuda.stream(self.copy_stream):
            self.copy_stream.wait_event(ready)
            buf["slices"][:k].copy_(slices, non_blocking=True)
            buf["idx"][0, :k].copy_(r_idx, non_blocking=True)
            buf["idx"][1, :k].copy_(b_idx, non_blocking=True)
            for t in (slices, r_idx, b_idx):  # keep their memory until the copies have run
                t.record_stream(self.copy_stream)
            done = self.copy_stream.record_event()
        self.pending[slot] = (done, k)
        self.bytes_moved += slices.numel() * slices.element_size()

    def drain(self) -> None:
        """Waits for every copy in flight and hands it to ``on_host``."""
        for i in range(len(self.bufs)):
            slot = (self.next + i) % len(self.bufs)
            self._deliver(slot)


class BatchRunner:
    """Runs batches of particles backward through hourly met windows on one GPU.

    ``window_provider(hour)`` returns the ``[hour, hour + 1 h]`` window as device
    ``WindowFields`` (for example ``SyntheticMet``'s fields, or
    ``window_from_hourly`` of a reader's ``HourlyMetTensors``). ``noise_provider``
    (parity runs) returns injected normals for a list of step indices; without
    it the kernels draw Philox-4x32-10 normals keyed by ``seed``.
    """

    def __init__(self, *, grid: GridInfo, window_provider: Callable[[datetime], WindowFields], hanna: HannaConfig,
                 footprint: FootprintSpec, domain: DomainSpec, emanuel: EmanuelConfig | None = None,
                 met_dtype: str = "f32", device="cuda", seed: int = 0,
                 noise_provider: Callable | None = None, conv_uniform_provider: Callable | None = None,
                 footprint_sink: Callable | None = None, packed_provider: Callable | None = None,
                 pipeline: bool = True) -> None:
        self.device = torch.device(device)
        self.grid = grid if grid.level_sorted_dev is not None else grid.to_device(self.device)
        self.window_provider = window_provider
        self.hanna = hanna
        self.footprint = footprint
        self.domain = domain
        self.emanuel = emanuel
        self.met_dtype = met_dtype
        self.seed = int(seed)
        self.noise_provider = noise_provider
        self.conv_uniform_provider = conv_uniform_provider
        self.footprint_sink = footprint_sink  # ring mode: sink(release_idx, bin_idx, slices [k, Zb, Y, X])
        # packed_provider(hour) -> PackedWindow: windows packed elsewhere and shared (read-only)
        self.packed_provider = packed_provider
        self.pipeline = bool(pipeline)
        # step-kernel launch shape: None = default_launch_variant(batch size);
        # glide_b200.autotune.tune picks one for a workload
        self.launch_variant: int | None = None
        self.reorder = True  # group particles by work class each window (results do not depend on it)
        self.steps_per_launch: int | None = None  # split each window into launches of this many steps
        self.fuse_convection = True  # convection inside the step kernel (else its own kernel between two steps)
        self.column_cache: dict | None = None  # (hour, alpha) -> prebuilt convection column, shared by batches
        self.diagnostics = True  # per-step mean position and grid-mean wind (BatchOutput.diag_pos / diag_wind)
        self._step_stream = None
        self._slots: list[PackedWindow | None] = [None, None]

    @property
    def step_stream(self) -> torch.cuda.Stream:
        """The stream a batch's launches run on when ``step_window`` is given none: a
        high-priority stream, so that the block scheduler runs the step kernel's blocks
        ahead of the next window's preparation (packing, column build) on the side stream,
        which then fills the SMs the step kernel leaves idle."""
        if self._step_stream is None:
            lo, hi = torch.cuda.Stream.priority_range()
            self._step_stream = torch.cuda.Stream(device=self.device, priority=hi)
        return self._step_stream

    def release(self, return_to_driver: bool = True) -> None:
        """Free the runner's packed-window slots (they are rebuilt on the next window
        packed) and, with ``return_to_driver``, hand the blocks the caching allocator
        keeps back to the driver (``torch.cuda.empty_cache``) — the runner-level half of
        the per-batch reclaim, for a process that runs other work between jobs. The
        device is synchronised first (a batch may still be packing into a slot)."""
        torch.cuda.synchronize(self.device)
        self._slots = [None, None]
        if return_to_driver:
            torch.cuda.empty_cache()

    def packed_for(self, wf: WindowFields, stream=None, slot: int = 0) -> PackedWindow:
        """The packed bricks of ``wf`` (packed into brick slot ``slot`` unless a
        ``packed_provider`` serves prebuilt windows)."""
        if self.packed_provider is not None:
            return self.packed_provider(wf.time_start)
        if self._slots[slot] is None:
            self._slots[slot] = PackedWindow(self.grid, self.met_dtype, self.device)
        pw = self._slots[slot]
        if pw.key != wf.time_start:
            pw.pack(wf, meander_coefficient=self.hanna.meander_coefficient,
                    meander_radius=self.hanna.meander_stencil_radius, build_meander=self.hanna.meander_enabled,
                    stream=stream)
        return pw

    def start(self, state: ParticleState, *, batch_start: datetime, cursor_start: datetime,
              cursor_terminus: datetime, sim_length_s: float, dt_seconds: float,
              max_steps: int | None = None) -> BatchRun:
        steps = plan_steps(batch_start, cursor_start, cursor_terminus, dt_seconds)
        if max_steps is not None:
            steps = steps[:max_steps]
        return BatchRun(self, state, steps, sim_length_s)

    def run(self, state: ParticleState, **kw) -> BatchOutput:
        return self.start(state, **kw).run()
