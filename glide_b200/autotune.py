"""Autotuner of the fused step kernel's launch configuration.

Two knobs, neither of which changes any result:

* the launch shape (threads per block x resident blocks per SM, i.e. register
  budget; the last variant is the general kernel). Which is fastest depends on the
  particle count — a batch of N particles fills ``N / (148 SMs x resident
  threads)`` waves and a partly filled last wave idles SMs — and on the met
  storage type;
* the outer steps per launch: a met window's steps in one launch, or in shorter
  launches with the work-class particle order rebuilt between them, which keeps
  the lanes of a warp on the same branches as particles change regime.

``tune`` times the shapes, then the steps per launch at the best shape, on the
first full met window of the batch (on copies of the particle state, so the
batch itself is untouched), keeps the fastest on the runner and caches it per
workload.
"""

from __future__ import annotations

import ctypes as C
from dataclasses import fields as dc_fields

import torch

from glide_b200 import _abi
from glide_b200.runtime import BatchRunner, ParticleState

_CACHE: dict = {}


def launch_variants() -> list[tuple[int, int, int]]:
    """(variant, threads per block, resident blocks per SM) of every compiled shape."""
    n = C.c_int32()
    _abi.check(_abi.lib.glide_step_launch_variants(C.byref(n)), "glide_step_launch_variants")
    out = []
    for v in range(n.value):
        t, b = C.c_int32(), C.c_int32()
        _abi.check(_abi.lib.glide_step_launch_variant_info(v, C.byref(t), C.byref(b)), "glide_step_launch_variant_info")
        out.append((v, t.value, b.value))
    return out


def _clone(state: ParticleState) -> ParticleState:
    return ParticleState(**{f.name: getattr(state, f.name).clone() for f in dc_fields(state)})


def workload_key(runner: BatchRunner, state: ParticleState) -> tuple:
    dev = torch.cuda.get_device_name(runner.device)
    return (dev, state.n, runner.grid.shape, runner.met_dtype, runner.hanna.meander_enabled,
            runner.emanuel is not None, runner.hanna.max_substeps)


def _time_config(runner: BatchRunner, state: ParticleState, windows: int, start_kw: dict) -> float:
    """Device ms per window of the runner's current configuration on the batch's first
    full window(s), on a copy of the particle state."""
    stream = torch.cuda.current_stream(runner.device)
    run = runner.start(_clone(state), **start_kw)
    run.sink = lambda *a: None  # a tuning run hands no footprint slices to the caller's sink
    # skip a leading partial window (the cursor often starts on an hour boundary)
    if run.windows and run.windows[0][1] - run.windows[0][0] < 0.5 * max(b - a for a, b in run.windows):
        run.step_window()
    run.step_window()  # warm: prepares the next window too
    torch.cuda.synchronize(runner.device)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    n = 0
    while n < windows and run.step_window():
        n += 1
    e1.record(stream)
    torch.cuda.synchronize(runner.device)
    return e0.elapsed_time(e1) / max(n, 1)


def tune(runner: BatchRunner, state: ParticleState, *, windows: int = 1, use_cache: bool = True,
         steps_per_launch_options: tuple = (None, 60, 30), **start_kw) -> dict:
    """Times every launch variant on the batch's first full window(s), then, at the fastest,
    every number of steps per launch in ``steps_per_launch_options`` (None = the whole
    window in one launch; shorter launches rebuild the particle order more often), and sets
    the fastest pair on the runner. ``start_kw`` are ``BatchRunner.start``'s schedule
    arguments. Returns ``{"variant", "steps_per_launch", "times_ms", "steps_times_ms", "cached"}``."""
    key = workload_key(runner, state)
    if use_cache and key in _CACHE:
        runner.launch_variant, runner.steps_per_launch = _CACHE[key]
        return {"variant": runner.launch_variant, "steps_per_launch": runner.steps_per_launch, "times_ms": {},
                "steps_times_ms": {}, "cached": True}
    runner.steps_per_launch = None
    times = {}
    for v, _, _ in launch_variants():
        runner.launch_variant = v
        times[v] = _time_config(runner, state, windows, start_kw)
    best = min(times, key=times.get)
    runner.launch_variant = best
    steps_times = {}
    for spl in steps_per_launch_options:
        runner.steps_per_launch = spl
        steps_times[spl] = times[best] if spl is None else _time_config(runner, state, windows, start_kw)
    best_spl = min(steps_times, key=steps_times.get)
    runner.steps_per_launch = best_spl
    _CACHE[key] = (best, best_spl)
    return {"variant": best, "steps_per_launch": best_spl, "times_ms": times, "steps_times_ms": steps_times,
            "cached": False}
