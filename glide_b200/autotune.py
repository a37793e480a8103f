"""Launch-shape autotuner of the fused step kernel.

The step kernel is compiled for several launch shapes (threads per block x
resident blocks per SM, i.e. register budget); which is fastest depends on the
workload — chiefly the particle count, since a batch of N particles fills
``N / (148 SMs x resident threads)`` waves and a partly filled last wave idles
SMs — and on the met storage type. ``tune`` times every shape on the first full
met window of the batch (on copies of the particle state, so the batch itself
is untouched), keeps the fastest on the runner and caches it per workload
shape. Results do not depend on the shape.
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


def tune(runner: BatchRunner, state: ParticleState, *, windows: int = 1, use_cache: bool = True, **start_kw) -> dict:
    """Times every launch variant on the batch's first full window(s) and sets the
    fastest as ``runner.launch_variant``. ``start_kw`` are ``BatchRunner.start``'s
    schedule arguments. Returns ``{"variant", "times_ms", "cached"}``."""
    key = workload_key(runner, state)
    if use_cache and key in _CACHE:
        runner.launch_variant = _CACHE[key]
        return {"variant": _CACHE[key], "times_ms": {}, "cached": True}
    keep = runner.launch_variant
    times = {}
    stream = torch.cuda.current_stream(runner.device)
    for v, _, _ in launch_variants():
        runner.launch_variant = v
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
        times[v] = e0.elapsed_time(e1) / max(n, 1)
    best = min(times, key=times.get) if times else keep
    runner.launch_variant = best
    _CACHE[key] = best
    return {"variant": best, "times_ms": times, "cached": False}
