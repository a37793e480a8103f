"""Grouped launches (glide_step_batched): batches of different sizes, schedules and
met windows stepped together in one launch per window give exactly the particles
each batch gets alone (noise and state are keyed by each batch's own particle and
step numbers), with injected noise (the general kernel) and generated noise (the
fast kernel)."""

from __future__ import annotations

import numpy as np
import pytest
import torch

from fixtures import load_run
from gpu_cases import as_numpy, runner_for, state_from

pytestmark = pytest.mark.gpu


def _prepared_runner(run, device, injected):
    from glide_b200.window import PackedWindow

    r = runner_for(run, device, injected=injected)
    cache = {}

    def packed(hour):
        if hour not in cache:
            pw = PackedWindow(r.grid, r.met_dtype, device)
            pw.pack(r.window_provider(hour), meander_coefficient=r.hanna.meander_coefficient,
                    meander_radius=r.hanna.meander_stencil_radius, build_meander=r.hanna.meander_enabled)
            cache[hour] = pw
        return cache[hour]

    r.packed_provider = packed
    r.column_cache = {}
    return r


def _start(run, r, device):
    z = run.z
    st = state_from(z["particles0"], z["rel_off"], z["win_end_off"], z["release_idx"], device)
    return r.start(st, batch_start=run.dt_("batch_start"), cursor_start=run.dt_("cursor_start"),
                   cursor_terminus=run.dt_("cursor_terminus"), sim_length_s=float(z["sim_length_s"]),
                   dt_seconds=float(z["dt_s"]))


@pytest.mark.parametrize("injected", [True, False])
def test_grouped_windows_match_each_batch_alone(cuda_device, injected):
    from glide_b200.runtime import launch_grouped

    runs = [load_run("run_small"), load_run("run_c0")]
    alone = []
    for run in runs:
        r = _prepared_runner(run, cuda_device, injected)
        br = _start(run, r, cuda_device)
        while not br.done:
            a, keep = br.next_window_args(torch.cuda.current_stream())
            launch_grouped([a], torch.cuda.current_stream())
        alone.append(br.finish())
    batches = [_start(run, _prepared_runner(run, cuda_device, injected), cuda_device) for run in runs]
    stream = torch.cuda.current_stream()
    launches = 0
    while not all(b.done for b in batches):
        args, keep = [], []
        for b in batches:
            if not b.done:
                a, k = b.next_window_args(stream)
                args.append(a)
                keep.append(k)
        launch_grouped(args, stream)
        launches += 1
    together = [b.finish() for b in batches]
    assert launches == max(len(b.windows) for b in batches)
    for x, y in zip(alone, together):
        px, sx, ax, fx = as_numpy(x)
        py, sy, ay, fy = as_numpy(y)
        np.testing.assert_array_equal(px, py)
        for k in sx:
            np.testing.assert_array_equal(sx[k], sy[k])
        np.testing.assert_array_equal(ax, ay)
        np.testing.assert_array_equal(x.escaped_per_step, y.escaped_per_step)
        np.testing.assert_array_equal(x.active_per_step, y.active_per_step)
        np.testing.assert_allclose(fy, fx, rtol=1e-5, atol=1e-9)
        assert x.status == 0 and y.status == 0


def test_grouped_window_matches_step_window(cuda_device):
    """The grouped path (cached columns, no reorder) equals the runtime's per-window
    launches on the golden batch."""
    from gpu_cases import run_gpu

    from glide_b200.runtime import launch_grouped

    run = load_run("run_small")
    ref = run_gpu(run, cuda_device)
    br = _start(run, _prepared_runner(run, cuda_device, True), cuda_device)
    while not br.done:
        a, keep = br.next_window_args(torch.cuda.current_stream())
        launch_grouped([a], torch.cuda.current_stream())
    out = br.finish()
    np.testing.assert_array_equal(as_numpy(out)[0], as_numpy(ref)[0])
    np.testing.assert_array_equal(out.escaped_per_step, ref.escaped_per_step)


def test_batched_argument_checks(cuda_device):
    from glide_b200 import _abi

    arr = (_abi.StepArgs * 1)()
    assert _abi.lib.glide_step_batched(arr, _abi.GLIDE_STEP_BATCH_MAX + 1, None) == 1
    assert "count" in _abi.last_error()
    assert _abi.lib.glide_step_batched(arr, 0, None) == 0
