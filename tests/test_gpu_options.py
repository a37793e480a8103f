"""Scheme options and input layouts beyond the golden defaults, against the oracle
(one step from identical states, the tolerances of test_gpu_parity):

* ``surface_layer_override=True`` (Monin-Obukhov sigma_w and kappa z / sigma timescales
  below 0.1 h, hanna.py:1535-1553) and ``flexpart_tl_floors=False`` (legacy 1 s floor);
* met delivered top-down (descending level order, as from a pressure-level reader);
* bf16 and fp16 met storage run cleanly and stay close to float32 storage;
* empty batches.
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

from fixtures import flipped_levels, load_run, oracle_kwargs
from gpu_cases import as_numpy, cursor_of, run_gpu, runner_for, state_from

pytestmark = pytest.mark.gpu


def _scaled_err(a, b):
    scale = np.maximum(np.abs(b[:3]), np.array([[1.0], [1.0], [10.0]]))
    return (np.abs(a[:3] - b[:3]) / scale).max(axis=0)


def _one_step(run, device, step, hanna_kw=None):
    from oracle.runtime import run_batch

    z = run.z
    if step > 0:
        pre = run_batch(**oracle_kwargs(run, hanna_kw=hanna_kw), max_steps=step)
        p0, st0, alive0 = pre.particles, pre.state, pre.alive
    else:
        p0, st0, alive0 = z["particles0"], None, None
    cur = cursor_of(run, step)
    kw = oracle_kwargs(run, hanna_kw=hanna_kw)
    kw.update(particles=p0, cursor_start=cur)
    ora = run_batch(**kw, max_steps=1, init_state=st0, init_alive=alive0, step_offset=step)
    r = runner_for(run, device, step_offset=step, hanna_kw=hanna_kw)
    st = state_from(p0, z["rel_off"], z["win_end_off"], z["release_idx"], device, st0, alive0)
    out = r.start(st, batch_start=run.dt_("batch_start"), cursor_start=cur, cursor_terminus=run.dt_("cursor_terminus"),
                  sim_length_s=float(z["sim_length_s"]), dt_seconds=float(z["dt_s"]), max_steps=1).run()
    parts, state, alive, fp = as_numpy(out)
    assert out.status == 0
    assert int(out.escaped_per_step[0]) == ora.escaped_per_step[0]
    np.testing.assert_array_equal(alive, ora.alive)
    err = _scaled_err(parts, ora.particles)
    assert err.max() < 1e-4, err.max()
    assert np.mean(err < 1e-5) >= 0.995, np.mean(err < 1e-5)
    return parts, ora


@pytest.mark.parametrize("hanna_kw", [{"surface_layer_override": True}, {"flexpart_tl_floors": False},
                                      {"surface_layer_override": True, "flexpart_tl_floors": False},
                                      {"substep_c": 0.2, "z_ubl_m": 5.0}])
@pytest.mark.parametrize("step", [0, 51])
def test_scheme_options_one_step(cuda_device, hanna_kw, step):
    _one_step(load_run("run_small"), cuda_device, step, hanna_kw)


@pytest.mark.parametrize("step", [0, 51, 111])
def test_descending_levels_one_step(cuda_device, step):
    _one_step(flipped_levels(load_run("run_small")), cuda_device, step)


def test_descending_levels_batch_close_to_ascending(cuda_device):
    run = load_run("run_small")
    a = run_gpu(run, cuda_device)
    b = run_gpu(flipped_levels(run), cuda_device)
    pa, _, aa, fa = as_numpy(a)
    pb, _, ab, fb = as_numpy(b)
    np.testing.assert_array_equal(a.active_per_step, b.active_per_step)
    err = _scaled_err(pb, pa)
    assert np.median(err) < 1e-5
    assert np.abs(fa - fb).sum() / np.abs(fa).sum() < 5e-3


@pytest.mark.parametrize("met_dtype,l1_max", [("bf16", 0.2), ("f16", 0.1)])
def test_reduced_precision_storage(cuda_device, met_dtype, l1_max):
    run = load_run("run_small")
    ref = run_gpu(run, cuda_device)
    out = run_gpu(run, cuda_device, met_dtype=met_dtype)
    pr, _, _, fr = as_numpy(ref)
    po, so, ao, fo = as_numpy(out)
    assert out.status == 0
    assert np.all(np.isfinite(po)) and np.all(po[2] >= 0.0)
    assert abs(int(out.escaped_per_step.sum()) - int(ref.escaped_per_step.sum())) <= 0.1 * max(
        1, int(ref.escaped_per_step.sum()))
    l1 = np.abs(fo - fr).sum() / np.abs(fr).sum()
    assert l1 < l1_max, l1
    # the first step moves every particle by the float32 step to within the storage rounding
    one_ref = run_gpu(run, cuda_device, max_steps=1)
    one = run_gpu(run, cuda_device, met_dtype=met_dtype, max_steps=1)
    e = _scaled_err(as_numpy(one)[0], as_numpy(one_ref)[0])
    assert np.median(e) < (3e-4 if met_dtype == "bf16" else 5e-5), np.median(e)


def test_empty_batch(cuda_device):
    from glide_b200.runtime import ParticleState

    run = load_run("run_small")
    r = runner_for(run, cuda_device, injected=False)
    z = run.z
    st = ParticleState.from_particles(np.zeros((0, 4), np.float32), np.zeros(0, np.float32), np.zeros(0, np.float32),
                                      np.zeros(0, np.int32), cuda_device)
    out = r.start(st, batch_start=run.dt_("batch_start"), cursor_start=run.dt_("cursor_start"),
                  cursor_terminus=run.dt_("cursor_terminus"), sim_length_s=float(z["sim_length_s"]),
                  dt_seconds=float(z["dt_s"])).run()
    assert out.status == 0
    assert out.footprint.abs().sum().item() == 0.0
    assert int(out.active_per_step.sum()) == 0


def test_release_returns_the_batch_memory(cuda_device):
    """Per-batch reclaim: ``BatchRun.release()`` and ``BatchRunner.release()`` free the
    batch's working buffers, so that batch after batch on one runner the device memory
    in use returns to the same level (no growth over a long run), and a released batch
    refuses to step."""
    run = load_run("run_small")
    z = run.z
    r = runner_for(run, cuda_device, injected=False)
    kw = dict(batch_start=run.dt_("batch_start"), cursor_start=run.dt_("cursor_start"),
              cursor_terminus=run.dt_("cursor_terminus"), sim_length_s=float(z["sim_length_s"]),
              dt_seconds=float(z["dt_s"]))
    levels, during = [], []
    for _ in range(3):
        st = state_from(z["particles0"], z["rel_off"], z["win_end_off"], z["release_idx"], cuda_device)
        br = r.start(st, **kw)
        out = br.run()
        assert out.status == 0
        torch.cuda.synchronize(cuda_device)
        during.append(torch.cuda.memory_allocated(cuda_device))
        br.release()
        r.release()
        with pytest.raises(RuntimeError, match="released"):
            br.step_window()
        with pytest.raises(RuntimeError, match="released"):
            br.finish()
        del out, st, br
        torch.cuda.synchronize(cuda_device)
        levels.append(torch.cuda.memory_allocated(cuda_device))
    assert levels[1] == levels[2], levels  # the same level after every batch
    assert all(d > lv for d, lv in zip(during, levels)), (during, levels)  # the working buffers were freed


def test_default_launch_shape_by_batch_size(cuda_device):
    """Without a tuned shape the runner launches one 768-thread block per SM once the
    batch fills every SM with such a block, and 128-thread blocks below that."""
    from glide_b200.autotune import launch_variants
    from glide_b200.runtime import default_launch_variant

    shapes = {v: (t, b) for v, t, b in launch_variants()}
    sms = torch.cuda.get_device_properties(cuda_device).multi_processor_count
    assert shapes[default_launch_variant(1000, cuda_device)] == (128, 6)
    assert shapes[default_launch_variant(sms * 768 - 1, cuda_device)] == (128, 6)
    assert shapes[default_launch_variant(sms * 768, cuda_device)] == (768, 1)
