"""Particle ordering by work class (glide_reorder_by_key) and the step kernel's
order / work_key arguments: the permutation equals a stable descending sort of
the keys, and stepping through it changes no result."""

from __future__ import annotations

import ctypes as C

import numpy as np
import pytest
import torch

from fixtures import load_run
from gpu_cases import as_numpy, run_gpu

pytestmark = pytest.mark.gpu


def _reorder(keys: np.ndarray, device) -> np.ndarray:
    from glide_b200 import _abi

    n = keys.size
    nb = C.c_size_t()
    _abi.check(_abi.lib.glide_reorder_scratch_bytes(n, C.byref(nb)), "glide_reorder_scratch_bytes")
    key = torch.from_numpy(keys).to(device)
    order = torch.full((max(n, 1),), -7, dtype=torch.int32, device=device)
    scratch = torch.empty(nb.value, dtype=torch.uint8, device=device)
    stream = torch.cuda.current_stream(device)
    _abi.check(_abi.lib.glide_reorder_by_key(n, key.data_ptr() if n else None, order.data_ptr(), scratch.data_ptr(),
                                             nb.value, stream.cuda_stream), "glide_reorder_by_key")
    torch.cuda.synchronize(device)
    return order[:n].cpu().numpy()


def _expected(keys: np.ndarray) -> np.ndarray:
    top = 63  # GLIDE_WORK_PENDING: the largest class
    return np.argsort(top - np.minimum(keys.astype(np.int64), top), kind="stable").astype(np.int32)


@pytest.mark.parametrize("n", [1, 31, 1023, 1024, 1025, 4096 + 77, 200_001])
def test_reorder_is_a_stable_descending_sort(cuda_device, n):
    rng = np.random.default_rng(n)
    keys = rng.integers(0, 61, n).astype(np.uint8)
    keys[rng.random(n) < 0.1] = 63
    keys[rng.random(n) < 0.01] = 200  # counts as 63
    np.testing.assert_array_equal(_reorder(keys, cuda_device), _expected(keys))


def test_reorder_single_class_and_empty(cuda_device):
    keys = np.full(5000, 3, np.uint8)
    np.testing.assert_array_equal(_reorder(keys, cuda_device), np.arange(5000, dtype=np.int32))
    assert _reorder(np.zeros(0, np.uint8), cuda_device).size == 0


def test_reorder_rejects_small_scratch(cuda_device):
    from glide_b200 import _abi

    key = torch.zeros(3000, dtype=torch.uint8, device=cuda_device)
    order = torch.zeros(3000, dtype=torch.int32, device=cuda_device)
    scratch = torch.zeros(16, dtype=torch.uint8, device=cuda_device)
    st = _abi.lib.glide_reorder_by_key(3000, key.data_ptr(), order.data_ptr(), scratch.data_ptr(), 16, None)
    assert st == 1 and "scratch" in _abi.last_error()


@pytest.mark.parametrize("name", ["run_small", "run_c0"])
def test_ordered_steps_give_the_same_results(cuda_device, name):
    """Stepping through the work-class order is bit-identical to the identity order
    (noise and state are keyed by particle index; only float atomics of the footprint
    may sum in another order)."""
    run = load_run(name)
    a = run_gpu(run, cuda_device, reorder=False)
    b = run_gpu(run, cuda_device, reorder=True)
    pa, sa, aa, fa = as_numpy(a)
    pb, sb, ab, fb = as_numpy(b)
    np.testing.assert_array_equal(pa, pb)
    for k in sa:
        np.testing.assert_array_equal(sa[k], sb[k])
    np.testing.assert_array_equal(aa, ab)
    np.testing.assert_array_equal(a.escaped_per_step, b.escaped_per_step)
    np.testing.assert_array_equal(a.active_per_step, b.active_per_step)
    np.testing.assert_allclose(fb, fa, rtol=1e-5, atol=1e-9)
    assert a.status == 0 and b.status == 0


def test_ordered_steps_generated_noise(cuda_device):
    run = load_run("run_small")
    a = as_numpy(run_gpu(run, cuda_device, reorder=False, injected=False))
    b = as_numpy(run_gpu(run, cuda_device, reorder=True, injected=False))
    np.testing.assert_array_equal(a[0], b[0])
    np.testing.assert_array_equal(a[2], b[2])


@pytest.mark.parametrize("name,injected", [("run_small", True), ("run_small", False), ("run_c0", True)])
def test_steps_per_launch_gives_the_same_results(cuda_device, name, injected):
    """Windows split into launches of 7 steps, the order rebuilt between them, step
    every particle exactly as one launch per window does (injected noise rows offset
    per launch; generated noise keyed by step)."""
    run = load_run(name)
    a = run_gpu(run, cuda_device, injected=injected)
    b = run_gpu(run, cuda_device, injected=injected, steps_per_launch=7)
    pa, sa, aa, fa = as_numpy(a)
    pb, sb, ab, fb = as_numpy(b)
    np.testing.assert_array_equal(pa, pb)
    for k in sa:
        np.testing.assert_array_equal(sa[k], sb[k])
    np.testing.assert_array_equal(aa, ab)
    np.testing.assert_array_equal(a.escaped_per_step, b.escaped_per_step)
    np.testing.assert_array_equal(a.active_per_step, b.active_per_step)
    # each launch ends by flushing the particles' register-held residence sums, so shorter
    # launches group the float32 additions differently (observed up to 1.1e-5 relative)
    np.testing.assert_allclose(fb, fa, rtol=1e-4, atol=1e-9)


def test_work_keys_and_bad_order(cuda_device):
    """The work keys a window writes: DONE for escaped particles, a class 1..45 (substeps
    x height band x stability regime) or PENDING for live ones; an order entry outside
    [0, n) is skipped and flagged."""
    from glide_b200 import _abi
    from glide_b200.runtime import stream_handle
    from gpu_cases import runner_for, state_from

    run = load_run("run_small")
    z = run.z
    r = runner_for(run, cuda_device)
    st = state_from(z["particles0"], z["rel_off"], z["win_end_off"], z["release_idx"], cuda_device)
    br = r.start(st, batch_start=run.dt_("batch_start"), cursor_start=run.dt_("cursor_start"),
                 cursor_terminus=run.dt_("cursor_terminus"), sim_length_s=float(z["sim_length_s"]),
                 dt_seconds=float(z["dt_s"]))
    br.step_window()
    torch.cuda.synchronize()
    keys = br.work_key.cpu().numpy()
    alive = st.alive.cpu().numpy().astype(bool)
    ms = int(z["max_substeps"])
    assert np.all(keys[~alive] == _abi.GLIDE_WORK_DONE)
    live = keys[alive].astype(np.int64)
    stepped = (live >= 1) & (live <= 45)
    assert np.all(stepped | (live == _abi.GLIDE_WORK_PENDING))
    assert np.any(stepped)
    cls = live[stepped] - 1
    k = cls % 3 + 1  # substeps (capped at 3)
    band = (cls // 3) % 5  # height band relative to the BL top
    regime = cls // 15  # stable / neutral / unstable
    assert np.all(k <= min(ms, 3)) and np.all(band <= 4) and np.all(regime <= 2)
    assert len(np.unique(band)) > 1  # the batch spans several height bands

    # one single-step launch of the next window through a corrupted permutation
    k = br.next_window
    if k not in br.prepared:
        br._prepare(k)
    _, packed, _, ready = br.prepared.pop(k)
    stream = torch.cuda.current_stream(cuda_device)
    stream.wait_event(ready)
    bad = torch.arange(st.n, dtype=torch.int32, device=cuda_device)
    bad[0] = -1
    bad[1] = st.n + 5
    a = br._step_args(packed, br.windows[k][0], 1, 0, 1, None)
    a.order = bad.data_ptr()
    _abi.check(_abi.lib.glide_step(C.byref(a), stream_handle(stream)), "glide_step")
    torch.cuda.synchronize()
    assert int(br.status.item()) & _abi.GLIDE_STATUS_BAD_ORDER
