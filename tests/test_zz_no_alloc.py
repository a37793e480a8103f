"""The allocation-free convection entry point, ``glide_convect_noalloc``.

Callers that cannot allocate device memory (a serving loop whose HBM budget is
already committed, a process whose framework allocator owns nearly all device
memory, a foreign-language caller without a device allocator) use this entry
point: it keeps its scratch in a static device array of the library instead of
a caller buffer. These tests call it through the C ABI and check that its
output equals ``glide_convect``'s (with a caller scratch buffer) on the same
inputs — bit for bit, the tolerance the convection parity uses here being
exact, since both run the same kernels — on two calls in a row on different
met windows (the second call starts from the first call's leftover scratch), on a
call whose column does not fire after one that did, and on shorter columns after a
longer one.
This file is collected last so that a failure here leaves every other test run.
"""

from __future__ import annotations

import ctypes as C

import numpy as np
import pytest
import torch

from fixtures import conv_uniforms, load_run
from glide_b200 import _abi


def _args(run, h: int, z: torch.Tensor, moved: torch.Tensor, dev, keep: list, nz_use: int | None = None,
          min_cape: float = 50.0) -> _abi.ConvectArgs:
    """Arguments of one convection call on window h; ``nz_use`` keeps only the lowest
    levels of the column, ``min_cape`` is the trigger's CAPE threshold."""
    m = run.met
    n = z.numel()
    a = _abi.ConvectArgs()
    a.n = n
    a.z, a.z_stride = z.data_ptr(), 1
    mask = torch.ones(n, dtype=torch.uint8, device=dev)
    a.active_mask = mask.data_ptr()
    nz, ny, nx = m.fields["t"].shape[1:]
    nz = nz if nz_use is None else nz_use
    a.nz, a.ny, a.nx = nz, ny, nx
    for k in (0, 1):
        t = torch.as_tensor(m.fields["t"][h + k][:nz], device=dev).contiguous()
        q = torch.as_tensor(m.fields["q"][h + k][:nz], device=dev).contiguous()
        keep += [t, q]
        a.t[k], a.q[k] = t.data_ptr(), q.data_ptr()
    lev = torch.as_tensor(np.asarray(m.levels, dtype=np.float32)[:nz], device=dev)
    p = torch.as_tensor(np.asarray(m.p_hpa, dtype=np.float32)[:nz], device=dev)
    u = torch.as_tensor(np.stack(conv_uniforms(int(run["conv_seed"]), h, n)), device=dev).contiguous()
    keep += [mask, lev, p, u]
    a.height3d, a.height_level, a.pressure_hpa = None, lev.data_ptr(), p.data_ptr()
    a.alpha = 0.25 + 0.5 * h
    a.closure_c, a.trigger_dtv_k, a.min_cape_j_kg, a.min_cloud_depth_m = 0.03, 0.9, min_cape, 500.0
    a.uniforms = u.data_ptr()
    a.scratch = None
    a.n_moved = moved.data_ptr()
    return a


def _call(fn_name: str, run, h: int, z0: torch.Tensor, dev, scratch: torch.Tensor | None = None, **kw):
    keep: list = []
    z = z0.clone()
    moved = torch.zeros(1, dtype=torch.int32, device=dev)
    a = _args(run, h, z, moved, dev, keep, **kw)
    if scratch is not None:
        a.scratch = scratch.data_ptr()
    stream = torch.cuda.current_stream().cuda_stream
    _abi.check(getattr(_abi.lib, fn_name)(C.byref(a), stream), fn_name)
    torch.cuda.synchronize()
    return z.cpu().numpy(), int(moved.item())


@pytest.mark.gpu
def test_noalloc_matches_caller_scratch_on_two_calls(cuda_device):
    run = load_run("run_small")
    z0 = torch.as_tensor(run["particles0"][2].copy(), device=cuda_device)
    nz = run.met.fields["t"].shape[1]
    nb = C.c_size_t()
    _abi.check(_abi.lib.glide_convect_scratch_bytes(nz, C.byref(nb)), "glide_convect_scratch_bytes")
    for h in (1, 0):  # two calls in a row, on two different met windows
        scratch = torch.zeros(nb.value // 8, dtype=torch.float64, device=cuda_device)
        z_ref, moved_ref = _call("glide_convect", run, h, z0, cuda_device, scratch)
        z_new, moved_new = _call("glide_convect_noalloc", run, h, z0, cuda_device)
        assert moved_ref > 0  # the column triggers and particles move
        assert moved_new == moved_ref
        np.testing.assert_array_equal(z_new, z_ref)


@pytest.mark.gpu
def test_noalloc_after_a_firing_call(cuda_device):
    """Each call writes every part of the shared array it reads: a call whose column does
    not fire, after one that did, moves nothing; a call on a shorter column (fewer levels,
    so a different layout of the array) after a longer one equals glide_convect on it."""
    run = load_run("run_small")
    z0 = torch.as_tensor(run["particles0"][2].copy(), device=cuda_device)
    nz = run.met.fields["t"].shape[1]
    z_fire, moved_fire = _call("glide_convect_noalloc", run, 1, z0, cuda_device)
    assert moved_fire > 0
    z_quiet, moved_quiet = _call("glide_convect_noalloc", run, 1, z0, cuda_device, min_cape=1e9)
    assert moved_quiet == 0
    np.testing.assert_array_equal(z_quiet, z0.cpu().numpy())
    _call("glide_convect_noalloc", run, 1, z0, cuda_device)  # the full column fires again
    for nz_use in (nz - 2, nz // 2):
        nb = C.c_size_t()
        _abi.check(_abi.lib.glide_convect_scratch_bytes(nz_use, C.byref(nb)), "glide_convect_scratch_bytes")
        scratch = torch.zeros(nb.value // 8, dtype=torch.float64, device=cuda_device)
        z_ref, moved_ref = _call("glide_convect", run, 0, z0, cuda_device, scratch, nz_use=nz_use)
        z_new, moved_new = _call("glide_convect_noalloc", run, 0, z0, cuda_device, nz_use=nz_use)
        assert moved_new == moved_ref
        np.testing.assert_array_equal(z_new, z_ref)


def test_noalloc_rejects_grids_beyond_its_scratch():
    a = _abi.ConvectArgs()
    a.nz, a.ny, a.nx = 129, 4, 4
    assert _abi.lib.glide_convect_noalloc(C.byref(a), None) == 1
    assert "exceeds the 128 levels" in _abi.last_error()
