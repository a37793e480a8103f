"""The FP64 footprint mode and the per-step diagnostics on the device.

FP64 footprint (``FootprintSpec(value_dtype="f64")``, ``FootprintGridderB200(dtype=
torch.float64)``; the reference's ``FootprintGridder(dtype=torch.float64)``,
src/lpdm/footprint_gridder.py:50-115): each contribution weight * dt formed and
summed in FP64. Checked against the oracle's FP64 gridder on identical positions
(teacher-forced first step: to 1e-12 relative), against the float32 mode of the same
run (same trajectories: within float32 rounding), through the stand-alone
accumulate, the ring and the sparse compaction (bit-exact round trips).

Diagnostics (main.py:1565-1566): the per-step mean particle position summed on the
device in FP64, and the grid-mean wind from the window sums, against the reference's
golden rows and against the run's own final state.
"""

from __future__ import annotations

import dataclasses

import numpy as np
import pytest
import torch

from fixtures import load_run, oracle_kwargs
from gpu_cases import as_numpy, run_gpu, runner_for, state_from

pytestmark = pytest.mark.gpu


def _u64(a):
    return np.ascontiguousarray(a, dtype=np.float64).view(np.uint64)


def test_first_step_fp64_footprint_matches_oracle(cuda_device):
    """From the release state the first step's positions are bit-identical to the oracle's,
    so the FP64 footprint sums the same contributions: equal to 1e-12 relative."""
    from oracle.runtime import run_batch

    run = load_run("run_small")
    out = run_gpu(run, cuda_device, max_steps=1, fp_dtype="f64")
    assert out.status == 0
    assert out.footprint.dtype == torch.float64
    ora = run_batch(**oracle_kwargs(run), max_steps=1, fp_dtype=np.float64)
    fp = out.footprint.cpu().numpy()
    assert ora.footprint.dtype == np.float64
    np.testing.assert_allclose(fp, ora.footprint, rtol=1e-12, atol=0.0)


@pytest.mark.parametrize("name", ["run_small", "run_c0"])
def test_fp64_footprint_is_the_float32_run_in_fp64(cuda_device, name):
    """Same trajectories (the footprint mode does not touch them), footprints within
    float32 rounding of each other; the FP64 one against the oracle's FP64 gridder within
    the batch tolerance."""
    from oracle.runtime import run_batch

    run = load_run(name)
    o32 = run_gpu(run, cuda_device)
    o64 = run_gpu(run, cuda_device, fp_dtype="f64")
    p32, _, a32, f32 = as_numpy(o32)
    p64, _, a64, f64 = as_numpy(o64)
    np.testing.assert_array_equal(p32, p64)
    np.testing.assert_array_equal(a32, a64)
    assert f64.dtype == np.float64
    # the float32 mode rounds each cell's running total at every flush of a residence sum
    assert np.abs(f64 - f32).sum() <= 3e-5 * np.abs(f64).sum()
    r64 = run["out_footprint_f64"]  # the reference's trajectories through its float64 gridder
    assert np.abs(f64 - r64).sum() / np.abs(r64).sum() < 5e-3
    ora = run_batch(**oracle_kwargs(run), fp_dtype=np.float64)
    assert np.abs(f64 - ora.footprint).sum() / np.abs(ora.footprint).sum() < 5e-3
    assert abs(f64.sum() - ora.footprint.sum()) / ora.footprint.sum() < 1e-3


def test_gridder_fp64_accumulate_matches_oracle(cuda_device):
    """FootprintGridderB200(dtype=torch.float64).accumulate (glide_footprint_accumulate
    with value_f64) against the oracle's FP64 scatter-add on the same positions: equal to
    1e-12 relative (only the order of the FP64 additions differs)."""
    from oracle.runtime import GridSpec, accumulate

    from glide_b200.schemes import FootprintGridderB200

    rng = np.random.default_rng(3)
    n = 50_000
    g = GridSpec((0.0, 4.0), (40.0, 43.0), 16, 12, (0.0, 100.0, 500.0), 3, 2)
    p = np.stack([rng.uniform(-0.2, 4.2, n), rng.uniform(39.8, 43.2, n), rng.uniform(-5, 600, n),
                  rng.uniform(0.5, 1.5, n) / n]).astype(np.float32)
    # many particles in few cells: the warp-aggregated atomics are exercised
    p[:2, : n // 2] = np.float32([1.1, 41.3])[:, None]
    active = rng.random(n) < 0.9
    t_idx = rng.integers(-1, 4, n)
    ridx = rng.integers(0, 3, n)
    gr = FootprintGridderB200(g.lon_bounds, g.lat_bounds, g.z_edges, g.n_time_bins, g.n_y, g.n_x, n_releases=2,
                              device=cuda_device, dtype=torch.float64)
    pt = torch.from_numpy(p.T.copy()).to(cuda_device)
    for _ in range(2):
        gr.accumulate(pt[:, :3], torch.from_numpy(active).to(cuda_device), pt[:, 3],
                      torch.from_numpy(t_idx).to(cuda_device), torch.from_numpy(ridx).to(cuda_device), 30.0)
    fp = np.zeros(int(np.prod(g.shape)), dtype=np.float64)
    for _ in range(2):
        accumulate(fp, p[:3], active, p[3], t_idx, ridx, g, 30.0, np.float32, np.float64)
    got = gr.tensor.cpu().numpy().reshape(-1)
    assert gr.tensor.dtype == torch.float64
    np.testing.assert_allclose(got, fp, rtol=1e-12, atol=1e-300)
    assert np.count_nonzero(got) == np.count_nonzero(fp)


@pytest.mark.parametrize("cells", [1, 2049, 112681])
def test_compact_fp64_rows_bit_exact(cuda_device, cells):
    from oracle import sparse_slices as osp

    from glide_b200.sparse import compact_rows

    rng = np.random.default_rng(cells)
    x = np.zeros((5, cells), dtype=np.float64)
    mask = rng.random(x.shape) < 0.05
    x[mask] = rng.gamma(0.5, 2e-3, int(mask.sum()))
    x[1] = 0.0
    x[2] = rng.normal(size=cells)
    x[2][x[2] == 0.0] = 1.0
    sp = np.array([-0.0, np.nan, np.inf, 5e-324, 1e-310], dtype=np.float64)[: min(5, cells)]
    x[3, : sp.size] = sp
    rows = torch.from_numpy(x).to(cuda_device)
    sel = np.array([2, 1, 3, 0], dtype=np.int64)
    off, cell, val = compact_rows(rows, torch.from_numpy(sel).to(cuda_device), clear=True)
    torch.cuda.synchronize()
    o_off, o_cell, o_val = osp.compact(x[sel])
    off = off.cpu().numpy()
    np.testing.assert_array_equal(off, o_off)
    total = int(off[-1])
    assert val.dtype == torch.float64
    np.testing.assert_array_equal(cell[:total].cpu().numpy(), o_cell)
    np.testing.assert_array_equal(_u64(val[:total].cpu().numpy()), _u64(o_val))
    after = rows.cpu().numpy()
    assert not _u64(after[sel]).any()
    np.testing.assert_array_equal(_u64(after[4]), _u64(x[4]))


def test_ring_fp64_footprint_matches_dense(cuda_device):
    """The ring layout in FP64 (two live slices per release, flushed to the dense output):
    equal to the dense FP64 footprint of the same run."""
    run = load_run("run_small")
    dense = run_gpu(run, cuda_device, fp_dtype="f64").footprint.cpu().numpy()
    r = runner_for(run, cuda_device, fp_dtype="f64")
    r.footprint = dataclasses.replace(r.footprint, ring=2)
    z = run.z
    st = state_from(z["particles0"], z["rel_off"], z["win_end_off"], z["release_idx"], cuda_device)
    out = r.start(st, batch_start=run.dt_("batch_start"), cursor_start=run.dt_("cursor_start"),
                  cursor_terminus=run.dt_("cursor_terminus"), sim_length_s=float(z["sim_length_s"]),
                  dt_seconds=float(z["dt_s"])).run()
    assert out.status == 0 and out.footprint.dtype == torch.float64
    np.testing.assert_allclose(out.footprint.cpu().numpy(), dense, rtol=1e-12, atol=1e-300)


@pytest.mark.parametrize("name", ["run_small", "run_c0", "run_c1"])
def test_diagnostics_match_reference(cuda_device, name):
    """Grid-mean wind within float32 rounding of the reference's rows at every step; the
    mean position equal at the first step, within the batch's trajectory spread later
    (1e-6 at the EUROPE-box case), and equal to the mean of the run's own final state at
    the last step."""
    run = load_run(name)
    out = run_gpu(run, cuda_device)
    assert out.diag_pos is not None and out.diag_pos.shape == (out.n_steps, 3)
    gp = run["out_diag_pos"].astype(np.float64)
    pos = np.abs(out.diag_pos.astype(np.float64) - gp) / np.maximum(np.abs(gp), 1.0)
    wind = np.abs(out.diag_wind.astype(np.float64) - run["out_diag_wind"])
    assert wind.max() < 5e-6, wind.max()
    assert pos[0].max() < 1e-6, pos[0]
    # small and c0: the trajectory spread the reference's own CUDA path shows against its
    # CPU path (1.5e-3 at c0)
    assert pos.max() < (1e-6 if name == "run_c1" else 5e-3), pos.max()
    parts, _, _, _ = as_numpy(out)
    own = parts[:3].astype(np.float64).mean(axis=1).astype(np.float32)
    np.testing.assert_allclose(out.diag_pos[-1], own, rtol=1e-6)  # sums of positions quantised to 2^-20 deg, 2^-10 m
    rows = out.diagnostic_rows()
    assert len(rows) == out.n_steps and rows[-1]["alive_particles"] == int(out.state.alive.sum().item())


def test_diagnostics_do_not_change_results(cuda_device):
    run = load_run("run_small")
    a = run_gpu(run, cuda_device)
    r = runner_for(run, cuda_device)
    r.diagnostics = False
    z = run.z
    st = state_from(z["particles0"], z["rel_off"], z["win_end_off"], z["release_idx"], cuda_device)
    b = r.start(st, batch_start=run.dt_("batch_start"), cursor_start=run.dt_("cursor_start"),
                cursor_terminus=run.dt_("cursor_terminus"), sim_length_s=float(z["sim_length_s"]),
                dt_seconds=float(z["dt_s"])).run()
    assert b.diag_pos is None
    pa, sa, aa, fa = as_numpy(a)
    pb, sb, ab, fb = as_numpy(b)
    np.testing.assert_array_equal(pa, pb)
    np.testing.assert_array_equal(aa, ab)
    np.testing.assert_allclose(fa, fb, rtol=1e-6, atol=1e-12)
