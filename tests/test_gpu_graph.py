"""A whole batch captured into one CUDA graph (BatchRun.capture) and replayed gives
the particles and counts of the same batch run window by window."""

from __future__ import annotations

import numpy as np
import pytest
import torch

from fixtures import load_run
from gpu_cases import as_numpy, grid_of, state_from

pytestmark = pytest.mark.gpu


def _runner(run, device, windows):
    from glide_b200.runtime import BatchRunner, DomainSpec, EmanuelConfig, FootprintSpec, HannaConfig

    z = run.z
    nxy = z["grid_nxy"]
    return BatchRunner(
        grid=grid_of(run).to_device(device), window_provider=lambda hour: windows[run.met.index(hour)],
        hanna=HannaConfig(meander_enabled=bool(z["meander"]), max_substeps=int(z["max_substeps"])),
        footprint=FootprintSpec(tuple(z["grid_lon"]), tuple(z["grid_lat"]), int(nxy[0]), int(nxy[1]),
                                tuple(float(e) for e in z["grid_z"]), int(nxy[2]), int(z["release_idx"].max()) + 1),
        domain=DomainSpec(tuple(z["dom_lon"]), tuple(z["dom_lat"]), float(z["dom_alt"])),
        emanuel=EmanuelConfig() if bool(z["convection"]) else None, device=device, seed=321, pipeline=False)


@pytest.mark.parametrize("name", ["run_small", "run_c0"])
def test_captured_batch_matches_eager(cuda_device, name):
    from glide_b200.window import window_from_arrays

    run = load_run(name)
    m = run.met
    times = [m.time(h) for h in range(m.n_snapshots)]
    grid = grid_of(run).to_device(cuda_device)
    windows = {h: window_from_arrays(m.fields, h, times, grid, cuda_device, lowest=int(np.argmin(m.levels)))
               for h in range(m.n_snapshots - 1)}  # all met on the device before the capture
    z = run.z
    kw = dict(batch_start=run.dt_("batch_start"), cursor_start=run.dt_("cursor_start"),
              cursor_terminus=run.dt_("cursor_terminus"), sim_length_s=float(z["sim_length_s"]),
              dt_seconds=float(z["dt_s"]))

    def state():
        return state_from(z["particles0"], z["rel_off"], z["win_end_off"], z["release_idx"], cuda_device)

    eager = _runner(run, cuda_device, windows).start(state(), **kw).run()
    br = _runner(run, cuda_device, windows).start(state(), **kw)
    graph = br.capture()
    graph.replay()
    torch.cuda.synchronize()
    out = br.finish()
    pe, se, ae, fe = as_numpy(eager)
    pg, sg, ag, fg = as_numpy(out)
    np.testing.assert_array_equal(pg, pe)
    for k in se:
        np.testing.assert_array_equal(sg[k], se[k])
    np.testing.assert_array_equal(ag, ae)
    np.testing.assert_array_equal(out.escaped_per_step, eager.escaped_per_step)
    np.testing.assert_array_equal(out.active_per_step, eager.active_per_step)
    np.testing.assert_allclose(fg, fe, rtol=1e-5, atol=1e-9)
    assert out.status == 0
