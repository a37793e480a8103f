"""Trajectory and footprint agreement between three runs of a golden batch fed the
same injected noise and convection uniforms:

* ``ref_cpu``  — the reference's static step path on the CPU (the golden fixture);
* ``ref_cuda`` — the same reference code on CUDA (its eager torch ops; the
  ``torch.compile`` CUDA-graph path draws its own noise, so it cannot be fed the
  injected streams);
* ``b200``     — this library's fused CUDA path.

For each pair it reports the fraction of particles whose position agrees within
1e-6 / 1e-5 / 1e-4 / 1e-3 relative (lon and lat against max(|x|, 1), z against
max(|z|, 10 m)) at the snapshot steps and at the end, the footprint relative L1
and peak-cell error, and whether the per-step active / escaped counts are equal.

Needs a CUDA device and the reference installed as a package directory
(``pip install --no-deps --target <dir> <reference>``) or a source tree:

    python tests/golden/compare_reference_cuda.py --reference baseline/_ref --case c1
"""

from __future__ import annotations

import argparse
import json
import sys
import time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent))
sys.path.insert(0, str(HERE))

import make_golden  # noqa: E402


def _scaled_err(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    scale = np.maximum(np.abs(b[:3]), np.array([[1.0], [1.0], [10.0]]))
    return (np.abs(a[:3] - b[:3]) / scale).max(axis=0)


def compare(a: dict, b: dict) -> dict:
    """Agreement of run ``a`` with run ``b`` (both in the fixture's key layout)."""
    out = {}
    for step, pa, pb in zip(a["snap_steps"], a["snap_particles"], b["snap_particles"]):
        err = _scaled_err(pa, pb)
        out[f"within_1e-5_step{int(step)}"] = float(np.mean(err < 1e-5))
    err = _scaled_err(a["out_particles"], b["out_particles"])
    for tol in (1e-6, 1e-5, 1e-4, 1e-3):
        out[f"within_{tol:.0e}"] = float(np.mean(err < tol))
    out["median_rel_err"] = float(np.median(err))
    out["max_rel_err"] = float(err.max())
    fa, fb = a["out_footprint"].astype(np.float64), b["out_footprint"].astype(np.float64)
    out["footprint_rel_l1"] = float(np.abs(fa - fb).sum() / max(np.abs(fb).sum(), 1e-300))
    out["footprint_peak_rel_err"] = float(abs(fa.max() - fb.max()) / max(abs(fb.max()), 1e-300))
    out["active_equal"] = bool(np.array_equal(a["out_active"], b["out_active"]))
    out["escaped_equal"] = bool(np.array_equal(a["out_escaped"], b["out_escaped"]))
    out["alive_equal"] = bool(np.array_equal(a["out_alive"].astype(bool), b["out_alive"].astype(bool)))
    out["conv_moved"] = [a["out_conv"][:, 1].tolist(), b["out_conv"][:, 1].tolist()]
    if "out_diag_pos" in a and "out_diag_pos" in b:
        dp = np.abs(a["out_diag_pos"].astype(np.float64) - b["out_diag_pos"]) / np.maximum(
            np.abs(b["out_diag_pos"].astype(np.float64)), 1.0)
        out["diag_pos_max_rel"] = float(dp.max())
        dw = np.abs(a["out_diag_wind"].astype(np.float64) - b["out_diag_wind"])
        out["diag_wind_max_abs"] = float(dw.max())
    return out


def run_b200(case: str, golden: dict, device) -> dict:
    """The golden batch through ``BatchRunner`` (window by window, injected noise),
    with snapshots at the fixture's snapshot steps."""
    import torch

    from fixtures import load_run
    from gpu_cases import runner_for, state_from

    run = load_run(f"run_{case}")
    z = run.z
    r = runner_for(run, device)
    kw = dict(batch_start=run.dt_("batch_start"), cursor_start=run.dt_("cursor_start"),
              cursor_terminus=run.dt_("cursor_terminus"), sim_length_s=float(z["sim_length_s"]),
              dt_seconds=float(z["dt_s"]))
    snap_steps = [int(s) for s in golden["snap_steps"]]
    snaps = []
    for k in snap_steps:  # the state after step k: a run of k + 1 steps
        st_k = state_from(z["particles0"], z["rel_off"], z["win_end_off"], z["release_idx"], device)
        s = r.start(st_k, max_steps=k + 1, **kw).run().state
        snaps.append(np.stack([s.lon.cpu().numpy(), s.lat.cpu().numpy(), s.z.cpu().numpy(), s.weight.cpu().numpy()]))
    st = state_from(z["particles0"], z["rel_off"], z["win_end_off"], z["release_idx"], device)
    out = r.start(st, **kw).run()
    torch.cuda.synchronize()
    s = out.state
    res = dict(snap_steps=np.array(snap_steps), snap_particles=np.stack(snaps),
               out_particles=np.stack([s.lon.cpu().numpy(), s.lat.cpu().numpy(), s.z.cpu().numpy(),
                                       s.weight.cpu().numpy()]),
               out_alive=s.alive.cpu().numpy().astype(bool), out_footprint=out.footprint.cpu().numpy(),
               out_active=out.active_per_step, out_escaped=out.escaped_per_step,
               out_conv=np.array([[k, int(m.item())] for k, (_, m) in enumerate(out.convection)]).reshape(-1, 2))
    if out.diag_pos is not None:
        res["out_diag_pos"] = out.diag_pos
        res["out_diag_wind"] = out.diag_wind
    return res


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", required=True, help="reference package directory or source tree")
    ap.add_argument("--case", nargs="*", default=["c1"], choices=["small", "c0", "c1"])
    args = ap.parse_args()
    import torch

    if not torch.cuda.is_available():
        raise SystemExit("needs a CUDA device")
    ref = make_golden._import_reference(Path(args.reference).resolve())
    dev = torch.device("cuda", 0)
    for case in args.case:
        golden = dict(np.load(HERE / f"run_{case}.npz"))
        t = time.perf_counter()
        b200 = run_b200(case, golden, dev)
        t_b200 = time.perf_counter() - t
        print(f"{case}: b200 done in {t_b200:.1f} s", file=sys.stderr, flush=True)
        t = time.perf_counter()
        ref_cuda = make_golden.drive_batch(ref, case, make_golden.NOISE_SEEDS[case], device="cuda",
                                           snap_every=make_golden.SNAP_EVERY[case])
        t_ref = time.perf_counter() - t
        print(f"{case}: reference on CUDA done in {t_ref:.1f} s", file=sys.stderr, flush=True)
        report = {
            "particles": int(golden["particles0"].shape[1]), "steps": int(golden["n_steps"]),
            "ref_cuda_vs_ref_cpu": compare(ref_cuda, golden),
            "b200_vs_ref_cpu": compare(b200, golden),
            "b200_vs_ref_cuda": compare(b200, ref_cuda),
            "wall_s": {"ref_cuda": t_ref, "b200": t_b200},
        }
        print(json.dumps({case: report}), flush=True)


if __name__ == "__main__":
    main()
