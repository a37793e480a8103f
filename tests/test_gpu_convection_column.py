"""The convection column ``glide_convect`` builds for a met window against the FP64
oracle (``oracle.convection.build_column``, the restatement of emanuel.py:570-689 and
720-770): trigger, LCL / LNB levels, CAPE, cloud-base mass flux and the backward
transition CDF, on synthetic columns of 12, 60 and 90 levels. Up to 73 levels the
kernel builds the nz x nz matrix in shared memory, above that in the caller's
scratch buffer, so both forms are covered; the parcel lift's parallel bisection runs
in both.
"""

from __future__ import annotations

import ctypes as C

import numpy as np
import pytest
import torch

from fixtures import met_from_synthetic
from glide_b200 import _abi
from glide_b200.synthetic import SyntheticMet, SyntheticMetSpec
from oracle import convection as oconv

# trigger thresholds low enough that every synthetic column fires; the values as the C
# ABI carries them (float32, as the reference's float32 tensors use the scheme's
# Python floats), so that the FP64 oracle starts from the same closure constant
PARAMS = {k: float(np.float32(v)) for k, v in
          dict(closure_c=0.03, trigger_dtv_k=-50.0, min_cape_j_kg=0.0, min_cloud_depth_m=0.0).items()}


def _column_on_device(met, h: int, alpha: float, dev) -> np.ndarray:
    """glide_convect with no particles: the window's column, read back from the scratch."""
    t, q = met.fields["t"], met.fields["q"]
    nz, ny, nx = t.shape[1:]
    keep = []
    a = _abi.ConvectArgs()
    a.n = 0
    a.z_stride = 1
    a.nz, a.ny, a.nx = nz, ny, nx
    for k in (0, 1):
        tk = torch.as_tensor(t[h + k], device=dev).contiguous()
        qk = torch.as_tensor(q[h + k], device=dev).contiguous()
        keep += [tk, qk]
        a.t[k], a.q[k] = tk.data_ptr(), qk.data_ptr()
    lev = torch.as_tensor(np.asarray(met.levels, dtype=np.float32), device=dev)
    p = torch.as_tensor(np.asarray(met.p_hpa, dtype=np.float32), device=dev)
    keep += [lev, p]
    a.height3d, a.height_level, a.pressure_hpa = None, lev.data_ptr(), p.data_ptr()
    a.alpha = alpha
    a.closure_c, a.trigger_dtv_k = PARAMS["closure_c"], PARAMS["trigger_dtv_k"]
    a.min_cape_j_kg, a.min_cloud_depth_m = PARAMS["min_cape_j_kg"], PARAMS["min_cloud_depth_m"]
    nb = C.c_size_t()
    _abi.check(_abi.lib.glide_convect_scratch_bytes(nz, C.byref(nb)), "glide_convect_scratch_bytes")
    scratch = torch.full((nb.value // 8,), float("nan"), dtype=torch.float64, device=dev)
    a.scratch = scratch.data_ptr()
    _abi.check(_abi.lib.glide_convect(C.byref(a), torch.cuda.current_stream().cuda_stream), "glide_convect")
    torch.cuda.synchronize()
    return scratch.cpu().numpy()


@pytest.mark.gpu
@pytest.mark.parametrize("nz", [12, 60, 90])
def test_column_matches_fp64_oracle(cuda_device, nz):
    spec = SyntheticMetSpec(nz=nz, ny=24, nx=32, n_snapshots=3, moist_fraction=0.3, seed=20261204 + nz)
    met = met_from_synthetic(SyntheticMet(spec))
    h, alpha = 1, 0.375
    s = _column_on_device(met, h, alpha, cuda_device)
    height = np.broadcast_to(np.asarray(met.levels, dtype=np.float32).reshape(-1, 1, 1), met.fields["t"].shape[1:])
    col = oconv.build_column(met.fields["t"][h], met.fields["t"][h + 1], met.fields["q"][h], met.fields["q"][h + 1],
                             height, np.asarray(met.p_hpa, dtype=np.float32), alpha,
                             oconv.EmanuelParams(**PARAMS), dt=np.float64)
    assert col.fires, "the synthetic column should trigger with these thresholds"
    fires, i_lcl, i_lnb, cape, dtv, m_b = s[:6]
    assert fires == 1.0
    assert (int(i_lcl), int(i_lnb)) == (col.i_lcl, col.i_lnb)
    np.testing.assert_allclose([cape, dtv, m_b], [col.cape, col.dtv, col.m_b], rtol=1e-9, atol=1e-12)
    cum = s[8 + 4 * nz:8 + 4 * nz + nz * nz].reshape(nz, nz)
    assert np.all(np.isfinite(cum))
    # the CDF rows: the oracle's in FP64, to FP64 round-off of the column means
    np.testing.assert_allclose(cum, col.cum, rtol=0, atol=1e-9)
    np.testing.assert_allclose(cum[:, -1], 1.0, atol=1e-12)  # every row ends at 1
    assert np.all(np.diff(cum, axis=1) >= -1e-15)  # and never decreases
