"""The device regrid (glide_agl_regrid through glide_b200.regrid) against the
reference's own outputs (tests/golden/regrid.npz): brackets and channels bit for
bit, including the slope-corrected w; the per-level mean pressure to rounding."""

from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GOLDEN = Path(__file__).resolve().parent / "golden" / "regrid.npz"


@pytest.mark.parametrize("case", ["toa", "sfc"])
def test_device_regrid_matches_reference(cuda_device, case):
    from glide_b200.regrid import regrid_hour_to_agl

    z = np.load(GOLDEN)
    g = {k[len(case) + 1:]: z[k] for k in z.files if k.startswith(case + "_")}
    out, agl, p_level = regrid_hour_to_agl(g["fields"], g["height_agl"], g["agl"], ["u", "v", "w", "t"],
                                           z_sfc=g["z_sfc"], lat=g["lat"], lon=g["lon"], pressure_p_hpa=g["p_hpa"],
                                           device=cuda_device)
    np.testing.assert_array_equal(out.cpu().numpy(), g["out"])
    np.testing.assert_allclose(p_level, g["p_level"], rtol=1e-12)
    np.testing.assert_array_equal(agl, g["agl"])


def test_device_regrid_without_slope_or_pressure(cuda_device):
    from oracle import regrid as rg

    from glide_b200.regrid import regrid_hour_to_agl

    z = np.load(GOLDEN)
    f, h, agl = z["sfc_fields"], z["sfc_height_agl"], z["sfc_agl"]
    out, _, p_level = regrid_hour_to_agl(f, h, agl, ["a", "b", "c", "d"], device=cuda_device)
    lower, frac, flipped = rg.weights(h, agl)
    np.testing.assert_array_equal(out.cpu().numpy(), rg.apply(f, lower, frac, flipped))
    assert p_level is None
