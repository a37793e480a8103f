"""The regrid oracle (oracle/regrid.py) against the reference's own outputs
(tests/golden/regrid.npz, made by tests/golden/make_regrid_golden.py)."""

from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

GOLDEN = Path(__file__).resolve().parent / "golden" / "regrid.npz"


@pytest.mark.parametrize("case", ["toa", "sfc"])
def test_regrid_oracle_matches_reference(case):
    from oracle import regrid as rg

    z = np.load(GOLDEN)
    g = {k[len(case) + 1:]: z[k] for k in z.files if k.startswith(case + "_")}
    lower, frac, flipped = rg.weights(g["height_agl"], g["agl"])
    assert flipped == bool(g["flipped"])
    np.testing.assert_array_equal(lower, g["lower"])
    np.testing.assert_array_equal(frac, g["frac"])
    out = rg.apply(g["fields"], lower, frac, flipped)
    dhdx, dhdy = rg.terrain_gradient(g["z_sfc"] / 9.80665, g["lat"], g["lon"])
    np.testing.assert_array_equal(dhdx, g["dhdx"])
    np.testing.assert_array_equal(dhdy, g["dhdy"])
    out[2] = rg.slope_correct_w(out[2], out[0], out[1], dhdx, dhdy, g["agl"], float(g["agl"][-1]))
    np.testing.assert_array_equal(out, g["out"])
    p = rg.apply(np.ascontiguousarray(g["p_hpa"])[None], lower, frac, flipped)[0]
    np.testing.assert_allclose(p.mean(axis=(1, 2)), g["p_level"], rtol=1e-14)
