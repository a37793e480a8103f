"""The oracle against the closed-form known answers the reference's own unit tests
hold for this path (in float64, as those tests run): the surface-layer scaling
functions and Hanna's in-boundary-layer profiles (tests/test_hanna.py:48-260), the
free-troposphere Richardson closure (tests/test_hanna.py:270-340) and the footprint
scatter-add's exact cell and exact mass (tests/test_footprint.py:58-106). The
golden fixtures pin the oracle against the reference's outputs on sampled inputs;
these pin it against the formulae themselves at the points the reference checks."""

from __future__ import annotations

import math

import numpy as np

from oracle import hanna as oh
from oracle import runtime as ort

D = np.float64


def a(*v):
    return np.array(v, dtype=D)


def test_coriolis_density_obukhov_wstar():
    f = oh.coriolis_parameter(a(0.0, 30.0, 45.0, 60.0, -45.0), D)
    assert abs(f[0]) < 1e-10
    assert abs(f[2] - 2.0 * 7.2921e-5 * math.sin(math.radians(45.0))) < 1e-9
    assert f[3] > f[2] > f[1] > 0 > f[4] and abs(f[4] + f[2]) < 1e-12
    assert abs(oh.air_density(a(101325.0), a(288.0), D)[0] - 1.225) < 0.01
    L = oh.obukhov_length(a(0.4, 0.4, 0.4), a(100.0, -50.0, 0.0), a(288.0, 288.0, 288.0),
                          a(101325.0, 101325.0, 101325.0), D)
    assert L[0] < 0 < L[1] and math.isinf(L[2])
    w = oh.convective_velocity(a(1000.0, 1000.0, 1000.0), a(200.0, -50.0, 0.0), a(288.0, 288.0, 288.0),
                               a(101325.0, 101325.0, 101325.0), D)
    rho = 101325.0 / (287.05 * 288.0)
    assert abs(w[0] - ((9.80665 * 1000.0 * 200.0) / (288.0 * rho * 1005.0)) ** (1.0 / 3.0)) < 1e-6
    assert w[1] == 0.0 and w[2] == 0.0


def test_in_bl_profiles_at_the_surface():
    """z = 0: sigma_u = 2.0 u*, sigma_v = sigma_w = 1.3 u* (stable, neutral);
    unstable sigma_w^2 = 1.8 u*^2."""
    su, sv, sw, _, _, _ = oh.in_bl_sigma_TL(a(0.0, 0.0, 0.0), a(1000.0, 1000.0, 1000.0), a(0.5, 0.5, 0.5),
                                            a(0.0, 0.0, 1.5), a(5.0, 0.0, -5.0), a(45.0, 45.0, 45.0), D)
    for i in (0, 1):
        assert abs(su[i] - 1.0) < 1e-9 and abs(sw[i] - 0.65) < 1e-9 and abs(sv[i] - 0.65) < 1e-9
    assert abs(sw[2] - math.sqrt(1.8 * 0.25)) < 1e-6
    assert not np.allclose(su, sv)


def test_stable_profile_vanishes_at_the_top_and_timescales():
    _, _, sw, _, _, _ = oh.in_bl_sigma_TL(a(1000.0), a(1000.0), a(0.5), a(0.0), a(5.0), a(45.0), D)
    assert sw[0] < 1e-2
    us, h = 0.3, 500.0
    z = a(25.0, 100.0, 250.0, 400.0)
    n = z.size
    su, sv, sw, tu, tv, tw = oh.in_bl_sigma_TL(z, np.full(n, h), np.full(n, us), np.zeros(n), np.full(n, 5.0),
                                               np.full(n, 45.0), D)
    zeta = z / h
    np.testing.assert_allclose(su, 2.0 * us * (1 - zeta), atol=1e-9)
    np.testing.assert_allclose(sv, 1.3 * us * (1 - zeta), atol=1e-9)
    np.testing.assert_allclose(sw, 1.3 * us * (1 - zeta), atol=1e-9)
    np.testing.assert_allclose(tu, 0.15 * h / su * zeta**0.5, atol=1e-6)
    np.testing.assert_allclose(tv, 0.07 * h / sv * zeta**0.5, atol=1e-6)
    np.testing.assert_allclose(tw, 0.10 * h / sv * zeta**0.8, atol=1e-6)
    np.testing.assert_allclose(tv / tu, 0.718, rtol=1e-3)


def test_regime_selection_past_unit_h_over_L():
    z, h, us, lat = a(100.0), a(1000.0), a(0.5), a(45.0)
    neu = oh.in_bl_sigma_TL(z, h, us, a(0.0), a(0.5), lat, D)[0][0]
    stab = oh.in_bl_sigma_TL(z, h, us, a(0.0), a(1.5), lat, D)[0][0]
    unst = oh.in_bl_sigma_TL(z, h, us, a(1.5), a(-1.5), lat, D)[0][0]
    deep = oh.in_bl_sigma_TL(z, h, us, a(1.5), a(-10.0), lat, D)[0][0]
    assert deep > unst > 0 and neu != stab


def test_surface_layer_sigma_w():
    sw = oh.surface_layer_sigma_w(a(10.0, 10.0, 10.0), a(0.5, 0.5, 0.5), a(np.inf, -100.0, 200.0), D)
    assert abs(sw[0] - 0.65) < 1e-6 and abs(sw[1] - 0.65 * 1.3 ** (1.0 / 3.0)) < 1e-6 and abs(sw[2] - 0.65) < 1e-6
    sw = oh.surface_layer_sigma_w(a(10.0, 100.0), a(0.5, 0.5), a(200.0, 5.0), D)
    assert abs(sw[0] - 0.65) < 1e-9 and abs(sw[1] - 0.65) < 1e-9


def test_free_troposphere_closure():
    theta = oh.potential_temperature(a(280.0, 250.0), a(100000.0, 50000.0), D)
    assert abs(theta[0] - 280.0) < 1e-9 and abs(theta[1] - 250.0 * 2.0 ** (287.05 / 1005.0)) < 1e-6
    n2 = oh.brunt_vaisala_squared(a(300.0, 300.0), a(0.005, -0.005), D)
    assert n2[0] > 0 > n2[1]
    shear = a(0.01, 0.01, 0.01)
    ri = oh.gradient_richardson(a(0.0, 1e-5, 1e-3), shear**2, D)
    k = oh.free_trop_diffusivity(a(1000.0, 1000.0, 1000.0), shear, ri, D)
    assert k[0] > k[1] >= k[2] and abs(k[2] - 0.1) < 1e-9 and k[0] <= 50.0
    sw, tl = oh.free_trop_sigma_TL(a(0.1, 1.0, 10.0), a(1e-4, 1e-4, 1e-4), D)
    np.testing.assert_allclose(sw**2 * tl, a(0.1, 1.0, 10.0), rtol=1e-5)
    assert oh.free_trop_diffusivity(a(2000.0), a(0.001), a(100.0), D)[0] >= 0.1


def _grid():
    return ort.GridSpec(lon_bounds=(-1.0, 1.0), lat_bounds=(-1.0, 1.0), n_x=4, n_y=4, z_edges=(0.0, 500.0, 1000.0),
                        n_time_bins=2, n_releases=1)


def test_footprint_single_particle_exact_cell():
    g = _grid()
    fp = np.zeros(int(np.prod(g.shape)), dtype=D)
    xyz = a(-0.75, -0.75, 250.0).reshape(3, 1)  # lon bin 0, lat bin 0, z bin 0
    ort.accumulate(fp, xyz, np.array([True]), a(0.5), np.array([1]), np.array([0]), g, 10.0, D)
    fp = fp.reshape(g.shape)
    assert fp[0, 1, 0, 0, 0] == 5.0 and fp.sum() == 5.0


def test_footprint_mass_is_conserved_in_bounds():
    g = _grid()
    rng = np.random.default_rng(42)
    n = 100
    xyz = np.stack([rng.uniform(-0.99, 0.99, n), rng.uniform(-0.99, 0.99, n), rng.uniform(0.0, 999.0, n)])
    w = np.full(n, 1.0 / n)
    fp = np.zeros(int(np.prod(g.shape)), dtype=D)
    ort.accumulate(fp, xyz, np.ones(n, bool), w, np.zeros(n, np.int64), np.zeros(n, np.int64), g, 5.0, D)
    assert abs(fp.sum() - w.sum() * 5.0) < 1e-12
    # out of the grid, inactive, or past the last time bin: nothing lands
    fp[:] = 0.0
    xyz_out = np.stack([a(1.5, 0.0, 0.0), a(0.0, -1.5, 0.0), a(10.0, 10.0, 1500.0)])
    ort.accumulate(fp, xyz_out, np.array([True, True, True]), a(1.0, 1.0, 1.0), np.array([0, 0, 0]),
                   np.array([0, 0, 0]), g, 5.0, D)
    ort.accumulate(fp, xyz[:, :2], np.array([False, True]), a(1.0, 1.0), np.array([0, 2]), np.array([0, 0]), g,
                   5.0, D)
    assert fp.sum() == 0.0
