"""Oracle: Hanna turbulence scheme, static (full-set, mask-gated) step path.

Restates ``src/lpdm/turbulence/hanna.py`` and the ``GPUEngine`` primitives of
``src/lpdm/gpu_engine.py`` in numpy. Test infrastructure only (see the package
docstring).

Operation order follows the reference's torch expressions so that the float32
mode agrees with the reference to a few ulp per operation. Where torch's CPU
kernels use a fused multiply-add (2-D bilinear ``grid_sample`` accumulation,
``torch.lerp``) this module uses :func:`fma`; everywhere else it does not.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np

# Physical constants (hanna.py:46-106)
KARMAN = 0.4
GRAVITY = 9.80665
R_DRY = 287.05
C_P = 1005.0
OMEGA = 7.2921e-5
H_OVER_L_STABLE = 1.0
H_OVER_L_UNSTABLE = -1.0
SURFACE_LAYER_FRACTION = 0.1
SIGMA_MIN = 1e-3
T_L_MIN = 1.0
USTAR_MIN = 1e-3
BLH_MIN = 50.0
Z_MIN = 1.0
T_LU_FLOOR = 10.0
T_LV_FLOOR = 10.0
T_LW_FLOOR = 30.0
P0_PA = 100000.0
KAPPA_POISSON = R_DRY / C_P
FT_MIXING_LENGTH = 100.0
FT_RI_CRIT = 0.25
FT_KZ_FLOOR = 0.1
FT_KZ_CEIL = 50.0
FT_SHEAR_SQ_FLOOR = 1e-8
FT_N2_FLOOR = 1e-6
FT_T_L_DEFAULT = 100.0
FT_T_L_MAX = 1000.0
W_PRIME_SIGMA_RATIO_MAX = 4.0
DRIFT_FD_DELTA_M = 1.0
M_PER_DEG_LAT = 110540.0
M_PER_DEG_LON = 111320.0


@dataclass(frozen=True)
class HannaParams:
    """Scheme knobs (``HannaScheme.__init__``, hanna.py:440-520)."""

    meander_enabled: bool = False
    meander_coefficient: float = 0.16
    meander_stencil_radius: int = 1
    meander_timescale_seconds: float = 1800.0
    substep_c: float = 0.5
    max_substeps: int = 50
    z_ubl_m: float = 2.0
    flexpart_tl_floors: bool = True
    surface_layer_override: bool = False


@dataclass
class StepNoise:
    """Injected standard-normal draws for one outer step.

    ``substep[i, c, p]``: substep ``i``, component ``c`` (0 = u, 1 = v, 2 = w),
    particle ``p`` — what ``GPUEngine.update_langevin_velocity`` would draw with
    ``randn_like`` (gpu_engine.py:386-391) in the static loop (hanna.py:1320-1353).
    ``meander[c, p]``: the two meander draws (hanna.py:1039-1050).
    """

    substep: np.ndarray
    meander: np.ndarray | None = None


def _c(x, dt):
    return np.asarray(x, dtype=dt)


def fma(a, b, c, dt):
    """Fused multiply-add rounded once to ``dt`` (emulated in float64 for float32)."""
    if dt == np.float64:
        return np.asarray(a, np.float64) * np.asarray(b, np.float64) + np.asarray(c, np.float64)
    return (np.asarray(a, np.float64) * np.asarray(b, np.float64) + np.asarray(c, np.float64)).astype(np.float32)


def lerp(s, e, w: float, dt):
    """``torch.lerp(s, e, w)`` with a scalar weight (FMA form of torch's CPU kernel)."""
    w = dt(w)
    diff = e - s
    if abs(w) < 0.5:
        return fma(w, diff, s, dt)
    return fma(w - dt(1.0), diff, e, dt)


# ---------------------------------------------------------------------------
# Coordinate normalisation + grid sampling (gpu_engine.py:210-299; torch grid_sample)
# ---------------------------------------------------------------------------


@dataclass(frozen=True)
class GridBounds:
    """``GridInterpolationBounds`` (gpu_engine.py:100-121) as built by
    ``HannaScheme._grid_bounds`` (hanna.py:1832-1853)."""

    lon_first: float
    lon_last: float
    lat_first: float
    lat_last: float
    level: np.ndarray  # [Z] AGL heights in the grid's own order


def normalize_coords(lon, lat, z, gb: GridBounds, dt):
    """``normalize_particle_coordinates`` (gpu_engine.py:210-299) → (x, y, z) in [-1, 1]."""

    def scale(vals, v0, v1):
        denom = float(v1 - v0)
        return dt(2.0) * ((vals - dt(v0)) / dt(denom)) - dt(1.0)

    x = scale(lon, gb.lon_first, gb.lon_last)
    y = scale(lat, gb.lat_first, gb.lat_last)
    level = np.asarray(gb.level, dtype=dt)
    n = level.size
    ascending = bool(gb.level[-1] > gb.level[0])
    lv = level if ascending else level[::-1]
    idx_upper = np.clip(np.searchsorted(lv, z, side="left"), 1, n - 1)
    idx_lower = idx_upper - 1
    lo = lv[idx_lower]
    hi = lv[idx_upper]
    frac = (z - lo) / np.maximum(hi - lo, dt(1e-6))
    frac_idx = idx_lower.astype(dt) + np.clip(frac, dt(0.0), dt(1.0))
    if not ascending:
        frac_idx = dt(n - 1) - frac_idx
    zn = dt(2.0) * frac_idx / dt(n - 1) - dt(1.0)
    return (np.clip(x, dt(-1), dt(1)), np.clip(y, dt(-1), dt(1)), np.clip(zn, dt(-1), dt(1)))


def trilinear(vol, xn, yn, zn, dt):
    """``grid_sample(vol[None], grid, align_corners=True)`` for a ``[C, Z, Y, X]`` stack
    (torch's CPU 3-D kernel: unnormalise ``((c+1)/2)(size-1)``, eight corner weights,
    zero padding, accumulation tnw→bse)."""
    C, Z, Y, X = vol.shape
    ix = ((xn + dt(1)) / dt(2)) * dt(X - 1)
    iy = ((yn + dt(1)) / dt(2)) * dt(Y - 1)
    iz = ((zn + dt(1)) / dt(2)) * dt(Z - 1)
    x0 = np.floor(ix).astype(np.int64)
    y0 = np.floor(iy).astype(np.int64)
    z0 = np.floor(iz).astype(np.int64)
    x1, y1, z1 = x0 + 1, y0 + 1, z0 + 1
    fx0, fx1 = x0.astype(dt), x1.astype(dt)
    fy0, fy1 = y0.astype(dt), y1.astype(dt)
    fz0, fz1 = z0.astype(dt), z1.astype(dt)
    corners = (
        (z0, y0, x0, (fx1 - ix) * (fy1 - iy) * (fz1 - iz)),
        (z0, y0, x1, (ix - fx0) * (fy1 - iy) * (fz1 - iz)),
        (z0, y1, x0, (fx1 - ix) * (iy - fy0) * (fz1 - iz)),
        (z0, y1, x1, (ix - fx0) * (iy - fy0) * (fz1 - iz)),
        (z1, y0, x0, (fx1 - ix) * (fy1 - iy) * (iz - fz0)),
        (z1, y0, x1, (ix - fx0) * (fy1 - iy) * (iz - fz0)),
        (z1, y1, x0, (fx1 - ix) * (iy - fy0) * (iz - fz0)),
        (z1, y1, x1, (ix - fx0) * (iy - fy0) * (iz - fz0)),
    )
    out = np.zeros((C, xn.size), dtype=dt)
    for zz, yy, xx, wgt in corners:
        ok = (zz >= 0) & (zz < Z) & (yy >= 0) & (yy < Y) & (xx >= 0) & (xx < X)
        vals = vol[:, np.clip(zz, 0, Z - 1), np.clip(yy, 0, Y - 1), np.clip(xx, 0, X - 1)].astype(dt)
        out = np.where(ok, out + vals * wgt, out)
    return out


def bilinear_at(field, lon0, lon1, lat0, lat1, lon, lat, dt):
    """``HannaScheme._bilinear_at`` (hanna.py:1070-1085): 4-D ``grid_sample`` bilinear,
    align_corners=True, torch's vectorised CPU kernel (FMA accumulation)."""
    if lon1 == lon0 or lat1 == lat0:
        raise ValueError("Met grid has zero span in lon or lat")
    Y, X = field.shape
    xn = np.clip(dt(2.0) * (lon - dt(lon0)) / dt(lon1 - lon0) - dt(1.0), dt(-1), dt(1))
    yn = np.clip(dt(2.0) * (lat - dt(lat0)) / dt(lat1 - lat0) - dt(1.0), dt(-1), dt(1))
    ix = ((xn + dt(1)) / dt(2)) * dt(X - 1)
    iy = ((yn + dt(1)) / dt(2)) * dt(Y - 1)
    fx = np.floor(ix)
    fy = np.floor(iy)
    w = ix - fx
    e = dt(1) - w
    n = iy - fy
    s = dt(1) - n
    nw, ne, sw, se = s * e, s * w, n * e, n * w
    xi, yi = fx.astype(np.int64), fy.astype(np.int64)

    def get(yy, xx):
        ok = (yy >= 0) & (yy < Y) & (xx >= 0) & (xx < X)
        return np.where(ok, field[np.clip(yy, 0, Y - 1), np.clip(xx, 0, X - 1)].astype(dt), dt(0))

    a, b, c, d = get(yi, xi), get(yi, xi + 1), get(yi + 1, xi), get(yi + 1, xi + 1)
    return fma(d, se, fma(c, sw, fma(b, ne, a * nw, dt), dt), dt)


# ---------------------------------------------------------------------------
# Free physics functions (hanna.py:142-426)
# ---------------------------------------------------------------------------


def deg2rad(x, dt):
    return x * dt(np.pi / 180.0)


def coriolis_parameter(lat, dt):
    """hanna.py:142-145"""
    return dt(2.0 * OMEGA) * np.sin(deg2rad(lat, dt))


def air_density(sp, t, dt):
    """hanna.py:148-151"""
    return sp / (dt(R_DRY) * t)


def obukhov_length(ustar, shf, t, sp, dt):
    """hanna.py:154-173 (``+inf`` where ``|kappa g H| <= 1e-10``)."""
    rho = air_density(sp, t, dt)
    denom = dt(KARMAN * GRAVITY) * shf
    us = np.maximum(ustar, dt(USTAR_MIN))
    num = -(us * us * us) * t * rho * dt(C_P)
    finite = np.abs(denom) > dt(1e-10)
    safe = np.where(finite, denom, dt(1.0))
    with np.errstate(divide="ignore", invalid="ignore"):
        return np.where(finite, num / safe, dt(np.inf))


def convective_velocity(blh, shf, t, sp, dt):
    """hanna.py:176-189"""
    rho = air_density(sp, t, dt)
    cube = (dt(GRAVITY) * np.maximum(blh, dt(BLH_MIN)) * shf) / (t * rho * dt(C_P))
    return np.where(cube > 0, np.power(np.maximum(cube, dt(0)), dt(1.0 / 3.0)), dt(0))


def in_bl_stable(z, blh, ustar, dt):
    """hanna.py:192-222 (Hanna 1982 Eqs 7.19-7.24)."""
    zoh = np.clip(z / blh, dt(0), dt(1))
    om = np.maximum(dt(1) - zoh, dt(0))
    su = dt(2.0) * ustar * om
    sw = dt(1.3) * ustar * om
    sv = sw
    zf = np.maximum(zoh, dt(1e-6))
    tlu = dt(0.15) * blh / np.maximum(su, dt(SIGMA_MIN)) * np.sqrt(zf)
    tlv = dt(0.07) * blh / np.maximum(sv, dt(SIGMA_MIN)) * np.sqrt(zf)
    tlw = dt(0.10) * blh / np.maximum(sw, dt(SIGMA_MIN)) * np.power(zf, dt(0.8))
    return su, sv, sw, tlu, tlv, tlw


def in_bl_neutral(z, ustar, f_cor, dt):
    """hanna.py:225-252 (Hanna 1982 Eqs 7.25-7.27, |f| floored at 1e-5)."""
    us = np.maximum(ustar, dt(USTAR_MIN))
    fa = np.maximum(np.abs(f_cor), dt(1e-5))
    su = dt(2.0) * ustar * np.exp(dt(-3.0) * fa * z / us)
    sw = dt(1.3) * ustar * np.exp(dt(-2.0) * fa * z / us)
    sv = sw
    den = dt(1.0) + dt(15.0) * fa * z / us
    tlw = dt(0.5) * z / np.maximum(sw, dt(SIGMA_MIN)) / np.maximum(den, dt(1.0))
    return su, sv, sw, tlw, tlw, tlw


def in_bl_unstable(z, blh, ustar, w_star, h_over_L, dt):
    """hanna.py:255-298 (Caughey 1982, Ryall & Maryon 1998, Hanna 1982)."""
    zoh = np.clip(z / blh, dt(0), dt(1))
    hl = np.clip(h_over_L, dt(-1000.0), dt(0.0))
    su = np.power(np.maximum(dt(12.0) - dt(0.5) * hl, dt(1e-3)), dt(1.0 / 3.0)) * ustar
    sv = su
    sw2 = (dt(1.2) * (w_star * w_star) * np.maximum(dt(1.0) - dt(0.9) * zoh, dt(0))
           * np.power(zoh, dt(2.0 / 3.0)) + (dt(1.8) - dt(1.4) * zoh) * (ustar * ustar))
    sw = np.sqrt(np.maximum(sw2, dt(SIGMA_MIN**2)))
    tlu = dt(0.15) * blh / np.maximum(su, dt(SIGMA_MIN))
    tlv = tlu
    azl = np.maximum(zoh * (-hl), dt(0))
    swc = np.maximum(sw, dt(SIGMA_MIN))
    t_near = dt(0.1) * z / (swc * np.maximum(dt(0.55) - dt(0.38) * azl, dt(1e-2)))
    t_shallow = dt(0.59) * z / swc
    t_bulk = dt(0.15) * blh / swc * (dt(1.0) - np.exp(dt(-5.0) * zoh))
    tlw = np.where(azl < 1.0, t_near, np.where(zoh < 0.1, t_shallow, t_bulk))
    return su, sv, sw, tlu, tlv, tlw


def in_bl_sigma_TL(z, blh, ustar, w_star, h_over_L, lat, dt):
    """hanna.py:301-337: all three regimes, selected by h/L (>1 stable, <-1 unstable)."""
    f_cor = coriolis_parameter(lat, dt)
    with np.errstate(divide="ignore", invalid="ignore", over="ignore"):
        st = in_bl_stable(z, blh, ustar, dt)
        nu = in_bl_neutral(z, ustar, f_cor, dt)
        un = in_bl_unstable(z, blh, ustar, w_star, h_over_L, dt)
    in_st = h_over_L > H_OVER_L_STABLE
    in_un = h_over_L < H_OVER_L_UNSTABLE
    return tuple(np.where(in_st, a, np.where(in_un, c, b)) for a, b, c in zip(st, nu, un))


def surface_layer_sigma_w(z, ustar, L, dt):
    """hanna.py:405-426"""
    eps = dt(1e-6)
    finite = np.abs(L) > eps
    Ls = np.where(finite, L, dt(1.0))
    zl = np.where(finite, np.clip(z / Ls, dt(-50), dt(50)), dt(0))
    unst = dt(1.3) * ustar * np.power(np.maximum(dt(1.0) - dt(3.0) * zl, eps), dt(1.0 / 3.0))
    return np.where(zl < 0.0, unst, dt(1.3) * ustar)


def potential_temperature(t, p, dt):
    """hanna.py:340-343"""
    return t * np.power(dt(P0_PA) / p, dt(KAPPA_POISSON))


def brunt_vaisala_squared(theta, dtheta_dz, dt):
    """hanna.py:346-350"""
    return (dt(GRAVITY) / np.maximum(theta, dt(1.0))) * dtheta_dz


def gradient_richardson(n2, shear_sq, dt):
    """hanna.py:353-356"""
    return n2 / np.maximum(shear_sq, dt(FT_SHEAR_SQ_FLOOR))


def free_trop_diffusivity(z, shear_mag, ri, dt):
    """hanna.py:359-382: K = l^2 |dU/dz| f(Ri), clamped to [0.1, 50]."""
    ml = (dt(KARMAN) * z) / (dt(1.0) + dt(KARMAN) * z / dt(FT_MIXING_LENGTH))
    fs = np.maximum(dt(1.0) - ri / dt(FT_RI_CRIT), dt(0))
    fs = fs * fs
    fu = np.sqrt(np.maximum(dt(1.0) - dt(16.0) * ri, dt(0)))
    f = np.where(ri < 0.0, fu, fs)
    k = (ml * ml) * shear_mag * f
    return np.clip(k, dt(FT_KZ_FLOOR), dt(FT_KZ_CEIL))


def free_trop_sigma_TL(k_z, n2, dt):
    """hanna.py:385-402"""
    tl = np.where(n2 > FT_N2_FLOOR,
                  np.clip(dt(0.5) / np.sqrt(np.maximum(n2, dt(FT_N2_FLOOR))), dt(T_L_MIN), dt(FT_T_L_MAX)),
                  dt(FT_T_L_DEFAULT))
    sw = np.sqrt(np.maximum(k_z / tl, dt(SIGMA_MIN**2)))
    return sw, tl


# ---------------------------------------------------------------------------
# Per-window support stacks (hanna.py:1682-1869)
# ---------------------------------------------------------------------------


def vertical_gradient(field, height, dt):
    """``_vertical_gradient`` (hanna.py:1855-1869): centred inside, one-sided at the ends."""

    def safe(den):
        return np.where(np.abs(den) < 1e-6, dt(1e-6), den)

    g = np.empty_like(field)
    g[1:-1] = (field[2:] - field[:-2]) / safe(height[2:] - height[:-2])
    g[0] = (field[1] - field[0]) / safe(height[1] - height[0])
    g[-1] = (field[-1] - field[-2]) / safe(height[-1] - height[-2])
    return g


def window_mid(start, end, dt):
    """``_window_mid`` (hanna.py:1682-1692)."""
    return dt(0.5) * (start.astype(dt) + end.astype(dt))


def free_trop_fields(t_mid, u_mid, v_mid, height, p_hpa, dt):
    """``_free_trop_fields._build`` (hanna.py:1694-1745) → ``[4, Z, Y, X]``."""
    p = (np.asarray(p_hpa).astype(dt) * dt(100.0)).reshape(-1, 1, 1)
    h = height.astype(dt)
    theta = potential_temperature(t_mid, p, dt)
    n2 = brunt_vaisala_squared(theta, vertical_gradient(theta, h, dt), dt)
    du = vertical_gradient(u_mid, h, dt)
    dv = vertical_gradient(v_mid, h, dt)
    shear_sq = du * du + dv * dv
    shear_mag = np.sqrt(np.maximum(shear_sq, dt(FT_SHEAR_SQ_FLOOR)))
    ri = gradient_richardson(n2, shear_sq, dt)
    kz = free_trop_diffusivity(np.maximum(h, dt(Z_MIN)), shear_mag, ri, dt)
    sw, tl = free_trop_sigma_TL(kz, n2, dt)
    return np.stack([sw, sw, tl, tl], axis=0)


def density_fields(t_mid, height, p_hpa, dt):
    """``_density_fields._build`` (hanna.py:1747-1784) → ``[2, Z, Y, X]`` (rho, drho/dz)."""
    p = (np.asarray(p_hpa).astype(dt) * dt(100.0)).reshape(-1, 1, 1)
    rho = p / (dt(R_DRY) * np.maximum(t_mid, dt(1.0)))
    return np.stack([rho, vertical_gradient(rho, height.astype(dt), dt)], axis=0)


def windowed_std(field, radius, dt):
    """``_windowed_std`` (hanna.py:1813-1830): per-level std over a (2r+1)^2 stencil,
    edges averaging only in-grid neighbours (avg_pool2d, count_include_pad=False)."""
    Z, Y, X = field.shape
    s = np.zeros_like(field)
    s2 = np.zeros_like(field)
    cnt = np.zeros((Y, X), dtype=dt)
    sq = field * field
    for dy in range(-radius, radius + 1):
        for dx in range(-radius, radius + 1):
            ys = slice(max(0, -dy), Y - max(0, dy))
            xs = slice(max(0, -dx), X - max(0, dx))
            ys_src = slice(max(0, dy), Y - max(0, -dy))
            xs_src = slice(max(0, dx), X - max(0, -dx))
            s[:, ys, xs] += field[:, ys_src, xs_src]
            s2[:, ys, xs] += sq[:, ys_src, xs_src]
            cnt[ys, xs] += 1
    mean = s / cnt
    var = np.maximum(s2 / cnt - mean * mean, dt(0))
    return np.sqrt(var)


def meander_fields(u_mid, v_mid, coefficient, radius, dt):
    """``_meander_sigma_fields._build`` (hanna.py:1786-1811) → ``[2, Z, Y, X]``."""
    return np.stack([dt(coefficient) * windowed_std(u_mid, radius, dt),
                     dt(coefficient) * windowed_std(v_mid, radius, dt)], axis=0)


# ---------------------------------------------------------------------------
# Column turbulence (hanna.py:1500-1596)
# ---------------------------------------------------------------------------


def column_turbulence(zq, *, blh, ustar, w_star, h_over_L, L, lat, lon, ft_fields, gb, params, dt):
    su, sv, sw, tlu, tlv, tlw = in_bl_sigma_TL(zq, blh, ustar, w_star, h_over_L, lat, dt)
    if params.surface_layer_override:
        z_sl = dt(SURFACE_LAYER_FRACTION) * blh
        in_sl = zq < z_sl
        sw_sl = surface_layer_sigma_w(zq, ustar, L, dt)
        zc = np.maximum(zq, z_sl)
        su_c, sv_c, *_ = in_bl_sigma_TL(zc, blh, ustar, w_star, h_over_L, lat, dt)
        su = np.where(in_sl, su_c, su)
        sv = np.where(in_sl, sv_c, sv)
        sw = np.where(in_sl, sw_sl, sw)
        zt = np.maximum(zq, dt(Z_MIN))
        tlu = np.where(in_sl, dt(KARMAN) * zt / np.maximum(su, dt(SIGMA_MIN)), tlu)
        tlv = np.where(in_sl, dt(KARMAN) * zt / np.maximum(sv, dt(SIGMA_MIN)), tlv)
        tlw = np.where(in_sl, dt(KARMAN) * zt / np.maximum(sw, dt(SIGMA_MIN)), tlw)
    if params.flexpart_tl_floors:
        tlu = np.maximum(tlu, dt(T_LU_FLOOR))
        tlv = np.maximum(tlv, dt(T_LV_FLOOR))
        tlw = np.maximum(tlw, dt(T_LW_FLOOR))
    above = zq > blh
    xn, yn, zn = normalize_coords(lon, lat, zq, gb, dt)
    ft = trilinear(ft_fields, xn, yn, zn, dt)
    su = np.where(above, ft[1], su)
    sv = np.where(above, ft[1], sv)
    sw = np.where(above, ft[0], sw)
    tlu = np.where(above, ft[3], tlu)
    tlv = np.where(above, ft[3], tlv)
    tlw = np.where(above, ft[2], tlw)
    return (np.maximum(su, dt(SIGMA_MIN)), np.maximum(sv, dt(SIGMA_MIN)), np.maximum(sw, dt(SIGMA_MIN)),
            np.maximum(tlu, dt(T_L_MIN)), np.maximum(tlv, dt(T_L_MIN)), np.maximum(tlw, dt(T_L_MIN)))


# ---------------------------------------------------------------------------
# Engine primitives (gpu_engine.py:26-42, 345-507)
# ---------------------------------------------------------------------------


def ou_step(w_prev, tl, sigma2, sub_dt, eta, drift_dt, dt):
    """``_ou_step_kernel`` (gpu_engine.py:26-42): exact OU update."""
    with np.errstate(over="ignore", invalid="ignore"):
        a = np.exp(-sub_dt / tl)
    var = np.maximum(sigma2 * (dt(1.0) - a * a), dt(0))
    return a * w_prev + drift_dt + np.sqrt(var) * eta


def meters_per_deg_lon(lat, dt):
    return dt(M_PER_DEG_LON) * np.maximum(np.abs(np.cos(deg2rad(lat, dt))), dt(0.05))


def wind_rk2(xyz, m_start, m_end, alpha, gb, dt):
    """``wind`` of ``_advect_rk2`` (hanna.py:866-889) → (dlon/dt, dlat/dt, w)."""
    xn, yn, zn = normalize_coords(xyz[0], xyz[1], xyz[2], gb, dt)
    vs = trilinear(m_start, xn, yn, zn, dt)
    ve = trilinear(m_end, xn, yn, zn, dt)
    v = vs * (dt(1.0) - alpha) + ve * alpha
    m_lon = meters_per_deg_lon(xyz[1], dt)
    return np.stack([v[0] / m_lon, v[1] / dt(M_PER_DEG_LAT), v[2]])


def advect_rk2(xyz, m_start, m_end, alpha, gb, delta, dt):
    """``_advect_rk2`` (hanna.py:855-896): backward midpoint RK2."""
    v1 = wind_rk2(xyz, m_start, m_end, alpha, gb, dt)
    v2 = wind_rk2(xyz - dt(0.5 * delta) * v1, m_start, m_end, alpha, gb, dt)
    return xyz - dt(delta) * v2


# ---------------------------------------------------------------------------
# Whole static step core (hanna.py:898-1068 + 1162-1186 + 1224-1368)
# ---------------------------------------------------------------------------


@dataclass
class StepInputs:
    """Per-window device inputs of ``_step_core`` (hanna.py:798-853)."""

    m_start_uvw: np.ndarray  # [3, Z, Y, X]
    m_end_uvw: np.ndarray
    surf_start: dict  # name -> [Y, X]; blh, sp, ustar, shf, t (lowest level)
    surf_end: dict
    ft_fields: np.ndarray  # [4, Z, Y, X]
    density_fields: np.ndarray  # [2, Z, Y, X]
    meander_fields: np.ndarray | None  # [2, Z, Y, X]
    gb: GridBounds


def step_core(particles, state, active, inp: StepInputs, alpha: float, delta: float,
              params: HannaParams, noise: StepNoise, dt=np.float32):
    """One outer step of the static path with injected noise.

    ``particles``: ``[4, N]`` (lon, lat, z, weight); ``state``: dict of ``[N]``
    (u_prime, v_prime, w_prime[, u_meander, v_meander]); ``active``: bool ``[N]``.
    Returns ``(particles, state)`` with inactive entries unchanged.
    """
    p0 = particles.astype(dt)
    gb = inp.gb
    a_t = dt(alpha)
    xyz = advect_rk2(p0[:3], inp.m_start_uvw, inp.m_end_uvw, a_t, gb, delta, dt)
    lon, lat, z = xyz[0], xyz[1], xyz[2]

    def surf(name):
        return bilinear_at(lerp(inp.surf_start[name].astype(dt), inp.surf_end[name].astype(dt), alpha, dt),
                           gb.lon_first, gb.lon_last, gb.lat_first, gb.lat_last, lon, lat, dt)

    blh = np.maximum(surf("blh"), dt(BLH_MIN))
    sp = surf("sp")
    ustar = np.maximum(surf("ustar"), dt(USTAR_MIN))
    shf = surf("shf")
    t_s = surf("t")
    L = obukhov_length(ustar, shf, t_s, sp, dt)
    with np.errstate(divide="ignore", invalid="ignore"):
        h_over_L = blh / L
    w_star = convective_velocity(blh, shf, t_s, sp, dt)
    ck = dict(blh=blh, ustar=ustar, w_star=w_star, h_over_L=h_over_L, L=L, lat=lat, lon=lon,
              ft_fields=inp.ft_fields, gb=gb, params=params, dt=dt)
    z_ubl = dt(params.z_ubl_m)
    z_eval = np.maximum(z, z_ubl)
    su, sv, sw, tlu, tlv, tlw = column_turbulence(z_eval, **ck)
    z_hi = z_eval + dt(DRIFT_FD_DELTA_M)
    z_lo = np.maximum(z_eval - dt(DRIFT_FD_DELTA_M), z_ubl)
    sw_hi = column_turbulence(z_hi, **ck)[2]
    sw_lo = column_turbulence(z_lo, **ck)[2]
    dsig2 = (sw_hi * sw_hi - sw_lo * sw_lo) / np.maximum(z_hi - z_lo, dt(DRIFT_FD_DELTA_M))
    sw_sq = np.maximum(sw * sw, dt(SIGMA_MIN**2))
    xn, yn, zn = normalize_coords(lon, lat, z_eval, gb, dt)
    dens = trilinear(inp.density_fields, xn, yn, zn, dt)
    rho = np.maximum(dens[0], dt(1e-3))
    drift_fwd = sw_sq * dens[1] / rho
    half_bwd = dt(-0.5) * dsig2
    dens_bwd = -drift_fwd

    # substep counts (hanna.py:1162-1186)
    with np.errstate(over="ignore", invalid="ignore", divide="ignore"):
        kq = np.ceil(dt(delta) / (dt(params.substep_c) * np.maximum(tlw, dt(1e-3))))
    k = np.clip(np.nan_to_num(kq, nan=1.0, posinf=params.max_substeps), 1, params.max_substeps).astype(np.int64)
    k = np.where(active, k, 1)
    sub_dt = dt(delta) / k.astype(dt)

    # static substep loop (hanna.py:1224-1368)
    x = xyz.copy()
    u_p = state["u_prime"].astype(dt)
    v_p = state["v_prime"].astype(dt)
    w_p = state["w_prime"].astype(dt)
    su2, sv2, sw2 = su * su, sv * sv, sw * sw
    u_max, v_max, w_max = dt(4.0) * su, dt(4.0) * sv, dt(4.0) * sw
    n_iter = int(k.max()) if k.size else 0
    for i in range(n_iter):
        owing = (k > i) & active
        sdt = np.where(owing, sub_dt, dt(0))
        factor = dt(1.0) + (w_p * w_p) / sw_sq
        drift_w = factor * half_bwd + dens_bwd
        u_n = ou_step(u_p, tlu, su2, sdt, noise.substep[i, 0].astype(dt), dt(0.0) * sdt, dt)
        v_n = ou_step(v_p, tlv, sv2, sdt, noise.substep[i, 1].astype(dt), dt(0.0) * sdt, dt)
        w_n = ou_step(w_p, tlw, sw2, sdt, noise.substep[i, 2].astype(dt), drift_w * sdt, dt)
        w_n = np.clip(w_n, -w_max, w_max)
        u_n = np.clip(u_n, -u_max, u_max)
        v_n = np.clip(v_n, -v_max, v_max)
        # apply_vertical_turbulence then apply_horizontal_turbulence (gpu_engine.py:400-471)
        x2 = x[2] + dt(-1.0) * w_n * sdt
        m_lon = meters_per_deg_lon(x[1], dt)
        x0 = x[0] + dt(-1.0) * u_n * sdt / m_lon
        x1 = x[1] + dt(-1.0) * v_n * sdt / dt(M_PER_DEG_LAT)
        # reflect_surface (gpu_engine.py:473-507)
        below = x2 < dt(0.0)
        x2 = np.where(below, dt(0.0) - x2, x2)
        w_n = np.where(below, -w_n, w_n)
        x = np.stack([x0, x1, x2])
        u_p, v_p, w_p = u_n, v_n, w_n

    new_state = {"u_prime": u_p, "v_prime": v_p, "w_prime": w_p}
    if params.meander_enabled:
        sm = trilinear(inp.meander_fields, xn, yn, zn, dt)
        d = dt(delta)
        tm = dt(params.meander_timescale_seconds)
        um = ou_step(state["u_meander"].astype(dt), tm, sm[0] * sm[0], d, noise.meander[0].astype(dt), dt(0.0) * d, dt)
        vm = ou_step(state["v_meander"].astype(dt), tm, sm[1] * sm[1], d, noise.meander[1].astype(dt), dt(0.0) * d, dt)
        m_lon = meters_per_deg_lon(x[1], dt)
        x = np.stack([x[0] + dt(-1.0) * um * d / m_lon, x[1] + dt(-1.0) * vm * d / dt(M_PER_DEG_LAT), x[2]])
        new_state["u_meander"] = um
        new_state["v_meander"] = vm

    out = p0.copy()
    out[:3] = np.where(active, x, p0[:3])
    st = {}
    for key, val in new_state.items():
        st[key] = np.where(active, val, state[key].astype(dt))
    return out, st


def build_step_inputs(win, params: HannaParams, dt=np.float32) -> StepInputs:
    """Per-window inputs from an oracle window dict (see ``oracle.runtime.window_from_met``)."""
    d = dt
    m_start = np.stack([win["u"][0], win["v"][0], win["w"][0]]).astype(d)
    m_end = np.stack([win["u"][1], win["v"][1], win["w"][1]]).astype(d)
    t_mid = window_mid(win["t"][0], win["t"][1], d)
    u_mid = window_mid(win["u"][0], win["u"][1], d)
    v_mid = window_mid(win["v"][0], win["v"][1], d)
    height = win["height"].astype(d)
    ft = free_trop_fields(t_mid, u_mid, v_mid, height, win["p_hpa"], d)
    dens = density_fields(t_mid, height, win["p_hpa"], d)
    mea = (meander_fields(u_mid, v_mid, params.meander_coefficient, params.meander_stencil_radius, d)
           if params.meander_enabled else None)
    lowest = int(np.argmin(win["level"]))
    names = ("blh", "sp", "ustar", "shf")
    ss = {n: win[n][0] for n in names}
    se = {n: win[n][1] for n in names}
    ss["t"] = win["t"][0][lowest]
    se["t"] = win["t"][1][lowest]
    gb = GridBounds(float(win["lon"][0]), float(win["lon"][-1]), float(win["lat"][0]), float(win["lat"][-1]),
                    np.asarray(win["level"], dtype=np.float64))
    return StepInputs(m_start, m_end, ss, se, ft, dens, mea, gb)
