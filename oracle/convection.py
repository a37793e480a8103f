"""Oracle: reduced Emanuel convection (``src/lpdm/convection/emanuel.py``).

numpy restatement, test infrastructure only. ``dt`` is the arithmetic type of
the column build: ``np.float32`` mirrors the reference, ``np.float64`` is the
FP64 column build the CUDA path uses.
"""

from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

GRAVITY = 9.80665
R_DRY = 287.05
R_VAPOR = 461.5
EPS = R_DRY / R_VAPOR
C_P = 1005.0
L_V = 2.5e6
P0_PA = 100000.0
KAPPA = R_DRY / C_P
P_MIN_PA = 1.0
T_MIN_K = 150.0
UPDRAFT_W_MAX = 5.0
CFL_MAX_OUTFLUX_FRAC = 0.9
CALL_INTERVAL_S = 3600.0


@dataclass(frozen=True)
class EmanuelParams:
    """``EmanuelReducedConvection.__init__`` (emanuel.py:531-565)."""

    closure_c: float = 0.03
    trigger_dtv_k: float = 0.9
    min_cape_j_kg: float = 50.0
    min_cloud_depth_m: float = 500.0


def saturation_vapor_pressure(t, dt):
    """emanuel.py:124-132 (Bolton 1980 Eq. 10)."""
    tc = t - dt(273.15)
    return dt(611.2) * np.exp(dt(17.67) * tc / (tc + dt(243.5)))


def q_to_e(q, p, dt):
    """emanuel.py:135-142"""
    return q * p / (dt(EPS) + dt(1.0 - EPS) * q)


def e_to_q(e, p, dt):
    """emanuel.py:145-148"""
    return dt(EPS) * e / (np.maximum(p, dt(P_MIN_PA)) - dt(1.0 - EPS) * e)


def virtual_temperature(t, q, dt):
    """emanuel.py:151-154"""
    return t * (dt(1.0) + dt(1.0 / EPS - 1.0) * q)


def lcl_temperature_bolton(t, q, p, dt):
    """emanuel.py:157-170 (Bolton 1980 Eq. 22)."""
    e_hpa = np.maximum(q_to_e(q, p, dt), dt(1.0)) / dt(100.0)
    den = dt(3.5) * np.log(t) - np.log(e_hpa) - dt(4.805)
    return dt(2840.0) / np.maximum(den, dt(1e-3)) + dt(55.0)


def lcl_pressure_poisson(t, t_lcl, p, dt):
    """emanuel.py:173-181"""
    return p * np.power(t_lcl / np.maximum(t, dt(T_MIN_K)), dt(C_P / R_DRY))


def potential_temperature(t, p, dt):
    """emanuel.py:184-187"""
    return t * np.power(dt(P0_PA) / np.maximum(p, dt(P_MIN_PA)), dt(KAPPA))


def equivalent_potential_temperature(t, q, p, dt):
    """emanuel.py:190-204"""
    t_lcl = lcl_temperature_bolton(t, q, p, dt)
    theta = potential_temperature(t, p, dt)
    return theta * np.exp(dt(L_V) * q / (dt(C_P) * np.maximum(t_lcl, dt(T_MIN_K))))


def saturation_specific_humidity(t, p, dt):
    """emanuel.py:207-212"""
    return e_to_q(saturation_vapor_pressure(t, dt), p, dt)


def lift_parcel(theta_e, p, dt, max_iter=30, t_min=180.0, t_max=350.0):
    """``lift_parcel_moist_pseudo_adiabatic`` (emanuel.py:215-255): fixed 30-step bisection."""
    lo = np.full_like(p, dt(t_min))
    hi = np.full_like(p, dt(t_max))
    for _ in range(max_iter):
        mid = dt(0.5) * (lo + hi)
        qs = saturation_specific_humidity(mid, p, dt)
        te = equivalent_potential_temperature(mid, qs, p, dt)
        too_high = te > theta_e
        hi = np.where(too_high, mid, hi)
        lo = np.where(too_high, lo, mid)
    return dt(0.5) * (lo + hi)


def layer_masses(p, dt):
    """``_layer_masses_per_area`` (emanuel.py:263-279)."""
    dp = np.zeros_like(p)
    dp[1:-1] = dt(0.5) * np.abs(p[:-2] - p[2:])
    dp[0] = np.abs(p[0] - p[1]) * dt(0.5)
    dp[-1] = np.abs(p[-2] - p[-1]) * dt(0.5)
    return dp / dt(GRAVITY)


def compute_lcl_lnb_cape(t_env, q_env, p, dt):
    """emanuel.py:282-399 → (i_lcl, i_lnb, cape, dTv at LCL+1)."""
    n = t_env.size
    t0, q0, p0 = t_env[:1], q_env[:1], p[:1]
    t_lcl = lcl_temperature_bolton(t0, q0, p0, dt)
    p_lcl = lcl_pressure_poisson(t0, t_lcl, p0, dt)[0]
    theta_e = equivalent_potential_temperature(t0, q0, p0, dt)[0]
    theta_sfc = potential_temperature(t0, p0, dt)[0]
    dry_t = theta_sfc * np.power(p / dt(P0_PA), dt(KAPPA))
    moist_t = lift_parcel(theta_e, p, dt)
    below = p >= p_lcl
    t_parcel = np.where(below, dry_t, moist_t)
    tv_env = virtual_temperature(t_env, q_env, dt)
    q_parcel = np.where(below, np.full_like(t_parcel, q_env[0]), saturation_specific_humidity(t_parcel, p, dt))
    tv_parcel = virtual_temperature(t_parcel, q_parcel, dt)
    buoy = (tv_parcel - tv_env) / np.maximum(tv_env, dt(T_MIN_K))
    above_idx = np.nonzero(~below)[0]
    i_lcl = int(above_idx[0]) if above_idx.size else -1
    if i_lcl >= 0 and i_lcl + 1 < n:
        dtv = tv_parcel[i_lcl + 1] - tv_env[i_lcl + 1]
    else:
        dtv = dt(-1.0)
    if i_lcl < 0:
        return -1, -1, dt(0.0), dt(dtv)
    dz = np.zeros(n, dtype=dt)
    dz[1:] = (dt(R_DRY) * dt(0.5) * (t_env[:-1] + t_env[1:])
              * (np.log(np.maximum(p[:-1], dt(P_MIN_PA))) - np.log(np.maximum(p[1:], dt(P_MIN_PA))))
              / dt(GRAVITY))
    pos = np.maximum(buoy, dt(0))
    pos[:i_lcl] = 0
    cape = (dt(GRAVITY) * pos * dz).sum(dtype=dt)
    neg = (buoy <= 0.0) & (np.arange(n) > i_lcl)
    i_lnb = int(np.nonzero(neg)[0][0]) if neg.any() else n - 1
    return i_lcl, i_lnb, dt(cape), dt(dtv)


def detrainment_weights(i_lcl, i_lnb, n, dt):
    """emanuel.py:402-426"""
    w = np.zeros(n, dtype=dt)
    depth = i_lnb - i_lcl
    if depth <= 0:
        return w
    for k in range(i_lcl, i_lnb + 1):
        w[k] = 1.0 - (k - i_lcl) / depth
    return w


def compute_mass_flux_matrix(p, i_lcl, i_lnb, m_b, dt):
    """emanuel.py:429-506: non-divergent updraft + compensating subsidence, CFL-capped."""
    n = p.size
    fmass = np.zeros((n, n), dtype=dt)
    if i_lcl < 0 or i_lnb <= i_lcl or m_b <= 0.0:
        return fmass
    m = layer_masses(p, dt)
    e = np.zeros(n, dtype=dt)
    bl_total = max(m[:i_lcl].sum(dtype=dt), dt(1e-12))
    e[:i_lcl] = dt(m_b) * m[:i_lcl] / bl_total
    w = detrainment_weights(i_lcl, i_lnb, n, dt)
    d = dt(m_b) * w / max(w.sum(dtype=dt), dt(1e-12))
    fmass = fmass + np.outer(e, d) / dt(m_b)
    phi = np.maximum((np.cumsum(e, dtype=dt) - np.cumsum(d, dtype=dt))[:-1], dt(0))
    fmass = fmass + np.diag(phi, -1).astype(dt)
    max_out = (fmass.sum(axis=1, dtype=dt) / np.maximum(m, dt(1e-12))).max()
    if float(max_out) > CFL_MAX_OUTFLUX_FRAC:
        fmass = fmass * (dt(CFL_MAX_OUTFLUX_FRAC) / max_out)
    return fmass


@dataclass
class ConvectionColumn:
    """Result of the per-window column build: fires?, and the backward CDF rows."""

    fires: bool
    height_col: np.ndarray  # [Z] ascending
    cum: np.ndarray | None  # [Z, Z]: cum[host, dest]
    i_lcl: int = -1
    i_lnb: int = -1
    cape: float = 0.0
    dtv: float = -1.0
    m_b: float = 0.0


def build_column(t_start, t_end, q_start, q_end, height, p_hpa, alpha, params: EmanuelParams, dt=np.float32):
    """``maybe_convect`` up to the transition matrix (emanuel.py:570-689 + 720-770).

    Inputs ``[Z, Y, X]`` (start/end), ``height [Z, Y, X]``, ``p_hpa [Z]``.
    """
    a = dt(alpha)
    t_field = t_start.astype(dt) * (dt(1.0) - a) + t_end.astype(dt) * a
    q_field = q_start.astype(dt) * (dt(1.0) - a) + q_end.astype(dt) * a
    t_col = t_field.mean(axis=(1, 2), dtype=np.float64).astype(dt)
    q_col = np.maximum(q_field.mean(axis=(1, 2), dtype=np.float64).astype(dt), dt(0))
    h_col = height.astype(dt).mean(axis=(1, 2), dtype=np.float64).astype(dt)
    p = np.asarray(p_hpa).astype(dt) * dt(100.0)
    ascending = bool(h_col[-1] > h_col[0])
    if not ascending:
        t_col, q_col, p, h_col = t_col[::-1].copy(), q_col[::-1].copy(), p[::-1].copy(), h_col[::-1].copy()
    i_lcl, i_lnb, cape, dtv = compute_lcl_lnb_cape(t_col, q_col, p, dt)
    fires = (i_lcl >= 0 and i_lnb > i_lcl and float(cape) >= params.min_cape_j_kg
             and float(dtv) >= params.trigger_dtv_k)
    if fires and float(h_col[i_lnb] - h_col[i_lcl]) < params.min_cloud_depth_m:
        fires = False
    col = ConvectionColumn(fires=fires, height_col=h_col, cum=None, i_lcl=i_lcl, i_lnb=i_lnb,
                           cape=float(cape), dtv=float(dtv))
    if not fires:
        return col
    rho_lcl = p[i_lcl] / (dt(R_DRY) * max(t_col[i_lcl], dt(T_MIN_K)))
    w_buoy = min(math.sqrt(2.0 * max(float(cape), 0.0)), UPDRAFT_W_MAX)
    m_b = params.closure_c * float(rho_lcl) * w_buoy
    fmass = compute_mass_flux_matrix(p, i_lcl, i_lnb, m_b * CALL_INTERVAL_S, dt)
    layer_mass = np.maximum(layer_masses(p, dt), dt(1e-6))
    fmf = fmass + np.diag(np.maximum(layer_mass - fmass.sum(axis=1, dtype=dt), dt(0))).astype(dt)
    trans = fmf.T
    prob = np.maximum(trans / np.maximum(layer_mass, dt(1e-12))[:, None], dt(0))
    probs = prob / np.maximum(prob.sum(axis=1, keepdims=True, dtype=dt), dt(1e-12))
    col.cum = np.cumsum(probs, axis=1, dtype=dt)
    col.m_b = m_b
    return col


def redistribute(z, active, col: ConvectionColumn, u1, u2, dt=np.float32):
    """``_redistribute_particles`` (emanuel.py:720-805), backward (column) sampling with
    injected uniforms ``u1`` (destination) and ``u2`` (height within the layer).
    Returns the new ``z`` and the number of displaced particles."""
    if not col.fires or not bool(np.any(active)):
        return z, 0
    h = col.height_col
    n_lev = h.size
    zz = z.astype(dt)
    iu = np.clip(np.searchsorted(h, zz, side="left"), 1, n_lev - 1)
    il = iu - 1
    host = np.where((zz - h[il]) < (h[iu] - zz), il, iu)
    cum_rows = col.cum[host]  # [N, Z]
    u1 = u1.astype(dt)
    dest = np.minimum((cum_rows < u1[:, None]).sum(axis=1), n_lev - 1)
    moved = active & (dest != host)
    n_moved = int(moved.sum())
    if n_moved == 0:
        return zz, 0
    lo = h[np.maximum(dest - 1, 0)]
    hi = h[dest]
    z_new = lo + u2.astype(dt) * (hi - lo)
    return np.where(moved, z_new, zz), n_moved
