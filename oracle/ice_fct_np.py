"""CPU restatement of the sea-ice FCT advection (test infrastructure only: the oracle for
the CUDA kernels behind ``fct_ice_solve``; nothing in the product path imports it).

Follows fesom_jax/ice_adv.py:37-194 (``_mm_times``, ``_tg_rhs``, ``_solve_low_order``,
``_solve_high_order``, ``_fem_fct``, ``fct_solve``) on numpy arrays. Pinned against the
reference's own outputs in tests/golden/fct_ice_golden.npz
(tests/golden/make_ice_golden.py).
"""

from __future__ import annotations

import numpy as np

ICE_SCALE_AREA = 2.0e8   # ice_adv.py:33
ICE_FLUX_EPS = 1.0e-12   # ice_adv.py:34


def _scatter(contrib, en, n):
    out = np.zeros(n)
    np.add.at(out, en.reshape(-1), contrib.reshape(-1))
    return out


def mm_times(m, X):
    """FE consistent-mass product (ice_adv.py:37-44)."""
    en = m.elem_nodes
    Xv = X[en]
    contrib = (m.elem_area / 12.0)[:, None] * (Xv + Xv.sum(axis=1, keepdims=True))
    contrib = np.where((m.ulevels <= 1)[:, None], contrib, 0.0)
    return _scatter(contrib, en, m.nod2D)


def tg_rhs(m, u, v, X, *, dt, ice_diff):
    """Taylor-Galerkin RHS of one tracer (ice_adv.py:47-75)."""
    en = m.elem_nodes
    gs = m.gradient_sca
    dx, dy = gs[:, 0:3], gs[:, 3:6]
    vol = m.elem_area
    U, V = u[en], v[en]
    um, vm = U.sum(axis=1), V.sum(axis=1)
    diff = ice_diff * np.sqrt(vol / ICE_SCALE_AREA)
    a = (dx[:, :, None] * (um[:, None, None] + U[:, None, :])
         + dy[:, :, None] * (vm[:, None, None] + V[:, None, :])) / 12.0
    b = diff[:, None, None] * (dx[:, :, None] * dx[:, None, :] + dy[:, :, None] * dy[:, None, :])
    udn = um[:, None] * dx + vm[:, None] * dy
    c = 0.5 * dt * (udn[:, :, None] * udn[:, None, :]) / 9.0
    entries = vol[:, None, None] * dt * (a - b - c)
    on = (m.ulevels <= 1)[:, None]
    contrib = np.where(on, (entries * X[en][:, None, :]).sum(axis=2), 0.0)
    return _scatter(contrib, en, m.nod2D)


def fem_fct(m, vals, vals_l, dvals, *, gamma):
    """Zalesak limiter of one tracer (ice_adv.py:110-172)."""
    en = m.elem_nodes
    area = m.area[:, 0]
    inv_area = 1.0 / np.where(area > 0, area, 1.0)
    nc_e = m.ulevels <= 1
    nc_n = m.ulevels_nod2D <= 1
    vol = m.elem_area
    w = gamma * vals + dvals
    wv = w[en]
    s = wv.sum(axis=1, keepdims=True) - 3.0 * wv
    flux = np.where(nc_e[:, None], -s * (vol[:, None] * inv_area[en]) / 12.0, 0.0)
    elem_hi = np.maximum(vals_l[en].max(1), vals[en].max(1))
    elem_lo = np.minimum(vals_l[en].min(1), vals[en].min(1))
    hi = np.full(m.nod2D, -np.inf)
    lo = np.full(m.nod2D, np.inf)
    np.maximum.at(hi, en.reshape(-1), np.repeat(np.where(nc_e, elem_hi, -np.inf), 3))
    np.minimum.at(lo, en.reshape(-1), np.repeat(np.where(nc_e, elem_lo, np.inf), 3))
    hi = np.where(np.isfinite(hi), hi, 0.0)
    lo = np.where(np.isfinite(lo), lo, 0.0)
    tmax, tmin = hi - vals_l, lo - vals_l
    fp = _scatter(np.maximum(flux, 0.0), en, m.nod2D)
    fm = _scatter(np.minimum(flux, 0.0), en, m.nod2D)
    with np.errstate(divide="ignore", invalid="ignore"):
        pplus = np.where(fp > 0.0, np.minimum(tmax / np.where(fp > ICE_FLUX_EPS, fp, ICE_FLUX_EPS),
                                              1.0), 0.0)
        pminus = np.where(fm < 0.0, np.minimum(tmin / np.where(fm < -ICE_FLUX_EPS, fm,
                                                               -ICE_FLUX_EPS), 1.0), 0.0)
    pplus = np.where(nc_n, pplus, 0.0)
    pminus = np.where(nc_n, pminus, 0.0)
    cand = np.where(flux >= 0.0, pplus[en], pminus[en])
    ae = cand.min(axis=1)
    limited = np.where(nc_e[:, None], flux * ae[:, None], 0.0)
    return vals_l + _scatter(limited, en, m.nod2D)


def fct_solve(m, a_ice, m_ice, m_snow, u_ice, v_ice, *, dt, gamma=0.5, ice_diff=10.0):
    """One sea-ice FCT step of (a_ice, m_ice, m_snow) (ice_adv.py:175-194)."""
    area = m.area[:, 0]
    inv_area = 1.0 / np.where(area > 0, area, 1.0)
    nc = m.ulevels_nod2D <= 1
    out = []
    for X in (a_ice, m_ice, m_snow):
        rhs = tg_rhs(m, u_ice, v_ice, X, dt=dt, ice_diff=ice_diff)
        d = np.where(nc, rhs * inv_area, 0.0)
        for _ in range(2):
            d = np.where(nc, d + (rhs - mm_times(m, d)) * inv_area, d)
        X_l = np.where(nc, (rhs + gamma * mm_times(m, X)) * inv_area + (1.0 - gamma) * X, X)
        out.append(fem_fct(m, X, X_l, d, gamma=gamma))
    return tuple(out)
