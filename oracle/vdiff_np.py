"""CPU restatement of the implicit vertical tracer diffusion (test infrastructure only:
the oracle for the CUDA kernel ``fct_vert_diff``; nothing in the product path imports it).

Follows fesom_jax/tracer_diff.py:68-141 (``impl_vert_diff_one``, ``impl_vert_diff``) and
the tridiagonal solve of fesom_jax/ops.py:121-168 (``tdma``: forward elimination then
back substitution, rows initialised from zero), restated with numpy on ``[nod2D, nl]``
arrays. Pinned against the reference's own outputs in tests/golden/fct_vdiff_golden.npz
(tests/golden/make_vdiff_golden.py).
"""

from __future__ import annotations

import numpy as np


def _shift_down(x):
    """``out[..., k] = x[..., k-1]``, edge-replicated at k = 0 (tracer_diff.py:50-52)."""
    return np.concatenate([x[..., :1], x[..., :-1]], axis=-1)


def _shift_up(x):
    """``out[..., k] = x[..., k+1]``, zero at the last level (tracer_diff.py:55-57)."""
    return np.concatenate([x[..., 1:], np.zeros_like(x[..., :1])], axis=-1)


def tdma(a, b, c, d):
    """Per-row tridiagonal solve along the last axis (ops.py:121-168)."""
    n, K = d.shape
    cp = np.zeros((n, K))
    dp = np.zeros((n, K))
    cprev = np.zeros(n)
    dprev = np.zeros(n)
    for k in range(K):
        m = b[:, k] - a[:, k] * cprev
        cprev = c[:, k] / m
        dprev = (d[:, k] - a[:, k] * dprev) / m
        cp[:, k], dp[:, k] = cprev, dprev
    x = np.zeros((n, K))
    xn = np.zeros(n)
    for k in range(K - 1, -1, -1):
        xn = dp[:, k] - cp[:, k] * xn
        x[:, k] = xn
    return x


def impl_vert_diff_one(m, T, Kv, hnode_new, *, dt, bc_surf=None, sw_3d=None, Z3d=None):
    """One tracer (tracer_diff.py:68-123)."""
    nl = m.nl
    if Z3d is None:
        Zp = np.concatenate([m.Z, m.Z[-1:]])
        dZ_up = (_shift_down(Zp) - Zp)[None, :]
        dZ_dn = (Zp - _shift_up(Zp))[None, :]
    else:
        dZ_up = _shift_down(Z3d) - Z3d
        dZ_dn = Z3d - _shift_up(Z3d)
    dZ_up = np.where(dZ_up == 0.0, 1.0, dZ_up)
    dZ_dn = np.where(dZ_dn == 0.0, 1.0, dZ_dn)
    area = m.area
    safe_av = np.where(m.areasvol > 0.0, m.areasvol, 1.0)
    a_full = -Kv * dt / dZ_up * (area / safe_av)
    c_full = -_shift_up(Kv) * dt / dZ_dn * (_shift_up(area) / safe_av)
    k = np.arange(nl)[None, :]
    nzmin = (m.ulevels_nod2D - 1)[:, None]
    nzmax = (m.nlevels_nod2D - 1)[:, None]
    valid = m.node_layer_mask
    surf = k == nzmin
    bot = k == (nzmax - 1)
    a = np.where(surf, 0.0, a_full)
    c = np.where(bot, 0.0, c_full)
    b = np.where(valid, -a - c + hnode_new, 1.0)
    a = np.where(valid, a, 0.0)
    c = np.where(valid, c, 0.0)
    rhs = np.where(valid, a * (T - _shift_down(T)) + c * (T - _shift_up(T)), 0.0)
    if bc_surf is not None:
        rhs = rhs + np.where(surf & valid, bc_surf[:, None], 0.0)
    if sw_3d is not None:
        sw_div = (sw_3d - _shift_up(sw_3d) * (_shift_up(area) / safe_av)) * dt
        rhs = rhs + np.where(valid, sw_div, 0.0)
    dT = tdma(a, b, c, rhs)
    return T + np.where(valid, dT, 0.0)


def impl_vert_diff(m, T, S, Kv, hnode_new, *, dt, bc_T=None, bc_S=None, sw_3d=None,
                   Z3d=None):
    """T and S with one Kv; shortwave on T only (tracer_diff.py:126-141)."""
    return (impl_vert_diff_one(m, T, Kv, hnode_new, dt=dt, bc_surf=bc_T, sw_3d=sw_3d, Z3d=Z3d),
            impl_vert_diff_one(m, S, Kv, hnode_new, dt=dt, bc_surf=bc_S, sw_3d=None, Z3d=Z3d))
