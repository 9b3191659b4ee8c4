"""CPU oracle (test infrastructure only): vectorised numpy restatement of the reference
FCT tracer advection, fesom_jax/tracer_adv.py:43-578.

This module is the checker for the CUDA path. Only ``tests/``, ``__graft_entry__.smoke``
and ``bench.py``'s CPU-baseline leg may import it; the product path never calls it.

Each function restates one reference function (cited per function) with numpy in place
of ``jax.numpy``: ``segment_sum`` becomes ``np.add.at`` (ascending index order, the order
the reference's C ancestor used), ``segment_max/min`` become ``np.maximum.at`` /
``np.minimum.at`` from -inf / +inf (the identity elements ``jax.ops.segment_max/min``
use for empty segments). The mesh argument is any object with the reference ``Mesh``
field names (``fesom_jax_b200.mesh.Mesh`` qualifies).

Pinning: ``tests/golden/make_golden.py`` runs the reference's own ``tracer_adv`` (and the
loop-based ``_fct_ref`` of fesom_jax/tests/test_tracers.py:325-516) on seeded pi-mesh
inputs; ``tests/test_oracle_golden.py`` checks this module against those vectors.
"""

from __future__ import annotations

import numpy as np

R_EARTH = 6367500.0          # fesom_jax/config.py:41
AB_OLD = -(0.5 + 0.1)        # tracer_adv.py:44-46 (AB2, eps = 0.1)
AB_NEW = (1.5 + 0.1)
FLUX_EPS = 1e-16             # tracer_adv.py:192
BIG = 1e3                    # tracer_adv.py:193


def shift_down(x):
    """``out[..., k] = x[..., k-1]``, edge-replicated at k=0 (tracer_adv.py:49-51)."""
    return np.concatenate([x[..., :1], x[..., :-1]], axis=-1)


def shift_up(x):
    """``out[..., k] = x[..., k+1]``, zero at the last level (tracer_adv.py:54-56)."""
    return np.concatenate([x[..., 1:], np.zeros_like(x[..., :1])], axis=-1)


def scatter_add(vals, seg, num_segments):
    """Masked segment sum (fesom_jax/ops.py:56-81): entries with ``seg < 0`` dropped."""
    seg = np.asarray(seg)
    lead = seg.ndim
    seg_f = seg.reshape(-1)
    v = np.asarray(vals).reshape((seg_f.shape[0],) + np.asarray(vals).shape[lead:])
    ok = seg_f >= 0
    out = np.zeros((num_segments,) + v.shape[1:])
    np.add.at(out, seg_f[ok], v[ok])
    return out


def segment_max(vals, seg, num_segments):
    out = np.full((num_segments,) + vals.shape[1:], -np.inf)
    np.maximum.at(out, seg, vals)
    return out


def segment_min(vals, seg, num_segments):
    out = np.full((num_segments,) + vals.shape[1:], np.inf)
    np.minimum.at(out, seg, vals)
    return out


def tracer_ab(values, valuesold):
    """AB2 extrapolation (tracer_adv.py:59-66): ``(ttfAB, valuesold_new=values)``."""
    return AB_OLD * valuesold + AB_NEW * values, values


def edge_vflux(m, uv, helem):
    """Per-edge volume flux ``[edge2D, nl]`` (tracer_adv.py:69-93)."""
    el1, el2 = m.edge_tri[:, 0], m.edge_tri[:, 1]
    has1, has2 = el1 >= 0, el2 >= 0
    e1 = np.where(has1, el1, 0)
    e2 = np.where(has2, el2, 0)
    cr = m.edge_cross_dxdy
    U, V = uv[:, :, 0], uv[:, :, 1]
    lm = m.elem_layer_mask
    t1 = np.where(lm[e1] & has1[:, None], (U[e1] * cr[:, 1:2] - V[e1] * cr[:, 0:1]) * helem[e1], 0.0)
    t2 = np.where(lm[e2] & has2[:, None], (V[e2] * cr[:, 2:3] - U[e2] * cr[:, 3:4]) * helem[e2], 0.0)
    return t1 + t2


def adv_flux_hor(m, uv, helem, ttf, vflux=None):
    """Upwind horizontal edge flux (tracer_adv.py:96-105)."""
    vf = edge_vflux(m, uv, helem) if vflux is None else vflux
    T1, T2 = ttf[m.edges[:, 0]], ttf[m.edges[:, 1]]
    av = np.abs(vf)
    return -0.5 * (T1 * (vf + av) + T2 * (vf - av))


def adv_flux_ver(m, w_e, ttf):
    """Upwind vertical interface flux, layer-masked (tracer_adv.py:108-120)."""
    aw = np.abs(w_e)
    flux = -0.5 * (ttf * (w_e + aw) + shift_down(ttf) * (w_e - aw)) * m.area
    return np.where(m.node_layer_mask, flux, 0.0)


def compute_fct_lo(m, flux_h, flux_v, T, hnode, hnode_new, dt):
    """Low-order ALE solution (tracer_adv.py:298-313)."""
    div_h = scatter_add(np.stack([flux_h, -flux_h], axis=1), m.edges, m.nod2D)
    div_v = flux_v - shift_up(flux_v)
    a = m.areasvol
    safe_a = np.where(a > 0.0, a, 1.0)
    safe_hn = np.where(hnode_new > 0.0, hnode_new, 1.0)
    lo = (T * hnode + (div_h + div_v) * dt / safe_a) / safe_hn
    valid = m.node_layer_mask & (hnode_new > 0.0) & (a > 0.0)
    return np.where(valid, lo, 0.0)


def tracer_gradient_elements(m, ttf):
    """Element gradient ``[elem2D, nl, 2]`` (tracer_adv.py:316-326)."""
    t = ttf[m.elem_nodes]
    gs = m.gradient_sca
    gx = gs[:, 0:1] * t[:, 0] + gs[:, 1:2] * t[:, 1] + gs[:, 2:3] * t[:, 2]
    gy = gs[:, 3:4] * t[:, 0] + gs[:, 4:5] * t[:, 1] + gs[:, 5:6] * t[:, 2]
    em = m.elem_layer_mask
    return np.stack([np.where(em, gx, 0.0), np.where(em, gy, 0.0)], axis=-1)


def node_avg_grad(m, tr_xy):
    """Area-weighted node average of element gradients (tracer_adv.py:329-341)."""
    aw = np.where(m.elem_layer_mask, m.elem_area[:, None], 0.0)
    contrib = tr_xy * aw[:, :, None]
    E = m.elem2D
    cb = np.broadcast_to(contrib[:, None], (E, 3) + tr_xy.shape[1:])
    wb = np.broadcast_to(aw[:, None], (E, 3, m.nl))
    num = scatter_add(cb, m.elem_nodes, m.nod2D)
    den = scatter_add(wb, m.elem_nodes, m.nod2D)
    return num / np.where(den > 0.0, den, 1.0)[:, :, None]


def fill_up_dn_grad(m, tr_xy):
    """Per-edge MFCT gradients ``[edge2D, nl, 4]`` (tracer_adv.py:344-368)."""
    gnode = node_avg_grad(m, tr_xy)
    up, dn = m.edge_up_dn_tri[:, 0], m.edge_up_dn_tri[:, 1]
    interior = (up >= 0) & (dn >= 0)
    gup = tr_xy[np.where(up >= 0, up, 0)]
    gdn = tr_xy[np.where(dn >= 0, dn, 0)]
    n1, n2 = m.edges[:, 0], m.edges[:, 1]
    gn1, gn2 = gnode[n1], gnode[n2]
    k = np.arange(m.nl)[None, :]
    nzmin = np.maximum(m.ulevels_nod2D_max[n1], m.ulevels_nod2D_max[n2])[:, None] - 1
    nzmax = np.minimum(m.nlevels_nod2D_min[n1], m.nlevels_nod2D_min[n2])[:, None] - 1
    use = interior[:, None] & (k >= nzmin) & (k < nzmax)
    return np.stack([np.where(use, gup[:, :, 0], gn1[:, :, 0]),
                     np.where(use, gdn[:, :, 0], gn2[:, :, 0]),
                     np.where(use, gup[:, :, 1], gn1[:, :, 1]),
                     np.where(use, gdn[:, :, 1], gn2[:, :, 1])], axis=-1)


def adv_flux_hor_ho(m, uv, helem, ttf, eud, vflux=None):
    """MFCT 3rd-order horizontal flux (tracer_adv.py:196-225)."""
    vf = edge_vflux(m, uv, helem) if vflux is None else vflux
    n1, n2 = m.edges[:, 0], m.edges[:, 1]
    T1, T2 = ttf[n1], ttf[n2]
    diff = T2 - T1
    el1, el2 = m.edge_tri[:, 0], m.edge_tri[:, 1]
    has2 = el2 >= 0
    a = R_EARTH * m.elem_cos[np.where(el1 >= 0, el1, 0)]
    a = np.where(has2, 0.5 * (a + R_EARTH * m.elem_cos[np.where(has2, el2, 0)]), a)[:, None]
    edx, edy = m.edge_dxdy[:, 0:1], m.edge_dxdy[:, 1:2]
    Tm1 = T1 + (2.0 * diff + edx * a * eud[:, :, 0] + edy * R_EARTH * eud[:, :, 2]) / 6.0
    Tm2 = T2 - (2.0 * diff + edx * a * eud[:, :, 1] + edy * R_EARTH * eud[:, :, 3]) / 6.0
    av = np.abs(vf)
    return -0.5 * ((vf + av) * Tm1 + (vf - av) * Tm2)


def z_stencil(Z):
    """Padded mid-depths and their shifts (tracer_adv.py:228-238)."""
    Zp = np.concatenate([Z, Z[-1:]])
    return (Zp, np.concatenate([Zp[:1], Zp[:-1]]), np.concatenate([Zp[:2], Zp[:-2]]),
            np.concatenate([Zp[1:], Zp[-1:]]))


def adv_flux_ver_ho(m, w_e, ttf, Z3d=None, zbar3=None):
    """QR4C 4th-order vertical flux, interface-masked (tracer_adv.py:241-295)."""
    W, area, T = w_e, m.area, ttf
    Tm1 = shift_down(T)
    Tm2 = shift_down(Tm1)
    Tp1 = shift_up(T)
    surf = -T * W * area
    cent = -0.5 * (Tm1 + T) * W * area
    if Z3d is None:
        Z_nz, Z_m1, Z_m2, Z_p1 = z_stencil(m.Z)
        zb = m.zbar
    else:
        Z_nz = Z3d
        Z_m1 = shift_down(Z3d)
        Z_m2 = shift_down(Z_m1)
        Z_p1 = np.concatenate([Z3d[:, 1:], Z3d[:, -1:]], axis=1)
        zb = zbar3

    def safe(x):
        return np.where(x == 0.0, 1.0, x)

    qc = (Tm1 - T) / safe(Z_m1 - Z_nz)
    qu = (T - Tp1) / safe(Z_nz - Z_p1)
    qd = (Tm2 - Tm1) / safe(Z_m2 - Z_m1)
    Tmean1 = T + (2.0 * qc + qu) * (zb - Z_nz) / 3.0
    Tmean2 = Tm1 + (2.0 * qc + qd) * (zb - Z_m1) / 3.0
    quad = -0.5 * (Tmean1 + Tmean2) * W * area
    k = np.arange(m.nl)[None, :]
    nzmin = (m.ulevels_nod2D - 1)[:, None]
    nzmax = (m.nlevels_nod2D - 1)[:, None]
    is_surf = k == nzmin
    is_bot = k == nzmax
    is_cent = (k == nzmin + 1) | (k == nzmax - 1)
    is_int = (k >= nzmin + 2) & (k <= nzmax - 2)
    hi = np.where(is_surf, surf, np.where(is_bot, 0.0, np.where(is_cent, cent,
                                                                 np.where(is_int, quad, 0.0))))
    return np.where(m.node_iface_mask, hi, 0.0)


def zalesak_limit(m, T, LO, adf_h, adf_v, hnode_new, dt, aux=None):
    """Zalesak limiter (tracer_adv.py:371-466). Returns ``(adf_h_lim, adf_v_lim)``;
    when ``aux`` is a dict the limiter's intermediates are stored in it."""
    nl = m.nl
    nlm = m.node_layer_mask
    ttf_max = np.maximum(LO, T)
    ttf_min = np.minimum(LO, T)
    em = m.elem_layer_mask
    aux_max = np.where(em, np.max(ttf_max[m.elem_nodes], axis=1), -BIG)
    aux_min = np.where(em, np.min(ttf_min[m.elem_nodes], axis=1), BIG)
    seg = m.elem_nodes.reshape(-1)
    E = m.elem2D
    tvert_max = segment_max(np.repeat(aux_max, 3, axis=0), seg, m.nod2D)
    tvert_min = segment_min(np.repeat(aux_min, 3, axis=0), seg, m.nod2D)
    k = np.arange(nl)[None, :]
    nzmin = (m.ulevels_nod2D - 1)[:, None]
    nzmax = (m.nlevels_nod2D - 1)[:, None]
    use_own = (k == nzmin) | (k == nzmax - 1)
    tmax3 = np.maximum(np.maximum(shift_down(tvert_max), tvert_max), shift_up(tvert_max))
    tmin3 = np.minimum(np.minimum(shift_down(tvert_min), tvert_min), shift_up(tvert_min))
    with np.errstate(invalid="ignore"):
        fct_ttf_max = np.where(use_own, tvert_max, tmax3) - LO
        fct_ttf_min = np.where(use_own, tvert_min, tmin3) - LO
    fct_ttf_max = np.where(nlm, fct_ttf_max, 0.0)
    fct_ttf_min = np.where(nlm, fct_ttf_min, 0.0)
    fv_bot = shift_up(adf_v)
    pos_v = np.where(nlm, np.maximum(adf_v, 0.0) + np.maximum(-fv_bot, 0.0), 0.0)
    neg_v = np.where(nlm, np.minimum(adf_v, 0.0) + np.minimum(-fv_bot, 0.0), 0.0)
    ph = np.stack([np.maximum(adf_h, 0.0), np.maximum(-adf_h, 0.0)], axis=1)
    nh = np.stack([np.minimum(adf_h, 0.0), np.minimum(-adf_h, 0.0)], axis=1)
    fct_plus = pos_v + scatter_add(ph, m.edges, m.nod2D)
    fct_minus = neg_v + scatter_add(nh, m.edges, m.nod2D)
    a = m.areasvol
    safe_a = np.where(a > 0.0, a, 1.0)
    safe_hn = np.where(hnode_new > 0.0, hnode_new, 1.0)
    flux_pos = fct_plus * dt / safe_a / safe_hn + FLUX_EPS
    flux_neg = fct_minus * dt / safe_a / safe_hn - FLUX_EPS
    plus_fac = np.minimum(1.0, fct_ttf_max / flux_pos)
    minus_fac = np.minimum(1.0, fct_ttf_min / flux_neg)
    valid = nlm & (a > 0.0) & (hnode_new > 0.0)
    plus_fac = np.where(valid, plus_fac, 1.0)
    minus_fac = np.where(valid, minus_fac, 1.0)
    ae_surf = np.where(adf_v >= 0.0, plus_fac, minus_fac)
    ae_int = np.where(adf_v >= 0.0, np.minimum(shift_down(minus_fac), plus_fac),
                      np.minimum(shift_down(plus_fac), minus_fac))
    ae_v = np.where(k == nzmin, ae_surf, ae_int)
    adf_v_lim = np.where(m.node_iface_mask, ae_v * adf_v, 0.0)
    n1, n2 = m.edges[:, 0], m.edges[:, 1]
    ae_h = np.where(adf_h >= 0.0, np.minimum(plus_fac[n1], minus_fac[n2]),
                    np.minimum(minus_fac[n1], plus_fac[n2]))
    if aux is not None:
        aux.update(tvert_max=tvert_max, tvert_min=tvert_min, fct_ttf_max=fct_ttf_max,
                   fct_ttf_min=fct_ttf_min, fct_plus=fct_plus, fct_minus=fct_minus,
                   plus_fac=plus_fac, minus_fac=minus_fac, aux_max=aux_max, aux_min=aux_min)
    return ae_h * adf_h, adf_v_lim


def flux2dtracer_fct(m, T, LO, adf_h, adf_v, hnode, hnode_new, dt):
    """``del_ttf`` assembly for FCT (tracer_adv.py:469-484)."""
    nlm = m.node_layer_mask
    a = m.areasvol
    safe_a = np.where(a > 0.0, a, 1.0)
    lo_trans = -T * hnode + LO * hnode_new
    vdiv = np.where(a > 0.0, (adf_v - shift_up(adf_v)) * dt / safe_a, 0.0)
    dttf_v = np.where(nlm, lo_trans + vdiv, 0.0)
    hsc = scatter_add(np.stack([adf_h, -adf_h], axis=1), m.edges, m.nod2D)
    dttf_h = np.where(nlm, hsc * dt / safe_a, 0.0)
    return dttf_h + dttf_v


def ale_reconstruct(m, T, del_ttf, hnode, hnode_new):
    """ALE reconstruction; invalid lanes keep ``T`` (tracer_adv.py:142-151)."""
    d = del_ttf + T * (hnode - hnode_new)
    safe_hn = np.where(hnode_new > 0.0, hnode_new, 1.0)
    upd = m.node_layer_mask & (hnode_new > 0.0)
    return T + np.where(upd, d / safe_hn, 0.0)


def tdma(a, b, c, d):
    """Thomas solve along the last axis (fesom_jax/ops.py:121-168)."""
    K = b.shape[-1]
    cp = np.zeros_like(b)
    dp = np.zeros_like(b)
    cprev = np.zeros(b.shape[:-1])
    dprev = np.zeros(b.shape[:-1])
    for k in range(K):
        mden = b[..., k] - a[..., k] * cprev
        cprev = c[..., k] / mden
        dprev = (d[..., k] - a[..., k] * dprev) / mden
        cp[..., k], dp[..., k] = cprev, dprev
    x = np.zeros_like(b)
    nxt = np.zeros(b.shape[:-1])
    for k in range(K - 1, -1, -1):
        nxt = dp[..., k] - cp[..., k] * nxt
        x[..., k] = nxt
    return x


def adv_tra_vert_impl(m, w_i, T, hnode_new, dt):
    """Implicit vertical advection by the split ``w_i`` (tracer_adv.py:487-529)."""
    safe_av = np.where(m.areasvol > 0.0, m.areasvol, 1.0)
    v_top = dt * m.area / safe_av
    v_bot = dt * shift_up(m.area) / safe_av
    wu, wd = w_i, shift_up(w_i)
    k = np.arange(m.nl)[None, :]
    nzmin = (m.ulevels_nod2D - 1)[:, None]
    nzmax = (m.nlevels_nod2D - 1)[:, None]
    valid = m.node_layer_mask
    surf = k == nzmin
    bot = k == (nzmax - 1)
    a_adv = np.where(surf, 0.0, np.minimum(0.0, wu)) * v_top
    b_top = np.where(surf, wu, np.maximum(0.0, wu)) * v_top
    b_bot = np.where(bot, 0.0, -np.minimum(0.0, wd)) * v_bot
    c_adv = np.where(bot, 0.0, -np.maximum(0.0, wd)) * v_bot
    b_adv = b_top + b_bot
    a = np.where(valid, a_adv, 0.0)
    c = np.where(valid, c_adv, 0.0)
    b = np.where(valid, hnode_new + b_adv, 1.0)
    rhs = np.where(valid, -(a * shift_down(T) + b_adv * T + c * shift_up(T)), 0.0)
    dT = tdma(a, b, c, rhs)
    return T + np.where(valid, dT, 0.0)


def advect_one_fct(m, uv, w_e, helem, hnode, hnode_new, T, T_old, *, dt,
                   Z3d=None, zbar3=None, w_i=None, intermediates=None):
    """One tracer's FCT advection + ALE reconstruction (tracer_adv.py:532-578).
    Returns ``(T_new, T_old_new)``; ``intermediates`` (a dict) receives the stages."""
    ttfAB, T_old_new = tracer_ab(T, T_old)
    vflux = edge_vflux(m, uv, helem)
    flux_h_lo = adv_flux_hor(m, uv, helem, T, vflux)
    flux_v_lo = adv_flux_ver(m, w_e, T)
    LO = compute_fct_lo(m, flux_h_lo, flux_v_lo, T, hnode, hnode_new, dt)
    if w_i is not None:
        LO = adv_tra_vert_impl(m, w_i, LO, hnode_new, dt)
    tr_xy = tracer_gradient_elements(m, T)
    eud = fill_up_dn_grad(m, tr_xy)
    adf_h = adv_flux_hor_ho(m, uv, helem, ttfAB, eud, vflux) - flux_h_lo
    if w_i is None:
        adf_v = adv_flux_ver_ho(m, w_e, ttfAB, Z3d, zbar3) - flux_v_lo
    else:
        w_full = w_e + w_i
        adf_v = adv_flux_ver_ho(m, w_full, ttfAB, Z3d, zbar3) - adv_flux_ver(m, w_full, T)
    lim = {} if intermediates is not None else None
    adf_h_l, adf_v_l = zalesak_limit(m, T, LO, adf_h, adf_v, hnode_new, dt, aux=lim)
    del_ttf = flux2dtracer_fct(m, T, LO, adf_h_l, adf_v_l, hnode, hnode_new, dt)
    T_new = ale_reconstruct(m, T, del_ttf, hnode, hnode_new)
    if intermediates is not None:
        intermediates.update(lim)
        intermediates.update(vflux=vflux, flux_h_lo=flux_h_lo, flux_v_lo=flux_v_lo, LO=LO,
                             tr_xy=tr_xy, eud=eud, gnode=node_avg_grad(m, tr_xy),
                             adf_h=adf_h, adf_v=adf_v, adf_h_lim=adf_h_l,
                             adf_v_lim=adf_v_l, del_ttf=del_ttf)
    return T_new, T_old_new
