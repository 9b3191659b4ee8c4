"""Rebuild the inputs of the golden pi cases (``tests/golden/make_golden.py``) without the
reference checkout, and compare a result against the stored vectors."""

from __future__ import annotations

import hashlib
from pathlib import Path

import numpy as np

from fesom_jax_b200 import inputs as I

GOLDEN = Path(__file__).resolve().parent / "golden" / "fct_pi_golden.npz"
DT = 3600.0
SAMPLE = slice(0, None, 4)
# max-norm relative tolerance of the FCT path (per step, over wet lanes)
RTOL = 1e-12


def field_digest(m, x, mask=None):
    mask = m.node_layer_mask if mask is None else mask
    wts = np.random.default_rng(1234).normal(size=mask.shape)
    xm = np.where(mask, x, 0.0)
    return np.array([xm.sum(), (wts * xm).sum(), np.abs(wts * xm).sum(), (xm * xm).sum()])


def _sha(*arrays):
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.digest()


def cases(m):
    """name -> dict(uv, w_e, helem, hnode, hnode_new, T, T_old, kw)."""
    lm = m.node_layer_mask
    f = I.make_fields(m, seed=0)
    f_ab2 = I.make_fields(m, seed=0, ab2=True)
    f_white = I.make_fields(m, seed=0, kind="white")
    k = np.arange(m.nl)[None, :]
    sharp = np.where(lm, 10.0 + 5.0 * np.sin(np.arange(m.nod2D)[:, None] * 0.7)
                     * np.cos(k * 1.3), 0.0)
    ten = np.where(lm, 10.0, 0.0)
    const = np.where(lm, 20.0, 0.0)
    zbar3 = np.broadcast_to(m.zbar, (m.nod2D, m.nl)).copy()
    zbar3[:, 1:] *= 1.0 + 0.01 * np.sin(np.arange(m.nod2D))[:, None]
    Z3d = np.concatenate([0.5 * (zbar3[:, :-1] + zbar3[:, 1:]),
                          0.5 * (zbar3[:, -2:-1] + zbar3[:, -1:])], axis=1)
    w_i = 0.3 * f.w_e
    base = dict(helem=f.helem, hnode=f.hnode, hnode_new=f.hnode_new)
    out = {
        "T_step1": dict(uv=f.uv, w_e=f.w_e, T=f.tracers[0], T_old=f.tracers_old[0], kw={}),
        "S_step1": dict(uv=f.uv, w_e=f.w_e, T=f.tracers[1], T_old=f.tracers_old[1], kw={}),
        "T_ab2": dict(uv=f_ab2.uv, w_e=f_ab2.w_e, T=f_ab2.tracers[0],
                      T_old=f_ab2.tracers_old[0], kw={}),
        "sharp_x5": dict(uv=f_white.uv * 5.0, w_e=f_white.w_e * 5.0, T=sharp, T_old=ten, kw={}),
        "const": dict(uv=f.uv, w_e=f.w_e, T=const, T_old=const, kw={}),
        "T_wsplit_zstar": dict(uv=f.uv, w_e=f.w_e - w_i, T=f.tracers[0],
                               T_old=f_ab2.tracers_old[0],
                               kw=dict(w_i=w_i, Z3d=Z3d, zbar3=zbar3)),
    }
    for c in out.values():
        c.update(base)
    return out


def load_golden():
    return dict(np.load(GOLDEN))


def check_against_golden(m, g, name, case, T_new, rtol=RTOL):
    """Assert ``T_new`` matches the golden case: input digest, sampled lanes (max-norm
    relative), and the full-field digest. Returns the sampled relative error."""
    c = case
    assert _sha(c["uv"], c["w_e"], c["T"], c["T_old"], *c["kw"].values()) == \
        g[f"{name}__in_digest"].tobytes(), f"{name}: input generation drifted"
    lm = m.node_layer_mask
    ref = g[f"{name}__T_new"]
    got = T_new[SAMPLE][lm[SAMPLE]]
    scale = max(np.max(np.abs(ref)), 1e-300)
    err = np.max(np.abs(got - ref)) / scale
    assert err <= rtol, f"{name}: sampled max|d|/max|ref| = {err:.3e}"
    dg, dr = field_digest(m, T_new), g[f"{name}__digest"]
    assert abs(dg[0] - dr[0]) <= rtol * abs(dr[0]) * 10 + 1e-300, f"{name}: sum"
    assert abs(dg[1] - dr[1]) <= rtol * dr[2] * 10, f"{name}: weighted sum"
    assert abs(dg[3] - dr[3]) <= rtol * dr[3] * 10, f"{name}: sum of squares"
    return err


VDIFF_GOLDEN = Path(__file__).resolve().parent / "golden" / "fct_vdiff_golden.npz"


def vdiff_cases(m):
    """Implicit vertical diffusion cases on ``m``: name -> dict(T, Kv, hnode_new, kw)
    (``kw``: bc_surf / sw_3d / Z3d of fesom_jax/tracer_diff.py:68)."""
    rng = np.random.default_rng(77)
    f = I.make_fields(m, seed=0)
    lm, im = m.node_layer_mask, m.node_iface_mask
    frac = I.layer_depth_fraction(m)[None, :]
    Kv = np.where(im, 1e-5 + 1e-2 * np.exp(-5.0 * frac) * rng.uniform(0.5, 1.5, im.shape), 0.0)
    k = np.arange(m.nl)[None, :]
    zbar3 = np.broadcast_to(m.zbar, (m.nod2D, m.nl)).copy()
    zbar3[:, 1:] *= 1.0 + 0.01 * np.sin(np.arange(m.nod2D))[:, None]
    Z3d = np.concatenate([0.5 * (zbar3[:, :-1] + zbar3[:, 1:]),
                          0.5 * (zbar3[:, -2:-1] + zbar3[:, -1:])], axis=1)
    Zp = np.concatenate([m.Z, m.Z[-1:]])
    sw = np.where(im, 2e-5 * np.exp(Zp[None, :] / 20.0) * rng.uniform(0.8, 1.2, im.shape), 0.0)
    base = dict(Kv=Kv, hnode_new=f.hnode_new)
    out = {
        "T": dict(T=f.tracers[0], kw={}),
        "S_bc": dict(T=f.tracers[1], kw=dict(bc_surf=rng.normal(0.0, 0.01, m.nod2D))),
        "T_sw": dict(T=f.tracers[0], kw=dict(sw_3d=sw)),
        "T_zstar": dict(T=f.tracers[0], kw=dict(Z3d=Z3d)),
        "const": dict(T=np.where(lm, 20.0, 0.0), kw={}),
        "grad": dict(T=np.where(lm, 10.0 + 0.5 * k, 0.0), kw={}),
    }
    for c in out.values():
        c.update(base)
    return out


ICE_GOLDEN = Path(__file__).resolve().parent / "golden" / "fct_ice_golden.npz"


def ice_cases(m, seed=0):
    """Sea-ice FCT inputs on ``m``: name -> dict(a, m, ms, u, v, dt). A concentration
    blob with a sharp edge (limiter active), ice/snow thickness, nodal ice velocity."""
    rng = np.random.default_rng(seed)
    N = m.nod2D
    lon, lat = m.coord_nod2D[:, 0], m.coord_nod2D[:, 1]
    d = np.hypot(lon - np.median(lon), lat - np.median(lat))
    r = np.argsort(np.argsort(d)) / N          # distance rank in [0, 1)
    a = np.clip(2.0 - 3.3 * r + 0.05 * rng.normal(size=N), 0.0, 1.0)
    a = np.where(r < 0.3, 1.0, a)    # a flat top, a ramp, open water beyond r = 0.6
    hi = a * (1.0 + 2.0 * rng.uniform(size=N))
    hs = a * 0.3 * rng.uniform(size=N)
    u, v = rng.normal(0.0, 0.1, N), rng.normal(0.0, 0.1, N)
    return {
        "step_500": dict(a=a, m=hi, ms=hs, u=u, v=v, dt=500.0),
        "fast_3600": dict(a=a, m=hi, ms=hs, u=5.0 * u, v=5.0 * v, dt=3600.0),
    }


CAVITY_GOLDEN = Path(__file__).resolve().parent / "golden" / "fct_cavity_golden.npz"
CAVITY_ARRAYS = ("ulevels", "ulevels_nod2D", "ulevels_nod2D_max", "area", "areasvol")


def cavity_arrays(m):
    """An ice-shelf cavity on ``m`` (a cavity-free mesh): the cells whose three nodes lie in
    the northernmost ~15% of deep nodes start at level 3 (two dry layers on top); node
    ``ulevels_nod2D`` is the min and ``ulevels_nod2D_max`` the max over a node's cells;
    ``area``/``areasvol`` are zero above a node's first wet layer. Returns the five arrays."""
    lat = m.coord_nod2D[:, 1]
    deep = m.nlevels_nod2D >= 12
    cav = deep & (lat >= np.quantile(lat[deep], 0.85))
    en = m.elem_nodes
    ul = np.where(cav[en].all(axis=1), 3, 1).astype(np.int32)
    uln = np.full(m.nod2D, 10 ** 6, np.int64)
    ulx = np.zeros(m.nod2D, np.int64)
    for v in range(3):
        np.minimum.at(uln, en[:, v], ul)
        np.maximum.at(ulx, en[:, v], ul)
    uln = uln.astype(np.int32)
    ulx = ulx.astype(np.int32)
    k = np.arange(m.nl)[None, :]
    dry_top = k < (uln - 1)[:, None]
    area = np.where(dry_top, 0.0, m.area)
    areasvol = np.where(dry_top, 0.0, m.areasvol)
    return dict(ulevels=ul, ulevels_nod2D=uln, ulevels_nod2D_max=ulx, area=area,
                areasvol=areasvol)


def cavity_mesh(m):
    """``m`` with the cavity of :func:`cavity_arrays` (a new Mesh; masks re-derived)."""
    from fesom_jax_b200.mesh import FCT_FIELDS, Mesh
    fields = {f: getattr(m, f) for f in FCT_FIELDS}
    fields.update(cavity_arrays(m))
    return Mesh(**fields, name=m.name + "_cavity")
