"""Seeded synthetic FESOM2-style meshes (host numpy).

Builds the "raw" mesh (geographic nodes, triangles, edges with their adjacent
triangles, level counts, ``zbar``) of a Fibonacci-jittered spherical Delaunay
triangulation, then derives every geometric array the FCT reads with the FESOM2 mesh
metrics as restated from the reference's standalone preparation script
(scripts/prepare_mesh.py:117-300):

  * rotation to the model frame with Euler angles (50, 15, -90) deg and FESOM's
    truncated pi (prepare_mesh.py:27-104);
  * clockwise orientation of every triangle before any geometry (:125-132);
  * element-ascending node->element CSR (:134-140); node areas accumulated in that
    order (:159-169); element centres with the min-anchored cyclic convention
    (:171-181); ``gradient_sca`` (:183-188); edge geometry (:190-207);
  * the MFCT up/down triangle scan (:251-300), vectorised here.

Land: polar caps around the model-frame poles (where lon/lat geometry degenerates) and a
few seeded circular "continents" are removed, so the mesh has coastlines (boundary edges
with ``edge_tri[:,1] = -1`` and ``edge_up_dn_tri = -1``). Nodes are ordered by reverse
Cuthill-McKee for locality, elements by their lowest node, and edges interior-first
(the FESOM convention, ``edge2D_in``) with ``edge_tri[:,0]`` left of ``n1 -> n2``.
"""

from __future__ import annotations

import numpy as np

from .mesh import Mesh

PI = 3.14159265358979          # FESOM truncated pi (fesom_jax/config.py:34)
RAD = PI / 180.0
R_EARTH = 6367500.0
CYC = 2.0 * PI
HALF_CYC = 0.5 * CYC
EULER = (50.0, 15.0, -90.0)     # fesom_jax/config.py:50-52


def _trim(dx):
    dx = np.where(dx > HALF_CYC, dx - CYC, dx)
    return np.where(dx < -HALF_CYC, dx + CYC, dx)


def rotation_matrix():
    al, be, ga = (a * RAD for a in EULER)
    ca, sa, cb, sb, cg, sg = np.cos(al), np.sin(al), np.cos(be), np.sin(be), np.cos(ga), np.sin(ga)
    return np.array([cg * ca - sg * cb * sa, cg * sa + sg * cb * ca, sg * sb,
                     -sg * ca - cg * cb * sa, -sg * sa + cg * cb * ca, cg * sb,
                     sb * sa, -sb * ca, cb])


def geo_to_rot(glon, glat):
    M = rotation_matrix()
    xg, yg, zg = np.cos(glat) * np.cos(glon), np.cos(glat) * np.sin(glon), np.sin(glat)
    xr = M[0] * xg + M[1] * yg + M[2] * zg
    yr = M[3] * xg + M[4] * yg + M[5] * zg
    zr = M[6] * xg + M[7] * yg + M[8] * zg
    rlat = np.arcsin(np.clip(zr, -1.0, 1.0))
    rlon = np.where((yr == 0.0) & (xr == 0.0), 0.0, np.arctan2(yr, xr))
    return rlon, rlat


def stretched_zbar(nl: int, depth: float = 6000.0, top: float = 5.0) -> np.ndarray:
    """``nl`` interface depths (<= 0) with layer thickness growing geometrically from
    ``top`` metres to reach ``depth`` at the bottom interface."""
    n = nl - 1
    lo, hi = 1.0 + 1e-9, 2.0
    for _ in range(200):
        r = 0.5 * (lo + hi)
        tot = top * (r ** n - 1.0) / (r - 1.0)
        lo, hi = (r, hi) if tot < depth else (lo, r)
    dz = top * r ** np.arange(n)
    dz *= depth / dz.sum()
    return -np.concatenate([[0.0], np.cumsum(dz)])


def _smooth_field(xyz: np.ndarray, rng: np.random.Generator, n_waves: int = 24,
                  kmax: float = 6.0) -> np.ndarray:
    """A smooth seeded scalar field on the unit sphere, scaled to [0, 1]."""
    f = np.zeros(xyz.shape[0])
    for _ in range(n_waves):
        k = rng.normal(size=3)
        k *= rng.uniform(1.0, kmax) / np.linalg.norm(k)
        f += rng.normal() * np.cos(xyz @ k + rng.uniform(0, 2 * np.pi))
    f -= f.min()
    return f / max(f.max(), 1e-300)


def generate_raw(n_nodes: int, zbar: np.ndarray, seed: int = 0, bottom=(5, None),
                 cap_deg: float = 80.0, n_land: int = 3, land_radius_deg=(8.0, 20.0),
                 jitter: float = 0.25, node_order: str = "rcm") -> dict:
    """Raw mesh: geographic nodes (degrees), CW-agnostic triangles, and level counts.

    ``bottom=(lo, hi)`` bounds the per-node bottom level count (``hi`` defaults to
    ``len(zbar)``); it is drawn from a seeded smooth field. ``node_order``: ``"rcm"``
    (reverse Cuthill-McKee, the default: neighbours are close in index), ``"raw"`` (the
    Fibonacci point order: consecutive nodes are a golden angle apart) or ``"random"``
    (a seeded shuffle); elements follow as ascending smallest vertex. Returns the dict
    consumed by :func:`derive` (the same keys the reference preparation script reads).
    """
    if node_order not in ("rcm", "raw", "random"):
        raise ValueError(f"node_order={node_order!r}: expected rcm, raw or random")
    from scipy.spatial import ConvexHull
    from scipy.sparse import coo_matrix
    from scipy.sparse.csgraph import reverse_cuthill_mckee

    rng = np.random.default_rng(seed)
    nl = len(zbar)
    blo, bhi = bottom[0], (bottom[1] if bottom[1] is not None else nl)
    lands = []
    for _ in range(n_land):
        c = rng.normal(size=3)
        lands.append((c / np.linalg.norm(c), rng.uniform(*land_radius_deg) * RAD))
    jit_seed = int(rng.integers(0, 2**31 - 1))

    def sphere(M):
        i = np.arange(M) + 0.5
        z = 1.0 - 2.0 * i / M
        lon = (PI * (3.0 - np.sqrt(5.0)) * i) % (2 * PI)
        r = np.sqrt(1.0 - z * z)
        xyz = np.stack([r * np.cos(lon), r * np.sin(lon), z], axis=1)
        xyz += np.random.default_rng(jit_seed).normal(
            scale=jitter * np.sqrt(4.0 * PI / M) / 2.0, size=xyz.shape)
        xyz /= np.linalg.norm(xyz, axis=1, keepdims=True)
        glat = np.arcsin(np.clip(xyz[:, 2], -1, 1))
        glon = np.arctan2(xyz[:, 1], xyz[:, 0])
        rlon, rlat = geo_to_rot(glon, glat)
        ocean = np.abs(rlat) < cap_deg * RAD
        for c, rad in lands:
            ocean &= (xyz @ c) < np.cos(rad)
        return xyz, glon, glat, ocean

    # size the Fibonacci set so that about n_nodes ocean nodes remain
    M = int(n_nodes / max(np.sin(cap_deg * RAD), 0.2)) + 16
    for _ in range(4):
        xyz, glon, glat, ocean = sphere(M)
        kept = int(ocean.sum())
        if abs(kept - n_nodes) <= max(2, n_nodes // 1000):
            break
        M = max(16, int(round(M * n_nodes / max(kept, 1))))
    tri = ConvexHull(xyz).simplices
    tri = tri[np.all(ocean[tri], axis=1)]
    used = np.unique(tri)
    # keep the largest connected ocean: drop nodes only reached through a single vertex
    remap = -np.ones(M, np.int64)
    remap[used] = np.arange(used.size)
    tri = remap[tri]
    xyz, glon, glat = xyz[used], glon[used], glat[used]
    N = used.size
    # node order: reverse Cuthill-McKee for locality (default)
    if node_order == "rcm":
        a, b = np.concatenate([tri[:, 0], tri[:, 1], tri[:, 2]]), np.concatenate(
            [tri[:, 1], tri[:, 2], tri[:, 0]])
        adj = coo_matrix((np.ones(a.size), (a, b)), shape=(N, N)).tocsr()
        adj = adj + adj.T
        perm = np.asarray(reverse_cuthill_mckee(adj, symmetric_mode=True))
    elif node_order == "random":
        perm = np.random.default_rng(seed + 7919).permutation(N)
    else:
        perm = np.arange(N)
    inv = np.empty(N, np.int64)
    inv[perm] = np.arange(N)
    tri = inv[tri]
    xyz, glon, glat = xyz[perm], glon[perm], glat[perm]
    tri = tri[np.argsort(tri.min(axis=1), kind="stable")]
    # bathymetry: per-node bottom level count from a smooth seeded field
    f = _smooth_field(xyz, rng)
    node_bot = (blo + np.floor(f * (bhi - blo + 1 - 1e-9))).astype(np.int32)
    nlev_elem = node_bot[tri].min(axis=1).astype(np.int32)
    nlev_node = np.zeros(N, np.int32)
    np.maximum.at(nlev_node, tri.ravel(), np.repeat(nlev_elem, 3))
    nodes_deg = np.stack([glon / RAD, glat / RAD], axis=1)
    edges, edge_tri = _edges_from_triangles(tri, nodes_deg[:, 0] * RAD, nodes_deg[:, 1] * RAD)
    return dict(nodes_deg=nodes_deg, elem_nodes=tri.astype(np.int32),
                nl=nl, zbar=np.asarray(zbar, np.float64), depth=-np.asarray(zbar)[nlev_node - 1],
                nlevels_nod2D=nlev_node, nlevels=nlev_elem, edges=edges, edge_tri=edge_tri,
                nod2D=N, elem2D=tri.shape[0], coast=np.zeros(N, np.int32))


def _edges_from_triangles(tri: np.ndarray, glon, glat):
    """Unique edges with ``edge_tri``: element 1 left of ``n1 -> n2``, element 2 right
    (-1 on coasts); interior edges first, each group sorted by ``(n1, n2)``."""
    rlon, rlat = geo_to_rot(glon, glat)
    en = _orient_cw(tri, rlon, rlat)
    E = en.shape[0]
    # half-edges (a, b) of a CW triangle have the triangle on their right
    ha = np.concatenate([en[:, 0], en[:, 1], en[:, 2]])
    hb = np.concatenate([en[:, 1], en[:, 2], en[:, 0]])
    ht = np.tile(np.arange(E), 3)
    key_lo, key_hi = np.minimum(ha, hb), np.maximum(ha, hb)
    order = np.lexsort((key_hi, key_lo))
    ka, kb, ha, hb, ht = key_lo[order], key_hi[order], ha[order], hb[order], ht[order]
    first = np.ones(ka.size, bool)
    first[1:] = (ka[1:] != ka[:-1]) | (kb[1:] != kb[:-1])
    starts = np.flatnonzero(first)
    counts = np.diff(np.append(starts, ka.size))
    if np.any(counts > 2):
        raise ValueError("non-manifold triangulation")
    n1 = np.empty(starts.size, np.int64)
    n2 = np.empty(starts.size, np.int64)
    t1 = np.empty(starts.size, np.int64)
    t2 = -np.ones(starts.size, np.int64)
    inter = counts == 2
    s = starts
    # interior: n1 < n2; the half-edge (n1 -> n2) belongs to the right triangle (el2)
    for sel, idx in ((inter, s[inter]),):
        a0, b0, t0 = ha[idx], hb[idx], ht[idx]
        t_other = ht[idx + 1]
        lo_, hi_ = np.minimum(a0, b0), np.maximum(a0, b0)
        right_is_t0 = a0 == lo_          # half-edge lo->hi is in t0 -> t0 right of lo->hi
        n1[sel], n2[sel] = lo_, hi_
        t2[sel] = np.where(right_is_t0, t0, t_other)
        t1[sel] = np.where(right_is_t0, t_other, t0)
    bnd = ~inter
    idx = s[bnd]
    # coast: orient so the only triangle is on the left: n1 = b, n2 = a of its half-edge
    n1[bnd], n2[bnd], t1[bnd] = hb[idx], ha[idx], ht[idx]
    grp = np.where(inter, 0, 1)
    order = np.lexsort((n2, n1, grp))
    edges = np.stack([n1[order], n2[order]], axis=1).astype(np.int32)
    edge_tri = np.stack([t1[order], t2[order]], axis=1).astype(np.int32)
    return edges, edge_tri


def _orient_cw(en, rlon, rlat):
    en = np.array(en, copy=True)
    ax, ay = rlon[en[:, 0]], rlat[en[:, 0]]
    bx = _trim(rlon[en[:, 1]] - ax)
    by = rlat[en[:, 1]] - ay
    cx = _trim(rlon[en[:, 2]] - ax)
    cy = rlat[en[:, 2]] - ay
    ccw = (bx * cy - by * cx) > 0.0
    en[ccw, 1], en[ccw, 2] = en[ccw, 2].copy(), en[ccw, 1].copy()
    return en


def derive(raw: dict) -> dict:
    """Derived FCT geometry from a raw mesh (restates scripts/prepare_mesh.py:117-243)."""
    N, E, nl = raw["nod2D"], raw["elem2D"], raw["nl"]
    glon, glat = raw["nodes_deg"][:, 0] * RAD, raw["nodes_deg"][:, 1] * RAD
    rlon, rlat = geo_to_rot(glon, glat)
    en = _orient_cw(raw["elem_nodes"], rlon, rlat)
    n0, n1, n2 = en[:, 0], en[:, 1], en[:, 2]
    pair_node = en.reshape(-1)
    pair_elem = np.repeat(np.arange(E, dtype=np.int32), 3)
    order = np.argsort(pair_node, kind="stable")
    nie = pair_elem[order].astype(np.int32)
    counts = np.bincount(pair_node, minlength=N)
    offsets = np.zeros(N + 1, np.int32)
    offsets[1:] = np.cumsum(counts)
    nlevels = np.asarray(raw["nlevels"], np.int32)
    nlevels_nod2D = np.asarray(raw["nlevels_nod2D"], np.int32)
    nmin = np.full(N, np.iinfo(np.int32).max, np.int32)
    np.minimum.at(nmin, pair_node, nlevels[pair_elem])
    nlevels_nod2D_min = np.minimum(nmin, nlevels_nod2D)
    lat0, lat1, lat2 = rlat[n0], rlat[n1], rlat[n2]
    lon0, lon1, lon2 = rlon[n0], rlon[n1], rlon[n2]
    ay = np.cos((lat0 + lat1 + lat2) / 3.0)
    aX = _trim(lon1 - lon0) * ay
    aly = lat1 - lat0
    bX = _trim(lon2 - lon0) * ay
    bly = lat2 - lat0
    elem_area = 0.5 * np.abs(aX * bly - bX * aly) * (R_EARTH ** 2)
    # node areas per level, element-ascending accumulation (bincount keeps input order)
    third = elem_area / 3.0
    area = np.zeros((N, nl))
    for k in range(nl):
        sel = (nlevels - 1) > k
        if not np.any(sel):
            break
        area[:, k] = np.bincount(en[sel].reshape(-1), weights=np.repeat(third[sel], 3),
                                 minlength=N)
    kk = np.arange(nl)[None, :]
    areasvol = np.where(kk < (nlevels_nod2D - 1)[:, None], area, 0.0)
    axk = np.stack([lon0, lon1, lon2], axis=1)
    amin = axk.min(axis=1, keepdims=True)
    axk = np.where(axk - amin >= HALF_CYC, axk - CYC, axk)
    ecx = axk.sum(axis=1) / 3.0
    ecy = (lat0 + lat1 + lat2) / 3.0
    elem_cos = np.cos(ecy)
    dX31 = _trim(lon2 - lon0) * elem_cos
    dX21 = _trim(lon1 - lon0) * elem_cos
    dY31 = lat2 - lat0
    dY21 = lat1 - lat0
    df = -0.5 * R_EARTH / elem_area
    gradient_sca = np.stack([(-dY31 + dY21) * df, dY31 * df, (-dY21) * df,
                             (dX31 - dX21) * df, (-dX31) * df, dX21 * df], axis=1)
    edges = np.asarray(raw["edges"], np.int32)
    e0, e1 = edges[:, 0], edges[:, 1]
    edge_dxdy = np.stack([_trim(rlon[e1] - rlon[e0]), rlat[e1] - rlat[e0]], axis=1)
    eax, ebx = rlon[e0].copy(), rlon[e1].copy()
    d = rlon[e0] - rlon[e1]
    eax = np.where(d > HALF_CYC, eax - CYC, eax)
    ebx = np.where(d < -HALF_CYC, ebx - CYC, ebx)
    emx = 0.5 * (eax + ebx)
    emy = 0.5 * (rlat[e0] + rlat[e1])
    et = np.asarray(raw["edge_tri"], np.int32)
    el1, el2 = et[:, 0], et[:, 1]
    cross = np.zeros((edges.shape[0], 4))
    cross[:, 0] = _trim(ecx[el1] - emx) * elem_cos[el1] * R_EARTH
    cross[:, 1] = (ecy[el1] - emy) * R_EARTH
    has2 = el2 >= 0
    el2s = np.where(has2, el2, 0)
    cross[:, 2] = np.where(has2, _trim(ecx[el2s] - emx) * elem_cos[el2s] * R_EARTH, 0.0)
    cross[:, 3] = np.where(has2, (ecy[el2s] - emy) * R_EARTH, 0.0)
    zbar = np.asarray(raw["zbar"], np.float64)
    up_dn = edge_up_dn_tri(edges, en, rlon, rlat, nie, offsets)
    return dict(coord_nod2D=np.stack([rlon, rlat], axis=1), nlevels_nod2D=nlevels_nod2D,
                nlevels_nod2D_min=nlevels_nod2D_min, ulevels_nod2D=np.ones(N, np.int32),
                ulevels_nod2D_max=np.ones(N, np.int32), area=area, areasvol=areasvol,
                nod_in_elem2D_offsets=offsets, nod_in_elem2D=nie, elem_nodes=en.astype(np.int32),
                nlevels=nlevels, ulevels=np.ones(E, np.int32), elem_area=elem_area,
                elem_cos=elem_cos, gradient_sca=gradient_sca, edges=edges, edge_tri=et,
                edge_dxdy=edge_dxdy, edge_cross_dxdy=cross, edge_up_dn_tri=up_dn,
                zbar=zbar, Z=0.5 * (zbar[:-1] + zbar[1:]))


def _between(bx, by, cx, cy, xx, xy):
    """Is direction x inside the angle from c to b (scripts/prepare_mesh.py:251-265)?"""
    cr = cx * cx + cy * cy
    ok = cr != 0.0
    crs = np.where(ok, cr, 1.0)
    bxp = (bx * cx + by * cy) / crs
    byp = (-bx * cy + by * cx) / crs
    xxp = (xx * cx + xy * cy) / crs
    xyp = (-xx * cy + xy * cx) / crs
    ab = np.arctan2(byp, bxp)
    axg = np.arctan2(xyp, xxp)
    hit = ((ab > 0.0) & (axg > 0.0) & (axg < ab)) | ((ab < 0.0) & (axg < 0.0) & (axg > ab)) | \
          (ab == axg) | (axg == 0.0)
    return ok & hit


def edge_up_dn_tri(edges, en, rlon, rlat, nie, offsets, chunk: int = 1 << 20):
    """MFCT up/down triangles: for endpoint ``n1`` the first element (CSR order) of
    ``n1`` whose corner at ``n1`` contains the direction away from ``n2``, likewise for
    ``n2``; -1 when none (restates scripts/prepare_mesh.py:268-300)."""
    Ed = edges.shape[0]
    out = np.full((Ed, 2), -1, np.int32)
    x0 = _trim(rlon[edges[:, 1]] - rlon[edges[:, 0]])
    x1 = rlat[edges[:, 1]] - rlat[edges[:, 0]]
    for side in (0, 1):
        node = edges[:, side]
        sgn = -1.0 if side == 0 else 1.0
        cnt = offsets[node + 1] - offsets[node]
        maxc = int(cnt.max())
        for j in range(maxc):
            todo = np.flatnonzero((out[:, side] < 0) & (cnt > j))
            for s0 in range(0, todo.size, chunk):
                ids = todo[s0:s0 + chunk]
                nd = node[ids]
                el = nie[offsets[nd] + j]
                tri = en[el]
                js = np.where(tri[:, 0] == nd, 0, np.where(tri[:, 1] == nd, 1, 2))
                jb = np.where(js == 0, 1, 0)
                jc = np.where(js == 2, 1, 2)
                nb = tri[np.arange(ids.size), jb]
                nc = tri[np.arange(ids.size), jc]
                bx = _trim(rlon[nb] - rlon[nd])
                by = rlat[nb] - rlat[nd]
                cx = _trim(rlon[nc] - rlon[nd])
                cy = rlat[nc] - rlat[nd]
                hit = _between(bx, by, cx, cy, sgn * x0[ids], sgn * x1[ids])
                out[ids[hit], side] = el[hit]
    return out


def make_mesh(n_nodes: int, nl: int = 48, zbar=None, seed: int = 0, bottom=(5, None),
              name: str | None = None, **kw) -> Mesh:
    """A synthetic mesh with about ``n_nodes`` ocean nodes (see :func:`generate_raw`)."""
    if zbar is None:
        from .mesh import pi_mesh
        zbar = pi_mesh().zbar if nl == 48 else stretched_zbar(nl)
    raw = generate_raw(n_nodes, np.asarray(zbar), seed=seed, bottom=bottom, **kw)
    m = Mesh(**derive(raw), name=name or f"synthetic_{raw['nod2D']}")
    m.validate()
    return m
