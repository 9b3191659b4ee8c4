"""Seeded synthetic inputs for the FCT path (host numpy, float64).

The reference drives ``advect_one_fct`` from a full model step; here the inputs are
generated directly with the shapes, layouts and value ranges the workloads name:

  * rest layer thicknesses from ``zbar`` (fesom_jax/state.py:165-187):
    ``hnode[n,k] = zbar[k]-zbar[k+1]`` on wet layers, ``helem`` likewise, 0 elsewhere;
  * ``T`` 2-28 degC decreasing with the layer mid-depth ``Z`` plus N(0, 0.5) noise,
    ``S`` 34-36 psu increasing with depth plus N(0, 0.1), both 0 below the bottom;
  * element velocities with standard deviation ``sigma`` (default 0.1 m/s) from a smooth
    seeded streamfunction, with a linear decay with depth, masked to each element's
    layers (:func:`velocities`);
  * ``w`` from discrete continuity, :func:`compute_w` (fesom_jax/ale.py:309-365).
"""

from __future__ import annotations

import dataclasses

import numpy as np

from .mesh import Mesh, R_EARTH


def rest_thickness(mesh: Mesh):
    """``(hnode [N,nl], helem [E,nl])`` rest thicknesses (fesom_jax/state.py:165-187)."""
    nl = mesh.nl
    dz = np.zeros(nl)
    dz[:-1] = mesh.zbar[:-1] - mesh.zbar[1:]
    hnode = np.where(mesh.node_layer_mask, dz[None, :], 0.0)
    helem = np.where(mesh.elem_layer_mask, dz[None, :], 0.0)
    return hnode, helem


def layer_depth_fraction(mesh: Mesh) -> np.ndarray:
    """``|Z_k| / max|Z|`` per layer ``k`` (``[nl]``; the last slot repeats ``Z[-1]``)."""
    Zp = np.concatenate([mesh.Z, mesh.Z[-1:]])
    return np.abs(Zp) / np.max(np.abs(Zp))


def compute_w(mesh: Mesh, uv: np.ndarray, helem: np.ndarray) -> np.ndarray:
    """Vertical velocity at interfaces ``[N, nl]`` from continuity.

    Restates fesom_jax/ale.py:309-365: per-level antisymmetric edge->node divergence
    scatter of ``(v*dx - u*dy)*h`` (minus the second cell's), a bottom-to-top suffix
    sum over levels, division by ``area`` (safe where 0) and the interface mask.
    """
    et = mesh.edge_tri
    el1, el2 = et[:, 0], et[:, 1]
    has1, has2 = el1 >= 0, el2 >= 0
    e1 = np.where(has1, el1, 0)
    e2 = np.where(has2, el2, 0)
    cr = mesh.edge_cross_dxdy
    U, V = uv[:, :, 0], uv[:, :, 1]
    lm = mesh.elem_layer_mask
    t1 = np.where(lm[e1] & has1[:, None],
                  (V[e1] * cr[:, 0:1] - U[e1] * cr[:, 1:2]) * helem[e1], 0.0)
    t2 = np.where(lm[e2] & has2[:, None],
                  (V[e2] * cr[:, 2:3] - U[e2] * cr[:, 3:4]) * helem[e2], 0.0)
    c = t1 - t2
    div = np.zeros((mesh.nod2D, mesh.nl))
    np.add.at(div, mesh.edges[:, 0], c)
    np.add.at(div, mesh.edges[:, 1], -c)
    w = np.flip(np.cumsum(np.flip(div, axis=1), axis=1), axis=1)
    w = w / np.where(mesh.area > 0.0, mesh.area, 1.0)
    return np.where(mesh.node_iface_mask, w, 0.0)


def tracer_profiles(mesh: Mesh, rng: np.random.Generator):
    """``(T, S)`` ``[N, nl]``: depth profiles plus seeded noise, 0 below the bottom."""
    frac = layer_depth_fraction(mesh)[None, :]
    shape = (mesh.nod2D, mesh.nl)
    T = 28.0 - 26.0 * frac + rng.normal(0.0, 0.5, shape)
    S = 34.0 + 2.0 * frac + rng.normal(0.0, 0.1, shape)
    m = mesh.node_layer_mask
    return np.where(m, T, 0.0), np.where(m, S, 0.0)


def passive_tracer(mesh: Mesh, rng: np.random.Generator) -> np.ndarray:
    """A passive tracer ``U[0, 1]`` on wet layers, 0 below the bottom."""
    return np.where(mesh.node_layer_mask, rng.uniform(0.0, 1.0, (mesh.nod2D, mesh.nl)), 0.0)


def node_xyz(mesh: Mesh) -> np.ndarray:
    lon, lat = mesh.coord_nod2D[:, 0], mesh.coord_nod2D[:, 1]
    return np.stack([np.cos(lat) * np.cos(lon), np.cos(lat) * np.sin(lon), np.sin(lat)], 1)


def streamfunction_velocity(mesh: Mesh, psi: np.ndarray) -> np.ndarray:
    """Element velocity ``(u, v) = (-dpsi/dy, dpsi/dx)`` ``[E, 2]`` of a nodal P1
    streamfunction, using the mesh's own ``gradient_sca``. The edge face fluxes of such a
    field telescope around every interior node's dual cell, so its discrete divergence
    (and hence ``w``) comes only from coasts and bathymetry steps."""
    t = psi[mesh.elem_nodes]
    gs = mesh.gradient_sca
    gx = (gs[:, 0:3] * t).sum(1)
    gy = (gs[:, 3:6] * t).sum(1)
    return np.stack([-gy, gx], axis=1)


def velocities(mesh: Mesh, rng: np.random.Generator, sigma: float = 0.1, kind: str = "psi",
               n_vortices: int = 0, vortex_radius_km=(50.0, 200.0),
               vortex_speed: float = 0.5) -> np.ndarray:
    """Element velocities ``uv [E, nl, 2]`` (m/s): :func:`velocity_base` expanded over the
    levels with the linear decay and masked to each element's layers."""
    base = velocity_base(mesh, rng, sigma, kind, n_vortices, vortex_radius_km, vortex_speed)
    decay = 1.0 - 0.9 * layer_depth_fraction(mesh)
    uv = base[:, None, :] * decay[None, :, None]
    return np.where(mesh.elem_layer_mask[:, :, None], uv, 0.0)


def velocity_base(mesh: Mesh, rng: np.random.Generator, sigma: float = 0.1, kind: str = "psi",
                  n_vortices: int = 0, vortex_radius_km=(50.0, 200.0),
                  vortex_speed: float = 0.5) -> np.ndarray:
    """Depth-independent element velocity ``[E, 2]`` (m/s) with standard deviation ``sigma``.

    ``kind="psi"``: a smooth seeded random streamfunction (sum of random plane waves on the
    sphere) turned into velocities by :func:`streamfunction_velocity` and scaled to
    ``sigma``; ``kind="white"``: independent ``N(0, sigma)`` per element (strongly
    divergent, large vertical CFL). Both are multiplied by the linear decay
    ``1 - 0.9*|Z_k|/max|Z|`` and masked to each element's layers.
    ``n_vortices > 0`` adds seeded Gaussian streamfunction eddies (radius ``R`` drawn from
    ``vortex_radius_km``, peak azimuthal speed ``vortex_speed`` at ``r = R``).
    """
    E = mesh.elem2D
    if kind == "white":
        base = rng.normal(0.0, sigma, (E, 2))
    elif kind == "psi":
        xyz = node_xyz(mesh)
        psi = np.zeros(mesh.nod2D)
        for _ in range(24):
            k = rng.normal(size=3)
            k *= rng.uniform(2.0, 12.0) / np.linalg.norm(k)
            psi += rng.normal() * np.cos(xyz @ k + rng.uniform(0.0, 2.0 * np.pi))
        base = streamfunction_velocity(mesh, psi)
        base *= sigma / max(base.std(), 1e-300)
    else:
        raise ValueError(f"unknown velocity kind {kind!r}")
    if n_vortices:
        xyz = node_xyz(mesh)
        psi = np.zeros(mesh.nod2D)
        centres = xyz[rng.integers(0, mesh.nod2D, n_vortices)]
        radii = rng.uniform(*vortex_radius_km, n_vortices) * 1e3
        signs = rng.choice([-1.0, 1.0], n_vortices)
        for c, R, s in zip(centres, radii, signs):
            r = R_EARTH * np.arccos(np.clip(xyz @ c, -1.0, 1.0))
            near = r < 5.0 * R
            psi[near] += s * vortex_speed * R * np.exp(0.5) * np.exp(-0.5 * (r[near] / R) ** 2)
        base = base + streamfunction_velocity(mesh, psi)
    return base


def wall_rings(mesh: Mesh, rings: int = 3):
    """Per-node level bounds of the walls within ``r`` edge hops, for ``r = 0..rings-1``.

    A node is at a wall on layer ``k`` when it lies on a coast (an edge with one cell) or
    one of its cells is dry at ``k``: ``k < ulevels_nod2D_max - 1`` or
    ``k >= nlevels_nod2D_min - 1`` (fesom_jax/mesh.py:135-151 level conventions). Returns
    ``[(nlmin_r, ulmax_r, coast_r)]``: the smallest ``nlevels_nod2D_min``, the largest
    ``ulevels_nod2D_max`` and whether a coast node occurs among the nodes within ``r`` hops.
    """
    e = np.asarray(mesh.edges)
    a, b = e[:, 0], e[:, 1]
    nlmin = np.asarray(mesh.nlevels_nod2D_min, np.int32).copy()
    ulmax = np.asarray(mesh.ulevels_nod2D_max, np.int32).copy()
    coast = np.zeros(mesh.nod2D, bool)
    ce = np.asarray(mesh.edge_tri)[:, 1] < 0
    coast[a[ce]] = True
    coast[b[ce]] = True
    out = []
    for r in range(rings):
        out.append((nlmin.copy(), ulmax.copy(), coast.copy()))
        if r + 1 == rings:
            break
        n2, u2, c2 = nlmin.copy(), ulmax.copy(), coast.copy()
        np.minimum.at(n2, a, nlmin[b])
        np.minimum.at(n2, b, nlmin[a])
        np.maximum.at(u2, a, ulmax[b])
        np.maximum.at(u2, b, ulmax[a])
        np.logical_or.at(c2, a, coast[b])
        np.logical_or.at(c2, b, coast[a])
        nlmin, ulmax, coast = n2, u2, c2
    return out


def basin_taper(rings, nl: int, xp=np):
    """``[N, nl]`` factor in ``[0, 1]``: ``r / R`` where ``r`` is the hop distance to the
    nearest wall on that layer (:func:`wall_rings`, ``R = len(rings)``), 1 beyond ``R - 1``
    hops. ``xp`` is numpy or torch (the ring arrays must be of that kind)."""
    R = len(rings)
    nlmin0 = rings[0][0]
    k = xp.arange(nl).reshape(1, -1)
    taper = xp.ones((nlmin0.shape[0], nl), dtype=xp.float64)
    if xp is not np:
        k, taper = k.to(nlmin0.device), taper.to(nlmin0.device)
    for r in range(R - 1, -1, -1):
        nlmin, ulmax, coast = rings[r]
        wall = (coast.reshape(-1, 1) | (k < ulmax.reshape(-1, 1) - 1)
                | (k >= nlmin.reshape(-1, 1) - 1))
        taper = xp.where(wall, r / R, taper)
    return taper


def basin_psi(mesh: Mesh, rng: np.random.Generator, sigma: float = 0.1,
              n_vortices: int = 0, vortex_radius_km=(50.0, 200.0),
              vortex_speed: float = 0.5) -> np.ndarray:
    """Nodal streamfunction ``[N]`` (m^2/s): the seeded plane waves of
    :func:`velocity_base` (``kind="psi"``), scaled so their velocity has standard deviation
    ``sigma``, plus ``n_vortices`` seeded Gaussian eddies."""
    xyz = node_xyz(mesh)
    psi = np.zeros(mesh.nod2D)
    for _ in range(24):
        k = rng.normal(size=3)
        k *= rng.uniform(2.0, 12.0) / np.linalg.norm(k)
        psi += rng.normal() * np.cos(xyz @ k + rng.uniform(0.0, 2.0 * np.pi))
    psi *= sigma / max(streamfunction_velocity(mesh, psi).std(), 1e-300)
    if n_vortices:
        centres = xyz[rng.integers(0, mesh.nod2D, n_vortices)]
        radii = rng.uniform(*vortex_radius_km, n_vortices) * 1e3
        signs = rng.choice([-1.0, 1.0], n_vortices)
        for c, R, s in zip(centres, radii, signs):
            r = R_EARTH * np.arccos(np.clip(xyz @ c, -1.0, 1.0))
            near = r < 5.0 * R
            psi[near] += s * vortex_speed * R * np.exp(0.5) * np.exp(-0.5 * (r[near] / R) ** 2)
    return psi


# standard deviation (m/s) of the divergent white-noise part of ``kind="basin"`` velocities
BASIN_SIGMA_DIV = 0.002
# width (m) over which the basin streamfunction tapers to 0 at walls
BASIN_TAPER_M = 200e3


def basin_rings(mesh: Mesh, width_m: float = BASIN_TAPER_M) -> int:
    """Hops that span ``width_m`` at the mesh's median node spacing (3 to 12)."""
    a = np.asarray(mesh.area)[:, 0]
    dx = float(np.sqrt(np.median(a[a > 0]))) if np.any(a > 0) else width_m
    return int(np.clip(round(width_m / dx), 3, 12))


def basin_velocities(mesh: Mesh, rng: np.random.Generator, sigma: float = 0.1,
                     n_vortices: int = 0, sigma_div: float = BASIN_SIGMA_DIV,
                     rings: int | None = None) -> np.ndarray:
    """Element velocities ``uv [E, nl, 2]`` of closed basins (``kind="basin"``).

    On every layer ``k`` the flow is the curl of ``psi_k = psi * decay_k * taper_k``
    (:func:`basin_psi`, the linear decay ``1 - 0.9*|Z_k|/max|Z|``, :func:`basin_taper`
    over :func:`basin_rings` hops, about 200 km):
    ``psi_k`` vanishes at every node that touches a coast or a dry cell on that layer, so
    the P1 face fluxes telescope around every node's (partial) dual cell and the flow is
    discretely divergence-free layer by layer, walls included. A seeded ``N(0,
    sigma_div)`` white-noise part (same decay, masked to each element's layers) adds the
    divergence that ``compute_w`` turns into a vertical velocity. With ``sigma_div`` 0.002
    m/s the low-order scheme's outflow CFL stays far below 1 on the benchmark meshes (the
    plain streamfunction of ``kind="psi"`` carries column divergence wherever the
    bathymetry steps, which reaches a vertical CFL of 10-50 in the 5 m surface layer).
    """
    psi, noise = basin_draw(mesh, rng, sigma, n_vortices, sigma_div)
    rg = wall_rings(mesh, rings or basin_rings(mesh))
    return basin_combine(mesh, psi, noise, rg, np)


def basin_draw(mesh: Mesh, rng: np.random.Generator, sigma: float, n_vortices: int,
               sigma_div: float):
    """The seeded pieces of a basin flow: ``psi [N]`` and the white part ``[E, 2]``."""
    psi = basin_psi(mesh, rng, sigma=sigma, n_vortices=n_vortices)
    return psi, rng.normal(0.0, sigma_div, (mesh.elem2D, 2))


def basin_combine(mesh: Mesh, psi, noise, rings, xp=np, device=None):
    """``uv [E, nl, 2]`` from the pieces of :func:`basin_draw` and :func:`wall_rings`;
    ``xp`` is numpy or torch (torch: the pieces are moved to ``device`` and the result
    stays there)."""
    if xp is np:
        cv = np.asarray
    else:
        def cv(a):
            return xp.as_tensor(np.asarray(a), device=device)
    decay = cv(1.0 - 0.9 * layer_depth_fraction(mesh))
    taper = basin_taper([tuple(cv(x) for x in r) for r in rings], mesh.nl, xp)
    psik = cv(psi)[:, None] * decay[None, :] * taper
    t = psik[cv(np.asarray(mesh.elem_nodes, np.int64))]          # [E, 3, nl]
    gs = cv(mesh.gradient_sca)
    gx = xp.einsum("ev,evk->ek", gs[:, 0:3], t)
    gy = xp.einsum("ev,evk->ek", gs[:, 3:6], t)
    del t
    uv = xp.stack([-gy, gx], 2) + cv(noise)[:, None, :] * decay[None, :, None]
    return xp.where(cv(mesh.elem_layer_mask)[:, :, None], uv, 0.0)


def lo_outflow_cfl(mesh: Mesh, uv: np.ndarray, w: np.ndarray, hnode: np.ndarray,
                   dt: float) -> float:
    """Largest outflow Courant number of the low-order upwind step
    (fesom_jax/tracer_adv.py:96-120, 298-313) over wet node layers: ``dt / (areasvol *
    hnode)`` times the volume leaving the layer through its edges (``vflux`` out of the
    node) and interfaces (``w * area`` up at ``k``, down at ``k + 1``). Below 1 the
    low-order solution is a convex combination of the old values (monotone); above 1 it
    is not, and repeated steps can grow without bound."""
    et = mesh.edge_tri
    el1, el2 = et[:, 0], et[:, 1]
    has2 = el2 >= 0
    e2 = np.where(has2, el2, 0)
    cr = mesh.edge_cross_dxdy
    lm = mesh.elem_layer_mask
    helem = np.where(lm, hnode_layer_thickness(mesh)[None, :], 0.0)
    U, V = uv[:, :, 0], uv[:, :, 1]
    t1 = np.where(lm[el1], (U[el1] * cr[:, 1:2] - V[el1] * cr[:, 0:1]) * helem[el1], 0.0)
    t2 = np.where(lm[e2] & has2[:, None],
                  (V[e2] * cr[:, 2:3] - U[e2] * cr[:, 3:4]) * helem[e2], 0.0)
    vf = t1 + t2
    out = np.zeros((mesh.nod2D, mesh.nl))
    np.add.at(out, mesh.edges[:, 0], np.maximum(vf, 0.0))
    np.add.at(out, mesh.edges[:, 1], np.maximum(-vf, 0.0))
    area = mesh.area
    lay = mesh.node_layer_mask
    z = np.zeros((mesh.nod2D, 1))
    up = np.maximum(w, 0.0) * area
    w1 = np.concatenate([w[:, 1:], z], 1)
    a1 = np.concatenate([area[:, 1:], z], 1)
    lay1 = np.concatenate([lay[:, 1:], z.astype(bool)], 1)
    dn = np.where(lay1, np.maximum(-w1, 0.0) * a1, 0.0)
    av = mesh.areasvol
    ok = lay & (av > 0) & (hnode > 0)
    c = np.where(ok, dt * (out + up + dn) / np.where(ok, av * hnode, 1.0), 0.0)
    return float(c.max())


def hnode_layer_thickness(mesh: Mesh) -> np.ndarray:
    """Rest layer thickness ``zbar[k] - zbar[k+1]`` per layer ``[nl]`` (0 in the last)."""
    dz = np.zeros(mesh.nl)
    dz[:-1] = mesh.zbar[:-1] - mesh.zbar[1:]
    return dz


@dataclasses.dataclass
class Fields:
    """One FCT instance's inputs (host numpy, reference layouts)."""

    uv: np.ndarray          # [E, nl, 2]
    w_e: np.ndarray         # [N, nl]
    helem: np.ndarray       # [E, nl]
    hnode: np.ndarray       # [N, nl]
    hnode_new: np.ndarray   # [N, nl]
    tracers: np.ndarray     # [ntr, N, nl]  (T, then S, then passives)
    tracers_old: np.ndarray  # [ntr, N, nl]


def make_fields(mesh: Mesh, seed: int = 0, n_passive: int = 0, sigma: float = 0.1,
                ab2: bool = False, n_vortices: int = 0, uv: np.ndarray | None = None,
                tracers: np.ndarray | None = None, kind: str = "psi") -> Fields:
    """Seeded inputs for one instance: T, S (+ passive tracers), velocities, ``w``.

    ``ab2=False`` gives ``T_old = T`` (step-1 convention, fesom_jax/ic.py:91-110);
    ``ab2=True`` perturbs ``T_old`` so the AB2 extrapolation is exercised.
    """
    rng = np.random.default_rng(seed)
    if tracers is None:
        T, S = tracer_profiles(mesh, rng)
        tr = [T, S] + [passive_tracer(mesh, rng) for _ in range(n_passive)]
        tracers = np.stack(tr)
    hnode, helem = rest_thickness(mesh)
    if uv is None and kind == "basin":
        uv = basin_velocities(mesh, rng, sigma=sigma, n_vortices=n_vortices)
    elif uv is None:
        uv = velocities(mesh, rng, sigma=sigma, kind=kind, n_vortices=n_vortices)
    w = compute_w(mesh, uv, helem)
    if ab2:
        pert = rng.normal(0.0, 0.05, tracers.shape) * mesh.node_layer_mask[None]
        old = tracers + pert
    else:
        old = tracers.copy()
    return Fields(uv=uv, w_e=w, helem=helem, hnode=hnode, hnode_new=hnode.copy(),
                  tracers=np.ascontiguousarray(tracers), tracers_old=np.ascontiguousarray(old))


def max_cfl_z(mesh: Mesh, w: np.ndarray, hnode_new: np.ndarray, dt: float) -> float:
    """Max vertical CFL ``|w|*dt*(1/h[k] + 1/h[k-1])`` over interfaces
    (fesom_jax/ale.py:368-395)."""
    lm = mesh.node_layer_mask
    inv = np.where(lm & (hnode_new > 0), 1.0 / np.where(hnode_new > 0, hnode_new, 1.0), 0.0)
    inv_above = np.concatenate([np.zeros((mesh.nod2D, 1)), inv[:, :-1]], axis=1)
    return float(np.max(np.abs(w) * dt * (inv + inv_above)))
