"""Workload builders: synthetic meshes and per-member device inputs for the benchmark
configurations (pi plain, CORE2-size batched ensemble, 1.3M-node single instance).

Member inputs are built on the GPU from small seeded host pieces: the nodal streamfunction
and white-noise part of :func:`inputs.basin_draw` (or the depth-independent velocity of
:func:`inputs.velocity_base`), expanded over levels with torch; ``w`` from the CUDA
``compute_w``; tracers drawn with a seeded torch generator on the device.
"""

from __future__ import annotations

import dataclasses

import numpy as np

from . import inputs as I
from .mesh import Mesh, pi_mesh

WORKLOADS = {
    # name: mesh + member layout of each benchmark workload; ``velocity`` is the
    # velocity kind of :func:`member_inputs_gpu`: one step on pi takes the white noise
    # u, v ~ N(0, 0.1) of its configuration; the multi-step workloads take closed-basin
    # flows (:func:`inputs.basin_velocities`), whose low-order CFL stays below 1
    "pi": dict(n_nodes=None, nl=48, members=1, ntr=2, fct_steps=1, dt=3600.0, sigma=0.1,
               n_vortices=0, bottom=None, velocity="white"),
    "batched": dict(n_nodes=127000, nl=48, members=32, ntr=8, fct_steps=30, dt=1800.0,
                    sigma=0.1, n_vortices=0, bottom=(5, 48), velocity="basin"),
    "large": dict(n_nodes=1300000, nl=70, members=1, ntr=10, fct_steps=20, dt=600.0,
                  sigma=0.2, n_vortices=400, bottom=(10, 70), velocity="basin"),
}


def velocity_note(name: str) -> str:
    """One line naming the velocity field of workload ``name``."""
    w = WORKLOADS[name]
    if w["velocity"] == "white":
        return (f"u, v ~ N(0, {w['sigma']} m/s) per element with linear decay; w from "
                "compute_w")
    return (f"closed basins: per-layer streamfunction (velocity std {w['sigma']} m/s"
            + (f", {w['n_vortices']} eddies" if w["n_vortices"] else "")
            + f") tapered to 0 within {I.BASIN_TAPER_M / 1e3:.0f} km of each layer's walls, "
            f"plus white N(0, {I.BASIN_SIGMA_DIV} m/s); linear decay; w from compute_w")


_RINGS = {}


def _wall_rings(mesh: Mesh):
    r = _RINGS.get(id(mesh))
    if r is None or r[0] is not mesh:
        r = _RINGS[id(mesh)] = (mesh, I.wall_rings(mesh, I.basin_rings(mesh)))
    return r[1]


def make_workload_mesh(name: str, seed: int = 0, node_order: str = "rcm") -> Mesh:
    """The configuration's mesh; synthetic meshes in ``node_order`` (see
    :func:`meshgen.generate_raw`; the pi mesh keeps its shipped order)."""
    from . import meshgen
    w = WORKLOADS[name]
    if w["n_nodes"] is None:
        return pi_mesh()
    suffix = "" if node_order == "rcm" else f"_{node_order}"
    return meshgen.make_mesh(w["n_nodes"], nl=w["nl"], seed=seed, bottom=w["bottom"],
                             name=f"{name}_{w['n_nodes']}{suffix}", node_order=node_order)


@dataclasses.dataclass
class Thickness:
    helem: object
    hnode: object
    hnode_new: object


def rest_thickness_gpu(mesh: Mesh, device) -> Thickness:
    import torch
    hn, he = I.rest_thickness(mesh)
    d = lambda x: torch.from_numpy(np.ascontiguousarray(x)).to(device)  # noqa: E731
    hnode = d(hn)
    return Thickness(helem=d(he), hnode=hnode, hnode_new=hnode)


def member_inputs_gpu(mesh: Mesh, seed: int, ntr: int, device, thickness: Thickness,
                      sigma: float = 0.1, n_vortices: int = 0, kind: str = "basin",
                      ab2: bool = True) -> dict:
    """``uv, w_e, helem, hnode, hnode_new, T [ntr,N,nl], T_old`` as CUDA tensors.

    ``kind``: ``"basin"`` (closed basins, :func:`inputs.basin_velocities`, the same
    numbers as the host generator for the same seed), or ``"psi"`` / ``"white"``
    (:func:`inputs.velocity_base`)."""
    import torch

    from .ale import compute_w
    rng = np.random.default_rng(seed)
    if kind == "basin":
        psi, noise = I.basin_draw(mesh, rng, sigma, n_vortices, I.BASIN_SIGMA_DIV)
        uv = I.basin_combine(mesh, psi, noise, _wall_rings(mesh), torch, device)
    else:
        base = I.velocity_base(mesh, rng, sigma=sigma, kind=kind, n_vortices=n_vortices)
        decay = 1.0 - 0.9 * I.layer_depth_fraction(mesh)
        emask = torch.from_numpy(mesh.elem_layer_mask).to(device)
        b = torch.from_numpy(base).to(device)
        dcy = torch.from_numpy(decay).to(device)
        uv = (b[:, None, :] * dcy[None, :, None]) * emask[:, :, None]
    uv = uv.contiguous()
    w = compute_w(mesh, uv, thickness.helem)
    g = torch.Generator(device=device)
    g.manual_seed(int(seed) * 7919 + 17)
    N, nl = mesh.nod2D, mesh.nl
    nmask = torch.from_numpy(mesh.node_layer_mask).to(device)
    frac = torch.from_numpy(I.layer_depth_fraction(mesh)).to(device)[None, :]
    T = torch.empty((ntr, N, nl), dtype=torch.float64, device=device)
    for t in range(ntr):
        if t == 0:
            T[t] = 28.0 - 26.0 * frac + 0.5 * torch.randn((N, nl), generator=g, device=device,
                                                          dtype=torch.float64)
        elif t == 1:
            T[t] = 34.0 + 2.0 * frac + 0.1 * torch.randn((N, nl), generator=g, device=device,
                                                         dtype=torch.float64)
        else:
            T[t] = torch.rand((N, nl), generator=g, device=device, dtype=torch.float64)
    T *= nmask
    if ab2:
        T_old = T + 0.05 * torch.randn(T.shape, generator=g, device=device,
                                       dtype=torch.float64) * nmask
    else:
        T_old = T.clone()
    return dict(uv=uv, w_e=w, helem=thickness.helem, hnode=thickness.hnode,
                hnode_new=thickness.hnode_new, T=T, T_old=T_old)


def algorithmic_bytes(mesh: Mesh, ntr: int, n_instances: int, n_thickness_sets: int = 1,
                      n_meshes: int = 1) -> int:
    """Minimum DRAM bytes of one FCT step over ``n_instances`` instances of ``mesh``:
    per instance ``ntr*24*N_wl`` (read T, T_old; write T_new) + ``16*E_wl`` (uv) +
    ``8*N_wi`` (w_e); per thickness set ``16*N_wl + 8*E_wl``; per mesh ``8*N_wi`` (area)
    + ``8*N_wl`` (areasvol) + the static 2-D arrays (72 B/edge, 96 B/element, 24 B/node).
    """
    N_wl = mesh.n_wet_layers
    N_wi = N_wl + mesh.nod2D
    E_wl = mesh.n_wet_elem_layers
    per_inst = ntr * 24 * N_wl + 16 * E_wl + 8 * N_wi
    per_thick = 16 * N_wl + 8 * E_wl
    per_mesh = 8 * N_wi + 8 * N_wl + 72 * mesh.edge2D + 96 * mesh.elem2D + 24 * mesh.nod2D
    return n_instances * per_inst + n_thickness_sets * per_thick + n_meshes * per_mesh
