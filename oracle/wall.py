"""Wall shear stress on the CPU (oracle; restates ``zvcfd/fv/wall.py:66-137``)."""

from __future__ import annotations

import numpy as np

from oracle.geometry import boundary_subface_weights, boundary_subfaces
from zvcfd_b200.topology import FACES, REF_NODES, _parameters_of, shape_functions


def wall_shear(mesh, zone_ids, U, mu=1.0, viscosity=None):
    """``tau (N, 3)``: per wall sub-face ip the owning element's gradient, the tangential
    viscous traction, area-weighted per node."""
    faces = np.concatenate([mesh.zones[z].faces for z in zone_ids])
    on = np.zeros(mesh.n_nodes, bool)
    on[faces[faces >= 0]] = True
    W = boundary_subface_weights(faces)
    S = boundary_subfaces(mesh.nodes, faces)
    key = {tuple(sorted(f[f >= 0].tolist())): i for i, f in enumerate(faces)}
    acc = np.zeros((mesh.n_nodes, 3))
    wsum = np.zeros(mesh.n_nodes)
    for kind, E in mesh.elements.items():
        cand = np.flatnonzero(on[E].sum(1) >= 3)
        for fl in FACES[kind]:
            for e in cand:
                fn = tuple(sorted(E[e, list(fl)].tolist()))
                fi = key.get(fn)
                if fi is None:
                    continue
                f = faces[fi]
                for si in range(4):
                    if f[si] < 0:
                        continue
                    loc = [int(np.flatnonzero(E[e] == v)[0]) if v >= 0 else 0 for v in f]
                    ref = np.array([REF_NODES[kind][l] if v >= 0 else [0, 0, 0]
                                    for l, v in zip(loc, f)], float)
                    pt = W[fi, si] @ ref
                    _, dN = shape_functions(kind, _parameters_of(kind, pt[None]))
                    x = mesh.nodes[E[e]]
                    J = np.einsum("nk,nd->kd", x, dN[0])
                    G = dN[0] @ np.linalg.inv(J)
                    g = np.einsum("ni,nj->ij", U[E[e]], G)
                    D = g + g.T
                    m = mu
                    if viscosity is not None:
                        rate = np.sqrt(0.5 * (D * D).sum())
                        v = viscosity
                        m = v.mu_inf + (v.mu_0 - v.mu_inf) * (1 + (v.lam * rate) ** v.a) ** (
                            (v.n - 1) / v.a)
                    a = S[fi, si]
                    area = np.linalg.norm(a)
                    n = a / area
                    t = m * D @ n
                    t = t - (t @ n) * n
                    acc[f[si]] -= t * area
                    wsum[f[si]] += area
    return acc / np.maximum(wsum, 1e-300)[:, None]
