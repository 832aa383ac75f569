"""Velocity shapes of flow-rate inlets (``zvcfd/fv/profiles.py`` of the reference).

A flow-rate inlet takes a shape along the zone's inward normal and is then scaled so that its
discrete inflow is the prescribed flow:

- ``"plug"``: uniform;
- ``"poiseuille"`` (or ``"parabolic"``, the default): the fully developed laminar profile of
  the zone's own cross-section, the solution of ``-Δu = 1`` on the (planar) face set with
  ``u = 0`` on its rim (F. M. White, *Viscous Fluid Flow*, 3rd ed., §3-3), by linear finite
  elements on the faces' triangles (quadrilaterals split along their 0-2 diagonal), scaled to
  a maximum of 1: ``1 - (r/R)^2`` on a circle, the exact developed shape on any other section;
- a callable ``f(x)`` of the zone nodes' coordinates.
"""

from __future__ import annotations

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spl


def face_triangles(faces: np.ndarray) -> np.ndarray:
    """``(T, 3)``: the faces' triangles (a quadrilateral ``abcd`` as ``abc`` and ``acd``)."""
    quads = faces[faces[:, 3] >= 0]
    parts = [faces[:, :3]]
    if len(quads):
        parts.append(quads[:, [0, 2, 3]])
    return np.concatenate(parts)


def zone_normal(X: np.ndarray, faces: np.ndarray) -> np.ndarray:
    """The face set's area-weighted unit normal (the faces' own orientation)."""
    t = face_triangles(faces)
    s = np.cross(X[t[:, 1]] - X[t[:, 0]], X[t[:, 2]] - X[t[:, 0]]).sum(0)
    return s / np.linalg.norm(s)


def rim_nodes(faces: np.ndarray) -> np.ndarray:
    """The nodes on edges that only one face of the set uses (sorted)."""
    nv = np.where(faces[:, 3] >= 0, 4, 3)
    a, b = [], []
    for k in range(4):
        used = k < nv
        a.append(faces[used, k])
        b.append(np.where(k + 1 < nv[used], faces[used, (k + 1) % 4], faces[used, 0]))
    a, b = np.concatenate(a), np.concatenate(b)
    e = np.stack([np.minimum(a, b), np.maximum(a, b)], 1)
    edges, count = np.unique(e, axis=0, return_counts=True)
    return np.unique(edges[count == 1])


def developed_profile(X: np.ndarray, faces: np.ndarray):
    """``(nodes, u)``: the zone's nodes (sorted) and the developed laminar profile there,
    ``max u = 1`` (see the module docstring)."""
    nodes = np.unique(faces[faces >= 0])
    tri = np.searchsorted(nodes, face_triangles(faces))
    n = zone_normal(X, faces)
    # in-plane coordinates: any orthonormal pair perpendicular to the normal
    a = np.eye(3)[int(np.argmin(np.abs(n)))]
    e1 = np.cross(n, a)
    e1 /= np.linalg.norm(e1)
    e2 = np.cross(n, e1)
    xy = np.stack([X[nodes] @ e1, X[nodes] @ e2], 1)
    p = xy[tri]                                                   # (T, 3, 2)
    # the edge opposite each vertex; P1 stiffness K_ij = (e_i . e_j) / (4 A)
    opp = np.stack([p[:, 2] - p[:, 1], p[:, 0] - p[:, 2], p[:, 1] - p[:, 0]], 1)
    area = 0.5 * np.abs(opp[:, 2, 0] * (-opp[:, 1, 1]) - opp[:, 2, 1] * (-opp[:, 1, 0]))
    K = np.einsum("tik,tjk->tij", opp, opp) / (4.0 * area)[:, None, None]
    m = len(nodes)
    A = sp.coo_matrix((K.reshape(-1), (np.repeat(tri, 3, 1).reshape(-1),
                                       np.tile(tri, (1, 3)).reshape(-1))), shape=(m, m)).tocsr()
    load = np.bincount(tri.reshape(-1), np.repeat(area / 3.0, 3), m)
    free = np.ones(m, bool)
    free[np.searchsorted(nodes, rim_nodes(faces))] = False
    u = np.zeros(m)
    u[free] = spl.spsolve(A[free][:, free].tocsc(), load[free])
    return nodes, u / u.max()


def inlet_shape(X: np.ndarray, faces: np.ndarray, profile="poiseuille"):
    """``(nodes, shape (n, 3))``: the zone's nodes (sorted) and the unscaled inlet velocity,
    along the inward normal."""
    nodes = np.unique(faces[faces >= 0])
    inward = -zone_normal(X, faces)
    if callable(profile):
        s = np.asarray(profile(X[nodes]), float).reshape(-1)
    elif profile == "plug":
        s = np.ones(len(nodes))
    elif profile in ("poiseuille", "parabolic"):
        s = developed_profile(X, faces)[1]
    else:
        raise ValueError(f"profile {profile!r}: plug, poiseuille (parabolic) or a callable")
    return nodes, s[:, None] * inward


__all__ = ["developed_profile", "face_triangles", "inlet_shape", "rim_nodes", "zone_normal"]
