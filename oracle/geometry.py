"""Median-dual geometry on the CPU (oracle; restates ``zvcfd/fv/geometry.py``).

All functions take element node coordinates ``x (E, n, 3)`` of one type.
"""

from __future__ import annotations

import numpy as np

from zvcfd_b200.topology import tables


def element_points(x: np.ndarray, kind: str) -> np.ndarray:
    """Dual points ``(E, n_pts, 3)`` (``zvcfd/fv/geometry.py:177-179``)."""
    return np.einsum("pn,enk->epk", tables(kind).weights, x)


def _flux_triangles(P: np.ndarray, kind: str):
    """The three corners ``(E, n_ip, 3)`` each of every flux point's dual-face triangle."""
    T = P[:, tables(kind).tris]
    return T[:, :, 0], T[:, :, 1], T[:, :, 2]


def ip_areas(P: np.ndarray, kind: str) -> np.ndarray:
    """Flux-point area vectors ``(E, n_ip, 3)``, edge node a -> b (``geometry.py:182-185``)."""
    p0, p1, p2 = _flux_triangles(P, kind)
    return 0.5 * np.cross(p1 - p0, p2 - p0)


def ip_points(P: np.ndarray, kind: str) -> np.ndarray:
    """Flux-point centroids ``(E, n_ip, 3)`` (``geometry.py:188-190``)."""
    p0, p1, p2 = _flux_triangles(P, kind)
    return (p0 + p1 + p2) / 3.0


def scv_volumes(P: np.ndarray, kind: str) -> np.ndarray:
    """Sub-control volumes ``(E, n)`` by the divergence theorem (``geometry.py:193-215``): the
    volume of a node's part of the element is a third of the flux of ``x - x_node`` out of it,
    and only the dual faces (the flux-point triangles) carry any, the rest of its boundary
    lying in element faces through the node."""
    t = tables(kind)
    A, c = ip_areas(P, kind), ip_points(P, kind)
    x = P[:, :t.n]
    vol = np.zeros((len(P), t.n))
    for s, (a, b) in enumerate(t.edge):          # the area points from node a to node b
        vol[:, a] += np.einsum("ek,ek->e", c[:, s] - x[:, a], A[:, s]) / 3.0
        vol[:, b] -= np.einsum("ek,ek->e", c[:, s] - x[:, b], A[:, s]) / 3.0
    return vol


def gradients(x: np.ndarray, kind: str) -> np.ndarray:
    """Shape-function gradients at the flux points ``(E, n_ip, n, 3)`` (``geometry.py:218-223``):
    ``grad N = J^-T dN``, ``J`` the Jacobian of the element map there."""
    dN = tables(kind).dN_ip                                  # (n_ip, n, 3)
    J = np.einsum("enk,ind->eikd", x, dN)                    # dx_k / dxi_d
    Jt = np.swapaxes(J, -1, -2)
    rhs = np.broadcast_to(np.swapaxes(dN, -1, -2)[None], Jt.shape[:2] + (3, dN.shape[1]))
    return np.swapaxes(np.linalg.solve(Jt, rhs), -1, -2)


def boundary_subfaces(nodes: np.ndarray, faces: np.ndarray) -> np.ndarray:
    """Each node's share of each boundary face, area vectors ``(F, 4, 3)`` (``geometry.py:226-244``):
    the polygon node, next edge midpoint, face centroid, previous edge midpoint, by the vector
    shoelace formula, one face at a time."""
    out = np.zeros(faces.shape + (3,))
    for fi, face in enumerate(faces):
        P = nodes[[int(v) for v in face if v >= 0]]
        n = len(P)
        c = P.mean(0)
        for i in range(n):
            # taken about the centroid, so that far-off coordinates cost no precision
            poly = [P[i] - c, 0.5 * (P[i] + P[(i + 1) % n]) - c, np.zeros(3),
                    0.5 * (P[i] + P[(i - 1) % n]) - c]
            out[fi, i] = 0.5 * sum(np.cross(poly[k], poly[(k + 1) % 4]) for k in range(4))
    return out


def boundary_subface_weights(faces: np.ndarray) -> np.ndarray:
    """Weights ``(F, 4, 4)`` from face nodes to each sub-face's area centroid (``geometry.py:247-266``):
    22/36 for the node and 7/36 for each other on a triangle; on a quadrilateral 9/16, 3/16, 1/16
    by the distance around the face."""
    tri = (15.0 * np.eye(3) + 7.0) / 36.0
    gap = np.abs(np.subtract.outer(np.arange(4), np.arange(4)))
    quad = np.array([9.0, 3.0, 1.0])[np.minimum(gap, 4 - gap)] / 16.0
    w = np.zeros(faces.shape + (4,))
    for fi, face in enumerate(faces):
        if face[3] >= 0:
            w[fi] = quad
        else:
            w[fi, :3, :3] = tri
    return w


class ElementGeometry:
    """Per-type geometry of a mesh (``zvcfd/fv/reference.py:465-474``)."""

    def __init__(self, kind: str, elem: np.ndarray, nodes: np.ndarray):
        t = tables(kind)
        self.kind, self.elem, self.t = kind, elem, t
        x = nodes[elem]
        P = element_points(x, kind)
        self.A = ip_areas(P, kind)
        self.G = gradients(x, kind)
        self.N = t.N_ip
        self.xip = ip_points(P, kind)
        self.scv = scv_volumes(P, kind)
        self.gbar = self.G.mean(1)
        self.ea, self.eb = t.edge[:, 0], t.edge[:, 1]


def node_volumes(mesh, geoms) -> np.ndarray:
    V = np.zeros(mesh.n_nodes)
    for g in geoms:
        V += np.bincount(g.elem.ravel(), g.scv.ravel(), mesh.n_nodes)
    return V


__all__ = ["ElementGeometry", "boundary_subface_weights", "boundary_subfaces", "element_points",
           "gradients", "ip_areas", "ip_points", "node_volumes", "scv_volumes"]
