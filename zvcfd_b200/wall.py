"""Wall shear stress from velocity gradients at the wall integration points, on the device.

The evaluator of ``zvcfd/fv/wall.py:66-137`` (``WallGradientShear``, CFX's laminar-wall
method): each wall face is split among its nodes into sub-faces; each sub-face carries one
integration point at its area centroid, where the element owning the face gives
``grad u = sum_n u_n (x) grad N_n``; the shear stress is the tangential part of the viscous
traction, ``tau = -(t - (t . n) n)`` with ``t = mu (grad u + grad u^T) . n``, and a node's value
is the area-weighted mean over its wall sub-faces. The operator (owning elements, shape
gradients, normals, areas) is built once on the host; ``zvfv_wall_shear`` evaluates it, one
thread per wall node summing its sub-faces in a fixed order (deterministic, no atomics).
"""

from __future__ import annotations

import numpy as np
import torch

from zvcfd_b200._lib import call, ptr, stream_ptr
from zvcfd_b200.boundary import subface_weights, subfaces
from zvcfd_b200.topology import FACES, REF_NODES, _parameters_of, shape_functions

MAXN = 8


def _face_keys(faces: np.ndarray, n_nodes: int):
    """Two int64 keys per face from its sorted node ids (``-1`` pads count as 0): equal keys,
    equal faces."""
    k = np.sort(faces, axis=1) + 1
    base = np.int64(n_nodes + 1)
    return k[:, 0] * base + k[:, 1], k[:, 2] * base + k[:, 3]


def face_owners(mesh, faces: np.ndarray):
    """``(kind per face, element row)`` of the element owning each boundary face: the element
    faces and the queried faces are sorted together by key, and each queried face takes the
    element face next to it in that order when their keys agree."""
    owner_kind, owner_row, el_faces = [], [], []
    for kind, e in mesh.elements.items():
        for local in FACES[kind]:
            pad = np.full((len(e), 4 - len(local)), -1, np.int64)
            el_faces.append(np.concatenate([e[:, list(local)], pad], 1))
            owner_kind.append(np.full(len(e), kind, dtype=object))
            owner_row.append(np.arange(len(e)))
    el_faces = np.concatenate(el_faces)
    owner_kind, owner_row = np.concatenate(owner_kind), np.concatenate(owner_row)
    hi, lo = _face_keys(np.concatenate([el_faces, faces]), mesh.n_nodes)
    is_query = np.r_[np.zeros(len(el_faces), bool), np.ones(len(faces), bool)]
    # element faces sort before the queried copy of the same face
    order = np.lexsort((is_query, lo, hi))
    hit = np.full(len(faces), -1, np.int64)
    q = np.flatnonzero(is_query[order][1:]) + 1           # positions of queried faces
    prev = order[q - 1]
    same = (hi[prev] == hi[order[q]]) & (lo[prev] == lo[order[q]]) & ~is_query[prev]
    hit[order[q][same] - len(el_faces)] = prev[same]
    if (hit < 0).any():
        raise ValueError(f"{int((hit < 0).sum())} wall faces belong to no element")
    return owner_kind[hit], owner_row[hit]


def _local_positions(e: np.ndarray, f: np.ndarray, n_nodes: int) -> np.ndarray:
    """``(F, 4)``: where each node of face ``f[i]`` sits in element ``e[i]`` (0 for pads),
    found by a search in each element's sorted node list."""
    shift = (np.arange(len(e), dtype=np.int64) * (n_nodes + 1))[:, None]
    order = np.argsort(e, axis=1)
    flat = (np.take_along_axis(e, order, 1) + shift).ravel()
    at = np.searchsorted(flat, (np.where(f >= 0, f, e[:, :1]) + shift).ravel())
    at = at.reshape(f.shape) - np.arange(len(e))[:, None] * e.shape[1]
    return np.where(f >= 0, np.take_along_axis(order, at, 1), 0)


def wall_operator(mesh, zone_ids):
    """Per wall sub-face integration point: owning element's nodes ``(M, 8)`` (-1 padded),
    shape-function gradients ``(M, 8, 3)``, unit outward normal, area and wall node.

    The integration point of a sub-face is its area centroid; in the owning element's
    reference coordinates that is the same weights applied to the face nodes' reference
    positions, where the element's shape functions give ``grad N = J^-T dN``."""
    faces = np.concatenate([mesh.zones[z].faces for z in zone_ids])
    kind_of, erow = face_owners(mesh, faces)
    W = subface_weights(faces)
    S = subfaces(mesh.nodes, faces)
    parts = []
    for kind in mesh.elements:
        fsel = np.flatnonzero(kind_of == kind)
        if not len(fsel):
            continue
        e = mesh.elements[kind][erow[fsel]]
        f = faces[fsel]
        ref = np.asarray(REF_NODES[kind], float)[_local_positions(e, f, mesh.n_nodes)]
        ref[f < 0] = 0.0
        ips = np.einsum("fij,fjd->fid", W[fsel], ref)
        fi, si = np.nonzero(f >= 0)
        _, dN = shape_functions(kind, _parameters_of(kind, ips[fi, si]))    # (M, n, 3)
        x = mesh.nodes[e[fi]]
        J = np.einsum("mnk,mnd->mkd", x, dN)                                # dx_k / dxi_d
        grad = np.swapaxes(np.linalg.solve(np.swapaxes(J, 1, 2), np.swapaxes(dN, 1, 2)), 1, 2)
        vec = S[fsel][fi, si]
        size = np.linalg.norm(vec, axis=1)
        n = e.shape[1]
        elem = np.full((len(fi), MAXN), -1, np.int64)
        elem[:, :n] = e[fi]
        G = np.zeros((len(fi), MAXN, 3))
        G[:, :n] = grad
        parts.append((elem, G, vec / size[:, None], size, f[fi, si]))
    return tuple(np.concatenate(col) for col in zip(*parts))


class WallShear:
    """Wall shear stress ``(N, 3)`` of the wall zones, evaluated on the device."""

    def __init__(self, mesh, zone_ids, device="cuda"):
        elem, G, nrm, area, node = wall_operator(mesh, zone_ids)
        order = np.argsort(node, kind="stable")
        self.N = mesh.n_nodes
        counts = np.bincount(node, minlength=self.N)
        ptr_ = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
        dev = lambda a, t: torch.as_tensor(np.ascontiguousarray(a), dtype=t, device=device)  # noqa: E731
        self.elem = dev(elem[order], torch.int32)
        self.G = dev(G[order], torch.float64)
        self.nrm = dev(nrm[order], torch.float64)
        self.area = dev(area[order], torch.float64)
        self.node_ptr = dev(ptr_, torch.int64)
        self.wall_nodes = dev(np.flatnonzero(counts), torch.int64)
        self.node_area = dev(np.bincount(node, area, self.N), torch.float64)

    def __call__(self, U, viscosity=None, mu: float = 1.0):
        U = torch.as_tensor(U, device="cuda", dtype=torch.float64).contiguous()
        out = torch.zeros((self.N, 3), dtype=torch.float64, device="cuda")
        if viscosity is None:
            rh = (0, float(mu), float(mu), 0.0, 2.0, 1.0)
        else:
            v = viscosity
            rh = (1, float(v.mu_0), float(v.mu_inf), float(v.lam), float(v.a), float(v.n))
        call("zvfv_wall_shear", self.N, ptr(self.node_ptr), ptr(self.elem), ptr(self.G),
             ptr(self.nrm), ptr(self.area), ptr(U), *rh, ptr(out), stream_ptr())
        return out

    def mean(self, tau, nodes=None):
        """Area-weighted mean magnitude of ``tau`` over the wall nodes (or ``nodes``)."""
        mag = torch.linalg.norm(tau, dim=1)
        sel = self.wall_nodes if nodes is None else nodes
        a = self.node_area[sel]
        return (mag[sel] * a).sum() / a.sum()


__all__ = ["WallShear", "face_owners", "wall_operator"]
