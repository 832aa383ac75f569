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


def face_owners(mesh, faces: np.ndarray):
    """``(kind per face, element row)`` of the element owning each boundary face."""
    keys, kinds, rows = [], [], []
    for kind, e in mesh.elements.items():
        for fl in FACES[kind]:
            loc = e[:, list(fl)]
            if len(fl) == 3:
                loc = np.concatenate([loc, -np.ones((len(e), 1), np.int64)], 1)
            keys.append(np.sort(loc, 1))
            kinds.append(np.full(len(e), kind, dtype=object))
            rows.append(np.arange(len(e)))
    keys, kinds, rows = np.concatenate(keys), np.concatenate(kinds), np.concatenate(rows)
    fk = np.sort(faces, 1)
    allk = np.concatenate([keys, fk])
    _, inv = np.unique(allk, axis=0, return_inverse=True)
    inv = inv.reshape(-1)
    where = -np.ones(inv.max() + 1, np.int64)
    where[inv[:len(keys)]] = np.arange(len(keys))
    hit = where[inv[len(keys):]]
    if (hit < 0).any():
        raise ValueError(f"{int((hit < 0).sum())} wall faces belong to no element")
    return kinds[hit], rows[hit]


def wall_operator(mesh, zone_ids):
    """Per wall sub-face integration point: owning element's nodes ``(M, 8)`` (-1 padded),
    shape-function gradients ``(M, 8, 3)``, unit outward normal, area and wall node."""
    faces = np.concatenate([mesh.zones[z].faces for z in zone_ids])
    kind_of, erow = face_owners(mesh, faces)
    W = subface_weights(faces)
    S = subfaces(mesh.nodes, faces)
    elem, G, nrm, area, node = [], [], [], [], []
    for kind in mesh.elements:
        fsel = np.flatnonzero(kind_of == kind)
        if not len(fsel):
            continue
        e = mesh.elements[kind][erow[fsel]]
        f = faces[fsel]
        ok = f >= 0
        loc = np.argmax(e[:, None, :] == np.where(ok, f, -2)[:, :, None], axis=2)
        ref = np.asarray(REF_NODES[kind], float)[loc]
        ref = np.where(ok[..., None], ref, 0.0)
        pts = np.einsum("fij,fjd->fid", W[fsel], ref)
        fi, si = np.nonzero(ok)
        _, dN = shape_functions(kind, _parameters_of(kind, pts[fi, si]))
        x = mesh.nodes[e[fi]]
        J = np.einsum("mnk,mnd->mkd", x, dN)
        g = np.einsum("mnd,mdk->mnk", dN, np.linalg.inv(J))
        a = S[fsel][fi, si]
        ar = np.linalg.norm(a, axis=1)
        n = e.shape[1]
        ep = -np.ones((len(fi), MAXN), np.int64)
        ep[:, :n] = e[fi]
        gp = np.zeros((len(fi), MAXN, 3))
        gp[:, :n] = g
        elem.append(ep)
        G.append(gp)
        nrm.append(a / ar[:, None])
        area.append(ar)
        node.append(f[fi, si])
    return (np.concatenate(elem), np.concatenate(G), np.concatenate(nrm), np.concatenate(area),
            np.concatenate(node))


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
