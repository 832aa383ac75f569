"""Zone forces from consistent reactions, as the reference's ``GPUSolver.zone_forces``.

The boundary pass keeps, before Dirichlet rows replace them, the assembled rows of every node
with a fixed velocity component (and of the nodes of lumped outlets): row ``i``'s blocks sit
contiguously at ``rawoff[i]`` in the pattern's column order (``rawoff[i] = -1`` for rows not
kept), its right-hand side at ``rawb[i]``. :class:`RawRows` applies those rows to a state, the
reference's ``RawRows.residual`` (``zvcfd/fv/solver.py:1303-1328``); :func:`zone_forces`
shares the reactions among the zones (``zvcfd/fv/solver.py:1080-1124``) and
:func:`wall_shear_reaction` turns them into wall shear stress (``:1200-1230``). The residual
works on tensors of any device and the rest on host arrays, so the same code runs on the CPU
in the tests.
"""

from __future__ import annotations

import numpy as np
import torch


class RawRows:
    """The kept rows of the assembled block system.

    Args:
        indptr, indices: the block pattern (``(N+1,)``, ``(nnzb,)``).
        rawoff: ``(N,)`` int64: offset of row ``i``'s first kept block, ``-1`` if not kept.
        data: kept blocks, at least ``(Σ kept row lengths, 4, 4)`` (a flat buffer is viewed).
        b: ``(N, 4)`` right-hand side before Dirichlet replacement (read at kept rows only).
    """

    def __init__(self, indptr, indices, rawoff, data, b):
        dev = rawoff.device
        indptr = indptr.to(device=dev, dtype=torch.int64)
        self.N = N = rawoff.numel()
        self.kept = rawoff >= 0
        rows = torch.nonzero(self.kept).reshape(-1)
        counts = (indptr[1:] - indptr[:-1])[rows]
        self.nraw = int(counts.sum())
        self.rows = torch.repeat_interleave(rows, counts)
        j = torch.arange(self.nraw, device=dev, dtype=torch.int64)
        pos = indptr[self.rows] + j - rawoff[self.rows]
        self.cols = indices.to(device=dev, dtype=torch.int64)[pos]
        self.data = data.reshape(-1, 4, 4)[:self.nraw]
        self.b = b.reshape(N, 4)

    def residual(self, X) -> torch.Tensor:
        """``(N, 4)``: ``A x - b`` at the kept rows, zero elsewhere (``X`` is ``(N, 4)``)."""
        X = X.reshape(self.N, 4)
        r = torch.zeros_like(self.b)
        r.index_add_(0, self.rows, torch.einsum("kij,kj->ki", self.data, X[self.cols]))
        return torch.where(self.kept[:, None], r - self.b, torch.zeros_like(r))


def zone_forces(bc, residual: np.ndarray, P: np.ndarray, *, stokes: bool = False,
                lumped=()) -> dict:
    """Force of the fluid on each zone, ``{zone: (3,)}`` (N).

    At nodes with fixed velocity components the force is minus the momentum residual of the
    kept rows, shared among the zones that fix each component by sub-face area (walls and
    inlets fix all three, a symmetry plane its normal), less the momentum an inlet carries in.
    At a pressure zone it is the pressure force ``p S`` over its sub-faces, ``p`` the imposed
    value or, at a lumped outlet, the nodal pressure; the lagged viscous traction of the
    zero-gradient outlet is left out, as the reference's device solver leaves it out.

    Args:
        bc: the :class:`~zvcfd_b200.boundary.Boundary` of the solve (sub-faces, kinds, values).
        residual: ``(N, 3)`` momentum residual of the kept rows at the current state.
        P: ``(N,)`` nodal pressure.
        stokes: no advection (no momentum carried through inlets).
        lumped: ids of the lumped pressure zones.
    """
    N = bc.N
    react = np.where(bc.vel_fixed_comp, -np.asarray(residual)[:, :3], 0.0)
    per, tot = {}, np.zeros((N, 3))
    for zid, (f, S) in bc.sub.items():
        kind = bc.bcs[zid]["kind"]
        if kind == "pressure":
            continue
        ok = f >= 0
        a = np.bincount(f[ok], np.linalg.norm(S, axis=2)[ok], N)
        comp = np.ones(3, bool)
        if kind == "symmetry":
            sn = np.abs(S.reshape(-1, 3).sum(0))
            comp = sn == sn.max()
        per[zid] = a[:, None] * comp[None, :]
        tot += per[zid]
    lumped = set(lumped)
    out = {}
    for zid, (f, S) in bc.sub.items():
        ok = f >= 0
        kind = bc.bcs[zid]["kind"]
        if kind == "pressure":
            p_sub = P[np.where(ok, f, 0)] if zid in lumped else bc.p_sub[zid]
            out[zid] = (p_sub[..., None] * S * ok[..., None]).reshape(-1, 3).sum(0)
            continue
        share = np.divide(per[zid], tot, out=np.zeros_like(tot), where=tot > 0)
        F = (share * react).sum(0)
        if kind == "velocity" and not stokes:
            F = F - np.einsum("fi,fik->k", bc.sub_flow[zid] * ok, bc.sub_vel[zid])
        out[zid] = F
    return out


def wall_geometry(bc):
    """``(nodes, n, area, share)`` of the wall nodes (``zvcfd/fv/solver.py:1128-1161``): the
    nodes with wall sub-face area, their outward unit normals and wall areas, and the wall's
    fraction of the sub-face area of the zones fixing each node's velocity."""
    N = bc.N
    Sn, area = np.zeros((N, 3)), np.zeros(N)
    wall, tot = np.zeros(N), np.zeros(N)
    for zid, (f, S) in bc.sub.items():
        kind = bc.bcs[zid]["kind"]
        if kind not in ("wall", "velocity"):
            continue
        ok = f >= 0
        a = np.bincount(f[ok], np.linalg.norm(S, axis=2)[ok], N)
        tot += a
        if kind == "wall":
            wall += a
            area += a
            for k in range(3):
                Sn[:, k] += np.bincount(f[ok], S[ok][:, k], N)
    nodes = np.flatnonzero(area > 0)
    n = Sn[nodes] / np.linalg.norm(Sn[nodes], axis=1, keepdims=True)
    share = np.divide(wall, tot, out=np.zeros(N), where=tot > 0)[nodes]
    return nodes, n, area[nodes], share


def wall_shear_reaction(bc, residual: np.ndarray, P: np.ndarray, *, stokes: bool = False):
    """Wall shear stress from consistent reactions, ``(nodes, tau (n, 3))``
    (``zvcfd/fv/solver.py:1200-1230``): the tangential part of minus the momentum residual at
    each wall node, less the pressure force and the momentum of any inlet sub-faces the node
    also borders, over the node's wall area."""
    nodes, n, area, _ = wall_geometry(bc)
    N = bc.N
    F = -np.asarray(residual)[:, :3].copy()
    for zid, (f, S) in bc.sub.items():
        if bc.bcs[zid]["kind"] != "velocity":
            continue
        ok = f >= 0
        for k in range(3):
            F[:, k] -= np.bincount(f[ok], S[ok][:, k], N) * P
            if not stokes:
                mom = bc.sub_flow[zid] * bc.sub_vel[zid][..., k]
                F[:, k] -= np.bincount(f[ok], mom[ok], N)
    F = F[nodes]
    tau = F - np.einsum("nk,nk->n", F, n)[:, None] * n
    return nodes, tau / area[:, None]


__all__ = ["RawRows", "wall_geometry", "wall_shear_reaction", "zone_forces"]
