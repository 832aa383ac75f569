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


def _zone_areas(bc, zid) -> np.ndarray:
    """``(N,)``: each node's sub-face area in zone ``zid``."""
    f, S = bc.sub[zid]
    ok = f >= 0
    return np.bincount(f[ok], np.linalg.norm(S[ok], axis=-1), bc.N)


def _fixed_axes(bc, zid) -> np.ndarray:
    """The velocity components a zone fixes: all three, or a symmetry plane's normal axis."""
    if bc.bcs[zid]["kind"] != "symmetry":
        return np.ones(3, bool)
    total = np.abs(bc.sub[zid][1].reshape(-1, 3).sum(0))
    return total == total.max()


def _inlet_momentum(bc, zid) -> np.ndarray:
    """``(3,)``: the momentum flux ``Σ m_sub u_sub`` through a zone's sub-faces."""
    f = bc.sub[zid][0]
    return np.einsum("fi,fik->k", np.where(f >= 0, bc.sub_flow[zid], 0.0), bc.sub_vel[zid])


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
    reaction = -np.where(bc.vel_fixed_comp, np.asarray(residual)[:, :3], 0.0)
    fixing = [z for z in bc.sub if bc.bcs[z]["kind"] != "pressure"]
    # (zones, N, 3): each fixing zone's claim on each node's reaction components
    claim = np.stack([_zone_areas(bc, z)[:, None] * _fixed_axes(bc, z)[None, :]
                      for z in fixing]) if fixing else np.zeros((0, bc.N, 3))
    total = claim.sum(0)
    share = np.divide(claim, total[None], out=np.zeros_like(claim), where=total[None] > 0)
    forces = dict(zip(fixing, np.einsum("znk,nk->zk", share, reaction)))
    lumped = set(lumped)
    out = {}
    for zid, (f, S) in bc.sub.items():
        kind = bc.bcs[zid]["kind"]
        if kind == "pressure":
            p = P[np.where(f >= 0, f, 0)] if zid in lumped else bc.p_sub[zid]
            out[zid] = np.einsum("fi,fik->k", np.where(f >= 0, p, 0.0), S)
        elif kind == "velocity" and not stokes:
            out[zid] = forces[zid] - _inlet_momentum(bc, zid)
        else:
            out[zid] = forces[zid]
    return out


def wall_geometry(bc):
    """``(nodes, n, area, share)`` of the wall nodes (``zvcfd/fv/solver.py:1128-1161``): the
    nodes with wall sub-face area, their outward unit normals and wall areas, and the wall's
    fraction of the sub-face area of the zones fixing each node's velocity."""
    walls = [z for z in bc.sub if bc.bcs[z]["kind"] == "wall"]
    inlets = [z for z in bc.sub if bc.bcs[z]["kind"] == "velocity"]
    wall_area = sum((_zone_areas(bc, z) for z in walls), np.zeros(bc.N))
    fixed_area = wall_area + sum((_zone_areas(bc, z) for z in inlets), np.zeros(bc.N))
    outward = np.zeros((bc.N, 3))
    for z in walls:
        f, S = bc.sub[z]
        ok = f >= 0
        np.add.at(outward, f[ok], S[ok])
    nodes = np.flatnonzero(wall_area > 0)
    n = outward[nodes] / np.linalg.norm(outward[nodes], axis=1)[:, None]
    share = wall_area[nodes] / fixed_area[nodes]
    return nodes, n, wall_area[nodes], share


def wall_shear_reaction(bc, residual: np.ndarray, P: np.ndarray, *, stokes: bool = False):
    """Wall shear stress from consistent reactions, ``(nodes, tau (n, 3))``
    (``zvcfd/fv/solver.py:1200-1230``): the tangential part of minus the momentum residual at
    each wall node, less the pressure force and the momentum of any inlet sub-faces the node
    also borders, over the node's wall area."""
    nodes, n, area, _ = wall_geometry(bc)
    F = -np.asarray(residual, float)[:, :3].copy()
    for zid, (f, S) in bc.sub.items():
        if bc.bcs[zid]["kind"] != "velocity":
            continue
        ok = f >= 0
        carried = S * P[np.where(ok, f, 0)][..., None]
        if not stokes:
            carried = carried + bc.sub_flow[zid][..., None] * bc.sub_vel[zid]
        np.subtract.at(F, f[ok], carried[ok])
    F = F[nodes]
    normal_part = np.einsum("nk,nk->n", F, n)
    return nodes, (F - normal_part[:, None] * n) / area[:, None]


__all__ = ["RawRows", "wall_geometry", "wall_shear_reaction", "zone_forces"]
