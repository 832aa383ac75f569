"""Partitions of a mesh for the partitioned solve (:mod:`zvcfd_b200.multi`).

The reference partitions its meshes in ``zvcfd/fv/partition.py:1-147``; this module gives
the same partitions, so that a run split here has the reference's owners, local numbering
and halo plans:

- **ownership** (:func:`morton_owner`): nodes are binned into cubic chunks of edge
  ``chunk``; the chunks are ordered along a Morton (Z-order) curve, with bit ``b`` of the
  chunk's x, y, z index at key bit ``3b``, ``3b + 1``, ``3b + 2`` (21 bits per axis); the
  node sequence in that order is cut into ``n`` pieces at the chunk boundaries nearest to
  equal node counts (the first chunk start at or after ``k N / n``). A partition owns whole
  chunks. The default chunk edge gives about 64 chunks per partition.
- **local meshes** (:func:`local_meshes`): partition ``p`` holds every element with a node it
  owns and every boundary face touching such a node; its local nodes are its owned nodes
  (ascending), then its halo (the other nodes of those elements) grouped by owner, each group
  ascending. Every control volume of an owned node is then complete locally.
- **halo plans** (:func:`halo_plan`): for each partition, per owner of some of its halo, the
  owner's local rows to send and this partition's rows they fill.

The Morton key is built by spreading each 21-bit index to every third bit with the
shift-and-mask sequence of the classic bit-interleaving construction (one vector operation
per step) instead of a loop over bits.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from zvcfd_b200.mesh import Mesh, Zone

_SPREAD = ((32, 0x1F00000000FFFF), (16, 0x1F0000FF0000FF), (8, 0x100F00F00F00F00F),
           (4, 0x10C30C30C30C30C3), (2, 0x1249249249249249))


def _spread3(v: np.ndarray) -> np.ndarray:
    """The low 21 bits of ``v`` moved to bits 0, 3, 6, ... of a uint64."""
    v = v.astype(np.uint64) & np.uint64(0x1FFFFF)
    for shift, mask in _SPREAD:
        v = (v | (v << np.uint64(shift))) & np.uint64(mask)
    return v


def morton_key(ijk: np.ndarray) -> np.ndarray:
    """Z-order key of non-negative integer triples ``(M, 3)`` (21 bits per axis)."""
    return _spread3(ijk[:, 0]) | (_spread3(ijk[:, 1]) << np.uint64(1)) | \
        (_spread3(ijk[:, 2]) << np.uint64(2))


def default_chunk(nodes: np.ndarray, n_parts: int) -> float:
    """A chunk edge giving about 64 chunks per partition over the bounding box."""
    extent = np.maximum(nodes.max(0) - nodes.min(0), 1e-300)
    return (float(np.prod(extent)) / (64 * n_parts)) ** (1 / 3)


def morton_owner(nodes: np.ndarray, n_parts: int, chunk: float | None = None) -> np.ndarray:
    """Owner partition ``(N,)`` int64 of each node (whole Morton chunks, balanced by nodes;
    ``zvcfd/fv/partition.py:40-65``). Raises ``ValueError`` when whole chunks cannot give
    every partition a node."""
    if n_parts < 1:
        raise ValueError("n_parts must be at least 1")
    nodes = np.asarray(nodes, np.float64)
    n = len(nodes)
    if chunk is None:
        chunk = default_chunk(nodes, n_parts)
    cell = np.floor((nodes - nodes.min(0)) / chunk).astype(np.int64)
    key = morton_key(cell)
    order = np.argsort(key, kind="stable")
    sorted_key = key[order]
    first = np.ones(n, bool)
    first[1:] = sorted_key[1:] != sorted_key[:-1]
    chunk_start = np.flatnonzero(first)
    want = n * np.arange(1, n_parts) / n_parts
    at = np.minimum(np.searchsorted(chunk_start, want), len(chunk_start) - 1)
    bounds = np.concatenate([[0], chunk_start[at], [n]])
    part_of_rank = np.repeat(np.arange(n_parts), np.diff(bounds))
    owner = np.empty(n, np.int64)
    owner[order] = part_of_rank
    if np.unique(owner).size != n_parts:
        raise ValueError(f"cannot cut {n} nodes into {n_parts} partitions of whole chunks: "
                         "use a smaller chunk")
    return owner


@dataclass
class LocalMesh:
    """One partition: its local mesh and the maps back to the global mesh."""

    part: int
    mesh: Mesh                # local numbering: owned nodes first, then the halo
    nodes: np.ndarray         # (n_local,) global node of each local node
    n_own: int
    elements: dict            # kind -> global indices of the elements held
    faces: dict               # zone -> global indices of the faces held

    @property
    def n_halo(self) -> int:
        return len(self.nodes) - self.n_own


def local_meshes(mesh: Mesh, owner: np.ndarray) -> list:
    """Every partition's :class:`LocalMesh` (``zvcfd/fv/partition.py:83-114``)."""
    owner = np.asarray(owner, np.int64)
    out = []
    for p in range(int(owner.max()) + 1):
        mine = owner == p
        own = np.flatnonzero(mine)
        held = {k: np.flatnonzero(mine[e].any(1)) for k, e in mesh.elements.items()}
        touched = np.zeros(mesh.n_nodes, bool)
        for k, sel in held.items():
            touched[mesh.elements[k][sel].ravel()] = True
        halo = np.flatnonzero(touched & ~mine)
        halo = halo[np.argsort(owner[halo], kind="stable")]     # by owner, ascending within
        glob = np.concatenate([own, halo])
        local = np.full(mesh.n_nodes, -1, np.int64)
        local[glob] = np.arange(len(glob))
        elements = {k: local[mesh.elements[k][sel]] for k, sel in held.items() if len(sel)}
        zones, fmap = {}, {}
        for zid, z in mesh.zones.items():
            f = z.faces
            valid = f >= 0
            sel = np.flatnonzero((mine[np.where(valid, f, 0)] & valid).any(1))
            lf = np.where(valid[sel], local[np.where(valid[sel], f[sel], 0)], -1)
            zones[zid] = Zone(zid, z.kind, z.name, lf)
            fmap[zid] = sel
        out.append(LocalMesh(p, Mesh(mesh.nodes[glob], elements, zones), glob, len(own),
                             held, fmap))
    return out


def halo_plan(parts: list, owner: np.ndarray) -> list:
    """For each partition ``p``: ``[(q, send, recv)]`` in ascending ``q``: ``q``'s local owned
    rows ``send`` fill ``p``'s local halo rows ``recv`` (``zvcfd/fv/partition.py:117-135``)."""
    owner = np.asarray(owner, np.int64)
    row_in_owner = np.empty(len(owner), np.int64)
    for q in parts:
        row_in_owner[q.nodes[:q.n_own]] = np.arange(q.n_own)
    plans = []
    for p in parts:
        halo = p.nodes[p.n_own:]
        rows = np.arange(p.n_own, len(p.nodes))
        who = owner[halo]
        plans.append([(int(q), row_in_owner[halo[who == q]], rows[who == q])
                      for q in np.unique(who)])
    return plans


def partition_report(parts: list) -> dict:
    """Owned and halo nodes per partition, overlap (halo over owned) and imbalance."""
    own = [p.n_own for p in parts]
    halo = [p.n_halo for p in parts]
    return {"parts": len(parts), "owned": own, "halo": halo,
            "overlap": [h / o for h, o in zip(halo, own)],
            "imbalance": max(own) / (sum(own) / len(own)) - 1.0}


__all__ = ["LocalMesh", "default_chunk", "halo_plan", "local_meshes", "morton_key",
           "morton_owner", "partition_report"]
