"""Block pattern and element colouring on the CPU (oracle).

- :func:`node_graph` restates ``zvcfd/fv/pattern.py:18-33``: the union of the
  complete node graphs of all elements, self included, rows and columns sorted.
- :func:`colour` restates the device colouring ``gpu_colour`` of
  ``zvcfd/fv/fast.py:35-130`` round by round: deterministic 64-bit keys
  (:func:`element_keys`, ``fast.py:84-92``), then rounds in which every
  uncoloured element whose key is the smallest at all of its nodes takes the
  lowest colour none of its nodes has used. Winners of a round share no node,
  so the result does not depend on thread order, and a first fit does not
  depend on the width of the colour masks: unbounded masks give the same
  colours as the reference's doubling ones.
- :func:`slots` restates the slot order ``argsort(colour * E + e)`` and the
  per-colour offsets (``fast.py:199-203``).

Pinned: ``tests/test_colour.py`` holds :func:`colour` to the colours of the reference's own
``gpu_colour``, run on the CPU with its kernel source compiled by g++
(``tests/golden/make_golden.py colour``).
"""

from __future__ import annotations

import numpy as np

_M64 = (1 << 64) - 1


def node_graph(mesh):
    """``(indptr int64 (N+1,), indices int64)`` of node couplings (``pattern.py:18-33``): every
    ordered pair of nodes of every element, itself included, sorted and counted once."""
    rows, cols = [], []
    for e in mesh.elements.values():
        n = e.shape[1]
        rows.append(np.repeat(e, n, axis=1).ravel())
        cols.append(np.tile(e, (1, n)).ravel())
    r, c = np.concatenate(rows), np.concatenate(cols)
    order = np.lexsort((c, r))
    r, c = r[order], c[order]
    first = np.r_[True, (r[1:] != r[:-1]) | (c[1:] != c[:-1])]
    r, c = r[first], c[first]
    indptr = np.zeros(mesh.n_nodes + 1, np.int64)
    indptr[1:] = np.cumsum(np.bincount(r, minlength=mesh.n_nodes))
    return indptr, c.astype(np.int64)


def element_keys(E: int) -> np.ndarray:
    """A hash of the element index in the high 32 bits, the index in the low 32
    (``zvcfd/fv/fast.py:84-92``): distinct keys in a pseudo-random order. The hash is the
    SplitMix64 output function (Steele, Lea and Flood 2014) with its published constants."""
    e = np.arange(E, dtype=np.uint64)
    with np.errstate(over="ignore"):
        z = e + np.uint64(0x9E3779B97F4A7C15)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        z = z ^ (z >> np.uint64(31))
    return (z & np.uint64(0xFFFFFFFF00000000)) | e


def colour(conn: np.ndarray, n_nodes: int, max_rounds: int = 1_000_000) -> np.ndarray:
    """Colour ``(E,)`` int32 of each element: no two elements of a colour share a node."""
    conn = np.asarray(conn, np.int64)
    E, n = conn.shape
    key = element_keys(E)
    col = np.full(E, -1, np.int32)
    used = np.zeros((n_nodes, 64), bool)
    for _ in range(max_rounds):
        unc = np.flatnonzero(col < 0)
        if not len(unc):
            return col
        best = np.full(n_nodes, np.iinfo(np.uint64).max, np.uint64)
        np.minimum.at(best, conn[unc].ravel(), np.repeat(key[unc], n))
        win = unc[(best[conn[unc]] == key[unc, None]).all(1)]
        taken = used[conn[win]].any(1)                  # (W, C): colours a winner's nodes hold
        full = taken.all(1)
        if full.any():                                   # widen the masks, as the device doubles
            used = np.concatenate([used, np.zeros_like(used)], 1)
            taken = used[conn[win]].any(1)
        c = np.argmin(taken, axis=1).astype(np.int32)   # lowest free colour
        col[win] = c
        used[conn[win], c[:, None]] = True
    raise RuntimeError("colouring did not finish")


def slots(col: np.ndarray):
    """``(order slot -> element, offsets (C+1,))``: elements in colour order (stable)."""
    E = len(col)
    order = np.argsort(col.astype(np.int64) * E + np.arange(E), kind="stable")
    counts = np.bincount(col, minlength=int(col.max()) + 1 if E else 0)
    return order, np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)


def check_colouring(conn: np.ndarray, col: np.ndarray) -> None:
    """Raise if two elements of one colour share a node (``tests/test_fv_fast.py:72-75``)."""
    order = np.argsort(col, kind="stable")
    c_sorted = col[order]
    for c in np.unique(col):
        nodes = conn[order[c_sorted == c]].ravel()
        if len(np.unique(nodes)) != len(nodes):
            raise AssertionError(f"colour {c} has elements sharing a node")


__all__ = ["check_colouring", "colour", "element_keys", "node_graph", "slots"]
