"""Per-element-type tables of the median-dual finite-volume discretisation.

Every element type (tet, pyramid, wedge, hex) is split into one sub-control
volume per node. The surface between the sub-volumes of the two nodes of an
element edge is a four-point loop (edge midpoint, first face centroid,
element centroid, second face centroid); it is cut into two planar
triangles, and each triangle carries one **flux point** at its centroid.
So a type with ``ne`` edges has ``2 ne`` flux points, numbered
``2 e + half`` (half 0 is the triangle (m, f1, c), half 1 is (m, c, f2)).

These tables fix the layout that every kernel and every array of per-flux-
point values (mass flows ``(E, n_ip)``) shares with the reference solver:
the local node order and the edge and face lists are VTK's
(``zvcfd/mesh/core.py:34-52``), the loop construction and its orientation
follow ``zvcfd/fv/geometry.py:133-160``, and the shape functions and the
pyramid's collapsed-hexahedron map follow ``zvcfd/fv/geometry.py:64-109``
and ``:163-174``. The kernels receive the tables as compile-time constants
(``csrc/topology_tables.h``, written by :func:`write_header`).
"""

from __future__ import annotations

from dataclasses import dataclass
from functools import lru_cache
from pathlib import Path

import numpy as np

KINDS = ("tet", "pyramid", "wedge", "hex")
NODES_PER = {"tet": 4, "pyramid": 5, "wedge": 6, "hex": 8}

# VTK local orders: faces with outward normals by the right-hand rule, and edges
# (zvcfd/mesh/core.py:34-52). They are a data format shared with every mesh the
# reference reads or writes, so they are kept identical.
FACES = {
    "tet": ((0, 2, 1), (0, 1, 3), (1, 2, 3), (0, 3, 2)),
    "pyramid": ((0, 3, 2, 1), (0, 1, 4), (1, 2, 4), (2, 3, 4), (3, 0, 4)),
    "wedge": ((0, 2, 1), (3, 4, 5), (0, 1, 4, 3), (1, 2, 5, 4), (2, 0, 3, 5)),
    "hex": ((0, 3, 2, 1), (4, 5, 6, 7), (0, 1, 5, 4), (1, 2, 6, 5), (2, 3, 7, 6),
            (3, 0, 4, 7)),
}
EDGES = {
    "tet": ((0, 1), (1, 2), (2, 0), (0, 3), (1, 3), (2, 3)),
    "pyramid": ((0, 1), (1, 2), (2, 3), (3, 0), (0, 4), (1, 4), (2, 4), (3, 4)),
    "wedge": ((0, 1), (1, 2), (2, 0), (3, 4), (4, 5), (5, 3), (0, 3), (1, 4), (2, 5)),
    "hex": ((0, 1), (1, 2), (2, 3), (3, 0), (4, 5), (5, 6), (6, 7), (7, 4), (0, 4), (1, 5),
            (2, 6), (3, 7)),
}

# reference-element node coordinates (zvcfd/fv/geometry.py:56-63)
REF_NODES = {
    "tet": [[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1]],
    "wedge": [[0, 0, -1], [1, 0, -1], [0, 1, -1], [0, 0, 1], [1, 0, 1], [0, 1, 1]],
    "hex": [[-1, -1, -1], [1, -1, -1], [1, 1, -1], [-1, 1, -1],
            [-1, -1, 1], [1, -1, 1], [1, 1, 1], [-1, 1, 1]],
    "pyramid": [[-1, -1, -1], [1, -1, -1], [1, 1, -1], [-1, 1, -1], [0, 0, 1]],
}

MAX_IP_PER_NODE = 8          # a hex node touches 3 edges = 6 flux points; a pyramid apex 8


def shape_functions(kind: str, xi: np.ndarray):
    """Shape functions ``N (..., n)`` and parametric derivatives ``dN (..., n, 3)`` at ``xi``.

    tet: barycentric; wedge: triangle area coordinates times the linear
    ``(1 -+ zeta)/2``; hex: trilinear on ``[-1, 1]^3``; pyramid: the
    hexahedron with its top face collapsed to the apex (base nodes
    ``(1 +- xi)(1 +- eta)(1 - zeta)/8``, apex ``(1 + zeta)/2``).
    """
    xi = np.asarray(xi, float)
    u, v, w = xi[..., 0], xi[..., 1], xi[..., 2]
    if kind == "tet":
        N = np.stack([1.0 - u - v - w, u, v, w], -1)
        d = np.array([[-1.0, -1.0, -1.0], [1.0, 0.0, 0.0], [0.0, 1.0, 0.0], [0.0, 0.0, 1.0]])
        dN = np.broadcast_to(d, u.shape + (4, 3)).copy()
        return N, dN
    if kind == "wedge":
        L = [1.0 - u - v, u, v]
        dLu = [-np.ones_like(u), np.ones_like(u), np.zeros_like(u)]
        dLv = [-np.ones_like(u), np.zeros_like(u), np.ones_like(u)]
        bot, top = 0.5 * (1.0 - w), 0.5 * (1.0 + w)
        N = np.stack([L[i] * bot for i in range(3)] + [L[i] * top for i in range(3)], -1)
        rows = [np.stack([dLu[i] * bot, dLv[i] * bot, -0.5 * L[i]], -1) for i in range(3)]
        rows += [np.stack([dLu[i] * top, dLv[i] * top, 0.5 * L[i]], -1) for i in range(3)]
        return N, np.stack(rows, -2)
    if kind == "hex":
        s = np.asarray(REF_NODES["hex"], float)
        a = 1.0 + u[..., None] * s[:, 0]
        b = 1.0 + v[..., None] * s[:, 1]
        c = 1.0 + w[..., None] * s[:, 2]
        N = a * b * c / 8.0
        dN = np.stack([s[:, 0] * b * c, a * s[:, 1] * c, a * b * s[:, 2]], -1) / 8.0
        return N, dN
    if kind == "pyramid":
        s = np.asarray(REF_NODES["pyramid"], float)[:4]
        a = 1.0 + u[..., None] * s[:, 0]
        b = 1.0 + v[..., None] * s[:, 1]
        c = (1.0 - w)[..., None]
        base = a * b * c / 8.0
        dbase = np.stack([s[:, 0] * b * c, a * s[:, 1] * c, -a * b], -1) / 8.0
        N = np.concatenate([base, (0.5 * (1.0 + w))[..., None]], -1)
        apex = np.stack([np.zeros_like(u), np.zeros_like(u), np.full_like(u, 0.5)], -1)
        return N, np.concatenate([dbase, apex[..., None, :]], -2)
    raise ValueError(kind)


def _parameters_of(kind: str, x: np.ndarray) -> np.ndarray:
    """Parametric coordinates of points ``x`` given on the reference element.

    The identity except for the pyramid, whose collapsed map sends
    ``(xi, eta, zeta)`` to ``(xi (1 - zeta)/2, eta (1 - zeta)/2, zeta)``.
    """
    if kind != "pyramid":
        return np.array(x, float)
    z = x[:, 2]
    return np.stack([2.0 * x[:, 0] / (1.0 - z), 2.0 * x[:, 1] / (1.0 - z), z], 1)


@dataclass(frozen=True)
class ElementTables:
    """Constant tables of one element type.

    Dual points are numbered nodes ``0..n-1``, edge midpoints, face
    centroids, then the element centroid; ``weights[p]`` writes dual point
    ``p`` as a combination of the element's nodes.
    """

    kind: str
    n: int
    n_ip: int
    edge: np.ndarray          # (n_ip, 2) local nodes (a, b); the area points a -> b
    tris: np.ndarray          # (n_ip, 3) dual points of each flux point's triangle
    weights: np.ndarray       # (n_pts, n)
    xi_ip: np.ndarray         # (n_ip, 3)
    N_ip: np.ndarray          # (n_ip, n)
    dN_ip: np.ndarray         # (n_ip, n, 3)
    node_ips: np.ndarray      # (n, 8) flux points touching each node (-1 padded)
    node_sgn: np.ndarray      # (n, 8) +1 where the node is the edge's a side, -1 for b

    @property
    def n_pts(self) -> int:
        return self.weights.shape[0]

    @property
    def const_gradient(self) -> bool:
        """Linear shape functions: one gradient set per element (tetrahedra)."""
        return self.kind == "tet"

    @property
    def n_grad(self) -> int:
        return 1 if self.const_gradient else self.n_ip

    @property
    def record_doubles(self) -> int:
        """Doubles in a stored geometry record: flux-point areas and centroids, the inverse
        Jacobian of the element map at each flux point (one for tetrahedra), the
        sub-control volumes."""
        return 2 * self.n_ip * 3 + self.n_grad * 9 + self.n

    @property
    def corner_masks(self) -> np.ndarray:
        """``(n_ip, 3)`` bit masks of the element nodes whose mean is each corner of a flux
        point's triangle (edge midpoint, face centroid, element centroid)."""
        w = self.weights[self.tris]                              # (n_ip, 3, n)
        return ((w > 0) * (1 << np.arange(self.n))).sum(-1).astype(np.int64)


@lru_cache(maxsize=None)
def tables(kind: str) -> ElementTables:
    n = NODES_PER[kind]
    edges = np.asarray(EDGES[kind], np.int64)
    faces = FACES[kind]
    ne, nf = len(edges), len(faces)
    W = np.zeros((n + ne + nf + 1, n))
    W[np.arange(n), np.arange(n)] = 1.0
    for e, (a, b) in enumerate(edges):
        W[n + e, a] = W[n + e, b] = 0.5
    for f, nodes in enumerate(faces):
        W[n + ne + f, list(nodes)] = 1.0 / len(nodes)
    W[n + ne + nf] = 1.0 / n
    ref = W @ np.asarray(REF_NODES[kind], float)
    centre = n + ne + nf
    tris = np.zeros((2 * ne, 3), np.int64)
    for e, (a, b) in enumerate(edges):
        on = [f for f, nodes in enumerate(faces) if a in nodes and b in nodes]
        if len(on) != 2:
            raise AssertionError((kind, e, on))
        m, f1, f2 = n + e, n + ne + on[0], n + ne + on[1]
        area = 0.5 * np.cross(ref[centre] - ref[m], ref[f2] - ref[f1])
        if area @ (ref[b] - ref[a]) < 0:
            f1, f2 = f2, f1
        tris[2 * e] = (m, f1, centre)
        tris[2 * e + 1] = (m, centre, f2)
    edge_ip = np.repeat(edges, 2, axis=0)
    xi = _parameters_of(kind, ref[tris].mean(axis=1))
    N, dN = shape_functions(kind, xi)
    ips = -np.ones((n, MAX_IP_PER_NODE), np.int64)
    sgn = np.zeros((n, MAX_IP_PER_NODE))
    fill = np.zeros(n, np.int64)
    for s, (a, b) in enumerate(edge_ip):
        for node, sg in ((a, 1.0), (b, -1.0)):
            ips[node, fill[node]] = s
            sgn[node, fill[node]] = sg
            fill[node] += 1
    return ElementTables(kind, n, 2 * ne, edge_ip, tris, W, xi, N, dN, ips, sgn)


# ---------------------------------------------------------------- header generation

def _c_array(name: str, a: np.ndarray, ctype: str) -> str:
    a = np.asarray(a)
    if ctype == "double":
        body = ", ".join(repr(float(v)) for v in a.reshape(-1))
    else:
        body = ", ".join(str(int(v)) for v in a.reshape(-1))
    dims = "".join(f"[{d}]" for d in a.shape)
    return f"static __constant__ {ctype} {name}{dims} = {{{body}}};"


def _kernel_tables(t: ElementTables):
    """The tables as the element kernels index them: lanes of a warp take one flux point each,
    so every per-flux-point table has the flux point as its fastest index."""
    return (("EDGE", t.edge, "int"),                               # (n_ip, 2)
            ("MASK", t.corner_masks, "int"),                       # (n_ip, 3)
            ("NT", t.N_ip.T, "double"),                            # (n, n_ip)
            ("DNT", t.dN_ip.transpose(1, 2, 0).reshape(t.n * 3, t.n_ip), "double"),
            ("IPS", t.node_ips, "int"),                            # (n, MAXI)
            ("SGN", t.node_sgn, "int"))                            # (n, MAXI) +1 / -1 / 0


def header_source() -> str:
    """CUDA source of ``topology_tables.h``.

    Per type: the tables as ``__constant__`` arrays (``k<KIND>_<TABLE>``) and a ``Topo<K>``
    traits struct with the sizes as compile-time constants and pointers to its tables, so
    that kernels templated on the type size their staging and unroll their loops:
    ``EDGE`` the edge nodes of each flux point, ``MASK`` the nodes averaged into each corner
    of its triangle, ``NT[q][s]`` the shape function of node q at flux point s, ``DNT[q*3+d][s]``
    its derivative along parametric axis d, ``IPS``/``SGN`` the flux points at each node and
    the side the node is on (+1 the edge's first node, -1 its second).
    """
    out = ["// Generated by zvcfd_b200.topology.write_header(); do not edit.",
           "// Element tables of the median-dual discretisation (flux points, shape functions).",
           "#pragma once", "", "namespace zvfv {", "",
           "enum Kind { TET = 0, PYRAMID = 1, WEDGE = 2, HEX = 3 };",
           f"constexpr int MAXI = {MAX_IP_PER_NODE};", "",
           "template <int K> struct Topo;", ""]
    for kind in KINDS:
        t = tables(kind)
        K = kind.upper()
        for cname, arr, ctype in _kernel_tables(t):
            out.append(_c_array(f"k{K}_{cname}", arr, ctype))
        out.append(f"template <> struct Topo<{K}> {{")
        out.append(f"    static constexpr int N = {t.n};")
        out.append(f"    static constexpr int NIP = {t.n_ip};")
        out.append(f"    static constexpr int CONSTG = {int(t.const_gradient)};")
        out.append(f"    static constexpr int NG = {t.n_grad};")
        out.append(f"    static constexpr int REC = {t.record_doubles};")
        out.append(f"    static constexpr int MAXF = {int((t.node_ips >= 0).sum(1).max())};")
        out.append(f"    __device__ static const int (*edge())[2] {{ return k{K}_EDGE; }}")
        out.append(f"    __device__ static const int (*mask())[3] {{ return k{K}_MASK; }}")
        out.append(f"    __device__ static const double (*nt())[{t.n_ip}] {{ return k{K}_NT; }}")
        out.append(f"    __device__ static const double (*dnt())[{t.n_ip}] {{ return k{K}_DNT; }}")
        out.append(f"    __device__ static const int (*ips())[MAXI] {{ return k{K}_IPS; }}")
        out.append(f"    __device__ static const int (*sgn())[MAXI] {{ return k{K}_SGN; }}")
        out.append("};")
        out.append("")
    out.append("}  // namespace zvfv")
    return "\n".join(out) + "\n"


HEADER_PATH = Path(__file__).resolve().parent / "csrc" / "topology_tables.h"


def write_header(path: Path = HEADER_PATH) -> bool:
    """Write the tables header if it differs; returns whether it changed."""
    src = header_source()
    if path.exists() and path.read_text() == src:
        return False
    path.write_text(src)
    return True


__all__ = ["EDGES", "ElementTables", "FACES", "KINDS", "NODES_PER", "header_source",
           "shape_functions", "tables", "write_header"]
