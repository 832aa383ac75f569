"""Unstructured meshes (nodes, elements by type, boundary zones) and synthetic vessel meshes.

The container follows the reference's mesh conventions
(``zvcfd/mesh/core.py:1-30``): coordinates ``(N, 3)`` float64, elements
``{kind: (E, n) int64}`` in VTK local order with positive volume, and
boundary zones whose faces ``(F, 4)`` (``-1`` pads a triangle) point out of
the fluid. Zone ids start at 3, as the reference's generators number them.

Generators (all seeded, all conforming):

- :func:`box`: a structured box of hexahedra, wedges or tetrahedra (test cases);
- :func:`pipe`: a straight circular pipe on a five-block O-grid, in
  tetrahedra (each hexahedron cut into six) or hexahedra, with an optional
  seeded jitter of the interior nodes (the plain FP64 Poiseuille pipe);
- :func:`curved_tube`: a tube swept along a circular arc, hexahedral core and
  wedge wall layers, graded toward the wall (the curved Carreau-Yasuda tube).

Hexahedra are split conformingly by the smallest-global-index rule of
Dompierre, Labbe, Vallet and Camarero (Proc. 8th International Meshing
Roundtable, 1999): every shared quadrilateral is cut along the diagonal
through its smallest-index node, so neighbours agree without bookkeeping.
"""

from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from zvcfd_b200.topology import FACES, KINDS


@dataclass
class Zone:
    """One boundary zone: ``faces (F, 4)`` node indices, outward, ``-1`` padding triangles."""

    zone: int
    kind: str
    name: str
    faces: np.ndarray

    @property
    def n_faces(self) -> int:
        return len(self.faces)


@dataclass
class Mesh:
    """Nodes ``(N, 3)``, elements ``{kind: (E, n)}`` and boundary zones ``{id: Zone}``."""

    nodes: np.ndarray
    elements: dict
    zones: dict = field(default_factory=dict)

    def __post_init__(self):
        self.nodes = np.require(self.nodes, np.float64, "C")
        kept = {}
        for kind in KINDS:                       # canonical order, empty types dropped
            e = self.elements.get(kind)
            if e is not None and len(e):
                kept[kind] = np.require(e, np.int64, "C")
        self.elements = kept

    @property
    def n_nodes(self) -> int:
        return self.nodes.shape[0]

    @property
    def n_elements(self) -> int:
        return int(sum(e.shape[0] for e in self.elements.values()))

    def zone_id(self, name: str) -> int:
        found = [zid for zid, z in self.zones.items() if z.name == name]
        if not found:
            raise KeyError(name)
        return found[0]

    def element_volumes(self, kind: str) -> np.ndarray:
        """Volume of each element: the tetrahedra joining the element's centroid to every
        face, each face fanned about its own centroid (outward faces give negative signed
        volumes, hence the sign)."""
        x = self.nodes[self.elements[kind]]
        centre = x.mean(1)
        vol = np.zeros(len(x))
        for face in FACES[kind]:
            ring = x[:, list(face)]
            mid = ring.mean(1)
            for a, b in zip(ring.transpose(1, 0, 2), np.roll(ring, -1, axis=1).transpose(1, 0, 2)):
                vol -= np.einsum("ij,ij->i", np.cross(a - mid, b - mid), centre - mid) / 6.0
        return vol

    def boundary_faces(self) -> np.ndarray:
        """Faces ``(F, 4)`` that belong to one element only, outward."""
        keys, faces = [], []
        for kind, e in self.elements.items():
            for f in FACES[kind]:
                loc = e[:, list(f)]
                if len(f) == 3:
                    loc = np.concatenate([loc, -np.ones((len(e), 1), np.int64)], 1)
                faces.append(loc)
                k = np.sort(loc, axis=1)
                keys.append(k)
        keys = np.concatenate(keys) + 1                 # -1 padding -> 0
        faces = np.concatenate(faces)
        # two int64 keys per face (pairs of sorted node ids, each pair < (N + 1)^2) sorted
        # together: a face is shared when its neighbour in that order has the same pair
        base = np.int64(self.n_nodes + 1)
        hi = keys[:, 0] * base + keys[:, 1]
        lo = keys[:, 2] * base + keys[:, 3]
        order = np.lexsort((lo, hi))
        h, l_ = hi[order], lo[order]
        same = (h[1:] == h[:-1]) & (l_[1:] == l_[:-1])
        shared = np.zeros(len(order), bool)
        shared[1:] |= same
        shared[:-1] |= same
        single = np.empty(len(order), bool)
        single[order] = ~shared
        return faces[single]


# ---------------------------------------------------------------- splitting

def _wedge_symmetries() -> np.ndarray:
    """Row ``v``: the relabelling of a wedge (triangle 0 1 2 under triangle 3 4 5) that brings
    local vertex ``v`` to position 0 and keeps the element's orientation: a rotation of both
    triangles, for a top vertex with the triangles exchanged and their direction reversed
    (the vertex permutations of Dompierre et al. 1999, table 2)."""
    rows = []
    for v in range(6):
        r = v % 3
        if v < 3:
            tri = [r, (r + 1) % 3, (r + 2) % 3]
            rows.append(tri + [3 + i for i in tri])
        else:
            tri = [r, (r + 2) % 3, (r + 1) % 3]
            rows.append([3 + i for i in tri] + tri)
    return np.array(rows)


_WEDGE_SYM = _wedge_symmetries()
# the three tetrahedra of a wedge relabelled so that vertex 0 holds its smallest index, for
# either diagonal of the quadrilateral 1-2-5-4 opposite that vertex
_TETS_CUT_15 = np.array([[0, 1, 2, 5], [0, 1, 5, 4], [0, 4, 5, 3]])
_TETS_CUT_24 = np.array([[0, 1, 2, 4], [0, 4, 2, 5], [0, 4, 5, 3]])


def split_wedges(w: np.ndarray) -> np.ndarray:
    """Three tetrahedra per wedge, conforming: each quadrilateral is cut along the diagonal
    through its smallest global index, so the two elements sharing it cut it alike."""
    w = np.asarray(w, np.int64)
    rows = np.arange(len(w))[:, None]
    lab = w[rows, _WEDGE_SYM[np.argmin(w, axis=1)]]
    cut15 = np.minimum(lab[:, 1], lab[:, 5]) < np.minimum(lab[:, 2], lab[:, 4])
    local = np.where(cut15[:, None, None], _TETS_CUT_15, _TETS_CUT_24)
    return lab[rows[:, :, None], local].reshape(-1, 4)


def split_hexes(h: np.ndarray) -> np.ndarray:
    """Two wedges per hexahedron with their triangles on faces 0-1-2-3 and 4-5-6-7, both cut
    along the diagonal through the bottom quadrilateral's smallest node. Columns of
    hexahedra numbered the same way layer after layer therefore stay conforming."""
    h = np.asarray(h, np.int64)
    through13 = np.argmin(h[:, :4], axis=1) % 2 == 1
    halves = np.where(through13[:, None, None], np.array([[0, 1, 3], [1, 2, 3]]),
                      np.array([[0, 1, 2], [0, 2, 3]]))
    rows = np.arange(len(h))[:, None, None]
    return np.concatenate([h[rows, halves], h[rows, halves + 4]], axis=2).reshape(-1, 6)


# per kind: the three edges from local node 0 whose triple product is the volume's sign, and
# the mirror relabelling that reverses it
_ORIENTATION = {"tet": ([1, 2, 3], [0, 2, 1, 3]), "wedge": ([1, 2, 3], [0, 2, 1, 3, 5, 4]),
                "hex": ([1, 3, 4], [0, 3, 2, 1, 4, 7, 6, 5])}


def orient(nodes: np.ndarray, kind: str, e: np.ndarray) -> np.ndarray:
    """Reorder each element's local nodes so that its volume is positive."""
    e = np.array(e, np.int64)
    if kind not in _ORIENTATION:
        return e
    edges, mirror = _ORIENTATION[kind]
    x = nodes[e]
    d = x[:, edges] - x[:, :1]
    neg = np.einsum("ij,ij->i", d[:, 0], np.cross(d[:, 1], d[:, 2])) < 0
    e[neg] = e[neg][:, mirror]
    return e


def _zones(mesh: Mesh, classify, names) -> dict:
    """Zones 3, 4, ... named ``names[i] = (name, kind)``: the boundary faces ``classify``
    (from their centroids and unit normals) assigns to ``i``; every face must be assigned."""
    f = mesh.boundary_faces()
    quad = f[:, 3] >= 0
    P = mesh.nodes[np.where(f >= 0, f, f[:, :1])]
    centre = np.where(quad[:, None], P.mean(1), P[:, :3].mean(1))
    # twice the polygon's area vector, about its centroid: a triangle's pad repeats vertex 0,
    # which closes its loop and adds nothing
    rel = P - centre[:, None]
    area = np.cross(rel, np.roll(rel, -1, axis=1)).sum(1)
    normal = area / np.linalg.norm(area, axis=1, keepdims=True)
    which = classify(centre, normal)
    if np.any(which < 0) or np.any(which >= len(names)):
        raise ValueError("unclassified boundary faces")
    return {3 + i: Zone(3 + i, kind, name, f[which == i]) for i, (name, kind) in enumerate(names)}


def jitter(mesh: Mesh, amount: float, seed: int) -> None:
    """Move interior nodes at random by up to ``amount`` times their shortest edge."""
    if not amount:
        return
    from zvcfd_b200.topology import EDGES

    rng = np.random.default_rng(seed)
    fixed = np.zeros(mesh.n_nodes, bool)
    for z in mesh.zones.values():
        fixed[z.faces[z.faces >= 0]] = True
    shortest = np.full(mesh.n_nodes, np.inf)
    for kind, e in mesh.elements.items():
        for a, b in EDGES[kind]:
            length = np.linalg.norm(mesh.nodes[e[:, b]] - mesh.nodes[e[:, a]], axis=1)
            np.minimum.at(shortest, e[:, a], length)
            np.minimum.at(shortest, e[:, b], length)
    move = rng.uniform(-1.0, 1.0, (mesh.n_nodes, 3)) * (amount * shortest)[:, None]
    move[fixed] = 0.0
    mesh.nodes = mesh.nodes + move
    if any((mesh.element_volumes(k) <= 0).any() for k in mesh.elements):
        raise ValueError("the jitter inverted an element; use a smaller amount")


# ---------------------------------------------------------------- generators

# VTK corner order of a hexahedral lattice cell, as offsets (i, j, k)
_CELL_CORNERS = np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0],
                          [0, 0, 1], [1, 0, 1], [1, 1, 1], [0, 1, 1]])


def box(n=(4, 4, 4), lengths=(1.0, 1.0, 1.0), *, kind: str = "hex", perturb: float = 0.0,
        seed: int = 0) -> Mesh:
    """A structured box; zones 3-8 ``xmin xmax ymin ymax zmin zmax`` (walls)."""
    n = np.asarray(n, np.int64)
    axes = [np.linspace(0.0, L, k + 1) for L, k in zip(lengths, n)]
    lattice = np.indices(n + 1).reshape(3, -1).T            # (i, j, k), k fastest
    nodes = np.stack([axes[d][lattice[:, d]] for d in range(3)], 1)
    cells = np.indices(n).reshape(3, -1).T
    c = cells[:, None, :] + _CELL_CORNERS[None]
    hexes = (c[..., 0] * (n[1] + 1) + c[..., 1]) * (n[2] + 1) + c[..., 2]
    if kind == "hex":
        els = {"hex": hexes}
    elif kind == "wedge":
        els = {"wedge": split_hexes(hexes)}
    else:
        els = {"tet": split_wedges(split_hexes(hexes))}
    mesh = Mesh(nodes, {k: orient(nodes, k, v) for k, v in els.items()})
    tol = 1e-9 * max(lengths)
    planes = [(ax, side * lengths[ax]) for ax in range(3) for side in (0, 1)]

    def classify(centre, normal):
        w = np.full(len(centre), -1)
        for i, (ax, at) in enumerate(planes):
            w[np.abs(centre[:, ax] - at) < tol] = i
        return w

    mesh.zones = _zones(mesh, classify, [(nm, "wall") for nm in
                                         ("xmin", "xmax", "ymin", "ymax", "zmin", "zmax")])
    jitter(mesh, perturb, seed)
    return mesh


def _grid_quads(first: int, rows: int, cols: int) -> np.ndarray:
    """The quadrilaterals of a ``rows x cols`` cell grid whose ``(rows + 1) x (cols + 1)``
    nodes are numbered row by row from ``first``: corners (r, c), (r+1, c), (r+1, c+1),
    (r, c+1)."""
    r, c = (v.reshape(-1) for v in np.indices((rows, cols)))
    at = lambda rr, cc: first + rr * (cols + 1) + cc            # noqa: E731
    return np.stack([at(r, c), at(r + 1, c), at(r + 1, c + 1), at(r, c + 1)], 1)


def ogrid_section(radius: float, n_core: int, n_ring: int, *, core: float = 0.5,
                  growth: float = 1.0):
    """Cross-section of a circle: a square core and four blocks out to the wall.

    Returns ``(xy (P, 2), quads (Q, 4), layer (Q,))``, ``layer`` the quad's
    radial layer counted from the wall (0 = at the wall), -1 in the core.
    Each outer block's radial cells grow by ``growth`` from the core outward
    (``growth < 1`` makes the wall cells thinnest).
    """
    half = core * radius / np.sqrt(2.0)          # half the side of the core square
    s = np.linspace(-1.0, 1.0, n_core + 1)       # position along a side, or along an arc
    cell = growth ** np.arange(n_ring)
    frac = np.r_[0.0, np.cumsum(cell) / cell.sum()]
    xs, ys = np.meshgrid(half * s, half * s, indexing="ij")
    pts = [np.stack([xs.reshape(-1), ys.reshape(-1)], 1)]
    quads = [_grid_quads(0, n_core, n_core)]
    layer = [np.full(n_core * n_core, -1)]
    first = len(pts[0])
    # block q: from the core side x = half to the arc of +-45 degrees about the +x axis,
    # turned by q right angles
    inner = np.stack([np.full(n_core + 1, half), half * s], 1)
    outer = radius * np.stack([np.cos(s * np.pi / 4), np.sin(s * np.pi / 4)], 1)
    block = (1.0 - frac)[:, None, None] * inner[None] + frac[:, None, None] * outer[None]
    for q in range(4):
        c, sn = np.cos(q * np.pi / 2), np.sin(q * np.pi / 2)
        turn = np.array([[c, -sn], [sn, c]])
        pts.append(block.reshape(-1, 2) @ turn.T)
        quads.append(_grid_quads(first, n_ring, n_core))
        layer.append(np.repeat(n_ring - 1 - np.arange(n_ring), n_core))
        first += (n_ring + 1) * (n_core + 1)
    xy, quads, layer = np.concatenate(pts), np.concatenate(quads), np.concatenate(layer)
    # merge the nodes two blocks share, numbered in order of first appearance
    keys = np.round(xy / (radius * 1e-9)).astype(np.int64)
    number, new_id = {}, np.empty(len(xy), np.int64)
    for i, k in enumerate(map(tuple, keys)):
        new_id[i] = number.setdefault(k, len(number))
    kept = np.zeros(len(number), np.int64)
    kept[new_id[::-1]] = np.arange(len(xy))[::-1]                # first occurrence of each
    return xy[kept], new_id[quads], layer


def _sweep(quads: np.ndarray, per: int, n_axial: int) -> np.ndarray:
    """``(n_axial, Q, 8)``: the hexahedra between consecutive copies (``per`` nodes apart) of
    a section's quadrilaterals."""
    lower = quads[None] + (per * np.arange(n_axial))[:, None, None]
    return np.concatenate([lower, lower + per], axis=2)


def pipe(radius: float = 1e-3, length: float = 10e-3, *, n_core: int = 14, n_ring: int = 7,
         n_axial: int = 80, kind: str = "tet", growth: float = 1.0, jitter_amount: float = 0.0,
         seed: int = 0) -> Mesh:
    """A straight circular pipe along z. Zones: 3 ``inlet`` (z = 0), 4 ``outlet``
    (z = length), 5 ``wall``. ``kind``: ``"tet"`` (six per hexahedron) or ``"hex"``."""
    xy, quads, _ = ogrid_section(radius, n_core, n_ring, growth=growth)
    z = np.linspace(0.0, length, n_axial + 1)
    nodes = np.column_stack([np.tile(xy, (n_axial + 1, 1)), np.repeat(z, len(xy))])
    hexes = _sweep(quads, len(xy), n_axial).reshape(-1, 8)
    els = {"hex": hexes} if kind == "hex" else {"tet": split_wedges(split_hexes(hexes))}
    mesh = Mesh(nodes, {kk: orient(nodes, kk, v) for kk, v in els.items()})
    tol = 1e-9 * max(radius, length)

    def classify(c, nrm):
        w = np.full(len(c), 2)
        w[np.abs(c[:, 2]) < tol] = 0
        w[np.abs(c[:, 2] - length) < tol] = 1
        return w

    mesh.zones = _zones(mesh, classify, [("inlet", "velocity-inlet"),
                                         ("outlet", "pressure-outlet"), ("wall", "wall")])
    jitter(mesh, jitter_amount, seed)
    return mesh


def curved_tube(radius: float = 2e-3, bend: float = 20e-3, angle: float = np.pi / 2, *,
                n_core: int = 20, n_ring: int = 12, n_axial: int = 285, layers: int = 5,
                growth: float = 0.8, jitter_amount: float = 0.0, seed: int = 0) -> Mesh:
    """A tube swept along a circular arc of radius ``bend`` through ``angle``.

    The cross-section is the O-grid of :func:`ogrid_section`; its outer ``layers``
    rings are cut into triangles (wedges once swept: the prism wall layers) and the
    rest stays quadrilateral (the hexahedral core). The centreline starts at the
    origin along +z and bends toward +x about the axis through ``(bend, 0, 0)``.
    Zones: 3 ``inlet``, 4 ``outlet``, 5 ``wall``.
    """
    if bend <= radius:
        raise ValueError("the bend radius must exceed the tube radius")
    xy, quads, layer = ogrid_section(radius, n_core, n_ring, growth=growth)
    th = np.linspace(0.0, angle, n_axial + 1)
    rows = []
    for t in th:
        ctr = np.array([bend * (1.0 - np.cos(t)), 0.0, bend * np.sin(t)])
        ex = np.array([np.cos(t), 0.0, -np.sin(t)])
        rows.append(ctr[None] + xy[:, :1] * ex[None] + xy[:, 1:2] * np.array([[0.0, 1.0, 0.0]]))
    nodes = np.concatenate(rows)
    hexes = _sweep(quads, len(xy), n_axial)
    wall = (layer >= 0) & (layer < layers)
    els = {"hex": hexes[:, ~wall].reshape(-1, 8),
           "wedge": split_hexes(hexes[:, wall].reshape(-1, 8))}
    mesh = Mesh(nodes, {kk: orient(nodes, kk, v) for kk, v in els.items()})
    tol = 1e-9 * bend
    out_c = np.array([bend * (1.0 - np.cos(angle)), 0.0, bend * np.sin(angle)])
    out_t = np.array([np.sin(angle), 0.0, np.cos(angle)])

    def classify(c, nrm):
        w = np.full(len(c), 2)
        w[(np.abs(c[:, 2]) < tol) & (nrm[:, 2] < -0.999)] = 0
        w[(np.abs((c - out_c) @ out_t) < tol) & (nrm @ out_t > 0.999)] = 1
        return w

    mesh.zones = _zones(mesh, classify, [("inlet", "velocity-inlet"),
                                         ("outlet", "pressure-outlet"), ("wall", "wall")])
    jitter(mesh, jitter_amount, seed)
    return mesh


__all__ = ["Mesh", "Zone", "box", "curved_tube", "jitter", "ogrid_section", "orient", "pipe",
           "split_hexes", "split_wedges"]


def y_bifurcation(h: float = 0.25e-3, *, parent=(2e-3, 30e-3), daughters=((1.6e-3, 25e-3, 35.0),
                                                                      (1.4e-3, 25e-3, -35.0)),
                  jitter_amount: float = 0.0, seed: int = 0) -> Mesh:
    """A Y-bifurcation of seeded tetrahedra on a voxel lattice of spacing ``h``.

    The parent tube (radius, length) runs along +z and ends at the origin; each daughter
    (radius, length, angle in degrees in the x-z plane) starts there. Lattice cells whose
    centres lie inside a tube or the junction sphere are kept and cut into six tetrahedra
    each (conforming). The walls are stair-stepped at the lattice scale: a synthetic mesh
    with the sizes and coupling of a vessel, not a body-fitted one. Zones: 3 ``inlet``
    (the parent's end plane), 4 ``outlet1``, 5 ``outlet2`` (the daughters' end caps),
    6 ``wall``.
    """
    Rp, Lp = parent
    axes = [(np.array([0.0, 0.0, -Lp]), np.array([0.0, 0.0, 1.0]), Lp, Rp)]
    for R, L, ang in daughters:
        a = np.radians(ang)
        axes.append((np.zeros(3), np.array([np.sin(a), 0.0, np.cos(a)]), L, R))
    ends = [o + d * L for o, d, L, _ in axes[1:]]
    lo = np.minimum.reduce([np.array([-Rp, -Rp, -Lp])] + [e - max(R for *_, R in axes) for e in ends])
    hi = np.maximum.reduce([np.array([Rp, Rp, 0.0])] + [e + max(R for *_, R in axes) for e in ends])
    n = np.ceil((hi - lo) / h).astype(int)
    lo[2] = -Lp                                   # the inlet is a lattice plane
    n[2] = int(np.ceil((hi[2] - lo[2]) / h))

    def inside(p):
        ok = np.linalg.norm(p, axis=1) < Rp
        for o, d, L, R in axes:
            t = (p - o) @ d
            r = np.linalg.norm((p - o) - t[:, None] * d, axis=1)
            ok |= (t >= 0) & (t <= L) & (r < R)
        return ok

    ii, jj, kk = np.meshgrid(np.arange(n[0]), np.arange(n[1]), np.arange(n[2]), indexing="ij")
    cells = np.stack([ii.ravel(), jj.ravel(), kk.ravel()], 1)
    keep = cells[inside(lo + (cells + 0.5) * h)]
    # corner node ids on the (n+1)^3 lattice, renumbered densely in z-major order
    corners = np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0],
                        [0, 0, 1], [1, 0, 1], [1, 1, 1], [0, 1, 1]])
    lat = (keep[:, None, :] + corners[None]).reshape(-1, 3)
    key = (lat[:, 2] * (n[1] + 1) + lat[:, 1]) * (n[0] + 1) + lat[:, 0]
    ukey, inv = np.unique(key, return_inverse=True)
    hexes = inv.reshape(-1, 8)
    kz, rem = np.divmod(ukey, (n[1] + 1) * (n[0] + 1))
    ky, kx = np.divmod(rem, n[0] + 1)
    nodes = lo + np.stack([kx, ky, kz], 1) * h
    tets = split_wedges(split_hexes(hexes))
    mesh = Mesh(nodes, {"tet": orient(nodes, "tet", tets)})

    def classify(c, nrm):
        w = np.full(len(c), 3)
        w[np.abs(c[:, 2] + Lp) < 1e-9 * Lp] = 0
        for q, (o, d, L, R) in enumerate(axes[1:]):
            t = (c - o) @ d
            w[(w == 3) & (t > L - 0.75 * h) & (nrm @ d > 0.5)] = 1 + q
        return w

    mesh.zones = _zones(mesh, classify, [("inlet", "velocity-inlet"), ("outlet1", "pressure-outlet"),
                                         ("outlet2", "pressure-outlet"), ("wall", "wall")])
    jitter(mesh, jitter_amount, seed)
    return mesh
