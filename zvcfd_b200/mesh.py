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
    nodes: np.ndarray
    elements: dict
    zones: dict = field(default_factory=dict)

    def __post_init__(self):
        self.nodes = np.ascontiguousarray(self.nodes, np.float64)
        self.elements = {k: np.ascontiguousarray(self.elements[k], np.int64)
                         for k in KINDS if k in self.elements and len(self.elements[k])}

    @property
    def n_nodes(self) -> int:
        return len(self.nodes)

    @property
    def n_elements(self) -> int:
        return sum(len(e) for e in self.elements.values())

    def zone_id(self, name: str) -> int:
        for zid, z in self.zones.items():
            if z.name == name:
                return zid
        raise KeyError(name)

    def element_volumes(self, kind: str) -> np.ndarray:
        """Volume of each element, every face fanned about its centroid."""
        e = self.elements[kind]
        x = self.nodes[e]
        c = x.mean(1)
        vol = np.zeros(len(e))
        for f in FACES[kind]:
            p = x[:, list(f)]
            fc = p.mean(1)
            for i in range(len(f)):
                a, b = p[:, i], p[:, (i + 1) % len(f)]
                vol += np.einsum("ij,ij->i", np.cross(a - fc, b - fc), c - fc) / 6.0
        return -vol

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

# Dompierre et al. (1999), table 2: vertex permutations taking each vertex of a
# wedge to position 0 while keeping the wedge's topology (bottom 0 1 2, top 3 4 5)
_WEDGE_ROT = np.array([[0, 1, 2, 3, 4, 5], [1, 2, 0, 4, 5, 3], [2, 0, 1, 5, 3, 4],
                       [3, 5, 4, 0, 2, 1], [4, 3, 5, 1, 0, 2], [5, 4, 3, 2, 1, 0]])


def split_wedges(w: np.ndarray) -> np.ndarray:
    """Three tetrahedra per wedge, conforming by the smallest-global-index rule."""
    w = np.asarray(w, np.int64)
    p = w[np.arange(len(w))[:, None], _WEDGE_ROT[np.argmin(w, axis=1)]]
    v = [p[:, i] for i in range(6)]
    # the quad (1, 2, 5, 4) opposite vertex 0 is cut through its smallest vertex
    cut15 = np.minimum(v[1], v[5]) < np.minimum(v[2], v[4])
    t = np.empty((len(w), 3, 4), np.int64)
    t[:, 0] = np.where(cut15[:, None], np.stack([v[0], v[1], v[2], v[5]], 1),
                       np.stack([v[0], v[1], v[2], v[4]], 1))
    t[:, 1] = np.where(cut15[:, None], np.stack([v[0], v[1], v[5], v[4]], 1),
                       np.stack([v[0], v[4], v[2], v[5]], 1))
    t[:, 2] = np.stack([v[0], v[4], v[5], v[3]], 1)
    return t.reshape(-1, 4)


def split_hexes(h: np.ndarray) -> np.ndarray:
    """Two wedges per hexahedron (triangles on faces 0-3 and 4-7), both cut along the
    diagonal through the bottom quad's smallest node. Columns of hexahedra numbered
    the same way layer after layer therefore stay conforming."""
    h = np.asarray(h, np.int64)
    b = h[:, :4]
    diag13 = np.argmin(np.minimum(b[:, [0, 1, 2, 3]], b[:, [2, 3, 0, 1]]), axis=1) % 2
    sel = np.where(diag13[:, None] == 0, np.array([[0, 1, 2, 0, 2, 3]]),
                   np.array([[0, 1, 3, 1, 2, 3]]))
    r = np.arange(len(h))[:, None]
    bot, top = b[r, sel], h[:, 4:][r, sel]
    w1 = np.concatenate([bot[:, :3], top[:, :3]], 1)
    w2 = np.concatenate([bot[:, 3:], top[:, 3:]], 1)
    return np.stack([w1, w2], 1).reshape(-1, 6)


def orient(nodes: np.ndarray, kind: str, e: np.ndarray) -> np.ndarray:
    """Reorder each element's local nodes so that its volume is positive."""
    e = np.array(e, np.int64)
    x = nodes[e]
    if kind in ("tet", "wedge"):
        s = np.einsum("ij,ij->i", np.cross(x[:, 1] - x[:, 0], x[:, 2] - x[:, 0]),
                      x[:, 3] - x[:, 0])
        perm = [0, 2, 1, 3] if kind == "tet" else [0, 2, 1, 3, 5, 4]
    elif kind == "hex":
        s = np.einsum("ij,ij->i", np.cross(x[:, 1] - x[:, 0], x[:, 3] - x[:, 0]),
                      x[:, 4] - x[:, 0])
        perm = [0, 3, 2, 1, 4, 7, 6, 5]
    else:
        return e
    e[s < 0] = e[s < 0][:, perm]
    return e


def _zones(mesh: Mesh, classify, names) -> dict:
    f = mesh.boundary_faces()
    p = mesh.nodes[np.where(f < 0, f[:, :1], f)]
    tri = f[:, 3] < 0
    c = np.where(tri[:, None], p[:, :3].mean(1), p.mean(1))
    nrm = np.where(tri[:, None], np.cross(p[:, 1] - p[:, 0], p[:, 2] - p[:, 0]),
                   np.cross(p[:, 2] - p[:, 0], p[:, 3] - p[:, 1]))
    nrm /= np.linalg.norm(nrm, axis=1, keepdims=True)
    which = classify(c, nrm)
    zones = {}
    for i, (name, kind) in enumerate(names):
        zones[3 + i] = Zone(3 + i, kind, name, f[which == i])
    if sum(z.n_faces for z in zones.values()) != len(f):
        raise ValueError("unclassified boundary faces")
    return zones


def jitter(mesh: Mesh, amount: float, seed: int) -> None:
    """Move interior nodes at random by up to ``amount`` times their shortest edge."""
    if not amount:
        return
    rng = np.random.default_rng(seed)
    bnd = np.zeros(mesh.n_nodes, bool)
    for z in mesh.zones.values():
        bnd[z.faces[z.faces >= 0]] = True
    h = np.full(mesh.n_nodes, np.inf)
    for kind, e in mesh.elements.items():
        from zvcfd_b200.topology import EDGES
        for a, b in EDGES[kind]:
            ln = np.linalg.norm(mesh.nodes[e[:, b]] - mesh.nodes[e[:, a]], axis=1)
            np.minimum.at(h, e[:, a], ln)
            np.minimum.at(h, e[:, b], ln)
    d = rng.uniform(-1.0, 1.0, (mesh.n_nodes, 3)) * (amount * h)[:, None]
    d[bnd] = 0.0
    mesh.nodes = mesh.nodes + d
    for k in mesh.elements:
        if (mesh.element_volumes(k) <= 0).any():
            raise ValueError("the jitter inverted an element; use a smaller amount")


# ---------------------------------------------------------------- generators

def box(n=(4, 4, 4), lengths=(1.0, 1.0, 1.0), *, kind: str = "hex", perturb: float = 0.0,
        seed: int = 0) -> Mesh:
    """A structured box; zones 3-8 ``xmin xmax ymin ymax zmin zmax`` (walls)."""
    nx, ny, nz = n
    xs = [np.linspace(0.0, L, k + 1) for L, k in zip(lengths, n)]
    X, Y, Z = np.meshgrid(*xs, indexing="ij")
    nodes = np.stack([X.ravel(), Y.ravel(), Z.ravel()], 1)
    idx = np.arange(len(nodes)).reshape(nx + 1, ny + 1, nz + 1)
    i, j, k = (a.ravel() for a in np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz),
                                              indexing="ij"))
    hexes = np.stack([idx[i, j, k], idx[i + 1, j, k], idx[i + 1, j + 1, k], idx[i, j + 1, k],
                      idx[i, j, k + 1], idx[i + 1, j, k + 1], idx[i + 1, j + 1, k + 1],
                      idx[i, j + 1, k + 1]], 1)
    els = {"hex": hexes} if kind == "hex" else {"wedge": split_hexes(hexes)} \
        if kind == "wedge" else {"tet": split_wedges(split_hexes(hexes))}
    mesh = Mesh(nodes, {k: orient(nodes, k, v) for k, v in els.items()})
    tol = 1e-9 * max(lengths)

    def classify(c, nrm):
        w = np.full(len(c), -1)
        for s, (ax, side) in enumerate([(0, 0), (0, 1), (1, 0), (1, 1), (2, 0), (2, 1)]):
            w[np.abs(c[:, ax] - side * lengths[ax]) < tol] = s
        return w

    mesh.zones = _zones(mesh, classify, [(nm, "wall") for nm in
                                         ("xmin", "xmax", "ymin", "ymax", "zmin", "zmax")])
    jitter(mesh, perturb, seed)
    return mesh


def ogrid_section(radius: float, n_core: int, n_ring: int, *, core: float = 0.5,
                  growth: float = 1.0):
    """Cross-section of a circle: a square core and four blocks out to the wall.

    Returns ``(xy (P, 2), quads (Q, 4), layer (Q,))``, ``layer`` the quad's
    radial layer counted from the wall (0 = at the wall), -1 in the core.
    Each outer block's radial cells grow by ``growth`` from the core outward
    (``growth < 1`` makes the wall cells thinnest).
    """
    half = core * radius / np.sqrt(2.0)
    t = np.linspace(-1.0, 1.0, n_core + 1)
    w = growth ** np.arange(n_ring)
    frac = np.r_[0.0, np.cumsum(w) / w.sum()]
    pts, quads, layer = [], [], []
    gx, gy = np.meshgrid(t, t, indexing="ij")
    pts.append(np.stack([half * gx.ravel(), half * gy.ravel()], 1))
    ci = np.arange((n_core + 1) ** 2).reshape(n_core + 1, n_core + 1)
    a, b = (v.ravel() for v in np.meshgrid(np.arange(n_core), np.arange(n_core), indexing="ij"))
    quads.append(np.stack([ci[a, b], ci[a + 1, b], ci[a + 1, b + 1], ci[a, b + 1]], 1))
    layer.append(np.full(len(a), -1))
    base = (n_core + 1) ** 2
    for q in range(4):
        c, s = np.cos(q * np.pi / 2), np.sin(q * np.pi / 2)
        rot = np.array([[c, -s], [s, c]])
        side = np.stack([np.full_like(t, half), half * t], 1)
        ang = t * np.pi / 4
        arc = radius * np.stack([np.cos(ang), np.sin(ang)], 1)
        blk = (1.0 - frac[:, None, None]) * side[None] + frac[:, None, None] * arc[None]
        pts.append(blk.reshape(-1, 2) @ rot.T)
        bi = base + np.arange((n_ring + 1) * (n_core + 1)).reshape(n_ring + 1, n_core + 1)
        a, b = (v.ravel() for v in np.meshgrid(np.arange(n_ring), np.arange(n_core),
                                               indexing="ij"))
        quads.append(np.stack([bi[a, b], bi[a + 1, b], bi[a + 1, b + 1], bi[a, b + 1]], 1))
        layer.append(n_ring - 1 - a)
        base += bi.size
    xy = np.concatenate(pts)
    quads = np.concatenate(quads)
    layer = np.concatenate(layer)
    # merge the nodes the blocks share, keeping first occurrences in order
    key = np.round(xy / (radius * 1e-9)).astype(np.int64)
    _, first, inv = np.unique(key, axis=0, return_index=True, return_inverse=True)
    inv = inv.reshape(-1)
    renum = np.empty(len(first), np.int64)
    renum[np.argsort(first)] = np.arange(len(first))
    return xy[np.sort(first)], renum[inv[quads]], layer


def pipe(radius: float = 1e-3, length: float = 10e-3, *, n_core: int = 14, n_ring: int = 7,
         n_axial: int = 80, kind: str = "tet", growth: float = 1.0, jitter_amount: float = 0.0,
         seed: int = 0) -> Mesh:
    """A straight circular pipe along z. Zones: 3 ``inlet`` (z = 0), 4 ``outlet``
    (z = length), 5 ``wall``. ``kind``: ``"tet"`` (six per hexahedron) or ``"hex"``."""
    xy, quads, _ = ogrid_section(radius, n_core, n_ring, growth=growth)
    P = len(xy)
    z = np.linspace(0.0, length, n_axial + 1)
    nodes = np.concatenate([np.column_stack([xy, np.full(P, zk)]) for zk in z])
    k = np.arange(n_axial)[:, None, None] * P
    hexes = np.concatenate([quads[None] + k, quads[None] + k + P], axis=2).reshape(-1, 8)
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
    P = len(xy)
    th = np.linspace(0.0, angle, n_axial + 1)
    rows = []
    for t in th:
        ctr = np.array([bend * (1.0 - np.cos(t)), 0.0, bend * np.sin(t)])
        ex = np.array([np.cos(t), 0.0, -np.sin(t)])
        rows.append(ctr[None] + xy[:, :1] * ex[None] + xy[:, 1:2] * np.array([[0.0, 1.0, 0.0]]))
    nodes = np.concatenate(rows)
    k = np.arange(n_axial)[:, None, None] * P
    hexes = np.concatenate([quads[None] + k, quads[None] + k + P], axis=2)
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
