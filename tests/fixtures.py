"""Loading the golden vectors (``tests/golden/*.npz``) into meshes and solver inputs."""

from __future__ import annotations

from pathlib import Path

import numpy as np

from zvcfd_b200.mesh import Mesh, Zone
from zvcfd_b200.topology import KINDS

GOLDEN = Path(__file__).resolve().parent / "golden"
KERNEL_MESHES = ("tet", "pyramid", "wedge", "hex", "mixed", "delaunay")
KERNEL_VARIANTS = ("newt_steady", "gn_dt")


def load(name: str) -> dict:
    with np.load(GOLDEN / f"{name}.npz") as z:
        return {k: z[k] for k in z.files}


def mesh_of(g: dict) -> Mesh:
    els = {k: g[f"elem_{k}"] for k in KINDS if f"elem_{k}" in g}
    m = Mesh(g["nodes"], els)
    for zid, name in zip(g["zone_ids"], g["zone_names"]):
        m.zones[int(zid)] = Zone(int(zid), "", str(name), g[f"zone_{int(zid)}"])
    return m


def kernel_case(mesh_name: str, variant: str) -> dict:
    return load(f"kernel_{mesh_name}_{variant}")


def mdot_of(g: dict, prefix: str = "mdot") -> dict:
    return {k: g[f"{prefix}_{k}"] for k in KINDS if f"{prefix}_{k}" in g}


def fluid_of(g: dict):
    from zvcfd_b200.fluid import CarreauYasuda, Fluid

    cy = None
    if int(g.get("gn", 0)) or "cy" in g and "flow_rate" in g:
        c = g["cy"]
        cy = CarreauYasuda(float(c[0]), float(c[1]), float(c[2]), float(c[3]), float(c[4]))
    return Fluid(float(g["rho"]), float(g["mu"]), viscosity=cy)


def oracle_for_kernel_case(g: dict):
    """The oracle set up as the reference was when the kernel golden case was made."""
    from oracle.fv import OracleSolver

    m = mesh_of(g)
    gn = bool(int(g["gn"]))
    dt = float(g["dt"]) or None
    s = OracleSolver(m, fluid_of(g), {z: {"kind": "wall"} for z in m.zones},
                     advection="high-resolution", dt=dt, transpose=gn)
    s.U, s.P = g["U"].copy(), g["P"].copy()
    for K in s.kinds:
        K.mdot = g[f"mdot_{K.kind}"].copy()
    return s


def oracle_kernel_outputs(g: dict) -> dict:
    """Everything the kernel golden case pins, computed by the oracle."""
    s = oracle_for_kernel_case(g)
    rho = float(g["rho"])
    dt = float(g["dt"]) or None
    gradU, gradP = s.nodal_gradient(s.U), s.nodal_gradient(s.P)
    mdot = {K.kind: K.mdot.copy() for K in s.kinds}
    diag = s.momentum_diagonal()
    tdiag = rho * s.V / dt if dt else 0.0
    dnode, snode = s.V / (diag + tdiag), s.V / diag
    levels = [(1.0, s.U.copy(), mdot)] if dt else []
    data, b = s.assemble_elements(s.U, mdot, gradU, g["beta_frozen"], gradP, dnode, snode,
                                  levels)
    new, imb = s.mass_flows(g["U_new"], g["P_new"], s.nodal_gradient(g["P_new"]), dnode, snode,
                            [(1.0, g["U"], mdot)] if dt else [])
    return {"V": s.V, "gradU": gradU, "gradP": gradP, "diag": diag,
            "beta_limiter": s.limiter(gradU), "indptr": s.indptr, "indices": s.indices,
            "data_raw": data, "b_raw": b, "imbalance": imb, "mdot_new": new,
            "dnode": dnode, "snode": snode, "solver": s}


def axial_parabola(radius: float, peak: float = 1.0, pulse=None):
    """``u(x)`` (or ``u(x, t)`` with ``pulse(t)``): velocity along +z, ``peak (1 - r^2/R^2)``
    inside the radius and zero outside, ``r`` the distance from the z axis."""
    def shape(x):
        r2 = np.einsum("ij,ij->i", x[:, :2], x[:, :2]) / radius ** 2
        u = np.zeros((len(x), 3))
        u[:, 2] = peak * np.maximum(1.0 - r2, 0.0)
        return u

    if pulse is None:
        return shape
    return lambda x, t: pulse(t) * shape(x)


def _pipe_zones(m, inlet: dict) -> dict:
    z = {zz.name: k for k, zz in m.zones.items()}
    return {z["inlet"]: inlet, z["outlet"]: {"kind": "pressure", "value": 0.0},
            z["wall"]: {"kind": "wall"}}


def pipe_bcs(name: str, g: dict, m):
    """The boundary conditions the golden pipe case was solved with."""
    if name in ("pipe_reference_tube", "pipe_tet_si"):
        inlet = {"kind": "velocity", "value": axial_parabola(float(g["radius"]), float(g["umax"]))}
    else:
        profile = axial_parabola(2e-3)
        inlet = {"kind": "velocity", "flow_rate": float(g["flow_rate"]),
                 "profile": lambda x: profile(x)[:, 2]}
    return _pipe_zones(m, inlet)


PIPES = ("pipe_reference_tube", "pipe_tet_si", "curved_cy")


def transient_bcs(g: dict, m):
    pulse = axial_parabola(float(g["radius"]), float(g["umax"]),
                           pulse=lambda t: 1.0 + 0.5 * np.sin(2 * np.pi * t / 0.8))
    return _pipe_zones(m, {"kind": "velocity", "value": pulse})


def backflow_bcs(m, beta: float) -> dict:
    """The backflow box's conditions (``tests/test_fv_boundaries.py:182-207`` of the reference):
    walls, a uniform inflow at xmin, and at xmax a pressure ``1.5 cos(pi y)`` that pulls fluid
    back in over part of the outlet, stabilised by ``beta``."""
    z = {zz.name: k for k, zz in m.zones.items()}
    bcs = {k: {"kind": "wall"} for k in m.zones}
    bcs[z["xmin"]] = {"kind": "velocity", "value": (1.0, 0.0, 0.0)}
    bcs[z["xmax"]] = {"kind": "pressure", "value": lambda x: 1.5 * np.cos(np.pi * x[:, 1]),
                      "backflow_stabilisation": beta}
    return bcs


def forces_case(g: dict, tag: str):
    """A zone-force golden case: its mesh and boundary conditions, rebuilt from the arrays."""
    sub = {k[len(tag) + 1:]: v for k, v in g.items() if k.startswith(tag + "_")}
    m = mesh_of(sub)
    z = {zz.name: k for k, zz in m.zones.items()}
    if tag == "pipe":
        bcs = _pipe_zones(m, {"kind": "velocity", "value": axial_parabola(0.5, 2.0)})
    else:
        bcs = {z["xmin"]: {"kind": "velocity", "value": [1.0, 0.0, 0.0]},
               z["xmax"]: {"kind": "pressure", "value": 0.0},
               z["ymax"]: {"kind": "pressure", "value": 0.0},
               z["ymin"]: {"kind": "wall"}, z["zmin"]: {"kind": "symmetry"},
               z["zmax"]: {"kind": "symmetry"}}
    return m, bcs, sub


def tabulated(points: np.ndarray, values: np.ndarray):
    """``f(x)`` that returns the tabulated value at each of the points ``x`` (each must be one
    of ``points`` up to round-off): boundary data recorded where the reference evaluated it."""
    from scipy.spatial import cKDTree

    tree = cKDTree(points)
    scale = float(np.abs(points).max())

    def f(x):
        d, i = tree.query(np.asarray(x, float))
        if np.any(d > 1e-12 * scale):
            raise KeyError("a point the table does not hold")
        return values[i]

    return f


def gn_outlet_bcs(g: dict, m) -> dict:
    """The manufactured Carreau-Yasuda outlet case's conditions, from its tables."""
    z = {zz.name: k for k, zz in m.zones.items()}
    u, p, J = (tabulated(g["points"], g[k]) for k in ("u", "p", "J"))
    bcs = {k: {"kind": "velocity", "value": u} for k in m.zones}
    bcs[z["xmax"]] = {"kind": "pressure", "value": p, "grad": J}
    return bcs


def gn_outlet_fluid(g: dict):
    from zvcfd_b200.fluid import CarreauYasuda, Fluid

    return Fluid(float(g["rho"]), float(g["mu"]),
                 viscosity=CarreauYasuda(*[float(v) for v in g["cy"]]))
