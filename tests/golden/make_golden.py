"""Generate the golden vectors of the coupled FV path by running the reference itself.

Run once, in a container where the reference is importable, with ``ZVCFD_REFERENCE`` naming
the reference's source tree:

    PYTHONPATH=$ZVCFD_REFERENCE:. PYTHONDONTWRITEBYTECODE=1 python tests/golden/make_golden.py

It writes ``tests/golden/*.npz``: element tables, and for six distorted test
meshes (every element type) the reference's node volumes, nodal gradients,
momentum diagonal, limiter, raw assembled block system, pattern and new mass
flows on a seeded random state (the procedure of the reference's
``tests/test_fv_fast.py:98-159``), plus converged fields of three small pipes
solved by the reference's CPU solver with lagged Rhie-Chow; a pulsatile BDF2
pipe (``transient``); wall shear (``wall``); the 0-D RCR model, BDF
coefficients and Carreau-Yasuda viscosity (``lumped``); the backflow box with
and without stabilisation (``backflow``); zone forces, flows and both wall-shear
methods of two converged cases (``forces``); WSS time statistics (``wss``);
the manufactured Carreau-Yasuda outlet (``gn_outlet``); developed inlet
profiles and a pipe with the default flow-rate inlet (``profiles``); uneven BDF2 steps of
an oscillating pipe (``variable_steps``); a mid-size curved Carreau-Yasuda tube
(``curved_mid``, about 6k nodes, the bench tube's cross-section coarsened); Morton owners,
local meshes and halo plans of the reference's partitioner (``partition``); element colours of
the reference's device colouring ``gpu_colour`` run on the CPU (``colour``); the reference's ACM
levels, V-cycle and ACM-FGMRES solve on a system its CPU solver assembled (``acm``); its
device boundary pass run on the CPU (``boundary``); its whole device solver run on the CPU for
the RCR outlet, the average-pressure outlet and the opening (``gpu_path``), and for BDF2 steps
of the RCR outlet (``gpu_path_transient``); the CPU solver's second-order boundary
reconstruction (``reconstruction``). A single file is
rewritten by naming it (``python tests/golden/make_golden.py forces``). Nothing
at test or bench time reads the reference: the tests read these files.
"""

from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
import os  # noqa: E402

# the reference's source tree (also on PYTHONPATH); its validation helpers live beneath it
REFERENCE = os.environ.get("ZVCFD_REFERENCE", "")
if not REFERENCE:
    raise SystemExit("set ZVCFD_REFERENCE to the reference's source tree")
sys.path.insert(0, str(HERE.parents[1]))

from zvcfd.fv.geometry import topology  # noqa: E402  (the reference)
from zvcfd.fv.pattern import node_graph  # noqa: E402
from zvcfd.fv.reference import Fluid, ReferenceSolver  # noqa: E402
from zvcfd.mesh.core import BoundaryZone, UnstructuredMesh  # noqa: E402
from zvcfd.mesh.generate import box, delaunay_box, tube  # noqa: E402
from zvcfd.rheology import CarreauYasuda  # noqa: E402

from zvcfd_b200 import mesh as zmesh  # noqa: E402

MESHES = {
    "tet": lambda: box((3, 3, 3), kind="tet", perturb=0.25, seed=1),
    "pyramid": lambda: box((2, 2, 2), kind="pyramid", perturb=0.15, seed=2),
    "wedge": lambda: box((3, 3, 3), kind="wedge", perturb=0.25, seed=3),
    "hex": lambda: box((3, 3, 3), kind="hex", perturb=0.25, seed=4),
    "mixed": lambda: tube(0.5, 1.0, n_core=2, n_ring=2, n_axial=3, kind="mixed", layers=1,
                          perturb=0.1),
    "delaunay": lambda: delaunay_box((3, 3, 3), seed=5),
}
VARIANTS = [(False, None), (True, 0.3)]          # (Carreau-Yasuda + transpose, false dt)


def mesh_arrays(m) -> dict:
    out = {"nodes": m.nodes}
    for k, e in m.elements.items():
        out[f"elem_{k}"] = e
    zids = sorted(m.zones)
    out["zone_ids"] = np.array(zids, np.int64)
    out["zone_names"] = np.array([m.zones[z].name for z in zids])
    for z in zids:
        out[f"zone_{z}"] = m.zones[z].faces
    return out


def to_reference(m: zmesh.Mesh) -> UnstructuredMesh:
    um = UnstructuredMesh(m.nodes.copy(), {k: v.copy() for k, v in m.elements.items()})
    um.zones = {zid: BoundaryZone(zid, z.kind, z.name, z.faces.copy(),
                                  np.zeros(len(z.faces), np.int64))
                for zid, z in m.zones.items()}
    return um


def blocks_on_pattern(M, indptr, indices) -> np.ndarray:
    """The 4x4 blocks of a (4N x 4N) sparse matrix at the pattern's positions."""
    N = len(indptr) - 1
    rows = np.repeat(np.arange(N), np.diff(indptr))
    M = M.tocsr()
    data = np.zeros((len(indices), 4, 4))
    for r in range(4):
        for c in range(4):
            data[:, r, c] = np.asarray(M[4 * rows + r, 4 * indices + c]).reshape(-1)
    return data


# the random-state kernel test of the reference (tests/test_fv_fast.py:98-159): its fluid,
# viscosity law and seed, so that the vectors are those its own check compares
KERNEL_RHO, KERNEL_MU, KERNEL_SEED = 1.3, 0.7, 11
KERNEL_CY = dict(mu_0=0.9, mu_inf=0.1, lam=1.5)


def _without_time_terms(s, dt):
    """The reference's raw rows less its time diagonal ``rho V / dt`` on the momentum rows
    (and the matching right-hand side), which the device assembly adds later."""
    import scipy.sparse as sp

    M, b = s._raw
    if not dt:
        return M, b
    mass = KERNEL_RHO * s.V / dt
    M = M - sp.diags(np.kron(mass, [1.0, 1.0, 1.0, 0.0]))
    b = b - np.hstack([mass[:, None] * s.U, np.zeros((s.N, 1))]).ravel()
    return M, b


def kernel_case(name: str, gn: bool, dt) -> dict:
    m = MESHES[name]()
    cy = CarreauYasuda(**KERNEL_CY)
    s = ReferenceSolver(m, Fluid(KERNEL_RHO, KERNEL_MU, viscosity=cy if gn else None),
                        {zid: {"kind": "wall"} for zid in m.zones},
                        advection="high-resolution", lag_rhie_chow=True, dt=dt, transpose=gn)
    draw = np.random.default_rng(KERNEL_SEED)
    # a random state, drawn in this order: velocity, pressure, mass flows per kind, blend
    state = {"U": draw.normal(size=(s.N, 3)), "P": draw.normal(size=s.N)}
    mdot = {}
    for K in s.kinds:
        K.mdot = mdot[K.kind] = draw.normal(size=K.mdot.shape)
    state["beta_frozen"] = draw.uniform(0, 1, (s.N, 3))
    s.U, s.P, s._frozen_beta = state["U"].copy(), state["P"].copy(), state["beta_frozen"].copy()
    mdot = {k: v.copy() for k, v in mdot.items()}
    s._store_old(first=True)
    s.assemble()
    M_raw, b_raw = _without_time_terms(s, dt)
    indptr, indices = node_graph(m)
    gradU, gradP = s.nodal_gradient(state["U"]), s.nodal_gradient(state["P"])
    out = dict(mesh_arrays(m), **state)
    out.update({
        "rho": KERNEL_RHO, "mu": KERNEL_MU, "gn": int(gn), "dt": 0.0 if dt is None else dt,
        "cy": np.array([cy.mu_0, cy.mu_inf, cy.lam, cy.a, cy.n]),
        "V": s.V, "gradU": gradU, "gradP": gradP, "diag": s._a_space,
        "beta_limiter": s._beta(gradU), "indptr": indptr, "indices": indices,
        "data_raw": blocks_on_pattern(M_raw, indptr, indices), "b_raw": b_raw.reshape(-1, 4),
    })
    out.update({f"mdot_{k}": v for k, v in mdot.items()})
    # mass flows of a new random state, the drawn one being the old level
    s.U, s.P = draw.normal(size=(s.N, 3)), draw.normal(size=s.N)
    out.update({"U_new": s.U.copy(), "P_new": s.P.copy()})
    s.update_mass_flows()
    out["imbalance"] = s._interior_out
    out.update({f"mdot_new_{K.kind}": K.mdot for K in s.kinds})
    return out


def pipe_cases() -> dict:
    """Converged fields of the reference's CPU solver (lagged Rhie-Chow, fixed blend)."""
    cases = {}
    # the reference's own pipe test case (tests/test_fv_reference.py:152-162)
    R = 0.5
    m = tube(R, 2.0, n_core=2, n_ring=2, n_axial=8, kind="mixed", layers=1)
    zid = {z.name: k for k, z in m.zones.items()}

    def prof(x):
        r2 = (x[:, 0] ** 2 + x[:, 1] ** 2) / R ** 2
        return np.stack([0 * r2, 0 * r2, 2 * np.clip(1 - r2, 0, None)], 1)

    bcs = {zid["inlet"]: {"kind": "velocity", "value": prof},
           zid["outlet"]: {"kind": "pressure", "value": 0.0}, zid["wall"]: {"kind": "wall"}}
    s = ReferenceSolver(m, Fluid(1.0, 0.2), bcs, advection=1.0, lag_rhie_chow=True)
    rep = s.solve(max_iterations=400, tol=1e-12)
    assert rep.converged
    cases["pipe_reference_tube"] = dict(mesh_arrays(m), U=s.U, P=s.P, rho=1.0, mu=0.2,
                                        iterations=rep.iterations, radius=R, umax=2.0)
    # a small jittered tetrahedral pipe in SI units (the plain FP64 Poiseuille pipe, shrunk)
    R2 = 1e-3
    pm = zmesh.pipe(R2, 3e-3, n_core=4, n_ring=2, n_axial=6, kind="tet", jitter_amount=0.05,
                    seed=7)
    um = to_reference(pm)
    z = {zz.name: k for k, zz in pm.zones.items()}

    def prof2(x):
        r2 = (x[:, 0] ** 2 + x[:, 1] ** 2) / R2 ** 2
        return np.stack([0 * r2, 0 * r2, 0.2 * np.clip(1 - r2, 0, None)], 1)

    bcs2 = {z["inlet"]: {"kind": "velocity", "value": prof2},
            z["outlet"]: {"kind": "pressure", "value": 0.0}, z["wall"]: {"kind": "wall"}}
    s = ReferenceSolver(um, Fluid(1060.0, 3.5e-3), bcs2, advection=1.0, lag_rhie_chow=True)
    rep = s.solve(max_iterations=400, tol=1e-12)
    assert rep.converged
    cases["pipe_tet_si"] = dict(mesh_arrays(pm), U=s.U, P=s.P, rho=1060.0, mu=3.5e-3,
                                iterations=rep.iterations, radius=R2, umax=0.2)
    # a small curved tube, hexahedral core and wedge layers, Carreau-Yasuda, flow-rate inlet
    cm = zmesh.curved_tube(2e-3, 20e-3, np.pi / 2, n_core=4, n_ring=3, n_axial=8, layers=2,
                           growth=0.8)
    um = to_reference(cm)
    z = {zz.name: k for k, zz in cm.zones.items()}

    def shape(x):
        r2 = (x[:, 0] ** 2 + x[:, 1] ** 2) / (2e-3) ** 2
        return np.clip(1 - r2, 0, None)

    bcs3 = {z["inlet"]: {"kind": "velocity", "flow_rate": 1e-6, "profile": shape},
            z["outlet"]: {"kind": "pressure", "value": 0.0}, z["wall"]: {"kind": "wall"}}
    cy = CarreauYasuda()
    s = ReferenceSolver(um, Fluid(1060.0, 0.0035, viscosity=cy), bcs3, advection=1.0,
                        lag_rhie_chow=True)
    rep = s.solve(max_iterations=400, tol=1e-12)
    assert rep.converged
    cases["curved_cy"] = dict(mesh_arrays(cm), U=s.U, P=s.P, rho=1060.0, mu=0.0035,
                              iterations=rep.iterations, flow_rate=1e-6,
                              cy=np.array([cy.mu_0, cy.mu_inf, cy.lam, cy.a, cy.n]))
    return cases


def curved_mid_case() -> dict:
    """Converged fields of a mid-size curved Carreau-Yasuda tube (the headline tube's geometry
    and fluid at about 6k nodes: hexahedral core, three wedge wall layers, 1 ml/s), solved by
    the reference's CPU solver with lagged Rhie-Chow (SuperLU per linearisation,
    ``zvcfd/fv/reference.py:952-980``). The advection blend is fixed (1.0), as in the other
    converged goldens: a limiter frozen at iteration 10 would tie the converged state to the
    linear solver's path to that iteration, which an inexact Krylov solve does not share."""
    cm = zmesh.curved_tube(2e-3, 20e-3, np.pi / 2, n_core=8, n_ring=5, n_axial=24, layers=3,
                           growth=0.8)
    um = to_reference(cm)
    z = {zz.name: k for k, zz in cm.zones.items()}

    def shape(x):
        r2 = (x[:, 0] ** 2 + x[:, 1] ** 2) / (2e-3) ** 2
        return np.clip(1 - r2, 0, None)

    bcs = {z["inlet"]: {"kind": "velocity", "flow_rate": 1e-6, "profile": shape},
           z["outlet"]: {"kind": "pressure", "value": 0.0}, z["wall"]: {"kind": "wall"}}
    cy = CarreauYasuda()
    s = ReferenceSolver(um, Fluid(1060.0, 0.00345, viscosity=cy), bcs, advection=1.0,
                        lag_rhie_chow=True)
    rep = s.solve(max_iterations=300, tol=1e-11)
    assert rep.converged, rep.iterations
    return dict(mesh_arrays(cm), U=s.U, P=s.P, rho=1060.0, mu=0.00345,
                iterations=rep.iterations, flow_rate=1e-6,
                cy=np.array([cy.mu_0, cy.mu_inf, cy.lam, cy.a, cy.n]))


def transient_case() -> dict:
    """The reference pipe marched 6 BDF2 steps from its steady state with a pulsatile inlet.

    Each step runs its coefficient loops to convergence (tol 1e-13, cap 150; the reference
    needs about 64 per step): with a cap of 30 the reference stops every step short of
    convergence and its fields then depend on the linear solver's path (1.6e-7 of 2.8)."""
    R = 0.5
    m = tube(R, 2.0, n_core=2, n_ring=2, n_axial=8, kind="mixed", layers=1)
    zid = {z.name: k for k, z in m.zones.items()}

    def prof(x, t):
        r2 = (x[:, 0] ** 2 + x[:, 1] ** 2) / R ** 2
        amp = 1.0 + 0.5 * np.sin(2 * np.pi * t / 0.8)
        return np.stack([0 * r2, 0 * r2, 2 * amp * np.clip(1 - r2, 0, None)], 1)

    bcs = {zid["inlet"]: {"kind": "velocity", "value": prof},
           zid["outlet"]: {"kind": "pressure", "value": 0.0}, zid["wall"]: {"kind": "wall"}}
    s = ReferenceSolver(m, Fluid(1.0, 0.2), bcs, advection=1.0, lag_rhie_chow=True)
    rep = s.solve(max_iterations=400, tol=1e-12)
    assert rep.converged
    U0, P0 = s.U.copy(), s.P.copy()
    s.solve_transient(0.05, 6, scheme="bdf2", loops=150, tol=1e-13)
    return dict(mesh_arrays(m), U0=U0, P0=P0, U=s.U, P=s.P, rho=1.0, mu=0.2, radius=R, umax=2.0,
                dt=0.05, steps=6, t_end=s.t, loops=150, tol=1e-13)


def wall_case() -> dict:
    """The reference's wall shear stress (WallGradientShear) of two converged golden fields."""
    from zvcfd.fv.wall import WallGradientShear

    out = {}
    for tag in ("pipe_reference_tube", "curved_cy"):
        with np.load(HERE / f"{tag}.npz") as z:
            g = {k: z[k] for k in z.files}
        els = {k: g[f"elem_{k}"] for k in ("tet", "pyramid", "wedge", "hex") if f"elem_{k}" in g}
        um = UnstructuredMesh(g["nodes"], els)
        um.zones = {int(zid): BoundaryZone(int(zid), "", str(nm), g[f"zone_{int(zid)}"],
                                           np.zeros(len(g[f"zone_{int(zid)}"]), np.int64))
                    for zid, nm in zip(g["zone_ids"], g["zone_names"])}
        wall = [int(zid) for zid, nm in zip(g["zone_ids"], g["zone_names"]) if str(nm) == "wall"]
        op = WallGradientShear(um, wall)
        visc = CarreauYasuda() if tag == "curved_cy" else None
        out[f"{tag}_tau"] = op(g["U"], viscosity=visc, mu=float(g["mu"]))
    return out


def backflow_case() -> dict:
    """The reference's backflow box (``tests/test_fv_boundaries.py:182-207``): a warped tet
    channel with a cosine outlet pressure that drives backflow, solved by the reference's CPU
    solver with backflow stabilisation 0.5, and the same without stabilisation."""
    m = box((6, 4, 3), (1.5, 1.0, 0.6), kind="tet", warp=0.03)
    z = {b.name: k for k, b in m.zones.items()}
    out = {}
    for tag, beta in (("stab", 0.5), ("plain", 0.0)):
        bcs = {k: {"kind": "wall"} for k in m.zones}
        bcs[z["xmin"]] = {"kind": "velocity", "value": (1.0, 0.0, 0.0)}
        bcs[z["xmax"]] = {"kind": "pressure", "value": lambda x: 1.5 * np.cos(np.pi * x[:, 1]),
                          "backflow_stabilisation": beta}
        s = ReferenceSolver(m, Fluid(1.0, 0.05), bcs, advection=1.0)
        rep = s.solve(max_iterations=200, tol=1e-12)
        assert rep.converged
        out[f"U_{tag}"], out[f"P_{tag}"] = s.U.copy(), s.P.copy()
    return dict(mesh_arrays(m), **out, rho=1.0, mu=0.05)


def _host_gpusolver(s: ReferenceSolver):
    """The reference's ``GPUSolver`` post-processing methods (``zone_forces``, ``wall_shear``,
    ``zvcfd/fv/solver.py:1080-1245``) bound to the converged state of a CPU solve, with NumPy
    standing in for CuPy (they only use array calls NumPy also has), so that their outputs can be
    recorded here without a GPU."""
    import types

    from zvcfd.fv.solver import GPUSolver, RawRows

    cp = types.ModuleType("cupy")
    for k in dir(np):
        if not k.startswith("_"):
            setattr(cp, k, getattr(np, k))
    cp.asnumpy = np.asarray
    sys.modules.setdefault("cupy", cp)
    g = object.__new__(GPUSolver)
    g.cp, g.N, g._n_own = cp, s.N, s.N
    g.mesh, g.fluid, g.bcs, g.stokes = s.mesh, s.fluid, s.bcs, s.stokes
    g.sub, g.sub_flow, g.sub_vel = s.sub, s.sub_flow, s.sub_vel
    g._outlet, g._special = s._outlet, {}
    g.vel_fixed_comp = s.vel_fixed_comp
    g.U, g.P = s.U.copy(), s.P.copy()
    M, b = s._raw
    indptr, indices = node_graph(s.mesh)
    data = blocks_on_pattern(M, indptr, indices)
    rows = np.repeat(np.arange(s.N), np.diff(indptr))
    keep = np.flatnonzero(s.vel_fixed_comp.any(1)[rows])
    g._raw = RawRows(keep, rows[keep], indices[keep].astype(np.int64), data[keep],
                     b.reshape(-1, 4))
    return g


def forces_case() -> dict:
    """Zone forces, zone flows and balances of two converged cases solved by the reference's
    CPU solver: the mixed-element pipe of ``tests/test_fv_reference.py:152-162`` (walls, a
    parabolic inlet, a pressure outlet; the case of ``tests/test_fv_solver_gpu.py:129-141``)
    and the channel of ``tests/test_fv_boundaries.py:210-233`` (two pressure zones that share
    an edge of nodes, a wall, two symmetry planes)."""
    out = {}
    R = 0.5
    pipe = tube(R, 2.0, n_core=2, n_ring=2, n_axial=8, kind="mixed", layers=1)
    z = {zz.name: k for k, zz in pipe.zones.items()}

    def prof(x):
        r2 = (x[:, 0] ** 2 + x[:, 1] ** 2) / R ** 2
        return np.stack([0 * r2, 0 * r2, 2 * np.clip(1 - r2, 0, None)], 1)

    pipe_bcs = {z["inlet"]: {"kind": "velocity", "value": prof},
                z["outlet"]: {"kind": "pressure", "value": 0.0}, z["wall"]: {"kind": "wall"}}
    chan = box((10, 6, 1), (2.0, 1.0, 0.2), kind="hex")
    z = {zz.name: k for k, zz in chan.zones.items()}
    chan_bcs = {z["xmin"]: {"kind": "velocity", "value": [1.0, 0.0, 0.0]},
                z["xmax"]: {"kind": "pressure", "value": 0.0},
                z["ymax"]: {"kind": "pressure", "value": 0.0},
                z["ymin"]: {"kind": "wall"}, z["zmin"]: {"kind": "symmetry"},
                z["zmax"]: {"kind": "symmetry"}}
    for tag, m, bcs, mu in (("pipe", pipe, pipe_bcs, 0.2), ("channel", chan, chan_bcs, 0.05)):
        s = ReferenceSolver(m, Fluid(1.0, mu), bcs, advection=1.0)
        rep = s.solve(max_iterations=300, tol=1e-13)
        assert rep.converged
        F, q, bal = s.zone_forces(), s.zone_flows(), s.balances()
        zids = sorted(F)
        for k, v in mesh_arrays(m).items():
            out[f"{tag}_{k}"] = v
        out.update({f"{tag}_U": s.U.copy(), f"{tag}_P": s.P.copy(), f"{tag}_mu": mu,
                    f"{tag}_force_zones": np.array(zids, np.int64),
                    f"{tag}_forces": np.array([F[k] for k in zids]),
                    f"{tag}_flows": np.array([q[k] for k in zids]),
                    f"{tag}_momentum_outflow": np.array(
                        [s.zone_momentum_outflow()[k] for k in zids]),
                    f"{tag}_mass": bal["mass"], f"{tag}_momentum": bal["momentum"],
                    f"{tag}_identity": bal["identity"]})
        h = _host_gpusolver(s)
        Fg = h.zone_forces()
        out[f"{tag}_gpusolver_forces"] = np.array([Fg[k] for k in zids])
        nodes, tau = h.wall_shear("reaction")
        out[f"{tag}_reaction_nodes"], out[f"{tag}_reaction_tau"] = nodes, tau
        nodes, tau = h.wall_shear("gradient")
        out[f"{tag}_gradient_nodes"], out[f"{tag}_gradient_tau"] = nodes, tau
    return out


def wss_case() -> dict:
    """The reference's WSS time statistics (``zvcfd/fv/wss.py``) over a seeded series: 40 wall
    nodes, 9 samples at uneven times; node 0 never sheared, node 1 reverses in time."""
    from zvcfd.fv.wss import WallShearStats

    rng = np.random.default_rng(11)
    n, k = 40, 9
    t = np.cumsum(rng.uniform(0.5e-3, 2e-3, k))
    tau = rng.standard_normal((k, n, 3))
    tau[:, 0] = 0.0
    tau[:, 1] = np.sin(2 * np.pi * (t - t[0]) / (t[-1] - t[0]))[:, None] * np.array([1.0, 0.2, 0])
    st = WallShearStats(n)
    for ti, x in zip(t, tau):
        st.add(ti, x)
    r = st.results()
    return {"t": t, "tau": tau, "tawss": r["tawss"], "osi": r["osi"], "rrt": r["rrt"]}


def gn_outlet_case() -> dict:
    """The reference's Carreau-Yasuda manufactured outlet (``tests/test_fv_solver_gpu.py:76-101``):
    a warped tet box with the manufactured velocity on every face but ``xmax``, a pressure
    outlet there with the manufactured pressure and prescribed velocity gradient (traction),
    the manufactured body force, the transpose term on; solved by the reference's CPU solver.
    The manufactured fields are tabulated at the nodes and the outlet's sub-face points (where
    the conditions are evaluated), so that the tests can rebuild the conditions without it."""
    from zvcfd.fv.geometry import boundary_subface_weights
    from zvcfd.rheology import CarreauYasuda as RefCY

    sys.path.insert(0, str(Path(REFERENCE) / "benchmarks" / "validation"))
    from exact import manufactured_gn

    cy = RefCY(mu_0=0.5, mu_inf=0.05, lam=2.0)
    m = box((4, 4, 4), kind="tet", warp=0.03)

    def ex(x):
        return manufactured_gn(x, cy.of_gamma_squared, shift=(0.2, 0.1, 0.3),
                               mean=(1.5, 0.0, 0.0))

    z = {b.name: k for k, b in m.zones.items()}
    bcs = {k: {"kind": "velocity", "value": lambda x: ex(x)[0]} for k in m.zones}
    bcs[z["xmax"]] = {"kind": "pressure", "value": lambda x: ex(x)[1],
                      "grad": lambda x: ex(x)[3]}
    s = ReferenceSolver(m, Fluid(1.0, 0.1, viscosity=lambda g: cy.of_gamma_squared(g * g)),
                        bcs, source=lambda x: ex(x)[2], advection=1.0, transpose=True)
    rep = s.solve(max_iterations=200, tol=1e-13)
    assert rep.converged
    f = m.zones[z["xmax"]].faces
    ok = f >= 0
    xs = np.einsum("fij,fjk->fik", boundary_subface_weights(f), m.nodes[np.where(ok, f, 0)])
    pts = np.concatenate([m.nodes, xs[ok]])
    u, p, src, J = ex(pts)
    return dict(mesh_arrays(m), U=s.U.copy(), P=s.P.copy(), rho=1.0, mu=0.1,
                cy=np.array([cy.mu_0, cy.mu_inf, cy.lam, cy.a, cy.n]), points=pts, u=u, p=p,
                f=src, J=J, iterations=rep.iterations)


def profiles_case() -> dict:
    """The developed inlet profile (``zvcfd/fv/profiles.py``) on four inlet faces (a mixed
    quad/triangle circle, a triangulated circle, a quad and a triangulated rectangle), and a
    pipe with a flow-rate inlet of the default profile solved by the reference's CPU solver."""
    from zvcfd.fv.profiles import poiseuille, shape

    out = {}
    meshes = {"tube_mixed": tube(0.5, 2.0, n_core=2, n_ring=2, n_axial=8, kind="mixed",
                                 layers=1),
              "tube_tet": tube(1.0, 2.0, n_core=3, n_ring=3, n_axial=4, kind="tet"),
              "box_hex": box((5, 4, 3), (1.0, 0.7, 0.4), kind="hex"),
              "box_tet": box((5, 4, 3), (1.0, 0.7, 0.4), kind="tet", warp=0.03)}
    for tag, m in meshes.items():
        z = next(zz for zz in m.zones.values() if zz.name in ("inlet", "xmin"))
        u = poiseuille(m.nodes, z.faces)
        nodes, v = shape(m.nodes, z.faces, "poiseuille")
        out.update({f"{tag}_X": m.nodes, f"{tag}_faces": z.faces, f"{tag}_nodes": nodes,
                    f"{tag}_u": np.array([u[int(g)] for g in nodes]), f"{tag}_shape": v})
    m = meshes["tube_mixed"]
    zid = {zz.name: k for k, zz in m.zones.items()}
    bcs = {zid["inlet"]: {"kind": "velocity", "flow_rate": 0.3},
           zid["outlet"]: {"kind": "pressure", "value": 0.0}, zid["wall"]: {"kind": "wall"}}
    s = ReferenceSolver(m, Fluid(1.0, 0.2), bcs, advection=1.0)
    rep = s.solve(max_iterations=300, tol=1e-13)
    assert rep.converged
    for k, v in mesh_arrays(m).items():
        out[f"pipe_{k}"] = v
    out.update(pipe_U=s.U.copy(), pipe_P=s.P.copy(), pipe_flow_rate=0.3, pipe_rho=1.0,
               pipe_mu=0.2)
    return out


def variable_steps_case() -> dict:
    """The reference's variable-step BDF2 case (``tests/test_fv_boundaries.py:281-300``): a
    hexahedral tube driven by an oscillating inlet pressure (Womersley number about 4), six
    steps of uneven size, solved by the reference's CPU solver with lagged Rhie-Chow."""
    R = 0.5
    w = 2 * np.pi
    nu = R * R * w / 16
    m = tube(R, 0.5, n_core=2, n_ring=2, n_axial=2, kind="hex")
    z = {b.name: k for k, b in m.zones.items()}
    bcs = {z["inlet"]: {"kind": "pressure",
                        "value": lambda x, t: 0.5 * np.cos(w * t) * np.ones(len(x))},
           z["outlet"]: {"kind": "pressure", "value": 0.0}, z["wall"]: {"kind": "wall"}}
    steps = np.array([0.05, 0.08, 0.04, 0.06, 0.03, 0.07])
    s = ReferenceSolver(m, Fluid(1.0, nu), bcs, advection=1.0, lag_rhie_chow=True)
    rep = s.solve_transient(list(steps), loops=60, tol=1e-12)
    return dict(mesh_arrays(m), U=s.U.copy(), P=s.P.copy(), steps=steps, nu=nu, omega=w,
                converged=rep.converged)


def lumped_case() -> dict:
    """The reference's RCR model (``zvcfd/lumped.py:181-218``): steady coefficients, and the
    step coefficients and committed pressures of 40 steps under a pulsatile outflow, for the
    trapezoidal and backward-Euler steppings, with a constant and a tabulated venous pressure."""
    from zvcfd.lumped import RCR as RefRCR

    out = {}
    params = [(1e8, 1e-9, 1e9, 0.0), (2.0, 0.1, 5.0, 1.0), (0.5e8, 2e-9, 0.8e9, [(0.0, 100.0),
                                                                            (0.4, 300.0),
                                                                            (0.8, 100.0)])]
    for i, (rp, c, rd, pv) in enumerate(params):
        for method in ("trapezoidal", "euler"):
            m = RefRCR(rp=rp, c=c, rd=rd, pv=pv, method=method)
            a, r = m.steady_coefficients(0.0)
            m.initialise(1e-6 if rp > 10 else 0.3, 0.0)
            rows = []
            dt = 0.013
            for k in range(1, 41):
                t = k * dt
                q = (1e-6 if rp > 10 else 0.3) * (1.0 + 0.5 * np.sin(2 * np.pi * t / 0.8))
                ca, cr = m.coefficients(t, dt)
                p = m.advance(q, t, dt)
                rows.append((t, q, ca, cr, p))
            out[f"rcr{i}_{method}_steady"] = np.array([a, r])
            out[f"rcr{i}_{method}_steps"] = np.array(rows)
    # the variable-step BDF coefficients and the Carreau-Yasuda law of the same module family
    from zvcfd.fv.reference import bdf_coefficients
    from zvcfd.rheology import CarreauYasuda as RefCY

    cases = [("bdf1", 1e-3, None, 1), ("bdf2", 1e-3, None, 1), ("bdf2", 1e-3, 1e-3, 2),
             ("bdf2", 2e-3, 1e-3, 2), ("bdf2", 0.5e-3, 1.5e-3, 2)]
    out["bdf"] = np.array([bdf_coefficients(*c) for c in cases])
    gamma = np.concatenate([[0.0], np.logspace(-3, 4, 29)])
    out["cy_gamma"] = gamma
    out["cy_blood"] = RefCY()(gamma)
    out["cy_other"] = RefCY(mu_0=0.1, mu_inf=0.004, lam=1.5, a=1.7, n=0.4)(gamma)
    return out


def partition_case() -> dict:
    """The reference's partitions (``zvcfd/fv/partition.py``) of the meshes of its own
    partition test (``tests/test_fv_multi.py:40-43``: a mixed tube, 4 parts) and of the golden
    pipe (2, 3 and 4 parts, and 3 parts at a given chunk edge): owners, and per part the local
    nodes, owned count, held elements and faces and the halo plan, flattened."""
    from zvcfd.fv.partition import halo_plan, local_meshes, morton_owner

    out = {}
    tubes = {"mixed": tube(0.5, 2.0, n_core=3, n_ring=3, n_axial=16, kind="mixed", layers=1),
             "pipe": tube(0.5, 2.0, n_core=2, n_ring=2, n_axial=8, kind="mixed", layers=1)}
    runs = [("mixed", 4, None), ("pipe", 2, None), ("pipe", 3, None), ("pipe", 4, None),
            ("pipe", 3, 0.3)]
    for name, m in tubes.items():
        for k, v in mesh_arrays(m).items():
            out[f"{name}_{k}"] = v
    for i, (name, n, chunk) in enumerate(runs):
        m = tubes[name]
        owner = morton_owner(m.nodes, n, chunk)
        parts = local_meshes(m, owner)
        plans = halo_plan(parts, owner)
        tag = f"run{i}"
        out[f"{tag}_meta"] = np.array([n, -1.0 if chunk is None else chunk])
        out[f"{tag}_mesh"] = np.array(name)
        out[f"{tag}_owner"] = owner
        for p, (lm, plan) in enumerate(zip(parts, plans)):
            out[f"{tag}_p{p}_nodes"] = lm.nodes
            out[f"{tag}_p{p}_n_own"] = np.array(lm.n_own)
            for k, sel in lm.elements.items():
                out[f"{tag}_p{p}_elem_{k}"] = sel
            for z, sel in lm.faces.items():
                out[f"{tag}_p{p}_face_{z}"] = sel
            out[f"{tag}_p{p}_plan"] = np.array([q for q, _, _ in plan], np.int64)
            for q, send, recv in plan:
                out[f"{tag}_p{p}_send_{q}"] = send
                out[f"{tag}_p{p}_recv_{q}"] = recv
    out["runs"] = np.array(len(runs))
    return out


# ---------------------------------------------------------------- the reference's colouring

_SHIM = r"""
// CUDA's built-ins for running a kernel's threads on the CPU: one after another, or, for a
// kernel with block barriers, each block's threads as OpenMP threads (__syncthreads an
// OpenMP barrier, __shared__ storage static: blocks run one at a time)
#include <stdint.h>
#include <math.h>
#include <omp.h>
struct zv_dim { long long x; };
static zv_dim blockIdx, blockDim;
static thread_local zv_dim threadIdx;
#define __global__
#define __shared__ static
#define __constant__ static const
#define __device__
static inline void __syncthreads() {
    _Pragma("omp barrier")
}
struct double2 { double x, y; };
static inline double2 make_double2(double a, double b) { double2 r; r.x = a; r.y = b; return r; }
// a warp shuffle over the block's threads (all of them call it, as the kernels do): values
// exchanged through a block-wide buffer between two barriers
static double zv_shfl[1024];
static inline double __shfl_down_sync(unsigned mask, double v, int delta, int width) {
    int t = (int)threadIdx.x;
    zv_shfl[t] = v;
    _Pragma("omp barrier")
    double r = (t % width + delta < width) ? zv_shfl[t + delta] : v;
    _Pragma("omp barrier")
    return r;
}
static inline unsigned long long atomicMin(unsigned long long *a, unsigned long long v) {
    unsigned long long o = *a; if (v < o) *a = v; return o; }
static inline unsigned long long atomicAdd(unsigned long long *a, unsigned long long v) {
    unsigned long long o = *a; *a = o + v; return o; }
static inline int __ffsll(long long v) { return __builtin_ffsll(v); }
"""

def _launcher(src: str, name: str) -> str:
    """A C function ``launch_<name>(grid, block, <the kernel's parameters>)`` running the
    kernel's threads one after another over the grid."""
    import re

    m = re.search(r"__global__\s+void\s+" + name + r"\s*\(([^)]*)\)", src)
    params = [p.strip() for p in m.group(1).split(",")]
    names = [re.findall(r"[A-Za-z_]\w*", p)[-1] for p in params]
    head = (f'extern "C" void launch_{name}(long long grid, long long block, '
            f'{", ".join(params)}) {{\n    blockDim.x = block;\n')
    call = f"{name}({', '.join(names)});"
    if "__syncthreads" in src or "__shfl" in src:
        return (head + "    omp_set_dynamic(0);\n"
                "    for (long long zv_b = 0; zv_b < grid; ++zv_b) {\n"
                "        blockIdx.x = zv_b;\n#pragma omp parallel num_threads((int)block)\n"
                f"        {{ threadIdx.x = omp_get_thread_num(); {call} }}\n    }}\n}}\n")
    return (head + "    for (long long zv_b = 0; zv_b < grid; ++zv_b) "
            "for (long long zv_t = 0; zv_t < block; ++zv_t) "
            f"{{ blockIdx.x = zv_b; threadIdx.x = zv_t; {call} }}\n}}\n")


def _ctypes_of(src: str, name: str) -> list:
    import ctypes
    import re

    m = re.search(r"__global__\s+void\s+" + name + r"\s*\(([^)]*)\)", src)
    out = []
    for p in (q.strip() for q in m.group(1).split(",")):
        if "*" in p:
            out.append(ctypes.c_void_p)
        elif "long long" in p:
            out.append(ctypes.c_longlong)
        elif "double" in p:
            out.append(ctypes.c_double)
        else:
            out.append(ctypes.c_int)
    return out


def _cpu_cupy():
    """A stand-in for the ``cupy`` module on the CPU, enough for the reference's device path:
    its colouring (``zvcfd/fv/fast.py:35-130``), ``BlockMatrix`` product, ACM and FGMRES
    (``zvcfd/fv/linear.py:47-135``, ``:238-518``), fast element kernels
    (``zvcfd/fv/_cuda_fast.py``), boundary pass (``zvcfd/fv/_cuda_bc.py``) and so its whole
    ``GPUSolver``. Arrays are numpy arrays with CuPy's ``get``; array functions are numpy's;
    ``RawKernel``/``RawModule`` compile the kernel source the reference hands them with g++ for
    the CPU (``oracle/_ref/``, not committed): a kernel without block barriers or shuffles runs
    its threads one after another, one with them runs each block's threads as OpenMP threads
    (``_SHIM``). The kernels' results do not depend on the order of their threads (one writer
    per address: a thread per block row, colour-ordered element scatters, an ``atomicMin`` claim
    per node), so they are what the reference computes on a GPU, with one exception: the
    residual sums of squares of ``finalise``'s partial-sum tree, which only its report uses."""
    import ctypes
    import hashlib
    import subprocess
    import types

    class Arr(np.ndarray):
        def get(self):
            return np.asarray(self)

    def wrap(fn):
        return lambda *a, **k: np.asarray(fn(*a, **k)).view(Arr)

    out_dir = HERE.parents[1] / "oracle" / "_ref"
    out_dir.mkdir(parents=True, exist_ok=True)

    class RawKernel:
        libs = {}

        def __init__(self, src, name, options=()):
            tag = hashlib.sha1((src + name).encode()).hexdigest()[:12]
            if tag not in RawKernel.libs:
                cpp, so = out_dir / f"kernel_{tag}.cpp", out_dir / f"kernel_{tag}.so"
                cpp.write_text(_SHIM + src + _launcher(src, name))
                subprocess.run(["g++", "-O2", "-fopenmp", "-shared", "-fPIC", "-o", str(so),
                                str(cpp)], check=True)
                RawKernel.libs[tag] = ctypes.CDLL(str(so))
            self.fn = getattr(RawKernel.libs[tag], f"launch_{name}")
            self.types = _ctypes_of(src, name)

        def __call__(self, grid, block, args):
            conv = [ctypes.c_void_p(np.ascontiguousarray(a).ctypes.data) if t is ctypes.c_void_p
                    else t(a) for a, t in zip(args, self.types)]
            for a, t in zip(args, self.types):
                if t is ctypes.c_void_p and not a.flags.c_contiguous:
                    raise ValueError("a kernel argument must be contiguous")
            self.fn(ctypes.c_longlong(grid[0]), ctypes.c_longlong(block[0]), *conv)

    class CuPy(types.ModuleType):
        def __getattr__(self, name):
            return getattr(np, name)

    cp = CuPy("cupy")
    for name in ("arange", "ascontiguousarray", "asarray", "empty", "zeros", "ones", "full",
                 "zeros_like", "empty_like", "concatenate", "stack", "searchsorted",
                 "flatnonzero", "cumsum", "bincount", "argsort", "sqrt", "dot", "einsum"):
        setattr(cp, name, wrap(getattr(np, name)))
    cp.asnumpy = np.asarray
    cp.ndarray = np.ndarray
    cp.get_array_module = lambda *a: np
    cp.linalg = types.SimpleNamespace(inv=wrap(np.linalg.inv), norm=np.linalg.norm)
    nothing = lambda *a, **k: None                                   # noqa: E731
    cp.cuda = types.SimpleNamespace(
        Device=lambda *a: types.SimpleNamespace(id=0, mem_info=(64 << 30, 64 << 30),
                                                synchronize=nothing),
        runtime=types.SimpleNamespace(deviceSynchronize=nothing),
        get_current_stream=lambda: types.SimpleNamespace(synchronize=nothing, ptr=0))
    cp.get_default_memory_pool = lambda: types.SimpleNamespace(
        free_all_blocks=nothing, used_bytes=lambda: 0, free_bytes=lambda: 0)

    class RawModule:
        def __init__(self, code, options=()):
            self.code = code

        def get_function(self, name):
            return RawKernel(self.code, name)

    cp.RawKernel, cp.RawModule = RawKernel, RawModule
    return cp


def box_tets(n):
    """Five tetrahedra per cube of an n^3 grid of cubes (the reference's
    ``tests/test_fv_fast.py:59-69`` mesh)."""
    i, j, k = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")

    def v(a, b, c):
        return ((i + a) * (n + 1) + (j + b)) * (n + 1) + (k + c)

    c = [v(0, 0, 0), v(1, 0, 0), v(1, 1, 0), v(0, 1, 0), v(0, 0, 1), v(1, 0, 1), v(1, 1, 1),
         v(0, 1, 1)]
    tets = [(0, 1, 3, 4), (1, 2, 3, 6), (1, 4, 5, 6), (3, 4, 6, 7), (1, 3, 4, 6)]
    return np.stack([np.stack([c[t].ravel() for t in tet], 1) for tet in tets], 0) \
        .reshape(-1, 4).astype(np.int32), (n + 1) ** 3


def colour_case() -> dict:
    """The reference's ``gpu_colour`` (run on the CPU, :func:`_cpu_cupy`) on the meshes the
    device colouring is tested on: a jittered tetrahedral pipe, the hexahedra and wedges of a
    curved tube, a box of 40,960 tetrahedra, the six kernel meshes, and a fan of 200 tetrahedra
    on one node coloured with one 64-bit mask word (the masks widen twice)."""
    sys.modules["cupy"] = _cpu_cupy()
    from zvcfd.fv.fast import gpu_colour

    out = {}
    cases = {}
    pm = zmesh.pipe(1.0, 3.0, n_core=4, n_ring=3, n_axial=10, kind="tet", jitter_amount=0.1,
                    seed=3)
    cm = zmesh.curved_tube(1.0, 5.0, n_core=4, n_ring=4, n_axial=12, layers=2)
    for tag, m in (("pipe", pm), ("curved", cm)):
        for k, e in m.elements.items():
            cases[f"{tag}_{k}"] = (e, m.n_nodes, 4)
    for name, make in MESHES.items():
        m = make()
        for k, e in m.elements.items():
            cases[f"kernel_{name}_{k}"] = (e, m.n_nodes, 4)
    cases["box16"] = box_tets(16) + (4,)
    fan = np.column_stack([np.zeros(200, np.int64), 3 * np.arange(200) + 1,
                           3 * np.arange(200) + 2, 3 * np.arange(200) + 3])
    cases["fan"] = (fan, 601, 1)
    for tag, (e, n, words) in cases.items():
        col = np.asarray(gpu_colour(np.asarray(e), n, words=words))
        out[f"{tag}_conn"] = np.asarray(e, np.int32) if tag != "box16" else np.zeros(0)
        out[f"{tag}_meta"] = np.array([n, words])
        out[f"{tag}_colour"] = col.astype(np.int32)
    out["cases"] = np.array(sorted(cases))
    return out


def acm_case() -> dict:
    """The reference's own ACM (``zvcfd/fv/linear.py:328-518``) and device FGMRES
    (``:238-320``), run on the CPU through :func:`_cpu_cupy`, on a system the reference's CPU
    solver assembled: the golden tetrahedral pipe after three Picard iterations (Dirichlet rows
    in place), with ``coarse=40`` (one coarse level) and ``coarse=8`` (deeper). Recorded: the
    system, and per setting each
    level's aggregates and Galerkin operator, one V-cycle of the right-hand side, and the
    ACM-FGMRES solve to 1e-10 (solution, iterations, residual)."""
    sys.modules["cupy"] = _cpu_cupy()
    import scipy.sparse as sp  # noqa: F401

    from zvcfd.fv.linear import ACM, BlockMatrix

    g = np.load(HERE / "pipe_tet_si.npz")
    nodes = g["nodes"]
    elements = {k: g[f"elem_{k}"] for k in ("tet", "pyramid", "wedge", "hex") if f"elem_{k}" in g}
    pm = zmesh.Mesh(nodes, elements)
    for zid, name in zip(g["zone_ids"], g["zone_names"]):
        pm.zones[int(zid)] = zmesh.Zone(int(zid), "", str(name), g[f"zone_{int(zid)}"])
    um = to_reference(pm)
    z = {zz.name: k for k, zz in pm.zones.items()}
    R2 = float(g["radius"])

    def prof(x):
        r2 = (x[:, 0] ** 2 + x[:, 1] ** 2) / R2 ** 2
        return np.stack([0 * r2, 0 * r2, 0.2 * np.clip(1 - r2, 0, None)], 1)

    bcs = {z["inlet"]: {"kind": "velocity", "value": prof},
           z["outlet"]: {"kind": "pressure", "value": 0.0}, z["wall"]: {"kind": "wall"}}
    s = ReferenceSolver(um, Fluid(1060.0, 3.5e-3), bcs, advection=1.0, lag_rhie_chow=True)
    s.solve(max_iterations=3, tol=0.0)
    M, b = s.assemble()
    indptr, indices = node_graph(um)
    data = blocks_on_pattern(M, indptr, indices)
    A = BlockMatrix(np.asarray(indptr, np.int64), np.asarray(indices, np.int32), data)
    out = {"indptr": A.indptr, "indices": A.indices, "data": data, "b": b,
           "coarse": np.array([40, 8])}
    for coarse in (40, 8):
        acm = ACM(coarse=coarse)
        acm.setup(A)
        pre = f"c{coarse}_"
        out[pre + "levels"] = np.array(len(acm.levels))
        for i, L in enumerate(acm.levels):
            out[f"{pre}level{i}_n"] = np.array(L["A"].n)
            out[f"{pre}level{i}_dense"] = np.array("dense_inv" in L)
            if "agg" in L:
                out[f"{pre}level{i}_agg"] = np.asarray(L["agg"])
            if i:
                out[f"{pre}level{i}_indptr"] = np.asarray(L["A"].indptr)
                out[f"{pre}level{i}_indices"] = np.asarray(L["A"].indices)
                out[f"{pre}level{i}_data"] = np.asarray(L["A"].data)
        out[pre + "vcycle"] = np.asarray(acm.vcycle(np.asarray(b).copy()))
        x, info = acm.solve(A, np.asarray(b).copy(), rtol=1e-10)
        out.update({pre + "x": np.asarray(x), pre + "iterations": np.array(info.iterations),
                    pre + "residual": np.array(info.residual),
                    pre + "converged": np.array(info.converged)})
    return out


def boundary_case() -> dict:
    """The reference's boundary pass (its ``finalise`` kernel, ``zvcfd/fv/_cuda_bc.py:32-138``)
    run on the CPU (:func:`_cpu_cupy`) on the raw system the oracle assembles for the golden
    tetrahedral pipe after three outer iterations with a false time step, with and without
    elimination. The pass's own known terms (time, body force, outlet force, inflow, outflow
    momentum, lumped rows) are given as zeros, since the raw system holds them: so this is the
    part the oracle's ``boundary_pass`` restates (Dirichlet rows, elimination, residual
    statistics, row scaling). Recorded: the inputs, and per case the scaled blocks, right-hand
    side, row scales and the residual maxima per equation. Not the sums of squares: the
    kernel's partial-sum tree has the four threads of a row add the same pair, which a GPU
    warp, in lockstep, performs once and concurrent CPU threads do not."""
    import ctypes  # noqa: F401

    cp = _cpu_cupy()
    from zvcfd.fv._cuda_bc import FINALISE

    from oracle.fv import OracleSolver
    sys.path.insert(0, str(HERE.parent))
    from fixtures import fluid_of, load, mesh_of, pipe_bcs

    out = {}
    name = "pipe_tet_si"
    g = load(name)
    m = mesh_of(g)
    fl = fluid_of(g)
    kernel = cp.RawKernel(FINALISE, "finalise")
    for dt in (0.02,):
        o = OracleSolver(m, fl, pipe_bcs(name, g, m), advection=1.0, dt=dt)
        o.solve(max_iterations=3, tol=0.0)
        o.momentum_diagonal()
        o.assemble()
        raw, braw = o.raw
        N = o.N
        X = np.concatenate([o.U, o.P[:, None]], 1)
        tag = "dt" if dt else "steady"
        fixed = np.concatenate([o.vel_fixed_comp, o.p_fixed[:, None]], 1)
        uref = max(np.abs(o.U).max(), np.abs(o.vel_value).max(), 1e-30)
        pref = max(np.ptp(o.P), fl.rho * uref * uref, 1e-30)
        out.update({f"{tag}_indptr": o.indptr, f"{tag}_indices": o.indices,
                    f"{tag}_raw": raw, f"{tag}_braw": braw.reshape(N, 4), f"{tag}_x": X,
                    f"{tag}_fixed": fixed, f"{tag}_vel": o.vel_value, f"{tag}_pval": o.p_value,
                    f"{tag}_aP": o.aP, f"{tag}_V": o.V, f"{tag}_U": o.U, f"{tag}_P": o.P,
                    f"{tag}_rho": np.array(fl.rho)})
        rows = np.repeat(np.arange(N), np.diff(o.indptr))
        dpos = np.flatnonzero(rows == o.indices).astype(np.int64)
        zN, zN3 = np.zeros(N), np.zeros((N, 3))
        for elim in (1, 0):
            data = np.ascontiguousarray(raw, np.float64).copy()
            b = np.ascontiguousarray(braw.reshape(-1), np.float64).copy()
            nb = (4 * N + 255) // 256
            rs = np.zeros(4 * N)
            partial = np.zeros(nb * 8)
            kernel((nb,), (256,), (
                np.int64(N), np.asarray(o.indptr, np.int64), np.asarray(o.indices, np.int32),
                dpos, data, b, np.int32(0), zN, zN3, zN3, zN3, zN, zN, zN, zN, zN, np.int32(1),
                zN3, fixed.astype(np.uint8), fixed.astype(np.uint8), o.vel_value.copy(),
                o.p_value.copy(), np.int32(elim), np.full(N, -1, np.int64), np.zeros(16),
                np.zeros(4 * N), X.reshape(-1).copy(), o.aP.copy(), o.V.copy(),
                np.float64(fl.rho), np.array([uref, pref, np.abs(o.U).max()]), zN, rs,
                partial))
            part = partial.reshape(nb, 8)
            key = f"{tag}_e{elim}"
            out.update({f"{key}_data": data, f"{key}_b": b.reshape(N, 4),
                        f"{key}_scale": rs.reshape(N, 4), f"{key}_max": part[:, 4:].max(0)})
    return out


def gpu_path_case() -> dict:
    """The reference's device solver (``GPUSolver``, ``zvcfd/fv/solver.py``: fast kernels, fused
    boundary pass, SuperLU on the host as its ``host-direct`` tests use) run on the CPU through
    :func:`_cpu_cupy`, on the pipe of its boundary tests (``tests/test_fv_boundaries.py:37-49``)
    with what only that path has: an RCR outlet coupled implicitly (``:86-109``), an
    average-static-pressure outlet (``:236-250``) and an opening inlet (``:253-266``). First
    the harness itself is held to the reference's CPU solver on the golden pipe (same fields to
    1e-13). Recorded per case: the converged ``U``, ``P``, the zone flows, pressures and forces,
    and the wall shear stress from consistent reactions."""
    sys.modules["cupy"] = _cpu_cupy()
    import os

    os.environ.setdefault("OMP_WAIT_POLICY", "PASSIVE")
    from zvcfd.fv.solver import GPUSolver
    from zvcfd.lumped import RCR

    R = 0.5
    m = tube(R, 2.0, n_core=2, n_ring=2, n_axial=8, kind="mixed", layers=1)
    z = {zz.name: k for k, zz in m.zones.items()}
    fluid = Fluid(1.0, 0.2)

    def run(bcs, tol):
        s = GPUSolver(m, fluid, bcs, linear="host-direct", linear_rtol=0.0, advection=1.0)
        rep = s.solve(max_iterations=300, tol=tol)
        assert rep.converged
        f = s.fields()
        return s, f

    # the harness: the golden pipe (parabolic inlet) as the CPU solver converged it
    g = np.load(HERE / "pipe_reference_tube.npz")

    def prof(x):
        r2 = (x[:, 0] ** 2 + x[:, 1] ** 2) / R ** 2
        return np.stack([0 * r2, 0 * r2, 2 * np.clip(1 - r2, 0, None)], 1)

    _, f = run({z["inlet"]: {"kind": "velocity", "value": prof},
                z["outlet"]: {"kind": "pressure", "value": 0.0}, z["wall"]: {"kind": "wall"}},
               1e-12)
    assert np.abs(f["U"] - g["U"]).max() < 1e-13 * np.abs(g["U"]).max()
    out = {}
    cases = {
        "rcr": {z["inlet"]: {"kind": "velocity", "flow_rate": 0.3, "profile": "poiseuille"},
                z["outlet"]: {"kind": "pressure", "lumped": RCR(rp=2.0, c=0.1, rd=5.0, pv=1.0)},
                z["wall"]: {"kind": "wall"}},
        "average": {z["inlet"]: {"kind": "velocity", "flow_rate": 0.3},
                    z["outlet"]: {"kind": "pressure", "value": 2.0, "profile": "average"},
                    z["wall"]: {"kind": "wall"}},
        "opening": {z["inlet"]: {"kind": "pressure", "value": 1.0, "opening": True},
                    z["outlet"]: {"kind": "pressure", "value": 0.0}, z["wall"]: {"kind": "wall"}},
    }
    for tag, bcs in cases.items():
        s, f = run(bcs, 1e-11)
        q, p = s.patch_flows(), s.patch_pressures()
        zids = sorted(q)
        forces = s.zone_forces()
        nodes, tau = s.wall_shear("reaction")
        out.update({f"{tag}_U": f["U"], f"{tag}_P": f["P"], f"{tag}_zones": np.array(zids),
                    f"{tag}_flows": np.array([q[k] for k in zids]),
                    f"{tag}_pressures": np.array([p[k] for k in zids]),
                    f"{tag}_forces": np.array([forces[k] for k in zids]),
                    f"{tag}_shear_nodes": np.asarray(nodes), f"{tag}_shear": np.asarray(tau)})
    return out


def gpu_path_transient_case() -> dict:
    """The reference's device solver run on the CPU (as :func:`gpu_path_case`) on its transient
    RCR test (``tests/test_fv_boundaries.py:112-129``), shortened for the CPU: the pipe with a
    pulsing flow-rate inlet ``Q(t) = 0.3 + 0.1 sin(2 pi t)`` and an RCR outlet, solved steady to
    1e-11, then 3 BDF2 steps of 0.05 with up to 20 coefficient loops to 1e-12. Recorded per
    step: the time, the outlet's flow and pressure; and the final ``U``, ``P``."""
    sys.modules["cupy"] = _cpu_cupy()
    import os

    os.environ.setdefault("OMP_WAIT_POLICY", "PASSIVE")
    from zvcfd.fv.solver import GPUSolver
    from zvcfd.lumped import RCR

    m = tube(0.5, 2.0, n_core=2, n_ring=2, n_axial=8, kind="mixed", layers=1)
    z = {zz.name: k for k, zz in m.zones.items()}

    def Q(t):
        return 0.3 + 0.1 * np.sin(2 * np.pi * t)

    bcs = {z["inlet"]: {"kind": "velocity", "flow_rate": Q, "profile": "poiseuille"},
           z["outlet"]: {"kind": "pressure", "lumped": RCR(rp=2.0, c=0.1, rd=5.0, pv=1.0)},
           z["wall"]: {"kind": "wall"}}
    s = GPUSolver(m, Fluid(1.0, 0.2), bcs, linear="host-direct", linear_rtol=0.0, advection=1.0)
    assert s.solve(max_iterations=300, tol=1e-11).converged
    rec = []
    s.solve_transient(0.05, 3, loops=20, tol=1e-12,
                      callback=lambda sv: rec.append((sv.t, sv.patch_flows()[z["outlet"]],
                                                      sv.patch_pressures()[z["outlet"]])))
    f = s.fields()
    return {"steps": np.array(rec), "U": f["U"], "P": f["P"]}


def reconstruction_case() -> dict:
    """The reference CPU solver's opt-in second-order boundary reconstruction
    (``boundary_reconstruction = True``, ``zvcfd/fv/reference.py:766-790``,
    ``zvcfd/fv/boundary_advection.py:167-219``) on the golden pipe (its own boundary tests'
    tube): the raw system after three outer iterations with a fixed blend, and the converged
    fields with a fixed blend and with High Resolution."""
    R = 0.5
    m = tube(R, 2.0, n_core=2, n_ring=2, n_axial=8, kind="mixed", layers=1)
    zid = {z.name: k for k, z in m.zones.items()}

    def prof(x):
        r2 = (x[:, 0] ** 2 + x[:, 1] ** 2) / R ** 2
        return np.stack([0 * r2, 0 * r2, 2 * np.clip(1 - r2, 0, None)], 1)

    def bcs():
        return {zid["inlet"]: {"kind": "velocity", "value": prof},
                zid["outlet"]: {"kind": "pressure", "value": 0.0}, zid["wall"]: {"kind": "wall"}}

    out = {}
    s = ReferenceSolver(m, Fluid(1.0, 0.2), bcs(), advection=1.0, lag_rhie_chow=True)
    s.boundary_reconstruction = True
    s.solve(max_iterations=3, tol=0.0)
    s.assemble()
    M, b = s._raw
    indptr, indices = node_graph(m)
    out.update(raw=blocks_on_pattern(M, indptr, indices), braw=b.reshape(-1, 4),
               U3=s.U.copy(), P3=s.P.copy(), mb3=s._mb.copy())
    for tag, adv in (("blend", 1.0), ("hr", "high-resolution")):
        s = ReferenceSolver(m, Fluid(1.0, 0.2), bcs(), advection=adv, lag_rhie_chow=True)
        s.boundary_reconstruction = True
        rep = s.solve(max_iterations=400, tol=1e-12)
        assert rep.converged
        out.update({f"{tag}_U": s.U, f"{tag}_P": s.P, f"{tag}_iterations": np.array(rep.iterations)})
    return out


def main():
    if sys.argv[1:] == ["reconstruction"]:
        np.savez_compressed(HERE / "reconstruction.npz", **reconstruction_case())
        print("wrote reconstruction")
        return
    if sys.argv[1:] == ["gpu_path_transient"]:
        np.savez_compressed(HERE / "gpu_path_transient.npz", **gpu_path_transient_case())
        print("wrote gpu_path_transient")
        return
    if sys.argv[1:] == ["gpu_path"]:
        np.savez_compressed(HERE / "gpu_path.npz", **gpu_path_case())
        print("wrote gpu_path")
        return
    if sys.argv[1:] == ["boundary"]:
        np.savez_compressed(HERE / "boundary_pass.npz", **boundary_case())
        print("wrote boundary_pass")
        return
    if sys.argv[1:] == ["acm"]:
        np.savez_compressed(HERE / "acm.npz", **acm_case())
        print("wrote acm")
        return
    if sys.argv[1:] == ["colour"]:
        np.savez_compressed(HERE / "colour.npz", **colour_case())
        print("wrote colour")
        return
    if sys.argv[1:] == ["partition"]:
        np.savez_compressed(HERE / "partition.npz", **partition_case())
        print("wrote partition")
        return
    if sys.argv[1:] == ["kernels"]:
        for name in MESHES:
            for gn, dt in VARIANTS:
                tag = f"kernel_{name}_{'gn' if gn else 'newt'}_{'dt' if dt else 'steady'}"
                np.savez_compressed(HERE / f"{tag}.npz", **kernel_case(name, gn, dt))
        print("wrote kernels")
        return
    if sys.argv[1:] == ["curved_mid"]:
        np.savez_compressed(HERE / "curved_mid.npz", **curved_mid_case())
        print("wrote curved_mid")
        return
    if sys.argv[1:] == ["variable_steps"]:
        np.savez_compressed(HERE / "variable_steps.npz", **variable_steps_case())
        print("wrote variable_steps")
        return
    if sys.argv[1:] == ["profiles"]:
        np.savez_compressed(HERE / "profiles.npz", **profiles_case())
        print("wrote profiles")
        return
    if sys.argv[1:] == ["gn_outlet"]:
        np.savez_compressed(HERE / "gn_outlet.npz", **gn_outlet_case())
        print("wrote gn_outlet")
        return
    if sys.argv[1:] == ["wss"]:
        np.savez_compressed(HERE / "wss.npz", **wss_case())
        print("wrote wss")
        return
    if sys.argv[1:] == ["forces"]:
        np.savez_compressed(HERE / "forces.npz", **forces_case())
        print("wrote forces")
        return
    if sys.argv[1:] == ["backflow"]:
        np.savez_compressed(HERE / "backflow_box.npz", **backflow_case())
        print("wrote backflow_box")
        return
    if sys.argv[1:] == ["lumped"]:
        np.savez_compressed(HERE / "lumped.npz", **lumped_case())
        print("wrote lumped")
        return
    if sys.argv[1:] == ["wall"]:
        np.savez_compressed(HERE / "wall_shear.npz", **wall_case())
        print("wrote wall_shear")
        return
    if sys.argv[1:] == ["transient"]:
        np.savez_compressed(HERE / "transient_pipe.npz", **transient_case())
        print("wrote transient_pipe")
        return
    tabs = {}
    for k in ("tet", "pyramid", "wedge", "hex"):
        t = topology(k)
        tabs.update({f"{k}_edges": t.edges, f"{k}_tris": t.tris, f"{k}_N": t.N_ip,
                     f"{k}_dN": t.dN_ip, f"{k}_W": t.point_weights, f"{k}_xi": t.xi_ip})
    np.savez_compressed(HERE / "tables.npz", **tabs)
    for name in MESHES:
        for gn, dt in VARIANTS:
            tag = f"kernel_{name}_{'gn' if gn else 'newt'}_{'dt' if dt else 'steady'}"
            np.savez_compressed(HERE / f"{tag}.npz", **kernel_case(name, gn, dt))
            print("wrote", tag)
    for tag, arrays in pipe_cases().items():
        np.savez_compressed(HERE / f"{tag}.npz", **arrays)
        print("wrote", tag, arrays["iterations"])
    np.savez_compressed(HERE / "transient_pipe.npz", **transient_case())
    print("wrote transient_pipe")
    np.savez_compressed(HERE / "wall_shear.npz", **wall_case())
    print("wrote wall_shear")
    np.savez_compressed(HERE / "lumped.npz", **lumped_case())
    print("wrote lumped")
    np.savez_compressed(HERE / "backflow_box.npz", **backflow_case())
    print("wrote backflow_box")
    np.savez_compressed(HERE / "forces.npz", **forces_case())
    print("wrote forces")
    np.savez_compressed(HERE / "wss.npz", **wss_case())
    print("wrote wss")
    np.savez_compressed(HERE / "gn_outlet.npz", **gn_outlet_case())
    print("wrote gn_outlet")
    np.savez_compressed(HERE / "profiles.npz", **profiles_case())
    print("wrote profiles")
    np.savez_compressed(HERE / "variable_steps.npz", **variable_steps_case())
    print("wrote variable_steps")
    np.savez_compressed(HERE / "partition.npz", **partition_case())
    print("wrote partition")
    np.savez_compressed(HERE / "colour.npz", **colour_case())
    print("wrote colour")
    np.savez_compressed(HERE / "acm.npz", **acm_case())
    print("wrote acm")
    np.savez_compressed(HERE / "boundary_pass.npz", **boundary_case())
    print("wrote boundary_pass")
    np.savez_compressed(HERE / "gpu_path.npz", **gpu_path_case())
    print("wrote gpu_path")
    np.savez_compressed(HERE / "gpu_path_transient.npz", **gpu_path_transient_case())
    print("wrote gpu_path_transient")
    np.savez_compressed(HERE / "reconstruction.npz", **reconstruction_case())
    print("wrote reconstruction")


if __name__ == "__main__":
    main()
