"""The oracle reproduces the reference's own outputs (golden vectors made by the reference)."""

import numpy as np
import pytest

from fixtures import KERNEL_MESHES, KERNEL_VARIANTS, kernel_case, load, mdot_of, oracle_kernel_outputs
from zvcfd_b200.topology import KINDS, tables


def test_tables_match_reference():
    g = load("tables")
    for k in KINDS:
        t = tables(k)
        np.testing.assert_array_equal(t.edge, g[f"{k}_edges"])
        np.testing.assert_array_equal(t.tris, g[f"{k}_tris"])
        np.testing.assert_array_equal(t.N_ip, g[f"{k}_N"])
        np.testing.assert_array_equal(t.dN_ip, g[f"{k}_dN"])
        np.testing.assert_array_equal(t.weights, g[f"{k}_W"])


def test_kernel_tables_restate_the_reference_tables():
    """The element kernels' forms of the tables (corner node masks, flux point as the fastest
    index) hold the same numbers: each triangle corner is the plain mean of its mask's nodes,
    and the transposed shape functions and derivatives are the reference's."""
    from zvcfd_b200.topology import _kernel_tables

    g = load("tables")
    for k in KINDS:
        t = tables(k)
        arrays = {name: a for name, a, _ in _kernel_tables(t)}
        W = g[f"{k}_W"][g[f"{k}_tris"]]                          # (n_ip, 3, n)
        bits = (arrays["MASK"][..., None] >> np.arange(t.n)) & 1
        np.testing.assert_array_equal(W > 0, bits.astype(bool))
        np.testing.assert_allclose(W, bits / bits.sum(-1, keepdims=True), rtol=0, atol=1e-16)
        np.testing.assert_array_equal(arrays["NT"], g[f"{k}_N"].T)
        dnt = arrays["DNT"].reshape(t.n, 3, t.n_ip)
        np.testing.assert_array_equal(dnt.transpose(2, 0, 1), g[f"{k}_dN"])
        np.testing.assert_array_equal(arrays["EDGE"], g[f"{k}_edges"])


@pytest.mark.parametrize("variant", KERNEL_VARIANTS)
@pytest.mark.parametrize("name", KERNEL_MESHES)
def test_oracle_matches_reference_kernels(name, variant):
    g = kernel_case(name, variant)
    o = oracle_kernel_outputs(g)
    np.testing.assert_array_equal(o["indptr"], g["indptr"])
    np.testing.assert_array_equal(o["indices"], g["indices"])
    np.testing.assert_allclose(o["V"], g["V"], rtol=1e-12)
    np.testing.assert_allclose(o["gradU"], g["gradU"], atol=1e-11)
    np.testing.assert_allclose(o["gradP"], g["gradP"], atol=1e-11)
    np.testing.assert_allclose(o["diag"], g["diag"], rtol=1e-11, atol=1e-12)
    np.testing.assert_allclose(o["beta_limiter"], g["beta_limiter"], atol=1e-12)
    scale = np.abs(g["data_raw"]).max()
    assert np.abs(o["data_raw"] - g["data_raw"]).max() < 1e-12 * scale
    np.testing.assert_allclose(o["b_raw"], g["b_raw"], atol=1e-12 * np.abs(g["b_raw"]).max())
    np.testing.assert_allclose(o["imbalance"], g["imbalance"],
                               atol=1e-12 * np.abs(g["imbalance"]).max())
    for k, v in mdot_of(g, "mdot_new").items():
        np.testing.assert_allclose(o["mdot_new"][k], v, atol=1e-12 * np.abs(v).max())


@pytest.mark.parametrize("name", ["pipe_reference_tube", "pipe_tet_si", "curved_cy"])
def test_oracle_reaches_reference_solution(name):
    from fixtures import fluid_of, mesh_of, pipe_bcs
    from oracle.fv import OracleSolver

    g = load(name)
    m = mesh_of(g)
    s = OracleSolver(m, fluid_of(g), pipe_bcs(name, g, m), advection=1.0)
    rep = s.solve(max_iterations=400, tol=1e-12)
    assert rep["converged"]
    np.testing.assert_allclose(s.U, g["U"], atol=1e-9 * np.abs(g["U"]).max())
    np.testing.assert_allclose(s.P, g["P"], atol=1e-9 * np.ptp(g["P"]))
    flows = s.zone_flows()
    assert abs(sum(flows.values())) < 1e-11 * sum(abs(v) for v in flows.values())


def test_oracle_transient_matches_reference():
    from fixtures import fluid_of, mesh_of, transient_bcs
    from oracle.fv import OracleSolver

    g = load("transient_pipe")
    m = mesh_of(g)
    s = OracleSolver(m, fluid_of(g), transient_bcs(g, m), advection=1.0)
    rep = s.solve(max_iterations=400, tol=1e-12)
    assert rep["converged"]
    np.testing.assert_allclose(s.U, g["U0"], atol=1e-9 * np.abs(g["U0"]).max())
    s.solve_transient(float(g["dt"]), int(g["steps"]), scheme="bdf2", loops=int(g["loops"]),
                      tol=float(g["tol"]))
    np.testing.assert_allclose(s.U, g["U"], atol=1e-9 * np.abs(g["U"]).max())
    np.testing.assert_allclose(s.P, g["P"], atol=1e-9 * np.ptp(g["P"]))


@pytest.mark.parametrize("tag,beta", [("stab", 0.5), ("plain", 0.0)])
def test_oracle_backflow_stabilisation_matches_reference(tag, beta):
    """The reference's backflow box: part of the outlet carries inflow (m_b < 0), where the
    stabilisation adds beta max(-m_b, 0) to the outflow momentum weight."""
    from fixtures import backflow_bcs, fluid_of, mesh_of
    from oracle.fv import OracleSolver

    g = load("backflow_box")
    m = mesh_of(g)
    bcs = backflow_bcs(m, beta)
    s = OracleSolver(m, fluid_of(g), bcs, advection=1.0)
    rep = s.solve(max_iterations=200, tol=1e-12)
    assert rep["converged"]
    U, P = g[f"U_{tag}"], g[f"P_{tag}"]
    np.testing.assert_allclose(s.U, U, atol=1e-9 * np.abs(U).max())
    np.testing.assert_allclose(s.P, P, atol=1e-9 * np.ptp(P))
    assert (s._mb[s.outlet] < 0).any() and (s._mb[s.outlet] > 0).any()


def test_oracle_manufactured_carreau_outlet_matches_reference():
    """The reference's Carreau-Yasuda manufactured outlet (``tests/test_fv_solver_gpu.py``
    ``:76-101``): body force, prescribed outlet gradient (traction), transpose term."""
    from fixtures import gn_outlet_bcs, gn_outlet_fluid, mesh_of, tabulated
    from oracle.fv import OracleSolver

    g = load("gn_outlet")
    m = mesh_of(g)
    s = OracleSolver(m, gn_outlet_fluid(g), gn_outlet_bcs(g, m),
                     source=tabulated(g["points"], g["f"]), advection=1.0, transpose=True)
    assert s.solve(max_iterations=300, tol=1e-13)["converged"]
    np.testing.assert_allclose(s.U, g["U"], atol=1e-11 * np.abs(g["U"]).max())
    np.testing.assert_allclose(s.P, g["P"], atol=1e-11 * np.ptp(g["P"]))


@pytest.mark.parametrize("name", ["pipe_reference_tube", "curved_cy"])
def test_oracle_wall_shear_matches_reference(name):
    from fixtures import fluid_of, mesh_of
    from oracle.wall import wall_shear

    g = load(name)
    m = mesh_of(g)
    fl = fluid_of(g)
    wall = [z for z, zz in m.zones.items() if zz.name == "wall"]
    tau = wall_shear(m, wall, g["U"], mu=fl.mu, viscosity=fl.viscosity)
    ref = load("wall_shear")[f"{name}_tau"]
    np.testing.assert_allclose(tau, ref, atol=1e-12 * np.abs(ref).max())


def test_symmetrised_strength_keeps_pairwise_coarsening_under_convection():
    """On a 12^3 lattice with one strong upstream coupling per node (a convective 4x4 block
    system), the one-sided block-norm strength of the ACM's matching points every node at its
    upstream neighbour, mutual pairs become rare and two passes leave 55 % of the rows; the
    strength averaged over both directions of each coupling keeps the matching near 4:1."""
    from oracle.linear import aggregate, transpose_positions

    rng = np.random.default_rng(0)
    nx = 12
    n = nx ** 3
    idx = np.arange(n).reshape(nx, nx, nx)
    rows, cols, vals = [], [], []
    for d in [(0, 0, 0), (1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, 1), (0, 0, -1)]:
        sl = tuple(slice(max(0, -k), nx - max(0, k)) for k in d)
        sh = tuple(slice(max(0, k), nx - max(0, -k)) for k in d)
        a, b = idx[sl].ravel(), idx[sh].ravel()
        if d == (0, 0, 0):
            v = np.full(len(a), 10.0)
        elif d == (-1, 0, 0):
            v = -(5.0 + 0.1 * rng.random(len(a)))
        else:
            v = -(0.5 + 0.1 * rng.random(len(a)))
        rows.append(a), cols.append(b), vals.append(v)
    rows, cols, vals = (np.concatenate(x) for x in (rows, cols, vals))
    o = np.lexsort((cols, rows))
    rows, cols, vals = rows[o], cols[o], vals[o]
    ip = np.zeros(n + 1, np.int64)
    np.cumsum(np.bincount(rows, minlength=n), out=ip[1:])
    pos = transpose_positions(ip, cols)
    np.testing.assert_array_equal(rows[pos], cols)
    np.testing.assert_array_equal(cols[pos], rows)
    data = vals[:, None, None] * np.eye(4)[None]
    _, one_sided = aggregate(ip, cols, data, 2, 0)
    _, symmetric = aggregate(ip, cols, data, 2, 2)
    assert one_sided > 0.5 * n
    assert symmetric < 0.25 * n


def test_array_matching_equals_the_node_by_node_matching():
    """The whole-array pairwise matching (the CPU baseline's) picks, ties and numbers the
    aggregates exactly as the node-by-node restatement: on an assembled golden system (both
    strength modes, both passes) and on random strengths with many exact ties."""
    from fixtures import fluid_of, mesh_of, pipe_bcs
    from oracle.fv import OracleSolver
    from oracle.linear import aggregate, pairwise, pairwise_arrays

    g = load("pipe_tet_si")
    m = mesh_of(g)
    s = OracleSolver(m, fluid_of(g), pipe_bcs("pipe_tet_si", g, m), advection=1.0)
    s.solve(max_iterations=2, tol=0.0)
    data, _ = s.assemble()
    for mode in (0, 2):
        a1, n1 = aggregate(s.indptr, s.indices, data, 2, mode)
        a2, n2 = aggregate(s.indptr, s.indices, data, 2, mode, pairwise_arrays)
        assert n1 == n2
        np.testing.assert_array_equal(a1, a2)
    rng = np.random.default_rng(3)
    n = 400
    for trial in range(5):
        dense = rng.random((n, n)) < 0.02
        dense = dense | dense.T | np.eye(n, dtype=bool)
        if trial == 4:
            dense[:50] = dense[:, :50] = False           # isolated rows: singletons
            dense[np.arange(n), np.arange(n)] = True
        rows, cols = np.nonzero(dense)
        ptr = np.zeros(n + 1, np.int64)
        np.cumsum(np.bincount(rows, minlength=n), out=ptr[1:])
        strength = rng.integers(0, 4, len(cols)).astype(float)     # many ties
        a1, n1 = pairwise(n, ptr, cols, strength)
        a2, n2 = pairwise_arrays(n, ptr, cols, strength)
        assert n1 == n2
        np.testing.assert_array_equal(a1, a2)


def test_oracle_acm_fgmres_solves_an_assembled_system():
    """The oracle's linear solver (the reference ACM's V-cycle inside FGMRES) on a Dirichlet
    system the oracle assembled for a golden pipe reaches the direct solution."""
    import scipy.sparse.linalg as spl

    from fixtures import fluid_of, mesh_of, pipe_bcs
    from oracle.fv import OracleSolver
    from oracle.linear import ACM, fgmres

    g = load("pipe_tet_si")
    m = mesh_of(g)
    s = OracleSolver(m, fluid_of(g), pipe_bcs("pipe_tet_si", g, m), advection=1.0)
    s.solve(max_iterations=3, tol=0.0)
    data, b = s.assemble()
    A = s.to_csr(data)
    amg = ACM().setup(s.indptr, s.indices, data)
    assert len(amg.levels) >= 2
    x, its, res, ok = fgmres(lambda v: A @ v, b.reshape(-1), np.zeros(b.size), amg.vcycle,
                             rtol=1e-10, maxiter=300)
    assert ok and res <= 1e-10 * 1.01
    assert np.linalg.norm(A @ x - b.reshape(-1)) <= 1.01e-10 * np.linalg.norm(b)
    # the system's condition number is about 7e7: the fields agree to that times the residual
    X, R = x.reshape(-1, 4), spl.spsolve(A.tocsc(), b.reshape(-1)).reshape(-1, 4)
    assert np.abs(X[:, :3] - R[:, :3]).max() < 1e-5 * np.abs(R[:, :3]).max()
    assert np.abs(X[:, 3] - R[:, 3]).max() < 1e-5 * np.ptp(R[:, 3])


@pytest.mark.parametrize("name", ["pipe_tet_si", "curved_cy"])
def test_oracle_boundary_pass_keeps_the_solution(name):
    """The restated boundary pass: symmetric elimination and the dimensionless row scaling
    leave the solution of the Dirichlet system unchanged, the eliminated columns are empty,
    fixed rows are scaled unit rows, and the residual sums are those of the state."""
    import scipy.sparse.linalg as spl

    from fixtures import fluid_of, mesh_of, pipe_bcs
    from oracle.fv import OracleSolver

    g = load(name)
    m = mesh_of(g)
    s = OracleSolver(m, fluid_of(g), pipe_bcs(name, g, m), advection=1.0)
    s.solve(max_iterations=3, tol=0.0)
    dirichlet, b_dir = s.assemble()
    raw, b_raw = s.raw
    X = np.concatenate([s.U, s.P[:, None]], 1)
    ref = spl.spsolve(s.to_csr(dirichlet).tocsc(), b_dir.reshape(-1))
    for eliminate in (True, False):
        data, b, scale, stats = s.boundary_pass(raw, b_raw, X, eliminate=eliminate)
        x = spl.spsolve(s.to_csr(data).tocsc(), b.reshape(-1))
        np.testing.assert_allclose(x, ref, rtol=1e-9, atol=1e-12 * np.abs(ref).max())
        fixed = np.concatenate([s.vel_fixed_comp, s.p_fixed[:, None]], 1)
        rows = np.repeat(np.arange(s.N), np.diff(s.indptr))
        if eliminate:                      # free rows keep nothing in known columns
            for r in range(4):
                for c in range(4):
                    assert np.all(data[fixed[s.indices, c] & ~fixed[rows, r], r, c] == 0.0)
        dpos = s.diagonal_positions()
        for r in range(4):
            on = np.flatnonzero(fixed[:, r])
            np.testing.assert_allclose(data[dpos[on], r, r], scale[on, r], rtol=1e-15)
    # residual sums of the free rows, computed directly from the Dirichlet system
    res = (b_dir.reshape(-1) - s.to_csr(dirichlet) @ X.reshape(-1)).reshape(-1, 4)
    norm = np.concatenate([np.repeat(s.aP[:, None], 3, 1),
                           (s.fluid.rho * s.V ** (2 / 3))[:, None]], 1)
    v = np.where(fixed, 0.0, np.abs(res) / norm)
    np.testing.assert_allclose(stats["max"], v.max(0), rtol=1e-10, atol=1e-300)
    np.testing.assert_allclose(stats["sq"], (v * v).sum(0), rtol=1e-10, atol=1e-300)


def test_oracle_variable_steps_match_reference():
    """Six uneven BDF2 steps of the reference's oscillating-pressure tube
    (``tests/test_fv_boundaries.py:281-300``): the oracle's variable-step coefficients and time
    levels reach the reference's fields."""
    from fixtures import mesh_of
    from oracle.fv import OracleSolver
    from zvcfd_b200.fluid import Fluid

    g = load("variable_steps")
    m = mesh_of(g)
    z = {zz.name: k for k, zz in m.zones.items()}
    w = float(g["omega"])
    bcs = {z["inlet"]: {"kind": "pressure",
                        "value": lambda x, t: 0.5 * np.cos(w * t) * np.ones(len(x))},
           z["outlet"]: {"kind": "pressure", "value": 0.0}, z["wall"]: {"kind": "wall"}}
    s = OracleSolver(m, Fluid(1.0, float(g["nu"])), bcs, advection=1.0)
    s.solve_transient(list(g["steps"]), loops=60, tol=1e-12)
    np.testing.assert_allclose(s.U, g["U"], atol=1e-11)
    np.testing.assert_allclose(s.P, g["P"], atol=1e-11 * max(np.ptp(g["P"]), 1e-30))


@pytest.mark.parametrize("stokes", [True, False])
def test_oracle_symmetry_plane_reproduces_the_full_channel(stokes):
    """The reference's half-channel property (``tests/test_fv_reference.py:105-135``): a
    channel of height 1 with a symmetry plane on top equals the lower half of the channel of
    height 2 with two walls, to round-off, with symmetry planes on both z faces too."""
    from oracle.fv import OracleSolver
    from zvcfd_b200.fluid import Fluid
    from zvcfd_b200.mesh import box

    halves = {}
    for H, ny in ((2.0, 8), (1.0, 4)):
        m = box((6, ny, 2), (3.0, H, 0.5), kind="hex")
        z = {zz.name: k for k, zz in m.zones.items()}

        def inflow(x):
            u = np.zeros((len(x), 3))
            u[:, 0] = x[:, 1] * (2.0 - x[:, 1])
            return u

        bcs = {z["xmin"]: {"kind": "velocity", "value": inflow},
               z["xmax"]: {"kind": "pressure", "value": 0.0}, z["ymin"]: {"kind": "wall"},
               z["zmin"]: {"kind": "symmetry"}, z["zmax"]: {"kind": "symmetry"},
               z["ymax"]: {"kind": "wall"} if H == 2.0 else {"kind": "symmetry"}}
        s = OracleSolver(m, Fluid(1.0, 0.5), bcs, stokes=stokes)
        assert s.solve(max_iterations=60, tol=1e-12)["converged"]
        q = s.zone_flows()
        assert abs(sum(q.values())) < 1e-13 * abs(q[z["xmin"]])
        lower = m.nodes[:, 1] <= 1.0 + 1e-9
        order = np.lexsort(np.round(m.nodes[lower] * 1e6).astype(np.int64).T[::-1])
        halves[H] = (s.U[lower][order], s.P[lower][order])
    np.testing.assert_allclose(halves[1.0][0], halves[2.0][0], atol=1e-12)
    np.testing.assert_allclose(halves[1.0][1], halves[2.0][1], atol=1e-12)


@pytest.mark.parametrize("kind,perturb", [("tet", 0.25), ("tet", 0.0), ("wedge", 0.0),
                                          ("hex", 0.0)])
def test_oracle_hydrostatic_is_exact(kind, perturb):
    """The reference's exactness check (``tests/test_fv_reference.py:25-36``): at rest, a
    uniform body force balanced by a linear pressure, to round-off. The lagged Rhie-Chow
    iteration reaches it as its fixed point (the reference's implicit form in one solve)."""
    from oracle.fv import OracleSolver
    from zvcfd_b200.fluid import Fluid
    from zvcfd_b200.mesh import box

    m = box((5, 5, 5), kind=kind, perturb=perturb, seed=1)
    g = np.array([0.3, -1.1, 0.7])
    p = m.nodes @ g
    s = OracleSolver(m, Fluid(), {z: {"kind": "wall"} for z in m.zones}, stokes=True,
                     source=lambda x: np.broadcast_to(g, (len(x), 3)),
                     reference_pressure=(0, float(p[0])))
    s.solve(max_iterations=200, tol=0.0)
    assert np.abs(s.U).max() < 1e-12
    assert np.abs(s.P - p).max() < 1e-11


@pytest.mark.parametrize("perturb", [0.0, 0.2])
@pytest.mark.parametrize("kind", ["tet", "wedge", "hex"])
def test_oracle_couette_is_exact_on_affine_elements(kind, perturb):
    """A linear shear flow (``tests/test_fv_reference.py:39-60``): exact on every affine
    element (all tetrahedra, undistorted wedges and hexahedra), close on distorted ones."""
    from oracle.fv import OracleSolver
    from zvcfd_b200.fluid import Fluid
    from zvcfd_b200.mesh import box

    def shear(x):
        u = np.zeros((len(x), 3))
        u[:, 0] = 0.5 + 2.0 * x[:, 2] - x[:, 1]
        return u

    m = box((4, 4, 4), kind=kind, perturb=perturb, seed=2)
    s = OracleSolver(m, Fluid(1.0, 0.7), {z: {"kind": "velocity", "value": shear}
                                          for z in m.zones}, stokes=True,
                     reference_pressure=(0, 0.0))
    s.solve(max_iterations=3)
    err = np.abs(s.U - shear(m.nodes)).max() / 2.5
    affine = kind == "tet" or perturb == 0
    assert err < (1e-12 if affine else 5e-4)
    if affine:
        assert np.abs(s.P).max() < 1e-10


def test_oracle_steady_state_does_not_depend_on_the_false_time_step():
    """The reference's check (``tests/test_fv_reference.py:165-179``): relaxing with a false
    time step reaches the same steady state (the transient Rhie-Chow part cancels there)."""
    from fixtures import fluid_of, mesh_of, pipe_bcs
    from oracle.fv import OracleSolver

    g = load("pipe_reference_tube")
    m = mesh_of(g)
    bcs = pipe_bcs("pipe_reference_tube", g, m)
    for dt in (0.05, 0.5):
        s = OracleSolver(m, fluid_of(g), bcs, advection=1.0, dt=dt)
        assert s.solve(max_iterations=600, tol=1e-13)["converged"]
        np.testing.assert_allclose(s.P, g["P"], atol=1e-10 * np.ptp(g["P"]))
        np.testing.assert_allclose(s.U, g["U"], atol=1e-10 * np.abs(g["U"]).max())


def test_oracle_lumped_outlet_reaches_its_0d_law():
    """The oracle's lumped RCR outlet (implicit rows ``p_j - r Q = a``): at the steady state
    the outlet pressure is ``a + r Q`` of the model's resting pair, and over BDF2 steps of a
    pulsing inflow it follows the standalone 0-D model fed with the same flows (the laws of
    the reference's ``tests/test_fv_boundaries.py:88-130``)."""
    from fixtures import axial_parabola, fluid_of, mesh_of, pipe_bcs
    from oracle.fv import OracleSolver
    from zvcfd_b200.lumped import RCR

    g = load("pipe_reference_tube")
    m = mesh_of(g)
    z = {zz.name: k for k, zz in m.zones.items()}
    bcs = pipe_bcs("pipe_reference_tube", g, m)
    pulse = axial_parabola(float(g["radius"]), float(g["umax"]),
                           pulse=lambda t: 1.0 + 0.5 * np.sin(2 * np.pi * t / 0.8))
    bcs[z["inlet"]] = {"kind": "velocity", "value": pulse}
    model = RCR(rp=0.5, c=1e-3, rd=2.0, pv=1.0)
    bcs[z["outlet"]] = {"kind": "pressure", "lumped": model}
    s = OracleSolver(m, fluid_of(g), bcs, advection=1.0)
    assert s.solve(max_iterations=400, tol=1e-12)["converged"]
    nodes = s._zone_nodes[z["outlet"]]
    rho = s.fluid.rho
    q = s.zone_flows()
    a, r = RCR(rp=0.5, c=1e-3, rd=2.0, pv=1.0).steady_coefficients()
    np.testing.assert_allclose(s.P[nodes], a + r * q[z["outlet"]] / rho, rtol=1e-12)
    assert abs(sum(q.values())) < 1e-12 * sum(abs(v) for v in q.values())
    alone = RCR(rp=0.5, c=1e-3, rd=2.0, pv=1.0)
    alone.initialise(q[z["outlet"]] / rho, 0.0)
    seen = []
    for _ in range(3):
        s.solve_transient(0.05, 1, loops=200, tol=1e-12)
        Q = s.zone_flows()[z["outlet"]] / rho
        np.testing.assert_allclose(s.P[nodes], alone.advance(Q, s.t, 0.05), rtol=1e-10)
        seen.append(Q)
    assert np.ptp(seen) > 0.05 * abs(seen[0])          # the flow did change


def test_oracle_poiseuille_pipe_balances_mass_and_converges_at_second_order():
    """The reference's ``tests/test_fv_reference.py:82-104`` on the oracle: a Stokes
    Poiseuille pipe on hexahedra carries its inflow out to round-off, and its pressure gradient
    approaches ``8 mu U / R^2`` at second order under refinement."""
    from fixtures import axial_parabola
    from oracle.fv import OracleSolver
    from zvcfd_b200.fluid import Fluid
    from zvcfd_b200.mesh import pipe

    R, L = 0.5, 3.0
    errors = []
    for nc in (2, 4):
        m = pipe(R, L, n_core=nc, n_ring=nc, n_axial=6 * nc, kind="hex")
        z = {zz.name: k for k, zz in m.zones.items()}
        s = OracleSolver(m, Fluid(), {z["inlet"]: {"kind": "velocity",
                                                   "value": axial_parabola(R, 2.0)},
                                      z["outlet"]: {"kind": "pressure", "value": 0.0},
                                      z["wall"]: {"kind": "wall"}}, stokes=True)
        assert s.solve(max_iterations=300, tol=1e-10)["converged"]
        q = s.zone_flows()
        assert abs(q[z["outlet"]] + q[z["inlet"]]) < 1e-12 * abs(q[z["inlet"]])
        zc = m.nodes[:, 2]
        drop = s.P[np.isclose(zc, 0.25 * L)].mean() - s.P[np.isclose(zc, 0.75 * L)].mean()
        errors.append(abs(drop / (0.5 * L) / (8 / R ** 2) - 1))
    assert errors[1] < 0.04
    assert np.log2(errors[0] / errors[1]) > 1.8
