"""The B200 linear back end and outer loop reach the reference's solutions.

- The device aggregation is the oracle's, bit for bit (integer work); the hierarchy sizes
  agree with the oracle's Galerkin products.
- FGMRES with the device AMG solves an assembled system to the direct solution.
- The outer loop (lagged Rhie-Chow, linear solves to 0.1) reaches the converged fields of the
  reference's CPU solver (golden vectors) on three pipes, in FP64 and with the FP32 hierarchy.
"""

import numpy as np
import pytest
import torch

from fixtures import PIPES, fluid_of, load, mesh_of, pipe_bcs
from oracle.linear import aggregate, bsr, galerkin

pytestmark = pytest.mark.gpu


def _system(name="pipe_tet_si", iterations=3):
    """An assembled, scaled system of a golden pipe after a few outer iterations."""
    from zvcfd_b200.solver import B200Solver

    g = load(name)
    m = mesh_of(g)
    s = B200Solver(m, fluid_of(g), pipe_bcs(name, g, m), advection=1.0)
    for _ in range(iterations):
        s.iterate()
    A, b, _, x0 = s._assemble_fused()
    return s, A, b.reshape(-1).clone(), x0


@pytest.mark.parametrize("strength", ["symmetric", "block", "pressure"])
def test_aggregation_is_bit_exact(strength):
    from zvcfd_b200.linear import B200AMG

    s, A, b, _ = _system("curved_cy")
    solver = B200AMG(strength=strength, precision="double")
    solver.setup(A)
    ip, ix = A.indptr.cpu().numpy(), A.indices.cpu().numpy()
    data = A.data.cpu().numpy()
    mode = {"block": 0, "pressure": 1, "symmetric": 2}[strength]
    level = 0
    while True:
        n, nnz, nc, agg = solver.level(level, with_aggregates=True)
        assert n == len(ip) - 1 and nnz == len(ix)
        if not nc:
            break
        ref, rnc = aggregate(ip, ix, data, 2, mode)
        assert nc == rnc
        np.testing.assert_array_equal(agg.cpu().numpy(), ref)
        ip, ix, data = galerkin(ip, ix, data, ref, rnc)
        level += 1
    solver.close()
    s.close()


@pytest.mark.parametrize("precision", ["double", "mixed"])
def test_fgmres_amg_solves_to_direct_solution(precision):
    import scipy.sparse.linalg as spl

    from zvcfd_b200.linear import B200AMG

    s, A, b, x0 = _system("pipe_tet_si")
    solver = B200AMG(precision=precision, rtol=1e-10, maxiter=400)
    x, info = solver.solve(A, b, x0)
    assert info.converged, info
    M = bsr(A.indptr.cpu().numpy(), A.indices.cpu().numpy(), A.data.cpu().numpy(), A.n).tocsc()
    ref = spl.splu(M).solve(b.cpu().numpy())
    np.testing.assert_allclose(x.cpu().numpy(), ref, atol=1e-7 * np.abs(ref).max())
    r = b.cpu().numpy() - M @ x.cpu().numpy()
    r0 = b.cpu().numpy() - M @ x0.cpu().numpy()
    assert np.linalg.norm(r) <= 1.01e-10 * np.linalg.norm(r0) + 1e-13 * np.linalg.norm(b.cpu().numpy())
    solver.close()
    s.close()


@pytest.mark.parametrize("linear", ["b200", "b200-mixed"])
@pytest.mark.parametrize("name", PIPES)
def test_pipe_matches_reference(name, linear):
    from zvcfd_b200.solver import B200Solver

    g = load(name)
    m = mesh_of(g)
    s = B200Solver(m, fluid_of(g), pipe_bcs(name, g, m), advection=1.0, linear=linear)
    rep = s.solve(max_iterations=800, tol=1e-11)
    assert rep["converged"], rep["history"][-1]
    f = s.fields()
    U, P = g["U"], g["P"]
    assert np.linalg.norm(f["U"] - U) <= 1e-8 * np.linalg.norm(U)
    assert np.linalg.norm(f["P"] - P) <= 1e-8 * np.linalg.norm(P - P.mean()) + 1e-9 * np.ptp(P)
    np.testing.assert_allclose(f["U"], U, atol=1e-8 * np.abs(U).max())
    np.testing.assert_allclose(f["P"], P, atol=1e-8 * np.ptp(P))
    assert abs(rep["history"][-1]["imbalance"]) < 1e-11
    s.close()


def test_transient_bdf2_matches_reference():
    from fixtures import transient_bcs
    from zvcfd_b200.solver import B200Solver

    g = load("transient_pipe")
    m = mesh_of(g)
    s = B200Solver(m, fluid_of(g), transient_bcs(g, m), advection=1.0, linear_rtol=0.1)
    rep = s.solve(max_iterations=800, tol=1e-11)
    assert rep["converged"]
    np.testing.assert_allclose(s.fields()["U"], g["U0"], atol=1e-8 * np.abs(g["U0"]).max())
    rep = s.solve_transient(float(g["dt"]), int(g["steps"]), scheme="bdf2", loops=int(g["loops"]),
                            tol=float(g["tol"]))
    assert rep["converged"]
    f = s.fields()
    np.testing.assert_allclose(f["U"], g["U"], atol=1e-8 * np.abs(g["U"]).max())
    np.testing.assert_allclose(f["P"], g["P"], atol=1e-8 * np.ptp(g["P"]))
    s.close()


def test_steady_rcr_outlet_reaches_its_0d_law():
    """A steady RCR outlet ends at p = a + r Q with Q the outlet's flow (the property of the
    reference's tests/test_fv_boundaries.py:88-110), and the mass balance is exact."""
    from zvcfd_b200.lumped import RCR
    from zvcfd_b200.solver import B200Solver

    g = load("pipe_reference_tube")
    m = mesh_of(g)
    bcs = pipe_bcs("pipe_reference_tube", g, m)
    z = {zz.name: k for k, zz in m.zones.items()}
    model = RCR(rp=0.5, c=1e-3, rd=2.0)
    bcs[z["outlet"]] = {"kind": "pressure", "value": 0.0, "lumped": model}
    s = B200Solver(m, fluid_of(g), bcs, advection=1.0)
    rep = s.solve(max_iterations=800, tol=1e-11)
    assert rep["converged"], rep["history"][-1]
    q = s.patch_flows()
    Q = q[z["outlet"]]
    P = s.fields()["P"]
    nodes = np.unique(m.zones[z["outlet"]].faces)
    nodes = nodes[nodes >= 0]
    a, r = model.steady_coefficients()
    np.testing.assert_allclose(P[nodes], a + r * Q, rtol=1e-8, atol=1e-10)
    assert abs(sum(q.values())) < 1e-11 * sum(abs(v) for v in q.values())
    s.close()


@pytest.mark.parametrize("name", ["pipe_reference_tube", "curved_cy"])
def test_wall_shear_matches_reference(name):
    from zvcfd_b200.wall import WallShear

    g = load(name)
    m = mesh_of(g)
    fl = fluid_of(g)
    wall = [z for z, zz in m.zones.items() if zz.name == "wall"]
    tau = WallShear(m, wall)(g["U"], viscosity=fl.viscosity, mu=fl.mu).cpu().numpy()
    ref = load("wall_shear")[f"{name}_tau"]
    np.testing.assert_allclose(tau, ref, atol=1e-12 * np.abs(ref).max())
