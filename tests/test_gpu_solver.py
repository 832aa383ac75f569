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


@pytest.mark.parametrize("strength", ["block", "pressure"])
def test_aggregation_is_bit_exact(strength):
    from zvcfd_b200.linear import B200AMG

    s, A, b, _ = _system("curved_cy")
    solver = B200AMG(strength=strength, precision="double")
    solver.setup(A)
    ip, ix = A.indptr.cpu().numpy(), A.indices.cpu().numpy()
    data = A.data.cpu().numpy()
    mode = 1 if strength == "pressure" else 0
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
