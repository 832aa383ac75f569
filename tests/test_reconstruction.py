"""The opt-in second-order boundary reconstruction against the reference's CPU solver.

``tests/golden/reconstruction.npz`` holds the reference's ``ReferenceSolver`` with
``boundary_reconstruction = True`` (``zvcfd/fv/reference.py:766-790``,
``zvcfd/fv/boundary_advection.py:167-219``) on the golden pipe: the raw system after three
outer iterations with a fixed blend, and the converged fields with a fixed blend and with High
Resolution (whose limiter, and with it the sub-face factors, freezes). The oracle must give
the same raw system (1e-13) and converged fields (1e-12) in the same iteration counts; the
device path's tables, neighbour range and boundary moments (torch, here on CPU tensors) must
equal the oracle's.
"""

import numpy as np
import pytest
import torch

from fixtures import fluid_of, load, mesh_of, pipe_bcs
from oracle.fv import OracleSolver

G = load("reconstruction")


def _solver(advection):
    g = load("pipe_reference_tube")
    m = mesh_of(g)
    s = OracleSolver(m, fluid_of(g), pipe_bcs("pipe_reference_tube", g, m), advection=advection)
    s.boundary_reconstruction = True
    return g, m, s


def test_oracle_raw_system_equals_the_reference():
    _, _, s = _solver(1.0)
    s.solve(max_iterations=3, tol=0.0)
    np.testing.assert_allclose(s.U, G["U3"], rtol=0, atol=1e-13 * np.abs(G["U3"]).max())
    s.assemble()
    raw, braw = s.raw
    np.testing.assert_allclose(raw, G["raw"], rtol=0, atol=1e-13 * np.abs(G["raw"]).max())
    np.testing.assert_allclose(braw, G["braw"], rtol=0, atol=1e-13 * np.abs(G["braw"]).max())


@pytest.mark.parametrize("tag,advection", [("blend", 1.0), ("hr", "high-resolution")])
def test_oracle_converges_to_the_reference_fields(tag, advection):
    g, _, s = _solver(advection)
    rep = s.solve(max_iterations=400, tol=1e-12)
    assert rep["converged"] and rep["iterations"] == int(G[f"{tag}_iterations"])
    U, P = G[f"{tag}_U"], G[f"{tag}_P"]
    np.testing.assert_allclose(s.U, U, rtol=0, atol=1e-12 * np.abs(U).max())
    np.testing.assert_allclose(s.P, P, rtol=0, atol=1e-12 * np.ptp(P))
    # the reconstruction does change the solution (by about 2 % of the largest velocity)
    assert np.abs(s.U - g["U"]).max() > 1e-2 * np.abs(g["U"]).max()


def test_device_tables_range_and_moments_equal_the_oracle():
    from zvcfd_b200.boundary import Boundary
    from zvcfd_b200.solver import boundary_moments, neighbour_range

    g, m, s = _solver(1.0)
    s.solve(max_iterations=3, tol=0.0)
    gradU = s.nodal_gradient(s.U)
    beta = s.beta_for(gradU)
    want = s.boundary_moments(gradU, beta)
    O = s._bsf_tables
    T = Boundary(m, pipe_bcs("pipe_reference_tube", g, m), float(g["rho"])).reconstruction_tables()
    np.testing.assert_array_equal(T["node"], O["node"])
    np.testing.assert_array_equal(T["corners"], O["corners"])
    np.testing.assert_array_equal(T["outflow_only"], O["oonly"])
    for k, o in (("W", "W"), ("S", "S"), ("dx", "dx")):
        np.testing.assert_allclose(T[k], O[o], rtol=0, atol=1e-15 * np.abs(O[o]).max())
    rows = torch.as_tensor(np.repeat(np.arange(s.N), np.diff(s.indptr)))
    U = torch.as_tensor(s.U)
    lo, hi = neighbour_range(U, rows, torch.as_tensor(s.indices.astype(np.int64)))
    starts = s.indptr[:-1]
    np.testing.assert_array_equal(lo.numpy(), np.minimum.reduceat(s.U[s.indices], starts, axis=0))
    np.testing.assert_array_equal(hi.numpy(), np.maximum.reduceat(s.U[s.indices], starts, axis=0))
    Tt = {k: torch.as_tensor(v) for k, v in T.items()}
    D, bsf = boundary_moments(Tt, U, torch.as_tensor(s._mb), torch.as_tensor(gradU),
                              torch.as_tensor(np.broadcast_to(beta, (s.N, 3)).copy()), lo, hi,
                              s.fluid.rho, torch.as_tensor(s.sym))
    assert np.abs(want).max() > 0
    np.testing.assert_allclose(D.numpy(), want, rtol=0, atol=1e-14 * np.abs(want).max())
    # frozen factors are used as given
    D2, bsf2 = boundary_moments(Tt, U, torch.as_tensor(s._mb), torch.as_tensor(gradU), None,
                                None, None, s.fluid.rho, torch.as_tensor(s.sym), bsf=bsf)
    assert bsf2 is bsf and torch.equal(D2, D)
