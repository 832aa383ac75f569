"""The solver's surface beyond one outer iteration, against the reference's own outputs: zone
forces and both wall-shear methods on the reference's zone-force pipe, and the reference's
manufactured Carreau-Yasuda outlet (body force, prescribed outlet gradient, transpose term)."""

import numpy as np
import pytest

from fixtures import load, mesh_of

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("tag", ["pipe"])
def test_zone_forces_and_wall_shear_match_reference(tag):
    """The reference's ``test_zone_forces_match_reference`` (``tests/test_fv_solver_gpu.py``
    ``:129-141``, forces to 1e-8 of their scale) on its pipe, and both ``wall_shear`` methods
    against the reference device solver's own evaluation of the converged state."""
    from fixtures import forces_case
    from zvcfd_b200.fluid import Fluid
    from zvcfd_b200.solver import B200Solver

    m, bcs, sub = forces_case(load("forces"), tag)
    s = B200Solver(m, Fluid(1.0, float(sub["mu"])), bcs, advection=1.0)
    rep = s.solve(max_iterations=800, tol=1e-11)
    assert rep["converged"], rep["history"][-1]
    F = s.zone_forces()
    ref = sub["forces"]
    got = np.array([F[int(z)] for z in sub["force_zones"]])
    np.testing.assert_allclose(got, ref, atol=1e-8 * np.abs(ref).max())
    nodes, tau = s.wall_shear("reaction")
    np.testing.assert_array_equal(nodes, sub["reaction_nodes"])
    np.testing.assert_allclose(tau, sub["reaction_tau"],
                               atol=1e-6 * np.abs(sub["reaction_tau"]).max())
    nodes, tau = s.wall_shear()
    np.testing.assert_array_equal(nodes, sub["gradient_nodes"])
    np.testing.assert_allclose(tau, sub["gradient_tau"],
                               atol=1e-7 * np.abs(sub["gradient_tau"]).max())
    s.close()


def test_manufactured_carreau_outlet_matches_reference():
    """The reference's ``test_carreau_outlet_manufactured`` (``tests/test_fv_solver_gpu.py``
    ``:76-101``): a body force, a pressure outlet with a prescribed velocity gradient
    (traction), Carreau-Yasuda viscosity and the transpose term; velocity to 1e-8 of the
    reference's solution, as the reference's own test asks."""
    from fixtures import gn_outlet_bcs, gn_outlet_fluid, tabulated
    from zvcfd_b200.solver import B200Solver

    g = load("gn_outlet")
    m = mesh_of(g)
    s = B200Solver(m, gn_outlet_fluid(g), gn_outlet_bcs(g, m),
                   source=tabulated(g["points"], g["f"]), advection=1.0, transpose=True)
    rep = s.solve(max_iterations=800, tol=1e-11)
    assert rep["converged"], rep["history"][-1]
    f = s.fields()
    np.testing.assert_allclose(f["U"], g["U"], atol=1e-8 * np.abs(g["U"]).max())
    np.testing.assert_allclose(f["P"], g["P"], atol=1e-8 * np.ptp(g["P"]))
    s.close()
