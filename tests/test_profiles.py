"""Flow-rate inlet profiles against the reference's own (CPU): the developed laminar profile
of each inlet's cross-section, and a pipe whose inlet takes the default profile."""

import numpy as np
import pytest

from fixtures import load, mesh_of

TAGS = ["tube_mixed", "tube_tet", "box_hex", "box_tet"]


@pytest.mark.parametrize("tag", TAGS)
def test_developed_profile_matches_reference(tag):
    from oracle.fv import developed_profile as oracle_profile
    from zvcfd_b200.profiles import developed_profile, inlet_shape

    g = load("profiles")
    X, faces = g[f"{tag}_X"], g[f"{tag}_faces"]
    nodes, u = developed_profile(X, faces)
    np.testing.assert_array_equal(nodes, g[f"{tag}_nodes"])
    np.testing.assert_allclose(u, g[f"{tag}_u"], atol=1e-14)
    n2, v = inlet_shape(X, faces)
    np.testing.assert_array_equal(n2, nodes)
    np.testing.assert_allclose(v, g[f"{tag}_shape"], atol=1e-14)
    o = oracle_profile(X, faces)
    np.testing.assert_allclose([o[int(k)] for k in nodes], g[f"{tag}_u"], atol=1e-14)
    assert u.max() == 1.0 and u.min() == 0.0


def test_circle_profile_is_close_to_the_parabola():
    """On the finest circle the developed profile approaches ``1 - (r/R)^2``."""
    from zvcfd_b200.profiles import developed_profile

    g = load("profiles")
    X, faces = g["tube_tet_X"], g["tube_tet_faces"]
    nodes, u = developed_profile(X, faces)
    r2 = (X[nodes, 0] ** 2 + X[nodes, 1] ** 2) / np.max(X[nodes, 0] ** 2 + X[nodes, 1] ** 2)
    assert np.abs(u - (1 - r2)).max() < 0.1


def test_default_flow_rate_inlet_matches_reference():
    """A flow-rate inlet without a profile takes the developed one, as in the reference: the
    device path's boundary values equal the oracle's, and the oracle reaches the reference's
    converged pipe."""
    from oracle.fv import OracleSolver
    from zvcfd_b200.boundary import Boundary
    from zvcfd_b200.fluid import Fluid

    g = load("profiles")
    sub = {k[5:]: v for k, v in g.items() if k.startswith("pipe_")}
    m = mesh_of(sub)
    z = {zz.name: k for k, zz in m.zones.items()}
    bcs = {z["inlet"]: {"kind": "velocity", "flow_rate": float(sub["flow_rate"])},
           z["outlet"]: {"kind": "pressure", "value": 0.0}, z["wall"]: {"kind": "wall"}}
    b = Boundary(m, bcs, float(sub["rho"]))
    o = OracleSolver(m, Fluid(float(sub["rho"]), float(sub["mu"])), bcs, advection=1.0)
    np.testing.assert_allclose(b.vel_value, o.vel_value, atol=1e-15 * np.abs(o.vel_value).max())
    np.testing.assert_allclose(b.inflow, o.inflow, atol=1e-15 * np.abs(o.inflow).max())
    assert abs(-b.inflow.sum() - float(sub["flow_rate"]) * float(sub["rho"])) < 1e-14
    assert o.solve(max_iterations=300, tol=1e-13)["converged"]
    np.testing.assert_allclose(o.U, sub["U"], atol=1e-10 * np.abs(sub["U"]).max())
    np.testing.assert_allclose(o.P, sub["P"], atol=1e-10 * np.ptp(sub["P"]))
