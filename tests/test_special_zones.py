"""Pressure zones that only the reference's device solver has, against its own results.

``tests/golden/gpu_path.npz`` holds the converged fields, zone flows and zone pressures of the
reference's ``GPUSolver`` (``zvcfd/fv/solver.py``), run in this container on the CPU (its
kernels compiled for the CPU, ``tests/golden/make_golden.py gpu_path``, which first holds that
run to the reference's CPU solver on a plain pipe), for the pipe of the reference's boundary
tests (``tests/test_fv_boundaries.py:37-49``) with:

- an RCR outlet coupled implicitly (``:86-109``);
- an average-static-pressure outlet (``:236-250``);
- an opening inlet (``:253-266``);

and ``tests/golden/gpu_path_transient.npz`` its BDF2 steps of the RCR outlet under a pulsing
inflow (``:112-129``, shortened to 3 steps).

The oracle must reach the same solutions (the converged outer loops agree to their tolerance:
1e-9 of the largest velocity and of the pressure range), and the device path's two new pieces,
the upstream neighbours of an average zone and the per-iteration zone pressures, must equal
the oracle's on the CPU (bit for bit, and to round-off).
"""

import numpy as np
import pytest
import torch

from fixtures import load, mesh_of
from oracle.fv import OracleSolver

G = load("gpu_path")


def _case(tag):
    from zvcfd_b200.fluid import Fluid
    from zvcfd_b200.lumped import RCR

    g = load("pipe_reference_tube")
    m = mesh_of(g)
    z = {zz.name: k for k, zz in m.zones.items()}
    wall = {z["wall"]: {"kind": "wall"}}
    if tag == "rcr":
        bcs = {z["inlet"]: {"kind": "velocity", "flow_rate": 0.3, "profile": "poiseuille"},
               z["outlet"]: {"kind": "pressure", "lumped": RCR(rp=2.0, c=0.1, rd=5.0, pv=1.0)}}
    elif tag == "average":
        bcs = {z["inlet"]: {"kind": "velocity", "flow_rate": 0.3},
               z["outlet"]: {"kind": "pressure", "value": 2.0, "profile": "average"}}
    else:
        bcs = {z["inlet"]: {"kind": "pressure", "value": 1.0, "opening": True},
               z["outlet"]: {"kind": "pressure", "value": 0.0}}
    return m, z, bcs | wall, Fluid(1.0, 0.2)


@pytest.mark.parametrize("tag", ["rcr", "average", "opening"])
def test_oracle_reaches_the_reference_device_solution(tag):
    m, z, bcs, fluid = _case(tag)
    s = OracleSolver(m, fluid, bcs, advection=1.0)
    assert s.solve(max_iterations=300, tol=1e-11)["converged"]
    U, P = G[f"{tag}_U"], G[f"{tag}_P"]
    np.testing.assert_allclose(s.U, U, rtol=0, atol=1e-9 * np.abs(U).max())
    np.testing.assert_allclose(s.P, P, rtol=0, atol=1e-9 * np.ptp(P))
    flows = s.zone_flows()
    for zid, q in zip(G[f"{tag}_zones"], G[f"{tag}_flows"]):
        assert abs(flows[int(zid)] / fluid.rho - q) <= 1e-9 * 0.3
    if tag == "average":                           # the zone's area-mean pressure is its value
        f, S = s.sub[z["outlet"]]
        ok = f >= 0
        a = np.linalg.norm(S, axis=2) * ok
        mean = float((s.P[np.where(ok, f, 0)] * a).sum() / a.sum())
        assert abs(mean - 2.0) < 1e-10
    if tag == "opening":                           # total pressure where the flow enters
        nodes = s._zone_nodes[z["inlet"]]
        np.testing.assert_allclose(s.P[nodes], 1.0 - 0.5 * (s.U[nodes] ** 2).sum(1),
                                   atol=1e-9)


@pytest.mark.parametrize("tag", ["average", "opening"])
def test_device_zone_pressures_equal_the_oracle(tag):
    """``upstream_neighbours`` and ``special_pressure`` (the device path's, on CPU tensors)
    against the oracle's on a state a few iterations in."""
    from zvcfd_b200.boundary import upstream_neighbours
    from zvcfd_b200.solver import special_pressure

    m, z, bcs, fluid = _case(tag)
    s = OracleSolver(m, fluid, bcs, advection=1.0)
    s.solve(max_iterations=4, tol=0.0)
    zid = next(iter(s.special))
    gradP = s.nodal_gradient(s.P)
    s._special_pressures(gradP)
    want = s.p_value[s._special_geom[zid]["nodes"]].copy()
    geo = s._special_geom[zid]
    zone = {"nodes": torch.as_tensor(geo["nodes"]), "Sn": torch.as_tensor(geo["Sn"]),
            "area": torch.as_tensor(geo["area"])}
    if tag == "average":
        up, dx = upstream_neighbours(geo["nodes"], geo["Sn"], m.nodes, s.indptr, s.indices,
                                     s.outlet)
        np.testing.assert_array_equal(up, geo["up"])
        np.testing.assert_allclose(dx, geo["dx"], rtol=0, atol=0)
        zone.update(up=torch.as_tensor(up), dx=torch.as_tensor(dx), blend=geo["blend"])
    p0 = 2.0 if tag == "average" else 1.0
    got = special_pressure(tag, zone, torch.as_tensor(s.P), torch.as_tensor(gradP),
                           torch.as_tensor(s.U), torch.as_tensor(s._mb), fluid.rho, p0)
    np.testing.assert_allclose(got.numpy(), want, rtol=0, atol=1e-14 * max(np.abs(want).max(), 1))
    if tag == "opening":
        assert (s._mb[geo["nodes"]] < 0).any()      # some of the zone takes inflow


def test_oracle_rcr_march_equals_the_reference_device_march():
    """The reference's transient RCR test (``tests/test_fv_boundaries.py:112-129``), shortened:
    BDF2 steps of a pulsing inlet into an RCR outlet. The oracle's step flows, the outlet
    pressure and the final fields equal the reference device solver's (run on the CPU) to the
    loops' tolerance."""
    from zvcfd_b200.lumped import RCR

    T = load("gpu_path_transient")
    seen = []

    class Recording(RCR):
        def advance(self, q, t, dt):
            seen.append((t, q))
            return super().advance(q, t, dt)

    m, z, bcs, fluid = _case("rcr")
    bcs[z["inlet"]] = {"kind": "velocity", "flow_rate": lambda t: 0.3 + 0.1 * np.sin(2 * np.pi * t),
                       "profile": "poiseuille"}
    bcs[z["outlet"]] = {"kind": "pressure", "lumped": Recording(rp=2.0, c=0.1, rd=5.0, pv=1.0)}
    s = OracleSolver(m, fluid, bcs, advection=1.0)
    assert s.solve(max_iterations=300, tol=1e-11)["converged"]
    s.solve_transient(0.05, 3, loops=20, tol=1e-12)
    steps = T["steps"]                                  # (t, outlet flow, outlet pressure)
    assert len(seen) == len(steps) == 3
    for (t, q), (tr, qr, pr) in zip(seen, steps):
        assert abs(t - tr) < 1e-15 and abs(q - qr) < 1e-9 * 0.3
    f, S = s.sub[z["outlet"]]
    ok = f >= 0
    a = np.linalg.norm(S, axis=2) * ok
    assert abs(float((s.P[np.where(ok, f, 0)] * a).sum() / a.sum()) - steps[-1][2]) < 1e-9
    np.testing.assert_allclose(s.U, T["U"], rtol=0, atol=1e-9 * np.abs(T["U"]).max())
    np.testing.assert_allclose(s.P, T["P"], rtol=0, atol=1e-9 * np.ptp(T["P"]))


@pytest.mark.parametrize("tag", ["rcr", "average", "opening"])
def test_device_path_forces_on_these_zones(tag):
    """Zone forces and wall shear from consistent reactions, by the device path's host code
    (``zvcfd_b200.forces`` over the kept rows in the boundary pass's layout) on the oracle's
    converged state, against the reference device solver's own: a lumped, average-pressure or
    opening zone's pressure force takes the nodal pressures."""
    from test_forces import _compact
    from zvcfd_b200.boundary import Boundary
    from zvcfd_b200.forces import RawRows, wall_shear_reaction, zone_forces

    m, z, bcs, fluid = _case(tag)
    s = OracleSolver(m, fluid, bcs, advection=1.0)
    assert s.solve(max_iterations=300, tol=1e-11)["converged"]
    bc = Boundary(m, bcs, fluid.rho, mu=fluid.mu)
    raw = RawRows(*_compact(s, bc.vel_fixed_comp.any(1)))
    r = raw.residual(torch.as_tensor(np.concatenate([s.U, s.P[:, None]], 1))).numpy()
    nodal = list(bc.lumped_zones()) + list(bc.special_zones())
    F = zone_forces(bc, r, s.P, lumped=nodal)
    want = G[f"{tag}_forces"]
    got = np.array([F[int(k)] for k in G[f"{tag}_zones"]])
    np.testing.assert_allclose(got, want, rtol=0, atol=1e-9 * np.abs(want).max())
    nodes, tau = wall_shear_reaction(bc, r, s.P)
    np.testing.assert_array_equal(nodes, G[f"{tag}_shear_nodes"])
    ref = G[f"{tag}_shear"]
    np.testing.assert_allclose(tau, ref, rtol=0, atol=1e-9 * np.abs(ref).max())
