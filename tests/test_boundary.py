"""The host-side boundary data of the device path equal the oracle's (CPU)."""

import numpy as np
import pytest

from fixtures import PIPES, fluid_of, load, mesh_of, pipe_bcs
from oracle.fv import OracleSolver


@pytest.mark.parametrize("name", PIPES)
def test_boundary_arrays_match_oracle(name):
    from zvcfd_b200.boundary import Boundary

    g = load(name)
    m = mesh_of(g)
    bcs = pipe_bcs(name, g, m)
    o = OracleSolver(m, fluid_of(g), bcs, advection=1.0)
    b = Boundary(m, bcs, float(g["rho"]))
    np.testing.assert_array_equal(b.vel_fixed_comp, o.vel_fixed_comp)
    np.testing.assert_array_equal(b.p_fixed, o.p_fixed)
    np.testing.assert_allclose(b.vel_value, o.vel_value, rtol=1e-15, atol=1e-300)
    np.testing.assert_allclose(b.p_value, o.p_value)
    np.testing.assert_allclose(b.inflow, o.inflow, rtol=1e-14, atol=1e-14 * np.abs(o.inflow).max())
    np.testing.assert_allclose(b.pressure_area(), o._pressure_area(), rtol=1e-15)
    np.testing.assert_allclose(b.inflow_offsets(), o.inflow_offsets(), atol=1e-15)
    # the outlet force equals the oracle's outlet right-hand side for p = 0 (zero here)
    force, a_out, w_cons, w_only, w_stab = b.outlet_arrays()
    assert np.abs(force).max() == 0.0
    tot = o._pressure_area()
    assert np.all(w_cons[o.outlet] > 0) and np.all(w_cons[~o.outlet] == 0)
    np.testing.assert_allclose(w_cons[o.outlet].sum(), (tot > 0).sum(), rtol=1e-12)
    zids, W, c = b.flow_weights()
    assert len(zids) == len(m.zones)


def test_backflow_stabilisation_weights_match_oracle():
    """On the reference's backflow box the device path's outlet weights give, for the converged
    mass flows of the oracle, the oracle's outflow momentum coefficient
    ``m_b + beta max(-m_b, 0)`` shared by area, and the outlet force ``p S``."""
    from fixtures import backflow_bcs
    from zvcfd_b200.boundary import Boundary

    g = load("backflow_box")
    m = mesh_of(g)
    bcs = backflow_bcs(m, 0.5)
    o = OracleSolver(m, fluid_of(g), bcs, advection=1.0)
    o.solve(max_iterations=200, tol=1e-12)
    b = Boundary(m, bcs, float(g["rho"]))
    force, a_out, w_cons, w_only, w_stab = b.outlet_arrays()
    assert np.all(w_only == 0)
    np.testing.assert_allclose(w_stab, 0.5 * w_cons, rtol=1e-15)
    mb = o._mb
    coef = w_cons * mb + w_stab * np.maximum(-mb, 0.0)
    ref = np.zeros(o.N)
    tot = o._pressure_area()
    for zid, (f, S) in o.sub.items():
        if bcs[zid]["kind"] != "pressure":
            continue
        ok = f >= 0
        nodes = f[ok]
        share = np.linalg.norm(S[ok], axis=1)
        flow = mb[nodes] + 0.5 * np.maximum(-mb[nodes], 0.0)
        ref += np.bincount(nodes, flow * share / tot[nodes], o.N)
    np.testing.assert_allclose(coef, ref, atol=1e-14 * np.abs(ref).max())
    pS = np.zeros((o.N, 3))
    for zid, (f, S) in o.sub.items():
        if bcs[zid]["kind"] == "pressure":
            ok = f >= 0
            flux = (o._outlet[zid][..., None] * S)[ok]
            for k in range(3):
                pS[:, k] += np.bincount(f[ok], flux[:, k], o.N)
    assert np.abs(pS).max() > 0
    np.testing.assert_allclose(force, pS, atol=1e-15 * np.abs(pS).max())


@pytest.mark.parametrize("transpose", [True, False])
def test_prescribed_outlet_gradient_traction_matches_oracle(transpose):
    """A pressure zone with a prescribed velocity gradient: the device path's outlet force is
    the oracle's ``p S - mu(grad) tau S`` (``tau = grad + grad^T`` with the transpose term),
    and the zone takes no part in the lagged transpose traction."""
    from fixtures import gn_outlet_bcs, gn_outlet_fluid, tabulated
    from zvcfd_b200.boundary import Boundary

    g = load("gn_outlet")
    m = mesh_of(g)
    bcs = gn_outlet_bcs(g, m)
    fl = gn_outlet_fluid(g)
    o = OracleSolver(m, fl, bcs, source=tabulated(g["points"], g["f"]), advection=1.0,
                     transpose=transpose)
    b = Boundary(m, bcs, fl.rho, mu=fl.mu, viscosity=fl.viscosity, transpose=transpose)
    force, a_out, *_ = b.outlet_arrays()
    data = np.zeros((len(o.indices), 4, 4))
    rhs = np.zeros((o.N, 4))
    o._mb = np.zeros(o.N)
    o._outlet_terms(data, rhs, o.diagonal_positions(), np.zeros((o.N, 3, 3)))
    ref = -rhs[:, :3]
    assert np.abs(ref).max() > 0
    np.testing.assert_allclose(force, ref, atol=1e-14 * np.abs(ref).max())
    assert np.all(a_out == 0)
    z = {zz.name: k for k, zz in m.zones.items()}
    bad = dict(bcs)
    bad[z["xmax"]] = dict(bcs[z["xmax"]], lumped=object())
    with pytest.raises(ValueError, match="grad"):
        Boundary(m, bad, 1.0)


@pytest.mark.parametrize("extra,kind", [({"profile": "average"}, "average"),
                                        ({"opening": True}, "opening")])
def test_average_pressure_and_opening_zones(extra, kind):
    """Zones whose pressures the solve sets each iteration (the reference's device solver,
    ``zvcfd/fv/solver.py:25-47``): reported as such, their pressure force left out of the fixed
    outlet force (it comes with the iteration's pressures), and refused where they share nodes
    with another pressure zone (``:315-318``)."""
    from zvcfd_b200.boundary import Boundary
    from zvcfd_b200.mesh import box

    m = box((3, 2, 2), kind="hex")
    z = {zz.name: k for k, zz in m.zones.items()}
    bcs = {k: {"kind": "wall"} for k in m.zones}
    bcs[z["xmin"]] = {"kind": "velocity", "value": (1.0, 0.0, 0.0)}
    bcs[z["xmax"]] = {"kind": "pressure", "value": 3.0, **extra}
    bc = Boundary(m, bcs, 1.0)
    assert bc.special_zones() == {z["xmax"]: kind}
    assert not bc.outlet_force().any()
    plain = dict(bcs)
    plain[z["xmax"]] = {"kind": "pressure", "value": 3.0}
    assert Boundary(m, plain, 1.0).outlet_force().any()
    shared = dict(bcs)
    shared[z["ymin"]] = {"kind": "pressure", "value": 0.0}
    with pytest.raises(ValueError, match="share nodes"):
        Boundary(m, shared, 1.0)


def test_symmetry_and_pinned_pressure():
    from zvcfd_b200.boundary import Boundary
    from zvcfd_b200.mesh import box

    m = box((4, 3, 2), (3.0, 1.0, 0.5), kind="hex")
    z = {zz.name: k for k, zz in m.zones.items()}
    bcs = {z["xmin"]: {"kind": "velocity", "value": (1.0, 0.0, 0.0)},
           z["xmax"]: {"kind": "wall"}, z["ymin"]: {"kind": "wall"}, z["ymax"]: {"kind": "wall"},
           z["zmin"]: {"kind": "symmetry"}, z["zmax"]: {"kind": "symmetry"}}
    b = Boundary(m, bcs, 1.0)
    o = OracleSolver(m, fluid_of({"rho": 1.0, "mu": 0.1}), bcs, advection=1.0)
    np.testing.assert_array_equal(b.sym, o.sym)
    assert b.pin == o._pin
    np.testing.assert_array_equal(b.p_fixed, o.p_fixed)


def test_union_of_meshes_offsets_nodes_elements_and_zones():
    """The ensemble's disjoint union: node ranges, shifted connectivity and renumbered zones."""
    from zvcfd_b200.ensemble import union
    from zvcfd_b200.mesh import box, pipe

    a = pipe(1e-3, 5e-3, n_core=4, n_ring=2, n_axial=6)
    b = box((3, 3, 3), kind="tet")
    m, off, ids = union([a, b])
    assert list(off) == [0, a.n_nodes, a.n_nodes + b.n_nodes]
    np.testing.assert_array_equal(m.nodes[off[1]:], b.nodes)
    np.testing.assert_array_equal(m.elements["tet"][len(a.elements["tet"]):], b.elements["tet"] + off[1])
    assert sorted(ids[0].values()) + sorted(ids[1].values()) == list(range(3, 3 + len(a.zones) + len(b.zones)))
    for i, mesh in enumerate((a, b)):
        for z, u in ids[i].items():
            f, g = mesh.zones[z].faces, m.zones[u].faces
            np.testing.assert_array_equal(g, np.where(f >= 0, f + off[i], -1))
            assert m.zones[u].name.startswith(mesh.zones[z].name)


def test_time_dependent_boundary_data_refresh_consistently():
    """What a time step re-uploads (outlet pressure forces, known zone flows) equals the full
    arrays of the same time, for a pulsatile inlet and a time-dependent outlet pressure."""
    from zvcfd_b200.boundary import Boundary

    g = load("pipe_reference_tube")
    m = mesh_of(g)
    z = {zz.name: k for k, zz in m.zones.items()}
    R = float(g["radius"])

    def shape(x):
        return np.clip(1 - (x[:, 0] ** 2 + x[:, 1] ** 2) / R ** 2, 0, None)

    bcs = {z["inlet"]: {"kind": "velocity", "flow_rate": lambda t: 0.3 + 0.1 * np.sin(t),
                        "profile": shape},
           z["outlet"]: {"kind": "pressure", "value": lambda x, t: 2.0 + np.cos(t) + 0 * x[:, 0]},
           z["wall"]: {"kind": "wall"}}
    b = Boundary(m, bcs, 1.0)
    for t in (0.0, 0.7, 1.9):
        b.update(t)
        force = b.outlet_arrays()[0]
        np.testing.assert_array_equal(b.outlet_force(), force)
        assert np.abs(force).max() > 0
        zids, W, c = b.flow_weights()
        np.testing.assert_array_equal(b.flow_constants(zids), c)
        assert abs(c[zids.index(z["inlet"])] + (0.3 + 0.1 * np.sin(t))) < 1e-12


def test_segmented_fgmres_converges_every_segment_on_its_own():
    """The ensemble's per-instance Krylov recurrences (CPU tensors, dense stand-ins for the
    operator and a Jacobi preconditioner): three decoupled nonsymmetric blocks whose right-hand
    sides differ by 1e6 in size each reach their own relative residual of 1e-8 - one FGMRES
    over the whole vector would leave the small ones unreduced."""
    import torch

    from zvcfd_b200.ensemble import segmented_fgmres

    rng = np.random.default_rng(3)
    sizes = [40, 64, 24]
    blocks = []
    for n in sizes:
        M = np.eye(n) * 4 + rng.normal(scale=0.3, size=(n, n)) + np.diag(np.full(n - 1, -1.5), 1)
        blocks.append(M)
    N = sum(sizes)
    A = np.zeros((N, N))
    o = 0
    for Bk in blocks:
        A[o:o + len(Bk), o:o + len(Bk)] = Bk
        o += len(Bk)
    b = np.concatenate([rng.normal(size=n) * s for n, s in zip(sizes, (1.0, 1e-6, 1e3))])
    At = torch.as_tensor(A)
    dinv = 1.0 / torch.diagonal(At)
    bounds = np.concatenate([[0], np.cumsum(sizes)])
    x, its, res, ok = segmented_fgmres(lambda v: At @ v, lambda v: dinv * v, torch.as_tensor(b),
                                       torch.zeros(N, dtype=torch.float64), bounds, 1e-8,
                                       restart=10, maxiter=300)
    assert ok and res <= 1.01e-8
    xe = np.linalg.solve(A, b)
    o = 0
    for n in sizes:
        ref = xe[o:o + n]
        np.testing.assert_allclose(x.numpy()[o:o + n], ref, atol=1e-6 * np.abs(ref).max())
        o += n


def test_flow_rate_table_is_periodic_and_exact():
    """A flow-rate inlet given as a periodic ``[(t, Q), ...]`` table (the reference's
    ``_Signal``, ``zvcfd/lumped.py:57-70``): linear between entries, repeating with the period
    of its last time, and the discrete inflow equal to ``rho Q(t)``."""
    from zvcfd_b200.boundary import Boundary
    from zvcfd_b200.mesh import pipe

    m = pipe(1e-3, 3e-3, n_core=4, n_ring=2, n_axial=3, kind="tet")
    z = {zz.name: k for k, zz in m.zones.items()}
    table = [(0.0, 1e-6), (0.3, 4e-6), (0.8, 1e-6)]
    bcs = {z["inlet"]: {"kind": "velocity", "flow_rate": table},
           z["outlet"]: {"kind": "pressure", "value": 0.0}, z["wall"]: {"kind": "wall"}}
    b = Boundary(m, bcs, 1060.0)
    for t, q in ((0.0, 1e-6), (0.15, 2.5e-6), (0.3, 4e-6), (0.55, 2.5e-6), (0.95, 2.5e-6)):
        b.update(t)
        assert abs(-b.inflow.sum() - 1060.0 * q) < 1e-12 * 1060.0 * q
