"""Zone forces from consistent reactions: the oracle and the device path's host code against
the reference's own forces (CPU)."""

import numpy as np
import pytest
import torch

from fixtures import forces_case, load
from oracle.fv import OracleSolver
from zvcfd_b200.fluid import Fluid


def _solved(tag):
    g = load("forces")
    m, bcs, sub = forces_case(g, tag)
    s = OracleSolver(m, Fluid(1.0, float(sub["mu"])), bcs, advection=1.0)
    assert s.solve(max_iterations=300, tol=1e-13)["converged"]
    return m, bcs, sub, s


def _compact(s, keep):
    """The oracle's raw rows in the device path's layout: kept rows' blocks contiguous."""
    ip = s.indptr.astype(np.int64)
    cnt = np.where(keep, ip[1:] - ip[:-1], 0)
    rawoff = np.where(keep, np.cumsum(cnt) - cnt, -1)
    data, b = s.raw
    blocks = np.concatenate([data[ip[i]:ip[i + 1]] for i in np.flatnonzero(keep)])
    rawb = np.where(keep[:, None], b, 0.0)
    return (torch.as_tensor(ip), torch.as_tensor(s.indices.astype(np.int32)),
            torch.as_tensor(rawoff), torch.as_tensor(blocks.reshape(-1)), torch.as_tensor(rawb))


@pytest.mark.parametrize("tag", ["pipe", "channel"])
def test_oracle_zone_forces_match_reference(tag):
    """The reference's ``test_zone_forces_match_reference`` case (and the channel with two
    pressure zones and symmetry planes): forces to 1e-12 of their scale, flows to 1e-12."""
    _, _, sub, s = _solved(tag)
    # the fields first (the channel's two symmetry planes pin the oracle's mirrored gradients)
    np.testing.assert_allclose(s.U, sub["U"], atol=1e-10 * np.abs(sub["U"]).max())
    np.testing.assert_allclose(s.P, sub["P"], atol=1e-10 * np.ptp(sub["P"]))
    F, q = s.zone_forces(), s.zone_flows()
    zids = [int(z) for z in sub["force_zones"]]
    scale = np.abs(sub["forces"]).max()
    np.testing.assert_allclose(np.array([F[z] for z in zids]), sub["forces"], atol=1e-12 * scale)
    np.testing.assert_allclose(np.array([q[z] for z in zids]), sub["flows"],
                               atol=1e-12 * np.abs(sub["flows"]).max())
    # the momentum balance the forces close: sum of forces and momentum outflows
    Mo = sub["momentum_outflow"]
    assert np.abs((sub["forces"] + Mo).sum(0)).max() < 1e-12 * scale


@pytest.mark.parametrize("tag", ["pipe", "channel"])
def test_device_path_zone_forces_from_compact_raw_rows(tag):
    """:class:`zvcfd_b200.forces.RawRows` over the compact kept-row layout the boundary pass
    writes, and :func:`zvcfd_b200.forces.zone_forces` over the device path's boundary data,
    give the reference's forces."""
    from zvcfd_b200.boundary import Boundary
    from zvcfd_b200.forces import RawRows, zone_forces

    m, bcs, sub, s = _solved(tag)
    bc = Boundary(m, bcs, 1.0)
    keep = bc.vel_fixed_comp.any(1)
    raw = RawRows(*_compact(s, keep))
    X = torch.as_tensor(np.concatenate([s.U, s.P[:, None]], 1))
    r = raw.residual(X).numpy()
    full = s.momentum_residual()
    np.testing.assert_allclose(r[keep, :3], full[keep], atol=1e-13 * np.abs(full).max())
    assert np.all(r[~keep] == 0)
    F = zone_forces(bc, r, s.P)
    zids = [int(z) for z in sub["force_zones"]]
    scale = np.abs(sub["forces"]).max()
    np.testing.assert_allclose(np.array([F[z] for z in zids]), sub["forces"], atol=1e-12 * scale)


@pytest.mark.parametrize("tag", ["pipe", "channel"])
def test_device_path_reaction_wall_shear_matches_reference(tag):
    """``wall_shear(method="reaction")``: the reference device solver's own evaluation of the
    converged state (recorded with NumPy in place of CuPy) against the device path's host code
    over the compact kept rows; also its zone forces, which equal the CPU reference's."""
    from zvcfd_b200.boundary import Boundary
    from zvcfd_b200.forces import RawRows, wall_shear_reaction

    m, bcs, sub, s = _solved(tag)
    np.testing.assert_allclose(sub["gpusolver_forces"], sub["forces"],
                               atol=1e-13 * np.abs(sub["forces"]).max())
    bc = Boundary(m, bcs, 1.0)
    raw = RawRows(*_compact(s, bc.vel_fixed_comp.any(1)))
    r = raw.residual(torch.as_tensor(np.concatenate([s.U, s.P[:, None]], 1))).numpy()
    nodes, tau = wall_shear_reaction(bc, r, s.P)
    np.testing.assert_array_equal(nodes, sub["reaction_nodes"])
    ref = sub["reaction_tau"]
    np.testing.assert_allclose(tau, ref, atol=1e-11 * np.abs(ref).max())


@pytest.mark.parametrize("tag", ["pipe", "channel"])
def test_oracle_gradient_wall_shear_matches_reference_device_solver(tag):
    """``wall_shear()`` (the gradient method) of the reference device solver on the converged
    state equals the oracle's wall-gradient evaluator at the same nodes."""
    from oracle.wall import wall_shear

    m, bcs, sub, s = _solved(tag)
    walls = [z for z in m.zones if bcs[z]["kind"] == "wall"]
    tau = wall_shear(m, walls, s.U, mu=float(sub["mu"]))
    np.testing.assert_array_equal(sub["gradient_nodes"], sub["reaction_nodes"])
    ref = sub["gradient_tau"]
    np.testing.assert_allclose(tau[sub["gradient_nodes"]], ref, atol=1e-12 * np.abs(ref).max())


def test_zone_flows_split_a_shared_edge_by_area():
    """The channel whose outflow and top pressure zones share an edge of nodes
    (``tests/test_fv_boundaries.py:210-233`` of the reference): the device path's zone-flow
    weights (``W m_b + c``, read back once per iteration) applied to the oracle's converged
    boundary mass flows give the reference's zone flows, each shared node counted once."""
    from zvcfd_b200.boundary import Boundary

    m, bcs, sub, s = _solved("channel")
    zids, W, c = Boundary(m, bcs, 1.0).flow_weights()
    q = dict(zip(zids, W @ s._mb + c))
    ref = dict(zip([int(z) for z in sub["force_zones"]], sub["flows"]))
    assert sorted(q) == sorted(ref)
    scale = sum(abs(v) for v in ref.values())
    for z in ref:
        assert abs(q[z] - ref[z]) < 1e-12 * scale
    name = {zz.name: k for k, zz in m.zones.items()}
    assert q[name["xmax"]] > 0 and q[name["ymax"]] > 0
    assert abs(sum(q.values())) < 1e-12 * scale


def test_raw_rows_residual_on_a_random_state():
    """At a random state the kept rows' residual equals the full system's, row by row."""
    from zvcfd_b200.boundary import Boundary
    from zvcfd_b200.forces import RawRows

    m, bcs, sub, s = _solved("channel")
    keep = Boundary(m, bcs, 1.0).vel_fixed_comp.any(1)
    rng = np.random.default_rng(3)
    s.U, s.P = rng.standard_normal((s.N, 3)), rng.standard_normal(s.N)
    raw = RawRows(*_compact(s, keep))
    r = raw.residual(torch.as_tensor(np.concatenate([s.U, s.P[:, None]], 1))).numpy()
    data, b = s.raw
    full = (s.to_csr(data) @ np.concatenate([s.U, s.P[:, None]], 1).reshape(-1)
            - b.reshape(-1)).reshape(-1, 4)
    np.testing.assert_allclose(r[keep], full[keep], atol=1e-12 * np.abs(full).max())
    assert raw.nraw == int(np.sum((s.indptr[1:] - s.indptr[:-1])[keep]))


@pytest.mark.parametrize("tag", ["pipe", "channel"])
def test_solver_zone_forces_glue_on_cpu_tensors(tag):
    """``B200Solver.zone_forces`` and ``wall_shear("reaction")`` over the buffers the boundary
    pass fills (here from the oracle, as CPU tensors): the solver's own glue, without a GPU."""
    from zvcfd_b200.boundary import Boundary
    from zvcfd_b200.solver import B200Solver

    m, bcs, sub, s = _solved(tag)
    bc = Boundary(m, bcs, 1.0)
    ip, ix, rawoff, rawdata, rawb = _compact(s, bc.vel_fixed_comp.any(1))
    sv = object.__new__(B200Solver)
    sv.pattern, sv._rawoff, sv.rawdata, sv.rawb = (ip, ix), rawoff, rawdata, rawb.reshape(-1)
    sv.U, sv.P = torch.as_tensor(s.U), torch.as_tensor(s.P)
    sv.bc, sv.stokes, sv._lumped, sv._assembled, sv._raw_rows = bc, False, {}, True, None
    sv._special = {}
    F = sv.zone_forces()
    got = np.array([F[int(z)] for z in sub["force_zones"]])
    np.testing.assert_allclose(got, sub["forces"], atol=1e-12 * np.abs(sub["forces"]).max())
    nodes, tau = sv.wall_shear("reaction")
    np.testing.assert_array_equal(nodes, sub["reaction_nodes"])
    np.testing.assert_allclose(tau, sub["reaction_tau"],
                               atol=1e-11 * np.abs(sub["reaction_tau"]).max())
