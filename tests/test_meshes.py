"""The synthetic vessel meshes of the workloads (CPU): every element has positive volume, the
zones cover the boundary exactly once, the boundary is closed (its outward area vectors sum to
zero), the documented sizes hold, and the ensemble's instances are reproducible from the seed."""

import numpy as np
import pytest

from zvcfd_b200.boundary import subfaces


def _check(m, names):
    for kind in m.elements:
        assert (m.element_volumes(kind) > 0).all(), kind
    bf = m.boundary_faces()
    zf = np.concatenate([z.faces for z in m.zones.values()])
    assert len(zf) == len(bf)
    key = lambda f: {tuple(sorted(r)) for r in f.tolist()}  # noqa: E731
    assert key(zf) == key(bf)
    total = sum(subfaces(m.nodes, z.faces).reshape(-1, 3).sum(0) for z in m.zones.values())
    scale = sum(np.abs(subfaces(m.nodes, z.faces)).sum() for z in m.zones.values())
    assert np.abs(total).max() < 1e-12 * scale
    assert sorted(z.name for z in m.zones.values()) == sorted(names)


def test_poiseuille_pipe():
    from zvcfd_b200.mesh import pipe

    m = pipe(1e-3, 10e-3, n_core=14, n_ring=7, n_axial=80, kind="tet", jitter_amount=0.05, seed=0)
    assert m.n_nodes == 49977 and len(m.elements["tet"]) == 282240
    _check(m, ["inlet", "outlet", "wall"])


def test_curved_tube_short():
    from zvcfd_b200.mesh import curved_tube

    m = curved_tube(2e-3, 20e-3, np.pi / 2, n_core=20, n_ring=12, n_axial=8, layers=5, growth=0.8)
    per_section = m.n_nodes // 9
    assert per_section * 286 == 400686          # the 285-cell workload tube
    assert set(m.elements) == {"wedge", "hex"}
    _check(m, ["inlet", "outlet", "wall"])


def test_y_bifurcation():
    from zvcfd_b200.mesh import y_bifurcation

    m = y_bifurcation(0.5e-3)
    assert m.n_nodes == 8410
    _check(m, ["inlet", "outlet1", "outlet2", "wall"])


@pytest.mark.parametrize("kind,nodes", [("straight", 30000), ("curved", 40000),
                                        ("bifurcating", 30000)])
def test_ensemble_vessels_are_sized_and_seeded(kind, nodes):
    from zvcfd_b200.ensemble import vessel

    m, R, outlets = vessel(kind, nodes, 5)
    assert 0.7 * nodes < m.n_nodes < 1.3 * nodes
    again, _, _ = vessel(kind, nodes, 5)
    np.testing.assert_array_equal(m.nodes, again.nodes)
    assert all(o in {z.name for z in m.zones.values()} for o in outlets)


@pytest.mark.parametrize("name", ["pipe_reference_tube", "curved_cy"])
def test_wall_operator_gives_the_reference_wall_shear(name):
    """The device wall-shear operator's host data (owning elements, shape gradients at the
    wall integration points, normals, areas), applied here with NumPy the way the kernel
    applies it, reproduces the reference's wall shear on the converged golden fields."""
    from fixtures import fluid_of, load, mesh_of
    from zvcfd_b200.wall import wall_operator

    g = load(name)
    m = mesh_of(g)
    fl = fluid_of(g)
    walls = [z for z, zz in m.zones.items() if zz.name == "wall"]
    elem, G, nrm, area, node = wall_operator(m, walls)
    U = g["U"]
    grad = np.einsum("qar,qac->qrc", np.where(elem[..., None] >= 0, U[np.maximum(elem, 0)], 0.0), G)
    D = grad + np.swapaxes(grad, 1, 2)
    mu = np.full(len(D), fl.mu) if fl.viscosity is None else \
        fl.viscosity(np.sqrt(0.5 * np.einsum("qrc,qrc->q", D, D)))
    t = mu[:, None] * np.einsum("qrc,qc->qr", D, nrm)
    sub = -(t - np.einsum("qr,qr->q", t, nrm)[:, None] * nrm)
    tau = np.zeros((m.n_nodes, 3))
    np.add.at(tau, node, sub * area[:, None])
    weight = np.bincount(node, area, m.n_nodes)
    tau[weight > 0] /= weight[weight > 0, None]
    ref = load("wall_shear")[f"{name}_tau"]
    np.testing.assert_allclose(tau, ref, atol=1e-12 * np.abs(ref).max())
