"""The B200 element and node kernels evaluate the reference's discrete equations.

The procedure of the reference's ``tests/test_fv_fast.py``: seeded random states on
distorted meshes of every element type, with and without stored geometry, Newtonian and
Carreau-Yasuda fluids, with and without a time term. Node volumes, nodal gradients, the
momentum diagonal, the limiter, the block matrix and right-hand side, and the new mass
flows must match the reference's own outputs (golden vectors) and the oracle; the pattern
and the colouring must match bit for bit.
"""

import numpy as np
import pytest
import torch

from fixtures import KERNEL_MESHES, KERNEL_VARIANTS, fluid_of, kernel_case, mdot_of, mesh_of
from oracle import pattern as opat

pytestmark = pytest.mark.gpu


def _np(t):
    return t.detach().cpu().numpy()


def test_pattern_and_colouring_are_bit_exact():
    from zvcfd_b200.assembler import gpu_colour, node_graph
    from zvcfd_b200.mesh import curved_tube, pipe

    for m in (pipe(1.0, 3.0, n_core=4, n_ring=3, n_axial=10, kind="tet", jitter_amount=0.1,
                   seed=3),
              curved_tube(1.0, 5.0, n_core=4, n_ring=4, n_axial=12, layers=2)):
        for e in m.elements.values():
            col, nc = gpu_colour(e, m.n_nodes)
            col = _np(col)
            ref = opat.colour(e, m.n_nodes)
            np.testing.assert_array_equal(col, ref)
            assert nc == col.max() + 1
            opat.check_colouring(e, col)
            again, _ = gpu_colour(e, m.n_nodes)
            np.testing.assert_array_equal(_np(again), col)
        ip, ix = node_graph(m.elements, m.n_nodes)
        hp, hx = opat.node_graph(m)
        np.testing.assert_array_equal(_np(ip), hp)
        np.testing.assert_array_equal(_np(ix), hx)


def _box_tets(n):
    """Five tetrahedra per cube of an n^3 grid of cubes (tests/test_fv_fast.py:59-69)."""
    i, j, k = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")

    def v(a, b, c):
        return ((i + a) * (n + 1) + (j + b)) * (n + 1) + (k + c)

    c = [v(0, 0, 0), v(1, 0, 0), v(1, 1, 0), v(0, 1, 0), v(0, 0, 1), v(1, 0, 1), v(1, 1, 1),
         v(0, 1, 1)]
    tets = [(0, 1, 3, 4), (1, 2, 3, 6), (1, 4, 5, 6), (3, 4, 6, 7), (1, 3, 4, 6)]
    return np.stack([np.stack([c[t].ravel() for t in tet], 1) for tet in tets], 0) \
        .reshape(-1, 4).astype(np.int32), (n + 1) ** 3


def test_colouring_of_large_and_high_valence_meshes():
    from zvcfd_b200.assembler import gpu_colour

    conn, nn = _box_tets(76)
    assert len(conn) > 2 ** 21
    col, _ = gpu_colour(conn, nn)
    col = _np(col)
    assert col.min() == 0 and col.max() < 64
    opat.check_colouring(conn, col)
    np.testing.assert_array_equal(col, opat.colour(conn, nn))
    # 200 elements sharing one node need 200 colours: one 64-bit word overflows twice
    fan = np.column_stack([np.zeros(200, np.int64), 3 * np.arange(200) + 1,
                           3 * np.arange(200) + 2, 3 * np.arange(200) + 3]).astype(np.int32)
    narrow, _ = gpu_colour(fan, 601, words=1)
    wide, _ = gpu_colour(fan, 601, words=4)
    np.testing.assert_array_equal(_np(narrow), _np(wide))
    assert len(np.unique(_np(narrow))) == 200


@pytest.mark.parametrize("store", [True, False])
@pytest.mark.parametrize("variant", KERNEL_VARIANTS)
@pytest.mark.parametrize("name", KERNEL_MESHES)
def test_kernels_match_reference(name, variant, store):
    from zvcfd_b200.assembler import B200Assembler

    g = kernel_case(name, variant)
    m = mesh_of(g)
    fl = fluid_of(g)
    gn = bool(int(g["gn"]))
    dt = float(g["dt"]) or None
    rho = fl.rho
    a = B200Assembler(m, rho=rho, mu=fl.mu, rheology=fl.viscosity, transpose=gn,
                      store_geometry=store)
    np.testing.assert_array_equal(_np(a.pattern[0]), g["indptr"])
    np.testing.assert_array_equal(_np(a.pattern[1]), g["indices"])
    np.testing.assert_allclose(_np(a.node_volume), g["V"], rtol=1e-12)
    gU, gP = a.gradient(g["U"]), a.gradient(g["P"])
    np.testing.assert_allclose(_np(gU), g["gradU"], atol=1e-11)
    np.testing.assert_allclose(_np(gP), g["gradP"], atol=1e-11)
    mdot = a.to_slots(mdot_of(g))
    diag = a.diagonal(mdot, g["U"])
    np.testing.assert_allclose(_np(diag), g["diag"], rtol=1e-11, atol=1e-12)
    V = a.node_volume
    tdiag = rho * V / dt if dt else 0.0
    dnode, snode = V / (diag + tdiag), V / diag
    beta = a.limiter(g["U"], gU)
    np.testing.assert_allclose(_np(beta), g["beta_limiter"], atol=1e-12)
    U = torch.as_tensor(g["U"], device="cuda")
    levels = [(1.0, U, mdot)] if dt else []
    data, b = a.assemble(U, mdot, gU, g["beta_frozen"], gP, dnode, snode, levels=levels)
    ref = g["data_raw"]
    assert np.abs(_np(data) - ref).max() < 1e-12 * np.abs(ref).max()
    np.testing.assert_allclose(_np(b), g["b_raw"], atol=1e-12 * np.abs(g["b_raw"]).max())
    new, imb, adv = a.massflow(g["U_new"], g["P_new"], a.gradient(g["P_new"]), dnode, snode,
                               levels=levels)
    back = a.from_slots(new)
    for k, v in mdot_of(g, "mdot_new").items():
        np.testing.assert_allclose(_np(back[k]), v, atol=1e-11 * np.abs(v).max())
    np.testing.assert_allclose(_np(imb), g["imbalance"], atol=1e-11 * np.abs(g["imbalance"]).max())
    if not gn:        # the advective diagonal of the new flows: dvisc + adv = full diagonal
        full = a.diagonal(new, g["U_new"])
        np.testing.assert_allclose(_np(a.dvisc + adv), _np(full), rtol=1e-12, atol=1e-12)


def test_assembly_is_deterministic():
    from zvcfd_b200.assembler import B200Assembler
    from zvcfd_b200.mesh import curved_tube

    m = curved_tube(1.0, 5.0, n_core=4, n_ring=3, n_axial=6, layers=2, jitter_amount=0.05)
    rng = np.random.default_rng(0)
    U, P = rng.normal(size=(m.n_nodes, 3)), rng.normal(size=m.n_nodes)
    out = []
    for _ in range(2):
        a = B200Assembler(m, rho=1.0, mu=0.5)
        md = a.zero_mdot()
        gU = a.gradient(U)
        one = torch.ones(m.n_nodes, dtype=torch.float64, device="cuda")
        d, b = a.assemble(U, md, gU, torch.ones((m.n_nodes, 3), dtype=torch.float64,
                                                device="cuda"), a.gradient(P), one, one)
        out.append(_np(d).tobytes() + _np(b).tobytes())
    assert out[0] == out[1]
