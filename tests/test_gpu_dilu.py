"""The multicolour DILU smoother of the device AMG (``smoother="dilu"``).

- On a one-level hierarchy the V-cycle is the coarse smoothing alone: ``coarse_sweeps`` DILU
  steps from zero on the finest level. Restated here in NumPy (the greedy colouring in row
  order, the DILU diagonal ``E_i = A_ii - sum over earlier colours A_ij E_j^-1 A_ji``, the
  forward and backward colour solves, ``x += omega z``), it must agree to round-off.
- FGMRES preconditioned by the DILU V-cycle solves an assembled system and its transpose to
  the direct solutions, in FP64 and with the FP32 hierarchy.
"""

import numpy as np
import pytest
import torch

from fixtures import fluid_of, load, mesh_of, pipe_bcs
from oracle.linear import bsr

pytestmark = pytest.mark.gpu


def _system(name="pipe_tet_si", iterations=3):
    from zvcfd_b200.solver import B200Solver

    g = load(name)
    m = mesh_of(g)
    s = B200Solver(m, fluid_of(g), pipe_bcs(name, g, m), advection=1.0)
    for _ in range(iterations):
        s.iterate()
    A, b, _, x0 = s._assemble_fused()
    return s, A, b.reshape(-1).clone(), x0


def _dilu_steps(ip, ix, data, r, omega, steps):
    n = len(ip) - 1
    col = np.zeros(n, int)
    for i in range(n):
        used = {col[j] for j in ix[ip[i]:ip[i + 1]] if j < i}
        c = 0
        while c in used:
            c += 1
        col[i] = c
    blk = {(i, int(ix[p])): data[p] for i in range(n) for p in range(ip[i], ip[i + 1])}
    order = np.argsort(col, kind="stable")
    Einv = np.zeros((n, 4, 4))
    for i in order:
        E = blk[(i, i)].copy()
        for j in ix[ip[i]:ip[i + 1]]:
            if col[j] < col[i] and (j, i) in blk:
                E -= blk[(i, j)] @ Einv[j] @ blk[(j, i)]
        Einv[i] = np.linalg.inv(E)
    M = bsr(ip, ix, data, n).tocsr()
    x = np.zeros(4 * n)
    for _ in range(steps):
        res = (r - M @ x).reshape(n, 4)
        w = np.zeros((n, 4))
        for i in order:                                   # forward, colours in order
            s = res[i].copy()
            for j in ix[ip[i]:ip[i + 1]]:
                if col[j] < col[i]:
                    s -= blk[(i, j)] @ w[j]
            w[i] = Einv[i] @ s
        for i in order[::-1]:                             # backward, colours in reverse
            s = np.zeros(4)
            for j in ix[ip[i]:ip[i + 1]]:
                if col[j] > col[i]:
                    s += blk[(i, j)] @ w[j]
            w[i] = w[i] - Einv[i] @ s
        x = x + omega * w.reshape(-1)
    return x


def test_one_level_dilu_cycle_matches_restatement():
    from zvcfd_b200.linear import B200AMG

    s, A, b, x0 = _system()
    solver = B200AMG(smoother="dilu", precision="double", max_levels=1, coarse_sweeps=3)
    solver.setup(A)
    g = torch.Generator(device="cuda").manual_seed(3)
    r = torch.randn(A.n * 4, dtype=torch.float64, device="cuda", generator=g)
    z = solver.vcycle(r).cpu().numpy()
    ref = _dilu_steps(A.indptr.cpu().numpy(), A.indices.cpu().numpy(), A.data.cpu().numpy(),
                      r.cpu().numpy(), 0.75, 3)
    np.testing.assert_allclose(z, ref, rtol=0, atol=1e-11 * np.abs(ref).max())
    solver.close()
    s.close()


@pytest.mark.parametrize("precision", ["double", "mixed"])
def test_dilu_fgmres_solves_to_direct_solution(precision):
    import scipy.sparse.linalg as spl

    from zvcfd_b200.linear import B200AMG

    s, A, b, x0 = _system()
    M = bsr(A.indptr.cpu().numpy(), A.indices.cpu().numpy(), A.data.cpu().numpy(), A.n).tocsc()
    bh = b.cpu().numpy()
    for transposed in (False, True):
        solver = B200AMG(smoother="dilu", precision=precision, rtol=1e-10, maxiter=400)
        x, info = solver.solve(A, b, x0, transposed=transposed)
        assert info.converged, (transposed, info)
        Mt = M.T.tocsc() if transposed else M
        ref = spl.splu(Mt).solve(bh)
        np.testing.assert_allclose(x.cpu().numpy(), ref, atol=1e-7 * np.abs(ref).max())
        solver.close()
    s.close()
