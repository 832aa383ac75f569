"""The multicolour factorisation smoothers of the device AMG: DILU (``smoother="dilu"``, the
reference's ``dilu`` presets) and ILU(0) (``smoother="ilu0"``, its ``robust`` preset).

- On a one-level hierarchy the V-cycle is the coarse smoothing alone: ``coarse_sweeps`` steps
  from zero on the finest level. Restated here in NumPy (the greedy colouring in row order;
  the DILU diagonal ``E_i = A_ii - sum over earlier colours A_ij E_j^-1 A_ji``, or the ILU(0)
  factors of the colour-ordered matrix without fill; the forward and backward colour solves;
  ``x += omega z``), it must agree to round-off.
- FGMRES preconditioned by either V-cycle solves an assembled system and its transpose to the
  direct solutions, in FP64 and with the FP32 hierarchy.
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


def _colours(ip, ix):
    n = len(ip) - 1
    col = np.zeros(n, int)
    for i in range(n):
        used = {col[j] for j in ix[ip[i]:ip[i + 1]] if j < i}
        c = 0
        while c in used:
            c += 1
        col[i] = c
    return col


def _ilu_steps(ip, ix, data, r, omega, steps):
    n = len(ip) - 1
    col = _colours(ip, ix)
    order = np.argsort(col, kind="stable")
    pos = np.empty(n, int)
    pos[order] = np.arange(n)                             # colour-ordered index of each row
    lu = {(i, int(ix[p])): data[p].copy() for i in range(n) for p in range(ip[i], ip[i + 1])}
    row = {i: [int(j) for j in ix[ip[i]:ip[i + 1]]] for i in range(n)}
    Uinv = {}
    for i in order:
        for k in sorted((j for j in row[i] if pos[j] < pos[i]), key=lambda j: pos[j]):
            L = lu[(i, k)] @ Uinv[k]
            lu[(i, k)] = L
            for j in row[k]:
                if pos[j] > pos[k] and (i, j) in lu:
                    lu[(i, j)] = lu[(i, j)] - L @ lu[(k, j)]
        Uinv[i] = np.linalg.inv(lu[(i, i)])
    M = bsr(ip, ix, data, n).tocsr()
    x = np.zeros(4 * n)
    for _ in range(steps):
        res = (r - M @ x).reshape(n, 4)
        w = np.zeros((n, 4))
        for i in order:
            s = res[i].copy()
            for j in row[i]:
                if pos[j] < pos[i]:
                    s -= lu[(i, j)] @ w[j]
            w[i] = s
        for i in order[::-1]:
            s = w[i].copy()
            for j in row[i]:
                if pos[j] > pos[i]:
                    s -= lu[(i, j)] @ w[j]
            w[i] = Uinv[i] @ s
        x = x + omega * w.reshape(-1)
    return x


def _dilu_steps(ip, ix, data, r, omega, steps):
    n = len(ip) - 1
    col = _colours(ip, ix)
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


@pytest.mark.parametrize("smoother", ["dilu", "ilu0"])
def test_one_level_cycle_matches_restatement(smoother):
    from zvcfd_b200.linear import B200AMG

    s, A, b, x0 = _system()
    solver = B200AMG(smoother=smoother, precision="double", max_levels=1, coarse_sweeps=3)
    solver.setup(A)
    g = torch.Generator(device="cuda").manual_seed(3)
    r = torch.randn(A.n * 4, dtype=torch.float64, device="cuda", generator=g)
    z = solver.vcycle(r).cpu().numpy()
    steps, omega = (_dilu_steps, 0.75) if smoother == "dilu" else (_ilu_steps, 1.0)
    ref = steps(A.indptr.cpu().numpy(), A.indices.cpu().numpy(), A.data.cpu().numpy(),
                r.cpu().numpy(), omega, 3)
    np.testing.assert_allclose(z, ref, rtol=0, atol=1e-11 * np.abs(ref).max())
    solver.close()
    s.close()


@pytest.mark.parametrize("smoother", ["dilu", "ilu0"])
@pytest.mark.parametrize("precision", ["double", "mixed"])
def test_fgmres_solves_to_direct_solution(precision, smoother):
    import scipy.sparse.linalg as spl

    from zvcfd_b200.linear import B200AMG

    s, A, b, x0 = _system()
    M = bsr(A.indptr.cpu().numpy(), A.indices.cpu().numpy(), A.data.cpu().numpy(), A.n).tocsc()
    bh = b.cpu().numpy()
    for transposed in (False, True):
        solver = B200AMG(smoother=smoother, precision=precision, rtol=1e-10, maxiter=400)
        x, info = solver.solve(A, b, x0, transposed=transposed)
        assert info.converged, (transposed, info)
        Mt = M.T.tocsc() if transposed else M
        ref = spl.splu(Mt).solve(bh)
        np.testing.assert_allclose(x.cpu().numpy(), ref, atol=1e-7 * np.abs(ref).max())
        solver.close()
    s.close()
