"""The discrete adjoint of the linear solve: transposed products and V-cycle, autograd.

On an assembled, scaled system of a golden pipe: the transposed SpMV equals the oracle's
A^T x; the adjoint solve A^T lam = g equals the direct solution; and the autograd gradients
of J = g . A^{-1} b with respect to b and to block entries of A equal central finite
differences (step 1e-2 max|b| in b, where J is linear; relative step 1e-4 on the most
influential entries of A) to 1e-5.
"""

import numpy as np
import pytest
import scipy.sparse.linalg as spl
import torch

from oracle.linear import bsr

pytestmark = pytest.mark.gpu


def _system():
    from test_gpu_solver import _system as sys_

    s, A, b, x0 = sys_("pipe_tet_si", iterations=3)
    return s, A, b


def test_transposed_spmv_and_adjoint_solve():
    from zvcfd_b200._lib import call, ptr, stream_ptr
    from zvcfd_b200.linear import B200AMG

    s, A, b = _system()
    n, nnz = A.n, A.nnzb
    tptr = torch.empty(n + 1, dtype=torch.int64, device="cuda")
    trow = torch.empty(nnz, dtype=torch.int32, device="cuda")
    tperm = torch.empty(nnz, dtype=torch.int64, device="cuda")
    call("zvfv_bsr_transpose", n, nnz, ptr(A.indptr), ptr(A.indices), ptr(tptr), ptr(trow),
         ptr(tperm), stream_ptr())
    M = bsr(A.indptr.cpu().numpy(), A.indices.cpu().numpy(), A.data.cpu().numpy(), n).tocsr()
    x = torch.randn(4 * n, dtype=torch.float64, device="cuda")
    y = torch.empty_like(x)
    for lanes in (8, 16, 32):
        call("zvfv_bsr_spmv_t", n, ptr(tptr), ptr(trow), ptr(tperm), ptr(A.data), ptr(x), ptr(y),
             lanes, stream_ptr())
        ref = M.T @ x.cpu().numpy()
        np.testing.assert_allclose(y.cpu().numpy(), ref, rtol=1e-12, atol=1e-12 * np.abs(ref).max())
    for precision in ("double", "mixed"):
        solver = B200AMG(precision=precision, rtol=1e-10, maxiter=500)
        g = torch.randn(4 * n, dtype=torch.float64, device="cuda")
        solver.setup(A)
        lam, info = solver.solve(A, g, None, rtol=1e-10, transposed=True, setup=False)
        assert info.converged, info
        ref = spl.splu(M.T.tocsc()).solve(g.cpu().numpy())
        np.testing.assert_allclose(lam.cpu().numpy(), ref, atol=1e-7 * np.abs(ref).max())
        solver.close()
    s.close()


def test_linear_solve_gradients_match_finite_differences():
    """J = g . A^{-1} b: the device adjoint's dJ/db and dJ/dA equal the exact (direct-solve)
    adjoint, and central finite differences of J (direct solves) to 1e-5."""
    from zvcfd_b200.adjoint import linear_solve
    from zvcfd_b200.linear import B200AMG, BlockMatrix

    s, A, b = _system()
    torch.manual_seed(0)
    g = torch.randn(4 * A.n, dtype=torch.float64, device="cuda")
    data = A.data.clone().requires_grad_(True)
    bb = b.clone().requires_grad_(True)
    solver = B200AMG(rtol=1e-12, maxiter=800)
    x = linear_solve(BlockMatrix(A.indptr, A.indices, data), bb, solver, 1e-12)
    torch.dot(g, x).backward()
    gd, gb = data.grad.cpu().numpy(), bb.grad.cpu().numpy()
    ip, ix = A.indptr.cpu().numpy(), A.indices.cpu().numpy()
    D, bh, gh = A.data.cpu().numpy(), b.cpu().numpy(), g.cpu().numpy()
    M = bsr(ip, ix, D, A.n).tocsc()
    xe = spl.splu(M).solve(bh)
    lam = spl.splu(M.T.tocsc()).solve(gh)
    np.testing.assert_allclose(gb, lam, atol=1e-7 * np.abs(lam).max())
    rows = np.repeat(np.arange(A.n), np.diff(ip))
    gA = -(lam.reshape(-1, 4)[rows][:, :, None] * xe.reshape(-1, 4)[ix][:, None, :])
    np.testing.assert_allclose(gd.reshape(-1, 4, 4), gA, atol=1e-7 * np.abs(gA).max())

    def J(Dm, bv):
        return gh @ spl.splu(bsr(ip, ix, Dm, A.n).tocsc()).solve(bv)

    rng = np.random.default_rng(1)
    for k in rng.choice(4 * A.n, 4, replace=False):
        # J is linear in b: a step of 1e-2 of max|b| has no truncation error and keeps the
        # difference well above the direct solves' rounding
        h = 1e-2 * np.abs(bh).max()
        bp, bm = bh.copy(), bh.copy()
        bp[k] += h
        bm[k] -= h
        fd = (J(D, bp) - J(D, bm)) / (2 * h)
        assert abs(fd - gb[k]) <= 1e-5 * max(abs(fd), abs(gb[k]), 1e-12), (k, fd, gb[k])
    flat = D.reshape(-1)
    # entries whose perturbation moves J well above the direct solves' rounding: the 64 with
    # the largest |D_q dJ/dD_q|; a relative step of 1e-4 keeps the O(h^2) error below 1e-7
    influence = np.abs(flat * gA.reshape(-1))
    big = np.argsort(-influence)[:64]
    for q in rng.choice(big, 4, replace=False):
        h = 1e-4 * abs(flat[q])
        dp, dm = D.copy(), D.copy()
        dp.reshape(-1)[q] += h
        dm.reshape(-1)[q] -= h
        fd = (J(dp, bh) - J(dm, bh)) / (2 * h)
        an = gd.reshape(-1)[q]
        assert abs(fd - an) <= 1e-5 * max(abs(fd), abs(an), 1e-12), (q, fd, an)
    solver.close()
    s.close()
