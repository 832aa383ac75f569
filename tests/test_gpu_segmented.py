"""FGMRES with one Krylov recurrence per block (``zvfv_solver_solve_segmented``).

Two assembled golden systems of different sizes and kinds (a tetrahedral pipe and a curved
hexahedral/prismatic tube) form one block-diagonal system, the second block's right-hand side
scaled down by 1e-6 so that a single recurrence over the union would leave it unreduced. The
segmented solve must bring each block to 1e-10 of its own initial residual and to its own
direct solution, in FP64 and with the FP32 hierarchy, and report each block's residual; a
block with nothing to solve (zero right-hand side and guess) takes no steps and stays zero, and
a block marked inactive keeps its initial guess.
"""

import numpy as np
import pytest
import torch

from fixtures import fluid_of, load, mesh_of, pipe_bcs
from oracle.linear import bsr

pytestmark = pytest.mark.gpu


def _system(name, iterations=3):
    from zvcfd_b200.solver import B200Solver

    g = load(name)
    m = mesh_of(g)
    s = B200Solver(m, fluid_of(g), pipe_bcs(name, g, m), advection=1.0)
    for _ in range(iterations):
        s.iterate()
    A, b, _, x0 = s._assemble_fused()
    out = (A.indptr.clone(), A.indices.clone(), A.data.clone(), b.reshape(-1).clone(), x0.clone())
    s.close()
    return out


def _block_diagonal(parts):
    from zvcfd_b200.linear import BlockMatrix

    ip, ix, data, bounds = [torch.zeros(1, dtype=torch.int64, device="cuda")], [], [], [0]
    nnz = 0
    for p_, i_, d_, _, _ in parts:
        ip.append(p_[1:] + nnz)
        ix.append(i_ + bounds[-1])
        data.append(d_)
        nnz += int(i_.numel())
        bounds.append(bounds[-1] + int(p_.numel()) - 1)
    return (BlockMatrix(torch.cat(ip), torch.cat(ix).to(torch.int32).contiguous(),
                        torch.cat(data).contiguous()), np.array(bounds))


@pytest.mark.parametrize("precision", ["double", "mixed"])
def test_segmented_fgmres_reaches_every_block_on_its_own(precision):
    import scipy.sparse.linalg as spl

    from zvcfd_b200.linear import B200AMG

    parts = [_system("pipe_tet_si"), _system("curved_cy")]
    A, bounds = _block_diagonal(parts)
    scale = [1.0, 1e-6]
    b = torch.cat([p[3] * f for p, f in zip(parts, scale)])
    x0 = torch.zeros_like(b)
    solver = B200AMG(precision=precision, rtol=1e-10, maxiter=400, segments=bounds)
    x, info = solver.solve(A, b, x0)
    res, ok = solver.last_segments
    assert info.converged and ok.all(), (info, res)
    assert np.all(res <= 1.01e-10), res
    xh, bh = x.cpu().numpy(), b.cpu().numpy()
    for q, (p_, i_, d_, _, _) in enumerate(parts):
        lo, hi = 4 * bounds[q], 4 * bounds[q + 1]
        M = bsr(p_.cpu().numpy(), i_.cpu().numpy(), d_.cpu().numpy(), bounds[q + 1] - bounds[q])
        ref = spl.splu(M.tocsc()).solve(bh[lo:hi])
        r = bh[lo:hi] - M @ xh[lo:hi]
        assert np.linalg.norm(r) <= 1.01e-10 * np.linalg.norm(bh[lo:hi]) + 1e-300, q
        np.testing.assert_allclose(xh[lo:hi], ref, atol=1e-7 * np.abs(ref).max())
    # a block with a zero right-hand side and a zero guess starts converged: it takes no steps
    # and stays zero while the other block is solved
    b1 = torch.cat([parts[0][3], torch.zeros(4 * (bounds[2] - bounds[1]), dtype=torch.float64,
                                             device="cuda")])
    x2, info2 = solver.solve(A, b1, torch.zeros_like(b1))
    res2, ok2 = solver.last_segments
    assert ok2.all() and res2[1] == 0.0, res2
    assert not bool(x2[4 * bounds[1]:].any())
    np.testing.assert_allclose(x2[:4 * bounds[1]].cpu().numpy(), xh[:4 * bounds[1]],
                               atol=1e-8 * np.abs(xh[:4 * bounds[1]]).max())
    # a block marked inactive keeps its initial guess exactly while the other is solved
    guess = torch.cat([torch.zeros(4 * bounds[1], dtype=torch.float64, device="cuda"),
                       torch.ones(4 * (bounds[2] - bounds[1]), dtype=torch.float64, device="cuda")])
    solver.segment_active = [True, False]
    x3, info3 = solver.solve(A, b, guess)
    solver.segment_active = None
    assert info3.converged, info3
    assert torch.equal(x3[4 * bounds[1]:], guess[4 * bounds[1]:])
    np.testing.assert_allclose(x3[:4 * bounds[1]].cpu().numpy(), xh[:4 * bounds[1]],
                               atol=1e-8 * np.abs(xh[:4 * bounds[1]]).max())
    solver.close()
