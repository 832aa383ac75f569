"""Discrete adjoints of the coupled solve behind ``torch.autograd``.

:class:`LinearSolve` is ``x = A^{-1} b`` for a 4x4 block-CSR ``A`` as an autograd function:
the forward pass is the B200 back end's FGMRES-AMG solve; the backward pass solves the
adjoint system ``A^T lam = dJ/dx`` with the transposed block-CSR product and the transposed
V-cycle of the same hierarchy (``zvfv_solver_solve_t``), and returns
``dJ/db = lam`` and ``dJ/dA = -lam x^T`` restricted to the blocks of the pattern. The reference
has no adjoint; this is the component the outer-loop sensitivities are built from.
"""

from __future__ import annotations

import torch

from zvcfd_b200.linear import B200AMG, BlockMatrix


class LinearSolve(torch.autograd.Function):
    """``x = solve(data, b)`` on a fixed pattern; differentiable in ``data`` and ``b``."""

    @staticmethod
    def forward(ctx, data, b, indptr, indices, solver: B200AMG, rtol: float):
        A = BlockMatrix(indptr, indices, data.detach().reshape(-1, 4, 4).contiguous())
        x, info = solver.solve(A, b.detach().reshape(-1).contiguous(), None, rtol=rtol)
        if not info.converged:
            raise RuntimeError(f"forward solve not converged ({info.residual:.2e} after "
                               f"{info.iterations} iterations)")
        ctx.solver, ctx.rtol, ctx.A = solver, rtol, A
        ctx.save_for_backward(x, indptr, indices)
        return x.view_as(b)

    @staticmethod
    def backward(ctx, gx):
        x, indptr, indices = ctx.saved_tensors
        lam, info = ctx.solver.solve(ctx.A, gx.reshape(-1).contiguous(), None, rtol=ctx.rtol,
                                     transposed=True, setup=False)
        if not info.converged:
            raise RuntimeError(f"adjoint solve not converged ({info.residual:.2e})")
        n = indptr.numel() - 1
        rows = torch.repeat_interleave(torch.arange(n, device=x.device), indptr[1:] - indptr[:-1])
        L = lam.view(n, 4)[rows]
        X = x.view(n, 4)[indices.to(torch.int64)]
        gA = -(L[:, :, None] * X[:, None, :])
        return gA.reshape(ctx.A.data.shape), lam.view_as(gx), None, None, None, None


def linear_solve(A: BlockMatrix, b, solver: B200AMG | None = None, rtol: float = 1e-10):
    """Differentiable ``A^{-1} b`` (``A.data`` and ``b`` may require grad)."""
    solver = solver or B200AMG(rtol=rtol, maxiter=500)
    return LinearSolve.apply(A.data, b, A.indptr, A.indices, solver, rtol)


__all__ = ["LinearSolve", "linear_solve"]
