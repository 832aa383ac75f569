"""Host pieces of the parameter adjoint (CPU): the flexible GMRES that solves the adjoint
systems, and the zero-slope square root of the shear rate."""

import torch


def test_fgmres_reaches_the_direct_solution():
    from zvcfd_b200.sensitivity import fgmres

    g = torch.Generator().manual_seed(0)
    n = 200
    A = 4 * torch.eye(n, dtype=torch.float64) + 0.1 * torch.randn(n, n, generator=g,
                                                                   dtype=torch.float64)
    b = torch.randn(n, generator=g, dtype=torch.float64)
    d = torch.diag(A).clone()
    x, its, res = fgmres(lambda v: A @ v, b, lambda v: v / d, rtol=1e-12, restart=30)
    assert res <= 1e-12 and its < 60
    ref = torch.linalg.solve(A, b)
    assert torch.linalg.norm(x - ref) <= 1e-11 * torch.linalg.norm(ref)
    # restarts: a short restart length still gets there
    x, its, res = fgmres(lambda v: A @ v, b, lambda v: v / d, rtol=1e-12, restart=5)
    assert res <= 1e-12 and torch.linalg.norm(x - ref) <= 1e-11 * torch.linalg.norm(ref)
    # a zero right-hand side
    x, its, res = fgmres(lambda v: A @ v, torch.zeros(n, dtype=torch.float64), lambda v: v)
    assert its == 0 and float(x.abs().max()) == 0.0


def test_shear_rate_has_a_zero_slope_at_rest():
    from zvcfd_b200.sensitivity import _rate

    L = torch.zeros((3, 3, 3), dtype=torch.float64)
    L[1, 0, 1] = 2.0
    L.requires_grad_(True)
    r = _rate(L)
    assert float(r[0]) == 0.0 and abs(float(r[1]) - 2.0) < 1e-15
    (g,) = torch.autograd.grad(r.sum(), L)
    assert torch.isfinite(g).all() and float(g[0].abs().max()) == 0.0
