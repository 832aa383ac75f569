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


def test_batched_fgmres_matches_one_solve_per_system():
    """Lock-step recurrences: each system reaches its own solution; a zero right-hand side
    takes no steps; a system that converges early freezes while the others go on."""
    from zvcfd_b200.sensitivity import fgmres, fgmres_batched

    g = torch.Generator().manual_seed(1)
    n = 150
    A = 4 * torch.eye(n, dtype=torch.float64) + 0.1 * torch.randn(n, n, generator=g,
                                                                   dtype=torch.float64)
    d = torch.diag(A).clone()
    b = torch.randn(4, n, generator=g, dtype=torch.float64)
    b[2] = 0.0
    b[3] = A @ torch.ones(n, dtype=torch.float64) * 1e-3      # an easier system
    x, its, res = fgmres_batched(lambda v: v @ A.T, b, lambda v: v / d, rtol=1e-12, restart=7)
    assert (res <= 1e-12).all(), res
    assert float(x[2].abs().max()) == 0.0
    for q in (0, 1, 3):
        ref = torch.linalg.solve(A, b[q])
        assert torch.linalg.norm(x[q] - ref) <= 1e-11 * torch.linalg.norm(ref)
        x1, _, _ = fgmres(lambda v: A @ v, b[q], lambda v: v / d, rtol=1e-12, restart=7)
        assert torch.linalg.norm(x[q] - x1) <= 1e-11 * torch.linalg.norm(ref)


def test_rcr_step_restates_the_outlet_model():
    """The differentiable RCR step is the model's own affine step, trapezoidal and Euler."""
    from zvcfd_b200.lumped import RCR
    from zvcfd_b200.sensitivity import rcr_step

    for method in ("trapezoidal", "euler"):
        m = RCR(rp=1.2e8, c=0.8e-9, rd=1.1e9, pv=0.0, method=method)
        m.initialise(2e-6, 0.3)
        m.advance(2.1e-6, 0.301, 1e-3)
        want = m._affine_step(0.302, 1e-3)
        t = lambda v: torch.tensor(v, dtype=torch.float64, requires_grad=True)   # noqa: E731
        got = rcr_step(m, t(m.pc), t(m.q), t(m.rp), t(m.c), t(m.rd), 0.302, 1e-3)
        assert abs(float(got[0]) - want[0]) <= 1e-12 * abs(want[0])
        assert abs(float(got[1]) - want[1]) <= 1e-12 * abs(want[1])
