"""The Chebyshev smoother of the device AMG (``smoother="chebyshev"``).

- The spectral bound: ``cheb_power`` steps of the power iteration on ``D^-1 A`` of the finest
  level, restated here in NumPy from the same start vector, give the device's estimate to
  round-off.
- On a one-level hierarchy the V-cycle is ``coarse_sweeps`` Chebyshev steps from zero,
  restated here with the device's estimate: equal to round-off.
- FGMRES preconditioned by the Chebyshev V-cycle solves an assembled system (FP64 and FP32
  hierarchy) and its transpose to the direct solutions.
- The outer loop with it reaches the reference's converged fields of a golden pipe.
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


def _start(m):
    """The device's power-iteration start: 0.5 plus the top 53 bits of a 64-bit mix of the
    index as a fraction of one."""
    with np.errstate(over="ignore"):
        h = np.arange(m, dtype=np.uint64) * np.uint64(0x9E3779B97F4A7C15) + np.uint64(0x632BE59BD9B4E019)
        h ^= h >> np.uint64(31)
        h *= np.uint64(0xBF58476D1CE4E5B9)
        h ^= h >> np.uint64(27)
    return 0.5 + (h >> np.uint64(11)).astype(np.float64) / 2.0 ** 53


def test_spectral_estimate_matches_power_iteration():
    import ctypes

    from zvcfd_b200._lib import call
    from zvcfd_b200.linear import B200AMG

    s, A, b, x0 = _system()
    solver = B200AMG(smoother="chebyshev", precision="double", cheb_power=12)
    solver.setup(A)
    v = ctypes.c_double()
    call("zvfv_solver_get_option", solver._h, b"cheb_lmax", ctypes.byref(v))
    ip, ix, data = A.indptr.cpu().numpy(), A.indices.cpu().numpy(), A.data.cpu().numpy()
    M = bsr(ip, ix, data, A.n).tocsr()
    blocks = data.reshape(-1, 4, 4)
    diag = np.stack([blocks[ip[i] + np.flatnonzero(ix[ip[i]:ip[i + 1]] == i)[0]]
                     for i in range(A.n)])
    Dinv = np.linalg.inv(diag)
    x = _start(4 * A.n)
    for _ in range(12):
        w = np.einsum("nij,nj->ni", Dinv, (M @ x).reshape(-1, 4)).reshape(-1)
        lam = np.linalg.norm(w)
        x = w / lam
    assert abs(v.value - lam) <= 1e-10 * lam, (v.value, lam)
    # the bound covers the spectrum of D^-1 A (its dominant eigenvalue, by a dense solve)
    ev = np.linalg.eigvals(_dense_dinv_a(M, Dinv))
    rho = np.abs(ev).max()
    assert 0.8 * rho <= v.value <= 1.3 * rho, (v.value, rho)
    solver.close()
    s.close()


def _dense_dinv_a(M, Dinv):
    n = Dinv.shape[0]
    D = np.zeros((4 * n, 4 * n))
    for i in range(n):
        D[4 * i:4 * i + 4, 4 * i:4 * i + 4] = Dinv[i]
    return D @ M.toarray()


def test_one_level_chebyshev_cycle_matches_restatement():
    """One level: the V-cycle is ``coarse_sweeps`` Chebyshev steps from zero on the finest
    level, restated here with the device's spectral estimate."""
    import ctypes

    from zvcfd_b200._lib import call
    from zvcfd_b200.linear import B200AMG

    s, A, b, x0 = _system()
    solver = B200AMG(smoother="chebyshev", precision="double", max_levels=1, coarse_sweeps=4)
    solver.setup(A)
    v, ratio = ctypes.c_double(), ctypes.c_double()
    call("zvfv_solver_get_option", solver._h, b"cheb_lmax", ctypes.byref(v))
    call("zvfv_solver_get_option", solver._h, b"cheb_ratio", ctypes.byref(ratio))
    g = torch.Generator(device="cuda").manual_seed(5)
    r = torch.randn(A.n * 4, dtype=torch.float64, device="cuda", generator=g)
    z = solver.vcycle(r).cpu().numpy()
    ip, ix, data = A.indptr.cpu().numpy(), A.indices.cpu().numpy(), A.data.cpu().numpy()
    M = bsr(ip, ix, data, A.n).tocsr()
    blocks = data.reshape(-1, 4, 4)
    Dinv = np.linalg.inv(np.stack([blocks[ip[i] + np.flatnonzero(ix[ip[i]:ip[i + 1]] == i)[0]]
                                   for i in range(A.n)]))
    hi = 1.1 * v.value
    lo = hi / ratio.value
    theta, delta = 0.5 * (hi + lo), 0.5 * (hi - lo)
    sigma = theta / delta
    rh = r.cpu().numpy()
    x = np.zeros_like(rh)
    d = np.zeros_like(rh)
    rho = 1.0 / sigma
    for k in range(4):
        zk = np.einsum("nij,nj->ni", Dinv, (rh - M @ x).reshape(-1, 4)).reshape(-1)
        if k == 0:
            d = zk / theta
        else:
            nxt = 1.0 / (2.0 * sigma - rho)
            d = nxt * rho * d + 2.0 * nxt / delta * zk
            rho = nxt
        x = x + d
    np.testing.assert_allclose(z, x, rtol=0, atol=1e-11 * np.abs(x).max())
    solver.close()
    s.close()


@pytest.mark.parametrize("precision", ["double", "mixed"])
def test_chebyshev_fgmres_solves_to_direct_solution(precision):
    import scipy.sparse.linalg as spl

    from zvcfd_b200.linear import B200AMG

    s, A, b, x0 = _system()
    M = bsr(A.indptr.cpu().numpy(), A.indices.cpu().numpy(), A.data.cpu().numpy(), A.n).tocsc()
    bh = b.cpu().numpy()
    for transposed in (False, True):
        solver = B200AMG(smoother="chebyshev", precision=precision, rtol=1e-10, maxiter=400)
        x, info = solver.solve(A, b, x0, transposed=transposed)
        assert info.converged, (transposed, info)
        Mt = M.T.tocsc() if transposed else M
        ref = spl.splu(Mt).solve(bh)
        np.testing.assert_allclose(x.cpu().numpy(), ref, atol=1e-7 * np.abs(ref).max())
        r = bh - Mt @ x.cpu().numpy()
        r0 = bh - Mt @ x0.cpu().numpy()
        assert np.linalg.norm(r) <= 1.01e-10 * np.linalg.norm(r0) + 1e-13 * np.linalg.norm(bh)
        solver.close()
    s.close()


def test_chebyshev_outer_loop_matches_reference():
    from zvcfd_b200.solver import B200Solver

    name = "pipe_tet_si"
    g = load(name)
    m = mesh_of(g)
    s = B200Solver(m, fluid_of(g), pipe_bcs(name, g, m), advection=1.0,
                   linear_options={"smoother": "chebyshev"})
    rep = s.solve(max_iterations=800, tol=1e-11)
    assert rep["converged"], rep["history"][-1]
    f = s.fields()
    U, P = g["U"], g["P"]
    assert np.linalg.norm(f["U"] - U) <= 1e-8 * np.linalg.norm(U)
    assert np.linalg.norm(f["P"] - P) <= 1e-8 * np.linalg.norm(P - P.mean()) + 1e-9 * np.ptp(P)
    s.close()
