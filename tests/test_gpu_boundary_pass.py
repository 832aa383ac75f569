"""The device boundary pass row by row against the oracle's restatement.

``zvfv_finalise`` (``zvcfd/fv/_cuda_bc.py:32-138``, launched at ``zvcfd/fv/solver.py:669-677``)
turns the element-assembled system into the scaled Dirichlet system the linear solver sees:
time and boundary terms on the raw rows, the raw rows of fixed-velocity nodes kept, Dirichlet
rows, with ``eliminate`` the known values moved out of the free rows, the normalised residual
statistics of the current state, and the dimensionless row scaling. The oracle restates the
same pass (``OracleSolver.boundary_pass``). Both sides start from one state (the oracle's,
after three outer iterations of a golden pipe), so the device's element assembly reproduces the
oracle's raw system to round-off and every output of the pass can be compared directly: the
scaled blocks and right-hand side, the row scales, the kept raw rows and the residual partials,
with and without elimination, steady and with a false time step.
"""

import numpy as np
import pytest
import torch

from fixtures import fluid_of, load, mesh_of, pipe_bcs

pytestmark = pytest.mark.gpu


def _columns_close(dev, ref, rtol, what):
    """Each column of ``dev`` within ``rtol`` of that column's largest entry of ``ref``."""
    for c in range(ref.shape[1]):
        scale = max(np.abs(ref[:, c]).max(), 1e-300)
        err = np.abs(dev[:, c] - ref[:, c])
        worst = int(err.argmax())
        assert err.max() <= rtol * scale, (what, c, worst, dev[worst, c], ref[worst, c], scale)


def _rowwise_close(dev, ref, rtol):
    """``dev`` within ``rtol`` of each block row's largest entry of ``ref`` ((nnzb, 4, 4))."""
    scale = np.abs(ref).max(axis=2, keepdims=True)
    assert np.all(np.abs(dev - ref) <= rtol * scale + 1e-300), np.abs(dev - ref).max()


@pytest.mark.parametrize("dt", [None, 0.02])
@pytest.mark.parametrize("eliminate", [True, False])
def test_finalise_matches_the_oracle_boundary_pass(eliminate, dt):
    from oracle.fv import OracleSolver
    from zvcfd_b200._lib import call, ptr, stream_ptr
    from zvcfd_b200.solver import B200Solver

    name = "pipe_tet_si"
    g = load(name)
    m = mesh_of(g)
    fl = fluid_of(g)
    o = OracleSolver(m, fl, pipe_bcs(name, g, m), advection=1.0, dt=dt)
    o.solve(max_iterations=3, tol=0.0)
    diag_o = o.momentum_diagonal()
    o.assemble()
    raw, braw = o.raw
    X = np.concatenate([o.U, o.P[:, None]], 1)
    data_o, b_o, scale_o, stats_o = o.boundary_pass(raw, braw, X, eliminate=eliminate)

    s = B200Solver(m, fl, pipe_bcs(name, g, m), advection=1.0, dt=dt, eliminate=eliminate)
    s.U = torch.as_tensor(o.U, device="cuda").clone()
    s.P = torch.as_tensor(o.P, device="cuda").clone()
    s.mdot = s.asm.to_slots({K.kind: K.mdot for K in o.kinds})
    s._vdiag = None
    s._adv = torch.as_tensor(diag_o, device="cuda") - s.asm.dvisc     # a_P = dvisc + adv
    s._mb = torch.as_tensor(o._mb, device="cuda").clone()
    A, b, scal, x = s._assemble_fused()
    torch.cuda.synchronize()
    np.testing.assert_allclose(x.cpu().numpy(), X.reshape(-1), rtol=0, atol=0)
    # the scaled Dirichlet system, its right-hand side and the row scales
    _rowwise_close(A.data.cpu().numpy().reshape(-1, 4, 4), data_o, 1e-10)
    bd = b.cpu().numpy().reshape(-1, 4)
    _columns_close(bd, b_o, 1e-10, "b")
    _columns_close(s.rs.cpu().numpy().reshape(-1, 4), scale_o, 1e-10, "row scales")
    # fixed rows: scaled unit rows; eliminated columns of free rows: empty
    fixed = np.concatenate([o.vel_fixed_comp, o.p_fixed[:, None]], 1)
    rows = np.repeat(np.arange(o.N), np.diff(o.indptr))
    dev = A.data.cpu().numpy().reshape(-1, 4, 4)
    if eliminate:
        for r in range(4):
            for c in range(4):
                assert np.all(dev[fixed[o.indices, c] & ~fixed[rows, r], r, c] == 0.0)
    # the kept raw rows (fixed-velocity nodes: reactions and zone forces)
    off = s._rawoff.cpu().numpy()
    rawd = s.rawdata.cpu().numpy().reshape(-1, 4, 4)
    rawb = s.rawb.cpu().numpy().reshape(-1, 4)
    kept = np.flatnonzero(off >= 0)
    assert len(kept) == int(o.vel_fixed_comp.any(1).sum())
    for i in kept:
        span = slice(o.indptr[i], o.indptr[i + 1])
        _rowwise_close(rawd[off[i]:off[i] + o.indptr[i + 1] - o.indptr[i]], raw[span], 1e-10)
        assert np.abs(rawb[i] - braw[i]).max() <= 1e-10 * np.abs(braw).max(), (i, rawb[i], braw[i])
    # residual partials of the free rows, folded: sums of squares and maxima per equation
    out = torch.empty(8, dtype=torch.float64, device="cuda")
    call("zvfv_fold", s._nfin, 8, ptr(s._fin_part), ptr(s._fin_ops), ptr(out), stream_ptr())
    folded = out.cpu().numpy()
    np.testing.assert_allclose(folded[:4], stats_o["sq"], rtol=1e-8, atol=1e-300)
    np.testing.assert_allclose(folded[4:], stats_o["max"], rtol=1e-8, atol=1e-300)
    np.testing.assert_allclose(scal.cpu().numpy()[:2],
                               [max(np.abs(o.U).max(), np.abs(o.vel_value).max()),
                                max(np.ptp(o.P), fl.rho * max(np.abs(o.U).max(),
                                                              np.abs(o.vel_value).max()) ** 2)],
                               rtol=1e-14)
    s.close()
