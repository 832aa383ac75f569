"""The oracle's ACM and FGMRES against the reference's own.

``tests/golden/acm.npz`` holds the reference's ``ACM`` (``zvcfd/fv/linear.py:328-518``) and
its device FGMRES (``:238-320``), run in this container on the CPU (numpy in place of CuPy,
its ``bsr_mv`` kernel compiled for the CPU), on a system the reference's CPU solver assembled
(the golden tetrahedral pipe after three Picard iterations), with one coarse level
(``coarse=40``) and with two (``coarse=8``). The oracle's restatement (``oracle.linear``, set to
the reference's parameters) must give:

- the same levels and the same aggregates on every level, bit for bit;
- the same Galerkin patterns, and blocks equal to round-off (sums of the same blocks; the
  reference orders them by an unstable sort);
- the same V-cycle of the right-hand side to 1e-14, and the same ACM-FGMRES solve: the same
  number of iterations and the solution to 1e-13, the residual to 1e-3 of itself.

The bench's CPU reference arm runs this oracle ACM-FGMRES, so this pins what it times.
"""

import numpy as np
import pytest

from fixtures import load
from oracle.linear import ACM, bsr, fgmres

G = load("acm")


@pytest.mark.parametrize("coarse", [int(c) for c in G["coarse"]])
def test_oracle_acm_equals_the_reference(coarse):
    pre = f"c{coarse}_"
    acm = ACM(coarse=coarse, smooth=2, omega=0.7, passes=2, mode=0).setup(
        G["indptr"], G["indices"], G["data"])
    assert len(acm.levels) == int(G[pre + "levels"])
    for i, L in enumerate(acm.levels):
        assert L["n"] == int(G[f"{pre}level{i}_n"])
        assert ("dense_inv" in L) == bool(G[f"{pre}level{i}_dense"])
        if f"{pre}level{i}_agg" in G:
            np.testing.assert_array_equal(L["agg"], G[f"{pre}level{i}_agg"])
        if i:
            np.testing.assert_array_equal(L["ptr"], G[f"{pre}level{i}_indptr"])
            np.testing.assert_array_equal(L["idx"], G[f"{pre}level{i}_indices"])
            want = G[f"{pre}level{i}_data"]
            np.testing.assert_allclose(L["data"], want, rtol=0, atol=1e-14 * np.abs(want).max())
    z, want = acm.vcycle(G["b"].copy()), G[pre + "vcycle"]
    np.testing.assert_allclose(z, want, rtol=0, atol=1e-14 * np.abs(want).max())
    A = bsr(G["indptr"], G["indices"], G["data"], len(G["indptr"]) - 1).tocsr()
    x, it, res, ok = fgmres(lambda v: A @ v, G["b"], np.zeros_like(G["b"]), acm.vcycle,
                            rtol=1e-10, restart=30, maxiter=200)
    assert ok and bool(G[pre + "converged"])
    assert it == int(G[pre + "iterations"])
    assert abs(res - float(G[pre + "residual"])) <= 1e-3 * float(G[pre + "residual"])
    np.testing.assert_allclose(x, G[pre + "x"], rtol=0, atol=1e-13 * np.abs(G[pre + "x"]).max())
