"""The oracle's boundary pass against the reference's own ``finalise`` kernel.

``tests/golden/boundary_pass.npz`` holds the outputs of the reference's device boundary pass
(``zvcfd/fv/_cuda_bc.py:32-138``), run in this container on the CPU (its kernel source compiled
by g++, each thread block's threads as OpenMP threads with ``__syncthreads`` a barrier), on the
raw system the oracle assembles for the golden tetrahedral pipe after three outer iterations
with a false time step, with and without symmetric elimination. Its known-term inputs are zero
(the raw system holds those terms), so it computes what ``OracleSolver.boundary_pass``
restates: Dirichlet rows, elimination, the residual of the current state, the dimensionless row
scaling. The oracle must give the same scaled blocks, right-hand side and row scales to 1e-15
of their largest entries and the same residual maxima to 1e-13. The device pass is held to the
oracle's on a B200 (``tests/test_gpu_boundary_pass.py``), so it is pinned to the reference's.
"""

import types

import numpy as np
import pytest

from fixtures import load
from oracle.fv import OracleSolver

G = load("boundary_pass")


def _state(tag):
    g = {k[len(tag) + 1:]: v for k, v in G.items() if k.startswith(tag + "_")}
    fixed = g["fixed"]
    return g, types.SimpleNamespace(
        N=len(g["aP"]), fluid=types.SimpleNamespace(rho=float(g["rho"])),
        vel_fixed_comp=fixed[:, :3], p_fixed=fixed[:, 3], vel_value=g["vel"], p_value=g["pval"],
        U=g["U"], P=g["P"], V=g["V"], indptr=g["indptr"], indices=g["indices"], aP=g["aP"])


@pytest.mark.parametrize("eliminate", [1, 0])
def test_oracle_boundary_pass_equals_the_reference_kernel(eliminate):
    g, state = _state("dt")
    data, b, scale, stats = OracleSolver.boundary_pass(state, g["raw"], g["braw"], g["x"],
                                                       eliminate=bool(eliminate))
    key = f"e{eliminate}_"
    for got, name in ((data, "data"), (b, "b"), (scale, "scale")):
        want = g[key + name].reshape(got.shape)
        np.testing.assert_allclose(got, want, rtol=0, atol=1e-15 * np.abs(want).max())
    np.testing.assert_allclose(stats["max"], g[key + "max"], rtol=1e-13, atol=0)
    # with elimination the known columns of free rows are empty
    if eliminate:
        fixed = g["fixed"]
        rows = np.repeat(np.arange(state.N), np.diff(g["indptr"]))
        want = g[key + "data"].reshape(-1, 4, 4)
        for r in range(4):
            for c in range(4):
                assert np.all(want[fixed[g["indices"], c] & ~fixed[rows, r], r, c] == 0.0)
