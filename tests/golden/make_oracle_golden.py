"""Converged fields of the plain FP64 Poiseuille pipe (49,977 nodes) from the oracle.

The reference's own CPU solver does not finish at this size (its SuperLU factorisation of one
linearisation ran for half an hour without ending), so the golden fields come from the oracle,
the NumPy restatement of that solver which the other goldens pin to the reference on smaller
meshes: the same lagged Rhie-Chow outer iteration, each linearisation solved by the oracle's
restatement of the reference's ACM inside FGMRES to 1e-9 (with the whole-array pairwise
matching). The advection blend is fixed (1.0) so that the converged state does not depend on
the linear solver's path (a High Resolution limiter freezes at iteration 10).

    python tests/golden/make_oracle_golden.py       # writes tests/golden/c0_pipe.npz

The mesh is not stored: the test rebuilds it with ``zvcfd_b200.mesh.pipe`` (seeded) and checks
its node count and coordinate checksum against the ones recorded here.
"""

from __future__ import annotations

import sys
import time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parents[1]))

from oracle.fv import OracleSolver  # noqa: E402
from oracle.linear import ACM, fgmres, pairwise_arrays  # noqa: E402
from zvcfd_b200.fluid import Fluid  # noqa: E402
from zvcfd_b200.mesh import pipe  # noqa: E402

R, L, UMEAN, RHO, MU = 1e-3, 10e-3, 0.1, 1060.0, 3.5e-3


def c0_case():
    m = pipe(R, L, n_core=14, n_ring=7, n_axial=80, kind="tet", jitter_amount=0.05, seed=0)
    z = {zz.name: k for k, zz in m.zones.items()}

    def inlet(x):
        r2 = (x[:, 0] ** 2 + x[:, 1] ** 2) / R ** 2
        return np.stack([0 * r2, 0 * r2, 2 * UMEAN * np.clip(1 - r2, 0, None)], 1)

    bcs = {z["inlet"]: {"kind": "velocity", "value": inlet},
           z["outlet"]: {"kind": "pressure", "value": 0.0}, z["wall"]: {"kind": "wall"}}
    return m, Fluid(RHO, MU), bcs


def main():
    m, fl, bcs = c0_case()
    s = OracleSolver(m, fl, bcs, advection=1.0)
    acm = ACM(coarse=400, matcher=pairwise_arrays, rebuild_every=10)
    t0 = time.time()

    def linear(data, b, x0):
        A = s.system_matrix(data).tocsr()
        acm.setup(s.indptr, s.indices, data)
        x, its, res, ok = fgmres(lambda v: A @ v, b, x0, acm.vcycle, rtol=1e-9, maxiter=600)
        print(f"  linear {its} its, residual {res:.1e}, {time.time() - t0:.0f} s", flush=True)
        return x

    rep = s.solve(max_iterations=200, tol=1e-11, linear=linear,
                  log=lambda msg: print(msg, flush=True))
    assert rep["converged"], rep["history"][-1]
    np.savez_compressed(HERE / "c0_pipe.npz", U=s.U, P=s.P, n_nodes=m.n_nodes,
                        node_checksum=float(np.abs(m.nodes).sum()), iterations=rep["iterations"],
                        rho=RHO, mu=MU, radius=R, length=L, umean=UMEAN)
    print("wrote c0_pipe", rep["iterations"], "iterations", flush=True)


if __name__ == "__main__":
    main()
