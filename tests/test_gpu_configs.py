"""The plain FP64 Poiseuille pipe (the CPU-runnable benchmark case) on the device.

Geometry radius 1 mm, length 10 mm; an O-grid section of 14 core and 7 ring cells swept over
80 axial cells, each hexahedron split into six tets, interior nodes jittered by up to 5 % of
their shortest edge (seed 0): 49,977 nodes. Newtonian fluid rho 1060, mu 3.5e-3; a parabolic
inlet of mean velocity 0.1 m/s, p = 0 at the outlet, no-slip walls.

- The converged axial velocity equals the analytic profile u = 2 U (1 - r^2/R^2) in the
  middle of the pipe to 2 % relative L2, and the pressure gradient equals -8 mu U / R^2 to 2 %.
- The mixed-precision solve (FP32 hierarchy) reaches the same fields as the FP64 one to 1e-6
  relative (the field-error bound of the mixed-precision form).
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

R, L, UMEAN, RHO, MU = 1e-3, 10e-3, 0.1, 1060.0, 3.5e-3


def _case():
    from zvcfd_b200.fluid import Fluid
    from zvcfd_b200.mesh import pipe

    m = pipe(R, L, n_core=14, n_ring=7, n_axial=80, kind="tet", jitter_amount=0.05, seed=0)
    z = {zz.name: k for k, zz in m.zones.items()}

    def inlet(x):
        r2 = (x[:, 0] ** 2 + x[:, 1] ** 2) / R ** 2
        return np.stack([0 * r2, 0 * r2, 2 * UMEAN * np.clip(1 - r2, 0, None)], 1)

    bcs = {z["inlet"]: {"kind": "velocity", "value": inlet},
           z["outlet"]: {"kind": "pressure", "value": 0.0}, z["wall"]: {"kind": "wall"}}
    return m, Fluid(RHO, MU), bcs


def test_poiseuille_pipe_matches_the_analytic_profile_fp64_and_mixed():
    from zvcfd_b200.solver import B200Solver

    m, fl, bcs = _case()
    assert m.n_nodes == 49977
    out = {}
    for linear in ("b200", "b200-mixed"):
        s = B200Solver(m, fl, bcs, linear=linear, linear_rtol=0.1)
        rep = s.solve(max_iterations=400, tol=1e-8)
        assert rep["converged"], rep["history"][-1]
        out[linear] = s.fields()
        s.close()
    x = m.nodes
    mid = (x[:, 2] > 0.3 * L) & (x[:, 2] < 0.7 * L)
    r2 = (x[mid, 0] ** 2 + x[mid, 1] ** 2) / R ** 2
    exact = 2 * UMEAN * np.clip(1 - r2, 0, None)
    U, P = out["b200"]["U"], out["b200"]["P"]
    err = np.linalg.norm(U[mid, 2] - exact) / np.linalg.norm(exact)
    assert err < 0.02, err
    slope = np.polyfit(x[mid, 2], P[mid], 1)[0]
    dpdz = -8 * MU * UMEAN / R ** 2
    assert abs(slope - dpdz) < 0.02 * abs(dpdz), (slope, dpdz)
    Um, Pm = out["b200-mixed"]["U"], out["b200-mixed"]["P"]
    assert np.linalg.norm(Um - U) <= 1e-6 * np.linalg.norm(U)
    assert np.linalg.norm(Pm - P) <= 1e-6 * np.linalg.norm(P)
