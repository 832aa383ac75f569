"""The ``b200-auto`` ladder (the reference's ``Auto`` semantics, ``zvcfd/fv/linear.py:1060-1171``)
on the device solvers.

- Driving the outer loop of a golden pipe, the ladder reaches the reference's converged fields
  (relative L2 <= 1e-8), records its probe of the robust rung at the third solve, and every
  rung it used is one of the four device configurations.
- A first rung that cannot converge (its iteration budget cut to one) is abandoned for the next
  rung on the first solve, with the reason recorded, and the solve still reaches its tolerance.
"""

import numpy as np
import pytest

from fixtures import fluid_of, load, mesh_of, pipe_bcs

pytestmark = pytest.mark.gpu


def test_auto_ladder_reaches_the_reference_fields():
    from zvcfd_b200.linear import make
    from zvcfd_b200.solver import B200Solver

    g = load("pipe_tet_si")
    m = mesh_of(g)
    lad = make("b200-auto", rtol=0.1)
    s = B200Solver(m, fluid_of(g), pipe_bcs("pipe_tet_si", g, m), advection=1.0, linear=lad)
    rep = s.solve(max_iterations=800, tol=1e-11)
    assert rep["converged"], rep["history"][-1]
    f = s.fields()
    assert np.linalg.norm(f["U"] - g["U"]) <= 1e-8 * np.linalg.norm(g["U"])
    assert np.linalg.norm(f["P"] - g["P"]) <= 1e-8 * np.linalg.norm(g["P"] - g["P"].mean()) + \
        1e-9 * np.ptp(g["P"])
    assert lad.probe is not None and set(lad.probe) == {"first_s", "probe_s", "probe_converged"}
    assert lad.active in lad.names
    for a, b, why in lad.switches:
        assert a in lad.names and b in lad.names and why
    s.close()


def test_auto_ladder_moves_on_from_a_failing_rung():
    import torch

    from zvcfd_b200.linear import B200AMG, Ladder
    from zvcfd_b200.solver import B200Solver

    g = load("pipe_tet_si")
    m = mesh_of(g)
    s = B200Solver(m, fluid_of(g), pipe_bcs("pipe_tet_si", g, m), advection=1.0)
    for _ in range(2):
        s.iterate()
    A, b, _, x0 = s._assemble_fused()
    b = b.reshape(-1).clone()
    lad = Ladder([("starved", lambda: B200AMG(rtol=1e-8, maxiter=1)),
                  ("b200-gs", lambda: B200AMG(rtol=1e-8))], rtol=1e-8, probe_at=None)
    x, info = lad.solve(A, b, x0)
    assert lad.active == "b200-gs" and len(lad.switches) == 1
    assert lad.switches[0][:2] == ("starved", "b200-gs")
    assert "residual" in lad.switches[0][2]
    assert info.converged and info.residual <= 1.01e-8
    r = b - A.matvec(x)
    assert float(torch.linalg.norm(r)) <= 1.01e-8 * float(torch.linalg.norm(b - A.matvec(x0))) \
        + 1e-13 * float(torch.linalg.norm(b))
    lad.close()
    s.close()
