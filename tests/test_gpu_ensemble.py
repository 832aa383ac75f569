"""Batched solves of independent instances (:mod:`zvcfd_b200.ensemble`).

Three small vessels of different kinds and sizes (a straight tet pipe, a curved hex/prism
tube, a tet Y-bifurcation), each with its own inlet flow and RCR outlets, solved together as
one block-diagonal system with the FP32 hierarchy and the lanes autotuner (one Krylov
recurrence per instance, or one over the union), reach each
instance's own FP64 solution (solved alone; both to relative changes below 1e-9) to 1e-7,
and every instance's outflows balance its inflow.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _cases():
    from zvcfd_b200.lumped import RCR
    from zvcfd_b200.mesh import curved_tube, pipe, y_bifurcation

    def shape(R):
        return lambda x: np.clip(1.0 - (x[:, 0] ** 2 + x[:, 1] ** 2) / R ** 2, 0.0, None)

    out = []
    m = pipe(1e-3, 10e-3, n_core=6, n_ring=3, n_axial=30, kind="tet", jitter_amount=0.05, seed=1)
    z = {zz.name: k for k, zz in m.zones.items()}
    out.append((m, {z["inlet"]: {"kind": "velocity", "flow_rate": 0.8e-6, "profile": shape(1e-3)},
                    z["outlet"]: {"kind": "pressure", "lumped": RCR(rp=1e8, c=1e-9, rd=8e8)},
                    z["wall"]: {"kind": "wall"}}))
    m = curved_tube(2e-3, 20e-3, np.pi / 2, n_core=8, n_ring=5, n_axial=40, layers=2, growth=0.8)
    z = {zz.name: k for k, zz in m.zones.items()}
    out.append((m, {z["inlet"]: {"kind": "velocity", "flow_rate": 2.0e-6, "profile": shape(2e-3)},
                    z["outlet"]: {"kind": "pressure", "lumped": RCR(rp=2e8, c=1e-9, rd=1e9)},
                    z["wall"]: {"kind": "wall"}}))
    m = y_bifurcation(0.6e-3)
    z = {zz.name: k for k, zz in m.zones.items()}
    out.append((m, {z["inlet"]: {"kind": "velocity", "flow_rate": 1.5e-6, "profile": shape(2e-3)},
                    z["outlet1"]: {"kind": "pressure", "lumped": RCR(rp=1e8, c=1e-9, rd=1e9)},
                    z["outlet2"]: {"kind": "pressure", "lumped": RCR(rp=1.5e8, c=1e-9, rd=1.2e9)},
                    z["wall"]: {"kind": "wall"}}))
    return out


@pytest.mark.parametrize("krylov", ["segmented", "union"])
def test_ensemble_matches_instances_solved_alone(krylov):
    from zvcfd_b200.ensemble import B200Ensemble, solve_sequentially
    from zvcfd_b200.fluid import Fluid

    cases = _cases()
    fl = Fluid(1060.0, 3.5e-3)
    alone = solve_sequentially(cases, fl, tol=1e-9, max_iterations=800, advection=1.0)
    assert all(r["converged"] for r in alone["instances"])
    ens = B200Ensemble(cases, fl, krylov=krylov, advection=1.0, linear="b200-mixed",
                       linear_options={"autotune": True})
    rep = ens.solve(tol=1e-9, max_iterations=800)
    assert rep["converged"], rep["history"][-1]
    for i, r in enumerate(alone["instances"]):
        f = ens.fields(i)
        for k in ("U", "P"):
            ref = r["fields"][k]
            assert np.linalg.norm(f[k] - ref) <= 1e-7 * np.linalg.norm(ref), (i, k)
        q = ens.patch_flows(i)
        assert abs(sum(q.values())) < 1e-8 * sum(abs(v) for v in q.values())
    ens.close()
