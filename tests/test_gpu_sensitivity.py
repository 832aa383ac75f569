"""Steady sensitivities (:mod:`zvcfd_b200.sensitivity`) against finite differences.

On the Y-bifurcation at a lattice spacing of 0.5 mm (8,410 nodes) with Carreau-Yasuda blood
and two RCR outlets, the tangent Jacobian of the outputs (the two outlet flow fractions, the
mean wall shear stress on each daughter) with respect to the parameters (inlet flow, Rp and
Rd of both outlets, C of one outlet, mu_0) equals central finite differences of full
nonlinear solves (relative step 1e-4, each solve converged to 1e-12) to 1e-5 relative, with an
absolute floor of 1e-5 of the column's largest entry; C, which a steady state does not see,
has a zero column. The autograd function returns the same gradient.
"""

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _problem():
    from zvcfd_b200.fluid import CarreauYasuda, Fluid
    from zvcfd_b200.lumped import RCR
    from zvcfd_b200.mesh import y_bifurcation
    from zvcfd_b200.sensitivity import (FlowFractions, MeanWallShear, Outputs, inlet_flow, lumped,
                                        viscosity_mu0)
    from zvcfd_b200.solver import B200Solver

    m = y_bifurcation(0.5e-3)
    z = {zz.name: k for k, zz in m.zones.items()}

    def shape(x):
        return np.clip(1.0 - (x[:, 0] ** 2 + x[:, 1] ** 2) / 2e-3 ** 2, 0.0, None)

    bcs = {z["inlet"]: {"kind": "velocity", "flow_rate": 1e-6, "profile": shape},
           z["outlet1"]: {"kind": "pressure", "lumped": RCR(rp=1e8, c=1e-9, rd=1e9)},
           z["outlet2"]: {"kind": "pressure", "lumped": RCR(rp=1.5e8, c=1e-9, rd=1.2e9)},
           z["wall"]: {"kind": "wall"}}
    s = B200Solver(m, Fluid(1060.0, 3.5e-3, viscosity=CarreauYasuda()), bcs, linear="b200")
    wall = m.zones[z["wall"]].faces
    wn = np.unique(wall[wall >= 0])
    x = m.nodes[wn]
    d1 = wn[(x[:, 2] > 2e-3) & (x[:, 0] > 0)]
    d2 = wn[(x[:, 2] > 2e-3) & (x[:, 0] < 0)]
    outputs = Outputs(FlowFractions([z["outlet1"], z["outlet2"]]),
                      MeanWallShear(m, [z["wall"]], {"daughter1": d1, "daughter2": d2}))
    params = [inlet_flow(z["inlet"]), lumped(z["outlet1"], "rp"), lumped(z["outlet1"], "rd"),
              lumped(z["outlet2"], "rp"), lumped(z["outlet2"], "rd"), lumped(z["outlet1"], "c"),
              viscosity_mu0()]
    return s, params, outputs


def test_tangent_jacobian_matches_finite_differences():
    from zvcfd_b200.sensitivity import SteadySensitivity

    s, params, outputs = _problem()
    assert s.solve(max_iterations=600, tol=1e-12)["converged"]
    sens = SteadySensitivity(s, params, outputs)
    assert sens.fixed_point_residual() < 1e-10
    jac = sens.jacobian()
    dJ = jac["dJ"]
    z0 = sens.z0
    for k, p in enumerate(params):
        v0 = p.get(s)
        h = 1e-4 * abs(v0)
        out = []
        for v in (v0 + h, v0 - h):
            sens.set_state(z0)
            p.set(s, v)
            assert s.solve(max_iterations=600, tol=1e-12)["converged"]
            out.append(outputs(s).numpy())
        sens.set_state(z0)
        p.set(s, v0)
        fd = (out[0] - out[1]) / (2 * h)
        col = dJ[:, k]
        scale = max(np.abs(fd).max(), np.abs(col).max()) * v0
        if p.name.startswith("c["):
            assert np.abs(col).max() * v0 <= 1e-9 * np.abs(jac["outputs"]).max(), col
            continue
        np.testing.assert_allclose(col * v0, fd * v0, rtol=1e-5, atol=1e-5 * scale,
                                   err_msg=p.name)
    s.close()


def test_autograd_function_returns_the_tangent_gradient():
    from zvcfd_b200.sensitivity import SteadySensitivity, steady_outputs

    s, params, outputs = _problem()
    theta = torch.tensor([p.get(s) for p in params], dtype=torch.float64, requires_grad=True)
    J = steady_outputs(theta, s, params, outputs, tol=1e-12, max_iterations=600)
    w = torch.tensor([1.0, -1.0, 0.5, 0.25], dtype=torch.float64)
    (J * w).sum().backward()
    ref = SteadySensitivity(s, params, outputs).jacobian()["dJ"]
    np.testing.assert_allclose(theta.grad.numpy(), w.numpy() @ ref, rtol=1e-6,
                               atol=1e-9 * np.abs(w.numpy() @ ref).max())
    s.close()
