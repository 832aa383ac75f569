"""Steady sensitivities (:mod:`zvcfd_b200.sensitivity`) against finite differences.

On the golden curved Carreau-Yasuda tube (the reference's solution case) with an RCR outlet,
the gradient that the autograd function returns for a weighted sum of the outputs (the
outlet's mean pressure and the mean wall shear stress) with respect to the inlet flow, the
outlet's distal resistance and mu_0 equals the same weighted sum of central finite
differences of full nonlinear solves, to 2e-5 relative. The finite differences take a
relative step of 1e-3: each solve stops at a relative change of 1e-10, which leaves about
1e-9 in the outputs; a step of 1e-6 would turn that into errors of 1e-3, while at 1e-3 the
O(h^2) truncation stays near 1e-6.
"""

import numpy as np
import pytest
import torch

from fixtures import fluid_of, load, mesh_of, pipe_bcs

pytestmark = pytest.mark.gpu


def _problem():
    from zvcfd_b200.lumped import RCR
    from zvcfd_b200.sensitivity import (MeanWallShear, Outputs, ZonePressures, inlet_flow, lumped,
                                        viscosity_mu0)
    from zvcfd_b200.solver import B200Solver

    g = load("curved_cy")
    m = mesh_of(g)
    z = {zz.name: k for k, zz in m.zones.items()}
    bcs = pipe_bcs("curved_cy", g, m)
    bcs[z["outlet"]] = {"kind": "pressure", "lumped": RCR(rp=1e8, c=1e-9, rd=1e9)}
    s = B200Solver(m, fluid_of(g), bcs, linear="b200")
    wall = m.zones[z["wall"]].faces
    outputs = Outputs(ZonePressures([z["outlet"]]),
                      MeanWallShear(m, [z["wall"]], {"wall": np.unique(wall[wall >= 0])}))
    params = [inlet_flow(z["inlet"]), lumped(z["outlet"], "rd"), viscosity_mu0()]
    return s, params, outputs


def test_autograd_gradient_matches_finite_differences():
    from zvcfd_b200.sensitivity import steady_outputs

    s, params, outputs = _problem()
    theta0 = np.array([p.get(s) for p in params])
    theta = torch.tensor(theta0, dtype=torch.float64, requires_grad=True)
    J = steady_outputs(theta, s, params, outputs, tol=1e-10, max_iterations=800)
    w = np.array([1e-3, 1.0])
    (J * torch.as_tensor(w)).sum().backward()
    grad = theta.grad.numpy()
    U0, P0 = s.U.clone(), s.P.clone()
    mdot0 = {k: v.clone() for k, v in s.mdot.items()}
    fd = np.zeros(len(params))
    for k, p in enumerate(params):
        h = 1e-3 * abs(theta0[k])
        vals = []
        for v in (theta0[k] + h, theta0[k] - h):
            s.U, s.P = U0.clone(), P0.clone()
            s.mdot = {kk: vv.clone() for kk, vv in mdot0.items()}
            p.set(s, v)
            assert s.solve(max_iterations=800, tol=1e-10)["converged"]
            vals.append(float(w @ outputs(s).numpy()))
        p.set(s, theta0[k])
        fd[k] = (vals[0] - vals[1]) / (2 * h)
    scale = np.abs(fd * theta0).max()
    np.testing.assert_allclose(grad * theta0, fd * theta0, rtol=2e-5, atol=2e-5 * scale)
    s.close()
