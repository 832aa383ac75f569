"""Parameter gradients of a steady solve by the discrete adjoint, against finite differences.

A small Y-bifurcation (the adjoint workload's geometry shortened and coarsened: parent radius 2 mm,
daughters 1.6 and 1.4 mm at +-35 degrees), Carreau-Yasuda blood, a 1 ml/s flow-rate inlet and
RCR outlets (Rp 1e8, C 1e-9, Rd 1e9), a fixed advection blend, solved to round-off. Objectives:
the two outlet flow fractions and the mean wall shear stress on each daughter's wall.
Parameters: the inlet flow, each outlet's (Rp, C, Rd) and mu0. The adjoint gradient (the four
objectives' FGMRES solves in lock-step with batched reverse passes, preconditioned by the
forward hierarchy's transposed V-cycle; the same solved one after another agrees to 1e-6,
both adjoints being solved to 1e-10) must
match central differences of converged solves (step 1e-6 relative) to 1e-5 of each objective's
largest sensitivity, and the capacitances must not matter in a steady state.
"""

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

NAMES = ["Q_in", "Rp1", "C1", "Rd1", "Rp2", "C2", "Rd2", "mu0"]


def _case(theta):
    from zvcfd_b200.fluid import CarreauYasuda, Fluid
    from zvcfd_b200.lumped import RCR
    from zvcfd_b200.mesh import y_bifurcation

    q, rp1, c1, rd1, rp2, c2, rd2, mu0 = (float(v) for v in theta)
    m = y_bifurcation(0.5e-3, parent=(2e-3, 8e-3),
                      daughters=((1.6e-3, 6e-3, 35.0), (1.4e-3, 6e-3, -35.0)))
    z = {zz.name: k for k, zz in m.zones.items()}

    def shape(x):
        return np.clip(1.0 - (x[:, 0] ** 2 + x[:, 1] ** 2) / 2e-3 ** 2, 0.0, None)

    bcs = {z["inlet"]: {"kind": "velocity", "flow_rate": q, "profile": shape},
           z["outlet1"]: {"kind": "pressure", "lumped": RCR(rp=rp1, c=c1, rd=rd1)},
           z["outlet2"]: {"kind": "pressure", "lumped": RCR(rp=rp2, c=c2, rd=rd2)},
           z["wall"]: {"kind": "wall"}}
    fl = Fluid(1060.0, 0.00345, viscosity=CarreauYasuda(mu_0=mu0))
    return m, fl, bcs, z


def _walls(m, z):
    """Wall nodes of each daughter: beyond the junction, on either side of the x = 0 plane."""
    f = m.zones[z["wall"]].faces
    nodes = np.unique(f[f >= 0])
    x = m.nodes[nodes]
    beyond = x[:, 2] > 2.5e-3
    return {"daughter1": torch.as_tensor(nodes[beyond & (x[:, 0] > 0)], device="cuda"),
            "daughter2": torch.as_tensor(nodes[beyond & (x[:, 0] < 0)], device="cuda")}


def _solve(theta, start=None):
    from zvcfd_b200.sensitivity import SteadyResidual
    from zvcfd_b200.solver import B200Solver

    m, fl, bcs, z = _case(theta)
    s = B200Solver(m, fl, bcs, advection=1.0, linear_rtol=0.1)
    if start is not None:
        s.initialise(U=start[0], P=start[1])
    rep = s.solve(max_iterations=1500, tol=1e-12)
    assert rep["converged"], rep["history"][-1]
    return SteadyResidual(s, z["inlet"], [z["outlet1"], z["outlet2"]], _walls(m, z))


def test_adjoint_gradients_match_central_differences():
    theta0 = np.array([1e-6, 1e8, 1e-9, 1e9, 1e8, 1e-9, 1e9, 0.056])
    res = _solve(theta0)
    x, mdot = res.state()
    th = res.theta0()
    np.testing.assert_allclose(th.cpu().numpy(), theta0, rtol=1e-15)
    # the differentiable residual restates the device's converged system: at the solved state
    # it is at round-off next to its size at a state perturbed by 1e-6 (relative)
    r, gmd, mb = res.residual(x, mdot, th)
    gen = torch.Generator(device="cuda").manual_seed(0)
    xp = x * (1 + 1e-6 * torch.randn(x.shape, generator=gen, device="cuda", dtype=x.dtype))
    mp = [m * (1 + 1e-6 * torch.randn(m.shape, generator=gen, device="cuda", dtype=m.dtype))
          for m in mdot]
    rp_, gp_, _ = res.residual(xp, mp, th)
    for k in range(4):
        assert float(r[:, k].abs().max()) <= 1e-4 * float(rp_[:, k].abs().max()), k
    for g, g2 in zip(gmd, gp_):
        assert float(g.abs().max()) <= 1e-4 * float(g2.abs().max())
    J0 = res.objectives(x, mdot, th).cpu().numpy()
    assert abs(J0[0] + J0[1] - 1.0) < 1e-9              # the flow splits between the outlets
    grad, J, info = res.sensitivities()                  # the four adjoint systems batched
    grad = grad.cpu().numpy()
    assert all(i["residual"] <= 1e-10 for i in info), info
    one, _, info1 = res.sensitivities(batched=False)      # and one after another
    one = one.cpu().numpy()
    assert all(i["residual"] <= 1e-10 for i in info1), info1
    for k in range(grad.shape[0]):
        scale = np.abs(one[k] * theta0).max()
        assert np.abs((grad[k] - one[k]) * theta0).max() <= 1e-6 * scale, (k, grad[k], one[k])
    start = (res.s.U.cpu().numpy(), res.s.P.cpu().numpy())
    res.s.close()
    fd = np.zeros_like(grad)
    for p in range(len(theta0)):
        h = 1e-6 * theta0[p]
        vals = []
        for sgn in (1.0, -1.0):
            t = theta0.copy()
            t[p] += sgn * h
            rp = _solve(t, start)
            xp, mp = rp.state()
            vals.append(rp.objectives(xp, mp, rp.theta0()).cpu().numpy())
            rp.s.close()
        fd[:, p] = (vals[0] - vals[1]) / (2 * h)
    for k in range(grad.shape[0]):
        ref = np.abs(fd[k] * theta0).max()                 # sensitivities per relative change
        err = np.abs((grad[k] - fd[k]) * theta0)
        assert err.max() <= 1e-5 * ref, (k, dict(zip(NAMES, grad[k])), dict(zip(NAMES, fd[k])))
    # steady state: the capacitances do not enter
    assert np.all(grad[:, [2, 5]] == 0.0)
