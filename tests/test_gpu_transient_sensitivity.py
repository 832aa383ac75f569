"""Parameter gradients of a BDF2 march by the discrete adjoint, against finite differences.

The small Y-bifurcation of the steady adjoint test (parent radius 2 mm, daughters 1.6 and 1.4
mm at +-35 degrees), Carreau-Yasuda blood, a pulsatile inlet Q(t) = A (1 + 0.5 sin(2 pi t /
0.8)) with A = 1 ml/s, RCR outlets (Rp 1e8, C 1e-9, Rd 1e9), a fixed advection blend; 50 BDF2
steps of 1 ms from the steady state at Q(0), every step's coefficient loops solved to
round-off. Objectives: the two outlet flow fractions and the mean wall shear stress of each
daughter, averaged over the steps; parameters: A, each outlet's (Rp, C, Rd) and mu0. The
adjoint runs backward through the steps, recomputing each 10-step segment from its checkpoint;
its gradient must match central differences of whole marches (step 1e-6 relative, from the
same initial state) to 1e-5 of each objective's largest sensitivity, capacitances included
(they matter in a transient).
"""

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

NAMES = ["A", "Rp1", "C1", "Rd1", "Rp2", "C2", "Rd2", "mu0"]


def _wave(t):
    return 1.0 + 0.5 * np.sin(2 * np.pi * t / 0.8)


def _mesh():
    from zvcfd_b200.mesh import y_bifurcation

    m = y_bifurcation(0.5e-3, parent=(2e-3, 8e-3),
                      daughters=((1.6e-3, 6e-3, 35.0), (1.4e-3, 6e-3, -35.0)))
    return m, {zz.name: k for k, zz in m.zones.items()}


def _solver(m, z, theta, flow):
    from zvcfd_b200.fluid import CarreauYasuda, Fluid
    from zvcfd_b200.lumped import RCR
    from zvcfd_b200.solver import B200Solver

    _, rp1, c1, rd1, rp2, c2, rd2, mu0 = (float(v) for v in theta)

    def shape(x):
        return np.clip(1.0 - (x[:, 0] ** 2 + x[:, 1] ** 2) / 2e-3 ** 2, 0.0, None)

    bcs = {z["inlet"]: {"kind": "velocity", "flow_rate": flow, "profile": shape},
           z["outlet1"]: {"kind": "pressure", "lumped": RCR(rp=rp1, c=c1, rd=rd1)},
           z["outlet2"]: {"kind": "pressure", "lumped": RCR(rp=rp2, c=c2, rd=rd2)},
           z["wall"]: {"kind": "wall"}}
    fl = Fluid(1060.0, 0.00345, viscosity=CarreauYasuda(mu_0=mu0))
    return B200Solver(m, fl, bcs, advection=1.0, linear_rtol=0.1)


def _walls(m, z):
    f = m.zones[z["wall"]].faces
    nodes = np.unique(f[f >= 0])
    x = m.nodes[nodes]
    beyond = x[:, 2] > 2.5e-3
    return {"daughter1": torch.as_tensor(nodes[beyond & (x[:, 0] > 0)], device="cuda"),
            "daughter2": torch.as_tensor(nodes[beyond & (x[:, 0] < 0)], device="cuda")}


def test_transient_adjoint_matches_central_differences():
    from zvcfd_b200.sensitivity import TransientSensitivity

    theta0 = np.array([1e-6, 1e8, 1e-9, 1e9, 1e8, 1e-9, 1e9, 0.056])
    m, z = _mesh()
    steady = _solver(m, z, theta0, theta0[0] * _wave(0.0))
    rep = steady.solve(max_iterations=1500, tol=1e-12)
    assert rep["converged"]
    start = steady.snapshot()
    steady.close()

    def make(theta):
        A = float(theta[0])
        return _solver(m, z, theta, lambda t: A * _wave(t))

    ts = TransientSensitivity(make, z["inlet"], [z["outlet1"], z["outlet2"]], _walls(m, z),
                              start=start, amplitude=theta0[0], waveform=_wave, dt=1e-3,
                              steps=50, tol=1e-12, checkpoint_every=10)
    grad, J, info = ts.gradient(theta0)
    assert info["converged"], info["iterations"]
    assert all(k["residual"] <= 1e-10 for k in info["adjoint"]), info["adjoint"]
    fd = np.zeros_like(grad)
    for p in range(len(theta0)):
        h = 1e-6 * theta0[p]
        vals = []
        for sgn in (1.0, -1.0):
            t = theta0.copy()
            t[p] += sgn * h
            Jp, rp = ts.march(t)
            assert rp["converged"], (p, sgn)
            vals.append(Jp)
        fd[:, p] = (vals[0] - vals[1]) / (2 * h)
    ts.close()
    for k in range(grad.shape[0]):
        ref = np.abs(fd[k] * theta0).max()
        err = np.abs((grad[k] - fd[k]) * theta0)
        assert err.max() <= 1e-5 * ref, (k, dict(zip(NAMES, grad[k])), dict(zip(NAMES, fd[k])))
    # in a transient the capacitances shape the flows
    assert np.all(np.abs(grad[:2, [2, 5]]) > 0.0)
