"""Derivatives of steady outputs (outlet flow fractions, mean wall shear) with respect to
boundary and fluid parameters (inlet flow, lumped-outlet Rp/C/Rd, the Carreau-Yasuda mu_0).

The converged steady state is the fixed point ``z = Phi(z; theta)`` of the outer iteration of
:class:`~zvcfd_b200.solver.B200Solver`: ``z`` holds everything one iteration reads from the
previous one (velocity, pressure, the Rhie-Chow mass flows of every flux point, the
advective diagonal and the boundary mass flows they imply) and ``Phi`` is one iteration with
its linear solve converged tightly, so that ``Phi`` is a smooth map of ``z`` and ``theta``
(the limiter is frozen by then). Differentiating the fixed point gives the tangent system

    (I - dPhi/dz) dz/dtheta_k = dPhi/dtheta_k,

solved here by GMRES in block-scaled variables with matrix-free products: ``dPhi/dz v`` is a
central difference of two device iterations, so every product is the exact linearisation of
the discrete scheme up to O(eps^2) - including the lagged Rhie-Chow coupling, the
Carreau-Yasuda viscosity and the implicit lumped-outlet rows, which a frozen-coefficient
(Picard) adjoint would miss. The output derivative is then
``dJ/dtheta_k = dJ/dz dz/dtheta_k + dJ/dtheta_k`` with both terms again central differences of
cheap evaluations. One GMRES solve per parameter: the forward (tangent) counterpart of an
adjoint, chosen because the transpose of the device outer iteration is not formed; the
adjoint of the linear solve itself is :mod:`zvcfd_b200.adjoint`.

The reference has no sensitivities; the derivatives are checked against central finite
differences of full nonlinear solves.
"""

from __future__ import annotations

from dataclasses import dataclass, replace
from typing import Callable

import numpy as np
import torch

from zvcfd_b200.wall import WallShear


@dataclass
class Parameter:
    """A scalar input of the steady problem: ``get(solver)`` and ``set(solver, value)``."""

    name: str
    get: Callable
    set: Callable


def inlet_flow(zid: int) -> Parameter:
    """The volume flow rate (m^3/s) of a flow-rate inlet zone."""

    def get(s):
        return float(s.bcs[zid]["flow_rate"])

    def set_(s, v):
        s.bcs[zid]["flow_rate"] = float(v)
        s.bc.update(s.t)
        s._upload_boundary()
        s._apply_fixed()

    return Parameter(f"inlet_flow[{zid}]", get, set_)


def lumped(zid: int, attr: str) -> Parameter:
    """An attribute (``"rp"``, ``"c"``, ``"rd"``) of a zone's lumped outlet model."""

    def get(s):
        return float(getattr(s.bcs[zid]["lumped"], attr))

    def set_(s, v):
        model = s.bcs[zid]["lumped"]
        setattr(model, attr, float(v))
        model.__post_init__()

    return Parameter(f"{attr}[{zid}]", get, set_)


def viscosity_mu0() -> Parameter:
    """The zero-shear viscosity of the Carreau-Yasuda fluid."""

    def get(s):
        return float(s.fluid.viscosity.mu_0)

    def set_(s, v):
        s.fluid.viscosity = replace(s.fluid.viscosity, mu_0=float(v))
        r = s.asm.rheo
        s.asm.rheo = (r[0], float(v)) + tuple(r[2:])

    return Parameter("mu_0", get, set_)


class FlowFractions:
    """Outputs: each zone's share of the total outflow through ``zids``."""

    def __init__(self, zids):
        self.zids = list(zids)
        self.names = [f"flow_fraction[{z}]" for z in self.zids]

    def __call__(self, s) -> torch.Tensor:
        q = s.patch_flows()
        tot = sum(q[z] for z in self.zids)
        return torch.tensor([q[z] / tot for z in self.zids], dtype=torch.float64)


class ZonePressures:
    """Outputs: the area-mean pressure of each zone in ``zids``."""

    def __init__(self, zids):
        self.zids = list(zids)
        self.names = [f"pressure[{z}]" for z in self.zids]

    def __call__(self, s) -> torch.Tensor:
        p = s.patch_pressures()
        return torch.tensor([p[z] for z in self.zids], dtype=torch.float64)


class MeanWallShear:
    """Outputs: the area-weighted mean wall shear stress magnitude over each node group."""

    def __init__(self, mesh, wall_zones, groups: dict):
        self.op = WallShear(mesh, wall_zones)
        self.groups = {k: torch.as_tensor(np.asarray(v), dtype=torch.int64, device="cuda")
                       for k, v in groups.items()}
        self.names = [f"mean_wss[{k}]" for k in self.groups]

    def __call__(self, s) -> torch.Tensor:
        tau = self.op(s.U, viscosity=s.fluid.viscosity, mu=s.fluid.mu)
        return torch.stack([self.op.mean(tau, g) for g in self.groups.values()]).cpu()


class Outputs:
    """Several output groups evaluated together."""

    def __init__(self, *groups):
        self.groups = groups
        self.names = [n for g in groups for n in g.names]

    def __call__(self, s) -> torch.Tensor:
        return torch.cat([g(s) for g in self.groups])


class SteadySensitivity:
    """Tangent sensitivities of ``outputs`` to ``parameters`` at a converged steady state of
    ``solver`` (see the module docstring).

    Args:
        solver: a converged :class:`B200Solver` (its limiter frozen).
        parameters: :class:`Parameter` list.
        outputs: callable ``solver -> (n_out,) tensor``.
        linear_rtol: tolerance of the linear solve inside each evaluation of ``Phi``.
        eps: central-difference step in block-scaled state units. The error of a difference
            quotient is about the linear solves' absolute accuracy (FGMRES stops at 1e-13 of
            the right-hand side) times the condition of the system over ``eps``, plus
            ``eps^2``: 1e-3 balances the two.
        rel_step: central-difference step of each parameter, relative to its value.
    """

    def __init__(self, solver, parameters, outputs, *, linear_rtol: float = 1e-10,
                 eps: float = 1e-3, rel_step: float = 1e-4, gmres_tol: float = 1e-8,
                 restart: int = 40, maxiter: int = 200, linear_maxiter: int = 1000):
        self.s, self.params, self.outputs = solver, list(parameters), outputs
        self.linear_rtol, self.eps, self.rel_step = linear_rtol, eps, rel_step
        self.linear_maxiter = linear_maxiter
        self.gmres_tol, self.restart, self.maxiter = gmres_tol, restart, maxiter
        self.kinds = list(solver.mdot)
        self.z0 = self.state()
        self.scale = self._block_scale(self.z0)

    # ------------------------------------------------------------ the state vector
    def _blocks(self):
        s = self.s
        return [s.U.reshape(-1), s.P.reshape(-1)] + [s.mdot[k].reshape(-1) for k in self.kinds] + \
            [s._adv.reshape(-1), s._mb.reshape(-1)]

    def state(self) -> torch.Tensor:
        return torch.cat([b.clone() for b in self._blocks()])

    def set_state(self, z: torch.Tensor) -> None:
        s = self.s
        sizes = [b.numel() for b in self._blocks()]
        parts = torch.split(z, sizes)
        s.U = parts[0].reshape(-1, 3).clone()
        s.P = parts[1].clone()
        for k, p in zip(self.kinds, parts[2:2 + len(self.kinds)]):
            s.mdot[k] = p.reshape(s.mdot[k].shape).clone()
        s._adv = parts[-2].clone()
        s._mb = parts[-1].clone()

    def _block_scale(self, z):
        sizes = [b.numel() for b in self._blocks()]
        out = []
        for p in torch.split(z, sizes):
            m = float(p.abs().max()) if p.numel() else 1.0
            out.append(torch.full_like(p, m if m > 0 else 1.0))
        return torch.cat(out)

    # ------------------------------------------------------------ the fixed-point map
    def phi(self, z: torch.Tensor) -> torch.Tensor:
        """One outer iteration from ``z`` with a tight linear solve; the next state."""
        s = self.s
        self.set_state(z)
        keep = s.linear_rtol
        keep_its = getattr(s.linear, "maxiter", None)
        s.linear_rtol = self.linear_rtol
        if keep_its is not None:
            s.linear.maxiter = self.linear_maxiter
        try:
            rec = s.iterate()
        finally:
            s.linear_rtol = keep
            if keep_its is not None:
                s.linear.maxiter = keep_its
        # near the fixed point the initial residual is already small, and FGMRES stops at its
        # round-off floor (1e-13 of the right-hand side) before a relative 1e-10; a solve that
        # did not get within 1e-6 would put its error into every difference quotient
        if rec["linear_residual"] > 1e-6:
            raise RuntimeError(f"tight linear solve not converged ({rec['linear_residual']:.1e} "
                               f"after {rec['linear_iterations']} iterations)")
        return self.state()

    def _with_param(self, p: Parameter, value: float, fn):
        old = p.get(self.s)
        self.set_state(self.z0)           # some setters read the state (boundary uploads)
        p.set(self.s, value)
        try:
            return fn()
        finally:
            self.set_state(self.z0)
            p.set(self.s, old)

    def fixed_point_residual(self) -> float:
        """Scaled ``max |Phi(z) - z|`` at the stored state (how converged the state is)."""
        return float(((self.phi(self.z0) - self.z0) / self.scale).abs().max())

    # ------------------------------------------------------------ tangent solves
    def _jv(self, v):
        """(I - dPhi/dz) v in scaled variables, central differences."""
        d = self.eps * v * self.scale
        return v - (self.phi(self.z0 + d) - self.phi(self.z0 - d)) / (2 * self.eps * self.scale)

    def _gmres(self, b):
        n = b.numel()
        x = torch.zeros_like(b)
        bnorm = float(torch.linalg.norm(b)) or 1.0
        r = b.clone()
        its = 0
        while its < self.maxiter:
            beta = float(torch.linalg.norm(r))
            if beta <= self.gmres_tol * bnorm:
                break
            m = self.restart
            V = torch.zeros((m + 1, n), dtype=b.dtype, device=b.device)
            H = np.zeros((m + 1, m))
            V[0] = r / beta
            k_used = 0
            for k in range(m):
                w = self._jv(V[k])
                for j in range(k + 1):              # modified Gram-Schmidt, twice
                    h = float(torch.dot(V[j], w))
                    H[j, k] += h
                    w = w - h * V[j]
                for j in range(k + 1):
                    h = float(torch.dot(V[j], w))
                    H[j, k] += h
                    w = w - h * V[j]
                H[k + 1, k] = float(torch.linalg.norm(w))
                its += 1
                k_used = k + 1
                e1 = np.zeros(k + 2)
                e1[0] = beta
                y, *_ = np.linalg.lstsq(H[:k + 2, :k + 1], e1, rcond=None)
                res = np.linalg.norm(H[:k + 2, :k + 1] @ y - e1)
                if H[k + 1, k] > 0:
                    V[k + 1] = w / H[k + 1, k]
                if res <= self.gmres_tol * bnorm or H[k + 1, k] == 0 or its >= self.maxiter:
                    break
            x = x + torch.as_tensor(y, dtype=b.dtype, device=b.device) @ V[:k_used]
            r = b - self._jv(x)
        return x, its

    def jacobian(self) -> dict:
        """``{"dJ": (n_out, n_par) array, "outputs": J, "gmres_iterations": [...]}``."""
        s, z0, sc = self.s, self.z0, self.scale
        self.set_state(z0)
        J0 = self.outputs(s).numpy()
        cols, its = [], []
        for p in self.params:
            v0 = p.get(s)
            h = self.rel_step * abs(v0) if v0 != 0 else self.rel_step
            zp = self._with_param(p, v0 + h, lambda: self.phi(z0))
            zm = self._with_param(p, v0 - h, lambda: self.phi(z0))
            rhs = (zp - zm) / (2 * h) / sc                  # dPhi/dtheta, scaled
            dz, k = self._gmres(rhs)
            its.append(k)
            d = self.eps * dz * sc
            self.set_state(z0 + d)
            Jp = self.outputs(s).numpy()
            self.set_state(z0 - d)
            Jm = self.outputs(s).numpy()
            dJ_dz = (Jp - Jm) / (2 * self.eps)
            self.set_state(z0)
            Jt_p = self._with_param(p, v0 + h, lambda: self.outputs(s).numpy())
            Jt_m = self._with_param(p, v0 - h, lambda: self.outputs(s).numpy())
            cols.append(dJ_dz + (Jt_p - Jt_m) / (2 * h))
        self.set_state(z0)
        return {"dJ": np.stack(cols, 1), "outputs": J0, "gmres_iterations": its}


class SteadyOutputs(torch.autograd.Function):
    """``outputs(theta)`` at the converged steady state as an autograd function: the forward
    pass sets the parameters and solves to ``tol``; the backward pass applies the tangent
    Jacobian of :class:`SteadySensitivity` to the incoming gradient."""

    @staticmethod
    def forward(ctx, theta, solver, parameters, outputs, tol, max_iterations, options):
        vals = theta.detach().cpu().numpy().astype(float)
        for p, v in zip(parameters, vals):
            p.set(solver, float(v))
        rep = solver.solve(max_iterations=max_iterations, tol=tol)
        if not rep["converged"]:
            raise RuntimeError("steady solve not converged")
        sens = SteadySensitivity(solver, parameters, outputs, **(options or {}))
        jac = sens.jacobian()
        ctx.save_for_backward(torch.as_tensor(jac["dJ"]))
        return torch.as_tensor(jac["outputs"], dtype=theta.dtype)

    @staticmethod
    def backward(ctx, g):
        (dJ,) = ctx.saved_tensors
        return (g.to(dJ.dtype) @ dJ).to(g.dtype), None, None, None, None, None, None


def steady_outputs(theta, solver, parameters, outputs, *, tol=1e-10, max_iterations=400,
                   options=None):
    """Differentiable steady outputs of ``solver`` as functions of ``theta`` (one value per
    :class:`Parameter`)."""
    return SteadyOutputs.apply(theta, solver, parameters, outputs, tol, max_iterations, options)


__all__ = ["Parameter", "inlet_flow", "lumped", "viscosity_mu0", "FlowFractions",
           "ZonePressures", "MeanWallShear", "Outputs", "SteadySensitivity", "SteadyOutputs", "steady_outputs"]
