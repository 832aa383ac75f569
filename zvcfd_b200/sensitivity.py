"""Parameter sensitivities of a converged steady solve by the discrete adjoint.

The steady state of :class:`~zvcfd_b200.solver.B200Solver` is the fixed point of the lagged
Rhie-Chow outer iteration. Its unknowns are ``z = (x, mdot)``: the nodal velocities and
pressures ``x (N, 4)`` and the mass flows at the flux points (slot order, per element type).
At the fixed point the residual

    R(z, theta) = ( A(z, theta) x - b(z, theta) ,  mdot - M(x, z, theta) )

vanishes, where ``A x - b`` is the assembled system with its boundary rows (the element fluxes
of ``zvcfd/fv/reference.py:654-806``, the boundary terms of ``zvcfd/fv/_cuda_bc.py:32-138``, the
lumped RCR rows of ``zvcfd/fv/solver.py:719-767``) and ``M`` the Rhie-Chow mass flow
(``zvcfd/fv/reference.py:922-948``) with the pressure-dissipation coefficient of the momentum
diagonal at ``z``. For an objective ``J(z, theta)``,

    dJ/dtheta = dJ/dtheta|_z - lambda^T dR/dtheta,    (dR/dz)^T lambda = (dJ/dz)^T.

:class:`SteadyResidual` states ``R`` and the objectives (outlet flow fractions, mean wall shear
stress per wall part) as torch functions of ``(z, theta)``, element type by element type, so
that every transposed Jacobian product ``(dR/dz)^T v`` is one reverse pass through them. The
adjoint system is solved by restarted FGMRES whose preconditioner is the transposed V-cycle of
the AMG hierarchy the forward solve built for its last linearisation (``zvfv_solver_vcycle_t``:
``A^T``, ``D^-T`` and transposed Gauss-Seidel sweeps on every level) for the ``x`` block, with
the mass-flow rows' coupling to ``x`` applied exactly (a block-triangular preconditioner). The reference has no adjoint; the forward state, boundary data and
hierarchy are the device solver's own.

Parameters ``theta``: the inlet flow rate, per lumped outlet ``(Rp, C, Rd)`` and the fluid's
``mu0``. In a steady state the capacitance only shapes the transient, so ``dJ/dC = 0``. The
advection blend must be fixed (a number): the Barth-Jespersen limiter is not differentiable.
"""

from __future__ import annotations

import numpy as np
import torch

from zvcfd_b200._lib import call, ptr, stream_ptr
from zvcfd_b200.topology import tables
from zvcfd_b200.wall import WallShear


def _carreau_yasuda(rate, mu0, muinf, lam, a, n):
    return muinf + (mu0 - muinf) * (1.0 + (lam * rate) ** a) ** ((n - 1.0) / a)


def _sqrt0(v):
    """``sqrt(v)`` with a zero derivative where ``v = 0`` (a flux point inside an element whose
    nodes all lie on a no-slip wall has no shear; there the viscosity's slope in the shear rate
    is zero, while sqrt's derivative would be infinite and turn the reverse pass into NaN)."""
    pos = v > 0
    return torch.where(pos, torch.sqrt(torch.where(pos, v, torch.ones_like(v))),
                       torch.zeros_like(v))


def _rate(L):
    """Shear rate ``sqrt(2 D:D)`` of velocity gradients ``L (..., 3, 3)``."""
    D = 0.5 * (L + L.transpose(-1, -2))
    return _sqrt0(2.0 * (D * D).sum((-1, -2)))


def rcr_step(model, pc, q, rp, c, rd, t_new, dt):
    """``(pc0, pc1)`` of an RCR outlet's step as torch functions of its previous capacitor
    pressure ``pc`` and flow ``q`` and its parameters: the capacitor pressure at ``t_new`` is
    ``pc0 + pc1 Q`` (``zvcfd/lumped.py`` RCR; :meth:`zvcfd_b200.lumped.RCR._affine_step`,
    trapezoidal or backward Euler)."""
    tau = rd * c
    pv1 = float(model._venous(t_new))
    if model.method == "euler":
        h = dt
        known = pc + h * pv1 / tau
    else:
        h = 0.5 * dt
        pv0 = float(model._venous(t_new - dt))
        known = pc + h * ((pv0 + pv1 - pc) / tau + q / c)
    damp = 1.0 + h / tau
    return known / damp, (h / c) / damp


class _KindGeometry:
    """One element type's constant geometry in slot order: node ids, flux-point area vectors
    and centroids, shape functions and their gradients at the flux points."""

    def __init__(self, K, X):
        t = tables(K.kind)
        dev = X.device
        self.kind, self.n, self.nip = K.kind, t.n, t.n_ip
        self.conn = K.conn.to(torch.int64)                         # (E, n) slot order
        xe = X[self.conn]                                          # (E, n, 3)
        W = torch.as_tensor(t.weights, dtype=torch.float64, device=dev)
        pts = torch.einsum("pn,enk->epk", W, xe)
        tri = torch.as_tensor(t.tris, device=dev)
        p0, p1, p2 = pts[:, tri[:, 0]], pts[:, tri[:, 1]], pts[:, tri[:, 2]]
        self.A = 0.5 * torch.linalg.cross(p1 - p0, p2 - p0)       # (E, nip, 3)
        self.xs = (p0 + p1 + p2) / 3.0
        dN = torch.as_tensor(t.dN_ip, dtype=torch.float64, device=dev)       # (nip, n, 3)
        J = torch.einsum("enk,ind->eikd", xe, dN)                            # dx_k / dxi_d
        Ji = torch.linalg.inv(J)                                             # dxi_d / dx_k
        self.G = torch.einsum("ind,eidk->eink", dN, Ji)                      # (E, nip, n, 3)
        self.N = torch.as_tensor(t.N_ip, dtype=torch.float64, device=dev)    # (nip, n)
        self.ia = torch.as_tensor(t.edge[:, 0], device=dev)
        self.ib = torch.as_tensor(t.edge[:, 1], device=dev)
        self.node_a = self.conn[:, self.ia]                                  # (E, nip)
        self.node_b = self.conn[:, self.ib]


class SteadyResidual:
    """``R(z, theta)`` and the objectives of a converged :class:`B200Solver` state.

    Args:
        solver: a converged steady solver (fixed advection blend, no time step).
        inlet: the velocity zone whose ``flow_rate`` is the first parameter.
        outlets: the lumped (RCR) pressure zones, in parameter order.
        walls: ``{name: node ids}`` of the wall parts whose mean shear stress is an objective.
    """

    def __init__(self, solver, inlet: int, outlets: list, walls: dict, *, amplitude=None):
        s = solver
        if not isinstance(s.advection, (int, float)):
            raise ValueError("the adjoint needs a fixed advection blend (a number)")
        if s.dt or s._time is not None:
            raise ValueError("the adjoint is of the steady state or of BDF steps, not of a "
                             "false time step")
        if getattr(s, "_special", None) or getattr(s, "boundary_reconstruction", False):
            raise NotImplementedError("the restated residual has no average-pressure or opening "
                                      "zones and no boundary reconstruction")
        self.s = s
        self.rho = float(s.fluid.rho)
        self.visc = s.fluid.viscosity
        self.transpose = bool(s.transpose)
        self.beta = float(s.advection)
        self.N = s.N
        X = s.asm.X.reshape(-1, 3)
        self.X = X
        self.V = s.asm.node_volume
        self.geo = [_KindGeometry(K, X) for K in s.asm.kinds]
        indptr, indices = s.pattern
        self.rows = torch.repeat_interleave(torch.arange(self.N, device=X.device),
                                            indptr[1:] - indptr[:-1])
        self.cols = indices.to(torch.int64)
        self.gop = s.asm.gop.view(-1, 3)
        # boundary data of the device's boundary pass
        self.fixed = s._fixed_d.clone()                       # (N, 3) bool
        self.pfix = s._pfix_d.clone()
        self.outlet = s._outlet_d.clone()
        self.wsum = (s._wcons_d, s._wonly_d, s._wstab_d)
        self.snl, self.force, self.fV = s._snl, s._force_d, s._fV_d
        self.aout = s._aout_d if s._has_aout else None
        # theta-dependent boundary data at the reference parameters
        spec = s.bcs[inlet]
        self.q0 = float(spec["flow_rate"] if amplitude is None else amplitude)
        self.vel0, self.inflow0, self.pval = s._vel_d.clone(), s._inflow_d.clone(), s._pval_d
        self.outlets = list(outlets)
        self.lumped = [s._lumped[z] for z in self.outlets]
        self.zone_nodes = {z: s._lumped[z]["nodes"] for z in self.outlets}
        self.walls = walls
        wall_ids = [z for z in s.mesh.zones if s.bcs.get(z, {}).get("kind") == "wall"]
        self.wall = WallShear(s.mesh, wall_ids)

    # ------------------------------------------------------------ parameters

    def theta0(self) -> torch.Tensor:
        """The parameters of the solved state: ``(Q_in, Rp_1, C_1, Rd_1, ..., mu0)``."""
        vals = [self.q0]
        for z in self.lumped:
            m = z["model"]
            vals += [float(m.rp), float(m.c), float(m.rd)]
        vals.append(float(self.visc.mu_0) if self.visc is not None else float(self.s.fluid.mu))
        return torch.tensor(vals, dtype=torch.float64, device=self.X.device)

    def state(self):
        """``z`` of the solver: ``x (N, 4)`` and the mass flows (slot order, per type)."""
        x = torch.cat([self.s.U, self.s.P[:, None]], 1).detach().clone()
        return x, [self.s.mdot[g.kind].detach().clone() for g in self.geo]

    def _mu(self, rate, mu0):
        if self.visc is None:
            return mu0 + 0.0 * rate
        v = self.visc
        return _carreau_yasuda(rate, mu0, v.mu_inf, v.lam, v.a, v.n)

    # ------------------------------------------------------------ the residual

    def gradient(self, phi):
        """Nodal gradients through the device's gradient operator: ``(N, C, 3)``."""
        out = torch.zeros((self.N, phi.shape[1], 3), dtype=phi.dtype, device=phi.device)
        return out.index_add(0, self.rows, self.gop[:, None, :] * phi[self.cols][:, :, None])

    def residual(self, x, mdot, theta, step=None):
        """``(r (N, 4), [mdot residual per type], mb)``; ``r`` unscaled, one row per unknown.

        ``step``: a BDF time step's data (:meth:`TransientResidual.step_data`): ``c0, c1, c2,
        dt``, the earlier levels ``U1, m1`` (and ``U2, m2``), the boundary values ``vel,
        inflow`` at the step's time for the reference inlet amplitude, and per lumped outlet
        the previous step's capacitor pressure and flow ``pc, q`` (tensors: the adjoint
        differentiates through them). None: the steady residual."""
        rho, N = self.rho, self.N
        U, P = x[:, :3], x[:, 3]
        q, mu0 = theta[0], theta[-1]
        grads = self.gradient(x)
        gU, gP = grads[:, :3], grads[:, 3]                     # (N, 3, 3), (N, 3)
        # momentum diagonal a_P: viscous coefficients and upwind flows of every flux point
        aP = torch.zeros(N, dtype=x.dtype, device=x.device)
        per = []
        for g, m in zip(self.geo, mdot):
            L = torch.einsum("eink,enj->eijk", g.G, U[g.conn])           # (E, nip, 3, 3)
            mu = self._mu(_rate(L), mu0)                                  # (E, nip)
            Ga = g.G[:, torch.arange(g.nip), g.ia]                        # (E, nip, 3)
            Gb = g.G[:, torch.arange(g.nip), g.ib]
            va = (Ga * g.A).sum(-1) + (Ga[..., 0] * g.A[..., 0] if self.transpose else 0.0)
            vb = (Gb * g.A).sum(-1) + (Gb[..., 0] * g.A[..., 0] if self.transpose else 0.0)
            aP = aP.index_add(0, g.node_a.reshape(-1),
                              (-mu * va + torch.clamp(m, min=0.0)).reshape(-1))
            aP = aP.index_add(0, g.node_b.reshape(-1),
                              (mu * vb + torch.clamp(-m, min=0.0)).reshape(-1))
            per.append((L, mu))
        if step is None:
            dnode = snode = self.V / aP
            levels = []
        else:
            # BDF: a_P + c0 rho V / dt in the Rhie-Chow coefficient of the step; the transient
            # Rhie-Chow part carries the earlier levels' mass flows (zvcfd/fv/reference.py:796-801)
            tdiag = step["c0"] * rho * self.V / step["dt"]
            dnode, snode = self.V / (aP + tdiag), self.V / aP
            levels = [(step["c1"] / step["c0"], step["U1"], step["m1"])]
            if step.get("U2") is not None and step["c2"]:
                levels.append((step["c2"] / step["c0"], step["U2"], step["m2"]))
        r = torch.zeros((N, 4), dtype=x.dtype, device=x.device)
        gmd = []
        for t_, (g, m, (L, mu)) in enumerate(zip(self.geo, mdot, per)):
            A = g.A
            Ne = g.N                                                       # (nip, n)
            us = torch.einsum("in,enk->eik", Ne, U[g.conn])                # u at the flux point
            ps = torch.einsum("in,en->ei", Ne, P[g.conn])
            gps = torch.einsum("eink,en->eik", g.G, P[g.conn])             # grad p at s
            gbar = torch.einsum("in,enk->eik", Ne, gP[g.conn])             # mean grad p
            d = 0.5 * (dnode[g.node_a] + dnode[g.node_b])
            visc = torch.einsum("eijk,eik->eij", L, A)                     # (grad u) . A
            if self.transpose:
                visc = visc + torch.einsum("eikj,eik->eij", L, A)          # (grad u)^T . A
            up = torch.where(m >= 0, g.node_a, g.node_b)
            reach = g.xs - self.X[up]
            corr = m[..., None] * self.beta * torch.einsum("eijk,eik->eij", gU[up], reach)
            adv = (torch.clamp(m, min=0.0)[..., None] * U[g.node_a]
                   + torch.clamp(m, max=0.0)[..., None] * U[g.node_b])
            mom = -mu[..., None] * visc + ps[..., None] * A + adv + corr
            flow = rho * (us * A).sum(-1) - rho * d * ((gps - gbar) * A).sum(-1)
            if levels:
                share = 1.0 - d / (0.5 * (snode[g.node_a] + snode[g.node_b]))
                past = 0.0
                for c, Uo, mo in levels:
                    uo = torch.einsum("in,enk->eik", Ne, Uo[g.conn])
                    past = past + c * (mo[t_] - rho * (uo * A).sum(-1))
                flow = flow + share * past
            f = torch.cat([mom, flow[..., None]], -1)                      # (E, nip, 4)
            r = r.index_add(0, g.node_a.reshape(-1), f.reshape(-1, 4))
            r = r.index_add(0, g.node_b.reshape(-1), -f.reshape(-1, 4))
            gmd.append(m - flow)
        # the boundary pass: outflow advection at outlets, pressure forces, body forces,
        # known inflows, the outlet traction of the transpose term
        scale = q / self.q0
        inflow = (self.inflow0 if step is None else step["inflow"]) * scale
        imb = torch.zeros(N, dtype=x.dtype, device=x.device)
        for g, m in zip(self.geo, mdot):
            imb = imb.index_add(0, g.node_a.reshape(-1), m.reshape(-1))
            imb = imb.index_add(0, g.node_b.reshape(-1), -m.reshape(-1))
        mb = torch.where(self.outlet, -(imb + inflow), torch.zeros_like(imb))
        wc, wo, wst = self.wsum
        dd = wc * mb + wo * torch.clamp(mb, min=0.0) + wst * torch.clamp(-mb, min=0.0)
        mom = r[:, :3] + dd[:, None] * U + self.snl * P[:, None] - self.fV + self.force
        if self.aout is not None:
            mun = self._mu(_rate(gU), mu0) if self.visc is not None else mu0 + 0.0 * P
            mom = mom - mun[:, None] * torch.einsum("njk,nj->nk", gU, self.aout)
        if step is not None:                 # c0 rho V/dt U - rho V/dt (c1 U1 + c2 U2)
            mass = rho * self.V / step["dt"]
            past_u = step["c1"] * step["U1"]
            if step.get("U2") is not None and step["c2"]:
                past_u = past_u + step["c2"] * step["U2"]
            mom = mom + mass[:, None] * (step["c0"] * U - past_u)
        cont = r[:, 3] + inflow
        raw_cont = cont
        # Dirichlet rows
        vel = (self.vel0 if step is None else step["vel"]) * scale
        mom = torch.where(self.fixed, U - vel, mom)
        cont = torch.where(self.pfix, P - self.pval, cont)
        # lumped rows: p_j - (Rp + Rd) Q = a, Q the zone's outflow by its raw continuity rows
        for k, (z, zd) in enumerate(zip(self.outlets, self.lumped)):
            rp, c, rd = theta[1 + 3 * k], theta[2 + 3 * k], theta[3 + 3 * k]
            nodes = zd["nodes"]
            Q = -raw_cont[nodes].sum() / self.rho
            if step is None:
                a, _ = zd["model"].steady_coefficients(self.s.t)
                cont = cont.index_copy(0, nodes, P[nodes] - (rp + rd) * Q - a)
            else:
                pc0, pc1 = rcr_step(zd["model"], step["pc"][k], step["q"][k], rp, c, rd,
                                    step["t"], step["dt"])
                cont = cont.index_copy(0, nodes, P[nodes] - (pc1 + rp) * Q - pc0)
        return torch.cat([mom, cont[:, None]], 1), gmd, mb

    # ------------------------------------------------------------ objectives

    def objectives(self, x, mdot, theta, mb=None):
        """``(Q_1/Q_in, ..., mean |tau| of each wall part)``."""
        if mb is None:
            _, _, mb = self.residual(x, mdot, theta)
        out = []
        for z in self.outlets:                      # the device's zone flows: W mb + c
            k = self.s._flow_zones.index(z)
            q_z = (self.s._flow_W[k] @ mb + self.s._flow_c[k]) / self.rho
            out.append(q_z / theta[0])
        tau = self.wall_shear(x[:, :3], theta[-1])
        mag = _sqrt0((tau * tau).sum(1))
        for name, nodes in self.walls.items():
            a = self.wall.node_area[nodes]
            out.append((mag[nodes] * a).sum() / a.sum())
        return torch.stack(out)

    def wall_shear(self, U, mu0):
        """``(N, 3)`` wall shear stress (the device evaluator's operator, in torch)."""
        w = self.wall
        elem = w.elem.to(torch.int64)
        on = elem >= 0
        Uq = U[torch.where(on, elem, torch.zeros_like(elem))] * on[..., None]
        L = torch.einsum("qaj,qak->qjk", Uq, w.G)
        D = L + L.transpose(1, 2)
        rate = _sqrt0(0.5 * (D * D).sum((1, 2)))
        mu = self._mu(rate, mu0)
        t = mu[:, None] * torch.einsum("qjk,qk->qj", D, w.nrm)
        tn = (t * w.nrm).sum(1, keepdim=True)
        tq = -(t - tn * w.nrm) * w.area[:, None]
        node = torch.repeat_interleave(torch.arange(self.N, device=U.device),
                                       w.node_ptr[1:] - w.node_ptr[:-1])
        acc = torch.zeros((self.N, 3), dtype=U.dtype, device=U.device).index_add(0, node, tq)
        asum = torch.zeros(self.N, dtype=U.dtype, device=U.device).index_add(0, node, w.area)
        return acc / torch.clamp(asum, min=1e-300)[:, None]

    # ------------------------------------------------------------ the adjoint

    def _precondition(self, vx):
        """``S A^-T`` on the velocity-pressure block: the transposed V-cycle of the forward
        solve's hierarchy (its matrix carries the row scales S of the boundary pass)."""
        lin = self.s.linear
        out = torch.empty_like(vx)
        call("zvfv_solver_vcycle_t", lin._h, ptr(vx), ptr(out), stream_ptr())
        return out * self.s.rs

    def adjoint(self, gx, gm, x, mdot, theta, *, rtol=1e-11, restart=200, maxiter=1000):
        """``lambda`` with ``(dR/dz)^T lambda = (gx, gm)`` by right-preconditioned FGMRES."""
        xz = x.detach().requires_grad_(True)
        mz = [m.detach().requires_grad_(True) for m in mdot]
        r, gmd, _ = self.residual(xz, mz, theta.detach())
        outs = [r] + gmd
        sizes = [r.numel()] + [m.numel() for m in mz]

        def split(v):
            parts, o = [], 0
            for n_ in sizes:
                parts.append(v[o:o + n_])
                o += n_
            return parts

        def JT(v):
            parts = split(v)
            gs = torch.autograd.grad(outs, [xz] + mz,
                                     [parts[0].view_as(r)] + [p.view_as(g) for p, g in
                                                              zip(parts[1:], gmd)],
                                     retain_graph=True)
            return torch.cat([t.reshape(-1) for t in gs])

        def M(v):
            # block upper triangle of (dR/dz)^T: the mass-flow rows' coupling to x, (dG/dx)^T,
            # exactly (one reverse pass), the x block by the transposed V-cycle
            parts = split(v)
            if any(float(p.abs().max()) > 0 for p in parts[1:]):
                (gx,) = torch.autograd.grad(gmd, [xz], [p.view_as(g) for p, g in
                                                         zip(parts[1:], gmd)], retain_graph=True)
                rhs = parts[0] - gx.reshape(-1)
            else:
                rhs = parts[0]
            px = self._precondition(rhs.contiguous())
            return torch.cat([px] + parts[1:])

        b = torch.cat([gx.reshape(-1)] + [t.reshape(-1) for t in gm])
        lam, its, res = fgmres(JT, b, M, rtol=rtol, restart=restart, maxiter=maxiter)
        return split(lam), its, res

    def adjoint_batched(self, gx, gm, x, mdot, theta, *, rtol=1e-11, restart=60, maxiter=1000,
                        step=None):
        """The adjoint systems of B objectives at once: ``gx (B, N, 4)``, ``gm`` per type
        ``(B, ...)``. Every transposed Jacobian product is one batched reverse pass through the
        residual (``is_grads_batched``: the saved element tensors are read once for all B
        right-hand sides), and the B Krylov recurrences advance in lock-step
        (:func:`fgmres_batched`). Returns ``(lambda parts (B, ...), iterations, residuals)``."""
        B = gx.shape[0]
        xz = x.detach().requires_grad_(True)
        mz = [m.detach().requires_grad_(True) for m in mdot]
        r, gmd, _ = self.residual(xz, mz, theta.detach(), step)
        outs = [r] + gmd
        sizes = [r.numel()] + [m.numel() for m in mz]

        def split(v):
            parts, o = [], 0
            for n_ in sizes:
                parts.append(v[:, o:o + n_])
                o += n_
            return parts

        def JT(v):
            parts = split(v)
            gs = torch.autograd.grad(outs, [xz] + mz,
                                     [p.reshape(B, *o.shape) for p, o in zip(parts, outs)],
                                     retain_graph=True, is_grads_batched=True)
            return torch.cat([t.reshape(B, -1) for t in gs], 1)

        def M(v):
            parts = split(v)
            rhs = parts[0]
            if any(bool(p.any()) for p in parts[1:]):
                (gxm,) = torch.autograd.grad(gmd, [xz], [p.reshape(B, *g.shape) for p, g in
                                                          zip(parts[1:], gmd)],
                                             retain_graph=True, is_grads_batched=True)
                rhs = rhs - gxm.reshape(B, -1)
            px = torch.stack([self._precondition(rhs[i].contiguous()) for i in range(B)])
            return torch.cat([px] + parts[1:], 1)

        b = torch.cat([gx.reshape(B, -1)] + [t.reshape(B, -1) for t in gm], 1)
        lam, its, res = fgmres_batched(JT, b, M, rtol=rtol, restart=restart, maxiter=maxiter)
        return split(lam), its, res

    def sensitivities(self, rtol=1e-11, restart=200, maxiter=1000, *, batched=True):
        """``dJ/dtheta`` ``(n_objectives, n_parameters)``: the adjoint systems of all objectives
        solved together (``batched``, :meth:`adjoint_batched`), or one after another; they
        share the forward hierarchy and the residual graph."""
        x, mdot = self.state()
        theta = self.theta0()
        xz = x.detach().requires_grad_(True)
        mz = [m.detach().requires_grad_(True) for m in mdot]
        th = theta.detach().requires_grad_(True)
        J = self.objectives(xz, mz, th)
        if batched:
            return self._sensitivities_batched(J, xz, mz, th, x, mdot, theta, rtol, restart,
                                               maxiter)
        rows, info = [], []
        for k in range(J.numel()):
            gz = torch.autograd.grad(J[k], [xz, th] + mz, retain_graph=True, allow_unused=True)
            gx, gth, gm = gz[0], gz[1], gz[2:]
            gx = torch.zeros_like(xz) if gx is None else gx
            gth = torch.zeros_like(th) if gth is None else gth
            gm = [torch.zeros_like(m) if g is None else g for g, m in zip(gm, mz)]
            lam, its, res = self.adjoint(gx, gm, x, mdot, theta, rtol=rtol, restart=restart,
                                         maxiter=maxiter)
            th2 = theta.detach().requires_grad_(True)
            r, gmd, _ = self.residual(x, mdot, th2)
            outs = [r] + gmd
            dR = torch.autograd.grad(outs, th2, [lam[0].view_as(r)] +
                                     [p.view_as(g) for p, g in zip(lam[1:], gmd)],
                                     allow_unused=True)[0]
            dR = torch.zeros_like(th2) if dR is None else dR
            rows.append(gth - dR)
            info.append({"iterations": its, "residual": res})
        return torch.stack(rows).detach(), J.detach(), info

    def _sensitivities_batched(self, J, xz, mz, th, x, mdot, theta, rtol, restart, maxiter):
        nJ = J.numel()
        eye = torch.eye(nJ, dtype=J.dtype, device=J.device)
        gz = torch.autograd.grad(J, [xz, th] + mz, eye, allow_unused=True,
                                 is_grads_batched=True)
        gx = torch.zeros((nJ,) + xz.shape, dtype=xz.dtype, device=xz.device) \
            if gz[0] is None else gz[0]
        gth = torch.zeros((nJ,) + th.shape, dtype=th.dtype, device=th.device) \
            if gz[1] is None else gz[1]
        gm = [torch.zeros((nJ,) + m.shape, dtype=m.dtype, device=m.device) if g is None else g
              for g, m in zip(gz[2:], mz)]
        lam, its, res = self.adjoint_batched(gx, gm, x, mdot, theta, rtol=rtol,
                                             restart=restart, maxiter=maxiter)
        th2 = theta.detach().requires_grad_(True)
        r, gmd, _ = self.residual(x, mdot, th2)
        dR = torch.autograd.grad([r] + gmd, th2, [lam[0].reshape(nJ, *r.shape)] +
                                 [p.reshape(nJ, *g.shape) for p, g in zip(lam[1:], gmd)],
                                 allow_unused=True, is_grads_batched=True)[0]
        dR = torch.zeros_like(gth) if dR is None else dR
        info = [{"iterations": its, "residual": float(v)} for v in res]
        return (gth - dR).detach(), J.detach(), info


class TransientSensitivity:
    """Gradients of time-averaged objectives over a BDF march, by the discrete adjoint of the
    time steps with checkpointed recomputation.

    Step ``n`` solves ``R_n(z_n; z_{n-1}, z_{n-2}, s_{n-1}, theta) = 0`` (the step's converged
    coefficient loops: :meth:`SteadyResidual.residual` with the step's BDF data), then commits
    each lumped outlet's state ``s_n = (pc_n, q_n)``: its flow ``q_n`` and capacitor pressure
    ``pc_n = pc0(pc_{n-1}, q_{n-1}, theta) + pc1(theta) q_n`` (:func:`rcr_step`). The
    objectives are the per-step outlet flow fractions ``q_z / Q_in(t_n)`` and mean wall shear
    stress of each wall part, averaged over the ``steps`` steps. Backward, from the last step:

        (dR_n/dz_n)^T lambda_n = dj_n/dz_n + (ds_n/dz_n)^T sbar_n
                                 - (dR_{n+1}/dz_n)^T lambda_{n+1} - (dR_{n+2}/dz_n)^T lambda_{n+2}
        sbar_{n-1} = -(dR_n/ds_{n-1})^T lambda_n + (ds_n/ds_{n-1})^T sbar_n
        dJ/dtheta = sum_n dj_n/dtheta - lambda_n^T dR_n/dtheta + sbar_n^T ds_n/dtheta,

    all objectives at once (:meth:`SteadyResidual.adjoint_batched`, each step's own hierarchy
    transposed as the preconditioner). The forward march stores its state every
    ``checkpoint_every`` steps (with the level before it, for BDF2); the backward pass
    recomputes each segment's steps from its checkpoint. The initial state ``start`` (a
    :meth:`B200Solver.snapshot`) is the same for every ``theta``.

    Args:
        make_solver: ``theta -> B200Solver`` for those parameters (fixed advection blend), its
            inlet flow ``theta[0] * waveform(t)``.
        inlet, outlets, walls: as :class:`SteadyResidual`.
        start: the initial state; amplitude: the reference ``theta[0]``.
        waveform: ``f(t)``; dt, steps, scheme: the march; tol, loops: each step's coefficient
            loops (relative changes below ``tol``).
    """

    def __init__(self, make_solver, inlet, outlets, walls, *, start, amplitude, waveform, dt,
                 steps, scheme="bdf2", tol=1e-12, loops=400, checkpoint_every=10):
        self.make_solver, self.inlet, self.outlets, self.walls = make_solver, inlet, outlets, walls
        self.start, self.amplitude, self.waveform = start, float(amplitude), waveform
        self.dt, self.steps, self.scheme = float(dt), int(steps), scheme
        self.tol, self.loops, self.every = tol, loops, max(1, int(checkpoint_every))
        self.solver = None
        self.res = None

    # ------------------------------------------------------------ forward

    def _begin(self, theta):
        if self.solver is not None:
            self.solver.close()
        self.solver = s = self.make_solver(np.asarray(theta, float))
        s.restore(self.start)
        self.res = SteadyResidual(s, self.inlet, self.outlets, self.walls,
                                  amplitude=float(theta[0]))
        return s

    def _step(self, s, old, dt_prev, record):
        """One committed BDF step from the solver's state; returns the step's data."""
        from zvcfd_b200.solver import bdf_coefficients

        h = self.dt
        pre = {z: (d["model"].pc, d["model"].q) for z, d in s._lumped.items()}
        c0, c1, c2 = bdf_coefficients(self.scheme, h, dt_prev, len(old))
        s.t += h
        s._time = (self.scheme, h, old, dt_prev)
        s.bc.update(s.t)
        s._refresh_boundary()
        s._apply_fixed()
        its, ok = s._iterate(self.loops, self.tol, None, [])
        rec = {"t": s.t, "dt": h, "c0": c0, "c1": c1, "c2": c2, "iterations": its,
               "converged": ok, "f": float(self.waveform(s.t)),
               "pc": [float(pre[z][0]) for z in self.outlets],
               "q": [float(pre[z][1]) for z in self.outlets]}
        if record:
            rec.update({"snap": s.snapshot(), "old": [(U.clone(), {k: v.clone() for k, v in m.items()})
                                                      for U, m in old],
                        "dt_prev": dt_prev, "vel": s._vel_d.clone(), "inflow": s._inflow_d.clone()})
        q = s.patch_flows()
        for z, d in s._lumped.items():
            d["model"].advance(q[z], s.t, h)
        s._time = None
        return rec

    def _objectives(self, x, mdot, theta, mb, f):
        r = self.res
        out = []
        for z in r.outlets:
            k = r.s._flow_zones.index(z)
            q_z = (r.s._flow_W[k] @ mb + r.s._flow_c[k]) / r.rho
            out.append(q_z / (theta[0] * f))
        tau = r.wall_shear(x[:, :3], theta[-1])
        mag = _sqrt0((tau * tau).sum(1))
        for nodes in r.walls.values():
            a = r.wall.node_area[nodes]
            out.append((mag[nodes] * a).sum() / a.sum())
        return torch.stack(out)

    def march(self, theta, checkpoints=False):
        """The march at ``theta``: ``(time-averaged objectives, report)``; with
        ``checkpoints`` the report holds the stored states."""
        s = self._begin(theta)
        th = torch.as_tensor(np.asarray(theta, float), device="cuda")
        old = [(s.U.clone(), {k: v.clone() for k, v in s.mdot.items()})]
        dt_prev = None
        total, ok, its, ck = 0.0, True, [], []
        for n in range(1, self.steps + 1):
            if checkpoints and (n - 1) % self.every == 0:
                ck.append({"n": n - 1, "snap": s.snapshot(), "old": [
                    (U.clone(), {k: v.clone() for k, v in m.items()}) for U, m in old],
                    "dt_prev": dt_prev})
            rec = self._step(s, old, dt_prev, False)
            x = torch.cat([s.U, s.P[:, None]], 1)
            mdot = [s.mdot[g.kind] for g in self.res.geo]
            total = total + self._objectives(x, mdot, th, s._mb, rec["f"])
            ok &= rec["converged"]
            its.append(rec["iterations"])
            old = [(s.U.clone(), {k: v.clone() for k, v in s.mdot.items()})] + old[:1]
            dt_prev = self.dt
        J = (total / self.steps).cpu().numpy()
        return J, {"converged": ok, "iterations": its, "checkpoints": ck}

    # ------------------------------------------------------------ backward

    def _recompute(self, ck, upto):
        """The steps ``ck["n"] + 1 .. upto`` from a checkpoint, with their data."""
        s = self.solver
        s.restore(ck["snap"])
        old = [(U.clone(), {k: v.clone() for k, v in m.items()}) for U, m in ck["old"]]
        dt_prev = ck["dt_prev"]
        recs = {}
        for n in range(ck["n"] + 1, upto + 1):
            rec = self._step(s, old, dt_prev, True)
            rec["x"] = torch.cat([s.U, s.P[:, None]], 1).clone()
            rec["mdot"] = [s.mdot[g.kind].clone() for g in self.res.geo]
            recs[n] = rec
            old = [(s.U.clone(), {k: v.clone() for k, v in s.mdot.items()})] + old[:1]
            dt_prev = self.dt
        return recs

    def _precondition_at(self, rec):
        """Set the solver's hierarchy and row scales to step ``rec``'s final linearisation."""
        s = self.solver
        s.restore(rec["snap"])
        for k, z in enumerate(self.outlets):
            m = s._lumped[z]["model"]
            m.pc, m.q = rec["pc"][k], rec["q"][k]
        s.t = rec["t"]
        s._time = (self.scheme, rec["dt"], rec["old"], rec["dt_prev"])
        s.bc.update(s.t)
        s._refresh_boundary()
        A, _, _, _ = s._assemble_fused()
        s.linear.setup(A)
        s._time = None

    def gradient(self, theta, *, rtol=1e-11, restart=60, maxiter=2000):
        """``(dJ/dtheta (objectives, parameters), J, report)`` at ``theta``."""
        J, rep = self.march(theta, checkpoints=True)
        r = self.res
        dev = r.X.device
        th0 = torch.as_tensor(np.asarray(theta, float), device=dev)
        nJ, K, Nst = 2 + len(self.walls), len(self.outlets), self.steps
        zero_x = torch.zeros((nJ, r.N, 4), dtype=torch.float64, device=dev)
        zero_m = [torch.zeros((nJ,) + m.shape, dtype=torch.float64, device=dev)
                  for m in (self.solver.mdot[g.kind] for g in r.geo)]
        xbar = {}                 # step -> (gx, [gm]) from the later steps' residuals
        sbar = torch.zeros((nJ, K, 2), dtype=torch.float64, device=dev)
        grad = torch.zeros((nJ, th0.numel()), dtype=torch.float64, device=dev)
        eye = torch.eye(nJ, dtype=torch.float64, device=dev) / Nst
        krylov = []
        cks = rep["checkpoints"]
        for ci in range(len(cks) - 1, -1, -1):
            ck = cks[ci]
            upto = cks[ci + 1]["n"] if ci + 1 < len(cks) else Nst
            recs = self._recompute(ck, upto)
            for n in range(upto, ck["n"], -1):
                rec = recs[n]
                prev = [(recs[n - 1]["x"], recs[n - 1]["mdot"]) if n - 1 in recs else
                        self._level_of(ck, n - 1)]
                if n >= 2 and rec["c2"]:
                    prev.append((recs[n - 2]["x"], recs[n - 2]["mdot"]) if n - 2 in recs else
                                self._level_of(ck, n - 2))
                step, leaves = self._step_inputs(rec, prev, dev)
                xz = rec["x"].detach().requires_grad_(True)
                mz = [m.detach().requires_grad_(True) for m in rec["mdot"]]
                th = th0.clone().requires_grad_(True)
                rr, gmd, mb = r.residual(xz, mz, th, step)
                s_n = self._lumped_state(step, mb, th, rec)
                j_n = self._objectives(xz, mz, th, mb, rec["f"])
                gz = torch.autograd.grad([s_n, j_n], [xz] + mz, [sbar, eye], retain_graph=True,
                                         allow_unused=True, is_grads_batched=True)
                gx = zero_x.clone() if gz[0] is None else gz[0].clone()
                gm = [zm.clone() if g is None else g.clone() for g, zm in zip(gz[1:], zero_m)]
                if n in xbar:
                    gx = gx + xbar[n][0]
                    gm = [a + b for a, b in zip(gm, xbar.pop(n)[1])]
                self._precondition_at(rec)
                const = {k: (v.detach() if torch.is_tensor(v) else
                             ([t.detach() for t in v] if isinstance(v, list) and v and
                              torch.is_tensor(v[0]) else v)) for k, v in step.items()}
                lam, its, res = r.adjoint_batched(gx, gm, rec["x"], rec["mdot"], th0, rtol=rtol,
                                                  restart=restart, maxiter=maxiter, step=const)
                krylov.append({"step": n, "iterations": its, "residual": float(np.max(res))})
                cot = [-lam[0].reshape(nJ, *rr.shape)] + \
                      [-p.reshape(nJ, *g.shape) for p, g in zip(lam[1:], gmd)] + [sbar, eye]
                outs = [rr] + gmd + [s_n, j_n]
                wrt = [th] + leaves["pc"] + leaves["q"] + leaves["levels"]
                gs = torch.autograd.grad(outs, wrt, cot, allow_unused=True, is_grads_batched=True)
                grad = grad + (0.0 if gs[0] is None else gs[0])
                pcq = gs[1:1 + 2 * K]
                sbar = torch.stack([torch.stack([torch.zeros(nJ, dtype=torch.float64, device=dev)
                                                 if g is None else g for g in pcq[:K]], 1),
                                    torch.stack([torch.zeros(nJ, dtype=torch.float64, device=dev)
                                                 if g is None else g for g in pcq[K:]], 1)], 2)
                lv = gs[1 + 2 * K:]
                for j, (U_, ms) in enumerate(leaves["level_slots"]):
                    m_at = n - 1 - j
                    dU, dms = lv[U_], [lv[q] for q in ms]
                    if m_at < 1:
                        continue                              # the fixed initial state
                    ax, am = xbar.get(m_at, (zero_x.clone(), [zm.clone() for zm in zero_m]))
                    if dU is not None:
                        ax[:, :, :3] += dU
                    am = [a if d is None else a + d for a, d in zip(am, dms)]
                    xbar[m_at] = (ax, am)
                del rr, gmd, mb, s_n, j_n
        return grad.detach().cpu().numpy(), J, {**rep, "adjoint": krylov}

    def _level_of(self, ck, n):
        """The stored level ``n`` of a checkpoint (its state, or the level before it)."""
        U, m = ck["old"][ck["n"] - n]
        snap = ck["snap"] if n == ck["n"] else None
        P = snap["P"] if snap is not None else torch.zeros_like(U[:, 0])
        return torch.cat([U, P[:, None]], 1), [m[g.kind] for g in self.res.geo]

    def _step_inputs(self, rec, prev, dev):
        """The step's data with the earlier levels and the lumped state as differentiable
        leaves."""
        levels, slots = [], []
        step = {k: rec[k] for k in ("c0", "c1", "c2", "dt", "t", "vel", "inflow")}
        for j, (x, m) in enumerate(prev):
            U = x[:, :3].detach().clone().requires_grad_(True)
            ms = [t.detach().clone().requires_grad_(True) for t in m]
            step[f"U{j + 1}"], step[f"m{j + 1}"] = U, ms
            slots.append((len(levels), list(range(len(levels) + 1, len(levels) + 1 + len(ms)))))
            levels += [U] + ms
        pc = [torch.tensor(v, dtype=torch.float64, device=dev, requires_grad=True) for v in rec["pc"]]
        q = [torch.tensor(v, dtype=torch.float64, device=dev, requires_grad=True) for v in rec["q"]]
        step["pc"], step["q"] = pc, q
        return step, {"pc": pc, "q": q, "levels": levels, "level_slots": slots}

    def _lumped_state(self, step, mb, th, rec):
        """``s_n (K, 2)``: each outlet's committed capacitor pressure and flow."""
        r = self.res
        rows = []
        for k, (z, zd) in enumerate(zip(self.outlets, r.lumped)):
            i = r.s._flow_zones.index(z)
            q = (r.s._flow_W[i] @ mb + r.s._flow_c[i]) / r.rho
            pc0, pc1 = rcr_step(zd["model"], step["pc"][k], step["q"][k], th[1 + 3 * k],
                                th[2 + 3 * k], th[3 + 3 * k], step["t"], step["dt"])
            rows.append(torch.stack([pc0 + pc1 * q, q]))
        return torch.stack(rows)

    def close(self):
        if self.solver is not None:
            self.solver.close()
            self.solver = None


def fgmres_batched(A, b, M, *, rtol=1e-10, restart=40, maxiter=400):
    """B right-preconditioned GMRES recurrences in lock-step: ``b (B, n)``, ``A`` and ``M``
    map ``(B, n)`` to ``(B, n)`` row by row, ``M`` a fixed linear operator (the transposed
    V-cycle is one: fixed sweeps, no inner tolerance), so that only the basis is stored and
    each restart cycle's update is ``M`` applied once to its combination of basis vectors (half
    the memory of the flexible form). Classical Gram-Schmidt applied twice (one batched product
    per pass over a preallocated basis), Givens rotations per system on the host; a system that
    reaches ``rtol`` (relative to ``|b|``) or breaks down freezes (its later basis vectors are
    zero) while the others go on. Returns ``(x, steps, residuals (B,))``."""
    B, n = b.shape
    dt, dev = b.dtype, b.device
    x = torch.zeros_like(b)
    bn = torch.linalg.norm(b, dim=1).cpu().numpy()
    bn_safe = np.where(bn > 0, bn, 1.0)
    m = restart
    Vb = torch.zeros((m + 1, B, n), dtype=dt, device=dev)
    r = b.clone()
    it = 0
    res = np.zeros(B)
    while True:
        beta = torch.linalg.norm(r, dim=1).cpu().numpy()
        res = np.where(bn > 0, beta / bn_safe, 0.0)
        live = res > rtol
        if not live.any() or it >= maxiter or not np.all(np.isfinite(res)):
            break
        scale = np.where(live & (beta > 0), 1.0 / np.where(beta > 0, beta, 1.0), 0.0)
        Vb[0] = r * torch.as_tensor(scale, dtype=dt, device=dev)[:, None]
        H = np.zeros((B, m + 1, m))
        cs, sn = np.zeros((B, m)), np.zeros((B, m))
        g = np.zeros((B, m + 1))
        g[:, 0] = beta
        steps = np.where(live, -1, 0)                       # -1 while a system is active
        k_used = 0
        for k in range(m):
            w = A(M(Vb[k]))
            V = Vb[:k + 1]
            h = np.zeros((B, k + 1))
            for _ in range(2):
                c = torch.einsum("jbn,bn->bj", V, w)
                w = w - torch.einsum("bj,jbn->bn", c, V)
                h += c.cpu().numpy()
            hn = torch.linalg.norm(w, dim=1).cpu().numpy()
            it += 1
            k_used = k + 1
            for q in range(B):
                if steps[q] >= 0:
                    continue
                col = np.concatenate([h[q], [hn[q]]])
                for j in range(k):
                    t = cs[q, j] * col[j] + sn[q, j] * col[j + 1]
                    col[j + 1] = -sn[q, j] * col[j] + cs[q, j] * col[j + 1]
                    col[j] = t
                den = np.hypot(col[k], col[k + 1])
                cs[q, k], sn[q, k] = (col[k] / den, col[k + 1] / den) if den else (1.0, 0.0)
                col[k], col[k + 1] = den, 0.0
                H[q, :k + 2, k] = col
                g[q, k + 1] = -sn[q, k] * g[q, k]
                g[q, k] = cs[q, k] * g[q, k]
                est = abs(g[q, k + 1]) / bn_safe[q]
                if est <= rtol or hn[q] == 0.0 or den == 0.0 or not np.isfinite(est):
                    steps[q] = k if den == 0.0 else k + 1
            if (steps >= 0).all() or it >= maxiter:
                break
            nxt = np.where(steps < 0, 1.0 / np.where(hn > 0, hn, 1.0), 0.0)
            Vb[k + 1] = w * torch.as_tensor(nxt, dtype=dt, device=dev)[:, None]
        Y = np.zeros((B, k_used))
        for q in range(B):
            K = k_used if steps[q] < 0 else steps[q]
            if K:
                Y[q, :K] = np.linalg.solve(np.triu(H[q, :K, :K]), g[q, :K])
        x = x + M(torch.einsum("bj,jbn->bn", torch.as_tensor(Y, dtype=dt, device=dev),
                               Vb[:k_used]))
        r = b - A(x)
    return x, it, res


def fgmres(A, b, M, *, rtol=1e-10, restart=40, maxiter=400):
    """Right-preconditioned flexible GMRES on torch vectors (modified Gram-Schmidt, Givens
    rotations): ``(x, iterations, residual relative to ||b||)``."""
    x = torch.zeros_like(b)
    bn = float(torch.linalg.norm(b))
    if bn == 0.0:
        return x, 0, 0.0
    r = b.clone()
    it = 0
    res = 1.0
    while it < maxiter:
        beta = float(torch.linalg.norm(r))
        res = beta / bn
        if res <= rtol:
            break
        V = [r / beta]
        Z = []
        H = np.zeros((restart + 1, restart))
        cs, sn = np.zeros(restart), np.zeros(restart)
        g = np.zeros(restart + 1)
        g[0] = beta
        k_used = 0
        for k in range(restart):
            z = M(V[k])
            Z.append(z)
            w = A(z)
            for j in range(k + 1):
                H[j, k] = float(torch.dot(V[j], w))
                w = w - H[j, k] * V[j]
            hn = float(torch.linalg.norm(w))
            H[k + 1, k] = hn
            for j in range(k):
                t = cs[j] * H[j, k] + sn[j] * H[j + 1, k]
                H[j + 1, k] = -sn[j] * H[j, k] + cs[j] * H[j + 1, k]
                H[j, k] = t
            den = np.hypot(H[k, k], H[k + 1, k])
            cs[k], sn[k] = (H[k, k] / den, H[k + 1, k] / den) if den else (1.0, 0.0)
            H[k, k] = den
            H[k + 1, k] = 0.0
            g[k + 1] = -sn[k] * g[k]
            g[k] = cs[k] * g[k]
            it += 1
            k_used = k + 1
            res = abs(g[k + 1]) / bn
            if res <= rtol or it >= maxiter or hn == 0.0 or not np.isfinite(res):
                break
            V.append(w / hn)
        y = np.linalg.solve(np.triu(H[:k_used, :k_used]), g[:k_used])
        for j in range(k_used):
            x = x + float(y[j]) * Z[j]
        r = b - A(x)
        res = float(torch.linalg.norm(r)) / bn
        if res <= rtol:
            break
    return x, it, res


class SteadySensitivity(torch.autograd.Function):
    """``J(theta)`` of a steady solve with its adjoint gradient: forward runs ``solve(theta)``
    (a callable returning a converged :class:`SteadyResidual`), backward one adjoint solve
    for the incoming ``dL/dJ``."""

    @staticmethod
    def forward(ctx, theta, solve):
        res = solve(theta.detach())
        x, mdot = res.state()
        J = res.objectives(x, mdot, theta.detach()).detach()
        ctx.res, ctx.state = res, (x, mdot)
        ctx.save_for_backward(theta)
        return J

    @staticmethod
    def backward(ctx, gJ):
        (theta,) = ctx.saved_tensors
        res = ctx.res
        x, mdot = ctx.state
        xz = x.detach().requires_grad_(True)
        mz = [m.detach().requires_grad_(True) for m in mdot]
        th = theta.detach().requires_grad_(True)
        J = res.objectives(xz, mz, th)
        gz = torch.autograd.grad((J * gJ).sum(), [xz, th] + mz, allow_unused=True)
        gx = torch.zeros_like(xz) if gz[0] is None else gz[0]
        gth = torch.zeros_like(th) if gz[1] is None else gz[1]
        gm = [torch.zeros_like(m) if g is None else g for g, m in zip(gz[2:], mz)]
        lam, _, _ = res.adjoint(gx, gm, x, mdot, theta)
        th2 = theta.detach().requires_grad_(True)
        r, gmd, _ = res.residual(x, mdot, th2)
        dR = torch.autograd.grad([r] + gmd, th2, [lam[0].view_as(r)] +
                                 [p.view_as(g) for p, g in zip(lam[1:], gmd)],
                                 allow_unused=True)[0]
        dR = torch.zeros_like(th2) if dR is None else dR
        return gth - dR, None


__all__ = ["SteadyResidual", "SteadySensitivity", "TransientSensitivity", "rcr_step", "fgmres",
           "fgmres_batched"]
