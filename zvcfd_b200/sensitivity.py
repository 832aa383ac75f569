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

    def __init__(self, solver, inlet: int, outlets: list, walls: dict):
        s = solver
        if not isinstance(s.advection, (int, float)):
            raise ValueError("the adjoint needs a fixed advection blend (a number)")
        if s.dt or s._time is not None:
            raise ValueError("the adjoint is of the steady state")
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
        self.q0 = float(spec["flow_rate"])
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

    def residual(self, x, mdot, theta):
        """``(r (N, 4), [mdot residual per type])``; ``r`` unscaled, one row per unknown."""
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
        dnode = self.V / aP
        r = torch.zeros((N, 4), dtype=x.dtype, device=x.device)
        gmd = []
        for g, m, (L, mu) in zip(self.geo, mdot, per):
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
            f = torch.cat([mom, flow[..., None]], -1)                      # (E, nip, 4)
            r = r.index_add(0, g.node_a.reshape(-1), f.reshape(-1, 4))
            r = r.index_add(0, g.node_b.reshape(-1), -f.reshape(-1, 4))
            gmd.append(m - flow)
        # the boundary pass: outflow advection at outlets, pressure forces, body forces,
        # known inflows, the outlet traction of the transpose term
        scale = q / self.q0
        inflow = self.inflow0 * scale
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
        cont = r[:, 3] + inflow
        raw_cont = cont
        # Dirichlet rows
        vel = self.vel0 * scale
        mom = torch.where(self.fixed, U - vel, mom)
        cont = torch.where(self.pfix, P - self.pval, cont)
        # lumped rows: p_j - (Rp + Rd) Q = a, Q the zone's outflow by its raw continuity rows
        for k, (z, zd) in enumerate(zip(self.outlets, self.lumped)):
            rp, rd = theta[1 + 3 * k], theta[3 + 3 * k]
            nodes = zd["nodes"]
            Q = -raw_cont[nodes].sum() / self.rho
            a, _ = zd["model"].steady_coefficients(self.s.t)
            cont = cont.index_copy(0, nodes, P[nodes] - (rp + rd) * Q - a)
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

    def sensitivities(self, rtol=1e-11, restart=200, maxiter=1000):
        """``dJ/dtheta`` ``(n_objectives, n_parameters)``: one adjoint solve per objective (the
        objectives' right-hand sides share the forward hierarchy and residual graph)."""
        x, mdot = self.state()
        theta = self.theta0()
        xz = x.detach().requires_grad_(True)
        mz = [m.detach().requires_grad_(True) for m in mdot]
        th = theta.detach().requires_grad_(True)
        J = self.objectives(xz, mz, th)
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


__all__ = ["SteadyResidual", "SteadySensitivity", "fgmres"]
