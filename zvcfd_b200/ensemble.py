"""Batched solves: independent vessel problems assembled and solved as one system.

The instances of an ensemble (meshes of uneven size, each with its own inlet flow and lumped
outlets) share no nodes, so their union is one mesh whose coupled system is block diagonal.
:class:`B200Ensemble` builds that union and runs one :class:`~zvcfd_b200.solver.B200Solver`
on it: every stage of an outer iteration (gradients, element kernels per colour, the boundary
pass, SpMV, the V-cycle graph, the Arnoldi passes, the update) is one launch over all
instances instead of one per instance, the AMG aggregates never cross instances (they are
not coupled), and the FGMRES basis holds every instance's residual at once. What stays per
instance is the convergence test: an instance has converged when its own relative changes
of velocity and pressure are below ``tol`` (the reference's criterion,
``zvcfd/fv/solver.py:990-1005``, applied to its node range), and the ensemble stops when all
have converged with the last linear solve converged.

The reference solves instances one after the other; :func:`solve_sequentially` is that
baseline on the same GPU.

The linear solve has two forms. ``krylov="union"`` runs one FGMRES over the union, so its
inner products and its residual reduction are those of all instances together: instances of
similar size and residual converge together (the three-vessel test), but on the 12-vessel
workload (59k-909k nodes) the small instances get no reduction of their own.
``krylov="segmented"`` (the default) runs one Krylov recurrence per instance inside the device
FGMRES (``zvfv_solver_solve_segmented``): the operator products and V-cycles still cover all
instances in one launch each, while every inner product, Hessenberg column, rotation and step
length is per instance, and each instance's solve stops at ``linear_rtol`` of its own initial
residual. :func:`segmented_fgmres` restates that algorithm in torch (checked on the CPU).
"""

from __future__ import annotations

import time

import numpy as np
import torch

from zvcfd_b200.mesh import Mesh, Zone
from zvcfd_b200.solver import B200Solver
from zvcfd_b200.topology import KINDS


def union(meshes: list) -> tuple:
    """The disjoint union of ``meshes``: ``(mesh, node_offsets (M+1,), zone_ids)`` where
    ``zone_ids[i][z]`` is the union's id of zone ``z`` of instance ``i`` (ids from 3)."""
    offsets = np.zeros(len(meshes) + 1, np.int64)
    for i, m in enumerate(meshes):
        offsets[i + 1] = offsets[i] + m.n_nodes
    nodes = np.concatenate([m.nodes for m in meshes])
    kinds = [k for k in KINDS if any(k in m.elements for m in meshes)]
    elements = {k: np.concatenate([m.elements[k] + offsets[i] for i, m in enumerate(meshes)
                                   if k in m.elements]) for k in kinds}
    zones, ids, nxt = {}, [], 3
    for i, m in enumerate(meshes):
        ids.append({})
        for z, zz in sorted(m.zones.items()):
            f = np.where(zz.faces >= 0, zz.faces + offsets[i], -1)
            zones[nxt] = Zone(nxt, zz.kind, f"{zz.name}#{i}", f)
            ids[i][z] = nxt
            nxt += 1
    return Mesh(nodes, elements, zones), offsets, ids


def segmented_fgmres(apply_A, apply_M, b, x0, bounds, rtol: float, *, restart: int = 30,
                     maxiter: int = 200):
    """Right-preconditioned FGMRES with one Krylov recurrence per segment of a block-diagonal
    system: every inner product, norm, Hessenberg column, Givens rotation and step length is
    taken per segment (``bounds``: the segments' first positions and the end, contiguous),
    while the operator and the preconditioner are applied to all segments at once. Each segment
    stops by its own criterion, a reduction ``rtol`` of its initial residual (with the
    reference's round-off floor of ``1e-13`` of its right-hand side); the iteration ends when
    all have. The basis is one preallocated ``(restart + 1, n)`` block and each Gram-Schmidt
    pass is one product per segment, so a Krylov step costs a few launches per segment
    whatever its index. Returns ``(x, iterations, largest relative residual, all converged)``.
    """
    dt, dev = b.dtype, b.device
    sl = [slice(int(bounds[i]), int(bounds[i + 1])) for i in range(len(bounds) - 1)]
    nseg = len(sl)
    n = b.numel()

    def sdot(a, c):                                  # (nseg,) inner products
        return torch.stack([torch.dot(a[q], c[q]) for q in sl])

    def expand(v):                                   # a value per segment, per row
        out = torch.empty(n, dtype=dt, device=dev)
        for i, q in enumerate(sl):
            out[q] = v[i]
        return out

    m = restart
    Vb = torch.zeros((m + 1, n), dtype=dt, device=dev)
    Zb = torch.zeros((m, n), dtype=dt, device=dev)
    x = x0.clone()
    r = b - apply_A(x)
    beta0 = torch.sqrt(sdot(r, r))
    target = torch.maximum(rtol * beta0, 1e-13 * torch.sqrt(sdot(b, b)))
    beta = beta0.clone()
    its = 0
    while its < maxiter and bool((beta > target).any()):
        H = torch.zeros((nseg, m + 1, m), dtype=dt, device=dev)
        cs = torch.zeros((nseg, m), dtype=dt, device=dev)
        sn = torch.zeros_like(cs)
        g = torch.zeros((nseg, m + 1), dtype=dt, device=dev)
        g[:, 0] = beta
        Vb[0] = r * expand(torch.where(beta > 0, 1.0 / beta, torch.zeros_like(beta)))
        k_used = 0
        for k in range(m):
            Zb[k] = apply_M(Vb[k])
            w = apply_A(Zb[k])
            V = Vb[:k + 1]
            for _ in range(2):                                   # classical Gram-Schmidt, twice
                h = torch.stack([V[:, q] @ w[q] for q in sl], 1)          # (k+1, nseg)
                for i, q in enumerate(sl):
                    w[q] -= h[:, i] @ V[:, q]
                H[:, :k + 1, k] += h.T
            hn = torch.sqrt(sdot(w, w))
            H[:, k + 1, k] = hn
            Vb[k + 1] = w * expand(torch.where(hn > 0, 1.0 / hn, torch.zeros_like(hn)))
            for j in range(k):                                   # earlier rotations
                t = cs[:, j] * H[:, j, k] + sn[:, j] * H[:, j + 1, k]
                H[:, j + 1, k] = -sn[:, j] * H[:, j, k] + cs[:, j] * H[:, j + 1, k]
                H[:, j, k] = t
            den = torch.hypot(H[:, k, k], H[:, k + 1, k])
            ok = den > 0
            cs[:, k] = torch.where(ok, H[:, k, k] / torch.where(ok, den, 1.0), 1.0)
            sn[:, k] = torch.where(ok, H[:, k + 1, k] / torch.where(ok, den, 1.0), 0.0)
            H[:, k, k] = den
            H[:, k + 1, k] = 0.0
            g[:, k + 1] = -sn[:, k] * g[:, k]
            g[:, k] = cs[:, k] * g[:, k]
            its += 1
            k_used = k + 1
            if bool((g[:, k + 1].abs() <= target).all()) or its >= maxiter:
                break
        R = H[:, :k_used, :k_used].clone()
        rhs = g[:, :k_used].clone()
        zero = R.diagonal(dim1=1, dim2=2) == 0                  # segments with nothing to solve
        R.diagonal(dim1=1, dim2=2)[zero] = 1.0
        rhs[zero] = 0.0
        y = torch.linalg.solve_triangular(R, rhs[..., None], upper=True)[..., 0]   # (nseg, k)
        for i, q in enumerate(sl):
            x[q] += y[i] @ Zb[:k_used, q]
        r = b - apply_A(x)
        beta = torch.sqrt(sdot(r, r))
    rel = beta / torch.where(beta0 > 0, beta0, torch.ones_like(beta0))
    return x, its, float(rel.max()), bool((beta <= 1.01 * target).all())


class B200Ensemble:
    """Independent steady problems ``cases = [(mesh, bcs), ...]`` of one fluid, solved together
    (see the module docstring). ``solver_options`` go to :class:`B200Solver`."""

    def __init__(self, cases: list, fluid, *, krylov: str = "segmented", **solver_options):
        meshes = [m for m, _ in cases]
        self.mesh, self.offsets, self.zone_ids = union(meshes)
        bcs = {}
        for i, (_, b) in enumerate(cases):
            for z, spec in b.items():
                bcs[self.zone_ids[i][z]] = spec
        self.n = len(cases)
        if krylov == "segmented":
            from zvcfd_b200.linear import B200AMG

            lin = solver_options.pop("linear", "b200")
            if lin not in ("b200", "b200-mixed"):
                raise ValueError(f"krylov 'segmented' builds its own b200 back end, not {lin!r}")
            opts = dict(solver_options.pop("linear_options", None) or {})
            rtol = solver_options.get("linear_rtol", 0.1)
            solver_options["linear"] = B200AMG(
                rtol=rtol, precision="mixed" if lin == "b200-mixed" else "double",
                segments=self.offsets, **opts)
        elif krylov != "union":
            raise ValueError(f"krylov {krylov!r}: segmented or union")
        self.solver = B200Solver(self.mesh, fluid, bcs, **solver_options)
        self._len = torch.as_tensor(np.diff(self.offsets), device="cuda")

    def _per_instance(self, values, reduce):
        return torch.segment_reduce(values, reduce, lengths=self._len)

    def solve(self, *, max_iterations: int = 400, tol: float = 1e-8, log=None) -> dict:
        """Outer iterations until every instance's relative changes are below ``tol``
        (``log``: called every 10 iterations with the number of converged instances)."""
        s = self.solver
        t0 = time.time()
        done = np.zeros(self.n, bool)
        first = np.full(self.n, -1)
        hist = []
        seg = getattr(s.linear, "segments", None) is not None
        for it in range(max_iterations):
            U0, P0 = s.U.clone(), s.P.clone()
            if seg:                 # converged instances stop: their blocks keep the state
                s.linear.segment_active = ~done
            rec = s.iterate()
            du = self._per_instance((s.U - U0).abs().amax(1), "max")
            um = self._per_instance(s.U.abs().amax(1), "max")
            dp = self._per_instance((s.P - P0).abs(), "max")
            pr = self._per_instance(s.P, "max") - self._per_instance(s.P, "min")
            du = (du / um.clamp(min=1e-300)).cpu().numpy()
            dp = (dp / pr.clamp(min=1e-300)).cpu().numpy()
            ok = (du < tol) & (dp < tol) & (it > 0)
            first[ok & (first < 0)] = it + 1
            done = ok
            hist.append({"iteration": it + 1, "du": du, "dp": dp,
                         "linear_iterations": rec["linear_iterations"]})
            if log and (it + 1) % 10 == 0:
                log(f"ensemble iteration {it + 1}: {int(done.sum())}/{self.n} converged, "
                    f"{time.time() - t0:.1f} s")
            if done.all() and rec["linear_converged"]:
                break
        return {"iterations": len(hist), "converged": bool(done.all()), "first_converged": first,
                "history": hist, "seconds": time.time() - t0}

    def fields(self, i: int) -> dict:
        """Velocity and pressure of instance ``i``."""
        a, b = int(self.offsets[i]), int(self.offsets[i + 1])
        f = self.solver.fields()
        return {"U": f["U"][a:b], "P": f["P"][a:b]}

    def patch_flows(self, i: int) -> dict:
        """Volume outflow through each zone of instance ``i`` (its own zone ids)."""
        q = self.solver.patch_flows()
        return {z: q[u] for z, u in self.zone_ids[i].items()}

    def close(self):
        self.solver.close()


def solve_sequentially(cases: list, fluid, *, max_iterations: int = 400, tol: float = 1e-8,
                       log=None, **solver_options) -> dict:
    """The baseline: each instance solved on its own, one after the other (``log``: called
    with a line per instance)."""
    t0 = time.time()
    out = []
    for i, (m, bcs) in enumerate(cases):
        t = time.time()
        s = B200Solver(m, fluid, bcs, **solver_options)
        rep = s.solve(max_iterations=max_iterations, tol=tol)
        out.append({"iterations": rep["iterations"], "converged": rep["converged"],
                    "fields": s.fields(), "flows": s.patch_flows(), "seconds": time.time() - t})
        s.close()
        if log:
            log(f"instance {i}: {m.n_nodes} nodes, {rep['iterations']} outer iterations, "
                f"converged {rep['converged']}, {time.time() - t:.1f} s")
    return {"instances": out, "seconds": time.time() - t0}


def _section_nodes(radius, n_core, n_ring, growth):
    from zvcfd_b200.mesh import ogrid_section

    return len(ogrid_section(radius, n_core, n_ring, growth=growth)[0])


def vessel(kind: str, nodes: int, seed: int):
    """A seeded vessel mesh of about ``nodes`` nodes: ``"straight"`` (the tet pipe of the
    Poiseuille workload, radius 1 mm, length 10 mm), ``"curved"`` (the hexahedral/prismatic
    90-degree tube, radius 2 mm, bend 20 mm) or ``"bifurcating"`` (the tet Y-bifurcation).
    Returns ``(mesh, inlet radius, outlet zone names)``."""
    from zvcfd_b200.mesh import curved_tube, pipe, y_bifurcation

    if kind == "straight":
        k = (nodes / 49977.0) ** (1.0 / 3.0)
        nc, nr = max(3, round(14 * k)), max(2, round(7 * k))
        P = _section_nodes(1e-3, nc, nr, 1.0)
        return (pipe(1e-3, 10e-3, n_core=nc, n_ring=nr, n_axial=max(4, round(nodes / P) - 1),
                     kind="tet", jitter_amount=0.05, seed=seed), 1e-3, ["outlet"])
    if kind == "curved":
        k = (nodes / 400686.0) ** (1.0 / 3.0)
        nc, nr = max(4, round(20 * k)), max(6, round(12 * k))
        P = _section_nodes(2e-3, nc, nr, 0.8)
        return (curved_tube(2e-3, 20e-3, np.pi / 2, n_core=nc, n_ring=nr,
                            n_axial=max(4, round(nodes / P) - 1), layers=5, growth=0.8), 2e-3,
                ["outlet"])
    if kind == "bifurcating":
        h = 0.25e-3 * (56118.0 / nodes) ** (1.0 / 3.0)
        return y_bifurcation(h, jitter_amount=0.05, seed=seed), 2e-3, ["outlet1", "outlet2"]
    raise ValueError(f"vessel kind {kind!r}")


def synthetic_ensemble(count: int = 12, low: int = 50_000, high: int = 1_200_000, seed: int = 0):
    """The batched-ensemble workload: ``count`` vessels of log-uniform sizes in
    ``[low, high]`` nodes, kinds in turn straight / curved / bifurcating, each with a
    parabolic inlet of flow U(0.5, 3) ml/s and RCR outlets with log-uniform
    Rp in [0.5, 2]e8, C in [0.5, 2]e-9, Rd in [0.5, 2]e9 (SI). Returns ``[(mesh, bcs)]``."""
    from zvcfd_b200.lumped import RCR

    rng = np.random.default_rng(seed)
    kinds = ("straight", "curved", "bifurcating")
    cases = []
    for i in range(count):
        target = int(np.exp(rng.uniform(np.log(low), np.log(high))))
        m, R, outlets = vessel(kinds[i % 3], target, seed + i)
        z = {zz.name: k for k, zz in m.zones.items()}
        q = rng.uniform(0.5e-6, 3e-6)

        def shape(x, R=R):
            return np.clip(1.0 - (x[:, 0] ** 2 + x[:, 1] ** 2) / R ** 2, 0.0, None)

        bcs = {z["inlet"]: {"kind": "velocity", "flow_rate": q, "profile": shape},
               z["wall"]: {"kind": "wall"}}
        for name in outlets:
            rp, c, rd = np.exp(rng.uniform(np.log(0.5), np.log(2.0), 3)) * np.array([1e8, 1e-9, 1e9])
            bcs[z[name]] = {"kind": "pressure", "lumped": RCR(rp=rp, c=c, rd=rd)}
        cases.append((m, bcs))
    return cases


__all__ = ["union", "segmented_fgmres", "B200Ensemble", "solve_sequentially",
           "vessel", "synthetic_ensemble"]
