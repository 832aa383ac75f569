"""The coupled solve on partitions of the mesh: the reference's ``MultiGPUSolver``.

:class:`B200MultiSolver` has the interface of the reference's ``MultiGPUSolver``
(``zvcfd/fv/multi.py:139-597``) and solves the same discrete equations as
:class:`~zvcfd_b200.solver.B200Solver` on the partitions of :mod:`zvcfd_b200.partition`
(whole Morton chunks, a one-element halo). Each partition is a ``B200Solver`` on its local
mesh whose rows past ``n_own`` (the halo) are assembled but never solved; this class runs the
outer iteration across them:

1. per partition the nodal gradients, blend factors and momentum diagonal (valid at owned
   nodes), then one halo exchange of all four, since the flux points of halo elements need
   them at halo nodes;
2. per partition the element assembly and the boundary pass of the owned rows, with the row
   scales ``U_ref``/``p_ref`` reduced over all partitions on the device; a lumped outlet's flow
   ``Q = Σ_p (w_p . x + c_p)`` is summed over partitions, so its rank-one row is global;
3. one FGMRES (:func:`fgmres`) over the owned unknowns of every partition: each operator
   product fills the halo of the local vectors, runs the block SpMV of each partition's owned
   rows straight into the owned vector and adds the global rank-one terms; the preconditioner
   is block Jacobi over partitions, one AMG V-cycle on each partition's owned rows and columns;
4. the update of the owned values, a halo exchange of ``u`` and ``p``, then of ``∇p`` for the
   Rhie-Chow mass flows, which every partition evaluates identically on shared elements.

Residual statistics, changes, zone flows and convergence are reduced over owned nodes. With one
partition this is the single-GPU solve with a host-driven FGMRES; with several, the converged
solution is the same to the solver tolerance, because only the preconditioner changes.

**Placement.** Without a process group every partition lives in this process on the current
device (the reference's test setting, partitions sharing one device). The partitions' owned
rows form one vector, and their owned blocks one block-diagonal matrix: the preconditioner is
one hierarchy and one V-cycle graph for all of them (aggregates never cross partitions, since
no block joins two of them). With ``group`` (a ``torch.distributed`` process group, one
process per GPU over NCCL) the partitions are dealt to the ranks in contiguous runs of the
Morton order; halo rows between ranks travel as point-to-point sends and receives (one batch
per exchange, in the same global order on every rank), and inner products, scales and
statistics are all-reduced. Every rank builds the same partitions from the same mesh.

Not supported across partitions: average-pressure zones (as in the reference: their mean
couples a zone globally), openings, eddy viscosity.
"""

from __future__ import annotations

import time

import numpy as np
import torch
import torch.distributed as dist

from zvcfd_b200._lib import call, ptr, stream_ptr
from zvcfd_b200.boundary import Boundary, call_value, takes_two
from zvcfd_b200.forces import zone_forces
from zvcfd_b200.linear import BlockMatrix, SolveInfo, make
from zvcfd_b200.partition import halo_plan, local_meshes, morton_owner, partition_report
from zvcfd_b200.solver import BDF, B200Solver, _zone_flow, time_steps

ROUNDOFF = 1e-13


# ---------------------------------------------------------------- processes and halos

class Reducer:
    """Sums and maxima of small tensors over the processes of a group (nothing to do with
    one process)."""

    def __init__(self, group=None):
        self.group = group
        self.world = dist.get_world_size(group) if group is not None else 1
        self.rank = dist.get_rank(group) if group is not None else 0

    def sum(self, t: torch.Tensor) -> torch.Tensor:
        if self.world > 1:
            dist.all_reduce(t, op=dist.ReduceOp.SUM, group=self.group)
        return t

    def max(self, t: torch.Tensor) -> torch.Tensor:
        if self.world > 1:
            dist.all_reduce(t, op=dist.ReduceOp.MAX, group=self.group)
        return t

    def peer(self, rank: int) -> int:
        """The global rank of a rank of the group (point-to-point operations take those)."""
        if self.group is None or self.world == 1:
            return rank
        return dist.get_global_rank(self.group, rank)


def deal(n_parts: int, world: int) -> np.ndarray:
    """The rank holding each partition: contiguous runs of the Morton order, as even as
    possible (neighbouring partitions share most halos, so runs keep them in one process)."""
    if world > n_parts:
        raise ValueError(f"{n_parts} partitions cannot feed {world} processes")
    return (np.arange(n_parts) * world) // n_parts


class HaloExchange:
    """The halo plans of the partitions held by this process, compiled for its device.

    ``__call__(arrays)`` fills, in place, the halo rows of ``arrays[p]`` (a tensor whose first
    axis is ``p``'s local nodes, for every partition ``p`` held here) with their owners'
    values: copies between partitions held here are one gather and one scatter each; rows
    between processes go in one batch of point-to-point operations, listed in the same global
    ``(p, q)`` order on every rank, so the messages between two ranks pair up in order.
    """

    def __init__(self, plans: list, rank_of, reducer: Reducer, device):
        self.rank_of = [int(r) for r in rank_of]
        self.red = reducer
        me = reducer.rank
        idx = lambda a: torch.as_tensor(np.ascontiguousarray(a), dtype=torch.int64,   # noqa: E731
                                        device=device)
        self.local, self.remote = [], []
        for p, plan in enumerate(plans):
            for q, send, recv in plan:
                here_p, here_q = self.rank_of[p] == me, self.rank_of[q] == me
                if here_p and here_q:
                    self.local.append((p, q, idx(send), idx(recv)))
                elif here_p or here_q:
                    self.remote.append((p, q, idx(send), idx(recv)))

    @property
    def crosses_processes(self) -> bool:
        return bool(self.remote)

    def __call__(self, arrays) -> None:
        for p, q, send, recv in self.local:
            arrays[p].index_copy_(0, recv, arrays[q].index_select(0, send))
        if not self.remote:
            return
        me = self.red.rank
        ops, inbox = [], []
        for p, q, send, recv in self.remote:
            if self.rank_of[q] == me:                        # q's owned rows go to p's rank
                buf = arrays[q].index_select(0, send).contiguous()
                ops.append(dist.P2POp(dist.isend, buf, self.red.peer(self.rank_of[p]),
                                      self.red.group))
            else:
                a = arrays[p]
                buf = torch.empty((recv.numel(),) + tuple(a.shape[1:]), dtype=a.dtype,
                                  device=a.device)
                ops.append(dist.P2POp(dist.irecv, buf, self.red.peer(self.rank_of[q]),
                                      self.red.group))
                inbox.append((p, recv, buf))
        for req in dist.batch_isend_irecv(ops):
            req.wait()
        for p, recv, buf in inbox:
            arrays[p].index_copy_(0, recv, buf)


# ---------------------------------------------------------------- Krylov solve

def _givens(a: float, b: float):
    d = float(np.hypot(a, b))
    return (a / d, b / d, d) if d else (1.0, 0.0, 0.0)


def fgmres(matvec, precond, b, x0, *, rtol: float, restart: int = 30, maxiter: int = 200,
           reducer: Reducer | None = None):
    """Right-preconditioned flexible GMRES (Saad 1993) over a vector whose rows may be spread
    over processes: ``(x, iterations, residual relative to the initial one, converged)``.

    The semantics of the device FGMRES (``zvfv_solver_solve``) and of the reference's
    ``fgmres`` (``zvcfd/fv/linear.py:170-235``): convergence at ``rtol`` relative to the initial
    residual (AmgX's ``RELATIVE_INI``) or at round-off (``1e-13 ‖b‖``), restarts after
    ``restart`` steps, ``maxiter`` steps in all, a lucky breakdown ends a cycle; after every
    cycle the true residual decides whether another follows, and ``converged`` is that
    residual within 1 % of the target. The orthogonalisation is classical Gram-Schmidt applied
    twice (CGS2): the basis is one ``(restart + 1, n)`` device array, each pass one product
    with it and one reduction over processes, where the reference's host loop reduces once per
    basis vector.
    """
    red = reducer or Reducer()
    n = b.numel()

    def norm(v) -> float:
        return float(red.sum((v * v).sum().reshape(1)).sqrt())

    x = x0.reshape(-1).clone()
    r = b - matvec(x)
    beta = norm(r)
    r0 = beta or 1.0
    tol = max(rtol, ROUNDOFF * norm(b) / r0)
    res = beta / r0
    V = torch.empty((restart + 1, n), dtype=b.dtype, device=b.device)
    Z = torch.empty((restart, n), dtype=b.dtype, device=b.device)
    it = 0
    while res > tol and it < maxiter and np.isfinite(res):
        V[0] = r / beta
        H = np.zeros((restart + 1, restart))
        g = np.zeros(restart + 1)
        g[0] = beta
        rot = []
        k_used = 0
        for k in range(restart):
            Z[k] = precond(V[k])
            w = matvec(Z[k])
            basis = V[:k + 1]
            h = red.sum(basis @ w)
            w = w - h @ basis
            h2 = red.sum(basis @ w)
            w = w - h2 @ basis
            col = (h + h2).cpu().numpy()
            hnext = norm(w)
            for j, (c, s) in enumerate(rot):              # the earlier rotations
                u, v = col[j], col[j + 1]
                col[j], col[j + 1] = c * u + s * v, c * v - s * u
            c, s, d = _givens(col[k], hnext)
            rot.append((c, s))
            H[:k + 1, k] = col
            H[k, k] = d
            g[k + 1] = -s * g[k]
            g[k] = c * g[k]
            it += 1
            k_used = k + 1
            est = abs(g[k + 1]) / r0
            if est <= tol or it >= maxiter or hnext == 0.0 or not np.isfinite(est):
                break
            V[k + 1] = w / hnext
        y = np.linalg.solve(np.triu(H[:k_used, :k_used]), g[:k_used])
        x += torch.as_tensor(y, dtype=b.dtype, device=b.device) @ Z[:k_used]
        r = b - matvec(x)
        beta = norm(r)
        res = beta / r0
    return x, it, res, bool(res <= 1.01 * tol)


# ---------------------------------------------------------------- one partition

def _node_view(name):
    """A property: the global boundary's node array ``name`` at a partition's local nodes."""
    return property(lambda self: getattr(self.g, name)[self.idx])


def _face_view(name):
    """A property: the global boundary's per-face dict ``name`` at the faces a partition
    holds."""
    return property(lambda self: {z: None if v is None else v[self.lm.faces[z]]
                                  for z, v in getattr(self.g, name).items()})


class PartBoundary:
    """The global :class:`~zvcfd_b200.boundary.Boundary` seen from one partition.

    Node arrays are the global ones at the partition's local nodes and zones are the faces it
    holds, read through to the global object (so a time update of it shows). Whatever is a sum
    over the domain counts the partition's owned nodes only: the zone-flow weights vanish at
    halo nodes and the known flows of inlets are the owned nodes' shares
    (``zvcfd/fv/solver.py:1262-1269``).
    """

    def __init__(self, glob: Boundary, lm, cache: dict):
        self.g, self.lm, self.cache = glob, lm, cache
        self.mesh, self.bcs, self.rho = lm.mesh, glob.bcs, glob.rho
        self.N, self.n_own = len(lm.nodes), lm.n_own
        self.idx = lm.nodes
        self.mu, self.viscosity, self.transpose = glob.mu, glob.viscosity, glob.transpose
        self.sub = {zid: (lm.mesh.zones[zid].faces, S[lm.faces[zid]])
                    for zid, (f, S) in glob.sub.items()}
        self.zone_nodes = {zid: np.unique(f[f >= 0]) for zid, (f, _) in self.sub.items()}
        self.pin = None

    wall, inlet = _node_view("wall"), _node_view("inlet")
    outlet, sym = _node_view("outlet"), _node_view("sym")
    vel_fixed, vel_fixed_comp = _node_view("vel_fixed"), _node_view("vel_fixed_comp")
    p_fixed, vel_value = _node_view("p_fixed"), _node_view("vel_value")
    p_value, inflow = _node_view("p_value"), _node_view("inflow")
    sub_flow, sub_vel = _face_view("sub_flow"), _face_view("sub_vel")
    p_sub, p_grad = _face_view("p_sub"), _face_view("p_grad")

    def _global(self, key, fn):
        if key not in self.cache:
            self.cache[key] = fn()
        return self.cache[key]

    def update(self, t: float) -> None:
        """Nothing: the partitioned solver updates the global boundary."""

    def lumped_zones(self) -> list:
        return self.g.lumped_zones()

    def special_zones(self) -> dict:
        return self.g.special_zones()

    def has_pressure_zone(self) -> bool:
        return self.g.has_pressure_zone()

    def pressure_area(self) -> np.ndarray:
        return self._global("pressure_area", self.g.pressure_area)[self.idx]

    def outlet_force(self) -> np.ndarray:
        return self.g.outlet_force()[self.idx]

    def outlet_arrays(self):
        return tuple(a[self.idx] for a in self._global("outlet_arrays", self.g.outlet_arrays))

    def inflow_offsets(self) -> np.ndarray:
        return self._global("inflow_offsets", self.g.inflow_offsets)[self.idx]

    def outflow_only(self) -> np.ndarray:
        return self._global("outflow_only", self.g.outflow_only)[self.idx]

    def flow_constants(self, zids) -> np.ndarray:
        own = self.idx[:self.n_own]
        out = []
        for z in zids:
            if z not in self.g.sub_flow:
                out.append(0.0)
                continue
            f = self.g.sub[z][0]
            on = f >= 0
            per_node = np.bincount(f[on], self.g.sub_flow[z][on], self.g.N)
            out.append(float(per_node[own].sum()))
        return np.array(out)

    def flow_weights(self):
        zids, W, _ = self._global("flow_weights", self.g.flow_weights)
        W = W[:, self.idx].copy()
        W[:, self.n_own:] = 0.0
        return zids, W, self.flow_constants(zids)


class _NoLinear:
    """A partition solves nothing on its own: the partitioned solver runs the Krylov solve."""

    name = "partition"


class _Part(B200Solver):
    """One partition: a :class:`B200Solver` on a local mesh whose halo rows are not solved,
    fed its boundary data, control volumes, row scales and exchanged stage-one fields by the
    partitioned solver."""

    def __init__(self, G: "B200MultiSolver", lm):
        self.G, self.lm, self.n_own = G, lm, lm.n_own
        self._pre = None
        super().__init__(lm.mesh, G.fluid, G.bcs, source=G.source, advection=G.advection,
                         dt=G.dt, stokes=G.stokes, rhie_chow=G.rhie_chow,
                         transpose=G.transpose, freeze_limiter=G.freeze_limiter, t=G.t,
                         linear=_NoLinear(), store_geometry=G.store_geometry,
                         eliminate=G.eliminate)
        # a lumped zone's pressure is an unknown at every node of the zone this partition
        # holds (halo ones too, whose columns its owned rows couple to), and its rows are
        # scaled by the zone's whole area and node count
        known = self._known4.view(self.N, 4).clone()
        for zid in self.bc.lumped_zones():
            f = self.bc.sub[zid][0]
            nodes = torch.as_tensor(np.unique(f[f >= 0]), device=known.device)
            known[nodes, 3] = 0
            z = self._lumped[zid]
            if len(z["nodes_h"]):
                self._lscale[z["nodes"]] = G._lumped_scale[zid]
        self._known4 = known.reshape(self._known4.shape).contiguous()

    def _node_volume(self):
        return self.asm.node_volume.clone()          # whole at owned nodes; halo from owners

    def _make_boundary(self, reference_pressure):
        return PartBoundary(self.G.bc, self.lm, self.G._bcache)

    def _scales(self):
        return self.G._scal

    def _stage1(self):
        return self._pre

    def lumped_coefficients(self, zid):
        return self.G.lumped_coefficients(zid)

    def _finish_lumped(self, A, b, rs):
        self._system = (A, b, rs)                    # the partitioned solver finishes them

    def _initial_pressure(self):
        """Nothing: the partitioned solver sets the starting level of every partition."""


# ---------------------------------------------------------------- the partitioned solver

class B200MultiSolver:
    """Coupled finite-volume solve on partitions of the mesh (see the module docstring).

    Args:
        mesh, fluid, bcs, source, advection, dt, reference_pressure, stokes, rhie_chow,
            transpose, freeze_limiter, t, store_geometry, eliminate: as
            :class:`~zvcfd_b200.solver.B200Solver`.
        parts: number of partitions (``zvcfd/fv/multi.py:174-186``).
        chunk: the partitions' chunk edge (mesh units); default about 64 chunks per part.
        owner: a given owner partition per node instead of the Morton cut.
        group: a ``torch.distributed`` process group (NCCL, one process per GPU) to deal the
            partitions over; ``None`` keeps every partition in this process on the current
            device.
        linear: the per-partition preconditioner's AMG (``"b200"`` or ``"b200-mixed"``, with
            ``linear_options``), its aggregates rebuilt every ``rebuild_every`` set-ups (the
            reference's ACM rebuilds every 10).
        linear_rtol, restart, maxiter: of the global FGMRES.
    """

    def __init__(self, mesh, fluid, bcs, *, parts: int = 2, chunk=None, owner=None, group=None,
                 source=None, advection="high-resolution", dt=None, reference_pressure=None,
                 stokes=False, rhie_chow=1.0, transpose="auto", freeze_limiter=10, t=0.0,
                 linear="b200", linear_rtol=0.1, linear_options=None, restart=30,
                 maxiter=200, rebuild_every=10, store_geometry="auto", eliminate=True):
        t0 = time.time()
        for zid, spec in bcs.items():
            if spec.get("profile") == "average" or spec.get("opening"):
                # an average's mean couples the zone globally; an opening's halo nodes would be
                # eliminated from owned rows with their owner's last value
                raise NotImplementedError(f"zone {zid}: average-pressure and opening zones "
                                          "need one partition")
        self.mesh, self.fluid, self.bcs, self.source = mesh, fluid, bcs, source
        self.advection, self.dt, self.stokes = advection, dt, bool(stokes)
        self.rhie_chow, self.freeze_limiter = float(rhie_chow), freeze_limiter
        self.transpose = (fluid.viscosity is not None) if transpose == "auto" else bool(transpose)
        self.store_geometry, self.eliminate = store_geometry, bool(eliminate)
        self.t = float(t)
        self.N = mesh.n_nodes
        self.iteration = 0
        self._time = None
        self.bc = Boundary(mesh, bcs, fluid.rho, reference_pressure=reference_pressure, t=self.t,
                           mu=fluid.mu, viscosity=fluid.viscosity, transpose=self.transpose)
        self._bcache = {}
        self._lumped_scale = {}
        for zid in self.bc.lumped_zones():
            f, S = self.bc.sub[zid]
            on = f >= 0
            area = float(np.linalg.norm(S[on], axis=-1).sum())
            self._lumped_scale[zid] = 1.0 / (fluid.rho * area * np.sqrt(np.unique(f[on]).size))
        self.owner = morton_owner(mesh.nodes, parts, chunk) if owner is None \
            else np.asarray(owner, np.int64)
        self.local = local_meshes(mesh, self.owner)
        self.plan = halo_plan(self.local, self.owner)
        self.report = partition_report(self.local)
        self.red = Reducer(group)
        self.rank_of = deal(len(self.local), self.red.world)
        self.mine = [p for p in range(len(self.local)) if self.rank_of[p] == self.red.rank]
        self.device = torch.device("cuda", torch.cuda.current_device())
        self.exchange = HaloExchange(self.plan, self.rank_of, self.red, self.device)
        # the group's first collective involves every rank (a rank without remote halo rows
        # takes no part in the point-to-point batches, and NCCL wants the first call to be
        # everyone's)
        self.red.sum(torch.zeros(1, dtype=torch.float64, device=self.device))
        self._scal = torch.ones(3, dtype=torch.float64, device=self.device)
        self.parts = {p: _Part(self, self.local[p]) for p in self.mine}
        # whole control volumes at halo nodes, from their owners
        self.exchange({p: s.Vd for p, s in self.parts.items()})
        for s in self.parts.values():
            s.V = s.Vd.cpu().numpy()
            s._fV_d = s._body_force()
        # the owned unknowns of the partitions held here, in one vector
        off, o = {}, 0
        for p in self.mine:
            off[p] = o
            o += self.parts[p].n_own
        self._off, self.n_owned = off, o
        self._xl = {p: torch.zeros(s.N * 4, dtype=torch.float64, device=self.device)
                    for p, s in self.parts.items()}
        self._union_structure()
        if isinstance(linear, str):
            self.pre = make(linear, **({"rebuild_every": rebuild_every} | (linear_options or {})))
        else:
            self.pre = linear
        self.linear_rtol, self.restart, self.maxiter = linear_rtol, restart, maxiter
        self.linear = type("Linear", (), {"name": f"{getattr(self.pre, 'name', 'amg')}"
                                                  f"x{len(self.local)}"})()
        self._initial_pressure()
        for s in self.parts.values():
            s._apply_fixed()
        self.setup_seconds = time.time() - t0

    # ------------------------------------------------------------ plumbing

    def _union_structure(self):
        """The block-diagonal matrix of the held partitions' owned rows and columns: its
        pattern, and where each partition's blocks come from."""
        ptrs, idxs, self._upos = [torch.zeros(1, dtype=torch.int64, device=self.device)], [], {}
        base_b = 0
        for p in self.mine:
            s = self.parts[p]
            n = s.n_own
            cols = s.pattern[1].to(torch.int64)
            keep = (s._rows < n) & (cols < n)
            pos = torch.nonzero(keep).reshape(-1)
            counts = torch.bincount(s._rows[pos], minlength=n)
            ptrs.append(base_b + torch.cumsum(counts, 0))
            idxs.append((cols[pos] + self._off[p]).to(torch.int32))
            self._upos[p] = (base_b, pos)
            base_b += pos.numel()
        self._uptr = torch.cat(ptrs).contiguous()
        self._uidx = torch.cat(idxs).contiguous()
        self._udata = torch.empty((base_b, 16), dtype=torch.float64, device=self.device)

    def _each(self, fn):
        return {p: fn(s) for p, s in self.parts.items()}

    def lumped_coefficients(self, zid):
        model = self.bcs[zid]["lumped"]
        if self._time is None:
            return model.steady_coefficients(self.t)
        return model.coefficients(self.t, self._time[1])

    def _initial_pressure(self):
        """The boundary pressure level (``B200Solver._initial_pressure``) over the whole mesh,
        given to every partition."""
        inflow = -sum(float(v.sum()) for v in self.bc.sub_flow.values()) / self.fluid.rho
        pairs = {zid: self.lumped_coefficients(zid) for zid in self.bc.lumped_zones()}
        conductance = sum(1.0 / r for _, r in pairs.values() if r > 0)
        weighted, total, levels = 0.0, 0.0, {}
        for zid, (f, S) in self.bc.sub.items():
            if self.bcs[zid]["kind"] != "pressure":
                continue
            if zid in pairs:
                a, r = pairs[zid]
                share = max(inflow, 0.0) / (r * conductance) if r > 0 and conductance > 0 else None
                level = a + share * r if share is not None else a
                levels[zid] = level
            else:
                level = float(self.bc.p_value[self.bc.zone_nodes[zid]].mean())
            area = float((np.linalg.norm(S, axis=2) * (f >= 0)).sum())
            weighted += level * area
            total += area
        for s in self.parts.values():
            if total > 0:
                s.P[:] = weighted / total
            for zid, v in levels.items():
                s._pval_d[s._lumped[zid]["nodes"]] = v

    def _global_scales(self):
        """``[U_ref, p_ref, max |U|]`` over every partition's owned nodes, on the device."""
        parts = []
        for s in self.parts.values():
            n = s.n_own
            parts.append(torch.stack([s.U[:n].abs().max(), s._vel_d.abs().max(),
                                      s.P[:n].max(), -s.P[:n].min()]))
        m = self.red.max(torch.stack(parts).amax(0))
        umax, vmax, pmax, mpmin = m
        rho = self.fluid.rho
        uref = torch.clamp(torch.maximum(umax, vmax), min=1e-30)
        pref = torch.clamp(torch.maximum(pmax + mpmin, rho * uref * uref), min=1e-30)
        self._scal = torch.stack([uref, pref, torch.clamp(umax, min=1e-30)]).contiguous()

    def _owned(self, per_part) -> torch.Tensor:
        """One owned vector (4 unknowns per node) from per-partition local vectors."""
        return torch.cat([per_part[p].reshape(-1)[:4 * self.parts[p].n_own] for p in self.mine])

    # ------------------------------------------------------------ one outer iteration

    def _assemble_all(self):
        """Every held partition's owned rows, scaled, with the global lumped rows; returns the
        operator's pieces, the owned right-hand side and state."""
        pre = {}
        for p, s in self.parts.items():
            pre[p] = B200Solver._stage1(s)
        for k in range(4):
            self.exchange({p: v[k] for p, v in pre.items()})
        for p, s in self.parts.items():
            s._pre = pre[p]
        self._global_scales()
        systems, x0 = {}, {}
        for p, s in self.parts.items():
            A, b, _, x = s._assemble_fused()
            systems[p] = (A, b, s.rs)
            x0[p] = x
        lowrank = self._finish_lumped(systems)
        return systems, lowrank, self._owned({p: v[1] for p, v in systems.items()}), \
            self._owned(x0)

    def _finish_lumped(self, systems) -> list:
        """The lumped outlets' rows (``B200Solver._finish_lumped``) with each zone's flow summed
        over partitions: ``p_j - r Q = a`` at every owned node of the zone, the ``-r w`` part a
        global rank-one term ``[(p, u_dofs, u_values, w_dofs, w_values)]`` per zone."""
        zones = self.bc.lumped_zones()
        if not zones:
            return []
        rho = self.fluid.rho
        pieces = {}
        for p, s in self.parts.items():
            raw, rawb = s.rawdata.view(-1, 4, 4), s.rawb.view(-1, 4)
            pieces[p] = {zid: _zone_flow(raw, rawb, s._lumped[zid], rho) for zid in zones}
        const = torch.stack([sum(pieces[p][zid][2] for p in self.parts) for zid in zones])
        const = self.red.sum(const.reshape(-1).clone())
        terms = []
        for k, zid in enumerate(zones):
            a, r = self.lumped_coefficients(zid)
            sc = min(1.0, rho / r) if r > 0 else 1.0
            zone_terms = []
            for p, s in self.parts.items():
                A, b, rs = systems[p]
                z = s._lumped[zid]
                nodes = z["nodes"]
                s_row = rs.view(-1, 4)[nodes, 3]
                A.data[s._dpos[nodes], 3, 3] = sc * s_row
                b.view(-1, 4)[nodes, 3] = sc * (a + r * const[k]) * s_row
                dofs, weights, _ = pieces[p][zid]
                zone_terms.append((p, 4 * nodes + 3, -sc * r * s_row, dofs, weights))
                z["a"], z["r"], z["sc"] = a, r, sc
            terms.append(zone_terms)
        return terms

    def _operator(self, systems, lowrank):
        """``y = A x`` over the owned unknowns: halo exchange of the local vectors, each
        partition's owned block rows, the global rank-one terms."""
        views = {p: self._xl[p].view(-1, 4) for p in self.mine}

        def matvec(x):
            for p, s in self.parts.items():
                o, n = 4 * self._off[p], 4 * s.n_own
                self._xl[p][:n].copy_(x[o:o + n])
            self.exchange(views)
            y = torch.empty_like(x)
            st = stream_ptr()
            for p, s in self.parts.items():
                A = systems[p][0]
                o = 4 * self._off[p]
                call("zvfv_bsr_spmv", s.n_own, ptr(A.indptr), ptr(A.indices), ptr(A.data),
                     ptr(self._xl[p]), ptr(y[o:o + 4 * s.n_own]), 8, st)
            for zone_terms in lowrank:
                dots = [torch.dot(wv, self._xl[p][wi]) for p, _, _, wi, wv in zone_terms]
                total = self.red.sum(torch.stack(dots).sum().reshape(1))
                for p, ui, uv, _, _ in zone_terms:
                    o = 4 * self._off[p]
                    y.index_add_(0, ui + o, uv * total)
            return y

        return matvec

    def _solve(self, systems, lowrank, b, x0):
        """The global FGMRES, block-Jacobi preconditioned by the AMG of the owned blocks."""
        t = time.time()
        for p, s in self.parts.items():
            base, pos = self._upos[p]
            torch.index_select(systems[p][0].data.view(-1, 16), 0, pos,
                               out=self._udata[base:base + pos.numel()])
        self.pre.setup(BlockMatrix(self._uptr, self._uidx, self._udata.view(-1, 4, 4)))
        ts = time.time() - t
        t = time.time()
        x, it, res, ok = fgmres(self._operator(systems, lowrank), self.pre.vcycle, b, x0,
                                rtol=self.linear_rtol, restart=self.restart,
                                maxiter=self.maxiter, reducer=self.red)
        return x, SolveInfo(it, res, time.time() - t, ts, bool(ok))

    def _update(self, x):
        """Owned values from the solution, with the change statistics reduced over partitions;
        then the halo exchange of ``u`` and ``p`` and the new mass flows."""
        st = stream_ptr()
        stats = []
        for p, s in self.parts.items():
            o, n = 4 * self._off[p], s.n_own
            call("zvfv_update", n, ptr(x[o:o + 4 * n]), ptr(s.U), ptr(s.P), ptr(s._upd_part), st)
            call("zvfv_fold", s._nupd, 5, ptr(s._upd_part), ptr(s._upd_ops), ptr(s._small[8:]),
                 st)
            call("zvfv_fold", s._nfin, 8, ptr(s._fin_part), ptr(s._fin_ops), ptr(s._small), st)
            stats.append(s._small[:13])
        self.exchange({p: s.U for p, s in self.parts.items()})
        self.exchange({p: s.P for p, s in self.parts.items()})
        self.update_mass_flows()
        return torch.stack(stats)

    def update_mass_flows(self):
        grads = {p: s.asm.gradient(s.P, sym=s._sym_d, nvec=0) for p, s in self.parts.items()}
        self.exchange(grads)
        for p, s in self.parts.items():
            s._massflow_from(grads[p])

    def iterate(self) -> dict:
        """One outer iteration over every partition; returns its record."""
        t0 = time.time()
        for s in self.parts.values():
            s.iteration = self.iteration
            s.t = self.t
        systems, lowrank, b, x0 = self._assemble_all()
        t_asm = time.time() - t0
        x, info = self._solve(systems, lowrank, b, x0)
        st = self._update(x)
        # sums (residual squares) add, the rest are maxima; p min is stored negated for MAX
        sums = self.red.sum(st[:, 0:4].sum(0).clone())
        mx = st[:, [4, 5, 6, 7, 8, 9, 10, 12]].amax(0)
        mn = st[:, 11].amin(0)
        mx = self.red.max(torch.cat([mx, -mn.reshape(1)]))
        flows = torch.stack([s._flow_W @ s._mb for s in self.parts.values()]).sum(0) \
            if self.parts else torch.zeros(0)
        flows = self.red.sum(flows.clone())
        small = torch.cat([self._scal, sums, mx, flows]).cpu().numpy()
        uref = small[2]
        nfree = sum(s._nfree for s in self.parts.values())
        nfree = self.red.sum(torch.as_tensor(nfree, dtype=torch.float64,
                                             device=self.device)).cpu().numpy()
        rec = {"iteration": self.iteration + 1}
        for k, name in enumerate(("u", "v", "w", "p")):
            n = nfree[k]
            rec[f"rms_{name}"] = float(np.sqrt(small[3 + k] / n) / uref) if n else 0.0
            rec[f"max_{name}"] = float(small[7 + k] / uref) if n else 0.0
        du_, um, dp_, pmax, pmin = small[11], small[12], small[13], small[14], -small[15]
        du = float(du_) / max(float(um), 1e-300)
        dp = float(dp_) / max(float(pmax - pmin), 1e-300)
        if not (np.isfinite(du) and np.isfinite(dp)):
            raise FloatingPointError(f"non-finite update at outer iteration {self.iteration + 1} "
                                     f"(linear residual {info.residual:.2e})")
        any_part = next(iter(self.parts.values()))
        c = {z: 0.0 for z in any_part._flow_zones}
        for s in self.parts.values():
            for z, v in zip(s._flow_zones, s._flow_c):
                c[z] += v
        cz = self.red.sum(torch.as_tensor([c[z] for z in any_part._flow_zones],
                                          dtype=torch.float64, device=self.device)).cpu().numpy()
        q = {z: float(v) + float(k) for z, v, k in zip(any_part._flow_zones, small[16:], cz)}
        gross = sum(abs(v) for v in q.values()) or 1.0
        rec.update({"du": du, "dp": dp, "linear_iterations": info.iterations,
                    "linear_residual": info.residual, "linear_converged": bool(info.converged),
                    "linear_solver": self.linear.name, "assemble_s": t_asm,
                    "linear_setup_s": info.setup_seconds, "linear_solve_s": info.seconds,
                    "seconds": time.time() - t0, "imbalance": sum(q.values()) / gross,
                    "flows": q})
        self.iteration += 1
        return rec

    # ------------------------------------------------------------ the outer loop

    def _iterate(self, max_iterations, tol, log, hist, residual_target=None):
        for it in range(1, max_iterations + 1):
            rec = self.iterate()
            if self._time is not None:
                rec["t"] = self.t
            hist.append(rec)
            if log:
                log(f"  it {rec['iteration']:4d}  rms u {rec['rms_u']:.2e} p {rec['rms_p']:.2e}  "
                    f"du {rec['du']:.2e} dp {rec['dp']:.2e}  lin {rec['linear_iterations']} "
                    f"({rec['linear_residual']:.1e})  imb {rec['imbalance']:+.1e}  "
                    f"{rec['seconds']:.3f}s")
            rms = max(rec["rms_u"], rec["rms_v"], rec["rms_w"], rec["rms_p"])
            done = (rec["du"] < tol and rec["dp"] < tol) or \
                (residual_target is not None and rms < residual_target)
            if it > 1 and done and rec["linear_converged"]:
                return it, True
        return max_iterations, False

    def solve(self, *, max_iterations: int = 200, tol: float = 1e-10, log=None,
              residual_target: float | None = None) -> dict:
        """Outer iterations to ``tol`` as :meth:`B200Solver.solve`; lumped outlets are then put
        at rest at the converged flows."""
        t0 = time.time()
        hist = []
        _, converged = self._iterate(max_iterations, tol, log, hist, residual_target)
        q = self.patch_flows()
        for zid in self.bc.lumped_zones():
            self.bcs[zid]["lumped"].initialise(q[zid], self.t)
        return {"iterations": len(hist), "converged": converged, "history": hist,
                "seconds": time.time() - t0}

    def solve_transient(self, dt, steps: int | None = None, *, scheme: str = "bdf2",
                        loops: int = 5, tol: float = 1e-8, callback=None, log=None,
                        residual_target: float | None = None) -> dict:
        """As :meth:`B200Solver.solve_transient`, over the partitions
        (``zvcfd/fv/multi.py:496-544``)."""
        if scheme not in BDF:
            raise ValueError(f"scheme {scheme!r}")
        t0 = time.time()
        hist = []

        def level(s):
            return (s.U.clone(), {k: v.clone() for k, v in s.mdot.items()})

        old = {p: [level(s)] for p, s in self.parts.items()}
        dt_prev, all_ok, total = None, True, 0
        with_dt = callback is not None and takes_two(callback)
        for h in time_steps(dt, steps, self.t):
            self.t += h
            self._time = (scheme, h, None, dt_prev)
            self.bc.update(self.t)
            self._bcache.pop("outlet_arrays", None)
            for p, s in self.parts.items():
                s.t = self.t
                s._time = (scheme, h, old[p], dt_prev)
                s._refresh_boundary()
                s._apply_fixed()
            dt_prev = h
            n, ok = self._iterate(loops, tol, log, hist, residual_target)
            all_ok &= ok
            total += n
            q = self.patch_flows()
            for zid in self.bc.lumped_zones():
                self.bcs[zid]["lumped"].advance(q[zid], self.t, h)
            old = {p: [level(s)] + old[p][:1] for p, s in self.parts.items()}
            if callback is not None:
                callback(self, h) if with_dt else callback(self)
        self._time = None
        for s in self.parts.values():
            s._time = None
        return {"iterations": total, "converged": all_ok, "history": hist,
                "seconds": time.time() - t0}

    def initialise(self, U=None, P=None) -> None:
        """Initial fields (arrays over the whole mesh, constants, or functions of ``x`` or
        ``(x, t)``), then that state's linearisation and mass flows."""
        def local(F, s, width):
            shape = (s.N, width) if width else (s.N,)
            if callable(F):
                v = np.asarray(call_value(F, s.mesh.nodes, self.t), float)
                return np.broadcast_to(v, shape)
            v = np.asarray(F, float)
            if v.size == self.N * max(width, 1):
                return v.reshape((self.N, width) if width else (self.N,))[s.lm.nodes]
            return np.broadcast_to(v, shape)

        for s in self.parts.values():
            if U is not None:
                s.U = torch.as_tensor(np.ascontiguousarray(local(U, s, 3)), dtype=torch.float64,
                                      device=self.device)
            if P is not None:
                s.P = torch.as_tensor(np.ascontiguousarray(local(P, s, 0)), dtype=torch.float64,
                                      device=self.device)
            s._apply_fixed()
        self._assemble_all()
        self.update_mass_flows()

    # ------------------------------------------------------------ results

    def zone_flows(self) -> dict:
        """Mass outflow (kg/s) through each zone, summed over the partitions' owned nodes."""
        any_part = next(iter(self.parts.values()))
        zids = any_part._flow_zones
        flows = torch.stack([s._flow_W @ s._mb for s in self.parts.values()]).sum(0)
        flows = self.red.sum(flows.clone()).cpu().numpy()
        c = np.zeros(len(zids))
        for s in self.parts.values():
            c += np.asarray(s._flow_c)
        c = self.red.sum(torch.as_tensor(c, device=self.device)).cpu().numpy()
        return {z: float(v) + float(k) for z, v, k in zip(zids, flows, c)}

    def patch_flows(self) -> dict:
        return {z: v / self.fluid.rho for z, v in self.zone_flows().items()}

    def _gather(self, per_part) -> np.ndarray:
        """A global node array from the partitions' owned rows (summed over processes)."""
        first = next(iter(per_part.values()))
        out = torch.zeros((self.N,) + tuple(first.shape[1:]), dtype=first.dtype,
                          device=first.device)
        for p, v in per_part.items():
            lm = self.local[p]
            out[torch.as_tensor(lm.nodes[:lm.n_own], device=out.device)] = v[:lm.n_own]
        return self.red.sum(out).cpu().numpy()

    def fields(self) -> dict:
        """Node fields on the host, gathered: ``{"U": (N, 3), "P": (N,)}``."""
        return {"U": self._gather({p: s.U for p, s in self.parts.items()}),
                "P": self._gather({p: s.P for p, s in self.parts.items()})}

    def patch_pressures(self) -> dict:
        P = self.fields()["P"]
        out = {}
        for zid, (f, S) in self.bc.sub.items():
            ok = f >= 0
            a = np.linalg.norm(S, axis=2) * ok
            out[zid] = float((P[np.where(ok, f, 0)] * a).sum() / a.sum())
        return out

    def zone_forces(self) -> dict:
        """Force of the fluid on each zone (N) from consistent reactions, from the partitions'
        owned kept rows (:meth:`B200Solver.zone_forces` over the whole mesh)."""
        res = self._gather({p: torch.as_tensor(s._momentum_residual(), device=self.device)
                            for p, s in self.parts.items()})
        return zone_forces(self.bc, res, self.fields()["P"], stokes=self.stokes,
                           lumped=self.bc.lumped_zones())

    def wall_shear(self, method: str = "gradient"):
        """``(global wall nodes, tau (n, 3))`` gathered from the partitions' owned wall nodes
        (:meth:`B200Solver.wall_shear`)."""
        if method == "reaction":
            from zvcfd_b200.forces import wall_shear_reaction

            res = self._gather({p: torch.as_tensor(s._momentum_residual(), device=self.device)
                                for p, s in self.parts.items()})
            return wall_shear_reaction(self.bc, res, self.fields()["P"], stokes=self.stokes)
        nodes, taus = [], []
        for p, s in self.parts.items():
            n, tau = s.wall_shear(method)
            keep = n < s.n_own
            nodes.append(s.lm.nodes[n[keep]])
            taus.append(tau[keep])
        if self.red.world > 1:
            got = [None] * self.red.world
            dist.all_gather_object(got, (nodes, taus), group=self.red.group)
            nodes = [a for g in got for a in g[0]]
            taus = [a for g in got for a in g[1]]
        nodes, tau = np.concatenate(nodes), np.concatenate(taus)
        order = np.argsort(nodes)
        return nodes[order], tau[order]

    def close(self):
        if hasattr(self.pre, "close"):
            self.pre.close()


__all__ = ["B200MultiSolver", "HaloExchange", "PartBoundary", "Reducer", "deal", "fgmres"]
