"""Host side of the partitioned solve (``zvcfd_b200.multi``) on the CPU.

The device path of :class:`~zvcfd_b200.multi.B200MultiSolver` needs a GPU; what it is built
from is device-agnostic and runs here on CPU tensors:

- the halo exchange, in one process holding every partition and over two gloo ranks holding
  two partitions each (point-to-point batches): afterwards every partition's rows equal the
  global field at its local nodes;
- the distributed FGMRES, with an operator that exchanges halos and multiplies each
  partition's owned rows and a block-Jacobi preconditioner (each partition's owned block
  inverted exactly): one process and two gloo ranks reach the direct solution of a
  non-symmetric system on the golden pipe's node graph, and agree with each other;
- the partition's view of the boundary: node arrays are the global ones at local nodes, and
  the zone-flow weights and known inlet flows summed over partitions equal the global ones.
"""

import os
import socket

import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as spla
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from fixtures import load, mesh_of, pipe_bcs
from zvcfd_b200.boundary import Boundary
from zvcfd_b200.multi import HaloExchange, PartBoundary, Reducer, deal, fgmres
from zvcfd_b200.partition import halo_plan, local_meshes, morton_owner


def _case(parts=4):
    g = load("pipe_reference_tube")
    m = mesh_of(g)
    owner = morton_owner(m.nodes, parts)
    local = local_meshes(m, owner)
    return g, m, owner, local, halo_plan(local, owner)


def _system(m):
    """A non-symmetric diagonally dominant operator on the mesh's node graph (convection along
    z plus diffusion), and a right-hand side."""
    rows, cols = [], []
    for e in m.elements.values():
        n = e.shape[1]
        a, c = np.meshgrid(np.arange(n), np.arange(n), indexing="ij")
        rows.append(e[:, a.ravel()].ravel())
        cols.append(e[:, c.ravel()].ravel())
    rows, cols = np.concatenate(rows), np.concatenate(cols)
    keep = rows != cols
    key = np.unique(rows[keep] * m.n_nodes + cols[keep])
    i, j = key // m.n_nodes, key % m.n_nodes
    dz = m.nodes[j, 2] - m.nodes[i, 2]
    v = -1.0 - 0.4 * np.sign(dz)
    A = sp.csr_matrix((v, (i, j)), shape=(m.n_nodes, m.n_nodes))
    A = A + sp.diags(np.asarray(abs(A).sum(1)).ravel() + 0.05)
    b = np.random.default_rng(0).normal(size=m.n_nodes)
    return A.tocsr(), b


def _solve_parts(A, b, local, plan, rank_of, red):
    """Distributed FGMRES on the partitions this process holds (1 unknown per node)."""
    mine = [p for p in range(len(local)) if rank_of[p] == red.rank]
    ex = HaloExchange(plan, rank_of, red, "cpu")
    off, o = {}, 0
    for p in mine:
        off[p] = o
        o += local[p].n_own
    ops, inv, xl = {}, {}, {}
    for p in mine:
        lm = local[p]
        own = lm.nodes[:lm.n_own]
        ops[p] = torch.as_tensor(A[own][:, lm.nodes].toarray())
        inv[p] = torch.as_tensor(np.linalg.inv(A[own][:, own].toarray()))
        xl[p] = torch.zeros(len(lm.nodes), dtype=torch.float64)

    def matvec(x):
        for p in mine:
            xl[p][:local[p].n_own] = x[off[p]:off[p] + local[p].n_own]
        ex(xl)
        return torch.cat([ops[p] @ xl[p] for p in mine])

    def precond(r):
        return torch.cat([inv[p] @ r[off[p]:off[p] + local[p].n_own] for p in mine])

    bl = torch.as_tensor(np.concatenate([b[local[p].nodes[:local[p].n_own]] for p in mine]))
    x, it, res, ok = fgmres(matvec, precond, bl, torch.zeros_like(bl), rtol=1e-10, restart=8,
                            maxiter=400, reducer=red)
    out = np.zeros(len(b))
    for p in mine:
        out[local[p].nodes[:local[p].n_own]] = x[off[p]:off[p] + local[p].n_own].numpy()
    return out, it, res, ok


def test_deal_keeps_runs_and_feeds_every_rank():
    np.testing.assert_array_equal(deal(4, 2), [0, 0, 1, 1])
    np.testing.assert_array_equal(deal(5, 2), [0, 0, 0, 1, 1])
    np.testing.assert_array_equal(deal(3, 1), [0, 0, 0])
    for n, w in [(7, 3), (8, 8), (9, 4)]:
        r = deal(n, w)
        assert (np.diff(r) >= 0).all() and np.unique(r).size == w
    with pytest.raises(ValueError):
        deal(2, 3)


def test_exchange_in_one_process_restores_the_global_field():
    g, m, owner, local, plan = _case(4)
    field = np.random.default_rng(1).normal(size=(m.n_nodes, 3, 3))
    arrays = {}
    for p, lm in enumerate(local):
        a = torch.as_tensor(field[lm.nodes]).clone()
        a[lm.n_own:] = -7.0                                # stale halo
        arrays[p] = a
    ex = HaloExchange(plan, deal(4, 1), Reducer(), "cpu")
    assert not ex.crosses_processes
    ex(arrays)
    for p, lm in enumerate(local):
        np.testing.assert_array_equal(arrays[p].numpy(), field[lm.nodes])


def test_fgmres_of_the_partitions_reaches_the_direct_solution():
    g, m, owner, local, plan = _case(3)
    A, b = _system(m)
    want = spla.spsolve(A.tocsc(), b)
    x, it, res, ok = _solve_parts(A, b, local, plan, deal(3, 1), Reducer())
    assert ok and res <= 1e-10
    assert np.abs(x - want).max() <= 1e-8 * np.abs(want).max()
    # restarted cycles and the round-off floor: a second solve from the answer stops at once
    x2, it2, _, ok2 = _solve_parts(A, A @ want, local, plan, deal(3, 1), Reducer())
    assert ok2 and np.abs(x2 - want).max() <= 1e-8 * np.abs(want).max()


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        torch.set_num_threads(1)
        g, m, owner, local, plan = _case(4)
        red = Reducer(dist.group.WORLD)
        rank_of = deal(4, world)
        ex = HaloExchange(plan, rank_of, red, "cpu")
        field = np.random.default_rng(1).normal(size=(m.n_nodes, 4))
        arrays = {}
        for p, lm in enumerate(local):
            if rank_of[p] == rank:
                a = torch.as_tensor(field[lm.nodes]).clone()
                a[lm.n_own:] = np.nan
                arrays[p] = a
        ex(arrays)
        exchanged = all(np.array_equal(arrays[p].numpy(), field[local[p].nodes])
                        for p in arrays)
        A, b = _system(m)
        x, it, res, ok = _solve_parts(A, b, local, plan, rank_of, red)
        xs = torch.as_tensor(x)
        red.sum(xs)
        out[rank] = (ex.crosses_processes, exchanged, xs.numpy(), it, bool(ok))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_exchange_halos_and_solve_together():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    out = mp.get_context("spawn").Manager().dict()
    mp.start_processes(_rank, args=(2, port, out), nprocs=2, join=True, start_method="spawn")
    g, m, owner, local, plan = _case(4)
    A, b = _system(m)
    want = spla.spsolve(A.tocsc(), b)
    one, it1, _, _ = _solve_parts(A, b, local, plan, deal(4, 1), Reducer())
    for rank in (0, 1):
        crosses, exchanged, x, it, ok = out[rank]
        assert crosses and exchanged and ok
        assert np.abs(x - want).max() <= 1e-8 * np.abs(want).max()
        # the same partitions and recurrences in one process or two: equal to round-off
        assert it == it1
        np.testing.assert_allclose(x, one, rtol=0, atol=1e-12 * np.abs(want).max())


def test_partition_boundary_sums_to_the_global_boundary():
    g, m, owner, local, plan = _case(4)
    bcs = pipe_bcs("pipe_reference_tube", g, m)
    G = Boundary(m, bcs, float(g["rho"]), mu=float(g["mu"]))
    cache = {}
    views = [PartBoundary(G, lm, cache) for lm in local]
    zids, W, c = G.flow_weights()
    W_sum = np.zeros_like(W)
    c_sum = np.zeros_like(c)
    force, a_out, wc, wo, ws = G.outlet_arrays()
    for lm, v in zip(local, views):
        np.testing.assert_array_equal(v.vel_fixed_comp, G.vel_fixed_comp[lm.nodes])
        np.testing.assert_array_equal(v.vel_value, G.vel_value[lm.nodes])
        np.testing.assert_array_equal(v.p_fixed, G.p_fixed[lm.nodes])
        np.testing.assert_array_equal(v.inflow, G.inflow[lm.nodes])
        for got, want in zip(v.outlet_arrays(), (force, a_out, wc, wo, ws)):
            np.testing.assert_array_equal(got, want[lm.nodes])
        z2, Wp, cp = v.flow_weights()
        assert z2 == zids
        assert (Wp[:, lm.n_own:] == 0).all()
        np.add.at(W_sum.T, lm.nodes, Wp.T)
        c_sum += cp
        for zid, (f, S) in v.sub.items():                 # faces held: those touching owned
            gf = m.zones[zid].faces[lm.faces[zid]]
            np.testing.assert_array_equal(np.where(f >= 0, lm.nodes[np.where(f >= 0, f, 0)],
                                                   -1), gf)
    np.testing.assert_allclose(W_sum, W, atol=1e-15)
    np.testing.assert_allclose(c_sum, c, rtol=1e-12, atol=1e-15 * np.abs(c).max())


def test_fgmres_edge_cases():
    """The stopping rules shared with the device FGMRES: nothing to do, a lucky breakdown,
    the step budget, restarts."""
    rng = np.random.default_rng(4)
    ident = lambda v: v.clone()                                    # noqa: E731
    z = torch.zeros(12, dtype=torch.float64)
    x, it, res, ok = fgmres(ident, ident, z, z, rtol=1e-8)
    assert it == 0 and ok and res == 0.0 and not x.any()           # b = 0, x0 = 0
    b = torch.as_tensor(rng.normal(size=12))
    x, it, res, ok = fgmres(ident, ident, b, z, rtol=1e-12)
    assert it == 1 and ok                                          # exact after one step
    np.testing.assert_allclose(x.numpy(), b.numpy(), rtol=0, atol=1e-15 * b.abs().max().item())
    M = torch.as_tensor(np.diag(np.linspace(1.0, 100.0, 40)) + 0.3 * np.eye(40, k=1))
    b = torch.as_tensor(rng.normal(size=40))
    x, it, res, ok = fgmres(lambda v: M @ v, ident, b, torch.zeros(40, dtype=torch.float64),
                            rtol=1e-10, maxiter=3)
    assert it == 3 and not ok and res > 1e-10
    x, it, res, ok = fgmres(lambda v: M @ v, ident, b, torch.zeros(40, dtype=torch.float64),
                            rtol=1e-10, restart=5, maxiter=400)
    assert ok and it > 5 and res <= 1.01e-10
    want = np.linalg.solve(M.numpy(), b.numpy())
    assert np.abs(x.numpy() - want).max() <= 1e-8 * np.abs(want).max()


@pytest.mark.parametrize("extra", [{"profile": "average"}, {"opening": True}])
def test_partitioned_solver_refuses_zones_that_couple_partitions(extra):
    """An average-pressure zone's mean couples it globally, and an opening's halo nodes would
    be eliminated with stale values: the partitioned solver refuses both before it sets up."""
    from zvcfd_b200.fluid import Fluid
    from zvcfd_b200.multi import B200MultiSolver

    g, m, owner, local, plan = _case(2)
    bcs = pipe_bcs("pipe_reference_tube", g, m)
    z = {zz.name: k for k, zz in m.zones.items()}
    bcs[z["outlet"]] = {"kind": "pressure", "value": 0.0, **extra}
    with pytest.raises(NotImplementedError, match="one partition"):
        B200MultiSolver(m, Fluid(1.0, 0.2), bcs, parts=2)
