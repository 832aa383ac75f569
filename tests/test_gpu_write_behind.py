"""Snapshots written behind the device (``zvcfd_b200.snapshots.SnapshotWriter``) hold each
step's fields: a BDF2 march of the golden pulsatile pipe with the writer as its callback, every
second step, then every group read back against the state the solver had at that step (FP64
kept, and the default ``float32`` cast); the partitioned solver's gathered fields go the same
way."""

import numpy as np
import pytest

from fixtures import fluid_of, load, mesh_of, transient_bcs

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("dtype", [None, "float32"])
def test_snapshots_hold_each_steps_fields(tmp_path, dtype):
    from zvcfd_b200.snapshots import SnapshotWriter, read_node_fields
    from zvcfd_b200.solver import B200Solver

    g = load("transient_pipe")
    m = mesh_of(g)
    s = B200Solver(m, fluid_of(g), transient_bcs(g, m), advection=1.0)
    seen = {}
    writer = SnapshotWriter(tmp_path, every=2, wss=True, dtype=dtype)

    def both(solver, dt):
        writer(solver, dt)
        seen[writer.step] = (solver.fields(), solver.t)

    s.solve_transient(0.05, 6, loops=6, tol=1e-10, callback=both)
    writer.close()
    assert len(writer.paths) == 3
    nodes, _ = s.wall_shear()
    for p in writer.paths:
        f, meta = read_node_fields(p)
        want, t = seen[meta["step"]]
        assert meta["nodes"] == m.n_nodes and meta["time_s"] == pytest.approx(t)
        cast = (lambda a: a) if dtype is None else (lambda a: a.astype(np.float32))
        np.testing.assert_array_equal(f["velocity"], cast(want["U"]))
        np.testing.assert_array_equal(f["pressure"], cast(want["P"]))
        np.testing.assert_array_equal(f["wall_nodes"], nodes)
    s.close()


def test_partitioned_solver_snapshots(tmp_path):
    from zvcfd_b200.multi import B200MultiSolver
    from zvcfd_b200.snapshots import SnapshotWriter, read_node_fields

    g = load("transient_pipe")
    m = mesh_of(g)
    s = B200MultiSolver(m, fluid_of(g), transient_bcs(g, m), parts=2, advection=1.0)
    with SnapshotWriter(tmp_path, dtype=None) as w:
        s.solve_transient(0.05, 2, loops=6, tol=1e-10, callback=w)
    f, meta = read_node_fields(w.paths[-1])
    np.testing.assert_array_equal(f["velocity"], s.fields()["U"])
    assert meta["step"] == 2
    s.close()
