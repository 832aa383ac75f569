"""The partitioner (``zvcfd_b200.partition``) against the reference's own partitions.

``tests/golden/partition.npz`` holds the reference's owners, local meshes and halo plans
(``zvcfd/fv/partition.py``) for the mixed tube of its partition test
(``tests/test_fv_multi.py:40-43``) and for the golden pipe at 2, 3 and 4 parts and at a given
chunk edge; every array must be equal. The properties the reference's test checks are held
too: whole chunks, node balance, complete control volumes of owned nodes, and halo plans that
move each halo node's value from its owner.
"""

import numpy as np
import pytest

from fixtures import load, mesh_of
from zvcfd_b200.partition import (default_chunk, halo_plan, local_meshes, morton_key,
                                  morton_owner, partition_report)

G = load("partition")


def _mesh(name):
    pre = f"{name}_"
    return mesh_of({k[len(pre):]: v for k, v in G.items() if k.startswith(pre)})


def _runs():
    for i in range(int(G["runs"])):
        n, chunk = G[f"run{i}_meta"]
        yield i, str(G[f"run{i}_mesh"]), int(n), None if chunk < 0 else float(chunk)


@pytest.mark.parametrize("run", [r[0] for r in _runs()])
def test_partitions_equal_the_reference(run):
    i, name, n, chunk = list(_runs())[run]
    m = _mesh(name)
    owner = morton_owner(m.nodes, n, chunk)
    np.testing.assert_array_equal(owner, G[f"run{i}_owner"])
    parts = local_meshes(m, owner)
    plans = halo_plan(parts, owner)
    assert len(parts) == n
    for p, (lm, plan) in enumerate(zip(parts, plans)):
        tag = f"run{i}_p{p}"
        np.testing.assert_array_equal(lm.nodes, G[f"{tag}_nodes"])
        assert lm.n_own == int(G[f"{tag}_n_own"])
        for k, sel in lm.elements.items():
            np.testing.assert_array_equal(sel, G.get(f"{tag}_elem_{k}", np.zeros(0, np.int64)))
        for z, sel in lm.faces.items():
            np.testing.assert_array_equal(sel, G[f"{tag}_face_{z}"])
        np.testing.assert_array_equal([q for q, _, _ in plan], G[f"{tag}_plan"])
        for q, send, recv in plan:
            np.testing.assert_array_equal(send, G[f"{tag}_send_{q}"])
            np.testing.assert_array_equal(recv, G[f"{tag}_recv_{q}"])


def test_morton_key_interleaves_bits():
    rng = np.random.default_rng(3)
    ijk = rng.integers(0, 1 << 21, size=(200, 3))
    want = np.zeros(200, np.uint64)
    for b in range(21):
        for a in range(3):
            bit = (ijk[:, a].astype(np.uint64) >> np.uint64(b)) & np.uint64(1)
            want |= bit << np.uint64(3 * b + a)
    np.testing.assert_array_equal(morton_key(ijk), want)


def test_whole_chunks_balance_and_complete_control_volumes():
    m = _mesh("mixed")
    owner = morton_owner(m.nodes, 4)
    counts = np.bincount(owner)
    assert counts.max() / counts.mean() < 1.25
    chunk = default_chunk(m.nodes, 4)
    cell = np.floor((m.nodes - m.nodes.min(0)) / chunk).astype(np.int64)
    key = morton_key(cell)
    for k in np.unique(key):                          # every chunk has one owner
        assert np.unique(owner[key == k]).size == 1
    parts = local_meshes(m, owner)
    plans = halo_plan(parts, owner)
    assert sum(p.n_own for p in parts) == m.n_nodes
    for lm, plan in zip(parts, plans):
        own = set(lm.nodes[:lm.n_own].tolist())
        # every element with an owned node is held, and no other
        for k, e in m.elements.items():
            touching = np.flatnonzero(np.isin(e, list(own)).any(1))
            np.testing.assert_array_equal(lm.elements.get(k, np.zeros(0, np.int64)), touching)
        # the plan fills every halo row once, from the node's owner
        filled = np.zeros(lm.n_halo, int)
        for q, send, recv in plan:
            np.testing.assert_array_equal(parts[q].nodes[send], lm.nodes[recv])
            assert (owner[lm.nodes[recv]] == q).all() and (send < parts[q].n_own).all()
            filled[recv - lm.n_own] += 1
        assert (filled == 1).all()
    rep = partition_report(parts)
    assert rep["parts"] == 4 and rep["imbalance"] < 0.25 and min(rep["overlap"]) > 0


def test_one_part_is_the_whole_mesh():
    m = _mesh("pipe")
    owner = morton_owner(m.nodes, 1)
    (lm,) = local_meshes(m, owner)
    np.testing.assert_array_equal(lm.nodes, np.arange(m.n_nodes))
    assert lm.n_own == m.n_nodes and lm.n_halo == 0
    assert halo_plan([lm], owner) == [[]]
    for k in m.elements:
        np.testing.assert_array_equal(lm.mesh.elements[k], m.elements[k])


def test_too_many_parts_for_whole_chunks_is_an_error():
    m = _mesh("pipe")
    with pytest.raises(ValueError, match="whole chunks"):
        morton_owner(m.nodes, 3, chunk=100.0)
    with pytest.raises(ValueError):
        morton_owner(m.nodes, 0)
