"""The element colouring against the reference's own.

``tests/golden/colour.npz`` holds the colours of the reference's device colouring
``gpu_colour`` (``zvcfd/fv/fast.py:84-130``: SplitMix64 keys, Jones-Plassmann claim and
first-fit pick rounds, masks doubled when they overflow), run in this container with its kernel
source compiled for the CPU (the results do not depend on thread order). The oracle's
restatement (``oracle.pattern.colour``) must give the same colour to every element, on the
meshes the device colouring is checked against the oracle with on a B200
(``tests/test_gpu_assembler.py``): so the device colouring is pinned to the reference's.
"""

import numpy as np
import pytest

from fixtures import load
from oracle import pattern as opat

G = load("colour")


def _box_tets(n):
    """Five tetrahedra per cube of an n^3 grid of cubes (the reference's
    ``tests/test_fv_fast.py:59-69`` mesh)."""
    i, j, k = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")

    def v(a, b, c):
        return ((i + a) * (n + 1) + (j + b)) * (n + 1) + (k + c)

    c = [v(0, 0, 0), v(1, 0, 0), v(1, 1, 0), v(0, 1, 0), v(0, 0, 1), v(1, 0, 1), v(1, 1, 1),
         v(0, 1, 1)]
    tets = [(0, 1, 3, 4), (1, 2, 3, 6), (1, 4, 5, 6), (3, 4, 6, 7), (1, 3, 4, 6)]
    return np.stack([np.stack([c[t].ravel() for t in tet], 1) for tet in tets], 0) \
        .reshape(-1, 4).astype(np.int32), (n + 1) ** 3


@pytest.mark.parametrize("case", [str(c) for c in G["cases"]])
def test_oracle_colouring_equals_the_reference(case):
    n_nodes, words = (int(v) for v in G[f"{case}_meta"])
    conn = _box_tets(16)[0] if case == "box16" else G[f"{case}_conn"]
    want = G[f"{case}_colour"]
    got = opat.colour(conn, n_nodes)
    np.testing.assert_array_equal(got, want)
    opat.check_colouring(conn, got)
    if case == "fan":                         # one mask word, widened twice by the reference
        assert words == 1 and len(np.unique(want)) == 200
