"""WSS time statistics against the reference's own (CPU)."""

import numpy as np
import pytest
import torch

from fixtures import load
from zvcfd_b200.wss import WallShearStats


@pytest.mark.parametrize("as_tensor", [False, True])
def test_wss_statistics_match_reference(as_tensor):
    g = load("wss")
    st = WallShearStats(g["tau"].shape[1])
    for t, tau in zip(g["t"], g["tau"]):
        st.add(float(t), torch.as_tensor(tau) if as_tensor else tau)
    r = st.results()
    np.testing.assert_allclose(r["tawss"], g["tawss"], rtol=1e-14, atol=1e-300)
    np.testing.assert_allclose(r["osi"], g["osi"], rtol=1e-13, atol=1e-15)
    np.testing.assert_allclose(r["rrt"], g["rrt"], rtol=1e-11)
    assert r["osi"][0] == 0.5 and r["rrt"][0] == g["rrt"][0]      # never sheared


def test_wss_statistics_need_two_samples_and_the_right_shape():
    st = WallShearStats(4)
    st.add(0.0, np.zeros((4, 3)))
    with pytest.raises(ValueError):
        st.results()
    with pytest.raises(ValueError):
        st.add(1.0, np.zeros((5, 3)))
