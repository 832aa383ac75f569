"""The block-CSR SpMV (FP64 and FP32, every lanes-per-row setting) against the oracle's."""

import numpy as np
import pytest
import torch

from oracle.linear import bsr_matvec
from oracle.pattern import node_graph

pytestmark = pytest.mark.gpu


def _system(seed=0):
    from zvcfd_b200.mesh import curved_tube

    m = curved_tube(1.0, 5.0, n_core=6, n_ring=4, n_axial=20, layers=2)
    indptr, indices = node_graph(m)
    rng = np.random.default_rng(seed)
    data = rng.normal(size=(len(indices), 4, 4))
    x = rng.normal(size=(m.n_nodes, 4))
    return m.n_nodes, indptr, indices, data, x


@pytest.mark.parametrize("lanes", [4, 8, 16, 32])
def test_spmv_fp64(lanes):
    from zvcfd_b200._lib import call, ptr, stream_ptr

    n, indptr, indices, data, x = _system()
    d = lambda a, t: torch.as_tensor(np.ascontiguousarray(a), dtype=t, device="cuda")  # noqa: E731
    ip, ix, dd, xx = d(indptr, torch.int64), d(indices, torch.int32), d(data, torch.float64), \
        d(x, torch.float64)
    y = torch.empty_like(xx)
    call("zvfv_bsr_spmv", n, ip.data_ptr(), ix.data_ptr(), dd.data_ptr(), xx.data_ptr(),
         y.data_ptr(), lanes, stream_ptr())
    ref = bsr_matvec(indptr, indices, data, x)
    np.testing.assert_allclose(y.cpu().numpy().reshape(-1), ref, rtol=1e-13, atol=1e-12)
    b = d(np.ones_like(x), torch.float64)
    r = torch.empty_like(xx)
    call("zvfv_bsr_residual", n, ip.data_ptr(), ix.data_ptr(), dd.data_ptr(), xx.data_ptr(),
         b.data_ptr(), r.data_ptr(), lanes, stream_ptr())
    np.testing.assert_allclose(r.cpu().numpy().reshape(-1), 1.0 - ref, rtol=1e-13, atol=1e-12)
    del ptr


@pytest.mark.parametrize("lanes", [4, 8, 16, 32])
def test_spmv_fp32(lanes):
    from zvcfd_b200._lib import call, stream_ptr

    n, indptr, indices, data, x = _system(1)
    d = lambda a, t: torch.as_tensor(np.ascontiguousarray(a), dtype=t, device="cuda")  # noqa: E731
    ip, ix = d(indptr, torch.int64), d(indices, torch.int32)
    dd, xx = d(data, torch.float32), d(x, torch.float32)
    y = torch.empty_like(xx)
    call("zvfv_bsr_spmv_f32", n, ip.data_ptr(), ix.data_ptr(), dd.data_ptr(), xx.data_ptr(),
         y.data_ptr(), lanes, stream_ptr())
    ref = bsr_matvec(indptr, indices, data.astype(np.float32).astype(np.float64),
                     x.astype(np.float32).astype(np.float64))
    scale = np.abs(data).max() * np.abs(x).max() * 27
    np.testing.assert_allclose(y.cpu().numpy().reshape(-1), ref, atol=1e-6 * scale)
