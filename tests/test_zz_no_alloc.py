"""The allocation-free state update (zvfv_update_noalloc) against the allocating pair.

zvfv_update_noalloc is for callers that cannot allocate device memory (a host program under
a fixed memory budget, an outer loop that must not call cudaMalloc/cudaFree between steps):
its partial rows live in a static array of the library instead of a caller buffer. On the
same inputs it must give what zvfv_update + zvfv_fold (ops max, max, max, min, max) give, bit
for bit, on two calls in a row (the second sees the first call's leftovers in the shared
array), and it must refuse sizes beyond that array. This file is collected last.
"""

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

LIMIT = 1 << 24          # nodes the static scratch covers (65,536 CTAs of 256)


def _allocating(n, x, U, P):
    from zvcfd_b200._lib import call, lib, ptr, stream_ptr

    rows = int(lib.zvfv_update_partials(n))
    part = torch.empty(rows * 5, dtype=torch.float64, device="cuda")
    ops = torch.tensor([1, 1, 1, 2, 1], dtype=torch.int32, device="cuda")
    out = torch.empty(5, dtype=torch.float64, device="cuda")
    call("zvfv_update", n, ptr(x), ptr(U), ptr(P), ptr(part), stream_ptr())
    call("zvfv_fold", rows, 5, ptr(part), ptr(ops), ptr(out), stream_ptr())
    return out


def _noalloc(n, x, U, P):
    from zvcfd_b200._lib import call, ptr, stream_ptr

    out = torch.full((5,), np.nan, dtype=torch.float64, device="cuda")
    call("zvfv_update_noalloc", n, ptr(x), ptr(U), ptr(P), ptr(out), stream_ptr())
    return out


def test_noalloc_update_matches_allocating_update_twice():
    g = torch.Generator(device="cuda").manual_seed(7)
    for n in (300_001, 1_000):          # the smaller second call leaves rows of the first behind
        U0 = torch.randn(n, 3, dtype=torch.float64, device="cuda", generator=g)
        P0 = torch.randn(n, dtype=torch.float64, device="cuda", generator=g)
        x = torch.randn(n * 4, dtype=torch.float64, device="cuda", generator=g)
        Ua, Pa, Ub, Pb = U0.clone(), P0.clone(), U0.clone(), P0.clone()
        ref = _allocating(n, x, Ua, Pa)
        got = _noalloc(n, x, Ub, Pb)
        torch.cuda.synchronize()
        assert torch.equal(got, ref), (got, ref)
        assert torch.equal(Ub, Ua) and torch.equal(Pb, Pa)
        xv = x.view(n, 4).cpu().numpy()
        np.testing.assert_array_equal(got.cpu().numpy(), [
            np.abs(xv[:, :3] - U0.cpu().numpy()).max(), np.abs(xv[:, :3]).max(),
            np.abs(xv[:, 3] - P0.cpu().numpy()).max(), xv[:, 3].min(), xv[:, 3].max()])


def test_noalloc_update_rejects_sizes_beyond_its_scratch():
    from zvcfd_b200._lib import lib

    out = torch.zeros(5, dtype=torch.float64, device="cuda")
    dummy = torch.zeros(4, dtype=torch.float64, device="cuda")
    p = dummy.data_ptr()
    for n in (LIMIT + 1, 0):
        rc = lib.zvfv_update_noalloc(n, p, p, p, out.data_ptr(), None)
        assert rc == 1
        assert b"static scratch" in lib.zvfv_last_error()
    torch.cuda.synchronize()
    assert torch.count_nonzero(out) == 0
