"""The drop-in adapters over foreign device arrays.

``ReferenceLinear`` and ``ReferenceAssembler`` are what a maintainer binds into the reference
(``zvcfd.fv.linear.make("b200")`` and ``kernels="b200"``). The reference hands them CuPy
arrays; CuPy is not installed here, so the caller's arrays are stood in for by objects that
expose nothing but ``__cuda_array_interface__`` (version 3), the protocol CuPy arrays carry.
Every method must view them without a copy, accept the reference's dtypes (int32 rank-one
dofs, int64 row pointers), return the reference's shapes and ``SolveInfo`` contract, and give
the same numbers as the torch path it wraps.
"""

import numpy as np
import pytest
import torch

from fixtures import fluid_of, load, mesh_of, pipe_bcs

pytestmark = pytest.mark.gpu


class Foreign:
    """A device array known only through ``__cuda_array_interface__`` (kept alive by ``base``)."""

    def __init__(self, t: torch.Tensor):
        self.base = t.contiguous()
        self.__cuda_array_interface__ = {
            "shape": tuple(self.base.shape),
            "typestr": {torch.float64: "<f8", torch.float32: "<f4", torch.int32: "<i4",
                        torch.int64: "<i8"}[self.base.dtype],
            "data": (self.base.data_ptr(), False),
            "version": 3,
            "strides": None,
        }


class RefBlockMatrix:
    """The reference's BlockMatrix fields (``zvcfd/fv/linear.py:75-135``) over foreign arrays."""

    def __init__(self, indptr, indices, data, lowrank=()):
        self.indptr, self.indices, self.data = indptr, indices, data
        self.lowrank = list(lowrank)


def _solver(name="pipe_tet_si", iterations=3):
    from zvcfd_b200.solver import B200Solver

    g = load(name)
    m = mesh_of(g)
    s = B200Solver(m, fluid_of(g), pipe_bcs(name, g, m), advection=1.0)
    for _ in range(iterations):
        s.iterate()
    return g, m, s


def test_reference_linear_solves_foreign_arrays_with_rank_one_terms():
    from zvcfd_b200.interop import ReferenceLinear
    from zvcfd_b200.linear import B200AMG, BlockMatrix, SolveInfo

    _, _, s = _solver()
    A, b, _, x0 = s._assemble_fused()
    b = b.reshape(-1).clone()
    n4 = b.numel()
    # a rank-one term u w^T coupling the last pressure dof to a few others, as the lumped rows
    u_dofs = torch.tensor([n4 - 1], dtype=torch.int32, device="cuda")
    u_vals = torch.tensor([1e-3], dtype=torch.float64, device="cuda")
    w_dofs = torch.arange(3, n4, 97, dtype=torch.int32, device="cuda")
    w_vals = torch.linspace(0.5, 1.5, w_dofs.numel(), dtype=torch.float64, device="cuda")
    RA = RefBlockMatrix(Foreign(A.indptr), Foreign(A.indices), Foreign(A.data.reshape(-1, 4, 4)),
                        [(Foreign(u_dofs), Foreign(u_vals), Foreign(w_dofs), Foreign(w_vals))])
    ref = ReferenceLinear("b200", rtol=1e-8)
    x, info = ref.solve(RA, Foreign(b), Foreign(x0.clone()), rtol=1e-8)
    assert isinstance(info, SolveInfo)
    assert info.converged and info.iterations > 0 and info.residual <= 1e-8 * 1.01
    assert info.seconds >= 0 and info.setup_seconds >= 0
    assert x.shape == (n4,) and x.dtype == torch.float64 and x.is_cuda
    # the torch path on the same matrix gives the same iterate, bit for bit
    low = [(u_dofs.long(), u_vals, w_dofs.long(), w_vals)]
    own = B200AMG(rtol=1e-8)
    x2, info2 = own.solve(BlockMatrix(A.indptr, A.indices, A.data.reshape(-1, 4, 4), low), b,
                          x0.clone(), rtol=1e-8)
    assert info2.iterations == info.iterations
    assert torch.equal(x, x2)
    # the residual counts the rank-one term
    M = BlockMatrix(A.indptr, A.indices, A.data.reshape(-1, 4, 4), low)
    Ax, Ax0 = M.matvec(x), M.matvec(x0)
    assert torch.linalg.norm(b - Ax) <= 1.01e-8 * torch.linalg.norm(b - Ax0) + \
        1e-13 * torch.linalg.norm(b)
    # the V-cycle entry point the reference's multi-GPU solver calls
    z = ref.vcycle(Foreign(b))
    assert z.shape == (n4,) and torch.isfinite(z).all()
    assert ref.active == "b200" and ref.switches == []
    ref.close()
    own.close()
    s.close()


def test_reference_assembler_methods_over_foreign_arrays():
    from zvcfd_b200.assembler import B200Assembler
    from zvcfd_b200.interop import ReferenceAssembler

    g = load("curved_cy")
    m = mesh_of(g)
    fl = fluid_of(g)
    kw = dict(rho=fl.rho, mu=fl.mu, rheology=fl.viscosity, transpose=True)
    ra, ta = ReferenceAssembler(m, **kw), B200Assembler(m, **kw)
    N = m.n_nodes
    rng = np.random.default_rng(4)
    U = torch.as_tensor(rng.normal(size=(N, 3)) * 1e-2, device="cuda")
    P = torch.as_tensor(rng.normal(size=N), device="cuda")
    # pattern, statics and the element-order <-> slot-order maps
    assert ra.pattern[0].dtype == torch.int64 and ra.pattern[1].dtype == torch.int32
    assert torch.equal(ra.node_volume, ta.node_volume) and torch.equal(ra.gop, ta.gop)
    mdot_elem = {k: torch.as_tensor(rng.normal(size=(len(e), ra.kinds[i].nip)) * 1e-6,
                                    device="cuda")
                 for i, (k, e) in enumerate(m.elements.items())}
    slots = ra.to_slots({k: Foreign(v) for k, v in mdot_elem.items()})
    for k, v in slots.items():
        assert v.shape == mdot_elem[k].shape
    back = ra.from_slots({k: Foreign(v) for k, v in slots.items()})
    for k, v in back.items():
        assert torch.equal(v, mdot_elem[k])
    tslots = ta.to_slots(mdot_elem)
    # gradients, limiter, diagonal
    gU, gP = ra.gradient(Foreign(U)), ra.gradient(Foreign(P))
    assert gU.shape == (N, 3, 3) and gP.shape == (N, 3)
    assert torch.equal(gU, ta.gradient(U)) and torch.equal(gP, ta.gradient(P))
    beta = ra.limiter(Foreign(U), Foreign(gU))
    assert beta.shape == (N, 3) and torch.equal(beta, ta.limiter(U, gU))
    diag = ra.diagonal({k: Foreign(v) for k, v in slots.items()}, Foreign(U))
    assert diag.shape == (N,) and torch.equal(diag, ta.diagonal(tslots, U))
    V = ta.node_volume
    dnode, snode = V / (diag + 1.0), V / diag
    own = torch.zeros(N, dtype=torch.int32, device="cuda")
    own[::7] = 1
    levels = [(1.0, U, tslots)]
    data, b = ra.assemble(Foreign(U), {k: Foreign(v) for k, v in slots.items()}, Foreign(gU),
                          Foreign(beta), Foreign(gP), Foreign(dnode), Foreign(snode),
                          levels=[(1.0, Foreign(U), {k: Foreign(v) for k, v in slots.items()})],
                          own=Foreign(own))
    d2, b2 = ta.assemble(U, tslots, gU, beta, gP, dnode, snode, levels=levels, own=own)
    assert data.shape == (ra.nnzb, 4, 4) and b.shape == (N, 4)
    assert torch.equal(data, d2) and torch.equal(b, b2)
    new, imb, adv = ra.massflow(Foreign(U), Foreign(P), Foreign(gP), Foreign(dnode),
                                Foreign(snode), levels=[(1.0, Foreign(U),
                                                         {k: Foreign(v) for k, v in slots.items()})])
    new2, imb2, adv2 = ta.massflow(U, P, gP, dnode, snode, levels=levels)
    for k, v in new.items():
        assert v.shape == (len(m.elements[k]), ra.kinds[[K.kind for K in ra.kinds].index(k)].nip)
        assert torch.equal(v, new2[k])
    assert imb.shape == (N,) and adv.shape == (N,)
    assert torch.equal(imb, imb2) and torch.equal(adv, adv2)
