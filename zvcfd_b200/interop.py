"""Adapters for the reference's own objects: CuPy arrays in and out, zero-copy.

``ReferenceLinear`` is what ``zvcfd.fv.linear.make("b200")`` returns once the reference's
``make`` is given a ``"b200"`` branch: it takes the reference's ``BlockMatrix`` (``zvcfd/fv/linear.py:75-135``:
CuPy ``indptr``/``indices``/``data`` and the ``lowrank`` list) and CuPy vectors, views them as
torch tensors through ``__cuda_array_interface__`` (no copy), solves with
:class:`~zvcfd_b200.linear.B200AMG` (or the ``b200-auto`` ladder), and hands back a CuPy view of the solution and the
reference's ``SolveInfo`` fields. ``ReferenceAssembler`` does the same for
:class:`~zvcfd_b200.assembler.B200Assembler`'s ``FastAssembler`` interface.
"""

from __future__ import annotations

import torch

from zvcfd_b200.assembler import B200Assembler
from zvcfd_b200.linear import BlockMatrix, make


def as_torch(a):
    """A torch view of a device array (CuPy or torch); host arrays are copied to the device."""
    if a is None or isinstance(a, torch.Tensor):
        return a
    if hasattr(a, "__cuda_array_interface__") or hasattr(a, "__dlpack__"):
        try:
            return torch.as_tensor(a, device="cuda")
        except TypeError:
            return torch.from_dlpack(a)
    return torch.as_tensor(a, device="cuda")


def as_caller(t, like):
    """``t`` in the caller's array type: a CuPy view when the caller passed CuPy."""
    if like is None or isinstance(like, torch.Tensor) or t is None:
        return t
    mod = type(like).__module__.split(".")[0]
    if mod == "cupy":
        import cupy as cp

        return cp.asarray(t)
    return t


def block_matrix(A) -> BlockMatrix:
    """The reference's BlockMatrix (any device array type) as a torch BlockMatrix view."""
    low = [tuple(as_torch(v).to(torch.int64) if i in (0, 2) else as_torch(v)
                 for i, v in enumerate(term)) for term in getattr(A, "lowrank", [])]
    return BlockMatrix(as_torch(A.indptr).to(torch.int64), as_torch(A.indices).to(torch.int32),
                       as_torch(A.data).reshape(-1, 4, 4), low)


class ReferenceLinear:
    """``solve(A, b, x0=None, rtol=None) -> (x, SolveInfo)`` over the reference's objects."""

    def __init__(self, name: str = "b200", **kw):
        self.inner = make(name, **kw)
        self.name = name

    @property
    def active(self) -> str:
        """The rung in use (``"b200-auto"``), as the reference's ``Auto.active``."""
        return getattr(self.inner, "active", self.name)

    @property
    def switches(self) -> list:
        return getattr(self.inner, "switches", [])

    def solve(self, A, b, x0=None, rtol=None):
        x, info = self.inner.solve(block_matrix(A), as_torch(b).reshape(-1),
                                   None if x0 is None else as_torch(x0).reshape(-1), rtol=rtol)
        return as_caller(x, b), info

    def vcycle(self, r):
        return as_caller(self.inner.vcycle(as_torch(r)), r)

    def close(self):
        self.inner.close()


class ReferenceAssembler(B200Assembler):
    """``FastAssembler``'s interface over caller arrays (CuPy in, CuPy out)."""

    def gradient(self, phi, **kw):
        return as_caller(super().gradient(as_torch(phi), **kw), phi)

    def diagonal(self, mdot, U=None, *, mu_t=None, out=None):
        md = {k: as_torch(v) for k, v in mdot.items()}
        like = next(iter(mdot.values()), None)
        return as_caller(super().diagonal(md, as_torch(U), mu_t=as_torch(mu_t)), like)

    def assemble(self, U, mdot, gradU, beta, gradP, dnode, snode, *, levels=(), own=None,
                 mu_t=None, data=None, b=None):
        md = {k: as_torch(v) for k, v in mdot.items()}
        lv = [(c, as_torch(Uo), {k: as_torch(v) for k, v in mo.items()}) for c, Uo, mo in levels]
        d, bb = super().assemble(as_torch(U), md, as_torch(gradU), as_torch(beta),
                                 as_torch(gradP), as_torch(dnode), as_torch(snode), levels=lv,
                                 own=as_torch(own), mu_t=as_torch(mu_t))
        return as_caller(d, U), as_caller(bb, U)

    def massflow(self, U, P, gradP, dnode, snode, *, levels=(), out=None):
        lv = [(c, as_torch(Uo), {k: as_torch(v) for k, v in mo.items()}) for c, Uo, mo in levels]
        m, imb, adv = super().massflow(as_torch(U), as_torch(P), as_torch(gradP), as_torch(dnode),
                                       as_torch(snode), levels=lv)
        return {k: as_caller(v, U) for k, v in m.items()}, as_caller(imb, U), as_caller(adv, U)

    def limiter(self, U, gradU):
        return as_caller(super().limiter(as_torch(U), as_torch(gradU)), U)

    def to_slots(self, mdot):
        like = next(iter(mdot.values()), None)
        return {k: as_caller(v, like) for k, v in
                super().to_slots({k: as_torch(v) for k, v in mdot.items()}).items()}

    def from_slots(self, mdot):
        like = next(iter(mdot.values()), None)
        return {k: as_caller(v, like) for k, v in
                super().from_slots({k: as_torch(v) for k, v in mdot.items()}).items()}


__all__ = ["ReferenceAssembler", "ReferenceLinear", "as_torch", "block_matrix"]
