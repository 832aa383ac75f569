"""The B200 assembler: a drop-in for the reference's ``FastAssembler`` (``zvcfd/fv/fast.py:155-406``).

Same constructor arguments and method set (``pattern``, ``node_volume``, ``dvisc``,
``gop``, ``zero_mdot``, ``to_slots``/``from_slots``, ``gradient``, ``diagonal``,
``assemble``, ``massflow``, ``limiter``), with torch device tensors in place of CuPy
arrays. Every array operation runs in ``libzvfv_b200.so``: the pattern, the colouring and
slot order, the geometry records, block positions and statics at set-up, and the element
and node kernels per outer iteration. Element data live in slot order (each type's
elements sorted by colour), so that a colour is a contiguous range of one launch.
"""

from __future__ import annotations

import ctypes

import numpy as np
import torch

from zvcfd_b200._lib import call, lib, ptr, stream_ptr
from zvcfd_b200.topology import KINDS, tables

KIND_CODE = {k: i for i, k in enumerate(KINDS)}


def _f64(a, device):
    return torch.as_tensor(np.ascontiguousarray(a), dtype=torch.float64, device=device) \
        if not isinstance(a, torch.Tensor) else a.to(device=device, dtype=torch.float64).contiguous()


def node_graph(elements: dict, n_nodes: int, device="cuda"):
    """The block pattern on the device: ``(indptr int64 (N+1,), indices int32)``, sorted
    (``zvcfd/fv/fast.py:133-147``)."""
    conns = [torch.as_tensor(np.ascontiguousarray(e, np.int32), device=device)
             for e in elements.values()]
    k = len(conns)
    cptr = (ctypes.c_void_p * k)(*[c.data_ptr() for c in conns])
    nel = (ctypes.c_int64 * k)(*[c.shape[0] for c in conns])
    npe = (ctypes.c_int32 * k)(*[c.shape[1] for c in conns])
    h = ctypes.c_void_p()
    nnzb = ctypes.c_int64()
    call("zvfv_pattern_create", ctypes.byref(h), n_nodes, k, cptr, nel, npe, ctypes.byref(nnzb),
         stream_ptr())
    try:
        indptr = torch.empty(n_nodes + 1, dtype=torch.int64, device=device)
        indices = torch.empty(nnzb.value, dtype=torch.int32, device=device)
        call("zvfv_pattern_fill", h, ptr(indptr), ptr(indices), stream_ptr())
    finally:
        lib.zvfv_pattern_destroy(h)
    return indptr, indices


def gpu_colour(conn, n_nodes: int, words: int = 4):
    """Colour ``(E,)`` int32 of each element, bit-exact with ``zvcfd/fv/fast.py:94-130``."""
    conn = torch.as_tensor(conn).to(device="cuda", dtype=torch.int32).contiguous()
    E, n = conn.shape
    col = torch.empty(E, dtype=torch.int32, device=conn.device)
    nc = ctypes.c_int32()
    call("zvfv_colour", ptr(conn), n, E, n_nodes, words, ptr(col), ctypes.byref(nc), 1_000_000,
         stream_ptr())
    return col, nc.value


class Kind:
    """One element type's device data, in slot order."""

    def __init__(self, kind, elem, n_nodes, device):
        t = tables(kind)
        self.kind, self.t, self.code = kind, t, KIND_CODE[kind]
        self.n, self.nip, self.E = t.n, t.n_ip, len(elem)
        ed = torch.as_tensor(np.ascontiguousarray(elem, np.int32), device=device)
        col, ncol = gpu_colour(ed, n_nodes)
        self.colour = col
        self.order = torch.empty(self.E, dtype=torch.int64, device=device)    # slot -> element
        offsets = torch.empty(ncol + 1, dtype=torch.int64, device=device)
        call("zvfv_slot_order", ptr(col), self.E, ncol, ptr(self.order), ptr(offsets),
             stream_ptr())
        self.conn = torch.empty_like(ed)
        call("zvfv_permute_rows", ptr(ed), ptr(self.order), self.E, 4 * self.n, ptr(self.conn),
             0, stream_ptr())
        self.offsets = offsets.cpu().numpy().astype(np.int64)
        self.n_colours = ncol
        self.host_offsets = (ctypes.c_int64 * (ncol + 1))(*self.offsets.tolist())


class B200Assembler:
    """Device evaluation of the discrete equations, ``FastAssembler``'s interface.

    Args:
        mesh: nodes ``(N, 3)``, ``elements {kind: (E, n)}``.
        rho, mu, rheology, transpose, stokes: fluid and options, as the reference.
        store_geometry: ``True`` keeps per-element geometry records on the device;
            ``False`` rebuilds them in shared memory in every kernel (``"auto"``:
            rebuild, which on a B200 costs less than reading the records back).
        pattern: ``(indptr, indices)`` on the device, if already built.
    """

    def __init__(self, mesh, *, rho=1.0, mu=1.0, rheology=None, transpose=False, stokes=False,
                 store_geometry="auto", pattern=None, device="cuda"):
        self.device = torch.device(device)
        self.mesh, self.rho, self.mu = mesh, float(rho), float(mu)
        self.transpose, self.stokes = int(bool(transpose)), int(bool(stokes))
        if rheology is None:
            self.rheo = (0, float(mu), float(mu), 0.0, 2.0, 1.0)
        else:
            r = rheology
            self.rheo = (1, float(r.mu_0), float(r.mu_inf), float(r.lam), float(r.a), float(r.n))
        self.N = mesh.n_nodes
        self.X = _f64(mesh.nodes, self.device)
        self.pattern = pattern if pattern is not None else node_graph(mesh.elements, self.N,
                                                                      self.device)
        indptr, indices = self.pattern
        self.nnzb = int(indices.numel())
        stored = store_geometry is True
        self.store_mode = stored
        self.kinds = [Kind(k, e, self.N, self.device) for k, e in mesh.elements.items()]
        self.node_volume = torch.zeros(self.N, dtype=torch.float64, device=self.device)
        self.dvisc = torch.zeros_like(self.node_volume)
        self.gop = torch.zeros(self.nnzb * 3, dtype=torch.float64, device=self.device)
        self._dummy = torch.zeros(1, dtype=torch.float64, device=self.device)
        st = stream_ptr()
        for K in self.kinds:
            K.stored = stored
            if stored:
                K.geo = torch.empty(K.E * K.t.record_doubles, dtype=torch.float64,
                                    device=self.device)
                call("zvfv_geobuild", K.code, ptr(K.conn), K.E, ptr(self.X), ptr(K.geo), st)
            else:
                K.geo = self._dummy
            K.pos = torch.empty(K.E * K.n * K.n, dtype=torch.int32, device=self.device)
            call("zvfv_blockpos", K.code, ptr(K.conn), K.E, ptr(indptr), ptr(indices),
                 ptr(K.pos), st)
            call("zvfv_statics", K.code, int(K.stored), ptr(K.conn), K.n_colours,
                 K.host_offsets, ptr(self.X), ptr(K.geo), ptr(K.pos),
                 float(self.rheo[1] if rheology is None else 0.0), self.transpose,
                 ptr(self.node_volume), ptr(self.dvisc), ptr(self.gop), st)
        rows = torch.repeat_interleave(torch.arange(self.N, device=self.device),
                                       indptr[1:] - indptr[:-1])
        self.gop.view(-1, 3).div_(self.node_volume[rows][:, None])
        self._no_own = torch.zeros(self.N, dtype=torch.int32, device=self.device)
        self._no_mut = self._dummy

    # ------------------------------------------------------------ slot order

    def zero_mdot(self) -> dict:
        return {K.kind: torch.zeros((K.E, K.nip), dtype=torch.float64, device=self.device)
                for K in self.kinds}

    def to_slots(self, mdot: dict) -> dict:
        """Mass flows from element order to slot order."""
        out = {}
        for K in self.kinds:
            src = _f64(mdot[K.kind], self.device)
            dst = torch.empty_like(src)
            call("zvfv_permute_rows", ptr(src), ptr(K.order), K.E, 8 * K.nip, ptr(dst), 0,
                 stream_ptr())
            out[K.kind] = dst
        return out

    def from_slots(self, mdot: dict) -> dict:
        out = {}
        for K in self.kinds:
            src = mdot[K.kind].contiguous()
            dst = torch.empty_like(src)
            call("zvfv_permute_rows", ptr(src), ptr(K.order), K.E, 8 * K.nip, ptr(dst), 1,
                 stream_ptr())
            out[K.kind] = dst
        return out

    def _vec(self, a):
        return _f64(a, self.device).reshape(-1)

    def _levels(self, levels, kind):
        out = [len(levels)]
        for i in range(2):
            if i < len(levels):
                c, Uo, mo = levels[i]
                out += [float(c), ptr(self._vec(Uo)), ptr(mo[kind].contiguous())]
            else:
                out += [0.0, ptr(self._dummy), ptr(self._dummy)]
        return out

    def _mut(self, mu_t):
        if mu_t is None:
            return 0, ptr(self._no_mut)
        return 1, ptr(self._vec(mu_t))

    def _own(self, own):
        if own is None:
            return self._no_own
        return torch.as_tensor(own, device=self.device).to(torch.int32).contiguous()

    # ------------------------------------------------------------ kernels

    def gradient(self, phi, *, sym=None, nvec=None):
        """Nodal gradients of ``phi (N,)`` or ``(N, C)``, ``C <= 4``: ``(N, 3)`` or ``(N, C, 3)``.

        ``sym`` ``(N, 3)`` uint8 applies the symmetry-plane mirror on the way out (the
        first ``nvec`` fields forming a vector).
        """
        phi = _f64(phi, self.device)
        vec = phi.ndim == 2
        nc = phi.shape[1] if vec else 1
        if nc > 4:
            return torch.cat([self.gradient(phi[:, i:i + 4]) for i in range(0, nc, 4)], 1)
        out = torch.empty(self.N * nc * 3, dtype=torch.float64, device=self.device)
        flat = phi.reshape(self.N, nc).contiguous()
        indptr, indices = self.pattern
        nv = (3 if nc >= 3 else 0) if nvec is None else nvec
        call("zvfv_gradient", self.N, nc, nv, ptr(indptr), ptr(indices), ptr(self.gop),
             ptr(flat), ptr(sym), ptr(out), stream_ptr())
        g = out.view(self.N, nc, 3)
        return g if vec else g[:, 0]

    def diagonal(self, mdot: dict, U=None, *, mu_t=None, out=None):
        """Momentum diagonal ``a_P`` from slot-ordered mass flows."""
        diag = torch.zeros(self.N, dtype=torch.float64, device=self.device) if out is None \
            else out.zero_()
        U_ = self._vec(U if U is not None else torch.zeros((self.N, 3), dtype=torch.float64,
                                                           device=self.device))
        hm, mt = self._mut(mu_t)
        st = stream_ptr()
        for K in self.kinds:
            call("zvfv_diagonal", K.code, int(K.stored), ptr(K.conn), K.n_colours,
                 K.host_offsets, ptr(self.X), ptr(K.geo), ptr(mdot[K.kind].contiguous()),
                 ptr(U_), *self.rheo, self.transpose, self.stokes, hm, mt, ptr(diag), st)
        return diag

    def assemble(self, U, mdot: dict, gradU, beta, gradP, dnode, snode, *, levels=(), own=None,
                 mu_t=None, data=None, b=None):
        """Block values ``(nnzb, 4, 4)`` and right-hand side ``(N, 4)`` of the flux points."""
        if data is None:
            data = torch.zeros(self.nnzb * 16, dtype=torch.float64, device=self.device)
        else:
            data.zero_()
        if b is None:
            b = torch.zeros(self.N * 4, dtype=torch.float64, device=self.device)
        else:
            b.zero_()
        U_, gU, be, gP, dn, sn = (self._vec(a) for a in (U, gradU, beta, gradP, dnode, snode))
        own_ = self._own(own)
        hm, mt = self._mut(mu_t)
        st = stream_ptr()
        for K in self.kinds:
            call("zvfv_assemble", K.code, int(K.stored), ptr(K.conn), K.n_colours,
                 K.host_offsets, ptr(self.X), ptr(K.geo), ptr(U_), ptr(mdot[K.kind].contiguous()),
                 ptr(gU), ptr(be), ptr(gP), ptr(dn), ptr(sn), *self._levels(levels, K.kind),
                 self.rho, *self.rheo, self.transpose, self.stokes, hm, mt, ptr(own_),
                 ptr(K.pos), ptr(data), ptr(b), st)
        return data.view(-1, 4, 4), b.view(self.N, 4)

    def massflow(self, U, P, gradP, dnode, snode, *, levels=(), out=None, vdiag=None,
                 mu_t=None):
        """``(mdot {kind: (E, n_ip)} slot order, net outflow (N,), advective diagonal (N,))``.
        With ``vdiag`` (N,), the same element pass also accumulates into it the viscous part
        of the next momentum diagonal from ``U`` (``diagonal`` without its advective part)."""
        imb = torch.zeros(self.N, dtype=torch.float64, device=self.device)
        adv = torch.zeros(self.N, dtype=torch.float64, device=self.device)
        res = {}
        U_, P_, gP, dn, sn = (self._vec(a) for a in (U, P, gradP, dnode, snode))
        st = stream_ptr()
        hm, mt = self._mut(mu_t)
        for K in self.kinds:
            m = torch.empty((K.E, K.nip), dtype=torch.float64, device=self.device) \
                if out is None else out[K.kind]
            head = (K.code, int(K.stored), ptr(K.conn), K.n_colours, K.host_offsets,
                    ptr(self.X), ptr(K.geo), ptr(U_), ptr(P_), ptr(gP), ptr(dn), ptr(sn),
                    *self._levels(levels, K.kind), self.rho)
            if vdiag is None:
                call("zvfv_massflow", *head, ptr(m), ptr(imb), ptr(adv), st)
            else:
                call("zvfv_massflow_diag", *head, *self.rheo, self.transpose, hm, mt, ptr(m),
                     ptr(imb), ptr(adv), ptr(vdiag), st)
            res[K.kind] = m
        return res, imb, adv

    def limiter(self, U, gradU):
        """Barth-Jespersen blend factors ``(N, 3)``."""
        U_ = self._vec(U)
        lo = torch.empty(self.N * 3, dtype=torch.float64, device=self.device)
        hi = torch.empty_like(lo)
        indptr, indices = self.pattern
        st = stream_ptr()
        call("zvfv_minmax", self.N, ptr(indptr), ptr(indices), ptr(U_), ptr(lo), ptr(hi), st)
        beta = torch.ones(self.N * 3, dtype=torch.float64, device=self.device)
        gU = self._vec(gradU)
        for K in self.kinds:
            call("zvfv_limiter", K.code, int(K.stored), ptr(K.conn), K.n_colours,
                 K.host_offsets, ptr(self.X), ptr(K.geo), ptr(U_), ptr(gU), ptr(lo), ptr(hi),
                 ptr(beta), st)
        return beta.view(self.N, 3)

    # ------------------------------------------------------------ sizes

    def geometry_bytes(self) -> int:
        return int(sum(K.geo.numel() * 8 for K in self.kinds if K.stored))

    def static_bytes(self) -> int:
        return self.geometry_bytes() + int(sum(K.pos.numel() * 4 + K.conn.numel() * 4
                                               for K in self.kinds)) + int(self.gop.numel() * 8)


__all__ = ["B200Assembler", "gpu_colour", "node_graph"]
