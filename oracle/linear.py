"""Linear algebra of the coupled system on the CPU (oracle).

- :func:`bsr_matvec` restates ``bsr_mv`` + ``BlockMatrix.matvec`` (``zvcfd/fv/linear.py:47-61``,
  ``:93-103``): ``y = A x + sum u (w . x)`` with SciPy's block-CSR product.
"""

from __future__ import annotations

import numpy as np
import scipy.sparse as sp


def bsr(indptr, indices, data, n):
    return sp.bsr_matrix((np.asarray(data).reshape(-1, 4, 4), np.asarray(indices),
                          np.asarray(indptr)), shape=(4 * n, 4 * n))


def bsr_matvec(indptr, indices, data, x, lowrank=()):
    n = len(indptr) - 1
    y = bsr(indptr, indices, data, n) @ np.asarray(x).reshape(-1)
    for ui, uv, wi, wv in lowrank:
        y[ui] += uv * np.dot(wv, np.asarray(x).reshape(-1)[wi])
    return y


# ---------------------------------------------------------------- aggregation multigrid

def block_weights(data, mode=0):
    """Coupling measure per block: the Frobenius norm (``zvcfd/fv/linear.py:418``), summed in
    entry order with separately rounded products, or ``|a_pp|`` (AmgX component 3)."""
    d = np.asarray(data).reshape(-1, 16)
    if mode == 1:
        return np.abs(d[:, 15])
    s = np.zeros(len(d))
    for e in range(16):
        s += d[:, e] * d[:, e]
    return np.sqrt(s)


def pairwise(n, indptr, indices, strength):
    """Pairwise matching on coupling strength (``zvcfd/fv/linear.py:373-413``): four rounds of
    mutual strongest free neighbours (ties: first in column order), pairs numbered in order
    of their first node; unmatched nodes join their strongest aggregated neighbour, the rest
    stay single. Returns ``(agg (n,), count)``."""
    indptr = np.asarray(indptr, np.int64)
    rows = np.repeat(np.arange(n), np.diff(indptr))
    cols = np.asarray(indices, np.int64)
    agg = -np.ones(n, np.int64)
    off = rows != cols
    r, c, s = rows[off], cols[off], strength[off]
    nxt = 0
    for _ in range(4):
        m = (agg[r] < 0) & (agg[c] < 0)
        if not m.any():
            break
        rr, cc, ss = r[m], c[m], s[m]
        order = np.lexsort((-ss, rr))
        rr, cc = rr[order], cc[order]
        first = np.r_[True, rr[1:] != rr[:-1]]
        best = -np.ones(n, np.int64)
        best[rr[first]] = cc[first]
        i = np.flatnonzero(best >= 0)
        j = best[i]
        mutual = (best[j] == i) & (i < j)
        a, bb = i[mutual], j[mutual]
        ids = nxt + np.arange(len(a))
        agg[a] = ids
        agg[bb] = ids
        nxt += len(a)
    left = np.flatnonzero(agg < 0)
    if len(left):
        m = (agg[r] < 0) & (agg[c] >= 0)
        rr, cc, ss = r[m], c[m], s[m]
        join = -np.ones(n, np.int64)
        if len(rr):
            order = np.lexsort((-ss, rr))
            rr, cc = rr[order], cc[order]
            first = np.r_[True, rr[1:] != rr[:-1]]
            join[rr[first]] = agg[cc[first]]
        to = join[left]
        agg[left[to >= 0]] = to[to >= 0]
        single = left[to < 0]
        agg[single] = nxt + np.arange(len(single))
        nxt += len(single)
    return agg, nxt


def transpose_positions(indptr, indices):
    """Position of the entry (j, i) for every entry (i, j) of a structurally symmetric pattern."""
    n = len(indptr) - 1
    rows = np.repeat(np.arange(n), np.diff(indptr))
    cols = np.asarray(indices, np.int64)
    order = np.lexsort((rows, cols))          # entries by (column, row): the transpose's order
    pos = np.empty(len(cols), np.int64)
    pos[order] = np.arange(len(cols))
    return pos


def aggregate(indptr, indices, data, passes=2, mode=0):
    """``passes`` pairwise passes with the graph coarsened between them by summing strengths
    per aggregate pair (``zvcfd/fv/linear.py:415-433``). Returns ``(agg, count)``. ``mode`` 2
    (not in the reference) averages each block norm with that of its transpose position."""
    n = len(indptr) - 1
    rows = np.repeat(np.arange(n), np.diff(indptr))
    cols = np.asarray(indices, np.int64)
    w = block_weights(data, 1 if mode == 1 else 0)
    if mode == 2:
        w = 0.5 * (w + w[transpose_positions(indptr, indices)])
    total = np.arange(n)
    count = n
    ptr = np.asarray(indptr, np.int64)
    for p in range(passes):
        diag = np.zeros(count)
        dmask = rows == cols
        diag[rows[dmask]] = w[dmask]
        s = w / np.sqrt(np.maximum(diag[rows] * diag[cols], 1e-300))
        a, count_new = pairwise(count, ptr, cols, s)
        total = a[total]
        if p + 1 == passes:
            count = count_new
            break
        rows, cols = a[rows], a[cols]
        count = count_new
        key = rows * count + cols
        uk, inv = np.unique(key, return_inverse=True)
        w = np.bincount(inv.reshape(-1), w, len(uk))
        rows, cols = uk // count, uk % count
        ptr = np.zeros(count + 1, np.int64)
        np.cumsum(np.bincount(rows, minlength=count), out=ptr[1:])
    return total, count


def galerkin(indptr, indices, data, agg, nc):
    """Coarse operator: blocks summed per aggregate pair (``zvcfd/fv/linear.py:437-454``)."""
    n = len(indptr) - 1
    rows = np.repeat(np.arange(n), np.diff(indptr))
    key = agg[rows] * nc + agg[np.asarray(indices, np.int64)]
    uk, inv = np.unique(key, return_inverse=True)
    out = np.zeros((len(uk), 16))
    d = np.asarray(data).reshape(-1, 16)
    for e in range(16):
        out[:, e] = np.bincount(inv.reshape(-1), d[:, e], len(uk))
    crow = uk // nc
    cptr = np.zeros(nc + 1, np.int64)
    np.cumsum(np.bincount(crow, minlength=nc), out=cptr[1:])
    return cptr, (uk % nc).astype(np.int64), out.reshape(-1, 4, 4)


class ACM:
    """Additive-correction multigrid on the CPU (``zvcfd/fv/linear.py:328-518``): pairwise
    aggregation, Galerkin block sums, damped block-Jacobi smoothing, a dense coarsest solve."""

    def __init__(self, *, smooth=2, omega=0.7, coarse=24, passes=2, mode=0, max_levels=25,
                 coarse_sweeps=8):
        self.smooth, self.omega, self.coarse, self.passes = smooth, omega, coarse, passes
        self.mode, self.max_levels, self.coarse_sweeps = mode, max_levels, coarse_sweeps

    def setup(self, indptr, indices, data):
        self.levels = []
        ptr, idx, dat = np.asarray(indptr), np.asarray(indices, np.int64), np.asarray(data)
        while True:
            n = len(ptr) - 1
            A = bsr(ptr, idx, dat, n).tocsr()
            rows = np.repeat(np.arange(n), np.diff(ptr))
            dpos = np.flatnonzero(rows == idx)
            D = dat.reshape(-1, 4, 4)[dpos]
            Dinv = np.zeros_like(D)
            ok = np.abs(np.linalg.det(D)) > 0
            Dinv[ok] = np.linalg.inv(D[ok])
            L = {"A": A, "Dinv": Dinv, "n": n, "ptr": ptr, "idx": idx, "data": dat}
            self.levels.append(L)
            if n <= self.coarse:
                L["dense_inv"] = np.linalg.inv(A.toarray())
                break
            if len(self.levels) >= self.max_levels:
                break
            agg, nc = aggregate(ptr, idx, dat, self.passes, self.mode)
            if nc >= 0.9 * n or nc < 1:
                break
            L["agg"], L["nc"] = agg, nc
            ptr, idx, dat = galerkin(ptr, idx, dat, agg, nc)
        return self

    def _smooth(self, L, x, b, sweeps):
        for s in range(sweeps):
            r = (b - L["A"] @ x).reshape(-1, 4) if (s or x.any()) else b.reshape(-1, 4)
            x = x + self.omega * np.einsum("nij,nj->ni", L["Dinv"], r).reshape(-1)
        return x

    def vcycle(self, b, level=0):
        L = self.levels[level]
        if "dense_inv" in L:
            return L["dense_inv"] @ b
        last = "agg" not in L
        x = self._smooth(L, np.zeros_like(b), b, self.coarse_sweeps if last else self.smooth)
        if last:
            return x
        r = (b - L["A"] @ x).reshape(-1, 4)
        rc = np.zeros((L["nc"], 4))
        np.add.at(rc, L["agg"], r)
        ec = self.vcycle(rc.reshape(-1), level + 1)
        x = x + ec.reshape(-1, 4)[L["agg"]].reshape(-1)
        return self._smooth(L, x, b, self.smooth)


def fgmres(matvec, b, x0, precond, *, rtol=1e-6, restart=30, maxiter=300):
    """Right-preconditioned flexible GMRES with CGS2 (``zvcfd/fv/linear.py:172-320``):
    convergence relative to the initial residual, with the round-off floor 1e-13 ||b||.
    Returns ``(x, iterations, residual relative to the initial one, converged)``."""
    x = np.array(x0, float)
    r = b - matvec(x)
    bnorm = np.linalg.norm(r) or 1.0
    rtol = max(rtol, 1e-13 * np.linalg.norm(b) / bnorm)
    beta = np.linalg.norm(r)
    res = beta / bnorm
    it = 0
    while res > rtol and it < maxiter:
        V = [r / beta]
        Z = []
        H = np.zeros((restart + 1, restart))
        g = np.zeros(restart + 1)
        g[0] = beta
        cs, sn = np.zeros(restart), np.zeros(restart)
        kk = 0
        for k in range(restart):
            z = precond(V[k])
            Z.append(z)
            w = matvec(z)
            Vk = np.array(V)
            h1 = Vk @ w
            w = w - h1 @ Vk
            h2 = Vk @ w
            w = w - h2 @ Vk
            hn = np.linalg.norm(w)
            H[:k + 1, k] = h1 + h2
            H[k + 1, k] = hn
            for j in range(k):
                t = cs[j] * H[j, k] + sn[j] * H[j + 1, k]
                H[j + 1, k] = -sn[j] * H[j, k] + cs[j] * H[j + 1, k]
                H[j, k] = t
            den = np.hypot(H[k, k], H[k + 1, k])
            cs[k], sn[k] = (H[k, k] / den, H[k + 1, k] / den) if den else (1.0, 0.0)
            H[k, k], H[k + 1, k] = den, 0.0
            g[k + 1] = -sn[k] * g[k]
            g[k] = cs[k] * g[k]
            it += 1
            kk = k + 1
            res = abs(g[k + 1]) / bnorm
            if res <= rtol or it >= maxiter or hn == 0.0:
                break
            V.append(w / hn)
        y = np.linalg.solve(np.triu(H[:kk, :kk]), g[:kk])
        x = x + y @ np.array(Z)
        r = b - matvec(x)
        beta = np.linalg.norm(r)
        res = beta / bnorm
    return x, it, res, res <= 1.01 * rtol
