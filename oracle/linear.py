"""Linear algebra of the coupled system on the CPU (oracle).

- :func:`bsr_matvec` restates ``bsr_mv`` + ``BlockMatrix.matvec`` (``zvcfd/fv/linear.py:47-61``,
  ``:93-103``): ``y = A x + sum u (w . x)`` with SciPy's block-CSR product.

Pinned: ``tests/test_acm_reference.py`` holds :class:`ACM` (at the reference's parameters) and
:func:`fgmres` to the reference's own ACM and device FGMRES, run on the CPU
(``tests/golden/make_golden.py acm``): the same aggregates bit for bit, the same Krylov
iteration counts, V-cycles and solutions to 1e-14 and 1e-13.
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
    """Pairwise matching on coupling strength (``zvcfd/fv/linear.py:373-413``), node by node.

    Up to four rounds: every free node picks its strongest free neighbour (the first in
    column order among equals); nodes that pick each other form an aggregate, numbered in
    order of the smaller node; the rounds stop early once no two free nodes are coupled.
    Then every node still free joins the aggregate of its strongest already-aggregated
    neighbour (picks made before any joins), and the rest become aggregates of their own, in
    node order. Returns ``(agg (n,), count)``."""
    ptr = [int(v) for v in indptr]
    col = [int(v) for v in indices]
    agg = [-1] * n
    count = 0

    def strongest(i, wanted):
        pick, top = -1, None
        for p in range(ptr[i], ptr[i + 1]):
            j = col[p]
            if j != i and wanted(j) and (top is None or strength[p] > top):
                pick, top = j, strength[p]
        return pick

    for _ in range(4):
        choice = {i: strongest(i, lambda j: agg[j] < 0) for i in range(n) if agg[i] < 0}
        choice = {i: j for i, j in choice.items() if j >= 0}
        if not choice:
            break
        for i in sorted(choice):
            j = choice[i]
            if i < j and choice.get(j) == i:
                agg[i] = agg[j] = count
                count += 1
    free = [i for i in range(n) if agg[i] < 0]
    joins = {i: strongest(i, lambda j: agg[j] >= 0) for i in free}
    for i in free:
        if joins[i] >= 0:
            agg[i] = agg[joins[i]]
    for i in free:
        if joins[i] < 0:
            agg[i] = count
            count += 1
    return np.array(agg, np.int64), count


def pairwise_arrays(n, indptr, indices, strength):
    """:func:`pairwise` over whole arrays: the form the reference's own host aggregation takes
    (``zvcfd/fv/linear.py:355-396``), used where the node-by-node form is too slow (the CPU
    baseline at full size). Same rounds, picks, ties (the first maximum in column order) and
    numbering, so the aggregates are equal to :func:`pairwise`'s (checked in the tests)."""
    rows = np.repeat(np.arange(n), np.diff(np.asarray(indptr, np.int64)))
    cols = np.asarray(indices, np.int64)
    off = rows != cols
    r, c, s = rows[off], cols[off], np.asarray(strength)[off]
    agg = np.full(n, -1, np.int64)
    count = 0

    def first_pick(rr, cc, ss):
        """Each row's strongest column (ties: the smallest column), -1 for rows without one."""
        pick = np.full(n, -1, np.int64)
        if len(rr):
            order = np.lexsort((cc, -ss, rr))
            head = np.ones(len(order), bool)
            head[1:] = rr[order][1:] != rr[order][:-1]
            pick[rr[order][head]] = cc[order][head]
        return pick

    for _ in range(4):
        live = (agg[r] < 0) & (agg[c] < 0)
        if not live.any():
            break
        best = first_pick(r[live], c[live], s[live])
        i = np.flatnonzero(best >= 0)
        j = best[i]
        pair = (best[j] == i) & (i < j)
        a, b = i[pair], j[pair]                       # ascending in a: numbered in its order
        agg[a] = agg[b] = count + np.arange(len(a))
        count += len(a)
    free = np.flatnonzero(agg < 0)
    if len(free):
        reach = (agg[r] < 0) & (agg[c] >= 0)
        join = first_pick(r[reach], c[reach], s[reach])[free]
        joined = join >= 0
        target = agg[join[joined]]
        agg[free[joined]] = target
        alone = free[~joined]
        agg[alone] = count + np.arange(len(alone))
        count += len(alone)
    return agg, count


def transpose_positions(indptr, indices):
    """Position of the entry (j, i) for every entry (i, j) of a structurally symmetric pattern."""
    n = len(indptr) - 1
    rows = np.repeat(np.arange(n), np.diff(indptr))
    cols = np.asarray(indices, np.int64)
    order = np.lexsort((rows, cols))          # entries by (column, row): the transpose's order
    pos = np.empty(len(cols), np.int64)
    pos[order] = np.arange(len(cols))
    return pos


def aggregate(indptr, indices, data, passes=2, mode=0, matcher=None):
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
        a, count_new = (matcher or pairwise)(count, ptr, cols, s)
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
                 coarse_sweeps=8, matcher=None, rebuild_every=1):
        self.smooth, self.omega, self.coarse, self.passes = smooth, omega, coarse, passes
        self.mode, self.max_levels, self.coarse_sweeps = mode, max_levels, coarse_sweeps
        self.matcher = matcher
        # aggregates are kept between re-aggregations, the coefficients re-summed every set-up
        # (the reference ACM's rebuild_every, zvcfd/fv/linear.py:456-470)
        self.rebuild_every, self._setups, self._aggs = rebuild_every, 0, None

    def setup(self, indptr, indices, data):
        self.levels = []
        rebuild = self._aggs is None or self._setups % self.rebuild_every == 0
        self._setups += 1
        if rebuild:
            self._aggs = []
        ptr, idx, dat = np.asarray(indptr), np.asarray(indices, np.int64), np.asarray(data)
        depth = 0
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
            if rebuild:
                agg, nc = aggregate(ptr, idx, dat, self.passes, self.mode, self.matcher)
                if nc >= 0.9 * n or nc < 1:
                    break
                self._aggs.append((agg, nc))
            elif depth < len(self._aggs):
                agg, nc = self._aggs[depth]
            else:
                break
            depth += 1
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


def givens(a, b):
    """The 2x2 rotation that takes ``(a, b)`` to ``(hypot(a, b), 0)``."""
    r = np.hypot(a, b)
    c, s = (a / r, b / r) if r else (1.0, 0.0)
    return np.array([[c, s], [-s, c]])


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
        rot = [None] * restart
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
            for j in range(k):                    # the earlier plane rotations
                H[j:j + 2, k] = rot[j] @ H[j:j + 2, k]
            rot[k] = givens(H[k, k], H[k + 1, k])
            H[k:k + 2, k] = rot[k] @ H[k:k + 2, k]
            g[k:k + 2] = rot[k] @ g[k:k + 2]
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
