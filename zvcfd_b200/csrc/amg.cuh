// Aggregation multigrid for the coupled 4x4 block system, set up and applied on the device.
//
// The method is the reference's own additive-correction multigrid (ACM,
// zvcfd/fv/linear.py:328-518; Hutchinson & Raithby 1986, Notay 2010 pairwise aggregation):
//
//  * aggregation: pairwise matching on coupling strength, `passes` times per level (about
//    4:1), each pass: up to four rounds in which every free node picks its strongest free
//    neighbour (ties: the smallest column) and mutual picks (i < j) become pairs numbered in
//    order of i; then unmatched nodes join their strongest aggregated neighbour, and the
//    rest stay single (linear.py:373-413). Between passes the graph is coarsened by summing
//    strengths per aggregate pair (linear.py:415-433). Strength is the block's Frobenius norm
//    over the geometric mean of the two diagonal blocks' (ACM), or the pressure-pressure
//    entry in the same form (AmgX's `aggregation_edge_weight_component: 3`, linear.py:95-102);
//  * coarse operators: Galerkin with piecewise-constant transfer, the sum of the blocks of
//    each aggregate pair (linear.py:437-454), in a fixed order (deterministic);
//  * smoothing: damped block Jacobi with the inverse of each 4x4 diagonal block, symmetric
//    multicolour block Gauss-Seidel, DILU or ILU(0) on the finest levels, or
//    block-Jacobi-preconditioned Chebyshev polynomials (the largest eigenvalue of D^-1 A by
//    power iteration at set-up);
//  * coarsest level: the explicit inverse of the dense matrix (Gauss-Jordan with partial
//    pivoting in one CTA), or smoothing sweeps when coarsening stalls above that size.
//
// The hierarchy is always built in FP64; the V-cycle runs in FP64, or in FP32 with FP32
// copies of every level's blocks and diagonal inverses (the mixed-precision form: half the
// bytes per cycle, with FP64 kept in the outer FGMRES).
#pragma once

#include <cub/cub.cuh>

#include <vector>

#include "devmem.cuh"
#include "spmv.cuh"

namespace zvfv {
namespace amg {

constexpr int DENSE_MAX = 24;            // block rows of a dense coarsest level (96 x 96:
                                         // matrix and inverse fit one CTA's shared memory)

// ------------------------------------------------------------------ small kernels

__global__ void k_iota64(long long *p, long long n) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) p[i] = i;
}

__global__ void k_fill_int(int *p, long long n, int v) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) p[i] = v;
}

// strength measure of every block: Frobenius norm (mode 0) or |pressure-pressure| (mode 1)
__global__ void k_block_weight(long long nnz, const double *__restrict__ data, int mode,
                               double *__restrict__ w) {
    const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= nnz) return;
    const double *b = data + p * 16;
    if (mode == 1) {
        w[p] = fabs(b[15]);
        return;
    }
    double s = 0.0;        // products rounded separately (no contraction): reproducible on the CPU
#pragma unroll
    for (int e = 0; e < 16; ++e) s = __dadd_rn(s, __dmul_rn(b[e], b[e]));
    w[p] = sqrt(s);
}

// symmetrised coupling weights: ws[p] = (w[p] + w[p^T]) / 2 with p^T the entry (j, i) of the
// entry p = (i, j). On a symmetric pattern with sorted rows, the transpose's q-th entry is the
// entry q of A itself and holds A's block tperm[q], so p^T of tperm[q] is q.
__global__ void k_symmetric_weight(long long nnz, const long long *__restrict__ tperm,
                                   const double *__restrict__ w, double *__restrict__ ws) {
    const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= nnz) return;
    const long long p = tperm[q];
    ws[p] = 0.5 * (w[p] + w[q]);
}

// row of every entry (CSR)
__global__ void k_rows_of(long long n, const long long *__restrict__ indptr, long long *__restrict__ row) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    for (long long p = indptr[i]; p < indptr[i + 1]; ++p) row[p] = i;
}

// diagonal weight per row (0 if the row has no diagonal entry) and diagonal position
__global__ void k_diag_of(long long n, const long long *__restrict__ indptr, const int *__restrict__ idx,
                          const double *__restrict__ w, double *__restrict__ dw,
                          long long *__restrict__ dpos) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double d = 0.0;
    long long pd = -1;
    for (long long p = indptr[i]; p < indptr[i + 1]; ++p)
        if (idx[p] == i) {
            pd = p;
            if (w) d = w[p];
        }
    if (dw) dw[i] = d;
    if (dpos) dpos[i] = pd;
}

__global__ void k_strength(long long nnz, const long long *__restrict__ row, const int *__restrict__ col,
                           const double *__restrict__ w, const double *__restrict__ dw,
                           double *__restrict__ s) {
    const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= nnz) return;
    s[p] = w[p] / sqrt(fmax(dw[row[p]] * dw[col[p]], 1e-300));
}

// every free node's strongest free off-diagonal neighbour (first maximum in column order)
__global__ void k_best_free(long long n, const long long *__restrict__ indptr, const int *__restrict__ idx,
                            const double *__restrict__ s, const int *__restrict__ agg,
                            int *__restrict__ best, int *__restrict__ any) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int b = -1;
    if (agg[i] < 0) {
        double bs = 0.0;
        for (long long p = indptr[i]; p < indptr[i + 1]; ++p) {
            const int j = idx[p];
            if (j == i || agg[j] >= 0) continue;
            if (b < 0 || s[p] > bs) { b = j; bs = s[p]; }
        }
    }
    best[i] = b;
    if (b >= 0) *any = 1;
}

__global__ void k_leaders(long long n, const int *__restrict__ best, int *__restrict__ flag) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int j = best[i];
    flag[i] = (j >= 0 && j > i && best[j] == i) ? 1 : 0;
}

// pairs (i, best[i]) with leader flags take ids nxt + rank (exclusive scan of flags)
__global__ void k_assign_pairs(long long n, const int *__restrict__ best, const int *__restrict__ flag,
                               const int *__restrict__ rank, const int *__restrict__ nxt,
                               int *__restrict__ agg) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || !flag[i]) return;
    const int id = *nxt + rank[i];
    agg[i] = id;
    agg[best[i]] = id;
}

__global__ void k_advance(const int *__restrict__ flag, const int *__restrict__ rank, long long n,
                          int *__restrict__ nxt) {
    if (n > 0) *nxt += rank[n - 1] + flag[n - 1];
}

// unmatched nodes: the aggregate of their strongest aggregated neighbour, or -1
__global__ void k_join(long long n, const long long *__restrict__ indptr, const int *__restrict__ idx,
                       const double *__restrict__ s, const int *__restrict__ agg,
                       int *__restrict__ join) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int to = -1;
    if (agg[i] < 0) {
        double bs = 0.0;
        int bj = -1;
        for (long long p = indptr[i]; p < indptr[i + 1]; ++p) {
            const int j = idx[p];
            if (agg[j] < 0) continue;             // also skips i itself
            if (bj < 0 || s[p] > bs) { bj = j; bs = s[p]; }
        }
        if (bj >= 0) to = agg[bj];
    }
    join[i] = to;
}

__global__ void k_apply_join(long long n, const int *__restrict__ join, int *__restrict__ agg,
                             int *__restrict__ single) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const bool free_ = agg[i] < 0;
    single[i] = (free_ && join[i] < 0) ? 1 : 0;
    if (free_ && join[i] >= 0) agg[i] = join[i];
}

__global__ void k_assign_singles(long long n, const int *__restrict__ single, const int *__restrict__ rank,
                                 const int *__restrict__ nxt, int *__restrict__ agg) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n && single[i]) agg[i] = *nxt + rank[i];
}

__global__ void k_compose(long long n, const int *__restrict__ a, int *__restrict__ total) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) total[i] = a[total[i]];
}

__global__ void k_pair_key(long long m, const long long *__restrict__ row, const int *__restrict__ col,
                           const int *__restrict__ agg, unsigned long long nc,
                           unsigned long long *__restrict__ key) {
    const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p < m) key[p] = (unsigned long long)agg[row[p]] * nc + (unsigned long long)agg[col[p]];
}

__global__ void k_int_key(long long m, const int *__restrict__ a, unsigned long long *__restrict__ key) {
    const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p < m) key[p] = (unsigned long long)a[p];
}

__global__ void k_seg_flags(long long m, const unsigned long long *__restrict__ k, int *__restrict__ f) {
    const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p < m) f[p] = (p == 0 || k[p] != k[p - 1]) ? 1 : 0;
}

__global__ void k_seg_starts(long long m, const int *__restrict__ f, const int *__restrict__ rank,
                             const unsigned long long *__restrict__ k, long long *__restrict__ seg,
                             unsigned long long *__restrict__ ukey) {
    const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p < m && f[p]) {
        seg[rank[p]] = p;
        ukey[rank[p]] = k[p];
    }
}

__global__ void k_seg_end(long long m, long long nseg, long long *__restrict__ seg) {
    seg[nseg] = m;
}

// CSR of unique sorted keys key = row * nc + col
__global__ void k_keys_to_csr(long long nseg, long long nrows, unsigned long long nc,
                              const unsigned long long *__restrict__ ukey, long long *__restrict__ indptr,
                              int *__restrict__ idx) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < nseg) idx[i] = (int)(ukey[i] % nc);
    if (i <= nrows) {
        if (i == nrows) { indptr[nrows] = nseg; return; }
        const unsigned long long target = (unsigned long long)i * nc;
        long long lo = 0, hi = nseg;
        while (lo < hi) {
            const long long mid = (lo + hi) >> 1;
            if (ukey[mid] < target) lo = mid + 1; else hi = mid;
        }
        indptr[i] = lo;
    }
}

// segmented sums of width-W rows in segment order (the original order inside a segment)
__global__ void k_seg_sum(long long nseg, int W, const long long *__restrict__ seg,
                          const long long *__restrict__ perm, const double *__restrict__ src,
                          double *__restrict__ dst) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nseg * W) return;
    const long long s = t / W;
    const int c = (int)(t % W);
    double acc = 0.0;
    for (long long q = seg[s]; q < seg[s + 1]; ++q) acc += src[perm[q] * W + c];
    dst[t] = acc;
}

// The Galerkin sums of 4x4 blocks: dst[s] = sum of src[perm[q]] over q in [seg[s], seg[s+1]),
// in that order (bit-equal to k_seg_sum with W = 16). Sixteen lanes own one coarse block and
// take the segment four entries at a time: the four source indices, then the four blocks'
// entries, are loaded before any is added, so a segment (2-3 fine blocks on average) costs
// two dependent round trips instead of two per entry.
__global__ void __launch_bounds__(256)
k_block_seg_sum(long long nseg, const long long *__restrict__ seg, const long long *__restrict__ perm,
                const double *__restrict__ src, double *__restrict__ dst) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nseg * 16) return;
    const long long s = t / 16;
    const int c = (int)(t % 16);
    const long long q1 = seg[s + 1];
    double acc = 0.0;
    for (long long q = seg[s]; q < q1; q += 4) {
        long long p[4];
        double v[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) p[u] = q + u < q1 ? perm[q + u] : -1;
#pragma unroll
        for (int u = 0; u < 4; ++u) v[u] = p[u] >= 0 ? __ldcs(src + p[u] * 16 + c) : 0.0;
#pragma unroll
        for (int u = 0; u < 4; ++u)
            if (p[u] >= 0) acc += v[u];
    }
    dst[t] = acc;
}

// inverse of every row's 4x4 diagonal block (Gauss-Jordan, partial pivoting); a singular
// block leaves a zero inverse (the row is then not smoothed)
template <typename V>
__global__ void k_dinv(long long n, const double *__restrict__ data, const long long *__restrict__ dpos,
                       V *__restrict__ dinv) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double a[4][8];
    const long long pd = dpos[i];
    for (int r = 0; r < 4; ++r)
        for (int c = 0; c < 4; ++c) {
            a[r][c] = pd >= 0 ? data[pd * 16 + r * 4 + c] : 0.0;
            a[r][4 + c] = r == c ? 1.0 : 0.0;
        }
    bool ok = pd >= 0;
    for (int k = 0; k < 4 && ok; ++k) {
        int piv = k;
        for (int r = k + 1; r < 4; ++r)
            if (fabs(a[r][k]) > fabs(a[piv][k])) piv = r;
        if (!(fabs(a[piv][k]) > 0.0)) { ok = false; break; }
        if (piv != k)
            for (int c = 0; c < 8; ++c) { const double t = a[k][c]; a[k][c] = a[piv][c]; a[piv][c] = t; }
        const double inv = 1.0 / a[k][k];
        for (int c = 0; c < 8; ++c) a[k][c] *= inv;
        for (int r = 0; r < 4; ++r) {
            if (r == k) continue;
            const double f = a[r][k];
            if (f != 0.0)
                for (int c = 0; c < 8; ++c) a[r][c] -= f * a[k][c];
        }
    }
    for (int r = 0; r < 4; ++r)
        for (int c = 0; c < 4; ++c) dinv[i * 16 + r * 4 + c] = (V)(ok ? a[r][4 + c] : 0.0);
}

template <typename A, typename B>
__global__ void k_convert(long long n, const A *__restrict__ src, B *__restrict__ dst) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) dst[i] = (B)src[i];
}

// dense (4n x 4n) copy of a small block-CSR matrix, column-major free: row-major
__global__ void k_densify(long long n, const long long *__restrict__ indptr, const int *__restrict__ idx,
                          const double *__restrict__ data, double *__restrict__ dense) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const long long m = 4 * n;
    for (long long p = indptr[i]; p < indptr[i + 1]; ++p) {
        const int j = idx[p];
        for (int r = 0; r < 4; ++r)
            for (int c = 0; c < 4; ++c) dense[(4 * i + r) * m + 4 * j + c] = data[p * 16 + r * 4 + c];
    }
}

// Gauss-Jordan inverse of an m x m matrix (m <= 128) in shared memory by one CTA, partial
// pivoting; ok[0] = 0 if a pivot vanishes
__global__ void k_dense_inverse(int m, const double *__restrict__ A, double *__restrict__ inv,
                                int *__restrict__ ok) {
    extern __shared__ double sm[];
    double *a = sm;                 // m x m
    double *e = sm + m * m;         // m x m, the inverse being built
    __shared__ int piv;
    __shared__ int bad;
    for (int t = threadIdx.x; t < m * m; t += blockDim.x) {
        a[t] = A[t];
        e[t] = (t / m == t % m) ? 1.0 : 0.0;
    }
    if (threadIdx.x == 0) bad = 0;
    __syncthreads();
    for (int k = 0; k < m; ++k) {
        if (threadIdx.x == 0) {
            int p = k;
            double best = fabs(a[k * m + k]);
            for (int r = k + 1; r < m; ++r)
                if (fabs(a[r * m + k]) > best) { best = fabs(a[r * m + k]); p = r; }
            piv = p;
            if (!(best > 0.0)) bad = 1;
        }
        __syncthreads();
        if (bad) break;
        const int p = piv;
        if (p != k)
            for (int c = threadIdx.x; c < m; c += blockDim.x) {
                double t = a[k * m + c]; a[k * m + c] = a[p * m + c]; a[p * m + c] = t;
                t = e[k * m + c]; e[k * m + c] = e[p * m + c]; e[p * m + c] = t;
            }
        __syncthreads();
        const double d = 1.0 / a[k * m + k];
        __syncthreads();
        for (int c = threadIdx.x; c < m; c += blockDim.x) {
            a[k * m + c] *= d;
            e[k * m + c] *= d;
        }
        __syncthreads();
        for (int t = threadIdx.x; t < m * m; t += blockDim.x) {
            const int r = t / m, c = t % m;
            if (r == k) continue;
            const double f = a[r * m + k];
            if (c != k) a[t] -= f * a[k * m + c];
            e[t] -= f * e[k * m + c];
        }
        __syncthreads();
        for (int r = threadIdx.x; r < m; r += blockDim.x)
            if (r != k) a[r * m + k] = 0.0;
        __syncthreads();
    }
    for (int t = threadIdx.x; t < m * m; t += blockDim.x) inv[t] = e[t];
    if (threadIdx.x == 0) *ok = bad ? 0 : 1;
}

// ------------------------------------------------------------------ V-cycle kernels

// Damped block Jacobi: x_out = x_in + omega D^-1 (b - A x_in); FIRST: x_in = 0 (no product).
// Lane layout of the SpMV (G lanes per row, 4-lane slots), then the four residual components
// are gathered into each lane of slot 0 for the 4x4 inverse.
template <int G, bool FIRST, typename V, typename T>
__global__ void __launch_bounds__(256)
k_jacobi(long long n, const long long *__restrict__ indptr, const int *__restrict__ indices,
         const V *__restrict__ data, const V *__restrict__ dinv, const T *__restrict__ b,
         const T *__restrict__ xin, T *__restrict__ xout, T omega) {
    constexpr int S = G / 4;
    const long long gid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long row = gid / G;
    const int lane = threadIdx.x % G;
    const int slot = lane / 4, r = lane % 4;
    T acc = 0;
    if (!FIRST && row < n) {
        const long long p1 = indptr[row + 1];
        for (long long p = indptr[row] + slot; p < p1; p += S) {
            const int j = __ldcs(indices + p);
            const Vec4<V> a = Vec4<V>::load_stream(data + p * 16 + r * 4);
            const Vec4<T> xv = Vec4<T>::load(xin + (long long)j * 4);
#pragma unroll
            for (int c = 0; c < 4; ++c) acc += (T)a.v[c] * xv.v[c];
        }
    }
    if (!FIRST) {
#pragma unroll
        for (int off = 4; off < G; off <<= 1) acc += __shfl_xor_sync(0xffffffffu, acc, off, G);
    }
    T res = 0;
    if (row < n) res = b[row * 4 + r] - acc;
    // gather the row's 4 residual components (lanes 0..3 of the group hold them)
    const int base = (threadIdx.x % 32) / G * G;
    T rc[4];
#pragma unroll
    for (int c = 0; c < 4; ++c) rc[c] = __shfl_sync(0xffffffffu, res, base + c);
    if (row < n && slot == 0) {
        const Vec4<V> d = Vec4<V>::load(dinv + row * 16 + r * 4);
        T upd = 0;
#pragma unroll
        for (int c = 0; c < 4; ++c) upd += (T)d.v[c] * rc[c];
        const T x0 = FIRST ? (T)0 : xin[row * 4 + r];
        xout[row * 4 + r] = x0 + omega * upd;
    }
}

// The transposed sweep: x_out = x_in + omega D^-T (b - A^T x_in), A^T through the transpose
// structure (tptr, trow, tperm) of the level; D^-T: lane r takes column r of the inverse.
template <int G, bool FIRST, typename V, typename T>
__global__ void __launch_bounds__(256)
k_jacobi_t(long long n, const long long *__restrict__ tptr, const int *__restrict__ trow,
           const long long *__restrict__ tperm, const V *__restrict__ data,
           const V *__restrict__ dinv, const T *__restrict__ b, const T *__restrict__ xin,
           T *__restrict__ xout, T omega) {
    constexpr int S = G / 4;
    const long long gid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long row = gid / G;
    const int lane = threadIdx.x % G;
    const int slot = lane / 4, r = lane % 4;
    T acc = 0;
    if (!FIRST && row < n) {
        const long long q1 = tptr[row + 1];
        for (long long q = tptr[row] + slot; q < q1; q += S) {
            const int i = trow[q];
            const V *blk = data + tperm[q] * 16;
            const Vec4<T> xv = Vec4<T>::load(xin + (long long)i * 4);
#pragma unroll
            for (int c = 0; c < 4; ++c) acc += (T)__ldg(blk + c * 4 + r) * xv.v[c];
        }
    }
    if (!FIRST) {
#pragma unroll
        for (int off = 4; off < G; off <<= 1) acc += __shfl_xor_sync(0xffffffffu, acc, off, G);
    }
    T res = 0;
    if (row < n) res = b[row * 4 + r] - acc;
    const int base = (threadIdx.x % 32) / G * G;
    T rc[4];
#pragma unroll
    for (int c = 0; c < 4; ++c) rc[c] = __shfl_sync(0xffffffffu, res, base + c);
    if (row < n && slot == 0) {
        T upd = 0;
#pragma unroll
        for (int c = 0; c < 4; ++c) upd += (T)dinv[row * 16 + c * 4 + r] * rc[c];
        const T x0 = FIRST ? (T)0 : xin[row * 4 + r];
        xout[row * 4 + r] = x0 + omega * upd;
    }
}

// ------------------------------------------------------------------ Chebyshev smoothing

// One step of block-Jacobi-preconditioned Chebyshev iteration (Saad, Iterative Methods for
// Sparse Linear Systems, 2nd ed., Algorithm 12.1, on D^-1 A; Adams, Brezina, Hu and
// Tuminaro, J. Comput. Phys. 188 (2003), for its use as a multigrid smoother):
//   z = D^-1 (b - A x_in),  d <- cd d + cz z,  x_out = x_in + d.
// The row's update d is kept in place (each row reads and writes only its own four entries);
// FIRST: x_in = 0 and no previous update (x_out = d = cz D^-1 b); cd == 0 starts a sequence
// from a nonzero x_in without reading d. Rows split over G lanes as in the Jacobi sweep.
// TR: the same step on A^T (through the transpose structure) and D^-T.
template <int G, bool FIRST, bool TR, typename V, typename T>
__global__ void __launch_bounds__(256)
k_cheby(long long n, const long long *__restrict__ ptr_, const int *__restrict__ idx,
        const long long *__restrict__ tperm, const V *__restrict__ data,
        const V *__restrict__ dinv, const T *__restrict__ b, const T *__restrict__ xin,
        T *__restrict__ xout, T *__restrict__ d, T cd, T cz) {
    constexpr int S = G / 4;
    const long long gid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long row = gid / G;
    const int lane = threadIdx.x % G;
    const int slot = lane / 4, r = lane % 4;
    T acc = 0;
    if (!FIRST && row < n) {
        const long long p1 = ptr_[row + 1];
        for (long long p = ptr_[row] + slot; p < p1; p += S) {
            const int j = idx[p];
            const Vec4<T> xv = Vec4<T>::load(xin + (long long)j * 4);
            if (TR) {
                const V *blk = data + tperm[p] * 16;
#pragma unroll
                for (int c = 0; c < 4; ++c) acc += (T)__ldg(blk + c * 4 + r) * xv.v[c];
            } else {
                const Vec4<V> a = Vec4<V>::load_stream(data + p * 16 + r * 4);
#pragma unroll
                for (int c = 0; c < 4; ++c) acc += (T)a.v[c] * xv.v[c];
            }
        }
    }
    // every lane of the warp takes part in the full-mask shuffles, rows beyond n included
    if (!FIRST) {
#pragma unroll
        for (int off = 4; off < G; off <<= 1) acc += __shfl_xor_sync(0xffffffffu, acc, off, G);
    }
    T res = 0;
    if (row < n) res = b[row * 4 + r] - acc;
    const int base = (threadIdx.x % 32) / G * G;
    T rc[4];
#pragma unroll
    for (int c = 0; c < 4; ++c) rc[c] = __shfl_sync(0xffffffffu, res, base + c);
    if (row < n && slot == 0) {
        T z = 0;
#pragma unroll
        for (int c = 0; c < 4; ++c) z += (T)dinv[row * 16 + (TR ? c * 4 + r : r * 4 + c)] * rc[c];
        const long long i = row * 4 + r;
        T step = cz * z;
        if (!FIRST && cd != (T)0) step += cd * d[i];
        d[i] = step;
        xout[i] = (FIRST ? (T)0 : xin[i]) + step;
    }
}

// Per-CTA partial sums of squares of v[0..m) (a fixed grid: the fold is deterministic).
template <typename T>
__global__ void __launch_bounds__(256) k_sumsq(long long m, const T *__restrict__ v,
                                               double *__restrict__ partial) {
    __shared__ double red[8];
    double s = 0.0;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < m;
         i += (long long)gridDim.x * blockDim.x) {
        const double e = (double)v[i];
        s += e * e;
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
    if (threadIdx.x % 32 == 0) red[threadIdx.x / 32] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < (int)(blockDim.x / 32); ++w) t += red[w];
        partial[blockIdx.x] = t;
    }
}

// out = in / sqrt(sum of the nparts partials) (every CTA folds the partials in one order).
template <typename T>
__global__ void __launch_bounds__(256) k_scale_by(long long m, int nparts,
                                                  const double *__restrict__ partial,
                                                  const T *__restrict__ in, T *__restrict__ out) {
    __shared__ double inv;
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int k = 0; k < nparts; ++k) t += partial[k];
        inv = t > 0.0 ? 1.0 / sqrt(t) : 0.0;
    }
    __syncthreads();
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < m;
         i += (long long)gridDim.x * blockDim.x)
        out[i] = (T)((double)in[i] * inv);
}

// A deterministic start vector for the power iteration: values in [0.5, 1.5) from a hash of
// the index (positive, so that it is not orthogonal to the dominant eigenvector of D^-1 A).
template <typename T>
__global__ void k_fill_start(long long m, T *__restrict__ v) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m) return;
    unsigned long long h = (unsigned long long)i * 0x9E3779B97F4A7C15ull + 0x632BE59BD9B4E019ull;
    h ^= h >> 31;
    h *= 0xBF58476D1CE4E5B9ull;
    h ^= h >> 27;
    v[i] = (T)(0.5 + (double)(h >> 11) * (1.0 / 9007199254740992.0));
}

// ------------------------------------------------------------------ multicolour DILU

// Inverse of a 4x4 block by Gauss-Jordan with partial pivoting: false (and inv = 0) if singular.
__device__ inline bool invert4(const double (&m)[16], double (&inv)[16]) {
    double a[4][8];
#pragma unroll
    for (int r = 0; r < 4; ++r)
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            a[r][c] = m[r * 4 + c];
            a[r][4 + c] = r == c ? 1.0 : 0.0;
        }
    bool ok = true;
    for (int k = 0; k < 4 && ok; ++k) {
        int piv = k;
        for (int r = k + 1; r < 4; ++r)
            if (fabs(a[r][k]) > fabs(a[piv][k])) piv = r;
        if (!(fabs(a[piv][k]) > 0.0)) {
            ok = false;
            break;
        }
        if (piv != k)
            for (int c = 0; c < 8; ++c) {
                const double t = a[k][c];
                a[k][c] = a[piv][c];
                a[piv][c] = t;
            }
        const double s = 1.0 / a[k][k];
        for (int c = 0; c < 8; ++c) a[k][c] *= s;
        for (int r = 0; r < 4; ++r) {
            if (r == k) continue;
            const double f = a[r][k];
            if (f != 0.0)
                for (int c = 0; c < 8; ++c) a[r][c] -= f * a[k][c];
        }
    }
#pragma unroll
    for (int r = 0; r < 4; ++r)
#pragma unroll
        for (int c = 0; c < 4; ++c) inv[r * 4 + c] = ok ? a[r][4 + c] : 0.0;
    return ok;
}

// The DILU diagonal of one colour, after the earlier colours' (AmgX's MULTICOLOR_DILU, the
// reference's `dilu` presets, zvcfd/fv/linear.py:571-608):
//   E_i = A_ii - sum over neighbours j of an earlier colour of A_ij E_j^-1 A_ji,
// on a colour-ordered level (colour = the contiguous rows [first, first + count); an earlier
// colour's rows lie below first). The blocks are read in FP64 from the level's own numbering
// (psrc: the source of every colour-ordered block; ptrans: the colour-ordered position of the
// transposed block, -1 if absent); E_i^-1 is written in FP64 (a singular E leaves a zero
// inverse: the row is not smoothed). One thread per row; launched colour by colour in order.
__global__ void __launch_bounds__(128)
k_dilu_factor(long long count, long long first, const long long *__restrict__ pptr,
              const int *__restrict__ pidx, const long long *__restrict__ psrc,
              const long long *__restrict__ ptrans, const long long *__restrict__ pdpos,
              const double *__restrict__ data, double *__restrict__ einv) {
    const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= count) return;
    const long long row = first + k;
    double E[16];
    const long long pd = pdpos[row];
#pragma unroll
    for (int e = 0; e < 16; ++e) E[e] = pd >= 0 ? data[psrc[pd] * 16 + e] : 0.0;
    for (long long q = pptr[row]; q < pptr[row + 1]; ++q) {
        const int j = pidx[q];
        const long long qt = ptrans[q];
        if (j >= first || qt < 0) continue;
        const double *Aij = data + psrc[q] * 16, *Aji = data + psrc[qt] * 16;
        const double *Ej = einv + (long long)j * 16;
        double T[16];                                   // T = E_j^-1 A_ji
#pragma unroll
        for (int r = 0; r < 4; ++r)
#pragma unroll
            for (int c = 0; c < 4; ++c) {
                double s = 0.0;
#pragma unroll
                for (int m = 0; m < 4; ++m) s += Ej[r * 4 + m] * Aji[m * 4 + c];
                T[r * 4 + c] = s;
            }
#pragma unroll
        for (int r = 0; r < 4; ++r)
#pragma unroll
            for (int c = 0; c < 4; ++c) {
                double s = 0.0;
#pragma unroll
                for (int m = 0; m < 4; ++m) s += Aij[r * 4 + m] * T[m * 4 + c];
                E[r * 4 + c] -= s;
            }
    }
    double inv[16];
    invert4(E, inv);
#pragma unroll
    for (int e = 0; e < 16; ++e) einv[row * 16 + e] = inv[e];
}

// One colour of the solve M z = r of a multicolour factorisation smoother, on a
// colour-ordered level (L, U: the blocks of earlier and later colours).
// DILU (ILU false): M = (E + L) E^-1 (E + U), E^-1 per row in `dinv` (row-indexed):
//   forward (colours in order):     w_i = E_i^-1 (r_i - sum_{j earlier} A_ij w_j)
//   backward (colours in reverse):  z_i = w_i - E_i^-1 sum_{j later} A_ij z_j
// ILU(0) (ILU true): M = L U, `data` the factored blocks (L_ij below the colour, U_ij above,
// U_ii^-1 at the diagonal position pdpos[i]):
//   forward:  w_i = r_i - sum_{j earlier} L_ij w_j
//   backward: z_i = U_ii^-1 (w_i - sum_{j later} U_ij z_j)
// and x_i += omega z_i in the backward pass (w and z share the vector wz). Rows split over G
// lanes as in the Gauss-Seidel sweep; a lane loads only the blocks on its side of the colour
// (each pass reads half the level's blocks).
template <int G, bool BACKWARD, bool ILU, typename V, typename T>
__global__ void __launch_bounds__(256)
k_lu_colour(long long count, long long first, const long long *__restrict__ pptr,
            const int *__restrict__ pidx, const long long *__restrict__ pdpos,
            const V *__restrict__ data, const V *__restrict__ dinv, const T *__restrict__ r,
            T *__restrict__ wz, T *__restrict__ x, T omega) {
    constexpr int S = G / 4;
    const long long gid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long k = gid / G;
    const int lane = threadIdx.x % G;
    const int slot = lane / 4, rr = lane % 4;
    const bool on = k < count;
    const long long row = first + (on ? k : 0);
    const long long last = first + count;
    T acc = 0;
    if (on) {
        const long long p1 = pptr[row + 1];
        for (long long p = pptr[row] + slot; p < p1; p += S) {
            const int j = __ldcs(pidx + p);
            if (BACKWARD ? j < last : j >= first) continue;
            const Vec4<V> a = Vec4<V>::load_stream(data + p * 16 + rr * 4);
            const T *v = wz + (long long)j * 4;
#pragma unroll
            for (int c = 0; c < 4; ++c) acc += (T)a.v[c] * v[c];
        }
    }
#pragma unroll
    for (int off = 4; off < G; off <<= 1) acc += __shfl_xor_sync(0xffffffffu, acc, off, G);
    const long long i = row * 4 + rr;
    T lhs = 0;
    if (on) lhs = BACKWARD ? (ILU ? wz[i] - acc : acc) : r[i] - acc;
    const int base = (threadIdx.x % 32) / G * G;
    T rc[4];
#pragma unroll
    for (int c = 0; c < 4; ++c) rc[c] = __shfl_sync(0xffffffffu, lhs, base + c);
    if (on && slot == 0) {
        if (ILU && !BACKWARD) {
            wz[i] = lhs;
            return;
        }
        // ILU: a row without a diagonal block (none in these systems) is not smoothed
        const long long pd = ILU ? pdpos[row] : 0;
        T s = 0;
        if (pd >= 0) {
            const V *dr = ILU ? data + pd * 16 : dinv + row * 16;
            const Vec4<V> d = Vec4<V>::load(dr + rr * 4);
#pragma unroll
            for (int c = 0; c < 4; ++c) s += (T)d.v[c] * rc[c];
        }
        if (BACKWARD) {
            const T z = ILU ? s : wz[i] - s;
            wz[i] = z;
            x[i] += omega * z;
        } else {
            wz[i] = s;
        }
    }
}

// Multicolour ILU(0) of one colour, after the earlier colours' rows (AmgX's MULTICOLOR_ILU
// with sparsity level 0 of the reference's `robust` preset, zvcfd/fv/linear.py:571-611): on the
// colour-ordered level, row i (this colour) is copied from the FP64 blocks (psrc) and, for each
// of its neighbours k of an earlier colour in increasing order, L_ik = a_ik U_kk^-1 and
// a_ij -= L_ik U_kj for every j > k of row k that row i holds (no fill); then U_ii is inverted
// in place. Rows of one colour are not coupled, so a colour's rows factor independently; one
// thread per row.
__global__ void __launch_bounds__(128)
k_ilu_factor(long long count, long long first, const long long *__restrict__ pptr,
             const int *__restrict__ pidx, const long long *__restrict__ psrc,
             const long long *__restrict__ pdpos, const double *__restrict__ data,
             double *__restrict__ lu) {
    const long long k0 = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (k0 >= count) return;
    const long long row = first + k0;
    const long long q0 = pptr[row], q1 = pptr[row + 1];
    for (long long q = q0; q < q1; ++q)
        for (int e = 0; e < 16; ++e) lu[q * 16 + e] = data[psrc[q] * 16 + e];
    int prev = -1;
    for (;;) {
        // the next neighbour of an earlier colour, by increasing position
        long long qk = -1;
        int kk = (int)first;
        for (long long q = q0; q < q1; ++q) {
            const int j = pidx[q];
            if (j > prev && j < kk) {
                kk = j;
                qk = q;
            }
        }
        if (qk < 0) break;
        prev = kk;
        if (pdpos[kk] < 0) continue;                    // no diagonal block: nothing to divide by
        const double *Ukk = lu + pdpos[kk] * 16;       // the inverse, already in place
        double L[16];
        double *a = lu + qk * 16;
#pragma unroll
        for (int r = 0; r < 4; ++r)
#pragma unroll
            for (int c = 0; c < 4; ++c) {
                double s = 0.0;
#pragma unroll
                for (int m = 0; m < 4; ++m) s += a[r * 4 + m] * Ukk[m * 4 + c];
                L[r * 4 + c] = s;
            }
#pragma unroll
        for (int e = 0; e < 16; ++e) a[e] = L[e];
        for (long long q2 = pptr[kk]; q2 < pptr[kk + 1]; ++q2) {
            const int j = pidx[q2];
            if (j <= kk) continue;
            long long q3 = -1;
            for (long long q = q0; q < q1; ++q)
                if (pidx[q] == j) {
                    q3 = q;
                    break;
                }
            if (q3 < 0) continue;
            const double *Ukj = lu + q2 * 16;
            double *aij = lu + q3 * 16;
#pragma unroll
            for (int r = 0; r < 4; ++r)
#pragma unroll
                for (int c = 0; c < 4; ++c) {
                    double s = 0.0;
#pragma unroll
                    for (int m = 0; m < 4; ++m) s += L[r * 4 + m] * Ukj[m * 4 + c];
                    aij[r * 4 + c] -= s;
                }
        }
    }
    const long long pd = pdpos[row];
    if (pd < 0) return;
    double D[16], inv[16];
#pragma unroll
    for (int e = 0; e < 16; ++e) D[e] = lu[pd * 16 + e];
    invert4(D, inv);
#pragma unroll
    for (int e = 0; e < 16; ++e) lu[pd * 16 + e] = inv[e];
}

// ------------------------------------------------------------------ multicolour Gauss-Seidel

// In-place block Gauss-Seidel over the rows of one colour (rows[0..count)): rows of a colour
// are not coupled, so x_i <- x_i + omega D_i^-1 (b_i - (A x)_i) is a Jacobi step within the
// colour and a Gauss-Seidel step across colours. A colour holds only a fraction of the rows,
// so one launch is a few waves at most and the sweep is latency-bound: each lane keeps
// several blocks (and their column indices) in flight before it uses them, and the register
// budget is held to 40 so that six 256-thread blocks fit on an SM (four FP32 blocks, or two
// FP64 blocks, per lane fit in it without spilling).
template <typename V>
__host__ __device__ constexpr int gs_inflight() { return sizeof(V) == 4 ? 4 : 2; }

// CONTIG: the colour is the contiguous row range [first, first + count) of a colour-ordered
// copy (rows unused); otherwise its rows are rows[0..count) of the original numbering.
template <int G, bool CONTIG, typename V, typename T>
__global__ void __launch_bounds__(256, 6)
k_gs_colour(long long count, long long first, const int *__restrict__ rows,
            const long long *__restrict__ indptr, const int *__restrict__ indices,
            const V *__restrict__ data, const V *__restrict__ dinv, const T *__restrict__ b,
            T *__restrict__ x, T omega) {
    constexpr int S = G / 4;
    constexpr int U = gs_inflight<V>();
    const long long gid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long k = gid / G;
    const int lane = threadIdx.x % G;
    const int slot = lane / 4, r = lane % 4;
    const long long row = k < count ? (CONTIG ? first + k : (long long)rows[k]) : 0;
    T acc = 0;
    if (k < count) {
        const long long p1 = indptr[row + 1];
        for (long long p = indptr[row] + slot; p < p1; p += S * U) {
            int j[U];
            Vec4<V> a[U];
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const long long q = p + u * S;
                j[u] = q < p1 ? __ldcs(indices + q) : -1;
                if (q < p1) a[u] = Vec4<V>::load_stream(data + q * 16 + r * 4);
            }
#pragma unroll
            for (int u = 0; u < U; ++u) {
                if (j[u] < 0) continue;
                const T *xj = x + (long long)j[u] * 4;      // plain loads: x changes in the sweep
#pragma unroll
                for (int c = 0; c < 4; ++c) acc += (T)a[u].v[c] * xj[c];
            }
        }
    }
#pragma unroll
    for (int off = 4; off < G; off <<= 1) acc += __shfl_xor_sync(0xffffffffu, acc, off, G);
    T res = 0;
    if (k < count) res = b[row * 4 + r] - acc;
    const int base = (threadIdx.x % 32) / G * G;
    T rc[4];
#pragma unroll
    for (int c = 0; c < 4; ++c) rc[c] = __shfl_sync(0xffffffffu, res, base + c);
    if (k < count && slot == 0) {
        const Vec4<V> d = Vec4<V>::load(dinv + row * 16 + r * 4);
        T upd = 0;
#pragma unroll
        for (int c = 0; c < 4; ++c) upd += (T)d.v[c] * rc[c];
        x[row * 4 + r] += omega * upd;
    }
}

// Blocks per slot the colour sweep requests before it waits for the previous colour (16 lanes
// per row: the first 16 FP64 or 32 FP32 blocks of the row). Measured on the 400k-node tube
// against the launch-per-colour kernel without prefetch: a V-cycle 3.72 -> 3.07 ms (FP64) and
// 2.75 -> 2.01 ms (FP32 hierarchy); 1 and 2 gain less, 6 and 8 cost occupancy.
#ifndef ZV_GS_PREFETCH
#define ZV_GS_PREFETCH 4
#endif
template <typename V>
__host__ __device__ constexpr int gs_prefetch_depth() {
    return sizeof(V) == 4 ? 2 * ZV_GS_PREFETCH : ZV_GS_PREFETCH;
}

// The colour sweep launched as a programmatic dependent of the previous colour (PDL): a
// colour's blocks, column indices and 4x4 inverses do not depend on the previous colour's
// update, so each CTA lets the next colour's grid launch at once
// (griddepcontrol.launch_dependents), requests the first DEPTH blocks of every slot and its
// row's inverse, and only then waits for the previous grid to complete and flush
// (griddepcontrol.wait) before it reads b and gathers x. The next colour's CTAs thus fill the
// SMs as this colour's last wave drains, with their block loads already in flight. Launched
// without the programmatic attribute, both instructions are no-ops. The sums are those of
// k_gs_colour (same slots, same order), bit for bit.
template <int G, int DEPTH, typename V, typename T>
__global__ void __launch_bounds__(256)
k_gs_colour_pdl(long long count, long long first, const long long *__restrict__ indptr,
                const int *__restrict__ indices, const V *__restrict__ data,
                const V *__restrict__ dinv, const T *__restrict__ b, T *__restrict__ x,
                T omega) {
    constexpr int S = G / 4;
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    const long long gid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long k = gid / G;
    const int lane = threadIdx.x % G;
    const int slot = lane / 4, r = lane % 4;
    const bool on = k < count;
    const long long row = first + (on ? k : 0);
    long long p0 = 0, p1 = 0;
    Vec4<V> d;
    int j[DEPTH];
    Vec4<V> a[DEPTH];
    if (on) {
        p0 = indptr[row];
        p1 = indptr[row + 1];
        if (slot == 0) d = Vec4<V>::load(dinv + row * 16 + r * 4);
#pragma unroll
        for (int u = 0; u < DEPTH; ++u) {
            const long long q = p0 + slot + (long long)u * S;
            j[u] = q < p1 ? __ldcs(indices + q) : -1;
            if (q < p1) a[u] = Vec4<V>::load_stream(data + q * 16 + r * 4);
        }
    }
    asm volatile("griddepcontrol.wait;" ::: "memory");
    T acc = 0, bi = 0;
    if (on) {
        if (slot == 0) bi = b[row * 4 + r];
#pragma unroll
        for (int u = 0; u < DEPTH; ++u) {
            if (j[u] < 0) continue;
            const T *xj = x + (long long)j[u] * 4;
#pragma unroll
            for (int c = 0; c < 4; ++c) acc += (T)a[u].v[c] * xj[c];
        }
        // rows longer than the first DEPTH blocks per slot: the rest, one block at a time
        for (long long q = p0 + slot + (long long)DEPTH * S; q < p1; q += S) {
            const int jj = __ldcs(indices + q);
            const Vec4<V> aa = Vec4<V>::load_stream(data + q * 16 + r * 4);
            const T *xj = x + (long long)jj * 4;
#pragma unroll
            for (int c = 0; c < 4; ++c) acc += (T)aa.v[c] * xj[c];
        }
    }
#pragma unroll
    for (int off = 4; off < G; off <<= 1) acc += __shfl_xor_sync(0xffffffffu, acc, off, G);
    const int base = (threadIdx.x % 32) / G * G;
    const T res = __shfl_sync(0xffffffffu, bi, base + r) - acc;
    T rc[4];
#pragma unroll
    for (int c = 0; c < 4; ++c) rc[c] = __shfl_sync(0xffffffffu, res, base + c);
    if (on && slot == 0) {
        T upd = 0;
#pragma unroll
        for (int c = 0; c < 4; ++c) upd += (T)d.v[c] * rc[c];
        x[row * 4 + r] += omega * upd;
    }
}

// colour-ordered copies: out[q] = data[src[q]] for 4x4 blocks (two doubles per thread)
template <typename V>
__global__ void k_gather_blocks(long long nnz, const long long *__restrict__ src,
                                const double *__restrict__ data, V *__restrict__ out) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nnz * 8) return;
    const long long q = t / 8;
    const int h = (int)(t % 8);
    const double2 v = __ldcs(reinterpret_cast<const double2 *>(data + src[q] * 16) + h);
    out[q * 16 + 2 * h] = (V)v.x;
    out[q * 16 + 2 * h + 1] = (V)v.y;
}

// dst[k * W + e] = src[idx[k] * W + e] (GATHER) or dst[idx[k] * W + e] = src[k * W + e]
template <bool GATHER, typename A, typename B>
__global__ void k_permute_rows(long long n, int W, const int *__restrict__ idx,
                               const A *__restrict__ src, B *__restrict__ dst) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n * W) return;
    const long long k = t / W;
    const int e = (int)(t % W);
    const long long j = idx[k];
    if (GATHER) dst[t] = (B)src[j * W + e];
    else dst[j * W + e] = (B)src[t];
}

// dst[k] = src[idx[k]]
__global__ void k_gather_int(long long n, const int *__restrict__ idx, const int *__restrict__ src,
                             int *__restrict__ dst) {
    const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n) dst[k] = src[idx[k]];
}

// the same sweep on A^T (columns of A through the transpose structure, D^-T)
template <int G, typename V, typename T>
__global__ void __launch_bounds__(256)
k_gs_colour_t(long long count, const int *__restrict__ rows, const long long *__restrict__ tptr,
              const int *__restrict__ trow, const long long *__restrict__ tperm,
              const V *__restrict__ data, const V *__restrict__ dinv, const T *__restrict__ b,
              T *__restrict__ x, T omega) {
    constexpr int S = G / 4;
    const long long gid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long k = gid / G;
    const int lane = threadIdx.x % G;
    const int slot = lane / 4, r = lane % 4;
    const long long row = k < count ? rows[k] : 0;
    T acc = 0;
    if (k < count) {
        const long long q1 = tptr[row + 1];
        for (long long q = tptr[row] + slot; q < q1; q += S) {
            const int i = trow[q];
            const V *blk = data + tperm[q] * 16;
            const T *xi = x + (long long)i * 4;
#pragma unroll
            for (int c = 0; c < 4; ++c) acc += (T)__ldg(blk + c * 4 + r) * xi[c];
        }
    }
#pragma unroll
    for (int off = 4; off < G; off <<= 1) acc += __shfl_xor_sync(0xffffffffu, acc, off, G);
    T res = 0;
    if (k < count) res = b[row * 4 + r] - acc;
    const int base = (threadIdx.x % 32) / G * G;
    T rc[4];
#pragma unroll
    for (int c = 0; c < 4; ++c) rc[c] = __shfl_sync(0xffffffffu, res, base + c);
    if (k < count && slot == 0) {
        T upd = 0;
#pragma unroll
        for (int c = 0; c < 4; ++c) upd += (T)dinv[row * 16 + c * 4 + r] * rc[c];
        x[row * 4 + r] += omega * upd;
    }
}

// coarse residual: rc[I] = sum over the aggregate's members (ascending) of r[i]
template <typename T>
__global__ void k_restrict(long long nc, const long long *__restrict__ mptr, const int *__restrict__ mem,
                           const T *__restrict__ r, T *__restrict__ rc) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nc * 4) return;
    const long long I = t / 4;
    const int c = (int)(t % 4);
    T acc = 0;
    for (long long q = mptr[I]; q < mptr[I + 1]; ++q) acc += r[(long long)mem[q] * 4 + c];
    rc[t] = acc;
}

template <typename T>
__global__ void k_prolong_add(long long n, const int *__restrict__ agg, const T *__restrict__ e,
                              T *__restrict__ x) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n * 4) return;
    const long long i = t / 4;
    x[t] += e[(long long)agg[i] * 4 + (t % 4)];
}

// x = inv b (TRANS: inv^T b) for a dense coarsest level (m x m), one warp per output row
template <typename V, typename T, bool TRANS = false>
__global__ void k_dense_apply(int m, const V *__restrict__ inv, const T *__restrict__ b, T *__restrict__ x) {
    const int row = (blockIdx.x * blockDim.x + threadIdx.x) / 32;
    const int lane = threadIdx.x % 32;
    if (row >= m) return;
    T acc = 0;
    for (int c = lane; c < m; c += 32)
        acc += (T)inv[TRANS ? (long long)c * m + row : (long long)row * m + c] * b[c];
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, off);
    if (lane == 0) x[row] = acc;
}

// ------------------------------------------------------------------ host-side structures

struct Level {
    long long n = 0, nnz = 0;
    const long long *indptr = nullptr;
    const int *indices = nullptr;
    const double *data = nullptr;         // FP64 blocks (level 0: the caller's matrix)
    double *own = nullptr;                // a coarse level's own FP64 blocks
    long long *dpos = nullptr;
    long long *rows = nullptr;            // row of every entry
    long long *tptr = nullptr, *tperm = nullptr;   // the transpose's structure (adjoint)
    int *trow = nullptr;
    double *dinv64 = nullptr;
    float *data32 = nullptr, *dinv32 = nullptr;
    int lanes = 8;
    int gs_depth = 1;                     // Gauss-Seidel blocks in flight: 0 half, 1 base, 2 double
    // transfer to the next level (kept while the aggregation is kept)
    int *agg = nullptr;
    long long nc = 0;
    long long *mptr = nullptr;
    int *mem = nullptr;
    long long *gperm = nullptr, *gseg = nullptr;   // Galerkin: fine blocks by coarse key
    long long cnnz = 0;
    // multicolour Gauss-Seidel: rows sorted by colour, first row of each colour (host)
    int *gs_rows = nullptr;
    std::vector<long long> gs_off;
    // the Gauss-Seidel levels' colour-ordered copy: row k is row gs_rows[k], its blocks in
    // their original order with columns renumbered, so a colour is one contiguous row range
    // (a sweep streams it like an SpMV) and every sum keeps its original order
    long long *pptr = nullptr, *psrc = nullptr, *pdpos = nullptr;   // psrc: source block
    int *pidx = nullptr, *pinv = nullptr;                           // pinv: row -> position
    int *pagg = nullptr, *pmem = nullptr;        // aggregate of each position; members renumbered
    long long *ptrans = nullptr;                 // DILU: the position of each block's transpose
    double *lu64 = nullptr;                      // ILU(0): the factored colour-ordered blocks
    float *lu32 = nullptr;
    double *pdata64 = nullptr, *pdinv64 = nullptr;
    float *pdata32 = nullptr, *pdinv32 = nullptr;
    void *pb = nullptr;                          // the level's right-hand side, colour-ordered
    // Chebyshev smoothing: the estimated largest eigenvalue of D^-1 A (power iteration)
    double cheb_lmax = 0.0;
    // dense coarsest
    bool dense = false;
    double *inv64 = nullptr;
    float *inv32 = nullptr;
    // cycle vectors
    void *x = nullptr, *x2 = nullptr, *b = nullptr, *r = nullptr;
};

struct Params {
    int precision = 0;       // 0 FP64 cycle, 1 FP32 cycle
    int smoother = 1;        // 0 damped block Jacobi, 1 symmetric multicolour block Gauss-Seidel,
                             // 2 block-Jacobi-preconditioned Chebyshev (sweeps = degree),
                             // 3 multicolour DILU, 4 multicolour ILU(0) on the colour-ordered
                             // levels (Jacobi below)
    int gs_levels = 2;       // with Gauss-Seidel: the finest levels that use it (Jacobi below)
    int jacobi_sweeps = 2;   // damped block-Jacobi sweeps (pre and post) below them
    double jacobi_omega = 0.7;
    int strength = 2;        // 0 block norm, 1 pressure-pressure entry, 2 symmetrised block norm
    int passes = 2;
    int presweeps = 2, postsweeps = 2;
    double omega = 0.7;
    int coarse_sweeps = 8;
    int max_levels = 25;
    int rebuild_every = 0;   // > 0: re-aggregate every this many set-ups; 0: adaptively
    double rebuild_ratio = 1.5;   // adaptive: rebuild after a solve needing more iterations
    int autotune = 0;        // 1: time each level's smoother at 8, 16 and 32 lanes per row
    double cheb_ratio = 4.0;    // Chebyshev: the interval [hi / ratio, hi], hi = 1.1 lambda_max
    int cheb_power = 10;        // power-iteration steps estimating lambda_max of D^-1 A
};

inline int lanes_for(long long n, long long nnz) {
    const double per = n ? (double)nnz / n : 0.0;
    return per > 40 ? 32 : (per > 12 ? 16 : 8);
}

}  // namespace amg
}  // namespace zvfv
