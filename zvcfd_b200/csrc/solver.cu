// The linear back end: FGMRES (right-preconditioned, flexible) around the aggregation
// multigrid of amg.cuh, behind an opaque handle in the manner of the reference's AmgX binding
// (zvcfd/fv/linear.py:681-955): create, set up for a matrix (structure on the first call,
// coefficients later), solve, one V-cycle, destroy.
//
// FGMRES follows zvcfd/fv/linear.py:172-320: restart length `restart`, classical Gram-Schmidt
// with one reorthogonalisation pass (CGS2), convergence when the residual has fallen by
// `rtol` relative to the initial one or to round-off (1e-13 ||b||), and the rank-one terms
// u w^T of lumped outlets applied in every product. The Arnoldi step runs in three fused
// passes over the basis (dots; update + dots; update + norm) with deterministic two-stage
// reductions, and the Hessenberg matrix, its Givens rotations and the residual estimate stay
// on the device: the host reads 3 numbers per Krylov step.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "amg.cuh"

extern "C" int zvfv_bsr_transpose(int64_t n, int64_t nnz, const int64_t *indptr,
                                  const int32_t *indices, int64_t *tptr, int32_t *trow,
                                  int64_t *tperm, void *stream);

namespace zvfv {

using namespace amg;

namespace {

constexpr int MAXV = 32;         // basis vectors per reduction (restart + 1 <= 32)
constexpr int DOT_THREADS = 256;

__device__ inline double warp_sum(double v) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
    return v;
}

// partial[cta][j] = sum over the CTA's rows of V[j][i] * w[i], j < nv (MODE 0)
// MODE 1: w -= sum_j h[j] V[j] first, then the dots with the updated w
// MODE 2: w -= sum_j h[j] V[j], then partial[cta][0] = ||w||^2
template <int MODE>
__global__ void __launch_bounds__(DOT_THREADS)
k_arnoldi_pass(long long n, const double *__restrict__ V, long long ldv, int nv,
               const double *__restrict__ h, double *__restrict__ w, double *__restrict__ partial) {
    double acc[MAXV];
#pragma unroll
    for (int j = 0; j < MAXV; ++j) acc[j] = 0.0;
    __shared__ double hs[MAXV];
    if (MODE > 0 && threadIdx.x < MAXV) hs[threadIdx.x] = threadIdx.x < nv ? h[threadIdx.x] : 0.0;
    __syncthreads();
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        double wi = w[i];
        if (MODE > 0) {
            double s = 0.0;
#pragma unroll
            for (int j = 0; j < MAXV; ++j)
                if (j < nv) s += hs[j] * V[j * ldv + i];
            wi -= s;
            w[i] = wi;
        }
        if (MODE < 2) {
#pragma unroll
            for (int j = 0; j < MAXV; ++j)
                if (j < nv) acc[j] += V[j * ldv + i] * wi;
        } else {
            acc[0] += wi * wi;
        }
    }
    __shared__ double red[DOT_THREADS / 32][MAXV];
    const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
    const int cols = MODE < 2 ? nv : 1;
#pragma unroll
    for (int j = 0; j < MAXV; ++j)
        if (j < cols) {
            const double v = warp_sum(acc[j]);
            if (lane == 0) red[warp][j] = v;
        }
    __syncthreads();
    if (threadIdx.x < cols) {
        double v = 0.0;
        for (int q = 0; q < DOT_THREADS / 32; ++q) v += red[q][threadIdx.x];
        partial[(long long)blockIdx.x * MAXV + threadIdx.x] = v;
    }
}

// out[j] = sum over CTAs of partial[cta][j], one warp per column (launched with 32 * MAXV
// threads): lane l adds the CTAs l, l + 32, ... in order, then a fixed butterfly adds the lanes,
// so the result does not depend on scheduling. A single thread per column walking all CTAs
// was a chain of several hundred dependent loads.
__global__ void k_fold_cols(int ncta, int cols, const double *__restrict__ partial, double *__restrict__ out) {
    const int j = threadIdx.x / 32, lane = threadIdx.x % 32;
    if (j >= cols) return;
    double v = 0.0;
    for (int c = lane; c < ncta; c += 32) v += partial[(long long)c * MAXV + j];
    v = warp_sum(v);
    if (lane == 0) out[j] = v;
}

// partial dots of two vectors (a . b), MAXV-strided partials in column 0
__global__ void __launch_bounds__(DOT_THREADS)
k_dot_partial(long long n, const double *__restrict__ a, const double *__restrict__ b,
              double *__restrict__ partial) {
    double acc = 0.0;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
        acc += a[i] * b[i];
    __shared__ double red[DOT_THREADS / 32];
    acc = warp_sum(acc);
    if (threadIdx.x % 32 == 0) red[threadIdx.x / 32] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double v = 0.0;
        for (int q = 0; q < DOT_THREADS / 32; ++q) v += red[q];
        partial[(long long)blockIdx.x * MAXV] = v;
    }
}

// Column k of the Hessenberg matrix from the two Gram-Schmidt passes and ||w||, the earlier
// Givens rotations applied, a new one formed, the residual estimate updated.
// st: [0] |g[k+1]|, [1] h_{k+1,k}, [2] 1/h_{k+1,k} (0 if it vanished)
__global__ void k_arnoldi_finish(int k, int ldh, const double *__restrict__ h1,
                                 const double *__restrict__ h2, const double *__restrict__ nrm2,
                                 double *__restrict__ H, double *__restrict__ cs, double *__restrict__ sn,
                                 double *__restrict__ g, double *__restrict__ st) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double *col = H + (long long)k * ldh;          // column k, rows 0..k+1
    for (int j = 0; j <= k; ++j) col[j] = h1[j] + h2[j];
    const double hn = sqrt(nrm2[0]);
    col[k + 1] = hn;
    for (int j = 0; j < k; ++j) {
        const double t = cs[j] * col[j] + sn[j] * col[j + 1];
        col[j + 1] = -sn[j] * col[j] + cs[j] * col[j + 1];
        col[j] = t;
    }
    const double den = hypot(col[k], col[k + 1]);
    if (den != 0.0) {
        cs[k] = col[k] / den;
        sn[k] = col[k + 1] / den;
    } else {
        cs[k] = 1.0;
        sn[k] = 0.0;
    }
    col[k] = den;
    col[k + 1] = 0.0;
    g[k + 1] = -sn[k] * g[k];
    g[k] = cs[k] * g[k];
    st[0] = fabs(g[k + 1]);
    st[1] = hn;
    st[2] = hn != 0.0 ? 1.0 / hn : 0.0;
}

__global__ void k_init_g(int m, double beta, double *__restrict__ g) {
    const int i = threadIdx.x;
    if (i <= m) g[i] = i == 0 ? beta : 0.0;
}

// y = H(0:kk, 0:kk)^-1 g (upper triangular)
__global__ void k_upper_solve(int kk, int ldh, const double *__restrict__ H, const double *__restrict__ g,
                              double *__restrict__ y) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    for (int i = kk - 1; i >= 0; --i) {
        double s = g[i];
        for (int j = i + 1; j < kk; ++j) s -= H[(long long)j * ldh + i] * y[j];
        y[i] = s / H[(long long)i * ldh + i];
    }
}

// x += sum_j y[j] Z[j]
__global__ void k_combine(long long n, const double *__restrict__ Z, long long ldz, int kk,
                          const double *__restrict__ y, double *__restrict__ x) {
    __shared__ double ys[MAXV];
    if (threadIdx.x < MAXV) ys[threadIdx.x] = threadIdx.x < kk ? y[threadIdx.x] : 0.0;
    __syncthreads();
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        double s = 0.0;
#pragma unroll
        for (int j = 0; j < MAXV; ++j)
            if (j < kk) s += ys[j] * Z[j * ldz + i];
        x[i] += s;
    }
}

// out = a * scale (host scalar) or a * scale_dev[0] (device scalar)
__global__ void k_scale(long long n, const double *__restrict__ a, double scale,
                        const double *__restrict__ scale_dev, double *__restrict__ out) {
    const double s = scale_dev ? scale_dev[0] : scale;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
        out[i] = a[i] * s;
}

// rank-one terms: t = w . x over (wi, wv); y[ui] += sign * uv * t
__global__ void k_lr_dot(long long m, const long long *__restrict__ wi, const double *__restrict__ wv,
                         const double *__restrict__ x, double *__restrict__ t) {
    __shared__ double red[32];
    double acc = 0.0;
    for (long long q = threadIdx.x; q < m; q += blockDim.x) acc += wv[q] * x[wi[q]];
    acc = warp_sum(acc);
    if (threadIdx.x % 32 == 0) red[threadIdx.x / 32] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double v = 0.0;
        for (int q = 0; q < (int)(blockDim.x / 32); ++q) v += red[q];
        t[0] = v;
    }
}

__global__ void k_lr_axpy(long long m, const long long *__restrict__ ui, const double *__restrict__ uv,
                          const double *__restrict__ t, double sign, double *__restrict__ y) {
    const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q < m) y[ui[q]] += sign * uv[q] * t[0];
}

// ------------------------------------------------------------------ segmented Krylov
//
// FGMRES with one Krylov recurrence per segment of a block-diagonal system (the instances of
// an ensemble): the operator and the preconditioner act on all segments at once, every inner
// product, norm, Hessenberg column, Givens rotation and step length is taken per segment.
// A pass over the vectors runs one CTA per chunk of a segment: CTA c covers the entries
// [cfirst[c], cfirst[c + 1]) of segment cseg[c], and the CTAs of segment s are
// sfirst[s] .. sfirst[s + 1] - 1, so that a segment's sums fold over its own CTAs in a fixed
// order. Per-segment arrays are strided by MAXV (h, norms, y), by ldh (rotations) or by
// ldh * ldh (Hessenberg), ldh = restart + 1.

// MODE 0: partial[c][j] = (V_j . w) over the CTA's chunk, j < nv; 1: w -= sum_j h[s][j] V_j
// first, then the dots; 2: the update, then partial[c][0] = |w|^2; 3: |w|^2 alone (w unchanged)
template <int MODE>
__global__ void __launch_bounds__(DOT_THREADS)
k_seg_pass(const long long *__restrict__ cfirst, const int *__restrict__ cseg,
           const double *__restrict__ V, long long ldv, int nv, const double *__restrict__ h,
           double *__restrict__ w, double *__restrict__ partial) {
    constexpr bool UPDATE = MODE == 1 || MODE == 2;
    constexpr bool DOTS = MODE < 2;
    const int c = blockIdx.x;
    const long long i0 = cfirst[c], i1 = cfirst[c + 1];
    __shared__ double hs[MAXV];
    if (UPDATE && threadIdx.x < MAXV)
        hs[threadIdx.x] = (int)threadIdx.x < nv ? h[(long long)cseg[c] * MAXV + threadIdx.x] : 0.0;
    __syncthreads();
    double acc[MAXV];
#pragma unroll
    for (int j = 0; j < MAXV; ++j) acc[j] = 0.0;
    for (long long i = i0 + threadIdx.x; i < i1; i += blockDim.x) {
        double wi = w[i];
        if (UPDATE) {
            double s = 0.0;
#pragma unroll
            for (int j = 0; j < MAXV; ++j)
                if (j < nv) s += hs[j] * V[j * ldv + i];
            wi -= s;
            w[i] = wi;
        }
        if (DOTS) {
#pragma unroll
            for (int j = 0; j < MAXV; ++j)
                if (j < nv) acc[j] += V[j * ldv + i] * wi;
        } else {
            acc[0] += wi * wi;
        }
    }
    __shared__ double red[DOT_THREADS / 32][MAXV];
    const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
    const int cols = DOTS ? nv : 1;
#pragma unroll
    for (int j = 0; j < MAXV; ++j)
        if (j < cols) {
            const double v = warp_sum(acc[j]);
            if (lane == 0) red[warp][j] = v;
        }
    __syncthreads();
    if ((int)threadIdx.x < cols) {
        double v = 0.0;
        for (int q = 0; q < DOT_THREADS / 32; ++q) v += red[q][threadIdx.x];
        partial[(long long)c * MAXV + threadIdx.x] = v;
    }
}

// out[s][j] = sum over segment s's CTAs of partial[c][j] (one CTA of 32 * MAXV threads per
// segment, a warp per column: lane-strided sums, then a fixed butterfly); 0 for no CTAs
__global__ void k_seg_fold(const int *__restrict__ sfirst, int cols, const double *__restrict__ partial,
                           double *__restrict__ out) {
    const int s = blockIdx.x, j = threadIdx.x / 32, lane = threadIdx.x % 32;
    if (j >= cols) return;
    double v = 0.0;
    for (int c = sfirst[s] + lane; c < sfirst[s + 1]; c += 32) v += partial[(long long)c * MAXV + j];
    v = warp_sum(v);
    if (lane == 0) out[(long long)s * MAXV + j] = v;
}

// per segment at the start of a solve: beta0 = |r|, target = max(rtol beta0, 1e-13 |b|)
// (the floor of the single-recurrence solve); bb, rr: folded squares (MAXV-strided)
// A segment marked inactive (active[s] == 0) gets an infinite target: it takes no steps and
// keeps its initial guess.
__global__ void k_seg_targets(int nseg, double rtol, const double *__restrict__ bb,
                              const double *__restrict__ rr, const int *__restrict__ active,
                              double *__restrict__ beta0, double *__restrict__ target) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nseg) return;
    const double b0 = sqrt(rr[(long long)s * MAXV]);
    beta0[s] = b0;
    target[s] = active[s] ? fmax(rtol * b0, 1e-13 * sqrt(bb[(long long)s * MAXV])) : INFINITY;
}

// a restart cycle's first column: g = (beta, 0, ...), the segment active (kk = -1) while its
// residual is above target, else frozen with no steps (kk = 0); inv = 1 / beta when active.
// active: the number of active segments (zeroed by the caller)
__global__ void k_seg_init(int nseg, int ldh, const double *__restrict__ rr,
                           const double *__restrict__ target, double *__restrict__ g,
                           int *__restrict__ kk, double *__restrict__ inv, int *__restrict__ active) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nseg) return;
    const double beta = sqrt(rr[(long long)s * MAXV]);
    double *gs = g + (long long)s * (ldh + 1);
    for (int i = 0; i <= ldh; ++i) gs[i] = i == 0 ? beta : 0.0;
    const bool on = beta > target[s];
    kk[s] = on ? -1 : 0;
    inv[s * 4 + 2] = on && beta > 0.0 ? 1.0 / beta : 0.0;
    if (on) atomicAdd(active, 1);
}

// column k of each active segment's Hessenberg matrix (the per-segment form of
// k_arnoldi_finish); a segment that reaches its target or breaks down (h_{k+1,k} = 0) freezes
// with kk = k + 1 steps. st[s]: [0] |g[k+1]|, [1] h_{k+1,k}, [2] the scale of the next basis
// vector (0 once frozen). active: segments still active after this step.
__global__ void k_seg_finish(int k, int nseg, int ldh, const double *__restrict__ h1,
                             const double *__restrict__ h2, const double *__restrict__ nrm2,
                             const double *__restrict__ target, double *__restrict__ H,
                             double *__restrict__ cs, double *__restrict__ sn, double *__restrict__ g,
                             int *__restrict__ kk, double *__restrict__ st, int *__restrict__ active) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nseg) return;
    double *sts = st + (long long)s * 4;
    if (kk[s] >= 0) {
        sts[2] = 0.0;
        return;
    }
    const double *a = h1 + (long long)s * MAXV, *b = h2 + (long long)s * MAXV;
    double *col = H + (long long)s * ldh * ldh + (long long)k * ldh;
    double *c = cs + (long long)s * ldh, *sv = sn + (long long)s * ldh;
    double *gs = g + (long long)s * (ldh + 1);
    for (int j = 0; j <= k; ++j) col[j] = a[j] + b[j];
    const double hn = sqrt(nrm2[(long long)s * MAXV]);
    col[k + 1] = hn;
    for (int j = 0; j < k; ++j) {
        const double t = c[j] * col[j] + sv[j] * col[j + 1];
        col[j + 1] = -sv[j] * col[j] + c[j] * col[j + 1];
        col[j] = t;
    }
    const double den = hypot(col[k], col[k + 1]);
    if (den != 0.0) {
        c[k] = col[k] / den;
        sv[k] = col[k + 1] / den;
    } else {
        c[k] = 1.0;
        sv[k] = 0.0;
    }
    col[k] = den;
    col[k + 1] = 0.0;
    gs[k + 1] = -sv[k] * gs[k];
    gs[k] = c[k] * gs[k];
    sts[0] = fabs(gs[k + 1]);
    sts[1] = hn;
    // frozen: at its target, or a breakdown - a vanished h_{k+1,k} (the space holds the
    // solution: keep the column), or a vanished rotated diagonal (drop the column)
    const bool done = sts[0] <= target[s] || hn == 0.0 || den == 0.0;
    sts[2] = done ? 0.0 : 1.0 / hn;
    if (done) kk[s] = den == 0.0 ? k : k + 1;
    else atomicAdd(active, 1);
}

// out[i] = a[i] * sc[cseg(i) * 4 + 2]: a basis vector scaled per segment
__global__ void k_seg_scale(const long long *__restrict__ cfirst, const int *__restrict__ cseg,
                            const double *__restrict__ a, const double *__restrict__ sc,
                            double *__restrict__ out) {
    const int c = blockIdx.x;
    const double f = sc[(long long)cseg[c] * 4 + 2];
    for (long long i = cfirst[c] + threadIdx.x; i < cfirst[c + 1]; i += blockDim.x) out[i] = a[i] * f;
}

// y[s] = H_s(0:K, 0:K)^-1 g_s, K = the segment's steps (kk, or ku while still active);
// y[s][j] = 0 for j >= K
__global__ void k_seg_upper(int nseg, int ku, int ldh, const double *__restrict__ H,
                            const double *__restrict__ g, const int *__restrict__ kk,
                            double *__restrict__ y) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nseg) return;
    const int K = kk[s] < 0 ? ku : kk[s];
    const double *Hs = H + (long long)s * ldh * ldh, *gs = g + (long long)s * (ldh + 1);
    double *ys = y + (long long)s * MAXV;
    for (int j = K; j < MAXV; ++j) ys[j] = 0.0;
    for (int i = K - 1; i >= 0; --i) {
        double v = gs[i];
        for (int j = i + 1; j < K; ++j) v -= Hs[(long long)j * ldh + i] * ys[j];
        ys[i] = v / Hs[(long long)i * ldh + i];
    }
}

// x += sum_j y[s][j] Z_j over each segment's entries (j < ku; y is 0 past a segment's steps)
__global__ void k_seg_combine(const long long *__restrict__ cfirst, const int *__restrict__ cseg,
                              const double *__restrict__ Z, long long ldz, int ku,
                              const double *__restrict__ y, double *__restrict__ x) {
    const int c = blockIdx.x;
    __shared__ double ys[MAXV];
    if (threadIdx.x < MAXV) ys[threadIdx.x] = (int)threadIdx.x < ku ? y[(long long)cseg[c] * MAXV + threadIdx.x] : 0.0;
    __syncthreads();
    for (long long i = cfirst[c] + threadIdx.x; i < cfirst[c + 1]; i += blockDim.x) {
        double v = 0.0;
        for (int j = 0; j < ku; ++j) v += ys[j] * Z[j * ldz + i];
        x[i] += v;
    }
}

// the segments whose residual (folded squares rr) is above target
__global__ void k_seg_open(int nseg, const double *__restrict__ rr, const double *__restrict__ target,
                           int *__restrict__ open) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s < nseg && sqrt(rr[(long long)s * MAXV]) > target[s]) atomicAdd(open, 1);
}

struct LowRank {
    const long long *ui;
    const double *uv;
    long long nu;
    const long long *wi;
    const double *wv;
    long long nw;
};

// ------------------------------------------------------------------ the hierarchy

__global__ void k_iota_i32(int *p, long long n);

class Hierarchy {
   public:
    Params prm;
    std::vector<Level> L;
    int setups = 0;
    cudaStream_t st = 0;
    Arena structure, values, scratch;
    const long long *src_indptr = nullptr;
    long long src_n = -1, src_nnz = -1;

    int setup(long long n, long long nnz, const long long *indptr, const int *indices,
              const double *data, cudaStream_t s) {
        st = s;
        structure.set_stream(s);
        values.set_stream(s);
        scratch.set_stream(s);
        persist.set_stream(s);
        const bool same = L.size() && n == src_n && nnz == src_nnz && indptr == src_indptr;
        const bool periodic = prm.rebuild_every > 0 &&
                              (prm.rebuild_every == 1 || setups % prm.rebuild_every == 0);
        const bool rebuild = !same || periodic || rebuild_requested;
        ++setups;
        rebuilt_ = rebuild;
        if (rebuild) {
            rebuild_requested = false;
            base_iterations = -1;
            base_seen = 0;
            ++rebuilds;
            drop_graphs();
            values.release();
            structure.release();
            L.clear();
            Level l0;
            l0.n = n;
            l0.nnz = nnz;
            l0.indptr = indptr;
            l0.indices = indices;
            l0.data = data;
            L.push_back(l0);
            src_indptr = indptr;
            src_n = n;
            src_nnz = nnz;
            ZV_TRY(build_structure());
            ZV_TRY(allocate_values());
        } else {
            if (L[0].data != data || L[0].indices != indices) drop_graphs();
            L[0].data = data;
            L[0].indices = indices;
            for (size_t l = 1; l < L.size(); ++l) ZV_TRY(galerkin_values(l));
        }
        ZV_TRY(compute_values());
        if (rebuild && prm.autotune) ZV_TRY(prm.precision == 1 ? autotune<float>() : autotune<double>());
        // Chebyshev: the spectral bound of every level, with the aggregates (a rebuild); the
        // values re-summed between rebuilds move it little, and a solve that degrades triggers
        // the adaptive rebuild
        if (rebuild && prm.smoother == 2)
            ZV_TRY(prm.precision == 1 ? estimate_spectra<float>() : estimate_spectra<double>());
        return OK;
    }

    ~Hierarchy() {
        drop_graphs();
        if (capture_stream) cudaStreamDestroy(capture_stream);
    }

    void drop_graphs() {
        for (auto &row : graphs)
            for (cudaGraphExec_t &g : row)
                if (g) {
                    cudaGraphExecDestroy(g);
                    g = nullptr;
                }
    }

    template <typename T, bool TRANS = false>
    int vcycle();   // defined below

    // the transpose structure of every level (built on first use, kept with the structure)
    bool transposed_used = false;
    int ensure_transpose() {
        if (!transposed_used) {
            transposed_used = true;
            if (prm.precision == 1)
                for (Level &v : L)
                    if (v.pptr) ZV_TRY(convert_original(v));
        }
        for (Level &v : L) {
            if (v.tptr) continue;
            ZV_TRY(structure.get(&v.tptr, v.n + 1));
            ZV_TRY(structure.get(&v.trow, v.nnz));
            ZV_TRY(structure.get(&v.tperm, v.nnz));
            ZV_TRY(zvfv_bsr_transpose(v.n, v.nnz, (const int64_t *)v.indptr, v.indices,
                                      (int64_t *)v.tptr, v.trow, (int64_t *)v.tperm, st));
        }
        return OK;
    }

    // Adaptive reuse (rebuild_every 0), after the policy of the reference's AmgX binding
    // (zvcfd/fv/linear.py:686-698, :837-841): later matrices keep the aggregates and only
    // re-sum the coarse operators, until a solve fails or needs more than rebuild_ratio times
    // (and at least 2 more than) the base iterations. The reference takes the first solve after
    // a rebuild as the base; here it is the largest of the first BASE_SOLVES, because the
    // coefficient loops of a time step alternate hard and easy solves and a base set by an
    // easy one rebuilt the hierarchy on the next hard one, every step.
    static constexpr int BASE_SOLVES = 3;
    bool rebuild_requested = false;
    int base_iterations = -1, base_seen = 0;
    long long rebuilds = 0;
    void request_rebuild() { rebuild_requested = true; }
    void record_solve(int iterations, bool converged) {
        if (prm.rebuild_every > 0) return;
        if (base_seen < BASE_SOLVES) {
            base_iterations = std::max(base_iterations, iterations);
            ++base_seen;
            if (converged) return;
        }
        const double limit = std::max(prm.rebuild_ratio * base_iterations, base_iterations + 2.0);
        if (!converged || iterations > limit) rebuild_requested = true;
    }

    cudaGraphExec_t graphs[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};   // [FP32][TRANS]
    long long graph_kernels[2][2] = {{0, 0}, {0, 0}};                         // kernels per replay
    cudaStream_t capture_stream = nullptr;

   private:
    bool rebuilt_ = false;
    Arena persist;                         // kept across rebuilds: the finest level's colouring
    const long long *coloured_indptr = nullptr;
    long long coloured_n = -1, coloured_nnz = -1;
    Level c0;                              // the finest level's colouring and colour order

    // level l's blocks: the sums of level l-1's blocks over each aggregate pair
    int galerkin_values(size_t l) {
        Level &v = L[l];
        const Level &f = L[l - 1];
        if (!v.own) ZV_TRY(structure.get(&v.own, v.nnz * 16));
        k_block_seg_sum<<<grid_for(v.nnz * 16, 256), 256, 0, st>>>(v.nnz, f.gseg, f.gperm, f.data, v.own); count_launch();
        v.data = v.own;
        return launch_status("galerkin");
    }

    // ---------------------------------------------------------------- sorting helpers

    // keys (m) -> stable order perm, unique keys, segment starts (nseg + 1)
    int sort_segments(Arena &out, const unsigned long long *keys, long long m, int end_bit,
                      long long **perm, unsigned long long **ukeys, long long **seg, long long *nseg) {
        unsigned long long *kout;
        long long *idx;
        int *flags, *rank;
        ZV_TRY(scratch.get(&kout, m));
        ZV_TRY(scratch.get(&idx, m));
        ZV_TRY(out.get(perm, m));
        ZV_TRY(scratch.get(&flags, m));
        ZV_TRY(scratch.get(&rank, m));
        k_iota64<<<grid_for(m, 256), 256, 0, st>>>(idx, m); count_launch();
        size_t tb = 0, tb2 = 0;
        cub::DeviceRadixSort::SortPairs(nullptr, tb, keys, kout, idx, *perm, (int64_t)m, 0, end_bit, st);
        cub::DeviceScan::ExclusiveSum(nullptr, tb2, flags, rank, (int64_t)m, st);
        unsigned char *tmp;
        ZV_TRY(scratch.get(&tmp, tb > tb2 ? tb : tb2));
        ZV_TRY(cuda_status(cub::DeviceRadixSort::SortPairs(tmp, tb, keys, kout, idx, *perm, (int64_t)m, 0,
                                                           end_bit, st), "sort"));
        k_seg_flags<<<grid_for(m, 256), 256, 0, st>>>(m, kout, flags); count_launch();
        ZV_TRY(cuda_status(cub::DeviceScan::ExclusiveSum(tmp, tb2, flags, rank, (int64_t)m, st), "scan"));
        int last[2];
        cudaMemcpyAsync(&last[0], rank + m - 1, 4, cudaMemcpyDeviceToHost, st);
        cudaMemcpyAsync(&last[1], flags + m - 1, 4, cudaMemcpyDeviceToHost, st);
        ZV_TRY(cuda_status(cudaStreamSynchronize(st), "segments"));
        *nseg = (long long)last[0] + last[1];
        ZV_TRY(out.get(seg, *nseg + 1));
        ZV_TRY(out.get(ukeys, *nseg));
        k_seg_starts<<<grid_for(m, 256), 256, 0, st>>>(m, flags, rank, kout, *seg, *ukeys); count_launch();
        k_seg_end<<<1, 1, 0, st>>>(m, *nseg, *seg); count_launch();
        return launch_status("segments");
    }

    int exclusive_scan(const int *in, int *out, long long n) {
        size_t tb = 0;
        cub::DeviceScan::ExclusiveSum(nullptr, tb, in, out, (int64_t)n, st);
        unsigned char *tmp;
        ZV_TRY(scratch.get(&tmp, tb));
        return cuda_status(cub::DeviceScan::ExclusiveSum(tmp, tb, in, out, (int64_t)n, st), "scan");
    }

    static int bits(unsigned long long v) {
        int b = 1;
        while (b < 64 && (v >> b)) ++b;
        return b;
    }

    // ---------------------------------------------------------------- aggregation

    // pairwise matching on graph (n, indptr, idx) with strengths s (linear.py:373-413)
    int pairwise(long long n, const long long *indptr, const int *idx, const double *s, int *agg,
                 long long *count) {
        int *best, *flag, *rank, *join, *nxt, *any;
        ZV_TRY(scratch.get(&best, n));
        ZV_TRY(scratch.get(&flag, n));
        ZV_TRY(scratch.get(&rank, n));
        ZV_TRY(scratch.get(&join, n));
        ZV_TRY(scratch.get(&nxt, 1));
        ZV_TRY(scratch.get(&any, 1));
        const unsigned g = grid_for(n, 256);
        k_fill_int<<<g, 256, 0, st>>>(agg, n, -1); count_launch();
        cudaMemsetAsync(nxt, 0, 4, st);
        for (int round = 0; round < 4; ++round) {
            k_best_free<<<g, 256, 0, st>>>(n, indptr, idx, s, agg, best, any); count_launch();
            k_leaders<<<g, 256, 0, st>>>(n, best, flag); count_launch();
            ZV_TRY(exclusive_scan(flag, rank, n));
            k_assign_pairs<<<g, 256, 0, st>>>(n, best, flag, rank, nxt, agg); count_launch();
            k_advance<<<1, 1, 0, st>>>(flag, rank, n, nxt); count_launch();
        }
        k_join<<<g, 256, 0, st>>>(n, indptr, idx, s, agg, join); count_launch();
        k_apply_join<<<g, 256, 0, st>>>(n, join, agg, flag); count_launch();
        ZV_TRY(exclusive_scan(flag, rank, n));
        k_assign_singles<<<g, 256, 0, st>>>(n, flag, rank, nxt, agg); count_launch();
        k_advance<<<1, 1, 0, st>>>(flag, rank, n, nxt); count_launch();
        int c = 0;
        cudaMemcpyAsync(&c, nxt, 4, cudaMemcpyDeviceToHost, st);
        ZV_TRY(cuda_status(cudaStreamSynchronize(st), "pairwise"));
        *count = c;
        return launch_status("pairwise");
    }

    // `passes` pairwise passes (linear.py:415-433) -> agg (n), nc
    int aggregate(Level &v) {
        const long long n = v.n;
        double *w;
        ZV_TRY(scratch.get(&w, v.nnz));
        k_block_weight<<<grid_for(v.nnz, 256), 256, 0, st>>>(v.nnz, v.data, prm.strength == 1 ? 1 : 0,
                                                             w); count_launch();
        if (prm.strength == 2) {
            // Convection makes the strongest coupling of a node point upstream, so that mutual
            // strongest neighbours - the pairs of the matching - become rare and coarsening
            // stalls (one level left). The mean of both directions keeps the pairs.
            long long *tptr, *tperm;
            int *trow;
            double *ws;
            ZV_TRY(scratch.get(&tptr, v.n + 1));
            ZV_TRY(scratch.get(&trow, v.nnz));
            ZV_TRY(scratch.get(&tperm, v.nnz));
            ZV_TRY(scratch.get(&ws, v.nnz));
            ZV_TRY(zvfv_bsr_transpose(v.n, v.nnz, (const int64_t *)v.indptr, v.indices,
                                      (int64_t *)tptr, trow, (int64_t *)tperm, st));
            k_symmetric_weight<<<grid_for(v.nnz, 256), 256, 0, st>>>(v.nnz, tperm, w, ws); count_launch();
            w = ws;
        }
        long long gn = n, gnnz = v.nnz;
        const long long *gptr = v.indptr;
        const int *gidx = v.indices;
        const long long *grows = v.rows;
        const double *gw = w;
        int *total;
        ZV_TRY(structure.get(&total, n));
        k_iota_int(total, n);
        long long count = n;
        for (int pass = 0; pass < prm.passes; ++pass) {
            double *dw, *s;
            int *a;
            ZV_TRY(scratch.get(&dw, gn));
            ZV_TRY(scratch.get(&s, gnnz));
            ZV_TRY(scratch.get(&a, gn));
            k_diag_of<<<grid_for(gn, 256), 256, 0, st>>>(gn, gptr, gidx, gw, dw, nullptr); count_launch();
            k_strength<<<grid_for(gnnz, 256), 256, 0, st>>>(gnnz, grows, gidx, gw, dw, s); count_launch();
            ZV_TRY(pairwise(gn, gptr, gidx, s, a, &count));
            k_compose<<<grid_for(n, 256), 256, 0, st>>>(n, a, total); count_launch();
            if (pass + 1 == prm.passes) break;
            // the graph of the aggregates: strengths summed per aggregate pair
            unsigned long long *keys, *ukeys;
            long long *perm, *seg, nseg;
            ZV_TRY(scratch.get(&keys, gnnz));
            k_pair_key<<<grid_for(gnnz, 256), 256, 0, st>>>(gnnz, grows, gidx, a,
                                                            (unsigned long long)count, keys); count_launch();
            ZV_TRY(sort_segments(scratch, keys, gnnz, bits((unsigned long long)count * count), &perm,
                                 &ukeys, &seg, &nseg));
            long long *nptr, *nrows;
            int *nidx;
            double *nw;
            ZV_TRY(scratch.get(&nptr, count + 1));
            ZV_TRY(scratch.get(&nidx, nseg));
            ZV_TRY(scratch.get(&nw, nseg));
            ZV_TRY(scratch.get(&nrows, nseg));
            k_keys_to_csr<<<grid_for((nseg > count ? nseg : count) + 1, 256), 256, 0, st>>>(
                nseg, count, (unsigned long long)count, ukeys, nptr, nidx); count_launch();
            k_seg_sum<<<grid_for(nseg, 256), 256, 0, st>>>(nseg, 1, seg, perm, gw, nw); count_launch();
            k_rows_of<<<grid_for(count, 256), 256, 0, st>>>(count, nptr, nrows); count_launch();
            gn = count;
            gnnz = nseg;
            gptr = nptr;
            gidx = nidx;
            grows = nrows;
            gw = nw;
        }
        v.agg = total;
        v.nc = count;
        return launch_status("aggregate");
    }

    void k_iota_int(int *p, long long n) {
        k_iota_i32_launch(p, n);
    }
    void k_iota_i32_launch(int *p, long long n);

    // Node colouring of level v and its rows in colour order (multicolour Gauss-Seidel):
    // greedy first-fit in row order on the host. Row i takes the lowest colour that none of
    // its earlier neighbours holds; the level patterns are symmetric (element cliques and
    // their Galerkin products), so no two rows of a colour are coupled either way. On the
    // finest level of a hexahedral/prismatic tube this gives 8 large colours and 1-2 small
    // ones, against 17 for a random-key Jones-Plassmann colouring: fewer, fuller launches per
    // sweep. Run once per pattern on the finest level (kept in `persist`) and at each
    // rebuild on the coarser Gauss-Seidel levels.
    int colour_level(Level &v, Arena &keep) {
        const long long n = v.n, nnz = v.nnz;
        std::vector<long long> ip(n + 1);
        std::vector<int> ix(nnz);
        ZV_TRY(cuda_status(cudaMemcpyAsync(ip.data(), v.indptr, (n + 1) * sizeof(long long),
                                           cudaMemcpyDeviceToHost, st), "colouring: indptr"));
        ZV_TRY(cuda_status(cudaMemcpyAsync(ix.data(), v.indices, nnz * sizeof(int),
                                           cudaMemcpyDeviceToHost, st), "colouring: indices"));
        ZV_TRY(cuda_status(cudaStreamSynchronize(st), "colouring: pattern"));
        std::vector<int> col(n);
        std::vector<long long> seen;             // seen[c]: the last row with a neighbour of colour c
        for (long long i = 0; i < n; ++i) {
            for (long long p = ip[i]; p < ip[i + 1]; ++p) {
                const int j = ix[p];
                if (j < i) seen[col[j]] = i;
            }
            int c = 0;
            while (c < (int)seen.size() && seen[c] == i) ++c;
            if (c == (int)seen.size()) seen.push_back(-1);
            col[i] = c;
        }
        const int C = (int)seen.size();
        v.gs_off.assign(C + 1, 0);
        for (long long i = 0; i < n; ++i) ++v.gs_off[col[i] + 1];
        for (int c = 0; c < C; ++c) v.gs_off[c + 1] += v.gs_off[c];
        std::vector<int> order(n);
        std::vector<long long> at(v.gs_off.begin(), v.gs_off.end() - 1);
        for (long long i = 0; i < n; ++i) order[at[col[i]]++] = (int)i;
        // the colour-ordered structure: position k holds row order[k]
        std::vector<int> inv(n), pidx(nnz);
        std::vector<long long> pptr(n + 1), psrc(nnz), pdpos(n, -1);
        for (long long k = 0; k < n; ++k) inv[order[k]] = (int)k;
        pptr[0] = 0;
        for (long long k = 0; k < n; ++k) {
            const long long i = order[k], q0 = pptr[k];
            for (long long p = ip[i]; p < ip[i + 1]; ++p) {
                const long long q = q0 + (p - ip[i]);
                pidx[q] = inv[ix[p]];
                psrc[q] = p;
                if (ix[p] == i) pdpos[k] = q;
            }
            pptr[k + 1] = q0 + (ip[i + 1] - ip[i]);
        }
        int *rows, *dinv_, *didx;
        long long *dptr, *dsrc, *ddpos;
        ZV_TRY(keep.get(&rows, n));
        ZV_TRY(keep.get(&dinv_, n));
        ZV_TRY(keep.get(&didx, nnz));
        ZV_TRY(keep.get(&dptr, n + 1));
        ZV_TRY(keep.get(&dsrc, nnz));
        ZV_TRY(keep.get(&ddpos, n));
        ZV_TRY(cuda_status(cudaMemcpyAsync(rows, order.data(), n * sizeof(int), cudaMemcpyHostToDevice,
                                           st), "colouring: rows"));
        ZV_TRY(cuda_status(cudaMemcpyAsync(dinv_, inv.data(), n * sizeof(int), cudaMemcpyHostToDevice,
                                           st), "colouring: positions"));
        ZV_TRY(cuda_status(cudaMemcpyAsync(didx, pidx.data(), nnz * sizeof(int),
                                           cudaMemcpyHostToDevice, st), "colouring: columns"));
        ZV_TRY(cuda_status(cudaMemcpyAsync(dptr, pptr.data(), (n + 1) * sizeof(long long),
                                           cudaMemcpyHostToDevice, st), "colouring: row starts"));
        ZV_TRY(cuda_status(cudaMemcpyAsync(dsrc, psrc.data(), nnz * sizeof(long long),
                                           cudaMemcpyHostToDevice, st), "colouring: sources"));
        ZV_TRY(cuda_status(cudaMemcpyAsync(ddpos, pdpos.data(), n * sizeof(long long),
                                           cudaMemcpyHostToDevice, st), "colouring: diagonal"));
        if (prm.smoother == 3) {
            // the transposed block of every colour-ordered block: (j, i) is found in the sorted
            // original row j, and keeps its place there in the colour-ordered row
            std::vector<long long> ptr_t(nnz, -1);
            for (long long k = 0; k < n; ++k) {
                const long long i0 = order[k];
                for (long long p = ip[i0]; p < ip[i0 + 1]; ++p) {
                    const int jj = ix[p];
                    const int *lo = ix.data() + ip[jj], *hi = ix.data() + ip[jj + 1];
                    const int *f = std::lower_bound(lo, hi, (int)i0);
                    if (f != hi && *f == (int)i0)
                        ptr_t[pptr[k] + (p - ip[i0])] = pptr[inv[jj]] + (f - lo);
                }
            }
            long long *dt;
            ZV_TRY(keep.get(&dt, nnz));
            ZV_TRY(cuda_status(cudaMemcpyAsync(dt, ptr_t.data(), nnz * sizeof(long long),
                                               cudaMemcpyHostToDevice, st), "colouring: transposes"));
            ZV_TRY(cuda_status(cudaStreamSynchronize(st), "colouring: transposes"));
            v.ptrans = dt;
        }
        ZV_TRY(cuda_status(cudaStreamSynchronize(st), "colouring: upload"));
        v.gs_rows = rows;
        v.pinv = dinv_;
        v.pidx = didx;
        v.pptr = dptr;
        v.psrc = dsrc;
        v.pdpos = ddpos;
        return OK;
    }

    int build_structure() {
        for (size_t l = 0;; ++l) {
            Level &v = L[l];
            v.lanes = lanes_for(v.n, v.nnz);
            ZV_TRY(structure.get(&v.dpos, v.n));
            ZV_TRY(structure.get(&v.rows, v.nnz));
            k_diag_of<<<grid_for(v.n, 256), 256, 0, st>>>(v.n, v.indptr, v.indices, nullptr, nullptr,
                                                          v.dpos); count_launch();
            k_rows_of<<<grid_for(v.n, 256), 256, 0, st>>>(v.n, v.indptr, v.rows); count_launch();
            if ((prm.smoother == 1 || prm.smoother >= 3) && v.n > DENSE_MAX && (int)l < prm.gs_levels) {
                if (l == 0 && coloured_indptr == v.indptr && coloured_n == v.n &&
                    coloured_nnz == v.nnz && c0.gs_rows) {
                    // the finest pattern does not change: its colouring and colour order stay
                    v.gs_rows = c0.gs_rows;
                    v.gs_off = c0.gs_off;
                    v.pptr = c0.pptr;
                    v.pidx = c0.pidx;
                    v.psrc = c0.psrc;
                    v.pdpos = c0.pdpos;
                    v.pinv = c0.pinv;
                    v.ptrans = c0.ptrans;
                } else {
                    if (l == 0) persist.release();
                    ZV_TRY(colour_level(v, l == 0 ? persist : structure));
                    scratch.release();
                    if (l == 0) {
                        coloured_indptr = v.indptr;
                        coloured_n = v.n;
                        coloured_nnz = v.nnz;
                        c0 = v;
                    }
                }
            }
            if (v.n <= DENSE_MAX) {
                v.dense = true;
                break;
            }
            if ((int)l + 1 >= prm.max_levels) break;
            ZV_TRY(aggregate(v));
            scratch.release();
            if (v.nc >= 0.9 * v.n || v.nc < 1) {          // coarsening stalled: last level
                v.agg = nullptr;
                break;
            }
            // members of each aggregate, ascending (restriction)
            unsigned long long *keys, *ukeys;
            long long nseg;
            ZV_TRY(scratch.get(&keys, v.n));
            k_agg_keys(v.agg, v.n, keys);
            long long *perm, *seg;
            ZV_TRY(sort_segments(structure, keys, v.n, bits((unsigned long long)v.nc), &perm, &ukeys,
                                 &seg, &nseg));
            int *mem;
            ZV_TRY(structure.get(&mem, v.n));
            k_narrow(perm, v.n, mem);
            v.mem = mem;
            v.mptr = seg;
            if (v.pinv) {                      // the transfer in the colour order of the level
                ZV_TRY(structure.get(&v.pagg, v.n));
                ZV_TRY(structure.get(&v.pmem, v.n));
                k_gather_int<<<grid_for(v.n, 256), 256, 0, st>>>(v.n, v.gs_rows, v.agg, v.pagg); count_launch();
                k_gather_int<<<grid_for(v.n, 256), 256, 0, st>>>(v.n, v.mem, v.pinv, v.pmem); count_launch();
            }
            // the Galerkin map: fine blocks grouped by (agg row, agg col)
            unsigned long long *gk;
            ZV_TRY(scratch.get(&gk, v.nnz));
            k_pair_key<<<grid_for(v.nnz, 256), 256, 0, st>>>(v.nnz, v.rows, v.indices, v.agg,
                                                             (unsigned long long)v.nc, gk); count_launch();
            unsigned long long *gu;
            long long cn;
            ZV_TRY(sort_segments(structure, gk, v.nnz, bits((unsigned long long)v.nc * v.nc), &v.gperm,
                                 &gu, &v.gseg, &cn));
            v.cnnz = cn;
            long long *cptr;
            int *cidx;
            ZV_TRY(structure.get(&cptr, v.nc + 1));
            ZV_TRY(structure.get(&cidx, cn));
            k_keys_to_csr<<<grid_for((cn > v.nc ? cn : v.nc) + 1, 256), 256, 0, st>>>(
                cn, v.nc, (unsigned long long)v.nc, gu, cptr, cidx); count_launch();
            scratch.release();
            Level c;
            c.n = v.nc;
            c.nnz = cn;
            c.indptr = cptr;
            c.indices = cidx;
            L.push_back(c);
            ZV_TRY(galerkin_values(L.size() - 1));     // the next level aggregates on these
        }
        return launch_status("hierarchy structure");
    }

    void k_agg_keys(const int *agg, long long n, unsigned long long *keys);
    void k_narrow(const long long *src, long long n, int *dst);

    // buffers that live as long as the structure: pointers stay fixed across set-ups, so a
    // captured V-cycle graph stays valid until the next rebuild
    int allocate_values() {
        const size_t vs = prm.precision == 1 ? sizeof(float) : sizeof(double);
        for (Level &v : L) {
            ZV_TRY(values.get(&v.dinv64, v.n * 16));
            if (prm.precision == 1) {
                ZV_TRY(values.get(&v.data32, v.nnz * 16));
                ZV_TRY(values.get(&v.dinv32, v.n * 16));
            }
            if (v.pptr && prm.smoother == 4) {  // ILU(0) factors (FP64, and FP32 copies)
                ZV_TRY(values.get(&v.lu64, v.nnz * 16));
                if (prm.precision == 1) ZV_TRY(values.get(&v.lu32, v.nnz * 16));
            }
            if (v.pptr) {                      // the Gauss-Seidel levels' colour-ordered copy
                if (prm.precision == 1) {
                    ZV_TRY(values.get(&v.pdata32, v.nnz * 16));
                    ZV_TRY(values.get(&v.pdinv32, v.n * 16));
                } else {
                    ZV_TRY(values.get(&v.pdata64, v.nnz * 16));
                    ZV_TRY(values.get(&v.pdinv64, v.n * 16));
                }
                char *pb;
                ZV_TRY(values.get(&pb, vs * v.n * 4));
                v.pb = pb;
            }
            if (v.dense) {
                const size_t m = 4 * v.n;
                ZV_TRY(values.get(&v.inv64, m * m));
                if (prm.precision == 1) ZV_TRY(values.get(&v.inv32, m * m));
            }
            char *buf;
            ZV_TRY(values.get(&buf, 4 * vs * v.n * 4));
            v.x = buf;
            v.x2 = buf + vs * v.n * 4;
            v.b = buf + 2 * vs * v.n * 4;
            v.r = buf + 3 * vs * v.n * 4;
        }
        return OK;
    }

    int compute_values() {
        for (size_t l = 0; l < L.size(); ++l) {
            Level &v = L[l];
            k_dinv<double><<<grid_for(v.n, 128), 128, 0, st>>>(v.n, v.data, v.dpos, v.dinv64); count_launch();
            if (v.pptr) {
                const unsigned gb = grid_for(v.nnz * 8, 256), gd = grid_for(v.n * 16, 256);
                if (prm.precision == 1) {
                    k_gather_blocks<float><<<gb, 256, 0, st>>>(v.nnz, v.psrc, v.data, v.pdata32); count_launch();
                    k_permute_rows<true, double, float><<<gd, 256, 0, st>>>(v.n, 16, v.gs_rows, v.dinv64, v.pdinv32); count_launch();
                } else {
                    k_gather_blocks<double><<<gb, 256, 0, st>>>(v.nnz, v.psrc, v.data, v.pdata64); count_launch();
                    k_permute_rows<true, double, double><<<gd, 256, 0, st>>>(v.n, 16, v.gs_rows, v.dinv64, v.pdinv64); count_launch();
                }
            }
            if (v.pptr && prm.smoother == 3) ZV_TRY(dilu_factor(v));
            if (v.pptr && prm.smoother == 4) ZV_TRY(ilu_factor(v));
            // FP32 copies in the original numbering: every level but the Gauss-Seidel ones
            // (which sweep their colour-ordered copy), and those too once A^T is solved with
            if (prm.precision == 1 && (!v.pptr || transposed_used)) ZV_TRY(convert_original(v));
            if (v.inv64) {
                const int m = (int)(4 * v.n);
                double *dense;
                int *ok;
                ZV_TRY(scratch.get(&dense, (size_t)m * m));
                ZV_TRY(scratch.get(&ok, 1));
                cudaMemsetAsync(dense, 0, sizeof(double) * m * m, st);
                k_densify<<<grid_for(v.n, 64), 64, 0, st>>>(v.n, v.indptr, v.indices, v.data, dense); count_launch();
                const size_t smem = sizeof(double) * 2 * m * m;
                cudaFuncSetAttribute(k_dense_inverse, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
                k_dense_inverse<<<1, 512, smem, st>>>(m, dense, v.inv64, ok); count_launch();
                int okh = 0;
                cudaMemcpyAsync(&okh, ok, 4, cudaMemcpyDeviceToHost, st);
                ZV_TRY(cuda_status(cudaStreamSynchronize(st), "coarse inverse"));
                const bool was = v.dense;
                v.dense = okh != 0;              // singular: smooth the coarsest level instead
                if (was != v.dense) drop_graphs();
                if (v.dense && prm.precision == 1)
                    k_convert<double, float><<<grid_for((long long)m * m, 256), 256, 0, st>>>(
                        (long long)m * m, v.inv64, v.inv32); count_launch();
                scratch.release();
            }
        }
        return launch_status("hierarchy values");
    }

    // the DILU inverses of a colour-ordered level, colour by colour, in FP64 (into the level's
    // colour-ordered inverses, converted for the FP32 hierarchy)
    int dilu_factor(Level &v) {
        double *e = v.pdinv64;
        if (prm.precision == 1) ZV_TRY(scratch.get(&e, v.n * 16));
        const int C = (int)v.gs_off.size() - 1;
        for (int c = 0; c < C; ++c) {
            const long long o = v.gs_off[c], cnt = v.gs_off[c + 1] - o;
            if (cnt <= 0) continue;
            k_dilu_factor<<<grid_for(cnt, 128), 128, 0, st>>>(cnt, o, v.pptr, v.pidx, v.psrc, v.ptrans,
                                                               v.pdpos, v.data, e); count_launch();
        }
        if (prm.precision == 1) {
            k_convert<double, float><<<grid_for(v.n * 16, 256), 256, 0, st>>>(v.n * 16, e, v.pdinv32); count_launch();
            ZV_TRY(launch_status("dilu factor"));
            scratch.release();
        }
        return launch_status("dilu factor");
    }

    // the ILU(0) factors of a colour-ordered level, colour by colour, in FP64 (converted for
    // the FP32 hierarchy)
    int ilu_factor(Level &v) {
        const int C = (int)v.gs_off.size() - 1;
        for (int c = 0; c < C; ++c) {
            const long long o = v.gs_off[c], cnt = v.gs_off[c + 1] - o;
            if (cnt <= 0) continue;
            k_ilu_factor<<<grid_for(cnt, 128), 128, 0, st>>>(cnt, o, v.pptr, v.pidx, v.psrc, v.pdpos,
                                                             v.data, v.lu64); count_launch();
        }
        if (prm.precision == 1) {
            k_convert<double, float><<<grid_for(v.nnz * 16, 256), 256, 0, st>>>(v.nnz * 16, v.lu64, v.lu32); count_launch();
        }
        return launch_status("ilu factor");
    }

    int convert_original(Level &v) {
        k_convert<double, float><<<grid_for(v.nnz * 16, 256), 256, 0, st>>>(v.nnz * 16, v.data, v.data32); count_launch();
        k_convert<double, float><<<grid_for(v.n * 16, 256), 256, 0, st>>>(v.n * 16, v.dinv64, v.dinv32); count_launch();
        return launch_status("fp32 copy");
    }

    template <typename T, bool TRANS>
    int cycle(size_t l);
    template <typename T>
    int autotune();
    template <typename T>
    int estimate_spectra();
};

__global__ void k_iota_i32(int *p, long long n) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) p[i] = (int)i;
}

__global__ void k_agg_keys_kernel(const int *agg, long long n, unsigned long long *keys) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) keys[i] = (unsigned long long)agg[i];
}

__global__ void k_narrow_kernel(const long long *src, long long n, int *dst) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) dst[i] = (int)src[i];
}

void Hierarchy::k_iota_i32_launch(int *p, long long n) {
    k_iota_i32<<<grid_for(n, 256), 256, 0, st>>>(p, n); count_launch();
}
void Hierarchy::k_agg_keys(const int *agg, long long n, unsigned long long *keys) {
    k_agg_keys_kernel<<<grid_for(n, 256), 256, 0, st>>>(agg, n, keys); count_launch();
}
void Hierarchy::k_narrow(const long long *src, long long n, int *dst) {
    k_narrow_kernel<<<grid_for(n, 256), 256, 0, st>>>(src, n, dst); count_launch();
}

template <bool FIRST, typename V, typename T>
void jacobi(int lanes, long long n, const long long *indptr, const int *indices, const V *data,
            const V *dinv, const T *b, const T *xin, T *xout, T omega, cudaStream_t st) {
    switch (lanes) {
        case 8:
            k_jacobi<8, FIRST, V, T><<<grid_for(n * 8, 256), 256, 0, st>>>(n, indptr, indices, data, dinv, b,
                                                                         xin, xout, omega); count_launch();
            break;
        case 16:
            k_jacobi<16, FIRST, V, T><<<grid_for(n * 16, 256), 256, 0, st>>>(n, indptr, indices, data, dinv,
                                                                           b, xin, xout, omega); count_launch();
            break;
        default:
            k_jacobi<32, FIRST, V, T><<<grid_for(n * 32, 256), 256, 0, st>>>(n, indptr, indices, data, dinv,
                                                                           b, xin, xout, omega); count_launch();
    }
}

template <bool FIRST, typename V, typename T>
void jacobi_t(int lanes, long long n, const Level &v, const V *data, const V *dinv, const T *b,
              const T *xin, T *xout, T omega, cudaStream_t st) {
    switch (lanes) {
        case 8:
            k_jacobi_t<8, FIRST, V, T><<<grid_for(n * 8, 256), 256, 0, st>>>(n, v.tptr, v.trow, v.tperm, data,
                                                                           dinv, b, xin, xout, omega); count_launch();
            break;
        case 16:
            k_jacobi_t<16, FIRST, V, T><<<grid_for(n * 16, 256), 256, 0, st>>>(n, v.tptr, v.trow, v.tperm, data,
                                                                             dinv, b, xin, xout, omega); count_launch();
            break;
        default:
            k_jacobi_t<32, FIRST, V, T><<<grid_for(n * 32, 256), 256, 0, st>>>(n, v.tptr, v.trow, v.tperm, data,
                                                                             dinv, b, xin, xout, omega); count_launch();
    }
}

// one Chebyshev step on level v (k_cheby): A through the level's CSR, or with TR A^T through
// its transpose structure
template <bool FIRST, bool TR, typename V, typename T>
void cheby(const Level &v, const V *data, const V *dinv, const T *b, const T *xin, T *xout, T *d,
           T cd, T cz, cudaStream_t st) {
    const long long *p = TR ? v.tptr : v.indptr;
    const int *ix = TR ? v.trow : v.indices;
    const long long n = v.n;
    switch (v.lanes) {
        case 8:
            k_cheby<8, FIRST, TR, V, T><<<grid_for(n * 8, 256), 256, 0, st>>>(n, p, ix, v.tperm, data, dinv, b,
                                                                            xin, xout, d, cd, cz);
            break;
        case 16:
            k_cheby<16, FIRST, TR, V, T><<<grid_for(n * 16, 256), 256, 0, st>>>(n, p, ix, v.tperm, data, dinv, b,
                                                                              xin, xout, d, cd, cz);
            break;
        default:
            k_cheby<32, FIRST, TR, V, T><<<grid_for(n * 32, 256), 256, 0, st>>>(n, p, ix, v.tperm, data, dinv, b,
                                                                              xin, xout, d, cd, cz);
    }
    count_launch();
}

// A launch of 256-thread CTAs that may begin while the previous kernel in the stream is still
// draining (Programmatic Dependent Launch): the kernel must wait (griddepcontrol.wait) before it
// touches anything that kernel writes. Captured into a CUDA graph as a programmatic edge.
template <typename... P, typename... A>
void launch_dependent(void (*kern)(P...), unsigned grid, cudaStream_t st, A... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(256);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cudaLaunchKernelEx(&cfg, kern, static_cast<P>(args)...);
}

// one colour of a Gauss-Seidel pass with B blocks per slot in flight (the base for G lanes), or
// half (sel 0) or twice (sel 2) that many, capped at 16: the level's tile shape, which the
// autotuner picks with the lanes per row
template <int G, int B, typename V, typename T>
void gs_colour_launch(int sel, unsigned grid, cudaStream_t st, long long cnt, long long o, const Level &v,
                      const V *data, const V *dinv, const T *b, T *x, T omega) {
    constexpr int LO = B / 2 > 0 ? B / 2 : 1;
    constexpr int HI = 2 * B < 16 ? 2 * B : 16;
    if (sel == 0) launch_dependent(k_gs_colour_pdl<G, LO, V, T>, grid, st, cnt, o, v.pptr, v.pidx, data, dinv, b, x, omega);
    else if (sel == 2) launch_dependent(k_gs_colour_pdl<G, HI, V, T>, grid, st, cnt, o, v.pptr, v.pidx, data, dinv, b, x, omega);
    else launch_dependent(k_gs_colour_pdl<G, B, V, T>, grid, st, cnt, o, v.pptr, v.pidx, data, dinv, b, x, omega);
}

// one Gauss-Seidel pass over the colours of level v, forward or backward: on the colour-ordered
// copy (data, dinv, b, x colour-ordered; each colour a contiguous row range), or with TRANS on
// A^T in the original numbering (columns of A through the transpose structure, D^-T)
template <bool TRANS, typename V, typename T>
void gs_pass(const Level &v, const V *data, const V *dinv, const T *b, T *x, T omega, bool backward,
             cudaStream_t st) {
    const int C = (int)v.gs_off.size() - 1;
    for (int q = 0; q < C; ++q) {
        const int c = backward ? C - 1 - q : q;
        const long long o = v.gs_off[c], cnt = v.gs_off[c + 1] - v.gs_off[c];
        if (cnt <= 0) continue;
        const int G = v.lanes;
        const unsigned grid = grid_for(cnt * G, 256);
        if (TRANS) {
            const int *rows = v.gs_rows + o;
            if (G == 8) k_gs_colour_t<8, V, T><<<grid, 256, 0, st>>>(cnt, rows, v.tptr, v.trow, v.tperm, data, dinv, b, x, omega);
            else if (G == 16) k_gs_colour_t<16, V, T><<<grid, 256, 0, st>>>(cnt, rows, v.tptr, v.trow, v.tperm, data, dinv, b, x, omega);
            else k_gs_colour_t<32, V, T><<<grid, 256, 0, st>>>(cnt, rows, v.tptr, v.trow, v.tperm, data, dinv, b, x, omega);
        } else {
            constexpr int D = gs_prefetch_depth<V>();
            if (G == 8) gs_colour_launch<8, 2 * D, V, T>(v.gs_depth, grid, st, cnt, o, v, data, dinv, b, x, omega);
            else if (G == 16) gs_colour_launch<16, D, V, T>(v.gs_depth, grid, st, cnt, o, v, data, dinv, b, x, omega);
            else gs_colour_launch<32, (D + 1) / 2, V, T>(v.gs_depth, grid, st, cnt, o, v, data, dinv, b, x, omega);
        }
        count_launch();
    }
}

// one factorisation-smoother step on a colour-ordered level (DILU, or with ILU ILU(0)):
// r = b - A x (b itself while x is the zero start), the forward solve over the colours into w,
// the backward solve over them with x += omega z (k_lu_colour). data: the level's
// colour-ordered blocks (A for the residual); fac: the factored blocks for ILU(0), the DILU
// inverses E^-1 otherwise
template <bool ILU, typename V, typename T>
void lu_sweep(const Level &v, const V *data, const V *fac, const T *b, T *x, T *r, T *w, T omega,
              bool x_zero, cudaStream_t st) {
    const T *rr = b;
    if (!x_zero) {
        bsr_spmv_launch<true, V, T>(v.lanes, v.n, v.pptr, v.pidx, data, x, b, r, st);
        rr = r;
    }
    const V *blocks = ILU ? fac : data;
    const V *dinv = ILU ? nullptr : fac;
    const int C = (int)v.gs_off.size() - 1;
    const int G = v.lanes;
    for (int back = 0; back < 2; ++back)
        for (int q = 0; q < C; ++q) {
            const int c = back ? C - 1 - q : q;
            const long long o = v.gs_off[c], cnt = v.gs_off[c + 1] - v.gs_off[c];
            if (cnt <= 0) continue;
            const unsigned grid = grid_for(cnt * G, 256);
#define ZV_LU_LAUNCH(GG, BB)                                                                     \
    k_lu_colour<GG, BB, ILU, V, T><<<grid, 256, 0, st>>>(cnt, o, v.pptr, v.pidx, v.pdpos, blocks, \
                                                          dinv, rr, w, x, omega)
            if (back) {
                if (G == 8) ZV_LU_LAUNCH(8, true);
                else if (G == 16) ZV_LU_LAUNCH(16, true);
                else ZV_LU_LAUNCH(32, true);
            } else {
                if (G == 8) ZV_LU_LAUNCH(8, false);
                else if (G == 16) ZV_LU_LAUNCH(16, false);
                else ZV_LU_LAUNCH(32, false);
            }
#undef ZV_LU_LAUNCH
            count_launch();
        }
}

template <typename T>
struct CyclePick;
template <>
struct CyclePick<double> {
    static const double *data(const Level &v) { return v.data; }
    static const double *dinv(const Level &v) { return v.dinv64; }
    static const double *inv(const Level &v) { return v.inv64; }
    static const double *pdata(const Level &v) { return v.pdata64; }
    static const double *pdinv(const Level &v) { return v.pdinv64; }
    static const double *lu(const Level &v) { return v.lu64; }
};
template <>
struct CyclePick<float> {
    static const float *data(const Level &v) { return v.data32; }
    static const float *dinv(const Level &v) { return v.dinv32; }
    static const float *inv(const Level &v) { return v.inv32; }
    static const float *pdata(const Level &v) { return v.pdata32; }
    static const float *pdinv(const Level &v) { return v.pdinv32; }
    static const float *lu(const Level &v) { return v.lu32; }
};

// one V-cycle on level l: L[l].b -> L[l].x (zero initial guess); TRANS: the same cycle on
// every level's transpose (A^T, D^-T, inv^T), reusing the hierarchy built for A
template <typename T, bool TRANS>
int Hierarchy::cycle(size_t l) {
    Level &v = L[l];
    T *b = static_cast<T *>(v.b);
    if (v.dense) {
        const int m = (int)(4 * v.n);
        k_dense_apply<T, T, TRANS><<<grid_for((long long)m * 32, 256), 256, 0, st>>>(
            m, CyclePick<T>::inv(v), b, static_cast<T *>(v.x)); count_launch();
        return OK;
    }
    const auto *data = CyclePick<T>::data(v);
    const auto *dinv = CyclePick<T>::dinv(v);
    using V = typename std::remove_const<typename std::remove_pointer<decltype(data)>::type>::type;
    const bool coloured = prm.smoother == 1 || prm.smoother == 3 || prm.smoother == 4;
    const bool gs_level = coloured && !v.gs_off.empty();
    const bool jac_below = coloured && !gs_level;       // Jacobi below the GS / DILU levels
    const T omega = (T)(jac_below ? prm.jacobi_omega : prm.omega);
    const bool last = (l + 1 == L.size()) || v.agg == nullptr;
    const int pre = last ? prm.coarse_sweeps : (jac_below ? prm.jacobi_sweeps : prm.presweeps);
    const int post = jac_below ? prm.jacobi_sweeps : prm.postsweeps;
    if (gs_level && !TRANS) {
        // sweeps, residual, restriction and prolongation on the colour-ordered copy; b comes
        // in and x goes out in the level's own numbering
        const V *pdata = CyclePick<T>::pdata(v);
        const V *pdinv = CyclePick<T>::pdinv(v);
        T *pb = static_cast<T *>(v.pb), *px = static_cast<T *>(v.x2), *pr = static_cast<T *>(v.r);
        const unsigned g4 = grid_for(v.n * 4, 256);
        k_permute_rows<true, T, T><<<g4, 256, 0, st>>>(v.n, 4, v.gs_rows, b, pb); count_launch();
        cudaMemsetAsync(px, 0, v.n * 4 * sizeof(T), st);
        bool zero = true;                 // px is still the zero start
        auto sgs = [&](int sweeps) {      // symmetric: forward then backward over the colours
            if (prm.smoother == 3 || prm.smoother == 4) {
                const V *lu = CyclePick<T>::lu(v);
                for (int s = 0; s < sweeps; ++s, zero = false) {
                    if (prm.smoother == 4)
                        lu_sweep<true, V, T>(v, pdata, lu, pb, px, pr, static_cast<T *>(v.x), omega, zero, st);
                    else
                        lu_sweep<false, V, T>(v, pdata, pdinv, pb, px, pr, static_cast<T *>(v.x), omega, zero, st);
                }
                return;
            }
            for (int s = 0; s < sweeps; ++s) {
                gs_pass<false, V, T>(v, pdata, pdinv, pb, px, omega, false, st);
                gs_pass<false, V, T>(v, pdata, pdinv, pb, px, omega, true, st);
            }
        };
        sgs(pre);
        if (!last) {
            ZV_TRY((bsr_spmv_launch<true, V, T>(v.lanes, v.n, v.pptr, v.pidx, pdata, px, pb, pr, st)));
            Level &c = L[l + 1];
            k_restrict<T><<<grid_for(c.n * 4, 256), 256, 0, st>>>(c.n, v.mptr, v.pmem, pr, static_cast<T *>(c.b)); count_launch();
            ZV_TRY((cycle<T, TRANS>(l + 1)));
            k_prolong_add<T><<<g4, 256, 0, st>>>(v.n, v.pagg, static_cast<const T *>(c.x), px); count_launch();
            zero = false;
            sgs(prm.postsweeps);
        }
        k_permute_rows<false, T, T><<<g4, 256, 0, st>>>(v.n, 4, v.gs_rows, px, static_cast<T *>(v.x)); count_launch();
        return launch_status(last ? "coarse smoothing" : "v-cycle");
    }
    if (gs_level) {
        T *x = static_cast<T *>(v.x);
        auto sgs = [&](int sweeps) {      // symmetric: forward then backward over the colours
            for (int s = 0; s < sweeps; ++s) {
                gs_pass<TRANS, V, T>(v, data, dinv, b, x, omega, false, st);
                gs_pass<TRANS, V, T>(v, data, dinv, b, x, omega, true, st);
            }
        };
        cudaMemsetAsync(x, 0, v.n * 4 * sizeof(T), st);
        sgs(pre);
        if (last) return launch_status("coarse smoothing");
        T *r = static_cast<T *>(v.r);
        if (TRANS)
            ZV_TRY(bsr_spmv_t_launch<true, V, T>(v.lanes, v.n, v.tptr, v.trow, v.tperm, data, x, b, r, st));
        else
            ZV_TRY(bsr_spmv_launch<true, V, T>(v.lanes, v.n, v.indptr, v.indices, data, x, b, r, st));
        Level &c = L[l + 1];
        k_restrict<T><<<grid_for(c.n * 4, 256), 256, 0, st>>>(c.n, v.mptr, v.mem, r, static_cast<T *>(c.b)); count_launch();
        ZV_TRY((cycle<T, TRANS>(l + 1)));
        k_prolong_add<T><<<grid_for(v.n * 4, 256), 256, 0, st>>>(v.n, v.agg, static_cast<const T *>(c.x), x); count_launch();
        sgs(prm.postsweeps);
        return launch_status("v-cycle");
    }
    if (prm.smoother == 2) {
        // Chebyshev polynomials of degree pre and post in D^-1 A on [hi / ratio, hi],
        // hi = 1.1 lambda_max: centre theta, half-width delta, and the three-term recurrence
        // rho_k = 1 / (2 sigma - rho_{k-1}), sigma = theta / delta, rho_0 = 1 / sigma
        const double hi = 1.1 * v.cheb_lmax, lo = hi / prm.cheb_ratio;
        const double theta = 0.5 * (hi + lo), delta = 0.5 * (hi - lo), sigma = theta / delta;
        T *d = static_cast<T *>(v.r);          // the update: r is free while smoothing
        auto steps = [&](int degree, bool from_zero) {
            double rho = 1.0 / sigma;
            for (int k = 0; k < degree; ++k) {
                double cd = 0.0, cz = 1.0 / theta;
                if (k > 0) {
                    const double next = 1.0 / (2.0 * sigma - rho);
                    cd = next * rho;
                    cz = 2.0 * next / delta;
                    rho = next;
                }
                if (k == 0 && from_zero) {
                    cheby<true, TRANS, V, T>(v, data, dinv, b, nullptr, static_cast<T *>(v.x), d, (T)cd,
                                             (T)cz, st);
                    continue;
                }
                cheby<false, TRANS, V, T>(v, data, dinv, b, static_cast<const T *>(v.x),
                                          static_cast<T *>(v.x2), d, (T)cd, (T)cz, st);
                std::swap(v.x, v.x2);
            }
        };
        if (pre > 0) {
            steps(pre, true);
        } else {
            cudaMemsetAsync(v.x, 0, v.n * 4 * sizeof(T), st);
        }
        if (last) return launch_status("coarse smoothing");
        T *r = static_cast<T *>(v.r);
        if (TRANS)
            ZV_TRY(bsr_spmv_t_launch<true, V, T>(v.lanes, v.n, v.tptr, v.trow, v.tperm, data,
                                                 static_cast<const T *>(v.x), b, r, st));
        else
            ZV_TRY(bsr_spmv_launch<true, V, T>(v.lanes, v.n, v.indptr, v.indices, data,
                                               static_cast<const T *>(v.x), b, r, st));
        Level &c = L[l + 1];
        k_restrict<T><<<grid_for(c.n * 4, 256), 256, 0, st>>>(c.n, v.mptr, v.mem, r, static_cast<T *>(c.b)); count_launch();
        ZV_TRY((cycle<T, TRANS>(l + 1)));
        k_prolong_add<T><<<grid_for(v.n * 4, 256), 256, 0, st>>>(v.n, v.agg, static_cast<const T *>(c.x),
                                                                static_cast<T *>(v.x)); count_launch();
        steps(prm.postsweeps, false);
        return launch_status("v-cycle");
    }
    auto sweep = [&](bool first, const T *xin, T *xout) {
        if (TRANS) {
            if (first) jacobi_t<true>(v.lanes, v.n, v, data, dinv, b, xin, xout, omega, st);
            else jacobi_t<false>(v.lanes, v.n, v, data, dinv, b, xin, xout, omega, st);
        } else {
            if (first) jacobi<true>(v.lanes, v.n, v.indptr, v.indices, data, dinv, b, xin, xout, omega, st);
            else jacobi<false>(v.lanes, v.n, v.indptr, v.indices, data, dinv, b, xin, xout, omega, st);
        }
    };
    sweep(true, nullptr, static_cast<T *>(v.x));
    for (int s = 1; s < pre; ++s) {
        sweep(false, static_cast<const T *>(v.x), static_cast<T *>(v.x2));
        std::swap(v.x, v.x2);
    }
    if (last) return launch_status("coarse smoothing");
    T *r = static_cast<T *>(v.r);
    if (TRANS)
        ZV_TRY(bsr_spmv_t_launch<true, V, T>(v.lanes, v.n, v.tptr, v.trow, v.tperm, data,
                                             static_cast<const T *>(v.x), b, r, st));
    else
        ZV_TRY(bsr_spmv_launch<true, V, T>(v.lanes, v.n, v.indptr, v.indices, data,
                                           static_cast<const T *>(v.x), b, r, st));
    Level &c = L[l + 1];
    k_restrict<T><<<grid_for(c.n * 4, 256), 256, 0, st>>>(c.n, v.mptr, v.mem, r, static_cast<T *>(c.b)); count_launch();
    ZV_TRY((cycle<T, TRANS>(l + 1)));
    k_prolong_add<T><<<grid_for(v.n * 4, 256), 256, 0, st>>>(v.n, v.agg, static_cast<const T *>(c.x),
                                                            static_cast<T *>(v.x)); count_launch();
    for (int s = 0; s < post; ++s) {
        sweep(false, static_cast<const T *>(v.x), static_cast<T *>(v.x2));
        std::swap(v.x, v.x2);
    }
    return launch_status("v-cycle");
}

// The autotuner: after each rebuild, every level of at least AUTOTUNE_MIN_ROWS rows times one
// smoothing pass (a forward Gauss-Seidel pass over its colours, or a Jacobi sweep) with 8, 16
// and 32 lanes per row and, on a Gauss-Seidel level, with half, the base and twice the blocks
// in flight per slot, twice each after a warm-up, with CUDA events on the solver's stream, and
// keeps the fastest for all of that level's row kernels (smoothing, residual). Different lanes add a row's blocks in a different order, so with the autotuner
// on, two runs can differ in the last bits when their timings pick differently.
constexpr long long AUTOTUNE_MIN_ROWS = 2048;

template <typename T>
int Hierarchy::autotune() {
    using V = typename std::conditional<sizeof(T) == 4, float, double>::type;
    cudaEvent_t e0, e1;
    ZV_TRY(cuda_status(cudaEventCreate(&e0), "autotune event"));
    ZV_TRY(cuda_status(cudaEventCreate(&e1), "autotune event"));
    int rc = OK;
    for (size_t l = 0; l < L.size() && rc == OK; ++l) {
        Level &v = L[l];
        if (v.dense || v.n < AUTOTUNE_MIN_ROWS) continue;
        const bool gs = prm.smoother == 1 && !v.gs_off.empty();
        const V *data = gs ? CyclePick<T>::pdata(v) : CyclePick<T>::data(v);
        const V *dinv = gs ? CyclePick<T>::pdinv(v) : CyclePick<T>::dinv(v);
        T *b = static_cast<T *>(gs ? v.pb : v.b), *x = static_cast<T *>(v.x2), *y = static_cast<T *>(v.x);
        cudaMemsetAsync(b, 0, v.n * 4 * sizeof(T), st);
        cudaMemsetAsync(x, 0, v.n * 4 * sizeof(T), st);
        int best = v.lanes, best_depth = v.gs_depth;
        float best_ms = 1e30f;
        for (int G : {8, 16, 32})
            for (int sel = 0; sel < (gs ? 3 : 1); ++sel) {    // Gauss-Seidel: blocks in flight too
                v.lanes = G;
                v.gs_depth = gs ? sel : 1;
                float total = 0.0f;
                for (int rep = 0; rep < 3 && rc == OK; ++rep) {
                    cudaEventRecord(e0, st);
                    if (gs) gs_pass<false, V, T>(v, data, dinv, b, x, (T)0.5, false, st);
                    else jacobi<false>(G, v.n, v.indptr, v.indices, data, dinv, b, x, y, (T)0.5, st);
                    cudaEventRecord(e1, st);
                    rc = cuda_status(cudaEventSynchronize(e1), "autotune");
                    float ms = 0.0f;
                    cudaEventElapsedTime(&ms, e0, e1);
                    if (rep > 0) total += ms;
                }
                if (total < best_ms) {
                    best_ms = total;
                    best = G;
                    best_depth = v.gs_depth;
                }
            }
        v.lanes = best;
        v.gs_depth = best_depth;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc == OK) rc = launch_status("autotune");
    return rc;
}

// The largest eigenvalue of D^-1 A on every smoothed level, by cheb_power steps of the power
// iteration from a fixed positive start: x <- w / |w|, w = D^-1 A x (the bound of the
// Chebyshev interval; A^T shares it, D^-T A^T being similar to the transpose of D^-1 A).
// Runs in the cycle's precision on the level's work vectors; the last |w| (of a unit x) is the
// estimate, folded on the host in a fixed order.
template <typename T>
int Hierarchy::estimate_spectra() {
    using V = T;
    const int np = std::max(1, 2 * sm_count());
    double *partial;
    ZV_TRY(scratch.get(&partial, np));
    std::vector<double> host(np);
    for (Level &v : L) {
        if (v.dense) continue;
        const long long m = v.n * 4;
        const V *data = CyclePick<T>::data(v), *dinv = CyclePick<T>::dinv(v);
        T *x = static_cast<T *>(v.x), *y = static_cast<T *>(v.r), *w = static_cast<T *>(v.x2);
        const unsigned g = (unsigned)std::min<long long>(grid_for(m, 256), np);
        k_fill_start<T><<<grid_for(m, 256), 256, 0, st>>>(m, x); count_launch();
        for (int k = 0; k < std::max(prm.cheb_power, 2); ++k) {
            ZV_TRY((bsr_spmv_launch<false, V, T>(v.lanes, v.n, v.indptr, v.indices, data, x, nullptr, y, st)));
            jacobi<true, V, T>(v.lanes, v.n, v.indptr, v.indices, data, dinv, y, nullptr, w, (T)1, st);
            cudaMemsetAsync(partial, 0, np * sizeof(double), st);
            k_sumsq<T><<<g, 256, 0, st>>>(m, w, partial); count_launch();
            k_scale_by<T><<<g, 256, 0, st>>>(m, np, partial, w, x); count_launch();
        }
        ZV_TRY(cuda_status(cudaMemcpyAsync(host.data(), partial, np * sizeof(double),
                                           cudaMemcpyDeviceToHost, st), "spectral estimate"));
        ZV_TRY(cuda_status(cudaStreamSynchronize(st), "spectral estimate"));
        double sum = 0.0;
        for (double p : host) sum += p;
        const double lmax = std::sqrt(sum);
        v.cheb_lmax = std::isfinite(lmax) && lmax > 0.0 ? lmax : 2.0;
    }
    scratch.release();
    return launch_status("spectral estimate");
}

// ------------------------------------------------------------------ the solver handle

struct Solver {
    Hierarchy H;
    int restart = 30;
    int lanes0 = 8;
    cudaStream_t st = 0;
    Arena work;
    long long n4 = 0;
    double *V = nullptr, *Z = nullptr, *w = nullptr, *r = nullptr, *x = nullptr;
    double *Hm = nullptr, *cs = nullptr, *sn = nullptr, *g = nullptr, *y = nullptr;
    double *h1 = nullptr, *h2 = nullptr, *nrm = nullptr, *stat = nullptr, *partial = nullptr;
    double *lr_t = nullptr;
    double *host = nullptr;        // pinned: 4 doubles
    int ncta = 0;
    long long n = 0, nnz = 0;
    const long long *indptr = nullptr;
    const int *indices = nullptr;
    const double *data = nullptr;

    ~Solver() {
        if (host) cudaFreeHost(host);
    }

    int ensure_work(long long n4_) {
        if (n4_ == n4 && V) return OK;
        work.set_stream(st);
        work.release();
        n4 = n4_;
        const int m = restart;
        ZV_TRY(work.get(&V, (size_t)(m + 1) * n4));
        ZV_TRY(work.get(&Z, (size_t)m * n4));
        ZV_TRY(work.get(&w, n4));
        ZV_TRY(work.get(&r, n4));
        ZV_TRY(work.get(&x, n4));
        ZV_TRY(work.get(&Hm, (size_t)(m + 1) * (m + 1)));
        ZV_TRY(work.get(&cs, m + 1));
        ZV_TRY(work.get(&sn, m + 1));
        ZV_TRY(work.get(&g, m + 2));
        ZV_TRY(work.get(&y, m + 1));
        ZV_TRY(work.get(&h1, MAXV));
        ZV_TRY(work.get(&h2, MAXV));
        ZV_TRY(work.get(&nrm, MAXV));
        ZV_TRY(work.get(&stat, 4));
        ZV_TRY(work.get(&lr_t, 1));
        ncta = (int)std::min<long long>(grid_for(n4, DOT_THREADS * 4), 4LL * sm_count());
        ZV_TRY(work.get(&partial, (size_t)ncta * MAXV));
        if (!host) ZV_TRY(cuda_status(cudaMallocHost((void **)&host, 8 * sizeof(double)), "pinned"));
        return OK;
    }

    // y = A x (+ rank-one terms); resid: y = b - A x. trans: A^T, the rank-one terms w u^T.
    int apply(const double *xin, const double *b, double *out, const std::vector<LowRank> &lr,
              bool trans = false) {
        if (trans) {
            const Level &v0 = H.L[0];
            if (b) ZV_TRY(bsr_spmv_t_launch<true, double, double>(lanes0, n, v0.tptr, v0.trow, v0.tperm, data, xin, b, out, st));
            else ZV_TRY(bsr_spmv_t_launch<false, double, double>(lanes0, n, v0.tptr, v0.trow, v0.tperm, data, xin, nullptr, out, st));
        } else {
            if (b) ZV_TRY(bsr_spmv_launch<true, double, double>(lanes0, n, indptr, indices, data, xin, b, out, st));
            else ZV_TRY(bsr_spmv_launch<false, double, double>(lanes0, n, indptr, indices, data, xin, nullptr, out, st));
        }
        for (const LowRank &t : lr) {
            if (trans) {
                k_lr_dot<<<1, 256, 0, st>>>(t.nu, t.ui, t.uv, xin, lr_t); count_launch();
                k_lr_axpy<<<grid_for(t.nw, 256), 256, 0, st>>>(t.nw, t.wi, t.wv, lr_t, b ? -1.0 : 1.0, out); count_launch();
            } else {
                k_lr_dot<<<1, 256, 0, st>>>(t.nw, t.wi, t.wv, xin, lr_t); count_launch();
                k_lr_axpy<<<grid_for(t.nu, 256), 256, 0, st>>>(t.nu, t.ui, t.uv, lr_t, b ? -1.0 : 1.0, out); count_launch();
            }
        }
        return launch_status("operator");
    }

    int dot2(const double *a, const double *b, double *out_dev) {
        k_dot_partial<<<ncta, DOT_THREADS, 0, st>>>(n4, a, b, partial); count_launch();
        k_fold_cols<<<1, 32 * MAXV, 0, st>>>(ncta, 1, partial, out_dev); count_launch();
        return launch_status("dot");
    }

    int precondition(const double *in, double *out, bool trans = false) {
        Level &v0 = H.L[0];
        if (H.prm.precision == 1) {
            k_convert<double, float><<<grid_for(n4, 256), 256, 0, st>>>(n4, in, static_cast<float *>(v0.b)); count_launch();
            ZV_TRY(trans ? H.vcycle<float, true>() : H.vcycle<float, false>());
            k_convert<float, double><<<grid_for(n4, 256), 256, 0, st>>>(n4, static_cast<const float *>(v0.x), out); count_launch();
        } else {
            cudaMemcpyAsync(v0.b, in, n4 * sizeof(double), cudaMemcpyDeviceToDevice, st);
            ZV_TRY(trans ? H.vcycle<double, true>() : H.vcycle<double, false>());
            cudaMemcpyAsync(out, v0.x, n4 * sizeof(double), cudaMemcpyDeviceToDevice, st);
        }
        return launch_status("precondition");
    }

    int solve(const double *b, double *xio, double rtol, int maxiter, const std::vector<LowRank> &lr,
              int *iterations, double *residual, int *converged, bool trans = false) {
        const int m = restart;
        if (trans) ZV_TRY(H.ensure_transpose());
        const int ldh = m + 1;
        cudaMemcpyAsync(x, xio, n4 * sizeof(double), cudaMemcpyDeviceToDevice, st);
        ZV_TRY(apply(x, b, r, lr, trans));
        ZV_TRY(dot2(b, b, nrm));
        ZV_TRY(dot2(r, r, nrm + 1));
        cudaMemcpyAsync(host, nrm, 2 * sizeof(double), cudaMemcpyDeviceToHost, st);
        ZV_TRY(cuda_status(cudaStreamSynchronize(st), "solve start"));
        const double nb2 = host[0], nr2 = host[1];
        double bnorm = std::sqrt(nr2);
        if (bnorm == 0.0) bnorm = 1.0;
        const double rt = std::max(rtol, 1e-13 * std::sqrt(nb2) / bnorm);
        double beta = std::sqrt(nr2);
        double res = beta / bnorm;
        int it = 0;
        while (res > rt && it < maxiter && std::isfinite(res)) {
            k_scale<<<ncta, 256, 0, st>>>(n4, r, 1.0 / beta, nullptr, V); count_launch();
            k_init_g<<<1, 64, 0, st>>>(m, beta, g); count_launch();
            int kk = 0;
            for (int k = 0; k < m; ++k) {
                double *vk = V + (size_t)k * n4, *zk = Z + (size_t)k * n4;
                ZV_TRY(precondition(vk, zk, trans));
                ZV_TRY(apply(zk, nullptr, w, lr, trans));
                const int nv = k + 1;
                k_arnoldi_pass<0><<<ncta, DOT_THREADS, 0, st>>>(n4, V, n4, nv, nullptr, w, partial); count_launch();
                k_fold_cols<<<1, 32 * MAXV, 0, st>>>(ncta, nv, partial, h1); count_launch();
                k_arnoldi_pass<1><<<ncta, DOT_THREADS, 0, st>>>(n4, V, n4, nv, h1, w, partial); count_launch();
                k_fold_cols<<<1, 32 * MAXV, 0, st>>>(ncta, nv, partial, h2); count_launch();
                k_arnoldi_pass<2><<<ncta, DOT_THREADS, 0, st>>>(n4, V, n4, nv, h2, w, partial); count_launch();
                k_fold_cols<<<1, 32 * MAXV, 0, st>>>(ncta, 1, partial, nrm); count_launch();
                k_arnoldi_finish<<<1, 1, 0, st>>>(k, ldh, h1, h2, nrm, Hm, cs, sn, g, stat); count_launch();
                ZV_TRY(launch_status("arnoldi"));
                cudaMemcpyAsync(host, stat, 3 * sizeof(double), cudaMemcpyDeviceToHost, st);
                ZV_TRY(cuda_status(cudaStreamSynchronize(st), "arnoldi step"));
                ++it;
                kk = k + 1;
                res = host[0] / bnorm;
                const double hn = host[1];
                if (res <= rt || it >= maxiter || hn == 0.0 || !std::isfinite(res)) break;
                k_scale<<<ncta, 256, 0, st>>>(n4, w, 0.0, stat + 2, V + (size_t)(k + 1) * n4); count_launch();
            }
            k_upper_solve<<<1, 1, 0, st>>>(kk, ldh, Hm, g, y); count_launch();
            k_combine<<<ncta, 256, 0, st>>>(n4, Z, n4, kk, y, x); count_launch();
            ZV_TRY(apply(x, b, r, lr, trans));
            ZV_TRY(dot2(r, r, nrm));
            cudaMemcpyAsync(host, nrm, sizeof(double), cudaMemcpyDeviceToHost, st);
            ZV_TRY(cuda_status(cudaStreamSynchronize(st), "restart"));
            beta = std::sqrt(host[0]);
            res = beta / bnorm;
            if (!std::isfinite(res)) break;
        }
        cudaMemcpyAsync(xio, x, n4 * sizeof(double), cudaMemcpyDeviceToDevice, st);
        *iterations = it;
        *residual = res;
        *converged = res <= 1.01 * rt ? 1 : 0;
        if (!trans) H.record_solve(it, *converged != 0);
        ZV_TRY(launch_status("fgmres"));
        return std::isfinite(res) ? OK : NON_FINITE;
    }

    // ---- segmented FGMRES (one recurrence per segment; kernels above)
    Arena segwork;
    std::vector<long long> seg_rows;       // the segment bounds the buffers below were built for
    int nseg = 0, nsc = 0;                 // segments, CTAs of a segmented pass
    long long seg_n4 = 0;
    long long *cfirst = nullptr;
    int *cseg = nullptr, *sfirst = nullptr, *kk = nullptr, *cnt = nullptr, *sact = nullptr;
    double *spart = nullptr, *sh1 = nullptr, *sh2 = nullptr, *snrm = nullptr, *sbb = nullptr;
    double *srr = nullptr, *sbeta0 = nullptr, *starget = nullptr, *sH = nullptr, *scs = nullptr;
    double *ssn = nullptr, *sg = nullptr, *sy = nullptr, *sst = nullptr, *sinv = nullptr;

    int ensure_segments(int ns, const long long *rows) {
        std::vector<long long> want(rows, rows + ns + 1);
        if (want == seg_rows && cfirst && seg_n4 == n4) return OK;
        for (int q = 0; q < ns; ++q)
            if (want[q + 1] < want[q]) {
                set_error("solve_segmented: segment bounds must not decrease");
                return BAD_ARGUMENT;
            }
        if (want[0] != 0 || want[ns] != n) {
            set_error("solve_segmented: segments must cover rows 0 to %lld", (long long)n);
            return BAD_ARGUMENT;
        }
        segwork.set_stream(st);
        segwork.release();
        seg_rows = want;
        seg_n4 = n4;
        nseg = ns;
        // chunks of at least 2048 entries, about four CTAs per SM over the whole vector
        long long chunk = (n4 + 4LL * sm_count() - 1) / (4LL * sm_count());
        chunk = std::max<long long>(2048, (chunk + 255) / 256 * 256);
        std::vector<long long> cf;
        std::vector<int> cs_, sf(ns + 1);
        for (int q = 0; q < ns; ++q) {
            sf[q] = (int)cs_.size();
            for (long long a = 4 * want[q]; a < 4 * want[q + 1]; a += chunk) {
                cf.push_back(a);
                cs_.push_back(q);
            }
        }
        sf[ns] = (int)cs_.size();
        cf.push_back(n4);
        nsc = (int)cs_.size();
        const int ldh = restart + 1;
        ZV_TRY(segwork.get(&cfirst, cf.size()));
        ZV_TRY(segwork.get(&cseg, std::max(nsc, 1)));
        ZV_TRY(segwork.get(&sfirst, ns + 1));
        ZV_TRY(segwork.get(&kk, ns));
        ZV_TRY(segwork.get(&sact, ns));
        ZV_TRY(segwork.get(&cnt, 1));
        ZV_TRY(segwork.get(&spart, (size_t)std::max(nsc, 1) * MAXV));
        for (double **q : {&sh1, &sh2, &snrm, &sbb, &srr, &sy}) ZV_TRY(segwork.get(q, (size_t)ns * MAXV));
        ZV_TRY(segwork.get(&sbeta0, ns));
        ZV_TRY(segwork.get(&starget, ns));
        ZV_TRY(segwork.get(&sH, (size_t)ns * ldh * ldh));
        ZV_TRY(segwork.get(&scs, (size_t)ns * ldh));
        ZV_TRY(segwork.get(&ssn, (size_t)ns * ldh));
        ZV_TRY(segwork.get(&sg, (size_t)ns * (ldh + 1)));
        ZV_TRY(segwork.get(&sst, (size_t)ns * 4));
        ZV_TRY(segwork.get(&sinv, (size_t)ns * 4));
        ZV_TRY(cuda_status(cudaMemcpyAsync(cfirst, cf.data(), cf.size() * sizeof(long long),
                                           cudaMemcpyHostToDevice, st), "segments"));
        if (nsc)
            ZV_TRY(cuda_status(cudaMemcpyAsync(cseg, cs_.data(), nsc * sizeof(int),
                                               cudaMemcpyHostToDevice, st), "segments"));
        ZV_TRY(cuda_status(cudaMemcpyAsync(sfirst, sf.data(), (ns + 1) * sizeof(int),
                                           cudaMemcpyHostToDevice, st), "segments"));
        // the pageable host vectors above must outlive the copies
        return cuda_status(cudaStreamSynchronize(st), "segments");
    }

    // |v|^2 per segment into out (MAXV-strided)
    void seg_norm2(const double *v, double *out) {
        k_seg_pass<3><<<nsc, DOT_THREADS, 0, st>>>(cfirst, cseg, nullptr, 0, 0, nullptr,
                                                   const_cast<double *>(v), spart); count_launch();
        k_seg_fold<<<nseg, 32 * MAXV, 0, st>>>(sfirst, 1, spart, out); count_launch();
    }

    int read_count(const char *what, int *out) {
        ZV_TRY(cuda_status(cudaMemcpyAsync(host, cnt, sizeof(int), cudaMemcpyDeviceToHost, st), what));
        ZV_TRY(cuda_status(cudaStreamSynchronize(st), what));
        std::memcpy(out, host, sizeof(int));
        return OK;
    }

    int solve_segmented(int ns, const long long *rows, const int *active, const double *b,
                        double *xio, double rtol, int maxiter, const std::vector<LowRank> &lr,
                        int *iterations, double *residuals, int *converged) {
        ZV_TRY(ensure_segments(ns, rows));
        {
            std::vector<int> on(ns, 1);
            if (active)
                for (int q = 0; q < ns; ++q) on[q] = active[q] ? 1 : 0;
            ZV_TRY(cuda_status(cudaMemcpyAsync(sact, on.data(), ns * sizeof(int),
                                               cudaMemcpyHostToDevice, st), "segments: active"));
            ZV_TRY(cuda_status(cudaStreamSynchronize(st), "segments: active"));
        }
        if (nsc == 0) {
            *iterations = 0;
            for (int q = 0; q < ns; ++q) {
                residuals[q] = 0.0;
                converged[q] = 1;
            }
            return OK;
        }
        const int m = restart, ldh = m + 1;
        const unsigned gs = grid_for(ns, 128);
        cudaMemcpyAsync(x, xio, n4 * sizeof(double), cudaMemcpyDeviceToDevice, st);
        ZV_TRY(apply(x, b, r, lr));
        seg_norm2(b, sbb);
        seg_norm2(r, srr);
        k_seg_targets<<<gs, 128, 0, st>>>(ns, rtol, sbb, srr, sact, sbeta0, starget); count_launch();
        int it = 0, open = 0;
        while (it < maxiter) {
            cudaMemsetAsync(cnt, 0, sizeof(int), st);
            k_seg_init<<<gs, 128, 0, st>>>(ns, ldh, srr, starget, sg, kk, sinv, cnt); count_launch();
            ZV_TRY(read_count("segmented start", &open));
            if (open == 0) break;
            k_seg_scale<<<nsc, 256, 0, st>>>(cfirst, cseg, r, sinv, V); count_launch();
            int ku = 0;
            for (int k = 0; k < m; ++k) {
                double *vk = V + (size_t)k * n4, *zk = Z + (size_t)k * n4;
                ZV_TRY(precondition(vk, zk));
                ZV_TRY(apply(zk, nullptr, w, lr));
                const int nv = k + 1;
                k_seg_pass<0><<<nsc, DOT_THREADS, 0, st>>>(cfirst, cseg, V, n4, nv, nullptr, w, spart); count_launch();
                k_seg_fold<<<ns, 32 * MAXV, 0, st>>>(sfirst, nv, spart, sh1); count_launch();
                k_seg_pass<1><<<nsc, DOT_THREADS, 0, st>>>(cfirst, cseg, V, n4, nv, sh1, w, spart); count_launch();
                k_seg_fold<<<ns, 32 * MAXV, 0, st>>>(sfirst, nv, spart, sh2); count_launch();
                k_seg_pass<2><<<nsc, DOT_THREADS, 0, st>>>(cfirst, cseg, V, n4, nv, sh2, w, spart); count_launch();
                k_seg_fold<<<ns, 32 * MAXV, 0, st>>>(sfirst, 1, spart, snrm); count_launch();
                cudaMemsetAsync(cnt, 0, sizeof(int), st);
                k_seg_finish<<<gs, 128, 0, st>>>(k, ns, ldh, sh1, sh2, snrm, starget, sH, scs, ssn, sg,
                                                 kk, sst, cnt); count_launch();
                ZV_TRY(launch_status("segmented arnoldi"));
                ZV_TRY(read_count("segmented step", &open));
                ++it;
                ku = k + 1;
                if (open == 0 || it >= maxiter) break;
                k_seg_scale<<<nsc, 256, 0, st>>>(cfirst, cseg, w, sst, V + (size_t)(k + 1) * n4); count_launch();
            }
            k_seg_upper<<<gs, 128, 0, st>>>(ns, ku, ldh, sH, sg, kk, sy); count_launch();
            k_seg_combine<<<nsc, 256, 0, st>>>(cfirst, cseg, Z, n4, ku, sy, x); count_launch();
            ZV_TRY(apply(x, b, r, lr));
            seg_norm2(r, srr);
            cudaMemsetAsync(cnt, 0, sizeof(int), st);
            k_seg_open<<<gs, 128, 0, st>>>(ns, srr, starget, cnt); count_launch();
            ZV_TRY(read_count("segmented restart", &open));
            if (open == 0) break;
        }
        // per segment: |r| / beta0 and whether |r| <= 1.01 target
        std::vector<double> rr((size_t)ns * MAXV), b0(ns), tg(ns);
        ZV_TRY(cuda_status(cudaMemcpyAsync(rr.data(), srr, rr.size() * sizeof(double),
                                           cudaMemcpyDeviceToHost, st), "segmented result"));
        ZV_TRY(cuda_status(cudaMemcpyAsync(b0.data(), sbeta0, ns * sizeof(double),
                                           cudaMemcpyDeviceToHost, st), "segmented result"));
        ZV_TRY(cuda_status(cudaMemcpyAsync(tg.data(), starget, ns * sizeof(double),
                                           cudaMemcpyDeviceToHost, st), "segmented result"));
        cudaMemcpyAsync(xio, x, n4 * sizeof(double), cudaMemcpyDeviceToDevice, st);
        ZV_TRY(cuda_status(cudaStreamSynchronize(st), "segmented result"));
        bool all = true, finite = true;
        for (int q = 0; q < ns; ++q) {
            const double rn = std::sqrt(rr[(size_t)q * MAXV]);
            residuals[q] = b0[q] > 0.0 ? rn / b0[q] : rn;
            converged[q] = rn <= 1.01 * tg[q] ? 1 : 0;
            all = all && converged[q];
            finite = finite && std::isfinite(rn);
        }
        *iterations = it;
        H.record_solve(it, all);
        ZV_TRY(launch_status("segmented fgmres"));
        return finite ? OK : NON_FINITE;
    }
};

}  // namespace

// one V-cycle (L[0].b -> L[0].x) as a CUDA graph: captured on first use after each rebuild
// (on a stream of the handle's own: the caller's may be the legacy stream, which cannot be
// captured) and replayed on the caller's stream; every buffer it touches keeps its address
// until the next rebuild
template <typename T, bool TRANS>
int Hierarchy::vcycle() {
    cudaGraphExec_t &g = graphs[sizeof(T) == 4 ? 1 : 0][TRANS ? 1 : 0];
    long long &kernels = graph_kernels[sizeof(T) == 4 ? 1 : 0][TRANS ? 1 : 0];
    if (!g) {
        const long long before = launches_so_far();
        if (!capture_stream)
            ZV_TRY(cuda_status(cudaStreamCreateWithFlags(&capture_stream, cudaStreamNonBlocking),
                               "capture stream"));
        cudaStream_t caller = st;
        ZV_TRY(cuda_status(cudaStreamSynchronize(caller), "before capture"));
        st = capture_stream;
        cudaGraph_t graph = nullptr;
        int rc = cuda_status(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal), "capture");
        if (rc == OK) {
            rc = cycle<T, TRANS>(0);
            const int rc2 = cuda_status(cudaStreamEndCapture(st, &graph), "end capture");
            if (rc == OK) rc = rc2;
        }
        st = caller;
        // the launches recorded during capture ran nothing: count them at each replay instead
        kernels = launches_so_far() - before;
        count_launches(-kernels);
        if (rc == OK) rc = cuda_status(cudaGraphInstantiate(&g, graph, 0), "instantiate");
        if (graph) cudaGraphDestroy(graph);
        if (rc != OK) {
            g = nullptr;
            return rc;
        }
    }
    count_launches(kernels);
    return cuda_status(cudaGraphLaunch(g, st), "graph launch");
}

}  // namespace zvfv

using namespace zvfv;

extern "C" {

int zvfv_solver_create(void **handle, int precision, int smoother, int strength, int passes,
                       int presweeps, int postsweeps, double omega, int coarse_sweeps,
                       int max_levels, int rebuild_every, int restart) {
    if (!handle || precision < 0 || precision > 1 || smoother < 0 || smoother > 4 || restart < 1 ||
        restart > MAXV - 1 || passes < 1 || presweeps < 1 || postsweeps < 0 || max_levels < 1) {
        set_error("solver_create: bad arguments");
        return BAD_ARGUMENT;
    }
    Solver *s = new Solver;
    s->H.prm.precision = precision;
    s->H.prm.smoother = smoother;
    s->H.prm.strength = strength;
    s->H.prm.passes = passes;
    s->H.prm.presweeps = presweeps;
    s->H.prm.postsweeps = postsweeps;
    s->H.prm.omega = omega;
    s->H.prm.coarse_sweeps = coarse_sweeps;
    s->H.prm.max_levels = max_levels;
    s->H.prm.rebuild_every = rebuild_every;
    s->restart = restart;
    *handle = s;
    return OK;
}

int zvfv_solver_setup(void *handle, int64_t n, int64_t nnzb, const int64_t *indptr,
                      const int32_t *indices, const double *data, void *stream) {
    Solver *s = static_cast<Solver *>(handle);
    if (!s || n <= 0 || nnzb <= 0) {
        set_error("solver_setup: bad arguments");
        return BAD_ARGUMENT;
    }
    s->st = as_stream(stream);
    s->n = n;
    s->nnz = nnzb;
    s->indptr = (const long long *)indptr;
    s->indices = indices;
    s->data = data;
    s->lanes0 = lanes_for(n, nnzb);
    ZV_TRY(s->ensure_work(n * 4));
    return s->H.setup(n, nnzb, (const long long *)indptr, indices, data, s->st);
}

int zvfv_solver_solve(void *handle, const double *b, double *x, double rtol, int maxiter,
                      int n_lowrank, const int64_t *const *u_idx, const double *const *u_val,
                      const int64_t *u_len, const int64_t *const *w_idx, const double *const *w_val,
                      const int64_t *w_len, int *iterations, double *residual, int *converged,
                      void *stream) {
    Solver *s = static_cast<Solver *>(handle);
    if (!s || !s->data || !b || !x || maxiter < 0) {
        set_error("solver_solve: not set up or bad arguments");
        return BAD_ARGUMENT;
    }
    s->st = as_stream(stream);
    s->H.st = s->st;
    std::vector<LowRank> lr;
    for (int q = 0; q < n_lowrank; ++q)
        lr.push_back({(const long long *)u_idx[q], u_val[q], (long long)u_len[q],
                      (const long long *)w_idx[q], w_val[q], (long long)w_len[q]});
    return s->solve(b, x, rtol, maxiter, lr, iterations, residual, converged);
}

// FGMRES with one Krylov recurrence per segment of rows (row_bounds: n_segments + 1
// ascending host values from 0 to n): the block-diagonal system of independent instances.
// Each segment stops at its own target, rtol times its initial residual (floor 1e-13 |b_s|);
// the solve ends when every segment has, or after maxiter Krylov steps (shared by all).
// active: n_segments host flags or null; a segment marked 0 takes no steps and keeps its guess.
// residuals / converged: n_segments host values (relative residual, 0/1).
int zvfv_solver_solve_segmented(void *handle, int n_segments, const int64_t *row_bounds,
                                const int *active, const double *b, double *x, double rtol,
                                int maxiter,
                                int n_lowrank, const int64_t *const *u_idx,
                                const double *const *u_val, const int64_t *u_len,
                                const int64_t *const *w_idx, const double *const *w_val,
                                const int64_t *w_len, int *iterations, double *residuals,
                                int *converged, void *stream) {
    Solver *s = static_cast<Solver *>(handle);
    if (!s || !s->data || !b || !x || maxiter < 0 || n_segments < 1 || !row_bounds || !iterations ||
        !residuals || !converged) {
        set_error("solver_solve_segmented: not set up or bad arguments");
        return BAD_ARGUMENT;
    }
    s->st = as_stream(stream);
    s->H.st = s->st;
    std::vector<LowRank> lr;
    for (int q = 0; q < n_lowrank; ++q)
        lr.push_back({(const long long *)u_idx[q], u_val[q], (long long)u_len[q],
                      (const long long *)w_idx[q], w_val[q], (long long)w_len[q]});
    return s->solve_segmented(n_segments, (const long long *)row_bounds, active, b, x, rtol,
                              maxiter, lr, iterations, residuals, converged);
}

// the adjoint solve: A^T x = b with the same hierarchy, transposed (same arguments)
int zvfv_solver_solve_t(void *handle, const double *b, double *x, double rtol, int maxiter,
                        int n_lowrank, const int64_t *const *u_idx, const double *const *u_val,
                        const int64_t *u_len, const int64_t *const *w_idx,
                        const double *const *w_val, const int64_t *w_len, int *iterations,
                        double *residual, int *converged, void *stream) {
    Solver *s = static_cast<Solver *>(handle);
    if (!s || !s->data || !b || !x || maxiter < 0) {
        set_error("solver_solve_t: not set up or bad arguments");
        return BAD_ARGUMENT;
    }
    s->st = as_stream(stream);
    s->H.st = s->st;
    std::vector<LowRank> lr;
    for (int q = 0; q < n_lowrank; ++q)
        lr.push_back({(const long long *)u_idx[q], u_val[q], (long long)u_len[q],
                      (const long long *)w_idx[q], w_val[q], (long long)w_len[q]});
    return s->solve(b, x, rtol, maxiter, lr, iterations, residual, converged, true);
}

int zvfv_solver_vcycle(void *handle, const double *r, double *z, void *stream) {
    Solver *s = static_cast<Solver *>(handle);
    if (!s || !s->data) {
        set_error("solver_vcycle: not set up");
        return BAD_ARGUMENT;
    }
    s->st = as_stream(stream);
    s->H.st = s->st;
    return s->precondition(r, z);
}

// z = one transposed V-cycle applied to r: the hierarchy of A on every level's transpose
// (A^T, D^-T, transposed Gauss-Seidel sweeps, the dense inverse transposed), the
// preconditioner of adjoint solves outside this library. Builds the transposes on first use.
int zvfv_solver_vcycle_t(void *handle, const double *r, double *z, void *stream) {
    Solver *s = static_cast<Solver *>(handle);
    if (!s || !s->data) {
        set_error("solver_vcycle_t: not set up");
        return BAD_ARGUMENT;
    }
    s->st = as_stream(stream);
    s->H.st = s->st;
    ZV_TRY(s->H.ensure_transpose());
    return s->precondition(r, z, true);
}

// `passes` forward Gauss-Seidel passes over the colours of level `level` (one of the
// Gauss-Seidel levels), or with the Chebyshev smoother `passes` Chebyshev steps on any level
// but a dense coarsest one, on the level's own work vectors, in the hierarchy's precision: the
// smoother kernel alone, for timing it (the V-cycle graph runs the same launches). The work
// vectors' contents are overwritten; the V-cycle does not depend on them between cycles.
int zvfv_solver_smooth(void *handle, int level, int passes, void *stream) {
    Solver *s = static_cast<Solver *>(handle);
    if (!s || !s->data || level < 0 || level >= (int)s->H.L.size() || passes < 1) {
        set_error("solver_smooth: not set up, or no level %d", level);
        return BAD_ARGUMENT;
    }
    Level &v = s->H.L[level];
    const cudaStream_t st = as_stream(stream);
    if (s->H.prm.smoother == 2 && !v.dense) {
        // alternate x and x2 without swapping the level's pointers (the captured V-cycle
        // graph keeps them); after the first step, the recurrence's limiting coefficients
        const double hi = 1.1 * v.cheb_lmax, lo = hi / s->H.prm.cheb_ratio;
        const double theta = 0.5 * (hi + lo), delta = 0.5 * (hi - lo), sigma = theta / delta;
        const double rho = sigma - std::sqrt(sigma * sigma - 1.0);
        for (int q = 0; q < passes; ++q) {
            void *xin = (q % 2) ? v.x2 : v.x, *xout = (q % 2) ? v.x : v.x2;
            const double c = q == 0 ? 0.0 : rho * rho, cz = q == 0 ? 1.0 / theta : 2.0 * rho / delta;
            if (s->H.prm.precision == 1)
                cheby<false, false, float, float>(v, v.data32, v.dinv32, static_cast<const float *>(v.b),
                                                  static_cast<const float *>(xin), static_cast<float *>(xout),
                                                  static_cast<float *>(v.r), (float)c, (float)cz, st);
            else
                cheby<false, false, double, double>(v, v.data, v.dinv64, static_cast<const double *>(v.b),
                                                    static_cast<const double *>(xin),
                                                    static_cast<double *>(xout),
                                                    static_cast<double *>(v.r), c, cz, st);
        }
        return launch_status("solver_smooth");
    }
    if (v.gs_off.empty() || !v.pb || !v.x2) {
        set_error("solver_smooth: level %d is not smoothed by Gauss-Seidel, DILU or Chebyshev",
                  level);
        return BAD_ARGUMENT;
    }
    const int sm = s->H.prm.smoother;
    if (sm == 3 || sm == 4) {                // DILU / ILU(0) steps (residual, forward, backward)
        for (int q = 0; q < passes; ++q) {
            if (s->H.prm.precision == 1) {
                const float *fac = sm == 4 ? v.lu32 : v.pdinv32;
                float *x = static_cast<float *>(v.x2), *r = static_cast<float *>(v.r),
                      *w = static_cast<float *>(v.x);
                const float *b = static_cast<const float *>(v.pb);
                if (sm == 4) lu_sweep<true, float, float>(v, v.pdata32, fac, b, x, r, w, (float)s->H.prm.omega, false, st);
                else lu_sweep<false, float, float>(v, v.pdata32, fac, b, x, r, w, (float)s->H.prm.omega, false, st);
            } else {
                const double *fac = sm == 4 ? v.lu64 : v.pdinv64;
                double *x = static_cast<double *>(v.x2), *r = static_cast<double *>(v.r),
                       *w = static_cast<double *>(v.x);
                const double *b = static_cast<const double *>(v.pb);
                if (sm == 4) lu_sweep<true, double, double>(v, v.pdata64, fac, b, x, r, w, s->H.prm.omega, false, st);
                else lu_sweep<false, double, double>(v, v.pdata64, fac, b, x, r, w, s->H.prm.omega, false, st);
            }
        }
        return launch_status("solver_smooth");
    }
    for (int q = 0; q < passes; ++q) {
        if (s->H.prm.precision == 1)
            gs_pass<false, float, float>(v, v.pdata32, v.pdinv32, static_cast<const float *>(v.pb),
                                         static_cast<float *>(v.x2), (float)s->H.prm.omega, false, st);
        else
            gs_pass<false, double, double>(v, v.pdata64, v.pdinv64,
                                           static_cast<const double *>(v.pb),
                                           static_cast<double *>(v.x2), s->H.prm.omega, false, st);
    }
    return launch_status("solver_smooth");
}

// levels, and per level rows and blocks (arrays of max_levels entries)
int zvfv_solver_set_option(void *handle, const char *name, double value) {
    Solver *s = static_cast<Solver *>(handle);
    if (!s || !name) {
        set_error("solver_set_option: no handle or name");
        return BAD_ARGUMENT;
    }
    Params &p = s->H.prm;
    const std::string opt(name);
    if (opt == "autotune") p.autotune = value != 0.0 ? 1 : 0;
    else if (opt == "gs_levels" && value >= 0) p.gs_levels = (int)value;
    else if (opt == "jacobi_sweeps" && value >= 1) p.jacobi_sweeps = (int)value;
    else if (opt == "jacobi_omega" && value > 0) p.jacobi_omega = value;
    else if (opt == "rebuild_ratio" && value >= 1) p.rebuild_ratio = value;
    else if (opt == "cheb_ratio" && value > 1) p.cheb_ratio = value;
    else if (opt == "cheb_power" && value >= 2) p.cheb_power = (int)value;
    else {
        set_error("solver_set_option: unknown option or bad value: %s = %g", name, value);
        return BAD_ARGUMENT;
    }
    s->H.request_rebuild();                  // the next set-up builds with the new setting
    return OK;
}

int zvfv_solver_get_option(void *handle, const char *name, double *value) {
    Solver *s = static_cast<Solver *>(handle);
    if (!s || !name || !value) {
        set_error("solver_get_option: no handle, name or output");
        return BAD_ARGUMENT;
    }
    const Params &p = s->H.prm;
    const std::string opt(name);
    if (opt == "autotune") *value = p.autotune;
    else if (opt == "gs_levels") *value = p.gs_levels;
    else if (opt == "jacobi_sweeps") *value = p.jacobi_sweeps;
    else if (opt == "jacobi_omega") *value = p.jacobi_omega;
    else if (opt == "rebuild_ratio") *value = p.rebuild_ratio;
    else if (opt == "cheb_ratio") *value = p.cheb_ratio;
    else if (opt == "cheb_power") *value = p.cheb_power;
    else if (opt == "cheb_lmax") *value = s->H.L.empty() ? 0.0 : s->H.L[0].cheb_lmax;
    else if (opt == "rebuilds") *value = (double)s->H.rebuilds;
    else if (opt == "setups") *value = (double)s->H.setups;
    else {
        set_error("solver_get_option: unknown option %s", name);
        return BAD_ARGUMENT;
    }
    return OK;
}

int zvfv_solver_stats(void *handle, int max_levels, int *levels, int64_t *rows, int64_t *blocks) {
    Solver *s = static_cast<Solver *>(handle);
    if (!s) return BAD_ARGUMENT;
    *levels = (int)s->H.L.size();
    for (int l = 0; l < *levels && l < max_levels; ++l) {
        rows[l] = s->H.L[l].n;
        blocks[l] = s->H.L[l].nnz;
    }
    return OK;
}

// level l's size, and its aggregate of every row (into agg, n entries, if not null)
int zvfv_solver_level(void *handle, int level, int64_t *n, int64_t *nnzb, int64_t *n_coarse,
                      int32_t *agg, void *stream) {
    Solver *s = static_cast<Solver *>(handle);
    if (!s || level < 0 || level >= (int)s->H.L.size()) {
        set_error("solver_level: no level %d", level);
        return BAD_ARGUMENT;
    }
    const Level &v = s->H.L[level];
    *n = v.n;
    *nnzb = v.nnz;
    *n_coarse = v.agg ? v.nc : 0;
    if (agg && v.agg)
        return cuda_status(cudaMemcpyAsync(agg, v.agg, v.n * sizeof(int), cudaMemcpyDeviceToDevice,
                                           as_stream(stream)), "copy");
    return OK;
}

int zvfv_solver_destroy(void *handle) {
    Solver *s = static_cast<Solver *>(handle);
    if (!s) return OK;
    cudaStreamSynchronize(s->st);
    delete s;
    return OK;
}

}  // extern "C"
