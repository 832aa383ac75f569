// Node-based kernels: nodal gradients through the gradient operator on the block pattern,
// neighbour extremes for the limiter, the boundary/scaling pass that finishes every row of
// the assembled system, the state update, and the deterministic reduction of per-CTA
// partial statistics.
#include <mutex>

#include "common.cuh"

namespace zvfv {
namespace {

constexpr int LANES = 8;          // lanes per row of the gradient and min/max kernels

// Nodal gradients of nc <= 4 fields: out[i][c][k] = sum_p gop[p][k] phi[col(p)][c]
// (zvcfd/fv/fast.py:310-325). 8 lanes per row, xor-butterfly reduction. With sym (N, 3)
// the mirror-symmetry rule of symmetry-plane nodes is applied on the way out
// (zvcfd/fv/reference.py:385-407): the first nvec fields form a vector (u, v, w).
__global__ void k_gradient(long long n, int nc, int nvec, const long long *__restrict__ indptr,
                           const int *__restrict__ indices, const double *__restrict__ gop,
                           const double *__restrict__ phi, const unsigned char *__restrict__ sym,
                           double *__restrict__ out) {
    const long long gid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long row = gid / LANES;
    const int lane = threadIdx.x % LANES;
    double acc[12];
#pragma unroll
    for (int q = 0; q < 12; ++q) acc[q] = 0.0;
    if (row < n) {
        const long long p1 = indptr[row + 1];
        for (long long p = indptr[row] + lane; p < p1; p += LANES) {
            const long long j = indices[p];
            const double g0 = gop[p * 3], g1 = gop[p * 3 + 1], g2 = gop[p * 3 + 2];
#pragma unroll
            for (int c = 0; c < 4; ++c) {
                if (c < nc) {
                    const double v = phi[j * nc + c];
                    acc[c * 3] += g0 * v;
                    acc[c * 3 + 1] += g1 * v;
                    acc[c * 3 + 2] += g2 * v;
                }
            }
        }
    }
#pragma unroll
    for (int off = LANES / 2; off > 0; off >>= 1)
#pragma unroll
        for (int q = 0; q < 12; ++q) acc[q] += __shfl_xor_sync(0xffffffffu, acc[q], off, LANES);
    if (row >= n) return;
    bool on[3] = {false, false, false};
    if (sym) {
        on[0] = sym[row * 3];
        on[1] = sym[row * 3 + 1];
        on[2] = sym[row * 3 + 2];
    }
    for (int q = lane; q < nc * 3; q += LANES) {
        const int c = q / 3, k = q % 3;
        double v = acc[0];
#pragma unroll
        for (int w = 0; w < 12; ++w)
            if (w == q) v = acc[w];
        if (sym) {
            for (int ax = 0; ax < 3; ++ax) {
                if (!on[ax]) continue;
                if (c < nvec) {
                    if ((c == ax) != (k == ax)) v = 0.0;
                } else if (k == ax) {
                    v = 0.0;
                }
            }
        }
        out[row * nc * 3 + q] = v;
    }
}

// Extremes of each velocity component over the pattern row (the nodes sharing an element)
__global__ void k_minmax(long long n, const long long *__restrict__ indptr,
                         const int *__restrict__ indices, const double *__restrict__ U,
                         double *__restrict__ lo, double *__restrict__ hi) {
    const long long gid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long row = gid / LANES;
    const int lane = threadIdx.x % LANES;
    double l[3] = {1e300, 1e300, 1e300}, h[3] = {-1e300, -1e300, -1e300};
    if (row < n) {
        const long long p1 = indptr[row + 1];
        for (long long p = indptr[row] + lane; p < p1; p += LANES) {
            const long long j = indices[p];
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                const double u = U[j * 3 + k];
                l[k] = fmin(l[k], u);
                h[k] = fmax(h[k], u);
            }
        }
    }
#pragma unroll
    for (int off = LANES / 2; off > 0; off >>= 1)
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            l[k] = fmin(l[k], __shfl_xor_sync(0xffffffffu, l[k], off, LANES));
            h[k] = fmax(h[k], __shfl_xor_sync(0xffffffffu, h[k], off, LANES));
        }
    if (row < n && lane < 3) {
        lo[row * 3 + lane] = l[lane];
        hi[row * 3 + lane] = h[lane];
    }
}

struct FinaliseArgs {
    long long n;
    const long long *indptr;
    const int *indices;
    const long long *dpos;
    double *data, *b;
    int has_time;
    const double *tdiag, *trhs, *fV, *force, *inflow, *mb, *wcons, *wonly, *wstab;
    int stokes;
    const double *snl;
    const unsigned char *fixed, *known;
    const double *vel, *pval;
    int eliminate;
    const long long *rawoff;
    double *rawdata, *rawb;
    const double *x, *aP, *V;
    double rho;
    const double *scal, *lscale;
    double *rs_out, *partial;
};

constexpr int FIN_THREADS = 256;

// Thread (row i, component r) owns row 4i + r of the system in every block of the block row
// (zvcfd/fv/_cuda_bc.py:32-138). In order: the known terms; a copy of the row for the rows the
// solver keeps; Dirichlet rows (identity, or symmetric elimination of known columns); the
// residual of the current state for the report; the dimensionless row scaling. Per CTA:
// 8 partials (sum of squares and max of the normalised residual, per equation).
__global__ void __launch_bounds__(FIN_THREADS) k_finalise(const FinaliseArgs g) {
    const long long gid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long i = gid >> 2;
    const int r = (int)(gid & 3);
    double sq = 0.0, mx = 0.0;
    if (i < g.n) {
        const long long p0 = g.indptr[i], p1 = g.indptr[i + 1], pd = g.dpos[i];
        double bi = g.b[i * 4 + r];
        if (r < 3) {
            bi += (g.has_time ? g.trhs[i * 3 + r] : 0.0) + g.fV[i * 3 + r] - g.force[i * 3 + r];
            double dd = g.has_time ? g.tdiag[i] : 0.0;
            if (!g.stokes) {
                const double m = g.mb[i];
                dd += g.wcons[i] * m + g.wonly[i] * fmax(m, 0.0) + g.wstab[i] * fmax(-m, 0.0);
            }
            g.data[pd * 16 + r * 5] += dd;
            g.data[pd * 16 + r * 4 + 3] += g.snl[i * 3 + r];
        } else {
            bi -= g.inflow[i];
        }
        const long long ro = g.rawoff[i];
        if (ro >= 0) {
            for (long long p = p0; p < p1; ++p) {
                const double2 *src = reinterpret_cast<const double2 *>(g.data + p * 16 + r * 4);
                double2 *dst = reinterpret_cast<double2 *>(g.rawdata + (ro + (p - p0)) * 16 + r * 4);
                dst[0] = src[0];
                dst[1] = src[1];
            }
            g.rawb[i * 4 + r] = bi;
        }
        const bool fx = g.fixed[i * 4 + r];
        const double uref = g.scal[0], pref = g.scal[1];
        double s;
        if (g.lscale[i] > 0.0 && r == 3) s = g.lscale[i] / uref;
        else if (fx) s = r < 3 ? 1.0 / uref : 1.0 / pref;
        else s = r < 3 ? 1.0 / (g.aP[i] * uref) : 1.0 / (g.rho * uref * pow(g.V[i], 2.0 / 3.0));
        double ax = 0.0;
        if (fx) {
            for (long long p = p0; p < p1; ++p) {
                double2 *row = reinterpret_cast<double2 *>(g.data + p * 16 + r * 4);
                row[0] = make_double2(0.0, 0.0);
                row[1] = make_double2(0.0, 0.0);
            }
            g.data[pd * 16 + r * 5] = s;          // the identity row, scaled
            bi = r < 3 ? g.vel[i * 3 + r] : g.pval[i];
            ax = g.x[i * 4 + r];
        } else {
            // one pass over the row: symmetric elimination of known columns, the row's product
            // with the current state (for the residual report), and the scaled store - in the
            // order of the separate passes they replace, so every sum is unchanged
            const uchar4 *known4 = reinterpret_cast<const uchar4 *>(g.known);
            for (long long p = p0; p < p1; ++p) {
                const long long j = g.indices[p];
                double2 *row = reinterpret_cast<double2 *>(g.data + p * 16 + r * 4);
                double2 ra = row[0], rb = row[1];
                if (g.eliminate) {
                    const uchar4 kn = known4[j];
                    if (kn.x | kn.y | kn.z | kn.w) {
                        double a[4] = {ra.x, ra.y, rb.x, rb.y};
                        const unsigned char k4[4] = {kn.x, kn.y, kn.z, kn.w};
                        for (int c = 0; c < 4; ++c)
                            if (k4[c]) {
                                const double v = c < 3 ? g.vel[j * 3 + c] : g.pval[j];
                                bi -= a[c] * v;
                                a[c] = 0.0;
                            }
                        ra = make_double2(a[0], a[1]);
                        rb = make_double2(a[2], a[3]);
                    }
                }
                const double2 xa = reinterpret_cast<const double2 *>(g.x)[j * 2];
                const double2 xb = reinterpret_cast<const double2 *>(g.x)[j * 2 + 1];
                ax += ra.x * xa.x + ra.y * xa.y + rb.x * xb.x + rb.y * xb.y;
                row[0] = make_double2(ra.x * s, ra.y * s);
                row[1] = make_double2(rb.x * s, rb.y * s);
            }
            const double res = bi - ax;
            const double nrm = r < 3 ? g.aP[i] : g.rho * pow(g.V[i], 2.0 / 3.0);
            const double v = fabs(res) / nrm;
            sq = v * v;
            mx = v;
        }
        g.b[i * 4 + r] = bi * s;
        g.rs_out[i * 4 + r] = s;
    }
    // per-CTA partials: lanes of equal r reduce by xor over bits 2..4, then across warps
#pragma unroll
    for (int off = 4; off < 32; off <<= 1) {
        sq += __shfl_xor_sync(0xffffffffu, sq, off);
        mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, off));
    }
    __shared__ double red[FIN_THREADS / 32][8];
    const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
    if (lane < 4) {
        red[warp][lane] = sq;
        red[warp][4 + lane] = mx;
    }
    __syncthreads();
    if (threadIdx.x < 8) {
        const int q = threadIdx.x;
        double v = red[0][q];
        for (int w = 1; w < FIN_THREADS / 32; ++w) v = q < 4 ? v + red[w][q] : fmax(v, red[w][q]);
        g.partial[blockIdx.x * 8 + q] = v;
    }
}

constexpr int UPD_THREADS = 256;

// U, P <- x, with per-CTA partials max |dU|, max |U|, max |dp|, min p, max p
// (zvcfd/fv/_cuda_bc.py:140-175)
__global__ void __launch_bounds__(UPD_THREADS)
k_update(long long n, const double *__restrict__ X, double *__restrict__ U, double *__restrict__ P,
         double *__restrict__ partial) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    double du = 0.0, um = 0.0, dp = 0.0, pmin = 1e300, pmax = -1e300;
    if (i < n) {
        for (int k = 0; k < 3; ++k) {
            const double v = X[i * 4 + k];
            du = fmax(du, fabs(v - U[i * 3 + k]));
            um = fmax(um, fabs(v));
            U[i * 3 + k] = v;
        }
        const double p = X[i * 4 + 3];
        dp = fabs(p - P[i]);
        pmin = p;
        pmax = p;
        P[i] = p;
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        du = fmax(du, __shfl_xor_sync(0xffffffffu, du, off));
        um = fmax(um, __shfl_xor_sync(0xffffffffu, um, off));
        dp = fmax(dp, __shfl_xor_sync(0xffffffffu, dp, off));
        pmin = fmin(pmin, __shfl_xor_sync(0xffffffffu, pmin, off));
        pmax = fmax(pmax, __shfl_xor_sync(0xffffffffu, pmax, off));
    }
    __shared__ double red[UPD_THREADS / 32][5];
    const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
    if (lane == 0) {
        red[warp][0] = du;
        red[warp][1] = um;
        red[warp][2] = dp;
        red[warp][3] = pmin;
        red[warp][4] = pmax;
    }
    __syncthreads();
    if (threadIdx.x < 5) {
        const int q = threadIdx.x;
        double v = red[0][q];
        for (int w = 1; w < UPD_THREADS / 32; ++w) v = q == 3 ? fmin(v, red[w][q]) : fmax(v, red[w][q]);
        partial[blockIdx.x * 5 + q] = v;
    }
}

// One CTA folds rows of partials (nrows, width) column by column: op 0 sum, 1 max, 2 min.
// Sums are taken in a fixed order (strided per thread, then a fixed tree): deterministic.
__global__ void k_fold(long long nrows, int width, const double *__restrict__ partial,
                       const int *__restrict__ ops, double *__restrict__ out) {
    __shared__ double red[256];
    for (int c = 0; c < width; ++c) {
        const int op = ops[c];
        double v = op == 0 ? 0.0 : (op == 1 ? -1e300 : 1e300);
        for (long long r = threadIdx.x; r < nrows; r += blockDim.x) {
            const double w = partial[r * width + c];
            v = op == 0 ? v + w : (op == 1 ? fmax(v, w) : fmin(v, w));
        }
        red[threadIdx.x] = v;
        __syncthreads();
        for (int s = blockDim.x / 2; s > 0; s >>= 1) {
            if (threadIdx.x < s) {
                const double a = red[threadIdx.x], b = red[threadIdx.x + s];
                red[threadIdx.x] = op == 0 ? a + b : (op == 1 ? fmax(a, b) : fmin(a, b));
            }
            __syncthreads();
        }
        if (threadIdx.x == 0) out[c] = red[0];
        __syncthreads();
    }
}

// Scratch of the allocation-free update (zvfv_update_noalloc): the per-CTA partial rows of
// k_update for up to NOALLOC_MAX_PARTIAL_ROWS CTAs of UPD_THREADS nodes, and the fold
// operations of its five columns (max |dU|, max |U|, max |dp|, min p, max p). 2.5 MiB that
// every GPU which loads the library holds until the process exits.
constexpr long long NOALLOC_MAX_PARTIAL_ROWS = 1LL << 16;
constexpr long long NOALLOC_MAX_NODES = NOALLOC_MAX_PARTIAL_ROWS * UPD_THREADS;  // 16,777,216
static __device__ __align__(256) double g_update_scratch[NOALLOC_MAX_PARTIAL_ROWS * 5];
static __device__ __align__(256) int g_update_fold_ops[5] = {1, 1, 1, 2, 1};

// Device addresses of the two arrays, looked up once per device with that device current and
// kept with the CUDA context they belong to. In host code the arrays' names stand for
// host-side shadows, never for device memory. A context that is torn down and recreated
// (cudaDeviceReset, or a host program that destroys the primary context) reloads the module
// at new addresses, so a cached entry is used only while the device's current context is the
// one it was looked up in; otherwise the addresses are looked up again.
struct NoallocScratch {
    double *partial = nullptr;
    int *ops = nullptr;
    void *context = nullptr;
};

// The calling thread's current driver context (null before the runtime has made one), through
// the runtime's driver entry point so that the library needs no link to the driver library.
int current_context(void **ctx) {
    using CtxGetCurrent = int (*)(void **);
    static CtxGetCurrent get = nullptr;
    static std::once_flag once;
    static cudaError_t found = cudaSuccess;
    std::call_once(once, [] {
        void *fn = nullptr;
        cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
        found = cudaGetDriverEntryPoint("cuCtxGetCurrent", &fn, cudaEnableDefault, &q);
        if (found == cudaSuccess && q == cudaDriverEntryPointSuccess) get = (CtxGetCurrent)fn;
    });
    if (!get) {
        set_error("update_noalloc: the driver entry point cuCtxGetCurrent is unavailable (%s)",
                  cudaGetErrorString(found));
        return CUDA_FAILURE;
    }
    *ctx = nullptr;
    if (get(ctx) != 0) {
        set_error("update_noalloc: cuCtxGetCurrent failed");
        return CUDA_FAILURE;
    }
    return OK;
}

int noalloc_scratch(NoallocScratch *out) {
    constexpr int MAX_DEVICES = 64;
    static std::mutex lock;
    static NoallocScratch table[MAX_DEVICES];
    int dev = 0;
    if (int rc = cuda_status(cudaGetDevice(&dev), "update_noalloc: cudaGetDevice")) return rc;
    if (dev < 0 || dev >= MAX_DEVICES) {
        set_error("update_noalloc: device %d beyond the %d devices it keeps addresses for", dev,
                  MAX_DEVICES);
        return BAD_ARGUMENT;
    }
    void *ctx = nullptr;
    if (int rc = current_context(&ctx)) return rc;
    std::lock_guard<std::mutex> guard(lock);
    NoallocScratch &e = table[dev];
    if (!e.partial || !ctx || ctx != e.context) {
        void *partial = nullptr, *ops = nullptr;
        if (int rc = cuda_status(cudaGetSymbolAddress(&partial, g_update_scratch),
                                 "update_noalloc: cudaGetSymbolAddress(scratch)"))
            return rc;
        if (int rc = cuda_status(cudaGetSymbolAddress(&ops, g_update_fold_ops),
                                 "update_noalloc: cudaGetSymbolAddress(fold ops)"))
            return rc;
        // the lookup made the runtime's context current if there was none yet
        if (int rc = current_context(&ctx)) return rc;
        e.ops = static_cast<int *>(ops);
        e.partial = static_cast<double *>(partial);
        e.context = ctx;
    }
    *out = e;
    return OK;
}

}  // namespace
}  // namespace zvfv

using namespace zvfv;

extern "C" {

int zvfv_gradient(int64_t n, int nc, int nvec, const int64_t *indptr, const int32_t *indices,
                  const double *gop, const double *phi, const uint8_t *sym, double *out,
                  void *stream) {
    if (nc < 1 || nc > 4 || nvec < 0 || nvec > nc) {
        set_error("gradient: nc %d, nvec %d", nc, nvec);
        return BAD_ARGUMENT;
    }
    if (n <= 0) return OK;
    k_gradient<<<grid_for(n * LANES, 256), 256, 0, as_stream(stream)>>>(
        n, nc, nvec, (const long long *)indptr, indices, gop, phi, sym, out); count_launch();
    return launch_status("gradient");
}

int zvfv_minmax(int64_t n, const int64_t *indptr, const int32_t *indices, const double *U,
                double *lo, double *hi, void *stream) {
    if (n <= 0) return OK;
    k_minmax<<<grid_for(n * LANES, 256), 256, 0, as_stream(stream)>>>(
        n, (const long long *)indptr, indices, U, lo, hi); count_launch();
    return launch_status("minmax");
}

int64_t zvfv_finalise_partials(int64_t n) { return (int64_t)grid_for(n * 4, FIN_THREADS); }

int zvfv_finalise(int64_t n, const int64_t *indptr, const int32_t *indices, const int64_t *dpos,
                  double *data, double *b, int has_time, const double *tdiag, const double *trhs,
                  const double *fV, const double *force, const double *inflow, const double *mb,
                  const double *wcons, const double *wonly, const double *wstab, int stokes,
                  const double *snl, const uint8_t *fixed, const uint8_t *known,
                  const double *vel, const double *pval, int eliminate, const int64_t *rawoff,
                  double *rawdata, double *rawb, const double *x, const double *aP,
                  const double *V, double rho, const double *scal, const double *lscale,
                  double *rs_out, double *partial, void *stream) {
    if (n <= 0) return OK;
    FinaliseArgs g{n, (const long long *)indptr, indices, (const long long *)dpos, data, b,
                   has_time, tdiag, trhs, fV, force, inflow, mb, wcons, wonly, wstab, stokes, snl,
                   fixed, known, vel, pval, eliminate, (const long long *)rawoff, rawdata, rawb, x,
                   aP, V, rho, scal, lscale, rs_out, partial};
    k_finalise<<<grid_for(n * 4, FIN_THREADS), FIN_THREADS, 0, as_stream(stream)>>>(g); count_launch();
    return launch_status("finalise");
}

int64_t zvfv_update_partials(int64_t n) { return (int64_t)grid_for(n, UPD_THREADS); }

int zvfv_update(int64_t n, const double *x, double *U, double *P, double *partial, void *stream) {
    if (n <= 0) return OK;
    k_update<<<grid_for(n, UPD_THREADS), UPD_THREADS, 0, as_stream(stream)>>>(n, x, U, P, partial); count_launch();
    return launch_status("update");
}

int zvfv_fold(int64_t nrows, int width, const double *partial, const int32_t *ops, double *out,
              void *stream) {
    if (width <= 0) return OK;
    k_fold<<<1, 256, 0, as_stream(stream)>>>(nrows, width, partial, ops, out); count_launch();
    return launch_status("fold");
}

// The state update and its folded change statistics without any allocation, for callers
// that cannot allocate device memory: a host program that runs under a fixed device-memory
// budget handed out by another component, or a driver whose outer loop must not call
// cudaMalloc/cudaFree between steps. It launches the same two kernels as zvfv_update followed
// by zvfv_fold with ops {1, 1, 1, 2, 1}, with the partial rows in the file-scope array
// g_update_scratch instead of a caller buffer, so its results are those of that pair bit for
// bit. Every row the fold reads is written by k_update first: nothing has to start at zero.
int zvfv_update_noalloc(int64_t n, const double *x, double *U, double *P, double *stats,
                        void *stream) {
    if (n <= 0 || n > NOALLOC_MAX_NODES) {
        set_error("update_noalloc: %lld nodes; the static scratch holds partials for 1 to %lld "
                  "nodes (use zvfv_update with a caller buffer beyond that limit)",
                  (long long)n, (long long)NOALLOC_MAX_NODES);
        return BAD_ARGUMENT;
    }
    NoallocScratch scratch;
    if (int rc = noalloc_scratch(&scratch)) return rc;
    const unsigned rows = grid_for(n, UPD_THREADS);
    k_update<<<rows, UPD_THREADS, 0, as_stream(stream)>>>(n, x, U, P, scratch.partial);
    count_launch();
    if (int rc = launch_status("update_noalloc: update")) return rc;
    k_fold<<<1, 256, 0, as_stream(stream)>>>(rows, 5, scratch.partial, scratch.ops, stats);
    count_launch();
    return launch_status("update_noalloc: fold");
}

}  // extern "C"
