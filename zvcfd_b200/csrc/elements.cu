// Element kernels of the coupled 4x4 (u, v, w, p) finite-volume system, one template per
// element type: block positions, geometry records, statics (node volumes, the Newtonian
// viscous diagonal, the nodal-gradient operator), the momentum diagonal, the assembly of the
// lagged Rhie-Chow blocks and right-hand side, the Rhie-Chow mass flows and the
// Barth-Jespersen limiter. The discrete equations are the reference's
// (docs/spec/fv_numerics.md:95-116; zvcfd/fv/reference.py:654-806, :922-948).
//
// Layout (one warp-team per element, no block-wide barriers):
//
//  * A team of 16 lanes (tetrahedra: two elements per warp) or 32 lanes (the other types)
//    owns one element at a time and walks its colour's slots with a grid-stride loop; a CTA
//    of four warps loads the type's tables into shared memory once and keeps them for all
//    of its elements.
//  * Node lanes (lane < n) gather the element's node values into the team's own staging
//    area; at the same time every lane issues an L2 bulk prefetch of the element's 4x4 blocks
//    so that their read-modify-write later finds them on chip.
//  * Flux lanes (lane < n_ip, 12-24 flux points) each build one flux point: the corners of
//    its dual triangle as node means, the area vector and centroid, the inverse Jacobian of
//    the element map there, the viscosity, the mass flow and its right-hand-side terms. The
//    results form a per-flux-point record (structure of arrays) in shared memory.
//  * Pair lanes (one (row node a, column node c) pair each, two rounds for n^2 > 32) sum the
//    block's distinct coefficients over the flux points of node a: the momentum diagonal,
//    the pressure column N_c A, the continuity diagonal d G_c.A and the transpose terms.
//  * Store lanes: eight lanes per block, each one 16-byte pair of entries, so that a warp
//    reads and writes four whole 128-byte blocks per instruction.
//
// Only __syncwarp orders the phases. Elements of one colour share no node (slot order,
// zvcfd/fv/fast.py:199-207), so every read-modify-write of a block or a node value in one
// launch is done by one lane and the result is deterministic without atomics.
#include <mutex>
#include <utility>
#include <vector>

#include "fvmath.cuh"

namespace zvfv {
namespace {

constexpr int CTA_WARPS = 4;
constexpr int CTA_THREADS = CTA_WARPS * 32;
// Resident CTAs per SM the per-iteration kernels are compiled for: a register cap of 128. The
// kernels are latency-bound; uncapped (160-200 registers) only two or three CTAs fit on an SM,
// and four measured fastest (assembly on the 400k-node tube 6.6 ms uncapped, 4.7 ms at four).
#ifndef ZV_ELEMENT_MIN_CTAS
#define ZV_ELEMENT_MIN_CTAS 4
#endif

template <int K>
struct Team {
    using T = Topo<K>;
    static constexpr int N = T::N, NIP = T::NIP, NN = N * N;
    static constexpr int LANES = (NN <= 16 && NIP <= 16) ? 16 : 32;
    static constexpr int PER_WARP = 32 / LANES;
    static constexpr int PER_CTA = CTA_WARPS * PER_WARP;
    static constexpr int PAIR_ROUNDS = (NN + LANES - 1) / LANES;
    static constexpr int STORE_BLOCKS = LANES / 8;          // blocks per store instruction
    static_assert(NIP <= LANES && 4 * N <= LANES, "one flux point / rhs entry per lane");
};

// The type's tables in shared memory (per CTA). Lanes index the per-flux-point tables by
// their own flux point (fastest index), so a warp reads consecutive words.
template <int K>
struct Tab {
    using T = Topo<K>;
    static constexpr int N = T::N, NIP = T::NIP;
    double dnt[N * 3][NIP];
    double nt[N][NIP];
    double cw[NIP][3];                 // 1 / (nodes in each triangle corner)
    int ia[NIP], ib[NIP];
    int mask[NIP][3];
    int ips[N][MAXI], sgn[N][MAXI];

    __device__ void load() {
        for (int i = threadIdx.x; i < N * 3 * NIP; i += blockDim.x) (&dnt[0][0])[i] = (&T::dnt()[0][0])[i];
        for (int i = threadIdx.x; i < N * NIP; i += blockDim.x) (&nt[0][0])[i] = (&T::nt()[0][0])[i];
        for (int i = threadIdx.x; i < NIP * 3; i += blockDim.x) {
            const int m = (&T::mask()[0][0])[i];
            (&mask[0][0])[i] = m;
            (&cw[0][0])[i] = 1.0 / (double)__popc(m);
        }
        for (int i = threadIdx.x; i < NIP; i += blockDim.x) {
            ia[i] = T::edge()[i][0];
            ib[i] = T::edge()[i][1];
        }
        for (int i = threadIdx.x; i < N * MAXI; i += blockDim.x) {
            (&ips[0][0])[i] = (&T::ips()[0][0])[i];
            (&sgn[0][0])[i] = (&T::sgn()[0][0])[i];
        }
        __syncthreads();
    }
};

// Stored geometry record of one element (doubles): areas A[NIP][3], centroids X[NIP][3],
// inverse Jacobians Ji[NG][9] (row-major, d xi_d / d x_k), sub-control volumes S[N].
template <int K>
struct Record {
    using T = Topo<K>;
    static constexpr int A = 0, X = 3 * T::NIP, J = 6 * T::NIP, S = 6 * T::NIP + 9 * T::NG;
    static_assert(S + T::N == T::REC, "record size");
    __device__ static int jac(int s) { return J + (T::CONSTG ? 0 : s) * 9; }
};

// Corner c of flux point s's dual triangle: the mean of the nodes in its mask.
template <int K>
__device__ inline void corner(const Tab<K> &tb, const double (*X)[3], int s, int c, double p[3]) {
    const int m = tb.mask[s][c];
    double acc[3] = {0.0, 0.0, 0.0};
#pragma unroll
    for (int q = 0; q < Topo<K>::N; ++q) {
        const double on = (m >> q) & 1 ? 1.0 : 0.0;
#pragma unroll
        for (int k = 0; k < 3; ++k) acc[k] += on * X[q][k];
    }
#pragma unroll
    for (int k = 0; k < 3; ++k) p[k] = acc[k] * tb.cw[s][c];
}

// Area vector (edge node a -> b) and centroid of flux point s from node coordinates X.
template <int K>
__device__ inline void flux_area(const Tab<K> &tb, const double (*X)[3], int s, double A[3],
                                 double xs[3]) {
    double p0[3], p1[3], p2[3];
    corner<K>(tb, X, s, 0, p0);
    corner<K>(tb, X, s, 1, p1);
    corner<K>(tb, X, s, 2, p2);
    const double e1[3] = {p1[0] - p0[0], p1[1] - p0[1], p1[2] - p0[2]};
    const double e2[3] = {p2[0] - p0[0], p2[1] - p0[1], p2[2] - p0[2]};
    A[0] = 0.5 * (e1[1] * e2[2] - e1[2] * e2[1]);
    A[1] = 0.5 * (e1[2] * e2[0] - e1[0] * e2[2]);
    A[2] = 0.5 * (e1[0] * e2[1] - e1[1] * e2[0]);
#pragma unroll
    for (int k = 0; k < 3; ++k) xs[k] = (p0[k] + p1[k] + p2[k]) * (1.0 / 3.0);
}

// Inverse Jacobian Ji[d*3+k] = d xi_d / d x_k of the element map at flux point s.
template <int K>
__device__ inline void flux_jacobian(const Tab<K> &tb, const double (*X)[3], int s, double Ji[9]) {
    double J[9];
#pragma unroll
    for (int k = 0; k < 3; ++k)
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            double acc = 0.0;
#pragma unroll
            for (int q = 0; q < Topo<K>::N; ++q) acc += X[q][k] * tb.dnt[q * 3 + d][s];
            J[k * 3 + d] = acc;
        }
    invert3(J, Ji);
}

// Gradient of shape function c at flux point s: G[k] = sum_d dN_c/dxi_d Ji[d][k].
template <int K>
__device__ inline void shape_gradient(const Tab<K> &tb, int c, int s, const double Ji[9],
                                      double G[3]) {
    const double d0 = tb.dnt[c * 3][s], d1 = tb.dnt[c * 3 + 1][s], d2 = tb.dnt[c * 3 + 2][s];
#pragma unroll
    for (int k = 0; k < 3; ++k) G[k] = d0 * Ji[k] + d1 * Ji[3 + k] + d2 * Ji[6 + k];
}

// Gradient at flux point s of a nodal vector field F (N x 3): L[j*3+k] = d F_j / d x_k,
// formed along the parametric axes first (N*9 products) and mapped by Ji once.
template <int K>
__device__ inline void field_gradient(const Tab<K> &tb, const double (*F)[3], int s,
                                      const double Ji[9], double L[9]) {
    double H[9];
#pragma unroll
    for (int i = 0; i < 9; ++i) H[i] = 0.0;
#pragma unroll
    for (int q = 0; q < Topo<K>::N; ++q) {
        const double d0 = tb.dnt[q * 3][s], d1 = tb.dnt[q * 3 + 1][s], d2 = tb.dnt[q * 3 + 2][s];
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            H[j * 3] += F[q][j] * d0;
            H[j * 3 + 1] += F[q][j] * d1;
            H[j * 3 + 2] += F[q][j] * d2;
        }
    }
#pragma unroll
    for (int j = 0; j < 3; ++j)
#pragma unroll
        for (int k = 0; k < 3; ++k)
            L[j * 3 + k] = H[j * 3] * Ji[k] + H[j * 3 + 1] * Ji[3 + k] + H[j * 3 + 2] * Ji[6 + k];
}

// Flux-point geometry from the record or rebuilt from the staged coordinates.
template <int K, bool STORED>
__device__ inline void flux_geometry(const Tab<K> &tb, const double (*X)[3], const double *rec,
                                     int s, double A[3], double xs[3], double Ji[9]) {
    using R = Record<K>;
    if (STORED) {
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            A[k] = __ldg(rec + R::A + s * 3 + k);
            xs[k] = __ldg(rec + R::X + s * 3 + k);
        }
#pragma unroll
        for (int i = 0; i < 9; ++i) Ji[i] = __ldg(rec + R::jac(s) + i);
    } else {
        flux_area<K>(tb, X, s, A, xs);
        flux_jacobian<K>(tb, X, s, Ji);
    }
}

// Viscous coefficient of flux point s on the row of its node c, -mu (G_c . A) (plus
// -mu G_c,x A_x with the transpose term), as the momentum diagonal takes it.
template <int K>
__device__ inline double viscous_coefficient(const Tab<K> &tb, int c, int s, const double Ji[9],
                                             const double A[3], double mu, int transpose) {
    double G[3];
    shape_gradient<K>(tb, c, s, Ji, G);
    double r = G[0] * A[0] + G[1] * A[1] + G[2] * A[2];
    if (transpose) r += G[0] * A[0];
    return -mu * r;
}

// Send the element's 128-byte blocks towards L2 ahead of their read-modify-write.
__device__ inline void prefetch_block(const double *p) {
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], 128;" ::"l"(p) : "memory");
}

// One 128-byte line of node data towards L2 (the next element's gathers).
__device__ inline void prefetch_line(const void *p) {
    asm volatile("prefetch.global.L2 [%0];" ::"l"(p) : "memory");
}

// Team coordinates of this thread inside the grid-stride walk.
template <int K>
struct Walk {
    int team, lane, warp_in_cta;
    long long first, stride;
    __device__ Walk() {
        constexpr int L = Team<K>::LANES;
        const int w = threadIdx.x >> 5;
        warp_in_cta = w;
        team = (threadIdx.x & 31) / L;
        lane = threadIdx.x & (L - 1);
        const long long gw = (long long)blockIdx.x * CTA_WARPS + w;
        first = gw * Team<K>::PER_WARP;
        stride = (long long)gridDim.x * CTA_WARPS * Team<K>::PER_WARP;
    }
    __device__ int slot_in_cta() const { return warp_in_cta * Team<K>::PER_WARP + team; }
};

// --------------------------------------------------------------------------- blockpos

// Pattern position of every (row node, column node) pair of every slot; -1 if missing.
// One warp per (slot, row): the warp reads the row's sorted columns 32 at a time and finds
// each of the element's columns with a ballot.
template <int K>
__global__ void k_blockpos(const int *__restrict__ conn, long long nslots,
                           const long long *__restrict__ indptr, const int *__restrict__ indices,
                           int *__restrict__ pos) {
    constexpr int N = Topo<K>::N;
    const long long w = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (w >= nslots * N) return;
    const long long slot = w / N;
    const int a = (int)(w % N);
    const long long row = conn[slot * N + a];
    const int mycol = lane < N ? conn[slot * N + lane] : -1;
    int found = -1;
    const long long lo = indptr[row], hi = indptr[row + 1];
    for (long long p0 = lo; p0 < hi; p0 += 32) {
        const int v = p0 + lane < hi ? indices[p0 + lane] : -2;
#pragma unroll
        for (int c = 0; c < N; ++c) {
            const int col = __shfl_sync(0xffffffffu, mycol, c);
            const unsigned hit = __ballot_sync(0xffffffffu, v == col);
            if (lane == c && hit) found = (int)(p0 + __ffs(hit) - 1);
        }
    }
    if (lane < N) pos[slot * N * N + a * N + lane] = found;
}

// --------------------------------------------------------------------------- geometry

template <int K>
struct GeoStage {
    using T = Topo<K>;
    double X[T::N][3];
    double A[3][T::NIP], xs[3][T::NIP], Ji[9][T::NIP];
    int node[T::N];
};

// Geometry records of every slot (for store_geometry): flux lanes write areas, centroids and
// inverse Jacobians, node lanes the sub-control volumes.
template <int K>
__global__ void __launch_bounds__(CTA_THREADS)
k_geobuild(const int *__restrict__ conn, const double *__restrict__ Xn, long long nslots,
           double *__restrict__ georec) {
    using T = Topo<K>;
    using R = Record<K>;
    __shared__ Tab<K> tb;
    __shared__ GeoStage<K> st_all[Team<K>::PER_CTA];
    tb.load();
    Walk<K> wk;
    GeoStage<K> &st = st_all[wk.slot_in_cta()];
    for (long long e0 = wk.first; e0 < nslots; e0 += wk.stride) {
        const long long slot = e0 + wk.team;
        const bool on = slot < nslots;
        if (on && wk.lane < T::N) {
            const long long n = conn[slot * T::N + wk.lane];
#pragma unroll
            for (int k = 0; k < 3; ++k) st.X[wk.lane][k] = __ldg(Xn + n * 3 + k);
        }
        __syncwarp();
        double *rec = georec + slot * T::REC;
        if (on && wk.lane < T::NIP) {
            const int s = wk.lane;
            double A[3], xs[3], Ji[9];
            flux_area<K>(tb, st.X, s, A, xs);
            flux_jacobian<K>(tb, st.X, s, Ji);
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                rec[R::A + s * 3 + k] = A[k];
                rec[R::X + s * 3 + k] = xs[k];
                st.A[k][s] = A[k];
                st.xs[k][s] = xs[k];
            }
            if (!T::CONSTG || s == 0)
#pragma unroll
                for (int i = 0; i < 9; ++i) rec[R::jac(s) + i] = Ji[i];
        }
        __syncwarp();
        if (on && wk.lane < T::N) {
            const int a = wk.lane;
            double v = 0.0;
#pragma unroll
            for (int i = 0; i < T::MAXF; ++i) {
                const int s = tb.ips[a][i];
                if (s < 0) continue;
                double f = 0.0;
#pragma unroll
                for (int k = 0; k < 3; ++k) f += (st.xs[k][s] - st.X[a][k]) * st.A[k][s];
                v += tb.sgn[a][i] * f;
            }
            rec[R::S + a] = v * (1.0 / 3.0);
        }
        __syncwarp();
    }
}

// --------------------------------------------------------------------------- statics

template <int K>
struct StaticStage {
    using T = Topo<K>;
    double X[T::N][3];
    double A[3][T::NIP], xs[3][T::NIP], Ji[9][T::NIP];
    double S[T::N], gbar[T::N][3];
    int node[T::N];
};

// Node volumes, the Newtonian viscous diagonal and the nodal-gradient operator: pattern
// block (a, c) gets S_a times the element's mean gradient of N_c (over its flux points).
template <int K, bool STORED>
__global__ void __launch_bounds__(CTA_THREADS)
k_statics(const int *__restrict__ conn, long long base, long long count,
          const double *__restrict__ Xn, const double *__restrict__ georec,
          const int *__restrict__ pos, double mu, int transpose, double *__restrict__ vol,
          double *__restrict__ dvisc, double *__restrict__ gop) {
    using T = Topo<K>;
    using R = Record<K>;
    constexpr int N = T::N, L = Team<K>::LANES;
    __shared__ Tab<K> tb;
    __shared__ StaticStage<K> st_all[Team<K>::PER_CTA];
    tb.load();
    Walk<K> wk;
    StaticStage<K> &st = st_all[wk.slot_in_cta()];
    for (long long e0 = wk.first; e0 < count; e0 += wk.stride) {
        const long long le = e0 + wk.team;
        const bool on = le < count;
        const long long slot = base + le;
        const double *rec = georec + (STORED ? slot * T::REC : 0);
        if (on && wk.lane < N) {
            const int n = conn[slot * N + wk.lane];
            st.node[wk.lane] = n;
#pragma unroll
            for (int k = 0; k < 3; ++k) st.X[wk.lane][k] = __ldg(Xn + (long long)n * 3 + k);
        }
        __syncwarp();
        if (on && wk.lane < T::NIP) {
            const int s = wk.lane;
            double A[3], xs[3], Ji[9];
            flux_geometry<K, STORED>(tb, st.X, rec, s, A, xs, Ji);
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                st.A[k][s] = A[k];
                st.xs[k][s] = xs[k];
            }
#pragma unroll
            for (int i = 0; i < 9; ++i) st.Ji[i][s] = Ji[i];
        }
        __syncwarp();
        if (on && wk.lane < N) {
            const int a = wk.lane;
            double v = 0.0, dv = 0.0;
#pragma unroll
            for (int i = 0; i < T::MAXF; ++i) {
                const int s = tb.ips[a][i];
                if (s < 0) continue;
                const double A[3] = {st.A[0][s], st.A[1][s], st.A[2][s]};
                double Ji[9];
#pragma unroll
                for (int q = 0; q < 9; ++q) Ji[q] = st.Ji[q][s];
                double f = 0.0;
#pragma unroll
                for (int k = 0; k < 3; ++k) f += (st.xs[k][s] - st.X[a][k]) * A[k];
                v += tb.sgn[a][i] * f;
                dv += tb.sgn[a][i] * viscous_coefficient<K>(tb, a, s, Ji, A, mu, transpose);
            }
            const double S = STORED ? __ldg(rec + R::S + a) : v * (1.0 / 3.0);
            st.S[a] = S;
            double g[3] = {0.0, 0.0, 0.0};
            for (int s = 0; s < T::NG; ++s) {
                double Ji[9], G[3];
#pragma unroll
                for (int q = 0; q < 9; ++q) Ji[q] = st.Ji[q][s];
                shape_gradient<K>(tb, a, s, Ji, G);
#pragma unroll
                for (int k = 0; k < 3; ++k) g[k] += G[k];
            }
#pragma unroll
            for (int k = 0; k < 3; ++k) st.gbar[a][k] = g[k] * (1.0 / T::NG);
            vol[st.node[a]] += S;
            dvisc[st.node[a]] += dv;
        }
        __syncwarp();
        if (on) {
            for (int p = wk.lane; p < N * N; p += L) {
                const int a = p / N, c = p % N;
                const long long q = pos[slot * N * N + p];
                if (q < 0) continue;
#pragma unroll
                for (int k = 0; k < 3; ++k) gop[q * 3 + k] += st.S[a] * st.gbar[c][k];
            }
        }
        __syncwarp();
    }
}

// --------------------------------------------------------------------------- diag

struct DiagArgs {
    const int *conn;
    const double *X, *geo, *mdot, *U;
    Rheology rh;
    int transpose, stokes, has_mut;
    const double *mut;
    double *out;
};

template <int K>
struct DiagStage {
    using T = Topo<K>;
    double X[T::N][3], U[T::N][3], mut[T::N];
    double ca[T::NIP], cb[T::NIP];          // the flux point's terms on its two nodes' rows
    int node[T::N];
};

// The momentum diagonal a_P: per flux point the viscous coefficient of each edge node on its
// own row and the upwind part of the mass flow (zvcfd/fv/reference.py:694-724).
template <int K, bool STORED>
__global__ void __launch_bounds__(CTA_THREADS, ZV_ELEMENT_MIN_CTAS)
k_diag(const DiagArgs g, long long base, long long count) {
    using T = Topo<K>;
    constexpr int N = T::N;
    __shared__ Tab<K> tb;
    __shared__ DiagStage<K> st_all[Team<K>::PER_CTA];
    tb.load();
    Walk<K> wk;
    DiagStage<K> &st = st_all[wk.slot_in_cta()];
    for (long long e0 = wk.first; e0 < count; e0 += wk.stride) {
        const long long le = e0 + wk.team;
        const bool on = le < count;
        const long long slot = base + le;
        const double *rec = g.geo + (STORED ? slot * T::REC : 0);
        if (on && wk.lane < N) {
            const int a = wk.lane;
            const long long n = g.conn[slot * N + a];
            st.node[a] = (int)n;
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                st.X[a][k] = __ldg(g.X + n * 3 + k);
                st.U[a][k] = __ldg(g.U + n * 3 + k);
            }
            st.mut[a] = g.has_mut ? __ldg(g.mut + n) : 0.0;
        }
        __syncwarp();
        if (on && wk.lane < T::NIP) {
            const int s = wk.lane;
            double A[3], xs[3], Ji[9];
            flux_geometry<K, STORED>(tb, st.X, rec, s, A, xs, Ji);
            double mu = g.rh.mu0;
            if (g.rh.model) {
                double Lg[9];
                field_gradient<K>(tb, st.U, s, Ji, Lg);
                mu = viscosity_of_gradient(Lg, g.rh);
            }
            if (g.has_mut)
#pragma unroll
                for (int q = 0; q < N; ++q) mu += tb.nt[q][s] * st.mut[q];
            double ra = viscous_coefficient<K>(tb, tb.ia[s], s, Ji, A, mu, g.transpose);
            double rb = -viscous_coefficient<K>(tb, tb.ib[s], s, Ji, A, mu, g.transpose);
            if (!g.stokes) {
                const double m = g.mdot[slot * T::NIP + s];
                ra += fmax(m, 0.0);
                rb += fmax(-m, 0.0);
            }
            st.ca[s] = ra;
            st.cb[s] = rb;
        }
        __syncwarp();
        if (on && wk.lane < N) {
            const int a = wk.lane;
            double d = 0.0;
#pragma unroll
            for (int i = 0; i < T::MAXF; ++i) {
                const int s = tb.ips[a][i];
                if (s < 0) continue;
                d += tb.sgn[a][i] > 0 ? st.ca[s] : st.cb[s];
            }
            g.out[st.node[a]] += d;
        }
        __syncwarp();
    }
}

// --------------------------------------------------------------------------- assemble

struct AsmArgs {
    const int *conn;
    const double *X, *geo, *U, *mdot, *gradU, *beta, *gradP, *dnode, *snode;
    int nlev;
    double c1;
    const double *Uo1, *mo1;
    double c2;
    const double *Uo2, *mo2;
    double rho;
    Rheology rh;
    int transpose, stokes, has_mut;
    const double *mut;
    const int *own, *pos;
    double *data, *b;
};

// Distinct coefficients of one pair's block: the momentum diagonal, the pressure column
// N_c A (3), the continuity diagonal -d G_c.A, and the transpose terms -mu G_c,k A_j (9).
constexpr int PAIR_DIAG = 0, PAIR_PV = 1, PAIR_RCD = 4, PAIR_TR = 5, PAIR_VALUES = 14;

template <int K>
struct AsmStage {
    using T = Topo<K>;
    static constexpr int N = T::N, NIP = T::NIP, L = Team<K>::LANES;
    struct Nodes {
        double X[N][3], U[N][3], gP[N][3], gU[N][9], be[N][3], u1[N][3], u2[N][3];
        double dn[N], sn[N], mut[N];
    };
    union {
        Nodes nd;                           // read by the flux lanes
        double pair[PAIR_VALUES][L];        // one round of pair coefficients, read by stores
    };
    double A[3][NIP], Ji[9][NIP], mu[NIP], m[NIP], d[NIP], R[4][NIP];
    int node[N], own[N];
    int pos[N * N];
};

// Entries 2q and 2q+1 of a block (row-major 4x4) from its pair coefficients P (stride L).
template <int L>
__device__ inline double2 block_entries(const double (*P)[L], int j, int q, double rho,
                                        int transpose) {
    const int r = q >> 1, c0 = (q & 1) * 2;
    const double dg = P[PAIR_DIAG][j];
    double e[2];
#pragma unroll
    for (int h = 0; h < 2; ++h) {
        const int c = c0 + h;
        double v;
        if (r < 3 && c < 3) {
            v = (r == c ? dg : 0.0) + (transpose ? P[PAIR_TR + r * 3 + c][j] : 0.0);
        } else if (r < 3) {
            v = P[PAIR_PV + r][j];                          // pressure column
        } else if (c < 3) {
            v = rho * P[PAIR_PV + c][j];                    // continuity on the velocity
        } else {
            v = rho * P[PAIR_RCD][j];                       // continuity on the pressure
        }
        e[h] = v;
    }
    return make_double2(e[0], e[1]);
}

// Blocks and right-hand side of the flux points of one colour (see the file comment for the
// lane phases). Pair (a, c) sums over the flux points s at node a, sg = +1 on the edge's
// first node and -1 on its second: momentum diagonal -sg mu G_c.A (+ sg m on the upwind node
// c of s), transpose -sg mu G_c,k A_j, pressure sg N_c(s) A_k, continuity rho sg N_c(s) A_j and
// -rho sg d G_c.A. The right-hand side: momentum -sg m beta_up (grad u_up . (x_s - x_up)),
// except on an own inflow node's row for the faces it is upwind of; continuity -sg (rho d
// (N(s) grad p) . A + the transient Rhie-Chow part).
template <int K, bool STORED>
__global__ void __launch_bounds__(CTA_THREADS, ZV_ELEMENT_MIN_CTAS)
k_assemble(const AsmArgs g, long long base, long long count) {
    using T = Topo<K>;
    using TM = Team<K>;
    constexpr int N = T::N, NIP = T::NIP, NN = TM::NN, L = TM::LANES;
    __shared__ Tab<K> tb;
    __shared__ AsmStage<K> st_all[TM::PER_CTA];
    tb.load();
    Walk<K> wk;
    AsmStage<K> &st = st_all[wk.slot_in_cta()];
    const int lane = wk.lane;
    constexpr int PPL = (NN + L - 1) / L;                  // block positions per lane
    for (long long e0 = wk.first; e0 < count; e0 += wk.stride) {
        const long long le = e0 + wk.team;
        const bool on = le < count;
        const long long slot = base + le;
        const double *rec = g.geo + (STORED ? slot * T::REC : 0);
        // the next element of this team: its nodes and block positions, read now so that its
        // node data and blocks can be sent towards L2 while this element is worked on
        const long long nle = le + wk.stride;
        const bool next_on = nle < count;
        const long long nslot = base + nle;
        int next_node = -1, next_pos[PPL];
        if (next_on && lane < N) next_node = __ldg(g.conn + nslot * N + lane);
#pragma unroll
        for (int j = 0; j < PPL; ++j) {
            const int p = j * L + lane;
            next_pos[j] = next_on && p < NN ? __ldg(g.pos + nslot * NN + p) : -1;
        }
        // ---- node lanes: stage the element's node values; every lane: block positions
        if (on) {
            for (int p = lane; p < NN; p += L) {
                const int q = __ldg(g.pos + slot * NN + p);
                st.pos[p] = q;
                if (q >= 0 && e0 == wk.first) prefetch_block(g.data + (long long)q * 16);
            }
        }
        if (on && lane < N) {
            const int a = lane;
            const long long n = __ldg(g.conn + slot * N + a);
            st.node[a] = (int)n;
            st.own[a] = __ldg(g.own + n);
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                st.nd.X[a][k] = __ldg(g.X + n * 3 + k);
                st.nd.U[a][k] = __ldg(g.U + n * 3 + k);
                st.nd.gP[a][k] = __ldg(g.gradP + n * 3 + k);
            }
            st.nd.dn[a] = __ldg(g.dnode + n);
            st.nd.sn[a] = __ldg(g.snode + n);
            st.nd.mut[a] = g.has_mut ? __ldg(g.mut + n) : 0.0;
            if (!g.stokes) {
#pragma unroll
                for (int q = 0; q < 9; ++q) st.nd.gU[a][q] = __ldg(g.gradU + n * 9 + q);
#pragma unroll
                for (int k = 0; k < 3; ++k) st.nd.be[a][k] = __ldg(g.beta + n * 3 + k);
            }
            if (g.nlev > 0)
#pragma unroll
                for (int k = 0; k < 3; ++k) st.nd.u1[a][k] = __ldg(g.Uo1 + n * 3 + k);
            if (g.nlev > 1)
#pragma unroll
                for (int k = 0; k < 3; ++k) st.nd.u2[a][k] = __ldg(g.Uo2 + n * 3 + k);
        }
        __syncwarp();
        // ---- flux lanes: one flux point each
        if (on && lane < NIP) {
            const int s = lane, ia = tb.ia[s], ib = tb.ib[s];
            double A[3], xs[3], Ji[9];
            flux_geometry<K, STORED>(tb, st.nd.X, rec, s, A, xs, Ji);
            double mu = g.rh.mu0;
            if (g.rh.model) {
                double Lg[9];
                field_gradient<K>(tb, st.nd.U, s, Ji, Lg);
                mu = viscosity_of_gradient(Lg, g.rh);
            }
            double gA = 0.0, v1 = 0.0, v2 = 0.0, mt = 0.0;
#pragma unroll
            for (int q = 0; q < N; ++q) {
                const double w = tb.nt[q][s];
                gA += w * (st.nd.gP[q][0] * A[0] + st.nd.gP[q][1] * A[1] + st.nd.gP[q][2] * A[2]);
                if (g.nlev > 0)
                    v1 += w * (st.nd.u1[q][0] * A[0] + st.nd.u1[q][1] * A[1] + st.nd.u1[q][2] * A[2]);
                if (g.nlev > 1)
                    v2 += w * (st.nd.u2[q][0] * A[0] + st.nd.u2[q][1] * A[1] + st.nd.u2[q][2] * A[2]);
                mt += w * st.nd.mut[q];
            }
            if (g.has_mut) mu += mt;
            const double m = __ldg(g.mdot + slot * NIP + s);
            const double d = 0.5 * (st.nd.dn[ia] + st.nd.dn[ib]);
            double past = 0.0;
            if (g.nlev > 0) {
                past = g.c1 * (__ldg(g.mo1 + slot * NIP + s) - g.rho * v1);
                if (g.nlev > 1) past += g.c2 * (__ldg(g.mo2 + slot * NIP + s) - g.rho * v2);
                past *= 1.0 - d / (0.5 * (st.nd.sn[ia] + st.nd.sn[ib]));
            }
            st.R[3][s] = g.rho * d * gA + past;
            const int up = m >= 0 ? ia : ib;
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                double corr = 0.0;
                if (!g.stokes) {
                    double reach = 0.0;
#pragma unroll
                    for (int q = 0; q < 3; ++q)
                        reach += st.nd.gU[up][k * 3 + q] * (xs[q] - st.nd.X[up][q]);
                    corr = m * st.nd.be[up][k] * reach;
                }
                st.R[k][s] = corr;
                st.A[k][s] = A[k];
            }
#pragma unroll
            for (int i = 0; i < 9; ++i) st.Ji[i][s] = Ji[i];
            st.mu[s] = mu;
            st.m[s] = m;
            st.d[s] = d;
        }
        __syncwarp();
        // ---- the next element's node data, mass flows and blocks towards L2
        if (next_node >= 0) {
            const long long n = next_node;
            prefetch_line(g.X + n * 3);
            prefetch_line(g.U + n * 3);
            prefetch_line(g.gradP + n * 3);
            prefetch_line(g.dnode + n);
            prefetch_line(g.snode + n);
            prefetch_line(g.own + n);
            if (!g.stokes) {
                prefetch_line(g.gradU + n * 9);
                prefetch_line(g.gradU + n * 9 + 8);
                prefetch_line(g.beta + n * 3);
            }
            if (g.nlev > 0) prefetch_line(g.Uo1 + n * 3);
            if (g.nlev > 1) prefetch_line(g.Uo2 + n * 3);
        }
        if (next_on && lane < NIP) prefetch_line(g.mdot + nslot * NIP + lane);
#pragma unroll
        for (int j = 0; j < PPL; ++j)
            if (next_pos[j] >= 0) prefetch_block(g.data + (long long)next_pos[j] * 16);
        // ---- pair lanes, then store lanes, one round of L pairs at a time
#pragma unroll 1
        for (int round = 0; round < TM::PAIR_ROUNDS; ++round) {
            const int p = round * L + lane;
            if (on && p < NN) {
                const int a = p / N, c = p % N;
                double dg = 0.0, rcd = 0.0, pv[3] = {0.0, 0.0, 0.0}, tr[9];
#pragma unroll
                for (int i = 0; i < 9; ++i) tr[i] = 0.0;
#pragma unroll
                for (int i = 0; i < T::MAXF; ++i) {
                    const int s = tb.ips[a][i];
                    if (s < 0) continue;
                    const double sg = (double)tb.sgn[a][i];
                    const double A[3] = {st.A[0][s], st.A[1][s], st.A[2][s]};
                    double Ji[9], G[3];
#pragma unroll
                    for (int q = 0; q < 9; ++q) Ji[q] = st.Ji[q][s];
                    shape_gradient<K>(tb, c, s, Ji, G);
                    const double GA = G[0] * A[0] + G[1] * A[1] + G[2] * A[2];
                    const double smu = sg * st.mu[s], sN = sg * tb.nt[c][s];
                    dg -= smu * GA;
                    rcd -= sg * st.d[s] * GA;
#pragma unroll
                    for (int k = 0; k < 3; ++k) pv[k] += sN * A[k];
                    if (g.transpose)
#pragma unroll
                        for (int k = 0; k < 3; ++k)
#pragma unroll
                            for (int j = 0; j < 3; ++j) tr[k * 3 + j] -= smu * G[k] * A[j];
                    if (!g.stokes) {
                        const double m = st.m[s];
                        if ((c == tb.ia[s] && m > 0) || (c == tb.ib[s] && m < 0)) dg += sg * m;
                    }
                }
                st.pair[PAIR_DIAG][lane] = dg;
                st.pair[PAIR_RCD][lane] = rcd;
#pragma unroll
                for (int k = 0; k < 3; ++k) st.pair[PAIR_PV + k][lane] = pv[k];
                if (g.transpose)
#pragma unroll
                    for (int i = 0; i < 9; ++i) st.pair[PAIR_TR + i][lane] = tr[i];
            }
            __syncwarp();
            if (on) {
                // store lanes: lane = 8 * (block in the instruction) + q, entries 2q, 2q+1
                constexpr int SB = TM::STORE_BLOCKS, STEPS = L / SB;
                const int q = lane & 7, sub = lane >> 3;
                double2 v[STEPS];
                double2 *dst[STEPS];
#pragma unroll
                for (int t = 0; t < STEPS; ++t) {
                    const int j = t * SB + sub;                       // pair within the round
                    const int pj = round * L + j;
                    dst[t] = nullptr;
                    if (pj < NN && st.pos[pj] >= 0) {
                        dst[t] = reinterpret_cast<double2 *>(g.data + (long long)st.pos[pj] * 16) + q;
                        v[t] = *dst[t];
                    }
                }
#pragma unroll
                for (int t = 0; t < STEPS; ++t) {
                    if (!dst[t]) continue;
                    const double2 add = block_entries<L>(st.pair, t * SB + sub, q, g.rho, g.transpose);
                    v[t].x += add.x;
                    v[t].y += add.y;
                    *dst[t] = v[t];
                }
            }
            __syncwarp();
        }
        // ---- right-hand side: lane = 4 a + k
        if (on && lane < 4 * N) {
            const int a = lane >> 2, k = lane & 3;
            const bool keep_out = k < 3 && st.own[a];
            double r = 0.0;
#pragma unroll
            for (int i = 0; i < T::MAXF; ++i) {
                const int s = tb.ips[a][i];
                if (s < 0) continue;
                if (keep_out && (st.m[s] >= 0 ? tb.ia[s] : tb.ib[s]) == a) continue;
                r -= tb.sgn[a][i] * st.R[k][s];
            }
            g.b[(long long)st.node[a] * 4 + k] += r;
        }
        __syncwarp();
    }
}

// --------------------------------------------------------------------------- massflow

struct MassArgs {
    const int *conn;
    const double *X, *geo, *U, *P, *gradP, *dnode, *snode;
    int nlev;
    double c1;
    const double *Uo1, *mo1;
    double c2;
    const double *Uo2, *mo2;
    double rho;
    double *mdot, *imbalance, *adv;
    // VDIAG: the viscous part of the next momentum diagonal from the same (new) velocity
    Rheology rh;
    int transpose, has_mut;
    const double *mut;
    double *vdiag;
};

template <int K>
struct MassStage {
    using T = Topo<K>;
    double X[T::N][3], U[T::N][3], gP[T::N][3], u1[T::N][3], u2[T::N][3];
    double P[T::N], dn[T::N], sn[T::N], mut[T::N];
    double m[T::NIP], va[T::NIP], vb[T::NIP];
    int node[T::N];
};

// New Rhie-Chow mass flows rho u(s).A + rho d (N(s) grad p - grad p(s)).A (+ the transient
// part), each node's net outflow and the upwind part of the next momentum diagonal
// (zvcfd/fv/reference.py:922-948). With VDIAG the flux lanes also form the viscous terms of
// the next diagonal from the same velocity, which then needs no element pass of its own.
template <int K, bool STORED, bool VDIAG>
__global__ void __launch_bounds__(CTA_THREADS, ZV_ELEMENT_MIN_CTAS)
k_massflow(const MassArgs g, long long base, long long count) {
    using T = Topo<K>;
    constexpr int N = T::N, NIP = T::NIP;
    __shared__ Tab<K> tb;
    __shared__ MassStage<K> st_all[Team<K>::PER_CTA];
    tb.load();
    Walk<K> wk;
    MassStage<K> &st = st_all[wk.slot_in_cta()];
    const int lane = wk.lane;
    for (long long e0 = wk.first; e0 < count; e0 += wk.stride) {
        const long long le = e0 + wk.team;
        const bool on = le < count;
        const long long slot = base + le;
        const double *rec = g.geo + (STORED ? slot * T::REC : 0);
        const long long nle = le + wk.stride;              // this team's next element
        const int next_node = nle < count && lane < N ? __ldg(g.conn + (base + nle) * N + lane) : -1;
        if (on && lane < N) {
            const int a = lane;
            const long long n = __ldg(g.conn + slot * N + a);
            st.node[a] = (int)n;
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                st.X[a][k] = __ldg(g.X + n * 3 + k);
                st.U[a][k] = __ldg(g.U + n * 3 + k);
                st.gP[a][k] = __ldg(g.gradP + n * 3 + k);
                if (g.nlev > 0) st.u1[a][k] = __ldg(g.Uo1 + n * 3 + k);
                if (g.nlev > 1) st.u2[a][k] = __ldg(g.Uo2 + n * 3 + k);
            }
            st.P[a] = __ldg(g.P + n);
            st.dn[a] = __ldg(g.dnode + n);
            st.sn[a] = __ldg(g.snode + n);
            st.mut[a] = (VDIAG && g.has_mut) ? __ldg(g.mut + n) : 0.0;
        }
        __syncwarp();
        if (on && lane < NIP) {
            const int s = lane, ia = tb.ia[s], ib = tb.ib[s];
            double A[3], xs[3], Ji[9];
            flux_geometry<K, STORED>(tb, st.X, rec, s, A, xs, Ji);
            // carried flow, lagged mean pressure gradient, and the gradient of p at s
            double ua = 0.0, gA = 0.0, v1 = 0.0, v2 = 0.0, h[3] = {0.0, 0.0, 0.0};
#pragma unroll
            for (int q = 0; q < N; ++q) {
                const double w = tb.nt[q][s];
                ua += w * (st.U[q][0] * A[0] + st.U[q][1] * A[1] + st.U[q][2] * A[2]);
                gA += w * (st.gP[q][0] * A[0] + st.gP[q][1] * A[1] + st.gP[q][2] * A[2]);
                if (g.nlev > 0)
                    v1 += w * (st.u1[q][0] * A[0] + st.u1[q][1] * A[1] + st.u1[q][2] * A[2]);
                if (g.nlev > 1)
                    v2 += w * (st.u2[q][0] * A[0] + st.u2[q][1] * A[1] + st.u2[q][2] * A[2]);
#pragma unroll
                for (int dd = 0; dd < 3; ++dd) h[dd] += st.P[q] * tb.dnt[q * 3 + dd][s];
            }
            double pA = 0.0;
#pragma unroll
            for (int k = 0; k < 3; ++k) pA += (h[0] * Ji[k] + h[1] * Ji[3 + k] + h[2] * Ji[6 + k]) * A[k];
            const double d = 0.5 * (st.dn[ia] + st.dn[ib]);
            double m = g.rho * ua + g.rho * d * (gA - pA);
            if (g.nlev > 0) {
                double past = g.c1 * (__ldg(g.mo1 + slot * NIP + s) - g.rho * v1);
                if (g.nlev > 1) past += g.c2 * (__ldg(g.mo2 + slot * NIP + s) - g.rho * v2);
                m += (1.0 - d / (0.5 * (st.sn[ia] + st.sn[ib]))) * past;
            }
            g.mdot[slot * NIP + s] = m;
            st.m[s] = m;
            if (VDIAG) {
                double mu = g.rh.mu0;
                if (g.rh.model) {
                    double Lg[9];
                    field_gradient<K>(tb, st.U, s, Ji, Lg);
                    mu = viscosity_of_gradient(Lg, g.rh);
                }
                if (g.has_mut)
#pragma unroll
                    for (int q = 0; q < N; ++q) mu += tb.nt[q][s] * st.mut[q];
                st.va[s] = viscous_coefficient<K>(tb, ia, s, Ji, A, mu, g.transpose);
                st.vb[s] = -viscous_coefficient<K>(tb, ib, s, Ji, A, mu, g.transpose);
            }
        }
        if (next_node >= 0) {
            const long long n = next_node;
            prefetch_line(g.X + n * 3);
            prefetch_line(g.U + n * 3);
            prefetch_line(g.gradP + n * 3);
            prefetch_line(g.P + n);
            prefetch_line(g.dnode + n);
            prefetch_line(g.snode + n);
            if (g.nlev > 0) prefetch_line(g.Uo1 + n * 3);
            if (g.nlev > 1) prefetch_line(g.Uo2 + n * 3);
        }
        __syncwarp();
        if (on && lane < N) {
            const int a = lane;
            double out = 0.0, ad = 0.0, vd = 0.0;
#pragma unroll
            for (int i = 0; i < T::MAXF; ++i) {
                const int s = tb.ips[a][i];
                if (s < 0) continue;
                const double m = st.m[s];
                if (tb.sgn[a][i] > 0) {
                    out += m;
                    ad += fmax(m, 0.0);
                    if (VDIAG) vd += st.va[s];
                } else {
                    out -= m;
                    ad += fmax(-m, 0.0);
                    if (VDIAG) vd += st.vb[s];
                }
            }
            const long long n = st.node[a];
            g.imbalance[n] += out;
            g.adv[n] += ad;
            if (VDIAG) g.vdiag[n] += vd;
        }
        __syncwarp();
    }
}

// --------------------------------------------------------------------------- limiter

template <int K>
struct LimStage {
    using T = Topo<K>;
    double X[T::N][3];
    double xs[3][T::NIP];
    int node[T::N];
};

// Barth-Jespersen blend per node and velocity component (zvcfd/fv/reference.py:578-601):
// the smallest clip((bound - u) / delta, 0, 1) over the flux points of the node's elements,
// delta the gradient's extrapolation from the node to the flux point and bound the extreme
// of the node's neighbours on delta's side. Lane 3 a + k of the team owns (node a, k).
template <int K, bool STORED>
__global__ void __launch_bounds__(CTA_THREADS)
k_limiter(const int *__restrict__ conn, long long base, long long count,
          const double *__restrict__ Xn, const double *__restrict__ georec,
          const double *__restrict__ U, const double *__restrict__ gradU,
          const double *__restrict__ lo, const double *__restrict__ hi,
          double *__restrict__ beta) {
    using T = Topo<K>;
    using R = Record<K>;
    constexpr int N = T::N;
    __shared__ Tab<K> tb;
    __shared__ LimStage<K> st_all[Team<K>::PER_CTA];
    tb.load();
    Walk<K> wk;
    LimStage<K> &st = st_all[wk.slot_in_cta()];
    const int lane = wk.lane;
    for (long long e0 = wk.first; e0 < count; e0 += wk.stride) {
        const long long le = e0 + wk.team;
        const bool on = le < count;
        const long long slot = base + le;
        if (on && lane < N) {
            const long long n = __ldg(conn + slot * N + lane);
            st.node[lane] = (int)n;
#pragma unroll
            for (int k = 0; k < 3; ++k) st.X[lane][k] = __ldg(Xn + n * 3 + k);
        }
        __syncwarp();
        if (on && lane < T::NIP) {
            const int s = lane;
            double A[3], xs[3];
            if (STORED) {
#pragma unroll
                for (int k = 0; k < 3; ++k) xs[k] = __ldg(georec + slot * T::REC + R::X + s * 3 + k);
            } else {
                flux_area<K>(tb, st.X, s, A, xs);
            }
#pragma unroll
            for (int k = 0; k < 3; ++k) st.xs[k][s] = xs[k];
        }
        __syncwarp();
        if (on && lane < 3 * N) {
            const int a = lane / 3, k = lane % 3;
            const long long n = st.node[a];
            const double g0 = __ldg(gradU + n * 9 + k * 3), g1 = __ldg(gradU + n * 9 + k * 3 + 1),
                         g2 = __ldg(gradU + n * 9 + k * 3 + 2);
            const double u = __ldg(U + n * 3 + k);
            const double up = __ldg(hi + n * 3 + k) - u, down = __ldg(lo + n * 3 + k) - u;
            double f = beta[n * 3 + k];
#pragma unroll
            for (int i = 0; i < T::MAXF; ++i) {
                const int s = tb.ips[a][i];
                if (s < 0) continue;
                const double delta = g0 * (st.xs[0][s] - st.X[a][0]) + g1 * (st.xs[1][s] - st.X[a][1]) +
                                     g2 * (st.xs[2][s] - st.X[a][2]);
                if (fabs(delta) > 1e-300)
                    f = fmin(f, fmin(fmax((delta > 0 ? up : down) / delta, 0.0), 1.0));
            }
            beta[n * 3 + k] = f;
        }
        __syncwarp();
    }
}

// --------------------------------------------------------------------------- launchers

// Resident CTAs of a kernel on the whole device (occupancy looked up once per kernel).
int resident_ctas(const void *kern) {
    static std::mutex lock;
    static std::vector<std::pair<const void *, int>> cache;
    std::lock_guard<std::mutex> guard(lock);
    for (const auto &e : cache)
        if (e.first == kern) return e.second;
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, CTA_THREADS, 0) != cudaSuccess)
        per_sm = 1;
    const int total = (per_sm > 0 ? per_sm : 1) * sm_count();
    cache.emplace_back(kern, total);
    return total;
}

// CTAs for a colour of `count` elements: enough for every team to own one element, capped
// at the resident limit (the grid-stride loop takes the rest).
template <int K, typename Kernel>
unsigned ctas_for(Kernel kern, long long count) {
    const long long resident = resident_ctas(reinterpret_cast<const void *>(kern));
    const long long need = (count + Team<K>::PER_CTA - 1) / Team<K>::PER_CTA;
    return (unsigned)(need < resident ? (need > 0 ? need : 1) : resident);
}

template <template <int, bool> class F, typename... A>
int dispatch(int kind, int stored, A &&...args) {
    switch (kind) {
        case TET: return stored ? F<TET, true>::run(args...) : F<TET, false>::run(args...);
        case PYRAMID: return stored ? F<PYRAMID, true>::run(args...) : F<PYRAMID, false>::run(args...);
        case WEDGE: return stored ? F<WEDGE, true>::run(args...) : F<WEDGE, false>::run(args...);
        case HEX: return stored ? F<HEX, true>::run(args...) : F<HEX, false>::run(args...);
    }
    set_error("unknown element kind %d", kind);
    return BAD_ARGUMENT;
}

// one launch per colour: slots [offsets[c], offsets[c + 1])
template <typename Launch>
void per_colour(int n_colours, const int64_t *offsets, Launch &&launch) {
    for (int c = 0; c < n_colours; ++c) {
        const long long base = offsets[c], count = offsets[c + 1] - offsets[c];
        if (count > 0) launch(base, count);
    }
}

template <int K, bool S>
struct StaticsL {
    static int run(const int *conn, int nc, const int64_t *off, const double *X, const double *geo,
                   const int *pos, double mu, int transpose, double *vol, double *dvisc,
                   double *gop, cudaStream_t st) {
        per_colour(nc, off, [&](long long base, long long count) {
            k_statics<K, S><<<ctas_for<K>(k_statics<K, S>, count), CTA_THREADS, 0, st>>>(
                conn, base, count, X, geo, pos, mu, transpose, vol, dvisc, gop);
            count_launch();
        });
        return launch_status("statics");
    }
};

template <int K, bool S>
struct DiagL {
    static int run(const DiagArgs &g, int nc, const int64_t *off, cudaStream_t st) {
        per_colour(nc, off, [&](long long base, long long count) {
            k_diag<K, S><<<ctas_for<K>(k_diag<K, S>, count), CTA_THREADS, 0, st>>>(g, base, count);
            count_launch();
        });
        return launch_status("diag");
    }
};

template <int K, bool S>
struct AssembleL {
    static int run(const AsmArgs &g, int nc, const int64_t *off, cudaStream_t st) {
        per_colour(nc, off, [&](long long base, long long count) {
            k_assemble<K, S><<<ctas_for<K>(k_assemble<K, S>, count), CTA_THREADS, 0, st>>>(
                g, base, count);
            count_launch();
        });
        return launch_status("assemble");
    }
};

template <int K, bool S>
struct MassL {
    static int run(const MassArgs &g, int nc, const int64_t *off, cudaStream_t st) {
        per_colour(nc, off, [&](long long base, long long count) {
            if (g.vdiag)
                k_massflow<K, S, true><<<ctas_for<K>(k_massflow<K, S, true>, count), CTA_THREADS,
                                         0, st>>>(g, base, count);
            else
                k_massflow<K, S, false><<<ctas_for<K>(k_massflow<K, S, false>, count),
                                          CTA_THREADS, 0, st>>>(g, base, count);
            count_launch();
        });
        return launch_status("massflow");
    }
};

template <int K, bool S>
struct LimiterL {
    static int run(const int *conn, int nc, const int64_t *off, const double *X, const double *geo,
                   const double *U, const double *gradU, const double *lo, const double *hi,
                   double *beta, cudaStream_t st) {
        per_colour(nc, off, [&](long long base, long long count) {
            k_limiter<K, S><<<ctas_for<K>(k_limiter<K, S>, count), CTA_THREADS, 0, st>>>(
                conn, base, count, X, geo, U, gradU, lo, hi, beta);
            count_launch();
        });
        return launch_status("limiter");
    }
};

template <int K, bool S>
struct GeoL {
    static int run(const int *conn, long long nslots, const double *X, double *geo, cudaStream_t st) {
        k_geobuild<K><<<ctas_for<K>(k_geobuild<K>, nslots), CTA_THREADS, 0, st>>>(conn, X, nslots,
                                                                                   geo);
        count_launch();
        return launch_status("geobuild");
    }
};

template <int K, bool S>
struct PosL {
    static int run(const int *conn, long long nslots, const long long *indptr, const int *indices,
                   int *pos, cudaStream_t st) {
        const long long warps = nslots * Topo<K>::N;
        k_blockpos<K><<<grid_for(warps * 32, 256), 256, 0, st>>>(conn, nslots, indptr, indices, pos);
        count_launch();
        return launch_status("blockpos");
    }
};

}  // namespace
}  // namespace zvfv

using namespace zvfv;

extern "C" {

int zvfv_record_doubles(int kind) {
    switch (kind) {
        case TET: return Topo<TET>::REC;
        case PYRAMID: return Topo<PYRAMID>::REC;
        case WEDGE: return Topo<WEDGE>::REC;
        case HEX: return Topo<HEX>::REC;
    }
    return -1;
}

int zvfv_geobuild(int kind, const int32_t *conn, int64_t n_slots, const double *X, double *geo,
                  void *stream) {
    if (n_slots <= 0) return OK;
    return dispatch<GeoL>(kind, 0, conn, (long long)n_slots, X, geo, as_stream(stream));
}

int zvfv_blockpos(int kind, const int32_t *conn, int64_t n_slots, const int64_t *indptr,
                  const int32_t *indices, int32_t *pos, void *stream) {
    if (n_slots <= 0) return OK;
    return dispatch<PosL>(kind, 0, conn, (long long)n_slots, (const long long *)indptr, indices,
                          pos, as_stream(stream));
}

int zvfv_statics(int kind, int stored, const int32_t *conn, int n_colours,
                 const int64_t *colour_offsets, const double *X, const double *geo,
                 const int32_t *pos, double mu, int transpose, double *vol, double *dvisc,
                 double *gop, void *stream) {
    return dispatch<StaticsL>(kind, stored, conn, n_colours, colour_offsets, X, geo, pos, mu,
                              transpose, vol, dvisc, gop, as_stream(stream));
}

int zvfv_diagonal(int kind, int stored, const int32_t *conn, int n_colours,
                  const int64_t *colour_offsets, const double *X, const double *geo,
                  const double *mdot, const double *U, int rheo, double mu0, double muinf,
                  double lam, double ca, double cn, int transpose, int stokes, int has_mut,
                  const double *mut, double *out, void *stream) {
    DiagArgs g{conn, X, geo, mdot, U, rheology_of(rheo, mu0, muinf, lam, ca, cn), transpose,
               stokes, has_mut, mut, out};
    return dispatch<DiagL>(kind, stored, g, n_colours, colour_offsets, as_stream(stream));
}

int zvfv_assemble(int kind, int stored, const int32_t *conn, int n_colours,
                  const int64_t *colour_offsets, const double *X, const double *geo,
                  const double *U, const double *mdot, const double *gradU, const double *beta,
                  const double *gradP, const double *dnode, const double *snode, int nlev,
                  double c1, const double *Uo1, const double *mo1, double c2, const double *Uo2,
                  const double *mo2, double rho, int rheo, double mu0, double muinf, double lam,
                  double ca, double cn, int transpose, int stokes, int has_mut, const double *mut,
                  const int32_t *own, const int32_t *pos, double *data, double *b, void *stream) {
    AsmArgs g{conn, X, geo, U, mdot, gradU, beta, gradP, dnode, snode, nlev, c1, Uo1, mo1, c2, Uo2,
              mo2, rho, rheology_of(rheo, mu0, muinf, lam, ca, cn), transpose, stokes, has_mut,
              mut, own, pos, data, b};
    return dispatch<AssembleL>(kind, stored, g, n_colours, colour_offsets, as_stream(stream));
}

int zvfv_massflow(int kind, int stored, const int32_t *conn, int n_colours,
                  const int64_t *colour_offsets, const double *X, const double *geo,
                  const double *U, const double *P, const double *gradP, const double *dnode,
                  const double *snode, int nlev, double c1, const double *Uo1, const double *mo1,
                  double c2, const double *Uo2, const double *mo2, double rho, double *mdot,
                  double *imbalance, double *adv, void *stream) {
    MassArgs g{conn, X, geo, U, P, gradP, dnode, snode, nlev, c1, Uo1, mo1, c2, Uo2, mo2, rho,
               mdot, imbalance, adv, rheology_of(0, 0.0, 0.0, 0.0, 2.0, 1.0), 0, 0, nullptr,
               nullptr};
    return dispatch<MassL>(kind, stored, g, n_colours, colour_offsets, as_stream(stream));
}

int zvfv_massflow_diag(int kind, int stored, const int32_t *conn, int n_colours,
                       const int64_t *colour_offsets, const double *X, const double *geo,
                       const double *U, const double *P, const double *gradP, const double *dnode,
                       const double *snode, int nlev, double c1, const double *Uo1,
                       const double *mo1, double c2, const double *Uo2, const double *mo2,
                       double rho, int rheo, double mu0, double muinf, double lam, double ca,
                       double cn, int transpose, int has_mut, const double *mut, double *mdot,
                       double *imbalance, double *adv, double *vdiag, void *stream) {
    if (!vdiag) {
        set_error("massflow_diag: no viscous-diagonal output");
        return BAD_ARGUMENT;
    }
    MassArgs g{conn, X, geo, U, P, gradP, dnode, snode, nlev, c1, Uo1, mo1, c2, Uo2, mo2, rho,
               mdot, imbalance, adv, rheology_of(rheo, mu0, muinf, lam, ca, cn), transpose,
               has_mut, mut, vdiag};
    return dispatch<MassL>(kind, stored, g, n_colours, colour_offsets, as_stream(stream));
}

int zvfv_limiter(int kind, int stored, const int32_t *conn, int n_colours,
                 const int64_t *colour_offsets, const double *X, const double *geo,
                 const double *U, const double *gradU, const double *lo, const double *hi,
                 double *beta, void *stream) {
    return dispatch<LimiterL>(kind, stored, conn, n_colours, colour_offsets, X, geo, U, gradU, lo,
                              hi, beta, as_stream(stream));
}

}  // extern "C"
