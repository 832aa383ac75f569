// Element kernels of the coupled 4x4 (u, v, w, p) finite-volume system, one template per
// element type: geometry records, block positions, statics (node volumes, the Newtonian
// viscous diagonal, the nodal-gradient operator), the momentum diagonal, the assembly of
// blocks and right-hand side, the Rhie-Chow mass flows and the Barth-Jespersen limiter.
//
// The discrete equations are the reference's (zvcfd/fv/reference.py:654-806 in lagged
// Rhie-Chow form, zvcfd/fv/_cuda_fast.py:239-603 on the device). Elements of one type are
// held in colour order ("slots": zvcfd/fv/fast.py:199-207); one launch covers one colour,
// whose elements share no node, so every read-modify-write of a block or a node value is
// owned by one thread and the result is deterministic without atomics.
#include "element.cuh"

namespace zvfv {

namespace {

template <int K>
constexpr int threads_of() { return Topo<K>::EPB * Topo<K>::N * Topo<K>::N; }

// The per-iteration element kernels are latency-bound (shared-memory phases separated by
// barriers); at their natural 72-96 registers only five blocks fit on an SM. Capping them
// at six blocks costs the hexahedral kernels about 100 bytes of spills per thread (L1) for
// 20 % more resident warps, with the shared-memory carveout at its maximum.
constexpr int ELEMENT_MIN_BLOCKS = 6;

template <typename Kernel>
void prefer_shared(Kernel k) {
    cudaFuncSetAttribute(k, cudaFuncAttributePreferredSharedMemoryCarveout,
                         (int)cudaSharedmemCarveoutMaxShared);
}

// --------------------------------------------------------------------------- geobuild

template <int K>
__global__ void __launch_bounds__(threads_of<K>())
k_geobuild(const int *__restrict__ conn, const double *__restrict__ X, long long nslots,
           double *__restrict__ georec) {
    using T = Topo<K>;
    constexpr int TE = T::N * T::N;
    __shared__ double s_x[T::EPB][T::N * 3];
    __shared__ double s_rec[T::EPB][T::REC];
    __shared__ SmemTab<K> tab;
    tab.load();
    const int le = threadIdx.x / TE, t = threadIdx.x % TE;
    const long long slot = (long long)blockIdx.x * T::EPB + le;
    const bool active = slot < nslots;
    if (active && t < T::N) {
        const long long n = conn[slot * T::N + t];
        for (int k = 0; k < 3; ++k) s_x[le][t * 3 + k] = X[n * 3 + k];
    }
    __syncthreads();
    element_geometry<K, false, true>(nullptr, slot, active, s_x[le], s_rec[le], t, tab);
    if (active)
        for (int i = t; i < T::REC; i += TE) georec[slot * T::REC + i] = s_rec[le][i];
}

// --------------------------------------------------------------------------- blockpos

// The pattern position of every (row node, column node) pair of every slot, by a binary
// search of the row (zvcfd/fv/_cuda_fast.py:605-623); -1 if the pair is missing.
template <int K>
__global__ void k_blockpos(const int *__restrict__ conn, long long nslots,
                           const long long *__restrict__ indptr, const int *__restrict__ indices,
                           int *__restrict__ pos) {
    using T = Topo<K>;
    constexpr int TE = T::N * T::N;
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nslots * TE) return;
    const long long slot = i / TE;
    const int t = (int)(i % TE), a = t / T::N, c = t % T::N;
    const long long row = conn[slot * T::N + a];
    const int col = conn[slot * T::N + c];
    long long lo = indptr[row], hi = indptr[row + 1] - 1, found = -1;
    while (lo <= hi) {
        const long long mid = (lo + hi) >> 1;
        const int v = indices[mid];
        if (v == col) { found = mid; break; }
        if (v < col) lo = mid + 1; else hi = mid - 1;
    }
    pos[i] = (int)found;
}

// --------------------------------------------------------------------------- statics

// Node volumes, the Newtonian viscous diagonal and the nodal-gradient operator (three
// coefficients per pattern block: row a, column c, the sub-volume of a times the element's
// mean gradient of N_c), zvcfd/fv/_cuda_fast.py:191-236.
template <int K, bool STORED>
__global__ void __launch_bounds__(threads_of<K>())
k_statics(const int *__restrict__ conn, long long base, long long count,
          const double *__restrict__ X, const double *__restrict__ georec,
          const int *__restrict__ pos, double mu, int transpose, double *__restrict__ vol,
          double *__restrict__ dvisc, double *__restrict__ gop) {
    using T = Topo<K>;
    using R = Rec<K>;
    constexpr int TE = T::N * T::N;
    __shared__ double s_x[T::EPB][T::N * 3];
    __shared__ double s_rec[T::EPB][T::REC];
    __shared__ int s_n[T::EPB][T::N];
    __shared__ SmemTab<K> tab;
    tab.load();
    const int le = threadIdx.x / TE, t = threadIdx.x % TE;
    const long long slot = base + (long long)blockIdx.x * T::EPB + le;
    const bool active = slot < base + count;
    if (active && t < T::N) {
        const int n = conn[slot * T::N + t];
        s_n[le][t] = n;
        for (int k = 0; k < 3; ++k) s_x[le][t * 3 + k] = X[(long long)n * 3 + k];
    }
    __syncthreads();
    element_geometry<K, STORED, true>(georec, slot, active, s_x[le], s_rec[le], t, tab);
    if (!active) return;
    const double *rec = s_rec[le];
    const int a = t / T::N, c = t % T::N;
    double gbar[3] = {0.0, 0.0, 0.0};
    for (int s = 0; s < T::NG; ++s)
        for (int k = 0; k < 3; ++k) gbar[k] += R::G(rec, s, c)[k];
    const long long p = pos[slot * TE + t];
    const double sa = rec[R::OFF_S + a];
    for (int k = 0; k < 3; ++k) gop[p * 3 + k] += sa * gbar[k] / T::NG;
    if (c == 0) {
        const int node = s_n[le][a];
        vol[node] += sa;
        double d = 0.0;
        for (int i = 0; i < MAXI; ++i) {
            const int s = tab.ips[a][i];
            if (s < 0) break;
            const double *A = R::A(rec, s);
            const double *G = R::G(rec, s, a);
            double r = -mu * (G[0] * A[0] + G[1] * A[1] + G[2] * A[2]);
            if (transpose) r -= mu * G[0] * A[0];
            d += tab.sgn[a][i] * r;
        }
        dvisc[node] += d;
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

// The momentum diagonal a_P with the viscosity at each flux point (zvcfd/fv/_cuda_fast.py:239-299)
template <int K, bool STORED>
__global__ void __launch_bounds__(threads_of<K>(), ELEMENT_MIN_BLOCKS)
k_diag(const DiagArgs g, long long base, long long count) {
    using T = Topo<K>;
    using R = Rec<K>;
    constexpr int TE = T::N * T::N;
    __shared__ double s_x[T::EPB][T::N * 3];
    __shared__ double s_u[T::EPB][T::N * 3];
    __shared__ double s_rec[T::EPB][T::REC];
    __shared__ double s_mu[T::EPB][T::NIP];
    __shared__ int s_n[T::EPB][T::N];
    __shared__ SmemTab<K> tab;
    tab.load();
    const int le = threadIdx.x / TE, t = threadIdx.x % TE;
    const long long slot = base + (long long)blockIdx.x * T::EPB + le;
    const bool active = slot < base + count;
    if (active && t < T::N) {
        const int n = g.conn[slot * T::N + t];
        s_n[le][t] = n;
        for (int k = 0; k < 3; ++k) {
            s_x[le][t * 3 + k] = g.X[(long long)n * 3 + k];
            s_u[le][t * 3 + k] = g.U[(long long)n * 3 + k];
        }
    }
    __syncthreads();
    element_geometry<K, STORED, false>(g.geo, slot, active, s_x[le], s_rec[le], t, tab);
    const double *rec = s_rec[le];
    if (active && t < T::NIP) {
        double mu = g.rh.mu0;
        if (g.rh.model) {
            double gu[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
            for (int q = 0; q < T::N; ++q) {
                const double *G = R::G(rec, t, q);
                for (int j = 0; j < 3; ++j)
                    for (int k = 0; k < 3; ++k) gu[j][k] += s_u[le][q * 3 + j] * G[k];
            }
            mu = viscosity(gu, g.rh);
        }
        if (g.has_mut)
            for (int q = 0; q < T::N; ++q) mu += tab.nip[t][q] * g.mut[s_n[le][q]];
        s_mu[le][t] = mu;
    }
    __syncthreads();
    if (!active || t >= T::N) return;
    const int a = t;
    double d = 0.0;
    for (int i = 0; i < MAXI; ++i) {
        const int s = tab.ips[a][i];
        if (s < 0) break;
        const double sg = tab.sgn[a][i], mu = s_mu[le][s];
        const double *A = R::A(rec, s);
        const double *G = R::G(rec, s, a);
        double r = -mu * (G[0] * A[0] + G[1] * A[1] + G[2] * A[2]);
        if (g.transpose) r -= mu * G[0] * A[0];
        d += sg * r;
        if (!g.stokes) {
            const double m = g.mdot[slot * T::NIP + s];
            d += sg > 0 ? fmax(m, 0.0) : fmax(-m, 0.0);
        }
    }
    g.out[s_n[le][a]] += d;
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

// Blocks and right-hand side of the flux points. Thread (a, c) owns block (row a, column c)
// of its element, summed over the flux points at a: viscous -mu G_c.A on the momentum
// diagonal (plus upwind advection), the transpose term -mu G_c[k] A[j], pressure N_c A,
// continuity rho N_c A and -rho d G_c.A. Threads (a, k < 4) add component k of row a's
// right-hand side: the deferred correction of the upwind node (momentum) and the lagged
// Rhie-Chow and transient parts (continuity).
template <int K, bool STORED>
__global__ void __launch_bounds__(threads_of<K>(), ELEMENT_MIN_BLOCKS)
k_assemble(const AsmArgs g, long long base, long long count) {
    using T = Topo<K>;
    using R = Rec<K>;
    constexpr int TE = T::N * T::N;
    constexpr int N = T::N;
    __shared__ double s_x[T::EPB][N * 3];
    __shared__ double s_u[T::EPB][N * 3];
    __shared__ double s_gp[T::EPB][N * 3];
    __shared__ double s_gu[T::EPB][N * 9];
    __shared__ double s_be[T::EPB][N * 3];
    __shared__ double s_u1[T::EPB][N * 3];
    __shared__ double s_u2[T::EPB][N * 3];
    __shared__ double s_dn[T::EPB][N];
    __shared__ double s_sn[T::EPB][N];
    __shared__ double s_rec[T::EPB][T::REC];
    __shared__ double s_ip[T::EPB][T::NIP][3];       // mu, mdot, d
    __shared__ double s_rhs[T::EPB][T::NIP][4];      // each flux point's right-hand side
    __shared__ int s_n[T::EPB][N];
    __shared__ SmemTab<K> tab;
    tab.load();
    const int le = threadIdx.x / TE, t = threadIdx.x % TE;
    const long long slot = base + (long long)blockIdx.x * T::EPB + le;
    const bool active = slot < base + count;
    if (active && t < N) {
        const int n = g.conn[slot * N + t];
        const long long n3 = (long long)n * 3;
        s_n[le][t] = n;
        for (int k = 0; k < 3; ++k) {
            s_x[le][t * 3 + k] = g.X[n3 + k];
            s_u[le][t * 3 + k] = g.U[n3 + k];
            s_gp[le][t * 3 + k] = g.gradP[n3 + k];
        }
        s_dn[le][t] = g.dnode[n];
        s_sn[le][t] = g.snode[n];
    } else if (active && t < 2 * N) {
        const int a = t - N;
        const long long n = g.conn[slot * N + a];
        if (!g.stokes) {
            for (int q = 0; q < 9; ++q) s_gu[le][a * 9 + q] = g.gradU[n * 9 + q];
            for (int k = 0; k < 3; ++k) s_be[le][a * 3 + k] = g.beta[n * 3 + k];
        }
        if (g.nlev > 0)
            for (int k = 0; k < 3; ++k) s_u1[le][a * 3 + k] = g.Uo1[n * 3 + k];
        if (g.nlev > 1)
            for (int k = 0; k < 3; ++k) s_u2[le][a * 3 + k] = g.Uo2[n * 3 + k];
    }
    __syncthreads();
    element_geometry<K, STORED, false>(g.geo, slot, active, s_x[le], s_rec[le], t, tab);
    const double *rec = s_rec[le];
    if (active && t < T::NIP) {
        const int s = t, ia = tab.edge[s][0], ib = tab.edge[s][1];
        double mu = g.rh.mu0;
        if (g.rh.model) {
            double gu[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
            for (int q = 0; q < N; ++q) {
                const double *G = R::G(rec, s, q);
                for (int j = 0; j < 3; ++j)
                    for (int k = 0; k < 3; ++k) gu[j][k] += s_u[le][q * 3 + j] * G[k];
            }
            mu = viscosity(gu, g.rh);
        }
        if (g.has_mut)
            for (int q = 0; q < N; ++q) mu += tab.nip[s][q] * g.mut[s_n[le][q]];
        const double m = g.mdot[slot * T::NIP + s];
        const double d = 0.5 * (s_dn[le][ia] + s_dn[le][ib]);
        s_ip[le][s][0] = mu;
        s_ip[le][s][1] = m;
        s_ip[le][s][2] = d;
        const double *A = R::A(rec, s);
        double gA = 0.0, u1 = 0.0, u2 = 0.0;
        for (int q = 0; q < N; ++q) {
            const double Nq = tab.nip[s][q];
            for (int j = 0; j < 3; ++j) {
                gA += Nq * s_gp[le][q * 3 + j] * A[j];
                if (g.nlev > 0) u1 += Nq * s_u1[le][q * 3 + j] * A[j];
                if (g.nlev > 1) u2 += Nq * s_u2[le][q * 3 + j] * A[j];
            }
        }
        double tr = 0.0;
        if (g.nlev > 0) {
            const double sbar = 0.5 * (s_sn[le][ia] + s_sn[le][ib]);
            tr = g.c1 * (g.mo1[slot * T::NIP + s] - g.rho * u1);
            if (g.nlev > 1) tr += g.c2 * (g.mo2[slot * T::NIP + s] - g.rho * u2);
            tr *= 1.0 - d / sbar;
        }
        s_rhs[le][s][3] = g.rho * d * gA + tr;
        const int up = m >= 0 ? ia : ib;
        for (int k = 0; k < 3; ++k) {
            double corr = 0.0;
            if (!g.stokes)
                for (int q = 0; q < 3; ++q)
                    corr += s_gu[le][up * 9 + k * 3 + q] * (R::X(rec, s)[q] - s_x[le][up * 3 + q]);
            s_rhs[le][s][k] = g.stokes ? 0.0 : m * s_be[le][up * 3 + k] * corr;
        }
    }
    __syncthreads();
    if (!active) return;
    const int a = t / N, c = t % N;
    double vis = 0.0, pv0 = 0.0, pv1 = 0.0, pv2 = 0.0, rcd = 0.0, adv = 0.0;
    double tr[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    for (int i = 0; i < MAXI; ++i) {
        const int s = tab.ips[a][i];
        if (s < 0) break;
        const double sg = tab.sgn[a][i];
        const double mu = s_ip[le][s][0], m = s_ip[le][s][1], d = s_ip[le][s][2];
        const double *A = R::A(rec, s);
        const double *G = R::G(rec, s, c);
        const double GA = G[0] * A[0] + G[1] * A[1] + G[2] * A[2];
        const double sN = sg * tab.nip[s][c];
        vis -= sg * mu * GA;
        rcd -= sg * d * GA;
        pv0 += sN * A[0];
        pv1 += sN * A[1];
        pv2 += sN * A[2];
        if (g.transpose) {
            const double smu = sg * mu;
            for (int k = 0; k < 3; ++k)
                for (int j = 0; j < 3; ++j) tr[k * 3 + j] -= smu * G[k] * A[j];
        }
        if (!g.stokes) {
            const int ia = tab.edge[s][0], ib = tab.edge[s][1];
            if ((c == ia && m > 0) || (c == ib && m < 0)) adv += sg * m;
        }
    }
    const double dg = vis + adv;
    const double acc[16] = {dg + tr[0], tr[1], tr[2], pv0,
                            tr[3], dg + tr[4], tr[5], pv1,
                            tr[6], tr[7], dg + tr[8], pv2,
                            g.rho * pv0, g.rho * pv1, g.rho * pv2, g.rho * rcd};
    const long long p = g.pos[slot * TE + t];
    double2 *blk = reinterpret_cast<double2 *>(g.data + p * 16);
#pragma unroll
    for (int q = 0; q < 8; ++q) {
        double2 v = blk[q];
        v.x += acc[2 * q];
        v.y += acc[2 * q + 1];
        blk[q] = v;
    }
    if (c < 4) {
        const int k = c;
        const bool mirror = k < 3 && g.own[s_n[le][a]];
        double r = 0.0;
        for (int i = 0; i < MAXI; ++i) {
            const int s = tab.ips[a][i];
            if (s < 0) break;
            // an inflow node keeps out of its own row the corrections of faces it is upwind of
            if (mirror && (s_ip[le][s][1] >= 0 ? tab.edge[s][0] : tab.edge[s][1]) == a) continue;
            r -= tab.sgn[a][i] * s_rhs[le][s][k];
        }
        g.b[(long long)s_n[le][a] * 4 + k] += r;
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

// New Rhie-Chow mass flows, each node's net interior outflow and the advective part of the
// next momentum diagonal (zvcfd/fv/_cuda_fast.py:469-553; reference.py:922-948). With VDIAG the
// same pass adds the viscous part of the next diagonal (the terms of k_diag,
// zvcfd/fv/_cuda_fast.py:239-299), so that the next iteration's a_P = vdiag + adv needs no
// element pass of its own: the velocity and mass flows k_diag would read at the start of that
// iteration are the ones at hand here.
template <int K, bool STORED, bool VDIAG>
__global__ void __launch_bounds__(threads_of<K>(), ELEMENT_MIN_BLOCKS)
k_massflow(const MassArgs g, long long base, long long count) {
    using T = Topo<K>;
    using R = Rec<K>;
    constexpr int TE = T::N * T::N;
    constexpr int N = T::N;
    __shared__ double s_x[T::EPB][N * 3];
    __shared__ double s_u[T::EPB][N * 3];
    __shared__ double s_gp[T::EPB][N * 3];
    __shared__ double s_u1[T::EPB][N * 3];
    __shared__ double s_u2[T::EPB][N * 3];
    __shared__ double s_p[T::EPB][N];
    __shared__ double s_dn[T::EPB][N];
    __shared__ double s_sn[T::EPB][N];
    __shared__ double s_rec[T::EPB][T::REC];
    __shared__ double s_m[T::EPB][T::NIP];
    __shared__ double s_mu[VDIAG ? T::EPB : 1][VDIAG ? T::NIP : 1];
    __shared__ int s_n[T::EPB][N];
    __shared__ SmemTab<K> tab;
    tab.load();
    const int le = threadIdx.x / TE, t = threadIdx.x % TE;
    const long long slot = base + (long long)blockIdx.x * T::EPB + le;
    const bool active = slot < base + count;
    if (active && t < N) {
        const int n = g.conn[slot * N + t];
        const long long n3 = (long long)n * 3;
        s_n[le][t] = n;
        for (int k = 0; k < 3; ++k) {
            s_x[le][t * 3 + k] = g.X[n3 + k];
            s_u[le][t * 3 + k] = g.U[n3 + k];
            s_gp[le][t * 3 + k] = g.gradP[n3 + k];
            if (g.nlev > 0) s_u1[le][t * 3 + k] = g.Uo1[n3 + k];
            if (g.nlev > 1) s_u2[le][t * 3 + k] = g.Uo2[n3 + k];
        }
        s_p[le][t] = g.P[n];
        s_dn[le][t] = g.dnode[n];
        s_sn[le][t] = g.snode[n];
    }
    __syncthreads();
    element_geometry<K, STORED, false>(g.geo, slot, active, s_x[le], s_rec[le], t, tab);
    const double *rec = s_rec[le];
    if (active && t < T::NIP) {
        const int s = t, ia = tab.edge[s][0], ib = tab.edge[s][1];
        const double *A = R::A(rec, s);
        double ua = 0.0, u1 = 0.0, u2 = 0.0, rc = 0.0;
        for (int q = 0; q < N; ++q) {
            const double Nq = tab.nip[s][q];
            const double *G = R::G(rec, s, q);
            for (int k = 0; k < 3; ++k) {
                ua += Nq * s_u[le][q * 3 + k] * A[k];
                if (g.nlev > 0) u1 += Nq * s_u1[le][q * 3 + k] * A[k];
                if (g.nlev > 1) u2 += Nq * s_u2[le][q * 3 + k] * A[k];
                rc += (Nq * s_gp[le][q * 3 + k] - G[k] * s_p[le][q]) * A[k];
            }
        }
        const double d = 0.5 * (s_dn[le][ia] + s_dn[le][ib]);
        double m = g.rho * ua + g.rho * d * rc;
        if (g.nlev > 0) {
            const double sbar = 0.5 * (s_sn[le][ia] + s_sn[le][ib]);
            double tr = g.c1 * (g.mo1[slot * T::NIP + s] - g.rho * u1);
            if (g.nlev > 1) tr += g.c2 * (g.mo2[slot * T::NIP + s] - g.rho * u2);
            m += (1.0 - d / sbar) * tr;
        }
        g.mdot[slot * T::NIP + s] = m;
        s_m[le][s] = m;
        if (VDIAG) {
            double mu = g.rh.mu0;
            if (g.rh.model) {
                double gu[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
                for (int q = 0; q < N; ++q) {
                    const double *G = R::G(rec, s, q);
                    for (int j = 0; j < 3; ++j)
                        for (int k = 0; k < 3; ++k) gu[j][k] += s_u[le][q * 3 + j] * G[k];
                }
                mu = viscosity(gu, g.rh);
            }
            if (g.has_mut)
                for (int q = 0; q < N; ++q) mu += tab.nip[s][q] * g.mut[s_n[le][q]];
            s_mu[le][s] = mu;
        }
    }
    __syncthreads();
    if (!active || t >= N) return;
    const int a = t;
    double out = 0.0, ad = 0.0, vd = 0.0;
    for (int i = 0; i < MAXI; ++i) {
        const int s = tab.ips[a][i];
        if (s < 0) break;
        const double sg = tab.sgn[a][i], m = s_m[le][s];
        out += sg * m;
        ad += sg > 0 ? fmax(m, 0.0) : fmax(-m, 0.0);
        if (VDIAG) {
            const double mu = s_mu[le][s];
            const double *A = R::A(rec, s);
            const double *G = R::G(rec, s, a);
            double r = -mu * (G[0] * A[0] + G[1] * A[1] + G[2] * A[2]);
            if (g.transpose) r -= mu * G[0] * A[0];
            vd += sg * r;
        }
    }
    g.imbalance[s_n[le][a]] += out;
    g.adv[s_n[le][a]] += ad;
    if (VDIAG) g.vdiag[s_n[le][a]] += vd;
}

// --------------------------------------------------------------------------- limiter

// Barth-Jespersen blend per node and velocity component over the flux points of the node's
// elements (zvcfd/fv/reference.py:578-601). The smallest ratio (h - u)/delta over delta > 0
// is (h - u)/max delta, as division is monotone in its denominator: two divisions per
// (node, component) instead of one per flux point, with the same result.
template <int K, bool STORED>
__global__ void __launch_bounds__(threads_of<K>(), ELEMENT_MIN_BLOCKS)
k_limiter(const int *__restrict__ conn, long long base, long long count,
          const double *__restrict__ X, const double *__restrict__ georec,
          const double *__restrict__ U, const double *__restrict__ gradU,
          const double *__restrict__ lo, const double *__restrict__ hi,
          double *__restrict__ beta) {
    using T = Topo<K>;
    using R = Rec<K>;
    constexpr int TE = T::N * T::N;
    __shared__ double s_x[T::EPB][T::N * 3];
    __shared__ double s_rec[T::EPB][T::REC];
    __shared__ int s_n[T::EPB][T::N];
    __shared__ SmemTab<K> tab;
    tab.load();
    const int le = threadIdx.x / TE, t = threadIdx.x % TE;
    const long long slot = base + (long long)blockIdx.x * T::EPB + le;
    const bool active = slot < base + count;
    if (active && t < T::N) {
        const int n = conn[slot * T::N + t];
        s_n[le][t] = n;
        for (int k = 0; k < 3; ++k) s_x[le][t * 3 + k] = X[(long long)n * 3 + k];
    }
    __syncthreads();
    element_geometry<K, STORED, false>(georec, slot, active, s_x[le], s_rec[le], t, tab);
    if (!active || t >= 3 * T::N) return;
    const int a = t / 3, k = t % 3;
    const long long n = s_n[le][a];
    const double *rec = s_rec[le];
    const double g0 = gradU[(n * 3 + k) * 3], g1 = gradU[(n * 3 + k) * 3 + 1],
                 g2 = gradU[(n * 3 + k) * 3 + 2];
    const double u = U[n * 3 + k], h = hi[n * 3 + k], l = lo[n * 3 + k];
    double dpos = 0.0, dneg = 0.0;
    for (int i = 0; i < MAXI; ++i) {
        const int s = tab.ips[a][i];
        if (s < 0) break;
        const double *xp = R::X(rec, s);
        const double delta = g0 * (xp[0] - s_x[le][a * 3]) + g1 * (xp[1] - s_x[le][a * 3 + 1]) +
                             g2 * (xp[2] - s_x[le][a * 3 + 2]);
        if (delta > 1e-300) dpos = fmax(dpos, delta);
        else if (delta < -1e-300) dneg = fmin(dneg, delta);
    }
    double bmin = beta[n * 3 + k];
    if (dpos > 0.0) bmin = fmin(bmin, fmin(fmax((h - u) / dpos, 0.0), 1.0));
    if (dneg < 0.0) bmin = fmin(bmin, fmin(fmax((l - u) / dneg, 0.0), 1.0));
    beta[n * 3 + k] = bmin;
}

// --------------------------------------------------------------------------- launchers

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
template <int K, typename Launch>
int per_colour(int n_colours, const int64_t *offsets, Launch &&launch) {
    for (int c = 0; c < n_colours; ++c) {
        const long long base = offsets[c], count = offsets[c + 1] - offsets[c];
        if (count <= 0) continue;
        launch(grid_for(count, Topo<K>::EPB), base, count);
    }
    return OK;
}

template <int K, bool S>
struct StaticsL {
    static int run(const int *conn, int nc, const int64_t *off, const double *X, const double *geo,
                   const int *pos, double mu, int transpose, double *vol, double *dvisc,
                   double *gop, cudaStream_t st) {
        per_colour<K>(nc, off, [&](unsigned grid, long long base, long long count) {
            k_statics<K, S><<<grid, threads_of<K>(), 0, st>>>(conn, base, count, X, geo, pos, mu,
                                                              transpose, vol, dvisc, gop); count_launch();
        });
        return launch_status("statics");
    }
};

template <int K, bool S>
struct DiagL {
    static int run(const DiagArgs &g, int nc, const int64_t *off, cudaStream_t st) {
        static const bool carveout = (prefer_shared(k_diag<K, S>), true);
        (void)carveout;
        per_colour<K>(nc, off, [&](unsigned grid, long long base, long long count) {
            k_diag<K, S><<<grid, threads_of<K>(), 0, st>>>(g, base, count); count_launch();
        });
        return launch_status("diag");
    }
};

template <int K, bool S>
struct AssembleL {
    static int run(const AsmArgs &g, int nc, const int64_t *off, cudaStream_t st) {
        static const bool carveout = (prefer_shared(k_assemble<K, S>), true);
        (void)carveout;
        per_colour<K>(nc, off, [&](unsigned grid, long long base, long long count) {
            k_assemble<K, S><<<grid, threads_of<K>(), 0, st>>>(g, base, count); count_launch();
        });
        return launch_status("assemble");
    }
};

template <int K, bool S>
struct MassL {
    static int run(const MassArgs &g, int nc, const int64_t *off, cudaStream_t st) {
        static const bool carveout = (prefer_shared(k_massflow<K, S, false>),
                                      prefer_shared(k_massflow<K, S, true>), true);
        (void)carveout;
        per_colour<K>(nc, off, [&](unsigned grid, long long base, long long count) {
            if (g.vdiag) k_massflow<K, S, true><<<grid, threads_of<K>(), 0, st>>>(g, base, count);
            else k_massflow<K, S, false><<<grid, threads_of<K>(), 0, st>>>(g, base, count);
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
        static const bool carveout = (prefer_shared(k_limiter<K, S>), true);
        (void)carveout;
        per_colour<K>(nc, off, [&](unsigned grid, long long base, long long count) {
            k_limiter<K, S><<<grid, threads_of<K>(), 0, st>>>(conn, base, count, X, geo, U, gradU,
                                                              lo, hi, beta); count_launch();
        });
        return launch_status("limiter");
    }
};

template <int K, bool S>
struct GeoL {
    static int run(const int *conn, long long nslots, const double *X, double *geo, cudaStream_t st) {
        k_geobuild<K><<<grid_for(nslots, Topo<K>::EPB), threads_of<K>(), 0, st>>>(conn, X, nslots,
                                                                                   geo); count_launch();
        return launch_status("geobuild");
    }
};

template <int K, bool S>
struct PosL {
    static int run(const int *conn, long long nslots, const long long *indptr, const int *indices,
                   int *pos, cudaStream_t st) {
        const long long work = nslots * Topo<K>::N * Topo<K>::N;
        k_blockpos<K><<<grid_for(work, 256), 256, 0, st>>>(conn, nslots, indptr, indices, pos); count_launch();
        return launch_status("blockpos");
    }
};

Rheology rheology_of(int model, double mu0, double muinf, double lam, double a, double n) {
    Rheology r;
    r.model = model;
    r.mu0 = mu0;
    r.muinf = muinf;
    r.lam = lam;
    r.a = a;
    r.n = n;
    return r;
}

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
