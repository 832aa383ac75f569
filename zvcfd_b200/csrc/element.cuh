// Per-element machinery of the element kernels: shared-memory copies of the type's tables,
// the element geometry record (flux-point areas and centroids, shape-function gradients,
// sub-control volumes), and the Carreau-Yasuda viscosity.
//
// Thread layout of every element kernel: a CTA holds EPB elements of one type and gives
// each element N*N threads (t = a*N + c, the (row node, column node) pair of a block).
// Everything an element needs is staged in shared memory once; the tables are copied
// there too, because threads of a warp index them by their own node or flux point and
// divergent constant-memory reads serialise.
#pragma once

#include "common.cuh"

namespace zvfv {

// Geometry record layout (doubles): areas A[NIP][3], centroids X[NIP][3],
// gradients G[NG][N][3], sub-volumes S[N]. Stored records use the same layout.
template <int K>
struct Rec {
    using T = Topo<K>;
    static constexpr int OFF_A = 0;
    static constexpr int OFF_X = T::NIP * 3;
    static constexpr int OFF_G = 2 * T::NIP * 3;
    static constexpr int OFF_S = 2 * T::NIP * 3 + T::NG * T::N * 3;
    static constexpr int SIZE = OFF_S + T::N;
    static_assert(SIZE == T::REC, "record size");
    __device__ static const double *A(const double *r, int s) { return r + OFF_A + s * 3; }
    __device__ static const double *X(const double *r, int s) { return r + OFF_X + s * 3; }
    __device__ static const double *G(const double *r, int s, int a) {
        return r + OFF_G + ((T::CONSTG ? 0 : s) * T::N + a) * 3;
    }
};

template <int K>
struct SmemTab {
    using T = Topo<K>;
    int ips[T::N][MAXI];
    double sgn[T::N][MAXI];
    double nip[T::NIP][T::N];
    int edge[T::NIP][2];
    int tris[T::NIP][3];
    double wpt[T::NPTS][T::N];
    double dn[T::NIP][T::N][3];

    __device__ void load() {
        const int nt = blockDim.x;
        for (int i = threadIdx.x; i < T::N * MAXI; i += nt) {
            (&ips[0][0])[i] = (&T::ips()[0][0])[i];
            (&sgn[0][0])[i] = (&T::sgn()[0][0])[i];
        }
        for (int i = threadIdx.x; i < T::NIP * T::N; i += nt) (&nip[0][0])[i] = (&T::nip()[0][0])[i];
        for (int i = threadIdx.x; i < T::NIP * 2; i += nt) (&edge[0][0])[i] = (&T::edge()[0][0])[i];
        for (int i = threadIdx.x; i < T::NIP * 3; i += nt) (&tris[0][0])[i] = (&T::tris()[0][0])[i];
        for (int i = threadIdx.x; i < T::NPTS * T::N; i += nt) (&wpt[0][0])[i] = (&T::wpt()[0][0])[i];
        for (int i = threadIdx.x; i < T::NIP * T::N * 3; i += nt)
            (&dn[0][0][0])[i] = (&T::dn()[0][0][0])[i];
    }
};

__device__ inline void inverse3(const double J[3][3], double I[3][3]) {
    // adjugate over determinant
    const double c00 = J[1][1] * J[2][2] - J[1][2] * J[2][1];
    const double c01 = J[1][2] * J[2][0] - J[1][0] * J[2][2];
    const double c02 = J[1][0] * J[2][1] - J[1][1] * J[2][0];
    const double det = J[0][0] * c00 + J[0][1] * c01 + J[0][2] * c02;
    const double r = 1.0 / det;
    I[0][0] = c00 * r;
    I[1][0] = c01 * r;
    I[2][0] = c02 * r;
    I[0][1] = (J[0][2] * J[2][1] - J[0][1] * J[2][2]) * r;
    I[1][1] = (J[0][0] * J[2][2] - J[0][2] * J[2][0]) * r;
    I[2][1] = (J[0][1] * J[2][0] - J[0][0] * J[2][1]) * r;
    I[0][2] = (J[0][1] * J[1][2] - J[0][2] * J[1][1]) * r;
    I[1][2] = (J[0][2] * J[1][0] - J[0][0] * J[1][2]) * r;
    I[2][2] = (J[0][0] * J[1][1] - J[0][1] * J[1][0]) * r;
}

struct Rheology {
    int model;            // 0 Newtonian, 1 Carreau-Yasuda
    double mu0, muinf, lam, a, n;
};

// mu(gamma_dot) at a flux point from the velocity gradient gu[j][k] = du_j/dx_k
__device__ inline double viscosity(const double gu[3][3], const Rheology &r) {
    if (r.model == 0) return r.mu0;
    double ss = 0.0;
#pragma unroll
    for (int j = 0; j < 3; ++j)
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            const double s = 0.5 * (gu[j][k] + gu[k][j]);
            ss += s * s;
        }
    const double g = sqrt(2.0 * ss);
    return r.muinf + (r.mu0 - r.muinf) * pow(1.0 + pow(r.lam * g, r.a), (r.n - 1.0) / r.a);
}

// The element's geometry record in shared memory, by its N*N threads (t = 0..N*N-1): copied
// from a stored record, or rebuilt from the node coordinates xs[N*3] (one thread per flux
// point, then one per node for the sub-volumes). Every thread of the CTA calls it.
template <int K, bool STORED, bool NEED_SCV>
__device__ void element_geometry(const double *__restrict__ georec, long long slot, bool active,
                                 const double *xs, double *rec, int t, const SmemTab<K> &tab) {
    using T = Topo<K>;
    using R = Rec<K>;
    constexpr int TE = T::N * T::N;
    if (STORED) {
        if (active)
            for (int i = t; i < T::REC; i += TE) rec[i] = georec[slot * T::REC + i];
        __syncthreads();
        return;
    }
    if (active) {
        for (int s = t; s < T::NIP; s += TE) {
            double p[3][3];
#pragma unroll
            for (int v = 0; v < 3; ++v) {
                const int q = tab.tris[s][v];
#pragma unroll
                for (int k = 0; k < 3; ++k) {
                    double acc = 0.0;
#pragma unroll
                    for (int a = 0; a < T::N; ++a) acc += tab.wpt[q][a] * xs[a * 3 + k];
                    p[v][k] = acc;
                }
            }
            double u[3], w[3];
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                u[k] = p[1][k] - p[0][k];
                w[k] = p[2][k] - p[0][k];
            }
            rec[R::OFF_A + s * 3 + 0] = 0.5 * (u[1] * w[2] - u[2] * w[1]);
            rec[R::OFF_A + s * 3 + 1] = 0.5 * (u[2] * w[0] - u[0] * w[2]);
            rec[R::OFF_A + s * 3 + 2] = 0.5 * (u[0] * w[1] - u[1] * w[0]);
#pragma unroll
            for (int k = 0; k < 3; ++k)
                rec[R::OFF_X + s * 3 + k] = (p[0][k] + p[1][k] + p[2][k]) / 3.0;
            if (!T::CONSTG || s == 0) {
                double J[3][3], I[3][3];
#pragma unroll
                for (int k = 0; k < 3; ++k)
#pragma unroll
                    for (int d = 0; d < 3; ++d) {
                        double acc = 0.0;
#pragma unroll
                        for (int a = 0; a < T::N; ++a) acc += xs[a * 3 + k] * tab.dn[s][a][d];
                        J[k][d] = acc;
                    }
                inverse3(J, I);
                double *G = rec + R::OFF_G + (T::CONSTG ? 0 : s) * T::N * 3;
#pragma unroll
                for (int a = 0; a < T::N; ++a)
#pragma unroll
                    for (int k = 0; k < 3; ++k)
                        G[a * 3 + k] = tab.dn[s][a][0] * I[0][k] + tab.dn[s][a][1] * I[1][k] +
                                       tab.dn[s][a][2] * I[2][k];
            }
        }
    }
    __syncthreads();
    if (NEED_SCV) {
        if (active && t < T::N) {
            double v = 0.0;
            for (int i = 0; i < MAXI; ++i) {
                const int s = tab.ips[t][i];
                if (s < 0) break;
                double d = 0.0;
#pragma unroll
                for (int k = 0; k < 3; ++k)
                    d += (rec[R::OFF_X + s * 3 + k] - xs[t * 3 + k]) * rec[R::OFF_A + s * 3 + k];
                v += tab.sgn[t][i] * d / 3.0;
            }
            rec[R::OFF_S + t] = v;
        }
        __syncthreads();
    }
}

}  // namespace zvfv
