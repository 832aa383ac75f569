// Small device math of the finite-volume kernels: the fluid's viscosity law and 3x3 algebra.
#pragma once

#include "common.cuh"

namespace zvfv {

// The fluid: model 0 Newtonian (mu0), 1 Carreau-Yasuda (zvcfd/rheology.py:37-62):
// mu = mu_inf + (mu0 - mu_inf) (1 + (lam g)^a)^((n - 1) / a), g the shear rate.
struct Rheology {
    int model;
    double mu0, muinf, lam, a, n;
};

inline Rheology rheology_of(int model, double mu0, double muinf, double lam, double a, double n) {
    Rheology r;
    r.model = model;
    r.mu0 = mu0;
    r.muinf = muinf;
    r.lam = lam;
    r.a = a;
    r.n = n;
    return r;
}

__device__ inline double carreau_yasuda(double rate, const Rheology &r) {
    const double shear = pow(r.lam * rate, r.a);
    return r.muinf + (r.mu0 - r.muinf) * pow(1.0 + shear, (r.n - 1.0) / r.a);
}

// Viscosity of a velocity gradient L (L[j*3+k] = du_j/dx_k): the shear rate is
// sqrt(2 D:D) with D the symmetric part of L, i.e. sqrt(sum_jk (L_jk + L_kj)^2 / 2).
__device__ inline double viscosity_of_gradient(const double *L, const Rheology &r) {
    if (r.model == 0) return r.mu0;
    double sum = 0.0;
#pragma unroll
    for (int j = 0; j < 3; ++j) {
        sum += 2.0 * L[j * 4] * L[j * 4];                         // diagonal: (2 L_jj)^2 / 2
#pragma unroll
        for (int k = j + 1; k < 3; ++k) {
            const double e = L[j * 3 + k] + L[k * 3 + j];
            sum += e * e;                                          // both (j,k) and (k,j)
        }
    }
    return carreau_yasuda(sqrt(sum), r);
}

// Inverse of a 3x3 matrix M (row-major) as adjugate / determinant; R = M^-1 (row-major).
__device__ inline void invert3(const double *M, double *R) {
    // cofactors of the first row, then the determinant along it
    const double c0 = M[4] * M[8] - M[5] * M[7];
    const double c1 = M[5] * M[6] - M[3] * M[8];
    const double c2 = M[3] * M[7] - M[4] * M[6];
    const double inv = 1.0 / (M[0] * c0 + M[1] * c1 + M[2] * c2);
    // R = adj(M) / det: column j of adj holds the cofactors of row j of M
    R[0] = c0 * inv;
    R[3] = c1 * inv;
    R[6] = c2 * inv;
    R[1] = (M[2] * M[7] - M[1] * M[8]) * inv;
    R[4] = (M[0] * M[8] - M[2] * M[6]) * inv;
    R[7] = (M[1] * M[6] - M[0] * M[7]) * inv;
    R[2] = (M[1] * M[5] - M[2] * M[4]) * inv;
    R[5] = (M[2] * M[3] - M[0] * M[5]) * inv;
    R[8] = (M[0] * M[4] - M[1] * M[3]) * inv;
}

}  // namespace zvfv
