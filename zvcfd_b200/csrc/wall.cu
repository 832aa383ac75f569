// Wall shear stress at wall nodes from the wall integration points of their sub-faces
// (zvcfd/fv/wall.py:66-137): per ip, grad u from the owning element's shape gradients, the
// traction t = mu (grad u + grad u^T) . n, its tangential part, area-weighted per node.
#include "fvmath.cuh"

namespace zvfv {
namespace {

constexpr int MAXN = 8;

// one thread per node; node_ptr groups the ips of each node (none off the wall)
__global__ void k_wall_shear(long long N, const long long *__restrict__ node_ptr,
                             const int *__restrict__ elem, const double *__restrict__ G,
                             const double *__restrict__ nrm, const double *__restrict__ area,
                             const double *__restrict__ U, Rheology rh, double *__restrict__ tau) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    const long long q0 = node_ptr[i], q1 = node_ptr[i + 1];
    if (q0 == q1) return;
    double acc[3] = {0.0, 0.0, 0.0}, asum = 0.0;
    for (long long q = q0; q < q1; ++q) {
        double g[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
        for (int a = 0; a < MAXN; ++a) {
            const int n = elem[q * MAXN + a];
            if (n < 0) break;
            const double *ga = G + (q * MAXN + a) * 3;
            for (int r = 0; r < 3; ++r) {
                const double u = U[(long long)n * 3 + r];
                for (int c = 0; c < 3; ++c) g[r][c] += u * ga[c];
            }
        }
        double D[3][3], dd = 0.0;
        for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 3; ++c) {
                D[r][c] = g[r][c] + g[c][r];
                dd += D[r][c] * D[r][c];
            }
        double mu = rh.mu0;
        if (rh.model) {
            const double rate = sqrt(0.5 * dd);
            mu = rh.muinf + (rh.mu0 - rh.muinf) * pow(1.0 + pow(rh.lam * rate, rh.a), (rh.n - 1.0) / rh.a);
        }
        const double *nv = nrm + q * 3;
        double t[3], tn = 0.0;
        for (int r = 0; r < 3; ++r) {
            t[r] = mu * (D[r][0] * nv[0] + D[r][1] * nv[1] + D[r][2] * nv[2]);
            tn += t[r] * nv[r];
        }
        const double ar = area[q];
        for (int r = 0; r < 3; ++r) acc[r] -= (t[r] - tn * nv[r]) * ar;
        asum += ar;
    }
    const double inv = 1.0 / fmax(asum, 1e-300);
    for (int r = 0; r < 3; ++r) tau[i * 3 + r] = acc[r] * inv;
}

}  // namespace
}  // namespace zvfv

using namespace zvfv;

extern "C" {

int zvfv_wall_shear(int64_t n_nodes, const int64_t *node_ptr, const int32_t *elem,
                    const double *grad, const double *normal, const double *area,
                    const double *U, int rheo, double mu0, double muinf, double lam, double ca,
                    double cn, double *tau, void *stream) {
    if (n_nodes <= 0) return OK;
    Rheology rh;
    rh.model = rheo;
    rh.mu0 = mu0;
    rh.muinf = muinf;
    rh.lam = lam;
    rh.a = ca;
    rh.n = cn;
    k_wall_shear<<<grid_for(n_nodes, 128), 128, 0, as_stream(stream)>>>(
        n_nodes, (const long long *)node_ptr, elem, grad, normal, area, U, rh, tau); count_launch();
    return launch_status("wall shear");
}

}  // extern "C"
