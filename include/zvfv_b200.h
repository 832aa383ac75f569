/*
 * zvfv_b200.h — C ABI of libzvfv_b200.so, the B200 (sm_100a) coupled finite-volume solve path.
 *
 * Conventions (those of the reference's AmgX binding, zvcfd/fv/linear.py:681-955, and of its
 * CuPy kernel launches): every array is a raw device pointer; sizes are int64_t; every entry
 * point returns an int status (0 = success, see ZVFV_* below) and zvfv_last_error() gives the
 * message of the last failure on the calling thread; `stream` is a cudaStream_t (NULL = the
 * legacy default stream). Nothing synchronises the stream unless its comment says so.
 * Element types: 0 tet, 1 pyramid, 2 wedge, 3 hex (VTK local node order). Per-type element
 * arrays are in "slot" order (elements sorted by colour) and the per-colour launches take
 * the host array colour_offsets[n_colours + 1] of first slots.
 */
#ifndef ZVFV_B200_H
#define ZVFV_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
    ZVFV_OK = 0,
    ZVFV_BAD_ARGUMENT = 1,
    ZVFV_CUDA_FAILURE = 2,
    ZVFV_OUT_OF_MEMORY = 3,
    ZVFV_NOT_CONVERGED = 4,
    ZVFV_TIMED_OUT = 5,
    ZVFV_NON_FINITE = 6,
    ZVFV_UNSUPPORTED = 7
};

/* ---------------------------------------------------------------- library */

const char *zvfv_last_error(void);
int zvfv_version(void);
/* kernels this library has launched since the process started (a replayed V-cycle graph
 * counts every kernel node it runs; its capture counts none) */
int64_t zvfv_launch_count(void);
/* doubles per stored geometry record of an element type (zvcfd/fv/fast.py:150-152) */
int zvfv_record_doubles(int kind);

/* ---------------------------------------------------------------- once-per-mesh setup */

/* The block pattern: sorted unique (row, col) node pairs of all elements, self included.
 * Replaces zvcfd/fv/fast.py:133-147 gpu_node_graph (host form zvcfd/fv/pattern.py:18-33).
 * create builds it in a handle and reports nnzb (synchronises the stream); fill writes
 * indptr int64 (N+1) and indices int32 (nnzb) into caller memory; destroy frees the handle. */
int zvfv_pattern_create(void **handle, int64_t n_nodes, int n_kinds, const int32_t *const *conn,
                        const int64_t *n_elems, const int32_t *nodes_per, int64_t *nnzb,
                        void *stream);
int zvfv_pattern_fill(void *handle, int64_t *indptr, int32_t *indices, void *stream);
int zvfv_pattern_destroy(void *handle);

/* Element colouring, bit-exact with zvcfd/fv/fast.py:84-130 gpu_colour (kernels
 * colour_claim/colour_pick, zvcfd/fv/fast.py:35-70): colour int32 (E), *n_colours on the host.
 * Synchronises the stream once per round. */
int zvfv_colour(const int32_t *conn, int n, int64_t E, int64_t n_nodes, int words,
                int32_t *colour, int32_t *n_colours, int64_t max_rounds, void *stream);

/* Slot order argsort(colour * E + e) and colour offsets (zvcfd/fv/fast.py:199-203):
 * order int64 (E, slot -> element), offsets int64 (n_colours + 1) on the device. */
int zvfv_slot_order(const int32_t *colour, int64_t E, int32_t n_colours, int64_t *order,
                    int64_t *offsets, void *stream);

/* dst[r] = src[idx[r]] (scatter = 0) or dst[idx[r]] = src[r] (scatter = 1), rows of `width`
 * bytes: FastAssembler.to_slots / from_slots (zvcfd/fv/fast.py:276-290). */
int zvfv_permute_rows(const void *src, const int64_t *idx, int64_t rows, int64_t width, void *dst,
                      int scatter, void *stream);

/* Geometry records of every slot (kernel geobuild, zvcfd/fv/_cuda_fast.py:169-188). */
int zvfv_geobuild(int kind, const int32_t *conn, int64_t n_slots, const double *X, double *geo,
                  void *stream);

/* Pattern position of every (row, col) pair of every slot (kernel blockpos,
 * zvcfd/fv/_cuda_fast.py:605-623); pos int32 (E * n * n). */
int zvfv_blockpos(int kind, const int32_t *conn, int64_t n_slots, const int64_t *indptr,
                  const int32_t *indices, int32_t *pos, void *stream);

/* Node volumes, Newtonian viscous diagonal, nodal-gradient operator (kernel statics,
 * zvcfd/fv/_cuda_fast.py:191-236); accumulates into vol (N), dvisc (N), gop (nnzb * 3). */
int zvfv_statics(int kind, int stored, const int32_t *conn, int n_colours,
                 const int64_t *colour_offsets, const double *X, const double *geo,
                 const int32_t *pos, double mu, int transpose, double *vol, double *dvisc,
                 double *gop, void *stream);

/* ---------------------------------------------------------------- per outer iteration */

/* Nodal gradients of nc <= 4 fields through the gradient operator (kernel csr_gradient,
 * zvcfd/fv/_cuda_fast.py:627-651, FastAssembler.gradient zvcfd/fv/fast.py:310-325), with the
 * symmetry-plane mirror of zvcfd/fv/solver.py:441-457 applied when sym (N*3 uint8) is given;
 * the first nvec fields form a vector. out (N, nc, 3). */
int zvfv_gradient(int64_t n, int nc, int nvec, const int64_t *indptr, const int32_t *indices,
                  const double *gop, const double *phi, const uint8_t *sym, double *out,
                  void *stream);

/* Neighbour extremes of U over the pattern (kernel csr_minmax, zvcfd/fv/_cuda_fast.py:653-667). */
int zvfv_minmax(int64_t n, const int64_t *indptr, const int32_t *indices, const double *U,
                double *lo, double *hi, void *stream);

/* Barth-Jespersen blend (kernel limiter, zvcfd/fv/_cuda_fast.py:555-603; FastAssembler.limiter
 * zvcfd/fv/fast.py:394-406); beta (N*3) initialised to 1 by the caller, min-accumulated. */
int zvfv_limiter(int kind, int stored, const int32_t *conn, int n_colours,
                 const int64_t *colour_offsets, const double *X, const double *geo,
                 const double *U, const double *gradU, const double *lo, const double *hi,
                 double *beta, void *stream);

/* Momentum diagonal a_P (kernel diag, zvcfd/fv/_cuda_fast.py:239-299; FastAssembler.diagonal
 * zvcfd/fv/fast.py:327-337); accumulates into out (N). rheo 0 Newtonian, 1 Carreau-Yasuda. */
int zvfv_diagonal(int kind, int stored, const int32_t *conn, int n_colours,
                  const int64_t *colour_offsets, const double *X, const double *geo,
                  const double *mdot, const double *U, int rheo, double mu0, double muinf,
                  double lam, double ca, double cn, int transpose, int stokes, int has_mut,
                  const double *mut, double *out, void *stream);

/* Blocks and right-hand side of the flux points, lagged Rhie-Chow (kernel assemble,
 * zvcfd/fv/_cuda_fast.py:301-467; FastAssembler.assemble zvcfd/fv/fast.py:339-360);
 * accumulates into data (nnzb * 16) and b (N * 4). */
int zvfv_assemble(int kind, int stored, const int32_t *conn, int n_colours,
                  const int64_t *colour_offsets, const double *X, const double *geo,
                  const double *U, const double *mdot, const double *gradU, const double *beta,
                  const double *gradP, const double *dnode, const double *snode, int nlev,
                  double c1, const double *Uo1, const double *mo1, double c2, const double *Uo2,
                  const double *mo2, double rho, int rheo, double mu0, double muinf, double lam,
                  double ca, double cn, int transpose, int stokes, int has_mut, const double *mut,
                  const int32_t *own, const int32_t *pos, double *data, double *b, void *stream);

/* Rhie-Chow mass flows (slot order), net interior outflow and advective diagonal (kernel
 * massflow, zvcfd/fv/_cuda_fast.py:469-553; FastAssembler.massflow zvcfd/fv/fast.py:380-392);
 * writes mdot (E * nip), accumulates imbalance and adv (N). */
int zvfv_massflow(int kind, int stored, const int32_t *conn, int n_colours,
                  const int64_t *colour_offsets, const double *X, const double *geo,
                  const double *U, const double *P, const double *gradP, const double *dnode,
                  const double *snode, int nlev, double c1, const double *Uo1, const double *mo1,
                  double c2, const double *Uo2, const double *mo2, double rho, double *mdot,
                  double *imbalance, double *adv, void *stream);
/* zvfv_massflow plus, in the same element pass, the viscous part of the next momentum
 * diagonal from the same velocity (the terms of zvfv_diagonal without the advective part,
 * which adv already holds): the next iteration's a_P = vdiag + adv (accumulated into vdiag,
 * N). No reference counterpart: the reference launches its diag kernel separately
 * (zvcfd/fv/_cuda_fast.py:239-299). */
int zvfv_massflow_diag(int kind, int stored, const int32_t *conn, int n_colours,
                       const int64_t *colour_offsets, const double *X, const double *geo,
                       const double *U, const double *P, const double *gradP, const double *dnode,
                       const double *snode, int nlev, double c1, const double *Uo1,
                       const double *mo1, double c2, const double *Uo2, const double *mo2,
                       double rho, int rheo, double mu0, double muinf, double lam, double ca,
                       double cn, int transpose, int has_mut, const double *mut, double *mdot,
                       double *imbalance, double *adv, double *vdiag, void *stream);

/* Boundary rows, raw-row copy, Dirichlet with symmetric elimination, residual partials and
 * dimensionless row scaling (kernel finalise, zvcfd/fv/_cuda_bc.py:32-138, launched at
 * zvcfd/fv/solver.py:669-677). partial: zvfv_finalise_partials(n) rows of 8 doubles. */
int64_t zvfv_finalise_partials(int64_t n);
int zvfv_finalise(int64_t n, const int64_t *indptr, const int32_t *indices, const int64_t *dpos,
                  double *data, double *b, int has_time, const double *tdiag, const double *trhs,
                  const double *fV, const double *force, const double *inflow, const double *mb,
                  const double *wcons, const double *wonly, const double *wstab, int stokes,
                  const double *snl, const uint8_t *fixed, const uint8_t *known,
                  const double *vel, const double *pval, int eliminate, const int64_t *rawoff,
                  double *rawdata, double *rawb, const double *x, const double *aP,
                  const double *V, double rho, const double *scal, const double *lscale,
                  double *rs_out, double *partial, void *stream);

/* U, P <- x with change partials (kernel update, zvcfd/fv/_cuda_bc.py:140-175, launched at
 * zvcfd/fv/solver.py:900-902). partial: zvfv_update_partials(n) rows of 5 doubles. */
int64_t zvfv_update_partials(int64_t n);
int zvfv_update(int64_t n, const double *x, double *U, double *P, double *partial, void *stream);

/* Deterministic column folds of partial rows: ops[c] 0 sum, 1 max, 2 min (the host reductions
 * of zvcfd/fv/solver.py:903-908, on the device). */
int zvfv_fold(int64_t nrows, int width, const double *partial, const int32_t *ops, double *out,
              void *stream);

/* The state update of zvfv_update folded into stats[5] = {max |dU|, max |U|, max |dp|, min p,
 * max p}, allocating nothing. No counterpart in the reference: it serves callers that cannot
 * allocate device memory (a host program under a fixed memory budget, an outer loop that must
 * not call cudaMalloc/cudaFree between steps). Its partial rows live in a 2.5 MiB array of the
 * library that every GPU loading it holds until exit, which limits n to 1..16,777,216 nodes;
 * larger n returns ZVFV_BAD_ARGUMENT with a message. The first call on each device looks up
 * that array's device address (with the device current) and should come before any stream
 * capture; the address is kept with the device's current context and looked up again when
 * that context changes (after a device reset). Calls share the array: two calls that overlap on the GPU (different streams, no
 * ordering between them) race and give wrong statistics. Results equal zvfv_update followed by
 * zvfv_fold with ops {1, 1, 1, 2, 1} bit for bit. */
int zvfv_update_noalloc(int64_t n, const double *x, double *U, double *P, double *stats,
                        void *stream);

/* Wall shear stress (N, 3) at wall nodes from the wall integration points of their sub-faces
 * (WallGradientShear.__call__, zvcfd/fv/wall.py:113-137): node_ptr int64 (N+1) groups the
 * ips by node; per ip the owning element's nodes elem int32 (M, 8, -1 padded), shape
 * gradients grad (M, 8, 3), unit outward normal (M, 3) and area (M). */
int zvfv_wall_shear(int64_t n_nodes, const int64_t *node_ptr, const int32_t *elem,
                    const double *grad, const double *normal, const double *area,
                    const double *U, int rheo, double mu0, double muinf, double lam, double ca,
                    double cn, double *tau, void *stream);

/* ---------------------------------------------------------------- block-CSR products */

/* y = A x for 4x4 block CSR (kernel bsr_mv, zvcfd/fv/linear.py:47-61; BlockMatrix.matvec
 * :93-103 without the rank-one terms); lanes per block row: 4, 8, 16 or 32. */
int zvfv_bsr_spmv(int64_t n, const int64_t *indptr, const int32_t *indices, const double *data,
                  const double *x, double *y, int lanes, void *stream);
/* r = b - A x (the residual form of the same product) */
int zvfv_bsr_residual(int64_t n, const int64_t *indptr, const int32_t *indices,
                      const double *data, const double *x, const double *b, double *r, int lanes,
                      void *stream);
/* y = A x with FP32 blocks and vectors (the mixed-precision hierarchy's product; AmgX mode
 * dDFI's matrix precision, zvcfd/fv/linear.py:523-524, :853-854) */
int zvfv_bsr_spmv_f32(int64_t n, const int64_t *indptr, const int32_t *indices,
                      const float *data, const float *x, float *y, int lanes, void *stream);

/* The structure of A^T (built once per pattern): tptr int64 (n+1), per entry the row trow
 * int32 (ascending within a column) and the block index tperm int64 of A. Replaces the
 * reference's host transposes (BlockMatrix.to_scipy().T, zvcfd/fv/linear.py:123-135). */
int zvfv_bsr_transpose(int64_t n, int64_t nnz, const int64_t *indptr, const int32_t *indices,
                       int64_t *tptr, int32_t *trow, int64_t *tperm, void *stream);
/* y = A^T x (the discrete adjoint's product; lanes 8, 16 or 32) */
int zvfv_bsr_spmv_t(int64_t n, const int64_t *tptr, const int32_t *trow, const int64_t *tperm,
                    const double *data, const double *x, double *y, int lanes, void *stream);

/* ---------------------------------------------------------------- linear back end */

/* FGMRES preconditioned by one V-cycle of a device-built aggregation AMG: replaces the AmgX C
 * API the reference binds (AMGX_config_create / resources / matrix / solver handles,
 * zvcfd/fv/linear.py:728-739, :846-868, :905-955) and its own ACM (linear.py:328-518).
 * create: precision 0 FP64, 1 FP32 hierarchy; smoother 0 damped block Jacobi, 1 symmetric
 * multicolour block Gauss-Seidel (AmgX's MULTICOLOR_GS of the `gs` preset, linear.py:571-598),
 * 2 block-Jacobi-preconditioned Chebyshev polynomials of degree presweeps / postsweeps
 * (coarse_sweeps on a coarsest level too large for the dense inverse) on every level, over
 * [hi / cheb_ratio, hi], hi = 1.1 x the largest eigenvalue of D^-1 A estimated by power
 * iteration at each rebuild (AmgX's CHEBYSHEV smoother, which the reference's presets do not
 * select; no colouring, every step one pass over the level), 3 multicolour DILU on the
 * Gauss-Seidel levels (AmgX's MULTICOLOR_DILU of the `dilu` presets, linear.py:571-608: the
 * diagonal E_i = A_ii - sum over earlier colours A_ij E_j^-1 A_ji, one step
 * x += omega M^-1 (b - A x) with M = (E + L) E^-1 (E + U); the transposed cycle smooths those
 * levels by transposed Gauss-Seidel), 4 multicolour ILU(0) on the Gauss-Seidel levels (AmgX's
 * MULTICOLOR_ILU at sparsity level 0 of the `robust` preset: the colour-ordered level factored
 * colour by colour without fill, one step x += omega (LU)^-1 (b - A x); transposed cycle as for
 * DILU); strength 0 block norm (the ACM's), 1 pressure entry, 2 block norm averaged over both
 * directions of each coupling (the default of the Python back end: convection otherwise
 * stalls the pairwise matching). rebuild_every > 0 re-aggregates every that many
 * set-ups (the reference's ACM, linear.py:337-348); 0 keeps the aggregates until a solve fails
 * or needs more than 1.5 times (and 2 more than) the most iterations of the first three solves
 * after the last rebuild (after the reuse policy of its AmgX binding, linear.py:686-698,
 * :837-841, which takes the first solve alone). */
int zvfv_solver_create(void **handle, int precision, int smoother, int strength, int passes,
                       int presweeps, int postsweeps, double omega, int coarse_sweeps,
                       int max_levels, int rebuild_every, int restart);
/* structure on the first call (or when it changes), coefficients after: AMGX_matrix_upload_all
 * / AMGX_matrix_replace_coefficients + AMGX_solver_setup (zvcfd/fv/linear.py:846-868, :812-840) */
int zvfv_solver_setup(void *handle, int64_t n, int64_t nnzb, const int64_t *indptr,
                      const int32_t *indices, const double *data, void *stream);
/* x (in: x0, out: solution) to a reduction rtol of the initial residual, with n_lowrank
 * rank-one terms u w^T (BlockMatrix.lowrank, zvcfd/fv/linear.py:81-103): AMGX_solver_solve
 * (linear.py:920-955) / fgmres (linear.py:172-320). Synchronises once per Krylov step. */
int zvfv_solver_solve(void *handle, const double *b, double *x, double rtol, int maxiter,
                      int n_lowrank, const int64_t *const *u_idx, const double *const *u_val,
                      const int64_t *u_len, const int64_t *const *w_idx, const double *const *w_val,
                      const int64_t *w_len, int *iterations, double *residual, int *converged,
                      void *stream);
/* the adjoint solve A^T x = b (same arguments): FGMRES on A^T preconditioned by the V-cycle of
 * the same hierarchy on every level's transpose (A^T, D^-T, the dense inverse transposed);
 * no reference counterpart (the reference has no adjoint); builds the transposes on first use */
int zvfv_solver_solve_t(void *handle, const double *b, double *x, double rtol, int maxiter,
                        int n_lowrank, const int64_t *const *u_idx, const double *const *u_val,
                        const int64_t *u_len, const int64_t *const *w_idx,
                        const double *const *w_val, const int64_t *w_len, int *iterations,
                        double *residual, int *converged, void *stream);
/* FGMRES with one Krylov recurrence per segment of rows: the block-diagonal system of
 * independent instances (an ensemble's union). row_bounds: n_segments + 1 ascending host values
 * from 0 to n. The operator and the V-cycle act on all segments at once; inner products, norms,
 * Hessenberg columns, rotations and step lengths are per segment, and each segment stops at
 * rtol times its own initial residual (floor 1e-13 of its right-hand side's norm). The solve
 * ends when all have, or after maxiter Krylov steps (shared). active: n_segments host flags,
 * or null for all; a segment marked 0 takes no steps and keeps its initial guess (an instance
 * that has already converged). residuals, converged: n_segments host values. No reference
 * counterpart (the reference solves one problem per solver). Other arguments as
 * zvfv_solver_solve. */
int zvfv_solver_solve_segmented(void *handle, int n_segments, const int64_t *row_bounds,
                                const int *active, const double *b, double *x, double rtol,
                                int maxiter,
                                int n_lowrank, const int64_t *const *u_idx,
                                const double *const *u_val, const int64_t *u_len,
                                const int64_t *const *w_idx, const double *const *w_val,
                                const int64_t *w_len, int *iterations, double *residuals,
                                int *converged, void *stream);
/* z = one V-cycle applied to r (AMGX.vcycle, zvcfd/fv/linear.py:905-918) */
int zvfv_solver_vcycle(void *handle, const double *r, double *z, void *stream);
/* z = one V-cycle of the transposed hierarchy applied to r (A^T, D^-T, transposed Gauss-Seidel
 * sweeps, the dense coarsest inverse transposed on every level): the preconditioner of the
 * parameter adjoint's FGMRES; no reference counterpart (the reference has no adjoint) */
int zvfv_solver_vcycle_t(void *handle, const double *r, double *z, void *stream);
/* `passes` forward multicolour Gauss-Seidel passes on level `level` (a Gauss-Seidel level),
 * or with the Chebyshev smoother `passes` Chebyshev steps on any level but a dense coarsest
 * one, over that level's own work vectors (overwritten): the smoother kernel alone, for timing
 * (no reference counterpart: AmgX's smoother is internal to its V-cycle). */
int zvfv_solver_smooth(void *handle, int level, int passes, void *stream);
/* Hierarchy options beyond create (each takes effect at the next set-up, which rebuilds):
 *   "autotune" (0/1, default 0): after each rebuild, every level of 2048 rows or more times one
 *       smoothing pass at 8, 16 and 32 lanes per row and keeps the fastest (AmgX fixes its
 *       kernels' shapes; no reference counterpart); runs can then differ in the last bits;
 *   "gs_levels" (default 2): the finest levels smoothed by Gauss-Seidel, Jacobi below;
 *   "jacobi_sweeps" (default 2), "jacobi_omega" (default 0.7): the block-Jacobi smoothing of
 *       the levels below (the reference ACM's damped Jacobi, zvcfd/fv/linear.py:343, :480-502);
 *   "rebuild_ratio" (default 1.5): the adaptive rebuild threshold;
 *   "cheb_ratio" (> 1, default 10), "cheb_power" (>= 2, default 10): the Chebyshev interval's
 *       ratio and the power-iteration steps of its bound.
 * Unknown names or out-of-range values return ZVFV_BAD_ARGUMENT. */
int zvfv_solver_set_option(void *handle, const char *name, double value);
/* The value of an option above, or a counter: "rebuilds" (hierarchy builds so far), "setups",
 * or "cheb_lmax" (the finest level's largest-eigenvalue estimate of the Chebyshev smoother). */
int zvfv_solver_get_option(void *handle, const char *name, double *value);
/* hierarchy sizes (ACM.stats, zvcfd/fv/linear.py:515-518) */
int zvfv_solver_stats(void *handle, int max_levels, int *levels, int64_t *rows, int64_t *blocks);
/* one level's size and aggregates (agg: n int32 entries, or NULL) */
int zvfv_solver_level(void *handle, int level, int64_t *n, int64_t *nnzb, int64_t *n_coarse,
                      int32_t *agg, void *stream);
/* AMGX_solver_destroy / matrix / vector / resources (AMGX.close, zvcfd/fv/linear.py:870-903) */
int zvfv_solver_destroy(void *handle);

#ifdef __cplusplus
}
#endif

#endif /* ZVFV_B200_H */
