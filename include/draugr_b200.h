/*
 * draugr_b200.h - extensions of the B200 AMG library beyond the reference
 * C API (draugr_amg.h).  All functions return -1 on error and set
 * draugr_amg_last_error().  "Device pointers" are CUDA device addresses on
 * the device that was current when the hierarchy was set up.
 */
#ifndef DRAUGR_B200_H
#define DRAUGR_B200_H

#include <stdint.h>

#include "draugr_amg.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Hierarchy structure only, built on the CPU with nothing sent to a GPU
 * (inspection and export; no counterpart in the reference, whose setup
 * always produces a solver).  A later device call uploads it. */
int32_t draugr_b200_setup_host(int32_t n, int32_t nnz, const int32_t *rowptr,
                               const int32_t *colval, const double *nzval, int32_t config_handle,
                               int32_t index_base, int32_t allow_partial_resetup);

/* Number of AMG levels (the coarsest dense level not counted), as
 * length(hierarchy.levels) in src/types.jl:457-467. */
int32_t draugr_b200_num_levels(int32_t handle);

/* Sizes of level lvl (0-based): info[0] n, [1] nnz(A), [2] n_coarse,
 * [3] nnz(P), [4] smoother kind, [5] colours, [6] nnz(A*P) or -1,
 * [7] [8] [9] 1 if every row of A, P and Pᵀ is reduced by the row kernel
 * in column order (the reference's summation order), 0 if some row is
 * longer than the kernel's tile capacity.  info must hold 10 values.
 * lvl = -1: the coarsest level, info[0] n_c, [1] nnz of its CSR. */
int32_t draugr_b200_level_info(int32_t handle, int32_t lvl, int64_t *info);

/* Copy one array of level lvl (0-based indices) into out.  Integer arrays
 * (int32): A_rowptr A_colval P_rowptr P_colval T_offsets T_rows T_pnz
 * colors color_order color_offsets AP_rowptr AP_colval cf (the C/F
 * splitting, 1 / -1, of splitting-based coarsening), ilu_diag
 * ilu_fwd_order ilu_fwd_offsets ilu_bwd_order ilu_bwd_offsets (ILU(0)
 * levels), sgs_order sgs_offsets (serial Gauss-Seidel schedule), and for
 * lvl = -1 C_rowptr C_colval C_piv.  Double arrays: A_nzval P_nzval
 * R_nzval invdiag omega AP_nzval, cheb_coef cheb_v0 (Chebyshev), ilu_L
 * ilu_U (ILU(0) factors), spai1_M (SPAI(1)), and for lvl = -1 C_nzval
 * C_dense C_lu.  Values come from the device when the hierarchy lives there
 * (so they reflect resetups).  out = NULL returns the element count.
 * Returns the element count. */
int64_t draugr_b200_export(int32_t handle, int32_t lvl, const char *what, void *out,
                           int64_t capacity_elems);

/* Hierarchy summary in the layout of the reference's verbose setup print
 * (src/setup.jl:405-473).  Valid until the next call. */
const char *draugr_b200_summary(int32_t handle);

/* Every field of a parsed configuration as JSON, for inspection: the
 * coarsening and initial coarsening as objects (type, theta, interpolation
 * with its options, aggregation filtering, smoothed-aggregation omega),
 * then smoother, jacobi_omega, level and step counts, verbose,
 * max_row_sum, cycle ("v" or "w"), strength, coarse_solve_on_cpu and seed.
 * Type names are the lower-case names draugr_amg_config_from_json accepts.
 * The reference's Julia callers read the same fields from the config object
 * behind the handle (src/cfunction_interface.jl:165-221).  Valid until the
 * next call on this thread; NULL on an invalid handle. */
const char *draugr_b200_config_json(int32_t config_handle);

/* Device memory held by the hierarchy, in bytes (0 if host-only). */
int64_t draugr_b200_device_bytes(int32_t handle);

/* Solve / cycle on device vectors (no host copies).  Same semantics as
 * draugr_amg_solve / draugr_amg_cycle. */
int32_t draugr_b200_solve_device(int32_t handle, int32_t n, double *x_dev, const double *b_dev,
                                 int32_t config_handle, double tol, int32_t maxiter);
int32_t draugr_b200_cycle_device(int32_t handle, int32_t n, double *x_dev, const double *b_dev,
                                 int32_t config_handle);

/* r = b - A x for the finest matrix of the hierarchy and ||r||_2 (device
 * vectors of length n; rnorm is a host pointer, may be NULL).  The residual
 * of amg_solve!'s convergence test (src/cycle.jl:138-139). */
int32_t draugr_b200_residual_device(int32_t handle, int32_t n, const double *x_dev,
                                    const double *b_dev, double *r_dev, double *rnorm);

/* The residual above for callers that cannot allocate device memory: hosts
 * whose own pool hands out every byte of device memory (a framework's
 * caching allocator, a solver that reserves all memory at start-up) and so
 * cannot let a library call cudaMalloc.  No counterpart in the reference.
 * All arrays belong to the caller and are device pointers: the n x n CSR
 * matrix (0-based rowptr[n+1], colval[nnz], nzval[nnz]), x and b (length n)
 * and the output r = b - A x (length n); rnorm (host pointer, may be NULL)
 * receives ||r||_2.  stream: a cudaStream_t, NULL for the default stream.
 * Nothing is allocated: the reduction's scratch is a static device array of
 * 16386 doubles (128 KB, held by every GPU that loads the library until the
 * process exits), so n is limited to 4,194,304 rows (16384 blocks of 256
 * rows); larger n is rejected with an error.  The first call on a device
 * looks up the scratch's device address (cudaGetSymbolAddress); make that
 * first call before any stream capture.  All calls share the scratch, so
 * calls that overlap on the GPU (different streams or threads) race.  Every
 * call copies ||r||_2 back to the host and synchronises `stream` before it
 * returns.  Rows are summed in column order with separately rounded
 * products and sums, as the reference's residual_kernel! does, so r equals
 * that kernel's result bit for bit.  Returns 0 or -1. */
int32_t draugr_b200_residual_noalloc(int32_t n, int32_t nnz, const int32_t *rowptr,
                                     const int32_t *colval, const double *nzval, const double *x,
                                     const double *b, double *r, double *rnorm, void *stream);

/* Partial resetup from new values of the finest matrix already on the
 * device (same pattern as at setup), nnz entries.  The first partial
 * resetup of a hierarchy also records its Galerkin product lists (8 bytes
 * per product, kept while under half of the free device memory), which
 * make later resetups faster.  A resetup synchronises its stream and may
 * allocate: do not capture it in a CUDA graph.  Replaces the device-side
 * part of amg_resetup! (src/resetup.jl:20-45); the reference copies the
 * values to the host first (ext/DraugrCUDAExt.jl:49). */
int32_t draugr_b200_resetup_values_device(int32_t handle, int64_t nnz, const double *nzval_dev);

/* Precision of the Galerkin products of later partial resetups: the first
 * fp64_levels products from the top (the ones that form levels 2 ..
 * fp64_levels + 1) in FP64, the rest in FP32 on the FP32 copies of A, P and
 * Pᵀ, each FP32-computed level's FP64 copy being its FP32 values widened.
 * Negative (the default): every product in FP64, as the reference.  The
 * smoother diagonals and the coarsest LU are always formed in FP64.  The
 * reference's resetup computes every level in the matrix's own precision
 * (src/resetup.jl:36-41). */
int32_t draugr_b200_set_resetup_precision(int32_t handle, int32_t fp64_levels);

/* The Galerkin product of level lvl computed on the host by the setup's
 * numeric product (A*P, then Pᵀ(AP), each entry accumulated in the same
 * order as the device's partial resetup): a_vals holds new values of level
 * lvl's matrix (nnz_in, its pattern), ac_vals receives the next level's
 * values (nnz_out, its pattern).  Needs a hierarchy set up with
 * allow_partial_resetup = 1.  For checking device resetups; the reference's
 * counterpart is galerkin_product! on the CPU backend
 * (src/galerkin.jl:194-222), which sums the same products per entry in its
 * triple map's order. */
int32_t draugr_b200_galerkin_host(int32_t handle, int32_t lvl, int64_t nnz_in, const double *a_vals,
                                  int64_t nnz_out, double *ac_vals);

/* Conjugate gradients preconditioned by one AMG cycle per iteration, until
 * ||b - A x|| / ||b|| < tol.  precision 0: FP64 cycle.  precision 1: cycle
 * on FP32 copies of the hierarchy with FP64 outer residual, products with A,
 * dot products and updates.  x holds the initial guess.  relres (may be
 * NULL) receives the final relative residual.  Returns iterations or -1.
 * The reference has no Krylov solver of its own (it hands amg_cycle! to
 * LinearSolve.jl through ldiv!, src/preconditioner.jl:76-102). */
int32_t draugr_b200_pcg(int32_t handle, int32_t n, double *x, const double *b,
                        int32_t config_handle, double tol, int32_t maxiter, int32_t precision,
                        double *relres);
int32_t draugr_b200_pcg_device(int32_t handle, int32_t n, double *x_dev, const double *b_dev,
                               int32_t config_handle, double tol, int32_t maxiter,
                               int32_t precision, double *relres);

/* Flexible GMRES(restart), right-preconditioned by one AMG cycle per
 * iteration, until ||b - A x|| / ||b|| < tol, for symmetric and
 * nonsymmetric systems.  precision 0: FP64 cycle; precision 1: FP32 cycle
 * (FP32 copies of the hierarchy) with the Arnoldi basis, Gram-Schmidt
 * products, least-squares update and residuals in FP64.  restart: 1 to 63
 * basis vectors before a restart from the true residual.  x holds the
 * initial guess; relres (may be NULL) receives the final true relative
 * residual.  Returns iterations or -1.  The reference hands amg_cycle! to
 * LinearSolve.jl's Krylov methods as a preconditioner instead
 * (ext/DraugrLinearSolveExt.jl:35-37, src/preconditioner.jl:76-102). */
int32_t draugr_b200_fgmres(int32_t handle, int32_t n, double *x, const double *b, int32_t config_handle,
                           double tol, int32_t maxiter, int32_t restart, int32_t precision, double *relres);
int32_t draugr_b200_fgmres_device(int32_t handle, int32_t n, double *x_dev, const double *b_dev,
                                  int32_t config_handle, double tol, int32_t maxiter, int32_t restart,
                                  int32_t precision, double *relres);

/* Iterative refinement: the residual r = b - A x is formed in FP64, the
 * correction equation A d = r is solved to inner_tol (relative to ||r||) by
 * AMG-PCG (inner_method 0) or FGMRES(30) (inner_method 1) with an FP64
 * (precision 0) or FP32 (precision 1) cycle, and x += d, until
 * ||b - A x|| / ||b|| < tol or max_outer steps.  relres (may be NULL): the
 * final FP64 relative residual; inner_iters (may be NULL): the inner
 * iterations in all.  Returns the refinement steps or -1.  No counterpart
 * in the reference (see draugr_b200_fgmres). */
int32_t draugr_b200_refine(int32_t handle, int32_t n, double *x, const double *b, int32_t config_handle,
                           double tol, int32_t max_outer, double inner_tol, int32_t inner_maxiter,
                           int32_t inner_method, int32_t precision, double *relres, int32_t *inner_iters);
int32_t draugr_b200_refine_device(int32_t handle, int32_t n, double *x_dev, const double *b_dev,
                                  int32_t config_handle, double tol, int32_t max_outer, double inner_tol,
                                  int32_t inner_maxiter, int32_t inner_method, int32_t precision,
                                  double *relres, int32_t *inner_iters);

/* Many independent systems solved as one batch.  batch_setup merges the
 * hierarchies of `nsys` systems (handles from draugr_amg_setup, each with at
 * least one AMG level, Jacobi, l1-Jacobi or SPAI(0) smoothing on every
 * level, the same smoother and weight where they share a level) level by
 * level into block-diagonal matrices, on the current device, and returns a
 * new hierarchy handle (free it with draugr_amg_free; the systems' own
 * handles stay valid).  The batch's vectors hold the systems' vectors one
 * after the other; batch_offsets writes the nsys + 1 row offsets (may be
 * NULL) and returns nsys.  batch_pcg_device runs conjugate gradients on
 * every system at once with the AMG V-cycle of the merged hierarchy as
 * preconditioner (precision 0: FP64, 1: FP32 cycle in the FP64 iteration):
 * each cycle stage, dot product and update is one launch for all systems,
 * every system keeps its own step sizes and stops changing once
 * ||b_s - A_s x_s|| < tol ||b_s||, and one iteration runs as a CUDA graph.
 * iters, relres (nsys entries each, may be NULL): per-system iterations and
 * final FP64 relative residuals.  Returns the largest iteration count, or
 * -1.  The reference solves one system per call; a caller loops over them
 * (src/cycle.jl:110-160). */
int32_t draugr_b200_batch_setup(int32_t nsys, const int32_t *handles);
int32_t draugr_b200_batch_offsets(int32_t handle, int64_t *offsets);
int32_t draugr_b200_batch_pcg_device(int32_t handle, int32_t n, double *x_dev, const double *b_dev,
                                     int32_t config_handle, double tol, int32_t maxiter, int32_t precision,
                                     int32_t *iters, double *relres);

/* BiCGStab preconditioned (on the right) by one AMG cycle per
 * application, until ||b - M x|| / ||b|| < tol, for nonsymmetric systems.
 * transpose 0: M = A.  transpose 1: M = A^T, the adjoint system of a
 * gradient computation, with cycles on the transposed hierarchy (A^T on
 * every level, the same P and P^T, the transposed coarsest LU solve);
 * every level must use Jacobi, l1-Jacobi or SPAI(0) smoothing.
 * precision 0: FP64 cycle; precision 1: FP32 cycle (FP32 copies of the
 * hierarchy, or of the transposed hierarchy) with the BiCGStab vectors,
 * products with M and dot products in FP64.  x holds the initial guess;
 * relres (may be NULL) receives the final true relative residual.  Returns
 * iterations or -1.  No counterpart in the reference, which has neither a
 * nonsymmetric Krylov solver nor adjoints. */
int32_t draugr_b200_bicgstab(int32_t handle, int32_t n, double *x, const double *b,
                             int32_t config_handle, double tol, int32_t maxiter,
                             int32_t transpose, int32_t precision, double *relres);
int32_t draugr_b200_bicgstab_device(int32_t handle, int32_t n, double *x_dev, const double *b_dev,
                                    int32_t config_handle, double tol, int32_t maxiter,
                                    int32_t transpose, int32_t precision, double *relres);

/* Conjugate gradients for k (1..32) right-hand sides of the same matrix
 * at once: X and B are device arrays of n x k doubles, row-major (column c
 * of row i at i*k + c); X holds the initial guesses.  Each product with a
 * level matrix serves all k columns in one pass over the matrix.
 * precision as for draugr_b200_pcg; every level must use Jacobi, l1-Jacobi or SPAI(0)
 * smoothing.  iters and relres (host arrays of k entries, may be NULL)
 * receive each column's iterations and final true relative residual.
 * Returns the largest iteration count or -1.  The first call for a given k
 * and precision on a hierarchy times the launch shapes of the cycle's
 * products (threads per row, blocks per SM) and keeps the fastest; results
 * do not depend on the shapes.  The environment variable
 * DRAUGR_B200_BLOCK_TUNE, read at each call: 0 keeps the default shapes,
 * 2/4/8/16 forces that many threads per row.  No counterpart in the
 * reference. */
int32_t draugr_b200_pcg_block_device(int32_t handle, int32_t n, int32_t k, double *X_dev,
                                     const double *B_dev, int32_t config_handle, double tol,
                                     int32_t maxiter, int32_t precision, int32_t *iters,
                                     double *relres);

/* Gradient of a loss L(x), x = A^-1 b, with respect to the nonzeros of the
 * finest matrix: grad[k] = -lambda_i x_j for nonzero k = (i, j) in CSR
 * order, where lambda = A^-T dL/dx (device vectors; grad has nnz entries).
 * dL/db is lambda itself.  No counterpart in the reference. */
int32_t draugr_b200_nz_gradient_device(int32_t handle, int32_t n, const double *x_dev,
                                       const double *lambda_dev, double *grad_dev);

/* One operation on one level, host arrays in and out (kernel-level checks).
 * op 0: y = A x (in1 = x)            op 1: r = b - A x (in1 = x, in2 = b)
 * op 2: `steps` smoother sweeps from x (in1) for rhs b (in2)
 * op 3: b_c = Pᵀ r (in1 = r)         op 4: x + P x_c (in1 = x, in2 = x_c)
 * op 5: coarsest solve (in1 = b_c; lvl ignored)
 * op 6: first Jacobi step from zero fused with the residual (in1 = b);
 *       out holds x1 then r (2n values)
 * precision 0 = FP64, 1 = FP32 kernels (inputs rounded to FP32). */
int32_t draugr_b200_level_op(int32_t handle, int32_t lvl, int32_t op, int32_t precision,
                             const double *in1, const double *in2, double *out, int32_t steps);

/* Mean device time of `reps` launches of a level kernel (op 2: one Jacobi
 * sweep, op 0: SpMV, 3: restriction, 4: prolongation, 6: first sweep from
 * zero fused with the residual), or of the V(1,1) cycle from level lvl >= 1
 * down from a zero guess (op 8, the coarse tail included), measured with
 * CUDA events on the hierarchy's stream. */
int32_t draugr_b200_time_level_op(int32_t handle, int32_t lvl, int32_t op, int32_t precision,
                                  int32_t reps, float *ms_per_launch);

/* Run this hierarchy's work on the caller's CUDA stream (a cudaStream_t;
 * NULL returns to the library's own non-blocking stream).  Entry points
 * still return only after their work on that stream is complete. */
int32_t draugr_b200_set_stream(int32_t handle, void *stream);

/* Number of CUDA kernels this library has launched in the process so far
 * (each launch of a captured CUDA graph adds the kernels it contains). */
int64_t draugr_b200_kernel_launches(void);

/* Test hook, no counterpart in the reference: the number of polls a row
 * kernel makes on a tile's copy (an mbarrier wait) before it gives up,
 * flags the timeout and returns; the entry point that launched it then
 * returns -1 with "timed out" in draugr_amg_last_error.  A negative value
 * restores the default (2^22).  0 makes every row kernel give up at once,
 * which is how the timeout path is tested without a stuck copy. */
void draugr_b200_set_tile_wait_limit(int32_t polls);

#ifdef __cplusplus
}
#endif

#endif /* DRAUGR_B200_H */
