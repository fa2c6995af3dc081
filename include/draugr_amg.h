/*
 * draugr_amg.h - C API of the B200 AMG library (libdraugr_b200.so).
 *
 * Drop-in for the C API of Draugr.jl (c_api/draugr_amg.h): the same symbols,
 * argument meanings, return codes and error reporting, so a C, C++ or
 * Fortran host linked against Draugr's PackageCompiler library can link
 * against this one instead.  Setup builds the hierarchy structure on the CPU
 * and uploads it to the current CUDA device; solve, cycle and the partial
 * resetup run on the device.  Extensions (device pointers, AMG-PCG, mixed
 * precision, hierarchy export) are declared in draugr_b200.h.
 *
 * Index arrays are int32 with a selectable base (0 or 1); values are double.
 */
#ifndef DRAUGR_AMG_H
#define DRAUGR_AMG_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Runtime lifecycle.  Replaces init_julia / shutdown_julia, which
 * PackageCompiler adds to the reference library (c_api/draugr_amg.h:30,36).
 * Here there is no runtime to start, so both are no-ops kept for link
 * compatibility. */
void init_julia(int argc, char **argv);
void shutdown_julia(int retcode);

/* Message of the last failed call, "" if none.  Valid until the next call.
 * Replaces draugr_amg_last_error (c_api/draugr_amg.h:49,
 * src/cfunction_interface.jl:18-28). */
const char *draugr_amg_last_error(void);

/* Configuration from a JSON object; NULL or "{}" gives the defaults of
 * AMGConfig() (HMIS θ=0.5 with extended+i interpolation, l1 colored
 * Gauss-Seidel, V(1,1), max_coarse_size 50).  Keys as in the reference
 * (coarsening, interpolation, smoother, strength, cycle, theta, max_levels,
 * max_coarse_size, pre_smoothing_steps, post_smoothing_steps, verbose,
 * jacobi_omega, max_row_sum, coarse_solve_on_cpu, initial_coarsening,
 * initial_coarsening_levels); unknown keys are ignored, string values are
 * case-insensitive, numbers may be given as strings.  One extra key, "seed",
 * seeds the random measures of PMIS/HMIS.  Returns a handle > 0 or -1.
 * Replaces draugr_amg_config_from_json (c_api/draugr_amg.h:86,
 * src/cfunction_interface.jl:178-221). */
int32_t draugr_amg_config_from_json(const char *json_str);

/* Build a hierarchy from an n x n CSR matrix (arrays are copied).
 * index_base 0 or 1.  allow_partial_resetup = 1 keeps the Galerkin maps for
 * draugr_amg_resetup(partial=1).  Returns a hierarchy handle > 0 or -1.
 * Replaces draugr_amg_setup (c_api/draugr_amg.h:106-111,
 * src/cfunction_interface.jl:242-270). */
int32_t draugr_amg_setup(int32_t n, int32_t nnz, const int32_t *rowptr, const int32_t *colval,
                         const double *nzval, int32_t config_handle, int32_t index_base,
                         int32_t allow_partial_resetup);

/* New coefficients.  partial = 1: same sparsity pattern (checked), values
 * copied to the device, Galerkin products, smoother diagonals and the
 * coarsest LU recomputed on the device.  partial = 0: the hierarchy is
 * rebuilt.  Returns 0 or -1.  Replaces draugr_amg_resetup
 * (c_api/draugr_amg.h:134-140, src/cfunction_interface.jl:302-330). */
int32_t draugr_amg_resetup(int32_t handle, int32_t n, int32_t nnz, const int32_t *rowptr,
                           const int32_t *colval, const double *nzval, int32_t config_handle,
                           int32_t index_base, int32_t partial, int32_t allow_partial_resetup);

/* Stationary AMG iteration until ||b - A x|| / ||b|| < tol; x (host, length
 * n) is the initial guess and receives the solution.  The cycle options
 * (V/W, smoothing steps, verbose) come from config_handle.  Returns the
 * number of cycles (maxiter if not converged) or -1.  Replaces
 * draugr_amg_solve (c_api/draugr_amg.h:159-162,
 * src/cfunction_interface.jl:361-386). */
int32_t draugr_amg_solve(int32_t handle, int32_t n, double *x, const double *b,
                         int32_t config_handle, double tol, int32_t maxiter);

/* One cycle improving x in place for A x = b (x is not zeroed).  Returns 0
 * or -1.  Replaces draugr_amg_cycle (c_api/draugr_amg.h:170-172,
 * src/cfunction_interface.jl:396-420). */
int32_t draugr_amg_cycle(int32_t handle, int32_t n, double *x, const double *b,
                         int32_t config_handle);

/* Release a hierarchy / a configuration.  0, or -1 for an unknown handle.
 * Replace draugr_amg_free / draugr_amg_config_free (c_api/draugr_amg.h:182,
 * :188; src/cfunction_interface.jl:435-476). */
int32_t draugr_amg_free(int32_t handle);
int32_t draugr_amg_config_free(int32_t handle);

#ifdef __cplusplus
}
#endif

#endif /* DRAUGR_AMG_H */
