/*
 * ORACLE — test infrastructure, not part of the product.
 *
 * A plain-C restatement of the arithmetic of Draugr.jl's AMG solve phase and
 * numeric resetup, used only by the tests, by __graft_entry__.smoke() and by
 * bench.py's CPU-baseline / reference arms to check and to time against.  It
 * follows the reference's loops in order (sums accumulated left to right,
 * products rounded separately), so for a given hierarchy it reproduces what
 * the reference computes on its CPU backend up to the order of dot-product
 * reductions.  Each function cites the reference routine it restates
 * (paths relative to the Draugr.jl repository).
 *
 * The reference is Julia and cannot run here; this restatement is pinned
 * against the reference's own test assertions (tests/test_oracle_pins.py):
 * restriction = explicit Pᵀr, Galerkin = explicit PᵀAP, Jacobi invdiag 0.5,
 * l1 invdiag 0.25, colouring validity, convergence thresholds.
 *
 * Row loops run under OpenMP with a static schedule in chunks of 64 rows,
 * as the reference's KernelAbstractions CPU(static=true) backend with
 * workgroup size 64 (src/Draugr.jl:10, src/setup.jl:48).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define CHUNK 64

/* ------------------------------------------------------------------ types */
typedef struct {
  int n, nc;
  const int *A_rp, *A_ci;
  double *A_v;
  const int *P_rp, *P_ci;
  const double *P_v;
  const int *T_off, *T_rows, *T_pnz;
  int smoother; /* 0 jacobi, 1 colored_gs, 2 serial_gs, 3 spai0, 4 spai1, 5 l1_jacobi,
                   6 l1_colored_gs, 7 l1_serial_gs, 8 chebyshev, 9 ilu0, 10 serial_ilu0 */
  double omega;
  double *invd;
  int ncolors;
  const int *color_off, *color_order;
  double *r, *xc, *bc, *tmp;
  /* Galerkin restriction map (orc_coarse_sparsity) for the resetup */
  const int64_t *nz_off;
  const int *tpi, *tai, *tpj;
  /* Chebyshev: inner steps, normalised power-iteration start vector,
   * coefficient table (2 * degree), update direction */
  int cheb_degree;
  const double *cheb_v0;
  double *cheb_coef, *cheb_d;
  /* ILU(0): diagonal positions and factors on A's pattern */
  const int *ilu_diag;
  double *ilu_L, *ilu_U;
  /* SPAI(1): M on A's pattern */
  double *spai1_M;
} olevel;

typedef struct {
  int nlevels;
  olevel *lv;
  int nc;
  double *dense; /* column-major nc x nc */
  double *lu;
  int *piv;
  double *cx, *cb;
  double *solve_r;
  double *coarse_v; /* values of the coarsest CSR when nlevels == 0 */
  const int *coarse_rp, *coarse_ci;
} ohier;

/* ------------------------------------------------------ CSR kernels */
/* y = A x : csr_mul_kernel!, src/csr_matrix.jl:150-159 */
void orc_spmv(int n, const int *rp, const int *ci, const double *v, const double *x, double *y) {
#pragma omp parallel for schedule(static, CHUNK)
  for (int i = 0; i < n; ++i) {
    double s = 0.0;
    for (int k = rp[i]; k < rp[i + 1]; ++k) s += v[k] * x[ci[k]];
    y[i] = s;
  }
}

/* r = b - A x : residual_kernel!, src/cycle.jl:32-43 */
void orc_residual(int n, const int *rp, const int *ci, const double *v, const double *x,
                  const double *b, double *r) {
#pragma omp parallel for schedule(static, CHUNK)
  for (int i = 0; i < n; ++i) {
    double ax = 0.0;
    for (int k = rp[i]; k < rp[i + 1]; ++k) ax += v[k] * x[ci[k]];
    r[i] = b[i] - ax;
  }
}

/* invdiag_kernel!, src/smoothers.jl:47-63 */
void orc_invdiag(int n, const int *rp, const int *ci, const double *v, double *invd) {
#pragma omp parallel for schedule(static, CHUNK)
  for (int i = 0; i < n; ++i) {
    double d = 0.0, rn = 0.0;
    for (int k = rp[i]; k < rp[i + 1]; ++k) {
      rn += fabs(v[k]);
      if (ci[k] == i) d = v[k];
    }
    double thr = 2.220446049250313e-16 * (rn > 1.0 ? rn : 1.0);
    invd[i] = fabs(d) > thr ? 1.0 / d : 0.0;
  }
}

/* l1_invdiag_kernel!, src/smoothers.jl:816-827 */
void orc_l1_invdiag(int n, const int *rp, const double *v, double *invd) {
#pragma omp parallel for schedule(static, CHUNK)
  for (int i = 0; i < n; ++i) {
    double l1 = 0.0;
    for (int k = rp[i]; k < rp[i + 1]; ++k) l1 += fabs(v[k]);
    invd[i] = l1 > 2.220446049250313e-16 ? 1.0 / l1 : 0.0;
  }
}

/* spai0_kernel!, src/smoothers.jl:524-538: m_i = a_ii / sum_j a_ij^2 (the
 * last diagonal entry of the row, 0 for a zero row) */
void orc_spai0(int n, const int *rp, const int *ci, const double *v, double *m) {
#pragma omp parallel for schedule(static, CHUNK)
  for (int i = 0; i < n; ++i) {
    double d = 0.0, s = 0.0;
    for (int k = rp[i]; k < rp[i + 1]; ++k) {
      s += v[k] * v[k];
      if (ci[k] == i) d = v[k];
    }
    m[i] = s > 0.0 ? d / s : 0.0;
  }
}

/* smooth!(::SPAI0Smoother): spai0_smooth_kernel! with the tmp/x ping-pong
 * and the copy back on odd step counts, src/smoothers.jl:546-583 */
void orc_spai0_smooth(int n, const int *rp, const int *ci, const double *v, const double *m,
                      double *x, const double *b, int steps, double *tmp) {
  double *src = x, *dst = tmp;
  for (int s = 0; s < steps; ++s) {
#pragma omp parallel for schedule(static, CHUNK)
    for (int i = 0; i < n; ++i) {
      double ri = b[i];
      for (int k = rp[i]; k < rp[i + 1]; ++k) ri -= v[k] * src[ci[k]];
      dst[i] = src[i] + m[i] * ri;
    }
    double *t = src;
    src = dst;
    dst = t;
  }
  if (steps & 1) memcpy(x, tmp, (size_t)n * sizeof(double));
}

/* _estimate_spectral_radius, src/smoothers.jl:869-887: `niter` power steps
 * w = (A v) .* invdiag (csr_mul_kernel! sums from zero), lambda = ||w||,
 * v = w / lambda when lambda > eps; v holds the normalised start vector and
 * is overwritten, w is work.  Returns the last lambda.  (norm is a plain
 * sum of squares here; the reference's BLAS nrm2 scales, which changes
 * only the last bits.) */
double orc_spectral_radius(int n, const int *rp, const int *ci, const double *a, const double *invd,
                           double *v, int niter, double *w) {
  double lam = 1.0;
  for (int it = 0; it < niter; ++it) {
#pragma omp parallel for schedule(static, CHUNK)
    for (int i = 0; i < n; ++i) {
      double s = 0.0;
      for (int k = rp[i]; k < rp[i + 1]; ++k) s += a[k] * v[ci[k]];
      w[i] = s * invd[i];
    }
    double ss = 0.0;
    for (int i = 0; i < n; ++i) ss += w[i] * w[i];
    lam = sqrt(ss);
    if (lam > 2.220446049250313e-16)
      for (int i = 0; i < n; ++i) v[i] = w[i] / lam;
  }
  return lam;
}

/* Chebyshev bounds and recurrence coefficients, build_chebyshev_smoother
 * (src/smoothers.jl:895-910: lambda_max = 1.1 rho, lambda_min =
 * lambda_max / 30) and smooth! (:947-986): coef[0] = 1/theta, coef[1] = 0,
 * then scale_r, scale_d of inner step k at [2k], [2k+1]. */
void orc_cheb_coef(double rho, int degree, double *coef) {
  double lmax = 1.1 * rho;
  double lmin = lmax / 30.0;
  double theta = (lmax + lmin) / 2.0;
  double delta = (lmax - lmin) / 2.0;
  coef[0] = 1.0 / theta;
  coef[1] = 0.0;
  double s_old = theta / delta;
  for (int k = 1; k < degree; ++k) {
    double s_new = 1.0 / (2.0 * theta / delta - s_old);
    coef[2 * k] = 2.0 * s_new / delta;
    coef[2 * k + 1] = s_new * s_old;
    s_old = s_new;
  }
}

/* residual_kernel_smoother!, src/smoothers.jl:988-999: Ax summed from zero,
 * then r = b - Ax */
static void cheb_residual(int n, const int *rp, const int *ci, const double *a, const double *x,
                          const double *b, double *r) {
#pragma omp parallel for schedule(static, CHUNK)
  for (int i = 0; i < n; ++i) {
    double s = 0.0;
    for (int k = rp[i]; k < rp[i + 1]; ++k) s += a[k] * x[ci[k]];
    r[i] = b[i] - s;
  }
}

/* smooth!(::ChebyshevSmoother), src/smoothers.jl:947-986, with
 * chebyshev_init_kernel! / chebyshev_iter_kernel! (:924-940): per step, the
 * residual of the whole vector, then d = invdiag r / theta, x += d; then
 * degree - 1 times the residual, d = scale_r invdiag r + scale_d d, x += d. */
void orc_chebyshev(int n, const int *rp, const int *ci, const double *a, const double *invd,
                   const double *coef, int degree, double *x, const double *b, int steps, double *r,
                   double *d) {
  for (int s = 0; s < steps; ++s) {
    cheb_residual(n, rp, ci, a, x, b, r);
    for (int i = 0; i < n; ++i) {
      d[i] = invd[i] * r[i] * coef[0];
      x[i] += d[i];
    }
    for (int k = 1; k < degree; ++k) {
      cheb_residual(n, rp, ci, a, x, b, r);
      for (int i = 0; i < n; ++i) {
        d[i] = coef[2 * k] * invd[i] * r[i] + coef[2 * k + 1] * d[i];
        x[i] += d[i];
      }
    }
  }
}

/* _ilu0_factorize!, src/smoothers.jl:1016-1080: U = A's values, L = 0; row
 * by row, for each k < i in row i: skip (L = U = 0) when |U_kk| is below
 * eps max(1, sum_k |a_kj|); l_ik = U_ik / U_kk clamped to magnitude 1e8;
 * U_ij -= l_ik U_kj for j > k where (i, j) exists (_find_nz_in_row's
 * binary search); then the diagonal safeguard U_ii = eps max(1, sum |a_ij|)
 * when |U_ii| is below it. */
void orc_ilu0_factor(int n, const int *rp, const int *ci, const double *a, const int *diag,
                     double *L, double *U) {
  const double eps = 2.220446049250313e-16;
  int nnz = rp[n];
  double *rn = (double *)malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
  for (int k = 0; k < nnz; ++k) {
    U[k] = a[k];
    L[k] = 0.0;
  }
  for (int i = 0; i < n; ++i) {
    double s = 0.0;
    for (int k = rp[i]; k < rp[i + 1]; ++k) s += fabs(a[k]);
    rn[i] = s;
  }
  for (int i = 0; i < n; ++i) {
    for (int nz = rp[i]; nz < diag[i]; ++nz) {
      int k = ci[nz];
      double ukk = U[diag[k]];
      if (fabs(ukk) < eps * (rn[k] > 1.0 ? rn[k] : 1.0)) {
        L[nz] = 0.0;
        U[nz] = 0.0;
        continue;
      }
      double lik = U[nz] / ukk;
      double nl = fabs(lik);
      if (nl > 1e8) lik = lik * (1e8 / nl);
      L[nz] = lik;
      U[nz] = 0.0;
      for (int nk = diag[k] + 1; nk < rp[k + 1]; ++nk) {
        int j = ci[nk], lo = rp[i], hi = rp[i + 1] - 1, at = -1;
        while (lo <= hi) {
          int mid = (lo + hi) >> 1;
          if (ci[mid] == j) { at = mid; break; }
          if (ci[mid] < j) lo = mid + 1;
          else hi = mid - 1;
        }
        if (at >= 0) U[at] -= lik * U[nk];
      }
    }
    double thr = eps * (rn[i] > 1.0 ? rn[i] : 1.0);
    if (fabs(U[diag[i]]) < thr) U[diag[i]] = thr;
  }
  free(rn);
}

/* smooth!(::SerialILU0Smoother), src/smoothers.jl:1143-1205 (the level-
 * scheduled ILU0Smoother computes the same values): per step the residual
 * (Ax summed from zero), forward substitution in row order, backward
 * substitution in reverse row order with t_i / U_ii (0 when |U_ii| <=
 * eps), then x += t where t is finite. */
void orc_ilu0_smooth(int n, const int *rp, const int *ci, const double *a, const int *diag,
                     const double *L, const double *U, double *x, const double *b, int steps, double *t) {
  for (int s = 0; s < steps; ++s) {
    cheb_residual(n, rp, ci, a, x, b, t);
    for (int i = 0; i < n; ++i)
      for (int nz = rp[i]; nz < diag[i]; ++nz) t[i] -= L[nz] * t[ci[nz]];
    for (int i = n - 1; i >= 0; --i) {
      for (int nz = diag[i] + 1; nz < rp[i + 1]; ++nz) t[i] -= U[nz] * t[ci[nz]];
      double u = U[diag[i]];
      t[i] = fabs(u) > 2.220446049250313e-16 ? t[i] / u : 0.0;
    }
    for (int i = 0; i < n; ++i)
      if (isfinite(t[i])) x[i] += t[i];
  }
}

/* G m = r for the small symmetric Gram matrix of SPAI(1) (row-major G,
 * overwritten): upper Cholesky (potf2 order), else partial-pivoting LU,
 * else m = 0 (the dense solve of Julia's `\` on a symmetric matrix) */
static void spai1_solve(int k, double *G, const double *r, double *m) {
  double *G2 = (double *)malloc(sizeof(double) * (size_t)k * k);
  memcpy(G2, G, sizeof(double) * (size_t)k * k);
  int ok = 1;
  for (int j = 0; j < k && ok; ++j) {
    double s = G[j * k + j];
    for (int t = 0; t < j; ++t) s -= G[t * k + j] * G[t * k + j];
    if (!(s > 0.0)) { ok = 0; break; }
    double u = sqrt(s);
    G[j * k + j] = u;
    for (int l = j + 1; l < k; ++l) {
      double v = G[j * k + l];
      for (int t = 0; t < j; ++t) v -= G[t * k + j] * G[t * k + l];
      G[j * k + l] = v / u;
    }
  }
  if (ok) {
    for (int j = 0; j < k; ++j) {
      double v = r[j];
      for (int t = 0; t < j; ++t) v -= G[t * k + j] * m[t];
      m[j] = v / G[j * k + j];
    }
    for (int j = k - 1; j >= 0; --j) {
      double v = m[j];
      for (int t = j + 1; t < k; ++t) v -= G[j * k + t] * m[t];
      m[j] = v / G[j * k + j];
    }
  } else {
    for (int j = 0; j < k; ++j) m[j] = r[j];
    for (int j = 0; j < k && !ok; ++j) {
      int p = j;
      for (int i = j + 1; i < k; ++i)
        if (fabs(G2[i * k + j]) > fabs(G2[p * k + j])) p = i;
      if (G2[p * k + j] == 0.0) { ok = -1; break; }
      if (p != j) {
        for (int c = 0; c < k; ++c) { double t = G2[p * k + c]; G2[p * k + c] = G2[j * k + c]; G2[j * k + c] = t; }
        double t = m[p]; m[p] = m[j]; m[j] = t;
      }
      for (int i = j + 1; i < k; ++i) {
        double f = G2[i * k + j] / G2[j * k + j];
        for (int c = j; c < k; ++c) G2[i * k + c] -= f * G2[j * k + c];
        m[i] -= f * m[j];
      }
    }
    if (ok == -1) {
      for (int j = 0; j < k; ++j) m[j] = 0.0;
    } else {
      for (int j = k - 1; j >= 0; --j) {
        double v = m[j];
        for (int c = j + 1; c < k; ++c) v -= G2[j * k + c] * m[c];
        m[j] = v / G2[j * k + j];
      }
    }
  }
  free(G2);
}

/* position of column c in row i's columns J (k entries), or -1 (the
 * reference's col_to_local map) */
static int spai1_local(const int *J, int k, int c) {
  for (int p = 0; p < k; ++p)
    if (J[p] == c) return p;
  return -1;
}

/* _compute_spai1!, src/smoothers.jl:620-690, loop for loop: for each row i
 * with columns J, every row r of A (in order) adds a_rp a_rq to G_pq for
 * its entries in J; rhs_p = a_i,Jp; G_pp += eps max(1, |G_pp|); m = G \ rhs
 * stored on row i's entries. */
void orc_spai1(int n, const int *rp, const int *ci, const double *a, double *M) {
  for (int i = 0; i < n; ++i) {
    const int rs = rp[i], k = rp[i + 1] - rs;
    if (k == 0) continue;
    const int *J = ci + rs;
    double *G = (double *)calloc((size_t)k * k, sizeof(double));
    double *rhs = (double *)malloc(sizeof(double) * (size_t)k);
    double *m = (double *)malloc(sizeof(double) * (size_t)k);
    for (int r = 0; r < n; ++r) /* every row, in order */
      for (int e1 = rp[r]; e1 < rp[r + 1]; ++e1) {
        const int p = spai1_local(J, k, ci[e1]);
        if (p < 0) continue;
        for (int e2 = rp[r]; e2 < rp[r + 1]; ++e2) {
          const int q = spai1_local(J, k, ci[e2]);
          if (q >= 0) G[p * k + q] += a[e1] * a[e2];
        }
      }
    for (int p = 0; p < k; ++p) rhs[p] = a[rs + p];
    for (int p = 0; p < k; ++p) {
      const double g = fabs(G[p * k + p]);
      G[p * k + p] += 2.220446049250313e-16 * (g > 1.0 ? g : 1.0);
    }
    spai1_solve(k, G, rhs, m);
    for (int p = 0; p < k; ++p) M[rs + p] = m[p];
    free(G);
    free(rhs);
    free(m);
  }
}

/* smooth!(::SPAI1Smoother), src/smoothers.jl:709-760: per step r = b - A x
 * (from b, column order), then x_i += sum_j M_ij r_j (summed from zero) */
void orc_spai1_smooth(int n, const int *rp, const int *ci, const double *a, const double *M, double *x,
                      const double *b, int steps, double *r) {
  for (int s = 0; s < steps; ++s) {
    for (int i = 0; i < n; ++i) {
      double ri = b[i];
      for (int nz = rp[i]; nz < rp[i + 1]; ++nz) ri -= a[nz] * x[ci[nz]];
      r[i] = ri;
    }
    for (int i = 0; i < n; ++i) {
      double v = 0.0;
      for (int nz = rp[i]; nz < rp[i + 1]; ++nz) v += M[nz] * r[ci[nz]];
      x[i] += v;
    }
  }
}

/* _serial_gs_compute_invdiag!, src/smoothers.jl:329-340: 1/a_ii from the
 * row's first diagonal entry, 0 when |a_ii| <= eps */
void orc_serial_gs_invdiag(int n, const int *rp, const int *ci, const double *v, double *invd) {
  for (int i = 0; i < n; ++i) {
    double d = 0.0;
    for (int k = rp[i]; k < rp[i + 1]; ++k)
      if (ci[k] == i) {
        d = v[k];
        break;
      }
    invd[i] = fabs(d) > 2.220446049250313e-16 ? 1.0 / d : 0.0;
  }
}

/* _serial_gs_sweep!, src/smoothers.jl:350-362: rows in order, in place:
 * r_i = b_i - sum_j a_ij x_j (current x), x_i += invdiag_i r_i */
void orc_serial_gs(int n, const int *rp, const int *ci, const double *v, const double *invd, double *x,
                   const double *b, int steps) {
  for (int s = 0; s < steps; ++s)
    for (int i = 0; i < n; ++i) {
      double r = b[i];
      for (int k = rp[i]; k < rp[i + 1]; ++k) r -= v[k] * x[ci[k]];
      x[i] += invd[i] * r;
    }
}

/* smooth!(::JacobiSmoother / ::L1JacobiSmoother): jacobi_kernel! with the
 * tmp/x ping-pong and the copy back on odd step counts,
 * src/smoothers.jl:78-124, :835-854 */
void orc_jacobi(int n, const int *rp, const int *ci, const double *v, const double *invd,
                double omega, double *x, const double *b, int steps, double *tmp) {
  double *src = x, *dst = tmp;
  for (int s = 0; s < steps; ++s) {
#pragma omp parallel for schedule(static, CHUNK)
    for (int i = 0; i < n; ++i) {
      double ri = b[i];
      for (int k = rp[i]; k < rp[i + 1]; ++k) ri -= v[k] * src[ci[k]];
      dst[i] = src[i] + omega * invd[i] * ri;
    }
    double *t = src;
    src = dst;
    dst = t;
  }
  if (steps & 1) memcpy(x, tmp, (size_t)n * sizeof(double));
}

/* greedy_coloring, src/smoothers.jl:136-159; returns the number of colours */
int orc_greedy_coloring(int n, const int *rp, const int *ci, int *colors) {
  int ncol = 0;
  int cap = 64;
  int *stamp = (int *)malloc(sizeof(int) * cap);
  for (int c = 0; c < cap; ++c) stamp[c] = -1;
  for (int i = 0; i < n; ++i) colors[i] = 0;
  for (int i = 0; i < n; ++i) {
    for (int k = rp[i]; k < rp[i + 1]; ++k) {
      int j = ci[k];
      if (j != i && colors[j] > 0) {
        int c = colors[j];
        if (c >= cap) {
          int nc2 = 2 * c + 2;
          stamp = (int *)realloc(stamp, sizeof(int) * nc2);
          for (int t = cap; t < nc2; ++t) stamp[t] = -1;
          cap = nc2;
        }
        stamp[c] = i;
      }
    }
    int c = 1;
    while (c < cap && stamp[c] == i) ++c;
    colors[i] = c;
    if (c > ncol) ncol = c;
  }
  free(stamp);
  return ncol;
}

/* colour-sorted node order, src/smoothers.jl:168-195 (0-based offsets) */
void orc_color_order(int n, const int *colors, int ncol, int *off, int *order) {
  for (int c = 0; c <= ncol; ++c) off[c] = 0;
  for (int i = 0; i < n; ++i) off[colors[i]]++;
  /* off[c] holds the count of colour c (1-based); prefix to starts */
  int acc = 0;
  for (int c = 1; c <= ncol; ++c) {
    int cnt = off[c];
    off[c] = acc + cnt;
    acc += cnt;
  }
  off[0] = 0;
  int *pos = (int *)malloc(sizeof(int) * (ncol + 1));
  for (int c = 1; c <= ncol; ++c) pos[c] = off[c - 1];
  for (int i = 0; i < n; ++i) order[pos[colors[i]]++] = i;
  free(pos);
}

/* smooth!(::ColoredGaussSeidelSmoother) / L1 variant: gs_color_kernel! per
 * colour in ascending colour order, src/smoothers.jl:203-241, :296-313 */
void orc_gs(int n, const int *rp, const int *ci, const double *v, const double *invd, int ncol,
            const int *off, const int *order, double *x, const double *b, int steps) {
  (void)n;
  for (int s = 0; s < steps; ++s)
    for (int c = 0; c < ncol; ++c) {
      int st = off[c], cnt = off[c + 1] - off[c];
#pragma omp parallel for schedule(static, CHUNK)
      for (int t = 0; t < cnt; ++t) {
        int i = order[st + t];
        double ri = b[i];
        for (int k = rp[i]; k < rp[i + 1]; ++k) ri -= v[k] * x[ci[k]];
        x[i] += invd[i] * ri;
      }
    }
}

/* build_transpose_map, src/prolongation.jl:767-800 */
void orc_transpose_map(int nf, int nc, const int *prp, const int *pci, int *off, int *rows,
                       int *pnz) {
  for (int j = 0; j <= nc; ++j) off[j] = 0;
  for (int i = 0; i < nf; ++i)
    for (int k = prp[i]; k < prp[i + 1]; ++k) off[pci[k] + 1]++;
  for (int j = 0; j < nc; ++j) off[j + 1] += off[j];
  int *pos = (int *)malloc(sizeof(int) * (nc > 0 ? nc : 1));
  for (int j = 0; j < nc; ++j) pos[j] = off[j];
  for (int i = 0; i < nf; ++i)
    for (int k = prp[i]; k < prp[i + 1]; ++k) {
      int J = pci[k];
      rows[pos[J]] = i;
      pnz[pos[J]] = k;
      pos[J]++;
    }
  free(pos);
}

/* restrict_kernel!, src/prolongation.jl:805-827 */
void orc_restrict(int nc, const int *off, const int *rows, const int *pnz, const double *pv,
                  const double *r, double *bc) {
#pragma omp parallel for schedule(static, CHUNK)
  for (int J = 0; J < nc; ++J) {
    double acc = 0.0;
    for (int k = off[J]; k < off[J + 1]; ++k) acc += pv[pnz[k]] * r[rows[k]];
    bc[J] = acc;
  }
}

/* prolongate_kernel!, src/prolongation.jl:742-760 (x updated per entry) */
void orc_prolongate(int nf, const int *prp, const int *pci, const double *pv, const double *xc,
                    double *x) {
#pragma omp parallel for schedule(static, CHUNK)
  for (int i = 0; i < nf; ++i)
    for (int k = prp[i]; k < prp[i + 1]; ++k) x[i] += pv[k] * xc[pci[k]];
}

/* ------------------------------------------------------ Galerkin product */
/* compute_coarse_sparsity, src/galerkin.jl:11-183: triples in the loop
 * order (fine row i, P entry of i, A entry, P entry of j), counting sort by
 * coarse row, sorted unique columns per coarse row, values accumulated in
 * triple order, and the RestrictionMap with triples grouped by destination
 * in stable order.  Call once with c_rp only (other outputs NULL) to get
 * the sizes: returns ntriples, writes c_rp (nc+1).  Call again with all
 * outputs allocated. */
static int cmp_int(const void *a, const void *b) {
  int x = *(const int *)a, y = *(const int *)b;
  return (x > y) - (x < y);
}

int64_t orc_coarse_sparsity(int nf, int nc, const int *arp, const int *aci, const double *av,
                            const int *prp, const int *pci, const double *pv, int *c_rp,
                            int *c_ci, double *c_v, int64_t *nz_off, int *tpi, int *tai, int *tpj) {
  int64_t nt = 0;
  for (int i = 0; i < nf; ++i)
    for (int a = prp[i]; a < prp[i + 1]; ++a)
      for (int k = arp[i]; k < arp[i + 1]; ++k) {
        int j = aci[k];
        nt += prp[j + 1] - prp[j];
      }
  int *rI = (int *)malloc(sizeof(int) * (nt ? nt : 1));
  int *rJ = (int *)malloc(sizeof(int) * (nt ? nt : 1));
  int *rpi = (int *)malloc(sizeof(int) * (nt ? nt : 1));
  int *rai = (int *)malloc(sizeof(int) * (nt ? nt : 1));
  int *rpj = (int *)malloc(sizeof(int) * (nt ? nt : 1));
  int64_t t = 0;
  for (int i = 0; i < nf; ++i)
    for (int a = prp[i]; a < prp[i + 1]; ++a) {
      int I = pci[a];
      for (int k = arp[i]; k < arp[i + 1]; ++k) {
        int j = aci[k];
        for (int b = prp[j]; b < prp[j + 1]; ++b) {
          rI[t] = I;
          rJ[t] = pci[b];
          rpi[t] = a;
          rai[t] = k;
          rpj[t] = b;
          ++t;
        }
      }
    }
  /* counting sort by coarse row */
  int64_t *rtmp = (int64_t *)calloc((size_t)nc + 1, sizeof(int64_t));
  for (int64_t s = 0; s < nt; ++s) rtmp[rI[s] + 1]++;
  for (int r = 0; r < nc; ++r) rtmp[r + 1] += rtmp[r];
  int64_t *perm = (int64_t *)malloc(sizeof(int64_t) * (nt ? nt : 1));
  int64_t *pos = (int64_t *)malloc(sizeof(int64_t) * ((size_t)nc + 1));
  for (int r = 0; r < nc; ++r) pos[r] = rtmp[r];
  for (int64_t s = 0; s < nt; ++s) perm[pos[rI[s]]++] = s;
  /* unique sorted columns per row */
  int *buf = (int *)malloc(sizeof(int) * (nt ? nt : 1));
  c_rp[0] = 0;
  for (int r = 0; r < nc; ++r) {
    int64_t rs = rtmp[r], re = rtmp[r + 1];
    int len = (int)(re - rs);
    int nu = 0;
    if (len > 0) {
      for (int64_t k = rs; k < re; ++k) buf[k - rs] = rJ[perm[k]];
      qsort(buf, len, sizeof(int), cmp_int);
      nu = 1;
      for (int k = 1; k < len; ++k)
        if (buf[k] != buf[k - 1]) ++nu;
    }
    c_rp[r + 1] = c_rp[r] + nu;
  }
  if (c_ci) {
    int *rci = (int *)malloc(sizeof(int) * (nt ? nt : 1));
    for (int r = 0; r < nc; ++r) {
      int64_t rs = rtmp[r], re = rtmp[r + 1];
      int len = (int)(re - rs);
      if (len == 0) continue;
      for (int64_t k = rs; k < re; ++k) buf[k - rs] = rJ[perm[k]];
      qsort(buf, len, sizeof(int), cmp_int);
      int p = c_rp[r];
      c_ci[p] = buf[0];
      for (int k = 1; k < len; ++k)
        if (buf[k] != buf[k - 1]) c_ci[++p] = buf[k];
      int lo0 = c_rp[r], hi0 = c_rp[r + 1] - 1;
      for (int64_t k = rs; k < re; ++k) {
        int64_t s = perm[k];
        int J = rJ[s], lo = lo0, hi = hi0, at = -1;
        while (lo <= hi) {
          int mid = (lo + hi) >> 1;
          if (c_ci[mid] == J) { at = mid; break; }
          if (c_ci[mid] < J) lo = mid + 1; else hi = mid - 1;
        }
        rci[s] = at;
      }
    }
    for (int k = 0; k < c_rp[nc]; ++k) c_v[k] = 0.0;
    /* values in row order, triples of a row in generation order */
    for (int r = 0; r < nc; ++r)
      for (int64_t k = rtmp[r]; k < rtmp[r + 1]; ++k) {
        int64_t s = perm[k];
        c_v[rci[s]] += pv[rpi[s]] * av[rai[s]] * pv[rpj[s]];
      }
    /* restriction map: stable grouping by destination */
    int nnzc = c_rp[nc];
    for (int k = 0; k <= nnzc; ++k) nz_off[k] = 0;
    for (int64_t s = 0; s < nt; ++s) nz_off[rci[s] + 1]++;
    for (int k = 0; k < nnzc; ++k) nz_off[k + 1] += nz_off[k];
    int64_t *wp = (int64_t *)malloc(sizeof(int64_t) * (nnzc ? nnzc : 1));
    for (int k = 0; k < nnzc; ++k) wp[k] = nz_off[k];
    for (int64_t s = 0; s < nt; ++s) {
      int64_t q = wp[rci[s]]++;
      tpi[q] = rpi[s];
      tai[q] = rai[s];
      tpj[q] = rpj[s];
    }
    free(wp);
    free(rci);
  }
  free(buf);
  free(pos);
  free(perm);
  free(rtmp);
  free(rI);
  free(rJ);
  free(rpi);
  free(rai);
  free(rpj);
  return nt;
}

/* galerkin_nz_kernel!, src/galerkin.jl:194-222 */
void orc_galerkin(int nnzc, const int64_t *nz_off, const int *tpi, const int *tai, const int *tpj,
                  const double *pv, const double *av, double *cv) {
#pragma omp parallel for schedule(static, CHUNK)
  for (int k = 0; k < nnzc; ++k) {
    double acc = 0.0;
    for (int64_t t = nz_off[k]; t < nz_off[k + 1]; ++t) acc += pv[tpi[t]] * av[tai[t]] * pv[tpj[t]];
    cv[k] = acc;
  }
}

/* _recompute_coarsest_dense!, src/resetup.jl:123-158 (column-major M) */
void orc_coarsest_dense(int nf, int nc, const int *arp, const int *aci, const double *av,
                        const int *prp, const int *pci, const double *pv, double *M) {
  memset(M, 0, sizeof(double) * (size_t)nc * nc);
  for (int i = 0; i < nf; ++i)
    for (int a = prp[i]; a < prp[i + 1]; ++a) {
      int I = pci[a];
      double p_i = pv[a];
      for (int k = arp[i]; k < arp[i + 1]; ++k) {
        int j = aci[k];
        double aij = av[k];
        for (int b = prp[j]; b < prp[j + 1]; ++b) M[(size_t)pci[b] * nc + I] += p_i * aij * pv[b];
      }
    }
}

/* _csr_to_dense!, src/setup.jl:495-516 (later entries of a row overwrite) */
void orc_csr_to_dense(int n, const int *rp, const int *ci, const double *v, double *M) {
  memset(M, 0, sizeof(double) * (size_t)n * n);
  for (int i = 0; i < n; ++i)
    for (int k = rp[i]; k < rp[i + 1]; ++k) M[(size_t)ci[k] * n + i] = v[k];
}

/* ------------------------------------------------------ coarsest LU */
/* lu(M) for the coarsest level (src/setup.jl:526-534, src/resetup.jl:44):
 * LAPACK dgetf2 semantics — pivot = first row of largest magnitude, column
 * scaled by the reciprocal of the pivot, rank-1 update.  Returns 0 or the
 * 1-based index of the first zero pivot (Julia raises SingularException). */
int orc_lu_factor(int n, double *a, int *piv) {
  for (int j = 0; j < n; ++j) {
    int p = j;
    double mx = fabs(a[(size_t)j * n + j]);
    for (int i = j + 1; i < n; ++i)
      if (fabs(a[(size_t)j * n + i]) > mx) { mx = fabs(a[(size_t)j * n + i]); p = i; }
    piv[j] = p;
    if (a[(size_t)j * n + p] == 0.0) return j + 1;
    if (p != j)
      for (int c = 0; c < n; ++c) {
        double t = a[(size_t)c * n + j];
        a[(size_t)c * n + j] = a[(size_t)c * n + p];
        a[(size_t)c * n + p] = t;
      }
    double r = 1.0 / a[(size_t)j * n + j];
    for (int i = j + 1; i < n; ++i) a[(size_t)j * n + i] *= r;
    for (int c = j + 1; c < n; ++c) {
      double t = a[(size_t)c * n + j];
      for (int i = j + 1; i < n; ++i) a[(size_t)c * n + i] -= a[(size_t)j * n + i] * t;
    }
  }
  return 0;
}

/* ldiv!(x, F, b) with dgetrs semantics: row interchanges, then the
 * column-oriented unit-lower and upper triangular solves of dtrsv. */
void orc_lu_solve(int n, const double *lu, const int *piv, double *y) {
  for (int j = 0; j < n; ++j)
    if (piv[j] != j) {
      double t = y[j];
      y[j] = y[piv[j]];
      y[piv[j]] = t;
    }
  for (int j = 0; j < n; ++j)
    if (y[j] != 0.0)
      for (int i = j + 1; i < n; ++i) y[i] -= y[j] * lu[(size_t)j * n + i];
  for (int j = n - 1; j >= 0; --j)
    if (y[j] != 0.0) {
      y[j] /= lu[(size_t)j * n + j];
      double t = y[j];
      for (int i = 0; i < j; ++i) y[i] -= t * lu[(size_t)j * n + i];
    }
}

/* ------------------------------------------------------ cycle and solve */
static void smooth(olevel *L, double *x, const double *b, int steps) {
  if (steps <= 0) return;
  if (L->smoother == 0 || L->smoother == 5)
    orc_jacobi(L->n, L->A_rp, L->A_ci, L->A_v, L->invd, L->omega, x, b, steps, L->tmp);
  else if (L->smoother == 3)
    orc_spai0_smooth(L->n, L->A_rp, L->A_ci, L->A_v, L->invd, x, b, steps, L->tmp);
  else if (L->smoother == 8)
    orc_chebyshev(L->n, L->A_rp, L->A_ci, L->A_v, L->invd, L->cheb_coef, L->cheb_degree, x, b, steps,
                  L->tmp, L->cheb_d);
  else if (L->smoother == 2 || L->smoother == 7)
    orc_serial_gs(L->n, L->A_rp, L->A_ci, L->A_v, L->invd, x, b, steps);
  else if (L->smoother == 4)
    orc_spai1_smooth(L->n, L->A_rp, L->A_ci, L->A_v, L->spai1_M, x, b, steps, L->tmp);
  else if (L->smoother == 9 || L->smoother == 10)
    orc_ilu0_smooth(L->n, L->A_rp, L->A_ci, L->A_v, L->ilu_diag, L->ilu_L, L->ilu_U, x, b, steps, L->tmp);
  else
    orc_gs(L->n, L->A_rp, L->A_ci, L->A_v, L->invd, L->ncolors, L->color_off, L->color_order, x, b,
           steps);
}

/* _vcycle_descend!, src/cycle.jl:63-99 */
static void vcycle(ohier *h, int lvl, double *x, const double *b, int pre, int post, int w) {
  olevel *L = &h->lv[lvl];
  smooth(L, x, b, pre);
  orc_residual(L->n, L->A_rp, L->A_ci, L->A_v, x, b, L->r);
  orc_restrict(L->nc, L->T_off, L->T_rows, L->T_pnz, L->P_v, L->r, L->bc);
  memset(L->xc, 0, sizeof(double) * (size_t)L->nc);
  if (lvl + 1 < h->nlevels) {
    int nr = w ? 2 : 1;
    for (int t = 0; t < nr; ++t) vcycle(h, lvl + 1, L->xc, L->bc, pre, post, w);
  } else {
    memcpy(h->cb, L->bc, sizeof(double) * (size_t)h->nc);
    memcpy(h->cx, h->cb, sizeof(double) * (size_t)h->nc);
    orc_lu_solve(h->nc, h->lu, h->piv, h->cx);
    memcpy(L->xc, h->cx, sizeof(double) * (size_t)h->nc);
  }
  orc_prolongate(L->n, L->P_rp, L->P_ci, L->P_v, L->xc, x);
  smooth(L, x, b, post);
}

/* amg_cycle!, src/cycle.jl:12-28 */
void orc_cycle(ohier *h, double *x, const double *b, int pre, int post, int w) {
  if (h->nlevels == 0) {
    memcpy(h->cx, b, sizeof(double) * (size_t)h->nc);
    orc_lu_solve(h->nc, h->lu, h->piv, h->cx);
    memcpy(x, h->cx, sizeof(double) * (size_t)h->nc);
    return;
  }
  vcycle(h, 0, x, b, pre, post, w);
}

static double dot(int n, const double *a, const double *b) {
  double s = 0.0;
#pragma omp parallel for schedule(static) reduction(+ : s)
  for (int i = 0; i < n; ++i) s += a[i] * b[i];
  return s;
}

/* amg_solve!, src/cycle.jl:110-160; returns iterations, relres[0] final */
int orc_solve(ohier *h, double *x, const double *b, int pre, int post, int w, double tol,
              int maxiter, double *relres) {
  int n = h->nlevels ? h->lv[0].n : h->nc;
  double bnorm = sqrt(dot(n, b, b));
  if (bnorm == 0.0) {
    memset(x, 0, sizeof(double) * (size_t)n);
    if (relres) *relres = 0.0;
    return 0;
  }
  if (h->nlevels == 0) {
    orc_cycle(h, x, b, pre, post, w);
    if (relres) *relres = NAN;
    return 1;
  }
  olevel *L = &h->lv[0];
  double rel = 1.0;
  for (int it = 1; it <= maxiter; ++it) {
    orc_cycle(h, x, b, pre, post, w);
    orc_residual(n, L->A_rp, L->A_ci, L->A_v, x, b, h->solve_r);
    rel = sqrt(dot(n, h->solve_r, h->solve_r)) / bnorm;
    if (rel < tol) {
      if (relres) *relres = rel;
      return it;
    }
  }
  if (relres) *relres = rel;
  return maxiter;
}

/* Textbook preconditioned CG around amg_cycle! with a zeroed iterate per
 * application (preconditioner_apply!, src/preconditioner.jl:76-80).  The
 * reference has no CG of its own; this is the standard algorithm.
 * work: 4n doubles (r, z, p, q). */
int orc_pcg(ohier *h, double *x, const double *b, int pre, int post, int w, double tol,
            int maxiter, double *relres, double *work) {
  int n = h->nlevels ? h->lv[0].n : h->nc;
  const int *rp = h->nlevels ? h->lv[0].A_rp : h->coarse_rp;
  const int *ci = h->nlevels ? h->lv[0].A_ci : h->coarse_ci;
  const double *v = h->nlevels ? h->lv[0].A_v : h->coarse_v;
  double *r = work, *z = work + n, *p = work + 2 * (size_t)n, *q = work + 3 * (size_t)n;
  orc_residual(n, rp, ci, v, x, b, r);
  double bnorm = sqrt(dot(n, b, b));
  if (bnorm == 0.0) {
    memset(x, 0, sizeof(double) * (size_t)n);
    if (relres) *relres = 0.0;
    return 0;
  }
  double rel = sqrt(dot(n, r, r)) / bnorm;
  if (rel < tol) {
    if (relres) *relres = rel;
    return 0;
  }
  memset(z, 0, sizeof(double) * (size_t)n);
  orc_cycle(h, z, r, pre, post, w);
  memcpy(p, z, sizeof(double) * (size_t)n);
  double rz = dot(n, r, z);
  int it;
  for (it = 1; it <= maxiter; ++it) {
    orc_spmv(n, rp, ci, v, p, q);
    double alpha = rz / dot(n, p, q);
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; ++i) {
      x[i] += alpha * p[i];
      r[i] -= alpha * q[i];
    }
    rel = sqrt(dot(n, r, r)) / bnorm;
    if (rel < tol || it == maxiter) break;
    memset(z, 0, sizeof(double) * (size_t)n);
    orc_cycle(h, z, r, pre, post, w);
    double rzn = dot(n, r, z);
    double beta = rzn / rz;
    rz = rzn;
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; ++i) p[i] = z[i] + beta * p[i];
  }
  if (it > maxiter) it = maxiter;
  if (relres) *relres = rel;
  return it;
}

/* ------------------------------------------------------ resetup */
/* amg_resetup!(partial=true), src/resetup.jl:20-45: new finest values,
 * smoother diagonals, Galerkin products through the restriction maps, the
 * coarsest dense product (src/resetup.jl:123-158) and its LU.  coarse_rp /
 * coarse_ci / coarse_v describe the coarsest CSR when nlevels == 0.
 * Returns 0 or the LU's zero-pivot index. */
static void upd_invd(olevel *L) {
  if (L->smoother == 5 || L->smoother == 6 || L->smoother == 7) orc_l1_invdiag(L->n, L->A_rp, L->A_v, L->invd);
  else if (L->smoother == 2) orc_serial_gs_invdiag(L->n, L->A_rp, L->A_ci, L->A_v, L->invd);
  else if (L->smoother == 3) orc_spai0(L->n, L->A_rp, L->A_ci, L->A_v, L->invd);
  else orc_invdiag(L->n, L->A_rp, L->A_ci, L->A_v, L->invd);
  if (L->smoother == 4) /* update_smoother!(::SPAI1Smoother), src/smoothers.jl:692-699 */
    orc_spai1(L->n, L->A_rp, L->A_ci, L->A_v, L->spai1_M);
  if (L->smoother == 9 || L->smoother == 10) /* update_smoother!, src/smoothers.jl:1332-1337 */
    orc_ilu0_factor(L->n, L->A_rp, L->A_ci, L->A_v, L->ilu_diag, L->ilu_L, L->ilu_U);
  if (L->smoother == 8) { /* update_smoother!(::ChebyshevSmoother), src/smoothers.jl:912-922 */
    memcpy(L->tmp, L->cheb_v0, (size_t)L->n * sizeof(double));
    double rho = orc_spectral_radius(L->n, L->A_rp, L->A_ci, L->A_v, L->invd, L->tmp, 10, L->r);
    orc_cheb_coef(rho, L->cheb_degree, L->cheb_coef);
  }
}

int orc_resetup(ohier *h, const double *v0, int64_t nnz0) {
  if (h->nlevels == 0) {
    memcpy(h->coarse_v, v0, sizeof(double) * (size_t)nnz0);
    orc_csr_to_dense(h->nc, h->coarse_rp, h->coarse_ci, h->coarse_v, h->dense);
  } else {
    memcpy(h->lv[0].A_v, v0, sizeof(double) * (size_t)nnz0);
    upd_invd(&h->lv[0]);
    for (int l = 0; l + 1 < h->nlevels; ++l) {
      olevel *L = &h->lv[l], *N = &h->lv[l + 1];
      int nnzc = N->A_rp[N->n];
      orc_galerkin(nnzc, L->nz_off, L->tpi, L->tai, L->tpj, L->P_v, L->A_v, N->A_v);
      upd_invd(N);
    }
    olevel *last = &h->lv[h->nlevels - 1];
    orc_coarsest_dense(last->n, h->nc, last->A_rp, last->A_ci, last->A_v, last->P_rp, last->P_ci,
                       last->P_v, h->dense);
  }
  memcpy(h->lu, h->dense, sizeof(double) * (size_t)h->nc * h->nc);
  return orc_lu_factor(h->nc, h->lu, h->piv);
}

/* ------------------------------------------------------ setup pieces */
/* absolute_strength_kernel!, src/strength.jl:38-76 */
void orc_strength_abs(int n, const int *rp, const int *ci, const double *v, double theta,
                      uint8_t *s) {
  for (int i = 0; i < n; ++i) {
    double mx = 0.0;
    for (int k = rp[i]; k < rp[i + 1]; ++k)
      if (ci[k] != i && fabs(v[k]) > mx) mx = fabs(v[k]);
    double thr = theta * mx;
    for (int k = rp[i]; k < rp[i + 1]; ++k) s[k] = (ci[k] != i) ? (fabs(v[k]) >= thr) : 0;
  }
}
