// Galerkin product structure, smoother data, coarsest LU and the level loop
// of the CPU setup phase.
//
//   transpose map        src/prolongation.jl:767-800
//   coarse sparsity      src/galerkin.jl:11-183 (the pattern of P^T A P:
//                        sorted unique columns per coarse row); here built
//                        row by row through A*P instead of from sorted triples
//   colouring            src/smoothers.jl:136-195
//   smoother diagonals   src/smoothers.jl:47-63, :816-827
//   coarse solver        src/setup.jl:177-209, :495-516, :526-534
//   level loop           src/setup.jl:123-166, θ fallback :219-237,
//                        coarsen+P :256-327
#include <omp.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <limits>
#include <numeric>
#include <sstream>

#include "dr_host.h"

namespace dr {

static const double kEps = std::numeric_limits<double>::epsilon();

TransposeMap build_transpose_map(const Prolong& P) {
  TransposeMap T;
  T.off.assign(P.nc + 1, 0);
  for (int64_t k = 0; k < P.nnz(); ++k) T.off[P.ci[k] + 1]++;
  for (int j = 0; j < P.nc; ++j) T.off[j + 1] += T.off[j];
  T.rows.resize(P.nnz());
  T.pnz.resize(P.nnz());
  std::vector<int> pos(T.off.begin(), T.off.end() - 1);
  for (int i = 0; i < P.nf; ++i)
    for (int k = P.rp[i]; k < P.rp[i + 1]; ++k) {
      int J = P.ci[k];
      T.rows[pos[J]] = i;
      T.pnz[pos[J]] = k;
      pos[J]++;
    }
  return T;
}

void symbolic_ap(const CSR& A, const Prolong& P, std::vector<int>& ap_rp, std::vector<int>& ap_ci) {
  const int n = A.n, nc = P.nc;
  ap_rp.assign(n + 1, 0);
#pragma omp parallel
  {
    std::vector<int> mark(nc, -1);
#pragma omp for schedule(static, 2048)
    for (int i = 0; i < n; ++i) {
      int cnt = 0;
      for (int k = A.rp[i]; k < A.rp[i + 1]; ++k) {
        int j = A.ci[k];
        for (int p = P.rp[j]; p < P.rp[j + 1]; ++p) {
          int J = P.ci[p];
          if (mark[J] != i) { mark[J] = i; ++cnt; }
        }
      }
      ap_rp[i + 1] = cnt;
    }
  }
  for (int i = 0; i < n; ++i) ap_rp[i + 1] += ap_rp[i];
  ap_ci.resize(ap_rp[n]);
#pragma omp parallel
  {
    std::vector<int> mark(nc, -1);
#pragma omp for schedule(static, 2048)
    for (int i = 0; i < n; ++i) {
      int w = ap_rp[i];
      for (int k = A.rp[i]; k < A.rp[i + 1]; ++k) {
        int j = A.ci[k];
        for (int p = P.rp[j]; p < P.rp[j + 1]; ++p) {
          int J = P.ci[p];
          if (mark[J] != i) { mark[J] = i; ap_ci[w++] = J; }
        }
      }
      std::sort(ap_ci.begin() + ap_rp[i], ap_ci.begin() + ap_rp[i + 1]);
    }
  }
}

void symbolic_ptap(const TransposeMap& T, int nc, const std::vector<int>& ap_rp,
                   const std::vector<int>& ap_ci, std::vector<int>& c_rp, std::vector<int>& c_ci) {
  c_rp.assign(nc + 1, 0);
#pragma omp parallel
  {
    std::vector<int> mark(nc, -1);
#pragma omp for schedule(dynamic, 256)
    for (int I = 0; I < nc; ++I) {
      int cnt = 0;
      for (int t = T.off[I]; t < T.off[I + 1]; ++t) {
        int i = T.rows[t];
        for (int q = ap_rp[i]; q < ap_rp[i + 1]; ++q) {
          int J = ap_ci[q];
          if (mark[J] != I) { mark[J] = I; ++cnt; }
        }
      }
      c_rp[I + 1] = cnt;
    }
  }
  for (int I = 0; I < nc; ++I) c_rp[I + 1] += c_rp[I];
  c_ci.resize(c_rp[nc]);
#pragma omp parallel
  {
    std::vector<int> mark(nc, -1);
#pragma omp for schedule(dynamic, 256)
    for (int I = 0; I < nc; ++I) {
      int w = c_rp[I];
      for (int t = T.off[I]; t < T.off[I + 1]; ++t) {
        int i = T.rows[t];
        for (int q = ap_rp[i]; q < ap_rp[i + 1]; ++q) {
          int J = ap_ci[q];
          if (mark[J] != I) { mark[J] = I; c_ci[w++] = J; }
        }
      }
      std::sort(c_ci.begin() + c_rp[I], c_ci.begin() + c_rp[I + 1]);
    }
  }
}

void numeric_ap(const CSR& A, const Prolong& P, const std::vector<int>& ap_rp,
                const std::vector<int>& ap_ci, std::vector<double>& ap_v) {
  const int n = A.n, nc = P.nc;
  ap_v.assign(ap_ci.size(), 0.0);
#pragma omp parallel
  {
    std::vector<double> acc(nc, 0.0);
#pragma omp for schedule(static, 2048)
    for (int i = 0; i < n; ++i) {
      for (int k = A.rp[i]; k < A.rp[i + 1]; ++k) {
        const double a = A.v[k];
        const int j = A.ci[k];
        for (int p = P.rp[j]; p < P.rp[j + 1]; ++p) {
          const double prod = a * P.v[p];
          acc[P.ci[p]] = acc[P.ci[p]] + prod;
        }
      }
      for (int q = ap_rp[i]; q < ap_rp[i + 1]; ++q) {
        ap_v[q] = acc[ap_ci[q]];
        acc[ap_ci[q]] = 0.0;
      }
    }
  }
}

void numeric_ptap(const TransposeMap& T, const std::vector<double>& Rv, const std::vector<int>& ap_rp,
                  const std::vector<int>& ap_ci, const std::vector<double>& ap_v,
                  const std::vector<int>& c_rp, const std::vector<int>& c_ci, std::vector<double>& c_v) {
  const int nc = (int)T.off.size() - 1;
  c_v.assign(c_ci.size(), 0.0);
#pragma omp parallel
  {
    std::vector<double> acc(nc, 0.0);
#pragma omp for schedule(dynamic, 256)
    for (int I = 0; I < nc; ++I) {
      for (int t = T.off[I]; t < T.off[I + 1]; ++t) {
        const double p = Rv[t];
        const int i = T.rows[t];
        for (int q = ap_rp[i]; q < ap_rp[i + 1]; ++q) {
          const double prod = p * ap_v[q];
          acc[ap_ci[q]] = acc[ap_ci[q]] + prod;
        }
      }
      for (int q = c_rp[I]; q < c_rp[I + 1]; ++q) {
        c_v[q] = acc[c_ci[q]];
        acc[c_ci[q]] = 0.0;
      }
    }
  }
}

void greedy_coloring(const CSR& A, std::vector<int>& colors, int& num_colors) {
  const int n = A.n;
  colors.assign(n, 0);
  num_colors = 0;
  std::vector<int> stamp(8, -1);
  for (int i = 0; i < n; ++i) {
    for (int k = A.rp[i]; k < A.rp[i + 1]; ++k) {
      int j = A.ci[k];
      if (j != i && colors[j] > 0) {
        int c = colors[j];
        if (c >= (int)stamp.size()) stamp.resize(2 * c + 2, -1);
        stamp[c] = i;
      }
    }
    int c = 1;
    while (c < (int)stamp.size() && stamp[c] == i) ++c;
    colors[i] = c;
    num_colors = std::max(num_colors, c);
  }
}

void color_order_from(const std::vector<int>& colors, int num_colors, std::vector<int>& off,
                      std::vector<int>& order) {
  // Counting sort of the rows by colour, ascending row index within a colour
  // (src/smoothers.jl:168-195); off[c-1] .. off[c] holds colour c.
  const int n = (int)colors.size();
  std::vector<int> cnt(num_colors + 1, 0);
  for (int i = 0; i < n; ++i) cnt[colors[i]]++;
  off.assign(num_colors + 1, 0);
  for (int c = 1; c <= num_colors; ++c) off[c] = off[c - 1] + cnt[c];
  order.resize(n);
  std::vector<int> pos(off.begin(), off.end() - 1);
  for (int i = 0; i < n; ++i) order[pos[colors[i] - 1]++] = i;
}

void inverse_diagonal(const CSR& A, std::vector<double>& invd) {
  invd.resize(A.n);
#pragma omp parallel for schedule(static, 4096)
  for (int i = 0; i < A.n; ++i) {
    double d = 0.0, rn = 0.0;
    for (int k = A.rp[i]; k < A.rp[i + 1]; ++k) {
      rn += std::fabs(A.v[k]);
      if (A.ci[k] == i) d = A.v[k];
    }
    double thr = kEps * std::max(1.0, rn);
    invd[i] = std::fabs(d) > thr ? 1.0 / d : 0.0;
  }
}

void l1_inverse_diagonal(const CSR& A, std::vector<double>& invd) {
  invd.resize(A.n);
#pragma omp parallel for schedule(static, 4096)
  for (int i = 0; i < A.n; ++i) {
    double l1 = 0.0;
    for (int k = A.rp[i]; k < A.rp[i + 1]; ++k) l1 += std::fabs(A.v[k]);
    invd[i] = l1 > kEps ? 1.0 / l1 : 0.0;
  }
}

// SPAI(0): m_i = a_ii / sum_j a_ij^2, the minimiser of ||e_i - m_i A_i,:||,
// 0 for a zero row; products and sums rounded separately, in column order.
void spai0_diagonal(const CSR& A, std::vector<double>& m) {
  m.resize(A.n);
#pragma omp parallel for schedule(static, 4096)
  for (int i = 0; i < A.n; ++i) {
    double d = 0.0, s = 0.0;
    for (int k = A.rp[i]; k < A.rp[i + 1]; ++k) {
      s += A.v[k] * A.v[k];
      if (A.ci[k] == i) d = A.v[k];
    }
    m[i] = s > 0.0 ? d / s : 0.0;
  }
}

double spectral_radius_estimate(const CSR& A, const std::vector<double>& invd, std::vector<double>& v,
                                int niter) {
  const int n = A.n;
  std::vector<double> w(n);
  double lam = 1.0;
  for (int it = 0; it < niter; ++it) {
#pragma omp parallel for schedule(static, 4096)
    for (int i = 0; i < n; ++i) {
      double s = 0.0;
      for (int k = A.rp[i]; k < A.rp[i + 1]; ++k) s += A.v[k] * v[A.ci[k]];
      w[i] = s * invd[i];
    }
    double ss = 0.0;
    for (int i = 0; i < n; ++i) ss += w[i] * w[i];
    lam = std::sqrt(ss);
    if (lam > kEps)
      for (int i = 0; i < n; ++i) v[i] = w[i] / lam;
  }
  return lam;
}

void chebyshev_coefficients(double rho, int degree, std::vector<double>& coef) {
  const double lmax = 1.1 * rho;
  const double lmin = lmax / 30.0;
  const double theta = (lmax + lmin) / 2.0;
  const double delta = (lmax - lmin) / 2.0;
  coef.assign(2 * (size_t)degree, 0.0);
  coef[0] = 1.0 / theta;
  double s_old = theta / delta;
  for (int k = 1; k < degree; ++k) {
    const double s_new = 1.0 / (2.0 * theta / delta - s_old);
    coef[2 * k] = 2.0 * s_new / delta;
    coef[2 * k + 1] = s_new * s_old;
    s_old = s_new;
  }
}

void csr_to_dense(const CSR& A, std::vector<double>& M) {
  const int n = A.n;
  M.assign((size_t)n * n, 0.0);
  for (int i = 0; i < n; ++i)
    for (int k = A.rp[i]; k < A.rp[i + 1]; ++k) M[(size_t)A.ci[k] * n + i] = A.v[k];
}

// Unblocked LU with partial pivoting, column-major (LAPACK dgetf2 order:
// pivot = first row of maximum magnitude, column scaled by the reciprocal
// of the pivot, rank-1 update of the trailing matrix).  A zero pivot is an
// error, as Julia's lu(A) throws SingularException for it.
void dense_lu(int n, std::vector<double>& a, std::vector<int>& piv) {
  piv.resize(n);
  for (int j = 0; j < n; ++j) {
    int p = j;
    double mx = std::fabs(a[(size_t)j * n + j]);
    for (int i = j + 1; i < n; ++i) {
      double v = std::fabs(a[(size_t)j * n + i]);
      if (v > mx) { mx = v; p = i; }
    }
    piv[j] = p;
    if (a[(size_t)j * n + p] == 0.0) fail("SingularException(" + std::to_string(j + 1) + ")");
    if (p != j)
      for (int c = 0; c < n; ++c) std::swap(a[(size_t)c * n + j], a[(size_t)c * n + p]);
    const double r = 1.0 / a[(size_t)j * n + j];
    for (int i = j + 1; i < n; ++i) a[(size_t)j * n + i] = a[(size_t)j * n + i] * r;
    for (int c = j + 1; c < n; ++c) {
      const double t = a[(size_t)c * n + j];
      for (int i = j + 1; i < n; ++i) {
        const double prod = a[(size_t)j * n + i] * t;
        a[(size_t)c * n + i] = a[(size_t)c * n + i] - prod;
      }
    }
  }
}

// ------------------------------------------------------------ level loop
namespace {

// cf receives the C/F splitting (empty for aggregation).
void coarsen_and_build_p(const CSR& A, const Coarsening& alg, const Config& cfg, uint64_t& rng,
                         Prolong& P, int& nc, std::vector<int>& cf) {
  std::vector<int> cmap;
  cf.clear();
  switch (alg.kind) {
    case CoarsenKind::PMIS:
    case CoarsenKind::HMIS:
    case CoarsenKind::RS: {  // coarsen_cf (coarsening.jl:1157-1187)
      CSR Aw;
      const CSR* Ap = &A;
      if (cfg.max_row_sum < 1.0) { Aw = apply_max_row_sum(A, cfg.max_row_sum); Ap = &Aw; }
      if (alg.kind == CoarsenKind::PMIS) coarsen_pmis(*Ap, alg.theta, rng, cf, cmap, nc);
      else if (alg.kind == CoarsenKind::HMIS) coarsen_hmis(*Ap, alg.theta, rng, cf, cmap, nc);
      else coarsen_rs(*Ap, alg.theta, cf, cmap, nc);
      P = build_interpolation(A, cf, cmap, nc, alg.interp, alg.theta);
      if (alg.interp.trunc_factor > 0) P = truncate_interpolation(P, alg.interp.trunc_factor);
      return;
    }
    case CoarsenKind::AggressivePMIS:
    case CoarsenKind::AggressiveHMIS: {
      coarsen_aggressive_cf(A, alg.theta, alg.kind == CoarsenKind::AggressiveHMIS, cfg, rng, cf,
                            cmap, nc);
      P = build_interpolation(A, cf, cmap, nc, alg.interp, alg.theta);
      if (alg.interp.trunc_factor > 0) P = truncate_interpolation(P, alg.interp.trunc_factor);
      return;
    }
    case CoarsenKind::Aggregation:
    case CoarsenKind::SmoothedAggregation: {
      std::vector<int> agg;
      if (cfg.max_row_sum < 1.0) coarsen_aggregation(apply_max_row_sum(A, cfg.max_row_sum), alg.theta, agg, nc);
      else coarsen_aggregation(A, alg.theta, agg, nc);
      P = build_aggregation_prolongation(A.n, agg, nc);
      if (alg.kind == CoarsenKind::SmoothedAggregation) P = smooth_prolongation(A, P, alg.sa_omega);
      if (alg.filtering) P = filter_prolongation(P, alg.filter_tol);
      return;
    }
  }
}

void coarsen_with_fallback(const CSR& A, const Coarsening& alg, const Config& cfg, uint64_t& rng,
                           Prolong& P, int& nc, std::vector<int>& cf) {
  const int n = A.n;
  coarsen_and_build_p(A, alg, cfg, rng, P, nc, cf);
  if (nc < 0.8 * n || n <= cfg.max_coarse_size) return;
  for (int attempt = 1; attempt <= 3; ++attempt) {
    Coarsening red = alg;
    red.theta = alg.theta * std::pow(0.5, attempt);
    Prolong P2;
    int nc2 = 0;
    std::vector<int> cf2;
    coarsen_and_build_p(A, red, cfg, rng, P2, nc2, cf2);
    if (nc2 < nc) { P = std::move(P2); nc = nc2; cf = std::move(cf2); }
    if (nc < 0.8 * n) break;
  }
}

}  // namespace

void ilu0_diag_indices(const CSR& A, std::vector<int>& diag) {
  diag.assign(A.n, -1);
  for (int i = 0; i < A.n; ++i) {
    for (int k = A.rp[i]; k < A.rp[i + 1]; ++k)
      if (A.ci[k] == i) {
        diag[i] = k;
        break;
      }
    if (diag[i] < 0) fail("ILU(0) needs a diagonal entry in every row (row " + std::to_string(i) + ")");
  }
}

void ilu0_factorize(const CSR& A, const std::vector<int>& diag, std::vector<double>& L,
                    std::vector<double>& U) {
  const int n = A.n;
  U = A.v;
  L.assign(A.v.size(), 0.0);
  const double kMaxFactor = 1e8;
  std::vector<double> rn(n);
  for (int i = 0; i < n; ++i) {
    double s = 0.0;
    for (int k = A.rp[i]; k < A.rp[i + 1]; ++k) s += std::fabs(A.v[k]);
    rn[i] = s;
  }
  auto safe = [&](double scale) { return kEps * std::max(1.0, scale); };
  for (int i = 0; i < n; ++i) {
    const int rs = A.rp[i], re = A.rp[i + 1];
    for (int nz = rs; nz < diag[i]; ++nz) {
      const int k = A.ci[nz];
      const double ukk = U[diag[k]];
      if (std::fabs(ukk) < safe(rn[k])) {
        L[nz] = 0.0;
        U[nz] = 0.0;
        continue;
      }
      double lik = U[nz] / ukk;
      const double nl = std::fabs(lik);
      if (nl > kMaxFactor) lik = lik * (kMaxFactor / nl);
      L[nz] = lik;
      U[nz] = 0.0;
      for (int nk = diag[k] + 1; nk < A.rp[k + 1]; ++nk) {
        const int j = A.ci[nk];
        // binary search of column j in row i (_find_nz_in_row)
        int lo = rs, hi = re - 1, at = -1;
        while (lo <= hi) {
          const int mid = (lo + hi) >> 1;
          const int c = A.ci[mid];
          if (c == j) { at = mid; break; }
          if (c < j) lo = mid + 1;
          else hi = mid - 1;
        }
        if (at >= 0) U[at] -= lik * U[nk];
      }
    }
    const double thr = safe(rn[i]);
    if (std::fabs(U[diag[i]]) < thr) U[diag[i]] = thr;
  }
}

void ilu0_levels(const CSR& A, const std::vector<int>& diag, std::vector<int>& fwd_order,
                 std::vector<int>& fwd_off, std::vector<int>& bwd_order, std::vector<int>& bwd_off) {
  const int n = A.n;
  auto order_by = [&](const std::vector<int>& level, int nlev, std::vector<int>& order,
                      std::vector<int>& off) {
    off.assign(nlev + 1, 0);
    for (int i = 0; i < n; ++i) ++off[level[i]];  // levels are 1-based
    for (int c = 0; c < nlev; ++c) off[c + 1] += off[c];
    std::vector<int> pos(off.begin(), off.end() - 1);
    order.resize(n);
    for (int i = 0; i < n; ++i) order[pos[level[i] - 1]++] = i;
  };
  std::vector<int> lev(n);
  int nf = 0;
  for (int i = 0; i < n; ++i) {
    int m = 0;
    for (int nz = A.rp[i]; nz < diag[i]; ++nz) m = std::max(m, lev[A.ci[nz]]);
    lev[i] = m + 1;
    nf = std::max(nf, lev[i]);
  }
  order_by(lev, nf, fwd_order, fwd_off);
  int nb = 0;
  for (int i = n - 1; i >= 0; --i) {
    int m = 0;
    for (int nz = diag[i] + 1; nz < A.rp[i + 1]; ++nz) m = std::max(m, lev[A.ci[nz]]);
    lev[i] = m + 1;
    nb = std::max(nb, lev[i]);
  }
  order_by(lev, nb, bwd_order, bwd_off);
}

namespace {

}  // namespace

void serial_gs_levels(const CSR& A, std::vector<int>& order, std::vector<int>& off) {
  const int n = A.n;
  // rows j < i with a_ji != 0, per row i (CSR: lo_off / lo_src)
  std::vector<int> lo_off(n + 1, 0);
  for (int j = 0; j < n; ++j)
    for (int k = A.rp[j]; k < A.rp[j + 1]; ++k)
      if (A.ci[k] > j) ++lo_off[A.ci[k] + 1];
  for (int i = 0; i < n; ++i) lo_off[i + 1] += lo_off[i];
  std::vector<int> lo_src(lo_off[n]);
  {
    std::vector<int> pos(lo_off.begin(), lo_off.end() - 1);
    for (int j = 0; j < n; ++j)
      for (int k = A.rp[j]; k < A.rp[j + 1]; ++k)
        if (A.ci[k] > j) lo_src[pos[A.ci[k]]++] = j;
  }
  std::vector<int> lev(n);
  int nl = 0;
  for (int i = 0; i < n; ++i) {
    int m = 0;
    for (int k = A.rp[i]; k < A.rp[i + 1]; ++k)
      if (A.ci[k] < i) m = std::max(m, lev[A.ci[k]]);
    for (int q = lo_off[i]; q < lo_off[i + 1]; ++q) m = std::max(m, lev[lo_src[q]]);
    lev[i] = m + 1;
    nl = std::max(nl, lev[i]);
  }
  off.assign(nl + 1, 0);
  for (int i = 0; i < n; ++i) ++off[lev[i]];
  for (int c = 0; c < nl; ++c) off[c + 1] += off[c];
  std::vector<int> pos(off.begin(), off.end() - 1);
  order.resize(n);
  for (int i = 0; i < n; ++i) order[pos[lev[i] - 1]++] = i;
}

void serial_gs_inverse_diagonal(const CSR& A, std::vector<double>& invd) {
  invd.resize(A.n);
  for (int i = 0; i < A.n; ++i) {
    double d = 0.0;
    for (int k = A.rp[i]; k < A.rp[i + 1]; ++k)
      if (A.ci[k] == i) {
        d = A.v[k];
        break;
      }
    invd[i] = std::fabs(d) > kEps ? 1.0 / d : 0.0;
  }
}

namespace {

}  // namespace

namespace {

// Solve the k x k symmetric system G m = r (row-major G, overwritten) by the
// upper Cholesky factor (G = U^T U, LAPACK potf2 order); false when a pivot
// is not positive.
bool cholesky_solve(int k, std::vector<double>& G, const std::vector<double>& r, std::vector<double>& m) {
  for (int j = 0; j < k; ++j) {
    double s = G[(size_t)j * k + j];
    for (int t = 0; t < j; ++t) s -= G[(size_t)t * k + j] * G[(size_t)t * k + j];
    if (!(s > 0.0)) return false;
    const double ujj = std::sqrt(s);
    G[(size_t)j * k + j] = ujj;
    for (int l = j + 1; l < k; ++l) {
      double v = G[(size_t)j * k + l];
      for (int t = 0; t < j; ++t) v -= G[(size_t)t * k + j] * G[(size_t)t * k + l];
      G[(size_t)j * k + l] = v / ujj;
    }
  }
  m = r;
  for (int j = 0; j < k; ++j) {  // U^T y = r
    double v = m[j];
    for (int t = 0; t < j; ++t) v -= G[(size_t)t * k + j] * m[t];
    m[j] = v / G[(size_t)j * k + j];
  }
  for (int j = k - 1; j >= 0; --j) {  // U m = y
    double v = m[j];
    for (int t = j + 1; t < k; ++t) v -= G[(size_t)j * k + t] * m[t];
    m[j] = v / G[(size_t)j * k + j];
  }
  return true;
}

// Partial-pivoting LU solve of the k x k system (row-major G, overwritten);
// false on a zero pivot.
bool lu_solve_small(int k, std::vector<double>& G, const std::vector<double>& r, std::vector<double>& m) {
  m = r;
  for (int j = 0; j < k; ++j) {
    int p = j;
    for (int i = j + 1; i < k; ++i)
      if (std::fabs(G[(size_t)i * k + j]) > std::fabs(G[(size_t)p * k + j])) p = i;
    if (G[(size_t)p * k + j] == 0.0) return false;
    if (p != j) {
      for (int c = 0; c < k; ++c) std::swap(G[(size_t)p * k + c], G[(size_t)j * k + c]);
      std::swap(m[p], m[j]);
    }
    for (int i = j + 1; i < k; ++i) {
      const double f = G[(size_t)i * k + j] / G[(size_t)j * k + j];
      for (int c = j; c < k; ++c) G[(size_t)i * k + c] -= f * G[(size_t)j * k + c];
      m[i] -= f * m[j];
    }
  }
  for (int j = k - 1; j >= 0; --j) {
    double v = m[j];
    for (int c = j + 1; c < k; ++c) v -= G[(size_t)j * k + c] * m[c];
    m[j] = v / G[(size_t)j * k + j];
  }
  return true;
}

}  // namespace

void spai1_values(const CSR& A, std::vector<double>& M) {
  const int n = A.n;
  M.assign(A.v.size(), 0.0);
  // rows of each column, ascending (the transpose pattern)
  std::vector<int> cp(n + 1, 0), cr(A.ci.size());
  for (int c : A.ci) ++cp[c + 1];
  for (int j = 0; j < n; ++j) cp[j + 1] += cp[j];
  {
    std::vector<int> f(cp.begin(), cp.end() - 1);
    for (int r = 0; r < n; ++r)
      for (int k = A.rp[r]; k < A.rp[r + 1]; ++k) cr[f[A.ci[k]]++] = r;
  }
#pragma omp parallel
  {
    std::vector<int> loc(n, -1), rows;
    std::vector<double> G, rhs, m;
#pragma omp for schedule(dynamic, 256)
    for (int i = 0; i < n; ++i) {
      const int rs = A.rp[i], k = A.rp[i + 1] - rs;
      if (k == 0) continue;
      for (int p = 0; p < k; ++p) loc[A.ci[rs + p]] = p;
      rows.clear();
      for (int p = 0; p < k; ++p) {
        const int c = A.ci[rs + p];
        rows.insert(rows.end(), cr.begin() + cp[c], cr.begin() + cp[c + 1]);
      }
      std::sort(rows.begin(), rows.end());
      rows.erase(std::unique(rows.begin(), rows.end()), rows.end());
      G.assign((size_t)k * k, 0.0);
      for (int r : rows) {
        for (int a = A.rp[r]; a < A.rp[r + 1]; ++a) {
          const int p = loc[A.ci[a]];
          if (p < 0) continue;
          const double vp = A.v[a];
          for (int b = A.rp[r]; b < A.rp[r + 1]; ++b) {
            const int q = loc[A.ci[b]];
            if (q >= 0) G[(size_t)p * k + q] += vp * A.v[b];
          }
        }
      }
      rhs.assign(A.v.begin() + rs, A.v.begin() + rs + k);
      for (int p = 0; p < k; ++p) {
        double& g = G[(size_t)p * k + p];
        g += kEps * std::max(1.0, std::fabs(g));
      }
      std::vector<double> G2 = G;
      if (!cholesky_solve(k, G, rhs, m) && !lu_solve_small(k, G2, rhs, m)) m.assign(k, 0.0);
      for (int p = 0; p < k; ++p) M[rs + p] = m[p];
      for (int p = 0; p < k; ++p) loc[A.ci[rs + p]] = -1;
    }
  }
}

namespace {

// Normalised start vector of the Chebyshev power iteration: standard normal
// entries (Box-Muller on splitmix64 uniforms), divided by their 2-norm.
std::vector<double> chebyshev_start(int n, uint64_t seed) {
  std::vector<double> v(n);
  uint64_t s = seed;
  for (int i = 0; i < n; ++i) {
    const double u1 = 1.0 - rng_uniform(s);  // (0, 1]
    const double u2 = rng_uniform(s);
    v[i] = std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
  }
  double ss = 0.0;
  for (int i = 0; i < n; ++i) ss += v[i] * v[i];
  const double nv = std::sqrt(ss);
  if (nv > 0.0)
    for (int i = 0; i < n; ++i) v[i] /= nv;
  return v;
}

void build_smoother(HostLevel& L, const Config& cfg, int level) {
  L.smoother = cfg.smoother;
  L.omega = cfg.jacobi_omega;
  switch (cfg.smoother) {
    case SmootherKind::Jacobi:
      inverse_diagonal(L.A, L.invdiag);
      break;
    case SmootherKind::L1Jacobi:
      l1_inverse_diagonal(L.A, L.invdiag);
      break;
    case SmootherKind::SPAI0:  // x + m (b - A x): the Jacobi sweep with omega = 1
      spai0_diagonal(L.A, L.invdiag);
      L.omega = 1.0;
      break;
    case SmootherKind::SPAI1:  // build_spai1_smoother, smoothers.jl:598-607
      spai1_values(L.A, L.spai1_M);
      inverse_diagonal(L.A, L.invdiag);  // not used by the sweep; kept for exports
      break;
    case SmootherKind::SerialGS:   // build_serial_gs_smoother, smoothers.jl:370-376
    case SmootherKind::L1SerialGS:  // build_l1_serial_gs_smoother, :428-434
      if (cfg.smoother == SmootherKind::SerialGS) serial_gs_inverse_diagonal(L.A, L.invdiag);
      else l1_inverse_diagonal(L.A, L.invdiag);
      serial_gs_levels(L.A, L.sgs_order, L.sgs_off);
      break;
    case SmootherKind::ILU0:
    case SmootherKind::SerialILU0:
      // build_ilu0_smoother / build_serial_ilu0_smoother (smoothers.jl:1112-1126,
      // :1309-1330): the same factors; both substitute row by row in column
      // order, which the level schedule reproduces exactly
      ilu0_diag_indices(L.A, L.ilu_diag);
      ilu0_levels(L.A, L.ilu_diag, L.ilu_fwd_order, L.ilu_fwd_off, L.ilu_bwd_order, L.ilu_bwd_off);
      ilu0_factorize(L.A, L.ilu_diag, L.ilu_L, L.ilu_U);
      inverse_diagonal(L.A, L.invdiag);  // not used by the sweep; kept for exports
      break;
    case SmootherKind::Chebyshev: {  // build_chebyshev_smoother, smoothers.jl:895-910 (degree 3)
      inverse_diagonal(L.A, L.invdiag);
      L.cheb_degree = 3;
      L.cheb_v0 = chebyshev_start(L.A.n, cfg.seed ^ (0xC6EB5E5ULL * (uint64_t)(level + 1)));
      std::vector<double> v = L.cheb_v0;
      L.cheb_rho = spectral_radius_estimate(L.A, L.invdiag, v, 10);
      chebyshev_coefficients(L.cheb_rho, L.cheb_degree, L.cheb_coef);
      break;
    }
    case SmootherKind::ColoredGS:
      greedy_coloring(L.A, L.colors, L.num_colors);
      color_order_from(L.colors, L.num_colors, L.color_off, L.color_order);
      inverse_diagonal(L.A, L.invdiag);
      break;
    case SmootherKind::L1ColoredGS:
      greedy_coloring(L.A, L.colors, L.num_colors);
      color_order_from(L.colors, L.num_colors, L.color_off, L.color_order);
      l1_inverse_diagonal(L.A, L.invdiag);
      break;
    default:
      fail("smoother \"" + smoother_name(cfg.smoother) +
           "\" is not supported by the B200 build (use jacobi, l1_jacobi, spai0, spai1, "
           "chebyshev, ilu0, serial_ilu0, colored_gs, l1_colored_gs, serial_gs or l1_serial_gs)");
  }
}

}  // namespace

void build_hierarchy(const CSR& A_in, const Config& cfg, bool allow_partial_resetup, HostHierarchy& H,
                     GalerkinDevice* gdev) {
  auto t0 = std::chrono::steady_clock::now();
  validate_csr(A_in, "matrix");
  if (A_in.n != A_in.m) fail("matrix must be square");
  // Check the smoother before any work, so an unsupported choice fails fast.
  switch (cfg.smoother) {
    case SmootherKind::Jacobi: case SmootherKind::L1Jacobi: case SmootherKind::SPAI0:
    case SmootherKind::Chebyshev: case SmootherKind::ILU0: case SmootherKind::SerialILU0:
    case SmootherKind::SerialGS: case SmootherKind::L1SerialGS: case SmootherKind::SPAI1:
    case SmootherKind::ColoredGS: case SmootherKind::L1ColoredGS: break;
    default:
      fail("smoother \"" + smoother_name(cfg.smoother) +
           "\" is not supported by the B200 build (use jacobi, l1_jacobi, spai0, spai1, "
           "chebyshev, ilu0, serial_ilu0, colored_gs, l1_colored_gs, serial_gs or l1_serial_gs)");
  }
  H = HostHierarchy();
  H.cfg = cfg;
  H.allow_partial_resetup = allow_partial_resetup;
  uint64_t rng = cfg.seed;
  CSR cur = A_in;
  for (int lvl = 1; lvl <= cfg.max_levels - 1; ++lvl) {
    const int n = cur.n;
    if (n <= cfg.max_coarse_size) break;
    const Coarsening& alg = lvl <= cfg.initial_coarsening_levels ? cfg.initial_coarsening : cfg.coarsening;
    Prolong P;
    int nc = 0;
    std::vector<int> cf;
    coarsen_with_fallback(cur, alg, cfg, rng, P, nc, cf);
    if (nc >= n) break;
    if (nc == 0) break;
    HostLevel L;
    L.cf = std::move(cf);
    L.T = build_transpose_map(P);
    L.Rv.resize(P.nnz());
    for (size_t k = 0; k < L.T.pnz.size(); ++k) L.Rv[k] = P.v[L.T.pnz[k]];
    std::vector<int> ap_rp, ap_ci;
    std::vector<double> ap_v;
    CSR next;
    next.n = next.m = nc;
    if (!gdev || !gdev->galerkin(cur, P, L.T, L.Rv, ap_rp, ap_ci, ap_v, next)) {
      symbolic_ap(cur, P, ap_rp, ap_ci);
      numeric_ap(cur, P, ap_rp, ap_ci, ap_v);
      symbolic_ptap(L.T, nc, ap_rp, ap_ci, next.rp, next.ci);
      numeric_ptap(L.T, L.Rv, ap_rp, ap_ci, ap_v, next.rp, next.ci, next.v);
    }
    if (allow_partial_resetup) {
      L.has_rap_map = true;
      L.ap_rp = std::move(ap_rp);
      L.ap_ci = std::move(ap_ci);
    }
    L.A = std::move(cur);
    L.P = std::move(P);
    build_smoother(L, cfg, (int)H.levels.size());
    H.levels.push_back(std::move(L));
    cur = std::move(next);
  }
  H.coarse = std::move(cur);
  H.nc = H.coarse.n;
  csr_to_dense(H.coarse, H.coarse_dense);
  H.coarse_lu = H.coarse_dense;
  dense_lu(H.nc, H.coarse_lu, H.coarse_piv);
  H.setup_seconds =
      std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

namespace {
// The smoother's configuration type name and its per-level display name, as
// the reference's verbose setup print shows them (src/setup.jl:426, :478-488).
const char* smoother_type_name(SmootherKind k) {
  switch (k) {
    case SmootherKind::Jacobi: return "JacobiSmootherType";
    case SmootherKind::ColoredGS: return "ColoredGaussSeidelType";
    case SmootherKind::SerialGS: return "SerialGaussSeidelType";
    case SmootherKind::SPAI0: return "SPAI0SmootherType";
    case SmootherKind::SPAI1: return "SPAI1SmootherType";
    case SmootherKind::L1Jacobi: return "L1JacobiSmootherType";
    case SmootherKind::L1ColoredGS: return "L1ColoredGaussSeidelType";
    case SmootherKind::L1SerialGS: return "L1SerialGaussSeidelType";
    case SmootherKind::Chebyshev: return "ChebyshevSmootherType";
    case SmootherKind::ILU0: return "ILU0SmootherType";
    case SmootherKind::SerialILU0: return "SerialILU0SmootherType";
  }
  return "?";
}

const char* smoother_display_name(SmootherKind k) {
  switch (k) {
    case SmootherKind::Jacobi: return "Jacobi";
    case SmootherKind::ColoredGS: return "Colored GS";
    case SmootherKind::SerialGS: return "Serial GS";
    case SmootherKind::SPAI0: return "SPAI(0)";
    case SmootherKind::SPAI1: return "SPAI(1)";
    case SmootherKind::L1Jacobi: return "l1-Jacobi";
    case SmootherKind::L1ColoredGS: return "l1-Colored GS";
    case SmootherKind::L1SerialGS: return "l1-Serial GS";
    case SmootherKind::Chebyshev: return "Chebyshev";
    case SmootherKind::ILU0: return "ILU(0)";
    case SmootherKind::SerialILU0: return "Serial ILU(0)";
  }
  return "?";
}
}  // namespace

std::string hierarchy_summary(const HostHierarchy& H, int n_finest) {
  // Layout of _print_hierarchy_info, src/setup.jl:405-473.
  std::ostringstream o;
  char buf[256];
  const Config& c = H.cfg;
  int nl = (int)H.levels.size();
  o << "+=============================================================================+\n";
  o << "                         AMG Hierarchy Summary                                  \n";
  o << "+=============================================================================+\n";
  std::snprintf(buf, sizeof buf, "  Setup time:      %.4f s\n", H.setup_seconds); o << buf;
  o << "  Levels:          " << nl + 1 << " (" << nl << " AMG + 1 coarse direct)\n";
  o << "  Cycle type:      " << (c.cycle_w ? "W" : "V") << "-cycle\n";
  o << "  Backend:         CUDA (sm_100a)\n";
  o << "  Block size:      256 (row kernels on rows of 12-32 entries: 128)\n";
  o << "  Coarse solve:    "
    << (c.coarse_solve_on_cpu ? "GPU (coarse_solve_on_cpu requested; same LU solve, same values)" : "GPU")
    << "\n";
  o << "  Strength:        " << (c.strength == StrengthKind::Absolute ? "AbsoluteStrength" : "SignedStrength") << "\n";
  o << "  Coarsening:      " << coarsening_name(c.coarsening) << "\n";
  if (c.initial_coarsening_levels > 0)
    o << "  Initial coars.:  " << coarsening_name(c.initial_coarsening) << " (first "
      << c.initial_coarsening_levels << " levels)\n";
  o << "  Smoother:        " << smoother_type_name(c.smoother) << "\n";
  if (c.smoother == SmootherKind::Jacobi || c.smoother == SmootherKind::L1Jacobi) {
    std::snprintf(buf, sizeof buf, "    omega = %.3f\n", c.jacobi_omega); o << buf;
  }
  std::snprintf(buf, sizeof buf, "  Pre-smooth:      %d steps, Post-smooth: %d steps\n",
                c.pre_smoothing_steps, c.post_smoothing_steps); o << buf;
  if (c.max_row_sum < 1.0) {
    std::snprintf(buf, sizeof buf, "  Max row sum:     %.2f\n", c.max_row_sum); o << buf;
  }
  o << "+-------+----------+-----------+---------+------------------------------------+\n";
  o << "  Level     Rows        NNZ      Ratio    Smoother                              \n";
  o << "+-------+----------+-----------+---------+------------------------------------+\n";
  int64_t tot_nnz = 0, tot_rows = 0;
  for (int i = 0; i < nl; ++i) {
    const auto& L = H.levels[i];
    tot_nnz += L.A.nnz();
    tot_rows += L.A.n;
    if (i == 0)
      std::snprintf(buf, sizeof buf, "  %5d   %7d    %8lld        -   %s\n", i + 1, L.A.n,
                    (long long)L.A.nnz(), smoother_display_name(L.smoother));
    else
      std::snprintf(buf, sizeof buf, "  %5d   %7d    %8lld    %5.3f   %s\n", i + 1, L.A.n,
                    (long long)L.A.nnz(), (double)L.A.n / H.levels[i - 1].A.n,
                    smoother_display_name(L.smoother));
    o << buf;
  }
  int64_t cnz = 0;
  for (double v : H.coarse_dense) cnz += (v != 0.0);
  tot_nnz += cnz;
  tot_rows += H.nc;
  if (nl > 0)
    std::snprintf(buf, sizeof buf, "  %5d   %7d    %8lld    %5.3f   %s\n", nl + 1, H.nc, (long long)cnz,
                  (double)H.nc / H.levels[nl - 1].A.n, "Direct (LU)");
  else
    std::snprintf(buf, sizeof buf, "  %5d   %7d    %8lld         -   %s\n", nl + 1, H.nc, (long long)cnz,
                  "Direct (LU)");
  o << buf;
  o << "+=============================================================================+\n";
  if (nl > 0) {
    std::snprintf(buf, sizeof buf, "  Operator complexity: %.3f\n",
                  (double)tot_nnz / (double)H.levels[0].A.nnz()); o << buf;
    std::snprintf(buf, sizeof buf, "  Grid complexity:     %.3f\n", (double)tot_rows / n_finest); o << buf;
  }
  o << "+=============================================================================+\n";
  return o.str();
}

}  // namespace dr
