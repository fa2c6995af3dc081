// Interpolation (prolongation) construction (CPU setup phase).
//
//   aggregation P        src/prolongation.jl:8-22
//   smoothed aggregation src/prolongation.jl:38-128
//   filter / truncate    src/prolongation.jl:134-186, src/setup.jl:348-384
//   direct               src/prolongation.jl:219-330
//   standard             src/prolongation.jl:345-455
//   extended+i           src/prolongation.jl:467-690
//   COO -> CSR           src/prolongation.jl:713-736 (sort by (row, col))
//
// Rows are independent, so each routine runs its row loop in parallel with
// thread-private marker arrays and assembles the rows in ascending order; the
// per-row arithmetic (and so every value) is the same as a sequential sweep.
#include <omp.h>

#include <algorithm>
#include <cmath>
#include <limits>
#include <map>
#include <numeric>

#include "dr_host.h"

namespace dr {

static const double kEps = std::numeric_limits<double>::epsilon();

namespace {
struct RowBuf {
  std::vector<int> row, col;
  std::vector<double> val, scale;
};

// Stable sort of every row by column (the (row, col) sortperm of
// _coo_to_prolongation, src/prolongation.jl:713-736).
void sort_rows_by_col(Prolong& P) {
  const int nf = P.nf;
  const bool with_scale = P.has_trunc_scaling;
#pragma omp parallel
  {
    std::vector<int> perm;
    std::vector<int> c2;
    std::vector<double> v2, s2;
#pragma omp for schedule(static, 4096)
    for (int i = 0; i < nf; ++i) {
      int s = P.rp[i], e = P.rp[i + 1];
      bool sorted = true;
      for (int k = s + 1; k < e; ++k)
        if (P.ci[k] < P.ci[k - 1]) { sorted = false; break; }
      if (sorted) continue;
      perm.resize(e - s);
      std::iota(perm.begin(), perm.end(), 0);
      std::stable_sort(perm.begin(), perm.end(),
                       [&](int x, int y) { return P.ci[s + x] < P.ci[s + y]; });
      c2.resize(e - s);
      v2.resize(e - s);
      s2.resize(e - s);
      for (int t = 0; t < e - s; ++t) {
        c2[t] = P.ci[s + perm[t]];
        v2[t] = P.v[s + perm[t]];
        if (with_scale) s2[t] = P.trunc_scaling[s + perm[t]];
      }
      for (int t = 0; t < e - s; ++t) {
        P.ci[s + t] = c2[t];
        P.v[s + t] = v2[t];
        if (with_scale) P.trunc_scaling[s + t] = s2[t];
      }
    }
  }
}

// Assemble per-thread row buffers (each holding a contiguous ascending row
// range) into a CSR prolongation, sorting every row by column (stable).
Prolong assemble(int nf, int nc, std::vector<RowBuf>& bufs, bool with_scale) {
  Prolong P;
  P.nf = nf;
  P.nc = nc;
  P.rp.assign(nf + 1, 0);
  for (auto& b : bufs)
    for (int r : b.row) P.rp[r + 1]++;
  for (int i = 0; i < nf; ++i) P.rp[i + 1] += P.rp[i];
  P.ci.resize(P.rp[nf]);
  P.v.resize(P.rp[nf]);
  if (with_scale) {
    P.has_trunc_scaling = true;
    P.trunc_scaling.resize(P.rp[nf]);
  }
  std::vector<int> pos(P.rp.begin(), P.rp.end() - 1);
  for (auto& b : bufs)
    for (size_t t = 0; t < b.row.size(); ++t) {
      int p = pos[b.row[t]]++;
      P.ci[p] = b.col[t];
      P.v[p] = b.val[t];
      if (with_scale) P.trunc_scaling[p] = b.scale[t];
    }
  sort_rows_by_col(P);
  return P;
}

int nearest_coarse(const CSR& A, int i, const std::vector<int>& cf, const std::vector<int>& cmap) {
  int best = -1;
  double bv = 0.0;
  for (int k = A.rp[i]; k < A.rp[i + 1]; ++k) {
    int j = A.ci[k];
    if (j == i) continue;
    if (cf[j] == 1 && std::fabs(A.v[k]) > bv) { bv = std::fabs(A.v[k]); best = cmap[j]; }
  }
  return best >= 0 ? best : 0;
}

inline double sgn(double x) { return x > 0 ? 1.0 : (x < 0 ? -1.0 : 0.0); }

inline double powi(double x, int p) {
  if (p == 1) return x;
  double r = 1.0;
  for (int t = 0; t < p; ++t) r *= x;
  return r;
}
}  // namespace

Prolong build_aggregation_prolongation(int nf, const std::vector<int>& agg, int nc) {
  Prolong P;
  P.nf = nf;
  P.nc = nc;
  P.rp.resize(nf + 1);
  P.ci.resize(nf);
  P.v.assign(nf, 1.0);
  for (int i = 0; i < nf; ++i) {
    P.rp[i] = i;
    P.ci[i] = agg[i];
  }
  P.rp[nf] = nf;
  return P;
}

Prolong filter_prolongation(const Prolong& P, double tol) {
  Prolong Q;
  Q.nf = P.nf;
  Q.nc = P.nc;
  Q.rp.assign(P.nf + 1, 0);
  Q.has_trunc_scaling = P.has_trunc_scaling;
  for (int i = 0; i < P.nf; ++i) {
    int s = P.rp[i], e = P.rp[i + 1];
    if (s < e) {
      double mx = 0.0;
      for (int k = s; k < e; ++k) mx = std::max(mx, std::fabs(P.v[k]));
      double thr = tol * mx;
      int cnt = 0;
      for (int k = s; k < e; ++k)
        if (std::fabs(P.v[k]) >= thr) {
          Q.ci.push_back(P.ci[k]);
          Q.v.push_back(P.v[k]);
          if (P.has_trunc_scaling) Q.trunc_scaling.push_back(P.trunc_scaling[k]);
          ++cnt;
        }
      if (cnt == 0) {
        int best = s;
        double bv = 0.0;
        for (int k = s; k < e; ++k)
          if (std::fabs(P.v[k]) > bv) { bv = std::fabs(P.v[k]); best = k; }
        Q.ci.push_back(P.ci[best]);
        Q.v.push_back(P.v[best]);
        if (P.has_trunc_scaling) Q.trunc_scaling.push_back(P.trunc_scaling[best]);
      }
    }
    Q.rp[i + 1] = (int)Q.ci.size();
  }
  sort_rows_by_col(Q);
  return Q;
}

Prolong truncate_interpolation(const Prolong& P, double tf) {
  // _filter_prolongation with the same threshold, trunc_scaling filtered in
  // step (src/setup.jl:348-384).
  return filter_prolongation(P, tf);
}

Prolong smooth_prolongation(const CSR& A, const Prolong& Pt, double omega) {
  const int nf = Pt.nf, nc = Pt.nc;
  std::vector<double> invd(nf);
  for (int i = 0; i < nf; ++i) {
    double d = 0.0;
    for (int k = A.rp[i]; k < A.rp[i + 1]; ++k)
      if (A.ci[k] == i) { d = A.v[k]; break; }
    double thr = kEps * std::max(1.0, std::fabs(d));
    invd[i] = std::fabs(d) > thr ? 1.0 / d : 0.0;
  }
  int nt = omp_get_max_threads();
  std::vector<RowBuf> bufs(nt);
#pragma omp parallel
  {
    RowBuf& B = bufs[omp_get_thread_num()];
    std::vector<double> acc(nc, 0.0);
    std::vector<int> mark(nc, -1), keys;
#pragma omp for schedule(static)
    for (int i = 0; i < nf; ++i) {
      keys.clear();
      auto add = [&](int J, double x) {
        if (mark[J] != i) { mark[J] = i; acc[J] = 0.0; keys.push_back(J); }
        acc[J] += x;
      };
      for (int p = Pt.rp[i]; p < Pt.rp[i + 1]; ++p) add(Pt.ci[p], Pt.v[p]);
      double f = -omega * invd[i];
      for (int k = A.rp[i]; k < A.rp[i + 1]; ++k) {
        int j = A.ci[k];
        if (j < 0 || j >= nf) continue;
        double w = f * A.v[k];
        for (int p = Pt.rp[j]; p < Pt.rp[j + 1]; ++p) add(Pt.ci[p], w * Pt.v[p]);
      }
      bool found = false;
      for (int J : keys)
        if (std::fabs(acc[J]) > kEps) {
          B.row.push_back(i); B.col.push_back(J); B.val.push_back(acc[J]);
          found = true;
        }
      if (!found && Pt.rp[i] < Pt.rp[i + 1]) {
        B.row.push_back(i); B.col.push_back(Pt.ci[Pt.rp[i]]); B.val.push_back(Pt.v[Pt.rp[i]]);
      }
    }
  }
  return assemble(nf, nc, bufs, false);
}

static Prolong interp_direct(const CSR& A, const std::vector<int>& cf, const std::vector<int>& cmap,
                             int nc, double theta) {
  const int nf = A.n;
  std::vector<uint8_t> st = strength_absolute(A, theta);
  int nt = omp_get_max_threads();
  std::vector<RowBuf> bufs(nt);
#pragma omp parallel
  {
    RowBuf& B = bufs[omp_get_thread_num()];
#pragma omp for schedule(static)
    for (int i = 0; i < nf; ++i) {
      if (cf[i] == 1) {
        B.row.push_back(i); B.col.push_back(cmap[i]); B.val.push_back(1.0);
        continue;
      }
      double aii = 0.0, ds = 0.0;
      for (int k = A.rp[i]; k < A.rp[i + 1]; ++k)
        if (A.ci[k] == i) { aii = A.v[k]; ds = sgn(aii); }
      double sum_nonc = 0.0;
      size_t first = B.row.size();
      std::vector<double> vals;
      std::vector<int> cols;
      for (int k = A.rp[i]; k < A.rp[i + 1]; ++k) {
        int j = A.ci[k];
        if (j == i) continue;
        bool ic = st[k] && cf[j] == 1 && (ds == 0 || sgn(A.v[k]) != ds);
        if (ic) { cols.push_back(cmap[j]); vals.push_back(A.v[k]); }
        else sum_nonc += A.v[k];
      }
      (void)first;
      double di = aii + sum_nonc;
      if (cols.empty()) {
        int best = -1;
        double bv = 0.0;
        for (int k = A.rp[i]; k < A.rp[i + 1]; ++k) {
          int j = A.ci[k];
          if (j == i) continue;
          if (cf[j] == 1 && std::fabs(A.v[k]) > bv) { bv = std::fabs(A.v[k]); best = cmap[j]; }
        }
        if (best < 0) best = 0;
        B.row.push_back(i); B.col.push_back(best); B.val.push_back(1.0);
      } else {
        double thr = kEps * std::max(1.0, std::fabs(di));
        for (size_t t = 0; t < cols.size(); ++t) {
          B.row.push_back(i); B.col.push_back(cols[t]);
          B.val.push_back(std::fabs(di) > thr ? -vals[t] / di : 0.0);
        }
      }
    }
  }
  // direct interpolation keeps the A-row order (no sort), src/prolongation.jl:262-330
  Prolong P;
  P.nf = nf;
  P.nc = nc;
  P.rp.assign(nf + 1, 0);
  for (auto& b : bufs)
    for (int r : b.row) P.rp[r + 1]++;
  for (int i = 0; i < nf; ++i) P.rp[i + 1] += P.rp[i];
  P.ci.resize(P.rp[nf]);
  P.v.resize(P.rp[nf]);
  std::vector<int> pos(P.rp.begin(), P.rp.end() - 1);
  for (auto& b : bufs)
    for (size_t t = 0; t < b.row.size(); ++t) {
      int p = pos[b.row[t]]++;
      P.ci[p] = b.col[t];
      P.v[p] = b.val[t];
    }
  return P;
}

static Prolong interp_standard(const CSR& A, const std::vector<int>& cf, const std::vector<int>& cmap,
                               int nc, double theta) {
  const int nf = A.n;
  std::vector<uint8_t> st = strength_absolute(A, theta);
  int nt = omp_get_max_threads();
  std::vector<RowBuf> bufs(nt);
#pragma omp parallel
  {
    RowBuf& B = bufs[omp_get_thread_num()];
#pragma omp for schedule(static)
    for (int i = 0; i < nf; ++i) {
      if (cf[i] == 1) {
        B.row.push_back(i); B.col.push_back(cmap[i]); B.val.push_back(1.0);
        continue;
      }
      double aii = 0.0, sum_weak = 0.0;
      std::map<int, double> strong_coarse;   // coarse id -> a_ij
      std::vector<std::pair<int, double>> strong_fine;
      for (int k = A.rp[i]; k < A.rp[i + 1]; ++k) {
        int j = A.ci[k];
        if (j == i) aii = A.v[k];
        else if (st[k] && cf[j] == 1) strong_coarse[cmap[j]] += A.v[k];
        else if (st[k] && cf[j] == -1) strong_fine.push_back({j, A.v[k]});
        else sum_weak += A.v[k];
      }
      double di = aii + sum_weak;
      std::map<int, double> contrib(strong_coarse.begin(), strong_coarse.end());
      for (auto& kf : strong_fine) {
        int kk = kf.first;
        double aik = kf.second;
        double dk = 0.0;
        for (int q = A.rp[kk]; q < A.rp[kk + 1]; ++q)
          if (A.ci[q] == kk) { dk = A.v[q]; break; }
        double s = dk < 0 ? -1.0 : 1.0;
        double sumck = 0.0;
        std::map<int, double> cvk;
        for (int q = A.rp[kk]; q < A.rp[kk + 1]; ++q) {
          int j2 = A.ci[q];
          if (j2 == kk) continue;
          double akj = A.v[q];
          if (cf[j2] == 1) {
            int cm2 = cmap[j2];
            if (strong_coarse.count(cm2) && s * akj < 0) { cvk[cm2] += akj; sumck += akj; }
          }
          if (j2 == i && s * akj < 0) sumck += akj;
        }
        if (std::fabs(sumck) > kEps) {
          double dist = aik / sumck;
          for (auto& e : cvk) contrib[e.first] += dist * e.second;
          for (int q = A.rp[kk]; q < A.rp[kk + 1]; ++q)
            if (A.ci[q] == i && s * A.v[q] < 0) { di += dist * A.v[q]; break; }
        } else {
          di += aik;
        }
      }
      if (contrib.empty()) {
        B.row.push_back(i); B.col.push_back(nearest_coarse(A, i, cf, cmap)); B.val.push_back(1.0);
      } else {
        for (auto& e : contrib) {
          double w = std::fabs(di) > kEps ? -e.second / di : 0.0;
          B.row.push_back(i); B.col.push_back(e.first); B.val.push_back(w);
        }
      }
    }
  }
  return assemble(nf, nc, bufs, false);
}

static Prolong interp_ext_i(const CSR& A, const std::vector<int>& cf, const std::vector<int>& cmap,
                            int nc, const Interp& ip, double theta) {
  const int nf = A.n;
  std::vector<uint8_t> st = strength_absolute(A, theta);
  const double tf = ip.trunc_factor;
  const int maxel = ip.max_elements;
  const int np = ip.norm_p;
  const bool resc = ip.rescale;
  int nt = omp_get_max_threads();
  std::vector<RowBuf> bufs(nt);
#pragma omp parallel
  {
    RowBuf& B = bufs[omp_get_thread_num()];
    std::vector<int> marker(nf, -1);
    std::vector<int> chat;
    std::vector<double> pdata;
    std::vector<int> keep;
    std::vector<char> kept;
#pragma omp for schedule(static)
    for (int i = 0; i < nf; ++i) {
      if (cf[i] == 1) {
        B.row.push_back(i); B.col.push_back(cmap[i]); B.val.push_back(1.0);
        if (resc) B.scale.push_back(1.0);
        continue;
      }
      const int SF = -2 - i;  // row-unique strong-F marker
      chat.clear();
      // Phase 1: C-hat = strong C nbrs of i and strong C nbrs of its strong F nbrs.
      for (int k = A.rp[i]; k < A.rp[i + 1]; ++k) {
        int j = A.ci[k];
        if (j == i || !st[k]) continue;
        if (cf[j] == 1) {
          if (marker[j] < 0) { marker[j] = (int)chat.size(); chat.push_back(j); }
        } else if (cf[j] == -1) {
          marker[j] = SF;
          for (int k2 = A.rp[j]; k2 < A.rp[j + 1]; ++k2) {
            int q = A.ci[k2];
            if (q == j || !st[k2]) continue;
            if (cf[q] == 1 && marker[q] < 0) { marker[q] = (int)chat.size(); chat.push_back(q); }
          }
        }
      }
      auto reset = [&]() {
        for (int j : chat) marker[j] = -1;
        for (int k = A.rp[i]; k < A.rp[i + 1]; ++k) {
          int j = A.ci[k];
          if (j == i || !st[k]) continue;
          marker[j] = -1;
          if (cf[j] == -1)
            for (int k2 = A.rp[j]; k2 < A.rp[j + 1]; ++k2) {
              int q = A.ci[k2];
              if (q == j || !st[k2]) continue;
              marker[q] = -1;
            }
        }
      };
      const int nch = (int)chat.size();
      if (nch == 0) {
        B.row.push_back(i); B.col.push_back(nearest_coarse(A, i, cf, cmap)); B.val.push_back(1.0);
        if (resc) B.scale.push_back(1.0);
        reset();
        continue;
      }
      // Phase 2: weights (hypre ExtPI formula).
      pdata.assign(nch, 0.0);
      double diag = 0.0;
      for (int k = A.rp[i]; k < A.rp[i + 1]; ++k) {
        int j = A.ci[k];
        double aij = A.v[k];
        if (j == i) { diag += aij; continue; }
        int pidx = marker[j];
        if (pidx >= 0) {
          pdata[pidx] += aij;
        } else if (pidx == SF) {
          double dj = 0.0;
          for (int q = A.rp[j]; q < A.rp[j + 1]; ++q)
            if (A.ci[q] == j) { dj = A.v[q]; break; }
          double s = dj < 0 ? -1.0 : 1.0;
          double sum = 0.0;
          for (int q = A.rp[j]; q < A.rp[j + 1]; ++q) {
            int mm = A.ci[q];
            if (mm == j) continue;
            double ajm = A.v[q];
            if (s * ajm < 0 && (marker[mm] >= 0 || mm == i)) sum += ajm;
          }
          if (std::fabs(sum) > kEps) {
            double dist = aij / sum;
            for (int q = A.rp[j]; q < A.rp[j + 1]; ++q) {
              int mm = A.ci[q];
              if (mm == j) continue;
              double ajm = A.v[q];
              if (s * ajm < 0) {
                int pm = marker[mm];
                if (pm >= 0) pdata[pm] += dist * ajm;
                else if (mm == i) diag += dist * ajm;
              }
            }
          } else {
            diag += aij;
          }
        } else {
          diag += aij;
        }
      }
      // Phase 3: normalise.
      if (std::fabs(diag) > kEps)
        for (int t = 0; t < nch; ++t) pdata[t] /= -diag;
      // Phase 4: truncation and max_elements.
      keep.resize(nch);
      std::iota(keep.begin(), keep.end(), 0);
      if (tf > 0) {
        double mw = 0.0;
        for (int t = 0; t < nch; ++t) mw = std::max(mw, powi(std::fabs(pdata[t]), np));
        double thr = tf * mw;
        keep.clear();
        for (int t = 0; t < nch; ++t)
          if (powi(std::fabs(pdata[t]), np) >= thr) keep.push_back(t);
      }
      if (maxel > 0 && (int)keep.size() > maxel) {
        std::stable_sort(keep.begin(), keep.end(),
                         [&](int x, int y) { return std::fabs(pdata[x]) > std::fabs(pdata[y]); });
        keep.resize(maxel);
      }
      double row_scale = 1.0;
      if (resc && (int)keep.size() < nch) {
        kept.assign(nch, 0);
        for (int t : keep) kept[t] = 1;
        double removed = 0.0;
        for (int t = 0; t < nch; ++t)
          if (!kept[t]) removed += pdata[t];
        double denom = 1.0 - removed;
        if (std::fabs(denom) > 1e-12) row_scale = 1.0 / denom;
      }
      for (int t : keep) {
        B.row.push_back(i);
        B.col.push_back(cmap[chat[t]]);
        B.val.push_back(pdata[t] * row_scale);
        if (resc) B.scale.push_back(row_scale);
      }
      reset();
    }
  }
  return assemble(nf, nc, bufs, resc);
}

Prolong build_interpolation(const CSR& A, const std::vector<int>& cf, const std::vector<int>& cmap,
                            int nc, const Interp& ip, double theta) {
  switch (ip.kind) {
    case InterpKind::Direct: return interp_direct(A, cf, cmap, nc, theta);
    case InterpKind::Standard: return interp_standard(A, cf, cmap, nc, theta);
    case InterpKind::ExtendedI: return interp_ext_i(A, cf, cmap, nc, ip, theta);
  }
  fail("unknown interpolation");
}

}  // namespace dr
