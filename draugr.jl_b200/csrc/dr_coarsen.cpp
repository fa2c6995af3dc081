// Strength of connection and coarsening (CPU setup phase).
//
// These routines produce the C/F splitting or aggregates that define the
// hierarchy structure.  They follow the sequential algorithms of Draugr.jl
// step by step (same visiting orders, same tie-breaking), so that for the
// same random measures the same splitting results:
//   strength         src/strength.jl:24-76 (absolute), :78-150 (signed),
//                    :183-218 (max row sum)
//   aggregation      src/coarsening.jl:14-171
//   PMIS             src/coarsening.jl:202-289
//   HMIS             src/coarsening.jl:330-404, RS first pass :406-573,
//                    PMIS on undecided :575-630
//   aggressive CF    src/coarsening.jl:990-1112
// The reference draws PMIS/HMIS measures from an unseeded global generator;
// here they come from a seeded generator (Config::seed).
#include <algorithm>
#include <cmath>
#include <limits>
#include <numeric>

#include "dr_host.h"

namespace dr {

static const double kEps = std::numeric_limits<double>::epsilon();

double rng_uniform(uint64_t& s) {
  // splitmix64 step, 53 random bits mapped to [0, 1).
  s += 0x9E3779B97F4A7C15ULL;
  uint64_t z = s;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  z ^= z >> 31;
  return (double)(z >> 11) * (1.0 / 9007199254740992.0);
}

void validate_csr(const CSR& A, const char* what) {
  if (A.n < 0 || A.m < 0) fail(std::string(what) + ": negative dimension");
  if ((int64_t)A.rp.size() != (int64_t)A.n + 1)
    fail(std::string(what) + ": rowptr must have n+1 entries");
  if (A.rp[0] != 0) fail(std::string(what) + ": rowptr must start at the index base");
  for (int i = 0; i < A.n; ++i)
    if (A.rp[i + 1] < A.rp[i]) fail(std::string(what) + ": rowptr is not monotone at row " + std::to_string(i + 1));
  if ((int64_t)A.rp[A.n] != A.nnz())
    fail(std::string(what) + ": rowptr[n+1]-base must equal nnz");
  if (A.v.size() != A.ci.size()) fail(std::string(what) + ": colval and nzval lengths differ");
  for (int64_t k = 0; k < A.nnz(); ++k)
    if (A.ci[k] < 0 || A.ci[k] >= A.m)
      fail(std::string(what) + ": column index out of range at entry " + std::to_string(k + 1));
}

// --------------------------------------------------------------- strength
std::vector<uint8_t> strength_absolute(const CSR& A, double theta) {
  std::vector<uint8_t> s(A.nnz(), 0);
#pragma omp parallel for schedule(static, 1024)
  for (int i = 0; i < A.n; ++i) {
    double mx = 0.0;
    for (int k = A.rp[i]; k < A.rp[i + 1]; ++k)
      if (A.ci[k] != i) mx = std::max(mx, std::fabs(A.v[k]));
    double thr = theta * mx;
    for (int k = A.rp[i]; k < A.rp[i + 1]; ++k)
      s[k] = (A.ci[k] != i) ? (std::fabs(A.v[k]) >= thr) : 0;
  }
  return s;
}

static inline double sgn(double x) { return x > 0 ? 1.0 : (x < 0 ? -1.0 : 0.0); }

std::vector<uint8_t> strength_signed(const CSR& A, double theta) {
  std::vector<uint8_t> s(A.nnz(), 0);
#pragma omp parallel for schedule(static, 1024)
  for (int i = 0; i < A.n; ++i) {
    double aii = 0.0;
    for (int k = A.rp[i]; k < A.rp[i + 1]; ++k)
      if (A.ci[k] == i) { aii = A.v[k]; break; }
    double ds = sgn(aii);
    if (ds == 0) ds = 1.0;
    double mx = 0.0;
    bool has = false;
    for (int k = A.rp[i]; k < A.rp[i + 1]; ++k)
      if (A.ci[k] != i && sgn(A.v[k]) != ds) { mx = std::max(mx, std::fabs(A.v[k])); has = true; }
    if (has) {
      double thr = theta * mx;
      for (int k = A.rp[i]; k < A.rp[i + 1]; ++k)
        s[k] = (A.ci[k] != i && sgn(A.v[k]) != ds) ? (std::fabs(A.v[k]) >= thr) : 0;
    } else {
      double mo = 0.0;
      for (int k = A.rp[i]; k < A.rp[i + 1]; ++k)
        if (A.ci[k] != i) mo = std::max(mo, std::fabs(A.v[k]));
      double thr = theta * mo;
      for (int k = A.rp[i]; k < A.rp[i + 1]; ++k)
        s[k] = (A.ci[k] != i) ? (std::fabs(A.v[k]) >= thr) : 0;
    }
  }
  return s;
}

CSR apply_max_row_sum(const CSR& A, double threshold) {
  CSR W = A;
  for (int i = 0; i < A.n; ++i) {
    double diag = 0.0, rs = 0.0;
    for (int k = A.rp[i]; k < A.rp[i + 1]; ++k) {
      rs += A.v[k];
      if (A.ci[k] == i) diag = A.v[k];
    }
    double ad = std::fabs(diag);
    if (ad < kEps) continue;
    if (std::fabs(rs) > ad * threshold && threshold < 1.0)
      for (int k = A.rp[i]; k < A.rp[i + 1]; ++k)
        if (A.ci[k] != i) W.v[k] = 0.0;
  }
  return W;
}

// ------------------------------------------------------------ union-find
static int find_root(std::vector<int>& parent, int i) {
  while (parent[i] != i) {
    parent[i] = parent[parent[i]];
    i = parent[i];
  }
  return i;
}
static void union_roots(std::vector<int>& parent, int a, int b) {
  int ra = find_root(parent, a), rb = find_root(parent, b);
  if (ra != rb) parent[rb] = ra;
}

// ------------------------------------------------------------ aggregation
void coarsen_aggregation(const CSR& A, double theta, std::vector<int>& agg, int& nc) {
  const int n = A.n;
  agg.assign(n, 0);
  if (n <= 1) {
    for (int i = 0; i < n; ++i) agg[i] = 0;
    nc = n;
    return;
  }
  std::vector<uint8_t> st = strength_absolute(A, theta);
  // aggregate ids are 1-based during construction (0 = unassigned)
  std::vector<int> a(n, 0);
  int ncoarse = 0;
  std::vector<int> scount(n, 0);
  for (int i = 0; i < n; ++i)
    for (int k = A.rp[i]; k < A.rp[i + 1]; ++k)
      if (A.ci[k] != i && st[k]) scount[i]++;
  // Phase 1: distance-2 MIS seeds in decreasing strong-count order (ties by
  // ascending index, as sortperm(...; rev=true) keeps equal keys in order).
  std::vector<int> order(n);
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(),
                   [&](int x, int y) { return scount[x] > scount[y]; });
  std::vector<int8_t> state(n, 0);
  for (int idx = 0; idx < n; ++idx) {
    int i = order[idx];
    if (state[i] != 0) continue;
    bool can_seed = true;
    for (int k = A.rp[i]; k < A.rp[i + 1]; ++k) {
      int j = A.ci[k];
      if (j != i && st[k] && (state[j] == 1 || state[j] == -1)) { can_seed = false; break; }
    }
    if (!can_seed) continue;
    state[i] = 1;
    ++ncoarse;
    a[i] = ncoarse;
    for (int k = A.rp[i]; k < A.rp[i + 1]; ++k) {
      int j = A.ci[k];
      if (j != i && st[k] && state[j] == 0) {
        state[j] = -1;
        a[j] = ncoarse;
        for (int k2 = A.rp[j]; k2 < A.rp[j + 1]; ++k2) {
          int q = A.ci[k2];
          if (q != j && st[k2] && state[q] == 0) state[q] = -2;
        }
      }
    }
  }
  // Phase 2: attach leftovers to the strongest aggregated neighbour.
  for (int i = 0; i < n; ++i) {
    if (a[i] != 0) continue;
    int best = 0;
    double bv = 0.0;
    for (int k = A.rp[i]; k < A.rp[i + 1]; ++k) {
      int j = A.ci[k];
      if (j != i && st[k] && a[j] != 0 && std::fabs(A.v[k]) > bv) { bv = std::fabs(A.v[k]); best = a[j]; }
    }
    if (best == 0)
      for (int k = A.rp[i]; k < A.rp[i + 1]; ++k) {
        int j = A.ci[k];
        if (j != i && a[j] != 0 && std::fabs(A.v[k]) > bv) { bv = std::fabs(A.v[k]); best = a[j]; }
      }
    if (best != 0) a[i] = best;
    else { ++ncoarse; a[i] = ncoarse; }
  }
  // Phase 3: merge singleton aggregates into their strongest neighbour.
  std::vector<int> size(ncoarse + 1, 0);
  for (int i = 0; i < n; ++i) size[a[i]]++;
  std::vector<int> mm(ncoarse + 1);
  std::iota(mm.begin(), mm.end(), 0);
  for (int i = 0; i < n; ++i) {
    int my = find_root(mm, a[i]);
    if (size[my] > 1) continue;
    int tgt = 0;
    double bv = 0.0;
    for (int k = A.rp[i]; k < A.rp[i + 1]; ++k) {
      int j = A.ci[k];
      if (j == i) continue;
      int jr = find_root(mm, a[j]);
      if (jr != my && std::fabs(A.v[k]) > bv) { bv = std::fabs(A.v[k]); tgt = jr; }
    }
    if (tgt != 0) {
      int om = size[my], ot = size[tgt];
      union_roots(mm, tgt, my);
      int nr = find_root(mm, tgt);
      size[nr] = om + ot;
    }
  }
  std::vector<int> nid(ncoarse + 1, 0);
  int cnt = 0;
  for (int i = 1; i <= ncoarse; ++i) {
    int r = find_root(mm, i);
    if (nid[r] == 0) nid[r] = ++cnt;
    nid[i] = nid[r];
  }
  for (int i = 0; i < n; ++i) agg[i] = nid[find_root(mm, a[i])] - 1;  // 0-based
  nc = cnt;
}

// ------------------------------------------------------------ helpers
static std::vector<int> strong_transpose_count(const CSR& A, const std::vector<uint8_t>& st) {
  std::vector<int> c(A.n, 0);
  for (int i = 0; i < A.n; ++i)
    for (int k = A.rp[i]; k < A.rp[i + 1]; ++k)
      if (A.ci[k] != i && st[k]) c[A.ci[k]]++;
  return c;
}

static void strong_transpose_adj(const CSR& A, const std::vector<uint8_t>& st,
                                 std::vector<int>& off, std::vector<int>& src) {
  const int n = A.n;
  off.assign(n + 1, 0);
  for (int i = 0; i < n; ++i)
    for (int k = A.rp[i]; k < A.rp[i + 1]; ++k)
      if (A.ci[k] != i && st[k]) off[A.ci[k] + 1]++;
  for (int j = 0; j < n; ++j) off[j + 1] += off[j];
  src.assign(off[n], 0);
  std::vector<int> pos(off.begin(), off.end() - 1);
  for (int i = 0; i < n; ++i)
    for (int k = A.rp[i]; k < A.rp[i + 1]; ++k)
      if (A.ci[k] != i && st[k]) src[pos[A.ci[k]]++] = i;
}

// Strong off-diagonal couplings of every row as a compact CSR: row i's
// entries k with ci[k] != i and st[k], in row order.  The sequential
// splitting loops walk these lists instead of A's rows and the strength
// flags (same entries, same order).
namespace {
struct StrongRows {
  std::vector<int> off, col;
  int begin(int i) const { return off[i]; }
  int end(int i) const { return off[i + 1]; }
};
}  // namespace

static StrongRows strong_rows(const CSR& A, const std::vector<uint8_t>& st) {
  const int n = A.n;
  StrongRows S;
  S.off.assign(n + 1, 0);
#pragma omp parallel for schedule(static, 4096)
  for (int i = 0; i < n; ++i) {
    int c = 0;
    for (int k = A.rp[i]; k < A.rp[i + 1]; ++k) c += (A.ci[k] != i && st[k]);
    S.off[i + 1] = c;
  }
  for (int i = 0; i < n; ++i) S.off[i + 1] += S.off[i];
  S.col.resize(S.off[n]);
#pragma omp parallel for schedule(static, 4096)
  for (int i = 0; i < n; ++i) {
    int w = S.off[i];
    for (int k = A.rp[i]; k < A.rp[i + 1]; ++k)
      if (A.ci[k] != i && st[k]) S.col[w++] = A.ci[k];
  }
  return S;
}

// Transpose of the strong couplings: for every j, the rows i that depend
// strongly on j, ascending (the lists of strong_transpose_adj).
static void strong_transpose(const StrongRows& S, int n, std::vector<int>& off, std::vector<int>& src) {
  off.assign(n + 1, 0);
  for (int j : S.col) off[j + 1]++;
  for (int j = 0; j < n; ++j) off[j + 1] += off[j];
  src.resize(off[n]);
  std::vector<int> pos(off.begin(), off.end() - 1);
  for (int i = 0; i < n; ++i)
    for (int t = S.begin(i); t < S.end(i); ++t) src[pos[S.col[t]]++] = i;
}

static bool has_strong_nbr(const CSR& A, const std::vector<uint8_t>& st, int i) {
  for (int k = A.rp[i]; k < A.rp[i + 1]; ++k)
    if (A.ci[k] != i && st[k]) return true;
  return false;
}

// PMIS sweeps over an adjacency (off, col), until no point is undecided
// (0): every undecided point that no neighbour outside F beats by measure
// becomes C, then every undecided point with a C neighbour becomes F.  With
// f_below_one (HMIS) an undecided point of measure below one becomes F
// instead of being tested.  Within a sweep no decision changes the outcome
// of another: C and undecided both count as "outside F", and a point made F
// for its measure could not beat any point that is tested.  So every sweep
// decides its points in parallel from the state before it, and gives the
// same states as deciding them one after another in row order.
static void pmis_sweeps(std::vector<int>& cf, const std::vector<int>& off, const std::vector<int>& col,
                        const std::vector<double>& meas, bool f_below_one) {
  const int n = (int)cf.size();
  std::vector<int8_t> nxt(n, 0);
  for (;;) {
    int undecided = 0;
#pragma omp parallel for schedule(static, 4096) reduction(+ : undecided)
    for (int i = 0; i < n; ++i) {
      nxt[i] = 0;
      if (cf[i] != 0) continue;
      ++undecided;
      if (f_below_one && meas[i] < 1.0) {
        nxt[i] = -1;
        continue;
      }
      bool is_max = true;
      for (int t = off[i]; t < off[i + 1]; ++t) {
        const int j = col[t];
        if (cf[j] != -1 && meas[j] > meas[i]) {
          is_max = false;
          break;
        }
      }
      if (is_max) nxt[i] = 1;
    }
    if (undecided == 0) break;
#pragma omp parallel for schedule(static, 4096)
    for (int i = 0; i < n; ++i)
      if (nxt[i]) cf[i] = nxt[i];
#pragma omp parallel for schedule(static, 4096)
    for (int i = 0; i < n; ++i) {
      nxt[i] = 0;
      if (cf[i] != 0) continue;
      for (int t = off[i]; t < off[i + 1]; ++t)
        if (cf[col[t]] == 1) {
          nxt[i] = -1;
          break;
        }
    }
#pragma omp parallel for schedule(static, 4096)
    for (int i = 0; i < n; ++i)
      if (nxt[i]) cf[i] = nxt[i];
  }
}

static void build_cmap(const std::vector<int>& cf, std::vector<int>& cmap, int& nc) {
  const int n = (int)cf.size();
  cmap.assign(n, -1);
  nc = 0;
  for (int i = 0; i < n; ++i)
    if (cf[i] == 1) cmap[i] = nc++;
}

// ------------------------------------------------------------ PMIS
void coarsen_pmis(const CSR& A, double theta, uint64_t& rng, std::vector<int>& cf,
                  std::vector<int>& cmap, int& nc) {
  const int n = A.n;
  if (n <= 1) {
    cf.assign(n, 1);
    build_cmap(cf, cmap, nc);
    return;
  }
  const StrongRows S = strong_rows(A, strength_absolute(A, theta));
  std::vector<int> stc(n, 0);
  for (int j : S.col) stc[j]++;
  std::vector<double> meas(n);
  for (int i = 0; i < n; ++i) meas[i] = (double)stc[i] + rng_uniform(rng);
  cf.assign(n, 0);
  for (int i = 0; i < n; ++i)
    if (S.begin(i) == S.end(i) && stc[i] == 0) cf[i] = 1;
  pmis_sweeps(cf, S.off, S.col, meas, false);
  build_cmap(cf, cmap, nc);
}

// ------------------------------------------------------------ RS first pass
// Bucket lists keyed by the measure lambda; insertion at the head.
namespace {
struct Buckets {
  std::vector<int> head, next, prev;
  std::vector<int>& lam;
  Buckets(int n, int maxl, std::vector<int>& l)
      : head(std::max(maxl + 1, 1), -1), next(n, -1), prev(n, -1), lam(l) {}
  void insert(int i) {
    int k = lam[i];
    if (k >= (int)head.size()) head.resize(k + 1, -1);
    int oh = head[k];
    head[k] = i;
    next[i] = oh;
    prev[i] = -1;
    if (oh != -1) prev[oh] = i;
  }
  void remove(int i) {
    int k = lam[i];
    int p = prev[i], nx = next[i];
    if (p != -1) next[p] = nx;
    else head[k] = nx;
    if (nx != -1) prev[nx] = p;
    next[i] = -1;
    prev[i] = -1;
  }
  void update(int i, int nl) {
    remove(i);
    lam[i] = nl;
    insert(i);
  }
};
}  // namespace

static std::vector<int> rs_first_pass(const StrongRows& S, int n, bool use_zpt) {
  const int f_pnt = use_zpt ? -2 : -1;
  std::vector<int> st_off, st_src;
  strong_transpose(S, n, st_off, st_src);
  std::vector<int> lam(n);
  for (int i = 0; i < n; ++i) lam[i] = st_off[i + 1] - st_off[i];
  std::vector<int> cf(n, 0);
  for (int i = 0; i < n; ++i)
    if (S.begin(i) == S.end(i) && lam[i] == 0) cf[i] = 1;
  for (int i = 0; i < n; ++i) {
    if (cf[i] != 0) continue;
    if (lam[i] == 0) {
      cf[i] = f_pnt;
      for (int t = S.begin(i); t < S.end(i); ++t) {
        const int j = S.col[t];
        if (cf[j] == 0) lam[j]++;
      }
    }
  }
  int maxl = 0;
  for (int i = 0; i < n; ++i)
    if (cf[i] == 0) maxl = std::max(maxl, lam[i]);
  Buckets B(n, maxl, lam);
  for (int i = 0; i < n; ++i)
    if (cf[i] == 0) B.insert(i);
  int top = maxl;
  for (;;) {
    while (top >= 0 && B.head[top] == -1) --top;
    if (top < 0) break;
    int best = B.head[top];
    if (best == -1) break;
    B.remove(best);
    cf[best] = 1;
    for (int idx = st_off[best]; idx < st_off[best + 1]; ++idx) {
      const int j = st_src[idx];
      if (cf[j] != 0) continue;
      B.remove(j);
      cf[j] = -1;
      for (int t = S.begin(j); t < S.end(j); ++t) {
        const int q = S.col[t];
        if (cf[q] == 0) {
          const int nv = lam[q] + 1;
          B.update(q, nv);
          if (nv > top) top = nv;
        }
      }
    }
    for (int t = S.begin(best); t < S.end(best); ++t) {
      const int j = S.col[t];
      if (cf[j] == 0) {
        const int nv = std::max(0, lam[j] - 1);
        B.update(j, nv);
        if (nv == 0) {
          B.remove(j);
          cf[j] = f_pnt;
          for (int t2 = S.begin(j); t2 < S.end(j); ++t2) {
            const int q = S.col[t2];
            if (cf[q] == 0) {
              const int nv2 = lam[q] + 1;
              B.update(q, nv2);
              if (nv2 > top) top = nv2;
            }
          }
        }
      }
    }
  }
  return cf;
}

static void pmis_on_undecided(std::vector<int>& cf, const StrongRows& S, const std::vector<double>& meas) {
  pmis_sweeps(cf, S.off, S.col, meas, true);
}

void coarsen_hmis(const CSR& A, double theta, uint64_t& rng, std::vector<int>& cf,
                  std::vector<int>& cmap, int& nc) {
  const int n = A.n;
  if (n <= 1) {
    cf.assign(n, 1);
    build_cmap(cf, cmap, nc);
    return;
  }
  const StrongRows S = strong_rows(A, strength_absolute(A, theta));
  cf = rs_first_pass(S, n, true);
  std::vector<int> stc(n, 0);
  for (int j : S.col) stc[j]++;
  std::vector<double> meas(n);
  for (int i = 0; i < n; ++i) meas[i] = (double)stc[i] + rng_uniform(rng);
  for (int i = 0; i < n; ++i) {
    if (cf[i] == -2) {
      if (meas[i] >= 1.0 || S.begin(i) != S.end(i)) cf[i] = 0;
      else cf[i] = -1;
    }
  }
  pmis_on_undecided(cf, S, meas);
  build_cmap(cf, cmap, nc);
}

static void ensure_fine_have_coarse_neighbor(std::vector<int>& cf, const CSR& A,
                                             const std::vector<uint8_t>& st) {
  bool changed = true;
  while (changed) {
    changed = false;
    for (int i = 0; i < A.n; ++i) {
      if (cf[i] != -1) continue;
      bool has_c = false;
      for (int k = A.rp[i]; k < A.rp[i + 1]; ++k) {
        int j = A.ci[k];
        if (j != i && st[k] && cf[j] == 1) { has_c = true; break; }
      }
      if (!has_c) { cf[i] = 1; changed = true; }
    }
  }
}

void coarsen_rs(const CSR& A, double theta, std::vector<int>& cf, std::vector<int>& cmap, int& nc) {
  const int n = A.n;
  if (n <= 1) {
    cf.assign(n, 1);
    build_cmap(cf, cmap, nc);
    return;
  }
  const std::vector<uint8_t> st = strength_absolute(A, theta);
  std::vector<int> lam = strong_transpose_count(A, st);
  std::vector<int> off, src;
  strong_transpose_adj(A, st, off, src);
  cf.assign(n, 0);  // 0 undecided, 1 C, -1 F
  for (int i = 0; i < n; ++i)
    if (!has_strong_nbr(A, st, i) && lam[i] == 0) cf[i] = 1;  // isolated
  // buckets of undecided points by lambda: doubly linked lists, new members
  // at the head
  int top = 0;
  for (int v : lam) top = std::max(top, v);
  std::vector<int> head(std::max(top + 1, n), -1), next(n, -1), prev(n, -1);
  auto push = [&](int i) {
    const int k = lam[i];
    if (k >= (int)head.size()) head.resize(k + 1, -1);
    next[i] = head[k];
    prev[i] = -1;
    if (head[k] >= 0) prev[head[k]] = i;
    head[k] = i;
  };
  auto remove = [&](int i) {
    const int k = lam[i];
    if (prev[i] >= 0) next[prev[i]] = next[i];
    else head[k] = next[i];
    if (next[i] >= 0) prev[next[i]] = prev[i];
    next[i] = prev[i] = -1;
  };
  auto update = [&](int i, int v) {
    remove(i);
    lam[i] = v;
    push(i);
  };
  for (int i = 0; i < n; ++i)
    if (cf[i] == 0) push(i);
  while (true) {
    while (top >= 0 && head[top] < 0) --top;
    if (top < 0) break;
    const int best = head[top];
    remove(best);
    cf[best] = 1;
    for (int q = off[best]; q < off[best + 1]; ++q) {  // points depending on best become F
      const int j = src[q];
      if (cf[j] != 0) continue;
      remove(j);
      cf[j] = -1;
      for (int k = A.rp[j]; k < A.rp[j + 1]; ++k) {  // their strong influences gain weight
        const int c = A.ci[k];
        if (c != j && st[k] && cf[c] == 0) {
          update(c, lam[c] + 1);
          top = std::max(top, lam[c]);
        }
      }
    }
    for (int k = A.rp[best]; k < A.rp[best + 1]; ++k) {  // best's strong influences lose weight
      const int c = A.ci[k];
      if (c != best && st[k] && cf[c] == 0) update(c, std::max(0, lam[c] - 1));
    }
  }
  ensure_fine_have_coarse_neighbor(cf, A, st);
  build_cmap(cf, cmap, nc);
}

void coarsen_aggressive_cf(const CSR& A_in, double theta, bool base_hmis, const Config& cfg,
                           uint64_t& rng, std::vector<int>& cf, std::vector<int>& cmap,
                           int& nc) {
  const int n = A_in.n;
  if (n <= 1) {
    cf.assign(n, 1);
    build_cmap(cf, cmap, nc);
    return;
  }
  CSR Aw;
  const CSR* Ap = &A_in;
  if (cfg.max_row_sum < 1.0) {
    Aw = apply_max_row_sum(A_in, cfg.max_row_sum);
    Ap = &Aw;
  }
  const CSR& A = *Ap;
  std::vector<int> cf1, cm1;
  int nc1 = 0;
  if (base_hmis) coarsen_hmis(A, theta, rng, cf1, cm1, nc1);
  else coarsen_pmis(A, theta, rng, cf1, cm1, nc1);
  std::vector<uint8_t> st = strength_absolute(A, theta);

  // C-points of the first pass and their local numbering.
  std::vector<int> cidx, clocal(n, -1);
  for (int i = 0; i < n; ++i)
    if (cf1[i] == 1) { clocal[i] = (int)cidx.size(); cidx.push_back(i); }
  const int m = (int)cidx.size();

  // Distance-2 graph among C-points: N(a) collects, over every node i with a
  // in its strong C-neighbour list cn(i), the other members of cn(i), plus i
  // itself when i is a C-point; and cn(node(a)) itself.
  std::vector<int> st_off, st_src;
  strong_transpose_adj(A, st, st_off, st_src);
  std::vector<int> noff(m + 1, 0);
  std::vector<int> nflat;
  {
    // the neighbours of a, in visiting order, each once (count, then fill)
    auto walk = [&](int a, std::vector<int>& mark, auto&& emit) {
      const int node = cidx[a];
      auto add = [&](int b) {
        if (b != a && mark[b] != a) {
          mark[b] = a;
          emit(b);
        }
      };
      // cn(node): strong C neighbours of node(a) (a -> them via "i is C")
      for (int k = A.rp[node]; k < A.rp[node + 1]; ++k) {
        const int j = A.ci[k];
        if (j != node && st[k] && cf1[j] == 1) add(clocal[j]);
      }
      // every i that has node(a) as a strong neighbour
      for (int t = st_off[node]; t < st_off[node + 1]; ++t) {
        const int i = st_src[t];
        if (cf1[i] == 1) add(clocal[i]);
        for (int k = A.rp[i]; k < A.rp[i + 1]; ++k) {
          const int j = A.ci[k];
          if (j != i && st[k] && cf1[j] == 1) add(clocal[j]);
        }
      }
    };
#pragma omp parallel
    {
      std::vector<int> mark(m, -1);
#pragma omp for schedule(dynamic, 256)
      for (int a = 0; a < m; ++a) {
        int cnt = 0;
        walk(a, mark, [&](int) { ++cnt; });
        noff[a + 1] = cnt;
      }
    }
    for (int a = 0; a < m; ++a) noff[a + 1] += noff[a];
    nflat.resize(noff[m]);
#pragma omp parallel
    {
      std::vector<int> mark(m, -1);
#pragma omp for schedule(dynamic, 256)
      for (int a = 0; a < m; ++a) {
        int w = noff[a];
        walk(a, mark, [&](int b) { nflat[w++] = b; });
      }
    }
  }
  std::vector<double> cmeas(m);
  for (int a = 0; a < m; ++a) cmeas[a] = (double)(noff[a + 1] - noff[a]) + rng_uniform(rng);
  std::vector<int> cf2(m, 0);
  pmis_sweeps(cf2, noff, nflat, cmeas, false);
  cf = cf1;
  for (int a = 0; a < m; ++a)
    if (cf2[a] == -1) cf[cidx[a]] = -1;
  ensure_fine_have_coarse_neighbor(cf, A, st);
  build_cmap(cf, cmap, nc);
}

}  // namespace dr
