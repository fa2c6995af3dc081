// Merging the hierarchies of independent systems into one batch (CPU).
//
// Merged level l holds, in system order, the rows of every system that has
// an AMG level l (its matrix, interpolation and smoother diagonal, placed
// block-diagonally), then the rows of every system whose coarsest level is
// l (solved by that system's own dense LU factors).  A system's rows keep
// their order, so every row of the merged matrices is the system's row
// with its columns shifted: the cycle kernels form the same per-row sums.
#include <stdexcept>
#include <string>

#include "dr_device.h"

namespace dr {

HostHierarchy merge_batch(const std::vector<const HostHierarchy*>& hs, BatchLayout& lay) {
  const int ns = (int)hs.size();
  if (ns < 1) fail("a batch needs at least one system");
  lay = BatchLayout();
  lay.nsys = ns;
  lay.depth.resize(ns);
  int lmax = 0;
  for (int s = 0; s < ns; ++s) {
    const HostHierarchy& h = *hs[s];
    lay.depth[s] = (int)h.levels.size();
    if (lay.depth[s] < 1)
      fail("system " + std::to_string(s) + " has no AMG level (n <= max_coarse_size): solve it alone");
    for (const HostLevel& L : h.levels)
      if (!(L.smoother == SmootherKind::Jacobi || L.smoother == SmootherKind::L1Jacobi ||
            L.smoother == SmootherKind::SPAI0))
        fail("batched systems need Jacobi, l1-Jacobi or SPAI(0) smoothing on every level");
    lmax = std::max(lmax, lay.depth[s]);
  }
  // row counts and offsets per merged level
  lay.nsmooth.assign(lmax + 1, 0);
  lay.ntotal.assign(lmax + 1, 0);
  lay.off.assign(lmax + 1, std::vector<int>(ns, -1));
  lay.coarse.resize(lmax + 1);
  for (int l = 0; l <= lmax; ++l) {
    int r = 0;
    for (int s = 0; s < ns; ++s)
      if (lay.depth[s] > l) {
        lay.off[l][s] = r;
        r += hs[s]->levels[l].A.n;
      }
    lay.nsmooth[l] = r;
    BatchLayout::Coarse& c = lay.coarse[l];
    for (int s = 0; s < ns; ++s)
      if (lay.depth[s] == l) {
        const HostHierarchy& h = *hs[s];
        lay.off[l][s] = r;
        c.off.push_back(r);
        c.nb.push_back(h.nc);
        c.luoff.push_back((long long)lay.lu.size());
        c.poff.push_back((int)lay.piv.size());
        c.maxn = std::max(c.maxn, h.nc);
        lay.lu.insert(lay.lu.end(), h.coarse_lu.begin(), h.coarse_lu.end());
        lay.piv.insert(lay.piv.end(), h.coarse_piv.begin(), h.coarse_piv.end());
        r += h.nc;
      }
    lay.ntotal[l] = r;
  }
  HostHierarchy M;
  M.cfg = hs[0]->cfg;
  M.allow_partial_resetup = false;
  M.levels.resize(lmax);
  for (int l = 0; l < lmax; ++l) {
    HostLevel& L = M.levels[l];
    const int n = lay.nsmooth[l];
    L.A.n = L.A.m = n;
    L.A.rp.assign(1, 0);
    L.P.nf = n;
    L.P.nc = lay.ntotal[l + 1];
    L.P.rp.assign(1, 0);
    bool first = true;
    for (int s = 0; s < ns; ++s) {
      if (lay.depth[s] <= l) continue;
      const HostLevel& h = hs[s]->levels[l];
      if (first) {
        L.smoother = h.smoother;
        L.omega = h.omega;
        first = false;
      } else if (h.smoother != L.smoother || h.omega != L.omega) {
        fail("batched systems must share the smoother and its weight on every level");
      }
      const int ro = lay.off[l][s], co = lay.off[l + 1][s];
      for (int i = 0; i < h.A.n; ++i) {
        for (int k = h.A.rp[i]; k < h.A.rp[i + 1]; ++k) {
          L.A.ci.push_back(h.A.ci[k] + ro);
          L.A.v.push_back(h.A.v[k]);
        }
        L.A.rp.push_back((int)L.A.ci.size());
        for (int k = h.P.rp[i]; k < h.P.rp[i + 1]; ++k) {
          L.P.ci.push_back(h.P.ci[k] + co);
          L.P.v.push_back(h.P.v[k]);
        }
        L.P.rp.push_back((int)L.P.ci.size());
      }
      L.invdiag.insert(L.invdiag.end(), h.invdiag.begin(), h.invdiag.end());
    }
    L.T = build_transpose_map(L.P);
    L.Rv.resize(L.P.nnz());
    for (size_t k = 0; k < L.T.pnz.size(); ++k) L.Rv[k] = L.P.v[L.T.pnz[k]];
    // the pattern of A·P, block-diagonal like P, when every system keeps
    // its own: it carries the fused correction on the way up (a batch has
    // no partial resetup, so has_rap_map stays false)
    L.has_rap_map = false;
    bool all_ap = true;
    for (int s = 0; s < ns; ++s)
      if (lay.depth[s] > l && !hs[s]->levels[l].has_rap_map) all_ap = false;
    if (all_ap) {
      L.ap_rp.assign(1, 0);
      for (int s = 0; s < ns; ++s) {
        if (lay.depth[s] <= l) continue;
        const HostLevel& h = hs[s]->levels[l];
        const int co = lay.off[l + 1][s];
        for (int i = 0; i < h.A.n; ++i) {
          for (int k = h.ap_rp[i]; k < h.ap_rp[i + 1]; ++k) L.ap_ci.push_back(h.ap_ci[k] + co);
          L.ap_rp.push_back((int)L.ap_ci.size());
        }
      }
    }
  }
  M.nc = lay.ntotal[lmax];
  M.coarse.n = M.coarse.m = M.nc;
  M.coarse.rp.assign((size_t)M.nc + 1, 0);
  return M;
}

}  // namespace dr
