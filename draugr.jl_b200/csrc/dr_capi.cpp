// C ABI of libdraugr_b200.so: the draugr_amg_* drop-in (include/draugr_amg.h)
// and the draugr_b200_* extensions (include/draugr_b200.h).
//
// Handle table and error convention follow src/cfunction_interface.jl of
// Draugr.jl: configs and hierarchies share one counter starting at 1
// (:165-174), every entry point catches its errors, stores the message for
// draugr_amg_last_error and returns -1 (:215-220 and the other entries).
#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>

#include "../../include/draugr_amg.h"
#include "../../include/draugr_b200.h"
#include "dr_device.h"
#include "dr_host.h"

namespace {

using namespace dr;

struct Hier {
  HostHierarchy host;
  std::unique_ptr<DevHier> dev;
  int device = 0;
  std::string summary;
  std::unique_ptr<BatchLayout> batch;  // set for a batch of merged systems
};

std::mutex g_mu;
std::map<int32_t, Config> g_cfg;
std::map<int32_t, std::shared_ptr<Hier>> g_hier;
int32_t g_next = 1;
// The last error of the calling thread (the reference keeps one per
// process; per thread, a host that calls from several threads reads the
// message of its own failed call).
thread_local std::string g_last_error;

void set_error(const std::string& m) { g_last_error = m; }

int32_t new_handle() { return g_next++; }

Config get_cfg(int32_t h) {
  std::lock_guard<std::mutex> lk(g_mu);
  auto it = g_cfg.find(h);
  if (it == g_cfg.end()) fail("Invalid config handle: " + std::to_string(h));
  return it->second;
}

std::shared_ptr<Hier> get_hier(int32_t h, int32_t cfg, Config* c) {
  std::lock_guard<std::mutex> lk(g_mu);
  auto it = g_hier.find(h);
  auto ic = g_cfg.find(cfg);
  if (it == g_hier.end() || (c && ic == g_cfg.end()))
    fail("Invalid handle (hierarchy=" + std::to_string(h) + ", config=" + std::to_string(cfg) + ")");
  if (c) *c = ic->second;
  return it->second;
}

std::shared_ptr<Hier> get_hier_only(int32_t h) {
  std::lock_guard<std::mutex> lk(g_mu);
  auto it = g_hier.find(h);
  if (it == g_hier.end()) fail("Invalid hierarchy handle: " + std::to_string(h));
  return it->second;
}

// Copy and shift raw CSR input to 0-based (csr_from_raw, src/csr_matrix.jl:133-143).
CSR csr_from_raw(int32_t n, int32_t nnz, const int32_t* rowptr, const int32_t* colval,
                 const double* nzval, int32_t base) {
  if (base != 0 && base != 1) fail("ArgumentError: index_base must be 0 or 1, got " + std::to_string(base));
  if (n < 0 || nnz < 0) fail("ArgumentError: n and nnz must be non-negative");
  if (!rowptr || (nnz > 0 && (!colval || !nzval))) fail("ArgumentError: NULL array");
  CSR A;
  A.n = A.m = n;
  A.rp.assign(rowptr, rowptr + n + 1);
  A.ci.assign(colval, colval + nnz);
  A.v.assign(nzval, nzval + nnz);
  if (base == 1) {
    for (auto& r : A.rp) r -= 1;
    for (auto& c : A.ci) c -= 1;
  }
  validate_csr(A, "matrix");
  return A;
}

CycleOpts opts_of(const Config& c) {
  CycleOpts o;
  o.pre = c.pre_smoothing_steps;
  o.post = c.post_smoothing_steps;
  o.w = c.cycle_w;
  return o;
}

DevHier& device_of(Hier& H) {
  if (!H.dev) {
    int dev = 0;
    DR_CK(cudaGetDevice(&dev));
    H.device = dev;
    H.dev.reset(new DevHier(H.host, dev, H.batch.get()));
  }
  DR_CK(cudaSetDevice(H.device));
  return *H.dev;
}

void print_summary(Hier& H) {
  int n0 = H.host.levels.empty() ? H.host.nc : H.host.levels[0].A.n;
  std::fputs(hierarchy_summary(H.host, n0).c_str(), stdout);
  std::fflush(stdout);
}

int32_t n_finest(const Hier& H) { return H.host.levels.empty() ? H.host.nc : H.host.levels[0].A.n; }

template <class F>
int32_t guarded(const char* name, F&& f) {
  try {
    set_error("");
    return f();
  } catch (const std::exception& e) {
    set_error(e.what());
    return -1;
  } catch (...) {
    set_error(std::string(name) + " failed");
    return -1;
  }
}

}  // namespace

namespace dr {
// Last-error text for entry points defined outside this file.
void set_last_error(const std::string& msg) { set_error(msg); }
}  // namespace dr

extern "C" {

void init_julia(int, char**) {}
void shutdown_julia(int) {}

const char* draugr_amg_last_error(void) {
  std::lock_guard<std::mutex> lk(g_mu);
  return g_last_error.c_str();
}

int32_t draugr_amg_config_from_json(const char* json_str) {
  return guarded("draugr_amg_config_from_json", [&]() -> int32_t {
    Config c = config_from_json(json_str);
    std::lock_guard<std::mutex> lk(g_mu);
    int32_t h = new_handle();
    g_cfg[h] = c;
    return h;
  });
}

static int32_t setup_impl(int32_t n, int32_t nnz, const int32_t* rowptr, const int32_t* colval,
                          const double* nzval, int32_t config_handle, int32_t index_base,
                          int32_t allow_partial_resetup, bool to_device) {
  CSR A = csr_from_raw(n, nnz, rowptr, colval, nzval, index_base);
  Config c = get_cfg(config_handle);
  auto H = std::make_shared<Hier>();
  // a setup for the device computes its Galerkin products there (same
  // hierarchy, bit for bit); a host-only setup stays on the CPU
  std::unique_ptr<GalerkinDevice> gdev = to_device ? make_galerkin_device() : nullptr;
  build_hierarchy(A, c, allow_partial_resetup != 0, H->host, gdev.get());
  if (to_device) device_of(*H);
  if (c.verbose >= 1) print_summary(*H);
  std::lock_guard<std::mutex> lk(g_mu);
  int32_t h = new_handle();
  g_hier[h] = H;
  return h;
}

int32_t draugr_amg_setup(int32_t n, int32_t nnz, const int32_t* rowptr, const int32_t* colval,
                         const double* nzval, int32_t config_handle, int32_t index_base,
                         int32_t allow_partial_resetup) {
  return guarded("draugr_amg_setup", [&]() {
    return setup_impl(n, nnz, rowptr, colval, nzval, config_handle, index_base, allow_partial_resetup, true);
  });
}

int32_t draugr_b200_setup_host(int32_t n, int32_t nnz, const int32_t* rowptr, const int32_t* colval,
                               const double* nzval, int32_t config_handle, int32_t index_base,
                               int32_t allow_partial_resetup) {
  return guarded("draugr_b200_setup_host", [&]() {
    return setup_impl(n, nnz, rowptr, colval, nzval, config_handle, index_base, allow_partial_resetup, false);
  });
}

int32_t draugr_amg_resetup(int32_t handle, int32_t n, int32_t nnz, const int32_t* rowptr,
                           const int32_t* colval, const double* nzval, int32_t config_handle,
                           int32_t index_base, int32_t partial, int32_t allow_partial_resetup) {
  return guarded("draugr_amg_resetup", [&]() -> int32_t {
    CSR A = csr_from_raw(n, nnz, rowptr, colval, nzval, index_base);
    Config c;
    auto H = get_hier(handle, config_handle, &c);
    if (partial) {
      const CSR& A0 = H->host.levels.empty() ? H->host.coarse : H->host.levels[0].A;
      if (A.n != A0.n || A.nnz() != A0.nnz() || A.rp != A0.rp || A.ci != A0.ci)
        fail("partial resetup: the sparsity pattern differs from the one given at setup");
      for (auto& L : H->host.levels)
        if (!L.has_rap_map)
          fail("partial resetup needs the Galerkin maps; set up the hierarchy with allow_partial_resetup=1");
      DevHier& D = device_of(*H);
      double* tmp = nullptr;
      DR_CK(cudaMalloc(&tmp, std::max<size_t>(1, A.v.size()) * sizeof(double)));
      cudaError_t e = cudaMemcpy(tmp, A.v.data(), A.v.size() * sizeof(double), cudaMemcpyHostToDevice);
      try {
        DR_CK(e);
        D.resetup_values(tmp);
      } catch (...) {
        cudaFree(tmp);
        throw;
      }
      cudaFree(tmp);
      if (H->host.levels.empty()) H->host.coarse.v = A.v;
      else H->host.levels[0].A.v = A.v;
    } else {
      auto NH = std::make_shared<Hier>();
      std::unique_ptr<GalerkinDevice> gdev = H->dev ? make_galerkin_device() : nullptr;
      build_hierarchy(A, c, allow_partial_resetup != 0, NH->host, gdev.get());
      if (H->dev) {
        H->dev.reset();
        device_of(*NH);
      }
      if (c.verbose >= 1) print_summary(*NH);
      H->host = std::move(NH->host);
      H->dev = std::move(NH->dev);
      H->device = NH->device;
    }
    return 0;
  });
}

int32_t draugr_amg_solve(int32_t handle, int32_t n, double* x, const double* b, int32_t config_handle,
                         double tol, int32_t maxiter) {
  return guarded("draugr_amg_solve", [&]() -> int32_t {
    Config c;
    auto H = get_hier(handle, config_handle, &c);
    if (n != n_finest(*H)) fail("DimensionMismatch: vector length " + std::to_string(n) + " != " + std::to_string(n_finest(*H)));
    if (!x || !b) fail("ArgumentError: NULL vector");
    DevHier& D = device_of(*H);
    DR_CK(cudaMemcpyAsync(D.xbuf(), x, (size_t)n * sizeof(double), cudaMemcpyHostToDevice, D.stream()));
    DR_CK(cudaMemcpyAsync(D.bbuf(), b, (size_t)n * sizeof(double), cudaMemcpyHostToDevice, D.stream()));
    int it = D.solve(D.xbuf(), D.bbuf(), opts_of(c), tol, maxiter, c.verbose, nullptr);
    DR_CK(cudaMemcpyAsync(x, D.xbuf(), (size_t)n * sizeof(double), cudaMemcpyDeviceToHost, D.stream()));
    DR_CK(cudaStreamSynchronize(D.stream()));
    return it;
  });
}

int32_t draugr_amg_cycle(int32_t handle, int32_t n, double* x, const double* b, int32_t config_handle) {
  return guarded("draugr_amg_cycle", [&]() -> int32_t {
    Config c;
    auto H = get_hier(handle, config_handle, &c);
    if (n != n_finest(*H)) fail("DimensionMismatch: vector length " + std::to_string(n) + " != " + std::to_string(n_finest(*H)));
    if (!x || !b) fail("ArgumentError: NULL vector");
    DevHier& D = device_of(*H);
    DR_CK(cudaMemcpyAsync(D.xbuf(), x, (size_t)n * sizeof(double), cudaMemcpyHostToDevice, D.stream()));
    DR_CK(cudaMemcpyAsync(D.bbuf(), b, (size_t)n * sizeof(double), cudaMemcpyHostToDevice, D.stream()));
    D.cycle(D.xbuf(), D.bbuf(), opts_of(c));
    DR_CK(cudaMemcpyAsync(x, D.xbuf(), (size_t)n * sizeof(double), cudaMemcpyDeviceToHost, D.stream()));
    D.check_errors();
    return 0;
  });
}

int32_t draugr_amg_free(int32_t handle) {
  return guarded("draugr_amg_free", [&]() -> int32_t {
    std::shared_ptr<Hier> H;
    {
      std::lock_guard<std::mutex> lk(g_mu);
      auto it = g_hier.find(handle);
      if (it == g_hier.end()) {
        g_last_error = "Invalid hierarchy handle: " + std::to_string(handle);
        return -1;
      }
      H = it->second;
      g_hier.erase(it);
    }
    return 0;  // H released here (device memory freed)
  });
}

int32_t draugr_amg_config_free(int32_t handle) {
  return guarded("draugr_amg_config_free", [&]() -> int32_t {
    std::lock_guard<std::mutex> lk(g_mu);
    auto it = g_cfg.find(handle);
    if (it == g_cfg.end()) {
      g_last_error = "Invalid config handle: " + std::to_string(handle);
      return -1;
    }
    g_cfg.erase(it);
    return 0;
  });
}

// ------------------------------------------------------------ extensions
int32_t draugr_b200_num_levels(int32_t handle) {
  return guarded("draugr_b200_num_levels", [&]() -> int32_t {
    return (int32_t)get_hier_only(handle)->host.levels.size();
  });
}

int32_t draugr_b200_level_info(int32_t handle, int32_t lvl, int64_t* info) {
  return guarded("draugr_b200_level_info", [&]() -> int32_t {
    auto H = get_hier_only(handle);
    if (!info) fail("ArgumentError: NULL info");
    if (lvl == -1) {
      info[0] = H->host.nc;
      info[1] = H->host.coarse.nnz();
      return 0;
    }
    if (lvl < 0 || lvl >= (int)H->host.levels.size()) fail("level index out of range");
    const HostLevel& L = H->host.levels[lvl];
    info[0] = L.A.n;
    info[1] = L.A.nnz();
    info[2] = L.P.nc;
    info[3] = L.P.nnz();
    info[4] = (int64_t)L.smoother;
    info[5] = L.num_colors;
    info[6] = L.has_rap_map ? (int64_t)L.ap_ci.size() : -1;
    info[7] = rows_in_order(L.A.rp);
    info[8] = rows_in_order(L.P.rp);
    info[9] = rows_in_order(L.T.off);
    return 0;
  });
}

int64_t draugr_b200_export(int32_t handle, int32_t lvl, const char* what, void* out, int64_t cap) {
  int64_t result = -1;
  guarded("draugr_b200_export", [&]() -> int32_t {
    auto H = get_hier_only(handle);
    if (!what) fail("ArgumentError: NULL name");
    const std::string w(what);
    const std::vector<int>* iv = nullptr;
    const std::vector<double>* dv = nullptr;
    std::vector<double> tmpd;
    std::vector<int> tmpi;
    if (lvl == -1) {
      const HostHierarchy& h = H->host;
      if (w == "C_rowptr") iv = &h.coarse.rp;
      else if (w == "C_colval") iv = &h.coarse.ci;
      else if (w == "C_piv") iv = &h.coarse_piv;
      else if (w == "C_nzval") dv = &h.coarse.v;
      else if (w == "C_dense") dv = &h.coarse_dense;
      else if (w == "C_lu") dv = &h.coarse_lu;
      if (dv && H->dev) { H->dev->export_values(-1, w, tmpd); dv = &tmpd; }
      if (iv == &h.coarse_piv && H->dev) { H->dev->export_piv(tmpi); iv = &tmpi; }
    } else {
      if (lvl < 0 || lvl >= (int)H->host.levels.size()) fail("level index out of range");
      const HostLevel& L = H->host.levels[lvl];
      if (w == "A_rowptr") iv = &L.A.rp;
      else if (w == "A_colval") iv = &L.A.ci;
      else if (w == "P_rowptr") iv = &L.P.rp;
      else if (w == "P_colval") iv = &L.P.ci;
      else if (w == "T_offsets") iv = &L.T.off;
      else if (w == "T_rows") iv = &L.T.rows;
      else if (w == "T_pnz") iv = &L.T.pnz;
      else if (w == "colors") iv = &L.colors;
      else if (w == "color_order") iv = &L.color_order;
      else if (w == "color_offsets") iv = &L.color_off;
      else if (w == "AP_rowptr") iv = &L.ap_rp;
      else if (w == "AP_colval") iv = &L.ap_ci;
      else if (w == "A_nzval") dv = &L.A.v;
      else if (w == "P_nzval") dv = &L.P.v;
      else if (w == "R_nzval") dv = &L.Rv;
      else if (w == "invdiag") dv = &L.invdiag;
      else if (w == "omega") { tmpd.assign(1, L.omega); dv = &tmpd; }
      else if (w == "cheb_coef") dv = &L.cheb_coef;
      else if (w == "cheb_v0") dv = &L.cheb_v0;
      else if (w == "ilu_L") dv = &L.ilu_L;
      else if (w == "ilu_U") dv = &L.ilu_U;
      else if (w == "ilu_diag") iv = &L.ilu_diag;
      else if (w == "ilu_fwd_order") iv = &L.ilu_fwd_order;
      else if (w == "ilu_fwd_offsets") iv = &L.ilu_fwd_off;
      else if (w == "ilu_bwd_order") iv = &L.ilu_bwd_order;
      else if (w == "ilu_bwd_offsets") iv = &L.ilu_bwd_off;
      else if (w == "spai1_M") dv = &L.spai1_M;
      else if (w == "sgs_order") iv = &L.sgs_order;
      else if (w == "cf") iv = &L.cf;
      else if (w == "sgs_offsets") iv = &L.sgs_off;
      else if (w == "AP_nzval") {
        if (!H->dev) fail("AP_nzval lives on the device only");
        dv = &tmpd;
      }
      if (dv && H->dev && w != "P_nzval" && w != "R_nzval" && w != "omega" && w != "cheb_v0" &&
          !(w == "cheb_coef" && L.cheb_coef.empty()) && !((w == "ilu_L" || w == "ilu_U") && L.ilu_L.empty()) &&
          !(w == "spai1_M" && L.spai1_M.empty())) {
        H->dev->export_values(lvl, w, tmpd);
        dv = &tmpd;
      }
    }
    if (!iv && !dv) fail("unknown export name: " + w);
    int64_t cnt = iv ? (int64_t)iv->size() : (int64_t)dv->size();
    if (out) {
      if (cap < cnt) fail("export buffer too small: need " + std::to_string(cnt));
      if (iv) std::memcpy(out, iv->data(), cnt * sizeof(int));
      else std::memcpy(out, dv->data(), cnt * sizeof(double));
    }
    result = cnt;
    return 0;
  });
  return result;
}

const char* draugr_b200_config_json(int32_t config_handle) {
  static thread_local std::string s;
  s.clear();
  const int32_t rc = guarded("draugr_b200_config_json", [&]() -> int32_t {
    s = config_to_json(get_cfg(config_handle));
    return 0;
  });
  return rc < 0 ? nullptr : s.c_str();
}

const char* draugr_b200_summary(int32_t handle) {
  static thread_local std::string s;
  s.clear();
  guarded("draugr_b200_summary", [&]() -> int32_t {
    auto H = get_hier_only(handle);
    s = hierarchy_summary(H->host, n_finest(*H));
    return 0;
  });
  return s.c_str();
}

int64_t draugr_b200_device_bytes(int32_t handle) {
  int64_t r = -1;
  guarded("draugr_b200_device_bytes", [&]() -> int32_t {
    auto H = get_hier_only(handle);
    r = H->dev ? (int64_t)H->dev->device_bytes() : 0;
    return 0;
  });
  return r;
}

int32_t draugr_b200_solve_device(int32_t handle, int32_t n, double* x_dev, const double* b_dev,
                                 int32_t config_handle, double tol, int32_t maxiter) {
  return guarded("draugr_b200_solve_device", [&]() -> int32_t {
    Config c;
    auto H = get_hier(handle, config_handle, &c);
    if (n != n_finest(*H)) fail("DimensionMismatch");
    DevHier& D = device_of(*H);
    return D.solve(x_dev, b_dev, opts_of(c), tol, maxiter, c.verbose, nullptr);
  });
}

int32_t draugr_b200_cycle_device(int32_t handle, int32_t n, double* x_dev, const double* b_dev,
                                 int32_t config_handle) {
  return guarded("draugr_b200_cycle_device", [&]() -> int32_t {
    Config c;
    auto H = get_hier(handle, config_handle, &c);
    if (n != n_finest(*H)) fail("DimensionMismatch");
    DevHier& D = device_of(*H);
    D.cycle(x_dev, b_dev, opts_of(c));
    D.check_errors();
    return 0;
  });
}

int32_t draugr_b200_resetup_values_device(int32_t handle, int64_t nnz, const double* nzval_dev) {
  return guarded("draugr_b200_resetup_values_device", [&]() -> int32_t {
    auto H = get_hier_only(handle);
    const CSR& A0 = H->host.levels.empty() ? H->host.coarse : H->host.levels[0].A;
    if (nnz != A0.nnz()) fail("partial resetup: nnz differs from the one given at setup");
    DevHier& D = device_of(*H);
    D.resetup_values(nzval_dev);
    return 0;
  });
}

int32_t draugr_b200_set_resetup_precision(int32_t handle, int32_t fp64_levels) {
  return guarded("draugr_b200_set_resetup_precision", [&]() -> int32_t {
    auto H = get_hier_only(handle);
    device_of(*H).set_resetup_fp64_levels(fp64_levels);
    return 0;
  });
}

int32_t draugr_b200_galerkin_host(int32_t handle, int32_t lvl, int64_t nnz_in, const double* a_vals,
                                  int64_t nnz_out, double* ac_vals) {
  return guarded("draugr_b200_galerkin_host", [&]() -> int32_t {
    auto H = get_hier_only(handle);
    if (lvl < 0 || lvl >= (int)H->host.levels.size()) fail("level index out of range");
    const HostLevel& L = H->host.levels[lvl];
    if (!L.has_rap_map) fail("the level keeps no A*P pattern (set up with allow_partial_resetup=1)");
    const CSR& next = lvl + 1 < (int)H->host.levels.size() ? H->host.levels[lvl + 1].A : H->host.coarse;
    if (nnz_in != L.A.nnz()) fail("nnz_in differs from the level's nonzeros");
    if (nnz_out != next.nnz()) fail("nnz_out differs from the next level's nonzeros");
    if ((nnz_in > 0 && !a_vals) || (nnz_out > 0 && !ac_vals)) fail("ArgumentError: NULL array");
    CSR A = L.A;
    A.v.assign(a_vals, a_vals + nnz_in);
    std::vector<double> ap_v, c_v;
    numeric_ap(A, L.P, L.ap_rp, L.ap_ci, ap_v);
    numeric_ptap(L.T, L.Rv, L.ap_rp, L.ap_ci, ap_v, next.rp, next.ci, c_v);
    std::copy(c_v.begin(), c_v.end(), ac_vals);
    return 0;
  });
}

int32_t draugr_b200_residual_device(int32_t handle, int32_t n, const double* x_dev, const double* b_dev,
                                    double* r_dev, double* rnorm) {
  return guarded("draugr_b200_residual_device", [&]() -> int32_t {
    auto H = get_hier_only(handle);
    if (n != n_finest(*H)) fail("DimensionMismatch");
    if (!x_dev || !b_dev || !r_dev) fail("ArgumentError: NULL vector");
    DevHier& D = device_of(*H);
    const double nr = D.residual_norm(x_dev, b_dev, r_dev);
    if (rnorm) *rnorm = nr;
    return 0;
  });
}

static int32_t pcg_impl(int32_t handle, int32_t n, double* x, const double* b, int32_t config_handle,
                        double tol, int32_t maxiter, int32_t precision, double* relres, bool host) {
  Config c;
  auto H = get_hier(handle, config_handle, &c);
  if (n != n_finest(*H)) fail("DimensionMismatch");
  if (precision != 0 && precision != 1) fail("precision must be 0 (FP64 cycle) or 1 (FP32 cycle)");
  if (!x || !b) fail("ArgumentError: NULL vector");
  DevHier& D = device_of(*H);
  double rr = 0;
  int it;
  if (host) {
    DR_CK(cudaMemcpyAsync(D.xbuf(), x, (size_t)n * sizeof(double), cudaMemcpyHostToDevice, D.stream()));
    DR_CK(cudaMemcpyAsync(D.bbuf(), b, (size_t)n * sizeof(double), cudaMemcpyHostToDevice, D.stream()));
    it = D.pcg(D.xbuf(), D.bbuf(), opts_of(c), tol, maxiter, precision == 1, &rr, c.verbose);
    DR_CK(cudaMemcpyAsync(x, D.xbuf(), (size_t)n * sizeof(double), cudaMemcpyDeviceToHost, D.stream()));
    DR_CK(cudaStreamSynchronize(D.stream()));
  } else {
    it = D.pcg(x, b, opts_of(c), tol, maxiter, precision == 1, &rr, c.verbose);
  }
  if (relres) *relres = rr;
  return it;
}

int32_t draugr_b200_pcg(int32_t handle, int32_t n, double* x, const double* b, int32_t config_handle,
                        double tol, int32_t maxiter, int32_t precision, double* relres) {
  return guarded("draugr_b200_pcg", [&]() {
    return pcg_impl(handle, n, x, b, config_handle, tol, maxiter, precision, relres, true);
  });
}

int32_t draugr_b200_pcg_device(int32_t handle, int32_t n, double* x_dev, const double* b_dev,
                               int32_t config_handle, double tol, int32_t maxiter, int32_t precision,
                               double* relres) {
  return guarded("draugr_b200_pcg_device", [&]() {
    return pcg_impl(handle, n, x_dev, b_dev, config_handle, tol, maxiter, precision, relres, false);
  });
}

static int32_t bicgstab_impl(int32_t handle, int32_t n, double* x, const double* b, int32_t config_handle,
                             double tol, int32_t maxiter, int32_t transpose, int32_t precision, double* relres,
                             bool host) {
  Config c;
  auto H = get_hier(handle, config_handle, &c);
  if (n != n_finest(*H)) fail("DimensionMismatch");
  if (!x || !b) fail("ArgumentError: NULL vector");
  if (precision != 0 && precision != 1) fail("precision must be 0 (FP64 cycle) or 1 (FP32 cycle)");
  const bool mixed = precision == 1;
  DevHier& D = device_of(*H);
  double rr = 0;
  int it;
  if (host) {
    DR_CK(cudaMemcpyAsync(D.xbuf(), x, (size_t)n * sizeof(double), cudaMemcpyHostToDevice, D.stream()));
    DR_CK(cudaMemcpyAsync(D.bbuf(), b, (size_t)n * sizeof(double), cudaMemcpyHostToDevice, D.stream()));
    it = D.bicgstab(D.xbuf(), D.bbuf(), opts_of(c), tol, maxiter, transpose != 0, &rr, c.verbose, mixed);
    DR_CK(cudaMemcpyAsync(x, D.xbuf(), (size_t)n * sizeof(double), cudaMemcpyDeviceToHost, D.stream()));
    DR_CK(cudaStreamSynchronize(D.stream()));
  } else {
    it = D.bicgstab(x, b, opts_of(c), tol, maxiter, transpose != 0, &rr, c.verbose, mixed);
  }
  if (relres) *relres = rr;
  return it;
}

int32_t draugr_b200_bicgstab(int32_t handle, int32_t n, double* x, const double* b, int32_t config_handle,
                             double tol, int32_t maxiter, int32_t transpose, int32_t precision, double* relres) {
  return guarded("draugr_b200_bicgstab", [&]() {
    return bicgstab_impl(handle, n, x, b, config_handle, tol, maxiter, transpose, precision, relres, true);
  });
}

int32_t draugr_b200_bicgstab_device(int32_t handle, int32_t n, double* x_dev, const double* b_dev,
                                    int32_t config_handle, double tol, int32_t maxiter, int32_t transpose,
                                    int32_t precision, double* relres) {
  return guarded("draugr_b200_bicgstab_device", [&]() {
    return bicgstab_impl(handle, n, x_dev, b_dev, config_handle, tol, maxiter, transpose, precision, relres,
                         false);
  });
}

static int32_t fgmres_impl(int32_t handle, int32_t n, double* x, const double* b, int32_t config_handle,
                           double tol, int32_t maxiter, int32_t restart, int32_t precision, double* relres,
                           bool host) {
  Config c;
  auto H = get_hier(handle, config_handle, &c);
  if (n != n_finest(*H)) fail("DimensionMismatch");
  if (!x || !b) fail("ArgumentError: NULL vector");
  if (precision != 0 && precision != 1) fail("precision must be 0 (FP64 cycle) or 1 (FP32 cycle)");
  if (restart < 1 || restart > 63) fail("restart must be between 1 and 63");
  DevHier& D = device_of(*H);
  double rr = 0;
  int it;
  if (host) {
    DR_CK(cudaMemcpyAsync(D.xbuf(), x, (size_t)n * sizeof(double), cudaMemcpyHostToDevice, D.stream()));
    DR_CK(cudaMemcpyAsync(D.bbuf(), b, (size_t)n * sizeof(double), cudaMemcpyHostToDevice, D.stream()));
    it = D.fgmres(D.xbuf(), D.bbuf(), opts_of(c), tol, maxiter, restart, precision == 1, &rr, c.verbose);
    DR_CK(cudaMemcpyAsync(x, D.xbuf(), (size_t)n * sizeof(double), cudaMemcpyDeviceToHost, D.stream()));
    DR_CK(cudaStreamSynchronize(D.stream()));
  } else {
    it = D.fgmres(x, b, opts_of(c), tol, maxiter, restart, precision == 1, &rr, c.verbose);
  }
  if (relres) *relres = rr;
  return it;
}

int32_t draugr_b200_fgmres(int32_t handle, int32_t n, double* x, const double* b, int32_t config_handle,
                           double tol, int32_t maxiter, int32_t restart, int32_t precision, double* relres) {
  return guarded("draugr_b200_fgmres", [&]() {
    return fgmres_impl(handle, n, x, b, config_handle, tol, maxiter, restart, precision, relres, true);
  });
}

int32_t draugr_b200_fgmres_device(int32_t handle, int32_t n, double* x_dev, const double* b_dev,
                                  int32_t config_handle, double tol, int32_t maxiter, int32_t restart,
                                  int32_t precision, double* relres) {
  return guarded("draugr_b200_fgmres_device", [&]() {
    return fgmres_impl(handle, n, x_dev, b_dev, config_handle, tol, maxiter, restart, precision, relres, false);
  });
}

static int32_t refine_impl(int32_t handle, int32_t n, double* x, const double* b, int32_t config_handle,
                           double tol, int32_t max_outer, double inner_tol, int32_t inner_maxiter,
                           int32_t inner_method, int32_t precision, double* relres, int32_t* inner_iters,
                           bool host) {
  Config c;
  auto H = get_hier(handle, config_handle, &c);
  if (n != n_finest(*H)) fail("DimensionMismatch");
  if (!x || !b) fail("ArgumentError: NULL vector");
  if (precision != 0 && precision != 1) fail("precision must be 0 (FP64 cycle) or 1 (FP32 cycle)");
  if (inner_method != 0 && inner_method != 1) fail("inner_method must be 0 (PCG) or 1 (FGMRES)");
  if (!(inner_tol > 0.0 && inner_tol < 1.0)) fail("inner_tol must lie in (0, 1)");
  DevHier& D = device_of(*H);
  double rr = 0;
  int inner = 0, steps;
  if (host) {
    DR_CK(cudaMemcpyAsync(D.xbuf(), x, (size_t)n * sizeof(double), cudaMemcpyHostToDevice, D.stream()));
    DR_CK(cudaMemcpyAsync(D.bbuf(), b, (size_t)n * sizeof(double), cudaMemcpyHostToDevice, D.stream()));
    steps = D.refine(D.xbuf(), D.bbuf(), opts_of(c), tol, max_outer, inner_tol, inner_maxiter, inner_method,
                     precision == 1, &rr, &inner, c.verbose);
    DR_CK(cudaMemcpyAsync(x, D.xbuf(), (size_t)n * sizeof(double), cudaMemcpyDeviceToHost, D.stream()));
    DR_CK(cudaStreamSynchronize(D.stream()));
  } else {
    steps = D.refine(x, b, opts_of(c), tol, max_outer, inner_tol, inner_maxiter, inner_method, precision == 1,
                     &rr, &inner, c.verbose);
  }
  if (relres) *relres = rr;
  if (inner_iters) *inner_iters = inner;
  return steps;
}

int32_t draugr_b200_refine(int32_t handle, int32_t n, double* x, const double* b, int32_t config_handle,
                           double tol, int32_t max_outer, double inner_tol, int32_t inner_maxiter,
                           int32_t inner_method, int32_t precision, double* relres, int32_t* inner_iters) {
  return guarded("draugr_b200_refine", [&]() {
    return refine_impl(handle, n, x, b, config_handle, tol, max_outer, inner_tol, inner_maxiter, inner_method,
                       precision, relres, inner_iters, true);
  });
}

int32_t draugr_b200_refine_device(int32_t handle, int32_t n, double* x_dev, const double* b_dev,
                                  int32_t config_handle, double tol, int32_t max_outer, double inner_tol,
                                  int32_t inner_maxiter, int32_t inner_method, int32_t precision,
                                  double* relres, int32_t* inner_iters) {
  return guarded("draugr_b200_refine_device", [&]() {
    return refine_impl(handle, n, x_dev, b_dev, config_handle, tol, max_outer, inner_tol, inner_maxiter,
                       inner_method, precision, relres, inner_iters, false);
  });
}

int32_t draugr_b200_batch_setup(int32_t nsys, const int32_t* handles) {
  return guarded("draugr_b200_batch_setup", [&]() -> int32_t {
    if (nsys < 1 || !handles) fail("ArgumentError: a batch needs at least one hierarchy handle");
    std::vector<std::shared_ptr<Hier>> keep;
    std::vector<const HostHierarchy*> hs;
    for (int32_t s = 0; s < nsys; ++s) {
      keep.push_back(get_hier_only(handles[s]));
      if (keep.back()->batch) fail("a batch cannot contain another batch");
      hs.push_back(&keep.back()->host);
    }
    auto B = std::make_shared<Hier>();
    B->batch = std::make_unique<BatchLayout>();
    B->host = merge_batch(hs, *B->batch);
    device_of(*B);
    std::lock_guard<std::mutex> lk(g_mu);
    int32_t h = new_handle();
    g_hier[h] = B;
    return h;
  });
}

int32_t draugr_b200_batch_offsets(int32_t handle, int64_t* offsets) {
  return guarded("draugr_b200_batch_offsets", [&]() -> int32_t {
    auto H = get_hier_only(handle);
    if (!H->batch) fail("not a batch handle");
    const BatchLayout& L = *H->batch;
    if (offsets) {
      for (int s = 0; s < L.nsys; ++s) offsets[s] = L.off[0][s];
      offsets[L.nsys] = L.ntotal[0];
    }
    return L.nsys;
  });
}

int32_t draugr_b200_batch_pcg_device(int32_t handle, int32_t n, double* x_dev, const double* b_dev,
                                     int32_t config_handle, double tol, int32_t maxiter, int32_t precision,
                                     int32_t* iters, double* relres) {
  return guarded("draugr_b200_batch_pcg_device", [&]() -> int32_t {
    Config c;
    auto H = get_hier(handle, config_handle, &c);
    if (!H->batch) fail("not a batch handle");
    if (n != H->batch->ntotal[0]) fail("DimensionMismatch: n must be the batch's total rows");
    if (precision != 0 && precision != 1) fail("precision must be 0 (FP64 cycle) or 1 (FP32 cycle)");
    if (!x_dev || !b_dev) fail("ArgumentError: NULL vector");
    if (c.cycle_w) fail("batched solves run V-cycles");
    return device_of(*H).pcg_batch_seg(x_dev, b_dev, opts_of(c), tol, maxiter, precision == 1, iters, relres,
                                       c.verbose);
  });
}

int32_t draugr_b200_pcg_block_device(int32_t handle, int32_t n, int32_t k, double* X_dev, const double* B_dev,
                                     int32_t config_handle, double tol, int32_t maxiter, int32_t precision,
                                     int32_t* iters, double* relres) {
  return guarded("draugr_b200_pcg_block_device", [&]() -> int32_t {
    Config c;
    auto H = get_hier(handle, config_handle, &c);
    if (n != n_finest(*H)) fail("DimensionMismatch");
    if (precision != 0 && precision != 1) fail("precision must be 0 (FP64 cycle) or 1 (FP32 cycle)");
    if (!X_dev || !B_dev) fail("ArgumentError: NULL block");
    return device_of(*H).pcg_block(X_dev, B_dev, k, opts_of(c), tol, maxiter, precision == 1, iters, relres,
                                   c.verbose);
  });
}

int32_t draugr_b200_nz_gradient_device(int32_t handle, int32_t n, const double* x_dev,
                                       const double* lambda_dev, double* grad_dev) {
  return guarded("draugr_b200_nz_gradient_device", [&]() -> int32_t {
    auto H = get_hier_only(handle);
    if (n != n_finest(*H)) fail("DimensionMismatch");
    if (!x_dev || !lambda_dev || !grad_dev) fail("ArgumentError: NULL vector");
    device_of(*H).nz_gradient(x_dev, lambda_dev, grad_dev);
    return 0;
  });
}

int32_t draugr_b200_level_op(int32_t handle, int32_t lvl, int32_t op, int32_t precision, const double* in1,
                             const double* in2, double* out, int32_t steps) {
  return guarded("draugr_b200_level_op", [&]() -> int32_t {
    auto H = get_hier_only(handle);
    DevHier& D = device_of(*H);
    const auto& levels = H->host.levels;
    const int nl = (int)levels.size();
    if (op != 5 && (lvl < 0 || lvl >= nl)) fail("level index out of range");
    const int n = op == 5 ? H->host.nc : levels[lvl].A.n;
    const int nc = op == 5 ? H->host.nc : levels[lvl].P.nc;
    int n_in1 = n, n_in2 = 0, n_out = n;
    switch (op) {
      case 0: break;
      case 1: n_in2 = n; break;
      case 2: n_in2 = n; break;
      case 3: n_out = nc; break;
      case 4: n_in2 = nc; break;
      case 5: break;
      case 6: n_out = 2 * n; break;
      default: fail("unknown level op " + std::to_string(op));
    }
    if (!in1 || (n_in2 && !in2) || !out) fail("ArgumentError: NULL array");
    double *d1 = nullptr, *d2 = nullptr, *d3 = nullptr;
    auto cleanup = [&]() { cudaFree(d1); cudaFree(d2); cudaFree(d3); };
    try {
      DR_CK(cudaMalloc(&d1, std::max(1, n_in1) * sizeof(double)));
      DR_CK(cudaMalloc(&d2, std::max(1, n_in2) * sizeof(double)));
      DR_CK(cudaMalloc(&d3, std::max(1, n_out) * sizeof(double)));
      DR_CK(cudaMemcpy(d1, in1, n_in1 * sizeof(double), cudaMemcpyHostToDevice));
      if (n_in2) DR_CK(cudaMemcpy(d2, in2, n_in2 * sizeof(double), cudaMemcpyHostToDevice));
      D.level_op(lvl, op, precision == 1, d1, d2, d3, steps);
      DR_CK(cudaMemcpy(out, d3, n_out * sizeof(double), cudaMemcpyDeviceToHost));
    } catch (...) {
      cleanup();
      throw;
    }
    cleanup();
    return 0;
  });
}

int32_t draugr_b200_time_level_op(int32_t handle, int32_t lvl, int32_t op, int32_t precision, int32_t reps,
                                  float* ms_per_launch) {
  return guarded("draugr_b200_time_level_op", [&]() -> int32_t {
    auto H = get_hier_only(handle);
    DevHier& D = device_of(*H);
    if (reps < 1) fail("reps must be >= 1");
    float ms = D.time_level_op(lvl, op, precision == 1, reps);
    if (ms_per_launch) *ms_per_launch = ms;
    return 0;
  });
}

int64_t draugr_b200_kernel_launches(void) { return kernel_launches(); }

void draugr_b200_set_tile_wait_limit(int32_t polls) { set_tile_wait_limit(polls); }

int32_t draugr_b200_set_stream(int32_t handle, void* stream) {
  return guarded("draugr_b200_set_stream", [&]() -> int32_t {
    auto H = get_hier_only(handle);
    device_of(*H).set_stream((cudaStream_t)stream);
    return 0;
  });
}

}  // extern "C"
