// Device hierarchy, V/W cycle, stationary AMG solve, AMG-preconditioned CG
// and the numeric resetup (sm_100a).
//
// Reference behaviour reproduced here (Draugr.jl):
//   amg_cycle! / _vcycle_descend!  src/cycle.jl:12-28, :63-99
//   amg_solve!                     src/cycle.jl:110-160
//   amg_resetup! (partial)         src/resetup.jl:20-45, :95-158
//   preconditioner_apply!          src/preconditioner.jl:76-80 (x zeroed, one cycle)
// Differences in form, not in result: the Jacobi ping-pong of
// src/smoothers.jl:103-124 swaps buffer pointers instead of copying back;
// the first Jacobi step from a zero iterate (every coarse level, and the
// finest level inside PCG) needs no product with A, so it is evaluated
// inside the residual kernel that follows it; restriction uses Pᵀ stored
// with values in transpose-map order, so no index indirection is needed.
#include <cuda_runtime.h>

#include <cub/device/device_scan.cuh>

#include <algorithm>
#include <chrono>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <type_traits>
#include <unordered_map>

#include "dr_device.h"
#include "dr_kernels.cuh"

namespace dr {

using namespace kern;

// Kernels launched by this library (host-side count; a CUDA graph adds the
// number of kernels captured in it on every launch).
static std::atomic<long long> g_launches{0};
long long kernel_launches() { return g_launches.load(); }
static inline void counted() { g_launches.fetch_add(1, std::memory_order_relaxed); }
void note_launch() { counted(); }

// SM count of the device in use and a device flag the row kernels set when a
// bounded wait gives up (checked after every solve / resetup).
static std::atomic<int> g_nsm{148};  // SM count (written by every hierarchy constructor)
// Flag a row kernel sets when a bounded wait gave up, one per device
// (allocated once, under a lock: hierarchies may be built from several
// host threads).  Shared by the hierarchies of a device; the host reads and
// clears it after each solve.
static std::mutex g_err_mu;
static std::atomic<int*> g_err_dev[64];

static int* err_flag() {
  int dev = 0;
  DR_CK(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) fail("device index out of range");
  int* p = g_err_dev[dev].load(std::memory_order_acquire);
  if (p) return p;
  std::lock_guard<std::mutex> lk(g_err_mu);
  p = g_err_dev[dev].load(std::memory_order_relaxed);
  if (!p) {
    DR_CK(cudaMalloc(&p, sizeof(int)));
    DR_CK(cudaMemset(p, 0, sizeof(int)));
    g_err_dev[dev].store(p, std::memory_order_release);
  }
  return p;
}

// Polls a row kernel makes on a tile's copy before it gives up.  Only the
// test hook draugr_b200_set_tile_wait_limit lowers it (0 makes every row
// kernel give up at once and report the timeout).
static std::atomic<int> g_tile_wait_limit{kern::kWaitLimit};
static int tile_wait_limit() { return g_tile_wait_limit.load(std::memory_order_relaxed); }
void set_tile_wait_limit(int polls) { g_tile_wait_limit.store(polls < 0 ? kern::kWaitLimit : polls); }

void cuda_check(cudaError_t e, const char* what, const char* file, int line) {
  if (e != cudaSuccess) {
    cudaGetLastError();
    char buf[512];
    std::snprintf(buf, sizeof buf, "CUDA error %d (%s) in %s at %s:%d", (int)e, cudaGetErrorString(e),
                  what, file, line);
    fail(buf);
  }
}

namespace {

// Lanes per row for the Gauss-Seidel colour kernel: about the mean row length.
int pick_G(long long nnz, int n) {
  if (n <= 0) return 1;
  double avg = (double)nnz / (double)n;
  int G = 1;
  while (G < 32 && G < avg * 0.75) G *= 2;
  return G;
}

// Greedy packing of consecutive rows into tiles of at most max_rows rows,
// kTileCap nonzeros and a column span below 65536 (so that a tile's columns
// are 16-bit offsets from its smallest column).  A row longer than kTileCap,
// or spanning 65536 columns or more by itself, is a tile of its own.
// Returns the tile row starts; `base` receives each tile's smallest column,
// -1 for a row too wide for offsets.
std::vector<int> make_tiles(const std::vector<int>& rp, const std::vector<int>& ci, int n,
                            int max_rows, std::vector<int>& base) {
  std::vector<int> tp;
  tp.reserve(n / std::max(1, max_rows) + 2);
  tp.push_back(0);
  base.clear();
  int r = 0;
  while (r < n) {
    int rows = 0, nz = 0;
    bool have = false;  // any column in the tile yet
    long long lo = 0, hi = 0;
    while (r < n && rows < max_rows) {
      const int len = rp[r + 1] - rp[r];
      long long rlo = 0, rhi = 0;
      if (len > 0) {
        rlo = rhi = ci[rp[r]];
        for (int k = rp[r] + 1; k < rp[r + 1]; ++k) {
          rlo = std::min<long long>(rlo, ci[k]);
          rhi = std::max<long long>(rhi, ci[k]);
        }
      }
      long long nlo = lo, nhi = hi;
      bool nhave = have;
      if (len > 0) {
        nlo = have ? std::min(lo, rlo) : rlo;
        nhi = have ? std::max(hi, rhi) : rhi;
        nhave = true;
      }
      if (rows > 0 && (nz + len > kTileCap || (nhave && nhi - nlo >= 65536))) break;
      nz += len;
      lo = nlo;
      hi = nhi;
      have = nhave;
      ++rows;
      ++r;
      if (len > kTileCap || (len > 0 && rhi - rlo >= 65536)) break;
    }
    tp.push_back(r);
    base.push_back(!have ? 0 : (hi - lo >= 65536 ? -1 : (int)lo));
  }
  return tp;
}

static_assert(kTileCap == kRowTileCap, "host and device tile capacities differ");

// Launch with programmatic stream serialization: the kernel may begin
// while the previous kernel in the stream drains.  Only for kernels that
// read nothing but sparsity patterns before pdl_wait() (k_tile_rows,
// k_coarse_tail, k_pcg_update).
template <typename... KArgs, typename... Args>
void launch_dependent(void (*kern)(KArgs...), int grid, int block, size_t smem, cudaStream_t st,
                      Args&&... args) {
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = dim3((unsigned)grid);
  cfg.blockDim = dim3((unsigned)block);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  DR_CK(cudaLaunchKernelEx(&cfg, kern, std::forward<Args>(args)...));
}

// Blocks of `nt` threads with `smem` dynamic shared memory that fit on one
// SM at once, per kernel (queried once).
int resident_blocks(const void* f, int nt, size_t smem) {
  static std::mutex mu;
  static std::unordered_map<const void*, int> cache;
  std::lock_guard<std::mutex> lk(mu);
  auto it = cache.find(f);
  if (it != cache.end()) return it->second;
  int nb = 0;
  DR_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, f, nt, smem));
  nb = std::max(1, nb);
  cache.emplace(f, nb);
  return nb;
}

template <typename TA, class XL, class EP, bool DOT, class Fin>
void launch_rows_impl(cudaStream_t st, int max_grid, const DevMat& M, const TA* av, XL xl, EP ep,
                      double* partials, unsigned* ticket, Fin fin) {
  const RowForm& f = M.form;
  const int n = M.n, ntiles = M.ntiles;
  const int *tp = M.tp, *ts = M.ts, *tb = M.tb, *rp = M.rp, *ci = M.ci;
  const uint16_t* cu = M.cu;
  if (n <= 0) {
    if constexpr (DOT) {
      // an empty reduction still has to deliver its (zero) result
      counted();
      k_dot<double, double, Fin><<<1, kBlock, 0, st>>>(0, nullptr, nullptr, partials, ticket, fin);
    }
    return;
  }
  counted();
  // one wave of resident blocks (registers and shared memory permitting)
#define DR_LAUNCH(F, g, O, NT, B, TC)                                                            \
  do {                                                                                           \
    auto kf = k_tile_rows<F, g, O, NT, B, TA, TC, XL, EP, DOT, Fin>;                             \
    const size_t smem = tile_smem_bytes<TA, TC>();                                               \
    const int grid = std::max(                                                                   \
        1, std::min({ntiles, max_grid, g_nsm * resident_blocks((const void*)kf, NT, smem)}));    \
    launch_dependent(kf, grid, NT, smem, st, ntiles, tp, ts, tb, rp, ci, cu, av, xl, ep, partials, \
                     ticket, fin, err_flag(), tile_wait_limit());                                \
  } while (0)
  // 16-bit column offsets where lanes read consecutive entries (flat and
  // tree forms), and for FP32 rows of 12-32 entries, where the bytes saved
  // outweigh the bank conflicts of 16-bit reads at a row stride; the
  // columns themselves for the other one-lane-per-row forms (measured on the
  // 128^3 hierarchy: both choices per form, FP64 and FP32)
  if (f.flat) DR_LAUNCH(true, 1, true, 256, 8, uint16_t);
  else if (f.G == 1 && f.nt == 128 && sizeof(TA) == 4) DR_LAUNCH(false, 1, true, 128, 32, uint16_t);
  else if (f.G == 1 && f.nt == 128) DR_LAUNCH(false, 1, true, 128, 32, int);
  else if (f.G == 1 && f.nt == 512) DR_LAUNCH(false, 1, true, 512, 4, int);
  else if (f.G == 1) DR_LAUNCH(false, 1, true, 256, 8, int);
  else if (f.G == 8) DR_LAUNCH(false, 8, false, 256, 12, uint16_t);
  else if (f.G == 16) DR_LAUNCH(false, 16, false, 256, 12, uint16_t);
  else if (f.G == 32) DR_LAUNCH(false, 32, false, 256, 4, uint16_t);
  else fail("bad row form");
#undef DR_LAUNCH
  DR_CK(cudaGetLastError());
}

template <typename TA, class XL, class EP>
void launch_rows(cudaStream_t st, int max_grid, const DevMat& M, const TA* av, XL xl, EP ep) {
  launch_rows_impl<TA, XL, EP, false, FinStore>(st, max_grid, M, av, xl, ep, nullptr, nullptr,
                                                FinStore{nullptr});
}

template <typename TA, class XL, class EP, class Fin>
void launch_rows_dot(cudaStream_t st, int max_grid, const DevMat& M, const TA* av, XL xl, EP ep,
                     double* partials, unsigned* ticket, Fin fin) {
  launch_rows_impl<TA, XL, EP, true, Fin>(st, max_grid, M, av, xl, ep, partials, ticket, fin);
}

int grid1d(long long n, int max_grid) {
  return (int)std::max<long long>(1, std::min<long long>((n + kBlock - 1) / kBlock, max_grid));
}

// Finalizer writing the same total to two places (r·z and its "old" copy).
struct FinStore2 {
  double* a;
  double* b;
  __device__ void operator()(double s) const {
    *a = s;
    *b = s;
  }
};

// ticket slots
enum : int { TK_DOT = 0, TK_RES = 1, TK_PQ = 2, TK_UPD = 3, TK_RZ = 4, TK_N = 8 };
// scalar slots
enum : int { SC_BB = 0, SC_RR = 1, SC_RZ = 2, SC_RZOLD = 3, SC_PQ = 4, SC_TMP = 5, SC_ALPHA = 6, SC_N = 8 };

}  // namespace

template <typename T>
T* DevHier::alloc(size_t n) {
  void* p = nullptr;
  // a multiple of 16 bytes, so a 16-byte-rounded bulk copy of any prefix of
  // the array stays inside the allocation
  size_t bytes = (std::max<size_t>(n, 1) * sizeof(T) + 15) & ~(size_t)15;
  DR_CK(cudaMalloc(&p, bytes));
  allocs_.push_back(p);
  bytes_ += bytes;
  return (T*)p;
}
template double* DevHier::alloc<double>(size_t);
template float* DevHier::alloc<float>(size_t);
template int* DevHier::alloc<int>(size_t);
template long long* DevHier::alloc<long long>(size_t);

template <typename T>
static void h2d(T* d, const std::vector<T>& h, cudaStream_t st) {
  if (!h.empty()) DR_CK(cudaMemcpyAsync(d, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice, st));
}

DevHier::DevHier(const HostHierarchy& H, int device, const BatchLayout* batch) {
  device_ = device;
  if (batch) batch_ = std::make_unique<BatchLayout>(*batch);
  DR_CK(cudaSetDevice(device));
  DR_CK(cudaDeviceGetAttribute(&nsm_, cudaDevAttrMultiProcessorCount, device));
  max_grid_ = nsm_ * 8;
  g_nsm = nsm_;
  err_flag();
  DR_CK(cudaStreamCreateWithFlags(&own_st_, cudaStreamNonBlocking));
  st_ = own_st_;
  own_stream_ = true;
  DR_CK(cudaEventCreateWithFlags(&ev_[0], cudaEventDisableTiming));
  DR_CK(cudaEventCreateWithFlags(&ev_[1], cudaEventDisableTiming));
  DR_CK(cudaStreamCreateWithFlags(&side_st_, cudaStreamNonBlocking));
  DR_CK(cudaEventCreateWithFlags(&ev_fork_, cudaEventDisableTiming));
  DR_CK(cudaEventCreateWithFlags(&ev_join_, cudaEventDisableTiming));
  try {
    const int nl = (int)H.levels.size();
    n0_ = nl ? H.levels[0].A.n : H.nc;
    nnz0_ = nl ? H.levels[0].A.nnz() : H.coarse.nnz();
    L_.resize(nl);
    auto up_csr = [&](DevMat& M, int n, int m, const std::vector<int>& rp, const std::vector<int>& ci,
                      const std::vector<double>* v) { upload_csr(M, n, m, rp, ci, v); };
    for (int l = 0; l < nl; ++l) {
      const HostLevel& h = H.levels[l];
      DevLevel& d = L_[l];
      up_csr(d.A, h.A.n, h.A.m, h.A.rp, h.A.ci, &h.A.v);
      up_csr(d.P, h.P.nf, h.P.nc, h.P.rp, h.P.ci, &h.P.v);
      up_csr(d.R, h.P.nc, h.P.nf, h.T.off, h.T.rows, &h.Rv);
      d.smoother = h.smoother;
      d.omega = h.omega;
      d.nv = batch ? batch->ntotal[l] : h.A.n;
      d.invd = alloc<double>(d.nv);
      if (d.nv > h.A.n) DR_CK(cudaMemsetAsync(d.invd, 0, (size_t)d.nv * sizeof(double), st_));
      h2d(d.invd, h.invdiag, st_);
      d.ncolors = h.num_colors;
      d.color_off = h.color_off;
      if (h.num_colors > 0) {
        d.color_order = alloc<int>(h.color_order.size());
        h2d(d.color_order, h.color_order, st_);
      }
      d.has_rap = h.has_rap_map;
      if (d.has_rap || !h.ap_rp.empty()) up_csr(d.AP, h.A.n, h.P.nc, h.ap_rp, h.ap_ci, nullptr);

      const int n = d.nv;
      if (l > 0) {
        d.v64.xa = alloc<double>(n);
        d.v64.b = alloc<double>(n);
      }
      d.v64.xb = alloc<double>(n);
      d.v64.r = alloc<double>(n);
      if (h.smoother == SmootherKind::SPAI1) {
        d.spai1_M = alloc<double>(h.A.v.size() + 4);
        h2d(d.spai1_M, h.spai1_M, st_);
        d.v64.d = alloc<double>(n);
        d.ilu_rp = h.A.rp;  // host pattern for recomputing M after a resetup
        d.ilu_ci = h.A.ci;
      }
      if (h.smoother == SmootherKind::SerialGS || h.smoother == SmootherKind::L1SerialGS) {
        d.sgs_order = alloc<int>(n);
        h2d(d.sgs_order, h.sgs_order, st_);
        d.sgs_off = h.sgs_off;
      }
      if (h.smoother == SmootherKind::ILU0 || h.smoother == SmootherKind::SerialILU0) {
        d.ilu_diag = alloc<int>(n);
        h2d(d.ilu_diag, h.ilu_diag, st_);
        d.ilu_L = alloc<double>(h.A.v.size() + 4);
        d.ilu_U = alloc<double>(h.A.v.size() + 4);
        h2d(d.ilu_L, h.ilu_L, st_);
        h2d(d.ilu_U, h.ilu_U, st_);
        d.ilu_fwd = alloc<int>(n);
        d.ilu_bwd = alloc<int>(n);
        h2d(d.ilu_fwd, h.ilu_fwd_order, st_);
        h2d(d.ilu_bwd, h.ilu_bwd_order, st_);
        d.ilu_fwd_off = h.ilu_fwd_off;
        d.ilu_bwd_off = h.ilu_bwd_off;
        d.ilu_rp = h.A.rp;
        d.ilu_ci = h.A.ci;
        d.ilu_diag_h = h.ilu_diag;
        d.v64.d = alloc<double>(n);
      }
      if (h.smoother == SmootherKind::Chebyshev) {
        d.cheb_degree = h.cheb_degree;
        d.cheb_v0 = alloc<double>(n);
        h2d(d.cheb_v0, h.cheb_v0, st_);
        d.cheb_coef = alloc<double>(2 * (size_t)h.cheb_degree + 2);
        h2d(d.cheb_coef, h.cheb_coef, st_);
        d.v64.d = alloc<double>(n);
      }
    }
    nc_ = H.nc;
    up_csr(C_, H.coarse.n, H.coarse.m, H.coarse.rp, H.coarse.ci, &H.coarse.v);
    info_ = alloc<int>(1);
    if (!batch) {
      cdense_ = alloc<double>((size_t)nc_ * nc_);
      clu_ = alloc<double>((size_t)nc_ * nc_);
      cpiv_ = alloc<int>(nc_);
      h2d(cdense_, H.coarse_dense, st_);
      h2d(clu_, H.coarse_lu, st_);
      h2d(cpiv_, H.coarse_piv, st_);
    } else {
      // the coarsest systems of the batch, per merged level
      blu_ = alloc<double>(batch->lu.size());
      bpiv_ = alloc<int>(batch->piv.size());
      h2d(blu_, batch->lu, st_);
      h2d(bpiv_, batch->piv, st_);
      batch_dev_.resize(batch->coarse.size());
      for (size_t l = 0; l < batch->coarse.size(); ++l) {
        const BatchLayout::Coarse& c = batch->coarse[l];
        BatchDev& b = batch_dev_[l];
        b.nblk = (int)c.off.size();
        b.maxn = c.maxn;
        if (!b.nblk) continue;
        b.off = alloc<int>(c.off.size());
        b.nb = alloc<int>(c.nb.size());
        b.poff = alloc<int>(c.poff.size());
        b.luoff = alloc<long long>(c.luoff.size());
        h2d(b.off, c.off, st_);
        h2d(b.nb, c.nb, st_);
        h2d(b.poff, c.poff, st_);
        h2d(b.luoff, c.luoff, st_);
        if (b.maxn <= kern::kInvMax) {
          // the merged cycle is not bit-exact against the systems' own
          // anyway: apply each coarsest system's explicit inverse
          if (!binv_) binv_ = alloc<double>(std::max<size_t>(batch->lu.size(), 1));
          counted();
          k_lu_inverse_batch<<<b.nblk, kern::kInvMax, 0, st_>>>(b.nb, b.luoff, b.poff, blu_, bpiv_, binv_);
          DR_CK(cudaGetLastError());
          b.inv = true;
        }
      }
      // finest-level segments: system s occupies rows off[0][s] .. off[0][s + 1] - 1
      std::vector<int> so(batch->nsys + 1, 0), sid(n0_);
      for (int q = 0; q < batch->nsys; ++q) so[q] = batch->off[0][q];
      so[batch->nsys] = n0_;
      for (int q = 0; q < batch->nsys; ++q)
        for (int i = so[q]; i < so[q + 1]; ++i) sid[i] = q;
      seg_off_ = alloc<int>(so.size());
      seg_id_ = alloc<int>(sid.size());
      h2d(seg_off_, so, st_);
      h2d(seg_id_, sid, st_);
      DR_CK(cudaStreamSynchronize(st_));
    }
    cb64_ = alloc<double>(nc_);
    cx64_ = alloc<double>(nc_);
    partials_ = alloc<double>(max_grid_ + 32);
    tickets_ = alloc<unsigned>(TK_N);
    DR_CK(cudaMemsetAsync(tickets_, 0, TK_N * sizeof(unsigned), st_));
    scal_ = alloc<double>(SC_N);
    DR_CK(cudaMemsetAsync(scal_, 0, SC_N * sizeof(double), st_));
    DR_CK(cudaMallocHost(&hscal_, SC_N * sizeof(double)));
    xd_ = alloc<double>(n0_);
    bd_ = alloc<double>(n0_);
    if (!batch && (size_t)nc_ * sizeof(double) > 48 * 1024) {
      size_t need = (size_t)nc_ * sizeof(double);
      if (need > 200 * 1024) fail("coarsest level too large for the on-chip LU solve (n_c = " + std::to_string(nc_) + ")");
      DR_CK(cudaFuncSetAttribute(k_lu_solve<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)need));
      DR_CK(cudaFuncSetAttribute(k_lu_solve<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)need));
    }
    if (!batch) {
      // the coarsest inverse, for hierarchies whose cycle is not bit-exact
      // anyway (some level sums its rows in a tree)
      bool any_tree = false;
      for (int l = 0; l < nl; ++l) any_tree = any_tree || !L_[l].A.form.ordered;
      cinv_ok_ = any_tree && nc_ >= 1 && nc_ <= kern::kInvMax;
      if (cinv_ok_) build_cinv();
    }
    if (batch) tail_ = nl;  // no shared-memory tail: every level runs as its own launches
    else build_tail();
    build_fused(H);
    DR_CK(cudaStreamSynchronize(st_));
  } catch (...) {
    for (void* p : allocs_) cudaFree(p);
    allocs_.clear();
    if (hscal_) cudaFreeHost(hscal_);
    cudaEventDestroy(ev_[0]);
    cudaEventDestroy(ev_[1]);
    cudaEventDestroy(ev_fork_);
    cudaEventDestroy(ev_join_);
    cudaStreamDestroy(side_st_);
    cudaStreamDestroy(own_st_);
    throw;
  }
}

// Upload a CSR pattern (and optionally values) with the row kernel's
// tiling and 16-bit column offsets.  Host arrays must outlive the stream's
// copies (callers synchronise the stream before releasing them).
void DevHier::upload_csr(DevMat& M, int n, int m, const std::vector<int>& rp, const std::vector<int>& ci,
                       const std::vector<double>* v) {
  M.n = n;
  M.m = m;
  M.nnz = (long long)ci.size();
  M.rp = alloc<int>(rp.size());
  // column and value arrays carry 4 padding entries for the tile
  // kernel's 128-bit loads
  M.ci = alloc<int>(ci.size() + 4);
  h2d(M.rp, rp, st_);
  h2d(M.ci, ci, st_);
  M.v = alloc<double>(ci.size() + 4);
  if (v) h2d(M.v, *v, st_);
  M.Ggs = pick_G(M.nnz, n);
  M.form = row_form(rp);
  M.maxlen = 0;
  for (int i = 0; i < n; ++i) M.maxlen = std::max(M.maxlen, rp[i + 1] - rp[i]);
  std::vector<int> base;
  std::vector<int> tiles = make_tiles(rp, ci, n, M.form.nt / M.form.G, base);
  std::vector<int> tstart(tiles.size());
  for (size_t t = 0; t < tiles.size(); ++t) tstart[t] = rp[tiles[t]];
  M.ntiles = (int)tiles.size() - 1;
  M.tp = alloc<int>(tiles.size());
  M.ts = alloc<int>(tiles.size());
  M.tb = alloc<int>(base.size());
  DR_CK(cudaMemcpy(M.tp, tiles.data(), tiles.size() * sizeof(int), cudaMemcpyHostToDevice));
  DR_CK(cudaMemcpy(M.ts, tstart.data(), tstart.size() * sizeof(int), cudaMemcpyHostToDevice));
  DR_CK(cudaMemcpy(M.tb, base.data(), base.size() * sizeof(int), cudaMemcpyHostToDevice));
  // 16-bit column offsets from each tile's smallest column (8 padding
  // entries for the tile kernel's 16-byte-rounded copies)
  std::vector<uint16_t> off(ci.size() + 8, 0);
  for (int t = 0; t < M.ntiles; ++t)
    if (base[t] >= 0)
      for (int k = tstart[t]; k < tstart[t + 1]; ++k) off[k] = (uint16_t)(ci[k] - base[t]);
  M.cu = alloc<uint16_t>(off.size());
  DR_CK(cudaMemcpy(M.cu, off.data(), off.size() * sizeof(uint16_t), cudaMemcpyHostToDevice));
  }

DevHier::~DevHier() {
  cudaSetDevice(device_);
  if (st_) cudaStreamSynchronize(st_);
  graphs_clear();
  if (seg_graph_) cudaGraphExecDestroy(seg_graph_);
  for (void* p : allocs_) cudaFree(p);
  if (hscal_) cudaFreeHost(hscal_);
  cudaEventDestroy(ev_[0]);
  cudaEventDestroy(ev_[1]);
  if (ev_fork_) cudaEventDestroy(ev_fork_);
  if (ev_join_) cudaEventDestroy(ev_join_);
  if (side_st_) cudaStreamDestroy(side_st_);
  if (own_stream_ && own_st_) cudaStreamDestroy(own_st_);
}

// Raise if a row kernel reported a bounded wait that gave up (the flag is
// cleared so the hierarchy stays usable).
static void check_kernel_flag(cudaStream_t st) {
  int e = 0;
  int* flag = err_flag();
  DR_CK(cudaMemcpyAsync(&e, flag, sizeof(int), cudaMemcpyDeviceToHost, st));
  DR_CK(cudaStreamSynchronize(st));
  if (e) {
    DR_CK(cudaMemsetAsync(flag, 0, sizeof(int), st));
    DR_CK(cudaStreamSynchronize(st));
    fail("a row kernel timed out waiting for its tile copy (results discarded)");
  }
}

void DevHier::check_errors() { check_kernel_flag(st_); }

void DevHier::set_stream(cudaStream_t s) {
  DR_CK(cudaStreamSynchronize(st_));
  st_ = s ? s : own_st_;
  graphs_clear();
}

void DevHier::graphs_clear() {
  for (int i = 0; i < 2; ++i)
    if (pg_.g1[i]) { cudaGraphExecDestroy(pg_.g1[i]); pg_.g1[i] = nullptr; }
  for (int i = 0; i < 2; ++i)
    if (pg_.g2[i]) { cudaGraphExecDestroy(pg_.g2[i]); pg_.g2[i] = nullptr; }
  pg_.valid = false;
}

// ------------------------------------------------------------ typed accessors
template <> LevelVecs<double>& DevHier::vecs<double>(int l) { return L_[l].v64; }
template <> LevelVecs<float>& DevHier::vecs<float>(int l) { return L_[l].v32; }
template <> double* DevHier::coarse_b<double>() { return cb64_; }
template <> float* DevHier::coarse_b<float>() { return cb32_; }
template <> double* DevHier::coarse_x<double>() { return cx64_; }
template <> float* DevHier::coarse_x<float>() { return cx32_; }
template <> const double* DevHier::mval<double>(const DevMat& M) const { return M.v; }
template <> const float* DevHier::mval<float>(const DevMat& M) const { return M.v32; }
template <> const double* DevHier::qval<double>(const DevLevel& d) const { return d.q; }
template <> const float* DevHier::qval<float>(const DevLevel& d) const { return d.q32; }
template <> const double* DevHier::invd<double>(const DevLevel& L) const { return tr_ ? L.invdT : L.invd; }
template <> const float* DevHier::invd<float>(const DevLevel& L) const { return tr_ ? L.invdT32 : L.invd32; }

// ------------------------------------------------------------ FP32 copies
void DevHier::ensure_fp32() {
  if (fp32_) return;
  graphs_clear();
  for (auto& d : L_) {
    d.A.v32 = alloc<float>(d.A.nnz + 4);
    d.P.v32 = alloc<float>(d.P.nnz + 4);
    d.R.v32 = alloc<float>(d.R.nnz + 4);
    d.invd32 = alloc<float>(d.nv);
    const int n = d.nv;
    d.v32.xa = alloc<float>(n);
    d.v32.xb = alloc<float>(n);
    d.v32.b = alloc<float>(n);
    d.v32.r = alloc<float>(n);
    if (d.smoother == SmootherKind::Chebyshev) d.v32.d = alloc<float>(n);
    if (d.spai1_M) {
      d.v32.d = alloc<float>(n);
      d.spai1_M32 = alloc<float>(d.A.nnz + 4);
    }
    if (d.ilu_L) {
      d.v32.d = alloc<float>(n);
      d.ilu_L32 = alloc<float>(d.A.nnz + 4);
      d.ilu_U32 = alloc<float>(d.A.nnz + 4);
    }
    if (d.fuse_up) d.q32 = alloc<float>(d.AP.nnz + 4);
  }
  cb32_ = alloc<float>(nc_);
  cx32_ = alloc<float>(nc_);
  fp32_ = true;
  if (at_built_) alloc_transpose_fp32();
  refresh_fp32();
  if (!batch_) build_tail();
}

// FP32 copies of the transposed levels' values and smoother diagonals.
void DevHier::alloc_transpose_fp32() {
  for (auto& d : L_) {
    if (!d.At.v32) d.At.v32 = alloc<float>(d.At.nnz + 4);
    if (!d.invdT32) d.invdT32 = alloc<float>(d.A.n);
  }
}

// Levels whose operands fit in the tail kernel's shared memory (all of them
// together, FP64 values, at most kTailSmem bytes), with Jacobi-type
// smoothers, from the coarsest up, run in one block (k_coarse_tail); never
// the finest level (its iterate is the caller's buffer).
static constexpr size_t kTailSmem = 200 * 1024;

static size_t a16(size_t b) { return (b + 15) & ~(size_t)15; }

// Thread -> row order of a tail level (see TailLevel): each warp of 32
// takes one row per starting position modulo 32 while such rows remain,
// then rows from the fullest positions.
static std::vector<int> bank_order(const std::vector<int>& rp) {
  const int n = (int)rp.size() - 1;
  std::vector<std::vector<int>> bucket(32);
  for (int i = 0; i < n; ++i) bucket[rp[i] & 31].push_back(i);
  std::vector<size_t> pos(32, 0);
  std::vector<int> ord;
  ord.reserve(n);
  auto left = [&](int r) { return bucket[r].size() - pos[r]; };
  while ((int)ord.size() < n) {
    int filled = 0;
    for (int r = 0; r < 32; ++r)
      if (left(r) > 0) {
        ord.push_back(bucket[r][pos[r]++]);
        ++filled;
      }
    while (filled < 32 && (int)ord.size() < n) {
      int best = 0;
      for (int r = 1; r < 32; ++r)
        if (left(r) > left(best)) best = r;
      ord.push_back(bucket[best][pos[best]++]);
      ++filled;
    }
  }
  return ord;
}

// Tail levels whose longest row exceeds this form their products flat
// (TailLevel::p), in a shared-memory scratch of one value per nonzero.  The
// environment variable DRAUGR_B200_TAIL_FLAT_ROW overrides it (read at each
// setup; a test hook: the results are the same either way).
static constexpr int kTailFlatRow = 48;
static int tail_flat_row() {
  const char* e = std::getenv("DRAUGR_B200_TAIL_FLAT_ROW");
  return e ? std::atoi(e) : kTailFlatRow;
}

template <typename T>
static size_t tail_level_bytes(const DevLevel& d, int flat_row) {
  const size_t n = d.A.n, nc = d.P.m, an = d.A.nnz, pn = d.P.nnz;
  return a16(4 * (n + 1)) + a16(4 * an) + a16(4 * n) + a16(sizeof(T) * an) + a16(sizeof(T) * n) +
         a16(4 * (n + 1)) + a16(4 * pn) + a16(sizeof(T) * pn) + a16(4 * (nc + 1)) + a16(4 * pn) +
         a16(sizeof(T) * pn) + 4 * a16(sizeof(T) * n) +
         (d.A.maxlen > flat_row ? a16(sizeof(T) * an) : 0);
}

template <typename T>
static size_t tail_coarse_bytes(int nc) {
  return a16(8 * ((size_t)nc * nc + nc)) + a16(4 * (size_t)nc) + 2 * a16(sizeof(T) * nc);
}

// The tail kernel's dynamic shared-memory limit is a per-function setting
// shared by every hierarchy of the process: raise it once per device to
// the opt-in maximum (a limit, not an allocation), so that no hierarchy's
// tail size lowers another's.
template <typename T>
static void allow_tail_smem() {
  static std::mutex mu;
  static bool done[64] = {false};
  int dev = 0;
  DR_CK(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lk(mu);
  if (dev < 0 || dev >= 64 || done[dev]) return;
  int optin = 0;
  DR_CK(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
  int stat = 0;
  {
    cudaFuncAttributes fa{};
    DR_CK(cudaFuncGetAttributes(&fa, k_coarse_tail<T>));
    stat = (int)fa.sharedSizeBytes;
  }
  DR_CK(cudaFuncSetAttribute(k_coarse_tail<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, optin - stat));
  done[dev] = true;
}

void DevHier::build_tail() {
  const int nl = nlevels();
  const int flat_row = tail_flat_row();
  tail_ = nl;
  size_t total = tail_coarse_bytes<double>(nc_);
  std::vector<std::vector<int>> ords;  // from the coarsest level up
  for (int l = nl - 1; l >= 1 && nl - l <= kern::kTailMaxLevels; --l) {
    const DevLevel& d = L_[l];
    const bool jac = jacobi_type(d.smoother);
    total += tail_level_bytes<double>(d, flat_row);
    if (!jac || d.A.n > 4096 || total > kTailSmem) break;
    std::vector<int> rp(d.A.n + 1);
    DR_CK(cudaMemcpy(rp.data(), d.A.rp, rp.size() * sizeof(int), cudaMemcpyDeviceToHost));
    ords.push_back(bank_order(rp));
    tail_ = l;
  }
  if (tail_ >= nl) return;
  tail_inv_ = cinv_ok_ && nc_ <= 32;
  const int cnt = nl - tail_;
  std::reverse(ords.begin(), ords.end());  // tail_ first
  std::vector<int*> ord_dev(cnt);
  for (int k = 0; k < cnt; ++k) {
    ord_dev[k] = alloc<int>(ords[k].size());
    DR_CK(cudaMemcpy(ord_dev[k], ords[k].data(), ords[k].size() * sizeof(int), cudaMemcpyHostToDevice));
  }
  auto make = [&](auto tag) {
    using T = decltype(tag);
    const int slot = sizeof(T) == 8 ? 0 : 1;
    std::vector<TailLevel<T>> v(cnt);
    size_t off = 0;
    auto take = [&](size_t bytes) {
      const unsigned o = (unsigned)off;
      off += a16(bytes);
      return o;
    };
    for (int k = 0; k < cnt; ++k) {
      DevLevel& d = L_[tail_ + k];
      LevelVecs<T>& V = vecs<T>(tail_ + k);
      TailLevel<T>& t = v[k];
      const size_t n = d.A.n, nc = d.P.m;
      t.n = d.A.n;
      t.nc = d.P.m;
      t.annz = (int)d.A.nnz;
      t.pnnz = (int)d.P.nnz;
      t.arp = d.A.rp;
      t.aci = d.A.ci;
      t.ord = ord_dev[k];
      t.av = mval<T>(d.A);
      t.invd = invd<T>(d);
      t.omega = (T)d.omega;
      t.prp = d.P.rp;
      t.pci = d.P.ci;
      t.pv = mval<T>(d.P);
      t.rrp = d.R.rp;
      t.rci = d.R.ci;
      t.rv = mval<T>(d.R);
      t.xa = V.xa;
      t.xb = V.xb;
      t.b = V.b;
      t.r = V.r;
      t.o_arp = take(4 * (n + 1));
      t.o_aci = take(4 * (size_t)d.A.nnz);
      t.o_ord = take(4 * n);
      t.o_av = take(sizeof(T) * (size_t)d.A.nnz);
      t.o_invd = take(sizeof(T) * n);
      t.o_prp = take(4 * (n + 1));
      t.o_pci = take(4 * (size_t)d.P.nnz);
      t.o_pv = take(sizeof(T) * (size_t)d.P.nnz);
      t.o_rrp = take(4 * (nc + 1));
      t.o_rci = take(4 * (size_t)d.P.nnz);
      t.o_rv = take(sizeof(T) * (size_t)d.P.nnz);
      t.o_xa = take(sizeof(T) * n);
      t.o_xb = take(sizeof(T) * n);
      t.o_b = take(sizeof(T) * n);
      t.o_r = take(sizeof(T) * n);
      // the product scratch has no global source: p only marks it (the
      // kernel points p at shared memory)
      const bool flat = d.A.maxlen > flat_row;
      t.o_p = flat ? take(sizeof(T) * (size_t)d.A.nnz) : 0;
      t.p = flat ? reinterpret_cast<T*>(V.r) : nullptr;
    }
    tail_co_[slot][0] = take(8 * ((size_t)nc_ * nc_ + nc_));
    tail_co_[slot][1] = take(4 * (size_t)nc_);
    tail_co_[slot][2] = take(sizeof(T) * (size_t)nc_);
    tail_co_[slot][3] = take(sizeof(T) * (size_t)nc_);
    tail_bytes_[slot] = off;
    // the prologue's bulk copies: patterns, then values, factors and the
    // top level's right-hand side (sizes rounded up to 16 bytes; every
    // source starts an allocation rounded the same way)
    std::vector<TailCopy> pat, val;
    auto rec = [&](std::vector<TailCopy>& l, unsigned o, const void* src, size_t bytes) {
      if (bytes) l.push_back(TailCopy{src, o, (unsigned)a16(bytes)});
    };
    for (int k = 0; k < cnt; ++k) {
      const TailLevel<T>& t = v[k];
      const size_t n = t.n;
      rec(pat, t.o_arp, t.arp, 4 * (n + 1));
      rec(pat, t.o_aci, t.aci, 4 * (size_t)t.annz);
      rec(pat, t.o_ord, t.ord, 4 * n);
      rec(pat, t.o_prp, t.prp, 4 * (n + 1));
      rec(pat, t.o_pci, t.pci, 4 * (size_t)t.pnnz);
      rec(pat, t.o_rrp, t.rrp, 4 * ((size_t)t.nc + 1));
      rec(pat, t.o_rci, t.rci, 4 * (size_t)t.pnnz);
      rec(val, t.o_av, t.av, sizeof(T) * (size_t)t.annz);
      rec(val, t.o_invd, t.invd, sizeof(T) * n);
      rec(val, t.o_pv, t.pv, sizeof(T) * (size_t)t.pnnz);
      rec(val, t.o_rv, t.rv, sizeof(T) * (size_t)t.pnnz);
    }
    rec(val, tail_co_[slot][0], tail_inv_ ? cinv_ : clu_, 8 * (size_t)nc_ * nc_);
    rec(val, tail_co_[slot][1], cpiv_, 4 * (size_t)nc_);
    rec(val, v[0].o_b, v[0].b, sizeof(T) * (size_t)v[0].n);
    TailCopyList& cl = tail_cp_[slot];
    cl.npat = (int)pat.size();
    cl.nval = (int)val.size();
    cl.pat_bytes = cl.val_bytes = 0;
    for (const TailCopy& c : pat) cl.pat_bytes += c.bytes;
    for (const TailCopy& c : val) cl.val_bytes += c.bytes;
    cl.xsrc = v[0].xa;
    cl.xoff = v[0].o_xa;
    cl.xbytes = (unsigned)a16(sizeof(T) * (size_t)v[0].n);
    pat.insert(pat.end(), val.begin(), val.end());
    TailCopy* dl = alloc<TailCopy>(pat.size());
    DR_CK(cudaMemcpy(dl, pat.data(), pat.size() * sizeof(TailCopy), cudaMemcpyHostToDevice));
    cl.list = dl;
    allow_tail_smem<T>();
    TailLevel<T>* dst = alloc<TailLevel<T>>(cnt);
    DR_CK(cudaMemcpy(dst, v.data(), cnt * sizeof(TailLevel<T>), cudaMemcpyHostToDevice));
    return (void*)dst;
  };
  tail64_ = make(double());
  if (fp32_) tail32_ = make(float());
}

// Levels that run the correction and the first post-smoothing step as one
// pass over Q = P - ω·D⁻¹·(A P) (EpCorrectJacobi): below the finest level
// and above the shared-memory tail, Jacobi-type smoothing, A's rows summed
// in a tree (not the reference's column order, so no bit-exact level loses
// it), and A·P no larger than A and P together.  A·P's values come from the
// Galerkin product on the device (refreshed by every partial resetup); a
// batch's A·P is the systems' patterns merged block-diagonally.
void DevHier::build_fused(const HostHierarchy& H) {
  const int nl = nlevels();
  for (int l = 1; l < std::min(nl, tail_); ++l) {
    DevLevel& d = L_[l];
    const HostLevel& h = H.levels[l];
    if (d.AP.n == 0 || !jacobi_type(d.smoother) || d.A.form.ordered) continue;
    if (d.AP.nnz > d.A.nnz + d.P.nnz) continue;
    // each P entry's position in AP's row (both rows sorted; P's pattern is
    // inside AP's when A's diagonal is stored)
    std::vector<int> pos(h.P.ci.size());
    bool ok = true;
    for (int i = 0; i < h.A.n && ok; ++i) {
      int k = h.ap_rp[i];
      const int ke = h.ap_rp[i + 1];
      for (int t = h.P.rp[i]; t < h.P.rp[i + 1]; ++t) {
        while (k < ke && h.ap_ci[k] < h.P.ci[t]) ++k;
        if (k == ke || h.ap_ci[k] != h.P.ci[t]) {
          ok = false;
          break;
        }
        pos[t] = k;
      }
    }
    if (!ok) continue;
    d.pq_pos = alloc<int>(pos.size());
    DR_CK(cudaMemcpy(d.pq_pos, pos.data(), pos.size() * sizeof(int), cudaMemcpyHostToDevice));
    d.q = alloc<double>(d.AP.nnz + 4);
    spgemm<double>(d.AP, d.A, d.P, d.AP.v, d.A.v, d.P.v, nullptr);
    d.fuse_up = true;
    build_q(d);
  }
}

void DevHier::build_q(DevLevel& d) {
  counted();
  k_build_q<<<grid1d(32LL * d.A.n, max_grid_), kBlock, 0, st_>>>(d.A.n, d.AP.rp, d.AP.v, d.invd, d.omega,
                                                                 d.P.rp, d.P.v, d.pq_pos, d.q);
  DR_CK(cudaGetLastError());
  if (fp32_) {
    if (!d.q32) d.q32 = alloc<float>(d.AP.nnz + 4);
    counted();
    k_convert<double, float><<<grid1d(d.AP.nnz, max_grid_), kBlock, 0, st_>>>(d.AP.nnz, d.q, d.q32);
    DR_CK(cudaGetLastError());
  }
}

void DevHier::build_cinv() {
  if (!cinv_) cinv_ = alloc<double>((size_t)nc_ * nc_);
  counted();
  k_lu_inverse<<<1, kern::kInvMax, 0, st_>>>(nc_, clu_, cpiv_, cinv_);
  DR_CK(cudaGetLastError());
}

void DevHier::refresh_fp32() {
  if (!fp32_) return;
  for (auto& d : L_) {
    counted();
    k_convert<double, float><<<grid1d(d.A.nnz, max_grid_), kBlock, 0, st_>>>(d.A.nnz, d.A.v, d.A.v32);
    counted();
    k_convert<double, float><<<grid1d(d.P.nnz, max_grid_), kBlock, 0, st_>>>(d.P.nnz, d.P.v, d.P.v32);
    counted();
    k_convert<double, float><<<grid1d(d.R.nnz, max_grid_), kBlock, 0, st_>>>(d.R.nnz, d.R.v, d.R.v32);
    counted();
    k_convert<double, float><<<grid1d(d.nv, max_grid_), kBlock, 0, st_>>>(d.nv, d.invd, d.invd32);
    if (d.spai1_M32) {
      counted();
      k_convert<double, float><<<grid1d(d.A.nnz, max_grid_), kBlock, 0, st_>>>(d.A.nnz, d.spai1_M, d.spai1_M32);
    }
    if (d.ilu_L32) {
      counted();
      k_convert<double, float><<<grid1d(d.A.nnz, max_grid_), kBlock, 0, st_>>>(d.A.nnz, d.ilu_L, d.ilu_L32);
      counted();
      k_convert<double, float><<<grid1d(d.A.nnz, max_grid_), kBlock, 0, st_>>>(d.A.nnz, d.ilu_U, d.ilu_U32);
    }
    if (d.fuse_up && d.q32) {
      counted();
      k_convert<double, float><<<grid1d(d.AP.nnz, max_grid_), kBlock, 0, st_>>>(d.AP.nnz, d.q, d.q32);
    }
    if (d.At.v32) {  // transposed copies (FP32 transposed cycles)
      counted();
      k_convert<double, float><<<grid1d(d.At.nnz, max_grid_), kBlock, 0, st_>>>(d.At.nnz, d.At.v, d.At.v32);
      counted();
      k_convert<double, float><<<grid1d(d.A.n, max_grid_), kBlock, 0, st_>>>(d.A.n, d.invdT, d.invdT32);
    }
  }
  DR_CK(cudaGetLastError());
}

// ------------------------------------------------------------ cycle pieces
template <typename T>
T* DevHier::smooth(int l, T* x, const T* b, int steps, T* ext, const double* rz_w, bool rz_first) {
  DevLevel& L = L_[l];
  LevelVecs<T>& V = vecs<T>(l);
  const DevMat& A = tr_ ? L.At : L.A;
  const T om = (T)L.omega;
  if (jacobi_type(L.smoother)) {
    for (int s = 0; s < steps; ++s) {
      T* dst = (l == 0) ? (x == V.xb ? ext : V.xb) : (x == V.xa ? V.xb : V.xa);
      if (rz_w && s == steps - 1) {
        EpJacobi<T> ep{x, b, invd<T>(L), dst, om, rz_w};
        if (rz_first)
          launch_rows_dot(st_, max_grid_, A, mval<T>(A), XPlain<T>{x}, ep, partials_,
                          tickets_ + TK_RZ, FinStore2{scal_ + SC_RZ, scal_ + SC_RZOLD});
        else
          launch_rows_dot(st_, max_grid_, A, mval<T>(A), XPlain<T>{x}, ep, partials_,
                          tickets_ + TK_RZ, FinShift{scal_ + SC_RZ, scal_ + SC_RZOLD});
      } else {
        launch_rows(st_, max_grid_, A, mval<T>(A), XPlain<T>{x},
                    EpJacobi<T>{x, b, invd<T>(L), dst, om, nullptr});
      }
      x = dst;
    }
  } else if (L.spai1_M) {
    // SPAI(1): r = b - A x, then x += M r, in place
    const T* Mv = std::is_same<T, float>::value ? (const T*)L.spai1_M32 : (const T*)L.spai1_M;
    for (int s = 0; s < steps; ++s) {
      launch_rows(st_, max_grid_, A, mval<T>(A), XPlain<T>{x}, EpResidualSub<T>{b, V.d});
      launch_rows(st_, max_grid_, A, Mv, XPlain<T>{V.d}, EpAddSum<T>{x});
    }
  } else if (L.sgs_order) {
    // serial (l1) Gauss-Seidel: the in-place sweep in row order, level by
    // level of its dependencies
    for (int s = 0; s < steps; ++s)
      for (size_t v = 0; v + 1 < L.sgs_off.size(); ++v) {
        const int off = L.sgs_off[v], cnt = L.sgs_off[v + 1] - off;
        counted();
        k_sgs_level<T><<<grid1d(cnt, max_grid_), kBlock, 0, st_>>>(cnt, L.sgs_order + off, A.rp, A.ci, mval<T>(A),
                                                                  b, invd<T>(L), x);
      }
    DR_CK(cudaGetLastError());
  } else if (L.ilu_L) {
    // ILU(0): dx = (LU)^-1 (b - A x) by the two level schedules, x += dx
    // (in place)
    T* t = V.d;
    const T* Lv = std::is_same<T, float>::value ? (const T*)L.ilu_L32 : (const T*)L.ilu_L;
    const T* Uv = std::is_same<T, float>::value ? (const T*)L.ilu_U32 : (const T*)L.ilu_U;
    for (int s = 0; s < steps; ++s) {
      residual<T>(l, x, b, t, nullptr);
      for (size_t v = 0; v + 1 < L.ilu_fwd_off.size(); ++v) {
        const int off = L.ilu_fwd_off[v], cnt = L.ilu_fwd_off[v + 1] - off;
        counted();
        k_ilu_fwd<T><<<grid1d(cnt, max_grid_), kBlock, 0, st_>>>(cnt, L.ilu_fwd + off, A.rp, A.ci, L.ilu_diag,
                                                                Lv, t);
      }
      for (size_t v = 0; v + 1 < L.ilu_bwd_off.size(); ++v) {
        const int off = L.ilu_bwd_off[v], cnt = L.ilu_bwd_off[v + 1] - off;
        counted();
        k_ilu_bwd<T><<<grid1d(cnt, max_grid_), kBlock, 0, st_>>>(cnt, L.ilu_bwd + off, A.rp, A.ci, L.ilu_diag,
                                                                Uv, t);
      }
      counted();
      k_ilu_apply<T><<<grid1d(A.n, max_grid_), kBlock, 0, st_>>>(A.n, t, x);
      DR_CK(cudaGetLastError());
    }
  } else if (L.smoother == SmootherKind::Chebyshev) {
    // each application: `cheb_degree` fused residual-and-update steps, the
    // iterate ping-ponging between two buffers as in the Jacobi sweeps
    for (int s = 0; s < steps; ++s)
      for (int j = 0; j < L.cheb_degree; ++j) {
        T* dst = (l == 0) ? (x == V.xb ? ext : V.xb) : (x == V.xa ? V.xb : V.xa);
        launch_rows(st_, max_grid_, A, mval<T>(A), XPlain<T>{x},
                    EpCheby<T>{x, b, invd<T>(L), V.d, dst, L.cheb_coef, j});
        x = dst;
      }
  } else {
    for (int s = 0; s < steps; ++s)
      for (int c = 0; c < L.ncolors; ++c) {
        const int off = L.color_off[c];
        const int cnt = L.color_off[c + 1] - off;
        if (cnt == 0) continue;
        const int grid = (int)std::max<long long>(1, std::min<long long>(((long long)cnt * A.Ggs + kBlock - 1) / kBlock, max_grid_));
        counted();
        switch (A.Ggs) {
#define DR_CASE(g)                                                                                  \
  case g:                                                                                           \
    k_gs_color<g, T><<<grid, kBlock, 0, st_>>>(cnt, L.color_order + off, A.rp, A.ci, mval<T>(A), b, \
                                               invd<T>(L), x);                                      \
    break;
          DR_CASE(1) DR_CASE(2) DR_CASE(4) DR_CASE(8) DR_CASE(16) DR_CASE(32)
#undef DR_CASE
        }
        DR_CK(cudaGetLastError());
      }
  }
  return x;
}

template <typename T>
void DevHier::residual(int l, const T* x, const T* b, T* r, double* rr_dst) {
  const DevMat& A = l < nlevels() ? (tr_ ? L_[l].At : L_[l].A) : C_;
  if (rr_dst)
    launch_rows_dot(st_, max_grid_, A, mval<T>(A), XPlain<T>{x}, EpResidual<T>{b, r}, partials_,
                    tickets_ + TK_RES, FinStore{rr_dst});
  else
    launch_rows(st_, max_grid_, A, mval<T>(A), XPlain<T>{x}, EpResidual<T>{b, r});
}

template <typename T>
void DevHier::coarse_solve(const T* b, T* x) {
  int threads = 32;
  while (threads < nc_ && threads < 1024) threads *= 2;
  // stage the factors in shared memory when they fit in 40 KB (n_c <= 70)
  const size_t ybytes = (size_t)((std::max(nc_, 1) + 1) & ~1) * sizeof(double);
  const size_t lbytes = (size_t)nc_ * nc_ * sizeof(double);
  const int staged = (ybytes + lbytes) <= 40 * 1024 ? 1 : 0;
  counted();
  if (tr_) {  // A_c^T y = b with the factors of A_c (adjoint solves)
    k_lu_solve_t<T><<<1, 32, ybytes, st_>>>(nc_, clu_, cpiv_, b, x);
    DR_CK(cudaGetLastError());
    return;
  }
  k_lu_solve<T><<<1, threads, ybytes + (staged ? lbytes : 0), st_>>>(nc_, clu_, cpiv_, b, x, staged);
  DR_CK(cudaGetLastError());
}

bool DevHier::fused_rz_ok(const CycleOpts& o) const {
  return !L_.empty() && o.post >= 1 &&
         jacobi_type(L_[0].smoother);
}

template <typename T>
T* DevHier::cycle_level(int l, T* x, const T* b, bool x_zero, const CycleOpts& o, T* ext,
                        const double* rz_w, bool rz_first, bool x1_ready) {
  if (!tr_ && l >= 1 && l == tail_ && x == vecs<T>(l).xa) {
    const void* desc = sizeof(T) == 8 ? tail64_ : tail32_;
    const int slot = sizeof(T) == 8 ? 0 : 1;
    TailCoarse<T> C{nc_, clu_, cpiv_, coarse_b<T>(), coarse_x<T>(), tail_co_[slot][0], tail_co_[slot][1],
                    tail_co_[slot][2], tail_co_[slot][3], tail_inv_ ? 1 : 0};
    counted();
    const TailCopyList& cl = tail_cp_[slot];
    const TailCopies cp{static_cast<const TailCopy*>(cl.list), cl.npat, cl.nval, cl.pat_bytes,
                        cl.val_bytes, TailCopy{cl.xsrc, cl.xoff, cl.xbytes}};
    launch_dependent(k_coarse_tail<T>, 1, kern::kTailThreads, tail_bytes_[slot], st_,
                     static_cast<const TailLevel<T>*>(desc), nlevels() - l, C, cp, o.pre, o.post,
                     o.w ? 1 : 0, x_zero ? 1 : 0, err_flag());
    DR_CK(cudaGetLastError());
    return x;
  }
  DevLevel& L = L_[l];
  LevelVecs<T>& V = vecs<T>(l);
  const DevMat& A = tr_ ? L.At : L.A;
  const T om = (T)L.omega;
  const bool jac = jacobi_type(L.smoother);
  bool have_r = false;
  // pre-smoothing
  if (x_zero && jac && o.pre >= 1) {
    if (o.pre == 1 && x1_ready) {
      // x already holds the zero-guess Jacobi step (written by the restriction)
      residual<T>(l, x, b, V.r, nullptr);
      have_r = true;
    } else if (o.pre == 1) {
      launch_rows(st_, max_grid_, A, mval<T>(A), XZeroJacobi<T>{b, invd<T>(L), om},
                  EpZeroJacobiResidual<T>{b, invd<T>(L), x, V.r, om});
      have_r = true;
    } else {
      counted();
      k_scale_jacobi_zero<T><<<grid1d(A.n, max_grid_), kBlock, 0, st_>>>(A.n, b, invd<T>(L), om, x);
      DR_CK(cudaGetLastError());
      x = smooth<T>(l, x, b, o.pre - 1, ext);
    }
  } else {
    if (x_zero) {
      counted();
      k_fill<T><<<grid1d(A.n, max_grid_), kBlock, 0, st_>>>(A.n, T(0), x);
      DR_CK(cudaGetLastError());
    }
    x = smooth<T>(l, x, b, o.pre, ext);
  }
  if (!have_r) residual<T>(l, x, b, V.r, nullptr);
  // restriction  b_{l+1} = Pᵀ r
  const bool last = (l + 1 == nlevels());
  T* bn = last ? coarse_b<T>() : vecs<T>(l + 1).b;
  bool x1n = false;
  if (!last && l + 1 != tail_ && o.pre == 1 &&
      jacobi_type(L_[l + 1].smoother)) {
    // the coarse level starts from zero with one Jacobi step: form it here
    DevLevel& Ln = L_[l + 1];
    launch_rows(st_, max_grid_, L.R, mval<T>(L.R), XPlain<T>{V.r},
                EpStoreZeroJacobi<T>{bn, invd<T>(Ln), vecs<T>(l + 1).xa, (T)Ln.omega});
    x1n = true;
  } else {
    launch_rows(st_, max_grid_, L.R, mval<T>(L.R), XPlain<T>{V.r}, EpStore<T>{bn});
  }
  // coarse-grid correction
  T* xn;
  if (!last) {
    xn = vecs<T>(l + 1).xa;
    xn = cycle_level<T>(l + 1, xn, bn, true, o, nullptr, nullptr, false, x1n);
    if (o.w) xn = cycle_level<T>(l + 1, xn, bn, false, o, nullptr);
    if (batch_) batch_coarse<T>(l + 1, bn, xn);  // the systems whose coarsest level is l + 1
  } else {
    xn = coarse_x<T>();
    if (batch_) batch_coarse<T>(l + 1, bn, xn);
    else coarse_solve<T>(bn, xn);
  }
  if (L.fuse_up && !tr_ && o.post >= 1 && !rz_w) {
    // correction and the first post-smoothing step in one pass over Q
    // (EpCorrectJacobi; V.r holds b - A x from the way down)
    launch_rows(st_, max_grid_, L.AP, qval<T>(L), XPlain<T>{xn},
                EpCorrectJacobi<T>{x, V.r, invd<T>(L), om});
    x = smooth<T>(l, x, b, o.post - 1, ext, rz_w, rz_first);
    return x;
  }
  // prolongation and correction  x += P xc
  launch_rows(st_, max_grid_, L.P, mval<T>(L.P), XPlain<T>{xn}, EpAddTo<T>{x});
  // post-smoothing
  x = smooth<T>(l, x, b, o.post, ext, rz_w, rz_first);
  return x;
}

void DevHier::cycle(double* x, const double* b, const CycleOpts& o) {
  if (L_.empty()) {
    coarse_solve<double>(b, x);
    return;
  }
  double* xo = cycle_level<double>(0, x, b, false, o, x);
  if (xo != x) DR_CK(cudaMemcpyAsync(x, xo, (size_t)n0_ * sizeof(double), cudaMemcpyDeviceToDevice, st_));
}

double DevHier::dot_host(const double* a, const double* b, int n) {
  counted();
  k_dot<double, double, FinStore><<<grid1d(n, max_grid_), kBlock, 0, st_>>>(n, a, b, partials_, tickets_ + TK_DOT,
                                                                           FinStore{scal_ + SC_TMP});
  DR_CK(cudaGetLastError());
  DR_CK(cudaMemcpyAsync(hscal_ + SC_TMP, scal_ + SC_TMP, sizeof(double), cudaMemcpyDeviceToHost, st_));
  DR_CK(cudaStreamSynchronize(st_));
  return hscal_[SC_TMP];
}

int DevHier::solve(double* x, const double* b, const CycleOpts& o, double tol, int maxiter, int verbose,
                   double* relres) {
  const auto t_solve = std::chrono::steady_clock::now();
  auto secs = [&]() { return std::chrono::duration<double>(std::chrono::steady_clock::now() - t_solve).count(); };
  const double bnorm = std::sqrt(dot_host(b, b, n0_));
  if (bnorm == 0.0) {
    counted();
    k_fill<double><<<grid1d(n0_, max_grid_), kBlock, 0, st_>>>(n0_, 0.0, x);
    DR_CK(cudaStreamSynchronize(st_));
    if (relres) *relres = 0.0;
    return 0;
  }
  if (L_.empty()) {
    coarse_solve<double>(b, x);
    DR_CK(cudaStreamSynchronize(st_));
    if (relres) *relres = NAN;
    return 1;
  }
  double* r = L_[0].v64.r;
  double rel = 1.0;
  for (int it = 1; it <= maxiter; ++it) {
    cycle(x, b, o);
    residual<double>(0, x, b, r, scal_ + SC_RR);
    DR_CK(cudaMemcpyAsync(hscal_ + SC_RR, scal_ + SC_RR, sizeof(double), cudaMemcpyDeviceToHost, st_));
    DR_CK(cudaStreamSynchronize(st_));
    const double rnorm = std::sqrt(hscal_[SC_RR]);
    rel = rnorm / bnorm;
    if (verbose >= 2) std::printf("  AMG iter %4d: residual norm = %.6e, relative = %.6e\n", it, rnorm, rel);
    if (rel < tol || it == maxiter) check_kernel_flag(st_);
    if (rel < tol) {
      if (verbose >= 1)
        std::printf("AMG solve converged: %d iterations, %.4f s, final residual %.2e\n", it, secs(), rel);
      if (relres) *relres = rel;
      return it;
    }
  }
  if (verbose >= 1)
    std::printf("AMG solve did NOT converge: %d iterations, %.4f s, final residual %.2e\n", maxiter, secs(), rel);
  if (relres) *relres = rel;
  return maxiter;
}

// ------------------------------------------------------------ transposed hierarchy
// A^T of every level (pattern transposed on the host once, values gathered
// from A's whenever those change) with the smoother diagonal of A^T, for
// cycles on A^T: the same P and R, coarse operators P^T A^T P = (P^T A P)^T,
// the coarsest solve with the transposed LU factors.  Jacobi-type smoothers.
void DevHier::build_transpose() {
  if (at_built_) return;
  for (auto& d : L_)
    if (!jacobi_type(d.smoother))
      fail("transposed cycles need Jacobi, l1-Jacobi or SPAI(0) smoothing on every level");
  DR_CK(cudaStreamSynchronize(st_));
  std::vector<std::vector<int>> keep_rp, keep_ci;  // alive until the uploads finish
  for (auto& d : L_) {
    const int n = d.A.n;
    std::vector<int> rp(n + 1), ci(d.A.nnz);
    DR_CK(cudaMemcpy(rp.data(), d.A.rp, rp.size() * sizeof(int), cudaMemcpyDeviceToHost));
    if (!ci.empty()) DR_CK(cudaMemcpy(ci.data(), d.A.ci, ci.size() * sizeof(int), cudaMemcpyDeviceToHost));
    std::vector<int> trp(n + 1, 0), tci(ci.size()), perm(ci.size());
    for (int k = 0; k < (int)ci.size(); ++k) ++trp[ci[k] + 1];
    for (int j = 0; j < n; ++j) trp[j + 1] += trp[j];
    std::vector<int> fill(trp.begin(), trp.end() - 1);
    for (int i = 0; i < n; ++i)  // rows in order: each transposed row's columns ascend
      for (int k = rp[i]; k < rp[i + 1]; ++k) {
        const int q = fill[ci[k]]++;
        tci[q] = i;
        perm[q] = k;
      }
    upload_csr(d.At, n, n, trp, tci, nullptr);
    d.at_perm = alloc<int>(perm.size());
    h2d(d.at_perm, perm, st_);
    d.invdT = alloc<double>(n);
    keep_rp.push_back(std::move(trp));
    keep_ci.push_back(std::move(tci));
    keep_ci.push_back(std::move(perm));
  }
  DR_CK(cudaStreamSynchronize(st_));
  at_built_ = true;
  refresh_transpose();
  if (fp32_) {
    alloc_transpose_fp32();
    refresh_fp32();
  }
  DR_CK(cudaStreamSynchronize(st_));
}

void DevHier::refresh_transpose() {
  for (auto& d : L_) {
    if (d.A.nnz > 0) {
      counted();
      k_gather_vals<<<grid1d(d.A.nnz, max_grid_), kBlock, 0, st_>>>(d.A.nnz, d.at_perm, d.A.v, d.At.v);
    }
    counted();
    if (d.smoother == SmootherKind::L1Jacobi)
      k_l1_invdiag<<<grid1d(d.A.n, max_grid_), kBlock, 0, st_>>>(d.A.n, d.At.rp, d.At.v, d.invdT);
    else if (d.smoother == SmootherKind::SPAI0)
      k_spai0_diag<<<grid1d(d.A.n, max_grid_), kBlock, 0, st_>>>(d.A.n, d.At.rp, d.At.ci, d.At.v, d.invdT);
    else
      k_invdiag<<<grid1d(d.A.n, max_grid_), kBlock, 0, st_>>>(d.A.n, d.At.rp, d.At.ci, d.At.v, d.invdT);
  }
  DR_CK(cudaGetLastError());
}

void DevHier::lin3(int n, double a, const double* x, double b, const double* y, double c, const double* z,
                   double* out) {
  counted();
  k_lin3<<<grid1d(n, max_grid_), kBlock, 0, st_>>>(n, a, x, b, y, c, z, out);
  DR_CK(cudaGetLastError());
}

// z = M r: one cycle from a zero iterate (FP64), result copied to `out`.
void DevHier::precond64(const double* r, double* out, const CycleOpts& o) {
  if (L_.empty()) {
    coarse_solve<double>(r, out);
    return;
  }
  const double* z = cycle_level<double>(0, out, r, true, o, out);
  if (z != out) DR_CK(cudaMemcpyAsync(out, z, (size_t)n0_ * sizeof(double), cudaMemcpyDeviceToDevice, st_));
}

// Right-preconditioned BiCGStab (FP64) on A or, with `transpose`, on A^T
// with cycles on the transposed hierarchy: x is the initial guess and the
// solution (device memory).  Returns the iterations; relres = |b - A x|/|b|.
int DevHier::bicgstab(double* x, const double* b, const CycleOpts& o, double tol, int maxiter,
                      bool transpose, double* relres, int verbose, bool mixed) {
  if (transpose) build_transpose();
  if (mixed) ensure_fp32();
  struct Mode {
    bool& f;
    bool old;
    ~Mode() { f = old; }
  } mode{tr_, tr_};
  tr_ = transpose;
  graphs_clear();
  const int n = n0_;
  if (!bk_[0])
    for (auto& p : bk_) p = alloc<double>(n);
  double *r = bk_[0], *rh = bk_[1], *p = bk_[2], *v = bk_[3], *sv = bk_[4], *t = bk_[5], *ph = bk_[6],
         *sh = bk_[7];
  auto spmv = [&](const double* in, double* out) {
    const DevMat& A = L_.empty() ? C_ : (tr_ ? L_[0].At : L_[0].A);
    launch_rows(st_, max_grid_, A, A.v, XPlain<double>{in}, EpStore<double>{out});
  };
  const double bnorm = std::sqrt(dot_host(b, b, n));
  if (bnorm == 0.0) {
    counted();
    k_fill<double><<<grid1d(n, max_grid_), kBlock, 0, st_>>>(n, 0.0, x);
    DR_CK(cudaStreamSynchronize(st_));
    if (relres) *relres = 0.0;
    return 0;
  }
  spmv(x, t);
  lin3(n, 1.0, b, -1.0, t, 0.0, nullptr, r);  // r = b - A x
  DR_CK(cudaMemcpyAsync(rh, r, (size_t)n * sizeof(double), cudaMemcpyDeviceToDevice, st_));
  double rel = std::sqrt(dot_host(r, r, n)) / bnorm;
  double rho = 1.0, alpha = 1.0, omega = 1.0;
  counted();
  k_fill<double><<<grid1d(n, max_grid_), kBlock, 0, st_>>>(n, 0.0, p);
  counted();
  k_fill<double><<<grid1d(n, max_grid_), kBlock, 0, st_>>>(n, 0.0, v);
  int it = 0;
  while (rel >= tol && it < maxiter) {
    ++it;
    const double rho1 = dot_host(rh, r, n);
    if (rho1 == 0.0) break;  // breakdown: r orthogonal to the shadow residual
    const double beta = (rho1 / rho) * (alpha / omega);
    lin3(n, 1.0, r, beta, p, -beta * omega, v, p);  // p = r + beta (p - omega v)
    if (mixed) precond32(p, ph, o);
    else precond64(p, ph, o);
    spmv(ph, v);
    alpha = rho1 / dot_host(rh, v, n);
    lin3(n, 1.0, r, -alpha, v, 0.0, nullptr, sv);  // s = r - alpha v
    const double snorm = std::sqrt(dot_host(sv, sv, n));
    if (snorm / bnorm < tol) {
      lin3(n, 1.0, x, alpha, ph, 0.0, nullptr, x);
      DR_CK(cudaMemcpyAsync(r, sv, (size_t)n * sizeof(double), cudaMemcpyDeviceToDevice, st_));
      rel = snorm / bnorm;
      break;
    }
    if (mixed) precond32(sv, sh, o);
    else precond64(sv, sh, o);
    spmv(sh, t);
    const double tt = dot_host(t, t, n);
    omega = tt > 0.0 ? dot_host(t, sv, n) / tt : 0.0;
    lin3(n, 1.0, x, alpha, ph, omega, sh, x);      // x += alpha p^ + omega s^
    lin3(n, 1.0, sv, -omega, t, 0.0, nullptr, r);  // r = s - omega t
    rel = std::sqrt(dot_host(r, r, n)) / bnorm;
    rho = rho1;
    if (verbose >= 2) std::printf("  BiCGStab iter %4d: relative residual %.6e\n", it, rel);
    if (omega == 0.0) break;
  }
  // true residual of the result
  spmv(x, t);
  lin3(n, 1.0, b, -1.0, t, 0.0, nullptr, r);
  rel = std::sqrt(dot_host(r, r, n)) / bnorm;
  check_kernel_flag(st_);
  if (relres) *relres = rel;
  return it;
}

// One FP32 AMG cycle from a zero guess on an FP64 right-hand side, the
// result returned in FP64 (the preconditioner of the mixed FGMRES).
void DevHier::precond32(const double* r, double* out, const CycleOpts& o) {
  ensure_fp32();
  const int n = n0_;
  if (!pr32_) {
    pr32_ = alloc<float>(n);
    pz32_ = alloc<float>(n);
  }
  counted();
  k_convert<double, float><<<grid1d(n, max_grid_), kBlock, 0, st_>>>(n, r, pr32_);
  const float* z = pz32_;
  if (L_.empty()) coarse_solve<float>(pr32_, pz32_);
  else z = cycle_level<float>(0, pz32_, pr32_, true, o, pz32_);
  counted();
  k_convert<float, double><<<grid1d(n, max_grid_), kBlock, 0, st_>>>(n, z, out);
  DR_CK(cudaGetLastError());
}

// Flexible GMRES(m) with right preconditioning (Saad's FGMRES): the
// preconditioned vectors z_j are kept, since the preconditioner (an FP32
// cycle rounds differently for every input) need not be a fixed linear map.
// Arnoldi in FP64 with classical Gram-Schmidt applied twice: h = Vᵀw and
// w -= V h by k_mdot / k_maxpy (deterministic reductions), then ||w||; the
// Hessenberg column, its Givens rotations and the least-squares update stay
// on the host (one device-to-host copy per iteration).  Restarts from the
// true residual; stops when the rotated residual estimate, and then the true
// residual, is below tol·||b||.
int DevHier::fgmres(double* x, const double* b, const CycleOpts& o, double tol, int maxiter, int restart,
                    bool mixed, double* relres, int verbose) {
  const int n = n0_;
  const int m = std::max(1, std::min(restart, 63));
  graphs_clear();
  const int gx = grid1d(n, max_grid_);
  if (gm_m_ < m) {
    // reallocation at a larger restart length (the old arrays stay with the
    // hierarchy until it is freed)
    gm_V_ = alloc<double>((size_t)(m + 1) * n);
    gm_Z_ = alloc<double>((size_t)m * n);
    gm_w_ = alloc<double>(n);
    gm_h_ = alloc<double>(2 * 64 + 2);
    gm_part_ = alloc<double>((size_t)65 * max_grid_);
    gm_tk_ = alloc<unsigned>(65);
    DR_CK(cudaMemsetAsync(gm_tk_, 0, 65 * sizeof(unsigned), st_));
    gm_m_ = m;
  }
  double *V = gm_V_, *Z = gm_Z_, *w = gm_w_;
  const DevMat& A = L_.empty() ? C_ : L_[0].A;
  auto spmv = [&](const double* in, double* out) {
    launch_rows(st_, max_grid_, A, A.v, XPlain<double>{in}, EpStore<double>{out});
  };
  auto mdot = [&](int k, const double* vw, double* h) {
    counted();
    k_mdot<<<dim3(gx, k), kBlock, 0, st_>>>(n, V, (long long)n, vw, gm_part_, gm_tk_, h);
  };
  auto maxpy = [&](int k, const double* Mv, const double* h, double sign, double* out) {
    counted();
    k_maxpy<<<gx, kBlock, 0, st_>>>(n, k, Mv, (long long)n, h, sign, out);
  };
  const double bnorm = std::sqrt(dot_host(b, b, n));
  if (bnorm == 0.0) {
    counted();
    k_fill<double><<<gx, kBlock, 0, st_>>>(n, 0.0, x);
    DR_CK(cudaStreamSynchronize(st_));
    if (relres) *relres = 0.0;
    return 0;
  }
  std::vector<double> H((size_t)(m + 1) * m), cs(m), sn(m), g(m + 1), y(m), hh(2 * 64 + 2);
  int it = 0;
  double rel = 1.0;
  while (true) {
    spmv(x, w);
    lin3(n, 1.0, b, -1.0, w, 0.0, nullptr, w);  // w = b - A x
    const double beta = std::sqrt(dot_host(w, w, n));
    rel = beta / bnorm;
    if (verbose >= 2) std::printf("  FGMRES restart at iter %4d: relative residual %.6e\n", it, rel);
    if (rel < tol || it >= maxiter) break;
    lin3(n, 1.0 / beta, w, 0.0, w, 0.0, nullptr, V);  // V_0 = w / beta
    std::fill(g.begin(), g.end(), 0.0);
    g[0] = beta;
    int jn = 0;  // columns in this cycle
    for (int j = 0; j < m && it < maxiter; ++j) {
      ++it;
      double* vj = V + (size_t)j * n;
      double* zj = Z + (size_t)j * n;
      if (mixed) precond32(vj, zj, o);
      else precond64(vj, zj, o);
      spmv(zj, w);
      // classical Gram-Schmidt, twice
      mdot(j + 1, w, gm_h_);
      maxpy(j + 1, V, gm_h_, -1.0, w);
      mdot(j + 1, w, gm_h_ + 64);
      maxpy(j + 1, V, gm_h_ + 64, -1.0, w);
      counted();
      k_dot<double, double, FinStore><<<gx, kBlock, 0, st_>>>(n, w, w, partials_, tickets_ + TK_DOT,
                                                             FinStore{gm_h_ + 128});
      DR_CK(cudaGetLastError());
      DR_CK(cudaMemcpyAsync(hh.data(), gm_h_, hh.size() * sizeof(double), cudaMemcpyDeviceToHost, st_));
      DR_CK(cudaStreamSynchronize(st_));
      const double hn = std::sqrt(hh[128]);
      double* col = &H[(size_t)j * (m + 1)];
      for (int i = 0; i <= j; ++i) col[i] = hh[i] + hh[64 + i];
      col[j + 1] = hn;
      if (hn > 0.0) lin3(n, 1.0 / hn, w, 0.0, w, 0.0, nullptr, V + (size_t)(j + 1) * n);
      // previous rotations, then a new one zeroing col[j+1]
      for (int i = 0; i < j; ++i) {
        const double t = cs[i] * col[i] + sn[i] * col[i + 1];
        col[i + 1] = -sn[i] * col[i] + cs[i] * col[i + 1];
        col[i] = t;
      }
      const double den = std::hypot(col[j], col[j + 1]);
      cs[j] = den > 0.0 ? col[j] / den : 1.0;
      sn[j] = den > 0.0 ? col[j + 1] / den : 0.0;
      col[j] = den;
      col[j + 1] = 0.0;
      g[j + 1] = -sn[j] * g[j];
      g[j] = cs[j] * g[j];
      jn = j + 1;
      const double est = std::fabs(g[j + 1]) / bnorm;
      if (verbose >= 2) std::printf("  FGMRES iter %4d: estimated relative residual %.6e\n", it, est);
      if (est < tol || hn == 0.0) break;
    }
    // y = H⁻¹ g (upper triangular), x += Z y
    for (int i = jn - 1; i >= 0; --i) {
      double t = g[i];
      for (int k = i + 1; k < jn; ++k) t -= H[(size_t)k * (m + 1) + i] * y[k];
      const double d = H[(size_t)i * (m + 1) + i];
      y[i] = d != 0.0 ? t / d : 0.0;
    }
    DR_CK(cudaMemcpyAsync(gm_h_, y.data(), (size_t)jn * sizeof(double), cudaMemcpyHostToDevice, st_));
    maxpy(jn, Z, gm_h_, 1.0, x);
    DR_CK(cudaStreamSynchronize(st_));  // y leaves scope only after the copy
  }
  check_kernel_flag(st_);
  if (verbose >= 1)
    std::printf("FGMRES (%s cycle) %s: %d iterations, final residual %.2e\n", mixed ? "FP32" : "FP64",
                rel < tol ? "converged" : "did NOT converge", it, rel);
  if (relres) *relres = rel;
  return it;
}

int DevHier::refine(double* x, const double* b, const CycleOpts& o, double tol, int max_outer,
                    double inner_tol, int inner_maxiter, int inner, bool mixed, double* relres,
                    int* inner_total, int verbose) {
  const int n = n0_;
  if (!ir_r_) {
    ir_r_ = alloc<double>(n);
    ir_d_ = alloc<double>(n);
    ir_x_ = alloc<double>(n);
  }
  const DevMat& A = L_.empty() ? C_ : L_[0].A;
  const double bnorm = std::sqrt(dot_host(b, b, n));
  int total = 0, outer = 0;
  double rel = 0.0;
  if (bnorm == 0.0) {
    counted();
    k_fill<double><<<grid1d(n, max_grid_), kBlock, 0, st_>>>(n, 0.0, x);
    DR_CK(cudaStreamSynchronize(st_));
  } else {
    // the iterate lives in a buffer of its own: the inner PCG works in the
    // hierarchy's iterate buffer, which may be the caller's x (host entry)
    double* const xout = x;
    DR_CK(cudaMemcpyAsync(ir_x_, xout, (size_t)n * sizeof(double), cudaMemcpyDeviceToDevice, st_));
    x = ir_x_;
    while (true) {
      launch_rows(st_, max_grid_, A, A.v, XPlain<double>{x}, EpStore<double>{ir_r_});
      lin3(n, 1.0, b, -1.0, ir_r_, 0.0, nullptr, ir_r_);  // r = b - A x (FP64)
      rel = std::sqrt(dot_host(ir_r_, ir_r_, n)) / bnorm;
      if (verbose >= 2) std::printf("  refinement step %3d: relative residual %.6e\n", outer, rel);
      if (rel < tol || outer >= max_outer) break;
      ++outer;
      counted();
      k_fill<double><<<grid1d(n, max_grid_), kBlock, 0, st_>>>(n, 0.0, ir_d_);
      double rr = 0.0;
      const int its = inner == 1 ? fgmres(ir_d_, ir_r_, o, inner_tol, inner_maxiter, 30, mixed, &rr, 0)
                                 : pcg(ir_d_, ir_r_, o, inner_tol, inner_maxiter, mixed, &rr, 0);
      total += its;
      lin3(n, 1.0, x, 1.0, ir_d_, 0.0, nullptr, x);  // x += d
      if (its == 0) break;  // the inner solver made no progress
    }
    DR_CK(cudaMemcpyAsync(xout, ir_x_, (size_t)n * sizeof(double), cudaMemcpyDeviceToDevice, st_));
  }
  check_kernel_flag(st_);
  if (verbose >= 1)
    std::printf("iterative refinement (%s inner, %s cycle): %d steps, %d inner iterations, residual %.2e\n",
                inner == 1 ? "FGMRES" : "PCG", mixed ? "FP32" : "FP64", outer, total, rel);
  if (relres) *relres = rel;
  if (inner_total) *inner_total = total;
  return outer;
}

// ------------------------------------------------------------ batch
// The coarsest solves of the systems whose coarsest level is merged level l
// (rows at the end of that level's vectors), one block per system.
template <typename T>
void DevHier::batch_coarse(int l, const T* b, T* x) {
  if (l >= (int)batch_dev_.size()) return;
  const BatchDev& c = batch_dev_[l];
  if (c.nblk == 0) return;
  counted();
  const size_t wsm = (size_t)(c.maxn + (size_t)c.maxn * c.maxn) * sizeof(double);
  if (c.inv) {  // one block per system, x = A^-1 b
    k_inv_apply_batch<T><<<c.nblk, kern::kInvMax, 0, st_>>>(c.off, c.nb, c.luoff, binv_, b, x);
  } else if (wsm <= 48 * 1024) {  // one warp per system, its factors staged in shared memory
    k_lu_solve_batch_warp<T><<<c.nblk, 32, wsm, st_>>>(c.off, c.nb, c.luoff, c.poff, blu_, bpiv_, b, x, c.maxn);
  } else {
    int threads = 32;
    while (threads < c.maxn && threads < 256) threads *= 2;
    k_lu_solve_batch<T><<<c.nblk, threads, (size_t)std::max(c.maxn, 1) * sizeof(double), st_>>>(
        c.off, c.nb, c.luoff, c.poff, blu_, bpiv_, b, x);
  }
  DR_CK(cudaGetLastError());
}
template void DevHier::batch_coarse<double>(int, const double*, double*);
template void DevHier::batch_coarse<float>(int, const float*, float*);

// Conjugate gradients on every system of a batch at once.  Each iteration
// (one CUDA graph) runs every stage once for all systems: q = A p (one
// launch over the block-diagonal finest matrix), the per-system dot
// products (k_seg_dot_part / k_seg_dot_final, deterministic), the step
// sizes (k_seg_alpha), the updates (k_seg_update), the preconditioner (one
// cycle of the merged hierarchy: one launch per stage and level, the
// systems' coarsest solves one launch per level), r·z and the new
// directions (k_seg_beta, k_seg_dir).  A system stops changing once its
// relative residual is below tol (its step sizes become 0); the host reads
// the count of converged systems after every iteration.
int DevHier::pcg_batch_seg(double* x, const double* b, const CycleOpts& o, double tol, int maxiter, bool mixed,
                           int* iters, double* relres, int verbose) {
  if (!batch_) fail("not a batch of systems");
  const int n = n0_, ns = batch_->nsys;
  if (mixed) ensure_fp32();
  if (!sx_) {
    sx_ = alloc<double>(n);
    sr_ = alloc<double>(n);
    sp_ = alloc<double>(n);
    sq_ = alloc<double>(n);
    sz_ = alloc<double>(n);
    seg_buf_ = alloc<double>(7 * (size_t)ns);
    seg_int_ = alloc<int>(2 * (size_t)ns + 1);
  }
  if (mixed && !pr32_) {
    pr32_ = alloc<float>(n);
    pz32_ = alloc<float>(n);
  }
  int maxlen = 0;
  for (int q = 0; q < ns; ++q)
    maxlen = std::max(maxlen, (q + 1 < ns ? batch_->off[0][q + 1] : n) - batch_->off[0][q]);
  const int PB = std::max(1, std::min(64, (maxlen + kBlock * 4 - 1) / (kBlock * 4)));
  if (!seg_part_) seg_part_ = alloc<double>((size_t)ns * 64);
  double* buf = seg_buf_;
  SegScal sc{buf, buf + ns, buf + 2 * ns, buf + 3 * ns, buf + 4 * ns, buf + 5 * ns, buf + 6 * ns, seg_int_,
             seg_int_ + ns};
  int* ndone = seg_int_ + 2 * ns;
  const DevMat& A = L_[0].A;
  auto segdot = [&](const double* a, const void* bb, bool bf32, double* out) {
    counted();
    if (bf32)
      k_seg_dot_part<double, float><<<dim3(PB, ns), kBlock, 0, st_>>>(seg_off_, a, (const float*)bb, seg_part_);
    else
      k_seg_dot_part<double, double><<<dim3(PB, ns), kBlock, 0, st_>>>(seg_off_, a, (const double*)bb,
                                                                         seg_part_);
    counted();
    k_seg_dot_final<<<(ns + 7) / 8, 256, 0, st_>>>(ns, PB, seg_part_, out);
    DR_CK(cudaGetLastError());
  };
  const void* zptr = nullptr;
  auto precond = [&]() {
    if (mixed) zptr = cycle_level<float>(0, pz32_, pr32_, true, o, pz32_);
    else zptr = cycle_level<double>(0, sz_, sr_, true, o, sz_);
  };
  // r = b - A x, |b|^2, |r|^2
  DR_CK(cudaMemcpyAsync(sx_, x, (size_t)n * sizeof(double), cudaMemcpyDeviceToDevice, st_));
  launch_rows(st_, max_grid_, A, A.v, XPlain<double>{sx_}, EpResidual<double>{b, sr_});
  segdot(b, b, false, sc.bb);
  segdot(sr_, sr_, false, sc.rr);
  std::vector<double> hb(2 * (size_t)ns);
  DR_CK(cudaMemcpyAsync(hb.data(), sc.rr, 2 * (size_t)ns * sizeof(double), cudaMemcpyDeviceToHost, st_));
  DR_CK(cudaStreamSynchronize(st_));
  std::vector<int> hint(2 * (size_t)ns + 1, 0);
  for (int q = 0; q < ns; ++q) {
    const double rr = hb[q], bb = hb[ns + q];
    if (bb == 0.0 || rr < tol * tol * bb) {  // nothing to do (b = 0: x = 0)
      hint[q] = 1;
      hint[2 * ns] += 1;
    }
  }
  for (int q = 0; q < ns; ++q)
    if (hb[ns + q] == 0.0)
      DR_CK(cudaMemsetAsync(sx_ + batch_->off[0][q], 0,
                            (size_t)((q + 1 < ns ? batch_->off[0][q + 1] : n) - batch_->off[0][q]) * sizeof(double),
                            st_));
  DR_CK(cudaMemcpyAsync(seg_int_, hint.data(), hint.size() * sizeof(int), cudaMemcpyHostToDevice, st_));
  if (mixed) {
    counted();
    k_convert<double, float><<<grid1d(n, max_grid_), kBlock, 0, st_>>>(n, sr_, pr32_);
  }
  precond();
  segdot(sr_, zptr, mixed, sc.rz);
  DR_CK(cudaMemsetAsync(sp_, 0, (size_t)n * sizeof(double), st_));
  DR_CK(cudaMemsetAsync(sc.beta, 0, (size_t)ns * sizeof(double), st_));
  auto dir = [&]() {
    counted();
    if (mixed)
      k_seg_dir<float><<<grid1d(n, max_grid_), kBlock, 0, st_>>>(n, seg_id_, (const float*)zptr, sc.beta, sp_);
    else
      k_seg_dir<double><<<grid1d(n, max_grid_), kBlock, 0, st_>>>(n, seg_id_, (const double*)zptr, sc.beta, sp_);
    DR_CK(cudaGetLastError());
  };
  dir();  // p = z
  const int gs = (ns + 127) / 128;
  auto iteration = [&]() {
    launch_rows(st_, max_grid_, A, A.v, XPlain<double>{sp_}, EpStore<double>{sq_});
    segdot(sp_, sq_, false, sc.pq);
    counted();
    k_seg_alpha<<<gs, 128, 0, st_>>>(ns, sc);
    counted();
    if (mixed)
      k_seg_update<float><<<grid1d(n, max_grid_), kBlock, 0, st_>>>(n, seg_id_, sc.alpha, sp_, sq_, sx_, sr_, pr32_);
    else
      k_seg_update<float><<<grid1d(n, max_grid_), kBlock, 0, st_>>>(n, seg_id_, sc.alpha, sp_, sq_, sx_, sr_,
                                                                   (float*)nullptr);
    DR_CK(cudaGetLastError());
    segdot(sr_, sr_, false, sc.rr);
    precond();
    DR_CK(cudaMemcpyAsync(sc.rzold, sc.rz, (size_t)ns * sizeof(double), cudaMemcpyDeviceToDevice, st_));
    segdot(sr_, zptr, mixed, sc.rz);
    counted();
    k_seg_beta<<<gs, 128, 0, st_>>>(ns, sc, tol * tol, ndone);
    DR_CK(cudaGetLastError());
    dir();
  };
  // one iteration as a CUDA graph (recaptured when the options change)
  if (seg_graph_ && (seg_graph_mixed_ != mixed || seg_graph_o_.pre != o.pre || seg_graph_o_.post != o.post ||
                     seg_graph_o_.w != o.w)) {
    cudaGraphExecDestroy(seg_graph_);
    seg_graph_ = nullptr;
  }
  if (!seg_graph_) {
    cudaGraph_t g;
    const long long c0 = g_launches.load();
    DR_CK(cudaStreamBeginCapture(st_, cudaStreamCaptureModeThreadLocal));
    iteration();
    DR_CK(cudaStreamEndCapture(st_, &g));
    const long long per_iter = g_launches.load() - c0;
    g_launches.fetch_sub(per_iter);
    DR_CK(cudaGraphInstantiate(&seg_graph_, g, 0));
    DR_CK(cudaGraphDestroy(g));
    seg_graph_mixed_ = mixed;
    seg_graph_o_ = o;
    seg_launches_ = per_iter;
  }
  int* hdone = reinterpret_cast<int*>(hscal_ + SC_N - 1);
  int it = 0;
  int done = hint[2 * ns];
  while (done < ns && it < maxiter) {
    DR_CK(cudaGraphLaunch(seg_graph_, st_));
    g_launches.fetch_add(seg_launches_);
    ++it;
    DR_CK(cudaMemcpyAsync(hdone, ndone, sizeof(int), cudaMemcpyDeviceToHost, st_));
    DR_CK(cudaStreamSynchronize(st_));
    done = *hdone;
    if (verbose >= 2) std::printf("  batch PCG iter %4d: %d of %d systems converged\n", it, done, ns);
  }
  // true residuals
  launch_rows(st_, max_grid_, A, A.v, XPlain<double>{sx_}, EpResidual<double>{b, sr_});
  segdot(sr_, sr_, false, sc.rr);
  DR_CK(cudaMemcpyAsync(x, sx_, (size_t)n * sizeof(double), cudaMemcpyDeviceToDevice, st_));
  std::vector<int> hit(ns);
  DR_CK(cudaMemcpyAsync(hb.data(), sc.rr, 2 * (size_t)ns * sizeof(double), cudaMemcpyDeviceToHost, st_));
  DR_CK(cudaMemcpyAsync(hit.data(), sc.iters, (size_t)ns * sizeof(int), cudaMemcpyDeviceToHost, st_));
  DR_CK(cudaStreamSynchronize(st_));
  check_kernel_flag(st_);
  int maxit = 0;
  for (int q = 0; q < ns; ++q) {
    if (iters) iters[q] = hit[q];
    if (relres) relres[q] = hb[ns + q] > 0.0 ? std::sqrt(hb[q] / hb[ns + q]) : 0.0;
    maxit = std::max(maxit, hit[q]);
  }
  if (verbose >= 1)
    std::printf("batch AMG-PCG (%s cycle): %d systems, %d of them converged, %d iterations at most\n",
                mixed ? "FP32" : "FP64", ns, done, maxit);
  return maxit;
}

// dL/da_ij = -lambda_i x_j over the finest matrix's nonzeros (CSR order).
void DevHier::nz_gradient(const double* x, const double* lam, double* grad) {
  const DevMat& A = L_.empty() ? C_ : L_[0].A;
  counted();
  k_nz_grad<<<grid1d(A.n, max_grid_), kBlock, 0, st_>>>(A.n, A.rp, A.ci, x, lam, grad);
  DR_CK(cudaGetLastError());
  DR_CK(cudaStreamSynchronize(st_));
}

double DevHier::residual_norm(const double* x, const double* b, double* r) {
  residual<double>(0, x, b, r, scal_ + SC_TMP);
  DR_CK(cudaMemcpyAsync(hscal_ + SC_TMP, scal_ + SC_TMP, sizeof(double), cudaMemcpyDeviceToHost, st_));
  check_kernel_flag(st_);
  return std::sqrt(hscal_[SC_TMP]);
}

// ------------------------------------------------------------ PCG
// Preconditioned conjugate gradients around one AMG cycle per iteration
// (x of the cycle zeroed, as preconditioner_apply! does,
// src/preconditioner.jl:76-80).  Outer vectors, products with A and dot
// products are FP64; with `mixed` the cycle runs on FP32 copies of the
// hierarchy values and vectors.  Per iteration:
//   K1  q = A p,  p = z + β p_old (on the fly),  p·q       (one pass over A)
//   K2  r -= α q, r·r (and the FP32 copy of r), α stored    (one vector pass)
//   M   z = M r                                              (the cycle)
//   D   r·z                                                  (fused into M's last sweep)
//   X   x += α p                                             (beside M)
// K1+K2 and M+D+X are captured once as CUDA graphs (two of each, for the
// alternating direction buffers); X is a forked branch of the second, so
// the iterate's update runs while the cycle's latency-bound coarse levels
// leave bandwidth free.  The host reads r·r of iteration k while the
// preconditioner of iteration k runs.
int DevHier::pcg(double* x, const double* b, const CycleOpts& o, double tol, int maxiter, bool mixed,
                 double* relres, int verbose) {
  if (mixed) ensure_fp32();
  if (!pr_) {
    pr_ = alloc<double>(n0_);
    pp_[0] = alloc<double>(n0_);
    pp_[1] = alloc<double>(n0_);
    pq_ = alloc<double>(n0_);
    pz_ = alloc<double>(n0_);
  }
  if (mixed && !pr32_) {
    pr32_ = alloc<float>(n0_);
    pz32_ = alloc<float>(n0_);
  }
  if (pg_.valid && (pg_.mixed != mixed || pg_.o.pre != o.pre || pg_.o.post != o.post || pg_.o.w != o.w))
    graphs_clear();
  const DevMat& A = L_.empty() ? C_ : L_[0].A;
  const int n = n0_;
  double* X = xd_;
  if (x != X) DR_CK(cudaMemcpyAsync(X, x, (size_t)n * sizeof(double), cudaMemcpyDeviceToDevice, st_));
  // r = b - A x, r·r ;  b·b
  residual<double>(0, X, b, pr_, scal_ + SC_RR);
  counted();
  k_dot<double, double, FinStore><<<grid1d(n, max_grid_), kBlock, 0, st_>>>(n, b, b, partials_, tickets_ + TK_DOT,
                                                                           FinStore{scal_ + SC_BB});
  DR_CK(cudaGetLastError());
  DR_CK(cudaMemcpyAsync(hscal_, scal_, 2 * sizeof(double), cudaMemcpyDeviceToHost, st_));
  DR_CK(cudaStreamSynchronize(st_));
  const double bnorm = std::sqrt(hscal_[SC_BB]);
  if (bnorm == 0.0) {
    counted();
    k_fill<double><<<grid1d(n, max_grid_), kBlock, 0, st_>>>(n, 0.0, x);
    DR_CK(cudaStreamSynchronize(st_));
    if (relres) *relres = 0.0;
    return 0;
  }
  double rel = std::sqrt(hscal_[SC_RR]) / bnorm;
  if (rel < tol) {
    if (x != X) DR_CK(cudaMemcpyAsync(x, X, (size_t)n * sizeof(double), cudaMemcpyDeviceToDevice, st_));
    DR_CK(cudaStreamSynchronize(st_));
    if (relres) *relres = rel;
    return 0;
  }
  // z = M r (the cycle writes where it ends; the location is the same for
  // every application with the same options)
  void* zptr = nullptr;
  const bool fuse_rz = fused_rz_ok(o);
  auto precond = [&](bool rz_first) {
    if (mixed) {
      if (L_.empty()) {
        counted();
        k_convert<double, float><<<grid1d(n, max_grid_), kBlock, 0, st_>>>(n, pr_, pr32_);
        coarse_solve<float>(pr32_, pz32_);
        zptr = pz32_;
      } else {
        zptr = cycle_level<float>(0, pz32_, pr32_, true, o, pz32_, fuse_rz ? pr_ : nullptr, rz_first);
      }
      if (!fuse_rz) {
        counted();
        if (rz_first)
          k_dot<double, float, FinStore2><<<grid1d(n, max_grid_), kBlock, 0, st_>>>(
              n, pr_, (const float*)zptr, partials_, tickets_ + TK_RZ, FinStore2{scal_ + SC_RZ, scal_ + SC_RZOLD});
        else
          k_dot<double, float, FinShift><<<grid1d(n, max_grid_), kBlock, 0, st_>>>(
              n, pr_, (const float*)zptr, partials_, tickets_ + TK_RZ, FinShift{scal_ + SC_RZ, scal_ + SC_RZOLD});
      }
    } else {
      if (L_.empty()) {
        coarse_solve<double>(pr_, pz_);
        zptr = pz_;
      } else {
        zptr = cycle_level<double>(0, pz_, pr_, true, o, pz_, fuse_rz ? pr_ : nullptr, rz_first);
      }
      if (!fuse_rz) {
        counted();
        if (rz_first)
          k_dot<double, double, FinStore2><<<grid1d(n, max_grid_), kBlock, 0, st_>>>(
              n, pr_, (const double*)zptr, partials_, tickets_ + TK_RZ, FinStore2{scal_ + SC_RZ, scal_ + SC_RZOLD});
        else
          k_dot<double, double, FinShift><<<grid1d(n, max_grid_), kBlock, 0, st_>>>(
              n, pr_, (const double*)zptr, partials_, tickets_ + TK_RZ, FinShift{scal_ + SC_RZ, scal_ + SC_RZOLD});
      }
    }
    DR_CK(cudaGetLastError());
  };
  if (mixed) {
    counted();
    k_convert<double, float><<<grid1d(n, max_grid_), kBlock, 0, st_>>>(n, pr_, pr32_);
  }
  precond(true);
  counted();
  k_fill<double><<<grid1d(n, max_grid_), kBlock, 0, st_>>>(n, 0.0, pp_[0]);
  DR_CK(cudaGetLastError());
  auto k1k2 = [&](int par) {
    double* pold = pp_[par];
    double* pnew = pp_[par ^ 1];
    if (mixed) {
      XPcgDir<float> dir{(const float*)zptr, pold, scal_ + SC_RZ, 0.0};
      launch_rows_dot(st_, max_grid_, A, A.v, dir, EpPcgDir<float>{dir, pnew, pq_}, partials_,
                      tickets_ + TK_PQ, FinStore{scal_ + SC_PQ});
      counted();
      launch_dependent(k_pcg_update<float>, grid1d(n, max_grid_), kBlock, 0, st_, n, (double*)nullptr, pr_,
                       (const double*)pnew, (const double*)pq_, (const double*)(scal_ + SC_RZ),
                       (const double*)(scal_ + SC_PQ), pr32_, scal_ + SC_ALPHA, partials_,
                       tickets_ + TK_UPD, FinStore{scal_ + SC_RR});
    } else {
      XPcgDir<double> dir{(const double*)zptr, pold, scal_ + SC_RZ, 0.0};
      launch_rows_dot(st_, max_grid_, A, A.v, dir, EpPcgDir<double>{dir, pnew, pq_}, partials_,
                      tickets_ + TK_PQ, FinStore{scal_ + SC_PQ});
      counted();
      launch_dependent(k_pcg_update<float>, grid1d(n, max_grid_), kBlock, 0, st_, n, (double*)nullptr, pr_,
                       (const double*)pnew, (const double*)pq_, (const double*)(scal_ + SC_RZ),
                       (const double*)(scal_ + SC_PQ), (float*)nullptr, scal_ + SC_ALPHA, partials_,
                       tickets_ + TK_UPD, FinStore{scal_ + SC_RR});
    }
    DR_CK(cudaGetLastError());
    DR_CK(cudaMemcpyAsync(hscal_ + SC_RR, scal_ + SC_RR, sizeof(double), cudaMemcpyDeviceToHost, st_));
  };
  // capture the iteration graphs once per option set
  if (!pg_.valid) {
    for (int par = 0; par < 2; ++par) {
      cudaGraph_t g;
      const long long c0 = g_launches.load();
      DR_CK(cudaStreamBeginCapture(st_, cudaStreamCaptureModeThreadLocal));
      k1k2(par);
      DR_CK(cudaStreamEndCapture(st_, &g));
      pg_.n1[par] = g_launches.load() - c0;
      g_launches.fetch_sub(pg_.n1[par]);
      DR_CK(cudaGraphInstantiate(&pg_.g1[par], g, 0));
      cudaGraphDestroy(g);
    }
    for (int par = 0; par < 2; ++par) {
      // the preconditioner, and beside it (a forked branch) x += α p with
      // the direction of the iteration just finished
      cudaGraph_t g;
      const long long c0 = g_launches.load();
      DR_CK(cudaStreamBeginCapture(st_, cudaStreamCaptureModeThreadLocal));
      DR_CK(cudaEventRecord(ev_fork_, st_));
      DR_CK(cudaStreamWaitEvent(side_st_, ev_fork_, 0));
      counted();
      k_pcg_x<<<grid1d(n, max_grid_), kBlock, 0, side_st_>>>(n, X, pp_[par ^ 1], scal_ + SC_ALPHA);
      DR_CK(cudaGetLastError());
      DR_CK(cudaEventRecord(ev_join_, side_st_));
      precond(false);
      DR_CK(cudaStreamWaitEvent(st_, ev_join_, 0));
      DR_CK(cudaStreamEndCapture(st_, &g));
      pg_.n2[par] = g_launches.load() - c0;
      g_launches.fetch_sub(pg_.n2[par]);
      DR_CK(cudaGraphInstantiate(&pg_.g2[par], g, 0));
      cudaGraphDestroy(g);
    }
    pg_.valid = true;
    pg_.mixed = mixed;
    pg_.o = o;
  }
  int it = 1;
  for (; it <= maxiter; ++it) {
    const int par = (it - 1) & 1;
    DR_CK(cudaGraphLaunch(pg_.g1[par], st_));
    g_launches.fetch_add(pg_.n1[par]);
    DR_CK(cudaEventRecord(ev_[par], st_));
    const bool more = it < maxiter;
    if (more) {
      DR_CK(cudaGraphLaunch(pg_.g2[par], st_));  // also x += α p of this iteration
      g_launches.fetch_add(pg_.n2[par]);
    } else {
      counted();
      k_pcg_x<<<grid1d(n, max_grid_), kBlock, 0, st_>>>(n, X, pp_[par ^ 1], scal_ + SC_ALPHA);
      DR_CK(cudaGetLastError());
    }
    DR_CK(cudaEventSynchronize(ev_[par]));
    rel = std::sqrt(hscal_[SC_RR]) / bnorm;
    if (verbose >= 2) std::printf("  PCG iter %4d: relative residual = %.6e\n", it, rel);
    if (rel < tol || !more) break;
  }
  if (it > maxiter) it = maxiter;
  if (x != X) DR_CK(cudaMemcpyAsync(x, X, (size_t)n * sizeof(double), cudaMemcpyDeviceToDevice, st_));
  check_kernel_flag(st_);
  if (verbose >= 1)
    std::printf("AMG-PCG (%s cycle) %s: %d iterations, final residual %.2e\n", mixed ? "FP32" : "FP64",
                rel < tol ? "converged" : "did NOT converge", it, rel);
  if (relres) *relres = rel;
  return it;
}

// ------------------------------------------------------------ resetup
// One Galerkin product O = S·B (k_spgemm_warp): 8 warps per block, output
// rows of up to 384 entries staged in shared memory (longer rows work in
// place in global memory; a wider stage at lower occupancy measured slower
// on the 128^3 27-point hierarchy).
// The staged pattern capacity per warp is the smallest of 128, 256 and 384
// entries that holds the output's longest row (longer rows search global
// memory): 128 and 256 leave room for 8 blocks of 8 warps per SM (the
// register limit), 384 for 5.
// Record the product lists of O = S B (k_spgemm_sym: counts, an exclusive
// scan into offsets, then the pairs).  They cost 8 bytes per product and
// are kept only when that is under half of the free device memory; false
// when they are not built (the warp kernel then stays in use).
bool DevHier::build_spgemm_list(const DevMat& O, const DevMat& S, const DevMat& B, SpgemmList& L) {
  L.tried = true;
  const long long nout = O.nnz;
  if (nout <= 0 || O.n <= 0) return false;
  constexpr int W = 8, CAP = 256;
  const int grid = std::max(1, std::min((O.n + W - 1) / W, max_grid_));
  int* cnt = nullptr;
  long long* cnt64 = nullptr;
  void* tmp = nullptr;
  size_t tmp_bytes = 0;
  bool ok = false;
  DR_CK(cudaMalloc(&cnt, (size_t)nout * sizeof(int)));
  DR_CK(cudaMalloc(&cnt64, (size_t)(nout + 1) * sizeof(long long)));
  long long* off = alloc<long long>(nout + 1);
  DR_CK(cudaMemsetAsync(cnt, 0, (size_t)nout * sizeof(int), st_));
  counted();
  k_spgemm_sym<CAP, W, false><<<grid, W * 32, 0, st_>>>(O.n, O.rp, O.ci, S.rp, S.ci, B.rp, B.ci, cnt, nullptr,
                                                         nullptr, nullptr);
  DR_CK(cudaGetLastError());
  // widen the counts (the last one 0) and scan them into the offsets
  DR_CK(cudaMemsetAsync(cnt64, 0, (size_t)(nout + 1) * sizeof(long long), st_));
  counted();
  k_convert<int, long long><<<grid1d(nout, max_grid_), kBlock, 0, st_>>>(nout, cnt, cnt64);
  DR_CK(cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, cnt64, off, nout + 1, st_));
  DR_CK(cudaMalloc(&tmp, std::max<size_t>(tmp_bytes, 16)));
  DR_CK(cub::DeviceScan::ExclusiveSum(tmp, tmp_bytes, cnt64, off, nout + 1, st_));
  long long total = 0;
  DR_CK(cudaMemcpyAsync(&total, off + nout, sizeof(long long), cudaMemcpyDeviceToHost, st_));
  DR_CK(cudaStreamSynchronize(st_));
  size_t free_b = 0, total_b = 0;
  DR_CK(cudaMemGetInfo(&free_b, &total_b));
  if (total > 0 && (size_t)total * 8 < free_b / 2) {
    L.ls = alloc<int>((size_t)total);
    L.lb = alloc<int>((size_t)total);
    DR_CK(cudaMemsetAsync(cnt, 0, (size_t)nout * sizeof(int), st_));
    counted();
    k_spgemm_sym<CAP, W, true><<<grid, W * 32, 0, st_>>>(O.n, O.rp, O.ci, S.rp, S.ci, B.rp, B.ci, cnt, off,
                                                          L.ls, L.lb);
    DR_CK(cudaGetLastError());
    L.off = off;
    L.total = total;
    ok = true;
  }
  DR_CK(cudaStreamSynchronize(st_));
  DR_CK(cudaFree(tmp));
  DR_CK(cudaFree(cnt64));
  DR_CK(cudaFree(cnt));
  return ok;
}

template <typename T>
void DevHier::spgemm(DevMat& O, const DevMat& S, const DevMat& B, T* ov, const T* sv, const T* bv,
                     SpgemmList* list) {
  if (list && !list->tried) build_spgemm_list(O, S, B, *list);
  if (list && list->off) {
    constexpr int WA = 8, CAPW = 768;  // 48 KB of staged pairs per block
    auto kf = k_spgemm_apply_staged<T, WA, CAPW>;
    const int grid = (int)std::max<long long>(
        1, std::min<long long>((O.nnz + 32 * WA - 1) / (32 * WA), (long long)g_nsm * resident_blocks((const void*)kf, WA * 32, 0)));
    counted();
    kf<<<grid, WA * 32, 0, st_>>>(O.nnz, list->off, list->ls, list->lb, sv, bv, ov);
    DR_CK(cudaGetLastError());
    return;
  }
  constexpr int W = 8;
  counted();
  const int grid = std::max(1, std::min((O.n + W - 1) / W, max_grid_));
#define DR_SPGEMM(CAP)                                                                      \
  k_spgemm_warp<T, CAP, W><<<grid, W * 32, spgemm_smem_bytes<T, CAP, W>(), st_>>>(        \
      O.n, O.rp, O.ci, ov, S.rp, S.ci, sv, B.rp, B.ci, bv)
  if (O.maxlen <= 128) DR_SPGEMM(128);
  else if (O.maxlen <= 256) DR_SPGEMM(256);
  else DR_SPGEMM(384);
#undef DR_SPGEMM
  DR_CK(cudaGetLastError());
}

void DevHier::set_resetup_fp64_levels(int n) {
  resetup_fp64_ = n;
}

// The numeric product O = S·B on O's pattern with the warp kernel, on raw
// device arrays (the setup's device Galerkin products).
void galerkin_numeric_raw(cudaStream_t st, int n, int maxlen, const int* o_rp, const int* o_ci, double* o_v,
                          const int* s_rp, const int* s_ci, const double* s_v, const int* b_rp,
                          const int* b_ci, const double* b_v, int max_grid) {
  if (n <= 0) return;
  constexpr int W = 8;
  const int grid = std::max(1, std::min((n + W - 1) / W, max_grid));
  counted();
#define DR_SPGEMM(CAP)                                                                      \
  k_spgemm_warp<double, CAP, W><<<grid, W * 32, spgemm_smem_bytes<double, CAP, W>(), st>>>( \
      n, o_rp, o_ci, o_v, s_rp, s_ci, s_v, b_rp, b_ci, b_v)
  if (maxlen <= 128) DR_SPGEMM(128);
  else if (maxlen <= 256) DR_SPGEMM(256);
  else DR_SPGEMM(384);
#undef DR_SPGEMM
  DR_CK(cudaGetLastError());
}

void DevHier::resetup_values(const double* v_dev) {
  const int nl = nlevels();
  for (int l = 0; l < nl; ++l)
    if (!L_[l].has_rap)
      fail("partial resetup needs the Galerkin maps; set up the hierarchy with allow_partial_resetup=1");
  graphs_clear();
  if (nl == 0) {
    DR_CK(cudaMemcpyAsync(C_.v, v_dev, (size_t)C_.nnz * sizeof(double), cudaMemcpyDeviceToDevice, st_));
  } else {
    DR_CK(cudaMemcpyAsync(L_[0].A.v, v_dev, (size_t)L_[0].A.nnz * sizeof(double), cudaMemcpyDeviceToDevice, st_));
  }
  auto upd_invd = [&](DevLevel& d) {
    counted();
    if (d.smoother == SmootherKind::L1Jacobi || d.smoother == SmootherKind::L1ColoredGS ||
        d.smoother == SmootherKind::L1SerialGS)
      k_l1_invdiag<<<grid1d(d.A.n, max_grid_), kBlock, 0, st_>>>(d.A.n, d.A.rp, d.A.v, d.invd);
    else if (d.smoother == SmootherKind::SerialGS)
      k_sgs_invdiag<<<grid1d(d.A.n, max_grid_), kBlock, 0, st_>>>(d.A.n, d.A.rp, d.A.ci, d.A.v, d.invd);
    else if (d.smoother == SmootherKind::SPAI0)
      k_spai0_diag<<<grid1d(d.A.n, max_grid_), kBlock, 0, st_>>>(d.A.n, d.A.rp, d.A.ci, d.A.v, d.invd);
    else
      k_invdiag<<<grid1d(d.A.n, max_grid_), kBlock, 0, st_>>>(d.A.n, d.A.rp, d.A.ci, d.A.v, d.invd);
    DR_CK(cudaGetLastError());
    if (d.spai1_M) {
      // update_smoother!(::SPAI1Smoother), src/smoothers.jl:692-699: M again
      // on the host from the level's new values, as in the reference
      CSR a;
      a.n = a.m = d.A.n;
      a.rp = d.ilu_rp;
      a.ci = d.ilu_ci;
      a.v.resize(d.A.nnz);
      DR_CK(cudaMemcpyAsync(a.v.data(), d.A.v, (size_t)d.A.nnz * sizeof(double), cudaMemcpyDeviceToHost, st_));
      DR_CK(cudaStreamSynchronize(st_));
      std::vector<double> Mh;
      spai1_values(a, Mh);
      h2d(d.spai1_M, Mh, st_);
      DR_CK(cudaStreamSynchronize(st_));
    }
    if (d.ilu_L) {
      // update_smoother!(::ILU0Smoother / ::SerialILU0Smoother), src/
      // smoothers.jl:1332-1337: the factorisation is sequential, so it runs
      // on the host from the level's new values, as in the reference
      CSR a;
      a.n = a.m = d.A.n;
      a.rp = d.ilu_rp;
      a.ci = d.ilu_ci;
      a.v.resize(d.A.nnz);
      DR_CK(cudaMemcpyAsync(a.v.data(), d.A.v, (size_t)d.A.nnz * sizeof(double), cudaMemcpyDeviceToHost, st_));
      DR_CK(cudaStreamSynchronize(st_));
      std::vector<double> Lh, Uh;
      ilu0_factorize(a, d.ilu_diag_h, Lh, Uh);
      h2d(d.ilu_L, Lh, st_);
      h2d(d.ilu_U, Uh, st_);
      DR_CK(cudaStreamSynchronize(st_));  // Lh, Uh leave scope
    }
    if (d.smoother == SmootherKind::Chebyshev) {
      // update_smoother!(::ChebyshevSmoother): the spectral radius of D^-1 A
      // again (10 power steps from the stored start vector, on the device),
      // then the coefficients
      double* v = d.v64.xb;
      double* w = d.v64.r;
      double* lam2 = d.cheb_coef + 2 * d.cheb_degree;
      DR_CK(cudaMemcpyAsync(v, d.cheb_v0, (size_t)d.A.n * sizeof(double), cudaMemcpyDeviceToDevice, st_));
      for (int it = 0; it < 10; ++it) {
        launch_rows_dot(st_, max_grid_, d.A, d.A.v, XPlain<double>{v}, EpPowerStep{d.invd, w}, partials_,
                        tickets_ + TK_DOT, FinStore{lam2});
        counted();
        k_cheb_rescale<<<grid1d(d.A.n, max_grid_), kBlock, 0, st_>>>(d.A.n, w, lam2, v);
      }
      counted();
      k_cheb_coef<<<1, 32, 0, st_>>>(lam2, d.cheb_degree, d.cheb_coef);
      DR_CK(cudaGetLastError());
    }
  };
  if (nl > 0) upd_invd(L_[0]);
  // Galerkin products 0 .. f64-1 in FP64, the rest in FP32 (on the FP32
  // copies of A, P and Pᵀ; the FP64 copy of each FP32-computed level is its
  // FP32 values widened, so both copies agree)
  const int f64 = resetup_fp64_ < 0 ? nl : std::min(resetup_fp64_, nl);
  if (f64 < nl) ensure_fp32();
  for (int l = 0; l < nl; ++l) {
    DevLevel& d = L_[l];
    DevMat& next = (l + 1 < nl) ? L_[l + 1].A : C_;
    if (l < f64) {
      spgemm<double>(d.AP, d.A, d.P, d.AP.v, d.A.v, d.P.v, &d.ap_list);
      spgemm<double>(next, d.R, d.AP, next.v, d.R.v, d.AP.v, &d.rap_list);
    } else {
      if (l == f64) {  // this level's values came from FP64 (a product above, or the input)
        counted();
        k_convert<double, float><<<grid1d(d.A.nnz, max_grid_), kBlock, 0, st_>>>(d.A.nnz, d.A.v, d.A.v32);
      }
      if (!d.AP.v32) d.AP.v32 = alloc<float>(d.AP.nnz + 4);
      if (!next.v32) next.v32 = alloc<float>(next.nnz + 4);
      spgemm<float>(d.AP, d.A, d.P, d.AP.v32, d.A.v32, d.P.v32, &d.ap_list);
      spgemm<float>(next, d.R, d.AP, next.v32, d.R.v32, d.AP.v32, &d.rap_list);
      counted();
      k_convert<float, double><<<grid1d(next.nnz, max_grid_), kBlock, 0, st_>>>(next.nnz, next.v32, next.v);
      DR_CK(cudaGetLastError());
    }
    if (d.fuse_up) {
      // Q from this level's new A·P (widened when formed in FP32) and the
      // inverse diagonal refreshed with the level's values above
      if (l >= f64) {
        counted();
        k_convert<float, double><<<grid1d(d.AP.nnz, max_grid_), kBlock, 0, st_>>>(d.AP.nnz, d.AP.v32, d.AP.v);
      }
      build_q(d);
    }
    if (l + 1 < nl) upd_invd(L_[l + 1]);
  }
  // coarsest dense matrix and its LU
  DR_CK(cudaMemsetAsync(cdense_, 0, (size_t)nc_ * nc_ * sizeof(double), st_));
  counted();
  k_csr_to_dense<<<grid1d(nc_, max_grid_), kBlock, 0, st_>>>(nc_, C_.rp, C_.ci, C_.v, cdense_);
  DR_CK(cudaMemcpyAsync(clu_, cdense_, (size_t)nc_ * nc_ * sizeof(double), cudaMemcpyDeviceToDevice, st_));
  int threads = 32;
  while (threads < nc_ && threads < 1024) threads *= 2;
  counted();
  k_lu_factor<<<1, threads, 0, st_>>>(nc_, clu_, cpiv_, info_);
  DR_CK(cudaGetLastError());
  if (cinv_ok_) build_cinv();
  if (at_built_) refresh_transpose();  // before the FP32 copies, which include the transposed ones
  refresh_fp32();
  check_kernel_flag(st_);
  int info = 0;
  DR_CK(cudaMemcpyAsync(&info, info_, sizeof(int), cudaMemcpyDeviceToHost, st_));
  DR_CK(cudaStreamSynchronize(st_));
  if (info != 0) fail("SingularException(" + std::to_string(info) + ")");
}

// ------------------------------------------------------------ level ops
void DevHier::level_op(int lvl, int op, bool fp32, const double* in1, const double* in2, double* out,
                       int steps) {
  const int nl = nlevels();
  if (op != 5 && (lvl < 0 || lvl >= nl)) fail("level index out of range");
  if (fp32) ensure_fp32();
  const int n = op == 5 ? nc_ : L_[lvl].A.n;
  const int ncn = op == 5 ? nc_ : (lvl + 1 < nl ? L_[lvl + 1].A.n : nc_);
  auto run = [&](auto tag) {
    using T = decltype(tag);
    LevelVecs<T>& V = vecs<T>(op == 5 ? 0 : lvl);
    auto to_t = [&](const double* s, T* d, int m) {
      counted();
      k_convert<double, T><<<grid1d(m, max_grid_), kBlock, 0, st_>>>(m, s, d);
    };
    auto from_t = [&](const T* s, double* d, int m) {
      counted();
      k_convert<T, double><<<grid1d(m, max_grid_), kBlock, 0, st_>>>(m, s, d);
    };
    // staging buffers in T: use level vectors (xa may be null at level 0)
    T* bufA = V.xb;
    T* bufB = V.r;
    switch (op) {
      case 0: {  // y = A x
        to_t(in1, bufA, n);
        const DevMat& A = L_[lvl].A;
        launch_rows(st_, max_grid_, A, mval<T>(A), XPlain<T>{bufA}, EpStore<T>{bufB});
        from_t(bufB, out, n);
        break;
      }
      case 1: {  // r = b - A x   (third buffer: level rhs, or the PCG z at level 0)
        T* tb = lvl > 0 ? V.b : nullptr;
        if (!tb) {
          if constexpr (sizeof(T) == 8) { if (!pz_) pz_ = alloc<double>(n0_); tb = (T*)pz_; }
          else { if (!pz32_) pz32_ = alloc<float>(n0_); tb = (T*)pz32_; }
        }
        to_t(in1, bufA, n);
        to_t(in2, tb, n);
        residual<T>(lvl, bufA, tb, bufB, nullptr);
        from_t(bufB, out, n);
        break;
      }
      case 2: {  // smoothing sweeps from x with rhs b (lvl >= 1: xa/b; lvl 0: xb + z)
        T* tb;
        T* x0;
        T* ext;
        if (lvl > 0) {
          tb = V.b;
          x0 = V.xa;
          ext = nullptr;
        } else {
          if constexpr (sizeof(T) == 8) { if (!pz_) pz_ = alloc<double>(n0_); tb = (T*)pz_; }
          else { if (!pz32_) pz32_ = alloc<float>(n0_); tb = (T*)pz32_; }
          x0 = V.r;   // caller-side x
          ext = V.r;
        }
        to_t(in1, x0, n);
        to_t(in2, tb, n);
        T* xr = smooth<T>(lvl, x0, tb, steps, ext);
        from_t(xr, out, n);
        break;
      }
      case 3: {  // bc = Pᵀ r
        to_t(in1, bufB, n);
        T* bc = (lvl + 1 < nl) ? vecs<T>(lvl + 1).b : coarse_b<T>();
        launch_rows(st_, max_grid_, L_[lvl].R, mval<T>(L_[lvl].R), XPlain<T>{bufB}, EpStore<T>{bc});
        from_t(bc, out, ncn);
        break;
      }
      case 4: {  // x += P xc
        T* xc = (lvl + 1 < nl) ? vecs<T>(lvl + 1).b : coarse_b<T>();
        to_t(in1, bufA, n);
        to_t(in2, xc, ncn);
        launch_rows(st_, max_grid_, L_[lvl].P, mval<T>(L_[lvl].P), XPlain<T>{xc}, EpAddTo<T>{bufA});
        from_t(bufA, out, n);
        break;
      }
      case 5: {  // coarsest solve
        to_t(in1, coarse_b<T>(), nc_);
        coarse_solve<T>(coarse_b<T>(), coarse_x<T>());
        from_t(coarse_x<T>(), out, nc_);
        break;
      }
      case 6: {  // first Jacobi step from zero fused with the residual: out = [x1, r]
        const DevLevel& L = L_[lvl];
        T* tb;
        if (lvl > 0) tb = V.b;
        else {
          if constexpr (sizeof(T) == 8) { if (!pz_) pz_ = alloc<double>(n0_); tb = (T*)pz_; }
          else { if (!pz32_) pz32_ = alloc<float>(n0_); tb = (T*)pz32_; }
        }
        to_t(in1, tb, n);
        const T om = (T)L.omega;
        launch_rows(st_, max_grid_, L.A, mval<T>(L.A), XZeroJacobi<T>{tb, invd<T>(L), om},
                    EpZeroJacobiResidual<T>{tb, invd<T>(L), bufA, bufB, om});
        from_t(bufA, out, n);
        from_t(bufB, out + n, n);
        break;
      }
      default:
        fail("unknown level op");
    }
    DR_CK(cudaGetLastError());
  };
  if (fp32) run(float());
  else run(double());
  check_kernel_flag(st_);
}

float DevHier::time_level_op(int lvl, int op, bool fp32, int reps) {
  if (lvl < 0 || lvl >= nlevels()) fail("level index out of range");
  if (op != 0 && op != 2 && op != 3 && op != 4 && op != 6 && op != 8)
    fail("time_level_op: op must be 0, 2, 3, 4, 6 or 8");
  if (op == 8 && (lvl < 1 || batch_)) fail("time_level_op: op 8 times a cycle from a level >= 1");
  if (fp32) ensure_fp32();
  cudaEvent_t e0, e1;
  DR_CK(cudaEventCreate(&e0));
  DR_CK(cudaEventCreate(&e1));
  float ms = 0.f;
  auto run = [&](auto tag) {
    using T = decltype(tag);
    DevLevel& L = L_[lvl];
    LevelVecs<T>& V = vecs<T>(lvl);
    const bool last = lvl + 1 == nlevels();
    const int n = L.A.n, nc = L.P.m;
    T* x0 = V.r;                                   // operand vectors of this level
    T* x1 = V.xb;
    T* cvec = last ? coarse_b<T>() : vecs<T>(lvl + 1).b;   // coarse-size vector
    if (!tout_) tout_ = alloc<double>(n0_);       // scratch: right-hand side of op 2,
    if (!tout2_) tout2_ = alloc<double>(n0_);     // second result of op 6
    T* bt = reinterpret_cast<T*>(tout_);
    T* x2 = reinterpret_cast<T*>(tout2_);
    counted();
    k_fill<T><<<grid1d(n, max_grid_), kBlock, 0, st_>>>(n, T(1), x0);
    counted();
    k_fill<T><<<grid1d(n, max_grid_), kBlock, 0, st_>>>(n, T(1), x1);
    counted();
    k_fill<T><<<grid1d(n, max_grid_), kBlock, 0, st_>>>(n, T(1), bt);
    counted();
    k_fill<T><<<grid1d(nc, max_grid_), kBlock, 0, st_>>>(nc, T(1), cvec);
    if (op == 8) {
      counted();
      k_fill<T><<<grid1d(n, max_grid_), kBlock, 0, st_>>>(n, T(1), V.b);
    }
    const T om = (T)L.omega;
    auto once = [&]() {
      switch (op) {
        case 0:
          launch_rows(st_, max_grid_, L.A, mval<T>(L.A), XPlain<T>{x0}, EpStore<T>{x1});
          break;
        case 2:
          launch_rows(st_, max_grid_, L.A, mval<T>(L.A), XPlain<T>{x0},
                      EpJacobi<T>{x0, bt, invd<T>(L), x1, om, nullptr});
          break;
        case 3:
          launch_rows(st_, max_grid_, L.R, mval<T>(L.R), XPlain<T>{x0}, EpStore<T>{cvec});
          break;
        case 4:
          launch_rows(st_, max_grid_, L.P, mval<T>(L.P), XPlain<T>{cvec}, EpAddTo<T>{x1});
          break;
        case 6:
          launch_rows(st_, max_grid_, L.A, mval<T>(L.A), XZeroJacobi<T>{x0, invd<T>(L), om},
                      EpZeroJacobiResidual<T>{x0, invd<T>(L), x1, x2, om});
          break;
        case 8:  // the V(1,1) cycle from level lvl down, from zero (the coarse tail included)
          cycle_level<T>(lvl, V.xa, V.b, true, CycleOpts{}, nullptr, nullptr, false, false);
          break;
      }
    };
    for (int w = 0; w < 3; ++w) once();
    DR_CK(cudaEventRecord(e0, st_));
    for (int r = 0; r < reps; ++r) once();
    DR_CK(cudaEventRecord(e1, st_));
    DR_CK(cudaEventSynchronize(e1));
    DR_CK(cudaEventElapsedTime(&ms, e0, e1));
  };
  if (fp32) run(float());
  else run(double());
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  check_kernel_flag(st_);
  return ms / reps;
}

void DevHier::export_values(int lvl, const std::string& what, std::vector<double>& out) const {
  const double* src = nullptr;
  long long n = 0;
  if (lvl == -1) {
    if (what == "C_nzval") { src = C_.v; n = C_.nnz; }
    else if (what == "C_lu") { src = clu_; n = (long long)nc_ * nc_; }
    else if (what == "C_dense") { src = cdense_; n = (long long)nc_ * nc_; }
  } else {
    const DevLevel& d = L_.at(lvl);
    if (what == "A_nzval") { src = d.A.v; n = d.A.nnz; }
    else if (what == "P_nzval") { src = d.P.v; n = d.P.nnz; }
    else if (what == "invdiag") { src = d.invd; n = d.A.n; }
    else if (what == "cheb_coef" && d.cheb_coef) { src = d.cheb_coef; n = 2LL * d.cheb_degree; }
    else if (what == "ilu_L" && d.ilu_L) { src = d.ilu_L; n = d.A.nnz; }
    else if (what == "spai1_M" && d.spai1_M) { src = d.spai1_M; n = d.A.nnz; }
    else if (what == "ilu_U" && d.ilu_U) { src = d.ilu_U; n = d.A.nnz; }
    else if (what == "AP_nzval" && d.has_rap) { src = d.AP.v; n = d.AP.nnz; }
  }
  if (!src) fail("unknown device export: " + what);
  out.resize(n);
  DR_CK(cudaMemcpyAsync(out.data(), src, n * sizeof(double), cudaMemcpyDeviceToHost, st_));
  DR_CK(cudaStreamSynchronize(st_));
}

void DevHier::export_piv(std::vector<int>& out) const {
  out.resize(nc_);
  DR_CK(cudaMemcpyAsync(out.data(), cpiv_, (size_t)nc_ * sizeof(int), cudaMemcpyDeviceToHost, st_));
  DR_CK(cudaStreamSynchronize(st_));
}

}  // namespace dr
