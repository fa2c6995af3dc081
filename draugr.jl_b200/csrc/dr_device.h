// Device-resident hierarchy and the solve / resetup drivers.
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <map>
#include <memory>
#include <set>
#include <string>
#include <utility>
#include <vector>

#include "dr_host.h"

namespace dr {

void cuda_check(cudaError_t e, const char* what, const char* file, int line);
long long kernel_launches();
void note_launch();  // counts one kernel launch (kernel_launches)
// Polls a row kernel makes on a tile copy before it reports a timeout
// (negative: the default).  A test hook.
void set_tile_wait_limit(int polls);
#define DR_CK(x) ::dr::cuda_check((x), #x, __FILE__, __LINE__)

// Nonzeros per tile of the row kernel (k_tile_rows); rows longer than this
// are reduced by a whole block in a fixed tree order instead of in column
// order.
constexpr int kRowTileCap = 2000;

// Form of the row kernel (k_tile_rows) for a CSR pattern:
//   flat    rows of very uneven length averaging at most 32 entries (a long
//           row among short ones): products formed flat over each tile,
//           then one thread per row sums them in column order;
//   G = 1   one lane per row, rows summed in column order: batches of 4
//           gathers with 512-thread blocks up to 5 entries per row on
//           average (interpolation rows: 512 rows fill a tile), batches of
//           8 with 256-thread blocks up to 12, batches of 32 with
//           128-thread blocks up to 32;
//   G > 1   longer rows, summed by G lanes and a fixed shuffle tree: 8 or
//           16 lanes gathering 12 entries each at once (about 27 or 13
//           rows fill a tile), or 32 lanes with 4 each when a few rows are
//           much longer than the rest.
struct RowForm {
  int G = 1;
  bool flat = false;
  bool ordered = true;  // every row (up to the tile capacity) in column order
  int nt = 256;         // threads per block
  int batch = 8;        // gathers in flight per lane (G = 1)
};

inline RowForm row_form(const std::vector<int>& rp) {
  RowForm f;
  const size_t n = rp.size() ? rp.size() - 1 : 0;
  if (n == 0) return f;
  int maxlen = 0;
  for (size_t i = 0; i < n; ++i) maxlen = std::max(maxlen, rp[i + 1] - rp[i]);
  const double avg = (double)(rp[n] - rp[0]) / (double)n;
  if (avg <= 32.0 && maxlen > 64 && maxlen > 4.0 * avg) {
    f.flat = true;
  } else if (avg <= 32.0) {
    if (avg > 12.0) {
      f.nt = 128;
      f.batch = 32;
    } else if (avg <= 5.0) {
      f.nt = 512;  // very short rows (interpolation): 512 rows fill a tile
      f.batch = 4;
    }
  } else {
    f.ordered = false;
    if (maxlen > 4.0 * avg) {
      f.G = 32;  // a few long rows set each tile's time: many lanes per row
      f.batch = 4;
    } else {
      f.G = avg <= 100 ? 8 : 16;  // full tiles, a row in one round of gathers
      f.batch = 12;
    }
  }
  return f;
}

// 1 when the row kernel reduces every row of the CSR pattern in column
// order (the reference's order, bit for bit): an ordered form and no row
// longer than the tile capacity.
inline int rows_in_order(const std::vector<int>& rp) {
  const size_t n = rp.size() ? rp.size() - 1 : 0;
  if (n == 0) return 1;
  int maxlen = 0;
  for (size_t i = 0; i < n; ++i) maxlen = std::max(maxlen, rp[i + 1] - rp[i]);
  return (maxlen <= kRowTileCap && row_form(rp).ordered) ? 1 : 0;
}

// Sparse matrix on the device: CSR pattern, FP64 values and (after the first
// mixed-precision use) an FP32 copy of the values, plus the row tiling of
// the row kernel.
struct DevMat {
  int n = 0, m = 0;
  long long nnz = 0;
  int* rp = nullptr;
  int* ci = nullptr;
  double* v = nullptr;
  float* v32 = nullptr;
  RowForm form;       // form of the row kernel
  int Ggs = 8;        // lanes per row of the Gauss-Seidel colour kernel
  int ntiles = 0;     // row tiles (see k_tile_rows)
  int* tp = nullptr;  // tile row starts, ntiles+1
  int* ts = nullptr;  // tile nonzero starts, ntiles+1
  int* tb = nullptr;       // tile smallest columns (-1: row too wide for offsets), ntiles
  uint16_t* cu = nullptr;  // columns as offsets from their tile's smallest column
  int maxlen = 0;          // longest row
};

template <typename T>
struct LevelVecs {
  T* xa = nullptr;  // iterate (levels >= 1) ...
  T* xb = nullptr;  // ... and its Jacobi ping-pong partner (level 0: partner of the caller's x)
  T* b = nullptr;   // right-hand side (levels >= 1: written by the restriction above)
  T* r = nullptr;   // residual
  T* d = nullptr;   // Chebyshev update direction (Chebyshev levels only)
};

// Product lists of one numeric Galerkin product on fixed patterns (see
// k_spgemm_sym): per output entry its (S entry, B entry) pairs.
struct SpgemmList {
  long long* off = nullptr;  // nout + 1
  int* ls = nullptr;         // total pairs
  int* lb = nullptr;
  long long total = 0;
  bool tried = false;        // a build was attempted (memory may have been short)
};

struct DevLevel {
  DevMat A, P, R;            // R = Pᵀ stored as the transpose map with values
  int nv = 0;                // length of the level's vectors (A.n, more in a batch)
  SmootherKind smoother = SmootherKind::Jacobi;
  double omega = 2.0 / 3.0;
  double* invd = nullptr;
  float* invd32 = nullptr;
  int ncolors = 0;
  std::vector<int> color_off;  // host copy, num_colors+1
  int* color_order = nullptr;
  bool has_rap = false;
  DevMat AP;                 // pattern and values of A·P (partial resetup)
  SpgemmList ap_list, rap_list;  // product lists of A·P and Pᵀ·(AP), built on the first resetup
  // Fused correction and first post-smoothing step (EpCorrectJacobi): Q =
  // P - ω·D⁻¹·(A P) on AP's pattern, on levels where A·P has fewer entries
  // than A and P together and A's rows are summed in a tree; pq_pos: each P
  // entry's position in AP's row
  bool fuse_up = false;
  double* q = nullptr;
  float* q32 = nullptr;
  int* pq_pos = nullptr;
  DevMat At;                 // A^T (transposed cycles; built on first use)
  int* at_perm = nullptr;    // At value k = A value at_perm[k]
  double* invdT = nullptr;   // smoother diagonal of A^T
  float* invdT32 = nullptr;  // its FP32 copy (FP32 transposed cycles)
  // Chebyshev: inner steps per application, the normalised power-iteration
  // start vector, and the coefficient table (2 * degree entries, then the
  // squared norm of the last power step)
  int cheb_degree = 0;
  double* cheb_v0 = nullptr;
  double* cheb_coef = nullptr;
  // ILU(0): diagonal positions, factors (FP64; FP32 after the first mixed
  // use), the substitution schedules (rows by level on the device, level
  // offsets on the host); ilu_rp / ilu_ci: the host pattern for recomputing
  // ILU(0) factors or SPAI(1)'s M after a resetup
  int* ilu_diag = nullptr;
  double *ilu_L = nullptr, *ilu_U = nullptr;
  float *ilu_L32 = nullptr, *ilu_U32 = nullptr;
  int *ilu_fwd = nullptr, *ilu_bwd = nullptr;
  std::vector<int> ilu_fwd_off, ilu_bwd_off, ilu_rp, ilu_ci, ilu_diag_h;
  // serial Gauss-Seidel: rows by level (device), level offsets (host)
  int* sgs_order = nullptr;
  std::vector<int> sgs_off;
  // SPAI(1): M on A's pattern (FP64; FP32 after the first mixed use)
  double* spai1_M = nullptr;
  float* spai1_M32 = nullptr;
  LevelVecs<double> v64;
  LevelVecs<float> v32;
};

struct CycleOpts {
  int pre = 1;
  int post = 1;
  bool w = false;
};

// Independent systems merged level by level (a batch).  Merged level l
// holds, in system order, the rows of the systems that still smooth there
// (the block-diagonal A, P and Pᵀ act on these), then the rows of the
// systems whose coarsest level it is (solved by their own dense LU).
struct BatchLayout {
  int nsys = 0;
  std::vector<int> depth;             // AMG levels of each system
  std::vector<int> nsmooth, ntotal;   // per merged level 0..Lmax
  std::vector<std::vector<int>> off;  // off[l][s]: first row of system s at level l (-1: absent)
  struct Coarse {
    std::vector<int> off, nb, poff;   // per system ending at the level: rows, size, pivot offset
    std::vector<long long> luoff;     // offset of its factors
    int maxn = 0;
  };
  std::vector<Coarse> coarse;         // per merged level
  std::vector<double> lu;             // all coarsest factors (column-major each)
  std::vector<int> piv;               // all pivots (0-based)
};

// Numeric product O = S·B on O's fixed pattern (k_spgemm_warp), raw device
// arrays, on stream st; maxlen: O's longest row.
void galerkin_numeric_raw(cudaStream_t st, int n, int maxlen, const int* o_rp, const int* o_ci, double* o_v,
                          const int* s_rp, const int* s_ci, const double* s_v, const int* b_rp,
                          const int* b_ci, const double* b_v, int max_grid);
// A device implementation of the setup's Galerkin products on the current
// device (nullptr when no device is usable or DRAUGR_B200_GPU_SETUP=0).
std::unique_ptr<GalerkinDevice> make_galerkin_device();

// Merge the hierarchies of independent systems into one (CPU); every
// level of every system must use a Jacobi-type smoother, and systems that
// share a level the same smoother and weight.
HostHierarchy merge_batch(const std::vector<const HostHierarchy*>& hs, BatchLayout& lay);

// Launch shape of a block (multi-right-hand-side) product: threads per row
// (32 / tpr rows per warp) and resident blocks per SM; 0 takes the default.
struct BlockShape {
  int tpr = 0, nb = 0;
};

// Per-launch timing of the dominant kernels, filled when enabled.
struct KernelClock {
  bool enabled = false;
  std::vector<cudaEvent_t> ev;  // pairs (start, stop)
  std::vector<int> tag;         // 0 = finest-level smoother sweep
};

class DevHier {
 public:
  DevHier(const HostHierarchy& H, int device, const BatchLayout* batch = nullptr);
  ~DevHier();
  DevHier(const DevHier&) = delete;
  DevHier& operator=(const DevHier&) = delete;

  int n0() const { return n0_; }
  int nlevels() const { return (int)L_.size(); }
  cudaStream_t stream() const { return st_; }
  // Run on the caller's stream (nullptr: back to the library's own stream).
  void set_stream(cudaStream_t s);
  size_t device_bytes() const { return bytes_; }

  // Raise if a kernel of this device reported a bounded wait that gave up
  // (synchronises the stream; clears the flag).
  void check_errors();

  // Galerkin products of a partial resetup computed in FP64 from the top:
  // n of them (the rest in FP32 on the FP32 copies); negative: all FP64.
  void set_resetup_fp64_levels(int n);
  int resetup_fp64_levels() const { return resetup_fp64_; }

  // Solve phase (device pointers, length n0).
  void cycle(double* x, const double* b, const CycleOpts& o);
  int solve(double* x, const double* b, const CycleOpts& o, double tol, int maxiter, int verbose,
            double* relres);
  int pcg(double* x, const double* b, const CycleOpts& o, double tol, int maxiter, bool mixed,
          double* relres, int verbose);
  // Right-preconditioned BiCGStab (FP64) on A, or on A^T with cycles on the
  // transposed hierarchy (adjoint solves); Jacobi-type smoothers.
  int bicgstab(double* x, const double* b, const CycleOpts& o, double tol, int maxiter, bool transpose,
               double* relres, int verbose, bool mixed = false);
  // Batch (a hierarchy built from merge_batch): conjugate gradients on every
  // system at once, each with its own step sizes and convergence test, one
  // launch per cycle stage for all systems; one iteration is captured in a
  // CUDA graph.  x, b: all systems' vectors, concatenated.  iters, relres:
  // per system.  Returns the largest iteration count.
  int pcg_batch_seg(double* x, const double* b, const CycleOpts& o, double tol, int maxiter, bool mixed,
                    int* iters, double* relres, int verbose);
  bool is_batch() const { return batch_ != nullptr; }
  int batch_systems() const { return batch_ ? batch_->nsys : 0; }
  const BatchLayout* batch_layout() const { return batch_.get(); }
  // Flexible GMRES(restart), right-preconditioned by one AMG cycle per
  // iteration (FP64, or with `mixed` the FP32 cycle), FP64 Arnoldi
  // (classical Gram-Schmidt, twice), until ||b - A x|| / ||b|| < tol.
  int fgmres(double* x, const double* b, const CycleOpts& o, double tol, int maxiter, int restart,
             bool mixed, double* relres, int verbose);
  // Iterative refinement: r = b - A x in FP64, A d = r solved to inner_tol
  // (relative to ||r||) by AMG-PCG (inner 0) or FGMRES (inner 1), x += d,
  // until ||b - A x|| / ||b|| < tol.  Returns the outer steps; inner_total
  // receives the inner iterations.
  int refine(double* x, const double* b, const CycleOpts& o, double tol, int max_outer, double inner_tol,
             int inner_maxiter, int inner, bool mixed, double* relres, int* inner_total, int verbose);
  // dL/da_ij = -lambda_i x_j for the finest matrix's nonzeros (CSR order).
  void nz_gradient(const double* x, const double* lam, double* grad);
  // Block PCG: k <= 32 right-hand sides at once, X and B row-major n x k
  // on the device (column c of row i at i*k + c).  One pass over each level
  // matrix per block product serves all k columns; per-column scalars, a
  // column stops changing once it has converged.  iters[k] and relres[k]
  // (host, may be null) receive each column's iterations and final relative
  // residual.  Returns the largest iteration count.
  int pcg_block(double* X, const double* B, int k, const CycleOpts& o, double tol, int maxiter, bool mixed,
                int* iters, double* relres, int verbose);

  // r = b - A x on the finest level and ||r||_2 (device vectors).
  double residual_norm(const double* x, const double* b, double* r);

  // Numeric resetup on the fixed structure; values of the finest matrix on
  // the device (nnz0 entries).
  void resetup_values(const double* v_dev);

  // Single operations on one level for kernel-level parity tests (device
  // pointers; precision 0 = FP64, 1 = FP32 buffers converted in/out).
  void level_op(int lvl, int op, bool fp32, const double* in1, const double* in2, double* out,
                int steps);
  float time_level_op(int lvl, int op, bool fp32, int reps);

  // Export device values (after a GPU resetup) into host vectors.
  void export_values(int lvl, const std::string& what, std::vector<double>& out) const;
  void export_piv(std::vector<int>& out) const;

  // Scratch host-pointer helpers
  double* xbuf() { return xd_; }
  double* bbuf() { return bd_; }

 private:
  template <typename T> LevelVecs<T>& vecs(int l);
  template <typename T> T* coarse_b();
  template <typename T> T* coarse_x();
  template <typename T> const T* mval(const DevMat& M) const;
  template <typename T> const T* qval(const DevLevel& d) const;
  template <typename T> const T* invd(const DevLevel& L) const;

  // rz_w: when set (finest level only), the last Jacobi sweep also forms
  // r·z with r = rz_w and stores it like the PCG's r·z (rz_first: first
  // application, else shift the previous value to "old").  x1_ready: x
  // already holds the zero-guess Jacobi step (formed by the restriction).
  template <typename T>
  T* cycle_level(int l, T* x, const T* b, bool x_zero, const CycleOpts& o, T* ext_partner,
                 const double* rz_w = nullptr, bool rz_first = false, bool x1_ready = false);
  template <typename T>
  T* smooth(int l, T* x, const T* b, int steps, T* ext_partner, const double* rz_w = nullptr,
            bool rz_first = false);
  bool fused_rz_ok(const CycleOpts& o) const;
  template <typename T>
  void residual(int l, const T* x, const T* b, T* r, double* rr_dst);
  template <typename T>
  void coarse_solve(const T* b, T* x);

  void ensure_fp32();
  void refresh_fp32();
  void build_tail();
  void build_fused(const HostHierarchy& H);
  void build_q(DevLevel& d);  // Q from d.AP.v, d.P.v and d.invd (and its FP32 copy)
  // block (multi-right-hand-side) solves: per-level n x k buffers
  template <typename T>
  struct BlockVecs {
    T *x = nullptr, *t = nullptr, *b = nullptr, *r = nullptr;
  };
  std::vector<BlockVecs<float>> blk32_;
  std::vector<BlockVecs<double>> blk64_;
  int blk_k_ = 0;  // columns the block buffers hold
  float *bcb32_ = nullptr, *bcx32_ = nullptr;
  double *bcb64_ = nullptr, *bcx64_ = nullptr;
  double* bpcg_[4] = {nullptr, nullptr, nullptr, nullptr};  // R, P, Q, Z
  float* bpcg32_[2] = {nullptr, nullptr};                   // R, Z in FP32
  double* bpart_ = nullptr;  // column-dot partial sums
  double* bdev_ = nullptr;   // k-vectors on the device (dot results, alpha, beta)
  double* bhost_ = nullptr;  // their pinned host mirror
  void ensure_block(int k);
  // Launch shapes of the block products, picked by timing (tune_block) per
  // matrix, product mode, precision and k.
  struct ShapeKey {
    const void* rp;
    int mode, bytes, k;
    bool operator<(const ShapeKey& o) const {
      return rp != o.rp ? rp < o.rp : mode != o.mode ? mode < o.mode : bytes != o.bytes ? bytes < o.bytes : k < o.k;
    }
  };
  std::map<ShapeKey, BlockShape> bshape_;
  std::set<std::pair<int, int>> btuned_;  // (k, bytes of the cycle's type) already tuned
  bool btune_on_ = true;                  // DRAUGR_B200_BLOCK_TUNE=0 at a solve: default shapes
  int bforce_tpr_ = 0;                    // DRAUGR_B200_BLOCK_TUNE=2/4/8/16: threads per row forced
  BlockShape shape_of(const void* rp, int mode, int bytes, int k) const;
  template <typename T>
  void tune_block(int k, int verbose);
  template <typename T>
  BlockVecs<T>& bvecs(int l);
  template <typename T>
  T* cycle_block(int l, T* X, const T* B, bool x_zero, const CycleOpts& o, int k);
  void col_dots(int n, int k, const double* a, const double* b, double* dst_dev);
  // transposed hierarchy (adjoint solves)
  bool at_built_ = false;
  bool tr_ = false;          // cycle pieces use A^T (and the transposed coarsest solve)
  void build_transpose();
  void refresh_transpose();
  double* bk_[8] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
  void lin3(int n, double a, const double* x, double b, const double* y, double c, const double* z,
            double* out);
  void precond64(const double* r, double* out, const CycleOpts& o);
  void precond32(const double* r, double* out, const CycleOpts& o);  // FP32 cycle, FP64 in and out
  // batch: layout, its device arrays per merged level (coarse blocks), the
  // finest level's segment offsets and row -> segment map
  std::unique_ptr<BatchLayout> batch_;
  struct BatchDev {
    int nblk = 0, maxn = 0;
    int *off = nullptr, *nb = nullptr, *poff = nullptr;
    long long* luoff = nullptr;
    bool inv = false;  // solved with the explicit inverses (binv_), every n <= 64
  };
  std::vector<BatchDev> batch_dev_;
  double* blu_ = nullptr;
  double* binv_ = nullptr;  // the systems' coarsest inverses, laid out like blu_
  int* bpiv_ = nullptr;
  int *seg_off_ = nullptr, *seg_id_ = nullptr;
  double* seg_buf_ = nullptr;    // per segment: rz, rzold, pq, rr, bb, alpha, beta
  double* seg_part_ = nullptr;   // dot partials
  int* seg_int_ = nullptr;       // per segment: done, iters; then the count of converged segments
  double *sx_ = nullptr, *sr_ = nullptr, *sp_ = nullptr, *sq_ = nullptr, *sz_ = nullptr;
  cudaGraphExec_t seg_graph_ = nullptr;
  long long seg_launches_ = 0;   // kernels in one captured batch iteration
  bool seg_graph_mixed_ = false;
  CycleOpts seg_graph_o_;
  template <typename T>
  void batch_coarse(int l, const T* b, T* x);
  void alloc_transpose_fp32();
  // FGMRES workspace: (restart + 1) basis vectors, restart preconditioned
  // vectors, one work vector, reduction partials and tickets per column.
  int gm_m_ = 0;
  double *gm_V_ = nullptr, *gm_Z_ = nullptr, *gm_w_ = nullptr, *gm_h_ = nullptr, *gm_part_ = nullptr;
  unsigned* gm_tk_ = nullptr;
  double *ir_r_ = nullptr, *ir_d_ = nullptr, *ir_x_ = nullptr;  // iterative refinement: residual, correction, iterate
  void upload_csr(DevMat& M, int n, int m, const std::vector<int>& rp, const std::vector<int>& ci,
                  const std::vector<double>* v);
  template <typename T>
  void spgemm(DevMat& O, const DevMat& S, const DevMat& B, T* ov, const T* sv, const T* bv,
              SpgemmList* list = nullptr);
  bool build_spgemm_list(const DevMat& O, const DevMat& S, const DevMat& B, SpgemmList& list);
  // Levels tail_ .. nlevels-1 run as one single-block kernel (k_coarse_tail);
  // tail_ = nlevels() when no level qualifies.
  int tail_ = 0;
  int resetup_fp64_ = -1;  // see set_resetup_fp64_levels
  void* tail64_ = nullptr;   // device TailLevel<double>[nlevels - tail_]
  void* tail32_ = nullptr;   // device TailLevel<float>[...] once FP32 buffers exist
  size_t tail_bytes_[2] = {0, 0};        // shared memory of the tail kernel (FP64, FP32)
  struct TailCopyList {  // its prologue's bulk copies (kern::TailCopies)
    const void* list = nullptr;
    int npat = 0, nval = 0;
    unsigned pat_bytes = 0, val_bytes = 0;
    const void* xsrc = nullptr;
    unsigned xoff = 0, xbytes = 0;
  } tail_cp_[2];
  unsigned tail_co_[2][4] = {{0}, {0}};  // its coarsest-system offsets (TailCoarse)
  void graphs_clear();
  double dot_host(const double* a, const double* b, int n);

  int device_ = 0;
  cudaStream_t st_ = nullptr;       // stream in use
  cudaStream_t own_st_ = nullptr;   // stream created by the library
  bool own_stream_ = false;
  int n0_ = 0;
  long long nnz0_ = 0;
  int nsm_ = 148;
  int max_grid_ = 148 * 8;
  std::vector<DevLevel> L_;
  DevMat C_;                 // coarsest CSR (pattern + values)
  int nc_ = 0;
  double* cdense_ = nullptr;
  double* clu_ = nullptr;
  int* cpiv_ = nullptr;
  // the coarsest system's explicit inverse, which the shared-memory tail
  // and the block cycle apply instead of the substitutions when the cycle
  // is not bit-exact anyway (some level sums its rows in a tree)
  double* cinv_ = nullptr;
  bool cinv_ok_ = false;   // cinv_ is kept (such a hierarchy, n_c <= 64)
  bool tail_inv_ = false;  // the tail applies it (n_c <= 32)
  void build_cinv();
  int* info_ = nullptr;
  double *cb64_ = nullptr, *cx64_ = nullptr;
  float *cb32_ = nullptr, *cx32_ = nullptr;
  bool fp32_ = false;
  // reductions: partial sums, tickets, scalars
  double* partials_ = nullptr;
  unsigned* tickets_ = nullptr;
  double* scal_ = nullptr;     // [0] bb [1] rr [2] rz [3] rz_old [4] pq [5] tmp
  double* hscal_ = nullptr;    // pinned host mirror
  // host-pointer staging and PCG workspace
  double *xd_ = nullptr, *bd_ = nullptr;
  double *pr_ = nullptr, *pp_[2] = {nullptr, nullptr}, *pq_ = nullptr, *pz_ = nullptr;
  float *pr32_ = nullptr, *pz32_ = nullptr;
  double *tin1_ = nullptr, *tin2_ = nullptr, *tout_ = nullptr;  // level_op staging
  double* tout2_ = nullptr;                                      // time_level_op scratch
  size_t bytes_ = 0;
  std::vector<void*> allocs_;
  template <typename T> T* alloc(size_t n);
  // CUDA graphs of the PCG iteration, keyed by (mixed, parity)
  struct PcgGraphs {
    bool valid = false;
    bool mixed = false;
    CycleOpts o;
    cudaGraphExec_t g1[2] = {nullptr, nullptr};  // direction + update of r
    cudaGraphExec_t g2[2] = {nullptr, nullptr};  // preconditioner + r·z, beside it x += α p
    long long n1[2] = {0, 0}, n2[2] = {0, 0};    // kernels per graph
  } pg_;
  cudaEvent_t ev_[2] = {nullptr, nullptr};
  // a second stream and two events, to fork and join a branch of a graph
  // capture (the PCG iterate update beside the preconditioner)
  cudaStream_t side_st_ = nullptr;
  cudaEvent_t ev_fork_ = nullptr, ev_join_ = nullptr;

  friend struct DevHierAccess;
};

// Value and smoother-diagonal arrays by precision (defined in dr_device.cu).
template <> const double* DevHier::mval<double>(const DevMat& M) const;
template <> const float* DevHier::mval<float>(const DevMat& M) const;
template <> const double* DevHier::qval<double>(const DevLevel& d) const;
template <> const float* DevHier::qval<float>(const DevLevel& d) const;
template <> const double* DevHier::invd<double>(const DevLevel& L) const;
template <> const float* DevHier::invd<float>(const DevLevel& L) const;

}  // namespace dr
