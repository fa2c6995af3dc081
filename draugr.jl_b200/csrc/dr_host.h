// Host-side data structures and setup routines of the B200 AMG library.
//
// All indices are 0-based int32 internally (the C ABI accepts 0- or 1-based
// input and converts once, like csr_from_raw in src/csr_matrix.jl:133-143 of
// Draugr.jl).  The setup phase (strength, coarsening, interpolation, symbolic
// Galerkin product, transpose map, colouring) runs on the CPU and produces the
// hierarchy *structure*; the solve phase and the numeric resetup run on the
// GPU (dr_device.h).
#pragma once

#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

namespace dr {

// ---------------------------------------------------------------------------
// Errors: every C entry point catches dr::Error and stores its message as the
// last error (src/cfunction_interface.jl:18-28).
struct Error : public std::runtime_error {
  explicit Error(const std::string& m) : std::runtime_error(m) {}
};
[[noreturn]] void fail(const std::string& msg);

// ---------------------------------------------------------------------------
// CSR matrix (src/csr_matrix.jl:19-33).  rp has n+1 entries.
struct CSR {
  int n = 0;     // rows
  int m = 0;     // columns
  std::vector<int> rp;
  std::vector<int> ci;
  std::vector<double> v;
  int64_t nnz() const { return (int64_t)ci.size(); }
};

// Prolongation operator P (n_fine x n_coarse), src/types.jl:368-376.
struct Prolong {
  int nf = 0, nc = 0;
  std::vector<int> rp, ci;
  std::vector<double> v;
  bool has_trunc_scaling = false;
  std::vector<double> trunc_scaling;
  int64_t nnz() const { return (int64_t)ci.size(); }
};

// Transpose map of P (src/types.jl:394-398, built by build_transpose_map,
// src/prolongation.jl:767-800): for coarse column J the fine rows with
// P[i,J] != 0 in ascending order and the index of that entry in P.
struct TransposeMap {
  std::vector<int> off;    // nc+1
  std::vector<int> rows;   // nnzP
  std::vector<int> pnz;    // nnzP
};

// ---------------------------------------------------------------------------
// Configuration (src/types.jl:497-536).
enum class InterpKind : int { Direct = 0, Standard = 1, ExtendedI = 2 };
struct Interp {
  InterpKind kind = InterpKind::ExtendedI;
  double trunc_factor = 0.0;
  int max_elements = 0;
  int norm_p = 1;
  bool rescale = false;
};

enum class CoarsenKind : int {
  Aggregation = 0,
  PMIS = 1,
  HMIS = 2,
  RS = 3,
  AggressivePMIS = 4,
  AggressiveHMIS = 5,
  SmoothedAggregation = 6,
};
struct Coarsening {
  CoarsenKind kind = CoarsenKind::HMIS;
  double theta = 0.5;
  Interp interp;
  bool filtering = false;   // aggregation / smoothed aggregation
  double filter_tol = 0.1;
  double sa_omega = 2.0 / 3.0;
};

enum class SmootherKind : int {
  Jacobi = 0,
  ColoredGS = 1,
  SerialGS = 2,
  SPAI0 = 3,
  SPAI1 = 4,
  L1Jacobi = 5,
  L1ColoredGS = 6,
  L1SerialGS = 7,
  Chebyshev = 8,
  ILU0 = 9,
  SerialILU0 = 10,
};

// Smoothers whose sweep is x + (omega d_i)(b - A x)_i with a per-row
// factor d: Jacobi and l1-Jacobi (d = 1/a_ii, 1/sum|a_ij|) and SPAI(0)
// (d = a_ii / sum a_ij^2, omega = 1).
inline bool jacobi_type(SmootherKind k) {
  return k == SmootherKind::Jacobi || k == SmootherKind::L1Jacobi || k == SmootherKind::SPAI0;
}

enum class StrengthKind : int { Absolute = 0, Signed = 1 };

struct Config {
  Coarsening coarsening;            // default HMIS(0.5, ExtendedI())
  Coarsening initial_coarsening;    // defaults to coarsening
  SmootherKind smoother = SmootherKind::L1ColoredGS;
  int max_levels = 20;
  int max_coarse_size = 50;
  int pre_smoothing_steps = 1;
  int post_smoothing_steps = 1;
  double jacobi_omega = 2.0 / 3.0;
  int verbose = 0;
  int initial_coarsening_levels = 0;
  double max_row_sum = 1.0;
  bool cycle_w = false;             // cycle_type :W
  StrengthKind strength = StrengthKind::Absolute;
  bool coarse_solve_on_cpu = false;
  uint64_t seed = 0x5eedULL;        // seeds the PMIS/HMIS random measures
};

Config default_config();
Config config_from_json(const char* json);   // src/cfunction_interface.jl:178-221
Config hypre_default_config(double agg_trunc_factor);
std::string smoother_name(SmootherKind k);
std::string coarsening_name(const Coarsening& c);
// Every field of a parsed configuration as JSON (lower-case type names as
// the parser accepts them; coarsening and initial coarsening as objects).
std::string config_to_json(const Config& c);

// ---------------------------------------------------------------------------
// Hierarchy (host side).  One HostLevel per AMG level (src/types.jl:431-440)
// plus the dense coarsest system (src/types.jl:457-467).
struct HostLevel {
  CSR A;
  Prolong P;
  TransposeMap T;
  // Values of R = P^T in transpose-map order: Rv[k] = P.v[T.pnz[k]].
  std::vector<double> Rv;
  // Symbolic Galerkin data kept for the partial resetup: the sparsity of
  // A*P (rows of the fine level, sorted unique coarse columns).
  bool has_rap_map = false;
  std::vector<int> ap_rp, ap_ci;
  // Smoother.
  SmootherKind smoother = SmootherKind::Jacobi;
  double omega = 2.0 / 3.0;
  std::vector<double> invdiag;
  int num_colors = 0;
  std::vector<int> colors;        // 1-based colours, per row
  std::vector<int> color_off;     // num_colors+1, 0-based offsets
  std::vector<int> color_order;   // rows sorted by colour
  // Chebyshev (src/smoothers.jl:860-1003): the normalised start vector of
  // the power iteration for the spectral radius of D^-1 A (seeded; the
  // reference draws an unseeded randn), the estimate, and the coefficients
  // of the `cheb_degree` inner steps: cheb_coef[0] = 1/theta, then
  // (scale_r, scale_d) of steps 1.. at [2j], [2j+1].
  int cheb_degree = 0;
  std::vector<double> cheb_v0;
  double cheb_rho = 0.0;
  std::vector<double> cheb_coef;
  // ILU(0) and serial ILU(0) (src/smoothers.jl:1016-1440): factors on A's
  // pattern (ilu_L: strictly lower part of L, unit diagonal implied;
  // ilu_U: upper part with the diagonal), the diagonal positions, and the
  // level schedules of the two substitutions (rows by level, offsets).
  std::vector<int> ilu_diag;
  std::vector<double> ilu_L, ilu_U;
  std::vector<int> ilu_fwd_order, ilu_fwd_off, ilu_bwd_order, ilu_bwd_off;
  // Serial and l1 serial Gauss-Seidel (src/smoothers.jl:318-491): rows by
  // level of the sweep's dependencies, level offsets.
  std::vector<int> sgs_order, sgs_off;
  // SPAI(1) (src/smoothers.jl:586-760): the approximate inverse M on A's
  // pattern.
  std::vector<double> spai1_M;
  // C/F splitting of the level (1 coarse, -1 fine) for splitting-based
  // coarsening; empty for aggregation.
  std::vector<int> cf;
};

struct HostHierarchy {
  std::vector<HostLevel> levels;
  CSR coarse;                      // coarsest CSR (pattern kept for resetup)
  int nc = 0;                      // coarsest size
  std::vector<double> coarse_dense;   // column-major n_c x n_c
  std::vector<double> coarse_lu;      // LU factors (column-major), getrf layout
  std::vector<int> coarse_piv;        // 0-based pivot rows (getrf ipiv - 1)
  bool allow_partial_resetup = true;
  double setup_seconds = 0.0;
  Config cfg;                      // configuration used at setup
};

// ---------------------------------------------------------------------------
// Setup routines (CPU).  Each cites the reference routine it reproduces.
void validate_csr(const CSR& A, const char* what);
std::vector<uint8_t> strength_absolute(const CSR& A, double theta);
std::vector<uint8_t> strength_signed(const CSR& A, double theta);
CSR apply_max_row_sum(const CSR& A, double threshold);

void coarsen_aggregation(const CSR& A, double theta, std::vector<int>& agg, int& nc);
void coarsen_pmis(const CSR& A, double theta, uint64_t& rng, std::vector<int>& cf,
                  std::vector<int>& cmap, int& nc);
void coarsen_hmis(const CSR& A, double theta, uint64_t& rng, std::vector<int>& cf,
                  std::vector<int>& cmap, int& nc);
// coarsen_rs (coarsening.jl:660-810): classical Ruge-Stueben splitting --
// isolated points coarse, then the greedy first pass over buckets of the
// measure lambda (points strongly depending on each point; the most
// recently bucketed point of the highest bucket first), then every F-point
// given a strong C-neighbour.  Deterministic.
void coarsen_rs(const CSR& A, double theta, std::vector<int>& cf, std::vector<int>& cmap, int& nc);
void coarsen_aggressive_cf(const CSR& A, double theta, bool base_hmis, const Config& cfg,
                           uint64_t& rng, std::vector<int>& cf, std::vector<int>& cmap,
                           int& nc);

Prolong build_aggregation_prolongation(int nf, const std::vector<int>& agg, int nc);
Prolong filter_prolongation(const Prolong& P, double tol);
Prolong truncate_interpolation(const Prolong& P, double tf);
Prolong smooth_prolongation(const CSR& A, const Prolong& Pt, double omega);
Prolong build_interpolation(const CSR& A, const std::vector<int>& cf,
                            const std::vector<int>& cmap, int nc, const Interp& ip,
                            double theta);

TransposeMap build_transpose_map(const Prolong& P);
// Sparsity of A*P (sorted unique coarse columns per fine row).
void symbolic_ap(const CSR& A, const Prolong& P, std::vector<int>& ap_rp,
                 std::vector<int>& ap_ci);
// Sparsity of P^T*(A*P) given the transpose map.
void symbolic_ptap(const TransposeMap& T, int nc, const std::vector<int>& ap_rp,
                   const std::vector<int>& ap_ci, std::vector<int>& c_rp,
                   std::vector<int>& c_ci);
// Numeric two-phase Galerkin product on fixed patterns.  Accumulation order
// per output entry: phase 1 in (A entry, P entry) order, phase 2 in transpose
// map order; the GPU resetup kernels use the same order.
void numeric_ap(const CSR& A, const Prolong& P, const std::vector<int>& ap_rp,
                const std::vector<int>& ap_ci, std::vector<double>& ap_v);
void numeric_ptap(const TransposeMap& T, const std::vector<double>& Rv,
                  const std::vector<int>& ap_rp, const std::vector<int>& ap_ci,
                  const std::vector<double>& ap_v, const std::vector<int>& c_rp,
                  const std::vector<int>& c_ci, std::vector<double>& c_v);

void greedy_coloring(const CSR& A, std::vector<int>& colors, int& num_colors);
void color_order_from(const std::vector<int>& colors, int num_colors,
                      std::vector<int>& off, std::vector<int>& order);
void inverse_diagonal(const CSR& A, std::vector<double>& invd);     // smoothers.jl:47-63
void l1_inverse_diagonal(const CSR& A, std::vector<double>& invd);  // smoothers.jl:816-827
void spai0_diagonal(const CSR& A, std::vector<double>& m);          // smoothers.jl:524-538
// _estimate_spectral_radius (smoothers.jl:869-887): `niter` power steps on
// D^-1 A from the normalised v (overwritten); returns the last ||w||.
double spectral_radius_estimate(const CSR& A, const std::vector<double>& invd, std::vector<double>& v,
                                int niter);
// Coefficients of one Chebyshev application of `degree` inner steps for the
// spectral-radius estimate rho (the bounds [rho * 1.1 / 30, rho * 1.1] and
// the recurrence of smoothers.jl:895-986); 2 * degree entries.
void chebyshev_coefficients(double rho, int degree, std::vector<double>& coef);
// _ilu0_diag_indices (smoothers.jl:1083-1097); fails on a row without a
// diagonal entry.
void ilu0_diag_indices(const CSR& A, std::vector<int>& diag);
// _ilu0_factorize! (smoothers.jl:1016-1080): sequential, with the
// reference's zero-pivot skip, 1e8 growth clamp and diagonal safeguard.
void ilu0_factorize(const CSR& A, const std::vector<int>& diag, std::vector<double>& L,
                    std::vector<double>& U);
// _compute_ilu_levels (smoothers.jl:1232-1299): rows grouped by level of
// the forward (L) and backward (U) substitutions, in row order within a
// level; offsets are 0-based, levels + 1 entries.
void ilu0_levels(const CSR& A, const std::vector<int>& diag, std::vector<int>& fwd_order,
                 std::vector<int>& fwd_off, std::vector<int>& bwd_order, std::vector<int>& bwd_off);
// Level schedule that reproduces the in-place forward Gauss-Seidel sweep in
// row order: row i follows every j < i with a_ij or a_ji nonzero (it reads
// the new x_j of its lower neighbours, and its upper neighbours must still
// read its old x_i).
void serial_gs_levels(const CSR& A, std::vector<int>& order, std::vector<int>& off);
// _serial_gs_compute_invdiag! (smoothers.jl:329-340): 1/a_ii (the first
// diagonal entry of the row), 0 when |a_ii| <= eps.
void serial_gs_inverse_diagonal(const CSR& A, std::vector<double>& invd);
// _compute_spai1! (smoothers.jl:620-690): per row i, the Gram matrix
// G_pq = sum_r a_r,Jp a_r,Jq over the rows r touching the row's columns J
// (ascending r, as the reference's loop over all rows), the right-hand side
// a_i,J, G_pp += eps max(1, |G_pp|), and G m = rhs (Cholesky, as Julia's
// `\` factorises a symmetric positive definite matrix; partial-pivoting LU
// if that breaks down).  The values of M on A's pattern.
void spai1_values(const CSR& A, std::vector<double>& M);
void csr_to_dense(const CSR& A, std::vector<double>& M);            // setup.jl:495-516
void dense_lu(int n, std::vector<double>& lu, std::vector<int>& piv);

// Optional device implementation of one level's Galerkin products during
// setup: the pattern and values of A·P (ap_*) and of Pᵀ(AP) (next),
// identical to symbolic_ap / numeric_ap / symbolic_ptap / numeric_ptap.
// Returns false to leave them to the host.
struct GalerkinDevice {
  virtual bool galerkin(const CSR& A, const Prolong& P, const TransposeMap& T, const std::vector<double>& Rv,
                        std::vector<int>& ap_rp, std::vector<int>& ap_ci, std::vector<double>& ap_v,
                        CSR& next) = 0;
  virtual ~GalerkinDevice() = default;
};
void build_hierarchy(const CSR& A, const Config& cfg, bool allow_partial_resetup, HostHierarchy& H,
                     GalerkinDevice* gdev = nullptr);
std::string hierarchy_summary(const HostHierarchy& H, int n_finest);

// Random measures: splitmix64-seeded xoshiro-like generator in [0,1).
double rng_uniform(uint64_t& state);

}  // namespace dr
