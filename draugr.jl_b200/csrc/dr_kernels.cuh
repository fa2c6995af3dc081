// sm_100a kernels of the AMG solve and resetup hot path.
//
// Row kernels use a group of G lanes per CSR row (G a power of two chosen
// per matrix from its mean row length): the G lanes read G consecutive
// (column, value) pairs per step, so a warp streams 32 consecutive entries
// of the value and index arrays, and the group sum is a fixed shuffle tree.
// Rows are walked with a warp-uniform grid-stride loop so every lane of a
// warp takes part in every shuffle.  Epilogue functors fuse what follows the
// product in the reference (residual, Jacobi update, prolongation add,
// Gauss-Seidel update, dot products) into the same pass.
//
// Dot products are deterministic: a fixed grid writes one partial per block,
// and the last block to finish (atomic ticket) sums the partials in index
// order; results do not depend on block scheduling.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace dr {
namespace kern {

constexpr int kBlock = 256;

// ------------------------------------------------------------ reductions
// Sum `v` over the block; result valid in thread 0.
__device__ __forceinline__ double block_sum(double v) {
  __shared__ double ws[32];
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  __syncthreads();  // ws may still be read by a previous call
  if (l == 0) ws[w] = v;
  __syncthreads();
  if (w == 0) {
    const int nw = (blockDim.x + 31) >> 5;
    v = (l < nw) ? ws[l] : 0.0;
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
  }
  return v;
}

// Finalizers applied by the last block to the grand total.
struct FinStore {
  double* dst;
  __device__ void operator()(double s) const { *dst = s; }
};
// Shift: old <- current, current <- s (used for r.z in PCG).
struct FinShift {
  double* cur;
  double* old;
  __device__ void operator()(double s) const {
    *old = *cur;
    *cur = s;
  }
};

// Each block contributes `v`; the last block sums all partials in order and
// applies `fin`.  `ticket` must be zero on entry and is zero again on exit.
template <class Fin>
__device__ __forceinline__ void grid_sum_finalize(double v, double* partials, unsigned* ticket,
                                                  Fin fin) {
  __shared__ bool am_last;
  v = block_sum(v);
  if (threadIdx.x == 0) {
    partials[blockIdx.x] = v;
    __threadfence();
    unsigned t = atomicAdd(ticket, 1u);
    am_last = (t == gridDim.x - 1);
  }
  __syncthreads();
  if (am_last) {
    __threadfence();
    double s = 0.0;
    for (int i = threadIdx.x; i < (int)gridDim.x; i += blockDim.x) s += __ldcg(partials + i);
    s = block_sum(s);
    if (threadIdx.x == 0) {
      fin(s);
      *ticket = 0u;
    }
  }
}

// ------------------------------------------------------------ operand loaders
template <typename T>
struct XPlain {
  const T* __restrict__ x;
  __device__ __forceinline__ T operator()(int j) const { return __ldg(x + j); }
};

// First weighted-Jacobi step from a zero guess: x1_j = 0 + (ω·invd_j)·(b_j - 0)
// (src/smoothers.jl:78-94 with x = 0), evaluated where it is consumed.
template <typename T>
struct XZeroJacobi {
  const T* __restrict__ b;
  const T* __restrict__ invd;
  T omega;
  __device__ __forceinline__ T operator()(int j) const;
};

// PCG search direction on the fly: p_j = z_j + β·p_old_j, with
// β = rz / rz_old read from device memory once per thread (bind()).
template <typename TZ>
struct XPcgDir {
  const TZ* __restrict__ z;
  const double* __restrict__ pold;
  const double* __restrict__ scal;  // [rz, rz_old]
  double beta;
  __device__ __forceinline__ void bind() { beta = __ldg(scal) / __ldg(scal + 1); }
  __device__ __forceinline__ double operator()(int j) const {
    return (double)__ldg(z + j) + beta * __ldg(pold + j);
  }
};
// Loaders without per-launch state.
template <class XL>
__device__ __forceinline__ void bind_loader(XL&) {}
template <typename TZ>
__device__ __forceinline__ void bind_loader(XPcgDir<TZ>& x) { x.bind(); }

// ------------------------------------------------------------ rounding
// Products and sums rounded separately (no contraction into FMA), as the
// reference's Julia loops evaluate them.
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double add_rn(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float add_rn(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ double sub_rn(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ float sub_rn(float a, float b) { return __fsub_rn(a, b); }

template <typename T>
__device__ __forceinline__ T XZeroJacobi<T>::operator()(int j) const {
  return mul_rn(mul_rn(omega, __ldg(invd + j)), __ldg(b + j));
}

// ------------------------------------------------------------ epilogues
// A row of a row kernel is reduced as  acc = init ± a_i1 x_1 ± a_i2 x_2 ...
// (kSign = +1 adds the products, -1 subtracts them) and then apply() writes
// the row's results and returns its contribution to a fused dot product.
// pre(i) loads the row's other operands; the tile kernel issues it before
// its barrier so those loads overlap the streaming of the tile.  With one
// lane per row the products are accumulated in column order, exactly as the
// reference's loops do; with G > 1 lanes they are summed in a fixed tree
// first and then added to (subtracted from) init.
template <typename T>
struct EpStore {  // y = A x                                (csr_matrix.jl:150-159)
  using acc_t = T;
  static constexpr int kSign = 1;
  struct Pre {};
  T* __restrict__ y;
  __device__ __forceinline__ Pre pre(int) const { return {}; }
  __device__ __forceinline__ T init(const Pre&) const { return T(0); }
  __device__ __forceinline__ double apply(int i, T v, const Pre&) const { y[i] = v; return 0.0; }
};

template <typename T>
struct EpResidual {  // Ax = Σ a x ; r = b - Ax                (cycle.jl:32-43)
  using acc_t = T;
  static constexpr int kSign = 1;
  struct Pre { T b; };
  const T* __restrict__ b;
  T* __restrict__ r;
  __device__ __forceinline__ Pre pre(int i) const { return {__ldg(b + i)}; }
  __device__ __forceinline__ T init(const Pre&) const { return T(0); }
  __device__ __forceinline__ double apply(int i, T v, const Pre& p) const {
    T ri = sub_rn(p.b, v);
    r[i] = ri;
    return (double)ri * (double)ri;
  }
};

template <typename T>
struct EpJacobi {  // r = b - a x - ... ; xn = x + (ω·invd)·r   (smoothers.jl:78-94)
  using acc_t = T;
  static constexpr int kSign = -1;
  struct Pre { T x, b, d; double w; };
  const T* __restrict__ x;
  const T* __restrict__ b;
  const T* __restrict__ invd;
  T* __restrict__ xn;
  T omega;
  const double* __restrict__ w;  // optional: returns w_i·xn_i for a fused dot
  __device__ __forceinline__ Pre pre(int i) const {
    return {__ldg(x + i), __ldg(b + i), __ldg(invd + i), w ? __ldg(w + i) : 0.0};
  }
  __device__ __forceinline__ T init(const Pre& p) const { return p.b; }
  __device__ __forceinline__ double apply(int i, T r, const Pre& p) const {
    T v = add_rn(p.x, mul_rn(mul_rn(omega, p.d), r));
    xn[i] = v;
    return p.w * (double)v;
  }
};

template <typename T>
struct EpZeroJacobiResidual {  // x1 = (ω·invd)·b ; r = b - A x1
  using acc_t = T;
  static constexpr int kSign = 1;
  struct Pre { T b, d; };
  const T* __restrict__ b;
  const T* __restrict__ invd;
  T* __restrict__ x1;
  T* __restrict__ r;
  T omega;
  __device__ __forceinline__ Pre pre(int i) const { return {__ldg(b + i), __ldg(invd + i)}; }
  __device__ __forceinline__ T init(const Pre&) const { return T(0); }
  __device__ __forceinline__ double apply(int i, T v, const Pre& p) const {
    x1[i] = mul_rn(mul_rn(omega, p.d), p.b);
    r[i] = sub_rn(p.b, v);
    return 0.0;
  }
};

// Restriction that also starts the coarse level's smoothing: b = Pᵀ r and
// the first weighted-Jacobi step from a zero guess, x1 = (ω·invd)·b, so the
// coarse level's first kernel is a plain residual r = b - A x1 with one
// gather per entry (the same values as XZeroJacobi forms on the fly).
template <typename T>
struct EpStoreZeroJacobi {
  using acc_t = T;
  static constexpr int kSign = 1;
  struct Pre { T d; };
  T* __restrict__ b;
  const T* __restrict__ invd;
  T* __restrict__ x1;
  T omega;
  __device__ __forceinline__ Pre pre(int i) const { return {__ldg(invd + i)}; }
  __device__ __forceinline__ T init(const Pre&) const { return T(0); }
  __device__ __forceinline__ double apply(int i, T v, const Pre& p) const {
    b[i] = v;
    x1[i] = mul_rn(mul_rn(omega, p.d), v);
    return 0.0;
  }
};

template <typename T>
struct EpAddTo {  // x += p xc, per entry                  (prolongation.jl:742-760)
  using acc_t = T;
  static constexpr int kSign = 1;
  struct Pre { T x; };
  T* __restrict__ x;
  __device__ __forceinline__ Pre pre(int i) const { return {x[i]}; }
  __device__ __forceinline__ T init(const Pre& p) const { return p.x; }
  __device__ __forceinline__ double apply(int i, T v, const Pre&) const { x[i] = v; return 0.0; }
};

// Prolongation, correction and the first weighted-Jacobi post-smoothing
// step in one pass.  With r = b - A x the residual of the iterate before the
// correction (formed on the way down), the reference's two steps
//   x' = x + P xc,  x_new = x' + (ω·invd)·(b - A x')
// equal  x_new = x + (ω·invd)·r + Q xc  with  Q = P - ω·D⁻¹·(A P)
// (src/prolongation.jl:742-760 then src/smoothers.jl:78-94, regrouped), so
// the row kernel runs over Q (the pattern of A·P) and gathers only the
// coarse vector.  x is updated in place: row i reads and writes only x_i.
template <typename T>
struct EpCorrectJacobi {
  using acc_t = T;
  static constexpr int kSign = 1;
  struct Pre { T base; };
  T* __restrict__ x;
  const T* __restrict__ r;
  const T* __restrict__ invd;
  T omega;
  __device__ __forceinline__ Pre pre(int i) const {
    return {add_rn(x[i], mul_rn(mul_rn(omega, __ldg(invd + i)), __ldg(r + i)))};
  }
  __device__ __forceinline__ T init(const Pre& p) const { return p.base; }
  __device__ __forceinline__ double apply(int i, T v, const Pre&) const { x[i] = v; return 0.0; }
};

template <typename T>
struct EpPcgDir {  // q = A p, p_new = z + β p_old, returns p_new·q
  using acc_t = double;
  static constexpr int kSign = 1;
  struct Pre { double p; };
  XPcgDir<T> dir;
  double* __restrict__ pnew;
  double* __restrict__ q;
  __device__ __forceinline__ void bind() { dir.bind(); }
  __device__ __forceinline__ Pre pre(int i) const { return {dir(i)}; }
  __device__ __forceinline__ double init(const Pre&) const { return 0.0; }
  __device__ __forceinline__ double apply(int i, double s, const Pre& pr) const {
    pnew[i] = pr.p;
    q[i] = s;
    return pr.p * s;
  }
};

// One inner step j of a Chebyshev application (src/smoothers.jl:947-986,
// residual_kernel_smoother! :988-999): Ax = sum a x from zero, r = b - Ax,
// then j = 0: d = (invd r) c0 with c0 = 1/theta; j > 0: d = (c0 invd) r +
// c1 d with (c0, c1) = (scale_r, scale_d) of step j; xn = x + d.  The
// coefficients are read from device memory once per thread (bind()), so a
// resetup can recompute them on the device.
template <typename T>
struct EpCheby {
  using acc_t = T;
  static constexpr int kSign = 1;
  struct Pre { T x, b, di, d; };
  const T* __restrict__ x;
  const T* __restrict__ b;
  const T* __restrict__ invd;
  T* d;
  T* __restrict__ xn;
  const double* __restrict__ coef;
  int j;
  T c0, c1;
  __device__ __forceinline__ void bind() {
    c0 = (T)__ldg(coef + 2 * j);
    c1 = j ? (T)__ldg(coef + 2 * j + 1) : T(0);
  }
  __device__ __forceinline__ Pre pre(int i) const {
    return {__ldg(x + i), __ldg(b + i), __ldg(invd + i), j ? d[i] : T(0)};
  }
  __device__ __forceinline__ T init(const Pre&) const { return T(0); }
  __device__ __forceinline__ double apply(int i, T v, const Pre& p) const {
    const T r = sub_rn(p.b, v);
    const T dn = j == 0 ? mul_rn(mul_rn(p.di, r), c0)
                        : add_rn(mul_rn(mul_rn(c0, p.di), r), mul_rn(c1, p.d));
    d[i] = dn;
    xn[i] = add_rn(p.x, dn);
    return 0.0;
  }
};

// The two passes of a SPAI(1) step (src/smoothers.jl:709-760): r = b -
// a_i1 x_1 - ... (from b, in column order), then x_i += (M_i1 r_1 + ...)
// (the sum formed from zero, then added).
template <typename T>
struct EpResidualSub {
  using acc_t = T;
  static constexpr int kSign = -1;
  struct Pre { T b; };
  const T* __restrict__ b;
  T* __restrict__ r;
  __device__ __forceinline__ Pre pre(int i) const { return {__ldg(b + i)}; }
  __device__ __forceinline__ T init(const Pre& p) const { return p.b; }
  __device__ __forceinline__ double apply(int i, T v, const Pre&) const { r[i] = v; return 0.0; }
};

template <typename T>
struct EpAddSum {
  using acc_t = T;
  static constexpr int kSign = 1;
  struct Pre { T x; };
  T* __restrict__ x;
  __device__ __forceinline__ Pre pre(int i) const { return {x[i]}; }
  __device__ __forceinline__ T init(const Pre&) const { return T(0); }
  __device__ __forceinline__ double apply(int i, T v, const Pre& p) const { x[i] = add_rn(p.x, v); return 0.0; }
};

// One power step of the spectral-radius estimate of D^-1 A
// (src/smoothers.jl:876-880): w = (A v) invd, returning w_i^2 for ||w||.
struct EpPowerStep {
  using acc_t = double;
  static constexpr int kSign = 1;
  struct Pre { double di; };
  const double* __restrict__ invd;
  double* __restrict__ w;
  __device__ __forceinline__ Pre pre(int i) const { return {__ldg(invd + i)}; }
  __device__ __forceinline__ double init(const Pre&) const { return 0.0; }
  __device__ __forceinline__ double apply(int i, double s, const Pre& p) const {
    const double wi = mul_rn(s, p.di);
    w[i] = wi;
    return mul_rn(wi, wi);
  }
};

// Warp barrier among the lanes executing together at this point: placed
// between a batch of independent gathers and their first use, it makes the
// compiler issue the whole batch first (without it, gathers whose indices
// come from shared memory are scheduled next to their uses, a few in flight
// at a time).  Every lane of the mask reaches it (no branch in between).
__device__ __forceinline__ void issue_fence() { __syncwarp(__activemask()); }

// ------------------------------------------------------------ dependent launch
// Kernels launched with programmatic stream serialization may start while
// the previous kernel in the stream is still running.  Before pdl_wait()
// such a kernel touches only what no kernel writes (sparsity patterns, tile
// bounds); pdl_wait() returns once the previous grid has completed and its
// writes are visible.  pdl_trigger() lets the next kernel launch early.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" :::); }

// ------------------------------------------------------------ TMA / mbarrier
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void fence_proxy_async() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Bounded wait: gives up after `limit` polls (each poll itself blocks for a
// hardware-defined time) and reports it; never spins forever.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity, int limit) {
  for (int i = 0; i < limit; ++i)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}
// 1-D bulk copy global -> shared (TMA engine), completion counted on `bar`.
// dst and src 16-byte aligned, bytes a multiple of 16.
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

// ------------------------------------------------------------ row kernel
// Rows are packed (on the host, once per matrix) into tiles of at most
// NT/G consecutive rows holding at most kTileCap nonzeros whose columns
// span fewer than 65536 indices; tp[t] is the first row, ts[t] the first
// nonzero and tb[t] the smallest column of tile t.  The columns are stored
// a second time as 16-bit offsets from their tile's smallest column (cu),
// which is what the kernel streams: 2 bytes per entry instead of 4.  A row
// that alone spans 65536 or more columns, or holds more than kTileCap
// entries, forms a tile of its own (tb = -1 marks the wide case) that is
// read from the 32-bit columns in global memory.
//
// Each block walks the tiles blockIdx.x, +gridDim.x, ... with two
// shared-memory stages: while it works on one tile, the TMA engine copies
// the column-offset and value arrays of the tile after next into the other
// stage (cp.async.bulk completing on an mbarrier), so HBM streaming never
// waits on the SM.  The row's other operands (row bounds, epilogue inputs)
// are loaded one tile ahead into registers.  Two ways to form the products
// a_ij·x_j (x is L2-resident):
//   row-gather (FLAT = false): G lanes per row gather their entries of the
//     row, B at once with one lane per row (8 for short rows; 32 with
//     128-thread blocks for rows of 12-32 entries, so that one L2 round trip
//     covers a row and the freed registers keep the same blocks resident),
//     12 (or 4 when a few rows are much longer) per lane with G > 1;
//   flat (FLAT = true, one row per thread): the whole block walks the tile's
//     nonzeros flat, so a long row among short ones costs no more than its
//     share (rows of very uneven length, e.g. the restriction Pᵀ).
// With one lane per row (ORDERED) a row is summed by one thread in column
// order — the reference's order, with products and sums rounded separately —
// so it is reproduced bit for bit.  With G > 1 lanes a row is summed by its
// lanes and a fixed shuffle tree (deterministic, not the reference's order).
// Rows read from global memory are summed by one thread in column order
// when ORDERED and no longer than kTileCap, else by the block in a fixed
// tree.  The offset and value arrays carry padding so the 16-byte-rounded
// copies stay in bounds.
constexpr int kTileCap = 2000;
constexpr int kStageEntries = 2008;  // kTileCap + alignment slack, a multiple of 8 entries
constexpr int kWaitLimit = 1 << 22;

// Dynamic shared memory of k_tile_rows: two stages of columns (TC: int, or
// uint16_t offsets) and values, 47 KB for FP64 values (under the 48 KB that
// needs no opt-in).  Sized for int columns whatever TC is: every row kernel
// of one value type then asks for the same shared memory, so consecutive
// kernels run in the same L1 / shared-memory split (kernels of different
// sizes interleaved in a cycle cost 1-3% of the solve time in SM
// reconfiguration and lost launch overlap).
template <typename TA, typename TC>
constexpr size_t tile_smem_bytes() {
  return 2 * (size_t)kStageEntries * (sizeof(int) + sizeof(TA));
}

template <class EP>
__device__ __forceinline__ void bind_epilogue(EP&) {}
template <typename T>
__device__ __forceinline__ void bind_epilogue(EpPcgDir<T>& e) { e.bind(); }
template <typename T>
__device__ __forceinline__ void bind_epilogue(EpCheby<T>& e) { e.bind(); }

// Resident blocks per SM the register allocation plans for: planning for 4
// lets 128-thread FP64 blocks keep a whole batch of 32 gathers in registers
// without spilling; 2 blocks of 512 threads (short rows, batches of 4).
template <int NT, typename TA>
constexpr int tile_min_blocks() {
  return NT == 128 ? (sizeof(TA) == 8 ? 4 : 5) : NT == 512 ? 2 : 1;
}

// TC: the staged column type — int (the columns themselves) or uint16_t
// (offsets from the tile's smallest column, from cu).  One lane per row
// reads its row's columns at a row stride, where 16-bit entries would
// collide on shared-memory banks; the other forms read consecutive entries.
template <bool FLAT, int G, bool ORDERED, int NT, int B, typename TA, typename TC, class XL, class EP,
          bool DOT, class Fin>
__global__ void __launch_bounds__(NT, (tile_min_blocks<NT, TA>()))
k_tile_rows(int ntiles, const int* __restrict__ tp, const int* __restrict__ ts,
            const int* __restrict__ tb, const int* __restrict__ rp, const int* __restrict__ ci,
            const uint16_t* __restrict__ cu, const TA* __restrict__ av, XL xl, EP ep,
            double* partials, unsigned* ticket, Fin fin, int* err, int wait_limit) {
  constexpr bool kOff = sizeof(TC) == 2;
  constexpr int kColAlign = 16 / (int)sizeof(TC);  // entries per 16 bytes
  const TC* const csrc = kOff ? reinterpret_cast<const TC*>(cu) : reinterpret_cast<const TC*>(ci);
  using acc_t = typename EP::acc_t;
  static_assert(sizeof(acc_t) == sizeof(TA), "flat products are stored over the staged values");
  static_assert(!FLAT || G == 1, "the flat form uses one row per thread");
  static_assert(!ORDERED || G == 1, "ordered sums use one lane per row");
  constexpr int kFlatIters = (kTileCap + NT - 1) / NT;
  using Pre = typename EP::Pre;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  // stage b: values at sv0 + b*kStageEntries, columns at sc0 + b*kStageEntries
  TA* const sv0 = reinterpret_cast<TA*>(smem_raw);
  TC* const sc0 = reinterpret_cast<TC*>(sv0 + 2 * kStageEntries);
  __shared__ __align__(8) uint64_t bar[2];
  __shared__ acc_t red[32];
  const int stride = gridDim.x;
  const int lane = threadIdx.x & (G - 1);
  const int grp = threadIdx.x / G;

  // A tile's bounds, and one thread's row bounds and epilogue operands in it.
  struct Head {
    int r0, r1, s, e, cb;  // cb: smallest column, -1 for a tile read from global memory
  };
  struct Ctx {
    int rs, re;
    bool valid;
    Pre pr;
  };
  auto head = [&](int t) -> Head {
    if (t >= ntiles) return Head{0, 0, 0, 0, 0};
    return Head{__ldg(tp + t), __ldg(tp + t + 1), __ldg(ts + t), __ldg(ts + t + 1),
                kOff ? __ldg(tb + t) : 0};
  };
  auto staged = [](const Head& h) { return (!kOff || h.cb >= 0) && h.e - h.s <= kTileCap; };
  auto ctx_rows = [&](const Head& h) -> Ctx {  // pattern only
    Ctx c{0, 0, false, Pre{}};
    const int row = h.r0 + grp;
    c.valid = staged(h) && row < h.r1;
    if (c.valid) {
      c.rs = __ldg(rp + row) - h.s;
      c.re = __ldg(rp + row + 1) - h.s;
    }
    return c;
  };
  auto ctx = [&](const Head& h) -> Ctx {
    Ctx c = ctx_rows(h);
    if (c.valid && lane == 0) c.pr = ep.pre(h.r0 + grp);
    return c;
  };
  // Stage a tile: the offset copy (and the expected byte count of both
  // copies) and the value copy are issued separately, so the offsets can be
  // requested before the previous kernel has finished.  Thread 0 only.
  // Copies start on 16-byte boundaries: kColAlign columns, 4 values.
  auto issue_cols = [&](const Head& h, int b) {
    if (!staged(h)) {
      mbar_arrive(bar + b);  // read from global memory: nothing to stage
      return;
    }
    const int sc = h.s & ~(kColAlign - 1), sv = h.s & ~3;
    const uint32_t cb = ((uint32_t)(h.e - sc) * (uint32_t)sizeof(TC) + 15u) & ~15u;
    const uint32_t vb = ((uint32_t)(h.e - sv) * (uint32_t)sizeof(TA) + 15u) & ~15u;
    mbar_expect_tx(bar + b, cb + vb);
    bulk_g2s(sc0 + b * kStageEntries, csrc + sc, cb, bar + b);
  };
  auto issue_vals = [&](const Head& h, int b) {
    if (!staged(h)) return;
    const int sv = h.s & ~3;
    const uint32_t vb = ((uint32_t)(h.e - sv) * (uint32_t)sizeof(TA) + 15u) & ~15u;
    bulk_g2s(sv0 + b * kStageEntries, av + sv, vb, bar + b);
  };
  auto issue = [&](const Head& h, int b) {
    issue_cols(h, b);
    issue_vals(h, b);
  };

  if (threadIdx.x == 0) {
    mbar_init(bar + 0, 1);
    mbar_init(bar + 1, 1);
    fence_mbar_init();
  }
  __syncthreads();
  // Software pipeline: while tile t is reduced, the TMA engine streams the
  // offsets and values of tile t + stride (issued one tile earlier), this
  // thread's row bounds and epilogue operands of tile t + stride are in
  // flight to registers, and so are the bounds of tile t + 2 stride.  What
  // is left on a tile's critical path is the L2 gather of x.
  // Up to pdl_wait() only the pattern is read (it never changes).
  Head h0 = head(blockIdx.x), h1 = head(blockIdx.x + stride);
  if (threadIdx.x == 0) {
    if (blockIdx.x < ntiles) issue_cols(h0, 0);
    if (blockIdx.x + stride < ntiles) issue_cols(h1, 1);
  }
  Ctx c0 = ctx_rows(h0);
  pdl_trigger();
  pdl_wait();
  bind_loader(xl);
  bind_epilogue(ep);
  if (threadIdx.x == 0) {
    if (blockIdx.x < ntiles) issue_vals(h0, 0);
    if (blockIdx.x + stride < ntiles) issue_vals(h1, 1);
  }
  if (c0.valid && lane == 0) c0.pr = ep.pre(h0.r0 + grp);

  double dacc = 0.0;
  int i = 0;
  for (int t = blockIdx.x; t < ntiles; t += stride, ++i) {
    const int b = i & 1;
    const uint32_t parity = (uint32_t)((i >> 1) & 1);
    const Head h2 = head(t + 2 * stride);
    const Ctx c1 = ctx(h1);
    const int r0 = h0.r0, s = h0.s, e = h0.e;
    const int len = e - s;
    const int row = r0 + grp;
    const bool valid = c0.valid;
    const int rs = c0.rs, re = c0.re;
    const Pre& pr = c0.pr;
    // A thread whose wait for the stage gives up reads nothing from it (its
    // rows are skipped); the block leaves the loop together at the barrier
    // that ends the tile.
    const bool ok = mbar_wait_bounded(bar + b, parity, wait_limit);
    if (staged(h0)) {
      TA* vs = sv0 + b * kStageEntries + (s - (s & ~3));
      const TC* cs = sc0 + b * kStageEntries + (s - (s & ~(kColAlign - 1)));
      const int cb = h0.cb;
      if constexpr (FLAT) {
        if (ok && len > 0) {
          // slots past the tile's end repeat its last entry (in bounds)
          acc_t p[kFlatIters];
#pragma unroll
          for (int j = 0; j < kFlatIters; ++j) {
            const int k = min((int)threadIdx.x + j * NT, len - 1);
            p[j] = (acc_t)xl(cb + (int)cs[k]);
          }
          issue_fence();
#pragma unroll
          for (int j = 0; j < kFlatIters; ++j) {
            const int k = threadIdx.x + j * NT;
            if (k < len) vs[k] = (TA)mul_rn((acc_t)vs[k], p[j]);
          }
        }
        __syncthreads();
        if (valid && ok) {
          acc_t a = ep.init(pr);
          for (int k = rs; k < re; ++k) {
            if constexpr (EP::kSign > 0) a = add_rn(a, (acc_t)vs[k]);
            else a = sub_rn(a, (acc_t)vs[k]);
          }
          dacc += ep.apply(row, a, pr);
        }
      } else if constexpr (G == 1) {
        if (valid && ok) {
          acc_t a = ep.init(pr);
          for (int k0 = rs; k0 < re; k0 += B) {
            // all B gathers issued unconditionally (slots past the row end
            // repeat its last column, in bounds), then the ordered sum
            acc_t xv[B];
#pragma unroll
            for (int j = 0; j < B; ++j) xv[j] = (acc_t)xl(cb + (int)cs[min(k0 + j, re - 1)]);
            issue_fence();
#pragma unroll
            for (int j = 0; j < B; ++j)
              if (k0 + j < re) {
                const acc_t p = mul_rn((acc_t)vs[k0 + j], xv[j]);
                if constexpr (EP::kSign > 0) a = add_rn(a, p);
                else a = sub_rn(a, p);
              }
          }
          dacc += ep.apply(row, a, pr);
        }
      } else {
        // longer rows: G lanes sum strided products, then a fixed shuffle tree
        acc_t sum = acc_t(0);
        const int rend = ok ? re : rs;
        for (int k0 = rs + lane; k0 < rend; k0 += B * G) {
          acc_t xv[B];
#pragma unroll
          for (int j = 0; j < B; ++j) xv[j] = (acc_t)xl(cb + (int)cs[min(k0 + j * G, re - 1)]);
          issue_fence();
#pragma unroll
          for (int j = 0; j < B; ++j) {
            const int k = k0 + j * G;
            if (k < re) sum = add_rn(sum, mul_rn((acc_t)vs[k], xv[j]));
          }
        }
#pragma unroll
        for (int o = G >> 1; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
        if (valid && ok && lane == 0) {
          acc_t a = ep.init(pr);
          if constexpr (EP::kSign > 0) a = add_rn(a, sum);
          else a = sub_rn(a, sum);
          dacc += ep.apply(row, a, pr);
        }
      }
    } else if (ORDERED && len <= kTileCap) {
      // a single wide row, from global memory, summed by one thread in order
      if (threadIdx.x == 0) {
        const Pre p0 = ep.pre(r0);
        acc_t a = ep.init(p0);
        for (int k = s; k < e; ++k) {
          const acc_t p = mul_rn((acc_t)__ldg(av + k), (acc_t)xl(__ldg(ci + k)));
          if constexpr (EP::kSign > 0) a = add_rn(a, p);
          else a = sub_rn(a, p);
        }
        dacc += ep.apply(r0, a, p0);
      }
    } else {
      // a single row longer than the tile capacity (or wide, in a form that
      // sums in a tree), from global memory, reduced by the block
      acc_t sum = acc_t(0);
      for (int k = s + threadIdx.x; k < e; k += NT)
        sum = add_rn(sum, mul_rn((acc_t)__ldg(av + k), (acc_t)xl(__ldg(ci + k))));
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
      if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = sum;
      __syncthreads();
      if (threadIdx.x < 32) {
        sum = threadIdx.x < (NT >> 5) ? red[threadIdx.x] : acc_t(0);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
        if (threadIdx.x == 0) {
          const Pre p0 = ep.pre(r0);
          acc_t a = ep.init(p0);
          if constexpr (EP::kSign > 0) a = add_rn(a, sum);
          else a = sub_rn(a, sum);
          dacc += ep.apply(r0, a, p0);
        }
      }
    }
    // stage b fully consumed; block-uniform abort if any thread gave up
    if (__syncthreads_or(!ok)) {
      // Flag the error, let the copies in flight land (stage b, and stage
      // 1-b if the next tile was issued) with bounded waits, and leave the
      // loop; the reduction below still completes, so its ticket is reset.
      if (threadIdx.x == 0) {
        atomicExch(err, 1);
        mbar_wait_bounded(bar + b, parity, kWaitLimit);
        if (t + stride < ntiles) mbar_wait_bounded(bar + (b ^ 1), (uint32_t)(((i + 1) >> 1) & 1), kWaitLimit);
      }
      __syncthreads();
      break;
    }
    if (threadIdx.x == 0 && t + 2 * stride < ntiles) {
      fence_proxy_async();
      issue(h2, b);
    }
    h0 = h1;
    h1 = h2;
    c0 = c1;
  }
  if constexpr (DOT) grid_sum_finalize(dacc, partials, ticket, fin);
}

// Gauss-Seidel update of one colour: rows taken from `order`.
// x_i += invd_i·(b_i - A_i x)                 (src/smoothers.jl:203-217)
template <int G, typename T>
__global__ void __launch_bounds__(kBlock)
k_gs_color(int cnt, const int* __restrict__ order, const int* __restrict__ rp,
           const int* __restrict__ ci, const T* __restrict__ av, const T* __restrict__ b,
           const T* __restrict__ invd, T* x) {
  constexpr int RPW = 32 / G;
  const int lane = threadIdx.x & (G - 1);
  const int g = (threadIdx.x & 31) / G;
  const long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
  for (long long base = warp * RPW; base < cnt; base += nwarps * RPW) {
    const int idx = (int)(base + g);
    const bool valid = idx < cnt;
    int row = 0, s = 0, e = 0;
    if (valid) {
      row = __ldg(order + idx);
      s = __ldg(rp + row);
      e = __ldg(rp + row + 1);
    }
    T sum = T(0);
    // x of the same colour is never a neighbour, so plain loads are safe
    for (int k = s + lane; k < e; k += G) sum += __ldg(av + k) * x[__ldg(ci + k)];
#pragma unroll
    for (int off = G >> 1; off > 0; off >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, off);
    if (valid && lane == 0) x[row] += __ldg(invd + row) * (__ldg(b + row) - sum);
  }
}

// ------------------------------------------------------------ vector kernels
template <typename T>
__global__ void k_scale_jacobi_zero(int n, const T* __restrict__ b, const T* __restrict__ invd,
                                    T omega, T* __restrict__ x) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    x[i] = (omega * invd[i]) * b[i];
}

template <typename T>
__global__ void k_fill(long long n, T v, T* __restrict__ x) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    x[i] = v;
}

template <typename TS, typename TD>
__global__ void k_convert(long long n, const TS* __restrict__ s, TD* __restrict__ d) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    d[i] = (TD)s[i];
}

// out = a x + b y + c z (out may be x, y or z; z may be null when c = 0)
__global__ void k_lin3(int n, double a, const double* x, double b, const double* y, double c,
                       const double* z, double* out) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double v = a * x[i] + b * y[i];
    if (z) v += c * z[i];
    out[i] = v;
  }
}

// Gradient of a loss L(x), x = A^-1 b, with respect to the nonzeros of A,
// given the adjoint lambda = A^-T dL/dx:  dL/da_ij = -lambda_i x_j, in CSR
// order.
// Q = P - (ω·invd_i)·(A P) on the pattern of A P (see EpCorrectJacobi):
// q_k = -(ω·invd_i)·ap_k over row i, then each P entry added at its
// position pos[p] in that row: q = p - (ω·invd)·ap, rounded once each.
// One warp per row (the row's P entries have distinct positions).
__global__ void __launch_bounds__(kBlock)
k_build_q(int n, const int* __restrict__ ap_rp, const double* __restrict__ ap_v,
          const double* __restrict__ invd, double omega, const int* __restrict__ p_rp,
          const double* __restrict__ p_v, const int* __restrict__ pos, double* __restrict__ q) {
  const int lane = threadIdx.x & 31;
  const long long w0 = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
  for (long long i = w0; i < n; i += nw) {
    const double w = __dmul_rn(omega, invd[i]);
    for (int k = ap_rp[i] + lane; k < ap_rp[i + 1]; k += 32) q[k] = -__dmul_rn(w, ap_v[k]);
    __syncwarp();
    for (int t = p_rp[i] + lane; t < p_rp[i + 1]; t += 32) q[pos[t]] = __dadd_rn(q[pos[t]], p_v[t]);
    __syncwarp();
  }
}

__global__ void k_nz_grad(int n, const int* __restrict__ rp, const int* __restrict__ ci,
                          const double* __restrict__ x, const double* __restrict__ lam,
                          double* __restrict__ grad) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double li = lam[i];
    for (int k = rp[i]; k < rp[i + 1]; ++k) grad[k] = -li * x[ci[k]];
  }
}

// dst[k] = src[perm[k]] (values of a transposed matrix from the original's)
__global__ void k_gather_vals(long long cnt, const int* __restrict__ perm, const double* __restrict__ src,
                              double* __restrict__ dst) {
  for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < cnt;
       k += (long long)gridDim.x * blockDim.x)
    dst[k] = src[perm[k]];
}

// dot(a, b) with deterministic finalize
template <typename TA, typename TB, class Fin>
__global__ void __launch_bounds__(kBlock)
k_dot(int n, const TA* __restrict__ a, const TB* __restrict__ b, double* partials, unsigned* ticket,
      Fin fin) {
  double s = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    s += (double)a[i] * (double)b[i];
  grid_sum_finalize(s, partials, ticket, fin);
}

// Krylov basis products for FGMRES (columns of V at stride ld):
//   k_mdot:  h_j = v_j · w for j < k; blockIdx.y = j, per-block partials,
//            the last block of column j sums them in block order
//            (deterministic);
//   k_maxpy: w += sign · Σ_j h_j v_j, the coefficients read once per block.
__global__ void __launch_bounds__(kBlock)
k_mdot(int n, const double* __restrict__ V, long long ld, const double* __restrict__ w, double* partials,
       unsigned* tickets, double* h) {
  const int j = blockIdx.y;
  const double* __restrict__ v = V + (long long)j * ld;
  double s = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    s = fma(v[i], w[i], s);
  grid_sum_finalize(s, partials + (size_t)j * gridDim.x, tickets + j, FinStore{h + j});
}

__global__ void __launch_bounds__(kBlock)
k_maxpy(int n, int k, const double* __restrict__ V, long long ld, const double* __restrict__ h, double sign,
        double* __restrict__ w) {
  __shared__ double hs[64];
  for (int j = threadIdx.x; j < k; j += blockDim.x) hs[j] = sign * h[j];
  __syncthreads();
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double s = w[i];
    for (int j = 0; j < k; ++j) s = fma(hs[j], V[(long long)j * ld + i], s);
    w[i] = s;
  }
}

// r -= α q ; rr = r·r ; optional r32 copy; α = rz / pq, also stored at
// alpha_out for k_pcg_x.  With x set it also updates x += α p (one pass);
// with x null the iterate is left to k_pcg_x, which the PCG graph runs
// beside the preconditioner (x is not on the iteration's critical path).
template <typename TR32>
__global__ void __launch_bounds__(kBlock)
k_pcg_update(int n, double* __restrict__ x, double* __restrict__ r, const double* __restrict__ p,
             const double* __restrict__ q, const double* __restrict__ rz, const double* __restrict__ pq,
             TR32* __restrict__ r32, double* alpha_out, double* partials, unsigned* ticket, FinStore fin) {
  pdl_trigger();
  pdl_wait();
  const double alpha = __ldg(rz) / __ldg(pq);
  if (alpha_out && blockIdx.x == 0 && threadIdx.x == 0) *alpha_out = alpha;
  double s = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    if (x) x[i] += alpha * p[i];
    double ri = r[i] - alpha * q[i];
    r[i] = ri;
    if (r32) r32[i] = (TR32)ri;
    s += ri * ri;
  }
  grid_sum_finalize(s, partials, ticket, fin);
}

// x += α p with α from k_pcg_update (the same expression, so the same
// values as the one-pass update).
__global__ void __launch_bounds__(kBlock)
k_pcg_x(int n, double* __restrict__ x, const double* __restrict__ p, const double* __restrict__ alpha_p) {
  const double alpha = __ldg(alpha_p);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    x[i] += alpha * p[i];
}

// ------------------------------------------------------------ coarsest level
// Solve with getrf-style factors (column-major LU, 0-based pivots) in one
// block: row interchanges, unit-lower forward substitution and upper back
// substitution in the column-oriented (axpy) order of LAPACK dgetrs/dtrsv,
// without contraction, so the result equals a sequential CPU solve bit for
// bit.  Input and output in T, arithmetic in double.
template <typename T>
__global__ void k_lu_solve(int n, const double* __restrict__ lu, const int* __restrict__ piv,
                           const T* __restrict__ bin, T* __restrict__ xout, int lu_in_smem) {
  extern __shared__ double sh[];
  double* y = sh;                            // n
  const double* a = lu;                      // factors (global or staged)
  if (lu_in_smem) {
    double* s = sh + ((n + 1) & ~1);
    for (int t = threadIdx.x; t < n * n; t += blockDim.x) s[t] = lu[t];
    a = s;
  }
  for (int i = threadIdx.x; i < n; i += blockDim.x) y[i] = (double)bin[i];
  __syncthreads();
  if (threadIdx.x == 0)
    for (int j = 0; j < n; ++j) {
      int p = piv[j];
      if (p != j) {
        double t = y[j];
        y[j] = y[p];
        y[p] = t;
      }
    }
  __syncthreads();
  for (int j = 0; j < n; ++j) {
    const double yj = y[j];
    if (yj != 0.0)
      for (int i = j + 1 + threadIdx.x; i < n; i += blockDim.x)
        y[i] = __dsub_rn(y[i], __dmul_rn(yj, a[(size_t)j * n + i]));
    __syncthreads();
  }
  for (int j = n - 1; j >= 0; --j) {
    if (threadIdx.x == 0 && y[j] != 0.0) y[j] = __ddiv_rn(y[j], a[(size_t)j * n + j]);
    __syncthreads();
    const double yj = y[j];
    if (yj != 0.0)
      for (int i = threadIdx.x; i < j; i += blockDim.x)
        y[i] = __dsub_rn(y[i], __dmul_rn(yj, a[(size_t)j * n + i]));
    __syncthreads();
  }
  for (int i = threadIdx.x; i < n; i += blockDim.x) xout[i] = (T)y[i];
}

// ------------------------------------------------------------ coarse tail
// The cycle from one small level down to the coarsest, in one block that
// first copies every operand of those levels (matrices, inverse diagonals,
// P and Pᵀ, the LU factors) into shared memory and then runs every phase
// (smoothing, residual, restriction, coarsest solve, prolongation) from
// there: a loop over rows by the block's threads, one thread per row
// summing in column order (the reference's order), separated by block
// barriers.  This replaces about four launches per level on levels whose
// work is a few microseconds, where launch and drain latency dominate.
// Only the top level's right-hand side (and iterate, when it does not start
// at zero) is read from global memory, and only its result is written back.
//
// Rows are handed to threads in a per-level order (ord) in which the 32
// rows of each warp start, as far as the pattern allows, at 32 different
// positions modulo 32: one thread per row then reads its row's columns and
// values from shared memory without bank conflicts (rows in natural order
// collide when their lengths are near multiples of 32), and still sums the
// row in column order.  On levels with long rows the products are first
// formed flat over the block (TailLevel::p), so the longest row's thread
// only adds.  The descriptor's pointers are the global sources of the
// copies; the kernel addresses the copies by their offsets from its
// shared-memory base.
template <typename T>
struct TailLevel {
  int n, nc, annz, pnnz;  // rows, coarse rows, nonzeros of A and of P
  const int *arp, *aci, *ord;
  const T *av, *invd;
  T omega;
  const int *prp, *pci;
  const T* pv;
  const int *rrp, *rci;
  const T* rv;
  T *xa, *xb, *b, *r;  // iterate pair, right-hand side, residual
  T* p;                // products a_ij x_j of A, flat (levels with long rows; else null)
  // byte offsets of the shared-memory copies (arrays above, in order; o_p:
  // the product scratch, 0 when p is null)
  unsigned o_arp, o_aci, o_ord, o_av, o_invd, o_prp, o_pci, o_pv, o_rrp, o_rci, o_rv, o_xa, o_xb,
      o_b, o_r, o_p;
};

template <typename T>
struct TailCoarse {
  int n;
  const double* lu;
  const int* piv;
  T *b, *x;
  // shared-memory offsets (bytes): factors followed by n doubles of work
  // space, pivots, right-hand side, solution
  unsigned o_lu, o_piv, o_b, o_x;
  int inv;  // 1: o_lu holds the explicit inverse (column-major), not the factors
};

constexpr int kTailMaxLevels = 8;
constexpr int kTailThreads = 256;

// The tail kernel's dynamic shared memory.  Arrays addressed from it by
// offset (tail_sh) compile to shared-memory loads; pointers read back from
// the level descriptors are generic.
extern __shared__ __align__(16) unsigned char tail_smem[];
template <typename U>
__device__ __forceinline__ U* tail_sh(unsigned off) {
  return reinterpret_cast<U*>(tail_smem + off);
}

// One bulk copy of the tail's prologue: `bytes` (a multiple of 16) from
// `src` to shared-memory offset `off`.
struct TailCopy {
  const void* src;
  unsigned off, bytes;
};

// The tail's copies: pattern arrays first (never written by a kernel),
// then the rest; x, the top level's iterate, is copied only when the
// visit does not start from zero.
struct TailCopies {
  const TailCopy* list;
  int npat, nval;
  unsigned pat_bytes, val_bytes;
  TailCopy x;
};

// a ± Σ_k v[k]·x[c[k]] over [s, e) in column order.  Eight entries at a
// time: their columns and values are loaded unconditionally (slots past the
// row end repeat its last entry), then the eight x reads, then the ordered
// sum, so each batch costs two shared-memory round trips instead of two per
// entry.
template <int SIGN, typename T>
__device__ __forceinline__ T tail_row(T a, const int* __restrict__ c, const T* __restrict__ v,
                                      const T* x, int s, int e) {
  for (int k0 = s; k0 < e; k0 += 8) {
    int cc[8];
    T vv[8], xv[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const int k = min(k0 + j, e - 1);
      cc[j] = c[k];
      vv[j] = v[k];
    }
#pragma unroll
    for (int j = 0; j < 8; ++j) xv[j] = x[cc[j]];
#pragma unroll
    for (int j = 0; j < 8; ++j)
      if (k0 + j < e) {
        const T p = mul_rn(vv[j], xv[j]);
        a = SIGN > 0 ? add_rn(a, p) : sub_rn(a, p);
      }
  }
  return a;
}

// a ± p[s] ± p[s+1] ... in order, eight products loaded at a time.
template <int SIGN, typename T>
__device__ __forceinline__ T tail_sum(T a, const T* __restrict__ p, int s, int e) {
  for (int k0 = s; k0 < e; k0 += 8) {
    T pv[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) pv[j] = p[min(k0 + j, e - 1)];
#pragma unroll
    for (int j = 0; j < 8; ++j)
      if (k0 + j < e) a = SIGN > 0 ? add_rn(a, pv[j]) : sub_rn(a, pv[j]);
  }
  return a;
}

// Levels with long rows (L.p set) form the products a_ij·x_j of A flat over
// the whole block first, so a long row no longer holds one thread for all
// of its gathers; each row then sums its products in column order (the
// same rounded products and sums as tail_row).
template <typename T>
__device__ __forceinline__ void tail_products(const TailLevel<T>& L, const T* x) {
  if (!L.p) return;
  T* __restrict__ p = tail_sh<T>(L.o_p);
  const int* __restrict__ c = tail_sh<const int>(L.o_aci);
  const T* __restrict__ v = tail_sh<const T>(L.o_av);
  const int nnz = L.annz;
  for (int k0 = threadIdx.x; k0 < nnz; k0 += 4 * kTailThreads) {
    int cc[4];
    T vv[4], xv[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int k = min(k0 + j * kTailThreads, nnz - 1);
      cc[j] = c[k];
      vv[j] = v[k];
    }
#pragma unroll
    for (int j = 0; j < 4; ++j) xv[j] = x[cc[j]];
#pragma unroll
    for (int j = 0; j < 4; ++j)
      if (k0 + j * kTailThreads < nnz) p[k0 + j * kTailThreads] = mul_rn(vv[j], xv[j]);
  }
  __syncthreads();
}

// a ± Σ_k a_ik x_k over row i of A, in column order.
template <int SIGN, typename T>
__device__ __forceinline__ T tail_arow(const TailLevel<T>& L, T a, const T* x, int i) {
  const int* rp = tail_sh<const int>(L.o_arp);
  return L.p ? tail_sum<SIGN>(a, tail_sh<const T>(L.o_p), rp[i], rp[i + 1])
             : tail_row<SIGN>(a, tail_sh<const int>(L.o_aci), tail_sh<const T>(L.o_av), x, rp[i],
                              rp[i + 1]);
}

template <typename T>
__device__ __forceinline__ void tail_jacobi(const TailLevel<T>& L, const T* x, const T* b, T* xn) {
  tail_products(L, x);
  const int* ord = tail_sh<const int>(L.o_ord);
  const T* invd = tail_sh<const T>(L.o_invd);
  for (int t = threadIdx.x; t < L.n; t += blockDim.x) {
    const int i = ord[t];
    const T ri = tail_arow<-1>(L, b[i], x, i);
    xn[i] = add_rn(x[i], mul_rn(mul_rn(L.omega, invd[i]), ri));
  }
  __syncthreads();
}

// Coarsest solve with the (shared-memory) LU factors, getrs order: row
// interchanges, then L (unit diagonal) and U substitutions by columns, a
// column's update skipped when its solution entry is zero.  Up to 32
// unknowns one warp holds y in registers (lane i: y_i); larger systems use
// the block with y in shared memory after the factors.
template <typename T>
__device__ __forceinline__ void tail_lu_solve(const TailCoarse<T>& C) {
  const int n = C.n;
  const double* lu = tail_sh<const double>(C.o_lu);
  const int* piv = tail_sh<const int>(C.o_piv);
  const T* cb = tail_sh<const T>(C.o_b);
  T* cx = tail_sh<T>(C.o_x);
  if (C.inv && n <= 32) {
    // x = A_c^-1 b, one row of the inverse per lane, summed in column order
    if (threadIdx.x < 32) {
      const int i = threadIdx.x;
      if (i < n) {
        double y = 0.0;
        for (int j = 0; j < n; ++j) y = __dadd_rn(y, __dmul_rn(lu[j * n + i], (double)cb[j]));
        cx[i] = (T)y;
      }
    }
    __syncthreads();
    return;
  }
  if (n <= 32) {
    if (threadIdx.x < 32) {
      const int i = threadIdx.x;
      double y = i < n ? (double)cb[i] : 0.0;
      for (int j = 0; j < n; ++j) {
        const int p = piv[j];
        if (p != j) {
          const double a = __shfl_sync(0xffffffffu, y, j);
          const double c = __shfl_sync(0xffffffffu, y, p);
          if (i == j) y = c;
          if (i == p) y = a;
        }
      }
      for (int j = 0; j < n; ++j) {
        const double yj = __shfl_sync(0xffffffffu, y, j);
        if (yj != 0.0 && i > j && i < n) y = __dsub_rn(y, __dmul_rn(yj, lu[j * n + i]));
      }
      for (int j = n - 1; j >= 0; --j) {
        if (i == j && y != 0.0) y = __ddiv_rn(y, lu[j * n + j]);
        const double yj = __shfl_sync(0xffffffffu, y, j);
        if (yj != 0.0 && i < j) y = __dsub_rn(y, __dmul_rn(yj, lu[j * n + i]));
      }
      if (i < n) cx[i] = (T)y;
    }
    __syncthreads();
    return;
  }
  double* y = tail_sh<double>(C.o_lu) + n * n;
  for (int i = threadIdx.x; i < n; i += blockDim.x) y[i] = (double)cb[i];
  __syncthreads();
  if (threadIdx.x == 0)
    for (int j = 0; j < n; ++j) {
      const int p = piv[j];
      if (p != j) {
        const double t = y[j];
        y[j] = y[p];
        y[p] = t;
      }
    }
  __syncthreads();
  for (int j = 0; j < n; ++j) {
    const double yj = y[j];
    if (yj != 0.0)
      for (int i = j + 1 + threadIdx.x; i < n; i += blockDim.x)
        y[i] = __dsub_rn(y[i], __dmul_rn(yj, lu[j * n + i]));
    __syncthreads();
  }
  for (int j = n - 1; j >= 0; --j) {
    if (threadIdx.x == 0 && y[j] != 0.0) y[j] = __ddiv_rn(y[j], lu[j * n + j]);
    __syncthreads();
    const double yj = y[j];
    if (yj != 0.0)
      for (int i = threadIdx.x; i < j; i += blockDim.x)
        y[i] = __dsub_rn(y[i], __dmul_rn(yj, lu[j * n + i]));
    __syncthreads();
  }
  for (int i = threadIdx.x; i < n; i += blockDim.x) cx[i] = (T)y[i];
  __syncthreads();
}

// One visit of level l = D (x_zero: the iterate starts at zero).  The
// result ends in the level's xa.  Levels l+1 .. nl-1 follow in `lv`; the
// coarsest system is C.  The level index is a template parameter so that
// the visits of all levels inline into the kernel (a recursive device
// function keeps a stack frame and spills around each call), and every
// array is addressed from the shared-memory base by its offset.
template <int D, typename T>
__device__ __forceinline__ void tail_visit(const TailLevel<T>* lv, int nl, const TailCoarse<T>& C,
                                           bool x_zero, int pre, int post, int wcycle) {
  constexpr int l = D;
  const TailLevel<T>& L = lv[l];
  const int n = L.n;
  T* const xa = tail_sh<T>(L.o_xa);
  T* x = xa;
  T* t = tail_sh<T>(L.o_xb);
  const T* b = tail_sh<const T>(L.o_b);
  const T* invd = tail_sh<const T>(L.o_invd);
  if (x_zero && pre >= 1) {
    // first Jacobi step from zero
    for (int i = threadIdx.x; i < n; i += blockDim.x) x[i] = mul_rn(mul_rn(L.omega, invd[i]), b[i]);
    __syncthreads();
    for (int s = 1; s < pre; ++s) {
      tail_jacobi(L, x, b, t);
      T* u = x; x = t; t = u;
    }
  } else {
    if (x_zero) {
      for (int i = threadIdx.x; i < n; i += blockDim.x) x[i] = T(0);
      __syncthreads();
    }
    for (int s = 0; s < pre; ++s) {
      tail_jacobi(L, x, b, t);
      T* u = x; x = t; t = u;
    }
  }
  {
    T* r = tail_sh<T>(L.o_r);
    const int* ord = tail_sh<const int>(L.o_ord);
    tail_products(L, x);
    for (int k = threadIdx.x; k < n; k += blockDim.x) {
      const int i = ord[k];
      r[i] = sub_rn(b[i], tail_arow<1>(L, T(0), x, i));
    }
    __syncthreads();
    const bool last = (l + 1 == nl);
    T* bn = last ? tail_sh<T>(C.o_b) : tail_sh<T>(lv[l + 1].o_b);
    const int* rrp = tail_sh<const int>(L.o_rrp);
    const int* rci = tail_sh<const int>(L.o_rci);
    const T* rv = tail_sh<const T>(L.o_rv);
    for (int J = threadIdx.x; J < L.nc; J += blockDim.x)
      bn[J] = tail_row<1>(T(0), rci, rv, r, rrp[J], rrp[J + 1]);
    __syncthreads();
  }
  const T* xc;
  if (l + 1 < nl) {
    if constexpr (D + 1 < kTailMaxLevels) {
      for (int rep = 0; rep < (wcycle ? 2 : 1); ++rep)
        tail_visit<D + 1>(lv, nl, C, rep == 0, pre, post, wcycle);
    }
    xc = tail_sh<const T>(lv[l + 1].o_xa);
  } else {
    tail_lu_solve(C);
    xc = tail_sh<const T>(C.o_x);
  }
  {
    const int* prp = tail_sh<const int>(L.o_prp);
    const int* pci = tail_sh<const int>(L.o_pci);
    const T* pv = tail_sh<const T>(L.o_pv);
    for (int i = threadIdx.x; i < n; i += blockDim.x)
      x[i] = tail_row<1>(x[i], pci, pv, xc, prp[i], prp[i + 1]);
    __syncthreads();
  }
  for (int s = 0; s < post; ++s) {
    tail_jacobi(L, x, b, t);
    T* u = x; x = t; t = u;
  }
  if (x != xa) {
    for (int i = threadIdx.x; i < n; i += blockDim.x) xa[i] = x[i];
    __syncthreads();
  }
}


// lv: nl (<= kTailMaxLevels) descriptors with global pointers and the
// shared-memory layout; dynamic shared memory holds that layout.  Every
// source array starts an allocation whose size is a multiple of 16 bytes
// and every destination is 16-byte aligned, so each array arrives by one
// bulk copy (TMA) rounded up to 16 bytes, all of them on one mbarrier.  A
// copy that does not complete within the wait limit sets *err and the block
// returns without touching global memory.
template <typename T>
__global__ void __launch_bounds__(kTailThreads, 1)
k_coarse_tail(const TailLevel<T>* __restrict__ lv, int nl, TailCoarse<T> C, TailCopies cp, int pre,
              int post, int wcycle, int x_zero, int* err) {
  unsigned char* const tsm = tail_smem;
  __shared__ TailLevel<T> sl[kTailMaxLevels];
  __shared__ TailCoarse<T> sc;
  __shared__ __align__(8) uint64_t bar;
  __shared__ int ok;
  // warp 0 issues the copies, one per lane at a time
  if (threadIdx.x < 32) {
    if (threadIdx.x == 0) {
      mbar_init(&bar, 1);
      fence_mbar_init();
      mbar_expect_tx(&bar, cp.pat_bytes + cp.val_bytes + (x_zero ? 0u : cp.x.bytes));
    }
    __syncwarp();
    for (int i = threadIdx.x; i < cp.npat; i += 32) {
      const TailCopy c = cp.list[i];
      bulk_g2s(tsm + c.off, c.src, c.bytes, &bar);
    }
  }
  pdl_trigger();
  pdl_wait();
  if (threadIdx.x < 32) {
    for (int i = threadIdx.x; i < cp.nval; i += 32) {
      const TailCopy c = cp.list[cp.npat + i];
      bulk_g2s(tsm + c.off, c.src, c.bytes, &bar);
    }
    if (threadIdx.x == 0 && !x_zero && cp.x.bytes) bulk_g2s(tsm + cp.x.off, cp.x.src, cp.x.bytes, &bar);
  }
  // the descriptors (sizes, ω, shared-memory offsets) into shared memory
  if (threadIdx.x < nl) sl[threadIdx.x] = lv[threadIdx.x];
  if (threadIdx.x == 32) sc = C;
  if (threadIdx.x == 0) ok = 1;
  __syncthreads();  // barrier initialised, descriptors published
  if (!mbar_wait_bounded(&bar, 0, kWaitLimit)) ok = 0;  // every thread observes the copies
  __syncthreads();
  if (!ok) {
    if (threadIdx.x == 0) {
      atomicExch(err, 1);
      mbar_wait_bounded(&bar, 0, kWaitLimit);  // let copies in flight land before exit
    }
    return;
  }
  tail_visit<0>(sl, nl, sc, x_zero != 0, pre, post, wcycle);
  // the top level's result back to global memory
  const T* xa0 = tail_sh<const T>(sl[0].o_xa);
  for (int i = threadIdx.x; i < sl[0].n; i += blockDim.x) lv[0].xa[i] = xa0[i];
}

// Solve A^T y = b with the dgetf2 factors of A (A = P L U, column-major,
// pivots piv): U^T z = b, L^T w = z, then the row interchanges in reverse
// (dgetrs with trans = 'T').  One thread: used by adjoint solves only.
template <typename T>
__global__ void k_lu_solve_t(int n, const double* __restrict__ lu, const int* __restrict__ piv,
                             const T* __restrict__ bin, T* __restrict__ xout) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  extern __shared__ double ys[];
  for (int i = 0; i < n; ++i) ys[i] = (double)bin[i];
  for (int j = 0; j < n; ++j) {  // U^T (lower triangular, non-unit)
    double t = ys[j];
    for (int i = 0; i < j; ++i) t -= lu[(size_t)j * n + i] * ys[i];
    ys[j] = t / lu[(size_t)j * n + j];
  }
  for (int j = n - 1; j >= 0; --j) {  // L^T (upper triangular, unit)
    double t = ys[j];
    for (int i = j + 1; i < n; ++i) t -= lu[(size_t)j * n + i] * ys[i];
    ys[j] = t;
  }
  for (int j = n - 1; j >= 0; --j) {
    const int p = piv[j];
    if (p != j) {
      const double t = ys[j];
      ys[j] = ys[p];
      ys[p] = t;
    }
  }
  for (int i = 0; i < n; ++i) xout[i] = (T)ys[i];
}

// In-place unblocked LU with partial pivoting (dgetf2 order) of a
// column-major n x n matrix in one block.  info = 0 or the 1-based index of
// the first zero pivot (factorisation stops there).
__global__ void k_lu_factor(int n, double* __restrict__ a, int* __restrict__ piv, int* info) {
  __shared__ double sv[1024];
  __shared__ int si[1024];
  __shared__ int sp;
  if (threadIdx.x == 0) *info = 0;
  for (int j = 0; j < n; ++j) {
    // pivot search: first index of the maximum magnitude in column j
    double best = -1.0;
    int bi = n;
    for (int i = j + threadIdx.x; i < n; i += blockDim.x) {
      double v = fabs(a[(size_t)j * n + i]);
      if (v > best) { best = v; bi = i; }
    }
    sv[threadIdx.x] = best;
    si[threadIdx.x] = bi;
    __syncthreads();
    for (int s = blockDim.x >> 1; s > 0; s >>= 1) {
      if (threadIdx.x < s) {
        double v2 = sv[threadIdx.x + s];
        int i2 = si[threadIdx.x + s];
        if (v2 > sv[threadIdx.x] || (v2 == sv[threadIdx.x] && i2 < si[threadIdx.x])) {
          sv[threadIdx.x] = v2;
          si[threadIdx.x] = i2;
        }
      }
      __syncthreads();
    }
    if (threadIdx.x == 0) {
      sp = si[0];
      piv[j] = sp;
    }
    __syncthreads();
    const int p = sp;
    if (a[(size_t)j * n + p] == 0.0) {
      if (threadIdx.x == 0) *info = j + 1;
      return;
    }
    if (p != j)
      for (int c = threadIdx.x; c < n; c += blockDim.x) {
        double t = a[(size_t)c * n + j];
        a[(size_t)c * n + j] = a[(size_t)c * n + p];
        a[(size_t)c * n + p] = t;
      }
    __syncthreads();
    const double r = __drcp_rn(a[(size_t)j * n + j]);
    for (int i = j + 1 + threadIdx.x; i < n; i += blockDim.x)
      a[(size_t)j * n + i] = __dmul_rn(a[(size_t)j * n + i], r);
    __syncthreads();
    const int m = n - j - 1;
    for (long long t = threadIdx.x; t < (long long)m * m; t += blockDim.x) {
      const int c = j + 1 + (int)(t / m);
      const int i = j + 1 + (int)(t % m);
      a[(size_t)c * n + i] =
          __dsub_rn(a[(size_t)c * n + i], __dmul_rn(a[(size_t)j * n + i], a[(size_t)c * n + j]));
    }
    __syncthreads();
  }
}

// Explicit inverse of A from its getrf factors (column-major, 0-based
// pivots), column j by thread j: A x = e_j solved in getrs order (row
// interchanges, unit-lower then upper substitution).  n <= kInvMax.  Used
// where the coarsest solve need not be the reference's substitutions bit for
// bit.
constexpr int kInvMax = 64;
__device__ __forceinline__ void lu_inverse_column(int n, const double* __restrict__ lu,
                                                  const int* __restrict__ piv, double* __restrict__ inv,
                                                  int j) {
  double y[kInvMax];
  for (int i = 0; i < n; ++i) y[i] = i == j ? 1.0 : 0.0;
  for (int k = 0; k < n; ++k) {
    const int p = piv[k];
    if (p != k) {
      const double t = y[k];
      y[k] = y[p];
      y[p] = t;
    }
  }
  for (int k = 0; k < n; ++k)
    if (y[k] != 0.0)
      for (int i = k + 1; i < n; ++i) y[i] = __dsub_rn(y[i], __dmul_rn(y[k], lu[k * n + i]));
  for (int k = n - 1; k >= 0; --k) {
    if (y[k] != 0.0) y[k] = __ddiv_rn(y[k], lu[k * n + k]);
    if (y[k] != 0.0)
      for (int i = 0; i < k; ++i) y[i] = __dsub_rn(y[i], __dmul_rn(y[k], lu[k * n + i]));
  }
  for (int i = 0; i < n; ++i) inv[j * n + i] = y[i];
}
__global__ void k_lu_inverse(int n, const double* __restrict__ lu, const int* __restrict__ piv,
                             double* __restrict__ inv) {
  if ((int)threadIdx.x < n) lu_inverse_column(n, lu, piv, inv, threadIdx.x);
}

// Scatter CSR values into a zeroed column-major dense matrix.
__global__ void k_csr_to_dense(int n, const int* __restrict__ rp, const int* __restrict__ ci,
                               const double* __restrict__ v, double* __restrict__ M) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    for (int k = rp[i]; k < rp[i + 1]; ++k) M[(size_t)ci[k] * n + i] = v[k];
}

// ------------------------------------------------------------ smoother diagonals
// src/smoothers.jl:47-63: 1/a_ii, or 0 if |a_ii| <= eps·max(1, Σ|a_ij|)
__global__ void k_invdiag(int n, const int* __restrict__ rp, const int* __restrict__ ci,
                          const double* __restrict__ v, double* __restrict__ invd) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double d = 0.0, rn = 0.0;
    for (int k = rp[i]; k < rp[i + 1]; ++k) {
      rn = __dadd_rn(rn, fabs(v[k]));
      if (ci[k] == i) d = v[k];
    }
    const double thr = 2.220446049250313e-16 * fmax(1.0, rn);
    invd[i] = fabs(d) > thr ? __drcp_rn(d) : 0.0;
  }
}

// src/smoothers.jl:816-827: 1/Σ|a_ij|, or 0 if the sum is <= eps
__global__ void k_l1_invdiag(int n, const int* __restrict__ rp, const double* __restrict__ v,
                             double* __restrict__ invd) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double l1 = 0.0;
    for (int k = rp[i]; k < rp[i + 1]; ++k) l1 = __dadd_rn(l1, fabs(v[k]));
    invd[i] = l1 > 2.220446049250313e-16 ? __drcp_rn(l1) : 0.0;
  }
}

// ------------------------------------------------------------ Galerkin product lists
// The numeric Galerkin product O = S B on fixed patterns as a list of
// product pairs per output entry: entry e of O is the sum, in list order,
// of s_v[ls[p]] * b_v[lb[p]] for p in [off[e], off[e + 1]).  The lists are
// recorded once by k_spgemm_sym (COUNT, then FILL after an exclusive scan
// of the counts) walking the products exactly as k_spgemm_warp does -- in
// the order (entry k of S's row, entry t of B's row j_k), grouped by output
// entry in lane order -- so k_spgemm_apply_staged adds every entry's products in
// the same order and gives the same values bit for bit, with a few
// instructions and 24 bytes of traffic per product.
template <int CAP, int WPB, bool FILL>
__global__ void __launch_bounds__(WPB * 32)
k_spgemm_sym(int nrows, const int* __restrict__ out_rp, const int* __restrict__ out_ci,
             const int* __restrict__ s_rp, const int* __restrict__ s_ci, const int* __restrict__ b_rp,
             const int* __restrict__ b_ci, int* cnt, const long long* __restrict__ off,
             int* __restrict__ ls, int* __restrict__ lb) {
  __shared__ int scol[WPB][CAP];
  __shared__ int sk[WPB][32], st[WPB][32];
  const int lane = threadIdx.x & 31;
  const int w = threadIdx.x >> 5;
  const unsigned full = 0xffffffffu;
  for (long long I0 = (long long)blockIdx.x * WPB + w; I0 < nrows; I0 += (long long)gridDim.x * WPB) {
    const int I = (int)I0;
    const int os = out_rp[I], oe = out_rp[I + 1];
    const int m = oe - os;
    const bool fits = m <= CAP;
    const int* pat = fits ? scol[w] : out_ci + os;
    if (fits)
      for (int t = lane; t < m; t += 32) scol[w][t] = out_ci[os + t];
    __syncwarp();
    const int ss = s_rp[I], se = s_rp[I + 1];
    for (int k0 = ss; k0 < se; k0 += 32) {
      const int k = k0 + lane;
      int bs = 0, len = 0;
      if (k < se) {
        const int j = s_ci[k];
        bs = b_rp[j];
        len = b_rp[j + 1] - bs;
      }
      int incl = len;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(full, incl, o);
        if (lane >= o) incl += y;
      }
      const int excl = incl - len;
      const int total = __shfl_sync(full, incl, 31);
      for (int f0 = 0; f0 < total; f0 += 32) {
        const int f = f0 + lane;
        int q = 0;
#pragma unroll
        for (int step = 16; step > 0; step >>= 1) {
          const int ex = __shfl_sync(full, excl, q + step);
          if (ex <= f) q += step;
        }
        const int qbs = __shfl_sync(full, bs, q);
        const int qex = __shfl_sync(full, excl, q);
        const bool act = f < total;
        int pos = -1, t = 0;
        if (act) {
          t = qbs + (f - qex);
          const int J = b_ci[t];
          int lo = 0, hi = m - 1;
          while (lo <= hi) {
            const int mid = (lo + hi) >> 1;
            const int c = pat[mid];
            if (c == J) {
              pos = mid;
              break;
            }
            if (c < J) lo = mid + 1;
            else hi = mid - 1;
          }
        }
        if (FILL) {
          sk[w][lane] = k0 + q;
          st[w][lane] = t;
        }
        const unsigned am = __ballot_sync(full, pos >= 0);
        __syncwarp();
        if (pos >= 0) {
          const unsigned peers = __match_any_sync(am, pos);
          if (lane == __ffs(peers) - 1) {
            const int e = os + pos;
            if (FILL) {
              long long slot = off[e] + cnt[e];
              for (unsigned mm = peers; mm; mm &= mm - 1) {
                const int src = __ffs(mm) - 1;
                ls[slot] = sk[w][src];
                lb[slot] = st[w][src];
                ++slot;
              }
            }
            cnt[e] += __popc(peers);
          }
        }
        __syncwarp();
      }
    }
  }
}

// O's values from the product lists (see k_spgemm_sym): a warp takes 32
// consecutive output entries, whose lists are contiguous, copies their
// (S entry, B entry) pairs into shared memory with coalesced loads when
// they number at most CAPW, and each lane then adds its entry's products
// in list order from there, multiplied and added with separate rounding
// (the warp kernel's values, bit for bit).  Spans longer than CAPW are read
// from global memory.
template <typename T, int WPB, int CAPW>
__global__ void __launch_bounds__(WPB * 32)
k_spgemm_apply_staged(long long nout, const long long* __restrict__ off, const int* __restrict__ ls,
                      const int* __restrict__ lb, const T* __restrict__ s_v, const T* __restrict__ b_v,
                      T* __restrict__ out_v) {
  __shared__ int2 stage[WPB][CAPW];
  const int lane = threadIdx.x & 31;
  const int w = threadIdx.x >> 5;
  for (long long e0 = ((long long)blockIdx.x * WPB + w) * 32; e0 < nout; e0 += (long long)gridDim.x * WPB * 32) {
    const long long e = e0 + lane;
    const long long p0 = __ldg(off + e0);
    const long long p1 = __ldg(off + min(e0 + 32, nout));
    const long long my0 = e < nout ? __ldg(off + e) : p1;
    const long long my1 = e < nout ? __ldg(off + e + 1) : p1;
    T a = T(0);
    if (p1 - p0 <= CAPW) {
      for (long long q = p0 + lane; q < p1; q += 32) stage[w][q - p0] = make_int2(__ldg(ls + q), __ldg(lb + q));
      __syncwarp();
#pragma unroll 4
      for (long long q = my0; q < my1; ++q) {
        const int2 pr = stage[w][q - p0];
        a = add_rn(a, mul_rn(__ldg(s_v + pr.x), __ldg(b_v + pr.y)));
      }
      __syncwarp();
    } else {
      for (long long q = my0; q < my1; ++q) a = add_rn(a, mul_rn(__ldg(s_v + __ldg(ls + q)), __ldg(b_v + __ldg(lb + q))));
    }
    if (e < nout) out_v[e] = a;
  }
}

// ILU(0) substitutions, one level of the schedule per launch (src/
// smoothers.jl:1398-1423; the serial smoother's loops, :1174-1192, give the
// same values): one thread per row, the row's products subtracted in column
// order with separately rounded products and differences.
// Forward: t_i -= L_ik t_k over the strictly lower part of row i.
template <typename T>
__global__ void k_ilu_fwd(int cnt, const int* __restrict__ order, const int* __restrict__ rp,
                          const int* __restrict__ ci, const int* __restrict__ diag, const T* __restrict__ Lv,
                          T* __restrict__ t) {
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < cnt; q += gridDim.x * blockDim.x) {
    const int i = order[q];
    T s = t[i];
    for (int nz = rp[i]; nz < diag[i]; ++nz) s = sub_rn(s, mul_rn(Lv[nz], t[ci[nz]]));
    t[i] = s;
  }
}

__device__ __forceinline__ double div_rn(double a, double b) { return __ddiv_rn(a, b); }
__device__ __forceinline__ float div_rn(float a, float b) { return __fdiv_rn(a, b); }
template <typename T>
__device__ __forceinline__ T eps_of();
template <>
__device__ __forceinline__ double eps_of<double>() { return 2.220446049250313e-16; }
template <>
__device__ __forceinline__ float eps_of<float>() { return 1.1920929e-07f; }

// Backward: t_i -= U_ij t_j over the strictly upper part, then t_i / U_ii
// (0 when |U_ii| <= eps).
template <typename T>
__global__ void k_ilu_bwd(int cnt, const int* __restrict__ order, const int* __restrict__ rp,
                          const int* __restrict__ ci, const int* __restrict__ diag, const T* __restrict__ Uv,
                          T* __restrict__ t) {
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < cnt; q += gridDim.x * blockDim.x) {
    const int i = order[q];
    const int di = diag[i];
    T s = t[i];
    for (int nz = di + 1; nz < rp[i + 1]; ++nz) s = sub_rn(s, mul_rn(Uv[nz], t[ci[nz]]));
    const T u = Uv[di];
    t[i] = fabs(u) > eps_of<T>() ? div_rn(s, u) : T(0);
  }
}

// One level of the serial Gauss-Seidel sweep (src/smoothers.jl:350-362):
// one thread per row, r = b_i - a_i1 x_1 - ... in column order, x_i +=
// invd_i r, in place.
template <typename T>
__global__ void k_sgs_level(int cnt, const int* __restrict__ order, const int* __restrict__ rp,
                            const int* __restrict__ ci, const T* __restrict__ av, const T* __restrict__ b,
                            const T* __restrict__ invd, T* x) {
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < cnt; q += gridDim.x * blockDim.x) {
    const int i = order[q];
    T r = b[i];
    for (int nz = rp[i]; nz < rp[i + 1]; ++nz) r = sub_rn(r, mul_rn(av[nz], x[ci[nz]]));
    x[i] = add_rn(x[i], mul_rn(invd[i], r));
  }
}

// _serial_gs_compute_invdiag! (src/smoothers.jl:329-340): 1/a_ii from the
// row's first diagonal entry, 0 when |a_ii| <= eps.
__global__ void k_sgs_invdiag(int n, const int* __restrict__ rp, const int* __restrict__ ci,
                              const double* __restrict__ v, double* __restrict__ invd) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double d = 0.0;
    for (int k = rp[i]; k < rp[i + 1]; ++k)
      if (ci[k] == i) {
        d = v[k];
        break;
      }
    invd[i] = fabs(d) > 2.220446049250313e-16 ? __drcp_rn(d) : 0.0;
  }
}

// x += dx where dx is finite (src/smoothers.jl:1426-1431).
template <typename T>
__global__ void k_ilu_apply(int n, const T* __restrict__ dx, T* __restrict__ x) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const T v = dx[i];
    if (isfinite(v)) x[i] = add_rn(x[i], v);
  }
}

// Power step, continued: lambda = ||w|| = sqrt(lam2[0]); v = w / lambda when
// lambda > eps (src/smoothers.jl:881-884).
__global__ void k_cheb_rescale(int n, const double* __restrict__ w, const double* __restrict__ lam2,
                               double* __restrict__ v) {
  const double lam = sqrt(__ldg(lam2));
  if (!(lam > 2.220446049250313e-16)) return;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    v[i] = __ddiv_rn(w[i], lam);
}

// Chebyshev coefficients from the spectral-radius estimate rho =
// sqrt(lam2[0]) (build_chebyshev_smoother and smooth!, src/smoothers.jl:
// 895-910, :947-986): lambda_max = 1.1 rho, lambda_min = lambda_max / 30,
// coef[0] = 1/theta, then (scale_r, scale_d) of inner steps 1.. at [2k],
// [2k+1].  One thread.
__global__ void k_cheb_coef(const double* __restrict__ lam2, int degree, double* __restrict__ coef) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  const double rho = sqrt(lam2[0]);
  const double lmax = __dmul_rn(1.1, rho);
  const double lmin = __ddiv_rn(lmax, 30.0);
  const double theta = __ddiv_rn(__dadd_rn(lmax, lmin), 2.0);
  const double delta = __ddiv_rn(__dsub_rn(lmax, lmin), 2.0);
  coef[0] = __ddiv_rn(1.0, theta);
  coef[1] = 0.0;
  double s_old = __ddiv_rn(theta, delta);
  for (int k = 1; k < degree; ++k) {
    const double s_new = __ddiv_rn(1.0, __dsub_rn(__ddiv_rn(__dmul_rn(2.0, theta), delta), s_old));
    coef[2 * k] = __ddiv_rn(__dmul_rn(2.0, s_new), delta);
    coef[2 * k + 1] = __dmul_rn(s_new, s_old);
    s_old = s_new;
  }
}

// src/smoothers.jl:524-538: SPAI(0) m_i = a_ii / sum_j a_ij^2 (0 for a
// zero row), products and sums rounded separately, in column order
__global__ void k_spai0_diag(int n, const int* __restrict__ rp, const int* __restrict__ ci,
                             const double* __restrict__ v, double* __restrict__ m) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double d = 0.0, s = 0.0;
    for (int k = rp[i]; k < rp[i + 1]; ++k) {
      const double a = v[k];
      s = __dadd_rn(s, __dmul_rn(a, a));
      if (ci[k] == i) d = a;
    }
    m[i] = s > 0.0 ? __ddiv_rn(d, s) : 0.0;
  }
}

// ------------------------------------------------------------ Galerkin product
// Phase 1 (A·P): S = A, B = P.  Phase 2 (Pᵀ·(AP)): S = R = Pᵀ in
// transpose-map order, B = A·P.
//
// Numeric sparse product O = S·B on O's fixed, sorted sparsity pattern (the
// Galerkin products A·P and Pᵀ·(AP) of a partial resetup), one warp per
// output row, deterministic and without atomics.
//
// The products of row I are numbered in the order (entry k of S's row,
// entry t of B's row j_k).  For each run of 32 entries of S's row the warp
// scans the lengths of the B rows they select; then, 32 products at a time,
// every lane finds its product's entry (a shuffle search over the scan),
// forms it and looks its column up in O's row pattern (binary search;
// staged in shared memory when the row has at most CAP entries).  Products
// that land on the same output entry are added by the lowest of their lanes
// in lane order, after the entry's earlier sum: every entry accumulates its
// products in the same order as a sequential loop over (k, t) — the order
// of the CPU setup's numeric product, bit for bit.
//
// WPB warps per block; the per-warp row patterns and sums (CAP entries each)
// live in dynamic shared memory: spgemm_smem_bytes<CAP, WPB>().
template <typename T, int CAP, int WPB>
constexpr size_t spgemm_smem_bytes() {
  return (size_t)WPB * CAP * (sizeof(T) + sizeof(int)) + (size_t)WPB * 32 * sizeof(T);
}

template <typename T, int CAP, int WPB>
__global__ void __launch_bounds__(WPB * 32)
k_spgemm_warp(int nrows, const int* __restrict__ out_rp, const int* __restrict__ out_ci,
              T* __restrict__ out_v, const int* __restrict__ s_rp, const int* __restrict__ s_ci,
              const T* __restrict__ s_v, const int* __restrict__ b_rp,
              const int* __restrict__ b_ci, const T* __restrict__ b_v) {
  extern __shared__ __align__(16) unsigned char gsm[];
  T (*sacc)[CAP] = reinterpret_cast<T (*)[CAP]>(gsm);
  T (*sprod)[32] = reinterpret_cast<T (*)[32]>(gsm + (size_t)WPB * CAP * sizeof(T));
  int (*scol)[CAP] = reinterpret_cast<int (*)[CAP]>(gsm + (size_t)WPB * (CAP + 32) * sizeof(T));
  const int lane = threadIdx.x & 31;
  const int w = threadIdx.x >> 5;
  const unsigned full = 0xffffffffu;
  for (long long I0 = (long long)blockIdx.x * WPB + w; I0 < nrows; I0 += (long long)gridDim.x * WPB) {
    const int I = (int)I0;
    const int os = out_rp[I], oe = out_rp[I + 1];
    const int m = oe - os;
    const bool fits = m <= CAP;
    const int* pat = fits ? scol[w] : out_ci + os;
    T* acc = fits ? sacc[w] : out_v + os;
    for (int t = lane; t < m; t += 32) {
      if (fits) scol[w][t] = out_ci[os + t];
      acc[t] = T(0);
    }
    __syncwarp();
    const int ss = s_rp[I], se = s_rp[I + 1];
    for (int k0 = ss; k0 < se; k0 += 32) {
      const int k = k0 + lane;
      int bs = 0, len = 0;
      T sv = T(0);
      if (k < se) {
        const int j = s_ci[k];
        sv = s_v[k];
        bs = b_rp[j];
        len = b_rp[j + 1] - bs;
      }
      int incl = len;  // inclusive scan of the selected B rows' lengths
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(full, incl, o);
        if (lane >= o) incl += y;
      }
      const int excl = incl - len;
      const int total = __shfl_sync(full, incl, 31);
      for (int f0 = 0; f0 < total; f0 += 32) {
        const int f = f0 + lane;
        // the entry of S's row that owns product f: the largest q with excl_q <= f
        int q = 0;
#pragma unroll
        for (int step = 16; step > 0; step >>= 1) {
          const int ex = __shfl_sync(full, excl, q + step);
          if (ex <= f) q += step;
        }
        const int qbs = __shfl_sync(full, bs, q);
        const int qex = __shfl_sync(full, excl, q);
        const T qsv = __shfl_sync(full, sv, q);
        const bool act = f < total;
        int pos = -1;
        T prod = T(0);
        if (act) {
          const int t = qbs + (f - qex);
          const int J = b_ci[t];
          prod = mul_rn(qsv, b_v[t]);
          int lo = 0, hi = m - 1;
          while (lo <= hi) {
            const int mid = (lo + hi) >> 1;
            const int c = pat[mid];
            if (c == J) {
              pos = mid;
              break;
            }
            if (c < J) lo = mid + 1;
            else hi = mid - 1;
          }
        }
        sprod[w][lane] = prod;
        const unsigned am = __ballot_sync(full, pos >= 0);
        __syncwarp();
        if (pos >= 0) {
          const unsigned peers = __match_any_sync(am, pos);
          if (lane == __ffs(peers) - 1) {
            T a = acc[pos];
            for (unsigned mm = peers; mm; mm &= mm - 1) a = add_rn(a, sprod[w][__ffs(mm) - 1]);
            acc[pos] = a;
          }
        }
        __syncwarp();
      }
    }
    if (fits)
      for (int t = lane; t < m; t += 32) out_v[os + t] = sacc[w][t];
    __syncwarp();
  }
}

// ------------------------------------------------------------ batched systems
// Many independent systems merged level by level into block-diagonal
// matrices (a "batch"): the vectors of a merged level hold the rows of the
// systems still smoothing there, then the rows of the systems whose
// coarsest level it is.  Segment s of the finest level is system s.

// Coarsest solves of the systems that end at one merged level: block k
// solves its system's dense LU (column-major factors at lu + luoff[k],
// 0-based pivots at piv + poff[k]) for rows off[k] .. off[k] + nb[k] - 1 of
// b into x, in the operation order of k_lu_solve (so each system's coarse
// solve gives what its own hierarchy's gives).
// The explicit inverses of the coarsest systems of a batch (block k: system
// k, thread j: column j; inverse stored where the factors are;
// n <= kInvMax),
// and their application x = A^-1 b, one block of kInvMax threads per
// system, each row of the inverse summed in column order.
__global__ void k_lu_inverse_batch(const int* __restrict__ nb, const long long* __restrict__ luoff,
                                   const int* __restrict__ poff, const double* __restrict__ lu_all,
                                   const int* __restrict__ piv_all, double* __restrict__ inv_all) {
  const int k = blockIdx.x;
  const int n = nb[k];
  if ((int)threadIdx.x < n)
    lu_inverse_column(n, lu_all + luoff[k], piv_all + poff[k], inv_all + luoff[k], threadIdx.x);
}

template <typename T>
__global__ void __launch_bounds__(kInvMax)
k_inv_apply_batch(const int* __restrict__ off, const int* __restrict__ nb, const long long* __restrict__ luoff,
                  const double* __restrict__ inv_all, const T* __restrict__ bin, T* __restrict__ xout) {
  const int k = blockIdx.x;
  const int n = nb[k], o = off[k];
  const double* inv = inv_all + luoff[k];
  const int i = threadIdx.x;
  if (i < n) {
    double y = 0.0;
    for (int j = 0; j < n; ++j) y = __dadd_rn(y, __dmul_rn(inv[j * n + i], (double)bin[o + j]));
    xout[o + i] = (T)y;
  }
}

template <typename T>
__global__ void k_lu_solve_batch(const int* __restrict__ off, const int* __restrict__ nb,
                                 const long long* __restrict__ luoff, const int* __restrict__ poff,
                                 const double* __restrict__ lu_all, const int* __restrict__ piv_all,
                                 const T* __restrict__ bin, T* __restrict__ xout) {
  extern __shared__ double shb[];
  const int k = blockIdx.x;
  const int n = nb[k];
  const double* __restrict__ a = lu_all + luoff[k];
  const int* __restrict__ piv = piv_all + poff[k];
  const T* __restrict__ b = bin + off[k];
  T* __restrict__ x = xout + off[k];
  double* y = shb;
  for (int i = threadIdx.x; i < n; i += blockDim.x) y[i] = (double)b[i];
  __syncthreads();
  if (threadIdx.x == 0)
    for (int j = 0; j < n; ++j) {
      const int p = piv[j];
      if (p != j) {
        const double t = y[j];
        y[j] = y[p];
        y[p] = t;
      }
    }
  __syncthreads();
  for (int j = 0; j < n; ++j) {
    const double yj = y[j];
    if (yj != 0.0)
      for (int i = j + 1 + threadIdx.x; i < n; i += blockDim.x)
        y[i] = __dsub_rn(y[i], __dmul_rn(yj, a[(size_t)j * n + i]));
    __syncthreads();
  }
  for (int j = n - 1; j >= 0; --j) {
    if (threadIdx.x == 0 && y[j] != 0.0) y[j] = __ddiv_rn(y[j], a[(size_t)j * n + j]);
    __syncthreads();
    const double yj = y[j];
    if (yj != 0.0)
      for (int i = threadIdx.x; i < j; i += blockDim.x)
        y[i] = __dsub_rn(y[i], __dmul_rn(yj, a[(size_t)j * n + i]));
    __syncthreads();
  }
  for (int i = threadIdx.x; i < n; i += blockDim.x) x[i] = (T)y[i];
}

// The same coarsest solves with one warp per system (one warp per block),
// warp barriers between the substitution steps in place of block barriers,
// and the system's factors first copied into shared memory (coalesced), so
// that the 2n dependent steps read them there rather than from L2; the
// operation order is k_lu_solve's.  Dynamic shared memory: (maxn + maxn²)
// doubles.
template <typename T>
__global__ void __launch_bounds__(32)
k_lu_solve_batch_warp(const int* __restrict__ off, const int* __restrict__ nb, const long long* __restrict__ luoff,
                      const int* __restrict__ poff, const double* __restrict__ lu_all,
                      const int* __restrict__ piv_all, const T* __restrict__ bin, T* __restrict__ xout, int maxn) {
  extern __shared__ double shw[];
  const int lane = threadIdx.x;
  const int k = blockIdx.x;
  const int n = nb[k];
  const double* __restrict__ ag = lu_all + luoff[k];
  const int* __restrict__ piv = piv_all + poff[k];
  const T* __restrict__ b = bin + off[k];
  T* __restrict__ x = xout + off[k];
  double* y = shw;
  double* a = shw + maxn;
  for (int t = lane; t < n * n; t += 32) a[t] = ag[t];
  for (int i = lane; i < n; i += 32) y[i] = (double)b[i];
  __syncwarp();
  if (lane == 0)
    for (int j = 0; j < n; ++j) {
      const int p = piv[j];
      if (p != j) {
        const double t = y[j];
        y[j] = y[p];
        y[p] = t;
      }
    }
  __syncwarp();
  for (int j = 0; j < n; ++j) {
    const double yj = y[j];
    if (yj != 0.0)
      for (int i = j + 1 + lane; i < n; i += 32) y[i] = __dsub_rn(y[i], __dmul_rn(yj, a[(size_t)j * n + i]));
    __syncwarp();
  }
  for (int j = n - 1; j >= 0; --j) {
    if (lane == 0 && y[j] != 0.0) y[j] = __ddiv_rn(y[j], a[(size_t)j * n + j]);
    __syncwarp();
    const double yj = y[j];
    if (yj != 0.0)
      for (int i = lane; i < j; i += 32) y[i] = __dsub_rn(y[i], __dmul_rn(yj, a[(size_t)j * n + i]));
    __syncwarp();
  }
  for (int i = lane; i < n; i += 32) x[i] = (T)y[i];
}

// Per-segment dot products, deterministic: blockIdx.y = segment, blocks
// along x stride its rows; partials[s * gridDim.x + bx]; then
// k_seg_dot_final sums each segment's partials in block order (one warp per
// segment) into out[s].
template <typename TA, typename TB>
__global__ void __launch_bounds__(kBlock)
k_seg_dot_part(const int* __restrict__ seg_off, const TA* __restrict__ a, const TB* __restrict__ b,
               double* __restrict__ partials) {
  const int s = blockIdx.y;
  const int lo = seg_off[s], hi = seg_off[s + 1];
  double v = 0.0;
  for (int i = lo + blockIdx.x * blockDim.x + threadIdx.x; i < hi; i += gridDim.x * blockDim.x)
    v = fma((double)a[i], (double)b[i], v);
  v = block_sum(v);
  if (threadIdx.x == 0) partials[(size_t)s * gridDim.x + blockIdx.x] = v;
}

__global__ void k_seg_dot_final(int nseg, int nparts, const double* __restrict__ partials,
                                double* __restrict__ out) {
  const int s = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (s >= nseg) return;
  double v = 0.0;
  for (int k = lane; k < nparts; k += 32) v += partials[(size_t)s * nparts + k];
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if (lane == 0) out[s] = v;
}

// Segmented PCG scalars (one thread per segment), from the dot products
// in `dots` (per segment: [rz, rz_old, pq, rr, bb]) and the convergence
// flags: alpha (0 once converged), beta, and, at the update step, the
// convergence test rr < tol^2 bb with the iteration count.
struct SegScal {
  double* rz;
  double* rzold;
  double* pq;
  double* rr;
  double* bb;
  double* alpha;
  double* beta;
  int* done;   // 1 once the segment has converged
  int* iters;  // iterations of each segment
};
__global__ void k_seg_alpha(int nseg, SegScal sc) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nseg) return;
  sc.alpha[s] = (sc.done[s] || sc.pq[s] == 0.0) ? 0.0 : sc.rz[s] / sc.pq[s];
}
__global__ void k_seg_beta(int nseg, SegScal sc, double tol2, int* ndone) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nseg) return;
  if (!sc.done[s]) {
    sc.iters[s] += 1;
    if (sc.rr[s] < tol2 * sc.bb[s]) {
      sc.done[s] = 1;
      atomicAdd(ndone, 1);
    }
  }
  sc.beta[s] = (sc.done[s] || sc.rzold[s] == 0.0) ? 0.0 : sc.rz[s] / sc.rzold[s];
}

// p = z + beta_s p (z of the cycle's type), per row's segment.
template <typename TZ>
__global__ void k_seg_dir(int n, const int* __restrict__ seg, const TZ* __restrict__ z,
                          const double* __restrict__ beta, double* __restrict__ p) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    p[i] = (double)z[i] + beta[seg[i]] * p[i];
}
// x += alpha_s p; r -= alpha_s q; optional FP32 copy of r.
template <typename TR32>
__global__ void k_seg_update(int n, const int* __restrict__ seg, const double* __restrict__ alpha,
                             const double* __restrict__ p, const double* __restrict__ q,
                             double* __restrict__ x, double* __restrict__ r, TR32* __restrict__ r32) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double a = alpha[seg[i]];
    x[i] = fma(a, p[i], x[i]);
    const double ri = fma(-a, q[i], r[i]);
    r[i] = ri;
    if (r32) r32[i] = (TR32)ri;
  }
}

}  // namespace kern
}  // namespace dr
