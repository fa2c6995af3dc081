// Block (multi-right-hand-side) solves: k <= 32 systems with the same
// operator, vectors stored row-major as n x k (column c of row i at
// i*k + c).  Every level matrix is read once per block product for all k
// columns, which turns the bandwidth of k separate solves (k passes over
// the matrices) into one pass plus the vector traffic.
//
// Kernels: one warp per row, lane c works on column c.  The warp reads 32
// of the row's entries at a time (coalesced) and hands them to every lane
// by shuffle; each lane gathers x[col][lane] (the k columns of a row are
// contiguous, so the warp's gather is one contiguous span) and sums its
// row in column order with separately rounded products and sums, as the
// reference's loops do.  Deterministic column dot products: per-warp
// partials reduced in a fixed order.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <mutex>
#include <string>
#include <type_traits>
#include <unordered_map>
#include <vector>

#include "dr_device.h"

namespace dr {

namespace {

constexpr int kBlock = 256;
constexpr int kWarps = kBlock / 32;

__device__ __forceinline__ double rn_mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float rn_mul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double rn_add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float rn_add(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ double rn_sub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ float rn_sub(float a, float b) { return __fsub_rn(a, b); }

enum : int { BM_STORE = 0, BM_RESID = 1, BM_JACOBI = 2, BM_ADDTO = 3, BM_CORRECT = 4 };

// Y = A X (STORE), Y = B - A X (RESID), Y = X + (omega d)(B - A X)
// (JACOBI), Y += A X (ADDTO, A = P), Y = Y + (omega d) B + A X (CORRECT:
// A = Q = P - omega D^-1 (A P), B = the residual of Y formed on the way
// down, X = the coarse correction; the fused correction and first
// post-smoothing step), for k columns.
template <typename TA, typename T, int MODE>
__global__ void __launch_bounds__(kBlock)
k_spmm(int nrows, int k, const int* __restrict__ rp, const int* __restrict__ ci, const TA* __restrict__ av,
       const T* __restrict__ X, const T* __restrict__ B, const T* __restrict__ dinv, T omega, T* Y) {
  const int lane = threadIdx.x & 31;
  const bool col = lane < k;
  const long long nw = (long long)gridDim.x * kWarps;
  for (long long r0 = (long long)blockIdx.x * kWarps + (threadIdx.x >> 5); r0 < nrows; r0 += nw) {
    const int row = (int)r0;
    const int rs = rp[row], re = rp[row + 1];
    T acc = T(0);
    if (col) {
      if (MODE == BM_ADDTO) acc = Y[(size_t)row * k + lane];
      if (MODE == BM_JACOBI) acc = B[(size_t)row * k + lane];
      if (MODE == BM_CORRECT)
        acc = rn_add(Y[(size_t)row * k + lane], rn_mul(rn_mul(omega, dinv[row]), B[(size_t)row * k + lane]));
    }
    for (int k0 = rs; k0 < re; k0 += 32) {
      const int my = k0 + lane;
      const int cj = my < re ? ci[my] : 0;
      const T vj = my < re ? (T)av[my] : T(0);
      const int cnt = min(32, re - k0);
      for (int j = 0; j < cnt; ++j) {
        const int c = __shfl_sync(0xffffffffu, cj, j);
        const T v = __shfl_sync(0xffffffffu, vj, j);
        if (col) {
          const T p = rn_mul(v, X[(size_t)c * k + lane]);
          acc = (MODE == BM_JACOBI) ? rn_sub(acc, p) : rn_add(acc, p);
        }
      }
    }
    if (col) {
      const size_t o = (size_t)row * k + lane;
      if (MODE == BM_RESID) Y[o] = rn_sub(B[o], acc);
      else if (MODE == BM_JACOBI) Y[o] = rn_add(X[o], rn_mul(rn_mul(omega, dinv[row]), acc));
      else Y[o] = acc;
    }
  }
}

// The same products with vector gathers, when each row's k columns split
// into pieces of V = 4 consecutive columns (k a multiple of 4, 16-byte
// aligned vectors; a piece is one 16-byte load in FP32, two in FP64): TPR
// threads per row, each owning one piece, 32 / TPR rows per warp.  A row's
// threads pass its (column, value) pairs round and gather one piece of X
// per entry, so an entry costs a few instructions per piece instead of
// shuffles and a scalar gather per column (four FP64 columns per thread
// rather than two took the 96^3 x 32 FP64 block solve from 97 to 90 ms).
// Each column is summed in column order with separately rounded products
// and sums: the results equal k_spmm's bit for bit.
template <typename T>
struct VecPiece;
template <>
struct VecPiece<float> {
  using type = float4;
  static constexpr int V = 4;
  __device__ static void get(const type& a, float* o) { o[0] = a.x; o[1] = a.y; o[2] = a.z; o[3] = a.w; }
  __device__ static type make(const float* o) { return make_float4(o[0], o[1], o[2], o[3]); }
};
struct __align__(16) double2x2 {
  double2 lo, hi;
};
template <>
struct VecPiece<double> {  // four FP64 columns: two 16-byte loads
  using type = double2x2;
  static constexpr int V = 4;
  __device__ static void get(const type& a, double* o) { o[0] = a.lo.x; o[1] = a.lo.y; o[2] = a.hi.x; o[3] = a.hi.y; }
  __device__ static type make(const double* o) {
    return double2x2{make_double2(o[0], o[1]), make_double2(o[2], o[3])};
  }
};

// Per-block partial sums of each column of a vector-layout kernel (TPR
// threads per row, V consecutive columns per thread): every thread's V sums
// go to shared memory, then thread c < k adds those of the threads owning
// column c, in thread order, into part[block * 32 + c] (deterministic for
// a given grid; k_bl_dot_final adds the blocks).
template <int TPR, int V>
__device__ __forceinline__ void block_col_partials(const double (&s)[V], int k, double* __restrict__ part) {
  __shared__ double red[kBlock * V];
#pragma unroll
  for (int q = 0; q < V; ++q) red[threadIdx.x * V + q] = s[q];
  __syncthreads();
  const int c = threadIdx.x;
  if (c < k) {
    const int g = c / V, q = c % V;
    double t = 0.0;
    for (int u = g; u < kBlock; u += TPR) t += red[u * V + q];
    part[(size_t)blockIdx.x * 32 + c] = t;
  }
}

// With `part` (STORE mode), also the column partials of X_row . Y_row (the
// p . q of block CG).
template <typename TA, typename T, int MODE, int TPR>
__global__ void __launch_bounds__(kBlock)
k_spmm_vec(int nrows, int k, const int* __restrict__ rp, const int* __restrict__ ci,
           const TA* __restrict__ av, const T* __restrict__ X, const T* __restrict__ B,
           const T* __restrict__ dinv, T omega, T* Y, double* __restrict__ part) {
  using VV = VecPiece<T>;
  using VT = typename VV::type;
  constexpr int V = VV::V;
  constexpr int RPW = 32 / TPR;
  const int lane = threadIdx.x & 31;
  const int sub = lane % TPR;
  const int c0 = sub * V;           // first column of this thread
  const bool act = c0 < k;
  const int cg = act ? c0 : k - V;  // lanes past k read (and drop) the last piece
  // the TPR lanes of one row (a row's lanes always run together)
  const unsigned gmask = TPR == 32 ? 0xffffffffu : (((1u << TPR) - 1u) << (lane & ~(TPR - 1)));
  double dsum[V];
#pragma unroll
  for (int q = 0; q < V; ++q) dsum[q] = 0.0;
  const long long w = (long long)blockIdx.x * kWarps + (threadIdx.x >> 5);
  const long long nw = (long long)gridDim.x * kWarps;
  for (long long r = w * RPW + lane / TPR; r < nrows; r += nw * RPW) {
    const int row = (int)r;
    const int rs = rp[row], re = rp[row + 1];
    const size_t o = (size_t)row * k + cg;
    T acc[V];
    if (MODE == BM_ADDTO) VV::get(*reinterpret_cast<const VT*>(Y + o), acc);
    else if (MODE == BM_JACOBI) VV::get(*reinterpret_cast<const VT*>(B + o), acc);
    else if (MODE == BM_CORRECT) {
      T yv[V], bv[V];
      VV::get(*reinterpret_cast<const VT*>(Y + o), yv);
      VV::get(*reinterpret_cast<const VT*>(B + o), bv);
      const T sc = rn_mul(omega, dinv[row]);
#pragma unroll
      for (int q = 0; q < V; ++q) acc[q] = rn_add(yv[q], rn_mul(sc, bv[q]));
    } else
#pragma unroll
      for (int q = 0; q < V; ++q) acc[q] = T(0);
    // the row's lanes load up to TPR (column, value) pairs at once and pass
    // them round; the X pieces of 4 entries are gathered before the first
    // is used (slots past the row's end repeat its last entry)
    for (int k0 = rs; k0 < re; k0 += TPR) {
      const int my = k0 + sub;
      const int cj = my < re ? ci[my] : 0;
      const T vj = my < re ? (T)av[my] : T(0);
      const int cnt = min(TPR, re - k0);
      for (int j0 = 0; j0 < cnt; j0 += 4) {
        T vv[4];
        VT xs[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          const int jj = min(j0 + u, cnt - 1);
          const int c = __shfl_sync(gmask, cj, jj, TPR);
          vv[u] = __shfl_sync(gmask, vj, jj, TPR);
          xs[u] = *reinterpret_cast<const VT*>(X + (size_t)c * k + cg);
        }
#pragma unroll
        for (int u = 0; u < 4; ++u)
          if (j0 + u < cnt) {
            T xv[V];
            VV::get(xs[u], xv);
#pragma unroll
            for (int q = 0; q < V; ++q) {
              const T p = rn_mul(vv[u], xv[q]);
              acc[q] = (MODE == BM_JACOBI) ? rn_sub(acc[q], p) : rn_add(acc[q], p);
            }
          }
      }
    }
    if (!act) continue;
    T out[V];
    if (MODE == BM_RESID) {
      T bv[V];
      VV::get(*reinterpret_cast<const VT*>(B + o), bv);
#pragma unroll
      for (int q = 0; q < V; ++q) out[q] = rn_sub(bv[q], acc[q]);
    } else if (MODE == BM_JACOBI) {
      T xo[V];
      VV::get(*reinterpret_cast<const VT*>(X + o), xo);
      const T sc = rn_mul(omega, dinv[row]);
#pragma unroll
      for (int q = 0; q < V; ++q) out[q] = rn_add(xo[q], rn_mul(sc, acc[q]));
    } else {
#pragma unroll
      for (int q = 0; q < V; ++q) out[q] = acc[q];
    }
    *reinterpret_cast<VT*>(Y + o) = VV::make(out);
    if (MODE == BM_STORE && part) {
      T xo[V];
      VV::get(*reinterpret_cast<const VT*>(X + o), xo);
#pragma unroll
      for (int q = 0; q < V; ++q) dsum[q] += (double)xo[q] * (double)out[q];
    }
  }
  if (MODE == BM_STORE && part) block_col_partials<TPR, V>(dsum, k, part);
}

// X += alpha_c P, R -= alpha_c Q, optionally R32 = (float) R, and the
// column partials of R . R; vector layout (TPR threads per row, 2 columns
// per thread).
template <int TPR>
__global__ void __launch_bounds__(kBlock)
k_bl_update_vec(int n, int k, const double* __restrict__ alpha, double* __restrict__ X,
                double* __restrict__ R, const double* __restrict__ P, const double* __restrict__ Q,
                float* __restrict__ R32, double* __restrict__ part) {
  constexpr int RPW = 32 / TPR;
  const int lane = threadIdx.x & 31;
  const int c0 = (lane % TPR) * 2;
  const bool act = c0 < k;
  double s[2] = {0.0, 0.0};
  const double a0 = act ? alpha[c0] : 0.0, a1 = act ? alpha[c0 + 1] : 0.0;
  const long long w = (long long)blockIdx.x * kWarps + (threadIdx.x >> 5);
  const long long nw = (long long)gridDim.x * kWarps;
  for (long long r = w * RPW + lane / TPR; act && r < n; r += nw * RPW) {
    const size_t o = (size_t)r * k + c0;
    double2 x = *reinterpret_cast<const double2*>(X + o);
    double2 rr = *reinterpret_cast<const double2*>(R + o);
    const double2 p = *reinterpret_cast<const double2*>(P + o);
    const double2 q = *reinterpret_cast<const double2*>(Q + o);
    x.x += a0 * p.x;
    x.y += a1 * p.y;
    rr.x = rr.x - a0 * q.x;
    rr.y = rr.y - a1 * q.y;
    *reinterpret_cast<double2*>(X + o) = x;
    *reinterpret_cast<double2*>(R + o) = rr;
    if (R32) *reinterpret_cast<float2*>(R32 + o) = make_float2((float)rr.x, (float)rr.y);
    s[0] += rr.x * rr.x;
    s[1] += rr.y * rr.y;
  }
  block_col_partials<TPR, 2>(s, k, part);
}

// Z = (double) z and the column partials of R . Z (the preconditioned
// residual handed back to block CG); vector layout, 2 columns per thread.
template <typename TS, int TPR>
__global__ void __launch_bounds__(kBlock)
k_bl_take_z(int n, int k, const TS* __restrict__ z, const double* __restrict__ R, double* __restrict__ Z,
            double* __restrict__ part) {
  constexpr int RPW = 32 / TPR;
  const int lane = threadIdx.x & 31;
  const int c0 = (lane % TPR) * 2;
  const bool act = c0 < k;
  double s[2] = {0.0, 0.0};
  const long long w = (long long)blockIdx.x * kWarps + (threadIdx.x >> 5);
  const long long nw = (long long)gridDim.x * kWarps;
  for (long long r = w * RPW + lane / TPR; act && r < n; r += nw * RPW) {
    const size_t o = (size_t)r * k + c0;
    const double z0 = (double)z[o], z1 = (double)z[o + 1];
    const double2 rr = *reinterpret_cast<const double2*>(R + o);
    *reinterpret_cast<double2*>(Z + o) = make_double2(z0, z1);
    s[0] += rr.x * z0;
    s[1] += rr.y * z1;
  }
  block_col_partials<TPR, 2>(s, k, part);
}

// X = A_c^-1 B for k columns (n x k row-major), A_c^-1 column-major: one
// thread per entry, its row of the inverse summed in column order.
template <typename T>
__global__ void __launch_bounds__(kBlock)
k_bl_inv(int n, int k, const double* __restrict__ inv, const T* __restrict__ B, T* __restrict__ X) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n * k) return;
  const int i = e / k, c = e % k;
  double y = 0.0;
  for (int j = 0; j < n; ++j) y = __dadd_rn(y, __dmul_rn(inv[j * n + i], (double)B[(size_t)j * k + c]));
  X[e] = (T)y;
}

template <typename T>
__global__ void k_bl_fill(long long n, T* __restrict__ x) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    x[i] = T(0);
}

// X = (omega d) B  (first Jacobi step from a zero iterate)
template <typename T>
__global__ void k_bl_jz(int n, int k, const T* __restrict__ B, const T* __restrict__ dinv, T omega,
                        T* __restrict__ X) {
  const long long tot = (long long)n * k;
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < tot;
       e += (long long)gridDim.x * blockDim.x)
    X[e] = rn_mul(rn_mul(omega, dinv[e / k]), B[e]);
}

// Coarsest solve for k columns with the dgetf2 factors (dgetrs order),
// one thread per column, its vector in shared memory (n * k doubles of
// dynamic shared memory; every thread reads the same factor entry at a
// time, a broadcast).  With `stage` the factors are first copied into
// shared memory after the vectors (n * n more doubles), so the
// substitutions' chains of dependent steps read shared memory instead of
// global memory.
template <typename T>
__global__ void k_bl_lu(int n, int k, const double* __restrict__ lu_g, const int* __restrict__ piv,
                        const T* __restrict__ B, T* __restrict__ X, int stage) {
  extern __shared__ double ysm[];
  const double* lu = lu_g;
  if (stage) {
    double* ls = ysm + (size_t)n * k;
    for (int e = threadIdx.x; e < n * n; e += blockDim.x) ls[e] = lu_g[e];
    __syncthreads();
    lu = ls;
  }
  const int c = threadIdx.x;
  if (c >= k) return;
  double* y = ysm + (size_t)c;  // element i at y[i * k]
  for (int i = 0; i < n; ++i) y[(size_t)i * k] = (double)B[(size_t)i * k + c];
  for (int j = 0; j < n; ++j) {
    const int p = piv[j];
    if (p != j) {
      const double t = y[(size_t)j * k];
      y[(size_t)j * k] = y[(size_t)p * k];
      y[(size_t)p * k] = t;
    }
  }
  for (int j = 0; j < n; ++j) {
    const double yj = y[(size_t)j * k];
    if (yj != 0.0)
      for (int i = j + 1; i < n; ++i)
        y[(size_t)i * k] = __dsub_rn(y[(size_t)i * k], __dmul_rn(yj, lu[(size_t)j * n + i]));
  }
  for (int j = n - 1; j >= 0; --j) {
    if (y[(size_t)j * k] != 0.0) y[(size_t)j * k] = __ddiv_rn(y[(size_t)j * k], lu[(size_t)j * n + j]);
    const double yj = y[(size_t)j * k];
    if (yj != 0.0)
      for (int i = 0; i < j; ++i)
        y[(size_t)i * k] = __dsub_rn(y[(size_t)i * k], __dmul_rn(yj, lu[(size_t)j * n + i]));
  }
  for (int i = 0; i < n; ++i) X[(size_t)i * k + c] = (T)y[(size_t)i * k];
}

// The same solve with one warp per column for n <= 64: the factors in
// shared memory (n * n doubles), each lane holding y_i for i = lane and
// lane + 32 in registers; at step j the lane owning y_j hands it to the
// others by shuffle.  Every y_i sees the same operations in the same order
// as in k_bl_lu (bit-identical results); the n steps of each substitution
// cost a shuffle and one update per lane instead of a sequential sweep.
template <typename T>
__global__ void __launch_bounds__(1024)
k_bl_lu_warp(int n, int k, const double* __restrict__ lu_g, const int* __restrict__ piv,
             const T* __restrict__ B, T* __restrict__ X) {
  extern __shared__ double lsm[];  // n * n factors, then n per warp (the pivoted column)
  double* lu = lsm;
  for (int e = threadIdx.x; e < n * n; e += blockDim.x) lu[e] = lu_g[e];
  __syncthreads();
  const int c = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (c >= k) return;  // whole warps leave; no block barrier follows
  double* ys = lsm + (size_t)n * n + (size_t)c * n;
  for (int i = lane; i < n; i += 32) ys[i] = (double)B[(size_t)i * k + c];
  __syncwarp();
  if (lane == 0)
    for (int j = 0; j < n; ++j) {
      const int p = piv[j];
      if (p != j) {
        const double t = ys[j];
        ys[j] = ys[p];
        ys[p] = t;
      }
    }
  __syncwarp();
  double y0 = lane < n ? ys[lane] : 0.0, y1 = lane + 32 < n ? ys[lane + 32] : 0.0;
  for (int j = 0; j < n; ++j) {  // L y = b (unit diagonal)
    const double yj = __shfl_sync(0xffffffffu, j < 32 ? y0 : y1, j & 31);
    if (yj != 0.0) {
      if (lane > j && lane < n) y0 = __dsub_rn(y0, __dmul_rn(yj, lu[(size_t)j * n + lane]));
      if (lane + 32 > j && lane + 32 < n) y1 = __dsub_rn(y1, __dmul_rn(yj, lu[(size_t)j * n + lane + 32]));
    }
  }
  for (int j = n - 1; j >= 0; --j) {  // U x = y
    const double d = lu[(size_t)j * n + j];
    if (lane == (j & 31)) {
      if (j < 32) {
        if (y0 != 0.0) y0 = __ddiv_rn(y0, d);
      } else if (y1 != 0.0) {
        y1 = __ddiv_rn(y1, d);
      }
    }
    const double yj = __shfl_sync(0xffffffffu, j < 32 ? y0 : y1, j & 31);
    if (yj != 0.0) {
      if (lane < j) y0 = __dsub_rn(y0, __dmul_rn(yj, lu[(size_t)j * n + lane]));
      if (lane + 32 < j) y1 = __dsub_rn(y1, __dmul_rn(yj, lu[(size_t)j * n + lane + 32]));
    }
  }
  if (lane < n) X[(size_t)lane * k + c] = (T)y0;
  if (lane + 32 < n) X[(size_t)(lane + 32) * k + c] = (T)y1;
}

// Column dot products a_c . b_c: per-block partials part[block][c]
// (warps take rows, lane c accumulates column c, warps summed in order).
__global__ void __launch_bounds__(kBlock)
k_bl_dot_part(int n, int k, const double* __restrict__ a, const double* __restrict__ b,
              double* __restrict__ part) {
  __shared__ double ws[kWarps][32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  double s = 0.0;
  if (lane < k)
    for (long long r = (long long)blockIdx.x * kWarps + w; r < n; r += (long long)gridDim.x * kWarps) {
      const size_t o = (size_t)r * k + lane;
      s += a[o] * b[o];
    }
  ws[w][lane] = s;
  __syncthreads();
  if (threadIdx.x < 32) {
    double t = 0.0;
    for (int q = 0; q < kWarps; ++q) t += ws[q][threadIdx.x];
    if (threadIdx.x < k) part[(size_t)blockIdx.x * 32 + threadIdx.x] = t;
  }
}

// Column totals of the partials: 32 groups of blocks per column (strided),
// then the groups in order — 1024 threads, a fixed summation order.
__global__ void __launch_bounds__(1024)
k_bl_dot_final(int nblocks, int k, const double* __restrict__ part, double* __restrict__ out) {
  __shared__ double g[32][33];
  const int c = threadIdx.x & 31, w = threadIdx.x >> 5;
  double t = 0.0;
  if (c < k)
    for (int q = w; q < nblocks; q += 32) t += part[(size_t)q * 32 + c];
  g[w][c] = t;
  __syncthreads();
  if (w == 0 && c < k) {
    double s = 0.0;
    for (int q = 0; q < 32; ++q) s += g[q][c];
    out[c] = s;
  }
}

// X += alpha_c P, R -= alpha_c Q (and R32 = (float) R when given)
__global__ void k_bl_update(int n, int k, const double* __restrict__ alpha, double* __restrict__ X,
                            double* __restrict__ R, const double* __restrict__ P, const double* __restrict__ Q,
                            float* __restrict__ R32) {
  const long long tot = (long long)n * k;
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < tot;
       e += (long long)gridDim.x * blockDim.x) {
    const double a = alpha[e % k];
    X[e] += a * P[e];
    const double r = R[e] - a * Q[e];
    R[e] = r;
    if (R32) R32[e] = (float)r;
  }
}

// P = Z + beta_c P
__global__ void k_bl_dir(int n, int k, const double* __restrict__ beta, const double* __restrict__ Z,
                         double* __restrict__ P) {
  const long long tot = (long long)n * k;
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < tot;
       e += (long long)gridDim.x * blockDim.x)
    P[e] = Z[e] + beta[e % k] * P[e];
}

template <typename TS, typename TD>
__global__ void k_bl_convert(long long n, const TS* __restrict__ s, TD* __restrict__ d) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    d[i] = (TD)s[i];
}

int grid_for(long long work, int max_grid) {
  return (int)std::max<long long>(1, std::min<long long>((work + kBlock - 1) / kBlock, max_grid));
}

int warp_grid(int rows, int max_grid) {
  return std::max(1, std::min((rows + kWarps - 1) / kWarps, max_grid));
}

bool aligned16(const void* p) { return p == nullptr || (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

// Threads per row for `per_row` vector pieces (a power of two up to 16).
int tpr_for(int per_row) {
  return per_row <= 1 ? 1 : per_row <= 2 ? 2 : per_row <= 4 ? 4 : per_row <= 8 ? 8 : 16;
}

// Blocks of a vector-layout kernel f (32 / tpr rows per warp): enough for
// the rows, at most one wave of resident blocks (max_grid allows 8 blocks
// of 256 threads per SM; registers may allow fewer, queried once per
// kernel), or nb_cap blocks per SM when that is smaller (0: no cap).
int vec_grid(const void* f, int nrows, int tpr, int max_grid, int nb_cap = 0) {
  static std::mutex mu;
  static std::unordered_map<const void*, int> occ;
  int nb;
  {
    std::lock_guard<std::mutex> lk(mu);
    auto it = occ.find(f);
    if (it == occ.end()) {
      nb = 0;
      DR_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, f, kBlock, 0));
      nb = std::max(1, std::min(nb, 8));
      occ.emplace(f, nb);
    } else {
      nb = it->second;
    }
  }
  if (nb_cap > 0) nb = std::min(nb, nb_cap);
  const int rows_per_block = kWarps * (32 / tpr);
  return std::max(1, std::min((nrows + rows_per_block - 1) / rows_per_block, max_grid / 8 * nb));
}

// Block product on `nrows` rows: the vector-gather kernel when the rows'
// k columns split into pieces of 4, else one warp per row.  With `part`
// (STORE mode only) the vector kernel also leaves the column partials of
// X_row . Y_row there; returns its grid (the number of partials per
// column), or 0 when the one-warp-per-row kernel ran (no partials).
// `sh` overrides the vector kernel's threads per row (a power of two from
// the default up to 16; the extra threads help load a row's entries and
// drop their sums) and caps its blocks per SM.  Every shape gives the same
// values: each column of a row is summed by one thread in column order.
template <typename TA, typename T, int MODE>
int spmm(cudaStream_t st, int max_grid, int nrows, int k, const int* rp, const int* ci, const TA* av,
         const T* X, const T* B, const T* dinv, T omega, T* Y, double* part = nullptr,
         BlockShape sh = {}) {
  constexpr int V = VecPiece<T>::V;
  if (k % V == 0 && aligned16(X) && aligned16(B) && aligned16(Y)) {
    const int t0 = tpr_for(k / V);
    const int tpr = (sh.tpr >= t0 && sh.tpr <= 16 && (sh.tpr & (sh.tpr - 1)) == 0) ? sh.tpr : t0;
    int grid = 1;
    switch (tpr) {
#define DR_SPMM_VEC(t)                                                                            \
  case t: {                                                                                       \
    auto kf = k_spmm_vec<TA, T, MODE, t>;                                                         \
    grid = vec_grid((const void*)kf, nrows, t, max_grid, sh.nb);                                  \
    kf<<<grid, kBlock, 0, st>>>(nrows, k, rp, ci, av, X, B, dinv, omega, Y, part);                \
    break;                                                                                        \
  }
      DR_SPMM_VEC(1) DR_SPMM_VEC(2) DR_SPMM_VEC(4) DR_SPMM_VEC(8) DR_SPMM_VEC(16)
#undef DR_SPMM_VEC
    }
    return grid;
  }
  k_spmm<TA, T, MODE><<<warp_grid(nrows, max_grid), kBlock, 0, st>>>(nrows, k, rp, ci, av, X, B, dinv, omega, Y);
  return 0;
}

}  // namespace

template <>
DevHier::BlockVecs<float>& DevHier::bvecs<float>(int l) {
  return blk32_[l];
}
template <>
DevHier::BlockVecs<double>& DevHier::bvecs<double>(int l) {
  return blk64_[l];
}

void DevHier::ensure_block(int k) {
  if (k <= blk_k_) return;
  const int nl = nlevels();
  blk32_.assign(nl, BlockVecs<float>{});
  blk64_.assign(nl, BlockVecs<double>{});
  for (int l = 0; l < nl; ++l) {
    const size_t m = (size_t)L_[l].A.n * k;
    blk32_[l] = BlockVecs<float>{alloc<float>(m), alloc<float>(m), alloc<float>(m), alloc<float>(m)};
    blk64_[l] = BlockVecs<double>{alloc<double>(m), alloc<double>(m), alloc<double>(m), alloc<double>(m)};
  }
  const size_t mc = (size_t)std::max(nc_, 1) * k;
  bcb32_ = alloc<float>(mc);
  bcx32_ = alloc<float>(mc);
  bcb64_ = alloc<double>(mc);
  bcx64_ = alloc<double>(mc);
  const size_t m0 = (size_t)n0_ * k;
  for (auto& p : bpcg_) p = alloc<double>(m0);
  for (auto& p : bpcg32_) p = alloc<float>(m0);
  bpart_ = alloc<double>((size_t)max_grid_ * 32);
  bdev_ = alloc<double>(8 * 32);
  if (!bhost_) DR_CK(cudaMallocHost(&bhost_, 8 * 32 * sizeof(double)));
  blk_k_ = k;
}

BlockShape DevHier::shape_of(const void* rp, int mode, int bytes, int k) const {
  if (!btune_on_) return BlockShape{};
  if (bforce_tpr_) return BlockShape{bforce_tpr_, 0};
  auto it = bshape_.find(ShapeKey{rp, mode, bytes, k});
  return it == bshape_.end() ? BlockShape{} : it->second;
}

// Picks the launch shape of each product of the block cycle (threads per
// row: 32 / tpr rows per warp, and blocks per SM) by timing the candidates
// on this hierarchy's own matrices, once per k and precision.  A candidate
// replaces the default only when it is at least 3% faster.  The candidates
// run on the block buffers, zeroed first, before a solve uses them, and
// every shape gives the same values, so tuning changes no result.  The
// FP64 product with A that also forms p.q keeps the default shape, so that
// the partial sums, and with them every dot product, do not depend on the
// timing.  The environment variable DRAUGR_B200_BLOCK_TUNE, read at each
// block solve, set to 0 keeps the default shapes and set to 2, 4, 8 or 16
// forces that many threads per row (at least the default) on every product
// of the cycle, without timing.
template <typename T>
void DevHier::tune_block(int k, int verbose) {
  btune_on_ = true;
  bforce_tpr_ = 0;
  if (const char* env = std::getenv("DRAUGR_B200_BLOCK_TUNE"); env && *env) {
    const int v = std::atoi(env);
    if (v == 0) {
      btune_on_ = false;
      return;
    }
    if (v == 2 || v == 4 || v == 8 || v == 16) {
      bforce_tpr_ = v;
      return;
    }
  }
  constexpr int V = VecPiece<T>::V;
  if (k % V != 0) return;  // the one-warp-per-row kernel has no shape to pick
  if (!btuned_.insert({k, (int)sizeof(T)}).second) return;
  const int t0 = tpr_for(k / V);
  std::vector<BlockShape> cand;
  for (int t = t0; t <= 16; t *= 2)
    for (int nb = 0; nb <= 2; nb += 2) cand.push_back(BlockShape{t, nb});
  constexpr int kReps = 3;
  cudaEvent_t e0, e1;
  DR_CK(cudaEventCreate(&e0));
  DR_CK(cudaEventCreate(&e1));
  static const char* kOpName[5] = {"A x (Jacobi)", "b - A x", "P^T r", "x + P x_c", "x + Q x_c"};
  static const int kOpMode[5] = {BM_JACOBI, BM_RESID, BM_STORE, BM_ADDTO, BM_CORRECT};
  const int nl = nlevels();
  for (int l = 0; l < nl; ++l) {
    DevLevel& L = L_[l];
    BlockVecs<T>& W = bvecs<T>(l);
    const size_t m = (size_t)L.A.n * k;
    T* const bufs[4] = {W.x, W.t, W.b, W.r};
    for (T* p : bufs) DR_CK(cudaMemsetAsync(p, 0, m * sizeof(T), st_));
    const bool last = (l + 1 == nl);
    T* bc = last ? (sizeof(T) == 8 ? (T*)bcb64_ : (T*)bcb32_) : bvecs<T>(l + 1).b;
    T* xc = last ? (sizeof(T) == 8 ? (T*)bcx64_ : (T*)bcx32_) : bvecs<T>(l + 1).x;
    const size_t mc = (size_t)std::max(last ? nc_ : L_[l + 1].A.n, 1) * k;
    DR_CK(cudaMemsetAsync(bc, 0, mc * sizeof(T), st_));
    DR_CK(cudaMemsetAsync(xc, 0, mc * sizeof(T), st_));
    const T* dinv = invd<T>(L);
    const T om = (T)L.omega;
    const DevMat &A = L.A, &R = L.R, &P = L.P;
    auto launch = [&](int op, BlockShape sh) {
      note_launch();
      switch (op) {
        case 0:
          spmm<T, T, BM_JACOBI>(st_, max_grid_, A.n, k, A.rp, A.ci, mval<T>(A), W.x, W.b, dinv, om, W.t, nullptr, sh);
          break;
        case 1:
          spmm<T, T, BM_RESID>(st_, max_grid_, A.n, k, A.rp, A.ci, mval<T>(A), W.x, W.b, nullptr, T(0), W.r,
                               nullptr, sh);
          break;
        case 2:
          spmm<T, T, BM_STORE>(st_, max_grid_, R.n, k, R.rp, R.ci, mval<T>(R), W.r, nullptr, nullptr, T(0), bc,
                               nullptr, sh);
          break;
        case 3:  // x += P x_c with x_c = 0 leaves x at zero
          spmm<T, T, BM_ADDTO>(st_, max_grid_, P.n, k, P.rp, P.ci, mval<T>(P), xc, nullptr, nullptr, T(0), W.x,
                               nullptr, sh);
          break;
        default:  // the fused correction, with r = 0 and x_c = 0 (x stays zero)
          spmm<T, T, BM_CORRECT>(st_, max_grid_, L.AP.n, k, L.AP.rp, L.AP.ci, qval<T>(L), xc, W.r, dinv, om,
                                 W.x, nullptr, sh);
      }
    };
    const void* rps[5] = {A.rp, A.rp, R.rp, P.rp, L.AP.rp};
    for (int op = 0; op < (L.fuse_up ? 5 : 4); ++op) {
      float best = 0.f, def = 0.f;
      BlockShape pick{};
      for (size_t c = 0; c < cand.size(); ++c) {
        launch(op, cand[c]);  // warm-up
        DR_CK(cudaEventRecord(e0, st_));
        for (int r = 0; r < kReps; ++r) launch(op, cand[c]);
        DR_CK(cudaEventRecord(e1, st_));
        DR_CK(cudaEventSynchronize(e1));
        float ms = 0.f;
        DR_CK(cudaEventElapsedTime(&ms, e0, e1));
        if (c == 0) {
          def = best = ms;
        } else if (ms < best && ms < 0.97f * def) {
          best = ms;
          pick = cand[c];
        }
      }
      if (pick.tpr) bshape_[ShapeKey{rps[op], kOpMode[op], (int)sizeof(T), k}] = pick;
      if (verbose >= 1)
        std::printf("block tuning (k = %d, FP%d) level %d %-12s: %2d threads per row, %s blocks per SM, "
                    "%.1f us (default %.1f us)\n",
                    k, 8 * (int)sizeof(T), l, kOpName[op], pick.tpr ? pick.tpr : t0,
                    pick.nb ? "2" : "all resident", 1e3 * best / kReps, 1e3 * def / kReps);
    }
  }
  DR_CK(cudaEventDestroy(e0));
  DR_CK(cudaEventDestroy(e1));
  DR_CK(cudaGetLastError());
}

void DevHier::col_dots(int n, int k, const double* a, const double* b, double* dst_dev) {
  const int grid = warp_grid(n, max_grid_);
  note_launch();
  k_bl_dot_part<<<grid, kBlock, 0, st_>>>(n, k, a, b, bpart_);
  note_launch();
  k_bl_dot_final<<<1, 1024, 0, st_>>>(grid, k, bpart_, dst_dev);
  DR_CK(cudaGetLastError());
}

// One cycle of level l on k columns; returns where the result ended (X or
// the level's partner buffer).
template <typename T>
T* DevHier::cycle_block(int l, T* X, const T* B, bool x_zero, const CycleOpts& o, int k) {
  DevLevel& L = L_[l];
  BlockVecs<T>& V = bvecs<T>(l);
  const DevMat& A = L.A;
  const int n = A.n;
  const T om = (T)L.omega;
  const T* dinv = invd<T>(L);
  const T* av = mval<T>(A);
  T* x = X;
  T* t = (X == V.x) ? V.t : V.x;
  const BlockShape sj = shape_of(A.rp, BM_JACOBI, sizeof(T), k);
  int pre = o.pre;
  if (x_zero) {
    note_launch();
    if (pre >= 1) {
      k_bl_jz<T><<<grid_for((long long)n * k, max_grid_), kBlock, 0, st_>>>(n, k, B, dinv, om, x);
      --pre;
    } else {
      k_bl_fill<T><<<grid_for((long long)n * k, max_grid_), kBlock, 0, st_>>>((long long)n * k, x);
    }
  }
  for (int s = 0; s < pre; ++s) {
    note_launch();
    spmm<T, T, BM_JACOBI>(st_, max_grid_, n, k, A.rp, A.ci, av, x, B, dinv, om, t, nullptr, sj);
    std::swap(x, t);
  }
  note_launch();
  spmm<T, T, BM_RESID>(st_, max_grid_, n, k, A.rp, A.ci, av, x, B, nullptr, T(0), V.r, nullptr,
                       shape_of(A.rp, BM_RESID, sizeof(T), k));
  const bool last = (l + 1 == nlevels());
  T* bc = last ? (sizeof(T) == 8 ? (T*)bcb64_ : (T*)bcb32_) : bvecs<T>(l + 1).b;
  const DevMat& R = L.R;
  note_launch();
  spmm<T, T, BM_STORE>(st_, max_grid_, R.n, k, R.rp, R.ci, mval<T>(R), V.r, nullptr, nullptr, T(0), bc, nullptr,
                       shape_of(R.rp, BM_STORE, sizeof(T), k));
  T* xc;
  if (!last) {
    xc = cycle_block<T>(l + 1, bvecs<T>(l + 1).x, bc, true, o, k);
    if (o.w) xc = cycle_block<T>(l + 1, xc, bc, false, o, k);
  } else {
    xc = sizeof(T) == 8 ? (T*)bcx64_ : (T*)bcx32_;
    note_launch();
    if (cinv_ok_) {  // the explicit inverse (a hierarchy with tree-summed levels)
      k_bl_inv<T><<<grid_for((long long)nc_ * k, max_grid_), kBlock, 0, st_>>>(nc_, k, cinv_, bc, xc);
    } else if (nc_ <= 64) {
      const size_t wsm = ((size_t)nc_ * nc_ + (size_t)k * nc_) * sizeof(double);  // <= 48 KB
      k_bl_lu_warp<T><<<1, 32 * k, wsm, st_>>>(nc_, k, clu_, cpiv_, bc, xc);
    } else {
      size_t smem = (size_t)nc_ * k * sizeof(double);
      int optin = 0;
      DR_CK(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device_));
      if (smem > (size_t)optin) fail("block solves: the coarsest system is too large for one block");
      // the factors too, when they fit beside the vectors
      const size_t with_lu = smem + (size_t)nc_ * nc_ * sizeof(double);
      const int stage = with_lu <= (size_t)optin ? 1 : 0;
      if (stage) smem = with_lu;
      if (smem > 48 * 1024)
        DR_CK(cudaFuncSetAttribute(k_bl_lu<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
      k_bl_lu<T><<<1, 32, smem, st_>>>(nc_, k, clu_, cpiv_, bc, xc, stage);
    }
  }
  const DevMat& P = L.P;
  int post0 = 0;
  note_launch();
  if (L.fuse_up && o.post >= 1) {
    // correction and the first post-smoothing step in one pass over Q (see
    // EpCorrectJacobi; V.r holds B - A x from the way down)
    spmm<T, T, BM_CORRECT>(st_, max_grid_, L.AP.n, k, L.AP.rp, L.AP.ci, qval<T>(L), xc, V.r, dinv, om, x,
                           nullptr, shape_of(L.AP.rp, BM_CORRECT, sizeof(T), k));
    post0 = 1;
  } else {
    spmm<T, T, BM_ADDTO>(st_, max_grid_, P.n, k, P.rp, P.ci, mval<T>(P), xc, nullptr, nullptr, T(0), x, nullptr,
                         shape_of(P.rp, BM_ADDTO, sizeof(T), k));
  }
  for (int s = post0; s < o.post; ++s) {
    note_launch();
    spmm<T, T, BM_JACOBI>(st_, max_grid_, n, k, A.rp, A.ci, av, x, B, dinv, om, t, nullptr, sj);
    std::swap(x, t);
  }
  DR_CK(cudaGetLastError());
  return x;
}

template float* DevHier::cycle_block<float>(int, float*, const float*, bool, const CycleOpts&, int);
template double* DevHier::cycle_block<double>(int, double*, const double*, bool, const CycleOpts&, int);

int DevHier::pcg_block(double* X, const double* B, int k, const CycleOpts& o, double tol, int maxiter,
                       bool mixed, int* iters, double* relres, int verbose) {
  if (k < 1 || k > 32) fail("pcg_block: k must be 1..32");
  if (L_.empty()) fail("pcg_block: the hierarchy has no levels");
  for (auto& d : L_)
    if (!jacobi_type(d.smoother))
      fail("block solves need Jacobi, l1-Jacobi or SPAI(0) smoothing on every level");
  if (mixed) ensure_fp32();
  ensure_block(k);
  if (mixed) tune_block<float>(k, verbose);
  else tune_block<double>(k, verbose);
  const int n = n0_;
  const long long m = (long long)n * k;
  double *R = bpcg_[0], *P = bpcg_[1], *Q = bpcg_[2], *Z = bpcg_[3];
  float* R32 = bpcg32_[0];
  const DevMat& A = L_[0].A;
  const int grid = warp_grid(n, max_grid_);
  const int vgrid = grid_for(m, max_grid_);
  // device k-vectors: 0 bb, 1 rr, 2 rz, 3 pq, 4 alpha, 5 beta
  double* dv = bdev_;
  double* hv = bhost_;
  auto fetch = [&](int slot) {
    DR_CK(cudaMemcpyAsync(hv + slot * 32, dv + slot * 32, k * sizeof(double), cudaMemcpyDeviceToHost, st_));
  };
  // Fused outer iteration (even k, 16-byte aligned vectors): p.q comes with
  // Q = A P, r.r and the FP32 copy of R with the update, r.z with taking Z
  // from the cycle; two columns per thread, column partials per block.
  const bool fused = (k % 2 == 0) && aligned16(X) && aligned16(B);
  const int tpr2 = tpr_for(k / 2);
  const int g2 = vec_grid((const void*)k_bl_update_vec<16>, n, tpr2, max_grid_);
  auto dot_final = [&](int nblocks, double* dst) {
    note_launch();
    k_bl_dot_final<<<1, 1024, 0, st_>>>(nblocks, k, bpart_, dst);
  };
  auto update = [&](bool r32) {  // X += alpha P, R -= alpha Q, r.r -> dv[1]
    note_launch();
    if (fused) {
      float* r32p = r32 ? R32 : nullptr;
      switch (tpr2) {
#define DR_UPD(t)                                                                             \
  case t:                                                                                     \
    k_bl_update_vec<t><<<g2, kBlock, 0, st_>>>(n, k, dv + 4 * 32, X, R, P, Q, r32p, bpart_); \
    break;
        DR_UPD(1) DR_UPD(2) DR_UPD(4) DR_UPD(8) DR_UPD(16)
#undef DR_UPD
      }
      dot_final(g2, dv + 1 * 32);
    } else {
      k_bl_update<<<vgrid, kBlock, 0, st_>>>(n, k, dv + 4 * 32, X, R, P, Q, nullptr);
      col_dots(n, k, R, R, dv + 1 * 32);
    }
  };
  bool r32_ready = false;  // R32 already holds (float) R
  auto take_z = [&](const auto* z) {  // Z = z, r.z -> dv[2]
    using TZ = std::remove_const_t<std::remove_pointer_t<decltype(z)>>;
    note_launch();
    if (fused) {
      switch (tpr2) {
#define DR_TZ(t)                                                                   \
  case t:                                                                          \
    k_bl_take_z<TZ, t><<<g2, kBlock, 0, st_>>>(n, k, z, R, Z, bpart_);            \
    break;
        DR_TZ(1) DR_TZ(2) DR_TZ(4) DR_TZ(8) DR_TZ(16)
#undef DR_TZ
      }
      dot_final(g2, dv + 2 * 32);
    } else {
      k_bl_convert<TZ, double><<<vgrid, kBlock, 0, st_>>>(m, z, Z);
      col_dots(n, k, R, Z, dv + 2 * 32);
    }
  };
  auto precond = [&]() {  // Z = M R, then r.z -> dv[2]
    if (mixed) {
      if (!r32_ready) {
        note_launch();
        k_bl_convert<double, float><<<vgrid, kBlock, 0, st_>>>(m, R, R32);
      }
      const float* z = cycle_block<float>(0, bvecs<float>(0).x, R32, true, o, k);
      take_z(z);
    } else {
      const double* z = cycle_block<double>(0, bvecs<double>(0).x, R, true, o, k);
      take_z(z);
    }
  };
  note_launch();
  spmm<double, double, BM_RESID>(st_, max_grid_, n, k, A.rp, A.ci, A.v, X, B, nullptr, 0.0, R);
  col_dots(n, k, B, B, dv + 0 * 32);
  col_dots(n, k, R, R, dv + 1 * 32);
  fetch(0);
  fetch(1);
  DR_CK(cudaStreamSynchronize(st_));
  std::vector<double> bb(hv, hv + k), rr(hv + 32, hv + 32 + k);
  std::vector<char> active(k);
  std::vector<int> its(k, 0);
  int nact = 0;
  for (int c = 0; c < k; ++c) {
    active[c] = bb[c] > 0.0 && std::sqrt(rr[c] / bb[c]) >= tol;
    nact += active[c];
  }
  precond();
  fetch(2);
  DR_CK(cudaMemcpyAsync(P, Z, (size_t)m * sizeof(double), cudaMemcpyDeviceToDevice, st_));
  DR_CK(cudaStreamSynchronize(st_));
  std::vector<double> rz(hv + 64, hv + 64 + k);
  int it = 0;
  while (nact > 0 && it < maxiter) {
    ++it;
    note_launch();
    const int gq = spmm<double, double, BM_STORE>(st_, max_grid_, n, k, A.rp, A.ci, A.v, P, nullptr, nullptr,
                                                  0.0, Q, fused ? bpart_ : nullptr);
    if (gq > 0 && fused) dot_final(gq, dv + 3 * 32);
    else col_dots(n, k, P, Q, dv + 3 * 32);
    fetch(3);
    DR_CK(cudaStreamSynchronize(st_));
    for (int c = 0; c < k; ++c) hv[4 * 32 + c] = (active[c] && hv[96 + c] != 0.0) ? rz[c] / hv[96 + c] : 0.0;
    DR_CK(cudaMemcpyAsync(dv + 4 * 32, hv + 4 * 32, k * sizeof(double), cudaMemcpyHostToDevice, st_));
    update(mixed);
    r32_ready = mixed && fused;
    fetch(1);
    DR_CK(cudaStreamSynchronize(st_));
    for (int c = 0; c < k; ++c)
      if (active[c]) {
        its[c] = it;
        if (std::sqrt(hv[32 + c] / bb[c]) < tol) {
          active[c] = 0;
          --nact;
        }
      }
    if (verbose >= 2) std::printf("  block PCG iter %4d: %d of %d columns active\n", it, nact, k);
    if (nact == 0) break;
    precond();
    fetch(2);
    DR_CK(cudaStreamSynchronize(st_));
    for (int c = 0; c < k; ++c) {
      const double rzn = hv[64 + c];
      hv[5 * 32 + c] = (active[c] && rz[c] != 0.0) ? rzn / rz[c] : 0.0;
      rz[c] = rzn;
    }
    DR_CK(cudaMemcpyAsync(dv + 5 * 32, hv + 5 * 32, k * sizeof(double), cudaMemcpyHostToDevice, st_));
    note_launch();
    k_bl_dir<<<vgrid, kBlock, 0, st_>>>(n, k, dv + 5 * 32, Z, P);
  }
  // true residuals of the result
  note_launch();
  spmm<double, double, BM_RESID>(st_, max_grid_, n, k, A.rp, A.ci, A.v, X, B, nullptr, 0.0, R);
  col_dots(n, k, R, R, dv + 1 * 32);
  fetch(1);
  DR_CK(cudaStreamSynchronize(st_));
  DR_CK(cudaGetLastError());
  int worst = 0;
  for (int c = 0; c < k; ++c) {
    if (iters) iters[c] = its[c];
    if (relres) relres[c] = bb[c] > 0.0 ? std::sqrt(hv[32 + c] / bb[c]) : 0.0;
    worst = std::max(worst, its[c]);
  }
  return worst;
}

}  // namespace dr
