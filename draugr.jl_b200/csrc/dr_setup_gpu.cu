// The setup's Galerkin products on the GPU (the setup offload): for each
// level, the sparsity patterns of A·P and Pᵀ(AP) (src/galerkin.jl:11-183,
// the sorted unique columns of each output row) and their numeric values,
// computed on the device and copied back for the CPU coarsening of the next
// level.  The patterns are sets, so they equal the CPU's symbolic_ap /
// symbolic_ptap; the values come from the warp kernel, whose per-entry
// order is the CPU numeric product's: the hierarchy is the CPU setup's, bit
// for bit.
//
// Pattern of row r of O = S·B: one warp inserts the columns of the B rows
// selected by S's row r into a hash set in shared memory (atomicCAS on
// empty slots), counting new insertions; a second pass inserts again,
// compacts the set and sorts it (bitonic, in shared memory) into O's
// columns.  A row with more than kSymMax distinct columns makes the device
// path give the level back to the host.
#include <cuda_runtime.h>

#include <cstdlib>
#include <memory>
#include <string>
#include <vector>

#include "dr_device.h"

namespace dr {
namespace {

constexpr int kSymWarps = 4;
constexpr int kSymSlots = 2048;  // hash slots per warp
constexpr int kSymMax = 1024;    // distinct columns a row may have (load factor 1/2)

__device__ __forceinline__ unsigned sym_hash(int c) { return ((unsigned)c * 0x9E3779B1u) >> 21; }  // 11 bits

// FILL = false: cnt[r] = number of distinct columns of row r.
// FILL = true: o_ci[o_rp[r] ..] = those columns, ascending.
template <bool FILL>
__global__ void __launch_bounds__(kSymWarps * 32)
k_sym_rows(int nrows, const int* __restrict__ s_rp, const int* __restrict__ s_ci, const int* __restrict__ b_rp,
           const int* __restrict__ b_ci, const int* __restrict__ o_rp, int* __restrict__ out, int* overflow) {
  __shared__ int tab[kSymWarps][kSymSlots];
  __shared__ int lst[kSymWarps][kSymMax];
  const int lane = threadIdx.x & 31;
  const int w = threadIdx.x >> 5;
  const unsigned full = 0xffffffffu;
  for (long long r0 = (long long)blockIdx.x * kSymWarps + w; r0 < nrows; r0 += (long long)gridDim.x * kSymWarps) {
    const int r = (int)r0;
    for (int q = lane; q < kSymSlots; q += 32) tab[w][q] = -1;
    __syncwarp();
    int added = 0;
    bool bad = false;
    const int ss = s_rp[r], se = s_rp[r + 1];
    for (int k = ss + lane; k < se; k += 32) {  // each lane takes whole B rows
      const int j = s_ci[k];
      for (int t = b_rp[j]; t < b_rp[j + 1]; ++t) {
        const int c = b_ci[t];
        unsigned h = sym_hash(c);
        int probe = 0;
        for (; probe < kSymSlots; ++probe) {
          const int old = atomicCAS(&tab[w][h], -1, c);
          if (old == -1) {
            ++added;
            break;
          }
          if (old == c) break;
          h = (h + 1) & (kSymSlots - 1);
        }
        if (probe == kSymSlots) bad = true;
      }
    }
    for (int o = 16; o > 0; o >>= 1) added += __shfl_xor_sync(full, added, o);
    bad = __any_sync(full, bad) || added > kSymMax;
    if (bad) {
      if (lane == 0) atomicExch(overflow, 1);
      __syncwarp();
      continue;
    }
    if (!FILL) {
      if (lane == 0) out[r] = added;
      __syncwarp();
      continue;
    }
    // compact the set, then sort it (padded with INT_MAX to a power of two)
    __syncwarp();
    int base = 0;
    for (int q0 = 0; q0 < kSymSlots; q0 += 32) {
      const int v = tab[w][q0 + lane];
      const unsigned m = __ballot_sync(full, v >= 0);
      if (v >= 0) lst[w][base + __popc(m & ((1u << lane) - 1u))] = v;
      base += __popc(m);
    }
    int P2 = 1;
    while (P2 < added) P2 <<= 1;
    for (int q = added + lane; q < P2; q += 32) lst[w][q] = 0x7fffffff;
    __syncwarp();
    for (int k = 2; k <= P2; k <<= 1)
      for (int jj = k >> 1; jj > 0; jj >>= 1) {
        for (int i = lane; i < P2; i += 32) {
          const int ixj = i ^ jj;
          if (ixj > i) {
            const int a = lst[w][i], b = lst[w][ixj];
            const bool asc = (i & k) == 0;
            if ((a > b) == asc) {
              lst[w][i] = b;
              lst[w][ixj] = a;
            }
          }
        }
        __syncwarp();
      }
    const int os = o_rp[r];
    for (int q = lane; q < added; q += 32) out[os + q] = lst[w][q];
    __syncwarp();
  }
}

template <typename T>
struct DevBuf {
  T* p = nullptr;
  size_t n = 0;
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  ~DevBuf() {
    if (p) cudaFree(p);
  }
  void alloc(size_t count) {
    if (p) cudaFree(p);
    p = nullptr;
    n = count;
    DR_CK(cudaMalloc(&p, std::max<size_t>(count, 1) * sizeof(T)));
  }
  void up(const std::vector<T>& h, cudaStream_t st) {
    alloc(h.size());
    if (!h.empty()) DR_CK(cudaMemcpyAsync(p, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice, st));
  }
  void down(std::vector<T>& h, size_t count, cudaStream_t st) const {
    h.resize(count);
    if (count) DR_CK(cudaMemcpyAsync(h.data(), p, count * sizeof(T), cudaMemcpyDeviceToHost, st));
  }
};

class DeviceGalerkin : public GalerkinDevice {
 public:
  DeviceGalerkin() {
    DR_CK(cudaStreamCreateWithFlags(&st_, cudaStreamNonBlocking));
    int dev = 0;
    DR_CK(cudaGetDevice(&dev));
    int nsm = 148;
    DR_CK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    max_grid_ = nsm * 8;
    ovf_.alloc(1);
  }
  ~DeviceGalerkin() override { cudaStreamDestroy(st_); }

  bool galerkin(const CSR& A, const Prolong& P, const TransposeMap& T, const std::vector<double>& Rv,
                std::vector<int>& ap_rp, std::vector<int>& ap_ci, std::vector<double>& ap_v, CSR& next) override {
    try {
      const int n = A.n, nc = P.nc;
      DevBuf<int> arp, aci, prp, pci, toff, trow, aprp, apci, crp, cci;
      DevBuf<double> av, pv, rv, apv, cv;
      arp.up(A.rp, st_);
      aci.up(A.ci, st_);
      av.up(A.v, st_);
      prp.up(P.rp, st_);
      pci.up(P.ci, st_);
      pv.up(P.v, st_);
      toff.up(T.off, st_);
      trow.up(T.rows, st_);
      rv.up(Rv, st_);
      // A·P
      if (!pattern(n, arp.p, aci.p, prp.p, pci.p, ap_rp, aprp, apci)) return fail_back();
      apv.alloc(ap_rp[n]);
      galerkin_numeric_raw(st_, n, maxlen(ap_rp), aprp.p, apci.p, apv.p, arp.p, aci.p, av.p, prp.p, pci.p, pv.p,
                           max_grid_);
      // Pᵀ(AP), Pᵀ in transpose-map order with P's values
      if (!pattern(nc, toff.p, trow.p, aprp.p, apci.p, next.rp, crp, cci)) return fail_back();
      cv.alloc(next.rp[nc]);
      galerkin_numeric_raw(st_, nc, maxlen(next.rp), crp.p, cci.p, cv.p, toff.p, trow.p, rv.p, aprp.p, apci.p,
                           apv.p, max_grid_);
      apci.down(ap_ci, ap_rp[n], st_);  // kept by the level for partial resetups
      ap_v.clear();                     // the host needs no A·P values: Pᵀ(AP) is done
      cci.down(next.ci, next.rp[nc], st_);
      cv.down(next.v, next.rp[nc], st_);
      DR_CK(cudaStreamSynchronize(st_));
      next.n = next.m = nc;
      return true;
    } catch (const std::exception&) {
      cudaGetLastError();
      return fail_back();
    }
  }

 private:
  cudaStream_t st_ = nullptr;
  int max_grid_ = 0;
  DevBuf<int> ovf_;

  bool fail_back() {
    cudaStreamSynchronize(st_);
    cudaGetLastError();
    return false;
  }
  static int maxlen(const std::vector<int>& rp) {
    int m = 0;
    for (size_t i = 0; i + 1 < rp.size(); ++i) m = std::max(m, rp[i + 1] - rp[i]);
    return m;
  }
  // pattern of S·B (S: nrows rows): counts, a host prefix sum, then the
  // sorted columns; false when some row has too many columns
  bool pattern(int nrows, const int* s_rp, const int* s_ci, const int* b_rp, const int* b_ci, std::vector<int>& o_rp,
               DevBuf<int>& d_rp, DevBuf<int>& d_ci) {
    DR_CK(cudaMemsetAsync(ovf_.p, 0, sizeof(int), st_));
    DevBuf<int> cnt;
    cnt.alloc(nrows);
    const int grid = std::max(1, std::min((nrows + kSymWarps - 1) / kSymWarps, max_grid_));
    note_launch();
    k_sym_rows<false><<<grid, kSymWarps * 32, 0, st_>>>(nrows, s_rp, s_ci, b_rp, b_ci, nullptr, cnt.p, ovf_.p);
    DR_CK(cudaGetLastError());
    std::vector<int> c;
    cnt.down(c, nrows, st_);
    int ovf = 0;
    DR_CK(cudaMemcpyAsync(&ovf, ovf_.p, sizeof(int), cudaMemcpyDeviceToHost, st_));
    DR_CK(cudaStreamSynchronize(st_));
    if (ovf) return false;
    o_rp.assign((size_t)nrows + 1, 0);
    for (int i = 0; i < nrows; ++i) o_rp[i + 1] = o_rp[i] + c[i];
    d_rp.up(o_rp, st_);
    d_ci.alloc(o_rp[nrows]);
    note_launch();
    k_sym_rows<true><<<grid, kSymWarps * 32, 0, st_>>>(nrows, s_rp, s_ci, b_rp, b_ci, d_rp.p, d_ci.p, ovf_.p);
    DR_CK(cudaGetLastError());
    DR_CK(cudaStreamSynchronize(st_));
    return true;
  }
};

}  // namespace

std::unique_ptr<GalerkinDevice> make_galerkin_device() {
  const char* e = std::getenv("DRAUGR_B200_GPU_SETUP");
  if (e && std::string(e) == "0") return nullptr;
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
    cudaGetLastError();
    return nullptr;
  }
  try {
    return std::make_unique<DeviceGalerkin>();
  } catch (const std::exception&) {
    cudaGetLastError();
    return nullptr;
  }
}

}  // namespace dr
