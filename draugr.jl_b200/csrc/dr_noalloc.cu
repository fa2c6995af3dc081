// Residual and residual norm for callers that cannot allocate device memory.
//
// draugr_b200_residual_device needs a hierarchy, and the library allocates
// every hierarchy, workspace and reduction buffer with cudaMalloc.  Some
// hosts cannot let a library do that: applications that hand all device
// memory out of their own pool (a framework's caching allocator, a solver
// that reserves everything at start-up and must not see the device's free
// memory change behind its back) own every byte the computation may touch.
// draugr_b200_residual_noalloc computes r = b - A x and ||r||_2 on CSR
// arrays and vectors the caller already owns, and allocates nothing: the
// only scratch it needs (one partial sum per block plus a completion
// counter) lives in the file-scope array below, which every GPU that loads
// the library holds (about 128 KB) until the process exits.
#include <cuda_runtime.h>

#include <cmath>
#include <mutex>
#include <string>

#include "../../include/draugr_b200.h"
#include "dr_host.h"

namespace dr {
void set_last_error(const std::string& msg);  // dr_capi.cpp
}

namespace {

constexpr int kNaBlock = 256;                       // rows per block
constexpr int kNaMaxBlocks = 16384;                 // partial sums the scratch holds
constexpr long long kNaMaxRows = (long long)kNaBlock * kNaMaxBlocks;  // 4,194,304
constexpr int kNaSlots = kNaMaxBlocks + 2;          // partials, result, counter

// Scratch: [0, kNaMaxBlocks) block partial sums, [kNaMaxBlocks] the total,
// [kNaMaxBlocks + 1] the completion counter (as an unsigned int).  Host
// code must not pass this name to a kernel (on the host it is only a
// stand-in); kernels get its device address from cudaGetSymbolAddress.
static __device__ __align__(256) double g_na_scratch[kNaSlots];

// One thread per row: Ax = sum of a_ij x_j in column order, r = b - Ax
// (the reference's residual_kernel!, src/cycle.jl:32-43, products and sums
// rounded separately); then r_i^2 summed per block, and the last block to
// finish sums the block totals in block order into the total.
__global__ void __launch_bounds__(kNaBlock)
k_residual_noalloc(int n, const int* __restrict__ rp, const int* __restrict__ ci,
                   const double* __restrict__ v, const double* __restrict__ x,
                   const double* __restrict__ b, double* __restrict__ r, double* scratch) {
  __shared__ double ws[kNaBlock / 32];
  __shared__ bool last;
  const int i = blockIdx.x * kNaBlock + threadIdx.x;
  double rr = 0.0;
  if (i < n) {
    double ax = 0.0;
    for (int k = rp[i]; k < rp[i + 1]; ++k) ax = __dadd_rn(ax, __dmul_rn(v[k], x[ci[k]]));
    const double ri = __dsub_rn(b[i], ax);
    r[i] = ri;
    rr = __dmul_rn(ri, ri);
  }
  for (int o = 16; o > 0; o >>= 1) rr += __shfl_xor_sync(0xffffffffu, rr, o);
  if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = rr;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int w = 0; w < kNaBlock / 32; ++w) s += ws[w];
    scratch[blockIdx.x] = s;
    __threadfence();
    unsigned* counter = reinterpret_cast<unsigned*>(scratch + kNaMaxBlocks + 1);
    last = atomicAdd(counter, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (last && threadIdx.x == 0) {
    __threadfence();
    double s = 0.0;
    for (int blk = 0; blk < (int)gridDim.x; ++blk) s += __ldcg(scratch + blk);
    scratch[kNaMaxBlocks] = s;
    *reinterpret_cast<unsigned*>(scratch + kNaMaxBlocks + 1) = 0u;
  }
}

// Device address of the scratch on each device, set up on the first call
// made while that device is current.
std::mutex g_na_mu;
double* g_na_addr[64] = {nullptr};

double* scratch_address() {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) dr::fail(std::string("cudaGetDevice: ") + cudaGetErrorString(e));
  if (dev < 0 || dev >= 64) dr::fail("device index out of range");
  std::lock_guard<std::mutex> lk(g_na_mu);
  if (!g_na_addr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_na_scratch);
    if (e != cudaSuccess || !p)
      dr::fail(std::string("cudaGetSymbolAddress of the residual scratch: ") + cudaGetErrorString(e));
    g_na_addr[dev] = static_cast<double*>(p);
  }
  return g_na_addr[dev];
}

void check(cudaError_t e, const char* what) {
  if (e != cudaSuccess) {
    cudaGetLastError();
    dr::fail(std::string(what) + ": " + cudaGetErrorString(e));
  }
}

}  // namespace

extern "C" int32_t draugr_b200_residual_noalloc(int32_t n, int32_t nnz, const int32_t* rowptr,
                                                const int32_t* colval, const double* nzval,
                                                const double* x, const double* b, double* r,
                                                double* rnorm, void* stream) {
  try {
    dr::set_last_error("");
    if (n < 0 || nnz < 0) dr::fail("ArgumentError: n and nnz must be non-negative");
    if ((long long)n > kNaMaxRows)
      dr::fail("draugr_b200_residual_noalloc: n = " + std::to_string(n) + " exceeds its maximum of " +
               std::to_string(kNaMaxRows) + " rows (its static scratch holds " +
               std::to_string(kNaMaxBlocks) + " block sums of " + std::to_string(kNaBlock) + " rows)");
    if (n > 0 && (!rowptr || !x || !b || !r || (nnz > 0 && (!colval || !nzval))))
      dr::fail("ArgumentError: NULL array");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    double* scratch = scratch_address();
    double total = 0.0;
    if (n > 0) {
      // the completion counter must start at zero (a call interrupted
      // before its last block finished would leave it set)
      check(cudaMemsetAsync(scratch + kNaMaxBlocks + 1, 0, sizeof(unsigned), st), "cudaMemsetAsync");
      const int grid = (n + kNaBlock - 1) / kNaBlock;
      k_residual_noalloc<<<grid, kNaBlock, 0, st>>>(n, rowptr, colval, nzval, x, b, r, scratch);
      check(cudaGetLastError(), "k_residual_noalloc launch");
      check(cudaMemcpyAsync(&total, scratch + kNaMaxBlocks, sizeof(double), cudaMemcpyDeviceToHost, st),
            "cudaMemcpyAsync");
      check(cudaStreamSynchronize(st), "cudaStreamSynchronize");
    }
    if (rnorm) *rnorm = std::sqrt(total);
    return 0;
  } catch (const std::exception& e) {
    dr::set_last_error(e.what());
    return -1;
  }
}
