// An IC(0) triangular solve that allocates nothing.
//
// Some callers cannot allocate GPU memory at the point where they need the
// preconditioner: code running inside a memory budget that another framework
// owns (a pool that must not grow, a process that has pre-reserved its
// device memory), callbacks invoked from code that forbids allocation, and
// hosts that replay a fixed set of buffers.  For them,
// ichol_solve_noalloc() solves L L^T x = b for a factor already on the device
// without any cudaMalloc/cudaFree: its scratch -- the forward-sweep result y
// and the factor's diagonal -- lives in the file-scope device array below,
// which every GPU that loads this library holds until the process exits
// (2 x 131072 doubles = 2 MiB).
//
// The arithmetic is the reference's ichol_solve (C_amg1/src/ichol.c:121-165),
// one operation at a time in the same order, so the result is bit-identical
// to the allocating ichol_solve entry point.  It runs in one thread block
// (the sweeps are sequential), which suits the small systems this entry point
// is meant for.
#include "common.cuh"
#include "../../include/amg_b200.h"

#include <cuda.h>

#include <mutex>

namespace bn {

constexpr int kNoAllocMaxRows = AMG_NOALLOC_MAX_ROWS;
constexpr int kNoAllocMaxDevices = 64;

// y[0..n) then diag[0..n).  Shared by every call on the device.
static __device__ __align__(256) double g_ichol_scratch[2 * kNoAllocMaxRows];

// Device address of g_ichol_scratch per device, looked up once per device
// with that device current (in host code the symbol is only a stand-in, not a
// device address), together with the context it belongs to: after a
// cudaDeviceReset the device gets a new primary context in which the array
// has a new address, so a changed context triggers a new lookup.
struct ScratchAddr {
  CUcontext ctx = nullptr;
  double* p = nullptr;
};
static ScratchAddr s_scratch[kNoAllocMaxDevices];
static std::mutex s_scratch_mutex;

// cuCtxGetCurrent through the runtime's driver entry point (no link-time
// dependency on the driver library)
typedef CUresult (*CtxGetCurrentFn)(CUcontext*);
static CUcontext current_context() {
  static CtxGetCurrentFn fn = [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      f = nullptr;
    return (CtxGetCurrentFn)f;
  }();
  CUcontext c = nullptr;
  if (fn) fn(&c);
  return c;
}

__global__ void __launch_bounds__(1024)
k_ichol_solve_static(int n, const int* __restrict__ ia, const int* __restrict__ ja,
                     const double* __restrict__ val, const double* __restrict__ b, double* x,
                     double* y, double* dg) {
  // diagonal of each row: its first entry with column i (0.0 if none, as
  // the reference's calloc'd Ldiag)
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    double d = 0.0;
    for (int k = ia[i]; k < ia[i + 1]; k++)
      if (ja[k] == i) { d = val[k]; break; }
    dg[i] = d;
  }
  __syncthreads();
  if (threadIdx.x == 0) {  // forward: L y = b
    for (int i = 0; i < n; i++) {
      double s = b[i], d = 1.0;
      for (int k = ia[i]; k < ia[i + 1]; k++) {
        const int j = ja[k];
        if (j < i) s = xsub(s, xmul(val[k], y[j]));
        else if (j == i) d = val[k];
      }
      y[i] = xdiv(s, d);
    }
  }
  __syncthreads();
  for (int i = threadIdx.x; i < n; i += blockDim.x) x[i] = y[i];
  __syncthreads();
  if (threadIdx.x == 0) {  // backward, column oriented: L^T x = y
    for (int i = n - 1; i >= 0; i--) {
      x[i] = xdiv(x[i], dg[i]);
      const double xi = x[i];
      for (int k = ia[i]; k < ia[i + 1]; k++) {
        const int j = ja[k];
        if (j < i) x[j] = xsub(x[j], xmul(val[k], xi));
      }
    }
  }
}

static int scratch_for_device(int dev, double** out) {
  if (dev < 0 || dev >= kNoAllocMaxDevices) return BN_ERR_ARG;
  std::lock_guard<std::mutex> lock(s_scratch_mutex);
  ScratchAddr& a = s_scratch[dev];
  const CUcontext ctx = current_context();
  if (!a.p || ctx != a.ctx) {
    double* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress((void**)&p, g_ichol_scratch);
    if (e != cudaSuccess || !p) return BN_ERR_CUDA;
    a.p = p;
    a.ctx = current_context();  // the lookup made the primary context current
  }
  *out = a.p;
  return BN_OK;
}

}  // namespace bn

// See include/amg_b200.h for the contract.
BN_API int ichol_solve_noalloc(int n, const int* d_ia, const int* d_ja, const double* d_val,
                               const double* d_b, double* d_x, void* stream) {
  using namespace bn;
  if (n < 0 || n > kNoAllocMaxRows) {
    set_last_error(BN_ERR_ARG, "ichol_solve_noalloc: n = " + std::to_string(n) +
                                   " is outside 0.." + std::to_string(kNoAllocMaxRows) +
                                   " (the size of its fixed device scratch)");
    return BN_ERR_ARG;
  }
  if (n == 0) {
    set_last_error(BN_OK, "");
    return BN_OK;
  }
  if (!d_ia || !d_ja || !d_val || !d_b || !d_x) {
    set_last_error(BN_ERR_ARG, "ichol_solve_noalloc: NULL device pointer");
    return BN_ERR_ARG;
  }
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) {
    set_last_error(BN_ERR_NO_DEVICE, std::string("ichol_solve_noalloc: ") + cudaGetErrorString(e));
    return BN_ERR_NO_DEVICE;
  }
  double* scratch = nullptr;
  int rc = scratch_for_device(dev, &scratch);
  if (rc != BN_OK) {
    set_last_error(rc, "ichol_solve_noalloc: device scratch address lookup failed");
    return rc;
  }
  g_launch_count++;
  k_ichol_solve_static<<<1, 1024, 0, (cudaStream_t)stream>>>(n, d_ia, d_ja, d_val, d_b, d_x,
                                                             scratch, scratch + kNoAllocMaxRows);
  e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_last_error(BN_ERR_CUDA, std::string("ichol_solve_noalloc: ") + cudaGetErrorString(e));
    return BN_ERR_CUDA;
  }
  set_last_error(BN_OK, "");
  return BN_OK;
}
