// Common device/host infrastructure for the B200 AMG-PCG library.
//
// Index type int32 (matches the reference's INT = int, C_amg1/include/
// agg_lib.h:29-31); values float64 (REAL = double) with float32 copies for
// the mixed-precision V-cycle.  All device memory is stream-ordered
// (cudaMallocAsync on the solver's stream) so setup temporaries recycle
// through the driver's pool.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>
#include <atomic>
#include <string>
#include <stdexcept>
#include <vector>
#include <utility>

#define BN_API extern "C" __attribute__((visibility("default")))

namespace bn {

// ---------------------------------------------------------------- status
enum Status : int {
  BN_OK = 0,
  BN_ERR_ARG = -1,        // invalid argument (sizes, NULL pointers, bad CSR)
  BN_ERR_CUDA = -2,       // CUDA runtime error
  BN_ERR_OOM = -3,        // device allocation failed
  BN_ERR_NOT_CONVERGED = -4,
  BN_ERR_NAN = -5,        // NaN / Inf detected in the iteration
  BN_ERR_SPIN = -6,       // a bounded device wait ran out
  BN_ERR_COARSE = -7,     // coarsest level too large for the dense solve
  BN_ERR_NO_DEVICE = -8,
  BN_ERR_DUP = -9,        // duplicate column index within a CSR row
};

struct Error : public std::runtime_error {
  int code;
  Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

void set_last_error(int code, const std::string& msg);

inline void cuda_check(cudaError_t e, const char* what, const char* file, int line) {
  if (e != cudaSuccess) {
    char buf[512];
    snprintf(buf, sizeof(buf), "%s failed at %s:%d: %s", what, file, line,
             cudaGetErrorString(e));
    throw Error(e == cudaErrorMemoryAllocation ? BN_ERR_OOM : BN_ERR_CUDA, buf);
  }
}
#define BN_CUDA(x) ::bn::cuda_check((x), #x, __FILE__, __LINE__)
#define BN_REQUIRE(cond, code, msg) \
  do { if (!(cond)) throw ::bn::Error((code), (msg)); } while (0)

// Launch accounting: every kernel launch in this library goes through
// BN_LAUNCH so the host can report how many of its kernels ran (atomic:
// entry points may be called from several host threads).
extern std::atomic<unsigned long long> g_launch_count;
#define BN_LAUNCH(kernel, grid, block, smem, stream, ...)                 \
  do {                                                                     \
    ::bn::g_launch_count++;                                                \
    kernel<<<(grid), (block), (smem), (stream)>>>(__VA_ARGS__);            \
    BN_CUDA(cudaGetLastError());                                           \
  } while (0)

// Programmatic dependent launch.  A solve-phase kernel starts with
// BN_PDL_ENTRY(): it waits until the kernel before it in the stream has
// finished and its writes are visible (griddepcontrol.wait), then lets the
// next kernel's blocks be scheduled (griddepcontrol.launch_dependents), so
// that launch and block scheduling of the next kernel overlap this kernel's
// tail.  BN_LAUNCH_PDL launches with programmatic stream serialization; only
// kernels that begin with BN_PDL_ENTRY() may be launched that way (a test
// checks the sources).  Off unless BN_PDL=1 (measured slower on the 20M
// solve); with plain launches the entry is a no-op.
__device__ __forceinline__ void pdl_entry() {
  asm volatile("griddepcontrol.wait;" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}
#define BN_PDL_ENTRY() ::bn::pdl_entry()
bool pdl_enabled();
#define BN_LAUNCH_PDL(kern_, grid_, block_, smem_, strm_, ...)                         \
  do {                                                                                  \
    ::bn::g_launch_count++;                                                             \
    if (::bn::pdl_enabled()) {                                                          \
      cudaLaunchConfig_t cfg_ = {};                                                     \
      cfg_.gridDim = dim3(grid_);                                                       \
      cfg_.blockDim = dim3(block_);                                                     \
      cfg_.dynamicSmemBytes = (smem_);                                                  \
      cfg_.stream = (strm_);                                                            \
      cudaLaunchAttribute at_[1];                                                       \
      at_[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;                  \
      at_[0].val.programmaticStreamSerializationAllowed = 1;                           \
      cfg_.attrs = at_;                                                                 \
      cfg_.numAttrs = 1;                                                                \
      BN_CUDA(cudaLaunchKernelEx(&cfg_, kern_, __VA_ARGS__));                           \
    } else {                                                                            \
      kern_<<<(grid_), (block_), (smem_), (strm_)>>>(__VA_ARGS__);                     \
      BN_CUDA(cudaGetLastError());                                                      \
    }                                                                                   \
  } while (0)

constexpr int kSMs = 148;  // B200: 2 dies x 74 SMs

inline int grid_for(long long n, int block, int per_sm = 16) {
  long long g = (n + block - 1) / block;
  long long cap = (long long)kSMs * per_sm;
  if (g > cap) g = cap;
  if (g < 1) g = 1;
  return (int)g;
}

// ---------------------------------------------------------------- buffers
// Owning device buffer, stream-ordered allocation.
template <class T>
struct DBuf {
  T* p = nullptr;
  size_t n = 0;
  cudaStream_t s = 0;
  DBuf() = default;
  DBuf(size_t count, cudaStream_t st) { alloc(count, st); }
  DBuf(const DBuf&) = delete;
  DBuf& operator=(const DBuf&) = delete;
  DBuf(DBuf&& o) noexcept : p(o.p), n(o.n), s(o.s) { o.p = nullptr; o.n = 0; }
  DBuf& operator=(DBuf&& o) noexcept {
    if (this != &o) { release(); p = o.p; n = o.n; s = o.s; o.p = nullptr; o.n = 0; }
    return *this;
  }
  ~DBuf() { release(); }
  void alloc(size_t count, cudaStream_t st) {
    release();
    s = st;
    n = count;
    if (count) BN_CUDA(cudaMallocAsync((void**)&p, count * sizeof(T) + 16, st));
  }
  void release() {
    if (p) cudaFreeAsync(p, s);
    p = nullptr;
    n = 0;
  }
  void zero() { if (n) BN_CUDA(cudaMemsetAsync(p, 0, n * sizeof(T), s)); }
  void fill_bytes(int v) { if (n) BN_CUDA(cudaMemsetAsync(p, v, n * sizeof(T), s)); }
  void upload(const T* h, size_t count) {
    BN_CUDA(cudaMemcpyAsync(p, h, count * sizeof(T), cudaMemcpyHostToDevice, s));
  }
  void download(T* h, size_t count) const {
    BN_CUDA(cudaMemcpyAsync(h, p, count * sizeof(T), cudaMemcpyDeviceToHost, s));
  }
  T* get() const { return p; }
  size_t bytes() const { return n * sizeof(T); }
};

// Copies of caller-owned host arrays: large pageable copies go through
// pinned staging buffers filled or drained by several host threads
// (host_copy.cu).  copy_h2d returns once the source has been read (the DMA
// may still run on s); copy_d2h returns with the data in place.
void copy_h2d(void* dst, const void* src, size_t bytes, cudaStream_t s);
void copy_d2h(void* dst, const void* src, size_t bytes, cudaStream_t s);

// Device CSR (0-based, int32 indices).
struct CSR {
  int n = 0, m = 0;  // rows, cols
  int nnz = 0;
  DBuf<int> ia, ja;
  DBuf<double> val;
  void alloc(int rows, int cols, int nz, cudaStream_t s, bool with_val = true) {
    n = rows; m = cols; nnz = nz;
    ia.alloc((size_t)rows + 1, s);
    ja.alloc((size_t)(nz > 0 ? nz : 1), s);
    if (with_val) val.alloc((size_t)(nz > 0 ? nz : 1), s);
  }
};

// read one scalar back (synchronous on the stream)
template <class T>
inline T read_scalar(const T* d, cudaStream_t s) {
  T h;
  BN_CUDA(cudaMemcpyAsync(&h, d, sizeof(T), cudaMemcpyDeviceToHost, s));
  BN_CUDA(cudaStreamSynchronize(s));
  return h;
}

// ---------------------------------------------------------------- scans
// Exclusive prefix sum in place over cnt[0..n] (n+1 entries; the last
// becomes the total).  Returns the total.
int scan_counts(int* cnt, int n, cudaStream_t s);
long long scan_counts64(long long* cnt, int n, cudaStream_t s);
// out[i] = sum of in[0..i) over n entries; out has n+1 entries.
void exclusive_scan_i32(const int* in, int* out, int n, cudaStream_t s);

// ---------------------------------------------------------------- exact arithmetic
// The setup kernels reproduce the reference's floating-point operation
// order exactly; x86-64 -O3 without -mfma performs every multiply and add
// separately, so these wrappers forbid contraction into FMA.
__device__ __forceinline__ double xmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double xadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double xsub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double xdiv(double a, double b) { return __ddiv_rn(a, b); }
__device__ __forceinline__ float xmulf(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float xaddf(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float xsubf(float a, float b) { return __fsub_rn(a, b); }

// ---------------------------------------------------------------- tracing
// BN_TRACE=1 in the environment prints per-phase device times to stderr
// (each phase is bracketed by a stream synchronisation, so tracing slows the
// run; it is off by default and never on inside a graph capture).
bool trace_on();
double wall_seconds();
struct Phase {
  const char* name;
  cudaStream_t s;
  double t0 = 0.0;
  int level;
  Phase(const char* nm, cudaStream_t st, int lev = -1) : name(nm), s(st), level(lev) {
    if (trace_on()) { cudaStreamSynchronize(s); t0 = wall_seconds(); }
  }
  bool live = true;
  // report now (instead of at the end of the scope)
  void done() {
    if (!live) return;
    live = false;
    if (trace_on()) {
      cudaStreamSynchronize(s);
      if (level >= 0)
        fprintf(stderr, "[bn] L%-2d %-26s %10.3f ms\n", level, name, (wall_seconds() - t0) * 1e3);
      else
        fprintf(stderr, "[bn]     %-26s %10.3f ms\n", name, (wall_seconds() - t0) * 1e3);
    }
  }
  ~Phase() { done(); }
};

}  // namespace bn
