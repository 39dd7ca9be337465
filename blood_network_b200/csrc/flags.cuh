// Sync-free sweeps over a dependency DAG: the value-as-flag primitives and
// the chunk schedule shared by the IC(0) triangular solves (ichol.cu) and
// the ordered Gauss-Seidel sweeps (gs_ordered.cu).
#pragma once
#include "common.cuh"

#include <vector>

namespace bn {

// Sync-free form: no barrier at all.  Every value of the output vector
// starts as an all-ones bit pattern (a NaN that arithmetic never produces:
// results are canonicalised below), so the value itself says whether it has
// been computed.  A row polls each of its dependencies with relaxed GPU-scope
// loads until the pattern is gone, then computes and publishes its value
// with one relaxed store.  Rows are taken in level order, 32 per warp,
// chunks dealt round-robin to the warps of a co-resident grid: a warp only
// waits on rows of earlier chunks, and the earliest unfinished chunk has all
// its dependencies done, so the sweep always advances.  Every wait is
// bounded; a wait that runs out records an error and uses NaN, so the
// kernel always ends and the failure surfaces as a non-finite result.
template <class T>
struct WordOf;
template <>
struct WordOf<float> {
  using U = unsigned;
  static constexpr U kPending = 0xFFFFFFFFu;
  static constexpr U kNaN = 0x7FFFFFFFu;
};
template <>
struct WordOf<double> {
  using U = unsigned long long;
  static constexpr U kPending = 0xFFFFFFFFFFFFFFFFull;
  static constexpr U kNaN = 0x7FFFFFFFFFFFFFFFull;
};

__device__ __forceinline__ unsigned ld_relaxed(const unsigned* p) {
  unsigned v;
  asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ unsigned long long ld_relaxed(const unsigned long long* p) {
  unsigned long long v;
  asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_relaxed(unsigned* p, unsigned v) {
  asm volatile("st.relaxed.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ void st_relaxed(unsigned long long* p, unsigned long long v) {
  asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ float word_value(unsigned u) { return __uint_as_float(u); }
__device__ __forceinline__ double word_value(unsigned long long u) {
  return __longlong_as_double((long long)u);
}
__device__ __forceinline__ unsigned value_word(float v) { return __float_as_uint(v); }
__device__ __forceinline__ unsigned long long value_word(double v) {
  return (unsigned long long)__double_as_longlong(v);
}

constexpr int kFlagThreads = 256;
constexpr int kSpinFast = 64;          // polls before backing off
constexpr int kSpinLimit = 1 << 22;    // polls before giving up (seconds with back-off)

// Waits until none of the first m words u[q] (loaded from o[j[q]]) is
// pending, re-polling all pending ones together so that the last arrival
// costs one round trip.
template <class U>
__device__ __forceinline__ void wait_group(const U* o, const int (&j)[4], U (&u)[4], int m,
                                           U pending, U nan, int* err) {
  for (int it = 0; it < kSpinLimit; it++) {
    bool pend = false;
#pragma unroll
    for (int q = 0; q < 4; q++) pend |= (q < m && u[q] == pending);
    if (!pend) return;
    if (it >= kSpinFast) __nanosleep(it < 4096 ? 32 : 256);
#pragma unroll
    for (int q = 0; q < 4; q++)
      if (q < m && u[q] == pending) u[q] = ld_relaxed(o + j[q]);
  }
  atomicExch(err, 1);
#pragma unroll
  for (int q = 0; q < 4; q++)
    if (q < m && u[q] == pending) u[q] = nan;
}

// Waits until the word at p (last read as u) is no longer pending (bounded;
// NaN and an error record when the wait runs out).
template <class U>
__device__ __forceinline__ U wait_word(const U* p, U u, U pending, U nan, int* err) {
  for (int it = 0; it < kSpinLimit && u == pending; it++) {
    if (it >= kSpinFast) __nanosleep(it < 4096 ? 32 : 256);
    u = ld_relaxed(p);
  }
  if (u == pending) {
    atomicExch(err, 1);
    u = nan;
  }
  return u;
}

// 32-row chunks of the level-ordered layout, cut at every level boundary
inline int upload_chunks(const std::vector<int>& ptr, DBuf<int2>& d, cudaStream_t s) {
  std::vector<int2> h;
  for (size_t l = 0; l + 1 < ptr.size(); l++)
    for (int t = ptr[l]; t < ptr[l + 1]; t += 32)
      h.push_back(make_int2(t, t + 32 < ptr[l + 1] ? t + 32 : ptr[l + 1]));
  d.alloc(h.size() > 0 ? h.size() : 1, s);
  if (!h.empty()) d.upload(h.data(), h.size());
  BN_CUDA(cudaStreamSynchronize(s));
  return (int)h.size();
}

// Dependency levels of a DAG (ichol.cu): rows in level order, level offsets.
void level_schedule(const CSR& deps, const CSR& users, DBuf<int>& order, std::vector<int>& lptr,
                    cudaStream_t s);

}  // namespace bn
