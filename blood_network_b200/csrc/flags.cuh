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
constexpr int kSpinFast = 64;            // polls before backing off
constexpr int kSpinHardCap = 1 << 27;    // polls: a last bound should the clock not advance

// ------------------------------------------------------------ bounded waits
// Every wait of a sync-free sweep is bounded in time, and the first wait that
// runs out abandons the whole launch: it raises the abort word of the
// sweep's wait record, and every other waiting thread polls that word while
// it backs off, so a sweep that cannot finish ends within about one limit
// (not one limit per waiting row).  A wait that gives up uses NaN for the
// missing value, so the kernel always ends and its output is non-finite.
//
// Wait record (kWaitWords ints in device memory, zero between sweeps):
//   [0] abort word: set by the first wait that gives up
//   [1] tag of that kernel (WaitTag)
//   [2] the waiting row (vector index)
//   [3] the dependency it waited for (vector index)
//   [4] how long it waited, microseconds
constexpr int kWaitWords = 8;
enum WaitTag : int { WT_IC_FWD = 1, WT_IC_BWD = 2, WT_GS_ORDERED = 3, WT_SELFTEST = 4 };

struct WaitCtl {
  int* rec;                      // the wait record
  unsigned long long limit_ns;   // give-up time of one wait
  int tag;                       // WaitTag of the launching sweep
};

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
__device__ __forceinline__ int ld_relaxed_i32(const int* p) {
  int v;
  asm volatile("ld.relaxed.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// The first thread to give up writes the record; later ones only read the
// abort word.
__device__ __forceinline__ void wait_give_up(const WaitCtl& w, int row, int dep,
                                             unsigned long long waited_ns) {
  if (atomicCAS(w.rec, 0, 1) == 0) {
    w.rec[1] = w.tag;
    w.rec[2] = row;
    w.rec[3] = dep;
    const unsigned long long us = waited_ns / 1000ull;
    w.rec[4] = us > 0x7fffffffull ? 0x7fffffff : (int)us;
  }
}

// Back-off step of poll number it (it >= kSpinFast): sleeps, and every 16th
// poll checks the abort word and the time waited.  Returns true when the
// wait must end now (*ran_out: this wait ran out, rather than another one).
__device__ __forceinline__ bool wait_backoff(const WaitCtl& w, int it,
                                             unsigned long long& t0, bool* ran_out) {
  __nanosleep(it < 4096 ? 32 : 256);
  if ((it & 15) != 0) return false;
  if (ld_relaxed_i32(w.rec) != 0) {
    *ran_out = false;
    return true;
  }
  const unsigned long long t = global_ns();
  if (t0 == 0) {
    t0 = t;
    return false;
  }
  if (t - t0 > w.limit_ns || it >= kSpinHardCap) {
    *ran_out = true;
    return true;
  }
  return false;
}

// Waits until none of the first m words u[q] (loaded from o[j[q]]) is
// pending, re-polling all pending ones together so that the last arrival
// costs one round trip.  row: the waiting row (for the record).
template <class U>
__device__ __forceinline__ void wait_group(const U* o, const int (&j)[4], U (&u)[4], int m,
                                           U pending, U nan, const WaitCtl& w, int row) {
  unsigned long long t0 = 0;
  for (int it = 0;; it++) {
    bool pend = false;
#pragma unroll
    for (int q = 0; q < 4; q++) pend |= (q < m && u[q] == pending);
    if (!pend) return;
    bool ran_out = false;
    if (it >= kSpinFast && wait_backoff(w, it, t0, &ran_out)) {
      int dep = -1;
#pragma unroll
      for (int q = 3; q >= 0; q--)
        if (q < m && u[q] == pending) dep = j[q];
      if (ran_out) wait_give_up(w, row, dep, global_ns() - t0);
      break;
    }
#pragma unroll
    for (int q = 0; q < 4; q++)
      if (q < m && u[q] == pending) u[q] = ld_relaxed(o + j[q]);
  }
#pragma unroll
  for (int q = 0; q < 4; q++)
    if (q < m && u[q] == pending) u[q] = nan;
}

// Waits until the word at o[j] (last read as u) is no longer pending
// (bounded as above; NaN when the wait is abandoned).
template <class U>
__device__ __forceinline__ U wait_word(const U* o, int j, U u, U pending, U nan,
                                       const WaitCtl& w, int row) {
  unsigned long long t0 = 0;
  for (int it = 0; u == pending; it++) {
    bool ran_out = false;
    if (it >= kSpinFast && wait_backoff(w, it, t0, &ran_out)) {
      if (ran_out) wait_give_up(w, row, j, global_ns() - t0);
      return nan;
    }
    u = ld_relaxed(o + j);
  }
  return u;
}

// Host side of a wait record: the device words, the limit, and the report.
struct WaitRecord {
  DBuf<int> rec;
  unsigned long long limit_ns = default_limit_ns();
  void init(cudaStream_t s) {  // never inside a stream capture
    if (!rec.p) rec.alloc(kWaitWords, s);
    rec.zero();
  }
  WaitCtl ctl(int tag) const { return WaitCtl{rec.p, limit_ns, tag}; }
  // 0, or BN_ERR_SPIN with *msg describing the wait that gave up; the
  // record is cleared (synchronous on s).
  int take(cudaStream_t s, std::string* msg);
  static unsigned long long default_limit_ns();
};

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
