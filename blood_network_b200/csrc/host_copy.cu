// Host <-> device copies of caller-owned host arrays (the C ABI's host
// CSR, right-hand sides and solutions).  A copy from pageable memory goes
// through the driver's own small staging buffer at one CPU thread's memcpy
// speed; here large copies go through pinned staging buffers filled (or
// drained) by several host threads, pipelined with the DMA.  Pinned caller
// memory and small copies take cudaMemcpyAsync directly.
#include "common.cuh"

#include <algorithm>
#include <map>
#include <mutex>
#include <thread>
#include <vector>

namespace bn {
namespace {

constexpr size_t kChunk = 32u << 20;     // bytes per staging buffer
constexpr int kStages = 4;               // staging buffers per device
constexpr size_t kDirect = 8u << 20;     // smaller copies go direct

struct Staging {
  char* buf[kStages] = {};
  cudaEvent_t ev[kStages] = {};
  bool ok = false;
};

std::mutex g_mu;                      // one staged copy at a time per process
std::map<int, Staging> g_stage;       // per device

Staging* staging_for_current_device() {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return nullptr;
  Staging& st = g_stage[dev];
  if (st.ok) return &st;
  for (int k = 0; k < kStages; k++) {
    if (cudaHostAlloc((void**)&st.buf[k], kChunk, cudaHostAllocPortable) != cudaSuccess ||
        cudaEventCreateWithFlags(&st.ev[k], cudaEventDisableTiming) != cudaSuccess) {
      cudaGetLastError();
      for (int j = 0; j <= k; j++) {
        if (st.buf[j]) cudaFreeHost(st.buf[j]);
        if (st.ev[j]) cudaEventDestroy(st.ev[j]);
        st.buf[j] = nullptr;
        st.ev[j] = nullptr;
      }
      return nullptr;
    }
  }
  st.ok = true;
  return &st;
}

bool is_pinned(const void* p) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeHost || a.type == cudaMemoryTypeDevice ||
         a.type == cudaMemoryTypeManaged;
}

int copy_threads() {
  static const int t = [] {
    const unsigned hw = std::thread::hardware_concurrency();
    return (int)std::max(1u, std::min(8u, hw ? hw : 1u));
  }();
  return t;
}

// memcpy split over the copy threads
void par_memcpy(char* dst, const char* src, size_t len) {
  const int nt = len >= (4u << 20) ? copy_threads() : 1;
  if (nt == 1) {
    memcpy(dst, src, len);
    return;
  }
  const size_t per = (len + nt - 1) / nt;
  std::vector<std::thread> th;
  for (int t = 1; t < nt; t++) {
    const size_t o = per * t;
    if (o >= len) break;
    th.emplace_back([=]() { memcpy(dst + o, src + o, std::min(per, len - o)); });
  }
  memcpy(dst, src, std::min(per, len));
  for (auto& x : th) x.join();
}

}  // namespace

// Enqueue a host -> device copy on s.  On return the host source has been
// read in full (the caller may reuse it); the DMA may still be running.
void copy_h2d(void* dst, const void* src, size_t bytes, cudaStream_t s) {
  if (bytes == 0) return;
  if (bytes < kDirect || is_pinned(src)) {
    BN_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s));
    return;
  }
  std::lock_guard<std::mutex> lock(g_mu);
  Staging* st = staging_for_current_device();
  if (!st) {
    BN_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s));
    return;
  }
  const char* sp = (const char*)src;
  char* dp = (char*)dst;
  for (size_t off = 0, c = 0; off < bytes; off += kChunk, c++) {
    const int k = (int)(c % kStages);
    const size_t len = std::min(kChunk, bytes - off);
    BN_CUDA(cudaEventSynchronize(st->ev[k]));  // its previous DMA has finished
    par_memcpy(st->buf[k], sp + off, len);
    BN_CUDA(cudaMemcpyAsync(dp + off, st->buf[k], len, cudaMemcpyHostToDevice, s));
    BN_CUDA(cudaEventRecord(st->ev[k], s));
  }
}

// Device -> host copy on s, complete on return (s is synchronised).
void copy_d2h(void* dst, const void* src, size_t bytes, cudaStream_t s) {
  if (bytes == 0) {
    BN_CUDA(cudaStreamSynchronize(s));
    return;
  }
  if (bytes < kDirect || is_pinned(dst)) {
    BN_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, s));
    BN_CUDA(cudaStreamSynchronize(s));
    return;
  }
  std::lock_guard<std::mutex> lock(g_mu);
  Staging* st = staging_for_current_device();
  if (!st) {
    BN_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, s));
    BN_CUDA(cudaStreamSynchronize(s));
    return;
  }
  const char* sp = (const char*)src;
  char* dp = (char*)dst;
  const size_t nchunks = (bytes + kChunk - 1) / kChunk;
  auto issue = [&](size_t c) {
    const int k = (int)(c % kStages);
    const size_t off = c * kChunk, len = std::min(kChunk, bytes - off);
    BN_CUDA(cudaMemcpyAsync(st->buf[k], sp + off, len, cudaMemcpyDeviceToHost, s));
    BN_CUDA(cudaEventRecord(st->ev[k], s));
  };
  // keep up to kStages - 1 chunks in flight ahead of the one being drained
  size_t issued = 0;
  for (; issued < nchunks && issued < (size_t)kStages - 1; issued++) issue(issued);
  for (size_t c = 0; c < nchunks; c++) {
    const int k = (int)(c % kStages);
    const size_t off = c * kChunk, len = std::min(kChunk, bytes - off);
    if (issued < nchunks) issue(issued++);  // reuses the buffer drained last round
    BN_CUDA(cudaEventSynchronize(st->ev[k]));
    par_memcpy(dp + off, st->buf[k], len);
  }
  BN_CUDA(cudaStreamSynchronize(s));
}

}  // namespace bn
