// Gauss-Seidel sweeps in a caller-given visiting order, computed exactly as
// the sequential sweep of the reference's MATLAB gateway
// (Matlab_amg/cf_gauss_seidel_mex.c:58-101):
//   for t in order (reversed when backward): i = order[t]
//     x_i = (b_i - sum_{j != i} a_ij x_j) / d_i,   d_i = first a_ii, else 1
// with the sum in row order and x_j already updated when j comes earlier in
// the order.  On the device: row i depends on its neighbours that come
// earlier; the rows are scheduled by dependency level and swept sync-free
// (flags.cuh), reading the new value of an earlier neighbour (waiting for
// it) and the old value of a later one.  Same operations in the same order,
// so the result is bit-identical to the sequential sweep.
#include "internal.cuh"
#include "flags.cuh"
#include "../../include/amg_b200.h"

#include <cub/cub.cuh>

namespace bn {
namespace {

__global__ void k_gs_pos(const int* __restrict__ order, int n, int backward, int* __restrict__ pos,
                         int* bad) {
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
    const int i = order[t];
    if (i < 0 || i >= n) { atomicExch(bad, 1); continue; }
    if (atomicExch(&pos[i], backward ? n - 1 - t : t) != -1) atomicExch(bad, 1);
  }
}

__global__ void k_gs_diag(const int* __restrict__ ia, const int* __restrict__ ja,
                          const double* __restrict__ a, int n, double* __restrict__ d) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double v = 1.0;
    for (int k = ia[i]; k < ia[i + 1]; k++)
      if (ja[k] == i) { v = a[k]; break; }
    d[i] = v;
  }
}

__global__ void k_gs_dep_count(const int* __restrict__ ia, const int* __restrict__ ja,
                               const int* __restrict__ pos, int n, int* __restrict__ cnt) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    int c = 0;
    for (int k = ia[i]; k < ia[i + 1]; k++) {
      const int j = ja[k];
      c += (j != i && pos[j] < pos[i]);
    }
    cnt[i] = c;
  }
}

__global__ void k_gs_dep_fill(const int* __restrict__ ia, const int* __restrict__ ja,
                              const int* __restrict__ pos, int n, const int* __restrict__ dia,
                              int* __restrict__ dja, double* __restrict__ dval) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    int p = dia[i];
    for (int k = ia[i]; k < ia[i + 1]; k++) {
      const int j = ja[k];
      if (j != i && pos[j] < pos[i]) { dja[p] = j; dval[p] = 0.0; p++; }
    }
  }
}

__device__ __forceinline__ void gs_row(int t, int t_end, const int* __restrict__ ia,
                                       const int* __restrict__ ja, const double* __restrict__ a,
                                       const double* __restrict__ d, const int* __restrict__ pos,
                                       const int* __restrict__ rows, const double* __restrict__ b,
                                       const double* __restrict__ xin,
                                       unsigned long long* o, const WaitCtl& wc) {
  using W = WordOf<double>;
  if (t >= t_end) return;
  const int i = rows[t];
  const int pi = pos[i];
  double s = b[i];
  for (int k = ia[i]; k < ia[i + 1]; k++) {
    const int j = ja[k];
    if (j == i) continue;
    double xj;
    if (pos[j] < pi) {  // updated earlier in this sweep
      unsigned long long u = ld_relaxed(o + j);
      u = wait_word(o, j, u, W::kPending, W::kNaN, wc, i);
      xj = word_value(u);
    } else {
      xj = xin[j];
    }
    s = xsub(s, xmul(a[k], xj));
  }
  unsigned long long r = value_word(xdiv(s, d[i]));
  if (r == W::kPending) r = W::kNaN;
  st_relaxed(o + i, r);
}

// chunks as for the IC(0) sweeps: 32-row pieces of one level, dealt
// round-robin to the warps of a co-resident grid, the warp reconverging
// after every chunk
__global__ void __launch_bounds__(kFlagThreads)
k_gs_flags(const int* __restrict__ ia, const int* __restrict__ ja, const double* __restrict__ a,
           const double* __restrict__ d, const int* __restrict__ pos,
           const int* __restrict__ rows, const int2* __restrict__ chunks, int nchunks,
           const double* __restrict__ b, const double* __restrict__ xin, double* xout,
           WaitCtl wc) {
  unsigned long long* o = reinterpret_cast<unsigned long long*>(xout);
  const int lane = threadIdx.x & 31;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  for (int c = warp; c < nchunks; c += nwarps) {
    const int2 ch = chunks[c];
    gs_row(ch.x + lane, ch.y, ia, ja, a, d, pos, rows, b, xin, o, wc);
    __syncwarp();
  }
}

}  // namespace

// nu sweeps on device data; x holds x0 on entry and the result on exit
void ordered_gs(const CSR& A, const int* d_order, const double* b, double* x, int nu,
                int backward, cudaStream_t s) {
  const int n = A.n;
  if (n == 0 || nu <= 0) return;
  const int g = grid_for(n, 256);
  DBuf<int> pos(n, s), bad(1, s);
  WaitRecord wait;
  wait.init(s);
  pos.fill_bytes(0xff);
  bad.zero();
  BN_LAUNCH(k_gs_pos, g, 256, 0, s, d_order, n, backward ? 1 : 0, pos.p, bad.p);
  BN_REQUIRE(read_scalar(bad.p, s) == 0, BN_ERR_ARG,
             "ordered Gauss-Seidel: the order is not a permutation of 0..n-1");
  DBuf<double> d(n, s);
  BN_LAUNCH(k_gs_diag, g, 256, 0, s, A.ia.p, A.ja.p, A.val.p, n, d.p);
  // dependencies (earlier neighbours) and their transpose
  CSR D, U;
  {
    DBuf<int> cnt((size_t)n + 1, s);
    cnt.zero();
    BN_LAUNCH(k_gs_dep_count, g, 256, 0, s, A.ia.p, A.ja.p, pos.p, n, cnt.p);
    const int dnnz = scan_counts(cnt.p, n, s);
    D.n = D.m = n;
    D.nnz = dnnz;
    D.ia = std::move(cnt);
    D.ja.alloc(dnnz > 0 ? dnnz : 1, s);
    D.val.alloc(dnnz > 0 ? dnnz : 1, s);
    BN_LAUNCH(k_gs_dep_fill, g, 256, 0, s, A.ia.p, A.ja.p, pos.p, n, D.ia.p, D.ja.p, D.val.p);
    transpose(D, U, s, true);
  }
  DBuf<int> rows;
  std::vector<int> lptr;
  level_schedule(D, U, rows, lptr, s);
  DBuf<int2> chunks;
  const int nchunks = upload_chunks(lptr, chunks, s);
  // co-resident grid: every wait ends
  int dev = 0, per_sm = 0, sms = 0;
  BN_CUDA(cudaGetDevice(&dev));
  BN_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_gs_flags, kFlagThreads, 0));
  BN_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  const int grid = sms * (per_sm < 2 ? per_sm : 2);
  BN_REQUIRE(grid > 0, BN_ERR_CUDA, "ordered Gauss-Seidel: sweep grid does not fit");
  DBuf<double> other(n, s);
  double* xin = x;
  double* xout = other.p;
  for (int sw = 0; sw < nu; sw++) {
    BN_CUDA(cudaMemsetAsync(xout, 0xFF, sizeof(double) * (size_t)n, s));
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(kFlagThreads);
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    g_launch_count++;
    BN_CUDA(cudaLaunchKernelEx(&cfg, k_gs_flags, (const int*)A.ia.p, (const int*)A.ja.p,
                               (const double*)A.val.p, (const double*)d.p, (const int*)pos.p,
                               (const int*)rows.p, (const int2*)chunks.p, nchunks, b,
                               (const double*)xin, xout, wait.ctl(WT_GS_ORDERED)));
    std::swap(xin, xout);
  }
  if (xin != x)
    BN_CUDA(cudaMemcpyAsync(x, xin, sizeof(double) * (size_t)n, cudaMemcpyDeviceToDevice, s));
  std::string msg;
  if (wait.take(s, &msg)) throw Error(BN_ERR_SPIN, "ordered Gauss-Seidel: " + msg);
}

}  // namespace bn

// See include/amg_b200.h for the contract.
BN_API int amg_gauss_seidel_ordered(int n, int nnz, const int* ia, const int* ja,
                                    const double* val, const double* b, double* x,
                                    const int* order, int nu, int backward) {
  using namespace bn;
  try {
    BN_REQUIRE(n >= 0 && nnz >= 0 && (n == 0 || (ia && ja && val && b && x && order)),
               BN_ERR_ARG, "amg_gauss_seidel_ordered: invalid arguments");
    if (n == 0 || nu <= 0) {
      set_last_error(BN_OK, "");
      return BN_OK;
    }
    cudaStream_t s = cudaStreamPerThread;
    CSR A;
    A.alloc(n, n, nnz, s, true);
    A.ia.upload(ia, (size_t)n + 1);
    if (nnz) {
      A.ja.upload(ja, (size_t)nnz);
      A.val.upload(val, (size_t)nnz);
    }
    const int f = validate(A.ia.p, A.ja.p, n, n, nnz, s);
    BN_REQUIRE(!(f & 1), BN_ERR_ARG, "CSR row pointers are not a valid 0-based prefix array");
    BN_REQUIRE(!(f & 2), BN_ERR_ARG, "CSR column index out of range");
    DBuf<int> dord(n, s);
    DBuf<double> db(n, s), dx(n, s);
    dord.upload(order, n);
    db.upload(b, n);
    dx.upload(x, n);
    ordered_gs(A, dord.p, db.p, dx.p, nu, backward, s);
    dx.download(x, n);
    BN_CUDA(cudaStreamSynchronize(s));
    set_last_error(BN_OK, "");
    return BN_OK;
  } catch (const Error& e) {
    set_last_error(e.code, e.what());
    return e.code;
  } catch (const std::exception& e) {
    set_last_error(BN_ERR_CUDA, e.what());
    return BN_ERR_CUDA;
  }
}
