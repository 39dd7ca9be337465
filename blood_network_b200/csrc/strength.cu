// Strength of connection, Ruge-Stuben criterion, on the device.
//
// Follows rs_strength (C_amg1/src/rs_classical.c:30-88):
//   row_max_i = max(0, max_{j != i} -a_ij)        (the running max starts at 0)
//   j is strong for i  iff  j != i  and  -a_ij >= theta * row_max_i
// S keeps A's values and A's in-row order; max_lam = max row length of A,
// floored at 1.  The threshold is one multiply then a compare, exactly as the
// reference, so S is bit-identical for a bit-identical A.
//
// Layout: a group of G lanes handles one row (G = 32 is warp-per-row; G = 8
// for the short rows of vessel-network Laplacians).  Three passes as in the
// reference -- max, count, fill -- with the count/fill order preserved by a
// ballot prefix inside the group.
#include "internal.cuh"

namespace bn {

template <int G>
__device__ __forceinline__ unsigned group_mask() {
  if constexpr (G == 32) {
    return 0xffffffffu;
  } else {
    unsigned lane = threadIdx.x & 31;
    return ((1u << G) - 1u) << (lane & ~(G - 1));
  }
}

template <int G>
__device__ __forceinline__ double row_threshold(const int* __restrict__ ia, const int* __restrict__ ja,
                                                const double* __restrict__ val, int i, double theta,
                                                int gl, unsigned mask) {
  double mx = 0.0;  // only strictly larger values replace it: never -0.0 or NaN
  for (int k = ia[i] + gl; k < ia[i + 1]; k += G) {
    if (ja[k] == i) continue;
    double v = -val[k];
    if (v > mx) mx = v;
  }
#pragma unroll
  for (int off = G / 2; off > 0; off >>= 1) {
    double o = __shfl_xor_sync(mask, mx, off, G);
    if (o > mx) mx = o;
  }
  return xmul(theta, mx);
}

template <int G>
__global__ void k_strength_count(const int* __restrict__ ia, const int* __restrict__ ja,
                                 const double* __restrict__ val, int n, double theta,
                                 int* __restrict__ cnt, double* __restrict__ thr_out,
                                 int* __restrict__ max_len) {
  const int gl = threadIdx.x & (G - 1);
  const unsigned mask = group_mask<G>();
  const int groups = (gridDim.x * blockDim.x) / G;
  int local_max = 0;
  for (int i = (blockIdx.x * blockDim.x + threadIdx.x) / G; i < n; i += groups) {
    double thr = row_threshold<G>(ia, ja, val, i, theta, gl, mask);
    int c = 0;
    for (int k = ia[i] + gl; k < ia[i + 1]; k += G)
      if (ja[k] != i && -val[k] >= thr) c++;
#pragma unroll
    for (int off = G / 2; off > 0; off >>= 1) c += __shfl_xor_sync(mask, c, off, G);
    if (gl == 0) {
      cnt[i] = c;
      thr_out[i] = thr;
      int len = ia[i + 1] - ia[i];
      if (len > local_max) local_max = len;
    }
  }
  if (gl == 0 && local_max > 0) atomicMax(max_len, local_max);
}

template <int G>
__global__ void k_strength_fill(const int* __restrict__ ia, const int* __restrict__ ja,
                                const double* __restrict__ val, int n,
                                const double* __restrict__ thr_in, const int* __restrict__ sia,
                                int* __restrict__ sja, double* __restrict__ sval) {
  const int gl = threadIdx.x & (G - 1);
  const unsigned mask = group_mask<G>();
  const int groups = (gridDim.x * blockDim.x) / G;
  const unsigned lt = (1u << (threadIdx.x & 31)) - 1u;
  for (int i = (blockIdx.x * blockDim.x + threadIdx.x) / G; i < n; i += groups) {
    double thr = thr_in[i];
    int p = sia[i];
    const int a0 = ia[i], a1 = ia[i + 1];
    for (int base = a0; base < a1; base += G) {
      int k = base + gl;
      bool strong = false;
      int c = 0;
      double v = 0.0;
      if (k < a1) {
        c = ja[k];
        v = val[k];
        strong = (c != i) && (-v >= thr);
      }
      unsigned b = __ballot_sync(mask, strong);
      if (strong) {
        int q = p + __popc(b & mask & lt);
        sja[q] = c;
        sval[q] = v;
      }
      p += __popc(b & mask);
    }
  }
}

template <int G>
static void strength_impl(const CSR& A, double theta, CSR& S, int* max_lam, cudaStream_t s) {
  const int n = A.n;
  DBuf<int> cnt((size_t)n + 1, s), mlen(1, s);
  DBuf<double> thr((size_t)(n > 0 ? n : 1), s);
  cnt.zero();
  mlen.zero();
  const int block = 256;
  long long threads = (long long)n * G;
  int grid = grid_for(threads, block, 8);
  if (n > 0)
    BN_LAUNCH(k_strength_count<G>, grid, block, 0, s, A.ia.p, A.ja.p, A.val.p, n, theta, cnt.p,
              thr.p, mlen.p);
  int snnz = scan_counts(cnt.p, n, s);
  int ml = read_scalar(mlen.p, s);
  if (ml < 1) ml = 1;
  *max_lam = ml;
  S.n = n;
  S.m = A.m;
  S.nnz = snnz;
  S.ia = std::move(cnt);
  S.ja.alloc((size_t)(snnz > 0 ? snnz : 1), s);
  S.val.alloc((size_t)(snnz > 0 ? snnz : 1), s);
  if (n > 0 && snnz > 0)
    BN_LAUNCH(k_strength_fill<G>, grid, block, 0, s, A.ia.p, A.ja.p, A.val.p, n, thr.p, S.ia.p,
              S.ja.p, S.val.p);
}

void strength(const CSR& A, double theta, CSR& S, int* max_lam, cudaStream_t s) {
  double avg = A.n > 0 ? (double)A.nnz / A.n : 0.0;
  if (avg <= 8.0)
    strength_impl<8>(A, theta, S, max_lam, s);
  else
    strength_impl<32>(A, theta, S, max_lam, s);
}

}  // namespace bn
