// C/F splitting on the device.
//
// PMIS (bit-exact with pmis_coarsening, C_amg1/src/rs_classical.c:246-371):
//  * G = S u S^T without the diagonal.  Only the neighbour SET matters to the
//    selection and marking rules, so G is never materialised: each kernel
//    walks row i of S and row i of S^T.
//  * w_i = |S^T_i| + rand()/RAND_MAX after srand(12345) (:293-300).  The
//    rand() values come from the host C library itself, so the sequence and
//    the side effect on its global generator state are the reference's.
//  * Rounds are Jacobi style: an undecided i becomes C if no undecided
//    G-neighbour has w_j > w_i (:312-323); with no new C every remaining node
//    becomes C (:325-330); then undecided nodes with a C neighbour become F
//    (:339-348).  One select and one mark kernel per round.
//  * Second pass (:357-364) promotes F points with no strong C neighbour.
//    The reference updates cf in place while scanning i = 0..n-1, so an
//    earlier promotion can keep a later point F.  That ordered rule is
//    reproduced exactly: only "orphan" F points (no C in S_i before the pass)
//    can be promoted, and orphan i is promoted iff no orphan j < i in S_i was
//    promoted -- solved in parallel rounds where a point decides once all of
//    its lower-index orphan dependencies have decided.
//
// RS / HMIS first pass (parallel counterpart of the sequential bucket greedy
// at rs_classical.c:108-229 and :390-486; the HMIS PMIS phase, :493-592,
// never runs because the first pass decides every point): rounds select the
// undecided local maxima of the RS measure lambda_i plus a tie-break in [0,1]
// over G -- for HMIS the reference's own weights lambda_i + rand()/RAND_MAX
// after srand(12345), for RS a hash of the index; undecided points that
// strongly depend on a new C become F;
// every undecided strong dependency of a new F gains lambda += 1.  The C/F
// split therefore differs from the sequential greedy's bucket order; the
// second pass is the reference's (ordered rule above).
#include "internal.cuh"
#include "crand.h"

#include <stdlib.h>
#include <string.h>

#include <vector>

namespace bn {

enum : int { kF = -1, kU = 0, kC = 1, kNewC = 2 };

// Points whose S and S^T rows together hold more than kLongPoint entries
// (hubs of the coarse tree levels, up to ~10^6 entries) are decided by a
// block each in a second launch of every round; the thread-per-point kernels
// skip them.  Every rule below is independent of the order in which points
// are decided within a round, so the split does not change.
constexpr int kLongPoint = 256;
constexpr int kLongThreads = 256;

__device__ __forceinline__ bool long_point(const int* __restrict__ sia,
                                           const int* __restrict__ tia, int i) {
  return (sia[i + 1] - sia[i]) + (tia[i + 1] - tia[i]) > kLongPoint;
}

__global__ void k_long_points(const int* __restrict__ sia, const int* __restrict__ tia, int n,
                              int* __restrict__ list, int* counter) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    if (long_point(sia, tia, i)) list[atomicAdd(counter, 1)] = i;
}

__global__ void k_lambda(const int* __restrict__ sja, int snnz, int* __restrict__ lam) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < snnz; k += gridDim.x * blockDim.x)
    atomicAdd(&lam[sja[k]], 1);
}

__global__ void k_pmis_weights(const int* __restrict__ lam, const int* __restrict__ rnd, int n,
                               double* __restrict__ w, int* __restrict__ cf) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    // (REAL)lambda_i + (REAL)rand() / (REAL)RAND_MAX
    w[i] = xadd((double)lam[i], xdiv((double)rnd[i], (double)RAND_MAX));
    cf[i] = kU;
  }
}

__device__ __forceinline__ bool undecided(int c) { return c == kU || c == kNewC; }

// select: undecided i with no undecided G-neighbour of larger weight -> kNewC
__global__ void k_select(const int* __restrict__ sia, const int* __restrict__ sja,
                         const int* __restrict__ tia, const int* __restrict__ tja,
                         const double* __restrict__ w, int n, int* cf, int* counter) {
  int local = 0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    if (cf[i] != kU || long_point(sia, tia, i)) continue;
    const double wi = w[i];
    bool is_max = true;
    for (int k = sia[i]; k < sia[i + 1] && is_max; k++) {
      int j = sja[k];
      if (undecided(((volatile int*)cf)[j]) && w[j] > wi) is_max = false;
    }
    for (int k = tia[i]; k < tia[i + 1] && is_max; k++) {
      int j = tja[k];
      if (undecided(((volatile int*)cf)[j]) && w[j] > wi) is_max = false;
    }
    if (is_max) {
      cf[i] = kNewC;
      local++;
    }
  }
  if (local) atomicAdd(counter, local);
}

__global__ void __launch_bounds__(kLongThreads)
k_select_long(const int* __restrict__ sia, const int* __restrict__ sja,
              const int* __restrict__ tia, const int* __restrict__ tja,
              const double* __restrict__ w, const int* __restrict__ list, int m, int* cf,
              int* counter) {
  for (int t = blockIdx.x; t < m; t += gridDim.x) {
    const int i = list[t];
    if (cf[i] != kU) continue;  // uniform over the block
    const double wi = w[i];
    bool beaten = false;
    for (int k = sia[i] + threadIdx.x; k < sia[i + 1] && !beaten; k += blockDim.x) {
      const int j = sja[k];
      beaten = undecided(((volatile int*)cf)[j]) && w[j] > wi;
    }
    for (int k = tia[i] + threadIdx.x; k < tia[i + 1] && !beaten; k += blockDim.x) {
      const int j = tja[k];
      beaten = undecided(((volatile int*)cf)[j]) && w[j] > wi;
    }
    if (!__syncthreads_or(beaten) && threadIdx.x == 0) {
      cf[i] = kNewC;
      atomicAdd(counter, 1);
    }
    __syncthreads();
  }
}

// PMIS mark: new C -> C; undecided with any C in G -> F
__global__ void k_pmis_mark(const int* __restrict__ sia, const int* __restrict__ sja,
                            const int* __restrict__ tia, const int* __restrict__ tja, int n,
                            int* cf, int* counter) {
  int local = 0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    if (long_point(sia, tia, i)) continue;
    int c = cf[i];
    if (c == kNewC) {
      ((volatile int*)cf)[i] = kC;
      continue;
    }
    if (c != kU) continue;
    bool hit = false;
    for (int k = sia[i]; k < sia[i + 1] && !hit; k++) {
      int cj = ((volatile int*)cf)[sja[k]];
      hit = (cj == kC || cj == kNewC);
    }
    for (int k = tia[i]; k < tia[i + 1] && !hit; k++) {
      int cj = ((volatile int*)cf)[tja[k]];
      hit = (cj == kC || cj == kNewC);
    }
    if (hit) {
      ((volatile int*)cf)[i] = kF;
      local++;
    }
  }
  if (local) atomicAdd(counter, local);
}

// mark for the long points (PMIS: S and S^T; RS: S only, new F flagged)
template <bool PMIS>
__global__ void __launch_bounds__(kLongThreads)
k_mark_long(const int* __restrict__ sia, const int* __restrict__ sja,
            const int* __restrict__ tia, const int* __restrict__ tja,
            const int* __restrict__ list, int m, int* cf, int* __restrict__ new_f, int* counter) {
  for (int t = blockIdx.x; t < m; t += gridDim.x) {
    const int i = list[t];
    const int c = ((volatile int*)cf)[i];
    __syncthreads();  // every thread has read cf[i] before thread 0 may change it
    if (!PMIS && threadIdx.x == 0) new_f[i] = 0;
    if (c == kNewC) {
      if (threadIdx.x == 0) ((volatile int*)cf)[i] = kC;
      continue;
    }
    if (c != kU) continue;
    bool hit = false;
    for (int k = sia[i] + threadIdx.x; k < sia[i + 1] && !hit; k += blockDim.x) {
      const int cj = ((volatile int*)cf)[sja[k]];
      hit = (cj == kC || cj == kNewC);
    }
    if (PMIS)
      for (int k = tia[i] + threadIdx.x; k < tia[i + 1] && !hit; k += blockDim.x) {
        const int cj = ((volatile int*)cf)[tja[k]];
        hit = (cj == kC || cj == kNewC);
      }
    if (__syncthreads_or(hit) && threadIdx.x == 0) {
      ((volatile int*)cf)[i] = kF;
      if (!PMIS) new_f[i] = 1;
      atomicAdd(counter, 1);
    }
  }
}

__global__ void k_all_undecided_to_c(int n, int* cf) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    if (cf[i] == kU || cf[i] == kNewC) cf[i] = kC;
}

// ---- RS-style first pass (HMIS / RS)
__device__ __forceinline__ double tie_frac(int i) {
  unsigned x = (unsigned)i * 0x9E3779B9u;
  x ^= x >> 16; x *= 0x7feb352du; x ^= x >> 15; x *= 0x846ca68bu; x ^= x >> 16;
  return (double)(x >> 1) * (1.0 / 2147483648.0);
}

__global__ void k_rs_measure(const int* __restrict__ lam, int n, double* __restrict__ w) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    w[i] = (double)lam[i] + tie_frac(i);
}

// RS mark: new C -> C; undecided i with a (new) C in S_i -> F (flagged new_f)
__global__ void k_rs_mark(const int* __restrict__ sia, const int* __restrict__ sja,
                          const int* __restrict__ tia, int n, int* cf,
                          int* __restrict__ new_f, int* counter) {
  int local = 0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    if (long_point(sia, tia, i)) continue;
    int c = cf[i];
    new_f[i] = 0;
    if (c == kNewC) {
      ((volatile int*)cf)[i] = kC;
      continue;
    }
    if (c != kU) continue;
    bool hit = false;
    for (int k = sia[i]; k < sia[i + 1] && !hit; k++) {
      int cj = ((volatile int*)cf)[sja[k]];
      hit = (cj == kC || cj == kNewC);
    }
    if (hit) {
      ((volatile int*)cf)[i] = kF;
      new_f[i] = 1;
      local++;
    }
  }
  if (local) atomicAdd(counter, local);
}

// each new F raises the measure of its undecided strong dependencies
// (w stays an integer plus a fixed fraction < 1, so the += 1.0 are exact and
// their order does not matter)
__global__ void k_rs_lambda_update(const int* __restrict__ sia, const int* __restrict__ sja,
                                   const int* __restrict__ tia, int n,
                                   const int* __restrict__ cf, const int* __restrict__ new_f,
                                   double* __restrict__ w) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    if (!new_f[i] || long_point(sia, tia, i)) continue;
    for (int k = sia[i]; k < sia[i + 1]; k++) {
      int j = sja[k];
      if (cf[j] == kU) atomicAdd(&w[j], 1.0);
    }
  }
}
__global__ void __launch_bounds__(kLongThreads)
k_rs_lambda_update_long(const int* __restrict__ sia, const int* __restrict__ sja,
                        const int* __restrict__ list, int m, const int* __restrict__ cf,
                        const int* __restrict__ new_f, double* __restrict__ w) {
  for (int t = blockIdx.x; t < m; t += gridDim.x) {
    const int i = list[t];
    if (!new_f[i]) continue;
    for (int k = sia[i] + threadIdx.x; k < sia[i + 1]; k += blockDim.x) {
      const int j = sja[k];
      if (cf[j] == kU) atomicAdd(&w[j], 1.0);
    }
  }
}

// ---- second pass (ordered promotion of orphan F points)
__global__ void k_orphans(const int* __restrict__ sia, const int* __restrict__ sja, int n,
                          const int* __restrict__ cf, int* __restrict__ orphan,
                          int* __restrict__ list, int* counter) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    int o = 0;
    if (cf[i] == kF) {
      o = 1;
      for (int k = sia[i]; k < sia[i + 1]; k++)
        if (cf[sja[k]] == kC) { o = 0; break; }
    }
    orphan[i] = o;
    if (o) list[atomicAdd(counter, 1)] = i;
  }
}

// state: 0 pending, 1 promoted, 2 stays F (only meaningful for orphans)
__global__ void k_orphan_round(const int* __restrict__ sia, const int* __restrict__ sja,
                               const int* __restrict__ list, int m,
                               const int* __restrict__ orphan, int* state, int* pending) {
  int local = 0;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < m; t += gridDim.x * blockDim.x) {
    int i = list[t];
    if (((volatile int*)state)[i] != 0) continue;
    bool wait = false, blocked = false;
    for (int k = sia[i]; k < sia[i + 1]; k++) {
      int j = sja[k];
      if (j >= i || !orphan[j]) continue;
      int st = ((volatile int*)state)[j];
      if (st == 1) { blocked = true; break; }
      if (st == 0) wait = true;
    }
    if (blocked)
      ((volatile int*)state)[i] = 2;
    else if (!wait)
      ((volatile int*)state)[i] = 1;
    else
      local++;
  }
  if (local) atomicAdd(pending, local);
}

__global__ void k_orphan_apply(const int* __restrict__ list, int m, const int* __restrict__ state,
                               int* __restrict__ cf) {
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < m; t += gridDim.x * blockDim.x) {
    int i = list[t];
    if (state[i] == 1) cf[i] = kC;
  }
}

__global__ void k_count_c(const int* __restrict__ cf, int n, int* counter) {
  int local = 0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    local += (cf[i] == kC);
  for (int off = 16; off > 0; off >>= 1) local += __shfl_xor_sync(0xffffffffu, local, off);
  if ((threadIdx.x & 31) == 0 && local) atomicAdd(counter, local);
}

// The first n draws of rand() after srand(seed) (crand.h), on the device:
// thread j produces draws [j C, (j+1) C) from its starting window, which it
// forms from the first window and the jump matrices of j's set bits.
constexpr int kCrandStep = 2048;  // draws per thread (a multiple of 32)

__global__ void __launch_bounds__(128)
k_crand_chunks(const uint32_t* __restrict__ pw, int nbits, const uint32_t* __restrict__ first,
               long long n, int* __restrict__ out) {
  const long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (j * kCrandStep >= n) return;
  uint32_t v[31];
#pragma unroll
  for (int i = 0; i < 31; i++) v[i] = first[i];
  for (int b = 0; b < nbits; b++) {
    if (!((j >> b) & 1)) continue;
    const uint32_t* m = pw + (size_t)b * 961;
    uint32_t t[31];
#pragma unroll
    for (int i = 0; i < 31; i++) {
      uint32_t acc = 0;
#pragma unroll
      for (int k = 0; k < 31; k++) acc += m[i * 31 + k] * v[k];
      t[i] = acc;
    }
#pragma unroll
    for (int i = 0; i < 31; i++) v[i] = t[i];
  }
  // ring slot (q & 31) holds position q of the chunk (q = -31 .. -1 first)
  uint32_t ring[32];
  ring[0] = 0;
#pragma unroll
  for (int i = 1; i < 32; i++) ring[i] = v[i - 1];
  const long long base = j * kCrandStep;
  for (int q0 = 0; q0 < kCrandStep; q0 += 32) {
#pragma unroll
    for (int i = 0; i < 32; i++) {
      const uint32_t r = ring[(i + 1) & 31] + ring[(i + 29) & 31];  // r[q-31] + r[q-3]
      ring[i] = r;
      const long long k = base + q0 + i;
      if (k < n) out[k] = (int)(r >> 1);
    }
  }
}

static void crand_device(unsigned seed, int* out, long long n, cudaStream_t s) {
  if (n <= 0) return;
  const long long nchunks = (n + kCrandStep - 1) / kCrandStep;
  int nbits = 1;
  while ((1LL << nbits) < nchunks) nbits++;
  std::vector<CrandMat> pw(nbits);
  crand_jump_matrices(kCrandStep, nbits, pw.data());
  std::vector<uint32_t> h((size_t)nbits * 961 + 31);
  for (int b = 0; b < nbits; b++)
    for (int i = 0; i < 31; i++)
      for (int k = 0; k < 31; k++) h[(size_t)b * 961 + i * 31 + k] = pw[b].a[i][k];
  crand_first_window(seed, h.data() + (size_t)nbits * 961);
  DBuf<uint32_t> d(h.size(), s);
  d.upload(h.data(), h.size());
  BN_LAUNCH(k_crand_chunks, (int)((nchunks + 127) / 128), 128, 0, s, d.p, nbits,
            d.p + (size_t)nbits * 961, n, out);
  BN_CUDA(cudaStreamSynchronize(s));  // h must outlive the copy
}

static void select_round(const CSR& S, const CSR& T, const double* w, int n, int* cf,
                         const int* longs, int nlong, int glong, int* ctr, cudaStream_t s) {
  BN_LAUNCH(k_select, grid_for(n, 256), 256, 0, s, S.ia.p, S.ja.p, T.ia.p, T.ja.p, w, n, cf, ctr);
  if (nlong)
    BN_LAUNCH(k_select_long, glong, kLongThreads, 0, s, S.ia.p, S.ja.p, T.ia.p, T.ja.p, w, longs,
              nlong, cf, ctr);
}

static void second_pass(const CSR& S, int* cf, cudaStream_t s) {
  const int n = S.n;
  DBuf<int> orphan(n, s), list(n, s), state(n, s), ctr(2, s);
  ctr.zero();
  state.zero();
  const int g = grid_for(n, 256);
  BN_LAUNCH(k_orphans, g, 256, 0, s, S.ia.p, S.ja.p, n, cf, orphan.p, list.p, ctr.p);
  int m = read_scalar(ctr.p, s);
  if (m == 0) return;
  int pending = m;
  for (int round = 0; round <= m && pending > 0; round++) {
    BN_CUDA(cudaMemsetAsync(ctr.p + 1, 0, sizeof(int), s));
    BN_LAUNCH(k_orphan_round, grid_for(m, 256), 256, 0, s, S.ia.p, S.ja.p, list.p, m, orphan.p,
              state.p, ctr.p + 1);
    pending = read_scalar(ctr.p + 1, s);
  }
  BN_REQUIRE(pending == 0, BN_ERR_SPIN, "second pass did not settle");
  BN_LAUNCH(k_orphan_apply, grid_for(m, 256), 256, 0, s, list.p, m, state.p, cf);
}

static int count_c(const int* cf, int n, cudaStream_t s) {
  DBuf<int> c(1, s);
  c.zero();
  BN_LAUNCH(k_count_c, grid_for(n, 256), 256, 0, s, cf, n, c.p);
  return read_scalar(c.p, s);
}

int coarsen(const CSR& S, int method, int max_lam, int* cf, cudaStream_t s) {
  (void)max_lam;
  const int n = S.n;
  if (n == 0) return 0;
  CSR T;  // S^T structure: row i lists the points that strongly depend on i
  transpose(S, T, s, false);
  DBuf<int> lam(n, s), ctr(2, s);
  DBuf<double> w(n, s);
  lam.zero();
  const int g = grid_for(n, 256);
  if (S.nnz > 0) BN_LAUNCH(k_lambda, grid_for(S.nnz, 256), 256, 0, s, S.ja.p, S.nnz, lam.p);
  DBuf<int> longs;
  int nlong = 0;
  {
    DBuf<int> lst(n, s);
    ctr.zero();
    BN_LAUNCH(k_long_points, g, 256, 0, s, S.ia.p, T.ia.p, n, lst.p, ctr.p);
    nlong = read_scalar(ctr.p, s);
    if (nlong > 0) longs = std::move(lst);
  }
  const int glong = nlong < 4096 ? nlong : 4096;

  if (method == COARSEN_PMIS) {
    // rand() sequence after srand(12345), drawn from the host C library
    std::vector<int> h(n);
    srand(12345);
    for (int i = 0; i < n; i++) h[i] = rand();
    DBuf<int> rnd(n, s);
    rnd.upload(h.data(), n);
    BN_LAUNCH(k_pmis_weights, g, 256, 0, s, lam.p, rnd.p, n, w.p, cf);
    BN_CUDA(cudaStreamSynchronize(s));  // h must outlive the copy
    long long undecided = n;
    for (long long round = 0; undecided > 0 && round <= n; round++) {
      ctr.zero();
      select_round(S, T, w.p, n, cf, longs.p, nlong, glong, ctr.p, s);
      int nc = read_scalar(ctr.p, s);
      if (nc == 0) {
        BN_LAUNCH(k_all_undecided_to_c, g, 256, 0, s, n, cf);
        undecided = 0;
        break;
      }
      BN_LAUNCH(k_pmis_mark, g, 256, 0, s, S.ia.p, S.ja.p, T.ia.p, T.ja.p, n, cf, ctr.p + 1);
      if (nlong)
        BN_LAUNCH(k_mark_long<true>, glong, kLongThreads, 0, s, S.ia.p, S.ja.p, T.ia.p, T.ja.p,
                  longs.p, nlong, cf, (int*)nullptr, ctr.p + 1);
      int nf = read_scalar(ctr.p + 1, s);
      undecided -= (long long)nc + nf;
    }
    BN_REQUIRE(undecided <= 0, BN_ERR_SPIN, "PMIS did not settle");
  } else {
    // RS measure: lambda_i = |S^T_i|; the classical RS routine leaves
    // lambda_0 at zero (rs_classical.c:118-123), reproduced here.
    if (method == COARSEN_RS) BN_CUDA(cudaMemsetAsync(lam.p, 0, sizeof(int), s));
    DBuf<int> rnd;
    if (method == COARSEN_HMIS) {
      // ties between equal measures: the reference HMIS's weights
      // lambda_i + rand()/RAND_MAX after srand(12345) (rs_classical.c:
      // 542-551), one draw per point in index order.  The sequence comes
      // from a restatement of the C library's generator (crand.h, drawn on the
      // device in chunks from jump-ahead windows), so the
      // caller's rand() state is left alone as the reference's first pass
      // leaves it.
      rnd.alloc(n, s);
      crand_device(12345u, rnd.p, n, s);
      BN_LAUNCH(k_pmis_weights, g, 256, 0, s, lam.p, rnd.p, n, w.p, cf);
    } else {
      BN_LAUNCH(k_rs_measure, g, 256, 0, s, lam.p, n, w.p);
    }
    BN_CUDA(cudaMemsetAsync(cf, 0, sizeof(int) * n, s));
    DBuf<int> new_f(n, s);
    long long undecided = n;
    for (long long round = 0; undecided > 0 && round <= n; round++) {
      ctr.zero();
      select_round(S, T, w.p, n, cf, longs.p, nlong, glong, ctr.p, s);
      int nc = read_scalar(ctr.p, s);
      if (nc == 0) {
        BN_LAUNCH(k_all_undecided_to_c, g, 256, 0, s, n, cf);
        undecided = 0;
        break;
      }
      BN_LAUNCH(k_rs_mark, g, 256, 0, s, S.ia.p, S.ja.p, T.ia.p, n, cf, new_f.p, ctr.p + 1);
      if (nlong)
        BN_LAUNCH(k_mark_long<false>, glong, kLongThreads, 0, s, S.ia.p, S.ja.p, T.ia.p, T.ja.p,
                  longs.p, nlong, cf, new_f.p, ctr.p + 1);
      BN_LAUNCH(k_rs_lambda_update, g, 256, 0, s, S.ia.p, S.ja.p, T.ia.p, n, cf, new_f.p, w.p);
      if (nlong)
        BN_LAUNCH(k_rs_lambda_update_long, glong, kLongThreads, 0, s, S.ia.p, S.ja.p, longs.p,
                  nlong, cf, new_f.p, w.p);
      int nf = read_scalar(ctr.p + 1, s);
      undecided -= (long long)nc + nf;
    }
    BN_REQUIRE(undecided <= 0, BN_ERR_SPIN, "RS first pass did not settle");
  }
  second_pass(S, cf, s);
  return count_c(cf, n, s);
}

}  // namespace bn
