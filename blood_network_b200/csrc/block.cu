// Many right-hand sides on one hierarchy: the PCG of every column runs at
// once over block vectors, so that each pass over a matrix serves all K
// columns (SpMM instead of K SpMVs) and each latency-bound step (a colour
// class, an IC(0) level, a coarse level) is taken once for all columns.
//
// Layout: a block vector is row-major n x K (K <= 64), row i's K values
// contiguous, so the gather of x_j for an entry a_ij is one coalesced
// 8K- (FP64) or 4K-byte (FP32) read.  A warp takes a row, lane c (and
// c + 32) a column; every row sum runs over the row's entries in storage
// order.  Rows longer than kLongRow take a block of 8 warps, each summing a
// fixed stride of the row, combined in warp order.
//
// Each column keeps its own PCG (amg_pcg, C_amg1/src/amg_pcg.c:12-101):
// its own alpha, beta, stopping test and iteration count; a column that has
// met the test is frozen (alpha = 0) while the others go on.  The
// preconditioner is the same three-stage AMG + IC(0) operator
// (amg_ichol_precond.c:22-48) applied to all columns; the IC(0) sweeps step
// through the factor's dependency levels once for all columns.
#include "solver.cuh"

namespace bn {
namespace {

constexpr int kMaxK = 64;
constexpr int kBlkWarps = 8;  // warps per block in the row kernels

template <class T> __device__ __forceinline__ T bmul(T a, T b);
template <> __device__ __forceinline__ double bmul(double a, double b) { return __dmul_rn(a, b); }
template <> __device__ __forceinline__ float bmul(float a, float b) { return __fmul_rn(a, b); }
template <class T> __device__ __forceinline__ T badd(T a, T b);
template <> __device__ __forceinline__ double badd(double a, double b) { return __dadd_rn(a, b); }
template <> __device__ __forceinline__ float badd(float a, float b) { return __fadd_rn(a, b); }
template <class T> __device__ __forceinline__ T bsub(T a, T b);
template <> __device__ __forceinline__ double bsub(double a, double b) { return __dsub_rn(a, b); }
template <> __device__ __forceinline__ float bsub(float a, float b) { return __fsub_rn(a, b); }

enum { BM_Y = 0, BM_RES = 1, BM_ADD = 2 };
constexpr int kLongWarps = 32;  // warps per block for rows longer than kLongRow

// Row sum of a warp over entries k0..k1-1 in storage order: the lanes load
// 32 entries at a time (one coalesced read of ja and a), then every entry is
// broadcast by shuffle and each lane accumulates its columns, so the x
// gathers of consecutive entries do not wait on one another's index loads.
// SUB: s -= a_ij x_j (triangular rows) instead of s += ; DIAG >= 0: the
// entry with column DIAG is not summed, its value goes to *d.
template <class T, bool SUB>
__device__ __forceinline__ void warp_row_sum(int k0, int k1, const int* __restrict__ ja,
                                             const T* __restrict__ a, const T* X, int K,
                                             int lane, bool c0, bool c1, int diag, T& s0, T& s1,
                                             T* d, bool* hit = nullptr) {
  for (int base = k0; base < k1; base += 32) {
    const int kk = base + lane;
    int jv = 0;
    T av = T(0);
    if (kk < k1) {
      jv = ja[kk];
      av = a[kk];
    }
    const int m = min(32, k1 - base);
#pragma unroll 4
    for (int e = 0; e < m; e++) {
      const int j = __shfl_sync(0xffffffffu, jv, e);
      const T v = __shfl_sync(0xffffffffu, av, e);
      if (j == diag) {  // uniform over the warp (j is broadcast)
        *d = v;
        if (hit) *hit = true;
        continue;
      }
      const T* xr = X + (size_t)j * K;
      if (SUB) {
        if (c0) s0 = bsub(s0, bmul(v, xr[lane]));
        if (c1) s1 = bsub(s1, bmul(v, xr[lane + 32]));
      } else {
        if (c0) s0 = badd(s0, bmul(v, xr[lane]));
        if (c1) s1 = badd(s1, bmul(v, xr[lane + 32]));
      }
    }
  }
}

// ---------------------------------------------------------------- SpMM
// Y = A X | B - A X | Y + A X for the rows of [0, n) (rows longer than
// kLongRow skipped when skip_long: k_spmm_long takes them)
template <class T, int MODE>
__global__ void __launch_bounds__(32 * kBlkWarps)
k_spmm(const int* __restrict__ ia, const int* __restrict__ ja, const T* __restrict__ a, int n,
       const T* __restrict__ X, const T* __restrict__ B, T* __restrict__ Y, int K, int skip_long) {
  const int lane = threadIdx.x & 31;
  const int nw = (gridDim.x * blockDim.x) >> 5;
  const bool c0 = lane < K, c1 = lane + 32 < K;
  for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < n; i += nw) {
    const int k0 = ia[i], k1 = ia[i + 1];
    if (skip_long && k1 - k0 > kLongRow) continue;
    T s0 = T(0), s1 = T(0);
    warp_row_sum<T, false>(k0, k1, ja, a, X, K, lane, c0, c1, -1, s0, s1, nullptr);
    T* yr = Y + (size_t)i * K;
    const T* br = B ? B + (size_t)i * K : nullptr;
    if (c0) yr[lane] = MODE == BM_Y ? s0 : (MODE == BM_RES ? bsub(br[lane], s0) : badd(yr[lane], s0));
    if (c1)
      yr[lane + 32] =
          MODE == BM_Y ? s1 : (MODE == BM_RES ? bsub(br[lane + 32], s1) : badd(yr[lane + 32], s1));
  }
}

// a block of kLongWarps warps per long row: warp w sums the w-th of
// kLongWarps consecutive pieces of the row (storage order within a piece),
// the pieces' sums are combined in piece order
__device__ __forceinline__ void long_piece(int k0, int k1, int w, int* p0, int* p1) {
  const int len = k1 - k0, per = (len + kLongWarps - 1) / kLongWarps;
  *p0 = min(k1, k0 + w * per);
  *p1 = min(k1, *p0 + per);
}

template <class T, int MODE>
__global__ void __launch_bounds__(32 * kLongWarps)
k_spmm_long(const int* __restrict__ ia, const int* __restrict__ ja, const T* __restrict__ a,
            const int* __restrict__ lrows, int nl, const T* __restrict__ X,
            const T* __restrict__ B, T* __restrict__ Y, int K) {
  __shared__ T part[kLongWarps][kMaxK];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const bool c0 = lane < K, c1 = lane + 32 < K;
  for (int q = blockIdx.x; q < nl; q += gridDim.x) {
    const int i = lrows[q];
    T s0 = T(0), s1 = T(0);
    int p0, p1;
    long_piece(ia[i], ia[i + 1], w, &p0, &p1);
    warp_row_sum<T, false>(p0, p1, ja, a, X, K, lane, c0, c1, -1, s0, s1, nullptr);
    part[w][lane] = s0;
    part[w][lane + 32] = s1;
    __syncthreads();
    if (w == 0) {
      T t0 = T(0), t1 = T(0);
      for (int u = 0; u < kLongWarps; u++) {
        t0 = badd(t0, part[u][lane]);
        t1 = badd(t1, part[u][lane + 32]);
      }
      T* yr = Y + (size_t)i * K;
      const T* br = B ? B + (size_t)i * K : nullptr;
      if (c0) yr[lane] = MODE == BM_Y ? t0 : (MODE == BM_RES ? bsub(br[lane], t0) : badd(yr[lane], t0));
      if (c1)
        yr[lane + 32] =
            MODE == BM_Y ? t1 : (MODE == BM_RES ? bsub(br[lane + 32], t1) : badd(yr[lane + 32], t1));
    }
    __syncthreads();
  }
}

template <class T>
void spmm(int mode, const DevMat<T>& A, const T* X, const T* B, T* Y, int K, cudaStream_t s) {
  if (A.n == 0) return;
  const int g = grid_for((long long)A.n * 32, 32 * kBlkWarps, 8);
  const int skip = A.lrows != nullptr && A.nlong > 0;
  const int gl = A.nlong < 4096 ? A.nlong : 4096;
  switch (mode) {
    case BM_Y:
      BN_LAUNCH((k_spmm<T, BM_Y>), g, 32 * kBlkWarps, 0, s, A.ia, A.ja, A.val, A.n, X, B, Y, K, skip);
      if (skip)
        BN_LAUNCH((k_spmm_long<T, BM_Y>), gl, 32 * kLongWarps, 0, s, A.ia, A.ja, A.val, A.lrows,
                  A.nlong, X, B, Y, K);
      break;
    case BM_RES:
      BN_LAUNCH((k_spmm<T, BM_RES>), g, 32 * kBlkWarps, 0, s, A.ia, A.ja, A.val, A.n, X, B, Y, K,
                skip);
      if (skip)
        BN_LAUNCH((k_spmm_long<T, BM_RES>), gl, 32 * kLongWarps, 0, s, A.ia, A.ja, A.val, A.lrows,
                  A.nlong, X, B, Y, K);
      break;
    default:
      BN_LAUNCH((k_spmm<T, BM_ADD>), g, 32 * kBlkWarps, 0, s, A.ia, A.ja, A.val, A.n, X, B, Y, K,
                skip);
      if (skip)
        BN_LAUNCH((k_spmm_long<T, BM_ADD>), gl, 32 * kLongWarps, 0, s, A.ia, A.ja, A.val, A.lrows,
                  A.nlong, X, B, Y, K);
      break;
  }
}

// ---------------------------------------------------------------- smoothers
// Gauss-Seidel on one colour class (rows r0 .. r0+nr-1 of the solve
// numbering, the last nlong of them long): x_i = (b_i - sum_{j != i} a_ij
// x_j) / a_ii (1 without a diagonal entry), written to X in place or, for an
// overflow (Jacobi) class, to OUT row t.
template <class T>
__global__ void __launch_bounds__(32 * kBlkWarps)
k_gsm(const int* __restrict__ ia, const int* __restrict__ ja, const T* __restrict__ a, int r0,
      int nshort, const T* __restrict__ B, T* X, T* __restrict__ OUT, int K) {
  const int lane = threadIdx.x & 31;
  const int nw = (gridDim.x * blockDim.x) >> 5;
  const bool c0 = lane < K, c1 = lane + 32 < K;
  for (int t = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; t < nshort; t += nw) {
    const int i = r0 + t;
    T s0 = T(0), s1 = T(0), d = T(1);
    warp_row_sum<T, false>(ia[i], ia[i + 1], ja, a, X, K, lane, c0, c1, i, s0, s1, &d);
    const T* br = B + (size_t)i * K;
    T* o = OUT ? OUT + (size_t)t * K : X + (size_t)i * K;
    if (c0) o[lane] = bsub(br[lane], s0) / d;
    if (c1) o[lane + 32] = bsub(br[lane + 32], s1) / d;
  }
}

template <class T>
__global__ void __launch_bounds__(32 * kLongWarps)
k_gsm_long(const int* __restrict__ ia, const int* __restrict__ ja, const T* __restrict__ a,
           int r0, int nshort, int nlong, const T* __restrict__ B, T* X, T* __restrict__ OUT,
           int K) {
  __shared__ T part[kLongWarps][kMaxK];
  __shared__ T dsh;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const bool c0 = lane < K, c1 = lane + 32 < K;
  for (int q = blockIdx.x; q < nlong; q += gridDim.x) {
    const int t = nshort + q, i = r0 + t;
    if (threadIdx.x == 0) dsh = T(1);
    __syncthreads();
    T s0 = T(0), s1 = T(0), d = T(1);
    int p0, p1;
    long_piece(ia[i], ia[i + 1], w, &p0, &p1);
    bool hit = false;
    warp_row_sum<T, false>(p0, p1, ja, a, X, K, lane, c0, c1, i, s0, s1, &d, &hit);
    if (hit && lane == 0) dsh = d;  // the warp whose piece holds the diagonal entry
    part[w][lane] = s0;
    part[w][lane + 32] = s1;
    __syncthreads();
    if (w == 0) {
      T t0 = T(0), t1 = T(0);
      for (int u = 0; u < kLongWarps; u++) {
        t0 = badd(t0, part[u][lane]);
        t1 = badd(t1, part[u][lane + 32]);
      }
      const T d = dsh;
      const T* br = B + (size_t)i * K;
      T* o = OUT ? OUT + (size_t)t * K : X + (size_t)i * K;
      if (c0) o[lane] = bsub(br[lane], t0) / d;
      if (c1) o[lane + 32] = bsub(br[lane + 32], t1) / d;
    }
    __syncthreads();
  }
}

template <class T>
void gs_class_block(const DevMat<T>& A, int r0, int nr, int nlong, const T* B, T* X, T* OUT,
                    int K, cudaStream_t s) {
  const int nshort = nr - nlong;
  if (nshort > 0)
    BN_LAUNCH(k_gsm<T>, grid_for((long long)nshort * 32, 32 * kBlkWarps, 8), 32 * kBlkWarps, 0, s,
              A.ia, A.ja, A.val, r0, nshort, B, X, OUT, K);
  if (nlong > 0)
    BN_LAUNCH(k_gsm_long<T>, nlong < 4096 ? nlong : 4096, 32 * kLongWarps, 0, s, A.ia, A.ja, A.val,
              r0, nshort, nlong, B, X, OUT, K);
}

// ---------------------------------------------------------------- element-wise
template <class T>
__global__ void k_bcopy_rows(const T* __restrict__ src, size_t m, T* __restrict__ dst) {
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < m;
       e += (size_t)gridDim.x * blockDim.x)
    dst[e] = src[e];
}
template <class T>
__global__ void k_badd(const T* __restrict__ u, const T* __restrict__ v, size_t m,
                       T* __restrict__ out) {
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < m;
       e += (size_t)gridDim.x * blockDim.x)
    out[e] = badd(u[e], v[e]);
}
template <class D, class S>
__global__ void k_bconv(const S* __restrict__ u, size_t m, D* __restrict__ out) {
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < m;
       e += (size_t)gridDim.x * blockDim.x)
    out[e] = (D)u[e];
}
// x_i += omega * r_i / d_i (Jacobi / L1 smoothers)
template <class T>
__global__ void k_bscaled(T* __restrict__ x, const T* __restrict__ r, const double* __restrict__ d,
                          T omega, int n, int K) {
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < (size_t)n * K;
       e += (size_t)gridDim.x * blockDim.x) {
    const T di = (T)d[e / K];
    x[e] = badd(x[e], bmul(omega, r[e] / di));
  }
}
// ---------------------------------------------------------------- coarse
// X = Ainv B (FP64 accumulation), one thread per (row, column)
template <class T>
__global__ void k_dense_apply_m(const double* __restrict__ Ainv, int n, const T* __restrict__ B,
                                T* __restrict__ X, int K) {
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < (size_t)n * K;
       e += (size_t)gridDim.x * blockDim.x) {
    const int i = (int)(e / K), c = (int)(e % K);
    const double* row = Ainv + (size_t)i * n;
    double acc = 0.0;
    for (int k = 0; k < n; k++) acc += row[k] * (double)B[(size_t)k * K + c];
    X[e] = (T)acc;
  }
}

// ---------------------------------------------------------------- IC(0)
// one level-ordered row of L (or L^T), all columns: warp per row
template <class T>
__device__ __forceinline__ void tri_row_m(int t, const int* __restrict__ ia,
                                          const int* __restrict__ ja, const T* __restrict__ val,
                                          const T* __restrict__ diag,
                                          const int* __restrict__ rows, const T* __restrict__ in,
                                          T* x, int K, int lane) {
  const int i = rows[t];
  const bool c0 = lane < K, c1 = lane + 32 < K;
  T s0 = c0 ? in[(size_t)i * K + lane] : T(0);
  T s1 = c1 ? in[(size_t)i * K + lane + 32] : T(0);
  warp_row_sum<T, true>(ia[t], ia[t + 1], ja, val, x, K, lane, c0, c1, -1, s0, s1, nullptr);
  const T d = diag[t];
  if (c0) x[(size_t)i * K + lane] = s0 / d;
  if (c1) x[(size_t)i * K + lane + 32] = s1 / d;
}

template <class T>
__global__ void __launch_bounds__(32 * kBlkWarps)
k_tri_wide_m(const int* __restrict__ ia, const int* __restrict__ ja, const T* __restrict__ val,
             const T* __restrict__ diag, const int* __restrict__ rows, int t0, int t1,
             const T* __restrict__ in, T* x, int K) {
  const int lane = threadIdx.x & 31;
  const int nw = (gridDim.x * blockDim.x) >> 5;
  for (int t = t0 + ((blockIdx.x * blockDim.x + threadIdx.x) >> 5); t < t1; t += nw)
    tri_row_m<T>(t, ia, ja, val, diag, rows, in, x, K, lane);
}

// a run of narrow levels in one block (a barrier between levels)
template <class T>
__global__ void __launch_bounds__(1024)
k_tri_batch_m(const int* __restrict__ ia, const int* __restrict__ ja, const T* __restrict__ val,
              const T* __restrict__ diag, const int* __restrict__ rows,
              const int* __restrict__ lptr, int l0, int l1, const T* __restrict__ in, T* x,
              int K) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int l = l0; l < l1; l++) {
    for (int t = lptr[l] + w; t < lptr[l + 1]; t += nw)
      tri_row_m<T>(t, ia, ja, val, diag, rows, in, x, K, lane);
    __syncthreads();
  }
}

// Tiled form of a many-column sweep: the single-vector tile schedule
// (IChol::Tiles), a warp per row, lane c (and c + 32) holding column c of
// the row; every value of the output block doubles as its ready flag (all
// ones = pending), so each lane polls its own column of a dependency in
// another tile, time-bounded like the single-vector sweep.  Dependencies in
// the block's own tile were published before a block barrier.
template <class T>
__global__ void __launch_bounds__(512, 2)
k_tri_tiles_m(const int* __restrict__ ia, const int* __restrict__ ja, const T* __restrict__ val,
              const T* __restrict__ diag, const int* __restrict__ rows,
              const unsigned* __restrict__ imask, const int2* __restrict__ tile_steps,
              const int2* __restrict__ steps, int ntiles, const T* __restrict__ in, T* out,
              int K, WaitCtl wc) {
  using W = WordOf<T>;
  using U = typename W::U;
  U* o = reinterpret_cast<U*>(out);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const bool c0 = lane < K, c1 = lane + 32 < K;
  for (int q = blockIdx.x; q < ntiles; q += gridDim.x) {
    const int2 ts = tile_steps[q];
    for (int st = ts.x; st < ts.y; st++) {
      const int2 sp = steps[st];
      for (int t = sp.x + w; t < sp.y; t += nw) {
        const int i = rows[t];
        const int k0 = ia[t], k1 = ia[t + 1];
        const unsigned im = imask[t];
        T s0 = c0 ? in[(size_t)i * K + lane] : T(0);
        T s1 = c1 ? in[(size_t)i * K + lane + 32] : T(0);
        for (int k = k0; k < k1; k++) {
          const int j = ja[k];
          const T v = val[k];
          const int bit = k - k0;
          const bool own = bit < 32 && ((im >> bit) & 1u);
          if (c0) {
            const U* p = o + (size_t)j * K + lane;
            U u = own ? __ldca(p) : ld_relaxed(p);
            u = wait_word(o, (int)((size_t)j * K + lane), u, W::kPending, W::kNaN, wc, i);
            if constexpr (sizeof(T) == 8) s0 = xsub(s0, xmul(v, word_value(u)));
            else s0 = xsubf(s0, xmulf(v, word_value(u)));
          }
          if (c1) {
            const U* p = o + (size_t)j * K + lane + 32;
            U u = own ? __ldca(p) : ld_relaxed(p);
            u = wait_word(o, (int)((size_t)j * K + lane + 32), u, W::kPending, W::kNaN, wc, i);
            if constexpr (sizeof(T) == 8) s1 = xsub(s1, xmul(v, word_value(u)));
            else s1 = xsubf(s1, xmulf(v, word_value(u)));
          }
        }
        const T d = diag[t];
        if (c0) {
          U r = value_word(s0 / d);
          if (r == W::kPending) r = W::kNaN;
          st_relaxed(o + (size_t)i * K + lane, r);
        }
        if (c1) {
          U r = value_word(s1 / d);
          if (r == W::kPending) r = W::kNaN;
          st_relaxed(o + (size_t)i * K + lane + 32, r);
        }
      }
      __syncthreads();
    }
  }
}

// Sync-free form of a many-column sweep: the rows in level order, a warp
// per row taken round-robin by the warps of a co-resident grid, lane c (and
// c + 32) holding column c.  Every value of the output block doubles as its
// ready flag; a lane polls its own column of up to four dependencies at a
// time and publishes its column as soon as those are in (the columns are
// independent, so a lane never waits for the others).  A warp only waits on
// rows of lower levels (earlier positions), and the earliest unfinished row
// has all its dependencies published, so the sweep always advances; every
// wait is bounded (flags.cuh).
template <class T>
__global__ void __launch_bounds__(256)
k_tri_flags_m(const int* __restrict__ ia, const int* __restrict__ ja, const T* __restrict__ val,
              const T* __restrict__ diag, const int* __restrict__ rows, int n,
              const T* __restrict__ in, T* out, int K, WaitCtl wc) {
  using W = WordOf<T>;
  using U = typename W::U;
  U* o = reinterpret_cast<U*>(out);
  const int lane = threadIdx.x & 31;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nw = (gridDim.x * blockDim.x) >> 5;
  for (int t = warp; t < n; t += nw) {
    const int i = rows[t];
    const int k0 = ia[t], k1 = ia[t + 1];
    const T d = diag[t];
#pragma unroll
    for (int h = 0; h < 2; h++) {
      const int c = lane + 32 * h;
      if (c >= K) continue;
      T sum = in[(size_t)i * K + c];
      for (int k = k0; k < k1; k += 4) {
        const int m = k1 - k < 4 ? k1 - k : 4;
        int jj[4];
        T v[4];
        U u[4];
#pragma unroll
        for (int q = 0; q < 4; q++) {
          jj[q] = q < m ? ja[k + q] * K + c : 0;
          v[q] = q < m ? val[k + q] : T(0);
        }
#pragma unroll
        for (int q = 0; q < 4; q++) u[q] = q < m ? ld_relaxed(o + jj[q]) : U(0);
        wait_group(o, jj, u, m, W::kPending, W::kNaN, wc, i);
#pragma unroll
        for (int q = 0; q < 4; q++) {
          if (q < m) {
            if constexpr (sizeof(T) == 8) sum = xsub(sum, xmul(v[q], word_value(u[q])));
            else sum = xsubf(sum, xmulf(v[q], word_value(u[q])));
          }
        }
      }
      U r = value_word(sum / d);
      if (r == W::kPending) r = W::kNaN;
      st_relaxed(o + (size_t)i * K + c, r);
    }
  }
}

template <class T>
static void sweep_flags_m(const IChol& ic, bool fwd, const T* in, T* x, int K, cudaStream_t s) {
  const int* ia = fwd ? ic.fia.p : ic.bia.p;
  const int* ja = fwd ? ic.vfja.p : ic.vbja.p;
  const int* rows = fwd ? ic.vorder.p : ic.vborder.p;
  const T* val;
  const T* diag;
  if constexpr (sizeof(T) == 8) {
    val = fwd ? ic.fval.p : ic.bval.p;
    diag = fwd ? ic.fdiag.p : ic.bdiag.p;
  } else {
    val = fwd ? ic.fval32.p : ic.bval32.p;
    diag = fwd ? ic.fdiag32.p : ic.bdiag32.p;
  }
  BN_CUDA(cudaMemsetAsync(x, 0xFF, sizeof(T) * (size_t)ic.n * K, s));
  int dev = 0, per_sm = 0, sms = 0;
  BN_CUDA(cudaGetDevice(&dev));
  BN_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_tri_flags_m<T>, 256, 0));
  BN_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  if (per_sm > 4) per_sm = 4;
  const int grid = sms * per_sm;
  BN_REQUIRE(grid > 0, BN_ERR_CUDA, "block IC(0): sweep grid does not fit");
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(256);
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;  // co-residency: waits always end
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  g_launch_count++;
  BN_CUDA(cudaLaunchKernelEx(&cfg, k_tri_flags_m<T>, ia, ja, val, diag, rows, ic.n, in, x, K,
                             ic.wait.ctl(fwd ? WT_IC_FWD : WT_IC_BWD)));
}

template <class T>
static void sweep_tiles_m(const IChol& ic, bool fwd, const T* in, T* x, int K, cudaStream_t s) {
  const IChol::Tiles& tl = fwd ? ic.tf : ic.tb;
  const int* ia = fwd ? ic.fia.p : ic.bia.p;
  const int* ja = fwd ? ic.vfja.p : ic.vbja.p;
  const int* rows = fwd ? ic.vorder.p : ic.vborder.p;
  const T* val;
  const T* diag;
  if constexpr (sizeof(T) == 8) {
    val = fwd ? ic.fval.p : ic.bval.p;
    diag = fwd ? ic.fdiag.p : ic.bdiag.p;
  } else {
    val = fwd ? ic.fval32.p : ic.bval32.p;
    diag = fwd ? ic.fdiag32.p : ic.bdiag32.p;
  }
  BN_CUDA(cudaMemsetAsync(x, 0xFF, sizeof(T) * (size_t)ic.n * K, s));
  int dev = 0, per_sm = 0, sms = 0;
  BN_CUDA(cudaGetDevice(&dev));
  BN_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_tri_tiles_m<T>, 512, 0));
  BN_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  const int cap = sms * per_sm;
  const int grid = tl.ntiles < cap ? tl.ntiles : cap;
  BN_REQUIRE(grid > 0, BN_ERR_CUDA, "IC(0): tiled block sweep grid does not fit");
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(512);
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;  // co-residency: waits always end
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  g_launch_count++;
  BN_CUDA(cudaLaunchKernelEx(&cfg, k_tri_tiles_m<T>, ia, ja, val, diag, rows,
                             (const unsigned*)tl.imask.p, (const int2*)tl.tile_steps.p,
                             (const int2*)tl.steps.p, tl.ntiles, in, x, K,
                             ic.wait.ctl(fwd ? WT_IC_FWD : WT_IC_BWD)));
}

template <class T>
void sweep_m(const IChol& ic, bool fwd, const T* in, T* x, int K, cudaStream_t s) {
  // the sync-free form by default (64 columns on the 5M network, mixed, true
  // residual 1e-8, same run: 23.5 ms per right-hand side for the whole block
  // solve, 24.7 ms with level launches, bit-identical); BN_BLOCK_IC_TILES=1
  // selects the tiled form (13.4 against 11.2 ms for level launches in an
  // earlier run), BN_BLOCK_IC_LEVELS=1 the level launches
  static const bool tiles = getenv("BN_BLOCK_IC_TILES") && atoi(getenv("BN_BLOCK_IC_TILES"));
  if (tiles && ic.tf.ntiles > 0 && (size_t)ic.n * K < (1ull << 31)) {
    sweep_tiles_m<T>(ic, fwd, in, x, K, s);
    return;
  }
  static const bool levels = getenv("BN_BLOCK_IC_LEVELS") && atoi(getenv("BN_BLOCK_IC_LEVELS"));
  if (!levels && (size_t)ic.n * K < (1ull << 31)) {
    sweep_flags_m<T>(ic, fwd, in, x, K, s);
    return;
  }
  const int* ia = fwd ? ic.fia.p : ic.bia.p;
  const int* ja = fwd ? ic.vfja.p : ic.vbja.p;
  const int* rows = fwd ? ic.vorder.p : ic.vborder.p;
  const int* lp = fwd ? ic.d_lptr.p : ic.d_bptr.p;
  const T* val;
  const T* diag;
  if constexpr (sizeof(T) == 8) {
    val = fwd ? ic.fval.p : ic.bval.p;
    diag = fwd ? ic.fdiag.p : ic.bdiag.p;
  } else {
    val = fwd ? ic.fval32.p : ic.bval32.p;
    diag = fwd ? ic.fdiag32.p : ic.bdiag32.p;
  }
  const std::vector<IChol::Seg>& segs = fwd ? ic.fseg : ic.bseg;
  for (const IChol::Seg& g : segs) {
    if (g.kind == 0) {
      BN_LAUNCH(k_tri_wide_m<T>, grid_for((long long)(g.t1 - g.t0) * 32, 32 * kBlkWarps, 8),
                32 * kBlkWarps, 0, s, ia, ja, val, diag, rows, g.t0, g.t1, in, x, K);
    } else {
      BN_LAUNCH(k_tri_batch_m<T>, 1, 1024, 0, s, ia, ja, val, diag, rows, lp, g.l0, g.l1, in, x,
                K);
    }
  }
}

// ---------------------------------------------------------------- PCG pieces
// per-column dot products: partial[b][c] over a block's rows, then a fixed-
// order sum over the blocks
constexpr int kDotBlocks = 592;
template <class T>
__global__ void __launch_bounds__(256)
k_dot_cols(const T* __restrict__ u, const T* __restrict__ v, int n, int K,
           double* __restrict__ partial) {
  __shared__ double red[256];
  const int per = 256 / K;  // rows handled at once (K divides 256: K in {1,2,4,...,64})
  const int c = threadIdx.x % K, r = threadIdx.x / K;
  double acc = 0.0;
  if (r < per)
    for (int i = blockIdx.x * per + r; i < n; i += gridDim.x * per)
      acc += (double)u[(size_t)i * K + c] * (double)v[(size_t)i * K + c];
  red[threadIdx.x] = acc;
  __syncthreads();
  if (threadIdx.x < K) {
    double t = 0.0;
    for (int q = 0; q < per; q++) t += red[q * K + threadIdx.x];
    partial[(size_t)blockIdx.x * K + threadIdx.x] = t;
  }
}
__global__ void k_dot_finish(const double* __restrict__ partial, int nb, int K,
                             double* __restrict__ out) {
  const int c = threadIdx.x;
  if (c >= K) return;
  double t = 0.0;
  for (int b = 0; b < nb; b++) t += partial[(size_t)b * K + c];
  out[c] = t;
}

__global__ void k_blk_update_xr(double* __restrict__ x, double* __restrict__ r,
                                const double* __restrict__ p, const double* __restrict__ ap,
                                const double* __restrict__ alpha, int n, int K) {
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < (size_t)n * K;
       e += (size_t)gridDim.x * blockDim.x) {
    const double a = alpha[e % K];
    x[e] = x[e] + p[e] * a;
    r[e] = r[e] + ap[e] * (-a);
  }
}
__global__ void k_blk_update_p(double* __restrict__ p, const double* __restrict__ z,
                               const double* __restrict__ beta, int n, int K) {
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < (size_t)n * K;
       e += (size_t)gridDim.x * blockDim.x)
    p[e] = z[e] + p[e] * beta[e % K];
}
// column-major n x K caller layout <-> row-major n x Kp block in the solve
// numbering: blk[t*Kp + c] = cm[c*n + perm[t]]; the Kp - K padding columns
// are zero (their PCG never starts)
__global__ void k_to_block(const double* __restrict__ cm, const int* __restrict__ perm, int n,
                           int K, int Kp, double* __restrict__ blk) {
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < (size_t)n * Kp;
       e += (size_t)gridDim.x * blockDim.x) {
    const int t = (int)(e / Kp), c = (int)(e % Kp);
    blk[e] = c < K ? cm[(size_t)c * n + perm[t]] : 0.0;
  }
}
__global__ void k_from_block(const double* __restrict__ blk, const int* __restrict__ perm, int n,
                             int K, int Kp, double* __restrict__ cm) {
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < (size_t)n * Kp;
       e += (size_t)gridDim.x * blockDim.x) {
    const int t = (int)(e / Kp), c = (int)(e % Kp);
    if (c < K) cm[(size_t)c * n + perm[t]] = blk[e];
  }
}
__global__ void k_blk_start(const double* __restrict__ rz, int K, int* __restrict__ active,
                            int* __restrict__ iters, int* nactive) {
  const int c = threadIdx.x;
  if (c >= K) return;
  const int a = rz[c] != 0.0;
  active[c] = a;
  iters[c] = 0;
  if (a) atomicAdd(nactive, 1);
}
__global__ void k_blk_relres(const double* __restrict__ rr, const double* __restrict__ bb, int K,
                             double* __restrict__ out) {
  const int c = threadIdx.x;
  if (c < K) out[c] = sqrt(rr[c]) / (bb[c] > 0.0 ? sqrt(bb[c]) : 1.0);
}

inline int eg(size_t m) { return grid_for((long long)m, 256, 16); }

}  // namespace

// ------------------------------------------------------------------ V-cycle
// Work vectors of one block solve (K columns), per level and for level 0.
struct BlockWork {
  int K = 0;
  std::vector<DBuf<double>> b, x, r;
  std::vector<DBuf<float>> b32, x32, r32;
  DBuf<double> u1, r1, icy, icx, xx, r2, corr;
  DBuf<float> g32, u1f, r1f, icyf, icxf, xxf, r2f, corrf;
};

template <class T>
static T* pick(std::vector<DBuf<double>>& d, std::vector<DBuf<float>>& f, int l) {
  if constexpr (sizeof(T) == 8) return d[l].p;
  else return f[l].p;
}

template <class T>
void Solver::smooth_block(BlockWork& W, int l, const T* bb, T* xl, bool forward) {
  Level& L = *lv[l];
  const int K = W.K;
  DevMat<T> A = mat<T>(L.Ap, &L.A32, &L.layA);
  const int n = L.A.n;
  T* tmp = pick<T>(W.r, W.r32, l);
  for (int sweep = 0; sweep < opt.nu; sweep++) {
    if (opt.smoother == SMOOTHER_CF_GS || opt.smoother == SMOOTHER_GS) {
      const int nseg = (int)L.cptr.size() - 1;
      for (int q = 0; q < nseg; q++) {
        const int c = forward ? q : nseg - 1 - q;
        const int r0 = L.cptr[c], nr = L.cptr[c + 1] - r0;
        if (L.cjac[c]) {
          gs_class_block<T>(A, r0, nr, L.clong[c], bb, xl, tmp, K, s);
          BN_CUDA(cudaMemcpyAsync(xl + (size_t)r0 * K, tmp, sizeof(T) * (size_t)nr * K,
                                  cudaMemcpyDeviceToDevice, s));
        } else {
          gs_class_block<T>(A, r0, nr, L.clong[c], bb, xl, nullptr, K, s);
        }
      }
    } else {
      spmm<T>(BM_RES, A, xl, bb, tmp, K, s);
      const double* d = opt.smoother == SMOOTHER_JACOBI ? L.dg.p : L.l1.p;
      const T om = opt.smoother == SMOOTHER_JACOBI ? (T)opt.omega : T(1);
      BN_LAUNCH(k_bscaled<T>, eg((size_t)n * K), 256, 0, s, xl, tmp, d, om, n, K);
    }
  }
}

template <class T>
void Solver::backslash_block(BlockWork& W, int l, const T* bb, T* xl) {
  const int nl = (int)lv.size();
  const int K = W.K;
  if (l == nl - 1) {
    BN_LAUNCH(k_dense_apply_m<T>, eg((size_t)coarse.n * K), 256, 0, s, coarse.inv.p, coarse.n, bb,
              xl, K);
    return;
  }
  Level& L = *lv[l];
  Level& C = *lv[l + 1];
  T* rr = pick<T>(W.r, W.r32, l);
  T* cb = pick<T>(W.b, W.b32, l + 1);
  T* cx = pick<T>(W.x, W.x32, l + 1);
  smooth_block<T>(W, l, bb, xl, true);
  spmm<T>(BM_RES, mat<T>(L.Ap, &L.A32, &L.layA), xl, bb, rr, K, s);
  spmm<T>(BM_Y, mat<T>(L.Rp, &L.R32, &L.layR), rr, nullptr, cb, K, s);
  if (l + 1 < nl - 1)
    BN_CUDA(cudaMemsetAsync(cx, 0, sizeof(T) * (size_t)C.A.n * K, s));
  backslash_block<T>(W, l + 1, cb, cx);
  spmm<T>(BM_ADD, mat<T>(L.Pp, &L.P32, &L.layP), cx, nullptr, xl, K, s);
}

template <class T>
void Solver::fwdslash_block(BlockWork& W, int l, const T* bb, T* xl) {
  const int nl = (int)lv.size();
  const int K = W.K;
  if (l == nl - 1) {
    BN_LAUNCH(k_dense_apply_m<T>, eg((size_t)coarse.n * K), 256, 0, s, coarse.inv.p, coarse.n, bb,
              xl, K);
    return;
  }
  Level& L = *lv[l];
  T* cb = pick<T>(W.b, W.b32, l + 1);
  T* cx = pick<T>(W.x, W.x32, l + 1);
  spmm<T>(BM_Y, mat<T>(L.Rp, &L.R32, &L.layR), bb, nullptr, cb, K, s);
  fwdslash_block<T>(W, l + 1, cb, cx);
  spmm<T>(BM_Y, mat<T>(L.Pp, &L.P32, &L.layP), cx, nullptr, xl, K, s);
  smooth_block<T>(W, l, bb, xl, false);
}

// the three-stage preconditioner (as precond_t) on K columns
template <class T>
void Solver::precond_block_t(BlockWork& W, const T* g, T* out) {
  const bool f64 = sizeof(T) == 8;
  const int n0 = n(), K = W.K;
  const size_t m = (size_t)n0 * K;
  T* U1 = f64 ? (T*)W.u1.p : (T*)W.u1f.p;
  T* R1 = f64 ? (T*)W.r1.p : (T*)W.r1f.p;
  T* IY = f64 ? (T*)W.icy.p : (T*)W.icyf.p;
  T* IX = f64 ? (T*)W.icx.p : (T*)W.icxf.p;
  T* XX = f64 ? (T*)W.xx.p : (T*)W.xxf.p;
  T* R2 = f64 ? (T*)W.r2.p : (T*)W.r2f.p;
  T* CO = f64 ? (T*)W.corr.p : (T*)W.corrf.p;
  DevMat<T> As = own_solve ? mat<T>(Aownp, &Aown32, &layOwn)
                           : mat<T>(lv[0]->Ap, &lv[0]->A32, &lv[0]->layA);
  BN_CUDA(cudaMemsetAsync(U1, 0, sizeof(T) * m, s));
  backslash_block<T>(W, 0, g, U1);
  spmm<T>(BM_RES, As, U1, g, R1, K, s);
  sweep_m<T>(ic, true, R1, IY, K, s);
  sweep_m<T>(ic, false, IY, IX, K, s);
  BN_LAUNCH(k_badd<T>, eg(m), 256, 0, s, U1, IX, m, XX);
  spmm<T>(BM_RES, As, XX, g, R2, K, s);
  BN_CUDA(cudaMemsetAsync(CO, 0, sizeof(T) * m, s));
  fwdslash_block<T>(W, 0, R2, CO);
  BN_LAUNCH(k_badd<T>, eg(m), 256, 0, s, XX, CO, m, out);
}

void Solver::precond_block(BlockWork& W, const double* g, double* out) {
  const size_t m = (size_t)n() * W.K;
  if (opt.precision == AMG_PREC_MIXED) {
    BN_LAUNCH((k_bconv<float, double>), eg(m), 256, 0, s, g, m, W.g32.p);
    precond_block_t<float>(W, W.g32.p, W.corrf.p);  // corrf is free after the last add
    BN_LAUNCH((k_bconv<double, float>), eg(m), 256, 0, s, W.corrf.p, m, out);
  } else {
    precond_block_t<double>(W, g, out);
  }
}

// ------------------------------------------------------------------ PCG
int Solver::pcg_block(int Kin, const double* d_Bcm, double* d_Xcm, double tol, int maxiter,
                      int* h_iters, double* h_relres) {
  BN_REQUIRE(Kin >= 1 && Kin <= kMaxK, BN_ERR_ARG, "block solve: 1 to 64 right-hand sides");
  BN_REQUIRE(opt.smoother == SMOOTHER_CF_GS || opt.smoother == SMOOTHER_GS ||
                 opt.smoother == SMOOTHER_JACOBI || opt.smoother == SMOOTHER_L1,
             BN_ERR_ARG, "block solve: unknown smoother");
  int K = 1;  // columns padded to a power of two (the dot kernels divide 256 rows)
  while (K < Kin) K <<= 1;
  const int n0 = n();
  const bool flexible = (opt.precision == AMG_PREC_MIXED);
  if (flexible && !f32_ready) prepare_f32();
  if (flexible && !ic.fval32.n) {
    ic.want_f32 = true;
    ic.refresh_values();
  }
  const size_t m = (size_t)n0 * K;
  // work vectors
  BlockWork W;
  W.K = K;
  const int nl = (int)lv.size();
  W.b.resize(nl); W.x.resize(nl); W.r.resize(nl);
  W.b32.resize(nl); W.x32.resize(nl); W.r32.resize(nl);
  for (int l = 0; l < nl; l++) {
    const size_t ml = (size_t)lv[l]->A.n * K;
    if (flexible) {
      if (l > 0) { W.b32[l].alloc(ml, s); W.x32[l].alloc(ml, s); }
      W.r32[l].alloc(ml, s);
    } else {
      if (l > 0) { W.b[l].alloc(ml, s); W.x[l].alloc(ml, s); }
      W.r[l].alloc(ml, s);
    }
  }
  if (flexible) {
    for (auto* v : {&W.g32, &W.u1f, &W.r1f, &W.icyf, &W.icxf, &W.xxf, &W.r2f, &W.corrf})
      v->alloc(m, s);
  } else {
    for (auto* v : {&W.u1, &W.r1, &W.icy, &W.icx, &W.xx, &W.r2, &W.corr}) v->alloc(m, s);
  }
  DBuf<double> B(m, s), X(m, s), R(m, s), Z(m, s), P(m, s), AP(m, s);
  enum { BB, RR, RZ, RZ0, PAP, RZNEW, RZON, ALPHA, BETA, NSC };
  DBuf<double> scal((size_t)NSC * K, s), part((size_t)kDotBlocks * K, s);
  auto S_ = [&](int w) { return scal.p + (size_t)w * K; };
  DBuf<int> ints((size_t)2 * K + 1, s);
  int* active = ints.p;
  int* iters = ints.p + K;
  int* nact_d = ints.p + 2 * K;
  ints.zero();
  auto dot = [&](const double* u, const double* v, double* out) {
    BN_LAUNCH(k_dot_cols<double>, kDotBlocks, 256, 0, s, u, v, n0, K, part.p);
    BN_LAUNCH(k_dot_finish, 1, 64, 0, s, part.p, kDotBlocks, K, out);
  };
  DevMat<double> A = mat<double>(Asolve_p(), nullptr, &lay_solve());
  const int* perm0 = lv[0]->perm.p;
  const int ge = eg(m);
  cudaEventRecord(ev0, s);
  BN_LAUNCH(k_to_block, ge, 256, 0, s, d_Bcm, perm0, n0, Kin, K, B.p);
  BN_LAUNCH(k_to_block, ge, 256, 0, s, d_Xcm, perm0, n0, Kin, K, X.p);
  spmm<double>(BM_RES, A, X.p, B.p, R.p, K, s);
  dot(B.p, B.p, S_(BB));
  precond_block(W, R.p, Z.p);
  BN_CUDA(cudaMemcpyAsync(P.p, Z.p, sizeof(double) * m, cudaMemcpyDeviceToDevice, s));
  dot(R.p, Z.p, S_(RZ));
  BN_CUDA(cudaMemcpyAsync(S_(RZ0), S_(RZ), sizeof(double) * K, cudaMemcpyDeviceToDevice, s));
  BN_LAUNCH(k_blk_start, 1, 64, 0, s, S_(RZ), K, active, iters, nact_d);
  int nact = read_scalar(nact_d, s);
  const int relres = (opt.stop == AMG_STOP_RELRES) ? 1 : 0;
  for (int iter = 1; iter <= maxiter && nact > 0; iter++) {
    spmm<double>(BM_Y, A, P.p, nullptr, AP.p, K, s);
    dot(P.p, AP.p, S_(PAP));
    seg_alpha(S_(RZ), S_(PAP), active, K, S_(ALPHA), s);
    BN_LAUNCH(k_blk_update_xr, ge, 256, 0, s, X.p, R.p, P.p, AP.p, S_(ALPHA), n0, K);
    if (relres) dot(R.p, R.p, S_(RR));
    if (flexible) dot(R.p, Z.p, S_(RZON));
    precond_block(W, R.p, Z.p);
    dot(R.p, Z.p, S_(RZNEW));
    BN_CUDA(cudaMemsetAsync(nact_d, 0, sizeof(int), s));
    seg_next(S_(RZ), S_(RZNEW), S_(RZON), S_(RR), S_(BB), S_(RZ0), active, iters, S_(BETA), K,
             flexible ? 1 : 0, relres, tol, iter, nact_d, s);
    BN_LAUNCH(k_blk_update_p, ge, 256, 0, s, P.p, Z.p, S_(BETA), n0, K);
    nact = read_scalar(nact_d, s);
    ic.check_waits(s);
  }
  spmm<double>(BM_RES, A, X.p, B.p, AP.p, K, s);
  dot(AP.p, AP.p, S_(RR));
  BN_LAUNCH(k_blk_relres, 1, 64, 0, s, S_(RR), S_(BB), K, S_(ALPHA));
  BN_LAUNCH(k_from_block, ge, 256, 0, s, X.p, perm0, n0, Kin, K, d_Xcm);
  cudaEventRecord(ev1, s);
  std::vector<int> hi(2 * (size_t)K);
  std::vector<double> hr(K);
  BN_CUDA(cudaMemcpyAsync(hi.data(), ints.p, sizeof(int) * 2 * K, cudaMemcpyDeviceToHost, s));
  BN_CUDA(cudaMemcpyAsync(hr.data(), S_(ALPHA), sizeof(double) * K, cudaMemcpyDeviceToHost, s));
  BN_CUDA(cudaStreamSynchronize(s));
  float ms = 0;
  cudaEventElapsedTime(&ms, ev0, ev1);
  stats.solve_seconds = ms * 1e-3;
  int worst = 0, failed = 0, nan = 0;
  for (int c = 0; c < Kin; c++) {
    int it = hi[K + c];
    if (hi[c]) { it = -maxiter; failed = 1; }
    else if (it < 0) nan = 1;
    if (h_iters) h_iters[c] = it;
    if (h_relres) h_relres[c] = hr[c];
    const int a = it < 0 ? -it : it;
    if (a > worst) worst = a;
  }
  stats.iterations = worst;
  stats.converged = !(failed || nan);
  if (nan) {
    set_last_error(BN_ERR_NAN, "block PCG: non-finite value in a column");
    return BN_ERR_NAN;
  }
  if (failed) {
    set_last_error(BN_ERR_NOT_CONVERGED, "block PCG: a column did not converge");
    return BN_ERR_NOT_CONVERGED;
  }
  set_last_error(BN_OK, "");
  return BN_OK;
}

}  // namespace bn

using bn::Solver;

// See include/amg_b200.h for the contract.
BN_API int amg_solver_solve_block(void* h, int k, const double* B, double* X, double tol,
                                  int maxiter, int* iterations, double* relres) {
  if (!h) { bn::set_last_error(bn::BN_ERR_ARG, "NULL handle"); return bn::BN_ERR_ARG; }
  Solver* S = (Solver*)h;
  return bn::guarded([&]() {
    BN_REQUIRE(k >= 1 && B && X, bn::BN_ERR_ARG, "amg_solver_solve_block: invalid arguments");
    BN_CUDA(cudaSetDevice(S->device));
    const size_t n = (size_t)S->n();
    bn::DBuf<double> db(n * k, S->s), dx(n * k, S->s);
    db.upload(B, n * k);
    dx.upload(X, n * k);
    const int rc = S->pcg_block(k, db.p, dx.p, tol, maxiter, iterations, relres);
    dx.download(X, n * k);
    BN_CUDA(cudaStreamSynchronize(S->s));
    return rc;
  }, bn::BN_ERR_CUDA);
}

BN_API int amg_solver_solve_block_device(void* h, int k, const double* d_B, double* d_X,
                                         double tol, int maxiter, int* iterations,
                                         double* relres) {
  if (!h) { bn::set_last_error(bn::BN_ERR_ARG, "NULL handle"); return bn::BN_ERR_ARG; }
  Solver* S = (Solver*)h;
  return bn::guarded([&]() {
    BN_REQUIRE(k >= 1 && d_B && d_X, bn::BN_ERR_ARG, "amg_solver_solve_block: invalid arguments");
    BN_CUDA(cudaSetDevice(S->device));
    return S->pcg_block(k, d_B, d_X, tol, maxiter, iterations, relres);
  }, bn::BN_ERR_CUDA);
}
