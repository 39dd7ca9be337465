// Solve-phase kernels: CSR SpMV family, coloured Gauss-Seidel, PCG vector
// updates with fused reductions.  Templated on the value type: float64 for
// the plain solver and the outer PCG, float32 (with float32 accumulation)
// for the mixed-precision V-cycle.
//
// SpMV layout ("CSR-stream"): a block of kRows rows loads the contiguous
// nonzero range of its rows with coalesced loads, forms the products
// a_ij * x_j into shared memory, then each thread sums its own row in
// storage order -- the reference's summation order for abyvg/abyvam/abyvcs
// (C_amg1/src/sparse_ops.c:19-56), with separate multiply and add.  Tiles
// whose nonzeros exceed the shared buffer fall back to a per-thread walk.
#include "solve_kernels.cuh"

#include <cub/cub.cuh>

namespace bn {

template <class T> __device__ __forceinline__ T dmul(T a, T b);
template <> __device__ __forceinline__ double dmul(double a, double b) { return __dmul_rn(a, b); }
template <> __device__ __forceinline__ float dmul(float a, float b) { return __fmul_rn(a, b); }
template <class T> __device__ __forceinline__ T dadd(T a, T b);
template <> __device__ __forceinline__ double dadd(double a, double b) { return __dadd_rn(a, b); }
template <> __device__ __forceinline__ float dadd(float a, float b) { return __fadd_rn(a, b); }
template <class T> __device__ __forceinline__ T dsub(T a, T b);
template <> __device__ __forceinline__ double dsub(double a, double b) { return __dsub_rn(a, b); }
template <> __device__ __forceinline__ float dsub(float a, float b) { return __fsub_rn(a, b); }

// -------------------------------------------------------------------- SpMV
// Each thread's tile header (the tile's nonzero range, its own row range,
// its b_i / y_i and dot weight) is loaded one tile ahead, so those loads are
// in flight while the current tile computes.
// ROWS < kRows: tiles of ROWS rows (denser operators, whose kRows-row
// tiles would overflow the product buffer); a kRows-row tile of the visiting
// order is taken as kRows/ROWS consecutive smaller tiles, the ones past the
// last row being empty.
template <class T, int MODE, bool DOT, int ROWS = kRows>
__global__ void __launch_bounds__(kRows, 8)
k_spmv(const int* __restrict__ ia, const int* __restrict__ ja, const T* __restrict__ a,
       const T* __restrict__ x, int n, const T* __restrict__ b, T* __restrict__ y,
       const T* __restrict__ dw, double* __restrict__ partial, int skip_long,
       const int* __restrict__ tiles) {
  BN_PDL_ENTRY();
  static_assert(ROWS <= kRows && kRows % ROWS == 0, "tile rows must divide kRows");
  constexpr int SUB = kRows / ROWS;
  __shared__ T prod[kTileNnz];
  __shared__ double red[kRows / 32];
  double dot = 0.0;
  const int ntiles = ((n + kRows - 1) / kRows) * SUB;
  int e0 = 0, e1 = 0, k0 = 0, k1 = 0;
  T hb = T(0), hw = T(0);
  auto head = [&](int t0) {  // t0 may lie past the last row (an empty tile)
    const int t1 = min(t0 + ROWS, n);
    e0 = ia[min(t0, n)];
    e1 = ia[t1];
    const int i = t0 + threadIdx.x;
    if (i < t1) {
      k0 = ia[i];
      k1 = ia[i + 1];
      if (MODE == SPMV_RES) hb = b[i];
      if (MODE == SPMV_ADD) hb = y[i];
      if (DOT) hw = dw[i];
    }
  };
  auto tile_row = [&](int slot) {
    return (tiles ? tiles[slot / SUB] : slot / SUB) * kRows + (slot % SUB) * ROWS;
  };
  int nxt = (int)blockIdx.x < ntiles ? tile_row(blockIdx.x) : 0;
  if ((int)blockIdx.x < ntiles) head(nxt);
  for (int slot = blockIdx.x; slot < ntiles; slot += gridDim.x) {
    const int r0 = nxt;
    const int r1 = min(r0 + ROWS, n);
    const int i = r0 + threadIdx.x;
    const int ce0 = e0, ce1 = e1, ck0 = k0, ck1 = k1;
    const T cb = hb, cw = hw;
    if (slot + (int)gridDim.x < ntiles) {
      nxt = tile_row(slot + gridDim.x);
      head(nxt);
    }
    T hold = (MODE == SPMV_Y) ? T(0) : cb;
    // this thread's row, unless the long-row kernel owns it
    const bool mine = i < r1 && !(skip_long && ck1 - ck0 > kLongRow);
    if (ce1 - ce0 <= kTileNnz) {
      // matrix entries are read once: evict-first, so that L2 keeps x
#pragma unroll 4
      for (int k = ce0 + threadIdx.x; k < ce1; k += kRows)
        prod[k - ce0] = dmul(__ldcs(a + k), x[__ldcs(ja + k)]);
      __syncthreads();
      if (mine) {
        for (int k = ck0 - ce0; k < ck1 - ce0; k++)
          hold = (MODE == SPMV_RES) ? dsub(hold, prod[k]) : dadd(hold, prod[k]);
      }
      __syncthreads();
    } else if (mine) {
      for (int k = ck0; k < ck1; k++) {
        T p = dmul(a[k], x[ja[k]]);
        hold = (MODE == SPMV_RES) ? dsub(hold, p) : dadd(hold, p);
      }
    }
    if (mine) {
      y[i] = hold;
      if (DOT) dot += (double)cw * (double)hold;
    }
  }
  if (DOT) {
    for (int off = 16; off > 0; off >>= 1) dot += __shfl_xor_sync(0xffffffffu, dot, off);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = dot;
    __syncthreads();
    if (threadIdx.x == 0) {
      double t = 0.0;
      for (int w = 0; w < kRows / 32; w++) t += red[w];
      partial[blockIdx.x] = t;
    }
  }
}

// ---- row tiles staged by the bulk-copy engine
// The same tiles and summation order as k_spmv (ROWS = kRows), but each
// tile's column indices and values reach shared memory by two 1D bulk
// copies (cp.async.bulk, completion on an mbarrier) issued one tile ahead by
// one thread, so the stream of A runs ahead of the arithmetic without
// occupying the threads' load slots; the threads then gather x with
// independent loads (indices already on chip) and sum each row in storage
// order.  Blocks are persistent and double-buffer their tiles.  A bulk copy
// moves 16-byte aligned pieces: the tile's range is rounded down to a 16-byte
// boundary at its start, and the last 0-3 entries past the last boundary are
// loaded by the threads.  Every mbarrier wait is bounded; one that runs out
// records an error (g_stage_err) and the launch goes on.
__device__ int g_stage_err = 0;
constexpr int kStageCap = kTileNnz;  // entries staged per tile

__device__ __forceinline__ unsigned smem_u32(const void* p) {
  return (unsigned)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(unsigned long long* b, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(b)), "r"(count)
               : "memory");
}
__device__ __forceinline__ void mbar_arrive_tx(unsigned long long* b, unsigned bytes) {
  asm volatile(
      "{\n\t.reg .b64 st;\n\t"
      "mbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n\t}" ::"r"(smem_u32(b)),
      "r"(bytes)
      : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned long long* b, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(b)), "r"(parity)
      : "memory");
  return ok != 0;
}
// bounded: about a second at most (try_wait suspends the thread between polls)
__device__ __forceinline__ void mbar_wait(unsigned long long* b, unsigned parity) {
  for (int it = 0; it < (1 << 22); it++)
    if (mbar_try_wait(b, parity)) return;
  atomicExch(&g_stage_err, 1);
}
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, unsigned bytes,
                                         unsigned long long* b) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
      ::"r"(smem_u32(dst)), "l"(src), "r"(bytes), "r"(smem_u32(b))
      : "memory");
}

// MODE: SPMV_Y / SPMV_RES / SPMV_ADD over rows [0, n) (tiles in the
// visiting order `tiles`), or kStagedGS: one Gauss-Seidel colour class,
// rows [r0, r0 + n) with x_i = (b_i - sum_{j != i} a_ij x_j) / d_i in place
// (into out[t] when out is given), the sum formed as the thread-per-row
// class kernel forms it.
constexpr int kStagedGS = 3;
template <class T, int MODE, bool DOT>
__global__ void __launch_bounds__(kRows)
k_spmv_staged(const int* __restrict__ ia, const int* __restrict__ ja, const T* __restrict__ a,
              const T* x, int n, const T* __restrict__ b, T* y, const T* __restrict__ dw,
              double* __restrict__ partial, int skip_long, const int* __restrict__ tiles,
              int r0base, T* __restrict__ out) {
  BN_PDL_ENTRY();
  constexpr bool kGs = (MODE == kStagedGS);
  extern __shared__ __align__(16) unsigned char stage_mem[];
  __shared__ __align__(8) unsigned long long bar[2];
  __shared__ double red[kRows / 32];
  constexpr int JB = ((kStageCap + 8) * 4 + 15) / 16 * 16;
  constexpr int AB = ((kStageCap + 8) * (int)sizeof(T) + 15) / 16 * 16;
  auto s_ja = [&](int q) { return (int*)(stage_mem + q * JB); };
  auto s_a = [&](int q) { return (T*)(stage_mem + 2 * JB + q * AB); };
  const int ntiles = (n + kRows - 1) / kRows;
  auto tile_row = [&](int slot) { return r0base + (tiles ? tiles[slot] : slot) * kRows; };
  const int rend = r0base + n;
  // thread 0: stage the tile at `slot` into buffer q (or just arrive)
  auto issue = [&](int q, int slot) {
    const int t0 = tile_row(slot);
    const int t1 = min(t0 + kRows, rend);
    const int e0 = ia[t0], e1 = ia[t1];
    const int s0 = e0 & ~3, fl = e1 & ~3;
    if (e1 - e0 <= kStageCap && fl > s0) {
      const unsigned nb = (unsigned)(fl - s0);
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      mbar_arrive_tx(&bar[q], nb * 4u + nb * (unsigned)sizeof(T));
      bulk_g2s(s_ja(q), ja + s0, nb * 4u, &bar[q]);
      bulk_g2s(s_a(q), a + s0, nb * (unsigned)sizeof(T), &bar[q]);
    } else {
      mbar_arrive_tx(&bar[q], 0u);
    }
  };
  if (threadIdx.x == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  if (threadIdx.x == 0 && (int)blockIdx.x < ntiles) issue(0, blockIdx.x);
  double dot = 0.0;
  int q = 0;
  for (int slot = blockIdx.x; slot < ntiles; slot += gridDim.x, q++) {
    const int st = q & 1;
    if (threadIdx.x == 0 && slot + (int)gridDim.x < ntiles) issue(st ^ 1, slot + gridDim.x);
    const int t0 = tile_row(slot);
    const int t1 = min(t0 + kRows, rend);
    const int e0 = ia[t0], e1 = ia[t1];
    const int i = t0 + threadIdx.x;
    int k0 = 0, k1 = 0;
    T hold = T(0), hw = T(0), di = T(1);
    if (i < t1) {
      k0 = ia[i];
      k1 = ia[i + 1];
      if (MODE == SPMV_RES || kGs) hold = b[i];
      if (MODE == SPMV_ADD) hold = y[i];
      if (kGs) di = y[i];  // y: the diagonal (1 where a row has none)
      if (DOT) hw = dw[i];
    }
    const bool mine = i < t1 && (kGs || !(skip_long && k1 - k0 > kLongRow));
    T sum = T(0);  // Gauss-Seidel: sum over j != i
    mbar_wait(&bar[st], (unsigned)((q >> 1) & 1));
    const int m = e1 - e0;
    if (m <= kStageCap) {
      const int s0 = e0 & ~3;
      const int fl = max(e1 & ~3, s0);
      int* sj = s_ja(st);
      T* sa = s_a(st);
      for (int k = fl + threadIdx.x; k < e1; k += kRows) {  // the last 0-3 entries
        sj[k - s0] = ja[k];
        sa[k - s0] = a[k];
      }
      __syncthreads();
#pragma unroll 4
      for (int k = e0 - s0 + threadIdx.x; k < e1 - s0; k += kRows)
        sa[k] = dmul(sa[k], x[sj[k]]);
      __syncthreads();
      if (mine) {
        for (int k = k0 - s0; k < k1 - s0; k++) {
          if (kGs) {
            if (sj[k] != i) sum = dadd(sum, sa[k]);
          } else {
            hold = (MODE == SPMV_RES) ? dsub(hold, sa[k]) : dadd(hold, sa[k]);
          }
        }
      }
    } else if (mine) {
      for (int k = k0; k < k1; k++) {
        const int j = ja[k];
        const T p = dmul(a[k], x[j]);
        if (kGs) {
          if (j != i) sum = dadd(sum, p);
        } else {
          hold = (MODE == SPMV_RES) ? dsub(hold, p) : dadd(hold, p);
        }
      }
    }
    if (mine) {
      if (kGs) {
        const T xi = dsub(hold, sum) / di;
        if (out) out[i - r0base] = xi;
        else const_cast<T*>(x)[i] = xi;
      } else {
        y[i] = hold;
        if (DOT) dot += (double)hw * (double)hold;
      }
    }
    __syncthreads();  // both buffers' readers are done before the next issue
  }
  if (DOT) {
    for (int off = 16; off > 0; off >>= 1) dot += __shfl_xor_sync(0xffffffffu, dot, off);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = dot;
    __syncthreads();
    if (threadIdx.x == 0) {
      double t = 0.0;
      for (int w = 0; w < kRows / 32; w++) t += red[w];
      partial[blockIdx.x] = t;
    }
  }
}

template <class T>
constexpr int staged_smem_bytes() {
  return 2 * (((kStageCap + 8) * 4 + 15) / 16 * 16) +
         2 * (((kStageCap + 8) * (int)sizeof(T) + 15) / 16 * 16);
}

int take_stage_error() {
  int e = 0;
  BN_CUDA(cudaMemcpyFromSymbol(&e, g_stage_err, sizeof(int)));
  if (e) {
    const int z = 0;
    BN_CUDA(cudaMemcpyToSymbol(g_stage_err, &z, sizeof(int)));
  }
  return e;
}

// Group-per-row SpMV for the denser coarse operators: G lanes stride a row
// (coalesced within the group) and combine with a fixed shuffle tree.
template <class T, int G, int MODE, bool DOT>
__global__ void __launch_bounds__(256)
k_spmv_vec(const int* __restrict__ ia, const int* __restrict__ ja, const T* __restrict__ a,
           const T* __restrict__ x, int n, const T* __restrict__ b, T* __restrict__ y,
           const T* __restrict__ dw, double* __restrict__ partial, int skip_long) {
  BN_PDL_ENTRY();
  __shared__ double red[8];
  const int gl = threadIdx.x & (G - 1);
  unsigned gmask = 0xffffffffu;
  if constexpr (G < 32) gmask = ((1u << G) - 1u) << ((threadIdx.x & 31) & ~(G - 1));
  const int groups = (gridDim.x * blockDim.x) / G;
  double dot = 0.0;
  for (int i = (blockIdx.x * blockDim.x + threadIdx.x) / G; i < n; i += groups) {
    const int k0 = ia[i], k1 = ia[i + 1];
    if (skip_long && k1 - k0 > kLongRow) continue;  // long-row kernel
    T sum = T(0);
#pragma unroll 4
    for (int k = k0 + gl; k < k1; k += G) sum = dadd(sum, dmul(a[k], x[ja[k]]));
#pragma unroll
    for (int off = G / 2; off > 0; off >>= 1) sum = dadd(sum, __shfl_xor_sync(gmask, sum, off, G));
    if (gl == 0) {
      T v = sum;
      if (MODE == SPMV_RES) v = dsub(b[i], sum);
      if (MODE == SPMV_ADD) v = dadd(y[i], sum);
      y[i] = v;
      if (DOT) dot += (double)dw[i] * (double)v;
    }
  }
  if (DOT) {
    for (int off = 16; off > 0; off >>= 1) dot += __shfl_xor_sync(0xffffffffu, dot, off);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = dot;
    __syncthreads();
    if (threadIdx.x == 0) {
      double t = 0.0;
      for (int w = 0; w < 8; w++) t += red[w];
      partial[blockIdx.x] = t;
    }
  }
}

// One block per long row.
template <class T, int MODE, bool DOT>
__global__ void __launch_bounds__(kLongThreads)
k_spmv_long(const int* __restrict__ ia, const int* __restrict__ ja, const T* __restrict__ a,
            const T* __restrict__ x, const int* __restrict__ lrows, const T* __restrict__ b,
            T* __restrict__ y, const T* __restrict__ dw, double* __restrict__ partial) {
  BN_PDL_ENTRY();
  __shared__ T red[kLongThreads / 32];
  const int i = lrows[blockIdx.x];
  T sum = T(0);
  for (int k = ia[i] + threadIdx.x; k < ia[i + 1]; k += kLongThreads)
    sum = dadd(sum, dmul(a[k], x[ja[k]]));
  for (int off = 16; off > 0; off >>= 1) sum = dadd(sum, __shfl_xor_sync(0xffffffffu, sum, off));
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = sum;
  __syncthreads();
  if (threadIdx.x == 0) {
    T t = T(0);
    for (int w = 0; w < kLongThreads / 32; w++) t = dadd(t, red[w]);
    T v = t;
    if (MODE == SPMV_RES) v = dsub(b[i], t);
    if (MODE == SPMV_ADD) v = dadd(y[i], t);
    y[i] = v;
    if (DOT) partial[blockIdx.x] = (double)dw[i] * (double)v;
  }
}

__global__ void k_long_rows(const int* __restrict__ ia, int n, int* __restrict__ lrows,
                            int* counter) {
  // warp-aggregated appends (the list is sorted afterwards)
  const int lane = threadIdx.x & 31;
  for (int base = blockIdx.x * blockDim.x; base < n; base += gridDim.x * blockDim.x) {
    const int i = base + threadIdx.x;
    const bool lng = i < n && ia[i + 1] - ia[i] > kLongRow;
    const unsigned m = __ballot_sync(0xffffffffu, lng);
    if (!m) continue;
    int pos0 = 0;
    if (lane == 0) pos0 = atomicAdd(counter, __popc(m));
    pos0 = __shfl_sync(0xffffffffu, pos0, 0);
    if (lng) lrows[pos0 + __popc(m & ((1u << lane) - 1u))] = i;
  }
}

void analyze_rows(const CSR& A, RowLayout& out, cudaStream_t s) {
  const double avg = A.n > 0 ? (double)A.nnz / A.n : 0.0;
  out.group = avg <= 8.0 ? 0 : (avg <= 16.0 ? 4 : (avg <= 48.0 ? 8 : 32));
  // BN_SPMV_GROUP=g pins every operator to one kernel variant (0-3: row
  // tiles of 256/128/64/32 rows, 5: staged 256-row tiles, 4/8/16/32: lanes
  // per row); the autotuner may still change it
  static const int forced = getenv("BN_SPMV_GROUP") ? atoi(getenv("BN_SPMV_GROUP")) : -1;
  if ((forced >= 0 && forced <= 5) || forced == 8 || forced == 16 || forced == 32)
    out.group = forced;
  DBuf<int> cnt(1, s);
  cnt.zero();
  out.lrows.alloc(A.n > 0 ? A.n : 1, s);
  if (A.n > 0)
    BN_LAUNCH(k_long_rows, grid_for(A.n, 256), 256, 0, s, A.ia.p, A.n, out.lrows.p, cnt.p);
  out.nlong = read_scalar(cnt.p, s);
  if (out.nlong > 1) {  // deterministic order
    DBuf<int> tmp_out(out.nlong, s);
    size_t tmp = 0;
    BN_CUDA(cub::DeviceRadixSort::SortKeys(nullptr, tmp, out.lrows.p, tmp_out.p, out.nlong, 0, 32, s));
    DBuf<unsigned char> t(tmp, s);
    BN_CUDA(cub::DeviceRadixSort::SortKeys(t.p, tmp, out.lrows.p, tmp_out.p, out.nlong, 0, 32, s));
    BN_CUDA(cudaMemcpyAsync(out.lrows.p, tmp_out.p, sizeof(int) * out.nlong,
                            cudaMemcpyDeviceToDevice, s));
    BN_CUDA(cudaStreamSynchronize(s));
  }
}

int spmv_partials(int n, int nlong) { return spmv_grid(n) + nlong; }

__global__ void k_tile_keys(const int* __restrict__ key, int n, int ntiles, int* __restrict__ tk,
                            int* __restrict__ ids) {
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < ntiles; t += gridDim.x * blockDim.x) {
    tk[t] = key[t * kRows];
    ids[t] = t;
  }
}

void order_tiles(int n, const int* key, RowLayout& out, cudaStream_t s) {
  const int ntiles = (n + kRows - 1) / kRows;
  if (ntiles <= 1 || !key) { out.tiles = DBuf<int>(); return; }
  DBuf<int> tk(ntiles, s), tk2(ntiles, s), ids(ntiles, s);
  out.tiles.alloc(ntiles, s);
  BN_LAUNCH(k_tile_keys, grid_for(ntiles, 256), 256, 0, s, key, n, ntiles, tk.p, ids.p);
  size_t tmp = 0;
  BN_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tmp, tk.p, tk2.p, ids.p, out.tiles.p, ntiles, 0,
                                          32, s));
  DBuf<unsigned char> t(tmp, s);
  BN_CUDA(cub::DeviceRadixSort::SortPairs(t.p, tmp, tk.p, tk2.p, ids.p, out.tiles.p, ntiles, 0, 32,
                                          s));
  BN_CUDA(cudaStreamSynchronize(s));
}

template <class T, int MODE, bool DOT>
static void spmv_dispatch(const DevMat<T>& A, const T* x, const T* b, T* y, cudaStream_t s,
                          const T* dw, double* partial) {
  const int grid = spmv_grid(A.n);
  const int skip = A.lrows != nullptr ? 1 : 0;
  switch (A.group) {
    case 0:
      BN_LAUNCH_PDL((k_spmv<T, MODE, DOT>), grid, kRows, 0, s, A.ia, A.ja, A.val, x, A.n, b, y, dw,
                partial, skip, A.tiles);
      break;
    case 1:
      BN_LAUNCH_PDL((k_spmv<T, MODE, DOT, 128>), grid, kRows, 0, s, A.ia, A.ja, A.val, x, A.n, b, y,
                dw, partial, skip, A.tiles);
      break;
    case 2:
      BN_LAUNCH_PDL((k_spmv<T, MODE, DOT, 64>), grid, kRows, 0, s, A.ia, A.ja, A.val, x, A.n, b, y,
                dw, partial, skip, A.tiles);
      break;
    case 3:
      BN_LAUNCH_PDL((k_spmv<T, MODE, DOT, 32>), grid, kRows, 0, s, A.ia, A.ja, A.val, x, A.n, b, y,
                dw, partial, skip, A.tiles);
      break;
    case 4:
      BN_LAUNCH_PDL((k_spmv_vec<T, 4, MODE, DOT>), grid, 256, 0, s, A.ia, A.ja, A.val, x, A.n, b, y,
                dw, partial, skip);
      break;
    case 5: {  // row tiles staged by bulk copies (persistent blocks)
      constexpr int smem = staged_smem_bytes<T>();
      static bool attr = false;
      if (!attr) {
        BN_CUDA(cudaFuncSetAttribute(k_spmv_staged<T, MODE, DOT>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
        attr = true;
      }
      BN_LAUNCH_PDL((k_spmv_staged<T, MODE, DOT>), grid, kRows, smem, s, A.ia, A.ja, A.val, x, A.n,
                b, y, dw, partial, skip, A.tiles, 0, (T*)nullptr);
      break;
    }
    case 8:
      BN_LAUNCH_PDL((k_spmv_vec<T, 8, MODE, DOT>), grid, 256, 0, s, A.ia, A.ja, A.val, x, A.n, b, y,
                dw, partial, skip);
      break;
    case 16:
      BN_LAUNCH_PDL((k_spmv_vec<T, 16, MODE, DOT>), grid, 256, 0, s, A.ia, A.ja, A.val, x, A.n, b,
                    y, dw, partial, skip);
      break;
    default:
      BN_LAUNCH_PDL((k_spmv_vec<T, 32, MODE, DOT>), grid, 256, 0, s, A.ia, A.ja, A.val, x, A.n, b, y,
                dw, partial, skip);
      break;
  }
  if (A.nlong > 0)
    BN_LAUNCH_PDL((k_spmv_long<T, MODE, DOT>), A.nlong, kLongThreads, 0, s, A.ia, A.ja, A.val, x,
              A.lrows, b, y, dw, DOT ? partial + grid : nullptr);
}

template <class T>
int spmv(int mode, const DevMat<T>& A, const T* x, const T* b, T* y, cudaStream_t s,
         const T* dot_w, double* partial) {
  if (A.n == 0) return 0;
  if (dot_w) {
    spmv_dispatch<T, SPMV_Y, true>(A, x, b, y, s, dot_w, partial);
    return spmv_partials(A.n, A.nlong);
  }
  switch (mode) {
    case SPMV_Y: spmv_dispatch<T, SPMV_Y, false>(A, x, b, y, s, nullptr, nullptr); break;
    case SPMV_RES: spmv_dispatch<T, SPMV_RES, false>(A, x, b, y, s, nullptr, nullptr); break;
    default: spmv_dispatch<T, SPMV_ADD, false>(A, x, b, y, s, nullptr, nullptr); break;
  }
  return 0;
}

// ----------------------------------------------------- coloured Gauss-Seidel
// x_i = (b_i - sum_{j != i} a_ij x_j) / a_ii for the rows of one colour
// (cf_fwd_gs / cf_bwd_gs, C_amg1/src/amg_cycle.c:52-80; diagonal 1.0 if
// missing).  Rows of one colour share no edge, so a colour is one launch.
// G lanes per row (1 for the short rows of fine levels, 8 or 32 for the
// denser coarse operators).  OUT == nullptr updates x in place; otherwise the
// new values go to out[t] (Jacobi-style overflow classes whose rows may be
// adjacent are computed into a buffer first, then scattered).
template <class T, int G>
__device__ __forceinline__ void gs_rows_short(const int* __restrict__ ia,
                                              const int* __restrict__ ja,
                                              const T* __restrict__ a,
                                              const int* __restrict__ rows, int r0, int nr,
                                              const T* __restrict__ b, T* x, T* __restrict__ out,
                                              int nblocks) {
  const int gl = threadIdx.x & (G - 1);
  const int groups = (nblocks * blockDim.x) / G;
  unsigned gmask = 0xffffffffu;
  if constexpr (G < 32) gmask = ((1u << G) - 1u) << ((threadIdx.x & 31) & ~(G - 1));
  for (int t = (blockIdx.x * blockDim.x + threadIdx.x) / G; t < nr; t += groups) {
    const int i = rows ? rows[t] : r0 + t;
    T sum = T(0), d = T(0);
    bool has_d = false;
#pragma unroll 4
    for (int k = ia[i] + gl; k < ia[i + 1]; k += G) {
      const int j = ja[k];
      const T v = a[k];
      if (j == i) { d = v; has_d = true; }
      else sum = dadd(sum, dmul(v, x[j]));
    }
    if (G > 1) {
#pragma unroll
      for (int off = G / 2; off > 0; off >>= 1) {
        sum = dadd(sum, __shfl_xor_sync(gmask, sum, off, G));
        T od = __shfl_xor_sync(gmask, d, off, G);
        bool oh = __shfl_xor_sync(gmask, has_d, off, G);
        if (oh) { d = od; has_d = true; }
      }
    }
    if (gl == 0) {
      const T xi = dsub(b[i], sum) / (has_d ? d : T(1));
      if (out) out[t] = xi; else x[i] = xi;
    }
  }
}

// one block per long row
template <class T>
__device__ __forceinline__ void gs_row_long(const int* __restrict__ ia,
                                            const int* __restrict__ ja, const T* __restrict__ a,
                                            int t, int i, const T* __restrict__ b, T* x,
                                            T* __restrict__ out) {
  __shared__ T red[kLongThreads / 32];
  __shared__ T dsh;
  __shared__ int has;
  if (threadIdx.x == 0) { has = 0; dsh = T(1); }
  __syncthreads();
  T sum = T(0);
  for (int k = ia[i] + threadIdx.x; k < ia[i + 1]; k += blockDim.x) {
    const int j = ja[k];
    if (j == i) { dsh = a[k]; has = 1; }
    else sum = dadd(sum, dmul(a[k], x[j]));
  }
  for (int off = 16; off > 0; off >>= 1) sum = dadd(sum, __shfl_xor_sync(0xffffffffu, sum, off));
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = sum;
  __syncthreads();
  if (threadIdx.x == 0) {
    T s = T(0);
    for (int w = 0; w < kLongThreads / 32; w++) s = dadd(s, red[w]);
    const T xi = dsub(b[i], s) / (has ? dsh : T(1));
    if (out) out[t] = xi; else x[i] = xi;
  }
}

// x_i = (b_i - sum_{j != i} a_ij x_j) / a_ii for the rows of one colour class
// (cf_fwd_gs / cf_bwd_gs, C_amg1/src/amg_cycle.c:52-80; diagonal 1.0 if
// missing).  Rows of a class share no edge, so a class is one launch: the
// first nb_short blocks take the short rows (G lanes per row: 1 for the
// short rows of fine levels, 8 or 32 for the denser coarse operators); each
// further block takes one of the class's long rows (stored last).  With out
// != nullptr the new values go to out[t] instead (an overflow class, whose
// rows may be adjacent, is computed into a buffer first, then scattered).
template <class T, int G>
__global__ void __launch_bounds__(kLongThreads)
k_gs_class(const int* __restrict__ ia, const int* __restrict__ ja, const T* __restrict__ a,
           const int* __restrict__ rows, int r0, int nshort, int nb_short,
           const T* __restrict__ b, T* x, T* __restrict__ out) {
  BN_PDL_ENTRY();
  if ((int)blockIdx.x < nb_short) {
    gs_rows_short<T, G>(ia, ja, a, rows, r0, nshort, b, x, out, nb_short);
  } else {
    const int t = nshort + (blockIdx.x - nb_short);
    gs_row_long<T>(ia, ja, a, t, rows ? rows[t] : r0 + t, b, x, out);
  }
}

template <class T>
__global__ void k_scatter(const int* __restrict__ rows, int r0, int nr, const T* __restrict__ v,
                          T* __restrict__ x) {
  BN_PDL_ENTRY();
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < nr; t += gridDim.x * blockDim.x)
    x[rows ? rows[t] : r0 + t] = v[t];
}

// Gauss-Seidel class on the staged row tiles (group 0; contiguous classes)
template <class T>
static void gs_staged(const DevMat<T>& A, int r0, int nr, const T* b, T* x, T* out,
                      const T* d, cudaStream_t s) {
  if (nr <= 0) return;
  constexpr int smem = staged_smem_bytes<T>();
  static bool attr = false;
  if (!attr) {
    BN_CUDA(cudaFuncSetAttribute(k_spmv_staged<T, kStagedGS, false>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    attr = true;
  }
  BN_LAUNCH_PDL((k_spmv_staged<T, kStagedGS, false>), spmv_grid(nr), kRows, smem, s, A.ia, A.ja,
            A.val, (const T*)x, nr, b, (T*)d, (const T*)nullptr, (double*)nullptr, 0,
            (const int*)nullptr, r0, out);
}

template <class T>
static void gs_launch(const DevMat<T>& A, const int* rows, int r0, int nr, const T* b, T* x,
                      T* out, int group, cudaStream_t s, int nlong = 0, const T* d = nullptr) {
  if (group == 0 && !rows && d) {  // staged tiles (long rows included: one thread walks each)
    gs_staged<T>(A, r0, nr, b, x, out, d, s);
    return;
  }
  if (group == 0) group = 1;
  const int lanes = group >= 32 ? 32 : group >= 16 ? 16 : group >= 8 ? 8 : group >= 4 ? 4
                                                                                      : group >= 2 ? 2 : 1;
  const int nshort = nr - nlong;
  int nb = 0;
  if (nshort > 0) nb = grid_for((long long)nshort * lanes, kLongThreads, 8);
  const int grid = nb + nlong;
  if (grid == 0) return;
  switch (lanes) {
    case 32:
      BN_LAUNCH_PDL((k_gs_class<T, 32>), grid, kLongThreads, 0, s, A.ia, A.ja, A.val, rows, r0,
                    nshort, nb, b, x, out);
      break;
    case 16:
      BN_LAUNCH_PDL((k_gs_class<T, 16>), grid, kLongThreads, 0, s, A.ia, A.ja, A.val, rows, r0,
                    nshort, nb, b, x, out);
      break;
    case 8:
      BN_LAUNCH_PDL((k_gs_class<T, 8>), grid, kLongThreads, 0, s, A.ia, A.ja, A.val, rows, r0,
                    nshort, nb, b, x, out);
      break;
    case 4:
      BN_LAUNCH_PDL((k_gs_class<T, 4>), grid, kLongThreads, 0, s, A.ia, A.ja, A.val, rows, r0,
                    nshort, nb, b, x, out);
      break;
    case 2:
      BN_LAUNCH_PDL((k_gs_class<T, 2>), grid, kLongThreads, 0, s, A.ia, A.ja, A.val, rows, r0,
                    nshort, nb, b, x, out);
      break;
    default:
      BN_LAUNCH_PDL((k_gs_class<T, 1>), grid, kLongThreads, 0, s, A.ia, A.ja, A.val, rows, r0,
                    nshort, nb, b, x, out);
  }
}

template <class T>
void scatter_range(const T* v, int r0, int nr, T* x, cudaStream_t s) {
  if (nr == 0) return;
  BN_LAUNCH_PDL(k_scatter<T>, grid_for(nr, 256), 256, 0, s, nullptr, r0, nr, v, x);
}
template void scatter_range<double>(const double*, int, int, double*, cudaStream_t);
template void scatter_range<float>(const float*, int, int, float*, cudaStream_t);

template <class T>
void gs_color(const DevMat<T>& A, const int* rows, int r0, int nr, const T* b, T* x, int group,
              cudaStream_t s, int nlong, const T* d) {
  if (nr == 0) return;
  gs_launch<T>(A, rows, r0, nr, b, x, nullptr, group, s, nlong, d);
}

template <class T>
void jacobi_class(const DevMat<T>& A, const int* rows, int r0, int nr, const T* b, T* x, T* tmp,
                  int group, cudaStream_t s, int nlong, const T* d) {
  if (nr == 0) return;
  gs_launch<T>(A, rows, r0, nr, b, x, tmp, group, s, nlong, d);
  BN_LAUNCH_PDL(k_scatter<T>, grid_for(nr, 256), 256, 0, s, rows, r0, nr, tmp, x);
}

// A whole sweep of a small level in one 1024-thread block: classes in
// order (or reverse), a barrier between classes; overflow classes are
// computed into tmp and copied back.  Warp per row.
template <class T>
__global__ void __launch_bounds__(1024)
k_gs_level_block(const int* __restrict__ ia, const int* __restrict__ ja, const T* __restrict__ a,
                 const int* __restrict__ cptr, const int* __restrict__ cjac, int ncls, int forward,
                 const T* __restrict__ b, T* x, T* tmp) {
  BN_PDL_ENTRY();
  for (int q = 0; q < ncls; q++) {
    const int c = forward ? q : ncls - 1 - q;
    const int r0 = cptr[c], r1 = cptr[c + 1];
    const bool jac = cjac[c] != 0;
    const int lane = threadIdx.x & 31;
    for (int i = r0 + (threadIdx.x >> 5); i < r1; i += (blockDim.x >> 5)) {
      T sum = T(0), d = T(0);
      int has = 0;
      for (int k = ia[i] + lane; k < ia[i + 1]; k += 32) {
        const int j = ja[k];
        if (j == i) { d = a[k]; has = 1; }
        else sum = dadd(sum, dmul(a[k], x[j]));
      }
      for (int off = 16; off > 0; off >>= 1) {
        sum = dadd(sum, __shfl_xor_sync(0xffffffffu, sum, off));
        const T od = __shfl_xor_sync(0xffffffffu, d, off);
        const int oh = __shfl_xor_sync(0xffffffffu, has, off);
        if (oh) { d = od; has = 1; }
      }
      if (lane == 0) {
        const T xi = dsub(b[i], sum) / (has ? d : T(1));
        if (jac) tmp[i - r0] = xi; else x[i] = xi;
      }
    }
    __syncthreads();
    if (jac) {
      for (int i = r0 + threadIdx.x; i < r1; i += blockDim.x) x[i] = tmp[i - r0];
      __syncthreads();
    }
  }
}

template <class T>
void gs_level_block(const DevMat<T>& A, const int* cptr, const int* cjac, int ncls, bool forward,
                    const T* b, T* x, T* tmp, cudaStream_t s) {
  if (ncls <= 0) return;
  BN_LAUNCH_PDL(k_gs_level_block<T>, 1, 1024, 0, s, A.ia, A.ja, A.val, cptr, cjac, ncls,
            forward ? 1 : 0, b, x, tmp);
}

// out[t] = in[map[t]]  (gather) ; out[map[t]] = in[t]  (scatter)
template <class T>
__global__ void k_permute(const T* __restrict__ in, const int* __restrict__ map, int n,
                          T* __restrict__ out, int scatter) {
  BN_PDL_ENTRY();
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
    if (scatter) out[map[t]] = in[t];
    else out[t] = in[map[t]];
  }
}
template <class T>
void vpermute(const T* in, const int* map, int n, T* out, bool scatter, cudaStream_t s) {
  if (n) BN_LAUNCH_PDL(k_permute<T>, grid_for(n, 256), 256, 0, s, in, map, n, out, scatter ? 1 : 0);
}

// ------------------------------------------------------------ vector ops
template <class T>
__global__ void k_zero(T* __restrict__ x, int n) {
  BN_PDL_ENTRY();
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) x[i] = T(0);
}
template <class T>
void vzero(T* x, int n, cudaStream_t s) {
  if (n) BN_LAUNCH_PDL(k_zero<T>, grid_for(n, 256), 256, 0, s, x, n);
}

template <class TO, class TI>
__global__ void k_convert(const TI* __restrict__ a, int n, TO* __restrict__ b) {
  BN_PDL_ENTRY();
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    b[i] = (TO)a[i];
}
template <class TO, class TI>
void vconvert(const TI* a, int n, TO* b, cudaStream_t s) {
  if (n) BN_LAUNCH_PDL((k_convert<TO, TI>), grid_for(n, 256), 256, 0, s, a, n, b);
}

// x = u + v  (x may alias u)
template <class T>
__global__ void k_add(const T* __restrict__ u, const T* __restrict__ v, int n, T* x) {
  BN_PDL_ENTRY();
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    x[i] = dadd(u[i], v[i]);
}
template <class T>
void vadd(const T* u, const T* v, int n, T* x, cudaStream_t s) {
  if (n) BN_LAUNCH_PDL(k_add<T>, grid_for(n, 256), 256, 0, s, u, v, n, x);
}

// block partial sums -> one scalar (deterministic order)
__device__ __forceinline__ double block_sum(double v, double* red) {
  for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  double t = 0.0;
  if (threadIdx.x == 0)
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) t += red[w];
  return t;
}

template <class T>
__global__ void k_dot2(const T* __restrict__ u, const T* __restrict__ v,
                       const T* __restrict__ w, int n, double* __restrict__ p0,
                       double* __restrict__ p1) {
  BN_PDL_ENTRY();
  __shared__ double red[32];
  double a = 0.0, c = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double ui = (double)u[i];
    a += ui * (double)v[i];
    if (w) c += ui * (double)w[i];
  }
  double ta = block_sum(a, red);
  __syncthreads();
  double tc = w ? block_sum(c, red) : 0.0;
  if (threadIdx.x == 0) {
    p0[blockIdx.x] = ta;
    if (w) p1[blockIdx.x] = tc;
  }
}

// u.v (and u.w) into partial arrays of kRedBlocks entries
template <class T>
void dot_partials(const T* u, const T* v, const T* w, int n, double* p0, double* p1,
                  cudaStream_t s) {
  BN_LAUNCH_PDL(k_dot2<T>, kRedBlocks, 256, 0, s, u, v, w, n, p0, p1);
}

// y += a u ;  p = z + b p   (uuplmv / umuplv of vector_ops.c with a host scalar)
__global__ void k_axpy(double* __restrict__ y, const double* __restrict__ u, double a, int n) {
  BN_PDL_ENTRY();
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    y[i] = y[i] + u[i] * a;
}
__global__ void k_xpby(double* __restrict__ p, const double* __restrict__ z, double b, int n) {
  BN_PDL_ENTRY();
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    p[i] = z[i] + p[i] * b;
}
void vaxpy(double* y, const double* u, double a, int n, cudaStream_t s) {
  if (n > 0) BN_LAUNCH_PDL(k_axpy, grid_for(n, 256), 256, 0, s, y, u, a, n);
}
void vxpby(double* p, const double* z, double b, int n, cudaStream_t s) {
  if (n > 0) BN_LAUNCH_PDL(k_xpby, grid_for(n, 256), 256, 0, s, p, z, b, n);
}

// ---- segmented PCG (independent systems packed block-diagonally)
// out[k] = sum over the rows of segment k (natural rows ptr[k]..ptr[k+1]-1,
// held at solve index idx[row]) of u*v: one block per segment, fixed order
__global__ void __launch_bounds__(256)
k_seg_dot(const double* __restrict__ u, const double* __restrict__ v,
          const int* __restrict__ ptr, const int* __restrict__ idx, int nseg,
          double* __restrict__ out) {
  BN_PDL_ENTRY();
  __shared__ double red[32];
  for (int k = blockIdx.x; k < nseg; k += gridDim.x) {
    double a = 0.0;
    for (int r = ptr[k] + threadIdx.x; r < ptr[k + 1]; r += blockDim.x) {
      const int t = idx[r];
      a += u[t] * v[t];
    }
    const double tot = block_sum(a, red);
    if (threadIdx.x == 0) out[k] = tot;
    __syncthreads();
  }
}
void seg_dot(const double* u, const double* v, const int* ptr, const int* idx, int nseg,
             double* out, cudaStream_t s) {
  if (nseg > 0) BN_LAUNCH_PDL(k_seg_dot, nseg < 4096 ? nseg : 4096, 256, 0, s, u, v, ptr, idx, nseg, out);
}

// segment of every solve-numbered row: perm[t] is its natural row
__global__ void k_seg_of_rows(const int* __restrict__ perm, int n, const int* __restrict__ ptr,
                              int nseg, int* __restrict__ seg) {
  BN_PDL_ENTRY();
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
    const int r = perm[t];
    int lo = 0, hi = nseg - 1;  // last segment starting at or before r
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (ptr[mid] <= r) lo = mid;
      else hi = mid - 1;
    }
    seg[t] = lo;
  }
}
void seg_of_rows(const int* perm, int n, const int* ptr, int nseg, int* seg, cudaStream_t s) {
  if (n > 0) BN_LAUNCH_PDL(k_seg_of_rows, grid_for(n, 256), 256, 0, s, perm, n, ptr, nseg, seg);
}

// x += alpha_k p ; r -= alpha_k Ap  (k the row's segment)
__global__ void k_seg_update_xr(double* __restrict__ x, double* __restrict__ r,
                                const double* __restrict__ p, const double* __restrict__ ap,
                                const int* __restrict__ seg, const double* __restrict__ alpha,
                                int n) {
  BN_PDL_ENTRY();
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double a = alpha[seg[i]];
    x[i] = x[i] + p[i] * a;
    r[i] = r[i] + ap[i] * (-a);
  }
}
void seg_update_xr(double* x, double* r, const double* p, const double* ap, const int* seg,
                   const double* alpha, int n, cudaStream_t s) {
  if (n > 0) BN_LAUNCH_PDL(k_seg_update_xr, grid_for(n, 256), 256, 0, s, x, r, p, ap, seg, alpha, n);
}

// p = z + beta_k p
__global__ void k_seg_update_p(double* __restrict__ p, const double* __restrict__ z,
                               const int* __restrict__ seg, const double* __restrict__ beta,
                               int n) {
  BN_PDL_ENTRY();
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    p[i] = z[i] + p[i] * beta[seg[i]];
}
void seg_update_p(double* p, const double* z, const int* seg, const double* beta, int n,
                  cudaStream_t s) {
  if (n > 0) BN_LAUNCH_PDL(k_seg_update_p, grid_for(n, 256), 256, 0, s, p, z, seg, beta, n);
}

// per-segment scalars.  sc layout: [SEG_* * nseg + k]
__global__ void k_seg_alpha(const double* __restrict__ rz, const double* __restrict__ pap,
                            const int* __restrict__ active, int nseg, double* __restrict__ alpha) {
  BN_PDL_ENTRY();
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nseg; k += gridDim.x * blockDim.x)
    alpha[k] = active[k] ? rz[k] / pap[k] : 0.0;
}
void seg_alpha(const double* rz, const double* pap, const int* active, int nseg, double* alpha,
               cudaStream_t s) {
  if (nseg > 0) BN_LAUNCH_PDL(k_seg_alpha, grid_for(nseg, 256), 256, 0, s, rz, pap, active, nseg, alpha);
}

// beta (standard or flexible), convergence test, rotate rz; counts the
// segments still iterating into *nactive
__global__ void k_seg_next(double* __restrict__ rz, const double* __restrict__ rznew,
                           const double* __restrict__ rzold_new, const double* __restrict__ rr,
                           const double* __restrict__ bb, const double* __restrict__ rz0,
                           int* __restrict__ active, int* __restrict__ iters,
                           double* __restrict__ beta, int nseg, int flexible, int relres,
                           double tol, int iter, const int* __restrict__ iters_done,
                           int* nactive) {
  BN_PDL_ENTRY();
  if (iters_done) iter = *iters_done + 1;  // device-driven loop: iterations done so far
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nseg; k += gridDim.x * blockDim.x) {
    if (!active[k]) { beta[k] = 0.0; continue; }
    const double b2 = bb[k] > 0.0 ? bb[k] : 1.0;
    const double crit = relres ? sqrt(rr[k] / b2) : sqrt(rznew[k] / rz0[k]);
    beta[k] = flexible ? (rznew[k] - rzold_new[k]) / rz[k] : rznew[k] / rz[k];
    rz[k] = rznew[k];
    if (crit < tol || rz0[k] == 0.0 || !isfinite(crit)) {
      active[k] = 0;
      iters[k] = isfinite(crit) ? iter : -iter;
    } else {
      atomicAdd(nactive, 1);
    }
  }
}
void seg_next(double* rz, const double* rznew, const double* rzold_new, const double* rr,
              const double* bb, const double* rz0, int* active, int* iters, double* beta,
              int nseg, int flexible, int relres, double tol, int iter, int* nactive,
              cudaStream_t s, const int* iters_done) {
  if (nseg > 0)
    BN_LAUNCH_PDL(k_seg_next, grid_for(nseg, 256), 256, 0, s, rz, rznew, rzold_new, rr, bb, rz0,
              active, iters, beta, nseg, flexible, relres, tol, iter, iters_done, nactive);
}

// Reduce a partial array into slot `dst` of the scalar block.
__global__ void k_reduce(const double* __restrict__ part, int m, double* __restrict__ out) {
  BN_PDL_ENTRY();
  __shared__ double red[32];
  double v = 0.0;
  for (int i = threadIdx.x; i < m; i += blockDim.x) v += part[i];
  double t = block_sum(v, red);
  if (threadIdx.x == 0) *out = t;
}
void reduce_partials(const double* part, int m, double* out, cudaStream_t s) {
  BN_LAUNCH_PDL(k_reduce, 1, 1024, 0, s, part, m, out);
}

// x += alpha p ; r -= alpha Ap ; partial r.r     (alpha = sc[RZ] / sc[PAP])
__global__ void k_pcg_update_xr(double* __restrict__ x, double* __restrict__ r,
                                const double* __restrict__ p, const double* __restrict__ ap,
                                int n, const double* __restrict__ sc, double* __restrict__ part) {
  BN_PDL_ENTRY();
  __shared__ double red[32];
  const double alpha = sc[SC_RZ] / sc[SC_PAP];
  double rr = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    x[i] = x[i] + p[i] * alpha;        // uuplmv: u + v * smult
    double ri = r[i] + ap[i] * (-alpha);
    r[i] = ri;
    rr += ri * ri;
  }
  double t = block_sum(rr, red);
  if (threadIdx.x == 0) part[blockIdx.x] = t;
}
void pcg_update_xr(double* x, double* r, const double* p, const double* ap, int n,
                   const double* sc, double* part, cudaStream_t s) {
  BN_LAUNCH_PDL(k_pcg_update_xr, kRedBlocks, 256, 0, s, x, r, p, ap, n, sc, part);
}

// p = z + beta p ; beta from the scalar block (standard or flexible)
__global__ void k_pcg_update_p(double* __restrict__ p, const double* __restrict__ z, int n,
                               const double* __restrict__ sc) {
  BN_PDL_ENTRY();
  const double beta = sc[SC_BETA];
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    p[i] = beta * p[i] + z[i];         // umuplv: smult * u + v
}
void pcg_update_p(double* p, const double* z, int n, const double* sc, cudaStream_t s) {
  BN_LAUNCH_PDL(k_pcg_update_p, grid_for(n, 256), 256, 0, s, p, z, n, sc);
}

// After z = M r: reduce r.z (and r.z_old), form beta, rotate rz, publish the
// convergence scalars.  One thread.
__global__ void k_pcg_scalars(double* sc, int flexible) {
  BN_PDL_ENTRY();
  const double rz_new = sc[SC_RZNEW];
  double beta;
  if (flexible)
    beta = (rz_new - sc[SC_RZOLD_NEW]) / sc[SC_RZ];  // r_{k+1}.(z_{k+1}-z_k) / r_k.z_k
  else
    beta = rz_new / sc[SC_RZ];
  sc[SC_BETA] = beta;
  sc[SC_RZ_PREV] = sc[SC_RZ];
  sc[SC_RZ] = rz_new;
}
void pcg_scalars(double* sc, int flexible, cudaStream_t s) {
  BN_LAUNCH_PDL(k_pcg_scalars, 1, 1, 0, s, sc, flexible);
}

// explicit instantiations
#define BN_INST(T)                                                                           \
  template int spmv<T>(int, const DevMat<T>&, const T*, const T*, T*, cudaStream_t, const T*,  \
                       double*);                                                             \
  template void gs_color<T>(const DevMat<T>&, const int*, int, int, const T*, T*, int,       \
                            cudaStream_t, int, const T*);                                    \
  template void jacobi_class<T>(const DevMat<T>&, const int*, int, int, const T*, T*, T*, int,\
                                cudaStream_t, int, const T*);                                \
  template void vpermute<T>(const T*, const int*, int, T*, bool, cudaStream_t);              \
  template void gs_level_block<T>(const DevMat<T>&, const int*, const int*, int, bool,       \
                                  const T*, T*, T*, cudaStream_t);                           \
  template void vzero<T>(T*, int, cudaStream_t);                                             \
  template void vadd<T>(const T*, const T*, int, T*, cudaStream_t);                          \
  template void dot_partials<T>(const T*, const T*, const T*, int, double*, double*,          \
                                cudaStream_t);
BN_INST(double)
BN_INST(float)
template void vconvert<float, double>(const double*, int, float*, cudaStream_t);
template void vconvert<double, float>(const float*, int, double*, cudaStream_t);

}  // namespace bn
