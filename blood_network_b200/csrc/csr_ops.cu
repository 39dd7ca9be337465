// CSR primitives on the device: prefix sums, stable transpose, the
// reference-order sparse add used for symmetrisation, and input validation.
//
// Reference behaviour reproduced:
//  * dcsr_transz (C_amg1/include/agg_lib.h:120-183): row j of A^T lists the
//    rows i of A that hold column j in increasing i (counting sort, stable).
//  * dcsr_mat_add (agg_lib.h:186-243): row i of C = A + B is A's row in A's
//    order followed by the entries of B's row whose column A's row lacks, in
//    B's order; values a, a+b, or b.  Symmetrisation then scales by 0.5
//    (amg_wrapper.c:59-76, build_hierarchy.c:118-130).
#include "internal.cuh"

#include <cub/cub.cuh>
#include <stdlib.h>
#include <time.h>

namespace bn {

std::atomic<unsigned long long> g_launch_count{0};

// Off by default: on the 20M network the solve measured slower with it
// (mixed 103.6 ms against 98.5 ms, FP64 139.2 against 122.9 ms, same run);
// BN_PDL=1 turns it on.
bool pdl_enabled() {
  static const bool on = getenv("BN_PDL") != nullptr && atoi(getenv("BN_PDL")) != 0;
  return on;
}

bool trace_on() {
  static int on = -1;
  if (on < 0) {
    const char* e = getenv("BN_TRACE");
    on = (e && e[0] && e[0] != '0') ? 1 : 0;
  }
  return on == 1;
}

double wall_seconds() {
  struct timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return ts.tv_sec + 1e-9 * ts.tv_nsec;
}

// ------------------------------------------------------------------ scans
int scan_counts(int* cnt, int n, cudaStream_t s) {
  // exclusive scan over n+1 entries (the last input entry is ignored/0)
  size_t tmp = 0;
  BN_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tmp, cnt, cnt, n + 1, s));
  DBuf<unsigned char> t(tmp, s);
  BN_CUDA(cub::DeviceScan::ExclusiveSum(t.p, tmp, cnt, cnt, n + 1, s));
  return read_scalar(cnt + n, s);
}

long long scan_counts64(long long* cnt, int n, cudaStream_t s) {
  size_t tmp = 0;
  BN_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tmp, cnt, cnt, n + 1, s));
  DBuf<unsigned char> t(tmp, s);
  BN_CUDA(cub::DeviceScan::ExclusiveSum(t.p, tmp, cnt, cnt, n + 1, s));
  return read_scalar(cnt + n, s);
}

void exclusive_scan_i32(const int* in, int* out, int n, cudaStream_t s) {
  size_t tmp = 0;
  BN_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tmp, in, out, n, s));
  DBuf<unsigned char> t(tmp, s);
  BN_CUDA(cub::DeviceScan::ExclusiveSum(t.p, tmp, in, out, n, s));
}

// ------------------------------------------------------------------ helpers
__global__ void k_row_of(const int* __restrict__ ia, int n, int* __restrict__ row) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    for (int k = ia[i]; k < ia[i + 1]; k++) row[k] = i;
}

__global__ void k_iota(int* __restrict__ a, int n) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) a[i] = i;
}

__global__ void k_col_count(const int* __restrict__ ja, int nnz, int* __restrict__ cnt) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nnz; k += gridDim.x * blockDim.x)
    atomicAdd(&cnt[ja[k]], 1);
}

__global__ void k_gather_transpose(const int* __restrict__ order, const int* __restrict__ row,
                                   const double* __restrict__ val, int nnz,
                                   int* __restrict__ tja, double* __restrict__ tval) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < nnz; p += gridDim.x * blockDim.x) {
    int k = order[p];
    tja[p] = row[k];
    if (tval) tval[p] = val[k];
  }
}

static int bits_for(int m) {
  int b = 1;
  while ((1LL << b) < (long long)m) b++;
  return b;
}

void transpose(const CSR& A, CSR& T, cudaStream_t s, bool with_val) {
  const int n = A.n, m = A.m, nnz = A.nnz;
  T.alloc(m, n, nnz, s, with_val);
  // column counts -> T.ia
  T.ia.zero();
  if (nnz > 0)
    BN_LAUNCH(k_col_count, grid_for(nnz, 256), 256, 0, s, A.ja.p, nnz, T.ia.p);
  scan_counts(T.ia.p, m, s);
  if (nnz == 0) return;
  // stable order: LSD radix sort of (column, k); equal columns keep k order,
  // i.e. increasing row -- the counting-sort order of dcsr_transz.
  DBuf<int> row(nnz, s), kin(nnz, s), keys_out(nnz, s), kout(nnz, s);
  BN_LAUNCH(k_row_of, grid_for(n, 256), 256, 0, s, A.ia.p, n, row.p);
  BN_LAUNCH(k_iota, grid_for(nnz, 256), 256, 0, s, kin.p, nnz);
  size_t tmp = 0;
  int eb = bits_for(m);
  BN_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tmp, A.ja.p, keys_out.p, kin.p, kout.p, nnz, 0, eb, s));
  DBuf<unsigned char> t(tmp, s);
  BN_CUDA(cub::DeviceRadixSort::SortPairs(t.p, tmp, A.ja.p, keys_out.p, kin.p, kout.p, nnz, 0, eb, s));
  BN_LAUNCH(k_gather_transpose, grid_for(nnz, 256), 256, 0, s, kout.p, row.p,
            with_val ? A.val.p : nullptr, nnz, T.ja.p, with_val ? T.val.p : nullptr);
}

// ------------------------------------------------------------------ merge-add
// Warp per row.  A's columns go into an open-addressing table (column ->
// position in A's row); B's entries are looked up in parallel.  A match adds
// into A's slot (one writer: rows hold no repeated column), misses are
// appended in B's order via a ballot prefix.  Rows up to kAddCap/2 entries
// use a per-warp table in shared memory; longer rows (coarse-level hubs) use
// a per-row table in global memory sized 2x the row.
constexpr int kAddCap = 512;   // shared table entries per warp
constexpr int kAddWarps = 4;   // warps per block

// rows longer than kAddHuge entries of A (coarse-level hubs of up to ~10^6
// entries): a block per row on the same global table, the misses appended in
// B's order through a block-wide ballot prefix
constexpr int kAddHuge = 8192;
constexpr int kAddBlock = 512;

__device__ __forceinline__ bool add_huge(const int* __restrict__ aia, int i) {
  return aia[i + 1] - aia[i] > kAddHuge;
}


struct AddTable {
  int* keys;
  int* vals;
  double* acc;
  unsigned mask;
};

__device__ __forceinline__ unsigned add_hash(int key, unsigned mask) {
  return ((unsigned)key * 2654435761u >> 9) & mask;
}
__device__ __forceinline__ void tbl_insert(AddTable t, int key, int v) {
  unsigned h = add_hash(key, t.mask);
  while (true) {
    int prev = atomicCAS(&t.keys[h], -1, key);
    if (prev == -1 || prev == key) { t.vals[h] = v; return; }
    h = (h + 1) & t.mask;
  }
}
__device__ __forceinline__ int tbl_find(AddTable t, int key) {
  unsigned h = add_hash(key, t.mask);
  while (true) {
    int k = t.keys[h];
    if (k == key) return t.vals[h];
    if (k == -1) return -1;
    h = (h + 1) & t.mask;
  }
}

__device__ int add_count_row(int i, AddTable t, int lane, const int* __restrict__ aia,
                             const int* __restrict__ aja, const int* __restrict__ bia,
                             const int* __restrict__ bja) {
  const int a0 = aia[i], la = aia[i + 1] - a0;
  const int b0 = bia[i], lb = bia[i + 1] - b0;
  for (unsigned e = lane; e <= t.mask; e += 32) t.keys[e] = -1;
  __syncwarp();
  for (int q = lane; q < la; q += 32) tbl_insert(t, aja[a0 + q], q);
  __syncwarp();
  int extra = 0;
  for (int q = lane; q < lb; q += 32) extra += (tbl_find(t, bja[b0 + q]) < 0);
  for (int off = 16; off > 0; off >>= 1) extra += __shfl_xor_sync(0xffffffffu, extra, off);
  __syncwarp();
  return la + extra;
}

__device__ void add_fill_row(int i, AddTable t, int lane, const int* __restrict__ aia,
                             const int* __restrict__ aja, const double* __restrict__ aval,
                             const int* __restrict__ bia, const int* __restrict__ bja,
                             const double* __restrict__ bval, double scale, int p0,
                             int* __restrict__ cja, double* __restrict__ cval) {
  const int a0 = aia[i], la = aia[i + 1] - a0;
  const int b0 = bia[i], lb = bia[i + 1] - b0;
  const unsigned lt = (1u << lane) - 1u;
  for (unsigned e = lane; e <= t.mask; e += 32) t.keys[e] = -1;
  __syncwarp();
  for (int q = lane; q < la; q += 32) {
    int c = aja[a0 + q];
    tbl_insert(t, c, q);
    t.acc[q] = aval[a0 + q];
    cja[p0 + q] = c;
  }
  __syncwarp();
  int appended = 0;
  for (int base = 0; base < lb; base += 32) {
    const int q = base + lane;
    int pos = -2, c = 0;
    double v = 0.0;
    if (q < lb) {
      c = bja[b0 + q];
      v = bval[b0 + q];
      pos = tbl_find(t, c);
      if (pos >= 0) t.acc[pos] = xadd(t.acc[pos], v);
    }
    const unsigned miss = __ballot_sync(0xffffffffu, pos == -1);
    if (pos == -1) {
      const int o = p0 + la + appended + __popc(miss & lt);
      cja[o] = c;
      cval[o] = xmul(v, scale);
    }
    appended += __popc(miss);
  }
  __syncwarp();
  for (int q = lane; q < la; q += 32) cval[p0 + q] = xmul(t.acc[q], scale);
  __syncwarp();
}

// short rows: per-warp shared tables; long rows are listed for the global path
__global__ void __launch_bounds__(32 * kAddWarps)
k_add_count_w(const int* __restrict__ aia, const int* __restrict__ aja,
              const int* __restrict__ bia, const int* __restrict__ bja, int n,
              int* __restrict__ cnt, int* __restrict__ long_rows, int* nlong) {
  __shared__ int keys_s[kAddWarps][kAddCap];
  __shared__ int vals_s[kAddWarps][kAddCap];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  AddTable t{keys_s[w], vals_s[w], nullptr, kAddCap - 1};
  for (int i = blockIdx.x * kAddWarps + w; i < n; i += gridDim.x * kAddWarps) {
    if (aia[i + 1] - aia[i] > kAddCap / 2) {
      if (lane == 0) long_rows[atomicAdd(nlong, 1)] = i;
      continue;
    }
    int c = add_count_row(i, t, lane, aia, aja, bia, bja);
    if (lane == 0) cnt[i] = c;
  }
}

__global__ void __launch_bounds__(32 * kAddWarps)
k_add_fill_w(const int* __restrict__ aia, const int* __restrict__ aja,
             const double* __restrict__ aval, const int* __restrict__ bia,
             const int* __restrict__ bja, const double* __restrict__ bval, int n, double scale,
             const int* __restrict__ cia, int* __restrict__ cja, double* __restrict__ cval) {
  __shared__ int keys_s[kAddWarps][kAddCap];
  __shared__ int vals_s[kAddWarps][kAddCap];
  __shared__ double acc_s[kAddWarps][kAddCap / 2];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  AddTable t{keys_s[w], vals_s[w], acc_s[w], kAddCap - 1};
  for (int i = blockIdx.x * kAddWarps + w; i < n; i += gridDim.x * kAddWarps) {
    if (aia[i + 1] - aia[i] > kAddCap / 2) continue;
    add_fill_row(i, t, lane, aia, aja, aval, bia, bja, bval, scale, cia[i], cja, cval);
  }
}

// long rows: warp per row, table in global memory at toff[q]
__global__ void k_add_count_g(const int* __restrict__ aia, const int* __restrict__ aja,
                              const int* __restrict__ bia, const int* __restrict__ bja,
                              const int* __restrict__ rows, int m,
                              const long long* __restrict__ toff, int* __restrict__ gkeys,
                              int* __restrict__ gvals, int* __restrict__ cnt) {
  const int lane = threadIdx.x & 31;
  const int warps = (gridDim.x * blockDim.x) >> 5;
  for (int q = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; q < m; q += warps) {
    if (add_huge(aia, rows[q])) continue;
    const long long off = toff[q];
    AddTable t{gkeys + off, gvals + off, nullptr, (unsigned)(toff[q + 1] - off) - 1};
    int c = add_count_row(rows[q], t, lane, aia, aja, bia, bja);
    if (lane == 0) cnt[rows[q]] = c;
  }
}

__global__ void k_add_fill_g(const int* __restrict__ aia, const int* __restrict__ aja,
                             const double* __restrict__ aval, const int* __restrict__ bia,
                             const int* __restrict__ bja, const double* __restrict__ bval,
                             const int* __restrict__ rows, int m, double scale,
                             const long long* __restrict__ toff, int* __restrict__ gkeys,
                             int* __restrict__ gvals, double* __restrict__ gacc,
                             const int* __restrict__ cia, int* __restrict__ cja,
                             double* __restrict__ cval) {
  const int lane = threadIdx.x & 31;
  const int warps = (gridDim.x * blockDim.x) >> 5;
  for (int q = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; q < m; q += warps) {
    if (add_huge(aia, rows[q])) continue;
    const long long off = toff[q];
    AddTable t{gkeys + off, gvals + off, gacc + off / 2, (unsigned)(toff[q + 1] - off) - 1};
    const int i = rows[q];
    add_fill_row(i, t, lane, aia, aja, aval, bia, bja, bval, scale, cia[i], cja, cval);
  }
}

__global__ void __launch_bounds__(kAddBlock)
k_add_count_b(const int* __restrict__ aia, const int* __restrict__ aja,
              const int* __restrict__ bia, const int* __restrict__ bja,
              const int* __restrict__ rows, int m, const long long* __restrict__ toff,
              int* __restrict__ gkeys, int* __restrict__ gvals, int* __restrict__ cnt) {
  __shared__ int red[kAddBlock / 32];
  for (int q = blockIdx.x; q < m; q += gridDim.x) {
    const int i = rows[q];
    if (!add_huge(aia, i)) continue;
    const long long off = toff[q];
    AddTable t{gkeys + off, gvals + off, nullptr, (unsigned)(toff[q + 1] - off) - 1};
    const int a0 = aia[i], la = aia[i + 1] - a0;
    const int b0 = bia[i], lb = bia[i + 1] - b0;
    for (unsigned e = threadIdx.x; e <= t.mask; e += blockDim.x) t.keys[e] = -1;
    __syncthreads();
    for (int k = threadIdx.x; k < la; k += blockDim.x) tbl_insert(t, aja[a0 + k], k);
    __syncthreads();
    int extra = 0;
    for (int k = threadIdx.x; k < lb; k += blockDim.x) extra += (tbl_find(t, bja[b0 + k]) < 0);
    for (int o = 16; o > 0; o >>= 1) extra += __shfl_xor_sync(0xffffffffu, extra, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = extra;
    __syncthreads();
    if (threadIdx.x == 0) {
      int tot = la;
      for (int w = 0; w < kAddBlock / 32; w++) tot += red[w];
      cnt[i] = tot;
    }
    __syncthreads();
  }
}

__global__ void __launch_bounds__(kAddBlock)
k_add_fill_b(const int* __restrict__ aia, const int* __restrict__ aja,
             const double* __restrict__ aval, const int* __restrict__ bia,
             const int* __restrict__ bja, const double* __restrict__ bval,
             const int* __restrict__ rows, int m, double scale,
             const long long* __restrict__ toff, int* __restrict__ gkeys,
             int* __restrict__ gvals, double* __restrict__ gacc, const int* __restrict__ cia,
             int* __restrict__ cja, double* __restrict__ cval) {
  __shared__ int wmiss[kAddBlock / 32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const unsigned lt = (1u << lane) - 1u;
  for (int q = blockIdx.x; q < m; q += gridDim.x) {
    const int i = rows[q];
    if (!add_huge(aia, i)) continue;
    const long long off = toff[q];
    AddTable t{gkeys + off, gvals + off, gacc + off / 2, (unsigned)(toff[q + 1] - off) - 1};
    const int a0 = aia[i], la = aia[i + 1] - a0;
    const int b0 = bia[i], lb = bia[i + 1] - b0;
    const int p0 = cia[i];
    for (unsigned e = threadIdx.x; e <= t.mask; e += blockDim.x) t.keys[e] = -1;
    __syncthreads();
    for (int k = threadIdx.x; k < la; k += blockDim.x) {
      const int c = aja[a0 + k];
      tbl_insert(t, c, k);
      t.acc[k] = aval[a0 + k];
      cja[p0 + k] = c;
    }
    __syncthreads();
    int appended = 0;
    for (int base = 0; base < lb; base += blockDim.x) {
      const int k = base + threadIdx.x;
      int pos = -2, c = 0;
      double v = 0.0;
      if (k < lb) {
        c = bja[b0 + k];
        v = bval[b0 + k];
        pos = tbl_find(t, c);
        if (pos >= 0) t.acc[pos] = xadd(t.acc[pos], v);  // one writer per slot
      }
      const unsigned miss = __ballot_sync(0xffffffffu, pos == -1);
      if (lane == 0) wmiss[w] = __popc(miss);
      __syncthreads();
      int before = 0, total = 0;
      for (int u = 0; u < kAddBlock / 32; u++) {
        before += (u < w) ? wmiss[u] : 0;
        total += wmiss[u];
      }
      if (pos == -1) {
        const int o = p0 + la + appended + before + __popc(miss & lt);
        cja[o] = c;
        cval[o] = xmul(v, scale);
      }
      appended += total;
      __syncthreads();
    }
    for (int k = threadIdx.x; k < la; k += blockDim.x) cval[p0 + k] = xmul(t.acc[k], scale);
    __syncthreads();
  }
}

__global__ void k_add_long_caps(const int* __restrict__ aia, const int* __restrict__ rows, int m,
                                long long* __restrict__ cap) {
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < m; q += gridDim.x * blockDim.x) {
    long long need = 2LL * (aia[rows[q] + 1] - aia[rows[q]]);
    long long c = 64;
    while (c < need) c <<= 1;
    cap[q] = c;
  }
}

// C = (A + B) * scale in the reference's entry order.  Neither A nor B may
// hold a repeated column within a row (inputs are validated for that).
void add_scaled(const CSR& A, const CSR& B, double scale, CSR& C, cudaStream_t s) {
  BN_REQUIRE(A.n == B.n && A.m == B.m, BN_ERR_ARG, "add: dimension mismatch");
  const int n = A.n;
  DBuf<int> cnt((size_t)n + 1, s), lrows(n > 0 ? n : 1, s), nl(1, s);
  cnt.zero();
  nl.zero();
  const int gw = grid_for((long long)n, kAddWarps, 64);
  if (n > 0)
    BN_LAUNCH(k_add_count_w, gw, 32 * kAddWarps, 0, s, A.ia.p, A.ja.p, B.ia.p, B.ja.p, n, cnt.p,
              lrows.p, nl.p);
  const int m = read_scalar(nl.p, s);
  DBuf<long long> toff;
  DBuf<int> gkeys, gvals;
  DBuf<double> gacc;
  const int gl = grid_for((long long)m * 32, 128, 16);
  if (m > 0) {
    toff.alloc((size_t)m + 1, s);
    toff.zero();
    BN_LAUNCH(k_add_long_caps, grid_for(m, 128), 128, 0, s, A.ia.p, lrows.p, m, toff.p);
    long long total = scan_counts64(toff.p, m, s);
    gkeys.alloc((size_t)total, s);
    gvals.alloc((size_t)total, s);
    gacc.alloc((size_t)total / 2 + 1, s);
    BN_LAUNCH(k_add_count_g, gl, 128, 0, s, A.ia.p, A.ja.p, B.ia.p, B.ja.p, lrows.p, m, toff.p,
              gkeys.p, gvals.p, cnt.p);
    BN_LAUNCH(k_add_count_b, m < 1024 ? m : 1024, kAddBlock, 0, s, A.ia.p, A.ja.p, B.ia.p,
              B.ja.p, lrows.p, m, toff.p, gkeys.p, gvals.p, cnt.p);
  }
  int nnz = scan_counts(cnt.p, n, s);
  C.n = n; C.m = A.m; C.nnz = nnz;
  C.ia = std::move(cnt);
  C.ja.alloc((size_t)(nnz > 0 ? nnz : 1), s);
  C.val.alloc((size_t)(nnz > 0 ? nnz : 1), s);
  if (n > 0)
    BN_LAUNCH(k_add_fill_w, gw, 32 * kAddWarps, 0, s, A.ia.p, A.ja.p, A.val.p, B.ia.p, B.ja.p,
              B.val.p, n, scale, C.ia.p, C.ja.p, C.val.p);
  if (m > 0) {
    BN_LAUNCH(k_add_fill_g, gl, 128, 0, s, A.ia.p, A.ja.p, A.val.p, B.ia.p, B.ja.p, B.val.p,
              lrows.p, m, scale, toff.p, gkeys.p, gvals.p, gacc.p, C.ia.p, C.ja.p, C.val.p);
    BN_LAUNCH(k_add_fill_b, m < 1024 ? m : 1024, kAddBlock, 0, s, A.ia.p, A.ja.p, A.val.p,
              B.ia.p, B.ja.p, B.val.p, lrows.p, m, scale, toff.p, gkeys.p, gvals.p, gacc.p,
              C.ia.p, C.ja.p, C.val.p);
  }
}

// (A + A^T) / 2 of a structurally symmetric A.  The reference's merge-add
// (row i of A, then the entries of row i of A^T that A's row lacks, times
// 0.5; agg_lib.h dcsr_mat_add, build_hierarchy.c:116-126) appends nothing
// then, so the result keeps A's pattern and entry order with
// c_ij = (a_ij + a_ji) * 0.5; a_ji is found by binary search in row i of A^T,
// whose columns are increasing (the transpose keeps rows in order).  A warp
// per row, its lanes striding the row's entries; rows longer than kSymLong
// go to a block each.  A missing a_ji sets *asym and the general merge-add
// runs instead.
constexpr int kSymLong = 1024;

__device__ __forceinline__ int sym_find(const int* __restrict__ tja, int lo, int hi, int key) {
  int a = lo, b = hi;
  while (a < b) {
    const int mid = (a + b) >> 1;
    if (tja[mid] < key) a = mid + 1;
    else b = mid;
  }
  return (a < hi && tja[a] == key) ? a : -1;
}

__global__ void k_sym_rows(const int* __restrict__ ia, const int* __restrict__ ja,
                           const double* __restrict__ a, const int* __restrict__ tia,
                           const int* __restrict__ tja, const double* __restrict__ ta, int n,
                           double* __restrict__ out, int* __restrict__ asym,
                           int* __restrict__ longs, int* __restrict__ nlong) {
  const int lane = threadIdx.x & 31;
  const int nw = (gridDim.x * blockDim.x) >> 5;
  for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < n; i += nw) {
    const int k0 = ia[i], k1 = ia[i + 1];
    if (tia[i + 1] - tia[i] != k1 - k0) {
      if (lane == 0) atomicOr(asym, 1);
      continue;
    }
    if (k1 - k0 > kSymLong) {
      if (lane == 0) longs[atomicAdd(nlong, 1)] = i;
      continue;
    }
    const int t0 = tia[i], t1 = tia[i + 1];
    for (int k = k0 + lane; k < k1; k += 32) {
      const int p = sym_find(tja, t0, t1, ja[k]);
      if (p < 0) {
        atomicOr(asym, 1);
        continue;
      }
      out[k] = xmul(xadd(a[k], ta[p]), 0.5);
    }
  }
}

__global__ void k_sym_long(const int* __restrict__ ia, const int* __restrict__ ja,
                           const double* __restrict__ a, const int* __restrict__ tia,
                           const int* __restrict__ tja, const double* __restrict__ ta,
                           const int* __restrict__ longs, double* __restrict__ out,
                           int* __restrict__ asym) {
  const int i = longs[blockIdx.x];
  for (int k = ia[i] + threadIdx.x; k < ia[i + 1]; k += blockDim.x) {
    const int p = sym_find(tja, tia[i], tia[i + 1], ja[k]);
    if (p < 0) {
      atomicOr(asym, 1);
      continue;
    }
    out[k] = xmul(xadd(a[k], ta[p]), 0.5);
  }
}

void symmetrize(const CSR& A, CSR& out, cudaStream_t s) {
  CSR T;
  transpose(A, T, s, true);
  const int n = A.n;
  if (n > 0 && A.n == A.m && A.nnz > 0) {
    DBuf<int> flags(2, s), longs(n, s);
    flags.zero();
    out.n = A.n;
    out.m = A.m;
    out.nnz = A.nnz;
    out.ia.alloc((size_t)n + 1, s);
    out.ja.alloc((size_t)A.nnz, s);
    out.val.alloc((size_t)A.nnz, s);
    BN_LAUNCH(k_sym_rows, grid_for((long long)n * 32, 256), 256, 0, s, A.ia.p, A.ja.p, A.val.p, T.ia.p, T.ja.p,
              T.val.p, n, out.val.p, flags.p, longs.p, flags.p + 1);
    int h[2];
    flags.download(h, 2);
    BN_CUDA(cudaStreamSynchronize(s));
    if (!h[0] && h[1] > 0)
      BN_LAUNCH(k_sym_long, h[1], 256, 0, s, A.ia.p, A.ja.p, A.val.p, T.ia.p, T.ja.p, T.val.p,
                longs.p, out.val.p, flags.p);
    if (!h[0] && h[1] > 0) h[0] = read_scalar(flags.p, s);
    if (!h[0]) {
      BN_CUDA(cudaMemcpyAsync(out.ia.p, A.ia.p, sizeof(int) * ((size_t)n + 1),
                              cudaMemcpyDeviceToDevice, s));
      BN_CUDA(cudaMemcpyAsync(out.ja.p, A.ja.p, sizeof(int) * (size_t)A.nnz,
                              cudaMemcpyDeviceToDevice, s));
      return;
    }
    out = CSR();
  }
  add_scaled(A, T, 0.5, out, s);
}

// ------------------------------------------------------------------ validation
// flags: bit0 bad row pointer, bit1 column out of range, bit2 duplicate column
__global__ void k_validate(const int* __restrict__ ia, const int* __restrict__ ja, int n, int m,
                           int nnz, int* __restrict__ flags) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    int a0 = ia[i], a1 = ia[i + 1];
    if (a0 < 0 || a1 < a0 || a1 > nnz || (i == 0 && a0 != 0) || (i == n - 1 && a1 != nnz)) {
      atomicOr(flags, 1);
      continue;
    }
    for (int k = a0; k < a1; k++) {
      int c = ja[k];
      if (c < 0 || c >= m) { atomicOr(flags, 2); break; }
      for (int k2 = a0; k2 < k; k2++)
        if (ja[k2] == c) { atomicOr(flags, 4); break; }
    }
  }
}

int validate(const int* ia, const int* ja, int n, int m, int nnz, cudaStream_t s) {
  DBuf<int> f(1, s);
  f.zero();
  if (n > 0) BN_LAUNCH(k_validate, grid_for(n, 128), 128, 0, s, ia, ja, n, m, nnz, f.p);
  return read_scalar(f.p, s);
}

}  // namespace bn
