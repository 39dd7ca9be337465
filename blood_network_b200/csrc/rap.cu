// Galerkin coarse operator Ac = R A P (R = P^T) as a two-pass SpGEMM with
// hash accumulators: pass 1 counts the distinct columns of every coarse row,
// a scan sizes Ac, pass 2 fills it.
//
// Bit-exact with dcsr_rap (C_amg1/src/sparse_ops.c:102-213).  The reference
// walks R row ic, then A row i1, then P row i2 in storage order, forms
// (r * a) * p and accumulates in that order; row ic starts with its diagonal
// (value 0.0, then accumulated), the other columns follow in order of first
// discovery and start from their first product.
//
// Layout: one warp per coarse row.  Pass 1 inserts the product columns of
// the row into a shared-memory open-addressing table in parallel
// (atomicCAS) and counts the new keys.  Pass 2 keeps the reference's
// sequential order without serialising the memory traffic: the 32 lanes walk
// A row i1 together (coalesced), form r*a, expand their P rows into an
// ordered product stream in shared memory (warp prefix sum), and consume the
// stream 32 products at a time: lanes holding the same column group up
// (match_any) and the group's first lane adds the group's products, in
// stream order, to that column's sum (a new column takes its first product
// and the next slot in order of first appearance), so every sum is formed in
// exactly the reference's order while distinct columns proceed in parallel.
// Rows with at most 64 products use small per-warp tables (many resident
// warps); rows whose column count exceeds the per-warp table use a one-warp
// block with a large dynamic table, and beyond that a table in global
// memory.
#include "internal.cuh"

#include <cub/cub.cuh>

namespace bn {

constexpr int kWarpCap = 1024;    // per-warp table (distinct columns <= 512)
constexpr int kBigCap = 8192;     // one-warp-per-block table (<= 4096)
constexpr int kRapWarps = 4;
constexpr int kBuf = 256;         // product stream chunk

__device__ __forceinline__ unsigned rap_hash(int key, unsigned mask) {
  return ((unsigned)key * 2654435761u >> 7) & mask;
}

struct Table {
  int* keys;
  int* slots;     // fill pass only
  double* vals;   // fill pass only (indexed by slot)
  unsigned mask;
};

__device__ __forceinline__ void table_clear(Table t, int lane) {
  for (unsigned e = lane; e <= t.mask; e += 32) t.keys[e] = -1;
}

// parallel insert; true if this call inserted the key
__device__ __forceinline__ bool table_insert_atomic(Table t, int key) {
  unsigned h = rap_hash(key, t.mask);
  while (true) {
    int prev = atomicCAS(&t.keys[h], -1, key);
    if (prev == -1) return true;
    if (prev == key) return false;
    h = (h + 1) & t.mask;
  }
}

// product-count bound per coarse row: 1 (diagonal) + sum |P_i2| over the
// entries i2 of the A rows i1 of R's row, computed as 1 + sum_{i1} w_{i1}
// with w_{i1} = sum_{i2 in A_{i1}} |P_{i2}| (one pass over A, one over R)
__global__ void k_fine_weights(const int* __restrict__ aia, const int* __restrict__ aja,
                               const int* __restrict__ pia, int n, long long* __restrict__ w) {
  const int lane = threadIdx.x & 31;
  const int warps = (gridDim.x * blockDim.x) >> 5;
  for (int i1 = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i1 < n; i1 += warps) {
    long long b = 0;
    for (int k2 = aia[i1] + lane; k2 < aia[i1 + 1]; k2 += 32) {
      const int i2 = aja[k2];
      b += pia[i2 + 1] - pia[i2];
    }
    for (int off = 16; off > 0; off >>= 1) b += __shfl_xor_sync(0xffffffffu, b, off);
    if (lane == 0) w[i1] = b;
  }
}

__global__ void k_rap_bound_w(const int* __restrict__ ria, const int* __restrict__ rja,
                              const long long* __restrict__ w, int nc, long long* __restrict__ ub) {
  const int lane = threadIdx.x & 31;
  const int warps = (gridDim.x * blockDim.x) >> 5;
  for (int ic = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; ic < nc; ic += warps) {
    long long b = 0;
    for (int k1 = ria[ic] + lane; k1 < ria[ic + 1]; k1 += 32) b += w[rja[k1]];
    for (int off = 16; off > 0; off >>= 1) b += __shfl_xor_sync(0xffffffffu, b, off);
    if (lane == 0) ub[ic] = 1 + b;
  }
}

__global__ void k_rap_bound(const int* __restrict__ ria, const int* __restrict__ rja,
                            const int* __restrict__ aia, const int* __restrict__ aja,
                            const int* __restrict__ pia, int nc, long long* __restrict__ ub) {
  const int lane = threadIdx.x & 31;
  const int warps = (gridDim.x * blockDim.x) >> 5;
  for (int ic = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; ic < nc; ic += warps) {
    long long b = 0;
    for (int k1 = ria[ic]; k1 < ria[ic + 1]; k1++) {
      int i1 = rja[k1];
      for (int k2 = aia[i1] + lane; k2 < aia[i1 + 1]; k2 += 32) {
        int i2 = aja[k2];
        b += pia[i2 + 1] - pia[i2];
      }
    }
    for (int off = 16; off > 0; off >>= 1) b += __shfl_xor_sync(0xffffffffu, b, off);
    if (lane == 0) ub[ic] = 1 + b;
  }
}

__device__ int rap_count_row(int ic, Table t, int lane, const int* __restrict__ ria,
                             const int* __restrict__ rja, const int* __restrict__ aia,
                             const int* __restrict__ aja, const int* __restrict__ pia,
                             const int* __restrict__ pja) {
  table_clear(t, lane);
  __syncwarp();
  int cnt = 0;
  if (lane == 0) cnt += table_insert_atomic(t, ic);
  for (int k1 = ria[ic]; k1 < ria[ic + 1]; k1++) {
    const int i1 = rja[k1];
    for (int k2 = aia[i1] + lane; k2 < aia[i1 + 1]; k2 += 32) {
      const int i2 = aja[k2];
      for (int k3 = pia[i2]; k3 < pia[i2 + 1]; k3++) cnt += table_insert_atomic(t, pja[k3]);
    }
  }
  for (int off = 16; off > 0; off >>= 1) cnt += __shfl_xor_sync(0xffffffffu, cnt, off);
  __syncwarp();
  return cnt;
}

// read-only probe: slot of key, or -1
__device__ __forceinline__ int table_find_slot(Table t, int key) {
  unsigned h = rap_hash(key, t.mask);
  while (true) {
    const int k = t.keys[h];
    if (k == key) return t.slots[h];
    if (k == -1) return -1;
    h = (h + 1) & t.mask;
  }
}
// insert a key known to be absent (lanes insert distinct keys concurrently)
__device__ __forceinline__ void table_put(Table t, int key, int slot) {
  unsigned h = rap_hash(key, t.mask);
  while (true) {
    if (atomicCAS(&t.keys[h], -1, key) == -1) {
      t.slots[h] = slot;
      return;
    }
    h = (h + 1) & t.mask;
  }
}

template <int BUF = kBuf>
__device__ void rap_fill_row(int ic, Table t, int lane, int* bcol, double* bval,
                             const int* __restrict__ ria, const int* __restrict__ rja,
                             const double* __restrict__ rval, const int* __restrict__ aia,
                             const int* __restrict__ aja, const double* __restrict__ aval,
                             const int* __restrict__ pia, const int* __restrict__ pja,
                             const double* __restrict__ pval, int cbase, int* __restrict__ cja,
                             double* __restrict__ cval) {
  table_clear(t, lane);
  __syncwarp();
  if (lane == 0) {
    table_put(t, ic, 0);
    t.vals[0] = 0.0;
    cja[cbase] = ic;
  }
  __syncwarp();
  int nslots = 1;  // warp-uniform
  const unsigned lt = (1u << lane) - 1u;
  for (int k1 = ria[ic]; k1 < ria[ic + 1]; k1++) {
    const double r = rval[k1];
    const int i1 = rja[k1];
    const int a1 = aia[i1 + 1];
    for (int base = aia[i1]; base < a1; base += 32) {
      const int k2 = base + lane;
      double ra = 0.0;
      int p0 = 0, plen = 0;
      if (k2 < a1) {
        ra = xmul(r, aval[k2]);
        const int i2 = aja[k2];
        p0 = pia[i2];
        plen = pia[i2 + 1] - p0;
      }
      // exclusive prefix of plen across the warp (stream positions)
      int incl = plen;
      for (int off = 1; off < 32; off <<= 1) {
        int v = __shfl_up_sync(0xffffffffu, incl, off);
        if (lane >= off) incl += v;
      }
      const int total = __shfl_sync(0xffffffffu, incl, 31);
      const int start = incl - plen;
      (void)lt;
      for (int cs = 0; cs < total; cs += BUF) {
        for (int q = 0; q < plen; q++) {
          const int sidx = start + q - cs;
          if (sidx >= 0 && sidx < BUF) {
            bcol[sidx] = pja[p0 + q];
            bval[sidx] = xmul(ra, pval[p0 + q]);
          }
        }
        __syncwarp();
        // consume the stream in order, 32 products at a time: lanes holding
        // the same column form a group whose lowest lane adds the group's
        // products to that column's sum in stream order (a new column takes
        // its first product and the next slot, numbered in order of first
        // appearance); distinct columns proceed in parallel
        const int m = min(BUF, total - cs);
        for (int q0 = 0; q0 < m; q0 += 32) {
          const int q = q0 + lane;
          const bool act = q < m;
          const int col = act ? bcol[q] : -1 - lane;
          const unsigned grp = __match_any_sync(0xffffffffu, col);
          const bool lead = act && (__ffs(grp) - 1 == lane);
          int slot = lead ? table_find_slot(t, col) : 0;
          const unsigned newm = __ballot_sync(0xffffffffu, lead && slot < 0);
          if (lead) {
            double acc;
            unsigned g = grp;
            if (slot < 0) {
              slot = nslots + __popc(newm & lt);
              table_put(t, col, slot);
              cja[cbase + slot] = col;
              acc = bval[q];
              g &= g - 1;
            } else {
              acc = t.vals[slot];
            }
            for (; g; g &= g - 1) acc = xadd(acc, bval[q0 + __ffs(g) - 1]);
            t.vals[slot] = acc;
          }
          nslots += __popc(newm);
          __syncwarp();
        }
      }
    }
  }
  for (int q = lane; q < nslots; q += 32) cval[cbase + q] = t.vals[q];
  __syncwarp();
}

// ---------------- small rows (at most kSmallCap/2 products): small tables
// and stream buffers, so that many more warps per SM hide the latency of the
// R -> A -> P walk (the fine and first coarse levels are almost all small)
constexpr int kSmallCap = 128;
constexpr int kSmallBuf = 64;
constexpr int kSmallWarps = 8;

__global__ void __launch_bounds__(32 * kSmallWarps)
k_rap_count_small(const int* __restrict__ ria, const int* __restrict__ rja,
                  const int* __restrict__ aia, const int* __restrict__ aja,
                  const int* __restrict__ pia, const int* __restrict__ pja,
                  const int* __restrict__ rows, int m, int* __restrict__ cnt_out) {
  __shared__ int keys_s[kSmallWarps][kSmallCap];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  Table t{keys_s[w], nullptr, nullptr, kSmallCap - 1};
  for (int q = blockIdx.x * kSmallWarps + w; q < m; q += gridDim.x * kSmallWarps) {
    const int ic = rows[q];
    int c = rap_count_row(ic, t, lane, ria, rja, aia, aja, pia, pja);
    if (lane == 0) cnt_out[ic] = c;
  }
}

__global__ void __launch_bounds__(32 * kSmallWarps)
k_rap_fill_small(const int* __restrict__ ria, const int* __restrict__ rja,
                 const double* __restrict__ rval, const int* __restrict__ aia,
                 const int* __restrict__ aja, const double* __restrict__ aval,
                 const int* __restrict__ pia, const int* __restrict__ pja,
                 const double* __restrict__ pval, const int* __restrict__ rows, int m,
                 const int* __restrict__ cia, int* __restrict__ cja, double* __restrict__ cval) {
  __shared__ double vals_s[kSmallWarps][kSmallCap / 2];
  __shared__ double bval_s[kSmallWarps][kSmallBuf];
  __shared__ int keys_s[kSmallWarps][kSmallCap];
  __shared__ int slots_s[kSmallWarps][kSmallCap];
  __shared__ int bcol_s[kSmallWarps][kSmallBuf];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  Table t{keys_s[w], slots_s[w], vals_s[w], kSmallCap - 1};
  for (int q = blockIdx.x * kSmallWarps + w; q < m; q += gridDim.x * kSmallWarps) {
    const int ic = rows[q];
    rap_fill_row<kSmallBuf>(ic, t, lane, bcol_s[w], bval_s[w], ria, rja, rval, aia, aja, aval,
                            pia, pja, pval, cia[ic], cja, cval);
  }
}

// ---------------- pass 1 kernels
// class 0: per-warp shared table; class 1: one warp per block, big table;
// class 2: global table (toff gives each listed row's table offset)
__global__ void __launch_bounds__(32 * kRapWarps)
k_rap_count_warp(const int* __restrict__ ria, const int* __restrict__ rja,
                 const int* __restrict__ aia, const int* __restrict__ aja,
                 const int* __restrict__ pia, const int* __restrict__ pja,
                 const int* __restrict__ rows, int m, int* __restrict__ cnt_out) {
  __shared__ int keys_s[kRapWarps][kWarpCap];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  Table t{keys_s[w], nullptr, nullptr, kWarpCap - 1};
  for (int q = blockIdx.x * kRapWarps + w; q < m; q += gridDim.x * kRapWarps) {
    const int ic = rows[q];
    int c = rap_count_row(ic, t, lane, ria, rja, aia, aja, pia, pja);
    if (lane == 0) cnt_out[ic] = c;
  }
}

__global__ void __launch_bounds__(32)
k_rap_count_big(const int* __restrict__ ria, const int* __restrict__ rja,
                const int* __restrict__ aia, const int* __restrict__ aja,
                const int* __restrict__ pia, const int* __restrict__ pja,
                const int* __restrict__ rows, int m, int* __restrict__ cnt_out) {
  extern __shared__ int dyn[];
  const int lane = threadIdx.x & 31;
  Table t{dyn, nullptr, nullptr, kBigCap - 1};
  for (int q = blockIdx.x; q < m; q += gridDim.x) {
    const int ic = rows[q];
    int c = rap_count_row(ic, t, lane, ria, rja, aia, aja, pia, pja);
    if (lane == 0) cnt_out[ic] = c;
  }
}

__global__ void k_rap_count_huge(const int* __restrict__ ria, const int* __restrict__ rja,
                                 const int* __restrict__ aia, const int* __restrict__ aja,
                                 const int* __restrict__ pia, const int* __restrict__ pja,
                                 const int* __restrict__ rows, int m,
                                 const long long* __restrict__ toff, int* __restrict__ gkeys,
                                 int* __restrict__ cnt_out) {
  const int lane = threadIdx.x & 31;
  const int warps = (gridDim.x * blockDim.x) >> 5;
  for (int q = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; q < m; q += warps) {
    const int ic = rows[q];
    const long long off = toff[q];
    Table t{gkeys + off, nullptr, nullptr, (unsigned)(toff[q + 1] - off) - 1};
    int c = rap_count_row(ic, t, lane, ria, rja, aia, aja, pia, pja);
    if (lane == 0) cnt_out[ic] = c;
  }
}

// ---------------- pass 2 kernels
constexpr size_t kWarpFillSmem =
    kRapWarps * (kWarpCap * 2 * sizeof(int) + (kWarpCap / 2) * sizeof(double) +
                 kBuf * (sizeof(int) + sizeof(double)));
constexpr size_t kBigFillSmem =
    kBigCap * 2 * sizeof(int) + (kBigCap / 2) * sizeof(double) + kBuf * (sizeof(int) + sizeof(double));
constexpr size_t kBigCountSmem = kBigCap * sizeof(int);

__device__ __forceinline__ void carve(unsigned char* base, int cap, Table* t, int** bcol,
                                      double** bval) {
  double* vals = (double*)base;                       // cap/2 doubles
  double* bv = vals + cap / 2;                        // kBuf doubles
  int* keys = (int*)(bv + kBuf);                      // cap ints
  int* slots = keys + cap;                            // cap ints
  int* bc = slots + cap;                              // kBuf ints
  *t = Table{keys, slots, vals, (unsigned)cap - 1};
  *bcol = bc;
  *bval = bv;
}

__global__ void __launch_bounds__(32 * kRapWarps)
k_rap_fill_warp(const int* __restrict__ ria, const int* __restrict__ rja,
                const double* __restrict__ rval, const int* __restrict__ aia,
                const int* __restrict__ aja, const double* __restrict__ aval,
                const int* __restrict__ pia, const int* __restrict__ pja,
                const double* __restrict__ pval, const int* __restrict__ rows, int m,
                const int* __restrict__ cia, int* __restrict__ cja, double* __restrict__ cval) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  Table t;
  int* bcol;
  double* bval;
  carve(smem + w * (kWarpFillSmem / kRapWarps), kWarpCap, &t, &bcol, &bval);
  for (int q = blockIdx.x * kRapWarps + w; q < m; q += gridDim.x * kRapWarps) {
    const int ic = rows[q];
    rap_fill_row(ic, t, lane, bcol, bval, ria, rja, rval, aia, aja, aval, pia, pja, pval, cia[ic],
                 cja, cval);
  }
}

__global__ void __launch_bounds__(32)
k_rap_fill_big(const int* __restrict__ ria, const int* __restrict__ rja,
               const double* __restrict__ rval, const int* __restrict__ aia,
               const int* __restrict__ aja, const double* __restrict__ aval,
               const int* __restrict__ pia, const int* __restrict__ pja,
               const double* __restrict__ pval, const int* __restrict__ rows, int m,
               const int* __restrict__ cia, int* __restrict__ cja, double* __restrict__ cval) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int lane = threadIdx.x & 31;
  Table t;
  int* bcol;
  double* bval;
  carve(smem, kBigCap, &t, &bcol, &bval);
  for (int q = blockIdx.x; q < m; q += gridDim.x) {
    const int ic = rows[q];
    rap_fill_row(ic, t, lane, bcol, bval, ria, rja, rval, aia, aja, aval, pia, pja, pval, cia[ic],
                 cja, cval);
  }
}

__global__ void k_rap_fill_huge(const int* __restrict__ ria, const int* __restrict__ rja,
                                const double* __restrict__ rval, const int* __restrict__ aia,
                                const int* __restrict__ aja, const double* __restrict__ aval,
                                const int* __restrict__ pia, const int* __restrict__ pja,
                                const double* __restrict__ pval, const int* __restrict__ rows,
                                int m, const long long* __restrict__ toff,
                                int* __restrict__ gkeys, int* __restrict__ gslots,
                                double* __restrict__ gvals, int* __restrict__ gbcol,
                                double* __restrict__ gbval, const int* __restrict__ cia,
                                int* __restrict__ cja, double* __restrict__ cval) {
  const int lane = threadIdx.x & 31;
  const int wid = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int warps = (gridDim.x * blockDim.x) >> 5;
  int* bcol = gbcol + (size_t)wid * kBuf;
  double* bval = gbval + (size_t)wid * kBuf;
  for (int q = wid; q < m; q += warps) {
    const int ic = rows[q];
    const long long off = toff[q];
    const unsigned cap = (unsigned)(toff[q + 1] - off);
    Table t{gkeys + off, gslots + off, gvals + off / 2, cap - 1};
    rap_fill_row(ic, t, lane, bcol, bval, ria, rja, rval, aia, aja, aval, pia, pja, pval, cia[ic],
                 cja, cval);
  }
}

// ---------------- hub rows: sort-based fill
// For rows with more than kSortProducts products the single-lane consumer
// above would serialise too much work.  Their ordered product streams are
// written out in full -- a (column, 0.0) seed for the diagonal first, then
// every (r*a)*p in the reference's order -- sorted stably by (row, column),
// so the products of one column stay in stream order; one thread per column
// then sums them in that order (the first product assigned, the rest added,
// exactly as the reference), and the columns are put back in order of first
// appearance, which places the diagonal first.
constexpr long long kSortProducts = 16384;
constexpr long long kLongSeg = 256;  // segments longer than this are summed by a warp

// products per (hub row, R entry) pair: sum over A row i1 of |P_i2|
__global__ void k_pair_counts(const int* __restrict__ ria, const int* __restrict__ rja,
                              const int* __restrict__ aia, const int* __restrict__ aja,
                              const int* __restrict__ pia, const int* __restrict__ pair_row,
                              const int* __restrict__ pair_k1, long long npairs,
                              long long* __restrict__ cnt) {
  const int lane = threadIdx.x & 31;
  const long long warps = ((long long)gridDim.x * blockDim.x) >> 5;
  for (long long p = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; p < npairs;
       p += warps) {
    const int k1 = pair_k1[p];
    if (k1 < 0) {  // diagonal seed slot
      if (lane == 0) cnt[p] = 1;
      continue;
    }
    const int i1 = rja[k1];
    long long c = 0;
    for (int k2 = aia[i1] + lane; k2 < aia[i1 + 1]; k2 += 32) {
      const int i2 = aja[k2];
      c += pia[i2 + 1] - pia[i2];
    }
    for (int off = 16; off > 0; off >>= 1) c += __shfl_xor_sync(0xffffffffu, c, off);
    if (lane == 0) cnt[p] = c;
  }
}

// list the (row, k1) pairs of the hub rows: row q owns pairs
// [pstart[q], pstart[q+1]) and one extra leading slot for its diagonal seed
__global__ void k_pairs(const int* __restrict__ ria, const int* __restrict__ rows, int m,
                        const long long* __restrict__ pstart, int* __restrict__ pair_row,
                        int* __restrict__ pair_k1) {
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < m; q += gridDim.x * blockDim.x) {
    const int ic = rows[q];
    long long p = pstart[q];
    pair_row[p] = q;   // seed slot
    pair_k1[p] = -1;
    p++;
    for (int k1 = ria[ic]; k1 < ria[ic + 1]; k1++, p++) {
      pair_row[p] = q;
      pair_k1[p] = k1;
    }
  }
}

// warp per pair: write the pair's products at its stream offset, in order
__global__ void k_rap_gen_stream(const int* __restrict__ rja, const double* __restrict__ rval,
                                 const int* __restrict__ aia, const int* __restrict__ aja,
                                 const double* __restrict__ aval, const int* __restrict__ pia,
                                 const int* __restrict__ pja, const double* __restrict__ pval,
                                 const int* __restrict__ rows, const int* __restrict__ pair_row,
                                 const int* __restrict__ pair_k1, long long npairs,
                                 const long long* __restrict__ poff,
                                 unsigned long long* __restrict__ keys,
                                 long long* __restrict__ idx, double* __restrict__ vals) {
  const int lane = threadIdx.x & 31;
  const long long warps = ((long long)gridDim.x * blockDim.x) >> 5;
  for (long long pr = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; pr < npairs;
       pr += warps) {
    const int q = pair_row[pr];
    const unsigned long long hi = (unsigned long long)q << 32;
    long long pos = poff[pr];
    const int k1 = pair_k1[pr];
    if (k1 < 0) {  // diagonal seed: value 0.0 ahead of every product
      if (lane == 0) {
        keys[pos] = hi | (unsigned)rows[q];
        idx[pos] = pos;
        vals[pos] = 0.0;
      }
      continue;
    }
    const double r = rval[k1];
    const int i1 = rja[k1];
    const int a1 = aia[i1 + 1];
    for (int base = aia[i1]; base < a1; base += 32) {
      const int k2 = base + lane;
      double ra = 0.0;
      int p0 = 0, plen = 0;
      if (k2 < a1) {
        ra = xmul(r, aval[k2]);
        const int i2 = aja[k2];
        p0 = pia[i2];
        plen = pia[i2 + 1] - p0;
      }
      int incl = plen;
      for (int off = 1; off < 32; off <<= 1) {
        int v = __shfl_up_sync(0xffffffffu, incl, off);
        if (lane >= off) incl += v;
      }
      const int total = __shfl_sync(0xffffffffu, incl, 31);
      const long long o = pos + incl - plen;
      for (int q3 = 0; q3 < plen; q3++) {
        keys[o + q3] = hi | (unsigned)pja[p0 + q3];
        idx[o + q3] = o + q3;
        vals[o + q3] = xmul(ra, pval[p0 + q3]);
      }
      pos += total;
    }
  }
}

__global__ void k_seed_counts(long long* __restrict__ cnt, const int* __restrict__ pair_k1,
                              long long npairs) {
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < npairs;
       p += (long long)gridDim.x * blockDim.x)
    if (pair_k1[p] < 0) cnt[p] = 1;
}

// per hub row: number of column segments (= distinct columns)
__global__ void k_seg_row_counts(const unsigned long long* __restrict__ keys,
                                 const long long* __restrict__ seg, long long nseg,
                                 const int* __restrict__ rows, int* __restrict__ cnt_out) {
  for (long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x; g < nseg;
       g += (long long)gridDim.x * blockDim.x) {
    const int q = (int)(keys[seg[g]] >> 32);
    atomicAdd(&cnt_out[rows[q]], 1);
  }
}

__global__ void k_seg_heads(const unsigned long long* __restrict__ keys, long long T,
                            unsigned char* __restrict__ head) {
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < T;
       p += (long long)gridDim.x * blockDim.x)
    head[p] = (p == 0 || keys[p] != keys[p - 1]) ? 1 : 0;
}

__global__ void k_iota64(long long* __restrict__ a, long long T) {
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < T;
       p += (long long)gridDim.x * blockDim.x)
    a[p] = p;
}

// one thread per column segment: ordered sum; key for reordering = first
// stream position of the column
__global__ void k_gather_sorted(const long long* __restrict__ idx, long long T,
                                const double* __restrict__ vals, double* __restrict__ out) {
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < T;
       p += (long long)gridDim.x * blockDim.x)
    out[p] = vals[idx[p]];
}

// svals: the products in sorted order (contiguous per column, stream order)
__global__ void k_seg_sum(const unsigned long long* __restrict__ keys,
                          const long long* __restrict__ idx, const double* __restrict__ svals,
                          const long long* __restrict__ seg, long long nseg, long long T,
                          double* __restrict__ sval, int* __restrict__ scol,
                          long long* __restrict__ sfirst) {
  for (long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x; g < nseg;
       g += (long long)gridDim.x * blockDim.x) {
    const long long b = seg[g], e = (g + 1 < nseg) ? seg[g + 1] : T;
    if (e - b > kLongSeg) continue;  // k_seg_sum_long
    double v = svals[b];
#pragma unroll 8
    for (long long p = b + 1; p < e; p++) v = xadd(v, svals[p]);
    sval[g] = v;
    scol[g] = (int)(keys[b] & 0xffffffffull);
    sfirst[g] = idx[b];
  }
}

// long segments, one warp each: the warp loads the next kSegChunk products
// (coalesced, into registers) while lane 0 adds the current chunk from
// shared memory in stream order; the loads' latency hides behind the adds.
constexpr int kSegChunk = 256;
__global__ void __launch_bounds__(32)
k_seg_sum_long(const unsigned long long* __restrict__ keys, const long long* __restrict__ idx,
               const double* __restrict__ svals, const long long* __restrict__ seg,
               long long nseg, long long T, const long long* __restrict__ lsegs, int nl,
               double* __restrict__ sval, int* __restrict__ scol,
               long long* __restrict__ sfirst) {
  __shared__ double buf[2][kSegChunk];
  const int lane = threadIdx.x;
  constexpr int kPer = kSegChunk / 32;
  for (int w = blockIdx.x; w < nl; w += gridDim.x) {
    const long long g = lsegs[w];
    const long long b = seg[g], e = (g + 1 < nseg) ? seg[g + 1] : T;
    double x[kPer];
#pragma unroll
    for (int r = 0; r < kPer; r++) {
      const long long q = b + r * 32 + lane;
      x[r] = q < e ? svals[q] : 0.0;
    }
#pragma unroll
    for (int r = 0; r < kPer; r++) buf[0][r * 32 + lane] = x[r];
    __syncwarp();
    double v = 0.0;
    int slot = 0;
    for (long long p0 = b; p0 < e; p0 += kSegChunk) {
      const long long pn = p0 + kSegChunk;
      if (pn < e) {
#pragma unroll
        for (int r = 0; r < kPer; r++) {
          const long long q = pn + r * 32 + lane;
          x[r] = q < e ? svals[q] : 0.0;
        }
      }
      if (lane == 0) {
        const int cnt = e - p0 < kSegChunk ? (int)(e - p0) : kSegChunk;
        int q0 = 0;
        if (p0 == b) { v = buf[slot][0]; q0 = 1; }
#pragma unroll 8
        for (int q = q0; q < cnt; q++) v = xadd(v, buf[slot][q]);
      }
      __syncwarp();
      if (pn < e) {
#pragma unroll
        for (int r = 0; r < kPer; r++) buf[slot ^ 1][r * 32 + lane] = x[r];
      }
      __syncwarp();
      slot ^= 1;
    }
    if (lane == 0) {
      sval[g] = v;
      scol[g] = (int)(keys[b] & 0xffffffffull);
      sfirst[g] = idx[b];
    }
    __syncwarp();
  }
}

__global__ void k_long_segs(const long long* __restrict__ seg, long long nseg, long long T,
                            long long* __restrict__ out, int* counter) {
  for (long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x; g < nseg;
       g += (long long)gridDim.x * blockDim.x) {
    const long long e = (g + 1 < nseg) ? seg[g + 1] : T;
    if (e - seg[g] > kLongSeg) out[atomicAdd(counter, 1)] = g;
    atomicMax(counter + 1, (int)(e - seg[g] < 0x7fffffff ? e - seg[g] : 0x7fffffff));
  }
}

// write the reordered columns of each hub row
__global__ void k_seg_write(const long long* __restrict__ order, long long nseg,
                            const unsigned long long* __restrict__ seg_key_row,
                            const double* __restrict__ sval, const int* __restrict__ scol,
                            const int* __restrict__ rows, const long long* __restrict__ rowseg,
                            const int* __restrict__ cia, int* __restrict__ cja,
                            double* __restrict__ cval) {
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < nseg;
       t += (long long)gridDim.x * blockDim.x) {
    const long long g = order[t];
    const int q = (int)(seg_key_row[g] >> 32);
    const int ic = rows[q];
    const long long rank = t - rowseg[q];
    cja[cia[ic] + rank] = scol[g];
    cval[cia[ic] + rank] = sval[g];
  }
}

__global__ void k_seg_rowkeys(const unsigned long long* __restrict__ keys,
                              const long long* __restrict__ seg, long long nseg,
                              unsigned long long* __restrict__ out) {
  for (long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x; g < nseg;
       g += (long long)gridDim.x * blockDim.x)
    out[g] = keys[seg[g]];
}

__global__ void k_rows_count64(const int* __restrict__ rows, int m, const long long* __restrict__ v,
                               long long sub, long long* __restrict__ out) {
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < m; q += gridDim.x * blockDim.x)
    out[q] = v[rows[q]] - sub;
}

__global__ void k_hub_pair_counts(const int* __restrict__ ria, const int* __restrict__ rows, int m,
                                  long long* __restrict__ out) {
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < m; q += gridDim.x * blockDim.x)
    out[q] = 1 + ria[rows[q] + 1] - ria[rows[q]];
}
__global__ void k_zero_rows(const int* __restrict__ rows, int m, int* __restrict__ cnt) {
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < m; q += gridDim.x * blockDim.x)
    cnt[rows[q]] = 0;
}
__global__ void k_rows_seglen(const int* __restrict__ rows, int m, const int* __restrict__ cia,
                              long long* __restrict__ out) {
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < m; q += gridDim.x * blockDim.x)
    out[q] = cia[rows[q] + 1] - cia[rows[q]];
}

struct HubStream {
  int m = 0;
  long long T = 0, nseg = 0;
  DBuf<unsigned long long> keys2;
  DBuf<long long> idx2, seg;
  DBuf<double> vals;
};

// Phase 1 (before the scan): build and sort the streams, count columns.
static void hub_prepare(const CSR& R, const CSR& A, const CSR& P, const int* rows, int m,
                        int* cnt_out, HubStream& H, cudaStream_t s) {
  H.m = m;
  // pairs: per row 1 seed + |R row|
  DBuf<long long> pstart((size_t)m + 1, s);
  pstart.zero();
  BN_LAUNCH(k_hub_pair_counts, grid_for(m, 128), 128, 0, s, R.ia.p, rows, m, pstart.p);
  const long long npairs = scan_counts64(pstart.p, m, s);
  DBuf<int> pair_row(npairs, s), pair_k1(npairs, s);
  BN_LAUNCH(k_pairs, grid_for(m, 128), 128, 0, s, R.ia.p, rows, m, pstart.p, pair_row.p,
            pair_k1.p);
  DBuf<long long> poff((size_t)npairs + 1, s);
  poff.zero();
  BN_LAUNCH(k_pair_counts, grid_for(npairs * 32, 256), 256, 0, s, R.ia.p, R.ja.p, A.ia.p, A.ja.p,
            P.ia.p, pair_row.p, pair_k1.p, npairs, poff.p);
  H.T = scan_counts64(poff.p, (int)npairs, s);
  const long long T = H.T;
  DBuf<unsigned long long> keys(T, s);
  DBuf<long long> idx(T, s);
  H.keys2.alloc(T, s);
  H.idx2.alloc(T, s);
  H.vals.alloc(T, s);
  BN_LAUNCH(k_rap_gen_stream, grid_for(npairs * 32, 256), 256, 0, s, R.ja.p, R.val.p, A.ia.p,
            A.ja.p, A.val.p, P.ia.p, P.ja.p, P.val.p, rows, pair_row.p, pair_k1.p, npairs, poff.p,
            keys.p, idx.p, H.vals.p);
  int eb = 33;
  while ((1LL << (eb - 32)) < (long long)m) eb++;
  size_t tmp = 0;
  BN_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tmp, keys.p, H.keys2.p, idx.p, H.idx2.p, T, 0,
                                          eb, s));
  DBuf<unsigned char> tb(tmp, s);
  BN_CUDA(cub::DeviceRadixSort::SortPairs(tb.p, tmp, keys.p, H.keys2.p, idx.p, H.idx2.p, T, 0, eb,
                                          s));
  DBuf<unsigned char> head(T, s);
  DBuf<long long> iota(T, s), nsel(1, s);
  H.seg.alloc(T, s);
  BN_LAUNCH(k_seg_heads, grid_for(T, 256), 256, 0, s, H.keys2.p, T, head.p);
  BN_LAUNCH(k_iota64, grid_for(T, 256), 256, 0, s, iota.p, T);
  tmp = 0;
  BN_CUDA(cub::DeviceSelect::Flagged(nullptr, tmp, iota.p, head.p, H.seg.p, nsel.p, T, s));
  DBuf<unsigned char> tb2(tmp, s);
  BN_CUDA(cub::DeviceSelect::Flagged(tb2.p, tmp, iota.p, head.p, H.seg.p, nsel.p, T, s));
  H.nseg = read_scalar(nsel.p, s);
  BN_LAUNCH(k_zero_rows, grid_for(m, 128), 128, 0, s, rows, m, cnt_out);
  BN_LAUNCH(k_seg_row_counts, grid_for(H.nseg, 256), 256, 0, s, H.keys2.p, H.seg.p, H.nseg, rows,
            cnt_out);
}

// Phase 2 (after the scan): ordered sums, reorder by first position, write.
static void hub_finish(const int* rows, HubStream& H, CSR& Ac, cudaStream_t s) {
  const long long nseg = H.nseg, T = H.T;
  const int m = H.m;
  if (trace_on())
    fprintf(stderr, "[bn]     hub rows %d products %lld columns %lld\n", m, T, nseg);
  Phase ph1("hub sums", s);
  DBuf<long long> rowseg((size_t)m + 1, s);
  rowseg.zero();
  BN_LAUNCH(k_rows_seglen, grid_for(m, 128), 128, 0, s, rows, m, Ac.ia.p, rowseg.p);
  scan_counts64(rowseg.p, m, s);
  DBuf<double> sval(nseg, s);
  DBuf<int> scol(nseg, s);
  DBuf<long long> sfirst(nseg, s), sfirst2(nseg, s), g_in(nseg, s), g_out(nseg, s);
  DBuf<unsigned long long> srow(nseg, s);
  DBuf<double> svals(T, s);
  BN_LAUNCH(k_gather_sorted, grid_for(T, 256), 256, 0, s, H.idx2.p, T, H.vals.p, svals.p);
  BN_LAUNCH(k_seg_sum, grid_for(nseg, 128), 128, 0, s, H.keys2.p, H.idx2.p, svals.p, H.seg.p,
            nseg, T, sval.p, scol.p, sfirst.p);
  {
    DBuf<long long> lsegs(nseg, s);
    DBuf<int> lc(2, s);
    lc.zero();
    BN_LAUNCH(k_long_segs, grid_for(nseg, 256), 256, 0, s, H.seg.p, nseg, T, lsegs.p, lc.p);
    const int nl = read_scalar(lc.p, s);
    if (trace_on())
      fprintf(stderr, "[bn]     hub columns over %lld products: %d, longest %d\n", kLongSeg, nl,
              read_scalar(lc.p + 1, s));
    if (nl > 0)
      BN_LAUNCH(k_seg_sum_long, nl < 32768 ? nl : 32768, 32, 0, s, H.keys2.p, H.idx2.p, svals.p,
                H.seg.p, nseg, T, lsegs.p, nl, sval.p, scol.p, sfirst.p);
  }
  ph1.done();
  Phase ph2("hub reorder+write", s);
  BN_LAUNCH(k_seg_rowkeys, grid_for(nseg, 256), 256, 0, s, H.keys2.p, H.seg.p, nseg, srow.p);
  BN_LAUNCH(k_iota64, grid_for(nseg, 256), 256, 0, s, g_in.p, nseg);
  int fb = 1;
  while ((1LL << fb) <= T) fb++;
  size_t tmp = 0;
  BN_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tmp, sfirst.p, sfirst2.p, g_in.p, g_out.p, nseg,
                                          0, fb, s));
  DBuf<unsigned char> tb3(tmp, s);
  BN_CUDA(cub::DeviceRadixSort::SortPairs(tb3.p, tmp, sfirst.p, sfirst2.p, g_in.p, g_out.p, nseg,
                                          0, fb, s));
  BN_LAUNCH(k_seg_write, grid_for(nseg, 256), 256, 0, s, g_out.p, nseg, srow.p, sval.p, scol.p,
            rows, rowseg.p, Ac.ia.p, Ac.ja.p, Ac.val.p);
}

// ---------------- classification helpers
// class by a size estimate: 3 (<= kSmallCap/2), 0 (<= kWarpCap/2),
// 1 (<= kBigCap/2), 2 (beyond)
__global__ void k_rap_classify(const long long* __restrict__ est, int nc, int cap_limit,
                               int* __restrict__ lists, int* __restrict__ counts) {
  // warp-aggregated appends: one atomic per class present in the warp
  const int lane = threadIdx.x & 31;
  const int stride = gridDim.x * blockDim.x;
  for (int base = blockIdx.x * blockDim.x; base < nc; base += stride) {
    const int ic = base + threadIdx.x;
    int c = -1;
    if (ic < nc) {
      long long e = est[ic];
      if (e >= 0) {  // e < 0: handled elsewhere
        if (e > cap_limit) e = cap_limit;
        c = e <= kSmallCap / 2 ? 3 : (e <= kWarpCap / 2 ? 0 : (e <= kBigCap / 2 ? 1 : 2));
      }
    }
    const unsigned grp = __match_any_sync(0xffffffffu, c);
    const int leader = __ffs(grp) - 1;
    int pos0 = 0;
    if (lane == leader && c >= 0) pos0 = atomicAdd(&counts[c], __popc(grp));
    pos0 = __shfl_sync(0xffffffffu, pos0, leader);
    if (c >= 0) lists[(size_t)c * nc + pos0 + __popc(grp & ((1u << lane) - 1u))] = ic;
  }
}

__global__ void k_rap_split_hubs(const long long* __restrict__ ub,
                                 const long long* __restrict__ exact, int nc,
                                 long long* __restrict__ est, int* __restrict__ hub, int* nh) {
  for (int ic = blockIdx.x * blockDim.x + threadIdx.x; ic < nc; ic += gridDim.x * blockDim.x) {
    if (ub[ic] > kSortProducts) {
      est[ic] = -1;
      hub[atomicAdd(nh, 1)] = ic;
    } else {
      est[ic] = exact[ic];
    }
  }
}

__global__ void k_rap_huge_caps(const long long* __restrict__ est, const int* __restrict__ rows,
                                int m, int cap_limit, long long* __restrict__ cap) {
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < m; q += gridDim.x * blockDim.x) {
    long long need = est[rows[q]];
    if (need > cap_limit) need = cap_limit;
    need *= 2;
    long long c = 64;
    while (c < need) c <<= 1;
    cap[q] = c;
  }
}

__global__ void k_i32_to_i64(const int* __restrict__ a, int n, long long* __restrict__ b) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    b[i] = a[i];
}

struct RapClasses {
  DBuf<int> lists;  // 4 x nc
  int count[4] = {0, 0, 0, 0};
};

static void classify(const long long* est, int nc, RapClasses& rc, cudaStream_t s) {
  rc.lists.alloc((size_t)4 * (nc > 0 ? nc : 1), s);
  DBuf<int> cnt(4, s);
  cnt.zero();
  if (nc > 0)
    BN_LAUNCH(k_rap_classify, grid_for(nc, 256), 256, 0, s, est, nc, nc, rc.lists.p, cnt.p);
  cnt.download(rc.count, 4);
  BN_CUDA(cudaStreamSynchronize(s));
}

void rap(const CSR& R, const CSR& A, const CSR& P, CSR& Ac, cudaStream_t s) {
  const int nc = R.n;
  BN_CUDA(cudaFuncSetAttribute(k_rap_fill_warp, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)kWarpFillSmem));
  BN_CUDA(cudaFuncSetAttribute(k_rap_fill_big, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)kBigFillSmem));
  BN_CUDA(cudaFuncSetAttribute(k_rap_count_big, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)kBigCountSmem));
  DBuf<long long> ub(nc > 0 ? nc : 1, s), est(nc > 0 ? nc : 1, s);
  DBuf<int> cnt((size_t)nc + 1, s), hub(nc > 0 ? nc : 1, s), nh(1, s);
  cnt.zero();
  nh.zero();
  Phase ph_bound("rap bound", s);
  if (nc > 0) {
    DBuf<long long> w(A.n > 0 ? A.n : 1, s);
    if (A.n > 0)
      BN_LAUNCH(k_fine_weights, grid_for((long long)A.n * 32, 256, 16), 256, 0, s, A.ia.p,
                A.ja.p, P.ia.p, A.n, w.p);
    BN_LAUNCH(k_rap_bound_w, grid_for((long long)nc * 32, 256, 16), 256, 0, s, R.ia.p, R.ja.p,
              w.p, nc, ub.p);
    BN_LAUNCH(k_rap_split_hubs, grid_for(nc, 256), 256, 0, s, ub.p, ub.p, nc, est.p, hub.p, nh.p);
  }
  const int nhub = read_scalar(nh.p, s);
  if (nhub > 1) {  // deterministic hub order
    DBuf<int> t_out(nhub, s);
    size_t tmp = 0;
    BN_CUDA(cub::DeviceRadixSort::SortKeys(nullptr, tmp, hub.p, t_out.p, nhub, 0, 32, s));
    DBuf<unsigned char> t(tmp, s);
    BN_CUDA(cub::DeviceRadixSort::SortKeys(t.p, tmp, hub.p, t_out.p, nhub, 0, 32, s));
    BN_CUDA(cudaMemcpyAsync(hub.p, t_out.p, sizeof(int) * nhub, cudaMemcpyDeviceToDevice, s));
  }
  ph_bound.done();
  HubStream H;
  // ---- pass 1: count; hub rows from their sorted streams, the rest
  // classified by min(bound, nc)
  if (nhub > 0) {
    Phase ph("rap hub streams", s);
    hub_prepare(R, A, P, hub.p, nhub, cnt.p, H, s);
  }
  {
    RapClasses rc;
    classify(est.p, nc, rc, s);
    const int* L0 = rc.lists.p;
    const int* L1 = rc.lists.p + nc;
    const int* L2 = rc.lists.p + 2 * (size_t)nc;
    const int* L3 = rc.lists.p + 3 * (size_t)nc;
    Phase ph("rap count", s);
    if (rc.count[3])
      BN_LAUNCH(k_rap_count_small, grid_for(rc.count[3], kSmallWarps, 64), 32 * kSmallWarps, 0,
                s, R.ia.p, R.ja.p, A.ia.p, A.ja.p, P.ia.p, P.ja.p, L3, rc.count[3], cnt.p);
    if (rc.count[0])
      BN_LAUNCH(k_rap_count_warp, grid_for(rc.count[0], kRapWarps, 64), 32 * kRapWarps, 0, s,
                R.ia.p, R.ja.p, A.ia.p, A.ja.p, P.ia.p, P.ja.p, L0, rc.count[0], cnt.p);
    if (rc.count[1])
      BN_LAUNCH(k_rap_count_big, grid_for(rc.count[1], 1, 16), 32, kBigCountSmem, s, R.ia.p,
                R.ja.p, A.ia.p, A.ja.p, P.ia.p, P.ja.p, L1, rc.count[1], cnt.p);
    if (rc.count[2]) {
      const int m = rc.count[2];
      DBuf<long long> toff((size_t)m + 1, s);
      toff.zero();
      BN_LAUNCH(k_rap_huge_caps, grid_for(m, 128), 128, 0, s, ub.p, L2, m, nc, toff.p);
      long long total = scan_counts64(toff.p, m, s);
      DBuf<int> gkeys((size_t)total, s);
      BN_LAUNCH(k_rap_count_huge, grid_for((long long)m * 32, 128), 128, 0, s, R.ia.p, R.ja.p,
                A.ia.p, A.ja.p, P.ia.p, P.ja.p, L2, m, toff.p, gkeys.p, cnt.p);
    }
  }
  // exact per-row counts (before the scan) drive the fill classes
  DBuf<long long> exact(nc > 0 ? nc : 1, s);
  if (nc > 0) BN_LAUNCH(k_i32_to_i64, grid_for(nc, 256), 256, 0, s, cnt.p, nc, exact.p);
  int nnz = scan_counts(cnt.p, nc, s);
  Ac.n = nc;
  Ac.m = P.m;
  Ac.nnz = nnz;
  Ac.ia = std::move(cnt);
  Ac.ja.alloc((size_t)(nnz > 0 ? nnz : 1), s);
  Ac.val.alloc((size_t)(nnz > 0 ? nnz : 1), s);
  // ---- pass 2: fill
  if (nhub > 0) {
    Phase ph("rap hub fill", s);
    hub_finish(hub.p, H, Ac, s);
  }
  {
    nh.zero();  // the hub list is rebuilt (and no longer needed)
    if (nc > 0)
      BN_LAUNCH(k_rap_split_hubs, grid_for(nc, 256), 256, 0, s, ub.p, exact.p, nc, est.p, hub.p,
                nh.p);
    RapClasses rc;
    classify(est.p, nc, rc, s);
    const int* L0 = rc.lists.p;
    const int* L1 = rc.lists.p + nc;
    const int* L2 = rc.lists.p + 2 * (size_t)nc;
    const int* L3 = rc.lists.p + 3 * (size_t)nc;
    if (trace_on())
      fprintf(stderr, "[bn]     rap fill classes: small %d warp %d big %d huge %d hubs %d\n",
              rc.count[3], rc.count[0], rc.count[1], rc.count[2], nhub);
    Phase ph_w("rap fill warp", s);
    if (rc.count[3])
      BN_LAUNCH(k_rap_fill_small, grid_for(rc.count[3], kSmallWarps, 64), 32 * kSmallWarps, 0, s,
                R.ia.p, R.ja.p, R.val.p, A.ia.p, A.ja.p, A.val.p, P.ia.p, P.ja.p, P.val.p, L3,
                rc.count[3], Ac.ia.p, Ac.ja.p, Ac.val.p);
    if (rc.count[0])
      BN_LAUNCH(k_rap_fill_warp, grid_for(rc.count[0], kRapWarps, 32), 32 * kRapWarps,
                kWarpFillSmem, s, R.ia.p, R.ja.p, R.val.p, A.ia.p, A.ja.p, A.val.p, P.ia.p,
                P.ja.p, P.val.p, L0, rc.count[0], Ac.ia.p, Ac.ja.p, Ac.val.p);
    ph_w.done();
    Phase ph_b("rap fill big", s);
    if (rc.count[1])
      BN_LAUNCH(k_rap_fill_big, grid_for(rc.count[1], 1, 2), 32, kBigFillSmem, s, R.ia.p, R.ja.p,
                R.val.p, A.ia.p, A.ja.p, A.val.p, P.ia.p, P.ja.p, P.val.p, L1, rc.count[1],
                Ac.ia.p, Ac.ja.p, Ac.val.p);
    ph_b.done();
    Phase ph_h("rap fill huge", s);
    if (rc.count[2]) {
      const int m = rc.count[2];
      DBuf<long long> toff((size_t)m + 1, s);
      toff.zero();
      BN_LAUNCH(k_rap_huge_caps, grid_for(m, 128), 128, 0, s, exact.p, L2, m, nc, toff.p);
      long long total = scan_counts64(toff.p, m, s);
      const int grid = grid_for((long long)m * 32, 128);
      const size_t nwarps = (size_t)grid * 4;
      DBuf<int> gkeys((size_t)total, s), gslots((size_t)total, s), gbcol(nwarps * kBuf, s);
      DBuf<double> gvals((size_t)total / 2 + 1, s), gbval(nwarps * kBuf, s);
      BN_LAUNCH(k_rap_fill_huge, grid, 128, 0, s, R.ia.p, R.ja.p, R.val.p, A.ia.p, A.ja.p,
                A.val.p, P.ia.p, P.ja.p, P.val.p, L2, m, toff.p, gkeys.p, gslots.p, gvals.p,
                gbcol.p, gbval.p, Ac.ia.p, Ac.ja.p, Ac.val.p);
    }
  }
}

}  // namespace bn
