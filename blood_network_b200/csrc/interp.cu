// Direct ("standard") interpolation on the device, two passes: count, then
// fill.  Follows rs_standard_interpolation_sparsity / _values
// (C_amg1/src/rs_classical.c:643-694, :703-805):
//   C row i:  P(i, cmap(i)) = 1
//   F row i:  columns = the C points of S_i in S order;
//     diag_hat = a_ii + sum of weak a_im (m not in S_i)
//     num_j    = a_ij                                   j in C_i
//             + sum_{k in S_i, F} a_ik a_kj / sum_{l in C_i} a_kl
//     (a strong F neighbour with |denominator| < 1e-15 is lumped into diag_hat)
//     w_ij = num_j / (-diag_hat)   if |diag_hat| > 1e-15
// Each F row is evaluated by one thread in exactly the reference's operation
// order (A's in-row order, separate multiply/divide/add), so P is
// bit-identical for bit-identical A, S and cf.
#include "internal.cuh"

namespace bn {

__global__ void k_is_c(const int* __restrict__ cf, int n, int* __restrict__ flag) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    flag[i] = (cf[i] == 1);
}

__global__ void k_interp_count(const int* __restrict__ sia, const int* __restrict__ sja,
                               const int* __restrict__ cf, int n, int* __restrict__ cnt) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    int c = 1;
    if (cf[i] != 1) {
      c = 0;
      for (int k = sia[i]; k < sia[i + 1]; k++) c += (cf[sja[k]] == 1);
    }
    cnt[i] = c;
  }
}

__global__ void k_interp_pattern(const int* __restrict__ sia, const int* __restrict__ sja,
                                 const int* __restrict__ cf, const int* __restrict__ cmap, int n,
                                 const int* __restrict__ pia, int* __restrict__ pja) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    int p = pia[i];
    if (cf[i] == 1) {
      pja[p] = cmap[i];
    } else {
      for (int k = sia[i]; k < sia[i + 1]; k++) {
        int j = sja[k];
        if (cf[j] == 1) pja[p++] = cmap[j];
      }
    }
  }
}

// slot of C point j in row i of P (rank among the C points of S_i), or -1
// when j is not in S_i.  *strong reports membership of j in S_i.
__device__ __forceinline__ int strong_slot(const int* __restrict__ sja, int s0, int s1,
                                           const int* __restrict__ cf, int j, bool* strong) {
  int r = 0;
  for (int k = s0; k < s1; k++) {
    int q = sja[k];
    if (q == j) {
      *strong = true;
      return cf[q] == 1 ? r : -1;
    }
    r += (cf[q] == 1);
  }
  *strong = false;
  return -1;
}

// Hub rows of A (longer than kInterpHub entries) get a column -> entry
// index hash table (open addressing, at most half full, so every probe
// sequence ends at an empty slot).  A row whose strong F neighbour is a hub
// then finds the entries of its own strong C points in that row by lookup
// instead of walking the hub's row, and visits them in row order -- the
// same entries, in the same order, as the walk.
constexpr int kInterpHub = 512;
constexpr int kInterpMaxC = 32;  // rows with more strong C points keep the walk

__device__ __forceinline__ unsigned hub_hash(int m) { return (unsigned)m * 2654435761u; }

__global__ void k_hub_mark(const int* __restrict__ aia, int n, int* __restrict__ hubidx,
                           int* __restrict__ hubrows, int* counter) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    int h = -1;
    if (aia[i + 1] - aia[i] > kInterpHub) {
      h = atomicAdd(counter, 1);
      hubrows[h] = i;
    }
    hubidx[i] = h;
  }
}

__global__ void k_hub_size(const int* __restrict__ aia, const int* __restrict__ hubrows, int nh,
                           int* __restrict__ hsz) {
  for (int h = blockIdx.x * blockDim.x + threadIdx.x; h < nh; h += gridDim.x * blockDim.x) {
    const int len = aia[hubrows[h] + 1] - aia[hubrows[h]];
    int sz = 1;
    while (sz < 2 * len) sz <<= 1;
    hsz[h] = sz;
  }
}

__global__ void k_hub_fill(const int* __restrict__ aia, const int* __restrict__ aja,
                           const int* __restrict__ hubrows, const int* __restrict__ hoff,
                           int* __restrict__ keys, int* __restrict__ vals) {
  const int h = blockIdx.x;
  const int i = hubrows[h];
  const int off = hoff[h], mask = hoff[h + 1] - off - 1;
  for (int l = aia[i] + threadIdx.x; l < aia[i + 1]; l += blockDim.x) {
    const int m = aja[l];
    int slot = (int)(hub_hash(m) & (unsigned)mask);
    while (true) {
      const int prev = atomicCAS(&keys[off + slot], -1, m);
      if (prev == -1) { vals[off + slot] = l; break; }
      slot = (slot + 1) & mask;
    }
  }
}

// entry index of column m in hub row h, or -1
__device__ __forceinline__ int hub_find(const int* __restrict__ keys, const int* __restrict__ vals,
                                        const int* __restrict__ hoff, int h, int m) {
  const int off = hoff[h], mask = hoff[h + 1] - off - 1;
  int slot = (int)(hub_hash(m) & (unsigned)mask);
  while (true) {
    const int k = keys[off + slot];
    if (k == m) return vals[off + slot];
    if (k == -1) return -1;
    slot = (slot + 1) & mask;
  }
}

// F rows with more than kWarpRow entries of A (and at most kInterpMaxC
// strong points) are evaluated by a warp.  The operations and their order
// are those of the thread-per-row kernel: the lanes classify A's entries and
// locate the strong C points, one lane adds the weak entries in row order,
// the strong F neighbours are taken from S_i (the same entries of A in the
// same order, S holding A's values), the entries of each neighbour's row
// that lie in C_i are collected in row order and one lane sums the
// denominator in that order; each slot of P's row receives its terms in the
// same sequence as in the thread kernel.
constexpr int kWarpRow = 32;

__device__ __forceinline__ bool warp_row(const int* __restrict__ aia, const int* __restrict__ sia,
                                         int i) {
  return aia[i + 1] - aia[i] > kWarpRow && sia[i + 1] - sia[i] <= kInterpMaxC;
}

__global__ void k_warp_rows(const int* __restrict__ aia, const int* __restrict__ sia,
                            const int* __restrict__ cf, int n, int* __restrict__ list,
                            int* counter) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    if (cf[i] != 1 && warp_row(aia, sia, i)) list[atomicAdd(counter, 1)] = i;
}

constexpr int kInterpWarps = 4;

__global__ void __launch_bounds__(32 * kInterpWarps)
k_interp_values_warp(const int* __restrict__ aia, const int* __restrict__ aja,
                     const double* __restrict__ aval, const int* __restrict__ sia,
                     const int* __restrict__ sja, const double* __restrict__ sval,
                     const int* __restrict__ cf, const int* __restrict__ rows, int m,
                     const int* __restrict__ pia, double* __restrict__ pval,
                     const int* __restrict__ hubidx, const int* __restrict__ hoff,
                     const int* __restrict__ hkeys, const int* __restrict__ hvals) {
  __shared__ int s_col[kInterpWarps][32];   // S_i columns, S order
  __shared__ int s_slot[kInterpWarps][32];  // slot in P's row (C) or -1 (F)
  __shared__ int s_cm[kInterpWarps][32];    // C_i columns by slot
  __shared__ double s_buf[kInterpWarps][32];
  __shared__ double s_af[kInterpWarps][32];  // a_ik of A (not S) for the strong F points
  __shared__ int s_el[kInterpWarps][32], s_sl[kInterpWarps][32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const unsigned lt = (1u << lane) - 1u;
  int* col = s_col[w];
  int* slt = s_slot[w];
  int* cm = s_cm[w];
  double* buf = s_buf[w];
  double* af = s_af[w];
  int* el = s_el[w];
  int* sl = s_sl[w];
  const int warps = (gridDim.x * blockDim.x) >> 5;
  for (int r = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; r < m; r += warps) {
    const int i = rows[r];
    const int p0 = pia[i];
    const int s0 = sia[i], ns = sia[i + 1] - s0;
    // strong points of i and their slots
    int q = -1, isc = 0;
    if (lane < ns) {
      q = sja[s0 + lane];
      isc = (cf[q] == 1);
    }
    const unsigned cmask = __ballot_sync(0xffffffffu, isc);
    const int nc = __popc(cmask);
    if (lane < ns) {
      col[lane] = q;
      slt[lane] = isc ? __popc(cmask & lt) : -1;
      if (isc) cm[__popc(cmask & lt)] = q;
    }
    if (lane < nc) pval[p0 + lane] = 0.0;
    __syncwarp();
    // A_i: diagonal, direct C terms, weak sum (one lane, row order)
    double diag = 0.0, weak = 0.0;
    const int a0 = aia[i], a1 = aia[i + 1];
    for (int base = a0; base < a1; base += 32) {
      const int k = base + lane;
      int cls = 0;  // 0 none, 1 weak, 2 diagonal
      double a = 0.0;
      if (k < a1) {
        const int j = aja[k];
        a = aval[k];
        if (j == i) {
          cls = 2;
        } else {
          int at = -1;
          for (int t = 0; t < ns; t++)
            if (col[t] == j) { at = t; break; }
          if (at < 0) cls = 1;
          else if (slt[at] >= 0) pval[p0 + slt[at]] = xadd(pval[p0 + slt[at]], a);  // once per slot
          else af[at] = a;  // strong F point: its a_ik, from A (a value refresh keeps S's old values)
        }
      }
      const unsigned wm = __ballot_sync(0xffffffffu, cls == 1);
      if (cls == 1) buf[__popc(wm & lt)] = a;
      const unsigned dm = __ballot_sync(0xffffffffu, cls == 2);
      if (dm) diag = __shfl_sync(0xffffffffu, a, __ffs(dm) - 1);
      __syncwarp();
      if (lane == 0) {
        const int nw = __popc(wm);
        for (int t = 0; t < nw; t++) weak = xadd(weak, buf[t]);
      }
      __syncwarp();
    }
    double diag_hat = xadd(diag, weak);  // meaningful on lane 0
    // strong F neighbours in S order (= A order)
    for (int t = 0; t < ns; t++) {
      if (slt[t] >= 0) continue;
      const int kk = col[t];
      const double a_ik = af[t];
      const int h = hubidx ? hubidx[kk] : -1;
      int ne = 0;
      if (h >= 0) {
        // entries of the hub row in C_i by lookup, then ranked by position
        const int l = lane < nc ? hub_find(hkeys, hvals, hoff, h, cm[lane]) : -1;
        const unsigned fm = __ballot_sync(0xffffffffu, l >= 0);
        ne = __popc(fm);
        int rank = 0;
        for (int u = 0; u < 32; u++) {
          const int lu = __shfl_sync(0xffffffffu, l, u);
          rank += (lu >= 0 && l >= 0 && lu < l);
        }
        if (l >= 0) {
          el[rank] = l;
          sl[rank] = lane;
        }
      } else {
        for (int base = aia[kk]; base < aia[kk + 1]; base += 32) {
          const int l = base + lane;
          int sidx = -1;
          if (l < aia[kk + 1]) {
            const int mcol = aja[l];
            if (cf[mcol] == 1)
              for (int u = 0; u < nc; u++)
                if (cm[u] == mcol) { sidx = u; break; }
          }
          const unsigned fm = __ballot_sync(0xffffffffu, sidx >= 0);
          if (sidx >= 0) {
            const int o = ne + __popc(fm & lt);
            el[o] = l;
            sl[o] = sidx;
          }
          ne += __popc(fm);
        }
      }
      __syncwarp();
      double denom = 0.0;
      if (lane == 0)
        for (int u = 0; u < ne; u++) denom = xadd(denom, aval[el[u]]);
      denom = __shfl_sync(0xffffffffu, denom, 0);
      if (fabs(denom) < 1e-15) {
        if (lane == 0) diag_hat = xadd(diag_hat, a_ik);
      } else if (lane < ne) {
        const int o = p0 + sl[lane];
        pval[o] = xadd(pval[o], xdiv(xmul(a_ik, aval[el[lane]]), denom));
      }
      __syncwarp();
    }
    diag_hat = __shfl_sync(0xffffffffu, diag_hat, 0);
    if (fabs(diag_hat) > 1e-15 && lane < nc) pval[p0 + lane] = xdiv(pval[p0 + lane], -diag_hat);
    __syncwarp();
  }
}

__global__ void k_interp_values(const int* __restrict__ aia, const int* __restrict__ aja,
                                const double* __restrict__ aval, const int* __restrict__ sia,
                                const int* __restrict__ sja, const int* __restrict__ cf, int n,
                                const int* __restrict__ pia, double* __restrict__ pval,
                                const int* __restrict__ hubidx, const int* __restrict__ hoff,
                                const int* __restrict__ hkeys, const int* __restrict__ hvals) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int p0 = pia[i], p1 = pia[i + 1];
    if (cf[i] == 1) {
      pval[p0] = 1.0;
      continue;
    }
    if (warp_row(aia, sia, i)) continue;  // k_interp_values_warp
    const int s0 = sia[i], s1 = sia[i + 1];
    for (int p = p0; p < p1; p++) pval[p] = 0.0;
    double diag = 0.0, weak = 0.0;
    for (int k = aia[i]; k < aia[i + 1]; k++) {
      int j = aja[k];
      double a = aval[k];
      if (j == i) {
        diag = a;
        continue;
      }
      bool strong;
      int slot = strong_slot(sja, s0, s1, cf, j, &strong);
      if (strong && cf[j] == 1)
        pval[p0 + slot] = xadd(pval[p0 + slot], a);
      else if (strong && cf[j] == -1) {
        // strong F neighbour: distributed below
      } else
        weak = xadd(weak, a);
    }
    double diag_hat = xadd(diag, weak);
    // this row's strong C points in S order (slot q = index in the list)
    int cm[kInterpMaxC];
    int nc = 0;
    if (hubidx) {
      for (int k = s0; k < s1 && nc <= kInterpMaxC; k++) {
        const int q = sja[k];
        if (cf[q] == 1) {
          if (nc < kInterpMaxC) cm[nc] = q;
          nc++;
        }
      }
    }
    for (int k = aia[i]; k < aia[i + 1]; k++) {
      int kk = aja[k];
      if (kk == i) continue;
      bool strong;
      strong_slot(sja, s0, s1, cf, kk, &strong);
      if (!strong || cf[kk] != -1) continue;
      const double a_ik = aval[k];
      const int h = hubidx ? hubidx[kk] : -1;
      if (h >= 0 && nc <= kInterpMaxC) {
        // entries of row kk in C_i, by lookup, then in row order
        int el[kInterpMaxC], sl[kInterpMaxC];
        int ne = 0;
        for (int q = 0; q < nc; q++) {
          const int l = hub_find(hkeys, hvals, hoff, h, cm[q]);
          if (l < 0) continue;
          int t = ne++;
          while (t > 0 && el[t - 1] > l) {
            el[t] = el[t - 1];
            sl[t] = sl[t - 1];
            t--;
          }
          el[t] = l;
          sl[t] = q;
        }
        double denom = 0.0;
        for (int t = 0; t < ne; t++) denom = xadd(denom, aval[el[t]]);
        if (fabs(denom) < 1e-15) {
          diag_hat = xadd(diag_hat, a_ik);
        } else {
          for (int t = 0; t < ne; t++)
            pval[p0 + sl[t]] = xadd(pval[p0 + sl[t]], xdiv(xmul(a_ik, aval[el[t]]), denom));
        }
        continue;
      }
      double denom = 0.0;
      for (int l = aia[kk]; l < aia[kk + 1]; l++) {
        int m = aja[l];
        if (cf[m] != 1) continue;
        bool sm;
        strong_slot(sja, s0, s1, cf, m, &sm);
        if (sm) denom = xadd(denom, aval[l]);
      }
      if (fabs(denom) < 1e-15) {
        diag_hat = xadd(diag_hat, a_ik);
      } else {
        for (int l = aia[kk]; l < aia[kk + 1]; l++) {
          int m = aja[l];
          if (cf[m] != 1) continue;
          bool sm;
          int slot = strong_slot(sja, s0, s1, cf, m, &sm);
          if (sm) pval[p0 + slot] = xadd(pval[p0 + slot], xdiv(xmul(a_ik, aval[l]), denom));
        }
      }
    }
    if (fabs(diag_hat) > 1e-15) {
      const double nd = -diag_hat;
      for (int p = p0; p < p1; p++) pval[p] = xdiv(pval[p], nd);
    }
  }
}

void interpolation_values(const CSR& A, const CSR& S, const int* cf, CSR& P, cudaStream_t s) {
  if (A.n == 0) return;
  const int n = A.n;
  DBuf<int> hubidx(n, s), hubrows(n, s), ctr(1, s);
  ctr.zero();
  BN_LAUNCH(k_hub_mark, grid_for(n, 256), 256, 0, s, A.ia.p, n, hubidx.p, hubrows.p, ctr.p);
  const int nh = read_scalar(ctr.p, s);
  DBuf<int> hoff((size_t)nh + 1, s), keys, vals;
  if (nh > 0) {
    hoff.zero();
    BN_LAUNCH(k_hub_size, grid_for(nh, 256), 256, 0, s, A.ia.p, hubrows.p, nh, hoff.p);
    const int tot = scan_counts(hoff.p, nh, s);
    keys.alloc(tot, s);
    vals.alloc(tot, s);
    keys.fill_bytes(0xff);
    BN_LAUNCH(k_hub_fill, nh, 256, 0, s, A.ia.p, A.ja.p, hubrows.p, hoff.p, keys.p, vals.p);
  }
  BN_LAUNCH(k_interp_values, grid_for(n, 128), 128, 0, s, A.ia.p, A.ja.p, A.val.p, S.ia.p,
            S.ja.p, cf, n, P.ia.p, P.val.p, nh > 0 ? hubidx.p : nullptr, hoff.p, keys.p,
            vals.p);
  ctr.zero();
  BN_LAUNCH(k_warp_rows, grid_for(n, 256), 256, 0, s, A.ia.p, S.ia.p, cf, n, hubrows.p, ctr.p);
  const int nw = read_scalar(ctr.p, s);
  if (nw > 0)
    BN_LAUNCH(k_interp_values_warp, grid_for((long long)nw * 32, 32 * kInterpWarps, 8),
              32 * kInterpWarps, 0, s, A.ia.p, A.ja.p, A.val.p, S.ia.p, S.ja.p, S.val.p, cf,
              hubrows.p, nw, P.ia.p, P.val.p, nh > 0 ? hubidx.p : nullptr, hoff.p, keys.p,
              vals.p);
}

void interpolation_pattern(const CSR& S, const int* cf, int n_coarse, CSR& P, cudaStream_t s) {
  const int n = S.n;
  DBuf<int> flag(n, s), cmap(n, s), cnt((size_t)n + 1, s);
  const int g = grid_for(n, 256);
  BN_LAUNCH(k_is_c, g, 256, 0, s, cf, n, flag.p);
  exclusive_scan_i32(flag.p, cmap.p, n, s);
  cnt.zero();
  BN_LAUNCH(k_interp_count, g, 256, 0, s, S.ia.p, S.ja.p, cf, n, cnt.p);
  int pnnz = scan_counts(cnt.p, n, s);
  P.n = n;
  P.m = n_coarse;
  P.nnz = pnnz;
  P.ia = std::move(cnt);
  P.ja.alloc((size_t)(pnnz > 0 ? pnnz : 1), s);
  P.val.alloc((size_t)(pnnz > 0 ? pnnz : 1), s);
  BN_LAUNCH(k_interp_pattern, g, 256, 0, s, S.ia.p, S.ja.p, cf, cmap.p, n, P.ia.p, P.ja.p);
}

void interpolation(const CSR& A, const CSR& S, const int* cf, int n_coarse, CSR& P,
                   cudaStream_t s) {
  interpolation_pattern(S, cf, n_coarse, P, s);
  interpolation_values(A, S, cf, P, s);
}

}  // namespace bn
