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

__global__ void k_interp_values(const int* __restrict__ aia, const int* __restrict__ aja,
                                const double* __restrict__ aval, const int* __restrict__ sia,
                                const int* __restrict__ sja, const int* __restrict__ cf, int n,
                                const int* __restrict__ pia, double* __restrict__ pval) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int p0 = pia[i], p1 = pia[i + 1];
    if (cf[i] == 1) {
      pval[p0] = 1.0;
      continue;
    }
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
    for (int k = aia[i]; k < aia[i + 1]; k++) {
      int kk = aja[k];
      if (kk == i) continue;
      bool strong;
      strong_slot(sja, s0, s1, cf, kk, &strong);
      if (!strong || cf[kk] != -1) continue;
      const double a_ik = aval[k];
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
  BN_LAUNCH(k_interp_values, grid_for(A.n, 128), 128, 0, s, A.ia.p, A.ja.p, A.val.p, S.ia.p,
            S.ja.p, cf, A.n, P.ia.p, P.val.p);
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
