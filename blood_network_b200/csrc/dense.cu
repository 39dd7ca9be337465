// Coarsest-level solve: dense FP64 Cholesky, then the explicit inverse, so
// that each V-cycle's coarse solve is one dense matrix-vector product.
//
// The reference solves the coarsest level with ichol-preconditioned PCG to a
// relative B-norm of 1e-12 (C_amg1/src/amg_cycle.c:188,229); a direct solve
// reaches the exact coarse solution up to cond(A_c) * eps.  The coarse
// operator is SPD (Galerkin product of an SPD matrix), so Cholesky applies.
#include "dense.cuh"

namespace bn {

__global__ void k_csr_to_dense(const int* __restrict__ ia, const int* __restrict__ ja,
                               const double* __restrict__ val, int n, double* __restrict__ D) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    for (int k = ia[i]; k < ia[i + 1]; k++) D[(size_t)i * n + ja[k]] += val[k];
}

// column j: pivot and scale (one block)
__global__ void k_chol_col(double* D, int n, int j, int* err) {
  __shared__ double piv;
  if (threadIdx.x == 0) {
    double d = D[(size_t)j * n + j];
    if (!(d > 0.0)) {
      atomicCAS(err, 0, 1);
      d = 1e-300;
    }
    piv = sqrt(d);
    D[(size_t)j * n + j] = piv;
  }
  __syncthreads();
  const double inv = 1.0 / piv;
  for (int i = j + 1 + threadIdx.x; i < n; i += blockDim.x) D[(size_t)i * n + j] *= inv;
}

// trailing update of the lower triangle: D[i][k] -= L[i][j] L[k][j], j<k<=i
__global__ void k_chol_update(double* D, int n, int j) {
  const int m = n - j - 1;
  const long long total = (long long)m * m;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    int i = j + 1 + (int)(t / m);
    int k = j + 1 + (int)(t % m);
    if (k <= i) D[(size_t)i * n + k] -= D[(size_t)i * n + j] * D[(size_t)k * n + j];
  }
}

// column c of A^{-1} = L^{-T} L^{-1} e_c, one thread per column, in place
__global__ void k_chol_inverse(const double* __restrict__ L, int n, double* __restrict__ X) {
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x) {
    for (int i = 0; i < c; i++) X[(size_t)i * n + c] = 0.0;
    for (int i = c; i < n; i++) {
      double s = (i == c) ? 1.0 : 0.0;
      for (int k = c; k < i; k++) s -= L[(size_t)i * n + k] * X[(size_t)k * n + c];
      X[(size_t)i * n + c] = s / L[(size_t)i * n + i];
    }
    for (int i = n - 1; i >= 0; i--) {
      double s = X[(size_t)i * n + c];
      for (int k = i + 1; k < n; k++) s -= L[(size_t)k * n + i] * X[(size_t)k * n + c];
      X[(size_t)i * n + c] = s / L[(size_t)i * n + i];
    }
  }
}

// Coarsest levels of up to kDenseBlock rows: the factorisation and the
// triangular inverse each run in one block (column j of L staged in shared
// memory; a barrier per column instead of two launches per column), then
// A^{-1} = X^T X with X = L^{-1} across the grid.
constexpr int kDenseBlock = 4096;
constexpr int kDenseThreads = 1024;

// right-looking Cholesky of the lower triangle, in place
__global__ void __launch_bounds__(kDenseThreads) k_chol_block(double* D, int n, int* err) {
  extern __shared__ double colj[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int j = 0; j < n; j++) {
    double* Dj = D + (size_t)j * n;
    if (threadIdx.x == 0) {
      double d = Dj[j];
      if (!(d > 0.0)) {
        *err = 1;
        d = 1e-300;
      }
      Dj[j] = sqrt(d);
    }
    __syncthreads();
    const double piv = Dj[j];
    for (int i = j + 1 + threadIdx.x; i < n; i += blockDim.x) {
      const double l = D[(size_t)i * n + j] / piv;
      D[(size_t)i * n + j] = l;
      colj[i] = l;
    }
    __syncthreads();
    // D[i][k] -= L[i][j] L[k][j], j < k <= i: a warp per row, lanes along k
    for (int i = j + 1 + warp; i < n; i += nw) {
      const double li = colj[i];
      double* Di = D + (size_t)i * n;
      for (int k = j + 1 + lane; k <= i; k += 32) Di[k] -= li * colj[k];
    }
    __syncthreads();
  }
}

// X = L^{-1} (lower triangle; the rest of X is zero), row by row: row k is
// final once the rows above have been subtracted, then it is divided by
// L[k][k] and subtracted from every later row
__global__ void __launch_bounds__(kDenseThreads)
k_trinv_block(const double* __restrict__ L, int n, double* __restrict__ X) {
  extern __shared__ double rowk[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (size_t t = threadIdx.x; t < (size_t)n * n; t += blockDim.x)
    X[t] = (t / n == t % n) ? 1.0 : 0.0;
  __syncthreads();
  for (int k = 0; k < n; k++) {
    const double d = L[(size_t)k * n + k];
    for (int c = threadIdx.x; c <= k; c += blockDim.x) {
      const double v = X[(size_t)k * n + c] / d;
      X[(size_t)k * n + c] = v;
      rowk[c] = v;
    }
    __syncthreads();
    for (int i = k + 1 + warp; i < n; i += nw) {
      const double lik = L[(size_t)i * n + k];
      double* Xi = X + (size_t)i * n;
      for (int c = lane; c <= k; c += 32) Xi[c] -= lik * rowk[c];
    }
    __syncthreads();
  }
}

// Ainv[i][j] = sum_{k >= max(i,j)} X[k][i] X[k][j]
__global__ void k_xtx(const double* __restrict__ X, int n, double* __restrict__ Ainv) {
  const long long total = (long long)n * n;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(t / n), j = (int)(t % n);
    double acc = 0.0;
    for (int k = i > j ? i : j; k < n; k++) acc += X[(size_t)k * n + i] * X[(size_t)k * n + j];
    Ainv[t] = acc;
  }
}

// x = Ainv b; one warp per row, FP64 accumulation
template <class T>
__global__ void k_dense_apply(const double* __restrict__ Ainv, int n, const T* __restrict__ b,
                              T* __restrict__ x) {
  BN_PDL_ENTRY();
  const int lane = threadIdx.x & 31;
  const int warps = (gridDim.x * blockDim.x) >> 5;
  for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < n; i += warps) {
    const double* row = Ainv + (size_t)i * n;
    double s = 0.0;
    for (int k = lane; k < n; k += 32) s += row[k] * (double)b[k];
    for (int off = 16; off > 0; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
    if (lane == 0) x[i] = (T)s;
  }
}

void DenseCoarse::setup(const CSR& A, cudaStream_t s) {
  n = A.n;
  BN_REQUIRE(n <= kDenseMax, BN_ERR_COARSE, "coarsest level too large for the dense solve");
  DBuf<double> D((size_t)n * n, s);
  D.zero();
  DBuf<int> err(1, s);
  err.zero();
  if (n > 0) BN_LAUNCH(k_csr_to_dense, grid_for(n, 128), 128, 0, s, A.ia.p, A.ja.p, A.val.p, n, D.p);
  if (n > 0 && n <= kDenseBlock) {
    const size_t sh = sizeof(double) * (size_t)n;
    BN_CUDA(cudaFuncSetAttribute(k_chol_block, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)(sizeof(double) * kDenseBlock)));
    BN_CUDA(cudaFuncSetAttribute(k_trinv_block, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)(sizeof(double) * kDenseBlock)));
    BN_LAUNCH(k_chol_block, 1, kDenseThreads, sh, s, D.p, n, err.p);
    BN_REQUIRE(read_scalar(err.p, s) == 0, BN_ERR_COARSE,
               "coarsest operator is not positive definite");
    DBuf<double> X((size_t)n * n, s);
    BN_LAUNCH(k_trinv_block, 1, kDenseThreads, sh, s, D.p, n, X.p);
    inv.alloc((size_t)n * n, s);
    BN_LAUNCH(k_xtx, grid_for((long long)n * n, 256), 256, 0, s, X.p, n, inv.p);
    return;
  }
  for (int j = 0; j < n; j++) {
    BN_LAUNCH(k_chol_col, 1, 256, 0, s, D.p, n, j, err.p);
    long long m = (long long)(n - j - 1) * (n - j - 1);
    if (m > 0) BN_LAUNCH(k_chol_update, grid_for(m, 256), 256, 0, s, D.p, n, j);
  }
  BN_REQUIRE(read_scalar(err.p, s) == 0, BN_ERR_COARSE,
             "coarsest operator is not positive definite");
  inv.alloc((size_t)n * n, s);
  if (n > 0) BN_LAUNCH(k_chol_inverse, grid_for(n, 64, 4), 64, 0, s, D.p, n, inv.p);
}

template <class T>
void DenseCoarse::apply(const T* b, T* x, cudaStream_t s) const {
  if (n == 0) return;
  BN_LAUNCH_PDL(k_dense_apply<T>, grid_for((long long)n * 32, 256, 8), 256, 0, s, inv.p, n, b, x);
}
template void DenseCoarse::apply<double>(const double*, double*, cudaStream_t) const;
template void DenseCoarse::apply<float>(const float*, float*, cudaStream_t) const;

}  // namespace bn
