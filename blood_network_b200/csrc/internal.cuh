// Internal (non-exported) interfaces shared by the library's translation units.
#pragma once
#include "common.cuh"

namespace bn {

// ---- csr_ops.cu
void transpose(const CSR& A, CSR& T, cudaStream_t s, bool with_val);
void add_scaled(const CSR& A, const CSR& B, double scale, CSR& C, cudaStream_t s);
void symmetrize(const CSR& A, CSR& out, cudaStream_t s);
int validate(const int* ia, const int* ja, int n, int m, int nnz, cudaStream_t s);

// ---- strength.cu
// S = strong part of A (reference rs_strength); returns max row length of A
// (floored at 1) in *max_lam.
void strength(const CSR& A, double theta, CSR& S, int* max_lam, cudaStream_t s);

// ---- coarsen.cu
enum Coarsening : int { COARSEN_RS = 0, COARSEN_PMIS = 1, COARSEN_HMIS = 2 };
// cf[i] = +1 (C) / -1 (F); returns the number of C points.
int coarsen(const CSR& S, int method, int max_lam, int* cf, cudaStream_t s);

// ---- interp.cu
void interpolation(const CSR& A, const CSR& S, const int* cf, int n_coarse, CSR& P,
                   cudaStream_t s);
void interpolation_pattern(const CSR& S, const int* cf, int n_coarse, CSR& P, cudaStream_t s);
void interpolation_values(const CSR& A, const CSR& S, const int* cf, CSR& P, cudaStream_t s);

// ---- rap.cu
void rap(const CSR& R, const CSR& A, const CSR& P, CSR& Ac, cudaStream_t s);

}  // namespace bn
