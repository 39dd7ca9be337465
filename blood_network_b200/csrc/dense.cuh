// Dense FP64 coarsest-level solver.
#pragma once
#include "common.cuh"

namespace bn {

constexpr int kDenseMax = 8192;

struct DenseCoarse {
  int n = 0;
  DBuf<double> inv;  // A_c^{-1}, row-major n x n
  void setup(const CSR& A, cudaStream_t s);
  template <class T>
  void apply(const T* b, T* x, cudaStream_t s) const;
};

}  // namespace bn
