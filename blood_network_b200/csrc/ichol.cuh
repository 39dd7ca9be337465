// IC(0) factor and level-scheduled triangular solves.
#pragma once
#include "internal.cuh"

namespace bn {

__global__ void k_iota_i(int* a, int n);

struct IChol {
  struct Seg {
    int kind;    // 0: one wide level (grid launch); 1: run of narrow levels (one block)
    int l0, l1;  // level range
    int t0, t1;  // row range in the level-ordered layout
  };
  int n = 0;
  int nlevels = 0;
  int offd_nnz = 0;
  bool want_f32 = false;
  cudaStream_t stream = 0;
  CSR L;                    // lower triangle, reference layout and values
  DBuf<int> pre, dpos;      // leading strictly-lower count, diagonal position
  DBuf<int> order, border;  // rows in level order / reverse level order
  std::vector<int> lptr, bptr;        // level offsets (forward / backward order)
  DBuf<int> d_lptr, d_bptr;
  std::vector<Seg> fseg, bseg;
  DBuf<int4> d_cfseg, d_cbseg;  // cooperative schedules (narrow = 1024 rows)
  int n_cfseg = 0, n_cbseg = 0;
  // sweep form: level launches, one cooperative launch with a grid barrier
  // per level, or the sync-free form (default; BN_IC_MODE=levels|coop|flags)
  enum { kSweepLevels = 0, kSweepCoop = 1, kSweepFlags = 2 };
  int mode = mode_from_env();
  int blocks_per_sm = blocks_from_env();  // sync-free grid: blocks per SM (0: occupancy)
  DBuf<int> err;                // sync-free form: a wait ran out
  DBuf<int2> d_fchunk, d_bchunk;  // sync-free form: 32-row chunks within levels
  int n_fchunk = 0, n_bchunk = 0;
  DBuf<int> fia, fja, fsrc; // forward rows (level order)
  DBuf<int> bia, bja, bsrc; // backward rows (reverse level order)
  // vector indices used by the solves: the rows/columns above mapped into
  // the numbering of the vectors (the solve phase's colour-ordered one)
  DBuf<int> vorder, vborder, vfja, vbja;
  DBuf<double> fval, bval, fdiag, bdiag;
  DBuf<float> fval32, bval32, fdiag32, bdiag32;

  void factor(const CSR& A, cudaStream_t s);   // pattern, levels, numeric factor
  void load(CSR&& Lf, cudaStream_t s);          // take a factor as given (solve only)
  void finish(const int* aia, const int* aja, const double* aval, bool numeric, cudaStream_t s);
  void refresh_values();                        // (re)gather solve values from L
  void remap(const int* inv, cudaStream_t s);   // vector numbering: inv[natural] (null: same)
  // x = (L L^T)^{-1} b ; y is scratch (n)
  template <class T>
  void solve(const T* b, T* y, T* x, cudaStream_t s);
  int take_error(cudaStream_t s);               // BN_ERR_SPIN if a wait ran out (then cleared)
  static int mode_from_env();
  static int blocks_from_env();
  int launches_per_solve() const { return (int)(fseg.size() + bseg.size()); }
};

}  // namespace bn
