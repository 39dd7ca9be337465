// IC(0) factor and level-scheduled triangular solves.
#pragma once
#include "internal.cuh"
#include "flags.cuh"

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
  // per level, the sync-free form over 32-row chunks (default) or the tiled
  // form (BN_IC_MODE=levels|coop|flags|tiles)
  enum { kSweepLevels = 0, kSweepCoop = 1, kSweepFlags = 2, kSweepTiles = 3 };
  int mode = mode_from_env();
  int blocks_per_sm = blocks_from_env();  // sync-free grid: blocks per SM (0: occupancy)
  WaitRecord wait;              // sync-free and tiled forms: bounded waits and their record
  DBuf<int2> d_fchunk, d_bchunk;  // sync-free form: 32-row chunks within levels
  int n_fchunk = 0, n_bchunk = 0;
  // tiled form: tile q holds the rows of index range [q R, (q+1) R) (the
  // forward sweep; the backward sweep takes the tiles in reverse); a step
  // is the tile's rows of one level, a contiguous range of the level-ordered
  // layout.  tile_steps[q] = [first step, end step), steps[k] = [first
  // position, end position).  imask[t]: bit q set when entry q of row t
  // depends on a row of the same tile (read from the block's own earlier
  // steps); other entries poll their dependency.
  struct Tiles {
    int ntiles = 0, rows_per_tile = 0, threads = 0, nsteps = 0;
    DBuf<int2> tile_steps, steps;
    DBuf<unsigned> imask;
  };
  Tiles tf, tb;
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
  // throws BN_ERR_SPIN (with the record's row, dependency and time) if a
  // wait of the last sweeps ran out; the record is cleared
  void check_waits(cudaStream_t s);
  static int mode_from_env();
  static int blocks_from_env();
  void build_tiles(bool forward, cudaStream_t s);
  int launches_per_solve() const { return (int)(fseg.size() + bseg.size()); }
};

}  // namespace bn
