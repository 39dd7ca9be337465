// IC(0) factor and level-scheduled triangular solves.
#pragma once
#include "internal.cuh"
#include "flags.cuh"

namespace bn {

__global__ void k_iota_i(int* a, int n);
// lev[t] = level of position t of a level-ordered layout (ptr: level offsets)
__global__ void k_pos_level(const int* __restrict__ ptr, int nlevels, int n, int* __restrict__ lev);
struct IChol;
// one sweep of the slab form (ic_slab.cu); out pre-filled with the pending pattern
template <class T>
void run_tri_slab(const IChol& ic, bool forward, const T* in, T* out, T* clear, WaitCtl wc,
                  cudaStream_t s);

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
  // per level, the sync-free form over 32-row chunks (default), the tiled
  // form or the slab form (the sync-free form runs where its rings do not
  // fit) or its chunked variant without barriers
  // (BN_IC_MODE=levels|coop|flags|tiles|slab|slabw)
  enum {
    kSweepLevels = 0, kSweepCoop = 1, kSweepFlags = 2, kSweepTiles = 3, kSweepSlab = 4,
    kSweepSlabW = 5
  };
  static constexpr int kSlabThreads = 512;
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
  // slab form: the rows are split into one slab per SM
  // (rows of wide, index-concentrated levels dealt evenly by their rank in
  // the level, all other rows by contiguous index ranges); a block owns a
  // slab and walks its rows in level order, at most kSlabThreads rows per
  // step with a block barrier after each step.  Row records, entries and
  // input values are staged into shared-memory rings by asynchronous
  // copies a few steps ahead; a dependency on a recent row of the same slab
  // is read from a shared-memory ring of computed values, every other one
  // from the output vector (value-as-flag, bounded polls), the first of
  // them pre-read into shared memory when its step is staged.
  struct Slab {
    int nsteps = 0, nnz = 0;
    int lead32 = 0, lead64 = 0;   // staging lead in steps (0: the rings do not fit)
    DBuf<int2> slab_steps;        // per slab (block): [first step, end step)
    DBuf<int2> steps;             // nsteps + 1: {first position, first entry}
    DBuf<int4> rec;               // per position: {vector row, first entry, pre-read dep, FP32 diagonal bits}
    DBuf<int> rnat, xnat;         // per position: natural row, natural pre-read dep (-1: none)
    DBuf<int> vrow, vx;           // the same in the vector numbering
    DBuf<int> cnat, code;         // per entry: ring code (< 0) or dependency (natural / vector numbering)
    DBuf<int> esrc;               // per entry: index of its value in L
    DBuf<double> ev64, d64;
    DBuf<float> ev32, d32;
  };
  Slab sf, sb;
  DBuf<int> slab_of;              // natural row -> slab
  int nslab = 0;
  void build_slab_partition(cudaStream_t s);
  void build_slab(bool forward, cudaStream_t s);
  void slab_values(Slab& sl, cudaStream_t s);
  void slab_pack(Slab& sl, const int* inv, cudaStream_t s);
  template <class T>
  bool slab_ready() const {
    return (mode == kSweepSlab || mode == kSweepSlabW) &&
           (sizeof(T) == 8 ? (sf.lead64 && sb.lead64) : (sf.lead32 && sb.lead32));
  }
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
