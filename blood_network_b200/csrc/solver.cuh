// Solver state shared by the solver's C ABI (solver.cu) and the
// reference-named host entry points (compat.cu).
#pragma once
#include "internal.cuh"
#include "ichol.cuh"
#include "dense.cuh"
#include "solve_kernels.cuh"
#include "packed.cuh"
#include "../../include/amg_b200.h"

#include <cstdlib>
#include <functional>
#include <memory>
#include <vector>

namespace bn {

// ------------------------------------------------------------ data
struct Level {
  // setup data in the natural numbering (bit-identical to the reference)
  CSR A, S, P, R;
  DBuf<int> cf;
  int n_coarse = 0;
  int max_lam = 0;
  // solve phase: the level's unknowns renumbered so that every colour class
  // is a contiguous range (perm[new] = natural, inv[natural] = new).  Ap is
  // A renumbered on both sides; Pp maps the next level's numbering into this
  // one; Rp = Pp^T.  FP32 value copies serve the mixed-precision V-cycle.
  DBuf<int> perm, inv;
  CSR Ap, Pp, Rp;
  RowLayout layA, layP, layR;  // SpMV row-length layouts of Ap, Pp, Rp
  DBuf<float> A32, P32, R32;
  // smoother colouring: rows grouped by (set, colour)
  DBuf<int> gs_rows;
  std::vector<int> cptr;   // colour class offsets into gs_rows
  std::vector<char> cjac;  // class is an overflow class (Jacobi update)
  std::vector<int> clong;  // long rows at the end of each class
  int colored_for = -1;    // smoother the colouring was built for
  int color_rounds = 0;
  int gs_group = 1;        // lanes per row in the GS kernel
  DBuf<int> d_cptr, d_cjac;  // class tables on the device (single-block sweeps)
  DBuf<double> l1, dg;
  DBuf<float> l1_32, dg32;
  // load-balanced kernels: packings of Ap, Pp, Rp (one range each) and of
  // the colour classes of Ap (one range per class)
  Packing pkA, pkP, pkR, pkG;
  // which operators run on the packed kernels: those with rows longer than
  // kLongRow (hub rows); the row-group kernels are faster on the others
  bool use_pkA = false, use_pkP = false, use_pkR = false;
  // Ap split by colour class for the first smoothing sweep from a zero
  // guess (coloured levels on the row-group kernels): AL row i holds the
  // entries of row i in earlier classes plus the diagonal, AU the other
  // off-diagonal entries negated.  A forward sweep from x = 0 reads only
  // AL (later classes are still zero), and afterwards b - A x = AU x (each
  // row's own equation held when it was updated), so the sweep and the
  // residual read A once instead of twice.
  bool split = false;
  CSR AL, AU;
  DBuf<float> AL32, AU32;
  RowLayout layAL, layAU;
  Packing pkAL, pkAU;  // levels with hub rows: AL per class, AU as one range
  // work vectors
  DBuf<double> b, x, r;
  DBuf<float> b32, x32, r32;
};

struct BlockWork;  // work vectors of a many-right-hand-side solve (block.cu)

struct Solver {
  int device = 0;
  cudaStream_t s = 0;
  amg_b200_options opt{};
  std::vector<std::unique_ptr<Level>> lv;
  DenseCoarse coarse;
  CSR Aown;               // solve matrix when set_matrix replaced it
  CSR Aownp;              // ... renumbered like level 0
  RowLayout layOwn;
  bool own_solve = false;
  DBuf<float> Aown32;
  IChol ic;
  bool f32_ready = false;
  // level-0 preconditioner vectors
  DBuf<double> u1, r1, icy, icx, xx, r2, corr;
  DBuf<float> g32, u1f, r1f, icyf, icxf, xxf, r2f, corrf;
  // PCG vectors
  DBuf<double> b, x, r, z, p, ap;
  DBuf<double> sc, part0, part1;
  double* h_sc = nullptr;
  cudaGraphExec_t graph[2] = {nullptr, nullptr};
  unsigned long long graph_kernels[2] = {0, 0};
  // PCG iterations as one graph each (a conditional WHILE node whose body
  // is one iteration, the stopping test evaluated on the device): [mode] for
  // the single solve, seg_loop for the segmented one (rebuilt per call)
  cudaGraphExec_t loop[2] = {nullptr, nullptr};
  unsigned long long loop_kernels[2] = {0, 0};
  DBuf<int> ctl;           // device loop state: [0] iterations done, [1] status, [2] maxiter
  bool loops_ok = getenv("BN_HOST_LOOP") == nullptr;  // BN_HOST_LOOP=1: host-driven loops
  bool capture_direct = false;  // precond(): emit the kernels (inside a loop capture)
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  amg_solve_stats stats{};

  ~Solver();
  const CSR& Asolve() const { return own_solve ? Aown : lv[0]->A; }
  int n() const { return Asolve().n; }
  void build(CSR&& A0);
  void rebuild_values(CSR&& A0);
  void finish_setup();
  void prepare_f32();
  void color_level(Level& L, int smoother);
  void alloc_vectors();
  void drop_graphs();
  template <class T> DevMat<T> mat(const CSR& M, const DBuf<float>* v32,
                                   const RowLayout* lay) const;
  template <class T> PackedMat<T> pmat(const CSR& M, const DBuf<float>& v32,
                                       const Packing& pk) const;
  // V-cycle SpMV and colour classes on the packed kernels (BN_PACKED=0: the
  // row-group kernels)
  bool use_packed = getenv("BN_PACKED") == nullptr || atoi(getenv("BN_PACKED")) != 0;
  const RowLayout& lay_solve() const { return own_solve ? layOwn : lv[0]->layA; }
  const CSR& Asolve_p() const { return own_solve ? Aownp : lv[0]->Ap; }
  void build_solve_layout();
  template <class T> void smooth(int l, const T* bb, T* xl, bool forward);
  // zero_guess: xl holds zeros on entry (every call inside the
  // preconditioner), which allows the split first sweep
  template <class T> void backslash(int l, const T* bb, T* xl, bool zero_guess);
  void build_split(Level& L);
  template <class T> void fwdslash(int l, const T* bb, T* xl);
  template <class T> void precond_t(const T* g, T* out);
  void precond(const double* g, double* out);  // z = M g (FP64 interface)
  int pcg(const double* d_b, double* d_x, double tol, int maxiter, int print_level);
  // K right-hand sides at once (column-major n x K device arrays), each
  // column with its own PCG; the V-cycle and IC(0) run on all columns
  int pcg_block(int K, const double* d_B, double* d_X, double tol, int maxiter, int* h_iters,
                double* h_relres);
  template <class T> void smooth_block(BlockWork& W, int l, const T* bb, T* xl, bool forward);
  template <class T> void backslash_block(BlockWork& W, int l, const T* bb, T* xl);
  template <class T> void fwdslash_block(BlockWork& W, int l, const T* bb, T* xl);
  template <class T> void precond_block_t(BlockWork& W, const T* g, T* out);
  void precond_block(BlockWork& W, const double* g, double* out);
  // times the candidate solve-phase kernels per level and keeps the fastest
  // (what: 1 SpMV/transfer row groups, 2 Gauss-Seidel lanes per row)
  template <class T> int autotune_t(int what, double* report, int nreport);
  // independent block-diagonal systems (natural row ranges d_ptr[k]..d_ptr[k+1]-1),
  // each with its own PCG scalars and stopping test; device b, x
  int pcg_segmented(int nseg, const int* d_ptr, const double* d_b, double* d_x, double tol,
                    int maxiter, int* h_iters, double* h_relres);
  // FP64 pieces for the reference-named host entry points (device vectors in
  // the solve numbering of the level)
  void vcycle_apply(const double* g, double* out);             // symmetric V-cycle
  void backslash_at(int l, const double* b, double* x);        // x: initial guess
  void fwdslash_at(int l, const double* b, double* x);         // x: initial guess
  void use_matrix_and_factor(CSR* A, CSR&& Lf);  // A null: the hierarchy's level 0
};

void l1_row_norms(const CSR& A, double* d_out, cudaStream_t s);  // sum_j |a_ij|

// Validated upload of host or device CSR, optionally symmetrised (the
// wrapper's (A + A^T)/2); a solver built from it.
void upload_csr(Solver& S, int n, int nnz, const int* ia, const int* ja, const double* val,
                bool device_ptrs, bool symmetrise, CSR& out);
Solver* make_solver(int n, int nnz, const int* ia, const int* ja, const double* val,
                    const amg_b200_options* o, bool device_ptrs, bool symmetrise = true);
void permute_csr(const CSR& A, const int* perm, const int* cinv, CSR& B, cudaStream_t s);


// runs f, turning errors into status codes (last error set)
template <class F>
int guarded(F&& f, int fail) {
  try {
    return f();
  } catch (const Error& e) {
    set_last_error(e.code, e.what());
    return fail;
  } catch (const std::exception& e) {
    set_last_error(BN_ERR_CUDA, e.what());
    return fail;
  }
}

}  // namespace bn
