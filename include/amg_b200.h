/*
 * amg_b200.h -- C ABI of the B200 AMG-PCG solver for vessel-network pressure
 * systems.  Drop-in for the reference library (liuzhengqi1996/blood_network,
 * C_amg1/lib/libamg.so): the same symbol names and signatures, host pointers
 * in and out, computed on one NVIDIA B200 (sm_100a).  0-based CSR with int32
 * indices and float64 values, exactly the reference's dcsr_mat.
 *
 * Link: -lamg_b200 (blood_network_b200/lib/libamg_b200.so).  No C++ or torch
 * types cross this boundary.
 */
#ifndef AMG_B200_H
#define AMG_B200_H

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------------
 * Types, identical in layout to the reference (C_amg1/include/agg_lib.h:37-44
 * and C_amg1/include/amg.h:333-342).
 * --------------------------------------------------------------------- */
typedef struct {
  int row;     /* number of rows */
  int col;     /* number of columns */
  int nnz;     /* number of nonzero entries */
  int* ia;     /* row pointers, size row+1 */
  int* ja;     /* column indices, size nnz */
  double* val; /* values, size nnz */
} dcsr_mat;

#define AMG_MAX_LEVELS 20
#define SMOOTHER_L1 0     /* l1-Jacobi */
#define SMOOTHER_GS 1     /* Gauss-Seidel (multicolour on the device) */
#define SMOOTHER_CF_GS 2  /* CF-ordered Gauss-Seidel (multicolour, C then F) */
#define SMOOTHER_JACOBI 3 /* damped Jacobi */
#define COARSEN_RS 0
#define COARSEN_PMIS 1
#define COARSEN_HMIS 2

/* Status codes returned by the extension entry points and reported by
 * amg_solver_last_status(). */
#define AMG_OK 0
#define AMG_ERR_ARG (-1)
#define AMG_ERR_CUDA (-2)
#define AMG_ERR_OOM (-3)
#define AMG_ERR_NOT_CONVERGED (-4)
#define AMG_ERR_NAN (-5)
#define AMG_ERR_SPIN (-6)
#define AMG_ERR_COARSE (-7)
#define AMG_ERR_NO_DEVICE (-8)
#define AMG_ERR_DUP (-9)

/* Precision forms */
#define AMG_PREC_FP64 0  /* everything FP64, standard PCG (the reference's) */
#define AMG_PREC_MIXED 1 /* FP32 hierarchy + V-cycle inside FP64 flexible PCG */

/* Stopping rules for the PCG */
#define AMG_STOP_BNORM 0  /* sqrt(r.z / r0.z0) < tol  (the reference's rule) */
#define AMG_STOP_RELRES 1 /* ||r||_2 / ||b||_2 < tol  (true relative residual) */

/* =====================================================================
 * Drop-in entry points (C_amg1/src/amg_wrapper.c)
 * ===================================================================== */

/* Replaces amg_solver_create (amg_wrapper.c:51-97).  Copies the host CSR to
 * the device, symmetrises A=(A+A^T)/2, builds the AMG hierarchy (PMIS, CF
 * Gauss-Seidel) and the fine-level IC(0).  max_levels outside 1..20 becomes
 * 20; nu <= 0 becomes 1.  Returns NULL on failure (reason in
 * amg_solver_last_error()). */
void* amg_solver_create(int n, int nnz, const int* ia, const int* ja, const double* val,
                        double threshold, int min_size, int max_levels, int nu);

/* Replaces amg_solver_update (amg_wrapper.c:114-149): same sparsity, new
 * values; recomputes P values, coarse operators and IC(0).  Returns 0. */
int amg_solver_update(void* handle, int n, int nnz, const int* ia, const int* ja,
                      const double* val);

/* Replaces amg_solver_set_matrix (amg_wrapper.c:168-199): new solve matrix
 * and fine IC(0); the hierarchy is kept.  Returns 0. */
int amg_solver_set_matrix(void* handle, int n, int nnz, const int* ia, const int* ja,
                          const double* val);

/* Replaces amg_solver_set_smoother (amg_wrapper.c:241-246). */
void amg_solver_set_smoother(void* handle, int smoother, double omega);

/* Replaces amg_solver_solve (amg_wrapper.c:214-225).  Host b and x; x is the
 * initial guess.  Returns the iteration count, or -maxiter when not
 * converged.  print_level >= 1 prints per-iteration rows to stderr. */
int amg_solver_solve(void* handle, const double* b, double* x, double tol, int maxiter,
                     int print_level);

/* Replace amg_solver_size / num_levels / free (amg_wrapper.c:249-268). */
int amg_solver_size(void* handle);
int amg_solver_num_levels(void* handle);
void amg_solver_free(void* handle);

/* =====================================================================
 * Extensions (no counterpart in the reference's wrapper)
 * ===================================================================== */
typedef struct {
  double threshold; /* strength threshold theta */
  int min_size;     /* coarsening stops below this size */
  int max_levels;   /* 1..20 */
  int nu;           /* smoothing sweeps */
  int coarsening;   /* COARSEN_RS / COARSEN_PMIS / COARSEN_HMIS (the reference
                       selects this only in its CLI, test_amg.c:91) */
  int smoother;     /* SMOOTHER_* */
  double omega;     /* damped-Jacobi factor */
  int precision;    /* AMG_PREC_FP64 / AMG_PREC_MIXED */
  int stop;         /* AMG_STOP_BNORM / AMG_STOP_RELRES */
  int device;       /* CUDA device ordinal */
} amg_b200_options;

/* Defaults: theta 0.25, min_size 500, 20 levels, nu 1, PMIS, CF-GS, omega
 * 0.5, FP64, B-norm stop, device 0. */
void amg_b200_default_options(amg_b200_options* opt);

/* Create with explicit options (host CSR). */
void* amg_solver_create_ex(int n, int nnz, const int* ia, const int* ja, const double* val,
                           const amg_b200_options* opt);
/* Create from CSR already resident on the device (device pointers). */
void* amg_solver_create_device(int n, int nnz, const int* d_ia, const int* d_ja,
                               const double* d_val, const amg_b200_options* opt);

int amg_solver_set_precision(void* handle, int precision);
int amg_solver_set_stop(void* handle, int stop);

/* Solve with device-resident b and x (x: initial guess in, solution out). */
int amg_solver_solve_device(void* handle, const double* d_b, double* d_x, double tol,
                            int maxiter, int print_level);

/* ---- Files in the reference's formats (host)
 * COO text matrix, C_amg1/src/io.c:71-124 (dcsr_mat_dcoo) with the COO -> CSR
 * conversion of io.c:19-58: header "nrows ncols nnz", then "row col value"
 * lines; shifted to 0-based when the smallest index is exactly 1; entries of
 * a row keep their file order and repeated pairs are not summed.  The arrays
 * are malloc'd: release each with amg_free_host.  AMG_ERR_ARG on a malformed
 * file or an index out of range (the reference does not check). */
int amg_read_coo(const char* path, int* nrow, int* ncol, int* nnz, int** ia, int** ja,
                 double** val);
void amg_free_host(void* p);
/* Right-hand side file of C_amg1/test_amg.c:126-148: "n" then n values. */
int amg_read_vector(const char* path, int n, double* out);
/* Labelled solution of Matlab_amg/label_solution.m:41-44: "%d %.16e" lines
 * (1-based node id, pressure). */
int amg_write_labeled_solution(const char* path, int n, const int* node, const double* p);

/* Many right-hand sides on one hierarchy (the batched scenarios of one
 * network): B and X are column-major n x k host arrays, X holding the initial
 * guesses; column j is solved exactly as amg_solver_solve would solve it.
 * iterations[j] (may be NULL) receives that call's return value.  Returns 0,
 * or AMG_ERR_NOT_CONVERGED (-4) when a column did not converge. */
int amg_solver_solve_batch(void* handle, int k, const double* B, double* X, double tol,
                           int maxiter, int* iterations);

/* Autotuner: for every level, times the candidate solve-phase kernels on
 * the level's own operators in the solver's current precision and keeps the
 * fastest -- rows per group / vector width of the SpMV, restriction and
 * prolongation kernels (row tiles of 256/128/64/32 rows, or 4, 8, 32 lanes
 * per row) when what & 1,
 * lanes per row of the Gauss-Seidel colour classes (1, 8, 32) when what & 2.
 * The choice changes only the rounding of row sums.  report (may be NULL)
 * receives up to nreport/4 records {level, operator (0 A, 1 R, 2 P, 3 GS),
 * choice, ms}; returns the number of records, or a negative status. */
int amg_solver_autotune(void* handle, int what, double* report, int nreport);

/* Many right-hand sides solved together (the boundary-pressure scenarios of
 * one network): the PCG of every column runs at once over block vectors, so
 * each pass over a matrix (SpMV -> SpMM) and each IC(0) level, colour class
 * and coarse level serves all k columns; every column keeps its own alpha,
 * beta, stopping test and iteration count.  B and X are column-major n x k
 * (1 <= k <= 64), X holding the initial guesses.  iterations[j] / relres[j]
 * (may be NULL): the column's iteration count (-maxiter if not converged)
 * and true ||b - A x|| / ||b||.  Returns 0, AMG_ERR_NOT_CONVERGED (-4) or
 * AMG_ERR_NAN (-5).  _device: B and X are device pointers. */
int amg_solver_solve_block(void* handle, int k, const double* B, double* X, double tol,
                           int maxiter, int* iterations, double* relres);
int amg_solver_solve_block_device(void* handle, int k, const double* d_B, double* d_X,
                                  double tol, int maxiter, int* iterations, double* relres);

/* Independent networks packed block-diagonally into one matrix (no entry
 * couples two segments; checked, AMG_ERR_ARG otherwise): segment k is the
 * row range seg_ptr[k] .. seg_ptr[k+1]-1 (host array of nseg + 1 offsets
 * from 0 to n).  One SpMV and one preconditioner application a step serve
 * all segments, while each keeps the scalars, stopping test and iteration
 * count of its own PCG; a converged segment is frozen while the others go
 * on.  iterations[k] (host, may be NULL): the segment's iteration count, or
 * -maxiter when it did not converge; relres[k] (may be NULL): its true
 * ||b - A x|| / ||b||.  Returns 0, AMG_ERR_NOT_CONVERGED (-4) or
 * AMG_ERR_NAN (-5).  _device: b and x are device pointers. */
int amg_solver_solve_segmented(void* handle, int nseg, const int* seg_ptr, const double* b,
                               double* x, double tol, int maxiter, int* iterations,
                               double* relres);
int amg_solver_solve_segmented_device(void* handle, int nseg, const int* seg_ptr,
                                      const double* d_b, double* d_x, double tol, int maxiter,
                                      int* iterations, double* relres);

/* One application of the AMG+IC(0) preconditioner, x = M g (host arrays),
 * the reference's amg_ichol_precond (C_amg1/src/amg_ichol_precond.c:51). */
int amg_solver_precond(void* handle, const double* g, double* x);

typedef struct {
  int iterations;       /* last solve */
  int converged;
  double relres;        /* true ||b - A x|| / ||b|| after the last solve */
  double bnorm_rel;     /* sqrt(r.z / r0.z0) at exit */
  double setup_seconds; /* device time of the last hierarchy build */
  double solve_seconds; /* device time of the last solve */
  int num_levels;
  long long nnz_total;  /* sum of nnz over levels (operator complexity numerator) */
  int ichol_levels;     /* dependency levels of the fine IC(0) */
  int device_loop;      /* 1: the last solve ran its PCG iterations as one CUDA
                           graph with the stopping test on the device (no host
                           round trip per iteration); 0: host-driven loop */
  int ichol_form;       /* form of the fine IC(0) sweeps at the solver's precision:
                           0 level launches, 1 one cooperative launch, 2 sync-free
                           32-row chunks, 3 tiles, 4 slabs (one block per SM) */
} amg_solve_stats;

int amg_solver_stats(void* handle, amg_solve_stats* out);

/* Per-level sizes: n, nnz(A), nnz(S), nnz(P), n_coarse. */
int amg_solver_level_info(void* handle, int level, int* out5);
/* Copy level data to host (any pointer may be NULL). */
int amg_solver_level_copy(void* handle, int level, int* a_ia, int* a_ja, double* a_val,
                          int* s_ia, int* s_ja, double* s_val, int* p_ia, int* p_ja,
                          double* p_val, int* cf);

/* Times `reps` launches of one hot operation with CUDA events on the
 * solver's stream; *ms receives the mean milliseconds per launch.
 * which: 0 fine residual SpMV, 1 fine forward Gauss-Seidel sweep,
 * 2 preconditioner application, 3 IC(0) solve (two sweeps), 4 the fine
 * level's first sweep from a zero guess plus the residual after it (the
 * split form where the level has it).  precision: 0 FP64, 1 FP32. */
int amg_solver_bench_kernel(void* handle, int which, int precision, int reps, double* ms);

const char* amg_solver_last_error(void);
int amg_solver_last_status(void);
unsigned long long amg_b200_launch_count(void);

/* =====================================================================
 * Kernel-level drop-ins: the reference's internal C entry points with host
 * dcsr_mat in/out, computed on the device.  Outputs are malloc'd as the
 * reference does (free with free()).
 * ===================================================================== */

/* rs_strength (C_amg1/src/rs_classical.c:30-88) */
void rs_strength(const dcsr_mat* A, double theta, dcsr_mat* S, int* max_lam);
/* pmis_coarsening (rs_classical.c:246-371); cf: +1 C, -1 F */
void pmis_coarsening(const dcsr_mat* S, int* cf, int* n_coarse);
/* hmis_coarsening (rs_classical.c:390-611): parallel RS first pass on the device */
void hmis_coarsening(const dcsr_mat* S, int* cf, int* n_coarse);
/* rs_coarsening (rs_classical.c:108-229): parallel RS first pass on the device */
void rs_coarsening(const dcsr_mat* S, int max_lam, int* cf, int* n_coarse);
/* rs_standard_interpolation[_sparsity|_values] (rs_classical.c:643-819) */
void rs_standard_interpolation_sparsity(const dcsr_mat* S, const int* cf, dcsr_mat* P);
void rs_standard_interpolation_values(const dcsr_mat* A, const dcsr_mat* S, const int* cf,
                                      dcsr_mat* P);
void rs_standard_interpolation(const dcsr_mat* A, const dcsr_mat* S, const int* cf,
                               dcsr_mat* P);
/* dcsr_rap (C_amg1/src/sparse_ops.c:102-213): rap_out = R A P */
void dcsr_rap(dcsr_mat* r_in, dcsr_mat* a_in, dcsr_mat* p_in, dcsr_mat* rap_out);
/* SpMV family (sparse_ops.c:19-75) */
void abyvg(const int* ia, const int* ja, const double* a, const double* x, int n, double* y);
void abyvcs(const int* ia, const int* ja, const double* a, const double* x, int n, double* y);
void abyvam(const double* x, const int* ia, const int* ja, const double* a, const double* y,
            int n, double* z);
void vbya(const int* ia, const int* ja, const double* a, const double* x, int n, int m_dim,
          double* y);

/* IC(0) factor (C_amg1/include/amg.h:344-351, ichol.c:12-172) */
typedef struct {
  int n;
  int* ia;
  int* ja;
  double* val;
  int nnz;
} ichol_factor;
void ichol_compute(const dcsr_mat* A, ichol_factor* L);
void ichol_solve(const ichol_factor* L, const double* b, double* x);
void ichol_free(ichol_factor* L);

/* ---------------------------------------------------------------------
 * The reference's internal hierarchy API (C_amg1/include/amg.h:42-124):
 * the same struct layout and function signatures, host pointers, backed by
 * the device solver.  amg_build_hierarchy reads the options from the struct
 * (threshold, min_size, max_levels, nu, smoother, omega_jacobi, coarsening),
 * builds the hierarchy on the GPU and fills every level's host fields (A, P,
 * A_filtered = S, mis, isolated, cf_order, n, n_coarse, l1_diag; the
 * coarsest level's L_ichol) as the reference does; the device hierarchy is
 * found again from the amg_data pointer, so the struct must stay at the same
 * address until amg_free.  Differences: the coarsest level is solved by a
 * dense FP64 Cholesky (not ichol-PCG to 1e-12) and the smoothers are the
 * device's multicolour forms.  No struct field is read back after
 * amg_build_hierarchy: change options through a new build.
 * --------------------------------------------------------------------- */
typedef struct {
  dcsr_mat A;          /* system matrix at this level */
  dcsr_mat P;          /* prolongation (n_fine x n_coarse) */
  dcsr_mat A_filtered; /* strength matrix S */
  int* mis;            /* 1 for a C point, 0 for an F point */
  int* isolated;       /* all zero */
  int* cf_order;       /* C points first, then F points */
  int n;               /* unknowns */
  int n_coarse;        /* coarse points */
  ichol_factor L_ichol;/* IC(0) factor of A (coarsest level only) */
  double* l1_diag;     /* sum_j |a_ij| per row */
} amg_level;

typedef struct {
  amg_level levels[AMG_MAX_LEVELS];
  int num_levels;
  double threshold;
  int min_size;
  int max_levels;
  int maxit_prol;
  int lump;
  int nu;
  int smoother;
  double omega_jacobi;
  int coarsening;
} amg_data;

/* build_hierarchy.c:29-156, :170-242, :245-260 */
void amg_build_hierarchy(amg_data* amg, const dcsr_mat* A);
void amg_rebuild_values(amg_data* amg, const dcsr_mat* A_new);
void amg_free(amg_data* amg);
/* amg_cycle.c:214-217, :250-253, :262-284 (x: initial guess for the slashes) */
void amg_backslash(const amg_data* amg, int lev, const double* b, double* x, int nu);
void amg_fwdslash(const amg_data* amg, int lev, const double* b, double* x, int nu);
void amg_vcycle_precond(const amg_data* amg, const double* g, double* x);
/* amg_ichol_precond.c:51-59.  The first call with a given (A, L) pair loads
 * them onto the device (A as given; A == &amg->levels[0].A reuses the
 * hierarchy's); later calls with the same two structs reuse the copies. */
void amg_ichol_precond(const amg_data* amg, const dcsr_mat* A, const ichol_factor* L,
                       const double* g, double* x);
/* amg_pcg.c:12-101: PCG with a host preconditioner callback; A is loaded
 * onto the device once per call, the vectors live there, and each iteration
 * hands r to the callback on the host and takes z back.  Returns the
 * iteration count, or -maxiter without convergence. */
int amg_pcg(const dcsr_mat* A, const double* b, double* x,
            void (*precond)(const void* data, const double* g, double* Bg),
            const void* precond_data, double tol, int maxiter, int print_level);

/* amg_gauss_seidel_ordered: the computation of the reference's MATLAB
 * gateway cf_gauss_seidel_mex (Matlab_amg/cf_gauss_seidel_mex.c:27-105), which
 * has no C-library counterpart: nu Gauss-Seidel sweeps visiting the rows in
 * `order` (0-based; reversed when backward != 0), x_i = (b_i - sum_{j != i}
 * a_ij x_j) / d_i with d_i the row's first diagonal entry (1 if none), the
 * sum in row order, updated values of the rows visited earlier.  Host CSR
 * and vectors; x holds x0 on entry and the result on exit; bit-identical to
 * the sequential sweep, computed on the device (rows scheduled by dependency
 * level).  Returns AMG_OK or a negative AMG_ERR_* code (AMG_ERR_ARG when
 * order is not a permutation). */
int amg_gauss_seidel_ordered(int n, int nnz, const int* ia, const int* ja, const double* val,
                             const double* b, double* x, const int* order, int nu,
                             int backward);

/* ---------------------------------------------------------------------
 * Vessel networks on the device (device pointers).  The reference assembles
 * in MATLAB (Matlab_amg/read_nwk.m:17-36, ConnectivityMx.m:10-13); these have
 * no counterpart in its C library.
 * --------------------------------------------------------------------- */
typedef struct {
  int n;            /* interior unknowns */
  int nnz;
  int n_nodes;      /* all nodes */
  int* ia;          /* device CSR of A = C_I^T G C_I (columns sorted) */
  int* ja;
  double* val;
  double* rhs;      /* device f = -C_I^T G C_B p_B */
  int* interior_of; /* device: node -> interior unknown, -1 at Dirichlet nodes */
  void* owner;      /* the library's; release with amg_network_system_free */
} amg_network_system;

/* Segments u[s] -- v[s] with conductance g[s] between nodes 0..n_nodes-1;
 * Dirichlet nodes bnd[] (distinct) held at p_bnd[].  Assembles A and f on the
 * device; entries summed in a fixed order (deterministic). */
int amg_network_assemble_device(int n_nodes, int n_seg, const int* d_u, const int* d_v,
                                const double* d_g, int n_bnd, const int* d_bnd,
                                const double* d_pbnd, amg_network_system* out);
void amg_network_system_free(amg_network_system* sys);
/* q[s] = g[s] (P_u - P_v) with P the interior solution p and p_B. */
int amg_network_flows_device(const amg_network_system* sys, int n_seg, const int* d_u,
                             const int* d_v, const double* d_g, const double* d_p,
                             double* d_q);
/* Adjoint of a loss L(p) through A(g) p = f(g): lambda = A^{-1} dL/dp by
 * one more solve on `solver` (a handle built for this A; A is symmetric),
 * then dL/dg[s] = -(Lambda_u - Lambda_v)(P_u - P_v), Lambda = 0 at Dirichlet
 * nodes.  d_lambda (n) receives lambda.  Returns AMG_OK or a negative
 * AMG_ERR_*; *iterations (may be NULL) the adjoint solve's count (-maxiter
 * when it did not converge). */
int amg_network_adjoint_device(void* solver, const amg_network_system* sys, int n_seg,
                               const int* d_u, const int* d_v, const double* d_p,
                               const double* d_dLdp, double tol, int maxiter, double* d_lambda,
                               double* d_dLdg, int* iterations);

/* amg_debug_wait_timeout: no counterpart in the reference (its solver has
 * no waits).  Exercises the give-up path of the sync-free sweeps' bounded
 * waits: runs the IC(0) forward-sweep kernel on an n-row chain (row t
 * depends on row t-1; 2 <= n <= 2^20) whose first row is left out of the
 * schedule, so row 1 waits for a value that is never published.  That wait
 * runs out after limit_ms (0 < limit_ms <= 10000), raises the sweep's abort
 * word, and every other waiting row ends at once.  The expected result is
 * AMG_ERR_SPIN, with the wait record (sweep, row, dependency, time waited)
 * in amg_solver_last_error(); *elapsed_ms (may be NULL) receives the
 * launch's device time, about limit_ms.  The device stays usable.  Any
 * other return means the give-up path is broken. */
int amg_debug_wait_timeout(int n, double limit_ms, double* elapsed_ms);

/* ichol_solve_noalloc: no counterpart in the reference.  Solves L L^T x = b
 * for an IC(0) factor already in device memory (0-based CSR d_ia[n+1],
 * d_ja/d_val[nnz] as ichol_compute returns it, lower triangle, diagonal
 * stored), with the same arithmetic as ichol_solve (bit-identical result),
 * without allocating any memory: for callers that may not call cudaMalloc
 * at the point where they apply the preconditioner (a memory budget owned by
 * another framework, allocation-free callbacks).  Its scratch is a fixed
 * device array of the library, so n <= AMG_NOALLOC_MAX_ROWS (larger n
 * returns AMG_ERR_ARG with a message in amg_solver_last_error()).
 * d_b and d_x are device pointers (n doubles each; they must not overlap);
 * the launch is queued on `stream` (a cudaStream_t, NULL = legacy default
 * stream) and the call returns without synchronising.  The first call on
 * each device looks up that device's scratch address, so make it once before
 * any stream capture.  All calls on a device share the scratch: calls that
 * may overlap in time (other streams, other host threads) race -- order them
 * on one stream.  Returns AMG_OK or a negative AMG_ERR_* code. */
#define AMG_NOALLOC_MAX_ROWS 131072
int ichol_solve_noalloc(int n, const int* d_ia, const int* d_ja, const double* d_val,
                        const double* d_b, double* d_x, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* AMG_B200_H */
