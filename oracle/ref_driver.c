/*
 * ref_driver.c -- test infrastructure: drives the reference C_amg1 library
 * (compiled from its own sources into _ref/) the way its C API does, but with
 * the coarsening selectable, because the reference exposes no setter for it
 * (only its CLI does: C_amg1/test_amg.c:91,199).
 *
 * refdrv_create mirrors amg_solver_create (C_amg1/src/amg_wrapper.c:51-97):
 * copy, symmetrise A=(A+A^T)/2, build the hierarchy with CF-GS smoothing,
 * then the fine-level ichol.  refdrv_solve mirrors amg_solver_solve
 * (amg_wrapper.c:214-225): amg_pcg with the AMG+ichol preconditioner.
 * Timing uses CLOCK_MONOTONIC.
 */
#include "amg.h"
#include <time.h>

typedef struct {
  dcsr_mat A;
  amg_data amg;
  ichol_factor L;
} refdrv;

typedef struct {
  const amg_data* amg;
  const dcsr_mat* A;
  const ichol_factor* L;
} refdrv_ctx;

static double now_s(void) {
  struct timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return ts.tv_sec + 1e-9 * ts.tv_nsec;
}

static void refdrv_precond(const void* data, const REAL* g, REAL* Bg) {
  const refdrv_ctx* c = (const refdrv_ctx*)data;
  amg_ichol_precond(c->amg, c->A, c->L, g, Bg);
}

void* refdrv_create(int n, int nnz, const int* ia, const int* ja,
                    const double* val, double theta, int min_size,
                    int max_levels, int nu, int coarsening) {
  refdrv* d = (refdrv*)calloc(1, sizeof(refdrv));
  dcsr_mat a, at, sum;
  dcsr_mat_alloc(&a, n, n, nnz);
  memcpy(a.ia, ia, (size_t)(n + 1) * sizeof(int));
  memcpy(a.ja, ja, (size_t)nnz * sizeof(int));
  memcpy(a.val, val, (size_t)nnz * sizeof(double));
  dcsr_mat_alloc(&at, n, n, nnz);
  dcsr_transz(&a, NULL, &at);
  dcsr_mat_add(&a, &at, &sum);
  for (int k = 0; k < sum.nnz; k++) sum.val[k] *= 0.5;
  dcsr_mat_free(&a);
  dcsr_mat_free(&at);
  d->A = sum;
  d->amg.threshold = theta;
  d->amg.min_size = min_size;
  d->amg.max_levels = (max_levels > 0 && max_levels <= AMG_MAX_LEVELS)
                          ? max_levels : AMG_MAX_LEVELS;
  d->amg.nu = nu > 0 ? nu : 1;
  d->amg.smoother = SMOOTHER_CF_GS;
  d->amg.omega_jacobi = 0.5;
  d->amg.coarsening = coarsening;
  amg_build_hierarchy(&d->amg, &d->A);
  ichol_compute(&d->A, &d->L);
  return d;
}

int refdrv_solve(void* h, const double* b, double* x, double tol, int maxiter) {
  refdrv* d = (refdrv*)h;
  refdrv_ctx c = {&d->amg, &d->A, &d->L};
  return amg_pcg(&d->A, b, x, refdrv_precond, &c, tol, maxiter, 0);
}

int refdrv_num_levels(void* h) { return ((refdrv*)h)->amg.num_levels; }

/* Level data access for golden dumps: sizes of level k (A, S, P). */
void refdrv_level_sizes(void* h, int k, int* out /* n, nnzA, nnzS, nnzP, ncoarse */) {
  refdrv* d = (refdrv*)h;
  const amg_level* L = &d->amg.levels[k];
  out[0] = L->n;
  out[1] = L->A.nnz;
  int last = (k == d->amg.num_levels - 1);
  out[2] = last ? 0 : L->A_filtered.nnz;
  out[3] = last ? 0 : L->P.nnz;
  out[4] = last ? 0 : L->n_coarse;
}

/* Copy level k's A, S, P and C/F marks (mis) into caller buffers. */
void refdrv_level_copy(void* h, int k, int* a_ia, int* a_ja, double* a_val,
                       int* s_ia, int* s_ja, double* s_val, int* p_ia,
                       int* p_ja, double* p_val, int* mis) {
  refdrv* d = (refdrv*)h;
  const amg_level* L = &d->amg.levels[k];
  int n = L->n;
  memcpy(a_ia, L->A.ia, (size_t)(n + 1) * sizeof(int));
  memcpy(a_ja, L->A.ja, (size_t)L->A.nnz * sizeof(int));
  memcpy(a_val, L->A.val, (size_t)L->A.nnz * sizeof(double));
  if (k == d->amg.num_levels - 1) return;
  memcpy(s_ia, L->A_filtered.ia, (size_t)(n + 1) * sizeof(int));
  memcpy(s_ja, L->A_filtered.ja, (size_t)L->A_filtered.nnz * sizeof(int));
  memcpy(s_val, L->A_filtered.val, (size_t)L->A_filtered.nnz * sizeof(double));
  memcpy(p_ia, L->P.ia, (size_t)(n + 1) * sizeof(int));
  memcpy(p_ja, L->P.ja, (size_t)L->P.nnz * sizeof(int));
  memcpy(p_val, L->P.val, (size_t)L->P.nnz * sizeof(double));
  memcpy(mis, L->mis, (size_t)n * sizeof(int));
}

/* Fine-level ichol factor sizes / copy. */
int refdrv_ichol_nnz(void* h) { return ((refdrv*)h)->L.nnz; }
void refdrv_ichol_copy(void* h, int* ia, int* ja, double* val) {
  refdrv* d = (refdrv*)h;
  memcpy(ia, d->L.ia, (size_t)(d->L.n + 1) * sizeof(int));
  memcpy(ja, d->L.ja, (size_t)d->L.nnz * sizeof(int));
  memcpy(val, d->L.val, (size_t)d->L.nnz * sizeof(double));
}

/* One application of the AMG+ichol preconditioner (amg_ichol_precond.c:51). */
/* refdrv_update mirrors amg_solver_update (C_amg1/src/amg_wrapper.c:114-149):
 * symmetrise the new values, amg_rebuild_values on the kept hierarchy, new
 * fine-level ichol. */
void refdrv_update(void* h, int n, int nnz, const int* ia, const int* ja, const double* val) {
  refdrv* d = (refdrv*)h;
  dcsr_mat a, at, sum;
  dcsr_mat_alloc(&a, n, n, nnz);
  memcpy(a.ia, ia, (size_t)(n + 1) * sizeof(int));
  memcpy(a.ja, ja, (size_t)nnz * sizeof(int));
  memcpy(a.val, val, (size_t)nnz * sizeof(double));
  dcsr_mat_alloc(&at, n, n, nnz);
  dcsr_transz(&a, NULL, &at);
  dcsr_mat_add(&a, &at, &sum);
  for (int k = 0; k < sum.nnz; k++) sum.val[k] *= 0.5;
  dcsr_mat_free(&a);
  dcsr_mat_free(&at);
  ichol_free(&d->L);
  dcsr_mat_free(&d->A);
  d->A = sum;
  amg_rebuild_values(&d->amg, &d->A);
  ichol_compute(&d->A, &d->L);
}

void refdrv_precond_apply(void* h, const double* g, double* x) {
  refdrv* d = (refdrv*)h;
  amg_ichol_precond(&d->amg, &d->A, &d->L, g, x);
}

/* Timed create+solve for the CPU baseline; returns iterations. */
int refdrv_timed(int n, int nnz, const int* ia, const int* ja,
                 const double* val, const double* b, double* x, double theta,
                 int min_size, int nu, int coarsening, double tol, int maxiter,
                 double* t_setup, double* t_solve) {
  double t0 = now_s();
  void* h = refdrv_create(n, nnz, ia, ja, val, theta, min_size, 20, nu,
                          coarsening);
  double t1 = now_s();
  int it = refdrv_solve(h, b, x, tol, maxiter);
  double t2 = now_s();
  *t_setup = t1 - t0;
  *t_solve = t2 - t1;
  refdrv* d = (refdrv*)h;
  ichol_free(&d->L);
  amg_free(&d->amg);
  dcsr_mat_free(&d->A);
  free(d);
  return it;
}

void refdrv_free(void* h) {
  if (!h) return;
  refdrv* d = (refdrv*)h;
  ichol_free(&d->L);
  amg_free(&d->amg);
  dcsr_mat_free(&d->A);
  free(d);
}
