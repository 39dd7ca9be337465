/*
 * amg_oracle.h -- TEST INFRASTRUCTURE ONLY.  CPU restatement of the
 * reference solver's algorithms (liuzhengqi1996/blood_network, C_amg1), used
 * by tests/ and the smoke check as the oracle of the CUDA library, never as
 * the thing measured or shipped.  Every function cites the reference
 * file:line it restates.  Parity of this restatement with the reference is
 * pinned by tests/golden/ (fixtures generated from the compiled reference).
 */
#ifndef AMG_ORACLE_H
#define AMG_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
  int n, m, nnz;
  int* ia;
  int* ja;
  double* val;
} orc_csr;

void orc_csr_free(orc_csr* a);

/* agg_lib.h:120-183 / :186-243 */
void orc_transpose(const orc_csr* a, orc_csr* t);
void orc_add_scaled(const orc_csr* a, const orc_csr* b, double scale, orc_csr* c);
void orc_symmetrize(const orc_csr* a, orc_csr* out);

/* rs_classical.c:30-88 */
void orc_strength(const orc_csr* a, double theta, orc_csr* s, int* max_lam);
/* rs_classical.c:108-229, :246-371, :390-611 ; cf: +1 C, -1 F */
void orc_rs(const orc_csr* s, int max_lam, int* cf, int* nc);
void orc_pmis(const orc_csr* s, int* cf, int* nc);
void orc_hmis(const orc_csr* s, int* cf, int* nc);
/* rs_classical.c:643-819 */
void orc_interp(const orc_csr* a, const orc_csr* s, const int* cf, orc_csr* p);
/* sparse_ops.c:102-213 */
void orc_rap(const orc_csr* r, const orc_csr* a, const orc_csr* p, orc_csr* ac);
/* ichol.c:12-165 */
void orc_ichol(const orc_csr* a, orc_csr* l);
void orc_ichol_solve(const orc_csr* l, const double* b, double* x);
/* sparse_ops.c:19-75 */
void orc_spmv(const orc_csr* a, const double* x, double* y);             /* y = A x */
void orc_residual(const orc_csr* a, const double* b, const double* x, double* r);
void orc_spmv_add(const orc_csr* a, const double* x, double* y);         /* y += A x */
void orc_spmv_t(const orc_csr* a, const double* x, int m, double* y);   /* y = A^T x */

/* Solver handle: amg_wrapper.c:51-268 with selectable coarsening */
void* orc_create(int n, int nnz, const int* ia, const int* ja, const double* val,
                 double theta, int min_size, int max_levels, int nu, int coarsening,
                 int smoother, double omega);
int orc_solve(void* h, const double* b, double* x, double tol, int maxiter);
void orc_precond(void* h, const double* g, double* x);
int orc_num_levels(void* h);
void orc_level_sizes(void* h, int k, int* out5);
void orc_level_copy(void* h, int k, int* a_ia, int* a_ja, double* a_val, int* s_ia,
                    int* s_ja, double* s_val, int* p_ia, int* p_ja, double* p_val, int* cf);
int orc_ichol_nnz(void* h);
void orc_ichol_copy(void* h, int* ia, int* ja, double* val);
void orc_free(void* h);

#ifdef __cplusplus
}
#endif
#endif
