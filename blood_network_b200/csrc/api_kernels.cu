// Kernel-level drop-ins: the reference's internal C entry points, with the
// reference's host dcsr_mat in/out, computed on the device.  Output arrays
// are malloc'd like the reference does, so callers free them with free().
// On error these entry points leave outputs zero-sized and record the
// reason in amg_solver_last_error().
#include "internal.cuh"
#include "ichol.cuh"
#include "solve_kernels.cuh"
#include "../../include/amg_b200.h"

#include <stdlib.h>
#include <string.h>

namespace bn {

static cudaStream_t api_stream() { return cudaStreamPerThread; }

static void to_device(const dcsr_mat* h, CSR& d, cudaStream_t s, bool with_val = true) {
  BN_REQUIRE(h && h->row >= 0 && h->nnz >= 0 && h->ia && (h->nnz == 0 || h->ja), BN_ERR_ARG,
             "invalid dcsr_mat");
  d.alloc(h->row, h->col, h->nnz, s, with_val && h->val);
  d.ia.upload(h->ia, (size_t)h->row + 1);
  if (h->nnz) d.ja.upload(h->ja, h->nnz);
  if (with_val && h->val && h->nnz) d.val.upload(h->val, h->nnz);
}

static void to_host(const CSR& d, dcsr_mat* h, cudaStream_t s) {
  h->row = d.n;
  h->col = d.m;
  h->nnz = d.nnz;
  h->ia = (int*)malloc(sizeof(int) * ((size_t)d.n + 1));
  h->ja = (int*)malloc(sizeof(int) * (size_t)(d.nnz > 0 ? d.nnz : 1));
  h->val = (double*)malloc(sizeof(double) * (size_t)(d.nnz > 0 ? d.nnz : 1));
  d.ia.download(h->ia, (size_t)d.n + 1);
  if (d.nnz) {
    d.ja.download(h->ja, d.nnz);
    d.val.download(h->val, d.nnz);
  }
  BN_CUDA(cudaStreamSynchronize(s));
}

template <class F>
static void api_call(F&& f) {
  try {
    f();
    set_last_error(0, "");
  } catch (const Error& e) {
    set_last_error(e.code, e.what());
  } catch (const std::exception& e) {
    set_last_error(BN_ERR_CUDA, e.what());
  }
}

static void coarsen_api(const dcsr_mat* S, int method, int max_lam, int* cf, int* n_coarse) {
  api_call([&]() {
    cudaStream_t s = api_stream();
    CSR d;
    to_device(S, d, s, false);
    DBuf<int> dcf(S->row > 0 ? S->row : 1, s);
    int nc = coarsen(d, method, max_lam, dcf.p, s);
    dcf.download(cf, S->row);
    BN_CUDA(cudaStreamSynchronize(s));
    *n_coarse = nc;
  });
}

}  // namespace bn

using namespace bn;

BN_API void rs_strength(const dcsr_mat* A, double theta, dcsr_mat* S, int* max_lam) {
  api_call([&]() {
    cudaStream_t s = api_stream();
    CSR dA, dS;
    to_device(A, dA, s);
    strength(dA, theta, dS, max_lam, s);
    to_host(dS, S, s);
  });
}

BN_API void pmis_coarsening(const dcsr_mat* S, int* cf, int* n_coarse) {
  coarsen_api(S, COARSEN_PMIS, 0, cf, n_coarse);
}
BN_API void hmis_coarsening(const dcsr_mat* S, int* cf, int* n_coarse) {
  coarsen_api(S, COARSEN_HMIS, 0, cf, n_coarse);
}
BN_API void rs_coarsening(const dcsr_mat* S, int max_lam, int* cf, int* n_coarse) {
  coarsen_api(S, COARSEN_RS, max_lam, cf, n_coarse);
}

BN_API void rs_standard_interpolation_sparsity(const dcsr_mat* S, const int* cf, dcsr_mat* P) {
  api_call([&]() {
    cudaStream_t s = api_stream();
    const int n = S->row;
    CSR dS, dP;
    to_device(S, dS, s);
    DBuf<int> dcf(n > 0 ? n : 1, s);
    dcf.upload(cf, n);
    int nc = 0;
    for (int i = 0; i < n; i++) nc += (cf[i] == 1);
    // pattern only: values are zero as in the reference
    interpolation_pattern(dS, dcf.p, nc, dP, s);
    dP.val.zero();
    to_host(dP, P, s);
  });
}

BN_API void rs_standard_interpolation_values(const dcsr_mat* A, const dcsr_mat* S, const int* cf,
                                             dcsr_mat* P) {
  api_call([&]() {
    cudaStream_t s = api_stream();
    const int n = A->row;
    CSR dA, dS, dP;
    to_device(A, dA, s);
    to_device(S, dS, s);
    to_device(P, dP, s);
    DBuf<int> dcf(n > 0 ? n : 1, s);
    dcf.upload(cf, n);
    interpolation_values(dA, dS, dcf.p, dP, s);
    dP.val.download(P->val, P->nnz);
    BN_CUDA(cudaStreamSynchronize(s));
  });
}

BN_API void rs_standard_interpolation(const dcsr_mat* A, const dcsr_mat* S, const int* cf,
                                      dcsr_mat* P) {
  api_call([&]() {
    cudaStream_t s = api_stream();
    const int n = A->row;
    CSR dA, dS, dP;
    to_device(A, dA, s);
    to_device(S, dS, s);
    DBuf<int> dcf(n > 0 ? n : 1, s);
    dcf.upload(cf, n);
    int nc = 0;
    for (int i = 0; i < n; i++) nc += (cf[i] == 1);
    interpolation(dA, dS, dcf.p, nc, dP, s);
    to_host(dP, P, s);
  });
}

BN_API void dcsr_rap(dcsr_mat* r_in, dcsr_mat* a_in, dcsr_mat* p_in, dcsr_mat* rap_out) {
  api_call([&]() {
    cudaStream_t s = api_stream();
    CSR dR, dA, dP, dC;
    to_device(r_in, dR, s);
    to_device(a_in, dA, s);
    to_device(p_in, dP, s);
    rap(dR, dA, dP, dC, s);
    to_host(dC, rap_out, s);
  });
}

// ---- SpMV family (host arrays); n rows, nnz = ia[n]
static void spmv_api(int mode, const int* ia, const int* ja, const double* a, const double* x,
                     int n, const double* b, double* y) {
  api_call([&]() {
    cudaStream_t s = api_stream();
    if (n <= 0) return;
    const int nnz = ia[n];
    int m = 0;
    for (int k = 0; k < nnz; k++) m = ja[k] + 1 > m ? ja[k] + 1 : m;
    DBuf<int> dia(n + 1, s), dja(nnz > 0 ? nnz : 1, s);
    DBuf<double> da(nnz > 0 ? nnz : 1, s), dx(m > 0 ? m : 1, s), dy(n, s), db;
    dia.upload(ia, n + 1);
    if (nnz) { dja.upload(ja, nnz); da.upload(a, nnz); }
    if (m) dx.upload(x, m);
    if (mode == SPMV_ADD) dy.upload(y, n);
    if (mode == SPMV_RES) { db.alloc(n, s); db.upload(b, n); }
    DevMat<double> A;
    A.n = n; A.m = m; A.nnz = nnz; A.ia = dia.p; A.ja = dja.p; A.val = da.p;
    // group 0 without long rows: every row summed by one thread in storage
    // order, the reference's sequential order
    spmv<double>(mode, A, dx.p, db.p, dy.p, s);
    dy.download(y, n);
    BN_CUDA(cudaStreamSynchronize(s));
  });
}

BN_API void abyvg(const int* ia, const int* ja, const double* a, const double* x, int n,
                  double* y) {
  spmv_api(SPMV_Y, ia, ja, a, x, n, nullptr, y);
}
BN_API void abyvcs(const int* ia, const int* ja, const double* a, const double* x, int n,
                   double* y) {
  spmv_api(SPMV_ADD, ia, ja, a, x, n, nullptr, y);
}
BN_API void abyvam(const double* x, const int* ia, const int* ja, const double* a,
                   const double* y, int n, double* z) {
  spmv_api(SPMV_RES, ia, ja, a, y, n, x, z);
}

// y = A^T x via the explicit transpose (gather; rows of A^T in increasing
// row order of A, the order the reference's scatter adds in)
BN_API void vbya(const int* ia, const int* ja, const double* a, const double* x, int n,
                 int m_dim, double* y) {
  api_call([&]() {
    cudaStream_t s = api_stream();
    if (m_dim <= 0) return;
    if (n <= 0) { for (int i = 0; i < m_dim; i++) y[i] = 0.0; return; }
    const int nnz = ia[n];
    CSR dA, dT;
    dA.alloc(n, m_dim, nnz, s, true);
    dA.ia.upload(ia, n + 1);
    if (nnz) { dA.ja.upload(ja, nnz); dA.val.upload(a, nnz); }
    transpose(dA, dT, s, true);
    DBuf<double> dx(n, s), dy(m_dim, s);
    dx.upload(x, n);
    DevMat<double> T;
    T.n = m_dim; T.m = n; T.nnz = nnz; T.ia = dT.ia.p; T.ja = dT.ja.p; T.val = dT.val.p;
    spmv<double>(SPMV_Y, T, dx.p, nullptr, dy.p, s);
    dy.download(y, m_dim);
    BN_CUDA(cudaStreamSynchronize(s));
  });
}

// ---- IC(0)
BN_API void ichol_compute(const dcsr_mat* A, ichol_factor* L) {
  memset(L, 0, sizeof(*L));
  api_call([&]() {
    cudaStream_t s = api_stream();
    CSR dA;
    to_device(A, dA, s);
    IChol ic;
    ic.factor(dA, s);
    dcsr_mat h;
    to_host(ic.L, &h, s);
    L->n = h.row;
    L->nnz = h.nnz;
    L->ia = h.ia;
    L->ja = h.ja;
    L->val = h.val;
  });
}

BN_API void ichol_solve(const ichol_factor* L, const double* b, double* x) {
  api_call([&]() {
    cudaStream_t s = api_stream();
    const int n = L->n;
    if (n <= 0) return;
    CSR dL;
    dL.alloc(n, n, L->nnz, s, true);
    dL.ia.upload(L->ia, n + 1);
    if (L->nnz) { dL.ja.upload(L->ja, L->nnz); dL.val.upload(L->val, L->nnz); }
    IChol ic;
    ic.load(std::move(dL), s);
    DBuf<double> db(n, s), dy(n, s), dx(n, s);
    db.upload(b, n);
    ic.solve<double>(db.p, dy.p, dx.p, s);
    dx.download(x, n);
    BN_CUDA(cudaStreamSynchronize(s));
    ic.check_waits(s);
  });
}

BN_API void ichol_free(ichol_factor* L) {
  if (!L) return;
  free(L->ia);
  free(L->ja);
  free(L->val);
  L->ia = L->ja = nullptr;
  L->val = nullptr;
  L->n = L->nnz = 0;
}
