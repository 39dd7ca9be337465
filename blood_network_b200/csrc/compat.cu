// The reference's internal hierarchy API on the device solver:
// amg_build_hierarchy / amg_rebuild_values / amg_free (build_hierarchy.c),
// amg_backslash / amg_fwdslash / amg_vcycle_precond (amg_cycle.c),
// amg_ichol_precond (amg_ichol_precond.c) and amg_pcg (amg_pcg.c).
//
// The caller's amg_data keeps the reference's layout and gets host copies of
// every level (so code that inspects the hierarchy keeps working); the device
// solver behind it is found through a registry keyed by the struct's
// address.  Vectors cross in the reference's (natural) numbering and are
// permuted into the solver's colour-ordered numbering on the device.
#include "solver.cuh"

#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <unordered_map>

namespace bn {
namespace {

struct Entry {
  Solver* S = nullptr;
  // amg_ichol_precond's (A, L) pair currently on the device
  const dcsr_mat* A = nullptr;
  const ichol_factor* L = nullptr;
};

std::mutex g_mu;
std::unordered_map<const amg_data*, Entry> g_reg;

Entry* find_entry(const amg_data* amg) {
  std::lock_guard<std::mutex> lock(g_mu);
  auto it = g_reg.find(amg);
  return it == g_reg.end() ? nullptr : &it->second;
}

template <class T>
T* host_copy(const DBuf<T>& d, size_t n, cudaStream_t s) {
  T* h = (T*)malloc(sizeof(T) * (n > 0 ? n : 1));
  BN_REQUIRE(h, BN_ERR_OOM, "host allocation failed");
  if (n) d.download(h, n);
  (void)s;
  return h;
}

void to_host_csr(const CSR& M, dcsr_mat* out, cudaStream_t s) {
  out->row = M.n;
  out->col = M.m;
  out->nnz = M.nnz;
  out->ia = host_copy(M.ia, (size_t)M.n + 1, s);
  out->ja = host_copy(M.ja, (size_t)M.nnz, s);
  out->val = host_copy(M.val, (size_t)M.nnz, s);
}

void free_csr(dcsr_mat* m) {
  free(m->ia);
  free(m->ja);
  free(m->val);
  memset(m, 0, sizeof(*m));
}

void free_levels(amg_data* amg) {
  for (int k = 0; k < amg->num_levels && k < AMG_MAX_LEVELS; k++) {
    amg_level* L = &amg->levels[k];
    free_csr(&L->A);
    free_csr(&L->P);
    free_csr(&L->A_filtered);
    free(L->mis);
    free(L->isolated);
    free(L->cf_order);
    free(L->l1_diag);
    free(L->L_ichol.ia);
    free(L->L_ichol.ja);
    free(L->L_ichol.val);
    memset(L, 0, sizeof(*L));
  }
  amg->num_levels = 0;
}

// host fields of every level, as build_hierarchy.c fills them
void fill_levels(amg_data* amg, Solver& S) {
  cudaStream_t s = S.s;
  const int nl = (int)S.lv.size();
  for (int k = 0; k < nl; k++) {
    Level& L = *S.lv[k];
    amg_level* H = &amg->levels[k];
    memset(H, 0, sizeof(*H));
    const int n = L.A.n;
    H->n = n;
    to_host_csr(L.A, &H->A, s);
    DBuf<double> l1(n > 0 ? n : 1, s);
    l1_row_norms(L.A, l1.p, s);
    H->l1_diag = host_copy(l1, (size_t)n, s);
    if (k < nl - 1) {
      H->n_coarse = L.n_coarse;
      to_host_csr(L.P, &H->P, s);
      to_host_csr(L.S, &H->A_filtered, s);
      int* cf = host_copy(L.cf, (size_t)n, s);
      BN_CUDA(cudaStreamSynchronize(s));
      H->mis = (int*)malloc(sizeof(int) * (n > 0 ? n : 1));
      H->isolated = (int*)calloc(n > 0 ? n : 1, sizeof(int));
      H->cf_order = (int*)malloc(sizeof(int) * (n > 0 ? n : 1));
      BN_REQUIRE(H->mis && H->isolated && H->cf_order, BN_ERR_OOM, "host allocation failed");
      int q = 0;
      for (int i = 0; i < n; i++) {
        H->mis[i] = cf[i] == 1 ? 1 : 0;
        if (cf[i] == 1) H->cf_order[q++] = i;
      }
      for (int i = 0; i < n; i++)
        if (cf[i] != 1) H->cf_order[q++] = i;
      free(cf);
    } else {  // coarsest: its IC(0) factor (ichol_compute)
      IChol ic;
      ic.factor(L.A, s);
      dcsr_mat f;
      to_host_csr(ic.L, &f, s);
      H->L_ichol.n = f.row;
      H->L_ichol.nnz = f.nnz;
      H->L_ichol.ia = f.ia;
      H->L_ichol.ja = f.ja;
      H->L_ichol.val = f.val;
    }
  }
  BN_CUDA(cudaStreamSynchronize(s));
  amg->num_levels = nl;
}

amg_b200_options options_of(const amg_data* amg) {
  amg_b200_options o;
  amg_b200_default_options(&o);
  o.threshold = amg->threshold;
  o.min_size = amg->min_size;
  o.max_levels = amg->max_levels;
  o.nu = amg->nu > 0 ? amg->nu : 1;
  o.smoother = amg->smoother;
  o.omega = amg->omega_jacobi;
  o.coarsening = amg->coarsening;
  o.precision = AMG_PREC_FP64;
  o.stop = AMG_STOP_BNORM;
  return o;
}

// host vector (natural numbering of level l) -> device, solve numbering
void to_solve(Solver& S, int l, const double* h, double* d, double* tmp) {
  const int n = S.lv[l]->A.n;
  BN_CUDA(cudaMemcpyAsync(tmp, h, sizeof(double) * n, cudaMemcpyHostToDevice, S.s));
  vpermute<double>(tmp, S.lv[l]->perm.p, n, d, false, S.s);
}

void from_solve(Solver& S, int l, const double* d, double* h, double* tmp) {
  const int n = S.lv[l]->A.n;
  vpermute<double>(d, S.lv[l]->perm.p, n, tmp, true, S.s);
  BN_CUDA(cudaMemcpyAsync(h, tmp, sizeof(double) * n, cudaMemcpyDeviceToHost, S.s));
  BN_CUDA(cudaStreamSynchronize(S.s));
}

const char* coarsen_name(int c) {
  return c == COARSEN_PMIS ? "PMIS" : (c == COARSEN_HMIS ? "HMIS" : "RS");
}

void report(const char* what) {
  fprintf(stderr, "%s: %s\n", what, amg_solver_last_error());
}

}  // namespace
}  // namespace bn

using bn::Entry;
using bn::Solver;

BN_API void amg_build_hierarchy(amg_data* amg, const dcsr_mat* A) {
  if (!amg || !A) {
    bn::set_last_error(bn::BN_ERR_ARG, "amg_build_hierarchy: NULL argument");
    return;
  }
  int rc = bn::guarded([&]() {
    amg_b200_options o = bn::options_of(amg);
    fprintf(stderr, "Building %s hierarchy on the GPU (threshold=%.2f, min_size=%d)\n",
            bn::coarsen_name(o.coarsening), o.threshold, o.min_size);
    Solver* S = bn::make_solver(A->row, A->nnz, A->ia, A->ja, A->val, &o, false, false);
    {
      std::lock_guard<std::mutex> lock(bn::g_mu);
      auto it = bn::g_reg.find(amg);
      if (it != bn::g_reg.end()) delete it->second.S;
      bn::g_reg[amg] = Entry{S, nullptr, nullptr};
    }
    bn::fill_levels(amg, *S);
    for (int k = 0; k < amg->num_levels; k++)
      fprintf(stderr, "  Level %d: n = %d, nnz = %d\n", k + 1, amg->levels[k].n,
              amg->levels[k].A.nnz);
    bn::set_last_error(0, "");
    return 0;
  }, -1);
  if (rc) bn::report("amg_build_hierarchy");
}

BN_API void amg_rebuild_values(amg_data* amg, const dcsr_mat* A_new) {
  Entry* e = amg ? bn::find_entry(amg) : nullptr;
  if (!e || !A_new) {
    bn::set_last_error(bn::BN_ERR_ARG, "amg_rebuild_values: no hierarchy for this amg_data");
    bn::report("amg_rebuild_values");
    return;
  }
  int rc = bn::guarded([&]() {
    Solver& S = *e->S;
    BN_CUDA(cudaSetDevice(S.device));
    BN_REQUIRE(A_new->row == S.lv[0]->A.n && A_new->nnz == S.lv[0]->A.nnz, bn::BN_ERR_ARG,
               "amg_rebuild_values: sparsity differs from the hierarchy");
    bn::CSR A;
    bn::upload_csr(S, A_new->row, A_new->nnz, A_new->ia, A_new->ja, A_new->val, false, false, A);
    S.rebuild_values(std::move(A));
    e->A = nullptr;
    e->L = nullptr;
    bn::free_levels(amg);
    bn::fill_levels(amg, S);
    bn::set_last_error(0, "");
    return 0;
  }, -1);
  if (rc) bn::report("amg_rebuild_values");
}

BN_API void amg_free(amg_data* amg) {
  if (!amg) return;
  Solver* S = nullptr;
  {
    std::lock_guard<std::mutex> lock(bn::g_mu);
    auto it = bn::g_reg.find(amg);
    if (it != bn::g_reg.end()) {
      S = it->second.S;
      bn::g_reg.erase(it);
    }
  }
  if (S) {
    cudaSetDevice(S->device);
    delete S;
  }
  bn::free_levels(amg);
}

// one level-l slash with host vectors; forward: backslash, else fwdslash
static void slash(const amg_data* amg, int lev, const double* b, double* x, int nu, bool back,
                  const char* what) {
  Entry* e = amg ? bn::find_entry(amg) : nullptr;
  if (!e || !b || !x) {
    bn::set_last_error(bn::BN_ERR_ARG, std::string(what) + ": no hierarchy or NULL vector");
    bn::report(what);
    return;
  }
  int rc = bn::guarded([&]() {
    Solver& S = *e->S;
    BN_CUDA(cudaSetDevice(S.device));
    BN_REQUIRE(lev >= 0 && lev < (int)S.lv.size(), bn::BN_ERR_ARG, "level out of range");
    const int n = S.lv[lev]->A.n;
    bn::DBuf<double> db(n, S.s), dx(n, S.s), tmp(n, S.s);
    bn::to_solve(S, lev, b, db.p, tmp.p);
    bn::to_solve(S, lev, x, dx.p, tmp.p);
    const int keep = S.opt.nu;
    S.opt.nu = nu > 0 ? nu : 1;
    if (back) S.backslash_at(lev, db.p, dx.p);
    else S.fwdslash_at(lev, db.p, dx.p);
    S.opt.nu = keep;
    bn::from_solve(S, lev, dx.p, x, tmp.p);
    bn::set_last_error(0, "");
    return 0;
  }, -1);
  if (rc) bn::report(what);
}

BN_API void amg_backslash(const amg_data* amg, int lev, const double* b, double* x, int nu) {
  slash(amg, lev, b, x, nu, true, "amg_backslash");
}

BN_API void amg_fwdslash(const amg_data* amg, int lev, const double* b, double* x, int nu) {
  slash(amg, lev, b, x, nu, false, "amg_fwdslash");
}

BN_API void amg_vcycle_precond(const amg_data* amg, const double* g, double* x) {
  Entry* e = amg ? bn::find_entry(amg) : nullptr;
  if (!e || !g || !x) {
    bn::set_last_error(bn::BN_ERR_ARG, "amg_vcycle_precond: no hierarchy or NULL vector");
    bn::report("amg_vcycle_precond");
    return;
  }
  int rc = bn::guarded([&]() {
    Solver& S = *e->S;
    BN_CUDA(cudaSetDevice(S.device));
    const int n = S.lv[0]->A.n;
    bn::DBuf<double> dg(n, S.s), dx(n, S.s), tmp(n, S.s);
    bn::to_solve(S, 0, g, dg.p, tmp.p);
    const int keep = S.opt.nu;
    S.opt.nu = amg->nu > 0 ? amg->nu : 1;
    S.vcycle_apply(dg.p, dx.p);
    S.opt.nu = keep;
    bn::from_solve(S, 0, dx.p, x, tmp.p);
    bn::set_last_error(0, "");
    return 0;
  }, -1);
  if (rc) bn::report("amg_vcycle_precond");
}

BN_API void amg_ichol_precond(const amg_data* amg, const dcsr_mat* A, const ichol_factor* L,
                              const double* g, double* x) {
  Entry* e = amg ? bn::find_entry(amg) : nullptr;
  if (!e || !A || !L || !g || !x) {
    bn::set_last_error(bn::BN_ERR_ARG, "amg_ichol_precond: no hierarchy or NULL argument");
    bn::report("amg_ichol_precond");
    return;
  }
  int rc = bn::guarded([&]() {
    Solver& S = *e->S;
    BN_CUDA(cudaSetDevice(S.device));
    const int n = S.lv[0]->A.n;
    BN_REQUIRE(A->row == n && L->n == n, bn::BN_ERR_ARG,
               "amg_ichol_precond: A or L does not match the hierarchy");
    if (e->A != A || e->L != L) {  // load this (A, L) pair
      bn::CSR Lf;
      Lf.alloc(n, n, L->nnz, S.s, true);
      Lf.ia.upload(L->ia, (size_t)n + 1);
      if (L->nnz) {
        Lf.ja.upload(L->ja, (size_t)L->nnz);
        Lf.val.upload(L->val, (size_t)L->nnz);
      }
      if (A == &amg->levels[0].A) {
        S.use_matrix_and_factor(nullptr, std::move(Lf));
      } else {
        bn::CSR Ad;
        bn::upload_csr(S, A->row, A->nnz, A->ia, A->ja, A->val, false, false, Ad);
        S.use_matrix_and_factor(&Ad, std::move(Lf));
      }
      e->A = A;
      e->L = L;
    }
    bn::DBuf<double> dg(n, S.s), dx(n, S.s), tmp(n, S.s);
    bn::to_solve(S, 0, g, dg.p, tmp.p);
    const int keep = S.opt.nu;
    S.opt.nu = amg->nu > 0 ? amg->nu : 1;
    S.precond(dg.p, dx.p);
    S.opt.nu = keep;
    S.ic.check_waits(S.s);
    bn::from_solve(S, 0, dx.p, x, tmp.p);
    bn::set_last_error(0, "");
    return 0;
  }, -1);
  if (rc) bn::report("amg_ichol_precond");
}

BN_API int amg_pcg(const dcsr_mat* A, const double* b, double* x,
                   void (*precond)(const void* data, const double* g, double* Bg),
                   const void* precond_data, double tol, int maxiter, int print_level) {
  if (!A || !b || !x || !precond) {
    bn::set_last_error(bn::BN_ERR_ARG, "amg_pcg: NULL argument");
    return bn::BN_ERR_ARG;
  }
  int result = 0;
  int rc = bn::guarded([&]() {
    BN_REQUIRE(A->row > 0, bn::BN_ERR_ARG, "amg_pcg: empty matrix");
    const int n = A->row;
    Solver S;  // only for its stream and the device upload helper
    int dev = 0;
    BN_CUDA(cudaGetDevice(&dev));
    S.device = dev;
    BN_CUDA(cudaStreamCreateWithFlags(&S.s, cudaStreamNonBlocking));
    struct StreamGuard {
      cudaStream_t s;
      ~StreamGuard() { cudaStreamDestroy(s); }
    } sg{S.s};
    cudaStream_t s = S.s;
    bn::CSR dA;
    bn::upload_csr(S, n, A->nnz, A->ia, A->ja, A->val, false, false, dA);
    bn::RowLayout lay;
    bn::analyze_rows(dA, lay, s);
    bn::DevMat<double> M;
    M.n = dA.n; M.m = dA.m; M.nnz = dA.nnz; M.ia = dA.ia.p; M.ja = dA.ja.p; M.val = dA.val.p;
    M.group = lay.group; M.lrows = lay.lrows.p; M.nlong = lay.nlong;
    bn::DBuf<double> db(n, s), dx(n, s), r(n, s), z(n, s), p(n, s), ap(n, s);
    bn::DBuf<double> part0(bn::kRedBlocks > bn::spmv_partials(n, lay.nlong)
                               ? bn::kRedBlocks : bn::spmv_partials(n, lay.nlong), s);
    bn::DBuf<double> part1(bn::kRedBlocks, s), sc(4, s);
    std::vector<double> hr(n), hz(n);
    db.upload(b, n);
    dx.upload(x, n);
    auto dot = [&](const double* u, const double* v) {  // u . v on the device
      bn::dot_partials<double>(u, v, (const double*)nullptr, n, part0.p, nullptr, s);
      bn::reduce_partials(part0.p, bn::kRedBlocks, sc.p, s);
      return bn::read_scalar(sc.p, s);
    };
    auto apply_precond = [&]() {  // z = B r through the host callback
      r.download(hr.data(), n);
      BN_CUDA(cudaStreamSynchronize(s));
      precond(precond_data, hr.data(), hz.data());
      z.upload(hz.data(), n);
    };
    auto axpy = [&](double* y, const double* u, double a) {  // y += a u
      bn::vaxpy(y, u, a, n, s);
    };
    bn::spmv<double>(bn::SPMV_RES, M, dx.p, db.p, r.p, s);  // r = b - A x
    double bnorm = std::sqrt(dot(db.p, db.p));
    if (bnorm == 0.0) bnorm = 1.0;
    apply_precond();
    BN_CUDA(cudaMemcpyAsync(p.p, z.p, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
    double rz_old = dot(r.p, z.p);
    const double rz0 = rz_old;
    double rnorm = std::sqrt(dot(r.p, r.p));
    if (print_level >= 1) {
      fprintf(stderr, "  %4s  %8s  %8s  %6s\n", "iter", "||r||_B", "rel", "rho");
      fprintf(stderr, "  %4d  %8.2e  %8.2e\n", 0, std::sqrt(rz0), 1.0);
    }
    int iter;
    for (iter = 1; iter <= maxiter; iter++) {
      bn::spmv<double>(bn::SPMV_Y, M, p.p, nullptr, ap.p, s);
      const double pap = dot(p.p, ap.p);
      const double alpha = rz_old / pap;
      axpy(dx.p, p.p, alpha);
      axpy(r.p, ap.p, -alpha);
      rnorm = std::sqrt(dot(r.p, r.p));
      apply_precond();
      const double rz_new = dot(r.p, z.p);
      const double bnorm_rel = std::sqrt(rz_new / rz0);
      if (print_level >= 1)
        fprintf(stderr, "  %4d  %8.2e  %8.2e  %6.4f\n", iter, std::sqrt(rz_new), bnorm_rel,
                rz_new / rz_old);
      if (bnorm_rel < tol) break;
      const double beta = rz_new / rz_old;
      rz_old = rz_new;
      bn::vxpby(p.p, z.p, beta, n, s);  // p = z + beta p
    }
    if (iter > maxiter) {
      fprintf(stderr, "  PCG: no convergence after %d iterations, relres = %.2e\n", maxiter,
              rnorm / bnorm);
      iter = -maxiter;
    }
    dx.download(x, n);
    BN_CUDA(cudaStreamSynchronize(s));
    S.s = 0;  // the guard destroys the stream
    result = iter;
    bn::set_last_error(0, "");
    return 0;
  }, -1);
  return rc ? bn::BN_ERR_CUDA : result;
}
