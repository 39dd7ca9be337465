// Vessel network on the device: the Dirichlet-reduced pressure system, the
// segment flows and the adjoint gradient with respect to the conductances.
//
// Assembly (Matlab_amg/read_nwk.m:17-36): with C the segment/node incidence
// (ConnectivityMx.m:10-13), G the segment conductances and I / B the
// interior and Dirichlet nodes,
//   A = C_I^T G C_I,   f = -C_I^T G C_B p_B
// i.e. a_ii = sum of g over the segments at interior node i, a_ij = -sum of
// g over the segments joining interior i and j, f_i = sum of g p_B over the
// segments joining i to a Dirichlet node.  Entries are emitted as
// (row * n + col, value) pairs -- diagonal contributions of the u ends, of
// the v ends, then the (u, v) and (v, u) off-diagonals, each block in
// segment order -- sorted stably by key and each run summed in order; the
// same for f.  The result is deterministic and equals the host assembly of
// the generator (blood_network_b200/network.py), which sums in that order.
//
// Adjoint: for a loss L(p) with A(g) p = f(g), lambda = A^{-1} dL/dp (A is
// symmetric: the same hierarchy solves it) and
//   dL/dg_e = -(Lambda_u - Lambda_v)(P_u - P_v)
// with P the pressures of all nodes (p_B at Dirichlet nodes) and Lambda the
// adjoint extended by 0 at Dirichlet nodes.
#include "solver.cuh"

#include <cub/cub.cuh>
#include <cstring>

namespace bn {
namespace {

__global__ void k_mark_boundary(const int* __restrict__ bnd, int nb, int n_nodes,
                                const double* __restrict__ pb, int* __restrict__ is_b,
                                double* __restrict__ pnode, int* bad) {
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < nb; t += gridDim.x * blockDim.x) {
    const int v = bnd[t];
    if (v < 0 || v >= n_nodes) { atomicExch(bad, 1); continue; }
    is_b[v] = 1;
    pnode[v] = pb[t];
  }
}

__global__ void k_interior_flag(const int* __restrict__ is_b, int n_nodes, int* __restrict__ f) {
  for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < n_nodes; v += gridDim.x * blockDim.x)
    f[v] = is_b[v] ? 0 : 1;
}

__global__ void k_interior_ids(const int* __restrict__ is_b, const int* __restrict__ scan,
                               int n_nodes, int* __restrict__ interior_of) {
  for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < n_nodes; v += gridDim.x * blockDim.x)
    interior_of[v] = is_b[v] ? -1 : scan[v];
}

// per segment: which of the four entry blocks and the rhs get an entry
__global__ void k_seg_flags(const int* __restrict__ u, const int* __restrict__ v, int ns,
                            int n_nodes, const int* __restrict__ io, int* __restrict__ fu,
                            int* __restrict__ fv, int* __restrict__ fb, int* __restrict__ ru,
                            int* __restrict__ rv, int* bad) {
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < ns; s += gridDim.x * blockDim.x) {
    const int a = u[s], b = v[s];
    if (a < 0 || a >= n_nodes || b < 0 || b >= n_nodes) {
      atomicExch(bad, 1);
      fu[s] = fv[s] = fb[s] = ru[s] = rv[s] = 0;
      continue;
    }
    const int ia = io[a], ib = io[b];
    fu[s] = ia >= 0;
    fv[s] = ib >= 0;
    fb[s] = ia >= 0 && ib >= 0;
    ru[s] = ia >= 0 && ib < 0;
    rv[s] = ib >= 0 && ia < 0;
  }
}

__global__ void k_seg_emit(const int* __restrict__ u, const int* __restrict__ v,
                           const double* __restrict__ g, int ns, const int* __restrict__ io,
                           const double* __restrict__ pnode, long long nint,
                           const int* __restrict__ ou, const int* __restrict__ ov,
                           const int* __restrict__ ob, const int* __restrict__ oru,
                           const int* __restrict__ orv, long long base_v, long long base_a,
                           long long base_b, long long rbase_v,
                           unsigned long long* __restrict__ key, double* __restrict__ val,
                           unsigned long long* __restrict__ rkey, double* __restrict__ rval) {
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < ns; s += gridDim.x * blockDim.x) {
    const int ia = io[u[s]], ib = io[v[s]];
    const double gs = g[s];
    if (ia >= 0) {
      key[ou[s]] = (unsigned long long)ia * nint + ia;
      val[ou[s]] = gs;
    }
    if (ib >= 0) {
      key[base_v + ov[s]] = (unsigned long long)ib * nint + ib;
      val[base_v + ov[s]] = gs;
    }
    if (ia >= 0 && ib >= 0) {
      key[base_a + ob[s]] = (unsigned long long)ia * nint + ib;
      val[base_a + ob[s]] = -gs;
      key[base_b + ob[s]] = (unsigned long long)ib * nint + ia;
      val[base_b + ob[s]] = -gs;
    }
    if (ia >= 0 && ib < 0) {
      rkey[oru[s]] = (unsigned long long)ia;
      rval[oru[s]] = xmul(gs, pnode[v[s]]);
    }
    if (ib >= 0 && ia < 0) {
      rkey[rbase_v + orv[s]] = (unsigned long long)ib;
      rval[rbase_v + orv[s]] = xmul(gs, pnode[u[s]]);
    }
  }
}

__global__ void k_run_heads(const unsigned long long* __restrict__ k, long long m,
                            unsigned char* __restrict__ head) {
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < m;
       p += (long long)gridDim.x * blockDim.x)
    head[p] = (p == 0 || k[p] != k[p - 1]) ? 1 : 0;
}

__global__ void k_iota_ll(long long* __restrict__ a, long long m) {
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < m;
       p += (long long)gridDim.x * blockDim.x)
    a[p] = p;
}

// each run (entries with equal key) summed in sorted (= emission) order
__global__ void k_run_sums(const unsigned long long* __restrict__ k, const double* __restrict__ v,
                           const long long* __restrict__ heads, long long nrun, long long m,
                           long long nint, int* __restrict__ rows, int* __restrict__ cols,
                           double* __restrict__ out) {
  for (long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x; r < nrun;
       r += (long long)gridDim.x * blockDim.x) {
    const long long b = heads[r], e = r + 1 < nrun ? heads[r + 1] : m;
    double s = v[b];
    for (long long p = b + 1; p < e; p++) s = xadd(s, v[p]);
    out[r] = s;
    if (rows) rows[r] = (int)(k[b] / nint);
    if (cols) cols[r] = (int)(k[b] % nint);
  }
}

__global__ void k_row_counts(const int* __restrict__ rows, long long nrun, int* __restrict__ cnt) {
  for (long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x; r < nrun;
       r += (long long)gridDim.x * blockDim.x)
    atomicAdd(&cnt[rows[r]], 1);
}

__global__ void k_rhs_scatter(const unsigned long long* __restrict__ k,
                              const double* __restrict__ sums, long long nrun,
                              const long long* __restrict__ heads, double* __restrict__ rhs) {
  for (long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x; r < nrun;
       r += (long long)gridDim.x * blockDim.x)
    rhs[k[heads[r]]] = sums[r];
}

__global__ void k_full_pressure(const int* __restrict__ io, const double* __restrict__ p,
                                const double* __restrict__ pnode, int n_nodes,
                                double* __restrict__ P) {
  for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < n_nodes; v += gridDim.x * blockDim.x)
    P[v] = io[v] >= 0 ? p[io[v]] : pnode[v];
}

__global__ void k_flows(const int* __restrict__ u, const int* __restrict__ v,
                        const double* __restrict__ g, int ns, const double* __restrict__ P,
                        double* __restrict__ q) {
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < ns; s += gridDim.x * blockDim.x)
    q[s] = xmul(g[s], xsub(P[u[s]], P[v[s]]));
}

// dL/dg_e = -(Lambda_u - Lambda_v)(P_u - P_v), Lambda = 0 at Dirichlet nodes
__global__ void k_adjoint_edges(const int* __restrict__ u, const int* __restrict__ v, int ns,
                                const int* __restrict__ io, const double* __restrict__ lam,
                                const double* __restrict__ P, double* __restrict__ out) {
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < ns; s += gridDim.x * blockDim.x) {
    const int a = io[u[s]], b = io[v[s]];
    const double la = a >= 0 ? lam[a] : 0.0, lb = b >= 0 ? lam[b] : 0.0;
    out[s] = -xmul(xsub(la, lb), xsub(P[u[s]], P[v[s]]));
  }
}

__global__ void k_gather_f64(const double* __restrict__ v, const long long* __restrict__ idx,
                             long long m, double* __restrict__ out) {
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < m;
       p += (long long)gridDim.x * blockDim.x)
    out[p] = v[idx[p]];
}

void gather_f64(const double* v, const long long* idx, long long m, double* out, cudaStream_t s) {
  if (m > 0) BN_LAUNCH(k_gather_f64, grid_for(m, 256), 256, 0, s, v, idx, m, out);
}

struct SortedRuns {
  DBuf<unsigned long long> keys;
  DBuf<double> vals;
  DBuf<long long> heads;
  long long nrun = 0;
};

// stable sort of (key, val) by key and the first position of each run
void sort_runs(DBuf<unsigned long long>& key, DBuf<double>& val, long long m, int key_bits,
               SortedRuns& out, cudaStream_t s) {
  out.keys.alloc(m > 0 ? m : 1, s);
  out.vals.alloc(m > 0 ? m : 1, s);
  if (m == 0) {
    out.nrun = 0;
    return;
  }
  DBuf<long long> idx(m, s), idx2(m, s);
  BN_LAUNCH(k_iota_ll, grid_for(m, 256), 256, 0, s, idx.p, m);
  size_t tmp = 0;
  BN_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tmp, key.p, out.keys.p, idx.p, idx2.p, m, 0,
                                          key_bits, s));
  DBuf<unsigned char> t(tmp, s);
  BN_CUDA(cub::DeviceRadixSort::SortPairs(t.p, tmp, key.p, out.keys.p, idx.p, idx2.p, m, 0,
                                          key_bits, s));
  // values in sorted order (a gather through the stable permutation)
  gather_f64(val.p, idx2.p, m, out.vals.p, s);
  DBuf<unsigned char> head(m, s);
  BN_LAUNCH(k_run_heads, grid_for(m, 256), 256, 0, s, out.keys.p, m, head.p);
  DBuf<long long> nsel(1, s);
  out.heads.alloc(m, s);
  tmp = 0;
  BN_CUDA(cub::DeviceSelect::Flagged(nullptr, tmp, idx.p, head.p, out.heads.p, nsel.p, m, s));
  DBuf<unsigned char> t2(tmp, s);
  BN_CUDA(cub::DeviceSelect::Flagged(t2.p, tmp, idx.p, head.p, out.heads.p, nsel.p, m, s));
  out.nrun = read_scalar(nsel.p, s);
}

int bits_for(unsigned long long maxkey) {
  int b = 1;
  while (b < 64 && (maxkey >> b) != 0) b++;
  return b;
}

}  // namespace

// The device system of one network (owner of the arrays handed out through
// amg_network_system).
struct NetSystem {
  cudaStream_t s = 0;
  int n_nodes = 0;
  CSR A;
  DBuf<double> rhs;
  DBuf<int> interior_of;
  DBuf<double> pnode;  // p_B at Dirichlet nodes, 0 elsewhere
};

void assemble_network(int n_nodes, int ns, const int* u, const int* v, const double* g, int nb,
                      const int* bnd, const double* pb, NetSystem& S) {
  cudaStream_t s = S.s;
  S.n_nodes = n_nodes;
  DBuf<int> is_b(n_nodes > 0 ? n_nodes : 1, s), bad(1, s), flag((size_t)n_nodes + 1, s);
  is_b.zero();
  bad.zero();
  S.pnode.alloc(n_nodes > 0 ? n_nodes : 1, s);
  S.pnode.zero();
  if (nb > 0)
    BN_LAUNCH(k_mark_boundary, grid_for(nb, 256), 256, 0, s, bnd, nb, n_nodes, pb, is_b.p,
              S.pnode.p, bad.p);
  BN_REQUIRE(read_scalar(bad.p, s) == 0, BN_ERR_ARG, "network: Dirichlet node id out of range");
  flag.zero();
  BN_LAUNCH(k_interior_flag, grid_for(n_nodes, 256), 256, 0, s, is_b.p, n_nodes, flag.p);
  const int n = scan_counts(flag.p, n_nodes, s);  // flag now holds interior ids
  BN_REQUIRE(n > 0, BN_ERR_ARG, "network: no interior node");
  S.interior_of.alloc(n_nodes, s);
  BN_LAUNCH(k_interior_ids, grid_for(n_nodes, 256), 256, 0, s, is_b.p, flag.p, n_nodes,
            S.interior_of.p);
  // offsets of every segment's entries in the five emission blocks
  DBuf<int> fu((size_t)ns + 1, s), fv((size_t)ns + 1, s), fb((size_t)ns + 1, s),
      ru((size_t)ns + 1, s), rv((size_t)ns + 1, s);
  for (auto* b : {&fu, &fv, &fb, &ru, &rv}) b->zero();
  if (ns > 0)
    BN_LAUNCH(k_seg_flags, grid_for(ns, 256), 256, 0, s, u, v, ns, n_nodes, S.interior_of.p,
              fu.p, fv.p, fb.p, ru.p, rv.p, bad.p);
  BN_REQUIRE(read_scalar(bad.p, s) == 0, BN_ERR_ARG, "network: segment end out of range");
  const long long nu_ = scan_counts(fu.p, ns, s), nv_ = scan_counts(fv.p, ns, s);
  const long long nb_ = scan_counts(fb.p, ns, s);
  const long long nru = scan_counts(ru.p, ns, s), nrv = scan_counts(rv.p, ns, s);
  const long long m = nu_ + nv_ + 2 * nb_, mr = nru + nrv;
  DBuf<unsigned long long> key(m > 0 ? m : 1, s), rkey(mr > 0 ? mr : 1, s);
  DBuf<double> val(m > 0 ? m : 1, s), rval(mr > 0 ? mr : 1, s);
  if (ns > 0)
    BN_LAUNCH(k_seg_emit, grid_for(ns, 256), 256, 0, s, u, v, g, ns, S.interior_of.p, S.pnode.p,
              (long long)n, fu.p, fv.p, fb.p, ru.p, rv.p, nu_, nu_ + nv_, nu_ + nv_ + nb_, nru,
              key.p, val.p, rkey.p, rval.p);
  // matrix: runs -> CSR (the diagonal is always present: every interior node
  // has a segment, else its row would be empty and the system singular)
  SortedRuns R;
  sort_runs(key, val, m, bits_for((unsigned long long)n * n), R, s);
  DBuf<int> rows(R.nrun > 0 ? R.nrun : 1, s);
  S.A.n = S.A.m = n;
  S.A.nnz = (int)R.nrun;
  BN_REQUIRE(R.nrun < (1LL << 31), BN_ERR_ARG, "network: too many entries for int32 indices");
  S.A.ja.alloc(R.nrun > 0 ? R.nrun : 1, s);
  S.A.val.alloc(R.nrun > 0 ? R.nrun : 1, s);
  if (R.nrun > 0)
    BN_LAUNCH(k_run_sums, grid_for(R.nrun, 256), 256, 0, s, R.keys.p, R.vals.p, R.heads.p, R.nrun,
              m, (long long)n, rows.p, S.A.ja.p, S.A.val.p);
  DBuf<int> cnt((size_t)n + 1, s);
  cnt.zero();
  if (R.nrun > 0)
    BN_LAUNCH(k_row_counts, grid_for(R.nrun, 256), 256, 0, s, rows.p, R.nrun, cnt.p);
  scan_counts(cnt.p, n, s);
  S.A.ia = std::move(cnt);
  // right-hand side
  S.rhs.alloc(n, s);
  S.rhs.zero();
  SortedRuns Q;
  sort_runs(rkey, rval, mr, bits_for((unsigned long long)n), Q, s);
  if (Q.nrun > 0) {
    DBuf<double> sums(Q.nrun, s);
    BN_LAUNCH(k_run_sums, grid_for(Q.nrun, 256), 256, 0, s, Q.keys.p, Q.vals.p, Q.heads.p,
              Q.nrun, mr, (long long)n, nullptr, nullptr, sums.p);
    BN_LAUNCH(k_rhs_scatter, grid_for(Q.nrun, 256), 256, 0, s, Q.keys.p, sums.p, Q.nrun,
              Q.heads.p, S.rhs.p);
  }
  BN_CUDA(cudaStreamSynchronize(s));
}

void full_pressure(const NetSystem& S, const double* p, double* P) {
  BN_LAUNCH(k_full_pressure, grid_for(S.n_nodes, 256), 256, 0, S.s, S.interior_of.p, p,
            S.pnode.p, S.n_nodes, P);
}

}  // namespace bn

using bn::NetSystem;

BN_API int amg_network_assemble_device(int n_nodes, int n_seg, const int* d_u, const int* d_v,
                                       const double* d_g, int n_bnd, const int* d_bnd,
                                       const double* d_pbnd, amg_network_system* out) {
  if (!out) {
    bn::set_last_error(bn::BN_ERR_ARG, "amg_network_assemble_device: NULL output");
    return bn::BN_ERR_ARG;
  }
  memset(out, 0, sizeof(*out));
  return bn::guarded([&]() {
    BN_REQUIRE(n_nodes > 0 && n_seg >= 0 && n_bnd >= 0 && (n_seg == 0 || (d_u && d_v && d_g)) &&
                   (n_bnd == 0 || (d_bnd && d_pbnd)),
               bn::BN_ERR_ARG, "amg_network_assemble_device: invalid arguments");
    std::unique_ptr<NetSystem> S(new NetSystem());
    BN_CUDA(cudaStreamCreateWithFlags(&S->s, cudaStreamNonBlocking));
    bn::assemble_network(n_nodes, n_seg, d_u, d_v, d_g, n_bnd, d_bnd, d_pbnd, *S);
    out->n = S->A.n;
    out->nnz = S->A.nnz;
    out->n_nodes = n_nodes;
    out->ia = S->A.ia.p;
    out->ja = S->A.ja.p;
    out->val = S->A.val.p;
    out->rhs = S->rhs.p;
    out->interior_of = S->interior_of.p;
    out->owner = S.release();
    bn::set_last_error(0, "");
    return 0;
  }, bn::BN_ERR_CUDA);
}

BN_API void amg_network_system_free(amg_network_system* sys) {
  if (!sys || !sys->owner) return;
  NetSystem* S = (NetSystem*)sys->owner;
  cudaStream_t s = S->s;
  delete S;  // frees on its stream
  cudaStreamSynchronize(s);
  cudaStreamDestroy(s);
  memset(sys, 0, sizeof(*sys));
}

BN_API int amg_network_flows_device(const amg_network_system* sys, int n_seg, const int* d_u,
                                    const int* d_v, const double* d_g, const double* d_p,
                                    double* d_q) {
  if (!sys || !sys->owner) {
    bn::set_last_error(bn::BN_ERR_ARG, "amg_network_flows_device: no system");
    return bn::BN_ERR_ARG;
  }
  NetSystem& S = *(NetSystem*)sys->owner;
  return bn::guarded([&]() {
    if (n_seg == 0) return 0;
    BN_REQUIRE(d_u && d_v && d_g && d_p && d_q, bn::BN_ERR_ARG,
               "amg_network_flows_device: NULL pointer");
    bn::DBuf<double> P(S.n_nodes, S.s);
    bn::full_pressure(S, d_p, P.p);
    BN_LAUNCH(bn::k_flows, bn::grid_for(n_seg, 256), 256, 0, S.s, d_u, d_v, d_g, n_seg, P.p, d_q);
    BN_CUDA(cudaStreamSynchronize(S.s));
    bn::set_last_error(0, "");
    return 0;
  }, bn::BN_ERR_CUDA);
}

BN_API int amg_network_adjoint_device(void* solver, const amg_network_system* sys, int n_seg,
                                      const int* d_u, const int* d_v, const double* d_p,
                                      const double* d_dLdp, double tol, int maxiter,
                                      double* d_lambda, double* d_dLdg, int* iterations) {
  if (!solver || !sys || !sys->owner) {
    bn::set_last_error(bn::BN_ERR_ARG, "amg_network_adjoint_device: no solver or system");
    return bn::BN_ERR_ARG;
  }
  NetSystem& S = *(NetSystem*)sys->owner;
  bn::Solver& V = *(bn::Solver*)solver;
  int it = 0;
  const int rc = bn::guarded([&]() {
    BN_REQUIRE(d_p && d_dLdp && d_lambda && (n_seg == 0 || (d_u && d_v && d_dLdg)),
               bn::BN_ERR_ARG, "amg_network_adjoint_device: NULL pointer");
    BN_REQUIRE(V.n() == S.A.n, bn::BN_ERR_ARG,
               "amg_network_adjoint_device: solver and system sizes differ");
    // lambda = A^{-1} dL/dp with the same hierarchy (A symmetric), x0 = 0
    BN_CUDA(cudaMemsetAsync(d_lambda, 0, sizeof(double) * (size_t)S.A.n, S.s));
    BN_CUDA(cudaStreamSynchronize(S.s));
    it = amg_solver_solve_device(solver, d_dLdp, d_lambda, tol, maxiter, 0);
    const int st = amg_solver_last_status();
    BN_REQUIRE(st == 0 || st == bn::BN_ERR_NOT_CONVERGED, st, amg_solver_last_error());
    if (n_seg > 0) {
      bn::DBuf<double> P(S.n_nodes, S.s);
      bn::full_pressure(S, d_p, P.p);
      BN_LAUNCH(bn::k_adjoint_edges, bn::grid_for(n_seg, 256), 256, 0, S.s, d_u, d_v, n_seg,
                S.interior_of.p, d_lambda, P.p, d_dLdg);
      BN_CUDA(cudaStreamSynchronize(S.s));
    }
    bn::set_last_error(0, "");
    return 0;
  }, bn::BN_ERR_CUDA);
  if (iterations) *iterations = it;
  return rc;
}
