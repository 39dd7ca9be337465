// IC(0) on the device: factorization and the two triangular solves.
//
// Follows ichol_compute / ichol_solve (C_amg1/src/ichol.c:12-165):
//  * L takes A's lower triangle (j <= i) in A's in-row order.
//  * Row i, in storage order, for each k < i:
//      L(i,k) = (w_k - sum_{j in pre(k), j in row i} w_j L(k,j)) / L(k,k)
//    where pre(k) is the leading part of row k before its first column
//    >= k (the reference breaks there) and w holds row i's current values.
//    Then L(i,i) = sqrt(w_i - sum_{j in pre(i)} w_j^2), a non-positive
//    pivot becomes 1e-14 (:102).
//  * Forward: y_i = (b_i - sum_{j<i} L(i,j) y_j) / L(i,i), row order.
//  * Backward (column oriented in the reference): x_j = (y_j - sum over
//    i > j, in decreasing i, of L(i,j) x_i) / L(j,j).
// Every row is computed by one thread in that exact operation order, so the
// factor and the solves are bit-identical to the reference.
//
// Parallel schedule: row i depends on the rows k < i of its own pattern.
// Dependency levels come from a Kahn frontier sweep (level l = rows whose
// dependencies all lie in levels < l); rows are stored and processed in
// level order.  The factorization runs one launch per level; runs of
// consecutive narrow levels (tree parts, lattice corners) are batched into a
// single 1024-thread block that steps through them with __syncthreads().
// The triangular solves run as one sync-free launch per sweep (rows wait on
// their dependencies' values, every wait bounded), or, selectable, as level
// launches or one cooperative launch with a grid barrier per level.
#include "ichol.cuh"
#include "flags.cuh"

#include <cstdlib>
#include <cstring>
#include <string>

#include <cooperative_groups.h>
#include <cub/cub.cuh>

namespace bn {

constexpr int kNarrow = 2048;     // levels up to this width are batched
constexpr int kBatchThreads = 1024;

// ---------------------------------------------------------------- pattern
__global__ void k_lower_count(const int* __restrict__ ia, const int* __restrict__ ja, int n,
                              int* __restrict__ cnt) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    int c = 0;
    for (int k = ia[i]; k < ia[i + 1]; k++) c += (ja[k] <= i);
    cnt[i] = c;
  }
}

// extract the lower triangle; pre = leading entries with col < i; dpos =
// first diagonal position (-1 if missing)
__global__ void k_lower_fill(const int* __restrict__ ia, const int* __restrict__ ja,
                             const double* __restrict__ val, int n, const int* __restrict__ lia,
                             int* __restrict__ lja, double* __restrict__ lval,
                             int* __restrict__ pre, int* __restrict__ dpos, int* flags) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    int p = lia[i];
    for (int k = ia[i]; k < ia[i + 1]; k++) {
      int j = ja[k];
      if (j <= i) {
        lja[p] = j;
        lval[p] = val[k];
        p++;
      }
    }
    int q = 0;
    while (lia[i] + q < lia[i + 1] && lja[lia[i] + q] < i) q++;
    pre[i] = q;
    int d = -1;
    for (int k = lia[i]; k < lia[i + 1]; k++)
      if (lja[k] == i) { d = k; break; }
    dpos[i] = d;
    if (d < 0) atomicOr(flags, 1);
  }
}

// pre/dpos for a factor given directly (every entry must satisfy j <= i)
__global__ void k_factor_meta(const int* __restrict__ lia, const int* __restrict__ lja, int n,
                              int* __restrict__ pre, int* __restrict__ dpos, int* flags) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    int q = 0;
    while (lia[i] + q < lia[i + 1] && lja[lia[i] + q] < i) q++;
    pre[i] = q;
    int d = -1;
    for (int k = lia[i]; k < lia[i + 1]; k++) {
      if (lja[k] > i) atomicOr(flags, 2);
      if (lja[k] == i && d < 0) d = k;
    }
    dpos[i] = d;
    if (d < 0) atomicOr(flags, 1);
  }
}

// strict lower part as CSR; values carry source positions in L (exact in double)
__global__ void k_strict_count(const int* __restrict__ lia, const int* __restrict__ lja, int n,
                               int* __restrict__ cnt) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    int c = 0;
    for (int k = lia[i]; k < lia[i + 1]; k++) c += (lja[k] < i);
    cnt[i] = c;
  }
}
__global__ void k_strict_fill(const int* __restrict__ lia, const int* __restrict__ lja, int n,
                              const int* __restrict__ sia, int* __restrict__ sja,
                              double* __restrict__ ssrc) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    int p = sia[i];
    for (int k = lia[i]; k < lia[i + 1]; k++)
      if (lja[k] < i) { sja[p] = lja[k]; ssrc[p] = (double)k; p++; }
  }
}

// ---------------------------------------------------------------- levels
__global__ void k_indeg(const int* __restrict__ sia, int n, int* __restrict__ indeg,
                        int* __restrict__ level, int* __restrict__ frontier, int* counter) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    int d = sia[i + 1] - sia[i];
    indeg[i] = d;
    if (d == 0) {
      level[i] = 0;
      frontier[atomicAdd(counter, 1)] = i;
    }
  }
}

// one Kahn step: rows of the current frontier release their dependents
__global__ void k_kahn_step(const int* __restrict__ uia, const int* __restrict__ uja,
                            const int* __restrict__ cur, int m, int lev, int* __restrict__ indeg,
                            int* __restrict__ level, int* __restrict__ next, int* counter) {
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < m; t += gridDim.x * blockDim.x) {
    const int k = cur[t];
    for (int q = uia[k]; q < uia[k + 1]; q++) {
      const int i = uja[q];
      if (atomicSub(&indeg[i], 1) == 1) {
        level[i] = lev;
        next[atomicAdd(counter, 1)] = i;
      }
    }
  }
}

// The whole sweep in one cooperative launch: each step releases the
// dependents of the current frontier [lo, hi); a grid barrier, then every
// thread reads the new end, then a second barrier before the next step
// appends to the frontier again.  Levels are fixed by the dependency graph;
// only the order inside a frontier depends on timing, and the rows are
// later sorted stably by level.
__global__ void k_kahn_all(const int* __restrict__ uia, const int* __restrict__ uja, int n,
                           int* __restrict__ indeg, int* __restrict__ level,
                           int* __restrict__ frontier, int* counter, int* nlev) {
  namespace cg = cooperative_groups;
  cg::grid_group grid = cg::this_grid();
  const int gtid = blockIdx.x * blockDim.x + threadIdx.x;
  const int gsz = gridDim.x * blockDim.x;
  int lo = 0;
  int hi = *(volatile int*)counter;
  int lev = 0;
  while (hi > lo && lev < n) {
    lev++;
    for (int t = lo + gtid; t < hi; t += gsz) {
      const int k = frontier[t];
      for (int q = uia[k]; q < uia[k + 1]; q++) {
        const int i = uja[q];
        if (atomicSub(&indeg[i], 1) == 1) {
          level[i] = lev;
          frontier[atomicAdd(counter, 1)] = i;
        }
      }
    }
    grid.sync();
    lo = hi;
    hi = *(volatile int*)counter;
    grid.sync();
  }
  if (gtid == 0) *nlev = lev;
}

__global__ void k_level_starts(const int* __restrict__ lev, int n, int nlevels,
                               int* __restrict__ ptr) {
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x)
    if (t == 0 || lev[t] != lev[t - 1]) ptr[lev[t]] = t;
  if (blockIdx.x == 0 && threadIdx.x == 0) ptr[nlevels] = n;
}

__global__ void k_iota_i(int* a, int n) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) a[i] = i;
}

// ---------------------------------------------------------------- factor
__device__ __forceinline__ void ic_factor_row(int i, const int* __restrict__ lia,
                                              const int* __restrict__ lja, double* lval,
                                              const int* __restrict__ pre,
                                              const int* __restrict__ dpos) {
  const int r0 = lia[i], r1 = lia[i + 1];
  for (int kk = r0; kk < r1; kk++) {
    const int k = lja[kk];
    if (k >= i) continue;
    double s = lval[kk];
    const int k0 = lia[k], kp = k0 + pre[k];
    for (int jj = k0; jj < kp; jj++) {
      const int j = lja[jj];
      for (int q = r0; q < r1; q++) {  // is j in row i?  (w_marker)
        if (lja[q] == j) {
          s = xsub(s, xmul(lval[q], lval[jj]));
          break;
        }
      }
    }
    lval[kk] = xdiv(s, lval[dpos[k]]);
  }
  const int di = dpos[i];
  double d = lval[di];
  for (int q = r0; q < r0 + pre[i]; q++) d = xsub(d, xmul(lval[q], lval[q]));
  if (d <= 0.0) d = 1e-14;
  lval[di] = __dsqrt_rn(d);
}

__global__ void k_ic_factor_wide(const int* __restrict__ lia, const int* __restrict__ lja,
                                 double* lval, const int* __restrict__ pre,
                                 const int* __restrict__ dpos, const int* __restrict__ order,
                                 int t0, int t1) {
  for (int t = t0 + blockIdx.x * blockDim.x + threadIdx.x; t < t1; t += gridDim.x * blockDim.x)
    ic_factor_row(order[t], lia, lja, lval, pre, dpos);
}

__global__ void __launch_bounds__(kBatchThreads)
k_ic_factor_batch(const int* __restrict__ lia, const int* __restrict__ lja, double* lval,
                  const int* __restrict__ pre, const int* __restrict__ dpos,
                  const int* __restrict__ order, const int* __restrict__ lptr, int l0, int l1) {
  for (int l = l0; l < l1; l++) {
    for (int t = lptr[l] + threadIdx.x; t < lptr[l + 1]; t += blockDim.x)
      ic_factor_row(order[t], lia, lja, lval, pre, dpos);
    __syncthreads();
  }
}

// ---------------------------------------------------------------- solves
// Row t of a layout: output index rows[t], entries [ia[t], ia[t+1]) of
// (column, value), divisor diag[t]:  out = (in - sum val*x[col]) / diag.
// x is read and written in the same kernel, so it is never marked
// read-only.
template <class T>
__device__ __forceinline__ void tri_row(int t, const int* __restrict__ ia,
                                        const int* __restrict__ ja, const T* __restrict__ val,
                                        const T* __restrict__ diag, const int* __restrict__ rows,
                                        const T* __restrict__ in, T* x) {
  const int i = rows[t];
  T s = in[i];
  for (int k = ia[t]; k < ia[t + 1]; k++) {
    if constexpr (sizeof(T) == 8)
      s = xsub(s, xmul(val[k], x[ja[k]]));
    else
      s = xsubf(s, xmulf(val[k], x[ja[k]]));
  }
  x[i] = s / diag[t];
}

template <class T>
__global__ void k_tri_wide(const int* __restrict__ ia, const int* __restrict__ ja,
                           const T* __restrict__ val, const T* __restrict__ diag,
                           const int* __restrict__ rows, int t0, int t1, const T* __restrict__ in,
                           T* x) {
  for (int t = t0 + blockIdx.x * blockDim.x + threadIdx.x; t < t1; t += gridDim.x * blockDim.x)
    tri_row<T>(t, ia, ja, val, diag, rows, in, x);
}

template <class T>
__global__ void __launch_bounds__(kBatchThreads)
k_tri_batch(const int* __restrict__ ia, const int* __restrict__ ja, const T* __restrict__ val,
            const T* __restrict__ diag, const int* __restrict__ rows,
            const int* __restrict__ lptr, int l0, int l1, const T* __restrict__ in, T* x) {
  for (int l = l0; l < l1; l++) {
    for (int t = lptr[l] + threadIdx.x; t < lptr[l + 1]; t += blockDim.x)
      tri_row<T>(t, ia, ja, val, diag, rows, in, x);
    __syncthreads();
  }
}

// Cooperative form: the whole sweep in one launch.  Segment s is either one
// wide level spread over the grid or a run of narrow levels stepped by block
// 0 with __syncthreads(); a grid-wide barrier separates segments.  Values of
// earlier levels are read with ld.global.cg (L2), since another SM wrote them.
constexpr int kCoopThreads = 256;
constexpr int kCoopNarrow = 4 * kCoopThreads;

template <class T>
__device__ __forceinline__ void tri_row_cg(int t, const int* __restrict__ ia,
                                           const int* __restrict__ ja, const T* __restrict__ val,
                                           const T* __restrict__ diag,
                                           const int* __restrict__ rows,
                                           const T* __restrict__ in, T* x) {
  const int i = rows[t];
  T s = in[i];
  for (int k = ia[t]; k < ia[t + 1]; k++) {
    if constexpr (sizeof(T) == 8)
      s = xsub(s, xmul(val[k], __ldcg(x + ja[k])));
    else
      s = xsubf(s, xmulf(val[k], __ldcg(x + ja[k])));
  }
  __stcg(x + i, s / diag[t]);
}

// A thread's first row of the next wide level, loaded before the grid
// barrier: everything but the values of the dependencies (which the
// barrier publishes) is known in advance.
constexpr int kPre = 4;
template <class T>
struct RowPre {
  int t;       // position in the layout, -1 if none
  int i, k0, k1;
  T in_i, d;
  int j[kPre];
  T v[kPre];
};

template <class T>
__device__ __forceinline__ void pre_load(RowPre<T>& p, int t, const int* __restrict__ ia,
                                         const int* __restrict__ ja, const T* __restrict__ val,
                                         const T* __restrict__ diag,
                                         const int* __restrict__ rows,
                                         const T* __restrict__ in) {
  p.t = t;
  p.i = rows[t];
  p.k0 = ia[t];
  p.k1 = ia[t + 1];
  p.in_i = in[p.i];
  p.d = diag[t];
#pragma unroll
  for (int q = 0; q < kPre; q++) {
    if (p.k0 + q < p.k1) {
      p.j[q] = ja[p.k0 + q];
      p.v[q] = val[p.k0 + q];
    }
  }
}

template <class T>
__device__ __forceinline__ void pre_finish(const RowPre<T>& p, const int* __restrict__ ja,
                                           const T* __restrict__ val, T* x) {
  T s = p.in_i;
  T xv[kPre];
#pragma unroll
  for (int q = 0; q < kPre; q++)
    if (p.k0 + q < p.k1) xv[q] = __ldcg(x + p.j[q]);  // independent loads in flight
#pragma unroll
  for (int q = 0; q < kPre; q++) {
    if (p.k0 + q < p.k1) {
      if constexpr (sizeof(T) == 8) s = xsub(s, xmul(p.v[q], xv[q]));
      else s = xsubf(s, xmulf(p.v[q], xv[q]));
    }
  }
  for (int k = p.k0 + kPre; k < p.k1; k++) {
    if constexpr (sizeof(T) == 8) s = xsub(s, xmul(val[k], __ldcg(x + ja[k])));
    else s = xsubf(s, xmulf(val[k], __ldcg(x + ja[k])));
  }
  __stcg(x + p.i, s / p.d);
}

template <class T>
__global__ void __launch_bounds__(kCoopThreads)
k_tri_coop(const int* __restrict__ ia, const int* __restrict__ ja, const T* __restrict__ val,
           const T* __restrict__ diag, const int* __restrict__ rows, const int* __restrict__ lptr,
           const int4* __restrict__ segs, int nseg, const T* __restrict__ in, T* x) {
  namespace cg = cooperative_groups;
  cg::grid_group grid = cg::this_grid();
  const int gtid = blockIdx.x * blockDim.x + threadIdx.x;
  const int gsz = gridDim.x * blockDim.x;
  RowPre<T> pre;
  pre.t = -1;
  if (nseg > 0 && segs[0].x == 0) {
    const int t = lptr[segs[0].y] + gtid;
    if (t < lptr[segs[0].y + 1]) pre_load<T>(pre, t, ia, ja, val, diag, rows, in);
  }
  for (int q = 0; q < nseg; q++) {
    const int4 sg = segs[q];
    if (sg.x == 0) {
      if (pre.t >= 0) pre_finish<T>(pre, ja, val, x);
      for (int t = lptr[sg.y] + gtid + gsz; t < lptr[sg.y + 1]; t += gsz)
        tri_row_cg<T>(t, ia, ja, val, diag, rows, in, x);
    } else if (blockIdx.x == 0) {
      for (int l = sg.y; l < sg.z; l++) {
        for (int t = lptr[l] + threadIdx.x; t < lptr[l + 1]; t += blockDim.x)
          tri_row_cg<T>(t, ia, ja, val, diag, rows, in, x);
        __syncthreads();
      }
    }
    // prefetch this thread's first row of the next segment if it is wide
    pre.t = -1;
    if (q + 1 < nseg) {
      const int4 nx = segs[q + 1];
      if (nx.x == 0) {
        const int t = lptr[nx.y] + gtid;
        if (t < lptr[nx.y + 1]) pre_load<T>(pre, t, ia, ja, val, diag, rows, in);
      }
    }
    grid.sync();
  }
}

// chunks[c] = [first, end) positions of chunk c: at most 32 rows, never
// crossing a level boundary, so no lane waits on a lane of its own warp.
// The warp reconverges after every chunk: lanes of one warp never spin on
// different chunks at once.
template <class T>
__global__ void __launch_bounds__(kFlagThreads)
k_tri_flags(const int* __restrict__ ia, const int* __restrict__ ja, const T* __restrict__ val,
            const T* __restrict__ diag, const int* __restrict__ rows,
            const int2* __restrict__ chunks, int nchunks, const T* __restrict__ in, T* out,
            T* clear, WaitCtl wc) {
  using W = WordOf<T>;
  using U = typename W::U;
  U* o = reinterpret_cast<U*>(out);
  const int lane = threadIdx.x & 31;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  for (int c = warp; c < nchunks; c += nwarps) {
    const int2 ch = chunks[c];
    const int t = ch.x + lane;
    if (t < ch.y) {
      const int i = rows[t];
      const int k0 = ia[t], k1 = ia[t + 1];
      T s = in[i];
      const T d = diag[t];
      if (clear) reinterpret_cast<U*>(clear)[i] = W::kPending;
      if (k1 - k0 <= 4) {
        // at most one group (nearly every row): the row is computed and
        // published inside its own polling loop, in the iteration its last
        // dependency arrives, instead of after the warp has reconverged
        // behind the chunk's slowest row
        const int m = k1 - k0;
        int j[4];
        T v[4];
        U u[4];
#pragma unroll
        for (int q = 0; q < 4; q++) {
          j[q] = q < m ? ja[k0 + q] : 0;
          v[q] = q < m ? val[k0 + q] : T(0);
          u[q] = U(0);
        }
        unsigned long long t0 = 0;
        for (int it = 0;; it++) {
#pragma unroll
          for (int q = 0; q < 4; q++)
            if (q < m && (it == 0 || u[q] == W::kPending)) u[q] = ld_relaxed(o + j[q]);
          bool pend = false;
#pragma unroll
          for (int q = 0; q < 4; q++) pend |= (q < m && u[q] == W::kPending);
          bool give_up = false;
          if (pend && it >= kSpinFast) {
            bool ran_out = false;
            if (wait_backoff(wc, it, t0, &ran_out)) {
              int dep = -1;
#pragma unroll
              for (int q = 3; q >= 0; q--)
                if (q < m && u[q] == W::kPending) dep = j[q];
              if (ran_out) wait_give_up(wc, i, dep, global_ns() - t0);
#pragma unroll
              for (int q = 0; q < 4; q++)
                if (q < m && u[q] == W::kPending) u[q] = W::kNaN;
              give_up = true;
            }
          }
          if (!pend || give_up) {
#pragma unroll
            for (int q = 0; q < 4; q++) {
              if (q < m) {
                if constexpr (sizeof(T) == 8) s = xsub(s, xmul(v[q], word_value(u[q])));
                else s = xsubf(s, xmulf(v[q], word_value(u[q])));
              }
            }
            U r = value_word(s / d);
            if (r == W::kPending) r = W::kNaN;
            st_relaxed(o + i, r);
            break;
          }
        }
      } else {
        for (int k = k0; k < k1; k += 4) {
          const int m = k1 - k < 4 ? k1 - k : 4;
          int j[4];
          T v[4];
          U u[4];
#pragma unroll
          for (int q = 0; q < 4; q++) {
            j[q] = q < m ? ja[k + q] : 0;
            v[q] = q < m ? val[k + q] : T(0);
          }
#pragma unroll
          for (int q = 0; q < 4; q++) u[q] = q < m ? ld_relaxed(o + j[q]) : U(0);
          wait_group(o, j, u, m, W::kPending, W::kNaN, wc, i);
#pragma unroll
          for (int q = 0; q < 4; q++) {
            if (q < m) {
              if constexpr (sizeof(T) == 8) s = xsub(s, xmul(v[q], word_value(u[q])));
              else s = xsubf(s, xmulf(v[q], word_value(u[q])));
            }
          }
        }
        U r = value_word(s / d);
        if (r == W::kPending) r = W::kNaN;
        st_relaxed(o + i, r);
      }
    }
    __syncwarp();
  }
}

// Tiled form.  Tile q is a range of consecutive row indices; a block takes
// its tiles in order (the backward sweep numbers the tiles from the end) and
// walks each tile's levels in order, one step per level with a block
// barrier after it.  A row's dependencies lie in its own tile at earlier
// levels (values this block published before a barrier: read through L1)
// or in earlier tiles (polled like the sync-free form).  Progress: every
// dependency of a tile lies in the same or an earlier tile, so the earliest
// unfinished tile always has its block working on it, and within a tile the
// earliest unfinished step has all its dependencies done.  A stale L1 copy
// can only hold the pending pattern (each value is written once per sweep,
// and L1 starts clean at a launch), which the poll loop treats as pending.
template <class T>
__global__ void __launch_bounds__(1024)
k_tri_tiles(const int* __restrict__ ia, const int* __restrict__ ja, const T* __restrict__ val,
            const T* __restrict__ diag, const int* __restrict__ rows,
            const unsigned* __restrict__ imask, const int2* __restrict__ tile_steps,
            const int2* __restrict__ steps, int ntiles, const T* __restrict__ in, T* out,
            T* clear, WaitCtl wc) {
  using W = WordOf<T>;
  using U = typename W::U;
  U* o = reinterpret_cast<U*>(out);
  for (int q = blockIdx.x; q < ntiles; q += gridDim.x) {
    const int2 ts = tile_steps[q];
    for (int st = ts.x; st < ts.y; st++) {
      const int2 sp = steps[st];
      for (int t = sp.x + threadIdx.x; t < sp.y; t += blockDim.x) {
        const int i = rows[t];
        const int k0 = ia[t], k1 = ia[t + 1];
        const unsigned im = imask[t];
        T s = in[i];
        const T d = diag[t];
        if (clear) reinterpret_cast<U*>(clear)[i] = W::kPending;
        for (int k = k0; k < k1; k += 4) {
          const int m = k1 - k < 4 ? k1 - k : 4;
          int j[4];
          T v[4];
          U u[4];
#pragma unroll
          for (int e = 0; e < 4; e++) {
            j[e] = e < m ? ja[k + e] : 0;
            v[e] = e < m ? val[k + e] : T(0);
          }
#pragma unroll
          for (int e = 0; e < 4; e++) {
            const int bit = k - k0 + e;
            const bool own = bit < 32 && ((im >> bit) & 1u);
            u[e] = e < m ? (own ? __ldca(o + j[e]) : ld_relaxed(o + j[e])) : U(0);
          }
          wait_group(o, j, u, m, W::kPending, W::kNaN, wc, i);
#pragma unroll
          for (int e = 0; e < 4; e++) {
            if (e < m) {
              if constexpr (sizeof(T) == 8) s = xsub(s, xmul(v[e], word_value(u[e])));
              else s = xsubf(s, xmulf(v[e], word_value(u[e])));
            }
          }
        }
        U r = value_word(s / d);
        if (r == W::kPending) r = W::kNaN;
        st_relaxed(o + i, r);
      }
      __syncthreads();
    }
  }
}

// schedule of the tiled form (IChol::build_tiles)
__global__ void k_pos_level(const int* __restrict__ ptr, int nlevels, int n, int* __restrict__ lev) {
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
    int lo = 0, hi = nlevels - 1;  // last level starting at or before t
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (ptr[mid] <= t) lo = mid;
      else hi = mid - 1;
    }
    lev[t] = lo;
  }
}
// tile of position t: forward = row / R, backward = ntiles - 1 - row / R
__device__ __forceinline__ int tile_of(int row, int R, int ntiles, bool forward) {
  const int q = row / R;
  return forward ? q : ntiles - 1 - q;
}
__global__ void k_step_heads(const int* __restrict__ rows, const int* __restrict__ lev, int n,
                             int R, int ntiles, int forward, int* __restrict__ head) {
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
    int h = 1;
    if (t > 0)
      h = lev[t] != lev[t - 1] || tile_of(rows[t], R, ntiles, forward) !=
                                      tile_of(rows[t - 1], R, ntiles, forward);
    head[t] = h;
  }
}
__global__ void k_step_tiles(const int* __restrict__ starts, int nsteps,
                             const int* __restrict__ rows, int R, int ntiles, int forward,
                             int* __restrict__ tile, int* __restrict__ ids) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nsteps; k += gridDim.x * blockDim.x) {
    tile[k] = tile_of(rows[starts[k]], R, ntiles, forward);
    ids[k] = k;
  }
}
__global__ void k_step_ranges(const int* __restrict__ sorted_ids, const int* __restrict__ starts,
                              int nsteps, int n, const int* __restrict__ sorted_tile,
                              int2* __restrict__ steps, int2* __restrict__ tile_steps) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nsteps; k += gridDim.x * blockDim.x) {
    const int id = sorted_ids[k];
    steps[k] = make_int2(starts[id], id + 1 < nsteps ? starts[id + 1] : n);
    const int q = sorted_tile[k];
    if (k == 0 || sorted_tile[k - 1] != q) tile_steps[q].x = k;
    if (k == nsteps - 1 || sorted_tile[k + 1] != q) tile_steps[q].y = k + 1;
  }
}
// bit e of imask[t]: entry e of row t depends on a row of the same tile
__global__ void k_tile_mask(const int* __restrict__ ia, const int* __restrict__ ja,
                            const int* __restrict__ rows, int n, int R,
                            unsigned* __restrict__ imask) {
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
    const int q = rows[t] / R;
    unsigned m = 0;
    const int k0 = ia[t];
    const int k1 = min(ia[t + 1], k0 + 32);
    for (int k = k0; k < k1; k++)
      if (ja[k] / R == q) m |= 1u << (k - k0);
    imask[t] = m;
  }
}

// ---------------------------------------------------------------- layout
__global__ void k_fwd_count(const int* __restrict__ lia, const int* __restrict__ lja,
                            const int* __restrict__ order, int n, int* __restrict__ cnt) {
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
    int i = order[t], c = 0;
    for (int k = lia[i]; k < lia[i + 1]; k++) c += (lja[k] < i);
    cnt[t] = c;
  }
}

__global__ void k_fwd_fill(const int* __restrict__ lia, const int* __restrict__ lja,
                           const int* __restrict__ order, int n, const int* __restrict__ fia,
                           int* __restrict__ fja, int* __restrict__ fsrc) {
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
    int i = order[t], p = fia[t];
    for (int k = lia[i]; k < lia[i + 1]; k++)
      if (lja[k] < i) { fja[p] = lja[k]; fsrc[p] = k; p++; }
  }
}

__global__ void k_bwd_count(const int* __restrict__ uia, const int* __restrict__ border, int n,
                            int* __restrict__ cnt) {
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
    int j = border[t];
    cnt[t] = uia[j + 1] - uia[j];
  }
}

// U row j lists i > j ascending (stable transpose); stored descending
__global__ void k_bwd_fill(const int* __restrict__ uia, const int* __restrict__ uja,
                           const int* __restrict__ usrc, const int* __restrict__ border, int n,
                           const int* __restrict__ bia, int* __restrict__ bja,
                           int* __restrict__ bsrc) {
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
    int j = border[t], p = bia[t];
    for (int k = uia[j + 1] - 1; k >= uia[j]; k--) { bja[p] = uja[k]; bsrc[p] = usrc[k]; p++; }
  }
}

__global__ void k_reverse(const int* __restrict__ a, int n, int* __restrict__ b) {
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x)
    b[t] = a[n - 1 - t];
}

template <class T>
__global__ void k_gather_vals(const int* __restrict__ src, int m, const double* __restrict__ lval,
                              T* __restrict__ out) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < m; p += gridDim.x * blockDim.x)
    out[p] = (T)lval[src[p]];
}

template <class T>
__global__ void k_gather_diag(const int* __restrict__ order, int n, const int* __restrict__ dpos,
                              const double* __restrict__ lval, T* __restrict__ out) {
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x)
    out[t] = (T)lval[dpos[order[t]]];
}

__global__ void k_map_ids(const int* __restrict__ src, int m, const int* __restrict__ inv,
                          int* __restrict__ dst) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < m; p += gridDim.x * blockDim.x)
    dst[p] = inv ? inv[src[p]] : src[p];
}

__global__ void k_double_to_int(const double* __restrict__ a, int m, int* __restrict__ b) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < m; p += gridDim.x * blockDim.x)
    b[p] = (int)a[p];
}

// ---------------------------------------------------------------- host
// Segments: a wide level is one grid launch; a run of narrow levels is one
// batched block.  Built from host level offsets.
static void make_segments(const std::vector<int>& ptr, std::vector<IChol::Seg>& segs,
                          int narrow = kNarrow) {
  segs.clear();
  const int nl = (int)ptr.size() - 1;
  int l = 0;
  while (l < nl) {
    int w = ptr[l + 1] - ptr[l];
    if (w > narrow) {
      segs.push_back({0, l, l + 1, ptr[l], ptr[l + 1]});
      l++;
    } else {
      int l1 = l;
      while (l1 < nl && ptr[l1 + 1] - ptr[l1] <= narrow) l1++;
      segs.push_back({1, l, l1, ptr[l], ptr[l1]});
      l = l1;
    }
  }
}

static void upload_segs(const std::vector<IChol::Seg>& segs, DBuf<int4>& d, cudaStream_t s) {
  std::vector<int4> h(segs.size());
  for (size_t q = 0; q < segs.size(); q++) h[q] = make_int4(segs[q].kind, segs[q].l0, segs[q].l1, 0);
  d.alloc(h.size() > 0 ? h.size() : 1, s);
  if (!h.empty()) d.upload(h.data(), h.size());
  BN_CUDA(cudaStreamSynchronize(s));
}

// Dependency levels by a Kahn frontier sweep (level l = rows whose
// dependencies all lie in levels < l), in one cooperative launch; rows in
// level order (stable: row order within a level) and the level offsets.
// deps: row i lists the rows it depends on; users: its transpose.
void level_schedule(const CSR& deps, const CSR& users, DBuf<int>& order, std::vector<int>& lptr,
                    cudaStream_t s) {
  const int n = deps.n;
  const int g = grid_for(n, 256);
  DBuf<int> indeg(n, s), level(n, s), frontier(n, s), ctr(1, s);
  ctr.zero();
  BN_LAUNCH(k_indeg, g, 256, 0, s, deps.ia.p, n, indeg.p, level.p, frontier.p, ctr.p);
  int nlevels = 0;
  {  // all Kahn steps in one cooperative launch
    DBuf<int> nlev(1, s);
    int dev = 0, per_sm = 0, sms = 0;
    BN_CUDA(cudaGetDevice(&dev));
    BN_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_kahn_all, 256, 0));
    BN_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const int grid = sms * (per_sm < 4 ? per_sm : 4);
    BN_REQUIRE(grid > 0, BN_ERR_CUDA, "level sweep grid does not fit");
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(256);
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    g_launch_count++;
    const int* uia = users.ia.p;
    const int* uja = users.ja.p;
    BN_CUDA(cudaLaunchKernelEx(&cfg, k_kahn_all, uia, uja, n, indeg.p, level.p, frontier.p, ctr.p,
                               nlev.p));
    const int reached = read_scalar(ctr.p, s);
    BN_REQUIRE(reached == n, BN_ERR_ARG, "dependency levels did not cover every row");
    // one step per level; the last one finds no new rows
    nlevels = read_scalar(nlev.p, s);
  }
  order.alloc(n, s);
  DBuf<int> ids(n, s), keys_out(n, s);
  BN_LAUNCH(k_iota_i, g, 256, 0, s, ids.p, n);
  size_t tmp = 0;
  int eb = 1;
  while ((1LL << eb) <= (long long)nlevels) eb++;
  BN_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tmp, level.p, keys_out.p, ids.p, order.p, n, 0,
                                          eb, s));
  DBuf<unsigned char> t(tmp, s);
  BN_CUDA(cub::DeviceRadixSort::SortPairs(t.p, tmp, level.p, keys_out.p, ids.p, order.p, n, 0, eb,
                                          s));
  // level offsets from the sorted levels (every level holds a row)
  DBuf<int> dptr((size_t)nlevels + 1, s);
  BN_LAUNCH(k_level_starts, g, 256, 0, s, keys_out.p, n, nlevels, dptr.p);
  lptr.assign(nlevels + 1, 0);
  dptr.download(lptr.data(), (size_t)nlevels + 1);
  BN_CUDA(cudaStreamSynchronize(s));
}

void IChol::factor(const CSR& A, cudaStream_t s) {
  stream = s;
  n = A.n;
  const int g = grid_for(n, 256);
  DBuf<int> cnt((size_t)n + 1, s);
  cnt.zero();
  BN_LAUNCH(k_lower_count, g, 256, 0, s, A.ia.p, A.ja.p, n, cnt.p);
  int lnnz = scan_counts(cnt.p, n, s);
  L.n = L.m = n;
  L.nnz = lnnz;
  L.ia = std::move(cnt);
  L.ja.alloc((size_t)(lnnz > 0 ? lnnz : 1), s);
  L.val.alloc((size_t)(lnnz > 0 ? lnnz : 1), s);
  finish(A.ia.p, A.ja.p, A.val.p, true, s);
}

void IChol::load(CSR&& Lf, cudaStream_t s) {
  stream = s;
  n = Lf.n;
  L = std::move(Lf);
  finish(L.ia.p, L.ja.p, L.val.p, false, s);
}

// Lower-triangle extraction (from A, or checks on a given factor), the
// dependency levels, the numeric factorization and the solve layouts.
void IChol::finish(const int* aia, const int* aja, const double* aval, bool numeric,
                   cudaStream_t s) {
  const int g = grid_for(n, 256);
  Phase ph_lower("ichol lower", s);
  DBuf<int> flags(1, s);
  flags.zero();
  pre.alloc(n, s);
  dpos.alloc(n, s);
  if (numeric) {
    BN_LAUNCH(k_lower_fill, g, 256, 0, s, aia, aja, aval, n, L.ia.p, L.ja.p, L.val.p, pre.p,
              dpos.p, flags.p);
  } else {
    BN_LAUNCH(k_factor_meta, g, 256, 0, s, L.ia.p, L.ja.p, n, pre.p, dpos.p, flags.p);
  }
  int f = read_scalar(flags.p, s);
  BN_REQUIRE(!(f & 1), BN_ERR_ARG, "IC(0): a row has no diagonal entry");
  BN_REQUIRE(!(f & 2), BN_ERR_ARG, "IC(0): factor holds an entry above the diagonal");

  ph_lower.done();
  // strict lower part and its transpose (the dependents of each row)
  CSR Sl, U;
  {
    Phase ph("ichol strict+transpose", s);
    DBuf<int> c((size_t)n + 1, s);
    c.zero();
    BN_LAUNCH(k_strict_count, g, 256, 0, s, L.ia.p, L.ja.p, n, c.p);
    int snnz = scan_counts(c.p, n, s);
    Sl.n = Sl.m = n;
    Sl.nnz = snnz;
    Sl.ia = std::move(c);
    Sl.ja.alloc((size_t)(snnz > 0 ? snnz : 1), s);
    Sl.val.alloc((size_t)(snnz > 0 ? snnz : 1), s);
    BN_LAUNCH(k_strict_fill, g, 256, 0, s, L.ia.p, L.ja.p, n, Sl.ia.p, Sl.ja.p, Sl.val.p);
    transpose(Sl, U, s, true);
  }
  offd_nnz = Sl.nnz;

  // dependency levels and the level order
  {
    Phase ph("ichol levels", s);
    level_schedule(Sl, U, order, lptr, s);
    nlevels = (int)lptr.size() - 1;
  }
  // backward processing order: reverse level order
  border.alloc(n, s);
  BN_LAUNCH(k_reverse, g, 256, 0, s, order.p, n, border.p);
  bptr.assign(nlevels + 1, 0);
  for (int l = 0; l <= nlevels; l++) bptr[l] = n - lptr[nlevels - l];
  make_segments(lptr, fseg);
  make_segments(bptr, bseg);
  {
    std::vector<Seg> cf, cb;
    make_segments(lptr, cf, kCoopNarrow);
    make_segments(bptr, cb, kCoopNarrow);
    upload_segs(cf, d_cfseg, s);
    upload_segs(cb, d_cbseg, s);
    n_cfseg = (int)cf.size();
    n_cbseg = (int)cb.size();
  }
  n_fchunk = upload_chunks(lptr, d_fchunk, s);
  n_bchunk = upload_chunks(bptr, d_bchunk, s);
  d_lptr.alloc(nlevels + 1, s);
  d_lptr.upload(lptr.data(), nlevels + 1);
  d_bptr.alloc(nlevels + 1, s);
  d_bptr.upload(bptr.data(), nlevels + 1);

  if (numeric) {
    Phase ph("ichol numeric", s);
    for (const Seg& sg : fseg) {
      if (sg.kind == 0)
        BN_LAUNCH(k_ic_factor_wide, grid_for(sg.t1 - sg.t0, 128), 128, 0, s, L.ia.p, L.ja.p,
                  L.val.p, pre.p, dpos.p, order.p, sg.t0, sg.t1);
      else
        BN_LAUNCH(k_ic_factor_batch, 1, kBatchThreads, 0, s, L.ia.p, L.ja.p, L.val.p, pre.p,
                  dpos.p, order.p, d_lptr.p, sg.l0, sg.l1);
    }
  }

  // forward solve layout (level order)
  Phase ph_lay("ichol layouts", s);
  fia.alloc((size_t)n + 1, s);
  fia.zero();
  BN_LAUNCH(k_fwd_count, g, 256, 0, s, L.ia.p, L.ja.p, order.p, n, fia.p);
  int fnnz = scan_counts(fia.p, n, s);
  fja.alloc((size_t)(fnnz > 0 ? fnnz : 1), s);
  fsrc.alloc((size_t)(fnnz > 0 ? fnnz : 1), s);
  BN_LAUNCH(k_fwd_fill, g, 256, 0, s, L.ia.p, L.ja.p, order.p, n, fia.p, fja.p, fsrc.p);
  // backward solve layout (reverse level order), rows of U = (strict L)^T
  {
    DBuf<int> usrc((size_t)(fnnz > 0 ? fnnz : 1), s);
    if (fnnz > 0)
      BN_LAUNCH(k_double_to_int, grid_for(fnnz, 256), 256, 0, s, U.val.p, fnnz, usrc.p);
    bia.alloc((size_t)n + 1, s);
    bia.zero();
    BN_LAUNCH(k_bwd_count, g, 256, 0, s, U.ia.p, border.p, n, bia.p);
    scan_counts(bia.p, n, s);
    bja.alloc((size_t)(fnnz > 0 ? fnnz : 1), s);
    bsrc.alloc((size_t)(fnnz > 0 ? fnnz : 1), s);
    BN_LAUNCH(k_bwd_fill, g, 256, 0, s, U.ia.p, U.ja.p, usrc.p, border.p, n, bia.p, bja.p, bsrc.p);
  }
  // the tiled schedule serves the tiled single-vector form and the
  // many-column sweeps of the block PCG
  build_tiles(true, s);
  build_tiles(false, s);
  if (mode == kSweepSlab || mode == kSweepSlabW) {
    build_slab_partition(s);
    build_slab(true, s);
    build_slab(false, s);
  }
  ph_lay.done();
  {
    Phase ph("ichol values", s);
    refresh_values();
    remap(nullptr, s);
  }
  wait.init(s);  // here, never inside a stream capture
}

void IChol::remap(const int* inv, cudaStream_t s) {
  const int m = offd_nnz > 0 ? offd_nnz : 1;
  vorder.alloc(n, s);
  vborder.alloc(n, s);
  vfja.alloc(m, s);
  vbja.alloc(m, s);
  if (mode == kSweepSlab || mode == kSweepSlabW) {
    slab_pack(sf, inv, s);
    slab_pack(sb, inv, s);
  }
  BN_LAUNCH(k_map_ids, grid_for(n, 256), 256, 0, s, order.p, n, inv, vorder.p);
  BN_LAUNCH(k_map_ids, grid_for(n, 256), 256, 0, s, border.p, n, inv, vborder.p);
  if (offd_nnz > 0) {
    BN_LAUNCH(k_map_ids, grid_for(offd_nnz, 256), 256, 0, s, fja.p, offd_nnz, inv, vfja.p);
    BN_LAUNCH(k_map_ids, grid_for(offd_nnz, 256), 256, 0, s, bja.p, offd_nnz, inv, vbja.p);
  }
}

void IChol::refresh_values() {
  cudaStream_t s = stream;
  const int g = grid_for(n, 256);
  const int m = offd_nnz > 0 ? offd_nnz : 1;
  fval.alloc(m, s);
  bval.alloc(m, s);
  fdiag.alloc(n, s);
  bdiag.alloc(n, s);
  if (offd_nnz > 0) {
    BN_LAUNCH(k_gather_vals<double>, grid_for(offd_nnz, 256), 256, 0, s, fsrc.p, offd_nnz,
              L.val.p, fval.p);
    BN_LAUNCH(k_gather_vals<double>, grid_for(offd_nnz, 256), 256, 0, s, bsrc.p, offd_nnz,
              L.val.p, bval.p);
  }
  BN_LAUNCH(k_gather_diag<double>, g, 256, 0, s, order.p, n, dpos.p, L.val.p, fdiag.p);
  BN_LAUNCH(k_gather_diag<double>, g, 256, 0, s, border.p, n, dpos.p, L.val.p, bdiag.p);
  if (want_f32) {
    fval32.alloc(m, s);
    bval32.alloc(m, s);
    fdiag32.alloc(n, s);
    bdiag32.alloc(n, s);
    if (offd_nnz > 0) {
      BN_LAUNCH(k_gather_vals<float>, grid_for(offd_nnz, 256), 256, 0, s, fsrc.p, offd_nnz,
                L.val.p, fval32.p);
      BN_LAUNCH(k_gather_vals<float>, grid_for(offd_nnz, 256), 256, 0, s, bsrc.p, offd_nnz,
                L.val.p, bval32.p);
    }
    BN_LAUNCH(k_gather_diag<float>, g, 256, 0, s, order.p, n, dpos.p, L.val.p, fdiag32.p);
    BN_LAUNCH(k_gather_diag<float>, g, 256, 0, s, border.p, n, dpos.p, L.val.p, bdiag32.p);
  }
  if (mode == kSweepSlab || mode == kSweepSlabW) {
    slab_values(sf, s);
    slab_values(sb, s);
  }
}

template <class T>
static void run_tri(const std::vector<IChol::Seg>& segs, const int* ia, const int* ja,
                    const T* val, const T* diag, const int* rows, const int* dptr, const T* in,
                    T* x, cudaStream_t s) {
  for (const IChol::Seg& sg : segs) {
    if (sg.kind == 0)
      BN_LAUNCH(k_tri_wide<T>, grid_for(sg.t1 - sg.t0, 128), 128, 0, s, ia, ja, val, diag, rows,
                sg.t0, sg.t1, in, x);
    else
      BN_LAUNCH(k_tri_batch<T>, 1, kBatchThreads, 0, s, ia, ja, val, diag, rows, dptr, sg.l0,
                sg.l1, in, x);
  }
}

template <class T>
static void run_tri_coop(int nseg, const int4* segs, const int* ia, const int* ja, const T* val,
                         const T* diag, const int* rows, const int* lptr, const T* in, T* x,
                         cudaStream_t s) {
  int dev = 0, per_sm = 0;
  BN_CUDA(cudaGetDevice(&dev));
  BN_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_tri_coop<T>, kCoopThreads, 0));
  int sms = 0;
  BN_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  int grid = sms * (per_sm < 4 ? per_sm : 4);
  BN_REQUIRE(grid > 0, BN_ERR_CUDA, "IC(0): cooperative grid does not fit");
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(kCoopThreads);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  g_launch_count++;
  BN_CUDA(cudaLaunchKernelEx(&cfg, k_tri_coop<T>, ia, ja, val, diag, rows, lptr, segs, nseg, in,
                             x));
}

template <class T>
static void run_tri_flags(int nchunks, const int2* chunks, int blocks_per_sm, const int* ia,
                          const int* ja, const T* val, const T* diag, const int* rows,
                          const T* in, T* out, T* clear, WaitCtl wc, cudaStream_t s) {
  int dev = 0, per_sm = 0, sms = 0;
  BN_CUDA(cudaGetDevice(&dev));
  BN_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_tri_flags<T>, kFlagThreads, 0));
  BN_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  if (blocks_per_sm > 0 && per_sm > blocks_per_sm) per_sm = blocks_per_sm;
  const int grid = sms * per_sm;
  BN_REQUIRE(grid > 0, BN_ERR_CUDA, "IC(0): sweep grid does not fit");
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(kFlagThreads);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;  // co-residency: waits always end
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  g_launch_count++;
  BN_CUDA(cudaLaunchKernelEx(&cfg, k_tri_flags<T>, ia, ja, val, diag, rows, chunks, nchunks, in,
                             out, clear, wc));
}

template <class T>
static void run_tri_tiles(const IChol::Tiles& tl, const int* ia, const int* ja, const T* val,
                          const T* diag, const int* rows, const T* in, T* out, T* clear,
                          WaitCtl wc, cudaStream_t s) {
  int dev = 0, per_sm = 0, sms = 0;
  BN_CUDA(cudaGetDevice(&dev));
  BN_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_tri_tiles<T>, tl.threads, 0));
  BN_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  const int cap = sms * per_sm;
  const int grid = tl.ntiles < cap ? tl.ntiles : cap;
  BN_REQUIRE(grid > 0, BN_ERR_CUDA, "IC(0): tiled sweep grid does not fit");
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(tl.threads);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;  // co-residency: waits always end
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  g_launch_count++;
  BN_CUDA(cudaLaunchKernelEx(&cfg, k_tri_tiles<T>, ia, ja, val, diag, rows,
                             (const unsigned*)tl.imask.p, (const int2*)tl.tile_steps.p,
                             (const int2*)tl.steps.p, tl.ntiles, in, out, clear, wc));
}

// The tiled schedule of one sweep direction: tiles of consecutive row
// indices (as many as the device holds blocks of tl.threads), each tile's
// rows of one level as one step.
void IChol::build_tiles(bool forward, cudaStream_t s) {
  Tiles& tl = forward ? tf : tb;
  const int* rows = forward ? order.p : border.p;  // natural row ids, layout order
  const DBuf<int>& dptr = forward ? d_lptr : d_bptr;
  const int* tia = forward ? fia.p : bia.p;
  const int* tja = forward ? fja.p : bja.p;
  static const int threads = getenv("BN_IC_TILE_THREADS") ? atoi(getenv("BN_IC_TILE_THREADS"))
                                                          : 512;
  static const int tiles_per_sm =
      getenv("BN_IC_TILES_PER_SM") ? atoi(getenv("BN_IC_TILES_PER_SM")) : 2;
  BN_REQUIRE(threads >= 32 && threads <= 1024 && threads % 32 == 0 && tiles_per_sm >= 1,
             BN_ERR_ARG, "IC(0): tiled sweep shape");
  int dev = 0, sms = 0, o64 = 0, o32 = 0;
  BN_CUDA(cudaGetDevice(&dev));
  BN_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  BN_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o64, k_tri_tiles<double>, threads, 0));
  BN_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o32, k_tri_tiles<float>, threads, 0));
  int per_sm = o64 < o32 ? o64 : o32;
  if (per_sm > tiles_per_sm) per_sm = tiles_per_sm;
  BN_REQUIRE(per_sm > 0, BN_ERR_CUDA, "IC(0): tiled sweep block does not fit");
  tl.threads = threads;
  tl.ntiles = sms * per_sm;
  tl.rows_per_tile = n > 0 ? (n + tl.ntiles - 1) / tl.ntiles : 1;
  const int R = tl.rows_per_tile;
  tl.tile_steps.alloc(tl.ntiles, s);
  tl.tile_steps.zero();  // empty tiles: [0, 0)
  tl.imask.alloc(n > 0 ? n : 1, s);
  tl.nsteps = 0;
  if (n == 0) {
    tl.steps.alloc(1, s);
    return;
  }
  const int g = grid_for(n, 256);
  DBuf<int> lev(n, s), head(n, s), starts(n, s), nsel(1, s);
  BN_LAUNCH(k_pos_level, g, 256, 0, s, dptr.p, nlevels, n, lev.p);
  BN_LAUNCH(k_step_heads, g, 256, 0, s, rows, lev.p, n, R, tl.ntiles, forward ? 1 : 0, head.p);
  DBuf<int> pos(n, s);
  BN_LAUNCH(k_iota_i, g, 256, 0, s, pos.p, n);
  size_t tmp = 0;
  BN_CUDA(cub::DeviceSelect::Flagged(nullptr, tmp, pos.p, head.p, starts.p, nsel.p, n, s));
  {
    DBuf<unsigned char> t(tmp, s);
    BN_CUDA(cub::DeviceSelect::Flagged(t.p, tmp, pos.p, head.p, starts.p, nsel.p, n, s));
  }
  const int ns = read_scalar(nsel.p, s);
  tl.nsteps = ns;
  DBuf<int> stile(ns, s), sids(ns, s), stile2(ns, s), sids2(ns, s);
  BN_LAUNCH(k_step_tiles, grid_for(ns, 256), 256, 0, s, starts.p, ns, rows, R, tl.ntiles,
            forward ? 1 : 0, stile.p, sids.p);
  int eb = 1;
  while ((1 << eb) <= tl.ntiles) eb++;
  tmp = 0;
  BN_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tmp, stile.p, stile2.p, sids.p, sids2.p, ns, 0,
                                          eb, s));
  {
    DBuf<unsigned char> t(tmp, s);
    BN_CUDA(cub::DeviceRadixSort::SortPairs(t.p, tmp, stile.p, stile2.p, sids.p, sids2.p, ns, 0,
                                            eb, s));
  }
  tl.steps.alloc(ns, s);
  BN_LAUNCH(k_step_ranges, grid_for(ns, 256), 256, 0, s, sids2.p, starts.p, ns, n, stile2.p,
            tl.steps.p, tl.tile_steps.p);
  BN_LAUNCH(k_tile_mask, g, 256, 0, s, tia, tja, rows, n, R, tl.imask.p);
  BN_CUDA(cudaStreamSynchronize(s));
}

template <class T>
void IChol::solve(const T* b, T* y, T* x, cudaStream_t s) {
  const T* fv;
  const T* fd;
  const T* bv;
  const T* bd;
  if constexpr (sizeof(T) == 8) {
    fv = fval.p; fd = fdiag.p; bv = bval.p; bd = bdiag.p;
  } else {
    fv = fval32.p; fd = fdiag32.p; bv = bval32.p; bd = bdiag32.p;
  }
  if (mode == kSweepTiles) {
    if (n == 0) return;
    BN_CUDA(cudaMemsetAsync(y, 0xFF, sizeof(T) * (size_t)n, s));
    run_tri_tiles<T>(tf, fia.p, vfja.p, fv, fd, vorder.p, b, y, x, wait.ctl(WT_IC_FWD), s);
    run_tri_tiles<T>(tb, bia.p, vbja.p, bv, bd, vborder.p, y, x, nullptr, wait.ctl(WT_IC_BWD), s);
    return;
  }
  if (slab_ready<T>()) {
    if (n == 0) return;
    BN_CUDA(cudaMemsetAsync(y, 0xFF, sizeof(T) * (size_t)n, s));
    run_tri_slab<T>(*this, true, b, y, x, wait.ctl(WT_IC_FWD), s);
    run_tri_slab<T>(*this, false, y, x, nullptr, wait.ctl(WT_IC_BWD), s);
    return;
  }
  if (mode == kSweepFlags || mode == kSweepSlab || mode == kSweepSlabW) {
    if (n == 0) return;
    BN_CUDA(cudaMemsetAsync(y, 0xFF, sizeof(T) * (size_t)n, s));
    run_tri_flags<T>(n_fchunk, d_fchunk.p, blocks_per_sm, fia.p, vfja.p, fv, fd, vorder.p, b, y,
                     x, wait.ctl(WT_IC_FWD), s);
    run_tri_flags<T>(n_bchunk, d_bchunk.p, blocks_per_sm, bia.p, vbja.p, bv, bd, vborder.p, y, x,
                     nullptr, wait.ctl(WT_IC_BWD), s);
    return;
  }
  if (mode == kSweepCoop) {
    run_tri_coop<T>(n_cfseg, d_cfseg.p, fia.p, vfja.p, fv, fd, vorder.p, d_lptr.p, b, y, s);
    run_tri_coop<T>(n_cbseg, d_cbseg.p, bia.p, vbja.p, bv, bd, vborder.p, d_bptr.p, y, x, s);
    return;
  }
  run_tri<T>(fseg, fia.p, vfja.p, fv, fd, vorder.p, d_lptr.p, b, y, s);
  run_tri<T>(bseg, bia.p, vbja.p, bv, bd, vborder.p, d_bptr.p, y, x, s);
}

template void IChol::solve<double>(const double*, double*, double*, cudaStream_t);
template void IChol::solve<float>(const float*, float*, float*, cudaStream_t);

void IChol::check_waits(cudaStream_t s) {
  if (!wait.rec.p) return;
  std::string msg;
  if (wait.take(s, &msg)) throw Error(BN_ERR_SPIN, "IC(0) solve: " + msg);
}

unsigned long long WaitRecord::default_limit_ns() {
  // A legitimate wait lasts at most the time the grid's other warps take
  // for their current chunks (milliseconds on the largest networks); a
  // second is far above that and still ends a stuck sweep promptly.
  static const unsigned long long v = [] {
    const char* e = getenv("BN_WAIT_LIMIT_MS");
    const double ms = e ? atof(e) : 1000.0;
    return (unsigned long long)((ms > 0.01 ? ms : 0.01) * 1e6);
  }();
  return v;
}

int WaitRecord::take(cudaStream_t s, std::string* msg) {
  int h[kWaitWords];
  rec.download(h, kWaitWords);
  BN_CUDA(cudaStreamSynchronize(s));
  if (h[0] == 0) return 0;
  rec.zero();
  static const char* names[] = {"?", "forward IC(0) sweep", "backward IC(0) sweep",
                                "ordered Gauss-Seidel sweep", "wait self-test"};
  const int tag = (h[1] >= 1 && h[1] <= 4) ? h[1] : 0;
  char buf[256];
  snprintf(buf, sizeof buf,
           "a bounded dependency wait ran out (%s: row %d waited %.3f ms for row %d; the "
           "sweep was abandoned)",
           names[tag], h[2], h[4] * 1e-3, h[3]);
  if (msg) *msg = buf;
  return BN_ERR_SPIN;
}

int IChol::blocks_from_env() {
  const char* v = getenv("BN_IC_BLOCKS");
  return v ? atoi(v) : 2;  // 2 blocks of 256 per SM measured fastest on the 20M network
}

// The give-up path of the bounded waits, on demand: the forward sweep
// kernel over an n-row chain (row t depends on row t-1) whose first row is
// left out of the schedule, so row 1 waits for a value that nothing
// publishes.  Its wait runs out after limit_ns, raises the abort word, and
// rows 2..n-1 end at once (they see NaN or the abort word).  Throws the
// sweep's BN_ERR_SPIN; *elapsed_ms receives the launch's device time.
void wait_selftest(int n, double limit_ms, double* elapsed_ms, cudaStream_t s) {
  BN_REQUIRE(n >= 2 && n <= (1 << 20), BN_ERR_ARG, "wait self-test: 2 <= n <= 2^20 rows");
  BN_REQUIRE(limit_ms > 0.0 && limit_ms <= 10000.0, BN_ERR_ARG,
             "wait self-test: 0 < limit <= 10000 ms");
  std::vector<int> ia(n + 1), ja(n - 1), rows(n);
  std::vector<double> val(n - 1, 0.5), diag(n, 1.0), in(n, 1.0);
  std::vector<int2> chunks;
  ia[0] = 0;
  for (int t = 0; t < n; t++) {
    ia[t + 1] = ia[t] + (t > 0);
    if (t > 0) ja[t - 1] = t - 1;
    rows[t] = t;
    if (t > 0) chunks.push_back(make_int2(t, t + 1));  // row 0 is never computed
  }
  DBuf<int> dia(n + 1, s), dja(n - 1, s), drows(n, s);
  DBuf<double> dval(n - 1, s), ddiag(n, s), din(n, s), dout(n, s);
  DBuf<int2> dch(chunks.size(), s);
  dia.upload(ia.data(), n + 1);
  dja.upload(ja.data(), n - 1);
  drows.upload(rows.data(), n);
  dval.upload(val.data(), n - 1);
  ddiag.upload(diag.data(), n);
  din.upload(in.data(), n);
  dch.upload(chunks.data(), chunks.size());
  dout.fill_bytes(0xff);
  WaitRecord wait;
  wait.init(s);
  wait.limit_ns = (unsigned long long)(limit_ms * 1e6);
  cudaEvent_t e0, e1;
  BN_CUDA(cudaEventCreate(&e0));
  BN_CUDA(cudaEventCreate(&e1));
  BN_CUDA(cudaEventRecord(e0, s));
  run_tri_flags<double>((int)chunks.size(), dch.p, 2, dia.p, dja.p, dval.p, ddiag.p, drows.p,
                        din.p, dout.p, nullptr, wait.ctl(WT_SELFTEST), s);
  BN_CUDA(cudaEventRecord(e1, s));
  BN_CUDA(cudaEventSynchronize(e1));
  float ms = 0.f;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (elapsed_ms) *elapsed_ms = ms;
  std::string msg;
  if (wait.take(s, &msg)) throw Error(BN_ERR_SPIN, "wait self-test: " + msg);
}

int IChol::mode_from_env() {
  // the chunked sync-free form measured fastest for the single-vector sweep
  // (20M network, FP32: 1.44 ms per sweep against 1.50 ms for the slab form
  // and 2.77 ms for the tiled form, whose block barriers make every level of
  // a tile wait for the slowest cross-tile dependency)
  const char* v = getenv("BN_IC_MODE");
  if (!v) return kSweepFlags;
  if (!strcmp(v, "levels")) return kSweepLevels;
  if (!strcmp(v, "coop")) return kSweepCoop;
  if (!strcmp(v, "tiles")) return kSweepTiles;
  if (!strcmp(v, "slab")) return kSweepSlab;
  if (!strcmp(v, "slabw")) return kSweepSlabW;
  return kSweepFlags;
}

}  // namespace bn

// See include/amg_b200.h for the contract.
BN_API int amg_debug_wait_timeout(int n, double limit_ms, double* elapsed_ms) {
  using namespace bn;
  try {
    wait_selftest(n, limit_ms, elapsed_ms, cudaStreamPerThread);
    set_last_error(BN_OK, "");
    return BN_OK;
  } catch (const Error& e) {
    set_last_error(e.code, e.what());
    return e.code;
  } catch (const std::exception& e) {
    set_last_error(BN_ERR_CUDA, e.what());
    return BN_ERR_CUDA;
  }
}
