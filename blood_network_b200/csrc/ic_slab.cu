// IC(0) triangular sweeps, slab form.
//
// The sync-free form spends one cross-SM round trip (a store reaching L2,
// then a poll reaching it) per dependency level, and the 20M-node vessel
// network has ~700 levels.  Here the rows are split into one slab per SM
// and a block owns a slab: it walks the slab's rows in level order, at most
// kSlabThreads rows (one per thread) per step, with a block barrier after
// each step.  A dependency on a row of the same slab computed a few steps
// earlier is read from a shared-memory ring of computed values (no round
// trip); only dependencies on other slabs, or on rows too old for the ring,
// are read from the output vector, and the first of them is pre-read by an
// asynchronous 16-byte copy when the step is staged, so that a value
// published in time costs nothing at the step itself.
//
// Staging (cp.async, one commit group per step and thread): the row
// records of step k+2G, then the entries, input values (and FP64
// diagonals) and the pre-read of step k+G; the wait for the group of step
// k-G+1 and the barrier end step k.  Every ring is indexed by the global
// position (or entry) modulo its size; the setup checks that the positions
// and entries in flight never exceed a ring (otherwise the form is off and
// the sync-free form runs).
//
// Slabs: rows of wide levels whose rows are packed in a narrow index range
// (the generations of a heap-numbered tree) are dealt evenly by their rank
// in the level; every other row goes by its rank in index order, so that a
// slab is a range of consecutive rows (planes of a capillary lattice).
//
// Progress: all slabs are co-resident (cooperative launch, one block per
// SM); a row waits only on rows of lower levels, and the slab holding the
// lowest unfinished level has all its dependencies published.  Every wait
// is bounded (flags.cuh): a wait that runs out raises the abort word and
// uses NaN, every block still runs its steps to the end.
//
// Arithmetic per row is the reference's (C_amg1/src/ichol.c:121-165): the
// input value minus the products in the row's entry order, then one
// division by the diagonal, so the result is bit-identical to the other
// sweep forms.
#include "ichol.cuh"
#include "flags.cuh"

#include <atomic>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <vector>
#include <cub/cub.cuh>

namespace bn {

namespace {

constexpr int kNT = IChol::kSlabThreads;
constexpr int kVS = 1024;  // ring of computed values (positions)
constexpr int kNS = 64;    // ring of step-table entries
// chunked slab form: kWT threads per block, 32-row chunks, a tagged ring of
// kVSW computed values
constexpr int kWT = 768, kWW = kWT / 32, kVSW = 4096;

template <class T>
struct SlabRings;
template <>
struct SlabRings<float> {
  static constexpr int A = 4096, B = 2048, E = 8192;
};
template <>
struct SlabRings<double> {
  static constexpr int A = 4096, B = 2048, E = 8192;
};

template <class T, int G>
constexpr size_t slab_smem_bytes() {
  using R = SlabRings<T>;
  return (size_t)R::A * 16 +                                     // row records
         (size_t)kNT * (G + 1) * 16 +                            // pre-read words
         (size_t)R::E * sizeof(T) +                              // entry values
         (size_t)R::B * sizeof(T) * (sizeof(T) == 8 ? 2 : 1) +   // diagonals (FP64), inputs
         (size_t)kVS * sizeof(T) +                               // computed values
         (size_t)kNS * 8 +                                       // step table
         (size_t)R::E * 4;                                       // entry codes
}

__device__ __forceinline__ unsigned smem_addr(const void* p) {
  return (unsigned)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void cpa16(void* dst, const void* src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_addr(dst)), "l"(src)
               : "memory");
}
template <int N>
__device__ __forceinline__ void cpa(void* dst, const void* src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], %2;" ::"r"(smem_addr(dst)), "l"(src),
               "n"(N)
               : "memory");
}
__device__ __forceinline__ void cpa_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cpa_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}
__device__ __forceinline__ void cpa_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

template <class T>
struct SlabArgs {
  const int2* slab_steps;  // per block: [first step, end step)
  const int2* steps;       // {first position, first entry}, one past the last step included
  const int4* rec;         // {vector row, first entry, pre-read dep or -1, FP32 diagonal bits}
  const int* code;         // entry: ring code (< 0: ~slot) or vector index of the dependency
  const T* ev;             // entry values
  const T* d;              // FP64 diagonals by position (FP32: rec.w)
  const T* in;
  T* out;
  T* clear;                // reset to the pending pattern row by row (or null)
  WaitCtl wc;
  int preread;             // 0: the output is not 16-byte aligned, no pre-reads
  unsigned long long* trace;  // diagnostics (BN_SLAB_TRACE): per block, time at each step end
  int trace_cap;              // steps recorded per block
};

template <class T, int G>
__global__ void __launch_bounds__(kNT, 1) k_tri_slab(SlabArgs<T> a) {
  using Wd = WordOf<T>;
  using U = typename Wd::U;
  using R = SlabRings<T>;
  constexpr int LA = 2 * G, GX = G + 1, WPS = 16 / (int)sizeof(U), LS = 3 * G + 1;
  constexpr int MA = R::A - 1, MB = R::B - 1, ME = R::E - 1, MV = kVS - 1, MS = kNS - 1;
  extern __shared__ __align__(16) unsigned char smem[];
  int4* sA = reinterpret_cast<int4*>(smem);
  uint4* sX = reinterpret_cast<uint4*>(sA + R::A);
  T* sV = reinterpret_cast<T*>(sX + kNT * GX);
  T* sD = sV + R::E;
  T* sIn = sD + (sizeof(T) == 8 ? R::B : 0);
  U* sXV = reinterpret_cast<U*>(sIn + R::B);
  int2* sS = reinterpret_cast<int2*>(sXV + kVS);
  int* sC = reinterpret_cast<int*>(sS + kNS);

  U* o = reinterpret_cast<U*>(a.out);
  const int tid = threadIdx.x;
  const int2 ss = a.slab_steps[blockIdx.x];
  const int s0 = ss.x, s1 = ss.y;
  if (s0 >= s1) return;
  // step-table entries s0 .. s0+LS now; later ones LS steps ahead (below)
  for (int i = tid; i <= LS && s0 + i <= s1; i += kNT) sS[(s0 + i) & MS] = a.steps[s0 + i];
  __syncthreads();

  // Issues this thread's copies for the steps ahead of step k.
  auto stage = [&](int k) {
    const int sa = k + LA;
    if (sa < s1) {
      const int p = sS[sa & MS].x + tid;
      if (p < sS[(sa + 1) & MS].x) cpa16(&sA[p & MA], a.rec + p);
    }
    const int sb = k + G;
    if (sb >= s0 && sb < s1) {
      const int2 b0 = sS[sb & MS], b1 = sS[(sb + 1) & MS];
      const int p = b0.x + tid;
      if (p < b1.x) {
        const int4 r = sA[p & MA];  // this thread's own copy, LA - G steps old
        cpa<sizeof(T)>(&sIn[p & MB], a.in + r.x);
        if constexpr (sizeof(T) == 8) cpa<8>(&sD[p & MB], a.d + p);
        if (a.preread && r.z >= 0) cpa16(&sX[(sb % GX) * kNT + tid], o + (r.z & ~(WPS - 1)));
      }
      for (int e = b0.y + tid; e < b1.y; e += kNT) {
        cpa<4>(&sC[e & ME], a.code + e);
        cpa<sizeof(T)>(&sV[e & ME], a.ev + e);
      }
    }
    if (tid == 0 && k > s0 && k + LS <= s1) cpa<8>(&sS[(k + LS) & MS], a.steps + k + LS);
  };

  // Computes this thread's row of step k (all its inputs staged and visible).
  auto compute = [&](int k) {
    const int2 c0 = sS[k & MS], c1 = sS[(k + 1) & MS];
    const int p = c0.x + tid;
    if (p >= c1.x) return;
    const int4 r = sA[p & MA];
    const int e1 = (p + 1 < c1.x) ? sA[(p + 1) & MA].y : c1.y;
    T s = sIn[p & MB];
    T d;
    if constexpr (sizeof(T) == 8) d = sD[p & MB];
    else d = __int_as_float(r.w);
    bool pre = a.preread && r.z >= 0;
    U pw = Wd::kPending;
    if (pre) pw = reinterpret_cast<const U*>(&sX[(k % GX) * kNT + tid])[r.z & (WPS - 1)];
    for (int e = r.y; e < e1; e += 4) {
      const int m = e1 - e < 4 ? e1 - e : 4;
      int j[4];
      T v[4];
      U u[4];
#pragma unroll
      for (int t = 0; t < 4; t++) {
        j[t] = 0;
        v[t] = T(0);
        u[t] = U(0);
        if (t < m) {
          const int c = sC[(e + t) & ME];
          v[t] = sV[(e + t) & ME];
          if (c < 0) {
            u[t] = sXV[~c];
          } else {
            j[t] = c;
            if (pre) {
              u[t] = pw;
              pre = false;
            } else {
              u[t] = ld_relaxed(o + c);
            }
          }
        }
      }
      wait_group(o, j, u, m, Wd::kPending, Wd::kNaN, a.wc, r.x);
#pragma unroll
      for (int t = 0; t < 4; t++) {
        if (t < m) {
          if constexpr (sizeof(T) == 8) s = xsub(s, xmul(v[t], word_value(u[t])));
          else s = xsubf(s, xmulf(v[t], word_value(u[t])));
        }
      }
    }
    U res = value_word(s / d);
    if (res == Wd::kPending) res = Wd::kNaN;
    sXV[p & MV] = res;
    st_relaxed(o + r.x, res);
    if (a.clear) reinterpret_cast<U*>(a.clear)[r.x] = Wd::kPending;
  };

  // prime the pipeline: the copies of the LA steps before s0
  for (int k = s0 - LA; k < s0; k++) {
    cpa_wait<G - 1>();
    stage(k);
    cpa_commit();
  }
  cpa_wait<G - 1>();
  __syncthreads();
  unsigned long long* tr = a.trace ? a.trace + (size_t)blockIdx.x * a.trace_cap : nullptr;
  if (tr && tid == 0) tr[0] = global_ns();
  for (int k = s0; k < s1; k++) {
    stage(k);
    cpa_commit();
    compute(k);
    cpa_wait<G - 1>();
    __syncthreads();
    if (tr && tid == 0 && k - s0 + 1 < a.trace_cap) tr[k - s0 + 1] = global_ns();
  }
  cpa_wait_all();
}

// ------------------------------------------------------------ layout build
struct MaxOp {
  __device__ __forceinline__ int operator()(int a, int b) const { return a > b ? a : b; }
};

// Largest number of rows of one level that a slab of consecutive rows
// (slab = row / R) would hold: rows of a level are in index order in the
// level-ordered layout, so each (level, slab) group is one run of positions.
__global__ void k_level_runs(const int* __restrict__ rows, const int* __restrict__ lev, int n,
                             int R, int* __restrict__ maxrun) {
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
    const int l = lev[t], q = rows[t] / R;
    const bool head = t == 0 || lev[t - 1] != l || rows[t - 1] / R != q;
    if (!head) continue;
    int e = t + 1;
    while (e < n && lev[e] == l && rows[e] / R == q && e - t <= 2 * kNT) e++;
    atomicMax(&maxrun[l], e - t);
  }
}

// rows of dealt levels: slab by rank in the level; flag[i] = 1 for the others
__global__ void k_slab_dealt(const int* __restrict__ order, const int* __restrict__ lev,
                             const int* __restrict__ lptr, const unsigned char* __restrict__ dealt,
                             int n, int nslab, int* __restrict__ slab_of, int* __restrict__ flag) {
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
    const int l = lev[t], i = order[t];
    if (dealt[l]) {
      const long long w = lptr[l + 1] - lptr[l];
      slab_of[i] = (int)((long long)(t - lptr[l]) * nslab / w);
      flag[i] = 0;
    } else {
      flag[i] = 1;
    }
  }
}

__global__ void k_slab_ranked(const int* __restrict__ rank, int n, long long m, int nslab,
                              int* __restrict__ slab_of) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    if (rank[i + 1] != rank[i]) slab_of[i] = (int)((long long)rank[i] * nslab / m);
}

__global__ void k_slab_key(const int* __restrict__ rows, const int* __restrict__ slab_of, int n,
                           int* __restrict__ key, int* __restrict__ ids) {
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
    key[t] = slab_of[rows[t]];
    ids[t] = t;
  }
}

// hv[p] = p at the first position of a (slab, level) run, else 0
__global__ void k_slab_runs(const int* __restrict__ perm, const int* __restrict__ keys,
                            const int* __restrict__ lev, int n, int* __restrict__ hv) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
    const bool h = p == 0 || keys[p] != keys[p - 1] || lev[perm[p]] != lev[perm[p - 1]];
    hv[p] = h ? p : 0;
  }
}

// step heads: run starts and every cap-th position of a run
__global__ void k_slab_heads(const int* __restrict__ runstart, int n, int cap,
                             int* __restrict__ head) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x)
    head[p] = ((p - runstart[p]) % cap) == 0;
}

__global__ void k_slab_counts(const int* __restrict__ perm, const int* __restrict__ tia,
                              const int* __restrict__ rows, int n, int* __restrict__ cnt,
                              int* __restrict__ rnat, int* __restrict__ newpos) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
    const int t = perm[p];
    cnt[p] = tia[t + 1] - tia[t];
    const int i = rows[t];
    rnat[p] = i;
    newpos[i] = p;
  }
}

__global__ void k_slab_steps(const int* __restrict__ head, const int* __restrict__ sid,
                             const int* __restrict__ eo, int n, int nsteps, int nnz,
                             int2* __restrict__ steps) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
    if (head[p]) steps[sid[p] - 1] = make_int2(p, eo[p]);
    if (p == 0) steps[nsteps] = make_int2(n, nnz);
  }
}

__global__ void k_slab_ranges(const int2* __restrict__ steps, const int* __restrict__ keys,
                              int nsteps, int2* __restrict__ slab_steps) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nsteps; k += gridDim.x * blockDim.x) {
    const int q = keys[steps[k].x];
    if (k == 0 || keys[steps[k - 1].x] != q) slab_steps[q].x = k;
    if (k == nsteps - 1 || keys[steps[k + 1].x] != q) slab_steps[q].y = k + 1;
  }
}

// entries in slab order: ring code for a dependency on the same slab that
// the ring still holds when the row is computed, the natural dependency
// otherwise.  Stepped form: code ~slot, held while the dependency is at most
// kVS positions before the end of the row's step.  Chunked form: code
// -(distance back), held while the distance is at most kVSW less the
// positions a block has in flight (kWW chunks of 32).
__global__ void k_slab_entries(const int* __restrict__ perm, const int* __restrict__ keys,
                               const int* __restrict__ sid, const int2* __restrict__ steps,
                               const int* __restrict__ eo, const int* __restrict__ tia,
                               const int* __restrict__ tja, const int* __restrict__ tsrc,
                               const int* __restrict__ slab_of, const int* __restrict__ newpos,
                               int n, int chunked, int* __restrict__ cnat, int* __restrict__ esrc,
                               int* __restrict__ xnat) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
    const int t = perm[p], q = keys[p];
    const int p1 = steps[sid[p]].x;  // first position of the next step
    const int b = tia[t], c = tia[t + 1] - b, o = eo[p];
    int xs = -1;
    for (int m = 0; m < c; m++) {
      const int j = tja[b + m];
      const int qp = newpos[j];
      bool ring;
      int code;
      if (chunked) {
        ring = slab_of[j] == q && p - qp <= kVSW - 32 * kWW;
        code = qp - p;
      } else {
        ring = slab_of[j] == q && qp >= p1 - kVS;
        code = ~(qp & (kVS - 1));
      }
      cnat[o + m] = ring ? code : j;
      esrc[o + m] = tsrc[b + m];
      if (!ring && xs < 0) xs = j;
    }
    xnat[p] = xs;
  }
}

// positions and entries in flight for staging leads 2 and 3:
// w[0..2] = lead 2 (records, inputs, entries), w[3..5] = lead 3
__global__ void k_slab_windows(const int2* __restrict__ steps, const int* __restrict__ keys,
                               const int2* __restrict__ slab_steps, int nsteps,
                               int* __restrict__ w) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nsteps; k += gridDim.x * blockDim.x) {
    const int end = slab_steps[keys[steps[k].x]].y;
    const int2 s = steps[k];
#pragma unroll
    for (int g = 2; g <= 3; g++) {
      const int ka = k + 2 * g + 1 < end ? k + 2 * g + 1 : end;
      const int kb = k + g + 1 < end ? k + g + 1 : end;
      atomicMax(&w[(g - 2) * 3 + 0], steps[ka].x - s.x);
      atomicMax(&w[(g - 2) * 3 + 1], steps[kb].x - s.x);
      atomicMax(&w[(g - 2) * 3 + 2], steps[kb].y - s.y);
    }
  }
}

__global__ void k_slab_vids(const int* __restrict__ rnat, const int* __restrict__ xnat, int n,
                            const int* __restrict__ inv, int* __restrict__ vrow,
                            int* __restrict__ vx) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
    vrow[p] = inv ? inv[rnat[p]] : rnat[p];
    int x = xnat[p];
    if (x >= 0) {
      x = inv ? inv[x] : x;
      if ((x & ~3) + 4 > n) x = -1;  // the 16-byte pre-read must lie inside the vector
    }
    vx[p] = x;
  }
}

__global__ void k_slab_codes(const int* __restrict__ cnat, int m, const int* __restrict__ inv,
                             int* __restrict__ code) {
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < m; e += gridDim.x * blockDim.x) {
    const int c = cnat[e];
    code[e] = (c < 0 || !inv) ? c : inv[c];
  }
}

__global__ void k_slab_rec(const int* __restrict__ vrow, const int* __restrict__ vx,
                           const float* __restrict__ d32, int n, int4* __restrict__ rec) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
    int4 r = rec[p];
    r.x = vrow[p];
    r.z = vx[p];
    r.w = d32 ? __float_as_int(d32[p]) : 0;
    rec[p] = r;
  }
}

__global__ void k_slab_init_rec(const int* __restrict__ eo, int n, int4* __restrict__ rec) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x)
    rec[p] = make_int4(0, eo[p], -1, 0);
}

template <class T>
__global__ void k_slab_gather(const int* __restrict__ src, int m, const double* __restrict__ lval,
                              T* __restrict__ out) {
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < m; e += gridDim.x * blockDim.x)
    out[e] = (T)lval[src[e]];
}

template <class T>
__global__ void k_slab_diag(const int* __restrict__ rnat, int n, const int* __restrict__ dpos,
                            const double* __restrict__ lval, T* __restrict__ out) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x)
    out[p] = (T)lval[dpos[rnat[p]]];
}

template <class T, int G>
void slab_launch(const IChol::Slab& sl, int nslab, const T* d, const T* ev, const T* in, T* out,
                 T* clear, WaitCtl wc, cudaStream_t s) {
  constexpr size_t smem = slab_smem_bytes<T, G>();
  static std::atomic<unsigned long long> attr_set{0};
  int dev = 0;
  BN_CUDA(cudaGetDevice(&dev));
  const unsigned long long bit = 1ull << (dev & 63);
  if (!(attr_set.load() & bit)) {
    BN_CUDA(cudaFuncSetAttribute(k_tri_slab<T, G>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)smem));
    attr_set.fetch_or(bit);
  }
  SlabArgs<T> a;
  a.slab_steps = sl.slab_steps.p;
  a.steps = sl.steps.p;
  a.rec = sl.rec.p;
  a.code = sl.code.p;
  a.ev = ev;
  a.d = d;
  a.in = in;
  a.out = out;
  a.clear = clear;
  a.wc = wc;
  a.preread = ((uintptr_t)out & 15) == 0;
  a.trace = nullptr;
  a.trace_cap = 0;
  // BN_SLAB_TRACE=<file>: append {nslab, cap, per-block [first step, end step), per-block step
  // end times} of every sweep (synchronous; diagnostics only)
  static const char* trace_path = getenv("BN_SLAB_TRACE");
  DBuf<unsigned long long> tbuf;
  if (trace_path) {
    a.trace_cap = 4096;
    tbuf.alloc((size_t)nslab * a.trace_cap, s);
    tbuf.zero();
    a.trace = tbuf.p;
  }
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(nslab);
  cfg.blockDim = dim3(kNT);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;  // co-residency: waits always end
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  g_launch_count++;
  BN_CUDA(cudaLaunchKernelEx(&cfg, k_tri_slab<T, G>, a));
  if (trace_path) {
    std::vector<unsigned long long> h((size_t)nslab * a.trace_cap);
    std::vector<int2> ss(nslab);
    tbuf.download(h.data(), h.size());
    sl.slab_steps.download(ss.data(), nslab);
    BN_CUDA(cudaStreamSynchronize(s));
    if (FILE* f = fopen(trace_path, "ab")) {
      const int hdr[2] = {nslab, a.trace_cap};
      fwrite(hdr, sizeof(int), 2, f);
      fwrite(ss.data(), sizeof(int2), nslab, f);
      fwrite(h.data(), sizeof(unsigned long long), h.size(), f);
      fclose(f);
    }
  }
}

template <class T, int G>
bool slab_fits_device() {
  constexpr size_t smem = slab_smem_bytes<T, G>();
  int dev = 0, optin = 0, per_sm = 0;
  BN_CUDA(cudaGetDevice(&dev));
  BN_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
  if ((size_t)optin < smem) return false;
  BN_CUDA(cudaFuncSetAttribute(k_tri_slab<T, G>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)smem));
  BN_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_tri_slab<T, G>, kNT, smem));
  return per_sm >= 1;
}

// ------------------------------------------------------------ chunked form
// The same slabs without block barriers: the warps of a block take the
// slab's 32-row chunks (cut at level boundaries) in order, chunk c to warp
// c mod kWW, and a row waits only for its own dependencies: a recent row of
// the slab through a ring of computed values in shared memory, each slot
// tagged with the position it holds (a reader waits for its position's
// tag), every other dependency through the output vector as in the
// sync-free form.  A warp starts chunk c only when every warp of the block
// is past chunk c - kWW (progress words in shared memory), so a block has at
// most kWW chunks in flight and a slot is rewritten (position q + kVSW)
// only after every reader of q has read it.
// Each warp loads the records of its chunk after next and the inputs and
// entries of its next chunk before it works on the current one.
template <class T>
struct ChunkRec {
  int p, p1, e1;  // this lane's position, the chunk's end position and end entry
  int4 r;         // record (r.y: first entry)
};
template <class T>
struct ChunkDat {
  T in, d;
  int cnt;        // entries of the row
  int code[4];
  T val[4];
};

template <class T>
__device__ __forceinline__ ChunkRec<T> chunk_rec(const SlabArgs<T>& a, int c, int s1, int lane) {
  ChunkRec<T> q;
  q.p = 0;
  q.p1 = 0;
  q.e1 = 0;
  q.r = make_int4(0, 0, -1, 0);
  if (c < s1) {
    const int2 b0 = a.steps[c], b1 = a.steps[c + 1];
    q.p = b0.x + lane;
    q.p1 = b1.x;
    q.e1 = b1.y;
    if (q.p < q.p1) q.r = a.rec[q.p];
  }
  return q;
}

template <class T>
__device__ __forceinline__ ChunkDat<T> chunk_dat(const SlabArgs<T>& a, const ChunkRec<T>& q) {
  ChunkDat<T> d;
  const int nxt = __shfl_down_sync(0xffffffffu, q.r.y, 1);
  d.cnt = 0;
  d.in = T(0);
  d.d = T(1);
#pragma unroll
  for (int t = 0; t < 4; t++) {
    d.code[t] = 0;
    d.val[t] = T(0);
  }
  if (q.p < q.p1) {
    const int e1 = q.p + 1 < q.p1 ? nxt : q.e1;
    d.cnt = e1 - q.r.y;
    d.in = a.in[q.r.x];
    if constexpr (sizeof(T) == 8) d.d = a.d[q.p];
    else d.d = __int_as_float(q.r.w);
#pragma unroll
    for (int t = 0; t < 4; t++) {
      if (t < d.cnt) {
        d.code[t] = a.code[q.r.y + t];
        d.val[t] = a.ev[q.r.y + t];
      }
    }
  }
  return d;
}

// Value of position q from the ring (waits for its tag; bounded).
template <class T>
__device__ __forceinline__ typename WordOf<T>::U ring_get(unsigned long long* sR, int* sTag,
                                                          int q, const WaitCtl& wc, int row) {
  using U = typename WordOf<T>::U;
  const int slot = q & (kVSW - 1);
  unsigned long long t0 = 0;
  for (int it = 0;; it++) {
    if constexpr (sizeof(T) == 4) {
      const unsigned long long v = *reinterpret_cast<volatile unsigned long long*>(&sR[slot]);
      if ((int)(unsigned)(v & 0xffffffffull) == q) return (U)(v >> 32);
    } else {
      if (*reinterpret_cast<volatile int*>(&sTag[slot]) == q) {
        __threadfence_block();
        return (U)(*reinterpret_cast<volatile unsigned long long*>(&sR[slot]));
      }
    }
    bool ran_out = false;
    if (it >= kSpinFast && wait_backoff(wc, it, t0, &ran_out)) {
      if (ran_out) wait_give_up(wc, row, q, global_ns() - t0);
      return WordOf<T>::kNaN;
    }
  }
}

template <class T>
__device__ __forceinline__ void ring_put(unsigned long long* sR, int* sTag, int p,
                                         typename WordOf<T>::U w) {
  const int slot = p & (kVSW - 1);
  if constexpr (sizeof(T) == 4) {
    *reinterpret_cast<volatile unsigned long long*>(&sR[slot]) =
        ((unsigned long long)w << 32) | (unsigned)p;
  } else {
    *reinterpret_cast<volatile unsigned long long*>(&sR[slot]) = w;
    __threadfence_block();
    *reinterpret_cast<volatile int*>(&sTag[slot]) = p;
  }
}

template <class T>
__global__ void __launch_bounds__(kWT, 1) k_tri_slabw(SlabArgs<T> a) {
  using Wd = WordOf<T>;
  using U = typename Wd::U;
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ int sProg[kWW];  // per warp: its next chunk (all its earlier ones done)
  unsigned long long* sR = reinterpret_cast<unsigned long long*>(smem);
  int* sTag = reinterpret_cast<int*>(sR + kVSW);  // FP64 only
  U* o = reinterpret_cast<U*>(a.out);
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  const int2 ss = a.slab_steps[blockIdx.x];
  const int s0 = ss.x, s1 = ss.y;
  if (s0 >= s1) return;
  for (int i = tid; i < kVSW; i += kWT) {
    if constexpr (sizeof(T) == 4) sR[i] = 0xffffffffull;  // tag -1
    else sTag[i] = -1;
  }
  if (tid < kWW) sProg[tid] = s0 + tid;
  __syncthreads();
  int c = s0 + w;
  ChunkRec<T> r0 = chunk_rec(a, c, s1, lane);
  ChunkRec<T> r1 = chunk_rec(a, c + kWW, s1, lane);
  ChunkDat<T> d0 = chunk_dat(a, r0);
  for (; c < s1; c += kWW) {
    const ChunkRec<T> r2 = chunk_rec(a, c + 2 * kWW, s1, lane);
    const ChunkDat<T> d1 = chunk_dat(a, r1);
    {  // gate: no warp of the block more than kWW chunks behind
      unsigned long long t0 = 0;
      for (int it = 0;; it++) {
        int m = lane < kWW ? *reinterpret_cast<volatile int*>(&sProg[lane]) : 0x7fffffff;
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) {
          const int v = __shfl_xor_sync(0xffffffffu, m, off);
          m = v < m ? v : m;
        }
        if (c < m + kWW) break;
        bool ran_out = false;
        if (it >= kSpinFast && wait_backoff(a.wc, it, t0, &ran_out)) {
          if (ran_out && lane == 0) wait_give_up(a.wc, -1, c, global_ns() - t0);
          break;
        }
      }
    }
    if (r0.p < r0.p1) {
      const int p = r0.p, vi = r0.r.x;
      T s = d0.in;
      for (int e = 0; e < d0.cnt; e += 4) {
        const int m = d0.cnt - e < 4 ? d0.cnt - e : 4;
        int j[4];
        T v[4];
        U u[4];
#pragma unroll
        for (int t = 0; t < 4; t++) {
          j[t] = 0;
          v[t] = T(0);
          u[t] = U(0);
          if (t < m) {
            int cd;
            if (e == 0) {
              cd = d0.code[t];
              v[t] = d0.val[t];
            } else {
              cd = a.code[r0.r.y + e + t];
              v[t] = a.ev[r0.r.y + e + t];
            }
            if (cd < 0) {
              u[t] = ring_get<T>(sR, sTag, p + cd, a.wc, vi);
            } else {
              j[t] = cd;
              u[t] = ld_relaxed(o + cd);
            }
          }
        }
        wait_group(o, j, u, m, Wd::kPending, Wd::kNaN, a.wc, vi);
#pragma unroll
        for (int t = 0; t < 4; t++) {
          if (t < m) {
            if constexpr (sizeof(T) == 8) s = xsub(s, xmul(v[t], word_value(u[t])));
            else s = xsubf(s, xmulf(v[t], word_value(u[t])));
          }
        }
      }
      U res = value_word(s / d0.d);
      if (res == Wd::kPending) res = Wd::kNaN;
      ring_put<T>(sR, sTag, p, res);
      st_relaxed(o + vi, res);
      if (a.clear) reinterpret_cast<U*>(a.clear)[vi] = Wd::kPending;
    }
    __syncwarp();
    if (lane == 0) *reinterpret_cast<volatile int*>(&sProg[w]) = c + kWW;
    r0 = r1;
    r1 = r2;
    d0 = d1;
  }
}

template <class T>
constexpr size_t slabw_smem_bytes() {
  return (size_t)kVSW * 8 + (sizeof(T) == 8 ? (size_t)kVSW * 4 : 0);
}

template <class T>
bool slab_fits_chunked() {
  int per_sm = 0;
  BN_CUDA(cudaFuncSetAttribute(k_tri_slabw<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)slabw_smem_bytes<T>()));
  BN_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_tri_slabw<T>, kWT,
                                                        slabw_smem_bytes<T>()));
  return per_sm >= 1;
}

template <class T>
void slabw_launch(const IChol::Slab& sl, int nslab, const T* d, const T* ev, const T* in, T* out,
                  T* clear, WaitCtl wc, cudaStream_t s) {
  constexpr size_t smem = slabw_smem_bytes<T>();
  static std::atomic<unsigned long long> attr_set{0};
  int dev = 0;
  BN_CUDA(cudaGetDevice(&dev));
  const unsigned long long bit = 1ull << (dev & 63);
  if (!(attr_set.load() & bit)) {
    BN_CUDA(cudaFuncSetAttribute(k_tri_slabw<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)smem));
    attr_set.fetch_or(bit);
  }
  SlabArgs<T> a;
  a.slab_steps = sl.slab_steps.p;
  a.steps = sl.steps.p;
  a.rec = sl.rec.p;
  a.code = sl.code.p;
  a.ev = ev;
  a.d = d;
  a.in = in;
  a.out = out;
  a.clear = clear;
  a.wc = wc;
  a.preread = 0;
  a.trace = nullptr;
  a.trace_cap = 0;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(nslab);
  cfg.blockDim = dim3(kWT);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;  // co-residency: waits always end
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  g_launch_count++;
  BN_CUDA(cudaLaunchKernelEx(&cfg, k_tri_slabw<T>, a));
}

}  // namespace

// One slab per SM.  A level of which a slab of consecutive rows would hold
// more than two steps' worth (a generation of a heap-numbered tree) has its
// rows dealt to all slabs by rank; the other rows go to slabs of
// consecutive rows.
void IChol::build_slab_partition(cudaStream_t s) {
  int dev = 0;
  BN_CUDA(cudaGetDevice(&dev));
  BN_CUDA(cudaDeviceGetAttribute(&nslab, cudaDevAttrMultiProcessorCount, dev));
  slab_of.alloc(n > 0 ? n : 1, s);
  if (n == 0) return;
  const int g = grid_for(n, 256);
  DBuf<int> maxrun(nlevels, s), lev(n, s);
  maxrun.zero();
  BN_LAUNCH(k_pos_level, g, 256, 0, s, d_lptr.p, nlevels, n, lev.p);
  const int R = (n + nslab - 1) / nslab;
  BN_LAUNCH(k_level_runs, g, 256, 0, s, order.p, lev.p, n, R, maxrun.p);
  std::vector<int> hrun(nlevels);
  maxrun.download(hrun.data(), nlevels);
  BN_CUDA(cudaStreamSynchronize(s));
  std::vector<unsigned char> hd(nlevels);
  for (int l = 0; l < nlevels; l++) hd[l] = hrun[l] > 2 * kSlabThreads ? 1 : 0;
  DBuf<unsigned char> dealt(nlevels, s);
  dealt.upload(hd.data(), nlevels);
  DBuf<int> flag((size_t)n + 1, s);
  BN_LAUNCH(k_slab_dealt, g, 256, 0, s, order.p, lev.p, d_lptr.p, dealt.p, n, nslab, slab_of.p,
            flag.p);
  const int m = scan_counts(flag.p, n, s);
  if (m > 0) BN_LAUNCH(k_slab_ranked, g, 256, 0, s, flag.p, n, (long long)m, nslab, slab_of.p);
}

void IChol::build_slab(bool forward, cudaStream_t s) {
  Slab& sl = forward ? sf : sb;
  sl.lead32 = sl.lead64 = 0;
  sl.nsteps = 0;
  sl.nnz = offd_nnz;
  const int* rows = forward ? order.p : border.p;
  const DBuf<int>& dptr = forward ? d_lptr : d_bptr;
  const int* tia = forward ? fia.p : bia.p;
  const int* tja = forward ? fja.p : bja.p;
  const int* tsrc = forward ? fsrc.p : bsrc.p;
  const int m = offd_nnz > 0 ? offd_nnz : 1;
  sl.slab_steps.alloc(nslab > 0 ? nslab : 1, s);
  sl.slab_steps.zero();
  sl.rec.alloc(n > 0 ? n : 1, s);
  sl.rnat.alloc(n > 0 ? n : 1, s);
  sl.xnat.alloc(n > 0 ? n : 1, s);
  sl.vrow.alloc(n > 0 ? n : 1, s);
  sl.vx.alloc(n > 0 ? n : 1, s);
  sl.cnat.alloc(m, s);
  sl.code.alloc(m, s);
  sl.esrc.alloc(m, s);
  if (n == 0) {
    sl.steps.alloc(1, s);
    return;
  }
  const int g = grid_for(n, 256);
  DBuf<int> lev(n, s), key(n, s), ids(n, s), keys(n, s), perm(n, s);
  BN_LAUNCH(k_pos_level, g, 256, 0, s, dptr.p, nlevels, n, lev.p);
  BN_LAUNCH(k_slab_key, g, 256, 0, s, rows, slab_of.p, n, key.p, ids.p);
  int eb = 1;
  while ((1 << eb) <= nslab) eb++;
  size_t tmp = 0;
  BN_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tmp, key.p, keys.p, ids.p, perm.p, n, 0, eb, s));
  {
    DBuf<unsigned char> t(tmp, s);
    BN_CUDA(cub::DeviceRadixSort::SortPairs(t.p, tmp, key.p, keys.p, ids.p, perm.p, n, 0, eb, s));
  }
  // steps: (slab, level) runs cut every kSlabThreads positions
  DBuf<int> hv(n, s), runstart(n, s), head(n, s), sid(n, s);
  BN_LAUNCH(k_slab_runs, g, 256, 0, s, perm.p, keys.p, lev.p, n, hv.p);
  tmp = 0;
  BN_CUDA(cub::DeviceScan::InclusiveScan(nullptr, tmp, hv.p, runstart.p, MaxOp(), n, s));
  {
    DBuf<unsigned char> t(tmp, s);
    BN_CUDA(cub::DeviceScan::InclusiveScan(t.p, tmp, hv.p, runstart.p, MaxOp(), n, s));
  }
  const bool chunked = mode == kSweepSlabW;
  BN_LAUNCH(k_slab_heads, g, 256, 0, s, runstart.p, n, chunked ? 32 : kNT, head.p);
  tmp = 0;
  BN_CUDA(cub::DeviceScan::InclusiveSum(nullptr, tmp, head.p, sid.p, n, s));
  {
    DBuf<unsigned char> t(tmp, s);
    BN_CUDA(cub::DeviceScan::InclusiveSum(t.p, tmp, head.p, sid.p, n, s));
  }
  const int nsteps = read_scalar(sid.p + (n - 1), s);
  sl.nsteps = nsteps;
  // entry offsets by position, natural rows, positions of the natural rows
  DBuf<int> eo((size_t)n + 1, s), newpos(n, s);
  BN_LAUNCH(k_slab_counts, g, 256, 0, s, perm.p, tia, rows, n, eo.p, sl.rnat.p, newpos.p);
  const int nnz = scan_counts(eo.p, n, s);
  BN_REQUIRE(nnz == offd_nnz, BN_ERR_CUDA, "IC(0) slab layout: entry count");
  sl.steps.alloc((size_t)nsteps + 1, s);
  BN_LAUNCH(k_slab_steps, g, 256, 0, s, head.p, sid.p, eo.p, n, nsteps, nnz, sl.steps.p);
  BN_LAUNCH(k_slab_ranges, grid_for(nsteps, 256), 256, 0, s, sl.steps.p, keys.p, nsteps,
            sl.slab_steps.p);
  BN_LAUNCH(k_slab_entries, g, 256, 0, s, perm.p, keys.p, sid.p, sl.steps.p, eo.p, tia, tja, tsrc,
            slab_of.p, newpos.p, n, chunked ? 1 : 0, sl.cnat.p, sl.esrc.p, sl.xnat.p);
  BN_LAUNCH(k_slab_init_rec, g, 256, 0, s, eo.p, n, sl.rec.p);
  if (chunked) {  // no staging rings: the chunked kernel only needs its value ring
    sl.lead32 = slab_fits_chunked<float>() ? 1 : 0;
    sl.lead64 = slab_fits_chunked<double>() ? 1 : 0;
  } else {
  // ring fit for the staging leads
  DBuf<int> w(6, s);
  w.zero();
  BN_LAUNCH(k_slab_windows, grid_for(nsteps, 256), 256, 0, s, sl.steps.p, keys.p, sl.slab_steps.p,
            nsteps, w.p);
  int hw[6];
  w.download(hw, 6);
  BN_CUDA(cudaStreamSynchronize(s));
  auto fits = [&](int gi, int ra, int rb, int re) {
    return hw[gi * 3] <= ra && hw[gi * 3 + 1] <= rb && hw[gi * 3 + 2] <= re;
  };
  using R32 = SlabRings<float>;
  using R64 = SlabRings<double>;
  if (fits(1, R32::A, R32::B, R32::E) && slab_fits_device<float, 3>()) sl.lead32 = 3;
  else if (fits(0, R32::A, R32::B, R32::E) && slab_fits_device<float, 2>()) sl.lead32 = 2;
  if (fits(1, R64::A, R64::B, R64::E) && slab_fits_device<double, 3>()) sl.lead64 = 3;
  else if (fits(0, R64::A, R64::B, R64::E) && slab_fits_device<double, 2>()) sl.lead64 = 2;
  if (const char* e = getenv("BN_SLAB_LEAD")) {  // cap the staging lead (2 or 3)
    const int cap = atoi(e);
    if (cap == 2) {
      sl.lead32 = fits(0, R32::A, R32::B, R32::E) && sl.lead32 ? 2 : 0;
      sl.lead64 = fits(0, R64::A, R64::B, R64::E) && sl.lead64 ? 2 : 0;
    }
  }
  if (getenv("BN_SLAB_TRACE"))
    fprintf(stderr,
            "IC(0) slab layout (%s): %d slabs, %d steps; in flight at lead 2: %d/%d/%d, "
            "lead 3: %d/%d/%d (records/inputs/entries); lead FP32 %d, FP64 %d\n",
            forward ? "forward" : "backward", nslab, nsteps, hw[0], hw[1], hw[2], hw[3], hw[4],
            hw[5], sl.lead32, sl.lead64);
  }
  // vector numbering: natural until remap()
  BN_LAUNCH(k_slab_vids, g, 256, 0, s, sl.rnat.p, sl.xnat.p, n, (const int*)nullptr, sl.vrow.p,
            sl.vx.p);
  if (offd_nnz > 0)
    BN_LAUNCH(k_slab_codes, grid_for(offd_nnz, 256), 256, 0, s, sl.cnat.p, offd_nnz,
              (const int*)nullptr, sl.code.p);
}

void IChol::slab_values(Slab& sl, cudaStream_t s) {
  const int m = offd_nnz > 0 ? offd_nnz : 1;
  sl.ev64.alloc(m, s);
  sl.d64.alloc(n > 0 ? n : 1, s);
  if (want_f32) {
    sl.ev32.alloc(m, s);
    sl.d32.alloc(n > 0 ? n : 1, s);
  }
  if (n == 0) return;
  if (offd_nnz > 0) {
    BN_LAUNCH(k_slab_gather<double>, grid_for(offd_nnz, 256), 256, 0, s, sl.esrc.p, offd_nnz,
              L.val.p, sl.ev64.p);
    if (want_f32)
      BN_LAUNCH(k_slab_gather<float>, grid_for(offd_nnz, 256), 256, 0, s, sl.esrc.p, offd_nnz,
                L.val.p, sl.ev32.p);
  }
  BN_LAUNCH(k_slab_diag<double>, grid_for(n, 256), 256, 0, s, sl.rnat.p, n, dpos.p, L.val.p,
            sl.d64.p);
  if (want_f32)
    BN_LAUNCH(k_slab_diag<float>, grid_for(n, 256), 256, 0, s, sl.rnat.p, n, dpos.p, L.val.p,
              sl.d32.p);
  BN_LAUNCH(k_slab_rec, grid_for(n, 256), 256, 0, s, sl.vrow.p, sl.vx.p,
            (const float*)(sl.d32.n ? sl.d32.p : nullptr), n, sl.rec.p);
}

void IChol::slab_pack(Slab& sl, const int* inv, cudaStream_t s) {
  if (n == 0) return;
  BN_LAUNCH(k_slab_vids, grid_for(n, 256), 256, 0, s, sl.rnat.p, sl.xnat.p, n, inv, sl.vrow.p,
            sl.vx.p);
  if (offd_nnz > 0)
    BN_LAUNCH(k_slab_codes, grid_for(offd_nnz, 256), 256, 0, s, sl.cnat.p, offd_nnz, inv,
              sl.code.p);
  BN_LAUNCH(k_slab_rec, grid_for(n, 256), 256, 0, s, sl.vrow.p, sl.vx.p,
            (const float*)(sl.d32.n ? sl.d32.p : nullptr), n, sl.rec.p);
}

template <class T>
void run_tri_slab(const IChol& ic, bool forward, const T* in, T* out, T* clear, WaitCtl wc,
                  cudaStream_t s) {
  const IChol::Slab& sl = forward ? ic.sf : ic.sb;
  if (ic.mode == IChol::kSweepSlabW) {
    if constexpr (sizeof(T) == 8)
      slabw_launch<double>(sl, ic.nslab, sl.d64.p, sl.ev64.p, in, out, clear, wc, s);
    else
      slabw_launch<float>(sl, ic.nslab, (const float*)nullptr, sl.ev32.p, in, out, clear, wc, s);
    return;
  }
  if constexpr (sizeof(T) == 8) {
    if (sl.lead64 == 3)
      slab_launch<double, 3>(sl, ic.nslab, sl.d64.p, sl.ev64.p, in, out, clear, wc, s);
    else
      slab_launch<double, 2>(sl, ic.nslab, sl.d64.p, sl.ev64.p, in, out, clear, wc, s);
  } else {
    if (sl.lead32 == 3)
      slab_launch<float, 3>(sl, ic.nslab, (const float*)nullptr, sl.ev32.p, in, out, clear, wc, s);
    else
      slab_launch<float, 2>(sl, ic.nslab, (const float*)nullptr, sl.ev32.p, in, out, clear, wc, s);
  }
}

template void run_tri_slab<double>(const IChol&, bool, const double*, double*, double*, WaitCtl,
                                   cudaStream_t);
template void run_tri_slab<float>(const IChol&, bool, const float*, float*, float*, WaitCtl,
                                  cudaStream_t);

}  // namespace bn
