// AMG-PCG solver on one B200: hierarchy setup, smoothers, the three-stage
// AMG + IC(0) preconditioner, PCG, and the amg_solver_* C ABI.
//
// Reference call structure (C_amg1):
//   amg_solver_create  amg_wrapper.c:51-97   copy, symmetrise, build, IC(0)
//   amg_build_hierarchy build_hierarchy.c:29-156
//   amg_ichol_precond  amg_ichol_precond.c:22-59
//   backslash/fwdslash amg_cycle.c:180-253
//   amg_pcg            amg_pcg.c:12-101
// Setup kernels reproduce the reference bit for bit (strength, PMIS,
// interpolation, RAP, symmetrisation, IC(0)); the solve phase uses a
// multicolour Gauss-Seidel in place of the sequential CF-ordered sweep and a
// dense direct coarse solve in place of the coarse PCG.
#include "solver.cuh"

#include <cub/cub.cuh>
#include <math.h>
#include <string.h>
#include <algorithm>
#include <memory>

namespace bn {

// ------------------------------------------------------------ colouring
__device__ __forceinline__ unsigned color_hash(unsigned x) {
  // bijective 32-bit mix: distinct rows get distinct priorities
  x ^= x >> 16; x *= 0x7feb352du; x ^= x >> 15; x *= 0x846ca68bu; x ^= x >> 16;
  return x;
}

// Jones-Plassmann-Luby rounds with first-fit colours (largest-degree-first
// priorities): an uncoloured row whose priority beats every uncoloured
// neighbour of its own set takes the
// smallest colour that no already-coloured neighbour of its set holds.
// Rows selected in one round are never adjacent, so the colouring is
// proper.  Colours are capped at kMaxColors per set; a row that finds all
// of them taken joins the set's overflow class (colour kMaxColors), which the
// smoother updates Jacobi-style.
constexpr int kMaxColors = 32;
// 20M network: 10 iterations at caps 1..8; cap 1 measured fastest (mixed
// 97.2 ms against 99.8 at cap 2 and 104.2 at cap 4; FP64 121.6 / 125.0 /
// 130.5 ms)
constexpr int kCoarseColors = 1;
constexpr double kCapAvgRow = 8.0;  // levels with more entries per row than this are capped
constexpr int kCappedRounds = 8;    // colouring rounds on capped levels
constexpr int kColorLong = 256;     // rows longer than this are coloured by a warp
constexpr int kColorHuge = 4096;    // ... and longer than this by a block
constexpr int kSmallLevel = 2048;  // levels up to this size (without hub rows) sweep in one block
// levels with at most this many entries take no split first sweep
constexpr long long kSmallLevelNnz = 65536;

__global__ void k_color_round(const int* __restrict__ ia, const int* __restrict__ ja,
                              const int* __restrict__ set, int n, const int* __restrict__ color,
                              int* __restrict__ newc, int* counter, int cap, int long_len) {
  int local = 0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    newc[i] = -1;
    if (color[i] >= 0) continue;
    if (ia[i + 1] - ia[i] > long_len) continue;  // k_color_round_long
    // priority: row length first (dense rows decide early), hash second
    const unsigned long long pi =
        ((unsigned long long)(ia[i + 1] - ia[i]) << 32) | color_hash((unsigned)i);
    const int si = set ? set[i] : 0;
    bool is_max = true;
    unsigned used = 0;
    for (int k = ia[i]; k < ia[i + 1]; k++) {
      const int j = ja[k];
      if (j == i) continue;
      if (set && set[j] != si) continue;
      const int cj = color[j];
      if (cj >= 0) {
        if (cj < kMaxColors) used |= 1u << cj;
      } else if ((((unsigned long long)(ia[j + 1] - ia[j]) << 32) | color_hash((unsigned)j)) > pi) {
        is_max = false;
        break;
      }
    }
    if (is_max) {
      const int c = (used == 0xffffffffu) ? kMaxColors : __ffs(~used) - 1;
      newc[i] = c < cap ? c : kMaxColors;
      local++;
    }
  }
  if (local) atomicAdd(counter, local);
}

// The same round for the long rows, one warp per row: the outcome (local
// maximum or not, colours in use) does not depend on the visiting order.
__global__ void k_color_round_long(const int* __restrict__ ia, const int* __restrict__ ja,
                                   const int* __restrict__ set, const int* __restrict__ lrows,
                                   int nl, const int* __restrict__ color, int* __restrict__ newc,
                                   int* counter, int cap) {
  const int lane = threadIdx.x & 31;
  const int warps = (gridDim.x * blockDim.x) >> 5;
  for (int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; w < nl; w += warps) {
    const int i = lrows[w];
    if (color[i] >= 0 || ia[i + 1] - ia[i] > kColorHuge) continue;
    const unsigned long long pi =
        ((unsigned long long)(ia[i + 1] - ia[i]) << 32) | color_hash((unsigned)i);
    const int si = set ? set[i] : 0;
    unsigned used = 0;
    bool blocked = false;
    for (int k0 = ia[i]; k0 < ia[i + 1]; k0 += 32) {
      const int k = k0 + lane;
      if (k < ia[i + 1]) {
        const int j = ja[k];
        if (j != i && !(set && set[j] != si)) {
          const int cj = color[j];
          if (cj >= 0) {
            if (cj < kMaxColors) used |= 1u << cj;
          } else if ((((unsigned long long)(ia[j + 1] - ia[j]) << 32) |
                      color_hash((unsigned)j)) > pi) {
            blocked = true;
          }
        }
      }
      if (__any_sync(0xffffffffu, blocked)) break;
    }
    blocked = __any_sync(0xffffffffu, blocked);
    used = __reduce_or_sync(0xffffffffu, used);
    if (lane == 0 && !blocked) {
      const int c = (used == 0xffffffffu) ? kMaxColors : __ffs(~used) - 1;
      newc[i] = c < cap ? c : kMaxColors;
      atomicAdd(counter, 1);
    }
  }
}

// rows longer than kColorHuge (coarse-level hubs): a block per row, the
// same decision as the warp kernel
__global__ void __launch_bounds__(512)
k_color_round_huge(const int* __restrict__ ia, const int* __restrict__ ja,
                   const int* __restrict__ set, const int* __restrict__ lrows, int nl,
                   const int* __restrict__ color, int* __restrict__ newc, int* counter, int cap) {
  __shared__ unsigned s_used;
  for (int w = blockIdx.x; w < nl; w += gridDim.x) {
    const int i = lrows[w];
    if (color[i] >= 0 || ia[i + 1] - ia[i] <= kColorHuge) continue;  // uniform
    const unsigned long long pi =
        ((unsigned long long)(ia[i + 1] - ia[i]) << 32) | color_hash((unsigned)i);
    const int si = set ? set[i] : 0;
    if (threadIdx.x == 0) s_used = 0;
    __syncthreads();
    unsigned used = 0;
    bool blocked = false;
    for (int k0 = ia[i]; k0 < ia[i + 1]; k0 += blockDim.x) {
      const int k = k0 + threadIdx.x;
      if (k < ia[i + 1]) {
        const int j = ja[k];
        if (j != i && !(set && set[j] != si)) {
          const int cj = color[j];
          if (cj >= 0) {
            if (cj < kMaxColors) used |= 1u << cj;
          } else if ((((unsigned long long)(ia[j + 1] - ia[j]) << 32) |
                      color_hash((unsigned)j)) > pi) {
            blocked = true;
          }
        }
      }
      if (__syncthreads_or(blocked)) {
        blocked = true;
        break;
      }
    }
    if (used) atomicOr(&s_used, used);
    __syncthreads();
    if (threadIdx.x == 0 && !blocked) {
      const unsigned u = s_used;
      const int c = (u == 0xffffffffu) ? kMaxColors : __ffs(~u) - 1;
      newc[i] = c < cap ? c : kMaxColors;
      atomicAdd(counter, 1);
    }
    __syncthreads();
  }
}

__global__ void k_class_counts(const int* __restrict__ key, int n, int* __restrict__ cnt) {
  __shared__ int h[256];
  for (int q = threadIdx.x; q < 256; q += blockDim.x) h[q] = 0;
  __syncthreads();
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
    const int cls = key[t] >> 1;
    atomicAdd(&h[cls], 1);
    if (key[t] & 1) atomicAdd(&h[128 + cls], 1);
  }
  __syncthreads();
  for (int q = threadIdx.x; q < 256; q += blockDim.x)
    if (h[q]) atomicAdd(&cnt[q], h[q]);
}

__global__ void k_long_list(const int* __restrict__ ia, int n, int long_len,
                            int* __restrict__ lrows, int* counter) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    if (ia[i + 1] - ia[i] > long_len) lrows[atomicAdd(counter, 1)] = i;
}

__global__ void k_color_rest(int n, int* __restrict__ color) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    if (color[i] < 0) color[i] = kMaxColors;
}

__global__ void k_color_commit(int n, const int* __restrict__ newc, int* __restrict__ color) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    if (newc[i] >= 0) color[i] = newc[i];
}

// key = ((set * 64 + colour) << 1) | long ; C points are set 0, F points
// set 1; long rows sort to the end of their class
__global__ void k_color_keys(const int* __restrict__ set, const int* __restrict__ color,
                             const int* __restrict__ ia, int n, int* __restrict__ key,
                             int* __restrict__ ids) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    key[i] = (((set ? set[i] : 0) * 64 + color[i]) << 1) | (ia[i + 1] - ia[i] > kLongRow ? 1 : 0);
    ids[i] = i;
  }
}

__global__ void k_cf_set(const int* __restrict__ cf, int n, int* __restrict__ set) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    set[i] = (cf[i] == 1) ? 0 : 1;
}

__global__ void k_l1_diag(const int* __restrict__ ia, const double* __restrict__ a, int n,
                          double* __restrict__ d) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double s = 0.0;
    for (int k = ia[i]; k < ia[i + 1]; k++) s += fabs(a[k]);
    d[i] = s;
  }
}

// diagonal value of each row (the last diagonal entry; 1 if none).  Rows
// longer than kLongRow are left to k_diag_long (a warp per listed row).
__global__ void k_diag(const int* __restrict__ ia, const int* __restrict__ ja,
                       const double* __restrict__ a, int n, double* __restrict__ d) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    if (ia[i + 1] - ia[i] > kLongRow) continue;
    double v = 1.0;
    for (int k = ia[i]; k < ia[i + 1]; k++)
      if (ja[k] == i) v = a[k];
    d[i] = v;
  }
}
__global__ void k_diag_long(const int* __restrict__ ia, const int* __restrict__ ja,
                            const double* __restrict__ a, const int* __restrict__ rows, int m,
                            double* __restrict__ d) {
  const int lane = threadIdx.x & 31;
  const int nw = (gridDim.x * blockDim.x) >> 5;
  for (int q = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; q < m; q += nw) {
    const int i = rows[q];
    int last = -1;
    for (int base = ia[i]; base < ia[i + 1]; base += 32) {
      const int k = base + lane;
      const unsigned hit = __ballot_sync(0xffffffffu, k < ia[i + 1] && ja[k] == i);
      if (hit) last = base + 31 - __clz(hit);
    }
    if (lane == 0) d[i] = last >= 0 ? a[last] : 1.0;
  }
}

// x += w_i * r_i  with w_i = scale / d_i
template <class T>
__global__ void k_scaled_update(T* __restrict__ x, const T* __restrict__ r,
                                const T* __restrict__ d, T scale, int n) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    x[i] += scale * (r[i] / d[i]);
}

template <class T>
__global__ void k_to_f32(const double* __restrict__ a, size_t m, T* __restrict__ b) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < m;
       i += (size_t)gridDim.x * blockDim.x)
    b[i] = (T)a[i];
}

Solver::~Solver() {
  drop_graphs();
  if (h_sc) cudaFreeHost(h_sc);
  if (ev0) cudaEventDestroy(ev0);
  if (ev1) cudaEventDestroy(ev1);
}

void Solver::drop_graphs() {
  for (auto& g : graph)
    if (g) { cudaGraphExecDestroy(g); g = nullptr; }
  for (auto& g : loop)
    if (g) { cudaGraphExecDestroy(g); g = nullptr; }
}

template <class T>
DevMat<T> Solver::mat(const CSR& M, const DBuf<float>* v32, const RowLayout* lay) const {
  DevMat<T> d;
  d.n = M.n; d.m = M.m; d.nnz = M.nnz; d.ia = M.ia.p; d.ja = M.ja.p;
  if constexpr (sizeof(T) == 8) d.val = M.val.p;
  else d.val = v32->p;
  if (lay) {
    d.group = lay->group;
    d.lrows = lay->lrows.p;
    d.nlong = lay->nlong;
    d.tiles = lay->tiles.n ? lay->tiles.p : nullptr;
  }
  return d;
}

template DevMat<double> Solver::mat<double>(const CSR&, const DBuf<float>*,
                                            const RowLayout*) const;
template DevMat<float> Solver::mat<float>(const CSR&, const DBuf<float>*,
                                          const RowLayout*) const;

template <class T>
PackedMat<T> Solver::pmat(const CSR& M, const DBuf<float>& v32, const Packing& pk) const {
  PackedMat<T> d;
  d.ia = M.ia.p;
  d.ja = M.ja.p;
  if constexpr (sizeof(T) == 8) d.val = M.val.p;
  else d.val = v32.p;
  d.pk = &pk;
  return d;
}

static std::vector<int> host_ia(const CSR& M, cudaStream_t s) {
  std::vector<int> h((size_t)M.n + 1);
  M.ia.download(h.data(), (size_t)M.n + 1);
  BN_CUDA(cudaStreamSynchronize(s));
  return h;
}

void Solver::color_level(Level& L, int smoother) {
  const int n = L.A.n;
  const int g = grid_for(n, 256);
  DBuf<int> color(n, s), newc(n, s), set, ctr(1, s);
  color.fill_bytes(0xff);  // -1
  bool cf_split = (smoother == SMOOTHER_CF_GS);
  if (cf_split) {
    set.alloc(n, s);
    BN_LAUNCH(k_cf_set, g, 256, 0, s, L.cf.p, n, set.p);
  }
  // dense coarse operators get fewer colour classes (rows beyond the cap
  // join the Jacobi-updated overflow class): each class costs a sequential
  // step per sweep
  const double avg_row = n > 0 ? (double)L.A.nnz / n : 0.0;
  static const int coarse_cap = getenv("BN_COARSE_COLORS") ? atoi(getenv("BN_COARSE_COLORS"))
                                                            : kCoarseColors;
  static const double cap_avg = getenv("BN_CAP_AVG") ? atof(getenv("BN_CAP_AVG")) : kCapAvgRow;
  const int cap = avg_row > cap_avg ? coarse_cap : kMaxColors;
  // capped levels: rows still uncoloured after kCappedRounds rounds join
  // the overflow class
  static const int capped_rounds =
      getenv("BN_CAP_ROUNDS") ? atoi(getenv("BN_CAP_ROUNDS")) : kCappedRounds;
  // long rows (order of the list is irrelevant: each row's outcome is)
  DBuf<int> lrows(n > 0 ? n : 1, s), lctr(1, s);
  lctr.zero();
  if (n > 0) BN_LAUNCH(k_long_list, g, 256, 0, s, L.A.ia.p, n, kColorLong, lrows.p, lctr.p);
  const int nlong_rows = read_scalar(lctr.p, s);
  int done = 0, round = 0;
  while (done < n) {
    BN_REQUIRE(round <= n, BN_ERR_ARG, "colouring did not finish");
    if (cap < kMaxColors && round >= capped_rounds) {
      BN_LAUNCH(k_color_rest, g, 256, 0, s, n, color.p);
      break;
    }
    ctr.zero();
    BN_LAUNCH(k_color_round, g, 256, 0, s, L.A.ia.p, L.A.ja.p, cf_split ? set.p : nullptr, n,
              color.p, newc.p, ctr.p, cap, kColorLong);
    if (nlong_rows > 0) {
      BN_LAUNCH(k_color_round_long, grid_for((long long)nlong_rows * 32, 256), 256, 0, s,
                L.A.ia.p, L.A.ja.p, cf_split ? set.p : nullptr, lrows.p, nlong_rows, color.p,
                newc.p, ctr.p, cap);
      BN_LAUNCH(k_color_round_huge, nlong_rows < 1024 ? nlong_rows : 1024, 512, 0, s, L.A.ia.p,
                L.A.ja.p, cf_split ? set.p : nullptr, lrows.p, nlong_rows, color.p, newc.p,
                ctr.p, cap);
    }
    BN_LAUNCH(k_color_commit, g, 256, 0, s, n, newc.p, color.p);
    // capped levels run their rounds without asking how many rows are left
    // (a round with nothing left to colour changes nothing)
    if (cap >= kMaxColors) done += read_scalar(ctr.p, s);
    round++;
  }
  DBuf<int> key(n, s), ids(n, s), key_out(n, s);
  L.gs_rows.alloc(n, s);
  BN_LAUNCH(k_color_keys, g, 256, 0, s, cf_split ? set.p : nullptr, color.p, L.A.ia.p, n, key.p,
            ids.p);
  size_t tmp = 0;
  BN_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tmp, key.p, key_out.p, ids.p, L.gs_rows.p, n,
                                          0, 8, s));
  DBuf<unsigned char> t(tmp, s);
  BN_CUDA(cub::DeviceRadixSort::SortPairs(t.p, tmp, key.p, key_out.p, ids.p, L.gs_rows.p, n, 0, 8,
                                          s));
  // class sizes and long-row counts per class id (key >> 1 < 128); the
  // sorted rows hold the classes in ascending id order
  DBuf<int> ccnt(256, s);
  ccnt.zero();
  if (n > 0) BN_LAUNCH(k_class_counts, g, 256, 0, s, key_out.p, n, ccnt.p);
  std::vector<int> hc(256);
  ccnt.download(hc.data(), 256);
  BN_CUDA(cudaStreamSynchronize(s));
  L.cptr.clear();
  L.cjac.clear();
  L.clong.clear();
  L.cptr.push_back(0);
  for (int cls = 0; cls < 128; cls++) {
    if (hc[cls] == 0) continue;
    L.cptr.push_back(L.cptr.back() + hc[cls]);
    L.cjac.push_back((cls & 63) == kMaxColors ? 1 : 0);
    L.clong.push_back(hc[128 + cls]);
  }
  L.colored_for = smoother;
  L.color_rounds = round;
  if (trace_on()) {
    int ov = 0;
    for (size_t c = 0; c + 1 < L.cptr.size(); c++)
      if (L.cjac[c]) ov += L.cptr[c + 1] - L.cptr[c];
    fprintf(stderr, "[bn]     colouring n=%d classes=%d overflow_rows=%d rounds=%d cap=%d\n", n,
            (int)L.cptr.size() - 1, ov, round, cap);
  }
  {
    const int nc = (int)L.cptr.size() - 1;
    std::vector<int> jac(nc);
    for (int c = 0; c < nc; c++) jac[c] = L.cjac[c];
    L.d_cptr.alloc(nc + 1, s);
    L.d_cptr.upload(L.cptr.data(), nc + 1);
    L.d_cjac.alloc(nc > 0 ? nc : 1, s);
    if (nc) L.d_cjac.upload(jac.data(), nc);
    BN_CUDA(cudaStreamSynchronize(s));
  }
  const double avg = n > 0 ? (double)L.A.nnz / n : 0.0;
  L.gs_group = avg <= 12.0 ? 1 : (avg <= 48.0 ? 8 : 32);
  // BN_GS_LANES=g pins the Gauss-Seidel kernel (0 staged row tiles, 1/2/4/8/
  // 16/32 lanes per row); the autotuner may still change it
  static const int gs_forced = getenv("BN_GS_LANES") ? atoi(getenv("BN_GS_LANES")) : -1;
  if (gs_forced == 0 || gs_forced == 1 || gs_forced == 2 || gs_forced == 4 || gs_forced == 8 ||
      gs_forced == 16 || gs_forced == 32)
    L.gs_group = gs_forced;
}

// B = rows perm[new] of A with columns renumbered by cinv (null: unchanged)
__global__ void k_perm_count(const int* __restrict__ ia, const int* __restrict__ perm, int n,
                             int* __restrict__ cnt) {
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
    const int o = perm ? perm[r] : r;
    cnt[r] = ia[o + 1] - ia[o];
  }
}
__global__ void k_perm_fill(const int* __restrict__ ia, const int* __restrict__ ja,
                            const double* __restrict__ val, const int* __restrict__ perm,
                            const int* __restrict__ cinv, int n, const int* __restrict__ bia,
                            int* __restrict__ bja, double* __restrict__ bval) {
  const int lane = threadIdx.x & 31;
  const int warps = (gridDim.x * blockDim.x) >> 5;
  for (int r = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; r < n; r += warps) {
    const int o = perm ? perm[r] : r;
    const int k0 = ia[o], len = ia[o + 1] - k0, q0 = bia[r];
    for (int q = lane; q < len; q += 32) {
      const int c = ja[k0 + q];
      bja[q0 + q] = cinv ? cinv[c] : c;
      bval[q0 + q] = val[k0 + q];
    }
  }
}
__global__ void k_inverse_perm(const int* __restrict__ perm, int n, int* __restrict__ inv) {
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x)
    inv[perm[r]] = r;
}
__global__ void k_iota_perm(int* __restrict__ a, int n) {
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) a[r] = r;
}

// ---- split of Ap by colour class (Level::AL / Level::AU)
__global__ void k_row_class_start(const int* __restrict__ cptr, int ncls, int n,
                                  int* __restrict__ cs) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    int lo = 0, hi = ncls - 1;  // last class starting at or before row i
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (cptr[mid] <= i) lo = mid;
      else hi = mid - 1;
    }
    cs[i] = cptr[lo];
  }
}
// Rows longer than kLongRow (the hub rows, listed in the layout's lrows) are
// left to the block-per-row kernels below.
__global__ void k_split_count(const int* __restrict__ ia, const int* __restrict__ ja,
                              const int* __restrict__ cs, int n, int* __restrict__ cl,
                              int* __restrict__ cu) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    if (ia[i + 1] - ia[i] > kLongRow) continue;
    int nlow = 0, nall = 0;
    for (int k = ia[i]; k < ia[i + 1]; k++) {
      const int j = ja[k];
      nlow += (j < cs[i] || j == i);
      nall++;
    }
    cl[i] = nlow;
    cu[i] = nall - nlow;
  }
}
__global__ void k_split_fill(const int* __restrict__ ia, const int* __restrict__ ja,
                             const double* __restrict__ a, const int* __restrict__ cs, int n,
                             const int* __restrict__ lia, int* __restrict__ lja,
                             double* __restrict__ la, const int* __restrict__ uia,
                             int* __restrict__ uja, double* __restrict__ ua) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    if (ia[i + 1] - ia[i] > kLongRow) continue;
    int pl = lia[i], pu = uia[i];
    for (int k = ia[i]; k < ia[i + 1]; k++) {
      const int j = ja[k];
      if (j < cs[i] || j == i) {
        lja[pl] = j;
        la[pl++] = a[k];
      } else {
        uja[pu] = j;
        ua[pu++] = -a[k];
      }
    }
  }
}

// A block per long row: counts, then the entries in chunks of blockDim.x,
// each chunk's AL entries placed by a block-wide prefix of the split flags
// (so both parts keep the row's order).
__global__ void __launch_bounds__(256)
k_split_count_long(const int* __restrict__ ia, const int* __restrict__ ja,
                   const int* __restrict__ cs, const int* __restrict__ lrows,
                   int* __restrict__ cl, int* __restrict__ cu) {
  __shared__ int red[8];
  const int i = lrows[blockIdx.x];
  const int c = cs[i];
  int nlow = 0;
  for (int k = ia[i] + threadIdx.x; k < ia[i + 1]; k += blockDim.x) {
    const int j = ja[k];
    nlow += (j < c || j == i);
  }
  for (int off = 16; off > 0; off >>= 1) nlow += __shfl_xor_sync(0xffffffffu, nlow, off);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = nlow;
  __syncthreads();
  if (threadIdx.x == 0) {
    int t = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) t += red[w];
    cl[i] = t;
    cu[i] = (ia[i + 1] - ia[i]) - t;
  }
}

__global__ void __launch_bounds__(256)
k_split_fill_long(const int* __restrict__ ia, const int* __restrict__ ja,
                  const double* __restrict__ a, const int* __restrict__ cs,
                  const int* __restrict__ lrows, const int* __restrict__ lia,
                  int* __restrict__ lja, double* __restrict__ la, const int* __restrict__ uia,
                  int* __restrict__ uja, double* __restrict__ ua) {
  __shared__ int wsum[8];
  const int i = lrows[blockIdx.x];
  const int c = cs[i];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  int pl = lia[i], pu = uia[i];
  for (int k0 = ia[i]; k0 < ia[i + 1]; k0 += blockDim.x) {
    const int k = k0 + threadIdx.x;
    const bool in = k < ia[i + 1];
    const int j = in ? ja[k] : 0;
    const bool low = in && (j < c || j == i);
    const unsigned bal = __ballot_sync(0xffffffffu, low);
    if (lane == 0) wsum[w] = __popc(bal);
    __syncthreads();
    int before = 0, total = 0;
    for (int q = 0; q < nw; q++) {
      before += q < w ? wsum[q] : 0;
      total += wsum[q];
    }
    const int rank = before + __popc(bal & ((1u << lane) - 1u));  // AL entries before k
    if (in) {
      if (low) {
        lja[pl + rank] = j;
        la[pl + rank] = a[k];
      } else {
        const int r = (k - k0) - rank;
        uja[pu + r] = j;
        ua[pu + r] = -a[k];
      }
    }
    const int chunk = (ia[i + 1] - k0) < (int)blockDim.x ? ia[i + 1] - k0 : (int)blockDim.x;
    pl += total;
    pu += chunk - total;
    __syncthreads();
  }
}

// AL / AU of a coloured level (entries keep their order within each part)
void Solver::build_split(Level& L) {
  const CSR& A = L.Ap;
  const int n = A.n;
  const int ncls = (int)L.cptr.size() - 1;
  const int g = grid_for(n, 256);
  DBuf<int> cs(n, s), cl((size_t)n + 1, s), cu((size_t)n + 1, s);
  cl.zero();
  cu.zero();
  BN_LAUNCH(k_row_class_start, g, 256, 0, s, L.d_cptr.p, ncls, n, cs.p);
  BN_LAUNCH(k_split_count, g, 256, 0, s, A.ia.p, A.ja.p, cs.p, n, cl.p, cu.p);
  const int nlong = L.layA.nlong;  // rows of Ap longer than kLongRow
  if (nlong > 0)
    BN_LAUNCH(k_split_count_long, nlong, 256, 0, s, A.ia.p, A.ja.p, cs.p, L.layA.lrows.p, cl.p,
              cu.p);
  const int nl = scan_counts(cl.p, n, s);
  const int nu = scan_counts(cu.p, n, s);
  L.AL.n = L.AU.n = n;
  L.AL.m = L.AU.m = A.m;
  L.AL.nnz = nl;
  L.AU.nnz = nu;
  L.AL.ia = std::move(cl);
  L.AU.ia = std::move(cu);
  L.AL.ja.alloc(nl > 0 ? nl : 1, s);
  L.AL.val.alloc(nl > 0 ? nl : 1, s);
  L.AU.ja.alloc(nu > 0 ? nu : 1, s);
  L.AU.val.alloc(nu > 0 ? nu : 1, s);
  BN_LAUNCH(k_split_fill, g, 256, 0, s, A.ia.p, A.ja.p, A.val.p, cs.p, n, L.AL.ia.p, L.AL.ja.p,
            L.AL.val.p, L.AU.ia.p, L.AU.ja.p, L.AU.val.p);
  if (nlong > 0)
    BN_LAUNCH(k_split_fill_long, nlong, 256, 0, s, A.ia.p, A.ja.p, A.val.p, cs.p,
              L.layA.lrows.p, L.AL.ia.p, L.AL.ja.p, L.AL.val.p, L.AU.ia.p, L.AU.ja.p, L.AU.val.p);
  analyze_rows(L.AL, L.layAL, s);
  analyze_rows(L.AU, L.layAU, s);
  order_tiles(n, L.perm.p, L.layAL, s);
  order_tiles(n, L.perm.p, L.layAU, s);
  L.split = true;
}

void permute_csr(const CSR& A, const int* perm, const int* cinv, CSR& B, cudaStream_t s) {
  const int n = A.n;
  DBuf<int> cnt((size_t)n + 1, s);
  cnt.zero();
  if (n > 0) BN_LAUNCH(k_perm_count, grid_for(n, 256), 256, 0, s, A.ia.p, perm, n, cnt.p);
  const int nnz = scan_counts(cnt.p, n, s);
  B.n = n;
  B.m = A.m;
  B.nnz = nnz;
  B.ia = std::move(cnt);
  B.ja.alloc((size_t)(nnz > 0 ? nnz : 1), s);
  B.val.alloc((size_t)(nnz > 0 ? nnz : 1), s);
  if (n > 0)
    BN_LAUNCH(k_perm_fill, grid_for((long long)n * 32, 256), 256, 0, s, A.ia.p, A.ja.p, A.val.p,
              perm, cinv, n, B.ia.p, B.ja.p, B.val.p);
}

// Colour-ordered renumbering of every level for the solve phase.
void Solver::build_solve_layout() {
  Phase ph("solve layout", s);
  const int nl = (int)lv.size();
  auto coloured_level = [&](int l) {
    return l < nl - 1 && lv[l]->gs_rows.n > 0 &&
           (opt.smoother == SMOOTHER_CF_GS || opt.smoother == SMOOTHER_GS);
  };
  for (int l = 0; l < nl; l++) {
    Level& L = *lv[l];
    const int n = L.A.n;
    L.perm.alloc(n > 0 ? n : 1, s);
    L.inv.alloc(n > 0 ? n : 1, s);
    const bool coloured = coloured_level(l);
    if (n == 0) continue;
    if (coloured)
      BN_CUDA(cudaMemcpyAsync(L.perm.p, L.gs_rows.p, sizeof(int) * n, cudaMemcpyDeviceToDevice,
                              s));
    else
      BN_LAUNCH(k_iota_perm, grid_for(n, 256), 256, 0, s, L.perm.p, n);
    BN_LAUNCH(k_inverse_perm, grid_for(n, 256), 256, 0, s, L.perm.p, n, L.inv.p);
  }
  for (int l = 0; l < nl; l++) {
    Level& L = *lv[l];
    {
      Phase p1("layout permute A", s, l);
      permute_csr(L.A, L.perm.p, L.inv.p, L.Ap, s);
    }
    {
      Phase p2("layout rows+tiles A", s, l);
      analyze_rows(L.Ap, L.layA, s);
      // row tiles in original row order: classes interleave, x gathers stay local
      if (coloured_level(l)) order_tiles(L.Ap.n, L.perm.p, L.layA, s);
    }
    if (l < nl - 1) {
      Level& C = *lv[l + 1];
      Phase p3("layout P, R", s, l);
      permute_csr(L.P, L.perm.p, C.inv.p, L.Pp, s);
      permute_csr(L.R, C.perm.p, L.inv.p, L.Rp, s);
      analyze_rows(L.Pp, L.layP, s);
      analyze_rows(L.Rp, L.layR, s);
      if (coloured_level(l)) order_tiles(L.Pp.n, L.perm.p, L.layP, s);
      if (coloured_level(l + 1)) order_tiles(L.Rp.n, C.perm.p, L.layR, s);
      p3.done();
      if (opt.smoother == SMOOTHER_L1) {
        L.l1.alloc(L.A.n, s);
        BN_LAUNCH(k_l1_diag, grid_for(L.A.n, 256), 256, 0, s, L.Ap.ia.p, L.Ap.val.p, L.A.n,
                  L.l1.p);
      }
      if (use_packed) {  // packings only for the operators that run on them
        Phase ph2("packing", s, l);
        L.use_pkA = L.layA.nlong > 0;
        L.use_pkP = L.layP.nlong > 0;
        L.use_pkR = L.layR.nlong > 0;
        if (L.use_pkA) {
          std::vector<int> ha = host_ia(L.Ap, s);
          L.pkA.build(ha, {make_int2(0, L.Ap.n)}, s);
          if (coloured_level(l)) {
            std::vector<int2> rg;
            for (size_t c = 0; c + 1 < L.cptr.size(); c++)
              rg.push_back(make_int2(L.cptr[c], L.cptr[c + 1]));
            L.pkG.build(ha, rg, s);
          }
        }
        if (L.use_pkP) L.pkP.build(host_ia(L.Pp, s), {make_int2(0, L.Pp.n)}, s);
        if (L.use_pkR) L.pkR.build(host_ia(L.Rp, s), {make_int2(0, L.Rp.n)}, s);
        if (trace_on())
          fprintf(stderr, "[bn] L%d packed kernels: A %d (%d long rows)  P %d  R %d (%d long rows)\n",
                  l, (int)L.use_pkA, L.layA.nlong, (int)L.use_pkP, (int)L.use_pkR, L.layR.nlong);
      }
      L.split = false;
      L.AL = CSR();
      L.AU = CSR();
      if (coloured_level(l) && L.A.n > kSmallLevel && L.A.nnz > kSmallLevelNnz &&
          ((use_packed && L.use_pkA) || L.layA.nlong == 0)) {
        Phase ph3("split by class", s, l);
        build_split(L);
        if (use_packed && L.use_pkA) {  // hub rows: the split runs on packed kernels too
          std::vector<int> hl = host_ia(L.AL, s);
          std::vector<int2> rg;
          for (size_t c = 0; c + 1 < L.cptr.size(); c++)
            rg.push_back(make_int2(L.cptr[c], L.cptr[c + 1]));
          L.pkAL.build(hl, rg, s);
          L.pkAU.build(host_ia(L.AU, s), {make_int2(0, L.AU.n)}, s);
        }
      }
      if (opt.smoother == SMOOTHER_JACOBI || coloured_level(l)) {
        L.dg.alloc(L.A.n, s);
        BN_LAUNCH(k_diag, grid_for(L.A.n, 256), 256, 0, s, L.Ap.ia.p, L.Ap.ja.p, L.Ap.val.p,
                  L.A.n, L.dg.p);
        if (L.layA.nlong > 0)
          BN_LAUNCH(k_diag_long, grid_for((long long)L.layA.nlong * 32, 256), 256, 0, s,
                    L.Ap.ia.p, L.Ap.ja.p, L.Ap.val.p, L.layA.lrows.p, L.layA.nlong, L.dg.p);
      }
    }
  }
  if (own_solve) {
    permute_csr(Aown, lv[0]->perm.p, lv[0]->inv.p, Aownp, s);
    analyze_rows(Aownp, layOwn, s);
    if (coloured_level(0)) order_tiles(Aownp.n, lv[0]->perm.p, layOwn, s);
  }
  ic.remap(lv[0]->inv.p, s);
  f32_ready = false;
}

void Solver::alloc_vectors() {
  drop_graphs();  // the graphs hold the vectors' addresses
  const int nl = (int)lv.size();
  for (int l = 0; l < nl; l++) {
    Level& L = *lv[l];
    int n = L.A.n;
    if (l > 0) { L.b.alloc(n, s); L.x.alloc(n, s); }
    if (l < nl - 1) L.r.alloc(n, s);
    if (opt.precision == AMG_PREC_MIXED) {
      if (l > 0) { L.b32.alloc(n, s); L.x32.alloc(n, s); }
      if (l < nl - 1) L.r32.alloc(n, s);
    }
  }
  const int n0 = n();
  for (auto* v : {&u1, &r1, &icy, &icx, &xx, &r2, &corr}) v->alloc(n0, s);
  for (auto* v : {&b, &x, &r, &z, &p, &ap}) v->alloc(n0, s);
  if (opt.precision == AMG_PREC_MIXED)
    for (auto* v : {&g32, &u1f, &r1f, &icyf, &icxf, &xxf, &r2f, &corrf}) v->alloc(n0, s);
  sc.alloc(SC_COUNT, s);
  sc.zero();
  ctl.alloc(4, s);
  ctl.zero();
  const int np = spmv_partials(n0, lay_solve().nlong);
  part0.alloc(kRedBlocks > np ? kRedBlocks : np, s);
  part1.alloc(kRedBlocks, s);
  if (!h_sc) BN_CUDA(cudaMallocHost((void**)&h_sc, sizeof(double) * SC_COUNT));
}

void Solver::prepare_f32() {
  const int nl = (int)lv.size();
  for (int l = 0; l < nl; l++) {
    Level& L = *lv[l];
    L.A32.alloc(L.Ap.nnz > 0 ? L.Ap.nnz : 1, s);
    BN_LAUNCH(k_to_f32<float>, grid_for(L.Ap.nnz, 256), 256, 0, s, L.Ap.val.p, (size_t)L.Ap.nnz,
              L.A32.p);
    if (L.split) {
      L.AL32.alloc(L.AL.nnz > 0 ? L.AL.nnz : 1, s);
      L.AU32.alloc(L.AU.nnz > 0 ? L.AU.nnz : 1, s);
      BN_LAUNCH(k_to_f32<float>, grid_for(L.AL.nnz, 256), 256, 0, s, L.AL.val.p,
                (size_t)L.AL.nnz, L.AL32.p);
      BN_LAUNCH(k_to_f32<float>, grid_for(L.AU.nnz, 256), 256, 0, s, L.AU.val.p,
                (size_t)L.AU.nnz, L.AU32.p);
    }
    if (l < nl - 1) {
      L.P32.alloc(L.Pp.nnz > 0 ? L.Pp.nnz : 1, s);
      L.R32.alloc(L.Rp.nnz > 0 ? L.Rp.nnz : 1, s);
      BN_LAUNCH(k_to_f32<float>, grid_for(L.Pp.nnz, 256), 256, 0, s, L.Pp.val.p,
                (size_t)L.Pp.nnz, L.P32.p);
      BN_LAUNCH(k_to_f32<float>, grid_for(L.Rp.nnz, 256), 256, 0, s, L.Rp.val.p,
                (size_t)L.Rp.nnz, L.R32.p);
      if (L.l1.n) {
        L.l1_32.alloc(L.l1.n, s);
        BN_LAUNCH(k_to_f32<float>, grid_for(L.l1.n, 256), 256, 0, s, L.l1.p, L.l1.n, L.l1_32.p);
      }
      if (L.dg.n) {
        L.dg32.alloc(L.dg.n, s);
        BN_LAUNCH(k_to_f32<float>, grid_for(L.dg.n, 256), 256, 0, s, L.dg.p, L.dg.n, L.dg32.p);
      }
    }
  }
  if (own_solve) {
    Aown32.alloc(Aownp.nnz > 0 ? Aownp.nnz : 1, s);
    BN_LAUNCH(k_to_f32<float>, grid_for(Aownp.nnz, 256), 256, 0, s, Aownp.val.p,
              (size_t)Aownp.nnz, Aown32.p);
  }
  f32_ready = true;
}

void Solver::finish_setup() {
  const int nl = (int)lv.size();
  { Phase ph("dense coarse", s, nl - 1); coarse.setup(lv[nl - 1]->A, s); }
  for (int l = 0; l < nl - 1; l++) {
    Level& L = *lv[l];
    const int sm = opt.smoother;
    if ((sm == SMOOTHER_CF_GS || sm == SMOOTHER_GS) && L.colored_for != sm) {
      Phase ph("colouring", s, l);
      color_level(L, sm);
    }
  }
  ic.want_f32 = (opt.precision == AMG_PREC_MIXED);
  { Phase ph("ichol factor", s); ic.factor(Asolve(), s); }
  build_solve_layout();
  if (opt.precision == AMG_PREC_MIXED) { Phase ph("fp32 copies", s); prepare_f32(); }
  { Phase ph("vectors", s); alloc_vectors(); }
  drop_graphs();
}

// Hierarchy loop of amg_build_hierarchy (build_hierarchy.c:59-147).
void Solver::build(CSR&& A0) {
  cudaEventRecord(ev0, s);
  lv.clear();
  lv.emplace_back(new Level());
  lv[0]->A = std::move(A0);
  const int max_levels =
      (opt.max_levels > 0 && opt.max_levels <= AMG_MAX_LEVELS) ? opt.max_levels : AMG_MAX_LEVELS;
  while (lv.back()->A.n >= opt.min_size && (int)lv.size() < max_levels) {
    Level& cur = *lv.back();
    const int nf = cur.A.n;
    const int li = (int)lv.size() - 1;
    { Phase ph("strength", s, li); strength(cur.A, opt.threshold, cur.S, &cur.max_lam, s); }
    cur.cf.alloc(nf, s);
    int nc;
    { Phase ph("coarsen", s, li); nc = coarsen(cur.S, opt.coarsening, cur.max_lam, cur.cf.p, s); }
    cur.n_coarse = nc;
    if (nc == 0 || nc >= nf) break;  // coarsening stalled (:78-83)
    { Phase ph("interpolation", s, li); interpolation(cur.A, cur.S, cur.cf.p, nc, cur.P, s); }
    { Phase ph("transpose P", s, li); transpose(cur.P, cur.R, s, true); }
    CSR Ac, Acs;
    { Phase ph("rap", s, li); rap(cur.R, cur.A, cur.P, Ac, s); }
    { Phase ph("symmetrize Ac", s, li); symmetrize(Ac, Acs, s); }
    lv.emplace_back(new Level());
    lv.back()->A = std::move(Acs);
  }
  finish_setup();
  cudaEventRecord(ev1, s);
  BN_CUDA(cudaEventSynchronize(ev1));
  float ms = 0;
  cudaEventElapsedTime(&ms, ev0, ev1);
  stats.setup_seconds = ms * 1e-3;
}

// amg_rebuild_values (build_hierarchy.c:170-242): same S, C/F and P pattern,
// new A; recompute P values, RAP and symmetrisation level by level.
void Solver::rebuild_values(CSR&& A0) {
  cudaEventRecord(ev0, s);
  lv[0]->A = std::move(A0);
  const int nl = (int)lv.size();
  for (int k = 0; k < nl - 1; k++) {
    Level& cur = *lv[k];
    interpolation_values(cur.A, cur.S, cur.cf.p, cur.P, s);
    transpose(cur.P, cur.R, s, true);
    CSR Ac, Acs;
    rap(cur.R, cur.A, cur.P, Ac, s);
    symmetrize(Ac, Acs, s);
    Level& nxt = *lv[k + 1];
    nxt.A = std::move(Acs);
  }
  own_solve = false;
  Aown = CSR();
  finish_setup();
  cudaEventRecord(ev1, s);
  BN_CUDA(cudaEventSynchronize(ev1));
  float ms = 0;
  cudaEventElapsedTime(&ms, ev0, ev1);
  stats.setup_seconds = ms * 1e-3;
}

// ------------------------------------------------------------ V-cycle
template <class T>
void Solver::smooth(int l, const T* bb, T* xl, bool forward) {
  Level& L = *lv[l];
  const bool f64 = sizeof(T) == 8;
  DevMat<T> A = mat<T>(L.Ap, &L.A32, &L.layA);
  const int n = L.A.n;
  for (int sweep = 0; sweep < opt.nu; sweep++) {
    switch (opt.smoother) {
      case SMOOTHER_CF_GS:
      case SMOOTHER_GS: {
        const int nseg = (int)L.cptr.size() - 1;
        T* tmp = f64 ? (T*)L.r.p : (T*)L.r32.p;
        // small levels sweep in one block, unless they hold hub rows (a warp
        // per row would serialise a class behind them)
        if (n <= kSmallLevel && L.layA.nlong == 0) {
          gs_level_block<T>(A, L.d_cptr.p, L.d_cjac.p, nseg, forward, bb, xl, tmp, s);
          break;
        }
        if (use_packed && L.use_pkA && L.pkG.ranges() == nseg) {
          const T* d = f64 ? (const T*)L.dg.p : (const T*)L.dg32.p;
          PackedMat<T> G = pmat<T>(L.Ap, L.A32, L.pkG);
          for (int q = 0; q < nseg; q++) {
            const int c = forward ? q : nseg - 1 - q;
            const int r0 = L.cptr[c];
            const int nr = L.cptr[c + 1] - r0;
            if (L.cjac[c]) {
              packed_apply<T>(PK_JAC, G, c, xl, bb, tmp, d, r0, s);
              scatter_range<T>(tmp, r0, nr, xl, s);
            } else {
              packed_apply<T>(PK_GS, G, c, xl, bb, xl, d, r0, s);
            }
          }
          break;
        }
        const T* dgl = f64 ? (const T*)L.dg.p : (const T*)L.dg32.p;
        for (int q = 0; q < nseg; q++) {
          int c = forward ? q : nseg - 1 - q;
          const int r0 = L.cptr[c];  // classes are contiguous in the solve numbering
          const int nr = L.cptr[c + 1] - r0;
          if (L.cjac[c])
            jacobi_class<T>(A, nullptr, r0, nr, bb, xl, tmp, L.gs_group, s, L.clong[c], dgl);
          else
            gs_color<T>(A, nullptr, r0, nr, bb, xl, L.gs_group, s, L.clong[c], dgl);
        }
        break;
      }
      case SMOOTHER_JACOBI: {
        T* rr = f64 ? (T*)L.r.p : (T*)L.r32.p;
        const T* d = f64 ? (const T*)L.dg.p : (const T*)L.dg32.p;
        spmv<T>(SPMV_RES, A, xl, bb, rr, s);
        BN_LAUNCH(k_scaled_update<T>, grid_for(n, 256), 256, 0, s, xl, rr, d, (T)opt.omega, n);
        break;
      }
      default: {  // SMOOTHER_L1
        T* rr = f64 ? (T*)L.r.p : (T*)L.r32.p;
        const T* d = f64 ? (const T*)L.l1.p : (const T*)L.l1_32.p;
        spmv<T>(SPMV_RES, A, xl, bb, rr, s);
        BN_LAUNCH(k_scaled_update<T>, grid_for(n, 256), 256, 0, s, xl, rr, d, (T)1, n);
        break;
      }
    }
  }
}

// backslash_rec (amg_cycle.c:180-212); xl is zero on entry
template <class T>
void Solver::backslash(int l, const T* bb, T* xl, bool zero_guess) {
  const int nl = (int)lv.size();
  if (l == nl - 1) {
    coarse.apply<T>(bb, xl, s);
    return;
  }
  Level& L = *lv[l];
  Level& C = *lv[l + 1];
  const bool f64 = sizeof(T) == 8;
  T* rr = f64 ? (T*)L.r.p : (T*)L.r32.p;
  T* cb = f64 ? (T*)C.b.p : (T*)C.b32.p;
  T* cx = f64 ? (T*)C.x.p : (T*)C.x32.p;
  const bool split = zero_guess && L.split && opt.nu == 1 &&
                     (opt.smoother == SMOOTHER_CF_GS || opt.smoother == SMOOTHER_GS);
  if (split) {
    // first sweep from x = 0 on AL (every class, Jacobi classes included,
    // reads only earlier classes: in place), then r = b - A x = AU x
    Phase ph("gs forward (split) + residual", s, l);
    const T* dgl = f64 ? (const T*)L.dg.p : (const T*)L.dg32.p;
    const int nseg = (int)L.cptr.size() - 1;
    if (use_packed && L.use_pkA) {  // levels with hub rows: packed blocks + row segments
      PackedMat<T> AL = pmat<T>(L.AL, L.AL32, L.pkAL);
      for (int c = 0; c < nseg; c++)
        packed_apply<T>(PK_GS, AL, c, xl, bb, xl, dgl, L.cptr[c], s);
      packed_apply<T>(PK_Y, pmat<T>(L.AU, L.AU32, L.pkAU), 0, xl, nullptr, rr, nullptr, 0, s);
    } else {
      DevMat<T> AL = mat<T>(L.AL, &L.AL32, &L.layAL);
      for (int c = 0; c < nseg; c++) {
        const int r0 = L.cptr[c];
        gs_color<T>(AL, nullptr, r0, L.cptr[c + 1] - r0, bb, xl, L.gs_group, s, L.clong[c], dgl);
      }
      spmv<T>(SPMV_Y, mat<T>(L.AU, &L.AU32, &L.layAU), xl, nullptr, rr, s);
    }
  } else {
    { Phase ph("gs forward", s, l); smooth<T>(l, bb, xl, true); }
    Phase ph("residual", s, l);
    if (use_packed && L.use_pkA)
      packed_apply<T>(PK_RES, pmat<T>(L.Ap, L.A32, L.pkA), 0, xl, bb, rr, nullptr, 0, s);
    else
      spmv<T>(SPMV_RES, mat<T>(L.Ap, &L.A32, &L.layA), xl, bb, rr, s);
  }
  {
    Phase ph("restrict", s, l);
    if (use_packed && L.use_pkR)
      packed_apply<T>(PK_Y, pmat<T>(L.Rp, L.R32, L.pkR), 0, rr, nullptr, cb, nullptr, 0, s);
    else
      spmv<T>(SPMV_Y, mat<T>(L.Rp, &L.R32, &L.layR), rr, nullptr, cb, s);
  }
  if (l + 1 < nl - 1) vzero<T>(cx, C.A.n, s);
  backslash<T>(l + 1, cb, cx, true);
  if (use_packed && L.use_pkP)  // x += P ec
    packed_apply<T>(PK_ADD, pmat<T>(L.Pp, L.P32, L.pkP), 0, cx, nullptr, xl, nullptr, 0, s);
  else
    spmv<T>(SPMV_ADD, mat<T>(L.Pp, &L.P32, &L.layP), cx, nullptr, xl, s);
}

// fwdslash_rec (amg_cycle.c:222-253); xl is zero on entry, so the first
// residual is b itself and the prolongation overwrites xl
template <class T>
void Solver::fwdslash(int l, const T* bb, T* xl) {
  const int nl = (int)lv.size();
  if (l == nl - 1) {
    coarse.apply<T>(bb, xl, s);
    return;
  }
  Level& L = *lv[l];
  Level& C = *lv[l + 1];
  const bool f64 = sizeof(T) == 8;
  T* cb = f64 ? (T*)C.b.p : (T*)C.b32.p;
  T* cx = f64 ? (T*)C.x.p : (T*)C.x32.p;
  if (use_packed && L.use_pkR)  // rc = P^T b
    packed_apply<T>(PK_Y, pmat<T>(L.Rp, L.R32, L.pkR), 0, bb, nullptr, cb, nullptr, 0, s);
  else
    spmv<T>(SPMV_Y, mat<T>(L.Rp, &L.R32, &L.layR), bb, nullptr, cb, s);
  fwdslash<T>(l + 1, cb, cx);
  if (use_packed && L.use_pkP)  // x = P ec
    packed_apply<T>(PK_Y, pmat<T>(L.Pp, L.P32, L.pkP), 0, cx, nullptr, xl, nullptr, 0, s);
  else
    spmv<T>(SPMV_Y, mat<T>(L.Pp, &L.P32, &L.layP), cx, nullptr, xl, s);
  smooth<T>(l, bb, xl, false);
}

// amg_ichol_apply (amg_ichol_precond.c:22-48):
//   u1 = backslash(g); x = u1 + IC^{-1}(g - A u1); x += fwdslash(g - A x)
template <class T>
void Solver::precond_t(const T* g, T* out) {
  const bool f64 = sizeof(T) == 8;
  const int n0 = n();
  T* U1 = f64 ? (T*)u1.p : (T*)u1f.p;
  T* R1 = f64 ? (T*)r1.p : (T*)r1f.p;
  T* IY = f64 ? (T*)icy.p : (T*)icyf.p;
  T* IX = f64 ? (T*)icx.p : (T*)icxf.p;
  T* XX = f64 ? (T*)xx.p : (T*)xxf.p;
  T* R2 = f64 ? (T*)r2.p : (T*)r2f.p;
  T* CO = f64 ? (T*)corr.p : (T*)corrf.p;
  DevMat<T> As = own_solve ? mat<T>(Aownp, &Aown32, &layOwn) : mat<T>(lv[0]->Ap, &lv[0]->A32, &lv[0]->layA);
  vzero<T>(U1, n0, s);
  { Phase ph("backslash", s); backslash<T>(0, g, U1, true); }
  const bool fine_packed = use_packed && !own_solve && lv[0]->use_pkA && lv[0]->pkA.ranges() == 1;
  PackedMat<T> Ap0 = pmat<T>(lv[0]->Ap, lv[0]->A32, lv[0]->pkA);
  if (fine_packed) {
    Phase ph("residual r1", s);
    packed_apply<T>(PK_RES, Ap0, 0, U1, g, R1, nullptr, 0, s);
  } else {
    Phase ph("residual r1", s);
    spmv<T>(SPMV_RES, As, U1, g, R1, s);
  }
  { Phase ph("ichol solve", s); ic.solve<T>(R1, IY, IX, s); }
  vadd<T>(U1, IX, n0, XX, s);
  if (fine_packed) {
    Phase ph("residual r2", s);
    packed_apply<T>(PK_RES, Ap0, 0, XX, g, R2, nullptr, 0, s);
  } else {
    Phase ph("residual r2", s);
    spmv<T>(SPMV_RES, As, XX, g, R2, s);
  }
  { Phase ph("fwdslash", s); fwdslash<T>(0, R2, CO); }
  vadd<T>(XX, CO, n0, out, s);
}

// amg_vcycle_precond (amg_cycle.c:262-284): x = backslash(g); r = g - A x;
// x += fwdslash(r), all on the hierarchy's level-0 operator, FP64
void Solver::vcycle_apply(const double* g, double* out) {
  const int n0 = lv[0]->A.n;
  vzero<double>(u1.p, n0, s);
  backslash<double>(0, g, u1.p, true);
  spmv<double>(SPMV_RES, mat<double>(lv[0]->Ap, nullptr, &lv[0]->layA), u1.p, g, r1.p, s);
  fwdslash<double>(0, r1.p, corr.p);
  vadd<double>(u1.p, corr.p, n0, out, s);
}

// amg_backslash (amg_cycle.c:180-215) at level l; x is the initial guess
void Solver::backslash_at(int l, const double* b, double* x) {
  backslash<double>(l, b, x, false);
}

// amg_fwdslash (amg_cycle.c:222-253) at level l with x as the initial guess:
// r = b - A x, coarse correction from R r, x += P e, post-smoothing
void Solver::fwdslash_at(int l, const double* b, double* x) {
  const int nl = (int)lv.size();
  if (l == nl - 1) {
    coarse.apply<double>(b, x, s);
    return;
  }
  Level& L = *lv[l];
  Level& C = *lv[l + 1];
  spmv<double>(SPMV_RES, mat<double>(L.Ap, nullptr, &L.layA), x, b, L.r.p, s);
  spmv<double>(SPMV_Y, mat<double>(L.Rp, nullptr, &L.layR), L.r.p, nullptr, C.b.p, s);
  fwdslash<double>(l + 1, C.b.p, C.x.p);
  spmv<double>(SPMV_ADD, mat<double>(L.Pp, nullptr, &L.layP), C.x.p, nullptr, x, s);
  smooth<double>(l, b, x, false);
}

// Solve matrix and IC(0) factor as given (amg_ichol_precond's A and L): the
// hierarchy stays; A is used as given (no symmetrisation), L as given.
void Solver::use_matrix_and_factor(CSR* A, CSR&& Lf) {
  if (A) {
    Aown = std::move(*A);
    own_solve = true;
    permute_csr(Aown, lv[0]->perm.p, lv[0]->inv.p, Aownp, s);
    analyze_rows(Aownp, layOwn, s);
  }
  ic.want_f32 = (opt.precision == AMG_PREC_MIXED);
  ic.load(std::move(Lf), s);
  ic.remap(lv[0]->inv.p, s);
  f32_ready = false;
  if (opt.precision == AMG_PREC_MIXED) prepare_f32();
  alloc_vectors();
  drop_graphs();
}

void l1_row_norms(const CSR& A, double* d_out, cudaStream_t s) {
  if (A.n > 0)
    BN_LAUNCH(k_l1_diag, grid_for(A.n, 256), 256, 0, s, A.ia.p, A.val.p, A.n, d_out);
}

// z = M r for the PCG: r -> z (captured once per precision as a CUDA graph)
void Solver::precond(const double* g, double* out) {
  const int mode = opt.precision == AMG_PREC_MIXED ? 1 : 0;
  const bool use_graph = (g == r.p && out == z.p) && !trace_on() && !capture_direct;
  if (use_graph && graph[mode]) {
    BN_CUDA(cudaGraphLaunch(graph[mode], s));
    g_launch_count += graph_kernels[mode];
    return;
  }
  auto body = [&]() {
    if (mode == 1) {
      vconvert<float, double>(g, n(), g32.p, s);
      precond_t<float>(g32.p, r2f.p);  // r2f is free once fwdslash has consumed it
      vconvert<double, float>(r2f.p, n(), out, s);
    } else {
      precond_t<double>(g, out);
    }
  };
  if (!use_graph) {
    body();
    return;
  }
  cudaGraph_t gr;
  BN_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
  unsigned long long before = g_launch_count;
  try {
    body();
  } catch (...) {
    cudaStreamEndCapture(s, &gr);
    if (gr) cudaGraphDestroy(gr);
    throw;
  }
  BN_CUDA(cudaStreamEndCapture(s, &gr));
  graph_kernels[mode] = g_launch_count - before;  // kernels recorded, launched on replay
  g_launch_count = before;
  BN_CUDA(cudaGraphInstantiate(&graph[mode], gr, 0));
  cudaGraphDestroy(gr);
  BN_CUDA(cudaGraphLaunch(graph[mode], s));
  g_launch_count += graph_kernels[mode];
}

// ------------------------------------------------------------ device loops
// Stopping test of one PCG iteration on the device (the host loop's test):
// ctl[0] iterations done, ctl[1] status (0 go on, 1 converged, 2 non-finite,
// 3 maxiter reached), ctl[2] maxiter, ctl[3] 1 = true relative residual
// test, else the reference's B-norm; sc[SC_TOL] the tolerance.
constexpr int SC_TOL = 9;
__global__ void k_pcg_check(const double* __restrict__ sc, int* ctl,
                            cudaGraphConditionalHandle h) {
  const int it = ++ctl[0];
  const double rz_new = sc[SC_RZ];
  const double rnorm = sqrt(sc[SC_RR]);
  double bn = sqrt(sc[SC_BB]);
  if (bn == 0.0) bn = 1.0;
  int st = 0;
  if (!isfinite(rz_new) || !isfinite(rnorm)) {
    st = 2;
  } else {
    const double crit = ctl[3] ? rnorm / bn : sqrt(rz_new / sc[SC_RZ0]);
    if (crit < sc[SC_TOL]) st = 1;
    else if (it >= ctl[2]) st = 3;
  }
  ctl[1] = st;
  cudaGraphSetConditional(h, st == 0 ? 1u : 0u);
}
// segmented loop: go on while a segment iterates and maxiter is not reached
__global__ void k_seg_cond(const int* __restrict__ nactive, int* ctl,
                           cudaGraphConditionalHandle h) {
  const int it = ++ctl[0];
  cudaGraphSetConditional(h, (*nactive > 0 && it < ctl[2]) ? 1u : 0u);
}

// Captures body() (the kernels of one iteration, ending with the kernel that
// sets the loop condition) as the body of a conditional WHILE node; the
// graph runs the body until the condition is cleared.  Returns null where
// the driver does not support it (the caller keeps the host loop).
template <class F>
static cudaGraphExec_t build_loop_graph(cudaStream_t s, F&& body,
                                        unsigned long long* body_kernels) {
  cudaGraph_t g = nullptr;
  if (cudaGraphCreate(&g, 0) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  cudaGraphConditionalHandle h;
  cudaGraphNodeParams cp = {};
  cp.type = cudaGraphNodeTypeConditional;
  cudaGraphNode_t node;
  if (cudaGraphConditionalHandleCreate(&h, g, 1, cudaGraphCondAssignDefault) != cudaSuccess ||
      (cp.conditional.handle = h, cp.conditional.type = cudaGraphCondTypeWhile,
       cp.conditional.size = 1, cudaGraphAddNode(&node, g, nullptr, 0, &cp) != cudaSuccess)) {
    cudaGetLastError();
    cudaGraphDestroy(g);
    return nullptr;
  }
  cudaGraph_t bg = cp.conditional.phGraph_out[0];
  if (cudaStreamBeginCaptureToGraph(s, bg, nullptr, nullptr, 0,
                                    cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
    cudaGetLastError();
    cudaGraphDestroy(g);
    return nullptr;
  }
  const unsigned long long before = g_launch_count;
  try {
    body(h);
  } catch (...) {
    cudaGraph_t dummy;
    cudaStreamEndCapture(s, &dummy);
    cudaGraphDestroy(g);
    g_launch_count = before;
    throw;
  }
  cudaGraph_t out = nullptr;
  const cudaError_t e = cudaStreamEndCapture(s, &out);
  *body_kernels = g_launch_count - before;  // launched once per iteration on replay
  g_launch_count = before;
  cudaGraphExec_t ex = nullptr;
  if (e != cudaSuccess || cudaGraphInstantiate(&ex, g, 0) != cudaSuccess) {
    cudaGetLastError();
    ex = nullptr;
  }
  cudaGraphDestroy(g);
  return ex;
}

// amg_pcg (amg_pcg.c:12-101) on device vectors.  FP64 throughout; the mixed
// form uses the flexible (Polak-Ribiere) beta because its preconditioner is
// not exactly symmetric.
int Solver::pcg(const double* d_b, double* d_x, double tol, int maxiter, int print_level) {
  const int n0 = n();
  const bool flexible = (opt.precision == AMG_PREC_MIXED);
  if (flexible && !f32_ready) prepare_f32();
  DevMat<double> A = mat<double>(Asolve_p(), nullptr, &lay_solve());
  const int* perm0 = lv[0]->perm.p;
  cudaEventRecord(ev0, s);
  vpermute<double>(d_b, perm0, n0, b.p, false, s);  // into the solve numbering
  vpermute<double>(d_x, perm0, n0, x.p, false, s);
  spmv<double>(SPMV_RES, A, x.p, b.p, r.p, s);            // r = b - A x
  dot_partials<double>(b.p, b.p, r.p, n0, part0.p, part1.p, s);
  reduce_partials(part0.p, kRedBlocks, sc.p + SC_BB, s);  // b.b
  reduce_partials(part1.p, kRedBlocks, sc.p + SC_RR, s);  // scratch
  precond(r.p, z.p);                                      // z = M r
  BN_CUDA(cudaMemcpyAsync(p.p, z.p, sizeof(double) * n0, cudaMemcpyDeviceToDevice, s));
  dot_partials<double>(r.p, z.p, r.p, n0, part0.p, part1.p, s);
  reduce_partials(part0.p, kRedBlocks, sc.p + SC_RZ, s);   // r.z
  reduce_partials(part1.p, kRedBlocks, sc.p + SC_RR, s);   // r.r
  BN_CUDA(cudaMemcpyAsync(h_sc, sc.p, sizeof(double) * SC_COUNT, cudaMemcpyDeviceToHost, s));
  BN_CUDA(cudaStreamSynchronize(s));
  ic.check_waits(s);
  double bnorm = sqrt(h_sc[SC_BB]);
  if (bnorm == 0.0) bnorm = 1.0;
  const double rz0 = h_sc[SC_RZ];
  double rnorm = sqrt(h_sc[SC_RR]);
  double bn_rel = 1.0;
  if (print_level >= 1) {
    fprintf(stderr, "  %4s  %8s  %8s  %6s\n", "iter", "||r||_B", "rel", "rho");
    fprintf(stderr, "  %4d  %8.2e  %8.2e\n", 0, sqrt(rz0), 1.0);
  }
  int iter;
  int status = BN_OK;
  const int mode = flexible ? 1 : 0;
  stats.device_loop = 0;
  if (loops_ok && print_level < 1 && !trace_on() && maxiter > 0 && !loop[mode]) {
    loop[mode] = build_loop_graph(s, [&](cudaGraphConditionalHandle h) {
      capture_direct = true;
      int np = spmv<double>(SPMV_Y, A, p.p, nullptr, ap.p, s, p.p, part0.p);
      reduce_partials(part0.p, np, sc.p + SC_PAP, s);
      pcg_update_xr(x.p, r.p, p.p, ap.p, n0, sc.p, part0.p, s);
      reduce_partials(part0.p, kRedBlocks, sc.p + SC_RR, s);
      if (flexible) {
        dot_partials<double>(r.p, z.p, nullptr, n0, part1.p, nullptr, s);
        reduce_partials(part1.p, kRedBlocks, sc.p + SC_RZOLD_NEW, s);
      }
      precond(r.p, z.p);
      dot_partials<double>(r.p, z.p, nullptr, n0, part0.p, nullptr, s);
      reduce_partials(part0.p, kRedBlocks, sc.p + SC_RZNEW, s);
      pcg_scalars(sc.p, flexible ? 1 : 0, s);
      g_launch_count++;
      k_pcg_check<<<1, 1, 0, s>>>(sc.p, ctl.p, h);
      BN_CUDA(cudaGetLastError());
      pcg_update_p(p.p, z.p, n0, sc.p, s);
      capture_direct = false;
    }, &loop_kernels[mode]);
    capture_direct = false;
    if (!loop[mode]) loops_ok = false;
  }
  if (loops_ok && print_level < 1 && !trace_on() && maxiter > 0 && loop[mode]) {
    // all iterations in one graph launch; the host reads the outcome once
    const int hc[4] = {0, 0, maxiter, opt.stop == AMG_STOP_RELRES ? 1 : 0};
    BN_CUDA(cudaMemcpyAsync(ctl.p, hc, sizeof hc, cudaMemcpyHostToDevice, s));
    h_sc[0] = tol;
    BN_CUDA(cudaMemcpyAsync(sc.p + SC_TOL, h_sc, sizeof(double), cudaMemcpyHostToDevice, s));
    BN_CUDA(cudaMemcpyAsync(sc.p + SC_RZ0, sc.p + SC_RZ, sizeof(double),
                            cudaMemcpyDeviceToDevice, s));
    BN_CUDA(cudaGraphLaunch(loop[mode], s));
    int hres[4];
    BN_CUDA(cudaMemcpyAsync(hres, ctl.p, sizeof hres, cudaMemcpyDeviceToHost, s));
    BN_CUDA(cudaMemcpyAsync(h_sc, sc.p, sizeof(double) * SC_COUNT, cudaMemcpyDeviceToHost, s));
    BN_CUDA(cudaStreamSynchronize(s));
    g_launch_count += (unsigned long long)hres[0] * loop_kernels[mode];
    ic.check_waits(s);
    stats.device_loop = 1;
    rnorm = sqrt(h_sc[SC_RR]);
    bn_rel = sqrt(h_sc[SC_RZ] / rz0);
    if (hres[1] == 1) {
      iter = hres[0];
    } else {
      iter = maxiter + 1;
      if (hres[1] == 2) status = BN_ERR_NAN;
    }
  } else
  for (iter = 1; iter <= maxiter; iter++) {
    int np = spmv<double>(SPMV_Y, A, p.p, nullptr, ap.p, s, p.p, part0.p);  // Ap, p.Ap
    reduce_partials(part0.p, np, sc.p + SC_PAP, s);
    pcg_update_xr(x.p, r.p, p.p, ap.p, n0, sc.p, part0.p, s);      // x, r, r.r
    reduce_partials(part0.p, kRedBlocks, sc.p + SC_RR, s);
    if (flexible) {  // r_{k+1}.z_k before z is overwritten
      dot_partials<double>(r.p, z.p, nullptr, n0, part1.p, nullptr, s);
      reduce_partials(part1.p, kRedBlocks, sc.p + SC_RZOLD_NEW, s);
    }
    precond(r.p, z.p);
    dot_partials<double>(r.p, z.p, nullptr, n0, part0.p, nullptr, s);
    reduce_partials(part0.p, kRedBlocks, sc.p + SC_RZNEW, s);
    pcg_scalars(sc.p, flexible ? 1 : 0, s);
    BN_CUDA(cudaMemcpyAsync(h_sc, sc.p, sizeof(double) * SC_COUNT, cudaMemcpyDeviceToHost, s));
    BN_CUDA(cudaStreamSynchronize(s));
    ic.check_waits(s);
    const double rz_new = h_sc[SC_RZ];  // rotated: SC_RZ now holds r_{k+1}.z_{k+1}
    rnorm = sqrt(h_sc[SC_RR]);
    bn_rel = sqrt(rz_new / rz0);
    if (print_level >= 1)
      fprintf(stderr, "  %4d  %8.2e  %8.2e  %6.4f\n", iter, sqrt(rz_new), bn_rel,
              rz_new / h_sc[SC_RZ_PREV]);
    if (!isfinite(rz_new) || !isfinite(rnorm)) {
      status = BN_ERR_NAN;
      iter = maxiter + 1;
      break;
    }
    const double crit = (opt.stop == AMG_STOP_RELRES) ? rnorm / bnorm : bn_rel;
    if (crit < tol) break;
    pcg_update_p(p.p, z.p, n0, sc.p, s);
  }
  // true residual for the stats
  spmv<double>(SPMV_RES, A, x.p, b.p, ap.p, s);
  dot_partials<double>(ap.p, ap.p, nullptr, n0, part0.p, nullptr, s);
  reduce_partials(part0.p, kRedBlocks, sc.p + SC_RR, s);
  vpermute<double>(x.p, perm0, n0, d_x, true, s);   // back to the caller's numbering
  cudaEventRecord(ev1, s);
  BN_CUDA(cudaMemcpyAsync(h_sc, sc.p, sizeof(double) * SC_COUNT, cudaMemcpyDeviceToHost, s));
  BN_CUDA(cudaStreamSynchronize(s));
  float ms = 0;
  cudaEventElapsedTime(&ms, ev0, ev1);
  stats.solve_seconds = ms * 1e-3;
  BN_REQUIRE(take_stage_error() == 0, BN_ERR_SPIN,
             "staged SpMV: a bounded wait for a bulk copy ran out");
  stats.relres = sqrt(h_sc[SC_RR]) / bnorm;
  stats.bnorm_rel = bn_rel;
  if (iter > maxiter) {
    if (status == BN_OK) status = BN_ERR_NOT_CONVERGED;
    fprintf(stderr, "  PCG: no convergence after %d iterations, relres = %.2e\n", maxiter,
            rnorm / bnorm);
    stats.iterations = maxiter;
    stats.converged = 0;
    set_last_error(status, status == BN_ERR_NAN ? "PCG: non-finite value in the iteration"
                                                : "PCG: no convergence");
    return -maxiter;
  }
  stats.iterations = iter;
  stats.converged = 1;
  set_last_error(BN_OK, "");
  return iter;
}

// ------------------------------------------------------------ segmented PCG
namespace {
// every entry of the solve matrix couples two rows of one segment
__global__ void k_seg_blockdiag(const int* __restrict__ ia, const int* __restrict__ ja, int n,
                                const int* __restrict__ seg, int* bad) {
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
    const int k = seg[t];
    for (int e = ia[t]; e < ia[t + 1]; e++)
      if (seg[ja[e]] != k) { atomicExch(bad, 1); break; }
  }
}
// start: a segment iterates unless its r0.z0 is zero (b = A x0 there)
__global__ void k_seg_start(const double* __restrict__ rz, int nseg, int* __restrict__ active,
                            int* __restrict__ iters, int* nactive) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nseg; k += gridDim.x * blockDim.x) {
    const int a = rz[k] != 0.0;
    active[k] = a;
    iters[k] = 0;
    if (a) atomicAdd(nactive, 1);
  }
}
__global__ void k_seg_relres(const double* __restrict__ rr, const double* __restrict__ bb,
                             int nseg, double* __restrict__ out) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nseg; k += gridDim.x * blockDim.x)
    out[k] = sqrt(rr[k]) / (bb[k] > 0.0 ? sqrt(bb[k]) : 1.0);
}
}  // namespace

// Independent systems packed block-diagonally (no entry couples two
// segments), solved together: one SpMV and one preconditioner application a
// step for all of them, while every segment keeps the scalars, stopping test
// and iteration count of its own PCG (Solver::pcg applied to that block
// alone).  The hierarchy of a block-diagonal matrix is block-diagonal (strength,
// coarsening, interpolation and RAP only follow entries), so the
// preconditioner acts on every segment separately; a segment that has met its
// stopping test is frozen (alpha = 0) while the others go on.  Segment dot
// products are one block per segment over its rows in natural order, so the
// result does not depend on how the other segments converge.
int Solver::pcg_segmented(int nseg, const int* d_ptr, const double* d_b, double* d_x,
                          double tol, int maxiter, int* h_iters, double* h_relres) {
  const int n0 = n();
  const bool flexible = (opt.precision == AMG_PREC_MIXED);
  if (flexible && !f32_ready) prepare_f32();
  DevMat<double> A = mat<double>(Asolve_p(), nullptr, &lay_solve());
  const int* perm0 = lv[0]->perm.p;
  const int* inv0 = lv[0]->inv.p;
  DBuf<int> seg(n0, s), ints((size_t)2 * nseg + 2, s);
  int* active = ints.p;
  int* iters = ints.p + nseg;
  int* flag = ints.p + 2 * nseg;  // [0] block-diagonal check, [1] segments iterating
  ints.zero();
  seg_of_rows(perm0, n0, d_ptr, nseg, seg.p, s);
  const CSR& Ap = Asolve_p();
  BN_LAUNCH(k_seg_blockdiag, grid_for(n0, 256), 256, 0, s, Ap.ia.p, Ap.ja.p, n0, seg.p, flag);
  BN_REQUIRE(read_scalar(flag, s) == 0, BN_ERR_ARG,
             "segmented solve: the matrix couples rows of different segments");
  enum { BB, RR, RZ, RZ0, PAP, RZNEW, RZON, ALPHA, BETA, NSC };
  DBuf<double> scal((size_t)NSC * nseg, s);
  auto S_ = [&](int w) { return scal.p + (size_t)w * nseg; };
  cudaEventRecord(ev0, s);
  vpermute<double>(d_b, perm0, n0, b.p, false, s);
  vpermute<double>(d_x, perm0, n0, x.p, false, s);
  spmv<double>(SPMV_RES, A, x.p, b.p, r.p, s);  // r = b - A x
  seg_dot(b.p, b.p, d_ptr, inv0, nseg, S_(BB), s);
  precond(r.p, z.p);
  BN_CUDA(cudaMemcpyAsync(p.p, z.p, sizeof(double) * n0, cudaMemcpyDeviceToDevice, s));
  seg_dot(r.p, z.p, d_ptr, inv0, nseg, S_(RZ), s);
  BN_CUDA(cudaMemcpyAsync(S_(RZ0), S_(RZ), sizeof(double) * nseg, cudaMemcpyDeviceToDevice, s));
  BN_LAUNCH(k_seg_start, grid_for(nseg, 256), 256, 0, s, S_(RZ), nseg, active, iters, flag + 1);
  int nact = read_scalar(flag + 1, s);
  ic.check_waits(s);
  const int relres = (opt.stop == AMG_STOP_RELRES) ? 1 : 0;
  int iter = 0;
  stats.device_loop = 0;
  // one CUDA graph for all iterations: the body is one iteration for every
  // segment, its last kernel keeps the loop going while a segment iterates
  cudaGraphExec_t seg_loop = nullptr;
  unsigned long long body_kernels = 0;
  if (loops_ok && !trace_on() && maxiter > 0 && nact > 0) {
    seg_loop = build_loop_graph(s, [&](cudaGraphConditionalHandle h) {
      capture_direct = true;
      spmv<double>(SPMV_Y, A, p.p, nullptr, ap.p, s);
      seg_dot(p.p, ap.p, d_ptr, inv0, nseg, S_(PAP), s);
      seg_alpha(S_(RZ), S_(PAP), active, nseg, S_(ALPHA), s);
      seg_update_xr(x.p, r.p, p.p, ap.p, seg.p, S_(ALPHA), n0, s);
      if (relres) seg_dot(r.p, r.p, d_ptr, inv0, nseg, S_(RR), s);
      if (flexible) seg_dot(r.p, z.p, d_ptr, inv0, nseg, S_(RZON), s);
      precond(r.p, z.p);
      seg_dot(r.p, z.p, d_ptr, inv0, nseg, S_(RZNEW), s);
      BN_CUDA(cudaMemsetAsync(flag + 1, 0, sizeof(int), s));
      seg_next(S_(RZ), S_(RZNEW), S_(RZON), S_(RR), S_(BB), S_(RZ0), active, iters, S_(BETA),
               nseg, flexible ? 1 : 0, relres, tol, 0, flag + 1, s, ctl.p);
      seg_update_p(p.p, z.p, seg.p, S_(BETA), n0, s);
      g_launch_count++;
      k_seg_cond<<<1, 1, 0, s>>>(flag + 1, ctl.p, h);
      BN_CUDA(cudaGetLastError());
      capture_direct = false;
    }, &body_kernels);
    capture_direct = false;
    if (!seg_loop) loops_ok = false;
  }
  if (seg_loop) {
    const int hc[4] = {0, 0, maxiter, 0};
    BN_CUDA(cudaMemcpyAsync(ctl.p, hc, sizeof hc, cudaMemcpyHostToDevice, s));
    BN_CUDA(cudaGraphLaunch(seg_loop, s));
    int hres[4];
    BN_CUDA(cudaMemcpyAsync(hres, ctl.p, sizeof hres, cudaMemcpyDeviceToHost, s));
    BN_CUDA(cudaStreamSynchronize(s));
    cudaGraphExecDestroy(seg_loop);
    g_launch_count += (unsigned long long)hres[0] * body_kernels;
    ic.check_waits(s);
    stats.device_loop = 1;
    iter = hres[0] + 1;
  } else
  for (iter = 1; iter <= maxiter && nact > 0; iter++) {
    spmv<double>(SPMV_Y, A, p.p, nullptr, ap.p, s);
    seg_dot(p.p, ap.p, d_ptr, inv0, nseg, S_(PAP), s);
    seg_alpha(S_(RZ), S_(PAP), active, nseg, S_(ALPHA), s);
    seg_update_xr(x.p, r.p, p.p, ap.p, seg.p, S_(ALPHA), n0, s);
    if (relres) seg_dot(r.p, r.p, d_ptr, inv0, nseg, S_(RR), s);
    if (flexible) seg_dot(r.p, z.p, d_ptr, inv0, nseg, S_(RZON), s);
    precond(r.p, z.p);
    seg_dot(r.p, z.p, d_ptr, inv0, nseg, S_(RZNEW), s);
    BN_CUDA(cudaMemsetAsync(flag + 1, 0, sizeof(int), s));
    seg_next(S_(RZ), S_(RZNEW), S_(RZON), S_(RR), S_(BB), S_(RZ0), active, iters, S_(BETA),
             nseg, flexible ? 1 : 0, relres, tol, iter, flag + 1, s);
    seg_update_p(p.p, z.p, seg.p, S_(BETA), n0, s);
    nact = read_scalar(flag + 1, s);
    ic.check_waits(s);
  }
  // true residual per segment
  spmv<double>(SPMV_RES, A, x.p, b.p, ap.p, s);
  seg_dot(ap.p, ap.p, d_ptr, inv0, nseg, S_(RR), s);
  BN_LAUNCH(k_seg_relres, grid_for(nseg, 256), 256, 0, s, S_(RR), S_(BB), nseg, S_(ALPHA));
  vpermute<double>(x.p, perm0, n0, d_x, true, s);
  cudaEventRecord(ev1, s);
  std::vector<int> hi(2 * (size_t)nseg);
  std::vector<double> hr(nseg);
  BN_CUDA(cudaMemcpyAsync(hi.data(), ints.p, sizeof(int) * 2 * nseg, cudaMemcpyDeviceToHost, s));
  BN_CUDA(cudaMemcpyAsync(hr.data(), S_(ALPHA), sizeof(double) * nseg, cudaMemcpyDeviceToHost, s));
  BN_CUDA(cudaStreamSynchronize(s));
  float ms = 0;
  cudaEventElapsedTime(&ms, ev0, ev1);
  stats.solve_seconds = ms * 1e-3;
  int worst = 0, failed = 0, nan = 0;
  for (int k = 0; k < nseg; k++) {
    int it = hi[nseg + k];
    if (hi[k]) { it = -maxiter; failed = 1; }           // still iterating: no convergence
    else if (it < 0) nan = 1;                            // stopped on a non-finite value
    if (h_iters) h_iters[k] = it;
    if (h_relres) h_relres[k] = hr[k];
    const int a = it < 0 ? -it : it;
    if (a > worst) worst = a;
  }
  stats.iterations = worst;
  stats.converged = !(failed || nan);
  if (nan) {
    set_last_error(BN_ERR_NAN, "segmented PCG: non-finite value in a segment");
    return BN_ERR_NAN;
  }
  if (failed) {
    set_last_error(BN_ERR_NOT_CONVERGED, "segmented PCG: a segment did not converge");
    return BN_ERR_NOT_CONVERGED;
  }
  set_last_error(BN_OK, "");
  return BN_OK;
}

// ------------------------------------------------------------ host helpers
static thread_local int t_status = 0;
static thread_local std::string t_msg;
void set_last_error(int code, const std::string& msg) {
  t_status = code;
  t_msg = msg;
}

static int current_device_count() {
  int c = 0;
  if (cudaGetDeviceCount(&c) != cudaSuccess) return 0;
  return c;
}

// Upload host or device CSR (validated), symmetrise on the device.
void upload_csr(Solver& S, int n, int nnz, const int* ia, const int* ja, const double* val,
                bool device_ptrs, bool symmetrise, CSR& out) {
  BN_REQUIRE(n > 0 && nnz >= 0 && ia && ja && val, BN_ERR_ARG, "invalid CSR arguments");
  CSR Ain;
  Ain.alloc(n, n, nnz, S.s, true);
  if (device_ptrs) {
    BN_CUDA(cudaMemcpyAsync(Ain.ia.p, ia, sizeof(int) * (n + 1), cudaMemcpyDeviceToDevice, S.s));
    BN_CUDA(cudaMemcpyAsync(Ain.ja.p, ja, sizeof(int) * (size_t)nnz, cudaMemcpyDeviceToDevice,
                            S.s));
    BN_CUDA(cudaMemcpyAsync(Ain.val.p, val, sizeof(double) * (size_t)nnz,
                            cudaMemcpyDeviceToDevice, S.s));
  } else {
    copy_h2d(Ain.ia.p, ia, sizeof(int) * (size_t)(n + 1), S.s);
    copy_h2d(Ain.ja.p, ja, sizeof(int) * (size_t)nnz, S.s);
    copy_h2d(Ain.val.p, val, sizeof(double) * (size_t)nnz, S.s);
  }
  int f = validate(Ain.ia.p, Ain.ja.p, n, n, nnz, S.s);
  BN_REQUIRE(!(f & 1), BN_ERR_ARG, "CSR row pointers are not a valid 0-based prefix array");
  BN_REQUIRE(!(f & 2), BN_ERR_ARG, "CSR column index out of range");
  BN_REQUIRE(!(f & 4), BN_ERR_DUP, "CSR row holds a duplicate column index");
  if (symmetrise) symmetrize(Ain, out, S.s);
  else out = std::move(Ain);
}

Solver* make_solver(int n, int nnz, const int* ia, const int* ja, const double* val,
                    const amg_b200_options* o, bool device_ptrs, bool symmetrise) {
  BN_REQUIRE(current_device_count() > 0, BN_ERR_NO_DEVICE, "no CUDA device available");
  std::unique_ptr<Solver> S(new Solver());
  S->opt = *o;
  if (S->opt.nu <= 0) S->opt.nu = 1;
  if (S->opt.max_levels <= 0 || S->opt.max_levels > AMG_MAX_LEVELS)
    S->opt.max_levels = AMG_MAX_LEVELS;
  S->device = o->device;
  BN_CUDA(cudaSetDevice(S->device));
  {
    // keep freed blocks in the stream-ordered pool instead of returning them
    // at every synchronisation (setup synchronises often)
    cudaMemPool_t pool;
    BN_CUDA(cudaDeviceGetDefaultMemPool(&pool, S->device));
    unsigned long long keep = ~0ull;
    BN_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep));
  }
  BN_CUDA(cudaStreamCreateWithFlags(&S->s, cudaStreamNonBlocking));
  BN_CUDA(cudaEventCreate(&S->ev0));
  BN_CUDA(cudaEventCreate(&S->ev1));
  CSR A;
  upload_csr(*S, n, nnz, ia, ja, val, device_ptrs, symmetrise, A);
  S->build(std::move(A));
  return S.release();
}


}  // namespace bn

using bn::Solver;

// ======================================================================
//                               C ABI
// ======================================================================
BN_API void amg_b200_default_options(amg_b200_options* o) {
  if (!o) return;
  o->threshold = 0.25;
  o->min_size = 500;
  o->max_levels = AMG_MAX_LEVELS;
  o->nu = 1;
  o->coarsening = COARSEN_PMIS;
  o->smoother = SMOOTHER_CF_GS;
  o->omega = 0.5;
  o->precision = AMG_PREC_FP64;
  o->stop = AMG_STOP_BNORM;
  o->device = 0;
}

BN_API void* amg_solver_create_ex(int n, int nnz, const int* ia, const int* ja,
                                  const double* val, const amg_b200_options* opt) {
  Solver* out = nullptr;
  amg_b200_options o;
  amg_b200_default_options(&o);
  if (opt) o = *opt;
  bn::guarded([&]() { out = bn::make_solver(n, nnz, ia, ja, val, &o, false); return 0; }, -1);
  if (out) bn::set_last_error(0, "");
  return out;
}

BN_API void* amg_solver_create_device(int n, int nnz, const int* ia, const int* ja,
                                      const double* val, const amg_b200_options* opt) {
  Solver* out = nullptr;
  amg_b200_options o;
  amg_b200_default_options(&o);
  if (opt) o = *opt;
  bn::guarded([&]() { out = bn::make_solver(n, nnz, ia, ja, val, &o, true); return 0; }, -1);
  if (out) bn::set_last_error(0, "");
  return out;
}

BN_API void* amg_solver_create(int n, int nnz, const int* ia, const int* ja, const double* val,
                               double threshold, int min_size, int max_levels, int nu) {
  amg_b200_options o;
  amg_b200_default_options(&o);
  o.threshold = threshold;
  o.min_size = min_size;
  o.max_levels = max_levels;
  o.nu = nu;
  return amg_solver_create_ex(n, nnz, ia, ja, val, &o);
}

BN_API int amg_solver_update(void* h, int n, int nnz, const int* ia, const int* ja,
                             const double* val) {
  if (!h) { bn::set_last_error(bn::BN_ERR_ARG, "NULL handle"); return bn::BN_ERR_ARG; }
  Solver* S = (Solver*)h;
  return bn::guarded([&]() {
    BN_CUDA(cudaSetDevice(S->device));
    BN_REQUIRE(n == S->lv[0]->A.n, bn::BN_ERR_ARG, "update: dimension differs from the hierarchy");
    bn::CSR A;
    bn::upload_csr(*S, n, nnz, ia, ja, val, false, true, A);
    BN_REQUIRE(A.nnz == S->lv[0]->A.nnz, bn::BN_ERR_ARG, "update: sparsity differs");
    S->rebuild_values(std::move(A));
    bn::set_last_error(0, "");
    return 0;
  }, bn::BN_ERR_ARG);
}

BN_API int amg_solver_set_matrix(void* h, int n, int nnz, const int* ia, const int* ja,
                                 const double* val) {
  if (!h) { bn::set_last_error(bn::BN_ERR_ARG, "NULL handle"); return bn::BN_ERR_ARG; }
  Solver* S = (Solver*)h;
  return bn::guarded([&]() {
    BN_CUDA(cudaSetDevice(S->device));
    BN_REQUIRE(n == S->lv[0]->A.n, bn::BN_ERR_ARG, "set_matrix: dimension differs");
    bn::CSR A;
    bn::upload_csr(*S, n, nnz, ia, ja, val, false, true, A);
    S->Aown = std::move(A);
    S->own_solve = true;
    S->ic.want_f32 = (S->opt.precision == AMG_PREC_MIXED);
    S->ic.factor(S->Aown, S->s);
    bn::permute_csr(S->Aown, S->lv[0]->perm.p, S->lv[0]->inv.p, S->Aownp, S->s);
    bn::analyze_rows(S->Aownp, S->layOwn, S->s);
    S->ic.remap(S->lv[0]->inv.p, S->s);
    S->f32_ready = false;
    if (S->opt.precision == AMG_PREC_MIXED) S->prepare_f32();
    S->alloc_vectors();
    S->drop_graphs();
    bn::set_last_error(0, "");
    return 0;
  }, bn::BN_ERR_ARG);
}

BN_API void amg_solver_set_smoother(void* h, int smoother, double omega) {
  if (!h) return;
  Solver* S = (Solver*)h;
  bn::guarded([&]() {
    BN_CUDA(cudaSetDevice(S->device));
    S->opt.smoother = smoother;
    if (smoother == SMOOTHER_JACOBI) S->opt.omega = omega;
    const int nl = (int)S->lv.size();
    for (int l = 0; l < nl - 1; l++) {
      bn::Level& L = *S->lv[l];
      if ((smoother == SMOOTHER_CF_GS || smoother == SMOOTHER_GS) && L.colored_for != smoother)
        S->color_level(L, smoother);
    }
    S->build_solve_layout();
    if (S->opt.precision == AMG_PREC_MIXED) S->prepare_f32();
    S->alloc_vectors();
    S->drop_graphs();
    return 0;
  }, -1);
}

BN_API int amg_solver_set_precision(void* h, int precision) {
  if (!h) return bn::BN_ERR_ARG;
  Solver* S = (Solver*)h;
  return bn::guarded([&]() {
    BN_REQUIRE(precision == AMG_PREC_FP64 || precision == AMG_PREC_MIXED, bn::BN_ERR_ARG,
               "unknown precision");
    BN_CUDA(cudaSetDevice(S->device));
    S->opt.precision = precision;
    if (precision == AMG_PREC_MIXED) {
      if (!S->ic.fval32.n) {
        S->ic.want_f32 = true;
        S->ic.refresh_values();
      }
      S->prepare_f32();
      S->alloc_vectors();
    }
    S->drop_graphs();
    return 0;
  }, bn::BN_ERR_ARG);
}

BN_API int amg_solver_set_stop(void* h, int stop) {
  if (!h) return bn::BN_ERR_ARG;
  ((Solver*)h)->opt.stop = stop;
  return 0;
}

BN_API int amg_solver_solve_device(void* h, const double* d_b, double* d_x, double tol,
                                   int maxiter, int print_level) {
  if (!h) { bn::set_last_error(bn::BN_ERR_ARG, "NULL handle"); return bn::BN_ERR_ARG; }
  Solver* S = (Solver*)h;
  int out = 0;
  int rc = bn::guarded([&]() {
    BN_CUDA(cudaSetDevice(S->device));
    out = S->pcg(d_b, d_x, tol, maxiter, print_level);
    return 0;
  }, -1);
  return rc < 0 ? -maxiter : out;
}

BN_API int amg_solver_solve(void* h, const double* b, double* x, double tol, int maxiter,
                            int print_level) {
  if (!h) { bn::set_last_error(bn::BN_ERR_ARG, "NULL handle"); return bn::BN_ERR_ARG; }
  Solver* S = (Solver*)h;
  int out = 0;
  int rc = bn::guarded([&]() {
    BN_CUDA(cudaSetDevice(S->device));
    const int n = S->n();
    bn::DBuf<double> db(n, S->s), dx(n, S->s);
    bn::copy_h2d(db.p, b, sizeof(double) * (size_t)n, S->s);
    bn::copy_h2d(dx.p, x, sizeof(double) * (size_t)n, S->s);
    out = S->pcg(db.p, dx.p, tol, maxiter, print_level);
    bn::copy_d2h(x, dx.p, sizeof(double) * (size_t)n, S->s);
    return 0;
  }, -1);
  return rc < 0 ? -maxiter : out;
}

// k right-hand sides on one hierarchy: column j of the column-major n x k
// arrays B, X is solved as amg_solver_solve would (X holds the initial guesses).
BN_API int amg_solver_solve_batch(void* h, int k, const double* B, double* X, double tol,
                                  int maxiter, int* iterations) {
  if (!h) { bn::set_last_error(bn::BN_ERR_ARG, "NULL handle"); return bn::BN_ERR_ARG; }
  Solver* S = (Solver*)h;
  return bn::guarded([&]() {
    BN_REQUIRE(k >= 0 && (k == 0 || (B && X)), bn::BN_ERR_ARG,
               "amg_solver_solve_batch: invalid arguments");
    BN_CUDA(cudaSetDevice(S->device));
    const size_t n = (size_t)S->n();
    bn::DBuf<double> db(n * k, S->s), dx(n * k, S->s);
    db.upload(B, n * k);
    dx.upload(X, n * k);
    int failed = 0;
    for (int j = 0; j < k; j++) {
      const int it = S->pcg(db.p + n * j, dx.p + n * j, tol, maxiter, 0);
      if (iterations) iterations[j] = it;
      failed |= it < 0;
    }
    dx.download(X, n * k);
    BN_CUDA(cudaStreamSynchronize(S->s));
    if (failed) {
      bn::set_last_error(bn::BN_ERR_NOT_CONVERGED, "a column did not converge");
      return (int)bn::BN_ERR_NOT_CONVERGED;
    }
    bn::set_last_error(bn::BN_OK, "");
    return 0;
  }, bn::BN_ERR_CUDA);
}

static int solve_segmented(Solver* S, int nseg, const int* seg_ptr, const double* b, double* x,
                           double tol, int maxiter, int* iterations, double* relres,
                           bool device) {
  return bn::guarded([&]() {
    const int n = S->n();
    BN_REQUIRE(nseg > 0 && seg_ptr && b && x, bn::BN_ERR_ARG,
               "segmented solve: invalid arguments");
    BN_REQUIRE(seg_ptr[0] == 0 && seg_ptr[nseg] == n, bn::BN_ERR_ARG,
               "segmented solve: segment offsets must run from 0 to n");
    for (int k = 0; k < nseg; k++)
      BN_REQUIRE(seg_ptr[k + 1] >= seg_ptr[k], bn::BN_ERR_ARG,
                 "segmented solve: segment offsets must not decrease");
    BN_CUDA(cudaSetDevice(S->device));
    bn::DBuf<int> dptr((size_t)nseg + 1, S->s);
    dptr.upload(seg_ptr, (size_t)nseg + 1);
    if (device) return S->pcg_segmented(nseg, dptr.p, b, x, tol, maxiter, iterations, relres);
    bn::DBuf<double> db(n, S->s), dx(n, S->s);
    db.upload(b, n);
    dx.upload(x, n);
    const int rc = S->pcg_segmented(nseg, dptr.p, db.p, dx.p, tol, maxiter, iterations, relres);
    dx.download(x, n);
    BN_CUDA(cudaStreamSynchronize(S->s));
    return rc;
  }, bn::BN_ERR_CUDA);
}

BN_API int amg_solver_solve_segmented(void* h, int nseg, const int* seg_ptr, const double* b,
                                      double* x, double tol, int maxiter, int* iterations,
                                      double* relres) {
  if (!h) { bn::set_last_error(bn::BN_ERR_ARG, "NULL handle"); return bn::BN_ERR_ARG; }
  return solve_segmented((Solver*)h, nseg, seg_ptr, b, x, tol, maxiter, iterations, relres,
                         false);
}

BN_API int amg_solver_solve_segmented_device(void* h, int nseg, const int* seg_ptr,
                                             const double* d_b, double* d_x, double tol,
                                             int maxiter, int* iterations, double* relres) {
  if (!h) { bn::set_last_error(bn::BN_ERR_ARG, "NULL handle"); return bn::BN_ERR_ARG; }
  return solve_segmented((Solver*)h, nseg, seg_ptr, d_b, d_x, tol, maxiter, iterations, relres,
                         true);
}

BN_API int amg_solver_precond(void* h, const double* g, double* xo) {
  if (!h) return bn::BN_ERR_ARG;
  Solver* S = (Solver*)h;
  return bn::guarded([&]() {
    BN_CUDA(cudaSetDevice(S->device));
    const int n = S->n();
    if (S->opt.precision == AMG_PREC_MIXED && !S->f32_ready) S->prepare_f32();
    bn::DBuf<double> dg(n, S->s), dx(n, S->s), pg(n, S->s), px(n, S->s);
    dg.upload(g, n);
    bn::vpermute<double>(dg.p, S->lv[0]->perm.p, n, pg.p, false, S->s);
    S->precond(pg.p, px.p);
    bn::vpermute<double>(px.p, S->lv[0]->perm.p, n, dx.p, true, S->s);
    dx.download(xo, n);
    BN_CUDA(cudaStreamSynchronize(S->s));
    S->ic.check_waits(S->s);
    return 0;
  }, bn::BN_ERR_CUDA);
}

// Times `reps` launches of one hot operation with CUDA events on the solver's
// stream (after one untimed launch).  which: 0 fine-level residual SpMV
// r = b - A x, 1 fine-level forward Gauss-Seidel sweep (all colour classes),
// 2 one preconditioner application, 3 one IC(0) solve (forward + backward).
// precision: 0 FP64, 1 FP32 (the mixed form's V-cycle copies).  Writes the
// mean milliseconds per launch to *ms.  Inputs are the PCG's own vectors.
BN_API int amg_solver_bench_kernel(void* h, int which, int precision, int reps, double* ms) {
  if (!h || !ms || reps <= 0) return bn::BN_ERR_ARG;
  Solver* S = (Solver*)h;
  return bn::guarded([&]() {
    BN_CUDA(cudaSetDevice(S->device));
    const bool f32 = precision == 1;
    if (f32 && !S->f32_ready) {
      if (!S->ic.fval32.n) { S->ic.want_f32 = true; S->ic.refresh_values(); }
      S->prepare_f32();
    }
    if (f32 && !S->g32.n) {
      const int keep = S->opt.precision;
      S->opt.precision = AMG_PREC_MIXED;
      S->alloc_vectors();
      S->opt.precision = keep;
    }
    const int n = S->n();
    bn::Level& L0 = *S->lv[0];
    auto run = [&]() {
      switch (which) {
        case 0:
          if (f32)
            bn::spmv<float>(bn::SPMV_RES, S->mat<float>(S->Asolve_p(),
                                                         S->own_solve ? &S->Aown32 : &L0.A32,
                                                         &S->lay_solve()),
                            S->xxf.p, S->g32.p, S->r1f.p, S->s);
          else
            bn::spmv<double>(bn::SPMV_RES, S->mat<double>(S->Asolve_p(), nullptr,
                                                          &S->lay_solve()),
                             S->x.p, S->b.p, S->r.p, S->s);
          break;
        case 1:
          if (S->lv.size() < 2) break;
          if (f32) S->smooth<float>(0, S->g32.p, S->u1f.p, true);
          else S->smooth<double>(0, S->b.p, S->u1.p, true);
          break;
        case 2:
          S->precond(S->b.p, S->z.p);
          break;
        case 4: {  // first sweep from zero + residual: split form where the level has it
          if (S->lv.size() < 2) break;
          bn::Level& L = L0;
          const int nseg = (int)L.cptr.size() - 1;
          if (!L.split) {
            if (f32) S->smooth<float>(0, S->g32.p, S->u1f.p, true);
            else S->smooth<double>(0, S->b.p, S->u1.p, true);
            if (f32)
              bn::spmv<float>(bn::SPMV_RES, S->mat<float>(L.Ap, &L.A32, &L.layA), S->u1f.p,
                              S->g32.p, L.r32.p, S->s);
            else
              bn::spmv<double>(bn::SPMV_RES, S->mat<double>(L.Ap, nullptr, &L.layA), S->u1.p,
                               S->b.p, L.r.p, S->s);
            break;
          }
          for (int c = 0; c < nseg; c++) {
            const int r0 = L.cptr[c];
            if (f32)
              bn::gs_color<float>(S->mat<float>(L.AL, &L.AL32, &L.layAL), nullptr, r0,
                                  L.cptr[c + 1] - r0, S->g32.p, S->u1f.p, L.gs_group, S->s,
                                  L.clong[c], L.dg32.p);
            else
              bn::gs_color<double>(S->mat<double>(L.AL, nullptr, &L.layAL), nullptr, r0,
                                   L.cptr[c + 1] - r0, S->b.p, S->u1.p, L.gs_group, S->s,
                                   L.clong[c], L.dg.p);
          }
          if (f32)
            bn::spmv<float>(bn::SPMV_Y, S->mat<float>(L.AU, &L.AU32, &L.layAU), S->u1f.p,
                            nullptr, L.r32.p, S->s);
          else
            bn::spmv<double>(bn::SPMV_Y, S->mat<double>(L.AU, nullptr, &L.layAU), S->u1.p,
                             nullptr, L.r.p, S->s);
          break;
        }
        default:
          if (f32) S->ic.solve<float>(S->g32.p, S->icyf.p, S->icxf.p, S->s);
          else S->ic.solve<double>(S->b.p, S->icy.p, S->icx.p, S->s);
          break;
      }
    };
    run();
    BN_CUDA(cudaStreamSynchronize(S->s));
    cudaEventRecord(S->ev0, S->s);
    for (int r = 0; r < reps; r++) run();
    cudaEventRecord(S->ev1, S->s);
    BN_CUDA(cudaEventSynchronize(S->ev1));
    float t = 0;
    cudaEventElapsedTime(&t, S->ev0, S->ev1);
    *ms = (double)t / reps;
    (void)n;
    return 0;
  }, bn::BN_ERR_CUDA);
}

BN_API int amg_solver_size(void* h) { return h ? ((Solver*)h)->n() : 0; }
BN_API int amg_solver_num_levels(void* h) { return h ? (int)((Solver*)h)->lv.size() : 0; }

BN_API void amg_solver_free(void* h) {
  if (!h) return;
  Solver* S = (Solver*)h;
  cudaSetDevice(S->device);
  cudaStream_t s = S->s;
  delete S;
  if (s) {
    cudaStreamSynchronize(s);
    cudaStreamDestroy(s);
  }
}

BN_API int amg_solver_stats(void* h, amg_solve_stats* out) {
  if (!h || !out) return bn::BN_ERR_ARG;
  Solver* S = (Solver*)h;
  S->stats.num_levels = (int)S->lv.size();
  long long t = 0;
  for (auto& L : S->lv) t += L->A.nnz;
  S->stats.nnz_total = t;
  S->stats.ichol_levels = S->ic.nlevels;
  {
    const bool f32 = S->opt.precision == AMG_PREC_MIXED;
    const int m = S->ic.mode;
    const bool slab = f32 ? S->ic.slab_ready<float>() : S->ic.slab_ready<double>();
    S->stats.ichol_form =
        (m == bn::IChol::kSweepSlab || m == bn::IChol::kSweepSlabW) ? (slab ? m : 2) : m;
  }
  *out = S->stats;
  return 0;
}

BN_API int amg_solver_level_info(void* h, int level, int* o) {
  if (!h || !o) return bn::BN_ERR_ARG;
  Solver* S = (Solver*)h;
  if (level < 0 || level >= (int)S->lv.size()) return bn::BN_ERR_ARG;
  bn::Level& L = *S->lv[level];
  const bool last = level == (int)S->lv.size() - 1;
  o[0] = L.A.n;
  o[1] = L.A.nnz;
  o[2] = last ? 0 : L.S.nnz;
  o[3] = last ? 0 : L.P.nnz;
  o[4] = last ? 0 : L.n_coarse;
  return 0;
}

BN_API int amg_solver_level_copy(void* h, int level, int* a_ia, int* a_ja, double* a_val,
                                 int* s_ia, int* s_ja, double* s_val, int* p_ia, int* p_ja,
                                 double* p_val, int* cf) {
  if (!h) return bn::BN_ERR_ARG;
  Solver* S = (Solver*)h;
  if (level < 0 || level >= (int)S->lv.size()) return bn::BN_ERR_ARG;
  return bn::guarded([&]() {
    BN_CUDA(cudaSetDevice(S->device));
    bn::Level& L = *S->lv[level];
    const bool last = level == (int)S->lv.size() - 1;
    const int n = L.A.n;
    if (a_ia) L.A.ia.download(a_ia, n + 1);
    if (a_ja) L.A.ja.download(a_ja, L.A.nnz);
    if (a_val) L.A.val.download(a_val, L.A.nnz);
    if (!last) {
      if (s_ia) L.S.ia.download(s_ia, n + 1);
      if (s_ja) L.S.ja.download(s_ja, L.S.nnz);
      if (s_val) L.S.val.download(s_val, L.S.nnz);
      if (p_ia) L.P.ia.download(p_ia, n + 1);
      if (p_ja) L.P.ja.download(p_ja, L.P.nnz);
      if (p_val) L.P.val.download(p_val, L.P.nnz);
      if (cf) L.cf.download(cf, n);
    }
    BN_CUDA(cudaStreamSynchronize(S->s));
    return 0;
  }, bn::BN_ERR_CUDA);
}

BN_API const char* amg_solver_last_error(void) { return bn::t_msg.c_str(); }
BN_API int amg_solver_last_status(void) { return bn::t_status; }
BN_API unsigned long long amg_b200_launch_count(void) { return bn::g_launch_count; }

// ------------------------------------------------------------ autotuner
// Per level, times the candidate kernels of the solve phase on the level's
// own operators and keeps the fastest:
//  * SpMV, restriction and prolongation (A, R, P): the row-tile kernel with
//    256, 128, 64 or 32 rows per tile (groups 0-3) or 4, 8 or 32 lanes per
//    row (the rows-per-warp / vector-width choice of the row-group kernels);
//  * Gauss-Seidel colour classes: 1, 8 or 32 lanes per row.
// Each candidate computes every row sum over the row's entries (tile
// kernel: in storage order; row groups: lane strides then a fixed shuffle
// tree), so the choice changes rounding only.  Timed in the precision the
// solver runs in; operators on the packed kernels keep them.
namespace bn {
namespace {
template <class T>
double time_ms(cudaStream_t s, cudaEvent_t e0, cudaEvent_t e1, int reps,
               const std::function<void()>& f) {
  f();
  cudaEventRecord(e0, s);
  for (int r = 0; r < reps; r++) f();
  cudaEventRecord(e1, s);
  BN_CUDA(cudaEventSynchronize(e1));
  float t = 0;
  cudaEventElapsedTime(&t, e0, e1);
  return (double)t / reps;
}
}  // namespace

template <class T>
int Solver::autotune_t(int what, double* report, int nreport) {
  const int nl = (int)lv.size();
  const int reps = 5;
  int written = 0;
  auto note = [&](int l, int op, int choice, double ms) {
    if (report && written + 4 <= nreport) {
      report[written++] = l;
      report[written++] = op;
      report[written++] = choice;
      report[written++] = ms;
    }
  };
  for (int l = 0; l + 1 < nl; l++) {
    Level& L = *lv[l];
    Level& C = *lv[l + 1];
    const int n = L.A.n, nc = C.A.n;
    DBuf<T> u(n, s), v(n, s), w(n, s), cu(nc, s);
    BN_CUDA(cudaMemsetAsync(u.p, 0, sizeof(T) * n, s));
    BN_CUDA(cudaMemsetAsync(v.p, 0, sizeof(T) * n, s));
    BN_CUDA(cudaMemsetAsync(cu.p, 0, sizeof(T) * nc, s));
    if (what & 1) {
      struct Op { const CSR* M; const DBuf<float>* v32; RowLayout* lay; bool packed; const T* x;
                  T* y; int id; };
      Op ops[4] = {{&L.Ap, &L.A32, &L.layA, L.use_pkA && use_packed, u.p, v.p, 0},
                   {&L.Rp, &L.R32, &L.layR, L.use_pkR && use_packed, u.p, cu.p, 1},
                   {&L.Pp, &L.P32, &L.layP, L.use_pkP && use_packed, cu.p, v.p, 2},
                   {&L.AU, &L.AU32, &L.layAU, !L.split || (use_packed && L.use_pkA), u.p,
                    v.p, 4}};
      for (Op& op : ops) {
        if (op.packed || op.M->n == 0) continue;
        int best = op.lay->group;
        double best_ms = 1e30;
        for (int g : {0, 1, 2, 3, 4, 5, 8, 16, 32}) {
          op.lay->group = g;
          DevMat<T> M = mat<T>(*op.M, op.v32, op.lay);
          const double ms = time_ms<T>(s, ev0, ev1, reps, [&]() {
            spmv<T>(SPMV_Y, M, op.x, nullptr, op.y, s);
          });
          if (ms < best_ms) { best_ms = ms; best = g; }
        }
        op.lay->group = best;
        note(l, op.id, best, best_ms);
      }
    }
    if ((what & 2) && L.cptr.size() > 1 && n > kSmallLevel && L.A.nnz > kSmallLevelNnz &&
        (opt.smoother == SMOOTHER_CF_GS || opt.smoother == SMOOTHER_GS) &&
        !(use_packed && L.use_pkA)) {
      int best = L.gs_group;
      double best_ms = 1e30;
      for (int g : {0, 1, 2, 4, 8, 16, 32}) {  // 0: staged row tiles
        L.gs_group = g;
        const double ms = time_ms<T>(s, ev0, ev1, reps, [&]() {
          smooth<T>(l, v.p, u.p, true);
        });
        if (ms < best_ms) { best_ms = ms; best = g; }
      }
      L.gs_group = best;
      note(l, 3, best, best_ms);
    }
  }
  drop_graphs();
  BN_CUDA(cudaStreamSynchronize(s));
  return written / 4;
}
template int Solver::autotune_t<double>(int, double*, int);
template int Solver::autotune_t<float>(int, double*, int);

}  // namespace bn

// See include/amg_b200.h for the contract.
BN_API int amg_solver_autotune(void* h, int what, double* report, int nreport) {
  if (!h) { bn::set_last_error(bn::BN_ERR_ARG, "NULL handle"); return bn::BN_ERR_ARG; }
  Solver* S = (Solver*)h;
  return bn::guarded([&]() {
    BN_CUDA(cudaSetDevice(S->device));
    if (S->opt.precision == AMG_PREC_MIXED) {
      if (!S->f32_ready) S->prepare_f32();
      return S->autotune_t<float>(what, report, nreport);
    }
    return S->autotune_t<double>(what, report, nreport);
  }, bn::BN_ERR_CUDA);
}
