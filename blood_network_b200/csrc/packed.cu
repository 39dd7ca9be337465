// Packed-block and long-row-segment CSR kernels (layout: packed.cuh).
#include "packed.cuh"

namespace bn {
namespace {

template <class T> __device__ __forceinline__ T pmul(T a, T b);
template <> __device__ __forceinline__ double pmul(double a, double b) { return __dmul_rn(a, b); }
template <> __device__ __forceinline__ float pmul(float a, float b) { return __fmul_rn(a, b); }
template <class T> __device__ __forceinline__ T padd(T a, T b);
template <> __device__ __forceinline__ double padd(double a, double b) { return __dadd_rn(a, b); }
template <> __device__ __forceinline__ float padd(float a, float b) { return __fadd_rn(a, b); }
template <class T> __device__ __forceinline__ T psub(T a, T b);
template <> __device__ __forceinline__ double psub(double a, double b) { return __dsub_rn(a, b); }
template <> __device__ __forceinline__ float psub(float a, float b) { return __fsub_rn(a, b); }

// The row's result from its sum: the operation's final step.  bi: b_i
// (RES, GS, JAC) or y_i (ADD); di: the diagonal (GS, JAC).
template <class T, int OP>
__device__ __forceinline__ void finish_row(int i, T sum, T bi, T di, T* y, int r0) {
  if (OP == PK_Y) y[i] = sum;
  if (OP == PK_RES) y[i] = psub(bi, sum);
  if (OP == PK_ADD) y[i] = padd(bi, sum);
  if (OP == PK_GS) y[i] = psub(bi, sum) / di;
  if (OP == PK_JAC) y[i - r0] = psub(bi, sum) / di;
}

// Inclusive segmented scan over the block's threads: (f, v) pairs combine
// as (fa, va) + (fb, vb) = (fa | fb, fb ? vb : va + vb), earlier first.
// Returns the inclusive value; *excl receives the previous thread's.
template <class T>
__device__ __forceinline__ T seg_scan(bool f, T v, T* excl) {
  __shared__ T wv[kPackThreads / 32];
  __shared__ int wf[kPackThreads / 32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
    const T ov = __shfl_up_sync(0xffffffffu, v, off);
    const bool of = __shfl_up_sync(0xffffffffu, f, off);
    if (lane >= off) {
      if (!f) v = padd(ov, v);
      f = f || of;
    }
  }
  if (lane == 31) { wv[w] = v; wf[w] = f; }
  __syncthreads();
  // prefix of the warps before this one
  T pv = T(0);
  bool pf = false;
  for (int q = 0; q < w; q++) {
    if (wf[q]) { pv = wv[q]; pf = true; }
    else pv = padd(pv, wv[q]);
  }
  (void)pf;
  if (w > 0 && !f) v = padd(pv, v);
  T prev = __shfl_up_sync(0xffffffffu, v, 1);
  if (lane == 0) prev = pv;  // previous warp's last thread (0 for the first warp)
  *excl = prev;
  return v;
}

// Shared slot of item q: one pad slot after every kPackItems items, so that
// the kPackThreads threads reading their own consecutive items hit distinct
// banks.
__device__ __forceinline__ int pad(int q) { return q + q / kPackItems; }
constexpr int kPadded = kPackNnz + kPackNnz / kPackItems;

template <class T, int OP>
__global__ void __launch_bounds__(kPackThreads, 8)
k_packed(const int* __restrict__ ia, const int* __restrict__ ja, const T* __restrict__ a,
         const T* x, const T* __restrict__ b, T* y, const T* __restrict__ d,
         const int4* __restrict__ blk, int nblk, const int4* __restrict__ seg, int seg_base,
         const int2* __restrict__ lrow, int* cnt, T* part, int r0) {
  BN_PDL_ENTRY();
  constexpr bool kGs = (OP == PK_GS || OP == PK_JAC);
  constexpr bool kRowB = (OP != PK_Y);  // per-row b_i (or y_i for ADD)
  if ((int)blockIdx.x < nblk) {
    __shared__ int s_ja[kGs ? kPadded : 1];
    __shared__ T s_p[kPadded];
    __shared__ int s_ia[kPackRows + 1];
    __shared__ T s_b[kRowB ? kPackRows : 1];
    __shared__ T s_d[kGs ? kPackRows : 1];
    const int4 bb = blk[blockIdx.x];
    const int rb = bb.x, nr = bb.y - bb.x;
    const int e0 = bb.z;
    const int m = bb.w - e0;
    // one load phase: nonzeros (and their x), row pointers, row data
#pragma unroll 4
    for (int q = threadIdx.x; q < m; q += kPackThreads) {
      const int j = ja[e0 + q];
      if (kGs) s_ja[pad(q)] = j;
      s_p[pad(q)] = pmul(a[e0 + q], x[j]);
    }
    for (int r = threadIdx.x; r <= nr; r += kPackThreads) {
      s_ia[r] = ia[rb + r] - e0;
      if (r < nr) {
        if (OP == PK_ADD) s_b[r] = y[rb + r];
        else if (kRowB) s_b[r] = b[rb + r];
        if (kGs) s_d[r] = d[rb + r];
      }
    }
    __syncthreads();
    auto fin = [&](int rr, T sum) {
      finish_row<T, OP>(rb + rr, sum, kRowB ? s_b[rr] : T(0), kGs ? s_d[rr] : T(0), y, r0);
    };
    // rows without entries
    for (int r = threadIdx.x; r < nr; r += kPackThreads)
      if (s_ia[r] == s_ia[r + 1]) fin(r, T(0));
    // this thread's items [q0, q1)
    const int q0 = threadIdx.x * kPackItems;
    const int q1 = min(q0 + kPackItems, m);
    int r = 0;
    bool first_cont = false, head_pending = false;
    T head = T(0), sum = T(0);
    int first = -1;
    if (q0 < m) {
      int lo = 0, hi = nr - 1;  // last row starting at or before q0
      while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (s_ia[mid] <= q0) lo = mid;
        else hi = mid - 1;
      }
      r = lo;
      first = r;
      first_cont = s_ia[r] < q0;
      for (int q = q0; q < q1; q++) {
        while (s_ia[r + 1] <= q) {  // row r ended inside this range
          if (r == first && first_cont) { head = sum; head_pending = true; }
          else if (s_ia[r] < s_ia[r + 1]) fin(r, sum);
          r++;
          sum = T(0);
        }
        if (!kGs || s_ja[pad(q)] != rb + r) sum = padd(sum, s_p[pad(q)]);
      }
      if (s_ia[r + 1] == q1) {  // the last row ends here too
        if (r == first && first_cont) { head = sum; head_pending = true; }
        else fin(r, sum);
      }
    }
    // the last row's partial, flagged where that row starts in this range
    const bool flag = (q0 >= m) || (s_ia[r] >= q0);
    T carry;
    seg_scan<T>(flag, q0 < m ? sum : T(0), &carry);
    if (head_pending) fin(first, padd(carry, head));
    return;
  }
  // a segment of a long row
  __shared__ T red[kPackThreads / 32];
  const int sidx = blockIdx.x - nblk;
  const int4 sg = seg[sidx];
  T sum = T(0);
#pragma unroll 4
  for (int k = sg.y + threadIdx.x; k < sg.z; k += kPackThreads) {
    const int j = ja[k];
    if (!kGs || j != sg.x) sum = padd(sum, pmul(a[k], x[j]));
  }
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) sum = padd(sum, __shfl_xor_sync(0xffffffffu, sum, off));
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = sum;
  __syncthreads();
  if (threadIdx.x == 0) {
    T t = T(0);
    for (int w = 0; w < kPackThreads / 32; w++) t = padd(t, red[w]);
    const int2 lr = lrow[sg.w];
    const int i = sg.x;
    const T bi = OP == PK_ADD ? y[i] : (kRowB ? b[i] : T(0));
    const T di = kGs ? d[i] : T(0);
    if (lr.y == 1) {
      finish_row<T, OP>(i, t, bi, di, y, r0);
    } else {
      part[seg_base + sidx] = t;
      __threadfence();
      const int ticket = atomicAdd(&cnt[sg.w], 1);
      if (ticket == lr.y - 1) {  // last segment of the row: add the partials in order
        __threadfence();
        T tot = T(0);
        for (int q = 0; q < lr.y; q++) tot = padd(tot, __ldcg(part + lr.x + q));
        finish_row<T, OP>(i, tot, bi, di, y, r0);
        cnt[sg.w] = 0;
      }
    }
  }
}

}  // namespace

void Packing::build(const std::vector<int>& ia, const std::vector<int2>& ranges, cudaStream_t s) {
  std::vector<int2> hl;
  std::vector<int4> hb, hs;
  auto block = [&](int r_first, int r_end) {
    hb.push_back(make_int4(r_first, r_end, ia[r_first], ia[r_end]));
  };
  rb.clear();
  rs.clear();
  for (const int2& rg : ranges) {
    rb.push_back((int)hb.size());
    rs.push_back((int)hs.size());
    int first = rg.x;
    long long acc = 0;
    for (int r = rg.x; r < rg.y; r++) {
      const int len = ia[r + 1] - ia[r];
      if (len > kPackNnz) {
        if (first < r) block(first, r);
        const int ns = (len + kPackNnz - 1) / kPackNnz;
        const int li = (int)hl.size();
        hl.push_back(make_int2((int)hs.size(), ns));
        for (int q = 0; q < ns; q++) {
          const int k0 = ia[r] + q * kPackNnz;
          const int k1 = k0 + kPackNnz < ia[r + 1] ? k0 + kPackNnz : ia[r + 1];
          hs.push_back(make_int4(r, k0, k1, li));
        }
        first = r + 1;
        acc = 0;
        continue;
      }
      const int w = len > 0 ? len : 1;  // an empty row still takes a slot
      if (acc + w > kPackNnz || r - first >= kPackRows) {
        block(first, r);
        first = r;
        acc = 0;
      }
      acc += w;
    }
    if (first < rg.y) block(first, rg.y);
  }
  rb.push_back((int)hb.size());
  rs.push_back((int)hs.size());
  nblk = (int)hb.size();
  nseg = (int)hs.size();
  nlong = (int)hl.size();
  blk.alloc(nblk > 0 ? nblk : 1, s);
  seg.alloc(nseg > 0 ? nseg : 1, s);
  lrow.alloc(nlong > 0 ? nlong : 1, s);
  cnt.alloc(nlong > 0 ? nlong : 1, s);
  part.alloc(nseg > 0 ? nseg : 1, s);
  cnt.zero();
  if (nblk) blk.upload(hb.data(), nblk);
  if (nseg) seg.upload(hs.data(), nseg);
  if (nlong) lrow.upload(hl.data(), nlong);
  BN_CUDA(cudaStreamSynchronize(s));
}

template <class T, int OP>
static void launch_packed(const PackedMat<T>& A, int q, const T* x, const T* b, T* y,
                          const T* d, int r0, cudaStream_t s) {
  const Packing& P = *A.pk;
  BN_REQUIRE(q >= 0 && q < P.ranges(), BN_ERR_ARG, "packed kernel: range outside the packing");
  const int b0 = P.rb[q], nb = P.rb[q + 1] - b0;
  const int s0 = P.rs[q], ns = P.rs[q + 1] - s0;
  if (nb + ns == 0) return;
  BN_LAUNCH_PDL((k_packed<T, OP>), nb + ns, kPackThreads, 0, s, A.ia, A.ja, A.val, x, b, y, d,
            P.blk.p + b0, nb, P.seg.p + s0, s0, P.lrow.p, P.cnt.p, (T*)P.part.p, r0);
}

template <class T>
void packed_apply(int op, const PackedMat<T>& A, int q, const T* x, const T* b, T* y, const T* d,
                  int r0, cudaStream_t s) {
  switch (op) {
    case PK_Y: launch_packed<T, PK_Y>(A, q, x, b, y, d, r0, s); break;
    case PK_RES: launch_packed<T, PK_RES>(A, q, x, b, y, d, r0, s); break;
    case PK_ADD: launch_packed<T, PK_ADD>(A, q, x, b, y, d, r0, s); break;
    case PK_GS: launch_packed<T, PK_GS>(A, q, x, b, y, d, r0, s); break;
    default: launch_packed<T, PK_JAC>(A, q, x, b, y, d, r0, s); break;
  }
}

template void packed_apply<double>(int, const PackedMat<double>&, int, const double*,
                                   const double*, double*, const double*, int, cudaStream_t);
template void packed_apply<float>(int, const PackedMat<float>&, int, const float*, const float*,
                                  float*, const float*, int, cudaStream_t);

}  // namespace bn
