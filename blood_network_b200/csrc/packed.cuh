// Load-balanced CSR kernels for the V-cycle: packed row blocks + long-row
// segments.
//
// A row range is cut, once at setup, into
//  * packed blocks: runs of consecutive rows holding at most kPackNnz
//    nonzeros together (at most kPackRows rows), one thread block each.  The
//    block stages the products a_ij * x_j of all its nonzeros, and the
//    rows' right-hand sides and diagonals, in shared memory in one load
//    phase (coalesced loads), each thread then sums kPackItems
//    consecutive products, and a segmented scan across the block's threads
//    completes the rows that straddle threads;
//  * segments: a row longer than kPackNnz is split into kPackNnz-entry
//    segments, one thread block each.  Each writes its partial sum; the last
//    segment of the row to finish (arrival counter after a memory fence)
//    adds the partials in segment order and finishes the row.
// Both summation orders are fixed, so the results are deterministic.  The
// same machinery serves y = A x, r = b - A x, y += A x and the Gauss-Seidel
// update x_i = (b_i - sum_{j != i} a_ij x_j) / a_ii of one colour class.
#pragma once
#include "common.cuh"

#include <vector>

namespace bn {

constexpr int kPackNnz = 1024;
constexpr int kPackRows = 512;   // rows per packed block at most
constexpr int kPackThreads = 256;
constexpr int kPackItems = kPackNnz / kPackThreads;

enum PackOp : int {
  PK_Y = 0,    // y_i = sum_j a_ij x_j
  PK_RES = 1,  // y_i = b_i - sum_j a_ij x_j
  PK_ADD = 2,  // y_i += sum_j a_ij x_j
  PK_GS = 3,   // x_i = (b_i - sum_{j != i} a_ij x_j) / d_i, in place
  PK_JAC = 4   // out[i - r0] = (b_i - sum_{j != i} a_ij x_j) / d_i
};

// The packing of one or more row ranges of a matrix (ranges: colour classes).
struct Packing {
  int nblk = 0, nseg = 0, nlong = 0;
  DBuf<int4> blk;      // packed blocks: {first row, end row, first entry, end entry}
  DBuf<int4> seg;      // segments: {row, first entry, end entry, long-row index}
  DBuf<int2> lrow;     // per long row: {first segment, segment count}
  DBuf<int> cnt;       // per long row: arrival counter, zero between launches
  DBuf<double> part;   // per segment: partial sum (float or double)
  std::vector<int> rb, rs;  // per range: first block, first segment (+ totals)
  void build(const std::vector<int>& ia, const std::vector<int2>& ranges, cudaStream_t s);
  int ranges() const { return rb.empty() ? 0 : (int)rb.size() - 1; }
};

template <class T>
struct PackedMat {
  const int* ia = nullptr;
  const int* ja = nullptr;
  const T* val = nullptr;
  const Packing* pk = nullptr;
};

// One range q of the packing.  b: right-hand side (RES, GS, JAC); d: the
// diagonal (GS, JAC; 1 where a row has none); out: JAC output indexed from
// r0, the range's first row.
template <class T>
void packed_apply(int op, const PackedMat<T>& A, int q, const T* x, const T* b, T* y,
                  const T* d, int r0, cudaStream_t s);

}  // namespace bn
