// Solve-phase kernel interfaces.
#pragma once
#include "common.cuh"

namespace bn {

constexpr int kRows = 256;        // rows per SpMV tile (= threads per block)
constexpr int kTileNnz = 2048;    // shared product buffer per tile
constexpr int kRedBlocks = 1184;  // blocks for reductions (8 per SM)

enum SpmvMode : int { SPMV_Y = 0, SPMV_RES = 1, SPMV_ADD = 2 };

// PCG scalar block slots (device memory)
enum ScalarSlot : int {
  SC_RZ = 0,        // r_k . z_k
  SC_PAP = 1,       // p . Ap
  SC_RR = 2,        // r . r
  SC_RZNEW = 3,     // r_{k+1} . z_{k+1}
  SC_RZOLD_NEW = 4, // r_{k+1} . z_k  (flexible beta)
  SC_BETA = 5,
  SC_RZ_PREV = 6,
  SC_RZ0 = 7,
  SC_BB = 8,
  SC_COUNT = 16
};

constexpr int kLongRow = 1024;    // rows longer than this get a block each
constexpr int kLongThreads = 256;

// Non-owning CSR view with values of type T, plus the row-length layout the
// kernels dispatch on: group 0-3 select the row-tile kernel (256/128/64/32
// rows per tile), 5 the row tiles staged by bulk copies, 4/8/32 that many
// lanes per row; rows longer than kLongRow are listed in lrows and handled
// by one block each.
template <class T>
struct DevMat {
  int n = 0, m = 0, nnz = 0;
  const int* ia = nullptr;
  const int* ja = nullptr;
  const T* val = nullptr;
  int group = 0;
  const int* lrows = nullptr;
  int nlong = 0;
  const int* tiles = nullptr;  // row-tile kernel: order in which tiles are visited (null: natural)
};

// Row-length layout of a CSR matrix (computed once at setup).
struct RowLayout {
  int group = 0;
  DBuf<int> tiles;  // visiting order of the kRows-row tiles (empty: natural)
  DBuf<int> lrows;
  int nlong = 0;
};
void analyze_rows(const CSR& A, RowLayout& out, cudaStream_t s);
// Visit the row tiles of a matrix in the order of key[first row of tile]
// (rows renumbered into colour classes: key = original row number, so that
// concurrently processed tiles gather from one neighbourhood of x).
void order_tiles(int n, const int* key, RowLayout& out, cudaStream_t s);

inline int spmv_grid(int n) {
  int tiles = (n + kRows - 1) / kRows;
  int cap = kSMs * 8;
  return tiles < cap ? tiles : cap;
}

// y = A x | b - A x | y + A x.  With dot_w, also writes partial sums of
// dot_w . y; returns the number of partial slots written (0 without dot_w).
template <class T>
int spmv(int mode, const DevMat<T>& A, const T* x, const T* b, T* y, cudaStream_t s,
         const T* dot_w = nullptr, double* partial = nullptr);
int spmv_partials(int n, int nlong);
// 1 if a bounded wait of the staged SpMV ran out since the last call (then cleared)
int take_stage_error();
// Rows of one colour class: rows[t] (or r0 + t when rows is null, a
// contiguous class); its last nlong rows are long rows (one block each).
// group: lanes per row (1/8/32), or 0 for the staged row tiles, which need
// a contiguous class and the diagonal d (1 where a row has none).
template <class T>
void gs_color(const DevMat<T>& A, const int* rows, int r0, int nr, const T* b, T* x, int group,
              cudaStream_t s, int nlong = 0, const T* d = nullptr);
template <class T>
void jacobi_class(const DevMat<T>& A, const int* rows, int r0, int nr, const T* b, T* x, T* tmp,
                  int group, cudaStream_t s, int nlong = 0, const T* d = nullptr);
// x[r0 + t] = v[t], t < nr
template <class T>
void scatter_range(const T* v, int r0, int nr, T* x, cudaStream_t s);
// all colour classes of a small level, one block, one launch
template <class T>
void gs_level_block(const DevMat<T>& A, const int* cptr, const int* cjac, int ncls, bool forward,
                    const T* b, T* x, T* tmp, cudaStream_t s);
// gather out[t] = in[map[t]] or scatter out[map[t]] = in[t]
template <class T>
void vpermute(const T* in, const int* map, int n, T* out, bool scatter, cudaStream_t s);
template <class T>
void vzero(T* x, int n, cudaStream_t s);
template <class TO, class TI>
void vconvert(const TI* a, int n, TO* b, cudaStream_t s);
template <class T>
void vadd(const T* u, const T* v, int n, T* x, cudaStream_t s);
template <class T>
void dot_partials(const T* u, const T* v, const T* w, int n, double* p0, double* p1,
                  cudaStream_t s);
void reduce_partials(const double* part, int m, double* out, cudaStream_t s);
void vaxpy(double* y, const double* u, double a, int n, cudaStream_t s);   // y += a u
// segmented PCG helpers: segments are natural row ranges ptr[k]..ptr[k+1]-1,
// idx maps a natural row to its solve index, seg a solve index to its segment
void seg_dot(const double* u, const double* v, const int* ptr, const int* idx, int nseg,
             double* out, cudaStream_t s);
void seg_of_rows(const int* perm, int n, const int* ptr, int nseg, int* seg, cudaStream_t s);
void seg_update_xr(double* x, double* r, const double* p, const double* ap, const int* seg,
                   const double* alpha, int n, cudaStream_t s);
void seg_update_p(double* p, const double* z, const int* seg, const double* beta, int n,
                  cudaStream_t s);
void seg_alpha(const double* rz, const double* pap, const int* active, int nseg, double* alpha,
               cudaStream_t s);
void seg_next(double* rz, const double* rznew, const double* rzold_new, const double* rr,
              const double* bb, const double* rz0, int* active, int* iters, double* beta,
              int nseg, int flexible, int relres, double tol, int iter, int* nactive,
              cudaStream_t s, const int* iters_done = nullptr);
void vxpby(double* p, const double* z, double b, int n, cudaStream_t s);   // p = z + b p
void pcg_update_xr(double* x, double* r, const double* p, const double* ap, int n,
                   const double* sc, double* part, cudaStream_t s);
void pcg_update_p(double* p, const double* z, int n, const double* sc, cudaStream_t s);
void pcg_scalars(double* sc, int flexible, cudaStream_t s);

}  // namespace bn
