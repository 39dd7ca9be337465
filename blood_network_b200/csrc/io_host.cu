// Host readers and writers for the reference's on-disk formats.
//   COO text matrix (C_amg1/src/io.c:71-124 dcsr_mat_dcoo, with the COO ->
//   CSR conversion of io.c:19-58 dcoo2dcsr):
//     "nrows ncols nnz" then nnz lines "row col value"; indices are shifted
//     down by one when the smallest row or column index is exactly 1; rows are
//     filled by a stable counting sort, so the entries of a row keep their
//     file order and repeated (row, col) pairs stay separate entries.
//   Right-hand side (C_amg1/test_amg.c:126-148): "n" then n values.
//   Labelled solution (Matlab_amg/label_solution.m:41-44): one line
//     "%d %.16e" per interior node (1-based node id, pressure).
// The reference trusts its input; these return AMG_ERR_ARG for a malformed
// file or an index out of range instead.
#include "common.cuh"
#include "../../include/amg_b200.h"

#include <algorithm>
#include <cctype>
#include <cerrno>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <string>
#include <thread>
#include <vector>

namespace {

struct Text {
  std::vector<char> buf;
  const char* p = nullptr;
  const char* end = nullptr;
  bool load(const char* path) {
    FILE* f = fopen(path, "rb");
    if (!f) return false;
    if (fseek(f, 0, SEEK_END) == 0) {  // size the buffer once when the file is seekable
      const long sz = ftell(f);
      if (sz > 0) buf.reserve((size_t)sz + 1);
      fseek(f, 0, SEEK_SET);
    }
    char tmp[1 << 16];
    size_t got;
    while ((got = fread(tmp, 1, sizeof tmp, f)) > 0) buf.insert(buf.end(), tmp, tmp + got);
    fclose(f);
    buf.push_back('\0');
    p = buf.data();
    end = buf.data() + buf.size() - 1;
    return true;
  }
  // same conversions as fscanf's %d and %lf (strtol / strtod)
  bool next_int(long long& v) {
    char* e = nullptr;
    errno = 0;
    v = strtoll(p, &e, 10);
    if (e == p || errno) return false;
    p = e;
    return true;
  }
  bool next_double(double& v) {
    char* e = nullptr;
    v = strtod(p, &e);
    if (e == p) return false;
    p = e;
    return true;
  }
};

// The COO entries of a large file are parsed by several threads: the text
// is cut at whitespace into one piece per thread, each piece's tokens are
// counted, and then each thread converts its tokens knowing their global
// position (token 3k and 3k+1 are the indices of entry k, 3k+2 its value).
// The conversions are strtoll / strtod as in the one-thread reader, so the
// result is the same; tokens past entry nz-1 are ignored, as there.
// Returns -1, or the first entry that cannot be read.
long long parse_entries(const char* p, const char* end, long long nz, int* r, int* c,
                        double* v) {
  const size_t len = (size_t)(end - p);
  const unsigned hw = std::thread::hardware_concurrency();
  const int nt = len < (1u << 20) ? 1 : (int)std::max(1u, std::min(16u, hw ? hw : 1u));
  std::vector<const char*> cut(nt + 1);
  cut[0] = p;
  cut[nt] = end;
  for (int t = 1; t < nt; t++) {
    const char* q = p + len * t / nt;
    if (q < cut[t - 1]) q = cut[t - 1];
    while (q < end && !isspace((unsigned char)*q)) q++;
    cut[t] = q;
  }
  std::vector<long long> count(nt + 1, 0), first_bad(nt, -1);
  auto run = [&](const std::function<void(int)>& f) {
    std::vector<std::thread> th;
    for (int t = 1; t < nt; t++) th.emplace_back(f, t);
    f(0);
    for (auto& x : th) x.join();
  };
  run([&](int t) {  // tokens per piece
    long long k = 0;
    bool in = false;
    for (const char* q = cut[t]; q < cut[t + 1]; q++) {
      const bool sp = isspace((unsigned char)*q) || *q == '\0';
      if (!sp && !in) k++;
      in = !sp;
    }
    count[t + 1] = k;
  });
  for (int t = 0; t < nt; t++) count[t + 1] += count[t];
  const long long need = 3 * nz;
  run([&](int t) {
    long long g = count[t];
    const char* q = cut[t];
    const char* stop = cut[t + 1];
    while (g < need) {
      while (q < stop && (isspace((unsigned char)*q) || *q == '\0')) q++;
      if (q >= stop) break;
      const char* tok_end = q;
      while (tok_end < stop && !isspace((unsigned char)*tok_end) && *tok_end != '\0') tok_end++;
      char* e = nullptr;
      bool ok;
      const long long entry = g / 3;
      if (g % 3 == 2) {
        v[entry] = strtod(q, &e);
        ok = e == tok_end;
      } else {
        errno = 0;
        const long long x = strtoll(q, &e, 10);
        ok = e == tok_end && !errno && x >= INT32_MIN && x <= INT32_MAX;
        (g % 3 == 0 ? r : c)[entry] = (int)x;
      }
      if (!ok) {
        first_bad[t] = entry;
        break;
      }
      q = tok_end;
      g++;
    }
  });
  long long bad = -1;
  for (int t = 0; t < nt; t++)
    if (first_bad[t] >= 0 && (bad < 0 || first_bad[t] < bad)) bad = first_bad[t];
  if (count[nt] < need) {
    const long long short_at = count[nt] / 3;
    if (bad < 0 || short_at < bad) bad = short_at;
  }
  return bad;
}

int fail(int code, const std::string& msg) {
  bn::set_last_error(code, msg);
  return code;
}

}  // namespace

BN_API void amg_free_host(void* p) { free(p); }

BN_API int amg_read_coo(const char* path, int* nrow, int* ncol, int* nnz, int** ia, int** ja,
                        double** val) {
  using namespace bn;
  if (!path || !nrow || !ncol || !nnz || !ia || !ja || !val)
    return fail(BN_ERR_ARG, "amg_read_coo: NULL argument");
  *ia = *ja = nullptr;
  *val = nullptr;
  Text t;
  if (!t.load(path)) return fail(BN_ERR_ARG, std::string("amg_read_coo: cannot open ") + path);
  long long m, n, nz;
  if (!t.next_int(m) || !t.next_int(n) || !t.next_int(nz) || m < 0 || n < 0 || nz < 0 ||
      m > 0x7fffffff || n > 0x7fffffff || nz > 0x7fffffff)
    return fail(BN_ERR_ARG, "amg_read_coo: cannot read the header \"nrows ncols nnz\"");
  std::vector<int> r((size_t)nz), c((size_t)nz);
  std::vector<double> v((size_t)nz);
  const long long bad = parse_entries(t.p, t.end, nz, r.data(), c.data(), v.data());
  if (bad >= 0) return fail(BN_ERR_ARG, "amg_read_coo: cannot read entry " + std::to_string(bad));
  long long lo = 0;
  for (long long k = 0; k < nz; k++) {
    if (k == 0) lo = r[k];
    if (r[k] < lo) lo = r[k];
    if (c[k] < lo) lo = c[k];
  }
  const int shift = (nz > 0 && lo == 1) ? 1 : 0;  // 1-based file
  std::vector<int> ptr((size_t)m + 1, 0);
  for (long long k = 0; k < nz; k++) {
    const long long a = (long long)r[k] - shift, b = (long long)c[k] - shift;
    if (a < 0 || a >= m || b < 0 || b >= n)
      return fail(BN_ERR_ARG, "amg_read_coo: entry " + std::to_string(k) + " is out of range");
    ptr[a + 1]++;
  }
  for (long long i = 0; i < m; i++) ptr[i + 1] += ptr[i];
  int* oia = (int*)malloc(sizeof(int) * ((size_t)m + 1));
  int* oja = (int*)malloc(sizeof(int) * (nz > 0 ? (size_t)nz : 1));
  double* ov = (double*)malloc(sizeof(double) * (nz > 0 ? (size_t)nz : 1));
  if (!oia || !oja || !ov) {
    free(oia);
    free(oja);
    free(ov);
    return fail(BN_ERR_OOM, "amg_read_coo: out of host memory");
  }
  memcpy(oia, ptr.data(), sizeof(int) * ((size_t)m + 1));
  for (long long k = 0; k < nz; k++) {  // stable: file order within a row
    const int row = r[k] - shift;
    const int at = ptr[row]++;
    oja[at] = c[k] - shift;
    ov[at] = v[k];
  }
  *nrow = (int)m;
  *ncol = (int)n;
  *nnz = (int)nz;
  *ia = oia;
  *ja = oja;
  *val = ov;
  set_last_error(BN_OK, "");
  return BN_OK;
}

BN_API int amg_read_vector(const char* path, int n, double* out) {
  using namespace bn;
  if (!path || n < 0 || (n > 0 && !out)) return fail(BN_ERR_ARG, "amg_read_vector: invalid arguments");
  Text t;
  if (!t.load(path)) return fail(BN_ERR_ARG, std::string("amg_read_vector: cannot open ") + path);
  long long len;
  if (!t.next_int(len)) return fail(BN_ERR_ARG, "amg_read_vector: cannot read the length");
  if (len != n)
    return fail(BN_ERR_ARG, "amg_read_vector: the file holds " + std::to_string(len) +
                                " values, expected " + std::to_string(n));
  for (int i = 0; i < n; i++)
    if (!t.next_double(out[i]))
      return fail(BN_ERR_ARG, "amg_read_vector: cannot read entry " + std::to_string(i));
  set_last_error(BN_OK, "");
  return BN_OK;
}

BN_API int amg_write_labeled_solution(const char* path, int n, const int* node, const double* p) {
  using namespace bn;
  if (!path || n < 0 || (n > 0 && (!node || !p)))
    return fail(BN_ERR_ARG, "amg_write_labeled_solution: invalid arguments");
  FILE* f = fopen(path, "w");
  if (!f) return fail(BN_ERR_ARG, std::string("amg_write_labeled_solution: cannot open ") + path);
  for (int i = 0; i < n; i++) fprintf(f, "%d %.16e\n", node[i], p[i]);
  const bool ok = fclose(f) == 0;
  if (!ok) return fail(BN_ERR_ARG, "amg_write_labeled_solution: write failed");
  set_last_error(BN_OK, "");
  return BN_OK;
}
