// The C library's rand() sequence after srand(seed), computed without
// touching the library's own generator state.
//
// glibc's rand() is random() on its default state, an additive feedback
// generator over 31 words (published description of the algorithm):
//   r[0] = seed (1 if seed is 0);
//   r[i] = 16807 * r[i-1] mod (2^31 - 1)   for i = 1..30 (Schrage's method,
//          no overflow in 32-bit signed arithmetic);
//   r[i] = r[i-31]                          for i = 31..33;
//   r[i] = r[i-31] + r[i-3]  (mod 2^32)     for i >= 34;
// the values r[34..343] are discarded and the k-th rand() returns
// r[344 + k] >> 1.  A 34-word ring holds the recurrence.
#pragma once
#include <stdint.h>

namespace bn {

inline void crand_sequence(unsigned seed, int* out, long long n) {
  uint32_t ring[34];
  int32_t w = seed == 0 ? 1 : (int32_t)seed;
  ring[0] = (uint32_t)w;
  for (int i = 1; i < 31; i++) {
    const int32_t hi = w / 127773, lo = w % 127773;
    int32_t word = 16807 * lo - 2836 * hi;
    if (word < 0) word += 2147483647;
    ring[i] = (uint32_t)word;
    w = word;
  }
  for (int i = 31; i < 34; i++) ring[i] = ring[i - 31];
  // position p of the recurrence lives in ring[p % 34]
  long long p = 34;
  auto next = [&]() {
    const uint32_t v = ring[(p - 31) % 34] + ring[(p - 3) % 34];
    ring[p % 34] = v;
    p++;
    return v;
  };
  for (int i = 34; i < 344; i++) next();
  for (long long k = 0; k < n; k++) out[k] = (int)(next() >> 1);
}

// Jump-ahead.  From position 34 on the recurrence is linear over Z/2^32:
// with the window s_p = (r[p-31], ..., r[p-1]), s_{p+1} = M s_p, where M
// shifts the window by one and appends s_0 + s_28.  The window before draw
// k (position 344 + k) is therefore M^k s_344, so the draws can be produced
// in independent chunks from their starting windows.
struct CrandMat {
  uint32_t a[31][31];
};

// z = x y (mod 2^32)
inline void crand_mat_mul(const CrandMat& x, const CrandMat& y, CrandMat& z) {
  for (int i = 0; i < 31; i++)
    for (int j = 0; j < 31; j++) {
      uint32_t t = 0;
      for (int k = 0; k < 31; k++) t += x.a[i][k] * y.a[k][j];
      z.a[i][j] = t;
    }
}

// w = m v (mod 2^32)
inline void crand_mat_vec(const CrandMat& m, const uint32_t* v, uint32_t* w) {
  for (int i = 0; i < 31; i++) {
    uint32_t t = 0;
    for (int k = 0; k < 31; k++) t += m.a[i][k] * v[k];
    w[i] = t;
  }
}

// The window before the first draw after srand(seed): r[313..343].
inline void crand_first_window(unsigned seed, uint32_t* win) {
  uint32_t r[344];
  int32_t w = seed == 0 ? 1 : (int32_t)seed;
  r[0] = (uint32_t)w;
  for (int i = 1; i < 31; i++) {
    const int32_t hi = w / 127773, lo = w % 127773;
    int32_t word = 16807 * lo - 2836 * hi;
    if (word < 0) word += 2147483647;
    r[i] = (uint32_t)word;
    w = word;
  }
  for (int i = 31; i < 34; i++) r[i] = r[i - 31];
  for (int i = 34; i < 344; i++) r[i] = r[i - 31] + r[i - 3];
  for (int i = 0; i < 31; i++) win[i] = r[313 + i];
}

// pw[b] = M^(step * 2^b) for b < nbits (step >= 1).
inline void crand_jump_matrices(long long step, int nbits, CrandMat* pw) {
  CrandMat m{}, t{};
  for (int i = 0; i < 30; i++) m.a[i][i + 1] = 1;
  m.a[30][0] = 1;
  m.a[30][28] = 1;
  CrandMat acc{};
  for (int i = 0; i < 31; i++) acc.a[i][i] = 1;
  for (long long e = step; e > 0; e >>= 1) {  // acc = M^step
    if (e & 1) {
      crand_mat_mul(acc, m, t);
      acc = t;
    }
    crand_mat_mul(m, m, t);
    m = t;
  }
  for (int b = 0; b < nbits; b++) {
    pw[b] = acc;
    crand_mat_mul(acc, acc, t);
    acc = t;
  }
}

// The window before draw j * step: the product of the matrices of j's set
// bits applied to the first window.
inline void crand_window_at(const CrandMat* pw, int nbits, const uint32_t* first, long long j,
                            uint32_t* win) {
  uint32_t v[31], t[31];
  for (int i = 0; i < 31; i++) v[i] = first[i];
  for (int b = 0; b < nbits; b++)
    if ((j >> b) & 1) {
      crand_mat_vec(pw[b], v, t);
      for (int i = 0; i < 31; i++) v[i] = t[i];
    }
  for (int i = 0; i < 31; i++) win[i] = v[i];
}

}  // namespace bn
