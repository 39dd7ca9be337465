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

}  // namespace bn
