// Checks bn::crand_sequence against the C library's srand/rand.
#include <stdio.h>
#include <stdlib.h>
#include <vector>
#include "crand.h"

int main(int argc, char** argv) {
  const long long n = argc > 1 ? atoll(argv[1]) : 1000000;
  const unsigned seeds[] = {12345u, 0u, 1u, 777u, 4294967295u};
  for (unsigned seed : seeds) {
    std::vector<int> v(n);
    bn::crand_sequence(seed, v.data(), n);
    srand(seed);
    for (long long k = 0; k < n; k++) {
      const int r = rand();
      if (r != v[k]) {
        printf("seed %u: mismatch at %lld: %d vs %d\n", seed, k, v[k], r);
        return 1;
      }
    }
  }
  // chunked generation from jump-ahead windows gives the same draws
  const long long step = 2048;
  const long long nchunks = (n + step - 1) / step;
  int nbits = 1;
  while ((1LL << nbits) < nchunks) nbits++;
  std::vector<bn::CrandMat> pw(nbits);
  bn::crand_jump_matrices(step, nbits, pw.data());
  for (unsigned seed : seeds) {
    std::vector<int> v(n);
    bn::crand_sequence(seed, v.data(), n);
    uint32_t first[31], win[31];
    bn::crand_first_window(seed, first);
    for (long long j = 0; j < nchunks; j += (j < 8 ? 1 : 37)) {
      bn::crand_window_at(pw.data(), nbits, first, j, win);
      uint32_t ring[32];
      for (int q = -31; q < 0; q++) ring[q & 31] = win[q + 31];
      for (long long q = 0; q < step && j * step + q < n; q++) {
        const uint32_t r = ring[(q + 1) & 31] + ring[(q - 3) & 31];
        ring[q & 31] = r;
        if ((int)(r >> 1) != v[j * step + q]) {
          printf("seed %u: chunk %lld draw %lld differs\n", seed, j, q);
          return 1;
        }
      }
    }
  }
  printf("ok\n");
  return 0;
}
