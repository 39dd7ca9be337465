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
  printf("ok\n");
  return 0;
}
