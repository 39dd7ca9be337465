/* A C caller written against the reference wrapper's API (amg_solver_create /
 * amg_solver_solve / amg_solver_free, C_amg1/src/amg_wrapper.c), built
 * unchanged against include/amg_b200.h and linked with libamg_b200.so.
 * Solves a diagonally dominant 1D operator (2.5 on the diagonal, -1 beside
 * it) and checks the residual. */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>

#include "amg_b200.h"

int main(int argc, char** argv) {
  const int n = argc > 1 ? atoi(argv[1]) : 10000;
  int* ia = malloc(sizeof(int) * (n + 1));
  int* ja = malloc(sizeof(int) * 3 * n);
  double* val = malloc(sizeof(double) * 3 * n);
  double* b = malloc(sizeof(double) * n);
  double* x = calloc(n, sizeof(double));
  int nnz = 0;
  for (int i = 0; i < n; i++) {
    ia[i] = nnz;
    if (i > 0) { ja[nnz] = i - 1; val[nnz++] = -1.0; }
    ja[nnz] = i; val[nnz++] = 2.5;
    if (i < n - 1) { ja[nnz] = i + 1; val[nnz++] = -1.0; }
    b[i] = 1.0;
  }
  ia[n] = nnz;
  void* h = amg_solver_create(n, nnz, ia, ja, val, 0.25, 500, 20, 1);
  if (!h) {
    fprintf(stderr, "create failed: %s\n", amg_solver_last_error());
    return 2;
  }
  const int it = amg_solver_solve(h, b, x, 1e-10, 500, 0);
  double r2 = 0.0, b2 = 0.0;
  for (int i = 0; i < n; i++) {
    double ax = 2.5 * x[i] - (i > 0 ? x[i - 1] : 0.0) - (i < n - 1 ? x[i + 1] : 0.0);
    r2 += (b[i] - ax) * (b[i] - ax);
    b2 += b[i] * b[i];
  }
  amg_solver_free(h);
  printf("n=%d iterations=%d relres=%.3e\n", n, it, sqrt(r2 / b2));
  free(ia); free(ja); free(val); free(b); free(x);
  return (it > 0 && sqrt(r2 / b2) < 1e-8) ? 0 : 1;
}
