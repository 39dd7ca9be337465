/*
 * x = cf_gauss_seidel_mex(A, b, x0, cf_order, nu, direction)
 * Gateway of the reference's Matlab_amg/cf_gauss_seidel_mex.c:27-105 on the
 * B200 library: same name, arguments (cf_order 1-based, direction 0 forward
 * / nonzero backward), error ids and output (x an n x 1 double).  A is
 * symmetric (CSC read as CSR).  The sweeps run on the device
 * (amg_gauss_seidel_ordered) and equal the sequential ones bit for bit.
 */
#include "bn_mex_util.h"

void mexFunction(int nlhs, mxArray* plhs[], int nrhs, const mxArray* prhs[]) {
  (void)nlhs;
  if (nrhs != 6)
    mexErrMsgIdAndTxt("cf_gs:nrhs", "Six inputs required: A, b, x, cf_order, nu, direction");
  if (!mxIsSparse(prhs[0])) mexErrMsgIdAndTxt("cf_gs:notSparse", "A must be sparse.");
  const size_t n = mxGetM(prhs[0]);
  const mwIndex* jc = mxGetJc(prhs[0]);
  int* ia = bn_mex_ints(jc, n + 1, "cf_gs:size");
  int* ja = bn_mex_ints(mxGetIr(prhs[0]), jc[n], "cf_gs:size");
  const double* b = mxGetPr(prhs[1]);
  const double* x0 = mxGetPr(prhs[2]);
  const double* ord = mxGetPr(prhs[3]);
  const int nu = (int)mxGetScalar(prhs[4]);
  const int backward = (int)mxGetScalar(prhs[5]);
  int* order = (int*)mxMalloc((n > 0 ? n : 1) * sizeof(int));
  for (size_t t = 0; t < n; t++) order[t] = (int)ord[t] - 1;  /* 1-based -> 0-based */
  plhs[0] = mxCreateDoubleMatrix(n, 1, mxREAL);
  double* x = mxGetPr(plhs[0]);
  memcpy(x, x0, n * sizeof(double));
  const int rc = amg_gauss_seidel_ordered((int)n, ia[n], ia, ja, mxGetPr(prhs[0]), b, x, order,
                                          nu, backward);
  mxFree(ia);
  mxFree(ja);
  mxFree(order);
  if (rc != AMG_OK) mexErrMsgIdAndTxt("cf_gs:device", "%s", amg_solver_last_error());
}
