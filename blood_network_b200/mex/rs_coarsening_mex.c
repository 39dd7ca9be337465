/*
 * [cf, nc] = rs_coarsening_mex(S, lam_max)
 * Gateway of the reference's Matlab_amg/rs_coarsening_mex.c:24-189 on the
 * B200 library: same name, arguments (lam_max an int32 scalar), error ids
 * and outputs (cf an n x 1 double of +1 for C / -1 for F points, nc a double
 * scalar).  The split comes from the device rs_coarsening (rs_classical.c:
 * 108-229), whose first pass runs in parallel: a valid Ruge-Stuben split
 * (every F point has a strong C neighbour), not necessarily the sequential
 * bucket order's.
 */
#include "bn_mex_util.h"

void mexFunction(int nlhs, mxArray* plhs[], int nrhs, const mxArray* prhs[]) {
  if (nrhs != 2) mexErrMsgIdAndTxt("rs_coarsen:nrhs", "Two inputs required: S, lam_max");
  if (!mxIsSparse(prhs[0])) mexErrMsgIdAndTxt("rs_coarsen:notSparse", "S must be sparse.");
  if (!mxIsInt32(prhs[1]) || mxGetNumberOfElements(prhs[1]) != 1)
    mexErrMsgIdAndTxt("rs_coarsen:badLamMax", "lam_max must be a scalar int32.");
  const int lam_max = *(const int*)mxGetData(prhs[1]);
  const size_t n = mxGetM(prhs[0]);
  int *ia, *ja;
  bn_mex_csc_to_csr(n, mxGetN(prhs[0]), mxGetJc(prhs[0]), mxGetIr(prhs[0]), &ia, &ja);
  double* val = (double*)mxCalloc(ia[n] > 0 ? (size_t)ia[n] : 1, sizeof(double));
  dcsr_mat S = {(int)n, (int)n, ia[n], ia, ja, val};
  int* cf = (int*)mxCalloc(n > 0 ? n : 1, sizeof(int));
  int nc = 0;
  rs_coarsening(&S, lam_max, cf, &nc);
  mxFree(ia);
  mxFree(ja);
  mxFree(val);
  bn_mex_check("rs_coarsen:device");
  plhs[0] = mxCreateDoubleMatrix(n, 1, mxREAL);
  double* out = mxGetPr(plhs[0]);
  for (size_t i = 0; i < n; i++) out[i] = (double)cf[i];
  mxFree(cf);
  if (nlhs > 1) plhs[1] = mxCreateDoubleScalar((double)nc);
}
