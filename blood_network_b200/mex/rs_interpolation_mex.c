/*
 * P = rs_interpolation_mex(A, S, cf)
 * Gateway of the reference's Matlab_amg/rs_interpolation_mex.c:29-238 on
 * the B200 library: same name, arguments (cf a double vector of +1 / -1),
 * error ids and output (P an n x nc sparse double).  A is symmetric (CSC
 * read as CSR); S arrives as MATLAB stores it (CSC) and is turned into CSR.
 * P is the device rs_standard_interpolation (rs_classical.c:643-805), the
 * direct interpolation the reference gateway also computes.
 */
#include "bn_mex_util.h"

void mexFunction(int nlhs, mxArray* plhs[], int nrhs, const mxArray* prhs[]) {
  (void)nlhs;
  if (nrhs != 3) mexErrMsgIdAndTxt("rs_interp:nrhs", "Three inputs required: A, S, cf");
  if (!mxIsSparse(prhs[0])) mexErrMsgIdAndTxt("rs_interp:A", "A must be sparse.");
  if (!mxIsSparse(prhs[1])) mexErrMsgIdAndTxt("rs_interp:S", "S must be sparse.");
  const size_t n = mxGetM(prhs[0]);
  const mwIndex* ajc = mxGetJc(prhs[0]);
  int* aia = bn_mex_ints(ajc, n + 1, "rs_interp:size");
  int* aja = bn_mex_ints(mxGetIr(prhs[0]), ajc[n], "rs_interp:size");
  dcsr_mat A = {(int)n, (int)n, aia[n], aia, aja, mxGetPr(prhs[0])};
  int *sia, *sja;
  bn_mex_csc_to_csr(n, mxGetN(prhs[1]), mxGetJc(prhs[1]), mxGetIr(prhs[1]), &sia, &sja);
  double* sval = (double*)mxCalloc(sia[n] > 0 ? (size_t)sia[n] : 1, sizeof(double));
  dcsr_mat S = {(int)n, (int)n, sia[n], sia, sja, sval};
  const double* cfd = mxGetPr(prhs[2]);
  int* cf = (int*)mxMalloc((n > 0 ? n : 1) * sizeof(int));
  for (size_t i = 0; i < n; i++) cf[i] = (int)cfd[i];
  dcsr_mat P;
  memset(&P, 0, sizeof(P));
  rs_standard_interpolation(&A, &S, cf, &P);
  mxFree(aia);
  mxFree(aja);
  mxFree(sia);
  mxFree(sja);
  mxFree(sval);
  mxFree(cf);
  bn_mex_check("rs_interp:device");
  plhs[0] = bn_mex_sparse_from_csr(n, (size_t)P.col, P.ia, P.ja, P.val);
  free(P.ia);
  free(P.ja);
  free(P.val);
}
