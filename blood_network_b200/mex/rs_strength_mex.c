/*
 * [S, lam_max] = rs_strength_mex(A, theta)
 * Gateway of the reference's Matlab_amg/rs_strength_mex.c:28-124 on the B200
 * library: same name, arguments, error ids and output classes (S sparse
 * double, lam_max int32).  A must be symmetric (its CSC arrays are read as
 * its CSR arrays, as the reference does).  S(i,j) != 0 when i depends
 * strongly on j: -a_ij >= theta * max_{k != i} (-a_ik), computed by the
 * device rs_strength (rs_classical.c:30-88).  The reference gateway also
 * keeps a row's non-negative off-diagonal entries when that row has no
 * negative one (max is 0); the C routine, used here, does not.  Graph
 * Laplacians have no such rows.
 */
#include "bn_mex_util.h"

void mexFunction(int nlhs, mxArray* plhs[], int nrhs, const mxArray* prhs[]) {
  if (nrhs != 2) mexErrMsgIdAndTxt("rs_str:nrhs", "Two inputs required: A, theta");
  if (!mxIsSparse(prhs[0])) mexErrMsgIdAndTxt("rs_str:notSparse", "A must be sparse.");
  const size_t n = mxGetM(prhs[0]);
  const mwIndex* jc = mxGetJc(prhs[0]);
  const double theta = mxGetScalar(prhs[1]);
  int* ia = bn_mex_ints(jc, n + 1, "rs_str:size");
  int* ja = bn_mex_ints(mxGetIr(prhs[0]), jc[n], "rs_str:size");
  dcsr_mat A = {(int)n, (int)n, ia[n], ia, ja, mxGetPr(prhs[0])};
  dcsr_mat S;
  int max_lam = 0;
  rs_strength(&A, theta, &S, &max_lam);
  mxFree(ia);
  mxFree(ja);
  bn_mex_check("rs_str:device");
  plhs[0] = bn_mex_sparse_from_csr(n, n, S.ia, S.ja, S.val);
  if (nlhs > 1) {
    plhs[1] = mxCreateNumericMatrix(1, 1, mxINT32_CLASS, mxREAL);
    *(int*)mxGetData(plhs[1]) = max_lam;
  }
  free(S.ia);
  free(S.ja);
  free(S.val);
}
