/*
 * MCcov_mex.c - MEX shim: [Ms, Mm] = MCcov(sigt, albedo, box_min, box_max, l,
 *     v, is_ff_l, is_ff_v, maxItr, lambda, doCBS, smpFlg, sct_type, ampfunc
 *     [, ampfunc0])                                                (MCcov.m:1)
 * on the GPU through scmc_cov (include/scmc_gpu.h).  Ms and Mm are
 * Nv x Nv x Nl x Nl complex, index (v1, v2, l1, l2) as the reference's.
 * Built as MCcov.mexa64 next to code/MCcov.m, it serves the unchanged scmc.m
 * (scmc.m:332-367, parfor workers included: each loads the MEX in its own
 * process and draws its own key from its own stream).
 *
 *     mex -R2018a mex/MCcov_mex.c -I include -I mex -L mcspeckle_b200 -lscmc_gpu -output MCcov
 */
#include "scmc_mex.h"

void mexFunction(int nlhs, mxArray *plhs[], int nrhs, const mxArray *prhs[])
{
    scmc_mex_nargin(nrhs, 14, 15); /* MCcov.m:45 */
    scmc_mex_scratch s = {{0}, 0};
    scmc_mc_args a;
    scmc_mex_mc_args(nrhs, prhs, &a, &s);
    const mwSize dims[4] = {(mwSize)a.nv, (mwSize)a.nv, (mwSize)a.nl, (mwSize)a.nl};
    plhs[0] = mxCreateNumericArray(4, dims, mxDOUBLE_CLASS, mxCOMPLEX);
    plhs[1] = mxCreateNumericArray(4, dims, mxDOUBLE_CLASS, mxCOMPLEX);
    /* a caller that asked for Ms only skips copying Mm back */
    double *mm = nlhs >= 2 ? (double *)mxGetComplexDoubles(plhs[1]) : NULL;
    scmc_mex_check(scmc_cov(&a, (double *)mxGetComplexDoubles(plhs[0]), mm), &s);
    scmc_mex_release(&s);
}
