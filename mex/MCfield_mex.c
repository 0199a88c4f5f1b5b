/*
 * MCfield_mex.c - MEX shim: u = MCfield(sigt, albedo, box_min, box_max, l, v,
 *     is_ff_l, is_ff_v, maxItr, lambda, doCBS, smpFlg, sct_type, ampfunc
 *     [, ampfunc0 [, lmean0]])                                   (MCfield.m:1)
 * on the GPU through scmc_field (include/scmc_gpu.h).  Built as MCfield.mexa64
 * next to code/MCfield.m, MATLAB calls it in place of the .m file, so the
 * unchanged scmc.m (scmc.m:387-423) renders fields on the GPU.
 *
 *     mex -R2018a mex/MCfield_mex.c -I include -I mex -L mcspeckle_b200 -lscmc_gpu -output MCfield
 */
#include "scmc_mex.h"

void mexFunction(int nlhs, mxArray *plhs[], int nrhs, const mxArray *prhs[])
{
    (void)nlhs;
    scmc_mex_nargin(nrhs, 14, 16); /* MCfield.m:41 */
    scmc_mex_scratch s = {{0}, 0};
    scmc_mc_args a;
    scmc_mex_mc_args(nrhs, prhs, &a, &s);
    plhs[0] = mxCreateNumericMatrix((mwSize)a.nv, (mwSize)a.nl, mxDOUBLE_CLASS, mxCOMPLEX);
    scmc_mex_check(scmc_field(&a, (double *)mxGetComplexDoubles(plhs[0])), &s);
    scmc_mex_release(&s);
}
