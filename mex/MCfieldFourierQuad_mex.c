/*
 * MCfieldFourierQuad_mex.c - MEX shim: u = MCfieldFourierQuad(sigt, albedo,
 *     box_min, box_max, l, v_max, v_stp, maxItr, lambda, doCBS, smpFlg
 *     [, lmean0 [, vsign]])                          (MCfieldFourierQuad.m:1)
 * on the GPU through scmc_field_fourier_quad (include/scmc_gpu.h).  u is
 * Nv0 x Nv0 x Nl complex on the angular grid -v_max:v_stp:v_max.  lmean0 may
 * be [] (then +z, lines 59-64); vsign defaults to -1 (line 66).  The box is
 * 3-D and l holds 3 x Nl light directions, as the reference assumes.
 *
 *     mex -R2018a mex/MCfieldFourierQuad_mex.c -I include -I mex -L mcspeckle_b200 -lscmc_gpu \
 *         -output MCfieldFourierQuad
 */
#include "scmc_mex.h"

void mexFunction(int nlhs, mxArray *plhs[], int nrhs, const mxArray *prhs[])
{
    (void)nlhs;
    scmc_mex_nargin(nrhs, 11, 13);
    scmc_mex_scratch s = {{0}, 0};
    scmc_fq_args a;
    memset(&a, 0, sizeof a);
    if (scmc_mex_box(prhs[2], prhs[3], a.box_min, a.box_max, &s) != 3)
        scmc_mex_fail(&s, "scmc:gpu:box", "Invalid box size");
    a.sigt = mxGetScalar(prhs[0]);
    a.albedo = mxGetScalar(prhs[1]);
    if (mxGetM(prhs[4]) != 3) scmc_mex_fail(&s, "scmc:gpu:source", "Invalid light source input");
    /* l is 3 x Nl column-major: the [nl][3] rows the ABI takes */
    a.l = mxGetDoubles(prhs[4]);
    a.nl = (int64_t)mxGetN(prhs[4]);
    a.v_max = mxGetScalar(prhs[5]);
    a.v_stp = mxGetScalar(prhs[6]);
    a.max_itr = (int64_t)mxGetScalar(prhs[7]);
    a.lambda = mxGetScalar(prhs[8]);
    a.do_cbs = mxGetScalar(prhs[9]) != 0.0;
    a.smp_flg = (int32_t)mxGetScalar(prhs[10]);
    if (nrhs >= 12 && !mxIsEmpty(prhs[11])) {
        if (mxGetNumberOfElements(prhs[11]) != 3) scmc_mex_fail(&s, "scmc:gpu:lmean0", "lmean0 must be 3 x 1");
        a.has_lmean0 = 1;
        memcpy(a.lmean0, mxGetDoubles(prhs[11]), 3 * sizeof(double));
    }
    a.vsign = nrhs >= 13 ? mxGetScalar(prhs[12]) : -1.0;
    a.seed = scmc_mex_seed();
    a.precision = scmc_mex_precision();
    a.device = scmc_mex_device();
    int64_t nv0 = 0;
    scmc_mex_check(scmc_fq_grid_size(a.v_max, a.v_stp, &nv0), &s);
    const mwSize dims[3] = {(mwSize)nv0, (mwSize)nv0, (mwSize)a.nl};
    plhs[0] = mxCreateNumericArray(3, dims, mxDOUBLE_CLASS, mxCOMPLEX);
    scmc_mex_check(scmc_field_fourier_quad(&a, (double *)mxGetComplexDoubles(plhs[0])), &s);
    scmc_mex_release(&s);
}
