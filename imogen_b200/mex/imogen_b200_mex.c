/*
 * MEX gateway over the imogen_b200 C ABI (include/imogen_b200.h).
 *
 * One mexFunction switching on a command string, the pattern of the reference's own MEX files
 * (gravity/utils/cudaCommon.cu:20-56), with the state resident on the device between calls:
 *
 *   h = imogen_b200_mex('create', grid, dgrid, gamma, cfl, minmass, bcinf, bcmodes, limiter,
 *                       fluid, magnet, timemax, itermax, updatemode, precision)
 *   imogen_b200_mex('set_state', h, mass, mom, ener, mag)     % FluidArray/MagnetArray setup
 *   imogen_b200_mex('upload', h, varid, array)                % X.array = ...
 *   a = imogen_b200_mex('download', h, varid)                 % X.array
 *   [dt, dir] = imogen_b200_mex('time_update', h, fluxdir)    % run.time.update(...)
 *   imogen_b200_mex('flux', h, order)                         % flux(run, ..., order)
 *   imogen_b200_mex('step', h)                                % one imogen.m loop body
 *   [t, dt, iter] = imogen_b200_mex('time', h)
 *   imogen_b200_mex('destroy', h)
 *
 * bcmodes is a 4x2x3 double array [class (mass, mom, ener, mag)][side][dim] of IMG_BC_* codes.
 * Errors map to mexErrMsgIdAndTxt('imogen_b200:<code>', img_last_error(ctx)).  The handle is the
 * context pointer carried in a uint64 scalar.
 */
#include <stdint.h>
#include <string.h>

#include "mex.h"
#include "imogen_b200.h"

static img_ctx* handle(const mxArray* a) {
    if (!mxIsUint64(a) || mxGetNumberOfElements(a) != 1) mexErrMsgIdAndTxt("imogen_b200:arg", "bad handle");
    return (img_ctx*)(uintptr_t)(*(uint64_t*)mxGetData(a));
}

static void check(int rc, img_ctx* ctx) {
    char id[64];
    if (rc == IMG_OK) return;
    sprintf(id, "imogen_b200:e%d", -rc);
    mexErrMsgIdAndTxt(id, "%s", img_last_error(ctx));
}

static double scalar(const mxArray* a) { return mxGetScalar(a); }

static size_t ncell(img_ctx* ctx, const mxArray* a) {
    (void)ctx;
    if (!mxIsDouble(a) || mxIsComplex(a)) mexErrMsgIdAndTxt("imogen_b200:arg", "arrays must be real double");
    return mxGetNumberOfElements(a);
}

void mexFunction(int nlhs, mxArray* plhs[], int nrhs, const mxArray* prhs[]) {
    char cmd[32];
    if (nrhs < 1 || mxGetString(prhs[0], cmd, sizeof cmd) != 0) mexErrMsgIdAndTxt("imogen_b200:arg", "command string expected");

    if (!strcmp(cmd, "create")) {
        img_config c;
        img_ctx* ctx = NULL;
        const double *grid, *dg, *bc, *lim;
        int i, k, s, d;
        if (nrhs != 15) mexErrMsgIdAndTxt("imogen_b200:arg", "create takes 14 arguments");
        img_config_default(&c);
        grid = mxGetPr(prhs[1]);
        dg = mxGetPr(prhs[2]);
        for (i = 0; i < 3; ++i) { c.grid[i] = (int)grid[i]; c.dgrid[i] = dg[i]; }
        c.gamma = scalar(prhs[3]);
        c.cfl = scalar(prhs[4]);
        c.minmass = scalar(prhs[5]);
        c.bc_infinity = (int)scalar(prhs[6]);
        bc = mxGetPr(prhs[7]);   /* MATLAB column-major 4x2x3 */
        for (k = 0; k < 4; ++k)
            for (s = 0; s < 2; ++s)
                for (d = 0; d < 3; ++d) c.bc_modes[k][s][d] = (int)bc[k + 4 * (s + 2 * d)];
        lim = mxGetPr(prhs[8]);
        for (i = 0; i < 3; ++i) c.limiter[i] = (int)lim[i];
        c.fluid_active = (int)scalar(prhs[9]);
        c.magnet_active = (int)scalar(prhs[10]);
        c.time_max = scalar(prhs[11]);
        c.iter_max = (int)scalar(prhs[12]);
        c.update_mode = (int)scalar(prhs[13]);
        c.precision = (int)scalar(prhs[14]);
        check(img_create(&ctx, &c), NULL);
        plhs[0] = mxCreateNumericMatrix(1, 1, mxUINT64_CLASS, mxREAL);
        *(uint64_t*)mxGetData(plhs[0]) = (uint64_t)(uintptr_t)ctx;
        return;
    }
    if (nrhs < 2) mexErrMsgIdAndTxt("imogen_b200:arg", "handle expected");
    {
        img_ctx* ctx = handle(prhs[1]);
        if (!strcmp(cmd, "destroy")) {
            check(img_destroy(ctx), NULL);
        } else if (!strcmp(cmd, "set_state")) {
            if (nrhs != 6) mexErrMsgIdAndTxt("imogen_b200:arg", "set_state(h, mass, mom, ener, mag)");
            check(img_set_state(ctx, mxGetPr(prhs[2]), mxGetPr(prhs[3]), mxGetPr(prhs[4]), mxGetPr(prhs[5])), ctx);
        } else if (!strcmp(cmd, "upload")) {
            if (nrhs != 4) mexErrMsgIdAndTxt("imogen_b200:arg", "upload(h, varid, array)");
            check(img_upload(ctx, (int)scalar(prhs[2]), mxGetPr(prhs[3]), ncell(ctx, prhs[3])), ctx);
        } else if (!strcmp(cmd, "download")) {
            const mwSize* dims;
            mwSize nd;
            if (nrhs != 4) mexErrMsgIdAndTxt("imogen_b200:arg", "download(h, varid, like) with an array of the grid's shape");
            dims = mxGetDimensions(prhs[3]);
            nd = mxGetNumberOfDimensions(prhs[3]);
            plhs[0] = mxCreateNumericArray(nd, dims, mxDOUBLE_CLASS, mxREAL);
            check(img_download(ctx, (int)scalar(prhs[2]), mxGetPr(plhs[0]), mxGetNumberOfElements(plhs[0])), ctx);
        } else if (!strcmp(cmd, "time_update")) {
            double dt = 0;
            int dir = 0;
            check(img_time_update(ctx, (int)scalar(prhs[2]), &dt, &dir), ctx);
            plhs[0] = mxCreateDoubleScalar(dt);
            if (nlhs > 1) plhs[1] = mxCreateDoubleScalar(dir);
        } else if (!strcmp(cmd, "flux")) {
            check(img_flux(ctx, (int)scalar(prhs[2])), ctx);
        } else if (!strcmp(cmd, "step")) {
            check(img_step(ctx), ctx);
        } else if (!strcmp(cmd, "time")) {
            double t = 0, dt = 0;
            int it = 0;
            check(img_get_time(ctx, &t, &dt, &it), ctx);
            plhs[0] = mxCreateDoubleScalar(t);
            if (nlhs > 1) plhs[1] = mxCreateDoubleScalar(dt);
            if (nlhs > 2) plhs[2] = mxCreateDoubleScalar(it);
        } else {
            mexErrMsgIdAndTxt("imogen_b200:arg", "unknown command");
        }
    }
}
