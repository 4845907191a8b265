/*
 * MEX gateway over the imogen_b200 C ABI (include/imogen_b200.h).
 *
 * One mexFunction switching on a command string, the pattern of the reference's own MEX files
 * (gravity/utils/cudaCommon.cu:20-56), with the state resident on the device between calls:
 *
 *   h = imogen_b200_mex('create', grid, dgrid, gamma, cfl, minmass, bcinf, bcmodes, limiter,
 *                       fluid, magnet, timemax, itermax, updatemode, precision
 *                       [, visc, visclin, viscquad, rad, radexp, radmax, treadmill
 *                        [, fademask, fadelocation, fadesize]])
 *   imogen_b200_mex('set_state', h, mass, mom, ener, mag)     % FluidArray/MagnetArray setup
 *   imogen_b200_mex('upload', h, varid, array)                % X.array = ...
 *   a = imogen_b200_mex('download', h, varid)                 % X.array
 *   [dt, dir] = imogen_b200_mex('time_update', h, fluxdir)    % run.time.update(...)
 *   imogen_b200_mex('flux', h, order)                         % flux(run, ..., order)
 *   imogen_b200_mex('step', h)                                % one imogen.m loop body
 *   [t, dt, iter] = imogen_b200_mex('time', h)
 *   imogen_b200_mex('source', h)                              % source(run, ...) (radiation)
 *   imogen_b200_mex('treadmill', h)                           % treadmillGrid(run, ...)
 *   imogen_b200_mex('save_slice', h, path, type, index, suffix)   % resultsHandler slice file
 *   imogen_b200_mex('load_slice', h, path)                    % resume from a slice file
 *   imogen_b200_mex('destroy', h)
 *
 * The job server (its handle is a uint64 scalar too):
 *
 *   s = imogen_b200_mex('server_create', budget_bytes, check_every, keep)
 *   id = imogen_b200_mex('submit', s, <the 14 or 21 create arguments>, mass, mom, ener, mag)
 *   [status, t, iter] = imogen_b200_mex('poll', s, id)        % IMG_JOB_* status
 *   imogen_b200_mex('cancel', s, id)
 *   a = imogen_b200_mex('result', s, id, varid, like)         % varid -1: the 8 totals
 *   imogen_b200_mex('server_destroy', s)
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

/* img_config from the create arguments prhs[0..n-1] (n = 14, 21 with the physics settings, 24 with a
 * point fade as well). */
static void read_config(img_config* c, const mxArray* const* a, int n) {
    const double *grid, *dg, *bc, *lim;
    int i, k, s, d;
    img_config_default(c);
    grid = mxGetPr(a[0]);
    dg = mxGetPr(a[1]);
    for (i = 0; i < 3; ++i) { c->grid[i] = (int)grid[i]; c->dgrid[i] = dg[i]; }
    c->gamma = scalar(a[2]);
    c->cfl = scalar(a[3]);
    c->minmass = scalar(a[4]);
    c->bc_infinity = (int)scalar(a[5]);
    bc = mxGetPr(a[6]);   /* MATLAB column-major 4x2x3 */
    for (k = 0; k < 4; ++k)
        for (s = 0; s < 2; ++s)
            for (d = 0; d < 3; ++d) c->bc_modes[k][s][d] = (int)bc[k + 4 * (s + 2 * d)];
    lim = mxGetPr(a[7]);
    for (i = 0; i < 3; ++i) c->limiter[i] = (int)lim[i];
    c->fluid_active = (int)scalar(a[8]);
    c->magnet_active = (int)scalar(a[9]);
    c->time_max = scalar(a[10]);
    c->iter_max = (int)scalar(a[11]);
    c->update_mode = (int)scalar(a[12]);
    c->precision = (int)scalar(a[13]);
    if (n >= 21) {   /* run.viscosity, run.radiation, ini.treadmill */
        c->viscosity_type = (int)scalar(a[14]);
        c->visc_linear = scalar(a[15]);
        c->visc_quadratic = scalar(a[16]);
        c->radiation_type = (int)scalar(a[17]);
        c->rad_exponent = scalar(a[18]);
        c->rad_initial_maximum = scalar(a[19]);
        c->treadmill = (int)scalar(a[20]);
    }
    if (n == 24) {   /* ini.fades with one point fade: IMG_FADE_* mask, 1-based location, radius */
        const double* loc = mxGetPr(a[22]);
        c->fade_active = (int)scalar(a[21]);
        for (i = 0; i < 3; ++i) c->fade_location[i] = (int)loc[i];
        c->fade_size = scalar(a[23]);
    }
}

static void* ptr(const mxArray* a) {
    if (!mxIsUint64(a) || mxGetNumberOfElements(a) != 1) mexErrMsgIdAndTxt("imogen_b200:arg", "bad handle");
    return (void*)(uintptr_t)(*(uint64_t*)mxGetData(a));
}

static mxArray* handle_out(void* p) {
    mxArray* h = mxCreateNumericMatrix(1, 1, mxUINT64_CLASS, mxREAL);
    *(uint64_t*)mxGetData(h) = (uint64_t)(uintptr_t)p;
    return h;
}

/* The job server's commands; returns 0 when cmd is not one of them. */
static int server_command(const char* cmd, int nlhs, mxArray* plhs[], int nrhs, const mxArray* prhs[]) {
    char id[64];
    int rc = IMG_OK;
    if (!strcmp(cmd, "server_create")) {
        img_server* srv = NULL;
        if (nrhs != 4) mexErrMsgIdAndTxt("imogen_b200:arg", "server_create(budget, check_every, keep)");
        rc = img_server_create(&srv, (size_t)scalar(prhs[1]), (int)scalar(prhs[2]), (int)scalar(prhs[3]));
        if (rc == IMG_OK) plhs[0] = handle_out(srv);
    } else if (!strcmp(cmd, "server_destroy")) {
        rc = img_server_destroy((img_server*)ptr(prhs[1]));
    } else if (!strcmp(cmd, "submit")) {
        img_config c;
        int job = -1, ncfg = nrhs - 6;
        if (ncfg != 14 && ncfg != 21 && ncfg != 24) mexErrMsgIdAndTxt("imogen_b200:arg", "submit(s, <create arguments>, mass, mom, ener, mag)");
        read_config(&c, prhs + 2, ncfg);
        rc = img_batch_submit((img_server*)ptr(prhs[1]), &c, mxGetPr(prhs[nrhs - 4]), mxGetPr(prhs[nrhs - 3]),
                              mxGetPr(prhs[nrhs - 2]), mxGetPr(prhs[nrhs - 1]), &job);
        if (rc == IMG_OK) plhs[0] = mxCreateDoubleScalar(job);
    } else if (!strcmp(cmd, "poll")) {
        img_job_info info;
        rc = img_batch_poll((img_server*)ptr(prhs[1]), (int)scalar(prhs[2]), &info);
        if (rc == IMG_OK) {
            plhs[0] = mxCreateDoubleScalar(info.status);
            if (nlhs > 1) plhs[1] = mxCreateDoubleScalar(info.time);
            if (nlhs > 2) plhs[2] = mxCreateDoubleScalar(info.iterations);
            if (nlhs > 3) plhs[3] = mxCreateString(info.error);
        }
    } else if (!strcmp(cmd, "cancel")) {
        rc = img_batch_cancel((img_server*)ptr(prhs[1]), (int)scalar(prhs[2]));
    } else if (!strcmp(cmd, "result")) {
        const mwSize* dims;
        int var;
        if (nrhs != 5) mexErrMsgIdAndTxt("imogen_b200:arg", "result(s, id, varid, like)");
        var = (int)scalar(prhs[3]);
        if (var == IMG_RESULT_TOTALS) {
            plhs[0] = mxCreateNumericMatrix(1, 8, mxDOUBLE_CLASS, mxREAL);
        } else {
            dims = mxGetDimensions(prhs[4]);
            plhs[0] = mxCreateNumericArray(mxGetNumberOfDimensions(prhs[4]), dims, mxDOUBLE_CLASS, mxREAL);
        }
        rc = img_batch_result((img_server*)ptr(prhs[1]), (int)scalar(prhs[2]), var, mxGetPr(plhs[0]),
                              mxGetNumberOfElements(plhs[0]));
    } else {
        return 0;
    }
    if (rc != IMG_OK) {
        sprintf(id, "imogen_b200:e%d", -rc);
        mexErrMsgIdAndTxt(id, "job server call failed (status %d)", rc);
    }
    return 1;
}

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
        if (nrhs != 15 && nrhs != 22 && nrhs != 25) mexErrMsgIdAndTxt("imogen_b200:arg", "create takes 14, 21 or 24 arguments");
        read_config(&c, prhs + 1, nrhs - 1);
        check(img_create(&ctx, &c), NULL);
        plhs[0] = handle_out(ctx);
        return;
    }
    if (nrhs >= 2 && server_command(cmd, nlhs, plhs, nrhs, prhs)) return;
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
        } else if (!strcmp(cmd, "source")) {
            check(img_source(ctx), ctx);
        } else if (!strcmp(cmd, "treadmill")) {
            check(img_treadmill(ctx), ctx);
        } else if (!strcmp(cmd, "save_slice")) {
            img_slice_meta m;
            char path[1024], suffix[64];
            const double* ix;
            int i;
            if (nrhs != 7) mexErrMsgIdAndTxt("imogen_b200:arg", "save_slice(h, path, type, index, suffix)");
            memset(&m, 0, sizeof m);
            mxGetString(prhs[2], path, sizeof path);
            m.type = (int)scalar(prhs[3]);
            ix = mxGetPr(prhs[4]);
            for (i = 0; i < 3; ++i) m.index[i] = (int)ix[i];
            mxGetString(prhs[5], suffix, sizeof suffix);
            m.suffix = suffix;
            m.wall_max = 1e5;
            check(img_save_slice(ctx, path, &m), ctx);
        } else if (!strcmp(cmd, "load_slice")) {
            char path[1024];
            if (nrhs != 3) mexErrMsgIdAndTxt("imogen_b200:arg", "load_slice(h, path)");
            mxGetString(prhs[2], path, sizeof path);
            check(img_load_slice(ctx, path), ctx);
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
