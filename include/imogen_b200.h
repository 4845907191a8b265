/*
 * imogen_b200 -- C ABI of the B200 relaxing-TVD fluid + magnet update.
 *
 * Plain C: opaque context handles, host pointers and sizes, int status codes.  No exception or
 * C++/torch type crosses this boundary.  Every entry point replaces one piece of the reference's
 * MATLAB call surface (paths are relative to the reference project root).
 *
 * Threading: a context is used by one host thread at a time.  All work of a context is issued on
 * its own CUDA stream; state stays resident on the device between calls.
 */
#ifndef IMOGEN_B200_H
#define IMOGEN_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes --------------------------------------------------------------------------- */
enum {
    IMG_OK = 0,
    IMG_ERR_ARG = -1,          /* invalid argument (message in img_last_error) */
    IMG_ERR_CUDA = -2,         /* CUDA runtime error */
    IMG_ERR_NOMEM = -3,        /* device allocation failed / over the HBM budget */
    IMG_ERR_UNSUPPORTED = -4,  /* setting that the reference itself cannot run (index error) */
    IMG_ERR_CFL = -5,          /* TimeManager.m:79-86: no direction exceeded the 1e-2 floor */
    IMG_ERR_NONFINITE = -6,    /* the timestep or (with nonfinite_check) the state became non-finite */
    IMG_ERR_STATE = -7         /* call out of order (e.g. step before state was set) */
};

/* ---- enumerations (enums/ENUM.m, enums/FluxLimiterEnum.m) ----------------------------------- */
enum { IMG_BC_CIRC = 0, IMG_BC_CONST = 1, IMG_BC_FADE = 2, IMG_BC_MIRROR = 3, IMG_BC_TRANS = 4, IMG_BC_WALL = 5,
       IMG_BC_FLIP = 6, IMG_BC_ZERO = 7, IMG_BC_LINEAR = 8, IMG_BC_WORMHOLE = 9 };
/* linear: rejected (IMG_ERR_UNSUPPORTED) -- linear_shift.m:20 indexes with an undefined variable, so the
 * reference stops at the first shift.  wormhole: the upper side is the constant shift (as in
 * wormhole_shift.m); a lower wormhole side couples pencils across the grid and is rejected
 * (IMG_ERR_UNSUPPORTED), as it is in 2-D by the reference itself. */
enum { IMG_LIM_VANLEER = 0, IMG_LIM_SUPERBEE = 1, IMG_LIM_MINMOD = 2 };
enum { IMG_CLS_MASS = 0, IMG_CLS_MOM = 1, IMG_CLS_ENER = 2, IMG_CLS_MAG = 3 };
enum { IMG_PREC_FP64 = 0, IMG_PREC_MIXED = 1 };
/* PointFade activeList entries (ImogenManager.addFades, classes/ImogenManager.m:262-280): only the
 * FluidArray primaries read fades (FluidArray.m:54), so MAG and GRAV are accepted and have no effect */
enum { IMG_FADE_MASS = 1, IMG_FADE_MOM = 2, IMG_FADE_ENER = 4, IMG_FADE_MAG = 8, IMG_FADE_GRAV = 16 };
/* ArtificialViscosity.type (fluid/ArtificialViscosity.m:45-56) and Radiation.type (fluid/Radiation.m:43-55) */
enum { IMG_VISC_NONE = 0, IMG_VISC_NEUMANN_RICHTMYER = 1, IMG_VISC_CARAMANA_SHASHKOV_WHALEN = 2 };
enum { IMG_RAD_NONE = 0, IMG_RAD_OPTICALLY_THIN = 1 };
/* variable ids for upload/download: rho, momentum x/y/z, energy, face-centred B x/y/z, and the
 * cell-centred B x/y/z (MagnetArray.cellMag, download only) */
enum {
    IMG_VAR_MASS = 0, IMG_VAR_MOMX = 1, IMG_VAR_MOMY = 2, IMG_VAR_MOMZ = 3, IMG_VAR_ENER = 4,
    IMG_VAR_MAGX = 5, IMG_VAR_MAGY = 6, IMG_VAR_MAGZ = 7,
    IMG_VAR_CMAGX = 8, IMG_VAR_CMAGY = 9, IMG_VAR_CMAGZ = 10
};

/* Run settings: the subset of the ini structure that initialize.m parses for this path
 * (initialize.m:24-190; defaults of experiment/Initializer.m:73-184). */
typedef struct img_config {
    int grid[3];              /* ini.grid (nx, ny, nz); nz == 1 gives a 2-D run */
    double dgrid[3];          /* ini.dGrid, uniform spacing per dimension (MINDGRID = dgrid) */
    double gamma;             /* ini.gamma */
    double cfl;               /* ini.cfl */
    double minmass;           /* ini.minMass */
    int bc_infinity;          /* ini.bcInfinity (trans extrapolation distance, fade width) */
    int bc_modes[4][2][3];    /* [class: mass, mom, ener, mag][side: lower, upper][dim] */
    int limiter[3];           /* ini.fluxLimiter.{x,y,z}; the magnet uses the same table */
    int fluid_active;         /* ini.mode.fluid */
    int magnet_active;        /* ini.mode.magnet */
    double time_max;          /* ini.timeMax */
    int iter_max;             /* ini.iterMax */
    int update_mode;          /* ini.timeUpdateMode: 0 per step, 1 per iteration */
    int precision;            /* IMG_PREC_FP64 (plain) or IMG_PREC_MIXED (FP32 state, FP64 pressure/CFL) */
    int nonfinite_check;      /* 1 (default): a CFL pass that meets a non-finite rho, momentum, energy or
                                 B stops the run with IMG_ERR_NONFINITE.  0: the reference's behaviour
                                 (its max ignores NaN, TimeManager.m:70-76; MINMASS replaces a NaN
                                 density, relaxingFluid.m:39,71) and the run goes on.  No reference
                                 counterpart. */
    /* run.viscosity (fluid/ArtificialViscosity.m:31-37): type, linear and quadratic strengths.  A
     * viscosity other than IMG_VISC_NONE needs circ or const ends on every dimension (the same mode
     * for mass, momentum, energy and B on each side) and pencils that fit one thread block (along x
     * N / C threads with C = 2 or 4 cells per thread a power of two up to 32 or a multiple of 32;
     * N / C <= 512 along every dimension); img_create returns IMG_ERR_UNSUPPORTED otherwise, and
     * such contexts do not join batches. */
    int viscosity_type;
    double visc_linear;
    double visc_quadratic;
    /* run.radiation (fluid/Radiation.m:32-37): type, exponent and initialMaximum (percent); the
     * strength is set from the state by img_set_state (Radiation.initialize).  Contexts with
     * radiation do not join batches. */
    int radiation_type;
    double rad_exponent;
    double rad_initial_maximum;
    /* ini.treadmill (initialize.m:328-331): 0 off, else the direction (1-3) along which treadmillGrid
     * keeps the steepest density rise in place (treadmill/treadmillGrid.m).  Pencils along it are
     * staged whole in shared memory (2 N values must fit one block); contexts with a treadmill take no
     * CUDA graph and do not join batches. */
    int treadmill;
    /* ini.fades (initialize.m:336-341) with one point fade (the reference's addFades takes one):
     * IMG_FADE_* mask of the arrays it acts on (0: none), its 1-based cell location and its radius in
     * cells.  Every assignment to a faded primary -- the sweeps' updates, relaxingFluid's MINMASS clamp,
     * the radiation sink, the treadmill's shift, img_upload / img_upload_many -- multiplies it by
     * 1 - 0.05 A, A the PointFade map (classes/PointFade.m:29-49).  Contexts with a fade do not join
     * batches. */
    int fade_active;
    int fade_location[3];
    double fade_size;
} img_config;

typedef struct img_ctx img_ctx;

/* Default config: Initializer.m defaults (gamma 5/3, cfl 0.7, minMass 1e-5, circ BCs,
 * bcInfinity 20, vanleer, fluid on, magnet off, timeMax 1e5, iterMax 10, per-iteration dt, no
 * viscosity (strengths 0), no radiation (exponent 0.5, initialMaximum 0)), plus nonfinite_check = 1. */
void img_config_default(img_config* cfg);

/* Create a context for one grid on the current CUDA device.  Replaces initialize.m:18-410 for
 * the settings above plus the FluidArray/MagnetArray allocations of imogen.m:34-45. */
int img_create(img_ctx** out, const img_config* cfg);
int img_destroy(img_ctx* ctx);

/* Construct the state from host FP64 arrays (x fastest, nx*ny*nz each; mom and mag hold the
 * three components back to back): FluidArray(...)/MagnetArray(...) of imogen.m:34-42, including
 * the initial stored edges of trans/wall boundaries and cellMag (MagnetArray.m:41-49). */
int img_set_state(img_ctx* ctx, const double* mass, const double* mom, const double* ener,
                  const double* mag);

/* X.array = value (ImogenArray.m:82-89) for one variable, and X.array reads (get.array). */
int img_upload(img_ctx* ctx, int var_id, const double* host, size_t n);
int img_download(img_ctx* ctx, int var_id, double* host, size_t n);
/* The same for several variables with one synchronisation at the end (hosts[i] holds n values of
 * variable var_ids[i]).  Mixed form: FP32 crosses PCIe; the values are rounded (IEEE
 * round-to-nearest, as the single-array calls do on the device) or widened on a small pool of host
 * threads, and the copy of one array overlaps the conversion of the next. */
int img_upload_many(img_ctx* ctx, int count, const int* var_ids, const double* const* hosts, size_t n);
int img_download_many(img_ctx* ctx, int count, const int* var_ids, double* const* hosts, size_t n);

/* TimeManager.update(mass, mom, ener, mag, fluxDirection) (time/TimeManager.m:55-99).  The new
 * dt is computed and applied on the device; dt_out / dir_out may be NULL (no host sync then). */
int img_time_update(img_ctx* ctx, int flux_direction, double* dt_out, int* dir_out);

/* flux(run, mass, mom, ener, mag, grav, order) (flux/flux.m:1-64) at the current iteration. */
int img_flux(img_ctx* ctx, int order);

/* directVec of flux.m:17-27: the three sweep dimensions (1-based, in sweep order) that img_flux uses
 * at 1-based `iteration` for order +1 (perms([1 2 3])) or -1 (perms([3 2 1])), with MATLAB
 * R2009a-R2010b's perms.  Host only; no device work. */
int img_sweep_order(int order, int iteration, int out[3]);

/* source(run, mass, mom, ener, mag, grav) (source.m:1-36) for this path: the radiation sink
 * E = E - dTime * radiation.solve (source.m:30), nothing without radiation.  Gravity is out of scope. */
int img_source(img_ctx* ctx);

/* treadmillGrid(run, mass, mom, ener, mag) (treadmill/treadmillGrid.m:1) at the current iteration;
 * nothing when the treadmill is off or before iteration 10.  img_step calls it after each flux. */
int img_treadmill(img_ctx* ctx);

/* ---- job server: img_batch_submit / poll / cancel ---------------------------------------------- */
/* Jobs admitted by HBM budget (img_bytes_required), in submission order, into the running batch of
 * their kind and advanced by one worker thread (see imogen_b200/csrc/server.cpp); a finished job's
 * result (its whole state, or its eight totals) is kept in host memory until the server is destroyed.
 * Every call returns at once and may come from any thread.  No reference counterpart: the reference
 * runs one simulation per MATLAB session. */
typedef struct img_server img_server;
enum { IMG_JOB_QUEUED = 0, IMG_JOB_RUNNING = 1, IMG_JOB_DONE = 2, IMG_JOB_FAILED = 3, IMG_JOB_CANCELLED = 4 };
enum { IMG_KEEP_STATE = 0, IMG_KEEP_TOTALS = 1 };
enum { IMG_RESULT_TOTALS = -1 };   /* img_batch_result var_id of the totals (IMG_KEEP_TOTALS) */
typedef struct img_job_info {
    int status;                  /* IMG_JOB_* */
    double time;                 /* simulated time reached (finished jobs) */
    int iterations;              /* iterations that advanced the state (finished jobs) */
    double submitted, admitted, completed;   /* img_monotonic_seconds() at those events (0: not yet) */
    int error_code;              /* IMG_ERR_* of a failed job */
    char error[256];
} img_job_info;
typedef struct img_server_info {
    size_t budget, used, peak;   /* bytes: the budget, held now, most ever held */
    int queued, running, finished;
    long long rounds;            /* scheduling rounds (one iteration of every running job each) */
} img_server_info;

/* check_every: rounds between checks for finished jobs (a check synchronises); keep: IMG_KEEP_*. */
int img_server_create(img_server** out, size_t hbm_budget, int check_every, int keep);
int img_server_destroy(img_server* s);   /* stops the worker; jobs still running are dropped */
/* Queue one job (settings + FP64 initial state as for img_set_state, copied).  IMG_ERR_NOMEM when
 * the job alone exceeds the budget. */
int img_batch_submit(img_server* s, const img_config* cfg, const double* mass, const double* mom, const double* ener,
                     const double* mag, int* job_id);
int img_batch_poll(img_server* s, int job_id, img_job_info* info);
/* A queued job is dropped at once; a running one is stopped by the worker before its next round
 * (poll until its status is IMG_JOB_CANCELLED).  IMG_ERR_STATE if the job already ended. */
int img_batch_cancel(img_server* s, int job_id);
/* The result of a finished job: variable var_id (IMG_VAR_*, n cells) or IMG_RESULT_TOTALS (8 values). */
int img_batch_result(img_server* s, int job_id, int var_id, double* host, size_t n);
int img_server_stats(img_server* s, img_server_info* info);
double img_monotonic_seconds(void);   /* the clock of the job times above: CLOCK_MONOTONIC seconds */

/* ---- slice files (save/resultsHandler.m:26-113) and resuming from them ------------------------ */
/* One slice save: SaveManager's slice type (1-3: X, Y, Z lines; 4-6: XY, XZ, YZ planes; 7: XYZ;
 * 8: SP-XYZ, SaveManager.SLICELABELS), SLICEINDEX (1-based cell of the cuts of types 1-6), the file
 * suffix ('START', 'FINAL' or the iteration label; the variable is sx_<label>_<suffix>, made a valid
 * name as genvarname does), and run.about / run.version / TimeManager.WALLMAX / the start date string
 * (NULL: '' or, through a context, its creation time in datestr's default form). */
typedef struct img_slice_meta {
    int type;
    int index[3];
    const char* suffix;
    const char* about;
    double version;
    double wall_max;
    const char* started;
} img_slice_meta;

/* Host view of a run for img_slice_write: FP64 arrays, x fastest, mom and mag three components back
 * to back; dt_history = TimeManager.history(1:n_history); tread_history = TreadmillManager.history. */
typedef struct img_slice_state {
    int grid[3];
    double dgrid[3];
    double gamma;
    double time;
    int iteration;
    int iter_max;
    double time_max;
    const double* dt_history;
    int n_history;
    int magnet_active;
    const double* mass;
    const double* mom;
    const double* ener;
    const double* mag;
    int treadmill;
    const int* tread_history;
    int n_tread;
} img_slice_state;

/* Write one slice file: a MAT-file Level 5 holding the struct resultsHandler saves (no device work). */
int img_slice_write(const char* path, const img_slice_meta* meta, const img_slice_state* state);
/* Read a slice file as Initializer.loadDataFromFile does (experiment/Initializer.m:269-292): the first
 * variable's mass, ener, momX/Y/Z and magX/Y/Z (zeros when empty).  Any output pointer may be NULL
 * (grid only: the extents of mass, trailing 1s added).  Uncompressed and zlib-compressed elements. */
int img_slice_read(const char* path, int grid[3], double* mass, double* mom, double* ener, double* mag, int* has_mag);
const char* img_slice_last_error(void);
/* The same through a context: its state, clock, dt and treadmill history (synchronises); and a
 * resume: img_set_state from a slice file whose arrays match the context's grid. */
int img_save_slice(img_ctx* ctx, const char* path, const img_slice_meta* meta);
int img_load_slice(img_ctx* ctx, const char* path);

/* TreadmillManager.history (treadmill/TreadmillManager.m:50-56) and .last: copies min(cap, count)
 * entries, *count = the number recorded (the device keeps the first 65536), synchronises. */
int img_treadmill_history(img_ctx* ctx, int* out, int cap, int* count, int* last);

/* Radiation.strength (fluid/Radiation.m:71-72; 0 without radiation), synchronises. */
int img_radiation_strength(img_ctx* ctx, double* strength);

/* relaxingFluid(run, mass, mom, ener, mag, grav, X) (fluid/relaxingFluid.m:1) -- one sweep. */
int img_fluid_sweep(img_ctx* ctx, int X);

/* magnetFlux(run, mass, mom, mag, X, magneticIndices) (magnet/magnetFlux.m:1) -- one sweep. */
int img_magnet_sweep(img_ctx* ctx, int X, int I1, int I2);

/* One pass of the imogen.m:58-72 loop body: two timesteps (CFL, flux, source), iteration+1.
 * Asynchronous: returns after enqueueing. */
int img_step(img_ctx* ctx);

/* while run.time.running: img_step (imogen.m:58-72), at most max_iters iterations (-1: no cap).
 * Returns after the device finished; *iters_done = iterations that advanced the state. */
int img_run(img_ctx* ctx, int max_iters, int* iters_done);

/* run.time.time, run.time.dTime, run.time.iteration (synchronises). */
int img_get_time(img_ctx* ctx, double* time, double* dt, int* iteration);
/* Overwrite the time manager state (time, dt, iteration). */
int img_set_time(img_ctx* ctx, double time, double dt, int iteration);

/* Simulated time, iterations that have run (TimeManager.running was true at their top), and whether
 * the run has stopped (TIMEMAX reached or ITERMAX passed).  Synchronises.  No reference counterpart
 * (the reference reads run.time and run.time.iteration). */
int img_progress(img_ctx* ctx, double* time, int* iterations_run, int* stopped);

/* Checkpoint / resume: the context's complete device state (arrays, stored edges, device clock)
 * and the host bookkeeping of its next launches, copied to a host buffer of img_checkpoint_bytes;
 * loading it into a context created with the same configuration resumes bit for bit.  The
 * reference's save/resume writes .mat slices (resultsHandler.m), which this does not replace. */
size_t img_checkpoint_bytes(const img_ctx* ctx);
int img_checkpoint_save(img_ctx* ctx, void* host, size_t bytes);
int img_checkpoint_load(img_ctx* ctx, const void* host, size_t bytes);

/* Compensated (Neumaier) FP64 totals of rho, px, py, pz, E, Bx, By, Bz over the grid. */
int img_totals(img_ctx* ctx, double out[8]);

/* The same totals as img_totals, bit for bit, computed without allocating anything, for callers
 * that may not call cudaMalloc (a MEX call whose device memory belongs to the MATLAB session's
 * allocator, or a host that has fixed its device footprint up front).  The scratch is a file-scope
 * device array of 128 KiB (16384 doubles: 1023 per-block partial pairs of 8 variables, the 8 results
 * and an 8-entry pointer table), whose device address the first call on each device looks up with
 * cudaGetSymbolAddress (make that first call before any stream capture on the device); grids of any
 * size. Each call copies the pointer table from the host, synchronises the context's stream and
 * copies the 8 results to `out` before it returns, so it cannot be captured into a graph: while the
 * context's stream is capturing it returns IMG_ERR_STATE and does nothing.  Every call overwrites all the scratch it reads,
 * so nothing needs to start at zero.  All contexts of a device share that scratch: calls that
 * overlap in time race on it and must be serialised by the caller.  The context's device must be
 * current.  No counterpart in the reference. */
int img_totals_static(img_ctx* ctx, double out[8]);

/* Block until the context's stream is idle; returns a pending device error if any. */
int img_sync(img_ctx* ctx);

/* Message of the last failing call on this context (or of img_create when ctx is NULL). */
const char* img_last_error(const img_ctx* ctx);

/* Device bytes a context with this config allocates (for HBM-budget admission). */
size_t img_bytes_required(const img_config* cfg);

/* The CUDA stream (cudaStream_t) all work of the context is issued on, for callers that record
 * CUDA events around calls or order their own work after it.  No reference counterpart. */
int img_get_stream(img_ctx* ctx, void** stream);

/* Autotuner: time every pencil tiling the kernels accept (cells per thread, CTA shape, cluster
 * size) for each swept direction and kernel (fluid sweep; magnet chain; magnet CT pass) on this
 * context's own state, `trials` sweeps each, keep the fastest, and remember it for later contexts
 * of the same shape.  The state, stored edges and clock are restored afterwards.  Needs a
 * temporary device copy of the context.  No reference counterpart. */
int img_autotune(img_ctx* ctx, int trials);
/* Tiling of slot dim: 1..3 the fluid sweeps along x, y, z, 4..6 the magnet chain along x, y, z
 * (after img_autotune the magnet CT pass may run on a tiling of its own);
 * out = {pencils per CTA, threads per pencil, CTAs per cluster, threads per CTA, cells per thread,
 * transverse components per CTA (magnet: 1 or 2; fluid: 1), segment layout: 1 when each thread owns
 * consecutive cells -- the segment fluid kernel or the window magnet kernels, used for the steady sweeps
 * of single-CTA pencils whose shifts are circ or const -- and 0 for the pencil-tile kernels}. */
int img_get_tiling(const img_ctx* ctx, int dim, int out[7]);
/* Set the tiling of slot dim to one of those the autotuner may pick (same field order); a magnet
 * slot sets the chain's and the CT pass's tiling. */
int img_set_tiling(img_ctx* ctx, int dim, const int cfg[7]);

/* Number of kernels the context has launched so far.  No reference counterpart. */
int img_launch_count(const img_ctx* ctx, uint64_t* count);

/* ---- batches: many grids, one batched launch per kernel --------------------------------------- */
/* A batch advances member contexts together: img_batch_step runs one iteration (imogen.m:58-72) of
 * every member, each with its own time step, issuing each kernel of the iteration as ONE launch
 * over all members that share its launch shape; steady iterations are replayed from a CUDA graph.
 * Members keep their state and stay usable on their own (upload/download/totals); while in a batch
 * their work runs on the batch's stream.  Members must agree in precision, physics (fluid/magnet),
 * the dimensions that are swept (extent >= 3) and the time update mode; they may sit at different
 * iterations, but must issue the same kinds of launches: a member joins after its first iteration
 * (which captures its stored edges) or all members start together.
 * No reference counterpart: the reference advances one grid per MATLAB session. */
typedef struct img_batch img_batch;
int img_batch_create(img_batch** out);
int img_batch_destroy(img_batch* b);                  /* members leave the batch; they are not destroyed */
int img_batch_add(img_batch* b, img_ctx* member);
int img_batch_remove(img_batch* b, img_ctx* member);  /* also done by img_destroy(member) */
int img_batch_size(const img_batch* b, int* n);
int img_batch_step(img_batch* b);                     /* asynchronous */
/* Step until every member has stopped (TIMEMAX reached, ITERMAX passed, or an error), checking the
 * members' flags every check_every iterations; at most max_iters iterations (-1: no cap). */
int img_batch_run(img_batch* b, int max_iters, int check_every, int* iters_done);
/* flags[i] of member i (in order of addition): bit 0 stopped, bit 1 error.  Synchronises. */
int img_batch_status(img_batch* b, int* flags, int n);
int img_batch_get_stream(img_batch* b, void** stream);
int img_batch_launch_count(const img_batch* b, uint64_t* count);
const char* img_batch_last_error(const img_batch* b);

#ifdef __cplusplus
}
#endif

#endif /* IMOGEN_B200_H */
