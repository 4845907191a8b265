// Shared device-side definitions for the relaxing-TVD sweep kernels.
//
// State layout in HBM: structure of arrays, one array per variable, x fastest (the MATLAB
// column-major order of the reference), each array 256-byte aligned.  The eleven arrays are
// rho, px, py, pz, E, the face-centred B (Bx, By, Bz; B_i(i) lives on face i-1/2,
// magnet/MagnetArray.m:36-38) and the cell-centred B used by the fluid (cBx, cBy, cBz).  The
// cell-centred copy is state, not a derived quantity: magnet/magnetFlux.m:30-31 refreshes only
// two of its three components per sweep, so one component is a step stale by design.
#pragma once

#include <cooperative_groups.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace img {

namespace cg = cooperative_groups;

// ---- enumerations shared with the host (values match include/imogen_b200.h) --------------------
enum BcMode { BC_CIRC = 0, BC_CONST = 1, BC_FADE = 2, BC_MIRROR = 3, BC_TRANS = 4, BC_WALL = 5, BC_FLIP = 6, BC_ZERO = 7,
              BC_LINEAR = 8, BC_WORMHOLE = 9 };
// Ghost flags of one array object: GF_NEG negates mirror/flip ghosts (the array's component is the
// shift direction, mirror_shift.m / flip_shift.m); GF_ZLO / GF_ZHI make a zero-BC ghost 0 on the
// lower / upper side (zero_shift.m: a FluxArray other than fluxl below and other than fluxr above).
constexpr int GF_NEG = 1;
constexpr int GF_ZLO = 2;
constexpr int GF_ZHI = 4;
constexpr int GF_FLUXR = GF_ZLO;             // fluxType 'fluxr'
constexpr int GF_FLUXL = GF_ZHI;             // fluxType 'fluxl'
constexpr int GF_FLUX = GF_ZLO | GF_ZHI;     // other flux types ('flux')
enum Limiter { LIM_VANLEER = 0, LIM_SUPERBEE = 1, LIM_MINMOD = 2 };
enum BcClass { CLS_MASS = 0, CLS_MOM = 1, CLS_ENER = 2, CLS_MAG = 3 };
enum Var { Q_RHO = 0, Q_PX, Q_PY, Q_PZ, Q_E, Q_BX, Q_BY, Q_BZ, Q_CBX, Q_CBY, Q_CBZ, NQ };

// Error bits written by kernels into DevTime::error (host reads them after a step).
enum DevError : int { DERR_NONFINITE_DT = 1, DERR_CFL = 2, DERR_NONFINITE_STATE = 4 };

// ---- stored-edge objects ------------------------------------------------------------------------
// Every array object of the reference that can be shifted under a stateful BC (trans, wall) owns a
// stored edge per (dim, side) (shifting/Edges.m).  Object ids:
//   fluid var v (0..4: rho,px,py,pz,E) x {store.fluxR, store.fluxL, fluxR, fluxL}: v*4 + k
//   primary mass, mom(1..3), mag(1..3):                                   20, 21+c, 24+c
//   mag(c) scratch for sweep dim X (c != X) x {velGrid, store.fluxR, wMag, flux}:
//                                                                   27 + (c*3+X)*4 + k
constexpr int OBJ_FLUID = 0;
constexpr int OBJ_PRIM_MASS = 20;
constexpr int OBJ_PRIM_MOM = 21;
constexpr int OBJ_PRIM_MAG = 24;
constexpr int OBJ_MAG = 27;
constexpr int OBJ_PRIM_ENER = 27 + 36;   // the energy primary: its edges serve only treadmillGrid's shift
constexpr int NOBJ = 27 + 36 + 1;
enum FluidObj { FO_STORE_R = 0, FO_STORE_L = 1, FO_R = 2, FO_L = 3 };
enum MagObj { MO_VELGRID = 0, MO_STORE_R = 1, MO_WMAG = 2, MO_FLUX = 3 };
__host__ __device__ constexpr int fluid_obj(int v, int k) { return OBJ_FLUID + v * 4 + k; }
__host__ __device__ constexpr int mag_obj(int c, int X, int k) { return OBJ_MAG + (c * 3 + X) * 4 + k; }

// Table of stored-edge slices: edge[obj][dim][side] -> face array (double) or nullptr.
struct EdgeTable {
    double* p[NOBJ][3][2];
};

// ---- device-resident time manager (time/TimeManager.m:55-99) ------------------------------------
struct DevTime {
    double time;
    double dt;
    double time_max;
    double cfl;
    double dgrid[3];
    double cmax;            // last CFL max (after the 1e-2 floor)
    int grid_index;         // 1-based argmax direction of the last CFL
    int update_mode;        // 0 per step, 1 per iteration
    int error;              // DevError bits
    int done;               // TimeManager.running turned false (time >= TIMEMAX)
    int iters_run;          // iterations that started (TimeManager.running was true at their top)
    int reserved1;
    unsigned long long maxbits[3];   // per-direction max of |v_i| + c_s (bit pattern, >= 0)
    unsigned int counter;            // CTAs finished in the current CFL reduction
    unsigned int pad2;
    double rad_strength;             // Radiation.strength (set by Radiation.initialize at set_state)
    unsigned long long rad_minbits;  // ordered bits of the running minimum of Radiation.initialize
    int tread_last;                  // TreadmillManager.last (-1 until the first treadmillGrid call)
    int tread_dc;                    // dCells of the current call
    int tread_go;                    // the current call shifts the grid
    int tread_count;                 // entries in TreadmillManager.history
    double* dt_hist;                 // TimeManager.history: dTime of iteration k at [k - 1] (k <= cap)
    int dt_hist_cap;
    int pad3;
};

// ---- batched launches -----------------------------------------------------------------------------
// A batched launch runs one kernel over the CTAs of many grids ("members"): CTA b of the launch
// works on block `block` of member `member`, whose own launch would have `nblocks` CTAs.  A
// member's CTAs are contiguous and start at a multiple of the cluster size.
struct BlockMap {
    int member;
    int block;
    int nblocks;
};

// Copy one member's kernel arguments into shared memory (all threads; a barrier follows).
template <typename Args>
__device__ __forceinline__ void load_member_args(Args& dst, const Args* src) {
    static_assert(sizeof(Args) % 4 == 0, "argument blocks are word multiples");
    const int* s = reinterpret_cast<const int*>(src);
    int* d = reinterpret_cast<int*>(&dst);
    for (int i = threadIdx.x; i < (int)(sizeof(Args) / 4); i += blockDim.x) d[i] = s[i];
}

// ---- grid geometry --------------------------------------------------------------------------------
struct Geom {
    int n[3];
    int ndims;        // 3 if nz > 1 else 2 (MATLAB squeeze + ndims)
    long long s[3];   // strides: 1, nx, nx*ny
    long long ncell;
};

// Index of a cell inside the face orthogonal to dim e (column-major order of the other two dims).
__host__ __device__ inline long long face_index(const Geom& g, int e, int x, int y, int z) {
    if (e == 0) return (long long)z * g.n[1] + y;
    if (e == 1) return (long long)z * g.n[0] + x;
    return (long long)y * g.n[0] + x;
}

// Select one of three values by a runtime index without indexing a register array.
template <typename T>
__host__ __device__ __forceinline__ T sel3(int i, T a, T b, T c) { return i == 0 ? a : (i == 1 ? b : c); }

// ---- small numeric helpers --------------------------------------------------------------------------
template <typename T> __device__ __forceinline__ T tmax(T a, T b) { return a > b ? a : b; }
__device__ __forceinline__ double msign(double v) { return v > 0 ? 1.0 : (v < 0 ? -1.0 : (v == 0 ? 0.0 : v)); }
__device__ __forceinline__ float msign(float v) { return v > 0 ? 1.f : (v < 0 ? -1.f : (v == 0 ? 0.f : v)); }

// TVD limiter correction (flux/vanleerLimiter.m:9-11, minmodLimiter.m:9, superbeeLimiter.m:9-10) for a
// limiter known at compile time.  The reference adds it to the flux in place:
// flux.array = flux.array + correction.
template <int LIM, typename T>
__device__ __forceinline__ T limiter_corr_t(T dL, T dR) {
    if constexpr (LIM == LIM_VANLEER) {
        T p = dL * dR;
        T num = p > T(0) ? p : T(0);
        T st;
        if constexpr (sizeof(T) == 4) st = __fdividef(num, dL + dR);   // mixed form: fast divide
        else st = num / (dL + dR);
        return isnan(st) ? T(0) : st;
    } else {
        if constexpr (LIM == LIM_SUPERBEE) {
            T c = fabs(dL) < fabs(dR) ? T(1) : T(0);
            dL = (T(1) + c) * dL;
            dR = (T(2) - c) * dR;
        }
        return T(0.125) * (msign(dL) + msign(dR)) * fmin(fabs(dL), fabs(dR));
    }
}

// The same for a limiter chosen at run time (uniform over a launch).
template <typename T>
__device__ __forceinline__ T limiter_corr(int lim, T dL, T dR) {
    if (lim == LIM_VANLEER) return limiter_corr_t<LIM_VANLEER>(dL, dR);
    if (lim == LIM_SUPERBEE) return limiter_corr_t<LIM_SUPERBEE>(dL, dR);
    return limiter_corr_t<LIM_MINMOD>(dL, dR);
}

// Stored-edge drift of a transparent edge (Edges.m:121-136): move toward the current edge value
// by at most TOLERANCE = 0.005.
__device__ __forceinline__ double edge_drift(double old_e, double cur) {
    double delta = fmin(fabs(cur - old_e), 0.005);
    bool st = (cur - old_e) > 0;
    return old_e + ((st ? 1.0 : 0.0) - (st ? 0.0 : 1.0)) * delta;
}

// One-sided shape-preserving end slope of MATLAB pchip (pchipslopes end formula).
__device__ __forceinline__ double pchip_end_slope(double h0, double h1, double d0, double d1) {
    double dd = ((2 * h0 + h1) * d0 - h0 * d1) / (h0 + h1);
    if (msign(dd) != msign(d0)) dd = 0.0;
    else if (msign(d0) != msign(d1) && fabs(dd) > fabs(3 * d0)) dd = 3 * d0;
    return dd;
}
// Interior slope: Fritsch-Butland weighted harmonic mean, 0 at sign changes.
__device__ __forceinline__ double pchip_mid_slope(double hl, double hr, double dl, double dr) {
    double w1 = 2 * hr + hl;
    double w2 = hr + 2 * hl;
    return (msign(dl) * msign(dr) > 0) ? (w1 + w2) / (w1 / dl + w2 / dr) : 0.0;
}

// MATLAB pchip through x = [1 2 3 inf inf+1] with values y0..y4, evaluated at xe >= 4 (Moler,
// "Numerical Computing with MATLAB", pchiptx; the interval is the last breakpoint <= xe, clamped
// to the last interval as ppval does).  For xe >= 4 the interval is [3, inf) or [inf, inf+1], so
// only the slopes at x = 3, inf and inf+1 are formed (y0 enters none of them).  Scalars only.
__device__ __forceinline__ double pchip5(double y1, double y2, double y3, double y4, double inf, double xe) {
    const double x3 = inf, x4 = inf + 1.0;
    const double h1 = 1.0, h2 = x3 - 3.0, h3 = x4 - x3;
    const double e1 = (y2 - y1) / h1, e2 = (y3 - y2) / h2, e3 = (y4 - y3) / h3;
    const double s3 = pchip_mid_slope(h2, h3, e2, e3);
    double xk, yk, hk, ek, dk, dk1;
    if (xe >= x3) { xk = x3; yk = y3; hk = h3; ek = e3; dk = s3; dk1 = pchip_end_slope(h3, h2, e3, e2); }
    else { xk = 3.0; yk = y2; hk = h2; ek = e2; dk = pchip_mid_slope(h1, h2, e1, e2); dk1 = s3; }
    const double s = xe - xk;
    const double c1 = (dk + dk1 - 2 * ek) / (hk * hk);
    const double c2 = (3 * ek - 2 * dk - dk1) / hk;
    return ((c1 * s + c2) * s + dk) * s + yk;
}

// Rows that transparent_shift.m:36-39 / :68-71 feed to pchip at x = 1, 2, 3 for a shift by
// n = -m (lower end) or n = +m (upper end): rows 2,1,0 / N-3,N-2,N-1, clamped for short lines.
__host__ __device__ __forceinline__ int trans_pick_lower(int N, int m, int q) {
    int p = 3 - q + m;
    p = p > N ? N : p;
    p = p - 1 - m;
    return p < 0 ? 0 : p;
}
__host__ __device__ __forceinline__ int trans_pick_upper(int N, int m, int q) {
    int p = N - (2 - q) - m;
    p = p < 1 ? 1 : p;
    p = p - 1 + m;
    return p > N - 1 ? N - 1 : p;
}

// Transparent ghost value (shifting/transparent_shift.m:23-99).  y1, y2 = the array values that
// the reference feeds at x = 2, 3 (x = 3 is the edge cell; the value at x = 1 does not affect the
// result at xe >= 4), edge = the stored edge after its drift (0 when the edge store is not
// ACTIVE(DIRECT)), xe = 4 or 5, orig = the unshifted array value at the ghost position (kept when
// the extrapolation is within 1e-4 of it).
__device__ __forceinline__ double trans_ghost(double y1, double y2, double edge, double inf, double xe, double orig) {
    double out = pchip5(y1, y2, edge, edge, inf, xe);
    bool t = fabs(orig - out) < 1e-4;
    return (t ? 0.0 : 1.0) * out + (t ? 1.0 : 0.0) * orig;
}

// Pressure recovery (pressure/pressure.m:23-64), always in FP64.  Returns P (clamped at 0).
// sound_mode = false: 'totsnd' (P_tot and c_s with the 2B^2 term); true: 'sound' (c_s in P).
struct PressOut {
    double p;
    double cs;
};
__device__ __forceinline__ PressOut pressure_totsnd(double G, double rho, double px, double py, double pz, double E,
                                                    double msq) {
    const double ir = 1.0 / rho;   // one division (a compiler CSE shares it with the flux terms)
    double vsq = (px * px + py * py + pz * pz) * (ir * ir);
    double r = (G - 1.0) * (E - 0.5 * rho * vsq);
    PressOut o;
    o.cs = sqrt(fabs((G * (r - (G - 1.0) * 0.5 * msq) + 2.0 * msq) * ir));
    r = r + 0.5 * (2.0 - G) * msq;
    o.p = r < 0 ? 0.0 : r;
    return o;
}
// Hardware approximations for the FP32 arithmetic of the mixed form: the reciprocal within 1 ulp and
// the square root within 2^-23 relative (PTX rcp.approx.f32 / sqrt.approx.f32), one instruction
// each instead of the correctly rounded sequences.
__device__ __forceinline__ float rcp_approx(float x) {
    float r;
    asm("rcp.approx.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}
__device__ __forceinline__ float sqrt_approx(float x) {
    float r;
    asm("sqrt.approx.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

// Mixed form of 'totsnd' for FP32 state: the pressure recovery P0 = (G-1)(E - rho v^2/2) and the
// magnetic terms are evaluated in FP64 (the reciprocal of rho is an FP32 estimate refined by one
// FP64 Newton step, exact to ~1e-15), the sound speed is taken in FP32.
struct PressOutF {
    float p;
    float cs;
};
__device__ __forceinline__ PressOutF pressure_totsnd_mixed(double G, float rho, float px, float py, float pz, float E,
                                                          double msq) {
    double r = rho;
    double inv = (double)rcp_approx(rho);   // FP32 seed, one FP64 Newton step
    inv = inv * (2.0 - r * inv);
    double psq = (double)px * px + (double)py * py + (double)pz * pz;
    double p0 = (G - 1.0) * ((double)E - 0.5 * psq * inv);
    double pg = p0 - (G - 1.0) * 0.5 * msq;
    PressOutF o;
    o.cs = sqrt_approx((float)fabs((G * pg + 2.0 * msq) * inv));
    double pt = p0 + 0.5 * (2.0 - G) * msq;
    o.p = pt < 0 ? 0.f : (float)pt;
    return o;
}

// CFL speed candidates |p_c / rho| + c_s of one cell, c = x, y, z (TimeManager.m:65-77 with the
// 'sound' speed of pressure.m): one FP64 reciprocal of rho serves the four quotients.
__device__ __forceinline__ void cfl_speeds(double G, double rho, double px, double py, double pz, double E,
                                           double msq, double s[3]) {
    const double inv = 1.0 / rho;
    const double vsq = (px * px + py * py + pz * pz) * (inv * inv);
    double r = (G - 1.0) * (E - 0.5 * rho * vsq);
    r = r - (G - 1.0) * 0.5 * msq;
    const double cs = sqrt(fabs((G * r + 2.0 * msq) * inv));
    s[0] = fabs(px * inv) + cs;
    s[1] = fabs(py * inv) + cs;
    s[2] = fabs(pz * inv) + cs;
}

// Barrier over every thread of the thread-block cluster, with release/acquire ordering of shared
// memory (DSMEM) accesses across it.  The warp is reconverged first and the per-thread (non-aligned)
// forms of barrier.cluster are used, so a warp that reaches the barrier after divergent work (halo
// jobs, stored-edge captures done by a few lanes) arrives exactly once per thread.
__device__ __forceinline__ void cluster_sync() {
    __syncwarp();
    asm volatile("barrier.cluster.arrive.release;\n\tbarrier.cluster.wait.acquire;" ::: "memory");
}

// Programmatic dependent launch: a pencil kernel launched with programmatic stream serialization may
// be scheduled before the previous kernel of its stream has finished.  pdl_wait() blocks until that
// kernel has completed and its memory is visible (a no-op for an ordinary launch); every read of data
// another kernel wrote comes after it.  pdl_trigger() lets the next kernel be scheduled; a kernel
// calls it at the start of its last stage, when every one of its CTAs is resident.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

// Flag a non-finite CFL speed candidate (a non-finite rho, momentum, energy or B in the cell) of any
// lane of the warp: one atomic per warp that saw one.
__device__ __forceinline__ void flag_nonfinite(DevTime* tm, bool bad) {
    if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) atomicOr(&tm->error, (int)DERR_NONFINITE_STATE);
}

// Atomic max of a non-negative double through its bit pattern (NaN never reaches here).
__device__ __forceinline__ void atomic_max_nonneg(unsigned long long* addr, double v) {
    atomicMax(addr, (unsigned long long)__double_as_longlong(v));
}

// PointFade.fadeArray (classes/PointFade.m:46-49): 0.95 u A + u (1 - A) in that order, without FMA
// contraction.
__device__ __forceinline__ float point_fade(float u, float A) {
    return __fadd_rn(__fmul_rn(__fmul_rn(0.95f, u), A), __fmul_rn(u, __fsub_rn(1.0f, A)));
}
__device__ __forceinline__ double point_fade(double u, double A) {
    return __dadd_rn(__dmul_rn(__dmul_rn(0.95, u), A), __dmul_rn(u, __dsub_rn(1.0, A)));
}

// Doubles of either sign as unsigned integers of the same order (the callers exclude NaN).
__device__ __forceinline__ unsigned long long ordered_bits(double v) {
    const unsigned long long b = (unsigned long long)__double_as_longlong(v);
    return (b >> 63) ? ~b : (b | 0x8000000000000000ull);
}
__device__ __forceinline__ double from_ordered_bits(unsigned long long b) {
    b = (b >> 63) ? (b & 0x7fffffffffffffffull) : ~b;
    return __longlong_as_double((long long)b);
}

}  // namespace img
