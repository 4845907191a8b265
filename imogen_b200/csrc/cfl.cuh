// Device-side TimeManager.update (time/TimeManager.m:55-99) and state construction helpers.
//
// The CFL maxima max_cells(|p_i/rho| + c_s) for i = 1..3 are accumulated into DevTime::maxbits,
// either by the last fluid sweep of the previous step (fused epilogue) or by cfl_reduce_kernel.
// cfl_finalize_kernel then applies the 1e-2 floor, the first-strictly-larger argmax, the CFL
// formula with MINDGRID(gridIndex), and the TIMEMAX clamp, all on the device, so a step never
// waits for the host.
#pragma once

#include "sweeps.cuh"

namespace img {

struct CflArgs {
    Geom g;
    void* q[NQ];
    DevTime* tm;
    double gamma;
    int mhd;
    int use_b[3];
    int check_nonfinite;   // flag a non-finite speed candidate (DERR_NONFINITE_STATE)
    int accumulate;        // accumulate the CFL maxima (0: the radiation sink alone)
    int radiate;           // first apply the optically thin radiation sink to E (source.m:30)
    double rad_exp;        // Radiation.exponent
    const void* fade_map;  // point-fade map (null: none); the sink's assignment to E fades it (fade_ener)
    int fade_ener;
};

// pressure(ENUM.PRESSURE_GAS, ...) of one cell (pressure.m:16-66): (G-1)(E - rho v^2/2) minus
// (G-1) B^2/2 (msq: the components without isZero), floored at 0; the reference's operation order,
// no FMA contraction.
__device__ __forceinline__ double gas_pressure(double G, double rho, double px, double py, double pz, double E,
                                               double msq) {
    const double vel_sq = __dadd_rn(__dadd_rn(__dmul_rn(px, px), __dmul_rn(py, py)), __dmul_rn(pz, pz)) / __dmul_rn(rho, rho);
    double r = __dmul_rn(G - 1.0, __dsub_rn(E, __dmul_rn(__dmul_rn(0.5, rho), vel_sq)));
    r = __dsub_rn(r, __dmul_rn(__dmul_rn(G - 1.0, 0.5), msq));
    return r < 0 ? 0.0 : r;
}

// Radiation.opticallyThinSolver (fluid/Radiation.m:86-88): (s rho^(2-a)) P_gas^a.
__device__ __forceinline__ double thin_radiation(double s, double a, double rho, double gas) {
    return __dmul_rn(__dmul_rn(s, pow(rho, 2.0 - a)), pow(gas, a));
}

// Sum of squares of the cell-centred B components without isZero, in component order.
template <typename T>
__device__ __forceinline__ double cell_msq(const CflArgs& a, const T* const cb[3], long long i) {
    double msq = 0.0;
    if (a.mhd) {
#pragma unroll
        for (int c = 0; c < 3; ++c)
            if (a.use_b[c]) { double b = cb[c][i]; msq = msq + b * b; }
    }
    return msq;
}

// CFL maxima of one grid, run by block vblock of vgrid blocks of that grid's launch; with `radiate`
// the radiation sink E <- E - dt * radiation.solve (source.m:30) is applied to each cell first (its
// CFL candidates are then those of the new E).
template <typename T>
__device__ __forceinline__ void cfl_reduce_body(const CflArgs& a, unsigned vblock, unsigned vgrid) {
    if (a.tm->done || a.tm->error || !(a.accumulate || a.radiate)) return;   // empty pass: nothing to do
    const T* rho = reinterpret_cast<const T*>(a.q[Q_RHO]);
    const T* p[3] = {reinterpret_cast<const T*>(a.q[Q_PX]), reinterpret_cast<const T*>(a.q[Q_PY]),
                     reinterpret_cast<const T*>(a.q[Q_PZ])};
    T* E = reinterpret_cast<T*>(a.q[Q_E]);
    const T* const cb[3] = {reinterpret_cast<const T*>(a.q[Q_CBX]), reinterpret_cast<const T*>(a.q[Q_CBY]),
                            reinterpret_cast<const T*>(a.q[Q_CBZ])};
    const double dt = a.tm->dt, rs = a.tm->rad_strength;
    double m3[3] = {0.0, 0.0, 0.0};
    bool bad = false;
    for (long long i = vblock * (long long)blockDim.x + threadIdx.x; i < a.g.ncell;
         i += (long long)vgrid * blockDim.x) {
        double r = rho[i], px = p[0][i], py = p[1][i], pz = p[2][i];
        const double msq = cell_msq<T>(a, cb, i);
        double e = (double)E[i];
        if (a.radiate) {
            const double gas = gas_pressure(a.gamma, r, px, py, pz, e, msq);
            T en = (T)__dsub_rn(e, __dmul_rn(dt, thin_radiation(rs, a.rad_exp, r, gas)));
            if (a.fade_ener) en = point_fade(en, reinterpret_cast<const T*>(a.fade_map)[i]);
            E[i] = en;
            e = (double)en;
        }
        if (!a.accumulate) continue;
        double sp[3];
        cfl_speeds(a.gamma, r, px, py, pz, e, msq, sp);
        bad = bad || !isfinite(sp[0] + sp[1] + sp[2]);
        m3[0] = fmax(m3[0], sp[0]);
        m3[1] = fmax(m3[1], sp[1]);
        m3[2] = fmax(m3[2], sp[2]);
    }
    if (!a.accumulate) return;   // uniform per launch
    if (a.check_nonfinite) flag_nonfinite(a.tm, bad);
    __shared__ double wp[3][32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        for (int o = 16; o > 0; o >>= 1) m3[c] = fmax(m3[c], __shfl_xor_sync(0xffffffffu, m3[c], o));
        if (lane == 0) wp[c][warp] = m3[c];
    }
    __syncthreads();
    if (threadIdx.x < 3) {   // one global atomic per block and direction
        double m = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) m = fmax(m, wp[threadIdx.x][w]);
        atomic_max_nonneg(&a.tm->maxbits[threadIdx.x], m);
    }
}

template <typename T>
__global__ void __launch_bounds__(256) cfl_reduce_kernel(const __grid_constant__ CflArgs a) {
    cfl_reduce_body<T>(a, blockIdx.x, gridDim.x);
}

template <typename T>
__global__ void __launch_bounds__(256) cfl_reduce_batch_kernel(const CflArgs* __restrict__ args,
                                                               const BlockMap* __restrict__ map) {
    __shared__ CflArgs sa;
    const BlockMap bm = map[blockIdx.x];
    load_member_args(sa, args + bm.member);
    __syncthreads();
    cfl_reduce_body<T>(sa, (unsigned)bm.block, (unsigned)bm.nblocks);
}

// Point-fade pass (classes/PointFade.m, ImogenArray.m:85-86).  var < 0: after a fluid sweep, whose
// relaxingFluid.m:64-71 assigns the five primaries (each faded when in `mask`: bit 0 rho, 1 momentum,
// 2 E) and then rho = max(rho, MINMASS) (faded again); the sweep itself left rho unclamped.  var >= 0:
// one array assigned from the host (img_upload), faded once.
struct FadeArgs {
    long long n;
    void* q[NQ];
    const void* map;
    int mask;
    int var;   // -1: the post-sweep pass; else the Q_* index of the assigned array
    double minmass;
    DevTime* tm;
};

template <typename T>
__global__ void __launch_bounds__(256) point_fade_kernel(const __grid_constant__ FadeArgs a) {
    if (a.var < 0 && (a.tm->done || a.tm->error)) return;
    const T* A = reinterpret_cast<const T*>(a.map);
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < a.n; i += (long long)gridDim.x * blockDim.x) {
        const T f = A[i];
        if (a.var >= 0) {
            T* X = reinterpret_cast<T*>(a.q[a.var]);
            X[i] = point_fade(X[i], f);
            continue;
        }
        if (a.mask & 2)
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                T* P = reinterpret_cast<T*>(a.q[Q_PX + c]);
                P[i] = point_fade(P[i], f);
            }
        if (a.mask & 4) {
            T* E = reinterpret_cast<T*>(a.q[Q_E]);
            E[i] = point_fade(E[i], f);
        }
        T* R = reinterpret_cast<T*>(a.q[Q_RHO]);
        T m = R[i];
        if (a.mask & 1) m = point_fade(m, f);
        m = m > (T)a.minmass ? m : (T)a.minmass;   // max(rho, MINMASS), NaN -> MINMASS
        if (a.mask & 1) m = point_fade(m, f);
        R[i] = m;
    }
}

// Radiation.initialize (fluid/Radiation.m:61-75), first part: the minimum over the cells of
// (E - KE - ME) / unscaledRadiation, KE = (p.p)/(2 rho), ME = (B.B)/2 of the face-centred B, the
// unscaled solver with strength 1 (NaN cells are skipped, as MATLAB's min does), into tm->rad_minbits
// (which the host sets to the bits of +inf first).
template <typename T>
__global__ void __launch_bounds__(256) rad_init_kernel(const __grid_constant__ CflArgs a) {
    const T* rho = reinterpret_cast<const T*>(a.q[Q_RHO]);
    const T* p[3] = {reinterpret_cast<const T*>(a.q[Q_PX]), reinterpret_cast<const T*>(a.q[Q_PY]),
                     reinterpret_cast<const T*>(a.q[Q_PZ])};
    const T* E = reinterpret_cast<const T*>(a.q[Q_E]);
    const T* const cb[3] = {reinterpret_cast<const T*>(a.q[Q_CBX]), reinterpret_cast<const T*>(a.q[Q_CBY]),
                            reinterpret_cast<const T*>(a.q[Q_CBZ])};
    const T* B[3] = {reinterpret_cast<const T*>(a.q[Q_BX]), reinterpret_cast<const T*>(a.q[Q_BY]),
                     reinterpret_cast<const T*>(a.q[Q_BZ])};
    double m = __longlong_as_double(0x7ff0000000000000ll);   // +inf
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < a.g.ncell;
         i += (long long)gridDim.x * blockDim.x) {
        const double r = rho[i], px = p[0][i], py = p[1][i], pz = p[2][i], e = E[i];
        const double bx = B[0][i], by = B[1][i], bz = B[2][i];
        const double unscaled = thin_radiation(1.0, a.rad_exp, r, gas_pressure(a.gamma, r, px, py, pz, e, cell_msq<T>(a, cb, i)));
        const double kinetic = __dmul_rn(0.5, __dadd_rn(__dadd_rn(__dmul_rn(px, px), __dmul_rn(py, py)), __dmul_rn(pz, pz))) / r;
        const double magnetic = __dmul_rn(0.5, __dadd_rn(__dadd_rn(__dmul_rn(bx, bx), __dmul_rn(by, by)), __dmul_rn(bz, bz)));
        const double ratio = __dsub_rn(__dsub_rn(e, kinetic), magnetic) / unscaled;
        if (ratio == ratio) m = fmin(m, ratio);
    }
    for (int o = 16; o > 0; o >>= 1) m = fmin(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) atomicMin(&a.tm->rad_minbits, ordered_bits(m));
}

// Radiation.initialize, second part: strength = initialMaximum / 100 * minimum.
__global__ void rad_init_finalize_kernel(DevTime* tm, double scale) {
    if (threadIdx.x == 0 && blockIdx.x == 0) tm->rad_strength = scale * from_ordered_bits(tm->rad_minbits);
}

// check_running: evaluate TimeManager.running (time < TIMEMAX) first, as imogen.m:58 does at the
// top of each iteration; the iteration limit is enforced by the host.
__device__ __forceinline__ void cfl_finalize_body(DevTime* tm, int check_running) {
    if (tm->done || tm->error) return;
    if (check_running && !(tm->time < tm->time_max)) {
        tm->done = 1;
        return;
    }
    if (check_running) tm->iters_run += 1;   // = run.time.iteration from here on
    double cmax = 1e-2;
    int gi = 0;
    for (int i = 0; i < 3; ++i) {
        double c = __longlong_as_double((long long)tm->maxbits[i]);
        tm->maxbits[i] = 0ull;
        if (c > cmax) { cmax = c; gi = i + 1; }
    }
    tm->cmax = cmax;
    tm->grid_index = gi;
    if (gi < 1) {   // TimeManager.m:79-86 (fireCFLError)
        tm->error |= DERR_CFL;
        return;
    }
    double dt = tm->cfl * tm->dgrid[gi - 1] / cmax;
    double nt = tm->time + (tm->update_mode + 1) * dt;
    if (nt > tm->time_max) {
        dt = (tm->time_max - tm->time) / (tm->update_mode + 1);
        nt = tm->time_max;
    }
    if (!isfinite(dt)) {
        tm->error |= DERR_NONFINITE_DT;
        return;
    }
    tm->dt = dt;
    tm->time = nt;
    // TimeManager.appendHistory: history(iteration) = dTime (the second update of a per-step
    // iteration overwrites the first)
    const int k = tm->iters_run - 1;
    if (tm->dt_hist && k >= 0 && k < tm->dt_hist_cap) tm->dt_hist[k] = dt;
}

__global__ void cfl_finalize_kernel(DevTime* tm, int check_running) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    cfl_finalize_body(tm, check_running);
}

// The finalisation for many grids: thread i handles member i.
__global__ void cfl_finalize_batch_kernel(DevTime* const* __restrict__ tms, int n, int check_running) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) cfl_finalize_body(tms[i], check_running);
}

// MagnetArray construction: cellMag = 0.5*(B + B.shift(component, +1)) (MagnetArray.m:36-38,41-49).
struct CellMagInitArgs {
    Geom g;
    void* q[NQ];
    int mode_hi[3];      // mag-class upper BC along dim c for component c
    int act[3];
    const EdgeTable* edges;
    const double* fade;
    int fade_f;
    double bc_inf;
};

template <typename T>
__global__ void cellmag_init_kernel(const __grid_constant__ CellMagInitArgs a) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < 3 * a.g.ncell;
         i += (long long)gridDim.x * blockDim.x) {
        int cpt = (int)(i / a.g.ncell);
        long long cell = i - cpt * a.g.ncell;
        const T* B = reinterpret_cast<const T*>(a.q[Q_BX + cpt]);
        T* CB = reinterpret_cast<T*>(a.q[Q_CBX + cpt]);
        int x, y, z;
        cell_coords(a.g, cell, x, y, z);
        T sh;
        if (cpt < a.g.ndims) {
            bool own = sel3(cpt, x, y, z) == a.g.n[cpt] - 1;
            sh = shift_along<T>(a.g, B, cell, x, y, z, cpt, +1, a.mode_hi[cpt], a.act[cpt], true,
                                a.edges->p[OBJ_PRIM_MAG + cpt][cpt][1], a.fade, a.fade_f, a.bc_inf, own);
        } else {
            sh = B[cell];
        }
        CB[cell] = T(0.5) * (B[cell] + sh);
    }
}

// Neumaier-compensated FP64 totals of the conserved variables (rho, px, py, pz, E, Bx, By, Bz):
// one partial (sum, compensation) pair per block and variable; the host finishes the sum.
template <typename T>
__global__ void totals_kernel(Geom g, const void* const* qp, double* partial) {
    __shared__ double ss[8][32], cc[8][32];
    double s[8], c[8];
#pragma unroll
    for (int v = 0; v < 8; ++v) { s[v] = 0.0; c[v] = 0.0; }
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < g.ncell;
         i += (long long)gridDim.x * blockDim.x) {
#pragma unroll
        for (int v = 0; v < 8; ++v) {
            double x = (double)reinterpret_cast<const T*>(qp[v])[i];
            double t = s[v] + x;
            c[v] += fabs(s[v]) >= fabs(x) ? (s[v] - t) + x : (x - t) + s[v];
            s[v] = t;
        }
    }
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int v = 0; v < 8; ++v) {
        // warp: pairwise Neumaier combine
        for (int o = 16; o > 0; o >>= 1) {
            double so = __shfl_xor_sync(0xffffffffu, s[v], o);
            double co = __shfl_xor_sync(0xffffffffu, c[v], o);
            double t = s[v] + so;
            double e = fabs(s[v]) >= fabs(so) ? (s[v] - t) + so : (so - t) + s[v];
            s[v] = t;
            c[v] = c[v] + co + e;
        }
        if (lane == 0) { ss[v][w] = s[v]; cc[v][w] = c[v]; }
    }
    __syncthreads();
    if (threadIdx.x < 8) {
        int v = threadIdx.x;
        double S = 0.0, Cc = 0.0;
        for (int k = 0; k < (int)(blockDim.x >> 5); ++k) {
            double x = ss[v][k];
            double t = S + x;
            Cc += fabs(S) >= fabs(x) ? (S - t) + x : (x - t) + S;
            S = t;
            Cc += cc[v][k];
        }
        partial[(blockIdx.x * 8 + v) * 2] = S;
        partial[(blockIdx.x * 8 + v) * 2 + 1] = Cc;
    }
}

// Final Neumaier combine of the per-block totals partials, in block order (the same operations, in
// the same order, as the host combine of img_totals): one thread per variable.
__global__ void totals_finalize_kernel(const double* partial, int nblocks, double* out) {
    const int v = threadIdx.x;
    if (v >= 8) return;
    double S = 0.0, C = 0.0;
    for (int b = 0; b < nblocks; ++b) {
        const double x = partial[(b * 8 + v) * 2];
        const double t = S + x;
        C += fabs(S) >= fabs(x) ? (S - t) + x : (x - t) + S;
        S = t;
        C += partial[(b * 8 + v) * 2 + 1];
    }
    out[v] = S + C;
}

// Host-transfer conversions of the mixed form (FP64 staging <-> FP32 state), 4 values per thread
// where the array's 16-byte alignment allows (arrays start 256-byte aligned).
__global__ void f64_to_f32_kernel(const double* __restrict__ src, float* __restrict__ dst, long long n) {
    const long long n4 = n / 4;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n4; i += (long long)gridDim.x * blockDim.x) {
        const double2 a = reinterpret_cast<const double2*>(src)[2 * i];
        const double2 b = reinterpret_cast<const double2*>(src)[2 * i + 1];
        reinterpret_cast<float4*>(dst)[i] = make_float4((float)a.x, (float)a.y, (float)b.x, (float)b.y);
    }
    for (long long i = 4 * n4 + blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        dst[i] = (float)src[i];
}

__global__ void f32_to_f64_kernel(const float* __restrict__ src, double* __restrict__ dst, long long n) {
    const long long n4 = n / 4;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n4; i += (long long)gridDim.x * blockDim.x) {
        const float4 a = reinterpret_cast<const float4*>(src)[i];
        reinterpret_cast<double2*>(dst)[2 * i] = make_double2(a.x, a.y);
        reinterpret_cast<double2*>(dst)[2 * i + 1] = make_double2(a.z, a.w);
    }
    for (long long i = 4 * n4 + blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        dst[i] = (double)src[i];
}

}  // namespace img
