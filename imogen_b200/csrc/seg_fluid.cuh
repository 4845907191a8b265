// Segment form of the fused fluid sweep (fluid/relaxingFluid.m:16-73, fluid/wFluidFlux.m:14-44,
// pressure/pressure.m:23-64, flux/*Limiter.m) for pencils that fit one CTA with circ or const ends.
//
// Each thread owns C consecutive cells of a pencil (a "segment"), so every stencil neighbour inside a
// segment is a register; only the cells at the two ends of a segment are exchanged, through shared
// memory, and the exchanges ride on the two barriers that the pencil maxima need anyway:
//   stage 1  load the segment (128-bit loads along x), 'totsnd' pressure, freezing-speed candidate and
//            the flux numerators F (w = F / c_f) of every cell; publish (u, F) of the first and last
//            cell; barrier; c_f = pencil max.
//   stage 2  predictor half step with R = (u + F/c_f)/2, L = (u - F/c_f)/2 (relaxingFluid.m:30-39);
//            pressure, speed and F of the half-step state; publish (u*, F*) of the first two and last
//            two cells; barrier; c_f* = pencil max.
//   stage 3  corrector fluxes R*, L* over the segment and the two neighbour cells each side, the TVD
//            limiter (relaxingFluid.m:57-62) -- the limited values of the neighbour cells next to the
//            segment are computed here as well, from the published cells -- and the update
//            (relaxingFluid.m:64-71); store; fused CFL maxima on the last sweep of a step.
// With artificial viscosity (fluid/ArtificialViscosity.m) stages 1 and 2 each publish the viscosity
// exchange set with the pencil maximum, then compute the viscous pressure and F and publish (u, F)
// behind one more barrier: four barriers instead of two.
// Per cell the formulas are those of the pencil-tile kernels (fluid_sweep.cuh); the momentum and
// cell-centred B are held in sweep-rotated order (the component along the sweep first), so sums over
// components run in that order, and the compiler may contract differently into FMAs: the two kernel
// families agree to round-off, not bit for bit.  The limiter is fixed per launch and compiled into the
// corrector (seg_correct).
//
// Thread placement (SweepGeom with G = S segments per pencil, RC = N): along x the S threads of a
// pencil are consecutive (thread t = b*S + s), along y and z the Wb pencils of the CTA are (t = s*Wb +
// b), so global loads and stores stay coalesced along x.  Pencil ends: a circ end's neighbour segment
// is the pencil's other end; a const end's ghost is the end cell itself (constant_shift.m), applied to
// every shifted array, the limited fluxes included.
#pragma once

#include <type_traits>

#include "fluid_sweep.cuh"

namespace img {

// FP64 words per thread of the artificial-viscosity exchange set (seg_visc_publish).
constexpr int VISC_ROWS = 9;

// Words per thread of the two exchange sets and of the pencil maxima: (u, F) of 2 cells, (u*, F*) of
// 4 cells, and 2 per-warp maxima slots of 32 columns; with artificial viscosity the FP64 viscosity
// exchange set after them.
template <typename T>
__host__ __device__ inline size_t seg_fluid_smem_bytes(int NT, bool visc = false) {
    return sizeof(T) * ((size_t)60 * NT + 2 * (size_t)(NT / 32) * 32) + (visc ? sizeof(double) * VISC_ROWS * NT : 0);
}

// Placement of one thread in the segment layout.
struct SegPos {
    int b, s;            // pencil within the CTA, segment within the pencil
    int rank = 0;        // cluster rank (one pencil per cluster)
    bool colok;          // the pencil exists (the last CTA may hold fewer than Wb) and so does the segment
    long long base;      // offset of the pencil's row 0
    // One pencil along x over the CL CTAs of a cluster (CL = 1: one CTA), S = ceil(N / C) segments of
    // which rank r holds r * NT .. r * NT + NT - 1; threads past the last segment idle.
    __device__ __forceinline__ void init_cluster(const SweepGeom& g, unsigned vblock) {
        const unsigned blk = g.div_cl.div(vblock);
        rank = (int)(vblock - blk * (unsigned)g.CL);
        b = 0;
        s = rank * g.NT + (int)threadIdx.x;
        colok = s < g.G && (long long)blk < g.ncol;
        const unsigned c = colok ? blk : 0u;
        const int c2 = (int)g.div_n1.div(c);
        const int c1 = (int)(c - (unsigned)c2 * (unsigned)g.n1);
        base = c1 * g.s1 + (long long)c2 * g.s2;
    }
    __device__ __forceinline__ void init(const SweepGeom& g, unsigned vblock) {
        const int t = threadIdx.x;
        const unsigned q = g.div_lanes.div((unsigned)t);   // t / S (x) or t / Wb (y, z)
        if (g.d == 0) { b = (int)q; s = t - b * g.G; }
        else { s = (int)q; b = t - s * g.Wb; }
        const int col = (int)(vblock * (unsigned)g.Wb + (unsigned)b);
        colok = col < g.ncol;
        const unsigned c = colok ? (unsigned)col : 0u;
        const int c2 = (int)g.div_n1.div(c);
        const int c1 = (int)(c - (unsigned)c2 * (unsigned)g.n1);
        base = c1 * g.s1 + (long long)c2 * g.s2;
    }
};

// C consecutive values of array p starting at offset o, stride sd (vector loads when sd == 1: the
// offset is a multiple of C and arrays start 256-byte aligned).
template <typename T, int C>
__device__ __forceinline__ void seg_load(const void* p, long long o, long long sd, bool vec, T (&out)[C]) {
    const T* a = reinterpret_cast<const T*>(p) + o;
    if (vec) {
        if constexpr (sizeof(T) == 4 && C % 4 == 0) {
#pragma unroll
            for (int k = 0; k < C; k += 4) {
                const float4 v = *reinterpret_cast<const float4*>(a + k);
                out[k] = v.x; out[k + 1] = v.y; out[k + 2] = v.z; out[k + 3] = v.w;
            }
            return;
        } else if constexpr (C % 2 == 0) {
            using V2 = typename std::conditional<sizeof(T) == 4, float2, double2>::type;
#pragma unroll
            for (int k = 0; k < C; k += 2) {
                const V2 v = *reinterpret_cast<const V2*>(a + k);
                out[k] = v.x; out[k + 1] = v.y;
            }
            return;
        }
    }
#pragma unroll
    for (int k = 0; k < C; ++k) out[k] = a[(long long)k * sd];
}

template <typename T, int C>
__device__ __forceinline__ void seg_store(void* p, long long o, long long sd, bool vec, const T (&v)[C]) {
    T* a = reinterpret_cast<T*>(p) + o;
    if (vec) {
        if constexpr (sizeof(T) == 4 && C % 4 == 0) {
#pragma unroll
            for (int k = 0; k < C; k += 4) *reinterpret_cast<float4*>(a + k) = make_float4(v[k], v[k + 1], v[k + 2], v[k + 3]);
            return;
        } else if constexpr (C % 2 == 0) {
#pragma unroll
            for (int k = 0; k < C; k += 2) {
                if constexpr (sizeof(T) == 4) *reinterpret_cast<float2*>(a + k) = make_float2(v[k], v[k + 1]);
                else *reinterpret_cast<double2*>(a + k) = make_double2(v[k], v[k + 1]);
            }
            return;
        }
    }
#pragma unroll
    for (int k = 0; k < C; ++k) a[(long long)k * sd] = v[k];
}

// The flux numerators F of wFluidFlux.m:31-44 (w = F * (1/c_f)) for one cell whose momentum and
// cell-centred B are held in sweep-rotated order (component 0 along the sweep): the mixed form with the
// one-instruction FP32 reciprocal of rho, FP64 with the IEEE reciprocal (the operations of wflux).
template <typename T>
__device__ __forceinline__ void flux_num_rot(const T u[5], const T bb[3], T press, T F[5]) {
    T ir;
    if constexpr (sizeof(T) == 4) ir = rcp_approx(u[0]);
    else ir = T(1) / u[0];
    const T velocity = u[1] * ir;
    F[0] = u[1];
    F[4] = velocity * (u[4] + press) - bb[0] * (bb[0] * u[1] + bb[1] * u[2] + bb[2] * u[3]) * ir;
    F[1] = velocity * u[1] + press - bb[0] * bb[0];
    F[2] = velocity * u[2] - bb[0] * bb[1];
    F[3] = velocity * u[3] - bb[0] * bb[2];
}

// 'totsnd' pressure and the freezing-speed candidate |p_X / rho| + c_s of one cell (rotated order).
template <typename T>
__device__ __forceinline__ T press_speed_rot(double G, const T u[5], double msq, T& p) {
    if constexpr (sizeof(T) == 4) {
        PressOutF o = pressure_totsnd_mixed(G, u[0], u[1], u[2], u[3], u[4], msq);
        p = o.p;
        return fabsf(u[1] * rcp_approx(u[0])) + o.cs;
    } else {
        PressOut o = pressure_totsnd(G, u[0], u[1], u[2], u[3], u[4], msq);
        p = o.p + 0.0;   // + viscosity.solve ('empty' -> 0)
        return fabs(u[1] * (1.0 / u[0])) + o.cs;
    }
}

// The same, also returning the 'totsnd' sound speed (the Neumann-Richtmyer viscosity reads it).
template <typename T>
__device__ __forceinline__ T press_speed_rot(double G, const T u[5], double msq, T& p, T& cs) {
    if constexpr (sizeof(T) == 4) {
        PressOutF o = pressure_totsnd_mixed(G, u[0], u[1], u[2], u[3], u[4], msq);
        p = o.p;
        cs = o.cs;
        return fabsf(u[1] * rcp_approx(u[0])) + o.cs;
    } else {
        PressOut o = pressure_totsnd(G, u[0], u[1], u[2], u[3], u[4], msq);
        p = o.p;
        cs = o.cs;
        return fabs(u[1] * (1.0 / u[0])) + o.cs;
    }
}

// ---- artificial viscosity (fluid/ArtificialViscosity.m) in the segment layout ---------------------
// Computed in FP64 for both forms, with explicit round-to-nearest products and sums (no FMA
// contraction), in the reference's operation order.  The stage's state is the one wFluidFlux.m
// receives: the primaries for the predictor, the half-step stores for the corrector; the viscous term
// is added to the 'totsnd' pressure after the freezing speed is taken (wFluidFlux.m:18-24).

// cswSoundSpeed's per-cell sound speed (ArtificialViscosity.m:157-190) from the natural-order
// momentum and cell-centred B of one cell.  As the reference writes it, only the z momentum of the
// velocity-squared sum is divided by rho^2, and every B component counts (no isZero test).
__device__ __forceinline__ double csw_cell_sound(double G, double rho, double px, double py, double pz, double E,
                                                 double bx, double by, double bz) {
    const double vel_sq = __dadd_rn(__dadd_rn(__dmul_rn(px, px), __dmul_rn(py, py)), __dmul_rn(pz, pz) / __dmul_rn(rho, rho));
    const double mag_sq = __dadd_rn(__dadd_rn(__dmul_rn(bx, bx), __dmul_rn(by, by)), __dmul_rn(bz, bz));
    double s = __dmul_rn(G - 1.0, __dsub_rn(E, __dmul_rn(__dmul_rn(0.5, rho), vel_sq)));
    s = __dsub_rn(s, __dmul_rn(__dmul_rn(G - 1.0, 0.5), mag_sq));
    return sqrt(fabs(__dadd_rn(__dmul_rn(G, s), __dmul_rn(2.0, mag_sq)) / rho));
}

// Per-cell viscosity inputs of one stage and their exchange set V ([VISC_ROWS][NT] FP64): v = p_X/rho
// of cells 0, 1, C-2, C-1 (rows 0-3), rho of cells 0 and C-1 (rows 4-5), the CSW cell sound speed of
// cells 0 and C-1 (rows 6-7) and p_X of cell 0 (row 8).  w holds the stage state in sweep-rotated order;
// (nx, ny, nz) give the rotated slot (0-2) of the natural components.
template <typename T, int C, int VT>
__device__ __forceinline__ void seg_visc_publish(const T (&w)[5][C], const T (&bb)[3][C], double G, int nx, int ny, int nz,
                                                 double* V, int NT, int t, double (&vel)[C], double (&snd)[C]) {
    static_assert(C >= 2, "the viscosity stencil reaches 2 cells: at least 2 cells per thread");
#pragma unroll
    for (int k = 0; k < C; ++k) {
        vel[k] = (double)w[1][k] / (double)w[0][k];
        if constexpr (VT == VISC_CSW) {
            const double p[3] = {(double)w[1][k], (double)w[2][k], (double)w[3][k]};
            const double b[3] = {(double)bb[0][k], (double)bb[1][k], (double)bb[2][k]};
            auto pick = [](const double (&a)[3], int s) { return s == 0 ? a[0] : (s == 1 ? a[1] : a[2]); };
            snd[k] = csw_cell_sound(G, (double)w[0][k], pick(p, nx), pick(p, ny), pick(p, nz), (double)w[4][k],
                                    pick(b, nx), pick(b, ny), pick(b, nz));
        } else {
            snd[k] = 0.0;
        }
    }
    if constexpr (VT == VISC_CSW) {
        V[0 * NT + t] = vel[0];
        V[1 * NT + t] = vel[1];
        V[2 * NT + t] = vel[C - 2];
        V[3 * NT + t] = vel[C - 1];
        V[4 * NT + t] = (double)w[0][0];
        V[5 * NT + t] = (double)w[0][C - 1];
        V[6 * NT + t] = snd[0];
        V[7 * NT + t] = snd[C - 1];
    } else {
        V[8 * NT + t] = (double)w[1][0];
    }
}

// The viscous pressure q of the C own cells (after the barrier that follows seg_visc_publish).  lt/rt:
// the threads of the neighbour segments; lo_own/hi_own: a const pencil end (its ghosts are the end
// cell, constant_shift.m); cs: the 'totsnd' sound speed of each cell (Neumann-Richtmyer).
template <typename T, int C, int VT>
__device__ __forceinline__ void seg_visc_terms(const FluidArgs& a, double G, const T (&w)[5][C], const T (&cs)[C],
                                               const double (&vel)[C], const double (&snd)[C], const double* V, int NT,
                                               int lt, int rt, bool lo_own, bool hi_own, double (&q)[C]) {
    if constexpr (VT == VISC_NR) {
        // viscousMagnitude = min(p_X.shift(X, 1) - p_X, 0); q = vm (c1 c_s + c2 vm / rho)
#pragma unroll
        for (int k = 0; k < C; ++k) {
            const double pn = k + 1 < C ? (double)w[1][k + 1] : (hi_own ? (double)w[1][C - 1] : V[8 * NT + rt]);
            const double vm = fmin(__dsub_rn(pn, (double)w[1][k]), 0.0);
            q[k] = __dmul_rn(vm, __dadd_rn(__dmul_rn(a.vc1, (double)cs[k]), __dmul_rn(a.vc2, vm) / (double)w[0][k]));
        }
    } else {
        double vv[C + 4], rr[C + 2], ss[C + 2];   // cells -2 .. C+1 and -1 .. C
#pragma unroll
        for (int k = 0; k < C; ++k) {
            vv[k + 2] = vel[k];
            rr[k + 1] = (double)w[0][k];
            ss[k + 1] = snd[k];
        }
        vv[1] = lo_own ? vel[0] : V[3 * NT + lt];
        vv[0] = lo_own ? vel[0] : V[2 * NT + lt];
        rr[0] = lo_own ? rr[1] : V[5 * NT + lt];
        ss[0] = lo_own ? ss[1] : V[7 * NT + lt];
        vv[C + 2] = hi_own ? vel[C - 1] : V[0 * NT + rt];
        vv[C + 3] = hi_own ? vel[C - 1] : V[1 * NT + rt];
        rr[C + 1] = hi_own ? rr[C] : V[4 * NT + rt];
        ss[C + 1] = hi_own ? ss[C] : V[6 * NT + rt];
#pragma unroll
        for (int k = 0; k < C; ++k) {
            const double mb = rr[k], mc = rr[k + 2];
            const double rho = __dmul_rn(__dmul_rn(2.0, mc), mb) / __dadd_rn(mc, mb);   // averaged density
            const double c = fmax(fmin(ss[k], ss[k + 2]), 0.0);                           // cswSoundSpeed
            const double v0 = vv[k], v1 = vv[k + 1], v2 = vv[k + 3], v3 = vv[k + 4];
            const double dv = __dsub_rn(v2, v1);
            const double rl = __dsub_rn(v3, v2) / __dmul_rn(2.0, dv);
            const double rr_ = __dsub_rn(v1, v0) / __dmul_rn(2.0, dv);
            const double lim = fmax(0.0, fmin(fmin(__dmul_rn(0.5, __dadd_rn(rl, rr_)),
                                                   fmin(__dmul_rn(2.0, rl), __dmul_rn(2.0, rr_))), 1.0));
            const double adv = fabs(dv);
            const double root = sqrt(__dadd_rn(__dmul_rn(a.vk2, __dmul_rn(dv, dv)), __dmul_rn(a.vc1sq, __dmul_rn(c, c))));
            const double mag = __dadd_rn(__dmul_rn(a.vk1, adv) / 4.0, root);
            q[k] = __dmul_rn(__dmul_rn(__dmul_rn(__dmul_rn(dv < 0.0 ? 1.0 : 0.0, rho), mag), __dsub_rn(1.0, lim)), adv);
        }
    }
}

// press + viscosity.solve: in FP64 the reference's sum; in the mixed form the FP32 pressure plus the
// rounded viscous term.
template <typename T>
__device__ __forceinline__ T visc_add(T p, double q) {
    if constexpr (sizeof(T) == 4) return p + (float)q;
    else return __dadd_rn(p, q);
}

// Corrector (relaxingFluid.m:52-71) of one variable over a segment: R* = (u* + F*/c_f*)/2 and
// L* = (u* - F*/c_f*)/2 at cells -2 .. C+1 (neighbour cells from the published exchange set X2), the
// TVD limiter at cells -1 .. C (only those the update reads), and the update of the C own cells.
// LIM: the launch's limiter (flux/*Limiter.m), fixed at compile time.  X2l/X2r: the exchange sets that
// hold the left and right neighbour segments (another CTA's, through DSMEM, across a cluster).
// nown < C: a ragged last segment with a const end after cell nown - 1 (its cells beyond hold copies of
// that cell's state), whose limited L takes the end cell's value one cell past it.
template <typename T, int C, int LIM>
__device__ __forceinline__ void seg_correct(const T (&u)[C], const T (&us)[C], const T (&Fs)[C], const T* X2l,
                                            const T* X2r, int NT, int lt, int rt, bool lo_own, bool hi_own, T ics,
                                            T ffc, T (&unew)[C], int nown = C) {
    const T* X2v = X2l;
    T Rs[C + 4], Ls[C + 4];
#pragma unroll
    for (int k = 0; k < C; ++k) {
        const T w = Fs[k] * ics;
        Rs[k + 2] = T(0.5) * (us[k] + w);
        Ls[k + 2] = T(0.5) * (us[k] - w);
    }
    if (lo_own) {
        Rs[1] = Rs[2]; Ls[1] = Ls[2];
        Rs[0] = Rs[2]; Ls[0] = Ls[2];
    } else {   // X2v holds [u*, F*] x [cell 0, cell 1, cell C-2, cell C-1] at strides of 5*NT
        const T u1 = X2v[30 * NT + lt], w1 = X2v[35 * NT + lt] * ics;   // left's last cell
        const T u2 = X2v[20 * NT + lt], w2 = X2v[25 * NT + lt] * ics;   // left's cell C-2
        Rs[1] = T(0.5) * (u1 + w1); Ls[1] = T(0.5) * (u1 - w1);
        Rs[0] = T(0.5) * (u2 + w2); Ls[0] = T(0.5) * (u2 - w2);
    }
    if (hi_own) {
        Rs[C + 2] = Rs[C + 1]; Ls[C + 2] = Ls[C + 1];
        Rs[C + 3] = Rs[C + 1]; Ls[C + 3] = Ls[C + 1];
    } else {
        const T u1 = X2r[rt], w1 = X2r[5 * NT + rt] * ics;                // right's first cell
        const T u2 = X2r[10 * NT + rt], w2 = X2r[15 * NT + rt] * ics;      // right's cell 1
        Rs[C + 2] = T(0.5) * (u1 + w1); Ls[C + 2] = T(0.5) * (u1 - w1);
        Rs[C + 3] = T(0.5) * (u2 + w2); Ls[C + 3] = T(0.5) * (u2 - w2);
    }
    // limited R at cells -1 .. C-1 and limited L at cells 0 .. C (index j + 1)
    T Rl[C + 1], Ll[C + 2];
#pragma unroll
    for (int j = -1; j < C; ++j) {
        const T r = Rs[j + 2];
        Rl[j + 1] = r + limiter_corr_t<LIM>(r - Rs[j + 1], Rs[j + 3] - r);
    }
#pragma unroll
    for (int j = 0; j <= C; ++j) {
        const T l = Ls[j + 2];
        Ll[j + 1] = l + limiter_corr_t<LIM>(Ls[j + 1] - l, l - Ls[j + 3]);
    }
    if (lo_own) Rl[0] = Rl[1];   // the limited flux's own const ghost
    if (hi_own) Ll[C + 1] = Ll[C];
    if (nown < C) {               // ragged end: the ghost one past cell nown - 1
        T e = Ll[1];
#pragma unroll
        for (int j = 1; j < C; ++j)
            if (j == nown) e = Ll[j];
#pragma unroll
        for (int j = 2; j <= C; ++j)
            if (j == nown + 1) Ll[j] = e;
    }
#pragma unroll
    for (int k = 0; k < C; ++k) unew[k] = u[k] - ffc * (Rl[k + 1] - Rl[k] + Ll[k + 1] - Ll[k + 2]);
}

// Pencil maximum of non-negative speeds in the segment layout.  publish: reduce over the lanes of the
// pencil inside the warp and leave the warp's value in pm where a pencil spans warps; collect, after
// a barrier, reduces those.  Along x the S segments of a pencil are consecutive lanes (S a power of
// two below 32, or a multiple of 32); along y and z the lanes of pencil b are b, b + Wb, ... (Wb a
// power of two, at most 32 when S > 1).  With S = 1 (a short pencil held whole by one thread, Wb up to
// the CTA) the thread's own maximum is the pencil's.
template <typename T>
__device__ __forceinline__ T seg_max_publish(const SweepGeom& g, T v, T* pm) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const unsigned full = 0xffffffffu;
    if (g.G == 1) return v;
    if (g.d == 0) {
        if (g.G >= 32) {
            v = warp_max_nonneg(v);
            if (lane == 0) pm[warp * 32] = v;
        } else {
            for (int o = g.G / 2; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(full, v, o));
        }
        return v;
    }
    for (int o = 16; o >= g.Wb; o >>= 1) v = fmax(v, __shfl_xor_sync(full, v, o));
    if (lane < g.Wb) pm[warp * 32 + lane] = v;
    return v;
}

template <typename T>
__device__ __forceinline__ T seg_max_collect(const SweepGeom& g, int b, T wv, const T* pm) {
    const int lane = threadIdx.x & 31;
    if (g.G == 1) return wv;
    if (g.d == 0) {
        if (g.G < 32) return wv;
        const int w0 = (b * g.G) >> 5, nw = g.G >> 5;
        return warp_max_nonneg(lane < nw ? pm[(w0 + lane) * 32] : T(0));
    }
    T m = T(0);
    const int nw = g.NT >> 5;
    for (int w = 0; w < nw; ++w) m = fmax(m, pm[w * 32 + b]);
    return m;
}

// Stage barrier of the segment kernel: the cluster's where a pencil spans a cluster.
template <bool CLU>
__device__ __forceinline__ void sp_sync(const SweepGeom& g) {
    if (CLU && g.CL > 1) cluster_sync();
    else __syncthreads();
}

// Pencil maximum for one pencil over a cluster (init_cluster placement): publish leaves each warp's
// maximum in pm; collect, after a barrier, reduces the CTA's warps and, with CL > 1, the CTAs' maxima
// through DSMEM (slot `slot` of cm) behind one more cluster barrier.  All threads call both.
template <typename T>
__device__ __forceinline__ void clu_max_publish(T v, T* pm) {
    v = warp_max_nonneg(v);
    if ((threadIdx.x & 31) == 0) pm[(threadIdx.x >> 5) * 32] = v;
}

template <typename T>
__device__ __forceinline__ T clu_max_collect(const SweepGeom& g, const T* pm, T* cm, int slot) {
    const int lane = threadIdx.x & 31;
    const T m = warp_max_nonneg(lane < (g.NT >> 5) ? pm[lane * 32] : T(0));
    if (g.CL == 1) return m;
    if (threadIdx.x == 0) cm[slot] = m;
    cluster_sync();
    T c = T(0);
    if (lane < g.CL) c = cg::this_cluster().map_shared_rank(cm, lane)[slot];
    return warp_max_nonneg(c);
}

// VT: the artificial viscosity (VISC_*), fixed per kernel.  With viscosity each of the first two
// stages takes one more barrier: the viscosity exchange set is published with the pencil maximum, and
// the flux numerators (which include the viscous pressure) are published after it.
// CLU: one pencil along x per cluster of CL CTAs (CL = 1: one CTA), placed by SegPos::init_cluster:
// the exchanges with segments in another CTA read its shared memory through DSMEM, the barriers and the
// pencil maxima span the cluster, and a length that C does not divide leaves the last segment ragged
// (const ends only: its cells past the pencil's end load the end cell and, after the predictor, take the
// end cell's half-step state, the const ghosts of every shifted array).
template <typename T, bool MHD, int C, int VT, bool CLU = false>
__device__ __forceinline__ void fluid_seg_body(const FluidArgs& a, unsigned vblock) {
    static_assert(!CLU || VT == VISC_NONE, "cluster segments carry no viscosity");
    extern __shared__ __align__(16) unsigned char smem[];
    pdl_wait();
    // cluster launches return on `done` only, as fluid_sweep_body_general's do
    if (a.tm->done || (a.sg.CL == 1 && a.tm->error)) return;
    __shared__ double cflp[3][MAX_WARPS];
    __shared__ T cmax[2];
    const SweepGeom& g = a.sg;
    const int NT = g.NT, S = g.G, d = g.d, d1 = g.d1, d2 = g.d2;
    const int N = g.N;
    const int t = threadIdx.x;
    SegPos sp;
    if constexpr (CLU) sp.init_cluster(g, vblock);
    else sp.init(g, vblock);
    const int s = sp.s;
    T* X1 = reinterpret_cast<T*>(smem);   // [20][NT]: (u, F) of the first cell, then of the last
    T* X2 = X1 + 20 * NT;                 // [40][NT]: (u*, F*) of cells 0, 1, C-2, C-1
    T* PM = X2 + 40 * NT;                 // [2][NT/32][32]: per-warp pencil maxima
    double* V = reinterpret_cast<double*>(PM + 2 * (NT >> 5) * 32);   // [VISC_ROWS][NT] (viscosity only)
    const bool circ_lo = a.mode[CLS_MASS][0] == BC_CIRC, circ_hi = a.mode[CLS_MASS][1] == BC_CIRC;
    const int ls = d == 0 ? 1 : g.Wb;     // thread distance between consecutive segments of a pencil
    const bool lo_own = s == 0 && !circ_lo, hi_own = s == S - 1 && !circ_hi;
    int lt = s > 0 ? t - ls : (circ_lo ? t + (S - 1) * ls : t);
    int rt = s < S - 1 ? t + ls : (circ_hi ? t - (S - 1) * ls : t);
    // the exchange sets holding the neighbour segments (another rank's across a cluster)
    const T* X1l = X1;
    const T* X1r = X1;
    const T* X2l = X2;
    const T* X2r = X2;
    int nown = C;   // own cells inside the pencil (a ragged last segment: fewer; idle threads: none)
    if constexpr (CLU) {
        const int sc = s < S ? s : S - 1;   // idle threads read a real segment's neighbours
        const int sl = sc > 0 ? sc - 1 : (circ_lo ? S - 1 : sc);
        const int sr = sc < S - 1 ? sc + 1 : (circ_hi ? 0 : sc);
        const int rl = sl / NT, rr = sr / NT;
        lt = sl - rl * NT;
        rt = sr - rr * NT;
        if (rl != sp.rank) {
            X1l = cg::this_cluster().map_shared_rank(X1, rl);
            X2l = cg::this_cluster().map_shared_rank(X2, rl);
        }
        if (rr != sp.rank) {
            X1r = cg::this_cluster().map_shared_rank(X1, rr);
            X2r = cg::this_cluster().map_shared_rank(X2, rr);
        }
        nown = N - s * C < C ? N - s * C : C;
    }
    const double G = a.gamma;
    const double dt = a.tm->dt;
    const T ff = (T)(dt / a.dx);
    const T half_ffx = (T)(0.5 * (dt / a.dx));
    // vector accesses need segments on multiples of C: pencils start on one where C divides N
    const bool vec = d == 0 && (!CLU || N % C == 0);
    const bool ragged = CLU && nown < C;   // cells past the pencil's end: load (and later take) the end cell
    const long long o0 = sp.base + (long long)s * C * g.sd;
    // momentum and cell-centred B in sweep-rotated order: component 0 along the sweep, then d1, d2
    void* qv[5] = {a.q[Q_RHO], a.q[Q_PX + d], a.q[Q_PX + d1], a.q[Q_PX + d2], a.q[Q_E]};
    const bool ub[3] = {a.use_b[d] != 0, a.use_b[d1] != 0, a.use_b[d2] != 0};
    // rotated slots of the natural x, y, z components (the CSW sound speed sums in natural order)
    const int nx = d == 0 ? 0 : (d1 == 0 ? 1 : 2), ny = d == 1 ? 0 : (d1 == 1 ? 1 : 2), nz = d == 2 ? 0 : (d1 == 2 ? 1 : 2);
    constexpr bool LOADB = MHD || VT == VISC_CSW;   // cswSoundSpeed reads every cell-centred component

    // ---- stage 1: load, pressure, speed, F -------------------------------------------------------
    T u[5][C], bb[3][C], F[5][C];
    // sum of squares of the cell-centred B components without isZero, in rotated order (recomputed
    // where needed instead of kept: it would hold 2C registers for the whole kernel)
    auto bsq = [&](const T (&b)[3][C], int k) {
        double m = 0.0;
#pragma unroll
        for (int c = 0; c < 3; ++c)
            if (MHD && ub[c]) m = m + (double)b[c][k] * (double)b[c][k];
        return m;
    };
    if (sp.colok && ragged) {
#pragma unroll
        for (int k = 0; k < C; ++k) {
            const long long o = sp.base + (long long)(k < nown ? s * C + k : N - 1) * g.sd;
#pragma unroll
            for (int v = 0; v < 5; ++v) u[v][k] = ldq<T>(qv[v], o);
            if (LOADB) {
                bb[0][k] = ldq<T>(a.q[Q_CBX + d], o);
                bb[1][k] = ldq<T>(a.q[Q_CBX + d1], o);
                bb[2][k] = ldq<T>(a.q[Q_CBX + d2], o);
            } else {
                bb[0][k] = bb[1][k] = bb[2][k] = T(0);
            }
        }
    } else if (sp.colok) {
#pragma unroll
        for (int v = 0; v < 5; ++v) seg_load<T, C>(qv[v], o0, g.sd, vec, u[v]);
        if (LOADB) {
            seg_load<T, C>(a.q[Q_CBX + d], o0, g.sd, vec, bb[0]);
            seg_load<T, C>(a.q[Q_CBX + d1], o0, g.sd, vec, bb[1]);
            seg_load<T, C>(a.q[Q_CBX + d2], o0, g.sd, vec, bb[2]);
        } else {
#pragma unroll
            for (int k = 0; k < C; ++k) bb[0][k] = bb[1][k] = bb[2][k] = T(0);
        }
    } else {
#pragma unroll
        for (int k = 0; k < C; ++k) {
            u[0][k] = T(1);
            u[1][k] = u[2][k] = u[3][k] = u[4][k] = T(0);
            bb[0][k] = bb[1][k] = bb[2][k] = T(0);
        }
    }
    T lmax = T(0);
    T cf;
    if constexpr (VT == VISC_NONE) {
#pragma unroll
        for (int k = 0; k < C; ++k) {
            const double m = bsq(bb, k);
            const T uu[5] = {u[0][k], u[1][k], u[2][k], u[3][k], u[4][k]};
            const T b3[3] = {bb[0][k], bb[1][k], bb[2][k]};
            T p;
            const T spd = press_speed_rot<T>(G, uu, m, p);
            if (sp.colok) lmax = fmax(lmax, spd);
            T Fk[5];
            flux_num_rot<T>(uu, b3, p, Fk);
#pragma unroll
            for (int v = 0; v < 5; ++v) F[v][k] = Fk[v];
        }
#pragma unroll
        for (int v = 0; v < 5; ++v) {
            X1[v * NT + t] = u[v][0];
            X1[(5 + v) * NT + t] = F[v][0];
            X1[(10 + v) * NT + t] = u[v][C - 1];
            X1[(15 + v) * NT + t] = F[v][C - 1];
        }
        if constexpr (CLU) {
            clu_max_publish(lmax, PM);
            sp_sync<CLU>(g);
            cf = clu_max_collect(g, PM, cmax, 0);   // freezing speed (wFluidFlux.m:18-22)
        } else {
            const T wv1 = seg_max_publish(g, lmax, PM);
            __syncthreads();
            cf = seg_max_collect(g, sp.b, wv1, PM);   // freezing speed (wFluidFlux.m:18-22)
        }
    } else {
        T P[C], CS[C];
        double vel[C], snd[C], q[C];
#pragma unroll
        for (int k = 0; k < C; ++k) {
            const double m = bsq(bb, k);
            const T uu[5] = {u[0][k], u[1][k], u[2][k], u[3][k], u[4][k]};
            const T spd = press_speed_rot<T>(G, uu, m, P[k], CS[k]);
            if (sp.colok) lmax = fmax(lmax, spd);
        }
        seg_visc_publish<T, C, VT>(u, bb, G, nx, ny, nz, V, NT, t, vel, snd);
        const T wv1 = seg_max_publish(g, lmax, PM);
        __syncthreads();
        cf = seg_max_collect(g, sp.b, wv1, PM);   // freezing speed (wFluidFlux.m:18-22), before the viscosity
        seg_visc_terms<T, C, VT>(a, G, u, CS, vel, snd, V, NT, lt, rt, lo_own, hi_own, q);
#pragma unroll
        for (int k = 0; k < C; ++k) {
            const T uu[5] = {u[0][k], u[1][k], u[2][k], u[3][k], u[4][k]};
            const T b3[3] = {MHD ? bb[0][k] : T(0), MHD ? bb[1][k] : T(0), MHD ? bb[2][k] : T(0)};
            T Fk[5];
            flux_num_rot<T>(uu, b3, visc_add<T>(P[k], q[k]), Fk);   // press + viscosity.solve (wFluidFlux.m:24)
#pragma unroll
            for (int v = 0; v < 5; ++v) F[v][k] = Fk[v];
        }
#pragma unroll
        for (int v = 0; v < 5; ++v) {
            X1[v * NT + t] = u[v][0];
            X1[(5 + v) * NT + t] = F[v][0];
            X1[(10 + v) * NT + t] = u[v][C - 1];
            X1[(15 + v) * NT + t] = F[v][C - 1];
        }
        __syncthreads();
    }
    T ic;
    if constexpr (sizeof(T) == 4) ic = __frcp_rn(cf);
    else ic = T(1) / cf;

    // ---- stage 2: predictor (relaxingFluid.m:30-39) and the half-step pressure, speed, F ----------
    T us[5][C], Fs[5][C];
    const T hfc = half_ffx * cf;
#pragma unroll
    for (int v = 0; v < 5; ++v) {
        // R = (u + F/c_f)/2 at cells -1 .. C-1 (index j + 1), L = (u - F/c_f)/2 at cells 0 .. C (index j)
        T R[C + 1], L[C + 1];
#pragma unroll
        for (int k = 0; k < C; ++k) {
            const T w = F[v][k] * ic;
            R[k + 1] = T(0.5) * (u[v][k] + w);
            L[k] = T(0.5) * (u[v][k] - w);
        }
        R[0] = lo_own ? R[1] : T(0.5) * (X1l[(10 + v) * NT + lt] + X1l[(15 + v) * NT + lt] * ic);
        L[C] = hi_own ? L[C - 1] : T(0.5) * (X1r[v * NT + rt] - X1r[(5 + v) * NT + rt] * ic);
#pragma unroll
        for (int k = 0; k < C; ++k) us[v][k] = u[v][k] - hfc * (R[k + 1] - R[k] + L[k] - L[k + 1]);
        if (ragged && nown > 0) {   // cells past the end take the end cell's half-step state
            T e = us[v][0];
#pragma unroll
            for (int k = 1; k < C; ++k)
                if (k == nown - 1) e = us[v][k];
#pragma unroll
            for (int k = 1; k < C; ++k)
                if (k >= nown) us[v][k] = e;
        }
    }
    T lmax2 = T(0);
    T P2[C], CS2[C];
#pragma unroll
    for (int k = 0; k < C; ++k) {
        us[0][k] = us[0][k] > (T)a.minmass ? us[0][k] : (T)a.minmass;   // max(rho, MINMASS), NaN -> MINMASS
        if (!sp.colok) { us[0][k] = T(1); us[1][k] = us[2][k] = us[3][k] = us[4][k] = T(0); }
        const T uu[5] = {us[0][k], us[1][k], us[2][k], us[3][k], us[4][k]};
        if constexpr (VT == VISC_NONE) {
            const T b3[3] = {bb[0][k], bb[1][k], bb[2][k]};
            T p2;
            const T spd = press_speed_rot<T>(G, uu, bsq(bb, k), p2);   // relaxingFluid.m:47-50
            if (sp.colok) lmax2 = fmax(lmax2, spd);
            T Fk[5];
            flux_num_rot<T>(uu, b3, p2, Fk);
#pragma unroll
            for (int v = 0; v < 5; ++v) Fs[v][k] = Fk[v];
        } else {
            const T spd = press_speed_rot<T>(G, uu, bsq(bb, k), P2[k], CS2[k]);
            if (sp.colok) lmax2 = fmax(lmax2, spd);
        }
    }
    if constexpr (VT != VISC_NONE) {
        // the viscosity of the half-step state: one more barrier before its fluxes are published
        double vel[C], snd[C], q[C];
        seg_visc_publish<T, C, VT>(us, bb, G, nx, ny, nz, V, NT, t, vel, snd);
        const T wv2 = seg_max_publish(g, lmax2, PM + (NT >> 5) * 32);
        __syncthreads();
        lmax2 = seg_max_collect(g, sp.b, wv2, PM + (NT >> 5) * 32);
        seg_visc_terms<T, C, VT>(a, G, us, CS2, vel, snd, V, NT, lt, rt, lo_own, hi_own, q);
#pragma unroll
        for (int k = 0; k < C; ++k) {
            const T uu[5] = {us[0][k], us[1][k], us[2][k], us[3][k], us[4][k]};
            const T b3[3] = {MHD ? bb[0][k] : T(0), MHD ? bb[1][k] : T(0), MHD ? bb[2][k] : T(0)};
            T Fk[5];
            flux_num_rot<T>(uu, b3, visc_add<T>(P2[k], q[k]), Fk);
#pragma unroll
            for (int v = 0; v < 5; ++v) Fs[v][k] = Fk[v];
        }
    }
    const int c1 = C > 1 ? 1 : 0;
#pragma unroll
    for (int v = 0; v < 5; ++v) {
        X2[v * NT + t] = us[v][0];
        X2[(5 + v) * NT + t] = Fs[v][0];
        X2[(10 + v) * NT + t] = us[v][c1];
        X2[(15 + v) * NT + t] = Fs[v][c1];
        X2[(20 + v) * NT + t] = us[v][C - 1 - c1];
        X2[(25 + v) * NT + t] = Fs[v][C - 1 - c1];
        X2[(30 + v) * NT + t] = us[v][C - 1];
        X2[(35 + v) * NT + t] = Fs[v][C - 1];
    }
    T cfs;   // freezing speed of the half step
    if constexpr (CLU) {
        clu_max_publish(lmax2, PM + (NT >> 5) * 32);
        sp_sync<CLU>(g);
        cfs = clu_max_collect(g, PM + (NT >> 5) * 32, cmax, 1);
    } else if constexpr (VT == VISC_NONE) {
        const T wv2 = seg_max_publish(g, lmax2, PM + (NT >> 5) * 32);
        __syncthreads();
        cfs = seg_max_collect(g, sp.b, wv2, PM + (NT >> 5) * 32);
    } else {
        __syncthreads();
        cfs = lmax2;
    }
    T ics;
    if constexpr (sizeof(T) == 4) ics = __frcp_rn(cfs);
    else ics = T(1) / cfs;

    pdl_trigger();
    // ---- stage 3: corrector fluxes, TVD limiter, update (relaxingFluid.m:52-71) -------------------
    T unew[5][C];
    const T ffc = ff * cfs;
#pragma unroll
    for (int v = 0; v < 5; ++v) {
        const T* Xl = X2l + v * NT;
        const T* Xr = X2r + v * NT;
        const int nc = CLU ? nown : C;
        if (a.limiter == LIM_VANLEER)
            seg_correct<T, C, LIM_VANLEER>(u[v], us[v], Fs[v], Xl, Xr, NT, lt, rt, lo_own, hi_own, ics, ffc, unew[v], nc);
        else if (a.limiter == LIM_SUPERBEE)
            seg_correct<T, C, LIM_SUPERBEE>(u[v], us[v], Fs[v], Xl, Xr, NT, lt, rt, lo_own, hi_own, ics, ffc, unew[v], nc);
        else
            seg_correct<T, C, LIM_MINMOD>(u[v], us[v], Fs[v], Xl, Xr, NT, lt, rt, lo_own, hi_own, ics, ffc, unew[v], nc);
    }
    // the other ranks have read this CTA's exchange sets before it moves on (and may exit)
    if (CLU && g.CL > 1) cluster_sync();
    double m3[3] = {0.0, 0.0, 0.0};   // rotated order
    bool bad = false;
    T cb[3][C];   // the CFL pass reloads the cell-centred B (cache hits; one sweep in six)
    if (a.cfl && sp.colok && MHD && ragged) {
#pragma unroll
        for (int k = 0; k < C; ++k) {
            const long long o = sp.base + (long long)(k < nown ? s * C + k : N - 1) * g.sd;
            cb[0][k] = ldq<T>(a.q[Q_CBX + d], o);
            cb[1][k] = ldq<T>(a.q[Q_CBX + d1], o);
            cb[2][k] = ldq<T>(a.q[Q_CBX + d2], o);
        }
    } else if (a.cfl && sp.colok && MHD) {
        seg_load<T, C>(a.q[Q_CBX + d], o0, g.sd, vec, cb[0]);
        seg_load<T, C>(a.q[Q_CBX + d1], o0, g.sd, vec, cb[1]);
        seg_load<T, C>(a.q[Q_CBX + d2], o0, g.sd, vec, cb[2]);
    }
#pragma unroll
    for (int k = 0; k < C; ++k) {
        unew[0][k] = unew[0][k] > (T)a.minmass_out ? unew[0][k] : (T)a.minmass_out;
        if (a.cfl && sp.colok && k < nown) {   // fused CFL maxima of the new state (TimeManager.m:65-77)
            double sp3[3];
            cfl_speeds(G, (double)unew[0][k], (double)unew[1][k], (double)unew[2][k], (double)unew[3][k],
                       (double)unew[4][k], MHD ? bsq(cb, k) : 0.0, sp3);
            bad = bad || !isfinite(sp3[0] + sp3[1] + sp3[2]);
#pragma unroll
            for (int c = 0; c < 3; ++c) m3[c] = fmax(m3[c], sp3[c]);
        }
    }
    if (sp.colok && ragged) {
#pragma unroll
        for (int k = 0; k < C; ++k)
            if (k < nown)
#pragma unroll
                for (int v = 0; v < 5; ++v) stq<T>(qv[v], o0 + (long long)k * g.sd, unew[v][k]);
    } else if (sp.colok) {
#pragma unroll
        for (int v = 0; v < 5; ++v) seg_store<T, C>(qv[v], o0, g.sd, vec, unew[v]);
    }
    if (a.cfl) {
        if (a.cfl & CFL_CHECK_NONFINITE) flag_nonfinite(a.tm, bad);
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            m3[c] = warp_max_nonneg(m3[c]);
            if (lane == 0) cflp[c][warp] = m3[c];
        }
        __syncthreads();
        if (threadIdx.x < 3) {   // one global atomic per CTA and direction (rotated slot of direction t)
            const int rc = threadIdx.x == d ? 0 : (threadIdx.x == d1 ? 1 : 2);
            double m = 0.0;
            for (int w = 0; w < (int)(blockDim.x >> 5); ++w) m = fmax(m, cflp[rc][w]);
            atomic_max_nonneg(&a.tm->maxbits[threadIdx.x], m);
        }
    }
}

template <typename T, bool MHD, int C, int VT = VISC_NONE>
__global__ void __launch_bounds__(512, 1) fluid_seg_kernel(const __grid_constant__ FluidArgs a) {
    fluid_seg_body<T, MHD, C, VT>(a, blockIdx.x);
}

template <typename T, bool MHD, int C>
__global__ void __launch_bounds__(512, 1) fluid_seg_batch_kernel(const FluidArgs* __restrict__ args,
                                                                  const BlockMap* __restrict__ map) {
    __shared__ FluidArgs sa;
    const BlockMap bm = map[blockIdx.x];
    load_member_args(sa, args + bm.member);
    __syncthreads();
    fluid_seg_body<T, MHD, C, VISC_NONE>(sa, (unsigned)bm.block);
}

// One pencil along x per cluster of CTAs, or per CTA with a ragged last segment (fluid_seg_body's CLU).
template <typename T, bool MHD, int C>
__global__ void __launch_bounds__(512, 1) fluid_seg_clu_kernel(const __grid_constant__ FluidArgs a) {
    fluid_seg_body<T, MHD, C, VISC_NONE, true>(a, blockIdx.x);
}

template <typename T, bool MHD, int C>
__global__ void __launch_bounds__(512, 1) fluid_seg_clu_batch_kernel(const FluidArgs* __restrict__ args,
                                                                      const BlockMap* __restrict__ map) {
    __shared__ FluidArgs sa;
    const BlockMap bm = map[blockIdx.x];
    load_member_args(sa, args + bm.member);
    __syncthreads();
    fluid_seg_body<T, MHD, C, VISC_NONE, true>(sa, (unsigned)bm.block);
}

}  // namespace img
