// Magnet sweep along X for the two transverse components (magnet/magnetFlux.m:14-31,
// magnet/relaxingMagnet.m:15-60, magnet/MagnetArray.m:36-38).
//
// The general path is five launches:
//   mag_chain  -- per X-pencil and component I: corner velocity (transverse average, then the
//                 1-2-1 smoothing along X), upwind predictor, TVD corrector, B_I update.  Writes
//                 B_I in place and the limited flux F_I to scratch.  Both components in one launch.
//   mag_ct1    -- C_I = F_I - F_I.shift(I,+1)                     (relaxingMagnet.m:56)
//   mag_ct2    -- D_I = C_I.shift(X,-1)                           (relaxingMagnet.m:57)
//   mag_bx     -- B_X' = (B_X - dt/dI1 D_I1) - dt/dI2 D_I2 to scratch; cell-centred B_I2
//   mag_cell   -- B_X = B_X'; cell-centred B_X                    (MagnetArray.m:36-38)
// Each pointwise pass reads neighbours of the previous pass's output, so no pass overwrites an
// array that another thread of the same pass still reads.
#pragma once

#include "fluid_sweep.cuh"

namespace img {

struct MagArgs {
    SweepGeom sg;              // sweep along d = X-1
    void* q[NQ];
    void* F[2];                // limited flux per component (scratch)
    void* C[2];                // CT differences per component (scratch)
    void* BXn;                 // new B_X (scratch)
    DevTime* tm;
    int X;                     // 1-based sweep dimension
    int I[2];                  // 1-based transverse components, in the reference's order
    int shiftI[2];             // shifting enabled along dim I (I-1 < ndims)
    double dx;                 // dgrid(X)
    double dI[2];              // dgrid(I)
    int limiter;
    int modeX[2];              // mag-class BC along X (lower, upper)
    int actX;                  // ACTIVE(DIRECT = X) of the mag-class edge store
    int modeI_mass[2][2];      // [component][side] mass-class BC along I
    int modeI_mom[2][2];       // mom-class BC along I
    int modeI_mag[2][2];       // mag-class BC along I
    int actI_mass[2], actI_mom[2], actI_mag[2];
    int modeX_magX[2];         // mag-class BC along X (for mag(X).shift(X,+1)); == modeX
    const double* fade;
    int fade_f;
    double bc_inf;
    const EdgeTable* edges;
    int init_mag[2];           // first assignment of velGrid/store.fluxR/wMag/flux of (I, X)
};

// ---- transverse (non-pencil) shifts used by the pointwise passes ----------------------------------
// Value of A.shift(dim e, n)[cell] for n = -1 or +1, computed from global memory along e.
// mode/act/flip/edge describe the array object; the edge state of a trans edge is drifted and
// written back when `own_update` (exactly one thread per face cell calls with own_update = true).
template <typename T>
__device__ T shift_along(const Geom& g, const T* A, long long cell, int x, int y, int z, int e, int n, int mode,
                         int act, bool flip, double* edge, const double* fc, int f, double bc_inf, bool own_update) {
    const int Ne = sel3(e, g.n[0], g.n[1], g.n[2]);
    const long long se = sel3(e, g.s[0], g.s[1], g.s[2]);
    const int i = sel3(e, x, y, z);
    const long long b = cell - (long long)i * se;   // row 0 of this line along e
    auto at = [&](int j) -> T { return A[b + (long long)j * se]; };
    const bool upper = n > 0;
    const bool is_ghost = upper ? (i == Ne - 1) : (i == 0);
    if (mode == BC_CIRC) return at(((i + n) % Ne + Ne) % Ne);
    if (!is_ghost) {
        T v = at(i + n);
        if (mode == BC_FADE) {
            T s0 = upper ? at(Ne > 1 ? 1 : 0) : at(0);
            T sN1 = upper ? at(Ne - 1) : at(Ne - 2);
            v = fade_apply(v, i, Ne, fc, f, s0, sN1);
        }
        return v;
    }
    long long fi = face_index(g, e, x, y, z);
    switch (mode) {
        case BC_MIRROR: { T v = upper ? at(Ne - 2) : at(1); return flip ? -v : v; }
        case BC_WALL: return (T)edge[fi];
        case BC_TRANS: {
            T a0, a1, a2;
            if (!upper) { a0 = at(trans_pick_lower(Ne, 1, 0)); a1 = at(trans_pick_lower(Ne, 1, 1)); a2 = at(0); }
            else { a0 = at(trans_pick_upper(Ne, 1, 0)); a1 = at(trans_pick_upper(Ne, 1, 1)); a2 = at(Ne - 1); }
            double ev = 0.0;
            if (act) {
                ev = edge_drift(edge[fi], (double)a2);
                if (own_update) edge[fi] = ev;
            }
            return (T)trans_ghost((double)a0, (double)a1, (double)a2, ev, bc_inf, 4.0, (double)a2);
        }
        case BC_FADE: {
            T v = upper ? at(Ne - 1) : at(0);
            T s0 = upper ? at(Ne > 1 ? 1 : 0) : at(0);
            T sN1 = upper ? at(Ne - 1) : at(Ne - 2);
            return fade_apply(v, i, Ne, fc, f, s0, sN1);
        }
        default: return upper ? at(Ne - 1) : at(0);   // const
    }
}

// ---- the X-chain ------------------------------------------------------------------------------------
constexpr int MAG_NSLOT = 2;

template <typename T, int CPT>
struct MagChain {
    using PC = Pencil<T, CPT, MAG_NSLOT, true>;
    const MagArgs& a;
    PC& pc;
    int N;
    __device__ MagChain(const MagArgs& aa, PC& p) : a(aa), pc(p), N(p.sg->N) {}

    // Ghost of a mag-class array at the pencil's lower end for shift(X,-1) (trans: one drift).
    __device__ T ghost_lo(int slot, double* edge, bool own) {
        int mode = a.modeX[0];
        switch (mode) {
            case BC_CIRC: return pc.endv(slot, N - 1);
            case BC_MIRROR: return pc.endv(slot, 1);
            case BC_WALL: return (T)edge[pc.col];
            case BC_TRANS: {
                double ev = 0.0;
                T y0 = pc.endv(slot, trans_pick_lower(N, 1, 0)), y1 = pc.endv(slot, trans_pick_lower(N, 1, 1));
                T y2 = pc.endv(slot, 0);
                if (a.actX) {
                    ev = edge_drift(edge[pc.col], (double)y2);
                    if (own) edge[pc.col] = ev;
                }
                return (T)trans_ghost((double)y0, (double)y1, (double)y2, ev, a.bc_inf, 4.0, (double)y2);
            }
            default: return pc.endv(slot, 0);
        }
    }
    // A.shift(X,-1) at row r (k = segment index) including fade damping.
    __device__ T sm(int slot, const T (&A)[CPT], int k, T glo) {
        int r = pc.r0 + k;
        T v = r == 0 ? glo : pc.prev(slot, A, k);
        if (a.modeX[0] == BC_FADE) v = fade_apply(v, r, N, a.fade, a.fade_f, pc.endv(slot, 0), pc.endv(slot, N - 2));
        return v;
    }
    // Upper ghosts for one shift(X,+m) call given the stored edge value after its drift (ev).
    // Returns the ghost for row N-1 (m=1) or rows N-2, N-1 (m=2) in g[0], g[1].
    __device__ void ghost_hi(int slot, int m, double ev, T g[2]) {
        int mode = a.modeX[1];
        switch (mode) {
            case BC_CIRC:   // rows N, N+1 wrap to 0, 1
                g[0] = pc.endv(slot, 0);
                g[1] = m == 2 ? pc.endv(slot, 1) : g[0];
                return;
            case BC_MIRROR:
                if (m == 1) g[0] = pc.endv(slot, N - 2);
                else { g[0] = pc.endv(slot, N - 2); g[1] = pc.endv(slot, N - 3); }
                return;
            case BC_WALL: g[0] = g[1] = (T)ev; return;
            case BC_TRANS: {
                double y0 = pc.endv(slot, trans_pick_upper(N, m, 0));
                double y1 = pc.endv(slot, trans_pick_upper(N, m, 1));
                double y2 = pc.endv(slot, trans_pick_upper(N, m, 2));
                if (m == 1) {
                    g[0] = (T)trans_ghost(y0, y1, y2, ev, a.bc_inf, 4.0, (double)pc.endv(slot, N - 1));
                } else {
                    g[0] = (T)trans_ghost(y0, y1, y2, ev, a.bc_inf, 4.0, (double)pc.endv(slot, N - 2));
                    g[1] = (T)trans_ghost(y0, y1, y2, ev, a.bc_inf, 5.0, (double)pc.endv(slot, N - 1));
                }
                return;
            }
            default: g[0] = g[1] = pc.endv(slot, N - 1); return;   // const, fade
        }
    }
    // A.shift(X,+m)[r] for this thread's row k given the upper ghosts g of this call.
    __device__ T sp(int slot, const T (&A)[CPT], int k, int m, const T g[2]) {
        int r = pc.r0 + k;
        T v;
        if (r + m <= N - 1) v = m == 1 ? pc.next(slot, A, k) : pc.next2(slot, A, k);
        else v = (m == 1) ? g[0] : g[(r + m) - N];   // m=2: r=N-2 -> g[0], r=N-1 -> g[1]
        if (a.modeX[1] == BC_FADE) {
            T s0 = pc.endv(slot, m < N ? m : N - 1);
            v = fade_apply(v, r, N, a.fade, a.fade_f, s0, pc.endv(slot, N - 1));
        }
        return v;
    }
};

template <typename T, int CPT>
__global__ void __launch_bounds__(512) mag_chain_kernel(const MagArgs a) {
    extern __shared__ __align__(16) unsigned char smem[];
    if (a.tm->done || a.tm->error) return;
    using PC = Pencil<T, CPT, MAG_NSLOT, true>;
    PC pc;
    pc.init(a.sg, smem);
    const int q = blockIdx.y;          // which transverse component
    const int X = a.X, I = q ? a.I[1] : a.I[0];
    const int shiftI = q ? a.shiftI[1] : a.shiftI[0];
    const int mode_mom_lo = q ? a.modeI_mom[1][0] : a.modeI_mom[0][0];
    const int mode_mass_lo = q ? a.modeI_mass[1][0] : a.modeI_mass[0][0];
    const int act_mom = q ? a.actI_mom[1] : a.actI_mom[0];
    const int act_mass = q ? a.actI_mass[1] : a.actI_mass[0];
    const int init_mag = q ? a.init_mag[1] : a.init_mag[0];
    const int d = X - 1, e = I - 1;
    const int N = a.sg.N;
    const Geom& g = a.sg.g;
    const double dt = a.tm->dt;
    const T ff = (T)(0.5 * dt / a.dx);
    const T ff2 = T(2) * ff;
    const EdgeTable* et = a.edges;
    MagChain<T, CPT> mc(a, pc);
    const int c = I - 1;   // component index of mag(I)
    double* e_vg_lo = et->p[mag_obj(c, d, MO_VELGRID)][d][0];
    double* e_vg_hi = et->p[mag_obj(c, d, MO_VELGRID)][d][1];
    double* e_sf_lo = et->p[mag_obj(c, d, MO_STORE_R)][d][0];
    double* e_sf_hi = et->p[mag_obj(c, d, MO_STORE_R)][d][1];
    double* e_wm_lo = et->p[mag_obj(c, d, MO_WMAG)][d][0];
    double* e_wm_hi = et->p[mag_obj(c, d, MO_WMAG)][d][1];
    double* e_fx_lo = et->p[mag_obj(c, d, MO_FLUX)][d][0];
    const bool own0 = pc.nv > 0 && pc.r0 == 0;
    const bool ownN = pc.nv > 0 && pc.r0 + pc.nv - 1 == N - 1;
    const bool ownN2 = pc.nv > 0 && pc.r0 <= N - 2 && pc.r0 + pc.nv - 1 >= N - 2;

    // ---- corner velocity (magnetFlux.m:18-19) --------------------------------------------------
    const T* rho = reinterpret_cast<const T*>(a.q[Q_RHO]);
    const T* pX = reinterpret_cast<const T*>(a.q[Q_PX + d]);
    T* BI = reinterpret_cast<T*>(a.q[Q_BX + c]);
    T vgr[CPT], bI[CPT];
#pragma unroll
    for (int k = 0; k < CPT; ++k) {
        vgr[k] = T(0);
        bI[k] = T(0);
        if (!pc.valid(k)) continue;
        long long o = pc.off(k);
        int x, y, z;
        pc.coords(k, x, y, z);
        T pm, rm;
        if (shiftI) {
            pm = shift_along<T>(g, pX, o, x, y, z, e, -1, mode_mom_lo, act_mom, false,
                                et->p[OBJ_PRIM_MOM + d][e][0], a.fade, a.fade_f, a.bc_inf, true);
            rm = shift_along<T>(g, rho, o, x, y, z, e, -1, mode_mass_lo, act_mass, false,
                                et->p[OBJ_PRIM_MASS][e][0], a.fade, a.fade_f, a.bc_inf, true);
        } else {
            pm = pX[o];
            rm = rho[o];
        }
        vgr[k] = (pm + pX[o]) / (rm + rho[o]);
        bI[k] = BI[o];
    }
    if (init_mag) init_edges(pc, et, mag_obj(c, d, MO_VELGRID), vgr);

    // vg = 0.25*(vg.shift(X,-1) + vg.shift(X,1) + 2*vg)   (magnetFlux.m:21-23)
    double s_vg_hi = 0.0;
    if (ownN && e_vg_hi) s_vg_hi = e_vg_hi[pc.col];
    pc.publish(0, vgr);
    pc.csync();
    T vg[CPT];
    {
        T glo = own0 ? mc.ghost_lo(0, e_vg_lo, true) : T(0);
        T gh[2] = {T(0), T(0)};
        if (ownN) {
            double ev = s_vg_hi;
            if (a.modeX[1] == BC_TRANS && a.actX) ev = edge_drift(ev, (double)pc.endv(0, N - 1));
            mc.ghost_hi(0, 1, ev, gh);
            s_vg_hi = ev;
        }
#pragma unroll
        for (int k = 0; k < CPT; ++k) {
            if (!pc.valid(k)) { vg[k] = T(0); continue; }
            T m1 = mc.sm(0, vgr, k, glo);
            T p1 = mc.sp(0, vgr, k, 1, gh);
            vg[k] = T(0.25) * (m1 + p1 + T(2) * vgr[k]);
        }
    }
    // velocityFlow = (vg + vg.shift(X,1)) < 0   (relaxingMagnet.m:17)
    pc.publish(1, vg);
    pc.csync();
    T vf[CPT], F[CPT];
    {
        T gh[2] = {T(0), T(0)};
        if (ownN) {
            double ev = s_vg_hi;
            if (a.modeX[1] == BC_TRANS && a.actX) ev = edge_drift(ev, (double)pc.endv(1, N - 1));
            mc.ghost_hi(1, 1, ev, gh);
            if (e_vg_hi && a.modeX[1] == BC_TRANS && a.actX) e_vg_hi[pc.col] = ev;
        }
#pragma unroll
        for (int k = 0; k < CPT; ++k) {
            if (!pc.valid(k)) { vf[k] = T(0); F[k] = T(0); continue; }
            T p1 = mc.sp(1, vg, k, 1, gh);
            vf[k] = (vg[k] + p1) < T(0) ? T(1) : T(0);
            F[k] = bI[k] * vg[k];
        }
    }
    if (init_mag) init_edges(pc, et, mag_obj(c, d, MO_STORE_R), F);
    // store.fluxR = F.*(1-vf) + F.shift(X,1).*vf   (relaxingMagnet.m:22-24)
    double s_sf_hi = (ownN && e_sf_hi) ? e_sf_hi[pc.col] : 0.0;
    pc.csync();
    pc.publish(0, F);
    pc.csync();
    T Fu[CPT];
    {
        T gh[2] = {T(0), T(0)};
        if (ownN) {
            double ev = s_sf_hi;
            if (a.modeX[1] == BC_TRANS && a.actX) {
                ev = edge_drift(ev, (double)pc.endv(0, N - 1));
                if (e_sf_hi) e_sf_hi[pc.col] = ev;
            }
            mc.ghost_hi(0, 1, ev, gh);
        }
#pragma unroll
        for (int k = 0; k < CPT; ++k) {
            if (!pc.valid(k)) { Fu[k] = T(0); continue; }
            Fu[k] = F[k] * (T(1) - vf[k]) + mc.sp(0, F, k, 1, gh) * vf[k];
        }
    }
    // store = B_I - ff*(fluxR - fluxR.shift(X,-1))   (relaxingMagnet.m:26-27)
    pc.csync();
    pc.publish(1, Fu);
    pc.csync();
    T W[CPT];
    {
        T glo = own0 ? mc.ghost_lo(1, e_sf_lo, true) : T(0);
#pragma unroll
        for (int k = 0; k < CPT; ++k) {
            if (!pc.valid(k)) { W[k] = T(0); continue; }
            T st = bI[k] - ff * (Fu[k] - mc.sm(1, Fu, k, glo));
            W[k] = st * vg[k];   // wMag = store .* velGrid   (relaxingMagnet.m:33)
        }
    }
    if (init_mag) init_edges(pc, et, mag_obj(c, d, MO_WMAG), W);

    // flux, dFluxR, dFluxL from wMag shifts (relaxingMagnet.m:34-45): upper edge drifts 4 times
    // (shift +1, +1, +2, +1 in evaluation order), the lower edge once.
    double s_wm_hi = ((ownN || ownN2) && e_wm_hi) ? e_wm_hi[pc.col] : 0.0;
    pc.csync();
    pc.publish(0, W);
    pc.csync();
    T Fl[CPT];
    {
        T g1[2] = {T(0), T(0)}, g2[2] = {T(0), T(0)}, g3[2] = {T(0), T(0)}, g4[2] = {T(0), T(0)};
        if (ownN || ownN2) {
            bool tr = a.modeX[1] == BC_TRANS && a.actX;
            double cur = (double)pc.endv(0, N - 1);
            double e1 = tr ? edge_drift(s_wm_hi, cur) : s_wm_hi;
            double e2 = tr ? edge_drift(e1, cur) : e1;
            double e3 = tr ? edge_drift(e2, cur) : e2;
            double e4 = tr ? edge_drift(e3, cur) : e3;
            mc.ghost_hi(0, 1, e1, g1);
            mc.ghost_hi(0, 1, e2, g2);
            mc.ghost_hi(0, 2, e3, g3);
            mc.ghost_hi(0, 1, e4, g4);
            s_wm_hi = e4;
        }
        T glo = own0 ? mc.ghost_lo(0, e_wm_lo, true) : T(0);
        T fx[CPT];
#pragma unroll
        for (int k = 0; k < CPT; ++k) {
            if (!pc.valid(k)) { fx[k] = T(0); Fl[k] = T(0); continue; }
            T w = W[k];
            T v = vf[k];
            fx[k] = w * (T(1) - v) + mc.sp(0, W, k, 1, g1) * v;
            T dFluxR = mc.sp(0, W, k, 1, g2) - (v * mc.sp(0, W, k, 2, g3) + (T(1) - v) * w);
            T dFluxL = w - (v * mc.sp(0, W, k, 1, g4) + (T(1) - v) * mc.sm(0, W, k, glo));
            Fl[k] = fx[k] + limiter_corr<T>(a.limiter, dFluxL, dFluxR);
        }
        if (init_mag) init_edges(pc, et, mag_obj(c, d, MO_FLUX), fx);
    }
    // B_I = B_I - 2ff*(flux - flux.shift(X,-1))   (relaxingMagnet.m:49)
    pc.csync();   // every thread has read the wMag slot (and the wMag upper state) by now
    if (ownN && e_wm_hi && a.modeX[1] == BC_TRANS && a.actX) e_wm_hi[pc.col] = s_wm_hi;
    pc.publish(1, Fl);
    pc.csync();
    {
        T glo = own0 ? mc.ghost_lo(1, e_fx_lo, true) : T(0);
        T* Fout = reinterpret_cast<T*>(q ? a.F[1] : a.F[0]);
#pragma unroll
        for (int k = 0; k < CPT; ++k) {
            if (!pc.valid(k)) continue;
            long long o = pc.off(k);
            BI[o] = bI[k] - ff2 * (Fl[k] - mc.sm(1, Fl, k, glo));
            Fout[o] = Fl[k];
        }
    }
}

// ---- pointwise passes ---------------------------------------------------------------------------------
__device__ __forceinline__ void cell_coords(const Geom& g, long long i, int& x, int& y, int& z) {
    x = (int)(i % g.n[0]);
    long long r = i / g.n[0];
    y = (int)(r % g.n[1]);
    z = (int)(r / g.n[1]);
}

// C_I = F_I - F_I.shift(I, +1)   (flux(X) object of mag(I): mag-class BC along I, component I)
template <typename T>
__global__ void mag_ct1_kernel(const MagArgs a) {
    if (a.tm->done || a.tm->error) return;
    const Geom& g = a.sg.g;
    const int d = a.X - 1;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < 2 * g.ncell;
         i += (long long)gridDim.x * blockDim.x) {
        int q = i >= g.ncell;
        long long cell = i - q * g.ncell;
        int x, y, z;
        cell_coords(g, cell, x, y, z);
        const T* F = reinterpret_cast<const T*>(q ? a.F[1] : a.F[0]);
        T* C = reinterpret_cast<T*>(q ? a.C[1] : a.C[0]);
        int I = q ? a.I[1] : a.I[0], e = I - 1;
        T fs;
        if (q ? a.shiftI[1] : a.shiftI[0]) {
            bool own = sel3(e, x, y, z) == sel3(e, g.n[0], g.n[1], g.n[2]) - 1;
            fs = shift_along<T>(g, F, cell, x, y, z, e, +1, q ? a.modeI_mag[1][1] : a.modeI_mag[0][1],
                                q ? a.actI_mag[1] : a.actI_mag[0], true,
                                a.edges->p[mag_obj(I - 1, d, MO_FLUX)][e][1], a.fade, a.fade_f, a.bc_inf, own);
        } else {
            fs = F[cell];
        }
        C[cell] = F[cell] - fs;
    }
}

// D_I = C_I.shift(X, -1)   (flux(X) object of mag(I), lower X edge) -> written over F_I
template <typename T>
__global__ void mag_ct2_kernel(const MagArgs a) {
    if (a.tm->done || a.tm->error) return;
    const Geom& g = a.sg.g;
    const int d = a.X - 1;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < 2 * g.ncell;
         i += (long long)gridDim.x * blockDim.x) {
        int q = i >= g.ncell;
        long long cell = i - q * g.ncell;
        int x, y, z;
        cell_coords(g, cell, x, y, z);
        const T* C = reinterpret_cast<const T*>(q ? a.C[1] : a.C[0]);
        T* D = reinterpret_cast<T*>(q ? a.F[1] : a.F[0]);
        int I = q ? a.I[1] : a.I[0];
        bool own = sel3(d, x, y, z) == 0;
        D[cell] = shift_along<T>(g, C, cell, x, y, z, d, -1, a.modeX[0], a.actX, I - 1 == d,
                                 a.edges->p[mag_obj(I - 1, d, MO_FLUX)][d][0], a.fade, a.fade_f, a.bc_inf, own);
    }
}

// B_X' = (B_X - dt/dI1 * D_I1) - dt/dI2 * D_I2 -> scratch; cell-centred B of I2 (the last component).
template <typename T>
__global__ void mag_bx_kernel(const MagArgs a) {
    if (a.tm->done || a.tm->error) return;
    const Geom& g = a.sg.g;
    const double dt = a.tm->dt;
    const T f0 = (T)(dt / a.dI[0]), f1 = (T)(dt / a.dI[1]);
    const int X = a.X;
    const T* BX = reinterpret_cast<const T*>(a.q[Q_BX + X - 1]);
    const T* D0 = reinterpret_cast<const T*>(a.F[0]);
    const T* D1 = reinterpret_cast<const T*>(a.F[1]);
    T* BXn = reinterpret_cast<T*>(a.BXn);
    const int I2 = a.I[1], e2 = I2 - 1;
    const T* BI2 = reinterpret_cast<const T*>(a.q[Q_BX + e2]);
    T* CB2 = reinterpret_cast<T*>(a.q[Q_CBX + e2]);
    for (long long cell = blockIdx.x * (long long)blockDim.x + threadIdx.x; cell < g.ncell;
         cell += (long long)gridDim.x * blockDim.x) {
        BXn[cell] = (BX[cell] - f0 * D0[cell]) - f1 * D1[cell];
        int x, y, z;
        cell_coords(g, cell, x, y, z);
        T sh;
        if (e2 < g.ndims) {
            bool own = sel3(e2, x, y, z) == sel3(e2, g.n[0], g.n[1], g.n[2]) - 1;
            sh = shift_along<T>(g, BI2, cell, x, y, z, e2, +1, a.modeI_mag[1][1], a.actI_mag[1], true,
                                a.edges->p[OBJ_PRIM_MAG + e2][e2][1], a.fade, a.fade_f, a.bc_inf, own);
        } else {
            sh = BI2[cell];
        }
        CB2[cell] = T(0.5) * (BI2[cell] + sh);
    }
}

// B_X = B_X'; cell-centred B_X = 0.5*(B_X + B_X.shift(X, +1))
template <typename T>
__global__ void mag_cell_kernel(const MagArgs a) {
    if (a.tm->done || a.tm->error) return;
    const Geom& g = a.sg.g;
    const int X = a.X, d = X - 1;
    const T* BXn = reinterpret_cast<const T*>(a.BXn);
    T* BX = reinterpret_cast<T*>(a.q[Q_BX + d]);
    T* CBX = reinterpret_cast<T*>(a.q[Q_CBX + d]);
    for (long long cell = blockIdx.x * (long long)blockDim.x + threadIdx.x; cell < g.ncell;
         cell += (long long)gridDim.x * blockDim.x) {
        int x, y, z;
        cell_coords(g, cell, x, y, z);
        bool own = sel3(d, x, y, z) == sel3(d, g.n[0], g.n[1], g.n[2]) - 1;
        T sh = shift_along<T>(g, BXn, cell, x, y, z, d, +1, a.modeX[1], a.actX, true, a.edges->p[OBJ_PRIM_MAG + d][d][1],
                              a.fade, a.fade_f, a.bc_inf, own);
        BX[cell] = BXn[cell];
        CBX[cell] = T(0.5) * (BXn[cell] + sh);
    }
}

}  // namespace img
