// Magnet sweep along X for the two transverse components (magnet/magnetFlux.m:14-31,
// magnet/relaxingMagnet.m:15-60, magnet/MagnetArray.m:36-38).
//
// Two launches per sweep, both on the same X-pencil tiling:
//   mag_chain   -- per X-pencil and component I: corner velocity (transverse average, then the
//                  1-2-1 smoothing along X), upwind predictor, TVD corrector, B_I update.  Writes
//                  B_I in place and the limited flux F_I to scratch.  Both components in one launch.
//   mag_ctcell  -- C_I = F_I - F_I.shift(I,+1) at own cells, D_I = C_I.shift(X,-1) through shared
//                  memory, B_X = (B_X - dt/dI1 D_I1) - dt/dI2 D_I2 in place, cell-centred B_I2 and
//                  B_X (relaxingMagnet.m:54-58, MagnetArray.m:36-38).
// The second launch needs the first's F_I at the neighbouring pencils along I, hence two launches.
#pragma once

#include "fluid_sweep.cuh"

namespace img {

struct MagArgs {
    SweepGeom sg;              // sweep along d = X-1
    void* q[NQ];
    void* F[2];                // limited flux per component (scratch)
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
// Value of A.shift(dim e, n) at index i of a line of Ne values along e, for n = -1 or +1, where
// at(j) returns A at index j of that line and fi is the line's index in the face orthogonal to e.
// mode/act/flip/edge describe the array object; the edge state of a trans edge is drifted and
// written back when `own_update` (exactly one thread per face cell calls with own_update = true).
template <typename T, typename At>
__device__ __forceinline__ T shift_line(const At& at, int i, int Ne, long long fi, int n, int mode, int act, int flip,
                                        double* edge, const double* fc, int f, double bc_inf, bool own_update) {
    const bool upper = n > 0;
    const bool is_ghost = upper ? (i == Ne - 1) : (i == 0);
    if (!is_ghost) {   // interior: the neighbour, damped under fade
        T v = at(i + n);
        if (mode == BC_FADE) {
            T s0 = upper ? at(Ne > 1 ? 1 : 0) : at(0);
            T sN1 = upper ? at(Ne - 1) : at(Ne - 2);
            v = fade_apply(v, i, Ne, fc, f, s0, sN1);
        }
        return v;
    }
    switch (mode) {
        case BC_CIRC: return at(upper ? 0 : Ne - 1);
        case BC_MIRROR: { T v = upper ? at(Ne - 2) : at(1); return (flip & GF_NEG) ? -v : v; }
        case BC_FLIP: { T v = upper ? at(Ne - 1) : at(0); return (flip & GF_NEG) ? -v : v; }
        case BC_ZERO: return (flip & (upper ? GF_ZHI : GF_ZLO)) ? T(0) : at(upper ? Ne - 1 : 0);
        case BC_WALL: return (T)edge[fi];
        case BC_TRANS: {
            T a1, a2;
            if (!upper) { a1 = at(trans_pick_lower(Ne, 1, 1)); a2 = at(0); }
            else { a1 = at(trans_pick_upper(Ne, 1, 1)); a2 = at(Ne - 1); }
            double ev = 0.0;
            if (act) {
                ev = edge_drift(edge[fi], (double)a2);
                if (own_update) edge[fi] = ev;
            }
            return (T)trans_ghost((double)a1, (double)a2, ev, bc_inf, 4.0, (double)a2);
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

// A.shift(dim e, n)[cell] for an array A in global memory.
template <typename T>
__device__ __forceinline__ T shift_along(const Geom& g, const T* A, long long cell, int x, int y, int z, int e, int n,
                                         int mode, int act, int flip, double* edge, const double* fc, int f,
                                         double bc_inf, bool own_update) {
    const int Ne = sel3(e, g.n[0], g.n[1], g.n[2]);
    const long long se = sel3(e, g.s[0], g.s[1], g.s[2]);
    const int i = sel3(e, x, y, z);
    const long long b = cell - (long long)i * se;   // row 0 of this line along e
    auto at = [&](int j) -> T { return A[b + (long long)j * se]; };
    return shift_line<T>(at, i, Ne, face_index(g, e, x, y, z), n, mode, act, flip, edge, fc, f, bc_inf, own_update);
}

// ---- the X-chain ------------------------------------------------------------------------------------
constexpr int MAG_NARR = 4;
constexpr int MAG_NSLOT = 6;   // per column: lower anchors, upper +1 (e1), +1 (e2), +2 row N, +2 row N+1, +1 (e4)

// Dynamic shared memory of the chain kernel for NQC components per CTA: 4 halo'd arrays + 6
// ghost/anchor slots per column, per component.
template <typename T>
__host__ __device__ inline size_t mag_smem_bytes(int RC, int Wb, int NQC = 1) {
    return NQC * (sizeof(T) * (size_t)MAG_NARR * tile_rows(RC) * Wb + sizeof(Ghost<T>) * MAG_NSLOT * (size_t)Wb);
}

// The four upper shift calls of wMag in relaxingMagnet.m:37-45 (+1, +1, +2, +1, in that order; a
// trans edge drifts once per call): their ghosts from the successive edge states e1..e4 go to slots
// 1, 2, (3, 4), 5, with the fade anchors of the +1 and +2 shifts.  Returns e4, the edge's new state.
template <typename T, int CPT>
__device__ __forceinline__ double wmag_upper_ghosts(const Tile<T, CPT>& tl, const T* A, Ghost<T>* GS, int mode,
                                                    int act, double* eh, double binf) {
    const int N = tl.N, Wb = tl.Wb, b = tl.b;
    const bool stateful = (mode == BC_TRANS || mode == BC_WALL) && eh != nullptr;
    const bool drift = mode == BC_TRANS && act && eh != nullptr;
    const double s0 = stateful ? eh[tl.col] : 0.0;
    const double cur = (double)tl.row(A, N - 1);
    const double e1 = drift ? edge_drift(s0, cur) : s0;
    const double e2 = drift ? edge_drift(e1, cur) : s0;
    const double e3 = drift ? edge_drift(e2, cur) : s0;
    const double e4 = drift ? edge_drift(e3, cur) : s0;
    Ghost<T> u = fade_anchors(tl, A, +1);
    u.g = bc_ghost(tl, A, +1, 1, mode, act, 0, eh, binf, e1);
    GS[1 * Wb + b] = u;
    u.g = bc_ghost(tl, A, +1, 1, mode, act, 0, eh, binf, e2);
    GS[2 * Wb + b] = u;
    u.g = bc_ghost(tl, A, +1, 1, mode, act, 0, eh, binf, e4);
    GS[5 * Wb + b] = u;
    Ghost<T> w2;
    w2.s0 = tl.row(A, N > 2 ? 2 : N - 1);
    w2.sN1 = tl.row(A, N - 1);
    w2.g = bc_ghost(tl, A, +2, 1, mode, act, 0, eh, binf, e3);
    GS[3 * Wb + b] = w2;
    w2.g = bc_ghost(tl, A, +2, 2, mode, act, 0, eh, binf, e3);
    GS[4 * Wb + b] = w2;
    return e4;
}

// Per-component constants of the chain: component I (1-based) of the transverse pair, its BC
// settings along I and its pointers.
template <typename T>
struct ChainComp {
    int I, e, shiftI, mode_mom_lo, mode_mass_lo, act_mom, act_mass, init_mag;
    T* BI;
    T* Fout;
    __device__ __forceinline__ void init(const MagArgs& a, int q) {
        I = q ? a.I[1] : a.I[0];
        e = I - 1;
        shiftI = q ? a.shiftI[1] : a.shiftI[0];
        mode_mom_lo = q ? a.modeI_mom[1][0] : a.modeI_mom[0][0];
        mode_mass_lo = q ? a.modeI_mass[1][0] : a.modeI_mass[0][0];
        act_mom = q ? a.actI_mom[1] : a.actI_mom[0];
        act_mass = q ? a.actI_mass[1] : a.actI_mass[0];
        init_mag = q ? a.init_mag[1] : a.init_mag[0];
        BI = reinterpret_cast<T*>(a.q[Q_BX + e]);
        Fout = reinterpret_cast<T*>(q ? a.F[1] : a.F[0]);
    }
};

// The chain of one grid, run by CTA (vblock, blockIdx.y) of that grid's launch: NQC = 1 handles
// component blockIdx.y, NQC = 2 both transverse components, interleaved stage by stage so that
// every barrier serves twice the work.
// FADE: a mag-class BC along X is fade (compiles the damping in).  CG (copy ghosts): single-CTA
// pencils with circ, const or fade mag-class shifts along X; the reader of a row next to a pencil end
// indexes the row its ghost copies, so no stage needs halo jobs or the barrier after them.
// INIT: this launch may capture stored edges of first-assigned objects (compiled out otherwise; the
// host never combines it with CG).
template <typename T, int CPT, bool FADE, int NQC, bool CG, bool INIT>
__device__ __forceinline__ void mag_chain_body(const MagArgs& a, unsigned vblock) {
    extern __shared__ __align__(16) unsigned char smem[];
    pdl_wait();
    if (a.tm->done || (a.sg.CL == 1 && a.tm->error)) return;   // clusters: as in the fluid sweeps
    Tile<T, CPT> tl;
    tl.init(a.sg, vblock);
    const int q0 = NQC == 2 ? 0 : (int)blockIdx.y;
    ChainComp<T> cp[NQC];
#pragma unroll
    for (int q = 0; q < NQC; ++q) cp[q].init(a, q0 + q);
    const int d = a.X - 1;
    const int N = a.sg.N, Wb = tl.Wb, b = tl.b;
    const Geom& g = a.sg.g;
    const double dt = a.tm->dt;
    const T ff = (T)(0.5 * dt / a.dx);
    const T ff2 = T(2) * ff;
    const EdgeTable* et = a.edges;
    const size_t AS = (size_t)tile_rows(tl.RC) * Wb;
    // component q: arrays S[q][0..3] at smem + (4q + i) * AS, ghost slots after all arrays
    T* const SB = reinterpret_cast<T*>(smem);
    Ghost<T>* const GSB = reinterpret_cast<Ghost<T>*>(SB + NQC * MAG_NARR * AS);
    auto S = [&](int q, int i) -> T* { return SB + (q * MAG_NARR + i) * AS; };
    auto GS = [&](int q) -> Ghost<T>* { return GSB + q * MAG_NSLOT * Wb; };
    const double* fc = a.fade;
    const int f = a.fade_f;
    const double binf = a.bc_inf;
    const int mlo = a.modeX[0], mhi = a.modeX[1];
    // copy ghosts: shared index of the row that row -1, row N and row N+1 copy
    const int dn_src = tl.ridx(mlo == BC_CIRC ? N - 1 : 0);
    const int up_src = tl.ridx(mhi == BC_CIRC ? 0 : N - 1);
    const int up2_src = tl.ridx(mhi == BC_CIRC ? 1 : N - 1);
    // A.shift(X, n) at own row k for n = -1 or +1 (anchors `an` read under fade only)
    auto sh = [&](const T* A, const Ghost<T>* an, int k, int n, int mode) -> T {
        if constexpr (CG) {
            const int r = tl.grow(k);
            const T v = A[n < 0 ? (r == 0 ? dn_src : tl.idx(k) - tl.rs) : (r == N - 1 ? up_src : tl.idx(k) + tl.rs)];
            if constexpr (FADE) {
                if (mode == BC_FADE) return cg_fade(tl, A, r, n, v, fc, f);
            }
            return v;
        } else {
            return shifted<FADE>(tl, A, an, k, n, mode, fc, f);
        }
    };
    // the scratch objects of mag(I) for this sweep (mag-class BC along X, no mirror flip)
    auto edge_of = [&](int q, int kind, int side) -> double* { return et->p[mag_obj(cp[q].e, d, kind)][d][side]; };
    // halo jobs: (component q, side) is done by thread g == (2q + side) mod G of the column
    auto job = [&](int q, int side) { return tl.colok && tl.g == (2 * q + side) % tl.G; };
    auto halo = [&](int q, T* A, int kind, bool lo_shift, bool hi_shift, int hi_rows) {
        // zero-BC flags by object: the store's fluxR and the flux are FluxArrays, velGrid/wMag are not
        const int gf = kind == MO_STORE_R ? GF_FLUXR : (kind == MO_FLUX ? GF_FLUX : 0);
        if (job(q, 0)) halo_job(tl, A, GS(q), 0, lo_shift, mlo, a.actX, gf, edge_of(q, kind, 0), binf, hi_rows);
        if (job(q, 1)) halo_job(tl, A, GS(q) + Wb, 1, hi_shift, mhi, a.actX, gf, edge_of(q, kind, 1), binf, hi_rows);
    };

    // ---- corner velocity (magnetFlux.m:18-19): transverse average with mass/mom BCs along I ------
    const T* rho = reinterpret_cast<const T*>(a.q[Q_RHO]);
    const T* pX = reinterpret_cast<const T*>(a.q[Q_PX + d]);
    T vgr[NQC][CPT], bI[NQC][CPT];
#pragma unroll
    for (int q = 0; q < NQC; ++q) {
        const ChainComp<T>& c = cp[q];
        // the transverse coordinate is the pencil's own (e != d): interior pencils read their lower
        // neighbour directly; the boundary and fade cases go through the reference's shift
        const int ie = c.e == a.sg.d1 ? tl.c1 : tl.c2;
        const long long se = sel3(c.e, g.s[0], g.s[1], g.s[2]);
        const bool direct = c.shiftI && ie > 0 && c.mode_mom_lo != BC_FADE && c.mode_mass_lo != BC_FADE;
#pragma unroll
        for (int k = 0; k < CPT; ++k) {
            vgr[q][k] = T(0);
            bI[q][k] = T(0);
            if (tl.ok(k)) {
                const long long o = tl.off(k);
                int x, y, z;
                tl.coords(k, x, y, z);
                T pm, rm;
                if (direct) {
                    pm = pX[o - se];
                    rm = rho[o - se];
                } else if (c.shiftI) {
                    pm = shift_along<T>(g, pX, o, x, y, z, c.e, -1, c.mode_mom_lo, c.act_mom, false,
                                        et->p[OBJ_PRIM_MOM + d][c.e][0], fc, f, binf, true);
                    rm = shift_along<T>(g, rho, o, x, y, z, c.e, -1, c.mode_mass_lo, c.act_mass, false,
                                        et->p[OBJ_PRIM_MASS][c.e][0], fc, f, binf, true);
                } else {
                    pm = pX[o];
                    rm = rho[o];
                }
                if constexpr (sizeof(T) == 4) vgr[q][k] = (pm + pX[o]) * rcp_approx(rm + rho[o]);
                else vgr[q][k] = (pm + pX[o]) / (rm + rho[o]);
                bI[q][k] = c.BI[o];
                if (INIT && c.init_mag && on_face(g, x, y, z))
                    init_edges_cell(g, et, mag_obj(c.e, d, MO_VELGRID), x, y, z, (double)vgr[q][k]);
            }
            S(q, 0)[tl.idx(k)] = vgr[q][k];
        }
    }
    tl.csync();
    if constexpr (!CG) {
#pragma unroll
        for (int q = 0; q < NQC; ++q) halo(q, S(q, 0), MO_VELGRID, true, true, 1);
        __syncthreads();
    }
    // vg = 0.25*(vg.shift(X,-1) + vg.shift(X,1) + 2*vg)   (magnetFlux.m:21-23)
    T vg[NQC][CPT];
#pragma unroll
    for (int q = 0; q < NQC; ++q)
#pragma unroll
        for (int k = 0; k < CPT; ++k) {
            const T m1 = sh((const T*)S(q, 0), GS(q), k, -1, mlo);
            const T p1 = sh((const T*)S(q, 0), GS(q) + Wb, k, +1, mhi);
            vg[q][k] = tl.ok(k) ? T(0.25) * (m1 + p1 + T(2) * vgr[q][k]) : T(0);
            S(q, 1)[tl.idx(k)] = vg[q][k];
        }
    tl.csync();
    if constexpr (!CG) {
#pragma unroll
        for (int q = 0; q < NQC; ++q) halo(q, S(q, 1), MO_VELGRID, false, true, 1);
        __syncthreads();
    }
    // velocityFlow = (vg + vg.shift(X,1)) < 0; store.fluxR = B_I.*vg   (relaxingMagnet.m:17,22)
    T vf[NQC][CPT];
#pragma unroll
    for (int q = 0; q < NQC; ++q)
#pragma unroll
        for (int k = 0; k < CPT; ++k) {
            const T p1 = sh((const T*)S(q, 1), GS(q) + Wb, k, +1, mhi);
            vf[q][k] = (vg[q][k] + p1) < T(0) ? T(1) : T(0);
            const T F = bI[q][k] * vg[q][k];
            S(q, 2)[tl.idx(k)] = F;
            if (INIT && cp[q].init_mag && tl.ok(k)) {
                int x, y, z;
                tl.coords(k, x, y, z);
                if (on_face(g, x, y, z)) init_edges_cell(g, et, mag_obj(cp[q].e, d, MO_STORE_R), x, y, z, (double)F);
            }
        }
    tl.csync();
    if constexpr (!CG) {
#pragma unroll
        for (int q = 0; q < NQC; ++q) halo(q, S(q, 2), MO_STORE_R, false, true, 1);
        __syncthreads();
    }
    // store.fluxR = F.*(1-vf) + F.shift(X,1).*vf   (relaxingMagnet.m:23-24)
#pragma unroll
    for (int q = 0; q < NQC; ++q)
#pragma unroll
        for (int k = 0; k < CPT; ++k) {
            const T F = S(q, 2)[tl.idx(k)];
            const T Fp = sh((const T*)S(q, 2), GS(q) + Wb, k, +1, mhi);
            S(q, 3)[tl.idx(k)] = F * (T(1) - vf[q][k]) + Fp * vf[q][k];
        }
    tl.csync();
    if constexpr (!CG) {
#pragma unroll
        for (int q = 0; q < NQC; ++q) halo(q, S(q, 3), MO_STORE_R, true, false, 1);
        __syncthreads();
    }
    // store = B_I - ff*(fluxR - fluxR.shift(X,-1)); wMag = store.*velGrid   (relaxingMagnet.m:26-33)
    T W[NQC][CPT];
#pragma unroll
    for (int q = 0; q < NQC; ++q)
#pragma unroll
        for (int k = 0; k < CPT; ++k) {
            const T Fu = S(q, 3)[tl.idx(k)];
            const T st = bI[q][k] - ff * (Fu - sh((const T*)S(q, 3), GS(q), k, -1, mlo));
            W[q][k] = st * vg[q][k];
            S(q, 0)[tl.idx(k)] = W[q][k];
            if (INIT && cp[q].init_mag && tl.ok(k)) {
                int x, y, z;
                tl.coords(k, x, y, z);
                if (on_face(g, x, y, z)) init_edges_cell(g, et, mag_obj(cp[q].e, d, MO_WMAG), x, y, z, (double)W[q][k]);
            }
        }
    tl.csync();
    // wMag: one lower shift (an ordinary halo job; the upper side only copies the next rank's two
    // rows) and four upper shift calls whose ghosts differ, kept in slots by every rank that owns
    // row N-1 or N-2.  The edge's new state is stored after the next cluster barrier, once every
    // rank has read the old one.
    double e4[NQC];
    const bool own_end = tl.rank == tl.rank_hi || (tl.rank + 1 == tl.rank_hi && tl.N - 1 == tl.rank_hi * tl.RC);
#pragma unroll
    for (int q = 0; q < NQC; ++q) {
        e4[q] = 0.0;
        if constexpr (CG) continue;
        halo(q, S(q, 0), MO_WMAG, true, false, 2);
        Ghost<T>* gs = GS(q);
        if (job(q, 1) && own_end)
            e4[q] = wmag_upper_ghosts(tl, (const T*)S(q, 0), gs, mhi, a.actX, edge_of(q, MO_WMAG, 1), binf);
        else if (job(q, 1) && mhi == BC_FADE) {   // fade anchors of the +1 and +2 shifts on the other ranks
            gs[1 * Wb + b] = gs[2 * Wb + b] = gs[5 * Wb + b] = fade_anchors(tl, (const T*)S(q, 0), +1);
            Ghost<T> w2;
            w2.g = T(0);
            w2.s0 = tl.row((const T*)S(q, 0), N > 2 ? 2 : N - 1);
            w2.sN1 = tl.row((const T*)S(q, 0), N - 1);
            gs[3 * Wb + b] = w2;
        }
    }
    if constexpr (!CG) __syncthreads();
    T Fl[NQC][CPT];
#pragma unroll
    for (int q = 0; q < NQC; ++q) {
        const T* A = S(q, 0);
        const Ghost<T>* gs = GS(q);
#pragma unroll
        for (int k = 0; k < CPT; ++k) {
            const T w = W[q][k], v = vf[q][k];
            const int ix = tl.idx(k);
            const int r = tl.grow(k);
            T p1a = A[ix + tl.rs], p1b = p1a, p1d = p1a, p2 = A[ix + 2 * tl.rs];
            if constexpr (CG) {   // the four upper calls share their ghosts
                p1a = p1b = p1d = A[r == N - 1 ? up_src : ix + tl.rs];
                p2 = A[r == N - 2 ? up_src : (r == N - 1 ? up2_src : ix + 2 * tl.rs)];
                if constexpr (FADE) {
                    if (mhi == BC_FADE && r < N && (r < f || r >= N - f)) {   // anchors of the +1 and +2 shifts
                        const T a1 = A[tl.ridx(N > 1 ? 1 : 0)], aN = A[tl.ridx(N - 1)], a2 = A[tl.ridx(N > 2 ? 2 : N - 1)];
                        p1a = p1b = p1d = fade_apply(p1a, r, N, fc, f, a1, aN);
                        p2 = fade_apply(p2, r, N, fc, f, a2, aN);
                    }
                }
            } else if (r >= N - 2 && r < N) {   // rows next to the upper end: ghosts of the four calls
                if (r == N - 1) {
                    p1a = gs[1 * Wb + b].g;
                    p1b = gs[2 * Wb + b].g;
                    p1d = gs[5 * Wb + b].g;
                    p2 = gs[4 * Wb + b].g;
                } else {
                    p2 = gs[3 * Wb + b].g;
                }
            }
            if (!CG && FADE && mhi == BC_FADE) {
                const Ghost<T>& u1 = gs[1 * Wb + b];
                const Ghost<T>& u2 = gs[3 * Wb + b];
                p1a = fade_apply(p1a, r, N, fc, f, u1.s0, u1.sN1);
                p1b = fade_apply(p1b, r, N, fc, f, u1.s0, u1.sN1);
                p1d = fade_apply(p1d, r, N, fc, f, u1.s0, u1.sN1);
                p2 = fade_apply(p2, r, N, fc, f, u2.s0, u2.sN1);
            }
            const T m1 = sh(A, gs, k, -1, mlo);
            const T fx = w * (T(1) - v) + p1a * v;
            const T dFluxR = p1b - (v * p2 + (T(1) - v) * w);
            const T dFluxL = w - (v * p1d + (T(1) - v) * m1);
            Fl[q][k] = fx + limiter_corr<T>(a.limiter, dFluxL, dFluxR);
            S(q, 1)[ix] = Fl[q][k];
            if (INIT && cp[q].init_mag && tl.ok(k)) {
                int x, y, z;
                tl.coords(k, x, y, z);
                if (on_face(g, x, y, z)) init_edges_cell(g, et, mag_obj(cp[q].e, d, MO_FLUX), x, y, z, (double)fx);
            }
        }
    }
    tl.csync();
    if constexpr (!CG) {
#pragma unroll
        for (int q = 0; q < NQC; ++q) {
            if (job(q, 1) && tl.rank == tl.rank_hi && mhi == BC_TRANS && a.actX) {
                double* eh = edge_of(q, MO_WMAG, 1);
                if (eh) eh[tl.col] = e4[q];
            }
            halo(q, S(q, 1), MO_FLUX, true, false, 1);
        }
        __syncthreads();
    }
    pdl_trigger();
    // B_I = B_I - 2ff*(flux - flux.shift(X,-1))   (relaxingMagnet.m:49); F_I -> scratch for CT
#pragma unroll
    for (int q = 0; q < NQC; ++q)
#pragma unroll
        for (int k = 0; k < CPT; ++k) {
            const T fm = sh((const T*)S(q, 1), GS(q), k, -1, mlo);
            if (!tl.ok(k)) continue;
            const long long o = tl.off(k);
            cp[q].BI[o] = bI[q][k] - ff2 * (Fl[q][k] - fm);
            cp[q].Fout[o] = Fl[q][k];
        }
    if (tl.CL > 1) cluster_sync();   // keep shared memory alive for DSMEM readers
}

// ---- CT and cell-centring, fused along X-pencils --------------------------------------------------------
// Per X-pencil, on the chain's tiling:
//   C_q  = F_q - F_q.shift(I_q, +1) at the thread's own cells        (relaxingMagnet.m:56)
//   D_q  = C_q.shift(X, -1), through shared memory                   (relaxingMagnet.m:57)
//   B_X  = (B_X - dt/dI_1 * D_1) - dt/dI_2 * D_2                      (relaxingMagnet.m:58, both calls)
//   cell-centred B_I2 along I2 and B_X along X, the latter from the new B_X in shared memory
//                                                                    (magnetFlux.m:30-31, MagnetArray.m:36-38)
// Every thread reads B_X only at its own cells, so B_X is updated in place.  Each flux object's
// shift(I, +1) call drifts its trans edge in the thread of the upper I face cell, which is also the
// only thread that reads that edge.
template <typename T>
__host__ __device__ inline size_t ctcell_smem_bytes(int RC, int Wb) {
    return 3 * (sizeof(T) * (size_t)tile_rows(RC) * Wb + sizeof(Ghost<T>) * (size_t)Wb);
}

template <typename T, int CPT, bool FADE, bool CG>
__device__ __forceinline__ void mag_ctcell_body(const MagArgs& a, unsigned vblock) {
    extern __shared__ __align__(16) unsigned char smem[];
    pdl_wait();
    if (a.tm->done || (a.sg.CL == 1 && a.tm->error)) return;   // clusters: as in the fluid sweeps
    Tile<T, CPT> tl;
    tl.init(a.sg, vblock);
    const int d = a.X - 1;
    const Geom& g = a.sg.g;
    const int Wb = tl.Wb;
    const double dt = a.tm->dt;
    const EdgeTable* et = a.edges;
    const double* fc = a.fade;
    const int f = a.fade_f;
    const double binf = a.bc_inf;
    const int mlo = a.modeX[0], mhi = a.modeX[1];
    const int N = tl.N;
    // copy ghosts (see mag_chain_body): the rows that row -1 and row N copy
    const int dn_src = tl.ridx(mlo == BC_CIRC ? N - 1 : 0);
    const int up_src = tl.ridx(mhi == BC_CIRC ? 0 : N - 1);
    const size_t AS = (size_t)tile_rows(tl.RC) * Wb;
    // shared: C_1, C_2, new B_X; then their ghost/anchor slots (C lower sides, B_X upper side)
    T* const S = reinterpret_cast<T*>(smem);
    Ghost<T>* const GS = reinterpret_cast<Ghost<T>*>(S + 3 * AS);

#pragma unroll
    for (int q = 0; q < 2; ++q) {
        const int e = (q ? a.I[1] : a.I[0]) - 1;
        const T* F = reinterpret_cast<const T*>(q ? a.F[1] : a.F[0]);
        const bool shI = q ? a.shiftI[1] : a.shiftI[0];
        const int modeI = q ? a.modeI_mag[1][1] : a.modeI_mag[0][1];
        const int actI = q ? a.actI_mag[1] : a.actI_mag[0];
        const int ie = e == a.sg.d1 ? tl.c1 : tl.c2;   // the pencil's coordinate along I (I != X)
        const bool directI = shI && ie < sel3(e, g.n[0], g.n[1], g.n[2]) - 1 && modeI != BC_FADE;
        const long long sI = sel3(e, g.s[0], g.s[1], g.s[2]);
#pragma unroll
        for (int k = 0; k < CPT; ++k) {
            T c = T(0);
            if (tl.ok(k)) {
                const long long o = tl.off(k);
                const T fv = F[o];
                if (!shI) c = fv - fv;
                else if (directI) c = fv - F[o + sI];
                else {
                    int x, y, z;
                    tl.coords(k, x, y, z);
                    c = fv - shift_along<T>(g, F, o, x, y, z, e, +1, modeI, actI, GF_NEG | GF_FLUX,
                                            et->p[mag_obj(e, d, MO_FLUX)][e][1], fc, f, binf, true);
                }
            }
            S[q * AS + tl.idx(k)] = c;
        }
    }
    tl.csync();
    if constexpr (!CG) {
        // lower ghosts of C_q along X: the flux object's mag-class BC, no mirror flip (I != X)
#pragma unroll
        for (int q = 0; q < 2; ++q)
            if (tl.colok && tl.g == q % tl.G)
                halo_job(tl, S + q * AS, GS + q * Wb, 0, true, mlo, a.actX, GF_FLUX,
                         et->p[mag_obj((q ? a.I[1] : a.I[0]) - 1, d, MO_FLUX)][d][0], binf, 1);
        __syncthreads();
    }
    T* BX = reinterpret_cast<T*>(a.q[Q_BX + d]);
    const T f0 = (T)(dt / a.dI[0]), f1 = (T)(dt / a.dI[1]);
    T bx[CPT];
#pragma unroll
    for (int k = 0; k < CPT; ++k) {
        T D0, D1;
        if constexpr (CG) {
            const int ix = tl.grow(k) == 0 ? dn_src : tl.idx(k) - tl.rs;
            D0 = S[ix];
            D1 = S[AS + ix];
            if constexpr (FADE) {
                if (mlo == BC_FADE) {
                    D0 = cg_fade(tl, (const T*)S, tl.grow(k), -1, D0, fc, f);
                    D1 = cg_fade(tl, (const T*)(S + AS), tl.grow(k), -1, D1, fc, f);
                }
            }
        } else {
            D0 = shifted<FADE>(tl, (const T*)S, GS, k, -1, mlo, fc, f);
            D1 = shifted<FADE>(tl, (const T*)(S + AS), GS + Wb, k, -1, mlo, fc, f);
        }
        bx[k] = T(0);
        if (tl.ok(k)) bx[k] = (BX[tl.off(k)] - f0 * D0) - f1 * D1;
        S[2 * AS + tl.idx(k)] = bx[k];
    }
    tl.csync();
    if constexpr (!CG) {
        // upper ghost of the new B_X along X: mag(X).shift(X, +1) of the primary array (mirror flips B_X)
        if (tl.colok && tl.g == 2 % tl.G)
            halo_job(tl, S + 2 * AS, GS + 2 * Wb, 1, true, mhi, a.actX, GF_NEG, et->p[OBJ_PRIM_MAG + d][d][1], binf, 1);
        __syncthreads();
    }
    pdl_trigger();
    T* CBX = reinterpret_cast<T*>(a.q[Q_CBX + d]);
    const int e2 = a.I[1] - 1;
    const T* BI2 = reinterpret_cast<const T*>(a.q[Q_BX + e2]);
    T* CB2 = reinterpret_cast<T*>(a.q[Q_CBX + e2]);
    const int i2 = e2 == a.sg.d1 ? tl.c1 : tl.c2;
    const int N2 = sel3(e2, g.n[0], g.n[1], g.n[2]);
    const int mode2 = a.modeI_mag[1][1];
    const bool direct2 = a.shiftI[1] && i2 < N2 - 1 && mode2 != BC_FADE;
    const long long s2 = sel3(e2, g.s[0], g.s[1], g.s[2]);
#pragma unroll
    for (int k = 0; k < CPT; ++k) {
        T up;
        if constexpr (CG) {
            up = S[2 * AS + (tl.grow(k) == N - 1 ? up_src : tl.idx(k) + tl.rs)];
            if constexpr (FADE) {
                if (mhi == BC_FADE) up = cg_fade(tl, (const T*)(S + 2 * AS), tl.grow(k), +1, up, fc, f);
            }
        } else {
            up = shifted<FADE>(tl, (const T*)(S + 2 * AS), GS + 2 * Wb, k, +1, mhi, fc, f);
        }
        if (!tl.ok(k)) continue;
        const long long o = tl.off(k);
        BX[o] = bx[k];
        CBX[o] = T(0.5) * (bx[k] + up);
        const T b2 = BI2[o];
        T sh;
        if (direct2) sh = BI2[o + s2];
        else if (a.shiftI[1]) {
            int x, y, z;
            tl.coords(k, x, y, z);
            sh = shift_along<T>(g, BI2, o, x, y, z, e2, +1, mode2, a.actI_mag[1], true,
                                et->p[OBJ_PRIM_MAG + e2][e2][1], fc, f, binf, i2 == N2 - 1);
        } else sh = b2;
        CB2[o] = T(0.5) * (b2 + sh);
    }
    if (tl.CL > 1) cluster_sync();   // keep shared memory alive for DSMEM readers
}

__device__ __forceinline__ void cell_coords(const Geom& g, long long i, int& x, int& y, int& z) {
    unsigned u = (unsigned)i, n0 = (unsigned)g.n[0], n1 = (unsigned)g.n[1];
    unsigned r = u / n0;
    x = (int)(u - r * n0);
    z = (int)(r / n1);
    y = (int)(r - (unsigned)z * n1);
}

template <typename T, int CPT, int NQC, int V>
__global__ void __launch_bounds__(512, CPT == 1 && NQC == 1 ? 2 : 1) mag_chain_kernel(const __grid_constant__ MagArgs a) {
    mag_chain_body<T, CPT, kv_fade<V>, NQC, kv_cg<V>, kv_init<V>>(a, blockIdx.x);
}

template <typename T, int CPT, bool FADE, bool CG>
__global__ void __launch_bounds__(512, 2) mag_ctcell_kernel(const __grid_constant__ MagArgs a) {
    mag_ctcell_body<T, CPT, FADE, CG>(a, blockIdx.x);
}

// The same passes over many grids in one launch (BlockMap per CTA, arguments per member).
template <typename T, int CPT, int NQC, int V>
__global__ void __launch_bounds__(512, CPT == 1 && NQC == 1 ? 2 : 1) mag_chain_batch_kernel(const MagArgs* __restrict__ args,
                                                                                const BlockMap* __restrict__ map) {
    __shared__ MagArgs sa;
    const BlockMap bm = map[blockIdx.x];
    load_member_args(sa, args + bm.member);
    __syncthreads();
    mag_chain_body<T, CPT, kv_fade<V>, NQC, kv_cg<V>, kv_init<V>>(sa, (unsigned)bm.block);
}

template <typename T, int CPT, bool FADE, bool CG>
__global__ void __launch_bounds__(512, 2) mag_ctcell_batch_kernel(const MagArgs* __restrict__ args,
                                                                  const BlockMap* __restrict__ map) {
    __shared__ MagArgs sa;
    const BlockMap bm = map[blockIdx.x];
    load_member_args(sa, args + bm.member);
    __syncthreads();
    mag_ctcell_body<T, CPT, FADE, CG>(sa, (unsigned)bm.block);
}

}  // namespace img
