// Window form of the magnet sweep along X (magnet/magnetFlux.m:14-31, magnet/relaxingMagnet.m:15-60,
// magnet/MagnetArray.m:36-38) for pencils that fit one CTA with circ or const ends.
//
// Each thread owns C consecutive cells of a pencil and computes the whole upwind/TVD chain for them in
// registers over a window that reaches 4 cells beyond each end (the chain's stencil depth): the corner
// velocity at C+8 cells, its smoothing at C+6, the upwind flux and predictor, the corrector fluxes and
// the limiter at C+1.  Nothing is exchanged between threads: the window's extra cells are recomputed
// from global memory (L1-resident: neighbouring threads load the same lines).  The only barrier
// separates the reads of B_I (and, in the CT pass, of B_X) from their in-place update, so a pencil's
// segments must share a CTA.
//   chain  per transverse component I: vg from rho, p_X at the pencil and its I-1 neighbour, the
//          1-2-1 smoothing, velocityFlow, store.fluxR, store, wMag, flux with the limiter; B_I updated
//          in place and the limited flux F_I written to scratch for the CT pass.
//   CT     C_I = F_I - F_I.shift(I,+1), D_I = C_I.shift(X,-1), B_X = (B_X - dt/dI1 D_1) - dt/dI2 D_2
//          in place, and the cell-centred B_X and B_I2.
// Pencil ends along X (mag-class BC): circ wraps the window; const makes every shifted array take its
// own end value (constant_shift.m), so after each stage the window cells beyond the pencil's end copy
// the stage's value at the end cell.  Transverse shifts (along I) use circ or const too; other
// boundaries and a run's first sweeps (stored-edge capture) take the tile kernels (magnet_sweep.cuh).
// Per cell the arithmetic is that of the tile kernels.
// Along x a pencil's length need not be a multiple of C (the last segment is ragged: S = ceil(N / C)
// segments, threads past them idle), and a pencil longer than one CTA's segments spans the CTAs of a
// thread-block cluster (one pencil per cluster; segment s = rank * NT + thread), whose barrier then
// separates the reads from the in-place writes.
#pragma once

#include "seg_fluid.cuh"

namespace img {

// Offset of the transverse neighbour pencil at I-1 (n = -1) or I+1 (n = +1) along dim e for a pencil
// whose coordinate along e is ie (of ne), under a circ or const BC on that side; 0 means the pencil
// itself (const edge, or dimension e not shifted).
__device__ __forceinline__ long long trans_offset(int ie, int ne, long long se, int n, int mode, bool shifted) {
    if (!shifted) return 0;
    if (n < 0) return ie > 0 ? -se : (mode == BC_CIRC ? (long long)(ne - 1) * se : 0);
    return ie < ne - 1 ? se : (mode == BC_CIRC ? -(long long)(ne - 1) * se : 0);
}

// Global row of window cell j of segment s (rows r0 + j, wrapped for circ, clamped for const ends).
// The window reaches at most 4 rows past a segment, so a pencil shorter than that wraps more than once
// (r >= -4 and r < N + C + 4: the loops run at most a few times).
__host__ __device__ __forceinline__ int win_row_multi(int r, int N, bool circ_lo, bool circ_hi) {
    if (r < 0) {
        if (!circ_lo) return 0;
        do r += N; while (r < 0);
        return r;
    }
    if (r >= N) {
        if (!circ_hi) return N - 1;
        do r -= N; while (r >= N);
        return r;
    }
    return r;
}

// The same where one wrap suffices: rows r >= -N and r < 2N (a window that reaches H rows past its
// segment, on a pencil of N >= C + H rows: the last segment starts at row N - 1 at most).  Selects
// only, no loop.
__host__ __device__ __forceinline__ int win_row_once(int r, int N, bool circ_lo, bool circ_hi) {
    const int lo = circ_lo ? r + N : 0, hi = circ_hi ? r - N : N - 1;
    return r < 0 ? lo : (r >= N ? hi : r);
}

// Global offsets of the W window rows r0 - H .. r0 - H + W - 1 (H rows of halo below the segment,
// W - C - H above).  The choice between the two row functions is uniform over the launch (N is).
template <int C, int W, int H>
__device__ __forceinline__ void win_rows(long long (&orow)[W], long long base, int r0, int N, long long sd,
                                         bool circ_lo, bool circ_hi) {
    constexpr int REACH = (H > W - C - H ? H : W - C - H);
    if (N >= C + REACH) {
#pragma unroll
        for (int j = 0; j < W; ++j) orow[j] = base + (long long)win_row_once(r0 + j - H, N, circ_lo, circ_hi) * sd;
    } else {
#pragma unroll
        for (int j = 0; j < W; ++j) orow[j] = base + (long long)win_row_multi(r0 + j - H, N, circ_lo, circ_hi) * sd;
    }
}

// Const ends: the window cells of a stage array A (local cells LO .. HI-1 at A[j + OFS]) past the
// pencil's lower end copy its row 0 (local cell lend = -r0), those past its upper end its last row
// (local cell hend = N - 1 - r0): the const ghost of every shifted array (constant_shift.m).  A window
// reaches 4 cells past its segment, so near an end several segments' windows cross it, and the end row
// may be a window cell rather than an own one (short segments, a ragged last segment).
template <typename T, int OFS, int LO, int HI>
__device__ __forceinline__ void const_fill(T* A, bool circ_lo, bool circ_hi, int lend, int hend) {
    if (!circ_lo && lend > LO) {
        T e = A[LO + OFS];
#pragma unroll
        for (int j = LO + 1; j < HI; ++j)
            if (j == lend) e = A[j + OFS];
#pragma unroll
        for (int j = LO; j < HI; ++j)
            if (j < lend) A[j + OFS] = e;
    }
    if (!circ_hi && hend < HI - 1) {
        T e = A[LO + OFS];
#pragma unroll
        for (int j = LO + 1; j < HI; ++j)
            if (j == hend) e = A[j + OFS];
#pragma unroll
        for (int j = LO; j < HI; ++j)
            if (j > hend) A[j + OFS] = e;
    }
}

// The segment placement of seg_fluid.cuh plus the pencil's coordinates along the transverse dims; G is
// the pencil's segment count S, over the CL CTAs of a cluster where CL > 1.
struct WinPos {
    int b, s, c1, c2;
    bool colok;
    long long base;
    __device__ __forceinline__ void init(const SweepGeom& g, unsigned vblock) {
        int t = threadIdx.x;
        unsigned blk = vblock;
        if (g.CL > 1) {   // cluster rank r holds segments r * NT .. r * NT + NT - 1 of the bundle's pencil
            blk = g.div_cl.div(vblock);
            t += (int)(vblock - blk * (unsigned)g.CL) * g.NT;
        }
        const unsigned q = g.div_lanes.div((unsigned)t);
        if (g.d == 0) { b = (int)q; s = t - b * g.G; }
        else { s = (int)q; b = t - s * g.Wb; }
        const int col = (int)(blk * (unsigned)g.Wb + (unsigned)b);
        colok = col < g.ncol && b < g.Wb && s < g.G;   // threads past the last segment idle
        const unsigned c = colok ? (unsigned)col : 0u;
        c2 = (int)g.div_n1.div(c);
        c1 = (int)(c - (unsigned)c2 * (unsigned)g.n1);
        base = c1 * g.s1 + (long long)c2 * g.s2;
    }
};

// Every read of the pencil's arrays before any in-place write: the CTA's barrier, or the cluster's.
__device__ __forceinline__ void win_barrier(const SweepGeom& g) {
    if (g.CL > 1) cluster_sync();
    else __syncthreads();
}

template <typename T, int C>
__device__ __forceinline__ void mag_chain_win_body(const MagArgs& a, unsigned vblock) {
    pdl_wait();
    if (a.tm->done || (a.sg.CL == 1 && a.tm->error)) return;   // clusters: as in the fluid sweeps
    constexpr int W = C + 8;   // window cells -4 .. C+3 (index j + 4)
    const SweepGeom& g = a.sg;
    const Geom& gg = g.g;
    const int N = g.N, d = a.X - 1;
    WinPos wp;
    wp.init(g, vblock);
    const int r0 = wp.s * C;
    const bool circ_lo = a.modeX[0] == BC_CIRC, circ_hi = a.modeX[1] == BC_CIRC;
    const bool fill_lo = !circ_lo && wp.s == 0;
    const int lend = -r0, hend = N - 1 - r0;    // local cells of the pencil's first and last rows
    const int nown = N - r0 < C ? N - r0 : C;   // own cells inside the pencil (fewer in a ragged last segment)
    // vector stores along x need every segment to start on a multiple of C: pencils (and the arrays,
    // 256-byte aligned) start on one only where C divides N; ragged pencils store cell by cell
    const bool vec = d == 0 && N % C == 0;
    const long long sd = g.sd;
    const T* rho = reinterpret_cast<const T*>(a.q[Q_RHO]);
    const T* pX = reinterpret_cast<const T*>(a.q[Q_PX + d]);
    const double dt = a.tm->dt;
    const T ff = (T)(0.5 * dt / a.dx);
    const T ff2 = T(2) * ff;

    // ---- loads: the corner velocity (magnetFlux.m:18-19) over the window, B_I over cells -3 .. C+2 ----
    long long orow[W];
    // idle threads (past the last segment) read rows of segment 0 and store nothing
    win_rows<C, W, 4>(orow, wp.base, wp.colok ? r0 : 0, N, sd, circ_lo, circ_hi);
    T vgr[2][W], bI[2][W - 2];
#pragma unroll
    for (int q = 0; q < 2; ++q) {
        const int e = a.I[q] - 1;
        const int ie = e == g.d1 ? wp.c1 : wp.c2;
        const int ne = sel3(e, gg.n[0], gg.n[1], gg.n[2]);
        const long long se = sel3(e, gg.s[0], gg.s[1], gg.s[2]);
        const long long nbp = trans_offset(ie, ne, se, -1, a.modeI_mom[q][0], a.shiftI[q] != 0);    // p_X: mom class
        const long long nbr = trans_offset(ie, ne, se, -1, a.modeI_mass[q][0], a.shiftI[q] != 0);   // rho: mass class
        const T* BI = reinterpret_cast<const T*>(a.q[Q_BX + e]);
#pragma unroll
        for (int j = 0; j < W; ++j) {
            const long long o = orow[j];
            const T pm = pX[o + nbp], rm = rho[o + nbr];
            if constexpr (sizeof(T) == 4) vgr[q][j] = (pm + pX[o]) * rcp_approx(rm + rho[o]);
            else vgr[q][j] = (pm + pX[o]) / (rm + rho[o]);
            if (j >= 1 && j < W - 1) bI[q][j - 1] = BI[o];
        }
    }
    win_barrier(g);   // every thread has read B_I before any writes it

#pragma unroll
    for (int q = 0; q < 2; ++q) {
        const int e = a.I[q] - 1;
        // vg = 0.25*(vg.shift(X,-1) + vg.shift(X,1) + 2*vg) at cells -3 .. C+2 (index j + 3)
        T vg[W - 2];
#pragma unroll
        for (int j = -3; j < C + 3; ++j) vg[j + 3] = T(0.25) * (vgr[q][j + 3] + vgr[q][j + 5] + T(2) * vgr[q][j + 4]);
        const_fill<T, 3, -3, C + 3>(vg, circ_lo, circ_hi, lend, hend);
        // velocityFlow = (vg + vg.shift(X,1)) < 0 and store.fluxR = F*(1-vf) + F.shift(X,1)*vf at cells
        // -3 .. C+1 (index j + 3), F = B_I * vg (relaxingMagnet.m:17-24)
        T Fr[W - 2], vf[W - 3], fR[W - 3];
#pragma unroll
        for (int j = -3; j < C + 3; ++j) Fr[j + 3] = bI[q][j + 3] * vg[j + 3];
        const_fill<T, 3, -3, C + 3>(Fr, circ_lo, circ_hi, lend, hend);
#pragma unroll
        for (int j = -3; j < C + 2; ++j) {
            vf[j + 3] = (vg[j + 3] + vg[j + 4]) < T(0) ? T(1) : T(0);
            fR[j + 3] = Fr[j + 3] * (T(1) - vf[j + 3]) + Fr[j + 4] * vf[j + 3];
        }
        const_fill<T, 3, -3, C + 2>(vf, circ_lo, circ_hi, lend, hend);
        const_fill<T, 3, -3, C + 2>(fR, circ_lo, circ_hi, lend, hend);
        // store = B_I - ff*(fluxR - fluxR.shift(X,-1)); wMag = store.*velGrid at cells -2 .. C+1 (j + 2)
        T Wm[W - 4];
#pragma unroll
        for (int j = -2; j < C + 2; ++j) {
            const T st = bI[q][j + 3] - ff * (fR[j + 3] - fR[j + 2]);
            Wm[j + 2] = st * vg[j + 3];
        }
        const_fill<T, 2, -2, C + 2>(Wm, circ_lo, circ_hi, lend, hend);
        // flux and its TVD correction (relaxingMagnet.m:32-51) at cells -1 .. C-1 (index j + 1)
        T Fl[C + 1];
#pragma unroll
        for (int j = -1; j < C; ++j) {
            const T w = Wm[j + 2], v = vf[j + 3];
            const T p1 = Wm[j + 3], p2 = Wm[j + 4], m1 = Wm[j + 1];
            const T fx = w * (T(1) - v) + p1 * v;
            const T dFluxR = p1 - (v * p2 + (T(1) - v) * w);
            const T dFluxL = w - (v * p1 + (T(1) - v) * m1);
            Fl[j + 1] = fx + limiter_corr<T>(a.limiter, dFluxL, dFluxR);
        }
        if (fill_lo) Fl[0] = Fl[1];
        // B_I = B_I - 2ff*(flux - flux.shift(X,-1)) (relaxingMagnet.m:49); flux -> scratch for CT
        if (wp.colok) {
            T* BI = reinterpret_cast<T*>(a.q[Q_BX + e]);
            T* Fo = reinterpret_cast<T*>(q ? a.F[1] : a.F[0]);
            T bnew[C], fo[C];
#pragma unroll
            for (int k = 0; k < C; ++k) {
                bnew[k] = bI[q][k + 3] - ff2 * (Fl[k + 1] - Fl[k]);
                fo[k] = Fl[k + 1];
            }
            const long long o0 = wp.base + (long long)r0 * sd;
            if (nown == C) {
                seg_store<T, C>(BI, o0, sd, vec, bnew);
                seg_store<T, C>(Fo, o0, sd, vec, fo);
            } else {
#pragma unroll
                for (int k = 0; k < C; ++k)
                    if (k < nown) { BI[o0 + k * sd] = bnew[k]; Fo[o0 + k * sd] = fo[k]; }
            }
        }
    }
    pdl_trigger();
}

template <typename T, int C>
__device__ __forceinline__ void mag_ct_win_body(const MagArgs& a, unsigned vblock) {
    pdl_wait();
    if (a.tm->done || (a.sg.CL == 1 && a.tm->error)) return;   // clusters: as in the fluid sweeps
    const SweepGeom& g = a.sg;
    const Geom& gg = g.g;
    const int N = g.N, d = a.X - 1;
    WinPos wp;
    wp.init(g, vblock);
    const int r0 = wp.s * C;
    const bool circ_lo = a.modeX[0] == BC_CIRC, circ_hi = a.modeX[1] == BC_CIRC;
    const bool fill_lo = !circ_lo && wp.s == 0, fill_hi = !circ_hi && r0 + C >= N;
    const int nown = N - r0 < C ? N - r0 : C;
    const bool vec = d == 0 && N % C == 0;   // as in the chain
    const long long sd = g.sd;
    const double dt = a.tm->dt;
    // window cells -1 .. C (index j + 1)
    long long orow[C + 2];
    win_rows<C, C + 2, 1>(orow, wp.base, wp.colok ? r0 : 0, N, sd, circ_lo, circ_hi);
    // C_q = F_q - F_q.shift(I_q, +1) over the window (relaxingMagnet.m:56)
    T Cq[2][C + 2];
#pragma unroll
    for (int q = 0; q < 2; ++q) {
        const int e = a.I[q] - 1;
        const int ie = e == g.d1 ? wp.c1 : wp.c2;
        const T* F = reinterpret_cast<const T*>(q ? a.F[1] : a.F[0]);
        const long long nb = trans_offset(ie, sel3(e, gg.n[0], gg.n[1], gg.n[2]), sel3(e, gg.s[0], gg.s[1], gg.s[2]), +1,
                                          a.modeI_mag[q][1], a.shiftI[q] != 0);
#pragma unroll
        for (int j = 0; j < C + 2; ++j) {
            const T fv = F[orow[j]];
            Cq[q][j] = fv - F[orow[j] + nb];
        }
    }
    T* BX = reinterpret_cast<T*>(a.q[Q_BX + d]);
    T bxo[C + 1];
#pragma unroll
    for (int j = 0; j <= C; ++j) bxo[j] = BX[orow[j + 1]];
    // cell-centred B_I2 needs B_I2 at the pencil and its I2+1 neighbour (read only here)
    const int e2 = a.I[1] - 1;
    const T* BI2 = reinterpret_cast<const T*>(a.q[Q_BX + e2]);
    const long long nb2 = trans_offset(e2 == g.d1 ? wp.c1 : wp.c2, sel3(e2, gg.n[0], gg.n[1], gg.n[2]),
                                       sel3(e2, gg.s[0], gg.s[1], gg.s[2]), +1, a.modeI_mag[1][1], a.shiftI[1] != 0);
    win_barrier(g);   // every thread has read B_X before any writes it
    // D_q = C_q.shift(X,-1); B_X = (B_X - dt/dI1 D_1) - dt/dI2 D_2 at cells 0 .. C (index j)
    const T f0 = (T)(dt / a.dI[0]), f1 = (T)(dt / a.dI[1]);
    T bx[C + 1];
#pragma unroll
    for (int j = 0; j <= C; ++j) {
        T D0 = Cq[0][j], D1 = Cq[1][j];
        if (j == 0 && fill_lo) { D0 = Cq[0][1]; D1 = Cq[1][1]; }
        bx[j] = (bxo[j] - f0 * D0) - f1 * D1;
    }
    if (fill_hi) {   // B_X.shift(X, +1) past the end cell nown - 1 is that cell's value (const)
        T e = bx[0];
#pragma unroll
        for (int j = 1; j < C; ++j)
            if (j == nown - 1) e = bx[j];
#pragma unroll
        for (int j = 1; j <= C; ++j)
            if (j == nown) bx[j] = e;
    }
    pdl_trigger();
    if (!wp.colok) return;
    T* CBX = reinterpret_cast<T*>(a.q[Q_CBX + d]);
    T* CB2 = reinterpret_cast<T*>(a.q[Q_CBX + e2]);
    const long long o0 = wp.base + (long long)r0 * sd;
    T bn[C], cbx[C], cb2[C];
#pragma unroll
    for (int k = 0; k < C; ++k) {
        bn[k] = bx[k];
        cbx[k] = T(0.5) * (bx[k] + bx[k + 1]);
        const long long o = o0 + (long long)k * sd;   // rows past a ragged end: not read (nor stored)
        const T b2 = k < nown ? BI2[o] : T(0);
        cb2[k] = k < nown ? T(0.5) * (b2 + BI2[o + nb2]) : T(0);
    }
    if (nown == C) {
        seg_store<T, C>(BX, o0, sd, vec, bn);
        seg_store<T, C>(CBX, o0, sd, vec, cbx);
        seg_store<T, C>(CB2, o0, sd, vec, cb2);
    } else {
#pragma unroll
        for (int k = 0; k < C; ++k)
            if (k < nown) {
                BX[o0 + k * sd] = bn[k];
                CBX[o0 + k * sd] = cbx[k];
                CB2[o0 + k * sd] = cb2[k];
            }
    }
}

template <typename T, int C>
__global__ void __launch_bounds__(512, 1) mag_chain_win_kernel(const __grid_constant__ MagArgs a) {
    mag_chain_win_body<T, C>(a, blockIdx.x);
}

template <typename T, int C>
__global__ void __launch_bounds__(512, 1) mag_ct_win_kernel(const __grid_constant__ MagArgs a) {
    mag_ct_win_body<T, C>(a, blockIdx.x);
}

template <typename T, int C>
__global__ void __launch_bounds__(512, 1) mag_chain_win_batch_kernel(const MagArgs* __restrict__ args,
                                                                      const BlockMap* __restrict__ map) {
    __shared__ MagArgs sa;
    const BlockMap bm = map[blockIdx.x];
    load_member_args(sa, args + bm.member);
    __syncthreads();
    mag_chain_win_body<T, C>(sa, (unsigned)bm.block);
}

template <typename T, int C>
__global__ void __launch_bounds__(512, 1) mag_ct_win_batch_kernel(const MagArgs* __restrict__ args,
                                                                   const BlockMap* __restrict__ map) {
    __shared__ MagArgs sa;
    const BlockMap bm = map[blockIdx.x];
    load_member_args(sa, args + bm.member);
    __syncthreads();
    mag_ct_win_body<T, C>(sa, (unsigned)bm.block);
}

}  // namespace img
