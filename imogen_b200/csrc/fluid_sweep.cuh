// Fused relaxing-TVD fluid sweep along one dimension (fluid/relaxingFluid.m:16-73,
// fluid/wFluidFlux.m:14-44, pressure/pressure.m:23-64, flux/*Limiter.m).
//
// One launch updates rho, p and E for every cell: per pencil it computes the freezing speed
// (pencil max of |v| + c_s, a column reduction), the predictor half step, the second freezing
// speed on the half-step state, and the TVD-limited corrector, with the boundary ghosts of the
// four flux arrays of each variable synthesised in the same pass.  State is read once and written
// once; nothing else touches HBM except the stored edges of stateful boundaries (trans, wall).
#pragma once

#include "pencil.cuh"

namespace img {

struct FluidArgs {
    SweepGeom sg;
    void* q[NQ];
    DevTime* tm;
    double gamma;
    double minmass;
    double dx;             // grid spacing along the sweep
    int limiter;
    int mode[4][2];        // BC mode per class (mass, mom, ener, mag) for dim d: [class][side]
    int act[4];            // trans edge store ACTIVE(DIRECT) per class (linear-index reading)
    const double* fade;    // fade_shift coefficients (length fade_f)
    int fade_f;
    double bc_inf;
    const EdgeTable* edges;
    int init_store;        // first assignment of store.fluxR/L: take their stored edges
    int init_flux;         // first assignment of fluxR/L
    int mhd;               // cell-centred B is nonzero / the magnet is active
    int use_b[3];          // pressure.m:28-33 skips components with isZero set
    int cfl;               // accumulate the CFL maxima of the new state (fused TimeManager pass)
};

constexpr int FLUID_NSLOT = 10;

template <typename T>
__device__ __forceinline__ T ldq(const void* p, long long i) { return reinterpret_cast<const T*>(p)[i]; }
template <typename T>
__device__ __forceinline__ void stq(void* p, long long i, T v) { reinterpret_cast<T*>(p)[i] = v; }

// w arrays of wFluidFlux.m:31-44 for one cell (X = sweep dim d).
template <typename T>
__device__ __forceinline__ void wflux(int d, const T u[5], const T bb[3], T press, T cf, T w[5]) {
    const T pX = sel3(d, u[1], u[2], u[3]);
    T velocity = pX / u[0];
    w[0] = pX / cf;
    T bX = sel3(d, bb[0], bb[1], bb[2]);
    T we = velocity * (u[4] + press) - bX * (bb[0] * u[1] + bb[1] * u[2] + bb[2] * u[3]) / u[0];
    w[4] = we / cf;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        T dirv = c == d ? T(1) : T(0);
        w[1 + c] = (velocity * u[1 + c] + press * dirv - bX * bb[c]) / cf;
    }
}

// Column max over the pencil (and over the cluster): returns the max for this thread's column.
template <typename T, int CPT, int NSLOT, bool H2>
__device__ double column_max(Pencil<T, CPT, NSLOT, H2>& pc, unsigned long long* red, double local) {
    const SweepGeom& s = *pc.sg;
    // lanes that share a column: d == 0 -> consecutive groups of min(G,32); else stride Wb
    unsigned mask = 0xffffffffu;
    if (s.d == 0) {
        int w = s.G < 32 ? s.G : 32;
        for (int o = w / 2; o > 0; o >>= 1) local = fmax(local, __shfl_xor_sync(mask, local, o));
    } else {
        for (int o = 16; o >= s.Wb; o >>= 1) local = fmax(local, __shfl_xor_sync(mask, local, o));
    }
    if (pc.colok) atomic_max_nonneg(&red[pc.b], local);
    pc.csync();
    double m = __longlong_as_double((long long)red[pc.b]);
    for (int r = 0; r < s.CL; ++r) {
        if (r == pc.rank) continue;
        unsigned long long* rp = pc.remote(red, r);
        m = fmax(m, __longlong_as_double((long long)rp[pc.b]));
    }
    return m;
}

// Ghost value at the pencil end for A.shift(d, -1)[0] (lower) or A.shift(d, +1)[N-1] (upper),
// for the modes without fade damping (fade uses the const ghost, damping applied by the caller).
// edge_ptr: stored edge slice of this object for (d, side) or nullptr.
template <typename T, int CPT, int NSLOT, bool H2>
__device__ T end_ghost(const Pencil<T, CPT, NSLOT, H2>& pc, int slot, bool upper, int mode, int act, bool flip,
                       double* edge_ptr, double bc_inf) {
    int N = pc.sg->N;
    switch (mode) {
        case BC_CIRC: return upper ? pc.endv(slot, 0) : pc.endv(slot, N - 1);
        case BC_MIRROR: { T v = upper ? pc.endv(slot, N - 2) : pc.endv(slot, 1); return flip ? -v : v; }
        case BC_WALL: return (T)edge_ptr[pc.col];
        case BC_TRANS: {
            double e = 0.0;
            T a0, a1, a2;   // array values at x = 1, 2, 3 (x = 3 is the edge cell)
            if (!upper) {
                a0 = pc.endv(slot, trans_pick_lower(N, 1, 0));
                a1 = pc.endv(slot, trans_pick_lower(N, 1, 1));
                a2 = pc.endv(slot, 0);
            } else {
                a0 = pc.endv(slot, trans_pick_upper(N, 1, 0));
                a1 = pc.endv(slot, trans_pick_upper(N, 1, 1));
                a2 = pc.endv(slot, N - 1);
            }
            if (act) {
                e = edge_drift(edge_ptr[pc.col], (double)a2);
                edge_ptr[pc.col] = e;
            }
            return (T)trans_ghost((double)a0, (double)a1, (double)a2, e, bc_inf, 4.0, (double)a2);
        }
        default:   // const and fade (const ghost)
            return upper ? pc.endv(slot, N - 1) : pc.endv(slot, 0);
    }
}

// A.shift(d, -1) (sm) and A.shift(d, +1) (sp) at this thread's rows for array A published in `slot`.
template <typename T, int CPT, int NSLOT, bool H2>
__device__ void shifted(const Pencil<T, CPT, NSLOT, H2>& pc, const FluidArgs& a, int slot, const T (&A)[CPT], int cls,
                        bool flip, bool need_m, bool need_p, double* e_lo, double* e_hi, T (&sm)[CPT], T (&sp)[CPT]) {
    const int N = pc.sg->N;
    const int mlo = a.mode[cls][0], mhi = a.mode[cls][1];
    T glo = T(0), ghi = T(0);
    bool own0 = pc.nv > 0 && pc.r0 == 0;
    bool ownN = pc.nv > 0 && pc.r0 + pc.nv - 1 == N - 1;
    if (need_m && own0) glo = end_ghost(pc, slot, false, mlo, a.act[cls], flip, e_lo, a.bc_inf);
    if (need_p && ownN) ghi = end_ghost(pc, slot, true, mhi, a.act[cls], flip, e_hi, a.bc_inf);
#pragma unroll
    for (int k = 0; k < CPT; ++k) {
        if (k >= pc.nv) { sm[k] = T(0); sp[k] = T(0); continue; }
        int r = pc.r0 + k;
        if (need_m) {
            T v = r == 0 ? glo : pc.prev(slot, A, k);
            if (mlo == BC_FADE) v = fade_apply(v, r, N, a.fade, a.fade_f, pc.endv(slot, 0), pc.endv(slot, N - 2));
            sm[k] = v;
        }
        if (need_p) {
            T v = r == N - 1 ? ghi : pc.next(slot, A, k);
            if (mhi == BC_FADE) v = fade_apply(v, r, N, a.fade, a.fade_f, pc.endv(slot, 1), pc.endv(slot, N - 1));
            sp[k] = v;
        }
    }
}

// First assignment of an InitializedArray takes its stored edges on every face it lies on
// (classes/InitializedArray.m:43-47 -> Edges.m:37-110).
template <typename T, int CPT, int NSLOT, bool H2>
__device__ void init_edges(const Pencil<T, CPT, NSLOT, H2>& pc, const EdgeTable* et, int obj, const T (&A)[CPT]) {
    const Geom& g = pc.sg->g;
#pragma unroll
    for (int k = 0; k < CPT; ++k) {
        if (k >= pc.nv) continue;
        int x, y, z;
        pc.coords(k, x, y, z);
#pragma unroll
        for (int e = 0; e < 3; ++e) {
            if (e >= g.ndims) continue;
            double* lo = et->p[obj][e][0];
            double* hi = et->p[obj][e][1];
            int ce = sel3(e, x, y, z);
            long long fi = face_index(g, e, x, y, z);
            if (lo && ce == 0) lo[fi] = (double)A[k];
            if (hi && ce == g.n[e] - 1) hi[fi] = (double)A[k];
        }
    }
}

template <typename T, bool MHD, int CPT>
__global__ void __launch_bounds__(512) fluid_sweep_kernel(const FluidArgs a) {
    extern __shared__ __align__(16) unsigned char smem[];
    if (a.tm->done || a.tm->error) return;   // uniform over the grid: a stopped or failed run does nothing
    __shared__ unsigned long long red[2][32];
    using PC = Pencil<T, CPT, FLUID_NSLOT>;
    PC pc;
    pc.init(a.sg, smem);
    const int d = a.sg.d;
    for (int i = threadIdx.x; i < 64; i += blockDim.x) (&red[0][0])[i] = 0ull;
    __syncthreads();

    const double G = a.gamma;
    const double dt = a.tm->dt;
    const T ff = (T)(dt / a.dx);
    const T half_ffx = (T)(0.5 * (dt / a.dx));

    // ---- load u (rho, px, py, pz, E) and cell-centred B --------------------------------------------
    T u[5][CPT], bb[3][CPT];
#pragma unroll
    for (int k = 0; k < CPT; ++k) {
        if (pc.valid(k)) {
            long long o = pc.off(k);
#pragma unroll
            for (int v = 0; v < 5; ++v) u[v][k] = ldq<T>(a.q[v], o);
#pragma unroll
            for (int c = 0; c < 3; ++c) bb[c][k] = MHD ? ldq<T>(a.q[Q_CBX + c], o) : T(0);
        } else {
#pragma unroll
            for (int v = 0; v < 5; ++v) u[v][k] = v == 0 ? T(1) : T(0);
#pragma unroll
            for (int c = 0; c < 3; ++c) bb[c][k] = T(0);
        }
    }

    auto msq_of = [&](int k) -> double {
        double m = 0.0;
        if (MHD) {
#pragma unroll
            for (int c = 0; c < 3; ++c)
                if (a.use_b[c]) m = m + (double)bb[c][k] * (double)bb[c][k];
        }
        return m;
    };

    // ---- freezing speed #1 (wFluidFlux.m:18-22) ----------------------------------------------------
    T press[CPT];
    double lmax = 0.0;
#pragma unroll
    for (int k = 0; k < CPT; ++k) {
        PressOut po = pressure_totsnd(G, u[0][k], u[1][k], u[2][k], u[3][k], u[4][k], msq_of(k));
        press[k] = (T)(po.p + 0.0);
        T cs = (T)po.cs;
        T spd = fabs(sel3(d, u[1][k], u[2][k], u[3][k]) / u[0][k]) + cs;
        if (pc.valid(k)) lmax = fmax(lmax, (double)spd);
    }
    const T cf = (T)column_max(pc, red[0], lmax);

    // ---- predictor (relaxingFluid.m:30-39) ----------------------------------------------------------
    T R[5][CPT], L[5][CPT];
#pragma unroll
    for (int k = 0; k < CPT; ++k) {
        T uu[5] = {u[0][k], u[1][k], u[2][k], u[3][k], u[4][k]};
        T b3[3] = {bb[0][k], bb[1][k], bb[2][k]};
        T w[5];
        wflux<T>(d, uu, b3, press[k], cf, w);
#pragma unroll
        for (int v = 0; v < 5; ++v) {
            R[v][k] = T(0.5) * (uu[v] + w[v]);
            L[v][k] = T(0.5) * (uu[v] - w[v]);
        }
    }
    const EdgeTable* et = a.edges;
    const int cls_of[5] = {CLS_MASS, CLS_MOM, CLS_MOM, CLS_MOM, CLS_ENER};
    if (a.init_store) {
#pragma unroll
        for (int v = 0; v < 5; ++v) {
            init_edges(pc, et, fluid_obj(v, FO_STORE_R), R[v]);
            init_edges(pc, et, fluid_obj(v, FO_STORE_L), L[v]);
        }
    }
#pragma unroll
    for (int v = 0; v < 5; ++v) {
        pc.publish(v, R[v]);
        pc.publish(5 + v, L[v]);
    }
    pc.csync();
    T us[5][CPT];
    {
        T sm[CPT], sp[CPT], dummy[CPT];
#pragma unroll
        for (int v = 0; v < 5; ++v) {
            bool flip = (v == 1 + d);
            int cls = cls_of[v];
            shifted(pc, a, v, R[v], cls, flip, true, false, et->p[fluid_obj(v, FO_STORE_R)][d][0], nullptr, sm, dummy);
            shifted(pc, a, 5 + v, L[v], cls, flip, false, true, nullptr, et->p[fluid_obj(v, FO_STORE_L)][d][1], dummy,
                    sp);
#pragma unroll
            for (int k = 0; k < CPT; ++k) us[v][k] = u[v][k] - half_ffx * cf * (R[v][k] - sm[k] + L[v][k] - sp[k]);
        }
    }
#pragma unroll
    for (int k = 0; k < CPT; ++k) us[0][k] = us[0][k] > (T)a.minmass ? us[0][k] : (T)a.minmass;

    // ---- freezing speed #2 on the half-step state (relaxingFluid.m:47-50) --------------------------
    lmax = 0.0;
#pragma unroll
    for (int k = 0; k < CPT; ++k) {
        if (!pc.valid(k)) { us[0][k] = T(1); us[1][k] = us[2][k] = us[3][k] = us[4][k] = T(0); }
        PressOut po = pressure_totsnd(G, us[0][k], us[1][k], us[2][k], us[3][k], us[4][k], msq_of(k));
        press[k] = (T)(po.p + 0.0);
        T spd = fabs(sel3(d, us[1][k], us[2][k], us[3][k]) / us[0][k]) + (T)po.cs;
        if (pc.valid(k)) lmax = fmax(lmax, (double)spd);
    }
    const T cfs = (T)column_max(pc, red[1], lmax);

    // ---- corrector fluxes and limiter (relaxingFluid.m:52-62) ---------------------------------------
#pragma unroll
    for (int k = 0; k < CPT; ++k) {
        T uu[5] = {us[0][k], us[1][k], us[2][k], us[3][k], us[4][k]};
        T b3[3] = {bb[0][k], bb[1][k], bb[2][k]};
        T w[5];
        wflux<T>(d, uu, b3, press[k], cfs, w);
#pragma unroll
        for (int v = 0; v < 5; ++v) {
            R[v][k] = T(0.5) * (uu[v] + w[v]);
            L[v][k] = T(0.5) * (uu[v] - w[v]);
        }
    }
    if (a.init_flux) {
#pragma unroll
        for (int v = 0; v < 5; ++v) {
            init_edges(pc, et, fluid_obj(v, FO_R), R[v]);
            init_edges(pc, et, fluid_obj(v, FO_L), L[v]);
        }
    }
    // the column_max sync above guarantees every thread is done reading the predictor slots
#pragma unroll
    for (int v = 0; v < 5; ++v) {
        pc.publish(v, R[v]);
        pc.publish(5 + v, L[v]);
    }
    pc.csync();
    {
        T sm[CPT], sp[CPT];
#pragma unroll
        for (int v = 0; v < 5; ++v) {
            bool flip = (v == 1 + d);
            int cls = cls_of[v];
            // fluxR: dL = R - R.shift(-1), dR = R.shift(+1) - R
            shifted(pc, a, v, R[v], cls, flip, true, true, et->p[fluid_obj(v, FO_R)][d][0],
                    et->p[fluid_obj(v, FO_R)][d][1], sm, sp);
            T Rn[CPT];
#pragma unroll
            for (int k = 0; k < CPT; ++k) Rn[k] = R[v][k] + limiter_corr<T>(a.limiter, R[v][k] - sm[k], sp[k] - R[v][k]);
            // fluxL: dL = L.shift(-1) - L, dR = L - L.shift(+1)
            shifted(pc, a, 5 + v, L[v], cls, flip, true, true, et->p[fluid_obj(v, FO_L)][d][0],
                    et->p[fluid_obj(v, FO_L)][d][1], sm, sp);
#pragma unroll
            for (int k = 0; k < CPT; ++k) {
                L[v][k] = L[v][k] + limiter_corr<T>(a.limiter, sm[k] - L[v][k], L[v][k] - sp[k]);
                R[v][k] = Rn[k];
            }
        }
    }
    pc.csync();   // all reads of the limiter-stage slots are done
#pragma unroll
    for (int v = 0; v < 5; ++v) {
        pc.publish(v, R[v]);
        pc.publish(5 + v, L[v]);
    }
    pc.csync();

    // ---- corrector update (relaxingFluid.m:64-71) ---------------------------------------------------
    T unew[5][CPT];
    {
        T sm[CPT], sp[CPT], dummy[CPT];
#pragma unroll
        for (int v = 0; v < 5; ++v) {
            bool flip = (v == 1 + d);
            int cls = cls_of[v];
            shifted(pc, a, v, R[v], cls, flip, true, false, et->p[fluid_obj(v, FO_R)][d][0], nullptr, sm, dummy);
            shifted(pc, a, 5 + v, L[v], cls, flip, false, true, nullptr, et->p[fluid_obj(v, FO_L)][d][1], dummy, sp);
#pragma unroll
            for (int k = 0; k < CPT; ++k) unew[v][k] = u[v][k] - ff * cfs * (R[v][k] - sm[k] + L[v][k] - sp[k]);
        }
    }
#pragma unroll
    for (int k = 0; k < CPT; ++k) unew[0][k] = unew[0][k] > (T)a.minmass ? unew[0][k] : (T)a.minmass;

#pragma unroll
    for (int k = 0; k < CPT; ++k) {
        if (!pc.valid(k)) continue;
        long long o = pc.off(k);
#pragma unroll
        for (int v = 0; v < 5; ++v) stq<T>(a.q[v], o, unew[v][k]);
    }

    // ---- fused CFL maxima of the new state (TimeManager.m:65-77) -----------------------------------
    if (a.cfl) {
        double m3[3] = {0.0, 0.0, 0.0};
#pragma unroll
        for (int k = 0; k < CPT; ++k) {
            if (!pc.valid(k)) continue;
            double cs = sound_speed(G, (double)unew[0][k], (double)unew[1][k], (double)unew[2][k], (double)unew[3][k],
                                    (double)unew[4][k], msq_of(k));
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                double v = fabs((double)unew[1 + c][k] / (double)unew[0][k]) + cs;
                m3[c] = fmax(m3[c], v);
            }
        }
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            for (int o = 16; o > 0; o >>= 1) m3[c] = fmax(m3[c], __shfl_xor_sync(0xffffffffu, m3[c], o));
            if ((threadIdx.x & 31) == 0) atomic_max_nonneg(&a.tm->maxbits[c], m3[c]);
        }
    }
}

}  // namespace img
