// Fused relaxing-TVD fluid sweep along one dimension (fluid/relaxingFluid.m:16-73,
// fluid/wFluidFlux.m:14-44, pressure/pressure.m:23-64, flux/*Limiter.m).
//
// One launch updates rho, p and E of every cell: per pencil it computes the freezing speed (the
// pencil max of |v| + c_s, a column reduction), the predictor half step, the second freezing speed
// on the half-step state, and the TVD-limited corrector; the boundary ghosts of the four flux
// arrays of each variable are synthesised in the same pass.  The state is read once and written
// once; the only other HBM traffic is the stored edges of stateful boundaries (trans, wall).
//
// Two kernel bodies.  The general one (halo jobs, FP64 copy ghosts, first sweeps): shared memory holds
// two sets of ten halo'd flux arrays (R and L of the five variables) -- set A the predictor fluxes
// and then the corrector fluxes, set B the half-step state and then the limited corrector fluxes --
// plus the fade anchors of the ten arrays of the current stage.  The mixed copy-ghost one
// (fluid_sweep_body_mixed_cg): two cell-major sets of the state and its flux numerators, three
// barriers per sweep (see there).
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
    int cfl;               // accumulate the CFL maxima of the new state (fused TimeManager pass);
                           // with CFL_CHECK_NONFINITE also flag a non-finite state
    // artificial viscosity (fluid/ArtificialViscosity.m; segment kernels only): VISC_* type, the
    // linear and quadratic strengths c1, c2, and c2 (G+1), c2^2 ((G+1)/4)^2, c1^2 formed on the host
    int visc;
    double vc1, vc2, vk1, vk2, vc1sq;
    double minmass_out;    // the final max(rho, MINMASS) (relaxingFluid.m:71); -inf when a point-fade pass
                           // follows the sweep (it fades, clamps and fades again, as the two sets do)
};
constexpr int VISC_NONE = 0;
constexpr int VISC_NR = 1;    // Neumann-Richtmyer (ArtificialViscosity.m:73-77)
constexpr int VISC_CSW = 2;   // Caramana-Shashkov-Whalen (ArtificialViscosity.m:81-148)
constexpr int CFL_ACCUMULATE = 1;
constexpr int CFL_CHECK_NONFINITE = 2;

constexpr int FLUID_NARR = 20;
constexpr int MAX_WARPS = 16;
constexpr int MIXED_CELL_WORDS = 11;   // mixed copy-ghost kernel: words per cell of a shared set

// Dynamic shared memory of the fluid kernel: 20 halo'd arrays + fade anchors of 10 arrays x 2 sides
// (FP32: room for the mixed copy-ghost kernel's two cell-major sets of 11 words per cell).
template <typename T>
__host__ __device__ inline size_t fluid_smem_bytes(int RC, int Wb) {
    const int words = sizeof(T) == 4 ? 2 * MIXED_CELL_WORDS : FLUID_NARR;
    return sizeof(T) * (size_t)words * tile_rows(RC) * Wb + sizeof(Ghost<T>) * 10 * 2 * (size_t)Wb;
}

template <typename T>
__device__ __forceinline__ T ldq(const void* p, long long i) { return reinterpret_cast<const T*>(p)[i]; }
template <typename T>
__device__ __forceinline__ void stq(void* p, long long i, T v) { reinterpret_cast<T*>(p)[i] = v; }

// BC class of fluid variable v (rho -> mass, p_i -> mom, E -> ener).
__device__ __forceinline__ int fluid_class(int v) { return v == 0 ? CLS_MASS : (v == 4 ? CLS_ENER : CLS_MOM); }

// Mixed form: the numerators F of the w arrays of wFluidFlux.m:31-44 (w = F / c_f) for one cell,
// with one reciprocal of rho.
__device__ __forceinline__ void flux_num(int d, const float u[5], const float bb[3], float press, float F[5]) {
    const float pX = sel3(d, u[1], u[2], u[3]);
    const float bX = sel3(d, bb[0], bb[1], bb[2]);
    const float ir = rcp_approx(u[0]);
    const float velocity = pX * ir;
    F[0] = pX;
    F[4] = velocity * (u[4] + press) - bX * (bb[0] * u[1] + bb[1] * u[2] + bb[2] * u[3]) * ir;
#pragma unroll
    for (int c = 0; c < 3; ++c) F[1 + c] = velocity * u[1 + c] + press * (c == d ? 1.f : 0.f) - bX * bb[c];
}

// w arrays of wFluidFlux.m:31-44 for one cell (X = sweep dim d).
template <typename T>
__device__ __forceinline__ void wflux(int d, const T u[5], const T bb[3], T press, T cf, T w[5]) {
    const T pX = sel3(d, u[1], u[2], u[3]);
    T bX = sel3(d, bb[0], bb[1], bb[2]);
    if constexpr (sizeof(T) == 4) {   // mixed form: w = F * (1 / c_f)
        const T ic = __frcp_rn(cf);
        flux_num(d, u, bb, press, w);
#pragma unroll
        for (int v = 0; v < 5; ++v) w[v] = w[v] * ic;
    } else {   // plain FP64: wFluidFlux.m's terms, its divisions by rho and c_f as products with one
               // reciprocal of each (a rounding-level difference)
        const T ir = T(1) / u[0], ic = T(1) / cf;
        T velocity = pX * ir;
        w[0] = pX * ic;
        T we = velocity * (u[4] + press) - bX * (bb[0] * u[1] + bb[1] * u[2] + bb[2] * u[3]) * ir;
        w[4] = we * ic;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            T dirv = c == d ? T(1) : T(0);
            w[1 + c] = (velocity * u[1 + c] + press * dirv - bX * bb[c]) * ic;
        }
    }
}

// 'totsnd' pressure and the freezing-speed candidate |p_X / rho| + c_s of one cell.
template <typename T>
__device__ __forceinline__ T press_speed(double G, int d, const T u[5], double msq, T& p) {
    const T pX = sel3(d, u[1], u[2], u[3]);
    if constexpr (sizeof(T) == 4) {
        PressOutF o = pressure_totsnd_mixed(G, u[0], u[1], u[2], u[3], u[4], msq);
        p = o.p;
        return fabsf(pX * rcp_approx(u[0])) + o.cs;
    } else {
        PressOut o = pressure_totsnd(G, u[0], u[1], u[2], u[3], u[4], msq);
        p = o.p + 0.0;   // + viscosity.solve ('empty' -> 0)
        return fabs(pX * (1.0 / u[0])) + o.cs;
    }
}

// Maximum over the full warp of non-negative, non-NaN values (speeds): the bit patterns of such
// values order like unsigned integers, so one hardware reduction (two for FP64: high words, then
// the low words of the lanes holding the largest high word) replaces a shuffle tree, exactly.
template <typename T>
__device__ __forceinline__ T warp_max_nonneg(T v) {
    const unsigned full = 0xffffffffu;
    if constexpr (sizeof(T) == 4) {
        return __uint_as_float(__reduce_max_sync(full, __float_as_uint(v + 0.0f)));   // + 0: no -0
    } else {
        const unsigned long long bits = (unsigned long long)__double_as_longlong(v + 0.0);
        const unsigned hi = (unsigned)(bits >> 32), lo = (unsigned)bits;
        const unsigned mh = __reduce_max_sync(full, hi);
        const unsigned ml = __reduce_max_sync(full, hi == mh ? lo : 0u);
        return __longlong_as_double((long long)(((unsigned long long)mh << 32) | ml));
    }
}

// Column max over the pencil (and the cluster); also a stage barrier that orders this CTA's shared
// reads before its next writes and, with a cluster, every rank's remote reads before them.  Lanes of
// a column reduce with warp shuffles; one lane per (warp, column) writes part[warp][b]; after a CTA
// barrier the lanes of each column share the reads of those local slots and reduce again.  With a
// cluster one thread per column then publishes the CTA's maximum in cpart[b], and after the cluster
// barrier each rank's value is read once (DSMEM) and reduced.  No atomics: every slot has one writer.
template <typename T, int CPT>
__device__ __forceinline__ T column_max(const Tile<T, CPT>& tl, int NT, T (*part)[33], T* cpart, T local) {
    const unsigned mask = 0xffffffffu;
    if (tl.d == 0 && tl.G <= 32 && tl.CL == 1) {   // each pencil lies inside one warp
        if (tl.G == 32) local = warp_max_nonneg(local);
        else
            for (int o = tl.G / 2; o > 0; o >>= 1) local = fmax(local, __shfl_xor_sync(mask, local, o));
        __syncthreads();
        return local;
    }
    if (tl.d != 0 && tl.Wb >= 32) {   // short pencils, one CTA: G rows of Wb columns, one value each
        T* flat = &part[0][0];          // G * Wb = blockDim.x <= 512 slots
        flat[tl.g * tl.Wb + tl.b] = local;
        __syncthreads();
        T m = T(0);
        for (int r = 0; r < tl.G; ++r) m = fmax(m, flat[r * tl.Wb + tl.b]);
        return m;
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int grp, lig, w0, nwc;   // lanes of the column in a warp, this lane's index among them, its warps
    if (tl.d == 0) {   // G is a multiple of 32: whole warps per column
        local = warp_max_nonneg(local);
        grp = 32;
        lig = lane;
        w0 = (tl.b * tl.G) >> 5;
        nwc = tl.G >> 5;
    } else {           // lanes b, b + Wb, ... belong to column b
        for (int o = 16; o >= tl.Wb; o >>= 1) local = fmax(local, __shfl_xor_sync(mask, local, o));
        grp = 32 / tl.Wb;
        lig = lane / tl.Wb;
        w0 = 0;
        nwc = NT >> 5;
    }
    if (lig == 0) part[warp][tl.b] = local;
    __syncthreads();
    T m = T(0);
    for (int j = lig; j < nwc; j += grp) m = fmax(m, part[w0 + j][tl.b]);
    const int olo = tl.d == 0 ? 1 : tl.Wb;
    if (tl.d == 0) m = warp_max_nonneg(m);
    else
        for (int o = 16; o >= olo; o >>= 1) m = fmax(m, __shfl_xor_sync(mask, m, o));
    if (tl.CL == 1) return m;
    if (tl.g == 0) cpart[tl.b] = m;
    cluster_sync();
    T c = T(0);
    if (lig < tl.CL) c = tl.remote(cpart, lig)[tl.b];
    if (tl.d == 0) c = warp_max_nonneg(c);
    else
        for (int o = 16; o >= olo; o >>= 1) c = fmax(c, __shfl_xor_sync(mask, c, o));
    return c;
}

// The two halves of column_max for single-CTA pencils, placed around a barrier the caller has anyway:
// colmax_publish reduces within the warp and leaves the warp's value in `part` where a column spans
// several warps; colmax_collect, after the barrier, reduces the column's warp values.
template <typename T, int CPT>
__device__ __forceinline__ T colmax_publish(const Tile<T, CPT>& tl, T (*part)[33], T local) {
    const unsigned mask = 0xffffffffu;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (tl.d == 0) {
        if (tl.G >= 32) {   // whole warps per column
            local = warp_max_nonneg(local);
            if (lane == 0) part[warp][tl.b] = local;
        } else {
            for (int o = tl.G / 2; o > 0; o >>= 1) local = fmax(local, __shfl_xor_sync(mask, local, o));
        }
        return local;
    }
    if (tl.Wb >= 32) {   // short pencils: one value per (row, column)
        (&part[0][0])[tl.g * tl.Wb + tl.b] = local;
        return local;
    }
    for (int o = 16; o >= tl.Wb; o >>= 1) local = fmax(local, __shfl_xor_sync(mask, local, o));
    if (lane < tl.Wb) part[warp][tl.b] = local;
    return local;
}

template <typename T, int CPT>
__device__ __forceinline__ T colmax_collect(const Tile<T, CPT>& tl, int NT, const T (*part)[33], T wv) {
    const unsigned mask = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    if (tl.d == 0) {
        if (tl.G <= 32) return wv;
        const int w0 = (tl.b * tl.G) >> 5, nwc = tl.G >> 5;
        return warp_max_nonneg(lane < nwc ? part[w0 + lane][tl.b] : T(0));
    }
    if (tl.Wb >= 32) {
        const T* flat = &part[0][0];
        T m = T(0);
        for (int r = 0; r < tl.G; ++r) m = fmax(m, flat[r * tl.Wb + tl.b]);
        return m;
    }
    const int grp = 32 / tl.Wb, lig = lane / tl.Wb, nwc = NT >> 5;
    T m = T(0);
    for (int j = lig; j < nwc; j += grp) m = fmax(m, part[j][tl.b]);
    for (int o = 16; o >= tl.Wb; o >>= 1) m = fmax(m, __shfl_xor_sync(mask, m, o));
    return m;
}

// First assignment of an InitializedArray takes its stored edges on every face it lies on
// (classes/InitializedArray.m:43-47 -> Edges.m:37-110).
__device__ __forceinline__ void init_edges_cell(const Geom& g, const EdgeTable* et, int obj, int x, int y, int z,
                                                double v) {
#pragma unroll
    for (int e = 0; e < 3; ++e) {
        if (e >= g.ndims) continue;
        const int ce = sel3(e, x, y, z);
        const int ne = sel3(e, g.n[0], g.n[1], g.n[2]);
        if (ce != 0 && ce != ne - 1) continue;
        double* lo = et->p[obj][e][0];
        double* hi = et->p[obj][e][1];
        const long long fi = face_index(g, e, x, y, z);
        if (lo && ce == 0) lo[fi] = v;
        if (hi && ce == ne - 1) hi[fi] = v;
    }
}

__device__ __forceinline__ bool on_face(const Geom& g, int x, int y, int z) {
    return x == 0 || x == g.n[0] - 1 || y == 0 || y == g.n[1] - 1 || (g.ndims > 2 && (z == 0 || z == g.n[2] - 1));
}

// Halo jobs of one stage for the ten arrays R_v (= base + v*AS) and L_v (= base + (5+v)*AS):
// `lo_mask`/`hi_mask` (bit 0: R, bit 1: L) say which sides the reference shifts in the coming stage
// (a pencil-end ghost is computed only for those); `kindR/kindL` name the fluid objects whose stored
// edges are used.  The 20 (array, side) jobs of a column are shared by its threads.
template <typename T, int CPT>
__device__ __forceinline__ void fluid_halo_jobs(const Tile<T, CPT>& tl, const FluidArgs& a, T* base, size_t AS,
                                                Ghost<T>* an, int lo_mask, int hi_mask, int kindR, int kindL) {
    if (!tl.colok) return;
    for (int j = tl.g; j < 20; j += tl.G) {   // job j: array j % 10 (R0..R4, L0..L4), side j / 10
        const int arr = j % 10, side = j / 10;
        const int isL = arr >= 5, v = arr - 5 * isL;
        const bool shift = ((side ? hi_mask : lo_mask) >> isL) & 1;
        const int cls = fluid_class(v);
        double* edge = a.edges->p[fluid_obj(v, isL ? kindL : kindR)][tl.d][side];
        halo_job(tl, base + arr * AS, an + (arr * 2 + side) * tl.Wb, side, shift, a.mode[cls][side], a.act[cls],
                 (v == 1 + tl.d ? GF_NEG : 0) | (isL ? GF_FLUXL : GF_FLUXR), edge, a.bc_inf, 1);
    }
}

// Mixed form with copy ghosts (single-CTA pencils, circ/const/fade shifts): the predictor and corrector
// stages store the flux numerators F beside the state they come from, so a stage is written before
// the pencil's freezing speed c_f is known and the two pencil maxima share the stage barriers.
// Readers form R = (u + F/c_f)/2 and L = (u - F/c_f)/2 (relaxingFluid.m:30-31, 52-56) at the rows
// they need, with the reciprocal of c_f the flux stage itself would use.  Three barriers per sweep.
// FADE: some side of this sweep is fade (copy of the near end row plus the damping of cg_fade).
template <bool MHD, int CPT, bool FADE>
__device__ __forceinline__ void fluid_sweep_body_mixed_cg(const FluidArgs& a, unsigned vblock) {
    using T = float;
    extern __shared__ __align__(16) unsigned char smem[];
    pdl_wait();
    if (a.tm->done || a.tm->error) return;
    __shared__ T part[2][MAX_WARPS][33];
    __shared__ double cflp[3][MAX_WARPS];
    Tile<T, CPT> tl;
    tl.init(a.sg, vblock);
    const int d = a.sg.d;
    const int NT = a.sg.NT;
    const int N = tl.N;
    // cell-major shared layout: cell i holds u[0..4] at S + i*CS and F[0..4] at S + i*CS + 5 (later the
    // limited R and L); a stride of 11 words keeps consecutive cells on distinct banks, and every
    // access is an immediate offset from one address per cell
    constexpr int CS = MIXED_CELL_WORDS;
    const size_t AS = (size_t)tile_rows(tl.RC) * tl.Wb;
    T* SA = reinterpret_cast<T*>(smem);   // the state and its F; later the limited R, L
    T* SB = SA + CS * AS;                 // half-step state and its F
    const int dn_src = tl.ridx(a.mode[CLS_MASS][0] == BC_CIRC ? N - 1 : 0);
    const int up_src = tl.ridx(a.mode[CLS_MASS][1] == BC_CIRC ? 0 : N - 1);
    // shared index of own row k shifted by n = -1 / +1 (copy ghosts at the pencil ends)
    auto nix = [&](int k, int n) -> int {
        const int r = tl.grow(k);
        return n < 0 ? (r == 0 ? dn_src : tl.idx(k) - tl.rs) : (r == N - 1 ? up_src : tl.idx(k) + tl.rs);
    };
    // fade damping of value v, the shift by n of an array whose row j is val(j), at own row k
    const bool fade_lo = FADE && a.mode[CLS_MASS][0] == BC_FADE, fade_hi = FADE && a.mode[CLS_MASS][1] == BC_FADE;
    const int fw = a.fade_f;
    auto fade = [&](T v, int k, int n, auto&& val) -> T {
        if constexpr (FADE) {
            const int r = tl.grow(k);
            if (!(n < 0 ? fade_lo : fade_hi) || r >= N || (r >= fw && r < N - fw)) return v;
            const T s0 = n < 0 ? val(0) : val(N > 1 ? 1 : 0);
            const T sN1 = n < 0 ? val(N >= 2 ? N - 2 : 0) : val(N - 1);
            return fade_apply(v, r, N, a.fade, fw, s0, sN1);
        } else {
            return v;
        }
    };
    const double G = a.gamma;
    const double dt = a.tm->dt;
    const T ff = (T)(dt / a.dx);
    const T half_ffx = (T)(0.5 * (dt / a.dx));

    // ---- load u and cell-centred B; pressure, speed and F of the state -> set A ------------------
    T u[5][CPT], bb[3][CPT];
    double msq[CPT];
    T lmax = T(0);
#pragma unroll
    for (int k = 0; k < CPT; ++k) {
        const bool ok = tl.ok(k);
        const long long o = tl.off(k);
#pragma unroll
        for (int v = 0; v < 5; ++v) u[v][k] = ok ? ldq<T>(a.q[v], o) : (v == 0 ? T(1) : T(0));
        double m = 0.0;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            bb[c][k] = (MHD && ok) ? ldq<T>(a.q[Q_CBX + c], o) : T(0);
            if (MHD && a.use_b[c]) m = m + (double)bb[c][k] * (double)bb[c][k];
        }
        msq[k] = m;
        T uu[5] = {u[0][k], u[1][k], u[2][k], u[3][k], u[4][k]};
        T b3[3] = {bb[0][k], bb[1][k], bb[2][k]};
        T p;
        const T spd = press_speed<T>(G, d, uu, m, p);
        if (ok) lmax = fmax(lmax, spd);
        T F[5];
        flux_num(d, uu, b3, p, F);
        T* c0 = SA + tl.idx(k) * CS;
#pragma unroll
        for (int v = 0; v < 5; ++v) {
            c0[v] = uu[v];
            c0[5 + v] = F[v];
        }
    }
    const T wv1 = colmax_publish(tl, part[0], lmax);
    __syncthreads();
    const T cf = colmax_collect(tl, NT, part[0], wv1);   // freezing speed (wFluidFlux.m:18-22)
    const T ic = __frcp_rn(cf);

    // ---- predictor (relaxingFluid.m:30-39); pressure, speed and F of the half-step state -> set B --
    T lmax2 = T(0);
#pragma unroll
    for (int k = 0; k < CPT; ++k) {
        const int ix = tl.idx(k);
        const T* cm = SA + nix(k, -1) * CS;
        const T* c0 = SA + ix * CS;
        const T* cp = SA + nix(k, +1) * CS;
        T us[5];
#pragma unroll
        for (int v = 0; v < 5; ++v) {
            const T w = c0[5 + v] * ic;
            T Rm = T(0.5) * (cm[v] + cm[5 + v] * ic);
            T Lp = T(0.5) * (cp[v] - cp[5 + v] * ic);
            if constexpr (FADE) {
                Rm = fade(Rm, k, -1, [&](int j) { const T* c = SA + tl.ridx(j) * CS; return T(0.5) * (c[v] + c[5 + v] * ic); });
                Lp = fade(Lp, k, +1, [&](int j) { const T* c = SA + tl.ridx(j) * CS; return T(0.5) * (c[v] - c[5 + v] * ic); });
            }
            us[v] = u[v][k] - half_ffx * cf * (T(0.5) * (u[v][k] + w) - Rm + T(0.5) * (u[v][k] - w) - Lp);
        }
        us[0] = us[0] > (T)a.minmass ? us[0] : (T)a.minmass;   // max(rho, MINMASS), NaN -> MINMASS
        if (!tl.ok(k)) { us[0] = T(1); us[1] = us[2] = us[3] = us[4] = T(0); }
        T b3[3] = {bb[0][k], bb[1][k], bb[2][k]};
        T p2;
        const T spd = press_speed<T>(G, d, us, msq[k], p2);   // relaxingFluid.m:47-50
        if (tl.ok(k)) lmax2 = fmax(lmax2, spd);
        T F[5];
        flux_num(d, us, b3, p2, F);
        T* b0 = SB + ix * CS;
#pragma unroll
        for (int v = 0; v < 5; ++v) {
            b0[v] = us[v];
            b0[5 + v] = F[v];
        }
    }
    const T wv2 = colmax_publish(tl, part[1], lmax2);
    __syncthreads();   // also orders the predictor's reads of set A before the limiter's writes
    const T cfs = colmax_collect(tl, NT, part[1], wv2);   // freezing speed of the half step
    const T ics = __frcp_rn(cfs);

    // ---- corrector fluxes and TVD limiter (relaxingFluid.m:52-62): limited R and L -> set A -------
#pragma unroll
    for (int k = 0; k < CPT; ++k) {
        const int ix = tl.idx(k);
        const T* bm = SB + nix(k, -1) * CS;
        const T* b0 = SB + ix * CS;
        const T* bp = SB + nix(k, +1) * CS;
        T* a0 = SA + ix * CS;
#pragma unroll
        for (int v = 0; v < 5; ++v) {
            const T wm = bm[5 + v] * ics, w0 = b0[5 + v] * ics, wp = bp[5 + v] * ics;
            const T um = bm[v], u0 = b0[v], up = bp[v];
            T Rm = T(0.5) * (um + wm), Rp = T(0.5) * (up + wp), Lm = T(0.5) * (um - wm), Lp = T(0.5) * (up - wp);
            const T r = T(0.5) * (u0 + w0), l = T(0.5) * (u0 - w0);
            if constexpr (FADE) {
                auto Rs = [&](int j) { const T* c = SB + tl.ridx(j) * CS; return T(0.5) * (c[v] + c[5 + v] * ics); };
                auto Ls = [&](int j) { const T* c = SB + tl.ridx(j) * CS; return T(0.5) * (c[v] - c[5 + v] * ics); };
                Rm = fade(Rm, k, -1, Rs);
                Rp = fade(Rp, k, +1, Rs);
                Lm = fade(Lm, k, -1, Ls);
                Lp = fade(Lp, k, +1, Ls);
            }
            a0[v] = r + limiter_corr<T>(a.limiter, r - Rm, Rp - r);
            a0[5 + v] = l + limiter_corr<T>(a.limiter, Lm - l, l - Lp);
        }
    }
    __syncthreads();

    pdl_trigger();
    // ---- corrector update (relaxingFluid.m:64-71), stored cell by cell ----------------------------
    double m3[3] = {0.0, 0.0, 0.0};
    bool bad = false;
#pragma unroll
    for (int k = 0; k < CPT; ++k) {
        const T* am = SA + nix(k, -1) * CS;
        const T* a0 = SA + tl.idx(k) * CS;
        const T* ap = SA + nix(k, +1) * CS;
        T unew[5];
#pragma unroll
        for (int v = 0; v < 5; ++v) {
            T Rm = am[v], Lp = ap[5 + v];
            if constexpr (FADE) {
                Rm = fade(Rm, k, -1, [&](int j) { return SA[tl.ridx(j) * CS + v]; });
                Lp = fade(Lp, k, +1, [&](int j) { return SA[tl.ridx(j) * CS + 5 + v]; });
            }
            unew[v] = u[v][k] - ff * cfs * (a0[v] - Rm + a0[5 + v] - Lp);
        }
        unew[0] = unew[0] > (T)a.minmass_out ? unew[0] : (T)a.minmass_out;
        if (!tl.ok(k)) continue;
        const long long o = tl.off(k);
#pragma unroll
        for (int v = 0; v < 5; ++v) stq<T>(a.q[v], o, unew[v]);
        if (a.cfl) {   // fused CFL maxima of the new state (TimeManager.m:65-77)
            double sp[3];
            cfl_speeds(G, (double)unew[0], (double)unew[1], (double)unew[2], (double)unew[3], (double)unew[4], msq[k],
                       sp);
            bad = bad || !isfinite(sp[0] + sp[1] + sp[2]);
#pragma unroll
            for (int c = 0; c < 3; ++c) m3[c] = fmax(m3[c], sp[c]);
        }
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
        if (threadIdx.x < 3) {   // one global atomic per CTA and direction
            double m = 0.0;
            for (int w = 0; w < (int)(blockDim.x >> 5); ++w) m = fmax(m, cflp[threadIdx.x][w]);
            atomic_max_nonneg(&a.tm->maxbits[threadIdx.x], m);
        }
    }
}

// One fluid sweep of one grid, run by CTA `vblock` of that grid's launch.
// FADE: some BC of this sweep direction is fade (compiles the damping in).
// CG (copy ghosts): single-CTA pencils whose three fluid classes share one circ, const or fade mode
// per side.  Those ghosts copy an own row (circ: the far end, const and fade: the near end, fade then
// damped by cg_fade), so the reader of row 0 or N-1 indexes that row directly: no halo jobs and no
// barrier after them.
// INIT: this launch may capture stored edges of first-assigned objects (compiled out otherwise).
template <typename T, bool MHD, int CPT, bool FADE, bool CG, bool INIT>
__device__ __forceinline__ void fluid_sweep_body_general(const FluidArgs& a, unsigned vblock) {
    extern __shared__ __align__(16) unsigned char smem[];
    pdl_wait();
    // A stopped or failed run does nothing.  Within a cluster every CTA must take the same branch before
    // its cluster barriers, and the error word can be raised by another cluster of this very launch (the
    // non-finite check of the fused CFL pass) while this one starts: cluster launches return on `done`
    // only (set between launches), and a failed run's clusters compute on without consequence.
    if (a.tm->done || (a.sg.CL == 1 && a.tm->error)) return;
    __shared__ T part[2][MAX_WARPS][33];   // per-warp column maxima (two freezing speeds; rows padded
                                           // so the lanes reading one column's warps hit distinct banks)
    __shared__ T cpart[2][32];             // per-CTA column maxima, read by the other cluster ranks
    __shared__ double cflp[3][MAX_WARPS];  // per-warp CFL maxima
    Tile<T, CPT> tl;
    tl.init(a.sg, vblock);
    const int d = a.sg.d;
    const int NT = a.sg.NT;
    const int Wb = tl.Wb;
    const size_t AS = (size_t)tile_rows(tl.RC) * Wb;
    T* SA = reinterpret_cast<T*>(smem);   // set A: R[v] at SA + v*AS, L[v] at SA + (5+v)*AS
    T* SB = SA + 10 * AS;                 // set B
    Ghost<T>* AN = reinterpret_cast<Ghost<T>*>(SA + 20 * AS);   // fade anchors [array][side][column]

    // copy ghosts: shared index of the row that row -1 (dn_src) and row N (up_src) copy
    const int N = tl.N;
    const int dn_src = tl.ridx(a.mode[CLS_MASS][0] == BC_CIRC ? N - 1 : 0);
    const int up_src = tl.ridx(a.mode[CLS_MASS][1] == BC_CIRC ? 0 : N - 1);
    // A.shift(d, n) at own row k, n = -1 or +1 (the anchors `an` are read under fade only)
    auto sh = [&](const T* A, const Ghost<T>* an, int k, int n, int mode) -> T {
        if constexpr (CG) {
            const int r = tl.grow(k);
            const int ix = n < 0 ? (r == 0 ? dn_src : tl.idx(k) - tl.rs) : (r == N - 1 ? up_src : tl.idx(k) + tl.rs);
            if constexpr (FADE) {
                if (mode == BC_FADE) return cg_fade(tl, A, r, n, A[ix], a.fade, a.fade_f);
            }
            return A[ix];
        } else {
            return shifted<FADE>(tl, A, an, k, n, mode, a.fade, a.fade_f);
        }
    };
    const double G = a.gamma;
    const double dt = a.tm->dt;
    const T ff = (T)(dt / a.dx);
    const T half_ffx = (T)(0.5 * (dt / a.dx));

    // ---- load u (rho, px, py, pz, E) and cell-centred B; freezing speed #1 (wFluidFlux.m:18-22) --
    T u[5][CPT], bb[3][CPT], press[CPT];
    double msq[CPT];
    T lmax = T(0);
#pragma unroll
    for (int k = 0; k < CPT; ++k) {
        const bool ok = tl.ok(k);
        const long long o = tl.off(k);
#pragma unroll
        for (int v = 0; v < 5; ++v) u[v][k] = ok ? ldq<T>(a.q[v], o) : (v == 0 ? T(1) : T(0));
        double m = 0.0;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            bb[c][k] = (MHD && ok) ? ldq<T>(a.q[Q_CBX + c], o) : T(0);
            if (MHD && a.use_b[c]) m = m + (double)bb[c][k] * (double)bb[c][k];
        }
        msq[k] = m;
        T uu[5] = {u[0][k], u[1][k], u[2][k], u[3][k], u[4][k]};
        T spd = press_speed<T>(G, d, uu, m, press[k]);
        if (ok) lmax = fmax(lmax, spd);
    }
    const T cf = column_max(tl, NT, part[0], cpart[0], lmax);

    // ---- predictor fluxes R = (u+w)/2, L = (u-w)/2 -> set A (relaxingFluid.m:30-31) ---------------
#pragma unroll
    for (int k = 0; k < CPT; ++k) {
        T uu[5] = {u[0][k], u[1][k], u[2][k], u[3][k], u[4][k]};
        T b3[3] = {bb[0][k], bb[1][k], bb[2][k]};
        T w[5];
        wflux<T>(d, uu, b3, press[k], cf, w);
        const int ix = tl.idx(k);
#pragma unroll
        for (int v = 0; v < 5; ++v) {
            SA[v * AS + ix] = T(0.5) * (uu[v] + w[v]);
            SA[(5 + v) * AS + ix] = T(0.5) * (uu[v] - w[v]);
        }
        if (INIT && a.init_store && tl.ok(k)) {   // first assignment of store.fluxR/L (InitializedArray.m:43-47)
            int x, y, z;
            tl.coords(k, x, y, z);
            if (on_face(a.sg.g, x, y, z)) {
#pragma unroll 1
                for (int arr = 0; arr < 10; ++arr)
                    init_edges_cell(a.sg.g, a.edges, fluid_obj(arr % 5, arr < 5 ? FO_STORE_R : FO_STORE_L), x, y,
                                    z, (double)SA[arr * AS + ix]);
            }
        }
    }
    tl.csync();
    if constexpr (!CG) {
        fluid_halo_jobs(tl, a, SA, AS, AN, /*lower: R*/ 1, /*upper: L*/ 2, FO_STORE_R, FO_STORE_L);
        __syncthreads();
    }

    // ---- predictor (relaxingFluid.m:32-39): half-step state -> set B; freezing speed #2 -----------
    T lmax2 = T(0);
    T press2[CPT];
#pragma unroll
    for (int k = 0; k < CPT; ++k) {
        const int ix = tl.idx(k);
        T us[5];
#pragma unroll
        for (int v = 0; v < 5; ++v) {
            const int cls = fluid_class(v);
            const T* R = SA + v * AS;
            const T* L = SA + (5 + v) * AS;
            const T Rm = sh(R, AN + (2 * v) * Wb, k, -1, a.mode[cls][0]);
            const T Lp = sh(L, AN + (2 * (5 + v) + 1) * Wb, k, +1, a.mode[cls][1]);
            us[v] = u[v][k] - half_ffx * cf * (R[ix] - Rm + L[ix] - Lp);
        }
        us[0] = us[0] > (T)a.minmass ? us[0] : (T)a.minmass;   // max(rho, MINMASS), NaN -> MINMASS
        if (!tl.ok(k)) { us[0] = T(1); us[1] = us[2] = us[3] = us[4] = T(0); }
#pragma unroll
        for (int v = 0; v < 5; ++v) SB[v * AS + ix] = us[v];
        T spd = press_speed<T>(G, d, us, msq[k], press2[k]);   // relaxingFluid.m:47-50
        if (tl.ok(k)) lmax2 = fmax(lmax2, spd);
    }
    const T cfs = column_max(tl, NT, part[1], cpart[1], lmax2);   // its barrier also ends the predictor reads of set A

    // ---- corrector fluxes (relaxingFluid.m:52-56) from the half-step state -> set A --------------
#pragma unroll
    for (int k = 0; k < CPT; ++k) {
        const int ix = tl.idx(k);
        T uu[5];
#pragma unroll
        for (int v = 0; v < 5; ++v) uu[v] = SB[v * AS + ix];
        T b3[3] = {bb[0][k], bb[1][k], bb[2][k]};
        T w[5];
        wflux<T>(d, uu, b3, press2[k], cfs, w);
#pragma unroll
        for (int v = 0; v < 5; ++v) {
            SA[v * AS + ix] = T(0.5) * (uu[v] + w[v]);
            SA[(5 + v) * AS + ix] = T(0.5) * (uu[v] - w[v]);
        }
        if (INIT && a.init_flux && tl.ok(k)) {   // first assignment of fluxR/L
            int x, y, z;
            tl.coords(k, x, y, z);
            if (on_face(a.sg.g, x, y, z)) {
#pragma unroll 1
                for (int arr = 0; arr < 10; ++arr)
                    init_edges_cell(a.sg.g, a.edges, fluid_obj(arr % 5, arr < 5 ? FO_R : FO_L), x, y, z,
                                    (double)SA[arr * AS + ix]);
            }
        }
    }
    tl.csync();
    if constexpr (!CG) {
        fluid_halo_jobs(tl, a, SA, AS, AN, 3, 3, FO_R, FO_L);
        __syncthreads();
    }

    // ---- TVD limiter (relaxingFluid.m:57-62): corrected R and L -> set B --------------------------
#pragma unroll
    for (int k = 0; k < CPT; ++k) {
        const int ix = tl.idx(k);
#pragma unroll
        for (int v = 0; v < 5; ++v) {
            const int cls = fluid_class(v);
            const T* R = SA + v * AS;
            const T* L = SA + (5 + v) * AS;
            const Ghost<T>* aR = AN + (2 * v) * Wb;
            const Ghost<T>* aL = AN + (2 * (5 + v)) * Wb;
            const int mlo = a.mode[cls][0], mhi = a.mode[cls][1];
            const T r = R[ix], l = L[ix];
            const T Rm = sh(R, aR, k, -1, mlo);
            const T Rp = sh(R, aR + Wb, k, +1, mhi);
            const T Lm = sh(L, aL, k, -1, mlo);
            const T Lp = sh(L, aL + Wb, k, +1, mhi);
            SB[v * AS + ix] = r + limiter_corr<T>(a.limiter, r - Rm, Rp - r);
            SB[(5 + v) * AS + ix] = l + limiter_corr<T>(a.limiter, Lm - l, l - Lp);
        }
    }
    tl.csync();
    if constexpr (!CG) {
        fluid_halo_jobs(tl, a, SB, AS, AN, 1, 2, FO_R, FO_L);
        __syncthreads();
    }

    pdl_trigger();
    // ---- corrector update (relaxingFluid.m:64-71), stored cell by cell ----------------------------
    double m3[3] = {0.0, 0.0, 0.0};
    bool bad = false;
#pragma unroll
    for (int k = 0; k < CPT; ++k) {
        const int ix = tl.idx(k);
        T unew[5];
#pragma unroll
        for (int v = 0; v < 5; ++v) {
            const int cls = fluid_class(v);
            const T* R = SB + v * AS;
            const T* L = SB + (5 + v) * AS;
            const T Rm = sh(R, AN + (2 * v) * Wb, k, -1, a.mode[cls][0]);
            const T Lp = sh(L, AN + (2 * (5 + v) + 1) * Wb, k, +1, a.mode[cls][1]);
            unew[v] = u[v][k] - ff * cfs * (R[ix] - Rm + L[ix] - Lp);
        }
        unew[0] = unew[0] > (T)a.minmass_out ? unew[0] : (T)a.minmass_out;
        if (!tl.ok(k)) continue;
        const long long o = tl.off(k);
#pragma unroll
        for (int v = 0; v < 5; ++v) stq<T>(a.q[v], o, unew[v]);
        if (a.cfl) {   // fused CFL maxima of the new state (TimeManager.m:65-77)
            double sp[3];
            cfl_speeds(G, (double)unew[0], (double)unew[1], (double)unew[2], (double)unew[3], (double)unew[4], msq[k],
                       sp);
            bad = bad || !isfinite(sp[0] + sp[1] + sp[2]);
#pragma unroll
            for (int c = 0; c < 3; ++c) m3[c] = fmax(m3[c], sp[c]);
        }
    }

    // peers of a cluster read this CTA's shared memory through DSMEM until their last stage ends
    if (tl.CL > 1) cluster_sync();

    if (a.cfl) {
        if (a.cfl & CFL_CHECK_NONFINITE) flag_nonfinite(a.tm, bad);
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            m3[c] = warp_max_nonneg(m3[c]);
            if (lane == 0) cflp[c][warp] = m3[c];
        }
        __syncthreads();
        if (threadIdx.x < 3) {   // one global atomic per CTA and direction
            double m = 0.0;
            for (int w = 0; w < (int)(blockDim.x >> 5); ++w) m = fmax(m, cflp[threadIdx.x][w]);
            atomic_max_nonneg(&a.tm->maxbits[threadIdx.x], m);
        }
    }
}

// Kernel variant V: 0 halo jobs, 1 halo jobs with fade, 2 copy ghosts, 3 and 4 as 0 and 1 with the
// capture of stored edges (a run's first sweeps), 5 copy ghosts with fade.
template <int V> constexpr bool kv_fade = V == 1 || V == 4 || V == 5;
template <int V> constexpr bool kv_cg = V == 2 || V == 5;
template <int V> constexpr bool kv_init = V == 3 || V == 4;

template <typename T, bool MHD, int CPT, int V>
__device__ __forceinline__ void fluid_sweep_body(const FluidArgs& a, unsigned vblock) {
    if constexpr (kv_cg<V> && sizeof(T) == 4) fluid_sweep_body_mixed_cg<MHD, CPT, kv_fade<V>>(a, vblock);
    else fluid_sweep_body_general<T, MHD, CPT, kv_fade<V>, kv_cg<V>, kv_init<V>>(a, vblock);
}

template <typename T, bool MHD, int CPT, int V>
__global__ void __launch_bounds__(512, CPT == 1 ? 2 : 1) fluid_sweep_kernel(const __grid_constant__ FluidArgs a) {
    fluid_sweep_body<T, MHD, CPT, V>(a, blockIdx.x);
}

// The same sweep over many grids in one launch (BlockMap per CTA, arguments per member).
template <typename T, bool MHD, int CPT, int V>
__global__ void __launch_bounds__(512, CPT == 1 ? 2 : 1) fluid_sweep_batch_kernel(const FluidArgs* __restrict__ args,
                                                                                  const BlockMap* __restrict__ map) {
    __shared__ FluidArgs sa;
    const BlockMap bm = map[blockIdx.x];
    load_member_args(sa, args + bm.member);
    __syncthreads();
    fluid_sweep_body<T, MHD, CPT, V>(sa, (unsigned)bm.block);
}

}  // namespace img
