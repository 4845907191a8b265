// Pencil tiles shared by the sweep kernels.
//
// A pencil is one line of cells along the sweep dimension d.  A CTA holds a bundle of Wb pencils
// ("columns") and RC = G*CPT rows of each (thread (b, g) owns rows g, g+G, ... of column b); a
// thread-block cluster of CL CTAs covers pencils longer than RC (rank r holds rows [r*RC, (r+1)*RC)),
// so every pencil stays on chip whatever its length.  Consecutive threads touch consecutive cells,
// so global loads/stores are coalesced along x for every sweep direction.
//
// Stencil operands live in shared-memory arrays with HALO rows: local row 0 is the row below the
// CTA's first row, local rows RC+1 and RC+2 the two rows above its last row (layout: Tile::rs/cs).
// Between stages a few threads fill the halos -- the neighbouring cluster rank's edge rows (read
// through DSMEM), or, at the pencil ends, the boundary-condition ghost of the reference's shift
// (shifting/*_shift.m), stateful edge drift included -- so every stencil read is one unconditional
// shared load.  Single-CTA pencils with circ, const or fade shifts skip the halos: their ghosts copy
// an own row, which the reader indexes directly (the copy-ghost kernel variants).
#pragma once

#include "common.cuh"

namespace img {

// Division by a launch-invariant divisor D >= 1 for dividends n < 2^31 by one 64-bit multiply and a
// shift (Granlund and Montgomery, "Division by invariant integers using multiplication", 1994,
// round-up method): with l = ceil(log2 D), s = 31 + l and M = floor(2^s / D) + 1, M*D lies in
// (2^s, 2^s + 2^l], so floor(n / D) = floor(n * M / 2^s) for every n < 2^31.
struct FastDiv {
    unsigned long long mul;
    int shift;
    __host__ __device__ unsigned div(unsigned n) const { return (unsigned)(((unsigned long long)n * mul) >> shift); }
};

inline FastDiv make_fastdiv(unsigned D) {
    int l = 0;
    while ((1ull << l) < D) ++l;
    FastDiv f;
    f.shift = 31 + l;
    f.mul = (1ull << f.shift) / D + 1;
    return f;
}

// Geometry of one directional sweep (host-filled; kernels read it from their grid-constant
// parameter, so the uniform values cost no registers).
struct SweepGeom {
    Geom g;
    int d;            // sweep dimension 0..2
    int d1, d2;       // the other two dimensions, in increasing order
    int N;            // pencil length g.n[d]
    long long ncol;   // number of pencils = ncell / N
    int Wb;           // pencils per CTA
    int G;            // threads per pencil per CTA
    int CL;           // CTAs per cluster along the pencil (1, 2 or 4)
    int NT;           // threads per CTA = Wb * G
    int RC;           // rows per CTA = G * cells per thread
    int rank_hi;      // cluster rank holding row N-1 = (N-1) / RC
    int n1;           // g.n[d1]
    long long sd, s1, s2;   // strides along d, d1, d2
    FastDiv div_lanes;      // by G (d == 0: threads of a pencil are consecutive) or Wb (d >= 1)
    FastDiv div_cl;         // by CL
    FastDiv div_n1;         // by n1
};

constexpr int HALO_LO = 1;   // halo rows below the CTA's rows
constexpr int HALO_HI = 2;   // halo rows above (two: the magnet's shift by +2)

// Rows of one shared array (own rows plus halos).
__host__ __device__ inline int tile_rows(int RC) { return RC + HALO_LO + HALO_HI; }

// Fade anchors of one (array, side): the constant-shifted values at rows 0 and N-1 (fade_shift.m
// damps toward them); `g` holds a ghost value where a stage needs more than one per side.
template <typename T>
struct Ghost {
    T g, s0, sN1;
};

template <typename T, int CPT>
struct Tile {
    // uniform (copies of parameter values)
    int N, Wb, G, CL, d, RC, rank_hi;
    // shared layout: element (local row l, column b) at l * rs + b * cs.  Along x a warp's lanes
    // walk the rows of one pencil, so rows are contiguous (rs = 1); along y/z the lanes walk the
    // columns, so columns are (cs = 1).  Either way consecutive lanes hit consecutive banks.
    int rs, cs;
    // per thread
    int b, g, rank;
    int row0;             // global row of own cell k = 0
    int ix0;              // shared index of own cell k = 0
    int col;              // global pencil index (ncell < 2^31)
    bool colok;
    long long base;       // linear offset of row 0 of this pencil
    long long sd;         // stride along the sweep
    int c1, c2;           // the pencil's coordinates along d1 and d2

    // vblock: this CTA's block index within its grid's launch (blockIdx.x for a single launch)
    __device__ __forceinline__ void init(const SweepGeom& s, unsigned vblock) {
        const int t = threadIdx.x;
        N = s.N;
        Wb = s.Wb;
        G = s.G;
        CL = s.CL;
        d = s.d;
        RC = s.RC;
        rank_hi = s.rank_hi;
        sd = s.sd;
        const unsigned tq = s.div_lanes.div((unsigned)t);   // t / G (x) or t / Wb (y, z)
        if (s.d == 0) { b = (int)tq; g = t - b * s.G; }
        else { g = (int)tq; b = t - g * s.Wb; }
        rs = s.d == 0 ? 1 : s.Wb;
        cs = s.d == 0 ? tile_rows(s.RC) : 1;
        rank = (int)(vblock & (unsigned)(s.CL - 1));   // CL is a power of two
        const unsigned bundle = s.div_cl.div(vblock);
        row0 = rank * s.RC + g;
        ix0 = (g + HALO_LO) * rs + b * cs;
        col = (int)(bundle * (unsigned)s.Wb + (unsigned)b);
        colok = col < s.ncol;
        const unsigned c = colok ? (unsigned)col : 0u;
        c2 = (int)s.div_n1.div(c);
        c1 = (int)(c - (unsigned)c2 * (unsigned)s.n1);
        base = c1 * s.s1 + (long long)c2 * s.s2;
    }
    __device__ __forceinline__ int grow(int k) const { return row0 + k * G; }
    __device__ __forceinline__ bool ok(int k) const { return colok && grow(k) < N; }
    __device__ __forceinline__ long long off(int k) const { return base + (long long)grow(k) * sd; }
    // shared index of own row k, and of local row l (0 = lower halo)
    __device__ __forceinline__ int idx(int k) const { return ix0 + k * G * rs; }
    __device__ __forceinline__ int lidx(int l) const { return l * rs + b * cs; }
    __device__ __forceinline__ void coords(int k, int& x, int& y, int& z) const {
        const int r = grow(k);
        if (d == 0) { x = r; y = c1; z = c2; }
        else if (d == 1) { x = c1; y = r; z = c2; }
        else { x = c1; y = c2; z = r; }
    }
    __device__ __forceinline__ void csync() const {
        if (CL > 1) cluster_sync();
        else __syncthreads();
    }
    template <typename U>
    __device__ __forceinline__ U* remote(U* p, int r) const {
        if (CL == 1 || r == rank) return p;
        return cg::this_cluster().map_shared_rank(p, r);
    }
    // Value of array A at global row r (0 <= r < N) of this column, on any cluster rank.
    template <typename U>
    __device__ __forceinline__ U row(const U* A, int r) const {
        int rk = r / RC;
        const U* p = remote(const_cast<U*>(A), rk);
        return p[(r - rk * RC + HALO_LO) * rs + b * cs];
    }
    // Local shared index of global row r (r may be N or N+1 on rank_hi: an idle row or a halo row).
    __device__ __forceinline__ int ridx(int r) const { return (r - rank * RC + HALO_LO) * rs + b * cs; }
};

// Fade damping of fade_shift.m:31-44 applied to the constant-shifted value sv at row r of a line of
// N cells: s0 and sN1 are the constant-shifted values at rows 0 and N-1 (the two anchors).
// Rows past the pencil's end (idle rows of the last CTA) are returned unchanged: their values are
// never read, and the coefficient index N-1-r would be negative there.
template <typename T>
__device__ __forceinline__ T fade_apply(T sv, int r, int N, const double* fc, int f, T s0, T sN1) {
    if (r >= N) return sv;
    T lf = sv;
    if (r < f) lf = (T(1) - T(fc[r])) * sv + T(fc[r]) * s0;
    if (r >= N - f) {
        T lfN1 = sN1;
        if (N - 1 < f) lfN1 = (T(1) - T(fc[N - 1])) * sN1 + T(fc[N - 1]) * s0;
        T c = T(fc[N - 1 - r]);
        lf = (T(1) - c) * lf + c * lfN1;
    }
    return lf;
}

// A.shift(d, n) at own row k for n = -1 / +1 (one shared load), fade damping included.  `an` is the
// array's anchor pair for that side, read only under fade; FADE = false (no fade BC on this sweep
// direction, known at launch) compiles the damping out.
template <bool FADE, typename T, int CPT>
__device__ __forceinline__ T shifted(const Tile<T, CPT>& tl, const T* A, const Ghost<T>* an, int k, int n, int mode,
                                     const double* fc, int f) {
    T v = A[tl.idx(k) + n * tl.rs];
    if (FADE && mode == BC_FADE) {
        const Ghost<T>& q = an[tl.b];
        v = fade_apply(v, tl.grow(k), tl.N, fc, f, q.s0, q.sN1);
    }
    return v;
}

// Copy-ghost form of the fade damping: v is A.shift(d, n) at own row r (the ghost copies the near end
// row, as a const shift); rows within f of either end are damped toward the shift's anchors, which
// are the array's own rows 0 and N-2 (n = -1) or 1 and N-1 (n = +1) (fade_shift.m:31-44).
template <typename T, int CPT>
__device__ __forceinline__ T cg_fade(const Tile<T, CPT>& tl, const T* A, int r, int n, T v, const double* fc, int f) {
    const int N = tl.N;
    if (r >= N || (r >= f && r < N - f)) return v;
    const T s0 = n < 0 ? A[tl.ridx(0)] : A[tl.ridx(N > 1 ? 1 : 0)];
    const T sN1 = n < 0 ? A[tl.ridx(N >= 2 ? N - 2 : 0)] : A[tl.ridx(N - 1)];
    return fade_apply(v, r, N, fc, f, s0, sN1);
}

// "No stored-edge value supplied" marker (stored edges are finite physical values).
constexpr double NO_EV = -1.0e300;

// Transparent ghost of one shift call (shifting/transparent_shift.m:23-99), out of line: it runs
// for a few threads per stage only, and keeping its FP64 interpolation out of the stencil code keeps
// the register allocation of the sweep kernels at the stencil's needs.
template <typename T, int CPT>
__device__ __noinline__ double trans_bc_ghost(const Tile<T, CPT> tl, const T* A, int n, int mp, int act, double* edge,
                                              double bc_inf, double ev) {
    const int N = tl.N;
    const bool upper = n > 0;
    const int m = n < 0 ? -n : n;
    double y1, y2, cur;
    if (upper) {
        y1 = (double)tl.row(A, trans_pick_upper(N, m, 1));
        y2 = (double)tl.row(A, trans_pick_upper(N, m, 2));
        cur = (double)tl.row(A, N - 1);
    } else {
        y1 = (double)tl.row(A, trans_pick_lower(N, m, 1));
        y2 = (double)tl.row(A, trans_pick_lower(N, m, 2));
        cur = (double)tl.row(A, 0);
    }
    double e = 0.0;
    if (act) {
        if (ev != NO_EV) e = ev;
        else {
            e = edge_drift(edge[tl.col], cur);
            edge[tl.col] = e;
        }
    }
    // the 1e-4 keep test compares with the unshifted array at the ghost's position
    const int gpos = upper ? N - 1 - (m - mp) : 0;
    return trans_ghost(y1, y2, e, bc_inf, 3.0 + mp, (double)tl.row(A, gpos));
}

// Ghost of array A beyond the pencil end for one shift call A.shift(d, n): n = -1 (row -1),
// n = +1 (row N) or n = +2 (rows N and N+1, mp = 1 or 2 selects which).  Stateful edges (trans,
// wall) use `ev` when given; otherwise a trans edge is drifted here and written back (the caller is
// the one thread per pencil end and shift call).  Rows are read through tl.row (any cluster rank).
template <typename T, int CPT>
__device__ __forceinline__ T bc_ghost(const Tile<T, CPT>& tl, const T* A, int n, int mp, int mode, int act, int flip,
                                      double* edge, double bc_inf, double ev) {
    const int N = tl.N;
    const bool upper = n > 0;
    switch (mode) {
        case BC_CIRC: return upper ? tl.row(A, mp - 1) : tl.row(A, N - 1);
        case BC_MIRROR: {
            T x = upper ? tl.row(A, N - 1 - mp) : tl.row(A, mp);
            return (flip & GF_NEG) ? -x : x;
        }
        case BC_FLIP: {   // flip_shift.m:22-40
            T x = upper ? tl.row(A, N - 1) : tl.row(A, 0);
            return (flip & GF_NEG) ? -x : x;
        }
        case BC_ZERO:     // zero_shift.m:14-46
            if (flip & (upper ? GF_ZHI : GF_ZLO)) return T(0);
            return upper ? tl.row(A, N - 1) : tl.row(A, 0);
        case BC_WALL: return (T)(ev != NO_EV ? ev : edge[tl.col]);
        case BC_TRANS: return (T)trans_bc_ghost<T, CPT>(tl, A, n, mp, act, edge, bc_inf, ev);
        default: return upper ? tl.row(A, N - 1) : tl.row(A, 0);   // const and fade: constant shift
    }
}

// Fade anchors of A for a shift by n = -1 or +1 (constant-shifted rows 0 and N-1).
template <typename T, int CPT>
__device__ __forceinline__ Ghost<T> fade_anchors(const Tile<T, CPT>& tl, const T* A, int n) {
    const int N = tl.N;
    Ghost<T> q;
    q.g = T(0);
    if (n < 0) { q.s0 = tl.row(A, 0); q.sN1 = tl.row(A, N - 2 < 0 ? 0 : N - 2); }
    else { q.s0 = tl.row(A, N > 1 ? 1 : 0); q.sN1 = tl.row(A, N - 1); }
    return q;
}

// Halo job for one (array, side) of this thread's column.  At the pencil end (rank 0 below, the
// rank holding row N-1 above) it writes the boundary ghost of one shift call -- only when `shift`
// says the reference shifts that side in the coming stage, since a trans edge drifts once per call;
// elsewhere it copies the neighbouring rank's edge rows (`hi_rows` of them above).  Under fade every
// rank keeps the side's anchors (the damping reaches up to bc_infinity rows from each end).  Called
// by exactly one thread per (array, side, column) and stage, after a cluster barrier; the values it
// writes are read by its own CTA only.
template <typename T, int CPT>
__device__ __forceinline__ void halo_job(const Tile<T, CPT>& tl, T* A, Ghost<T>* an, int side, bool shift, int mode,
                                         int act, int flip, double* edge, double bc_inf, int hi_rows) {
    if (shift && mode == BC_FADE) an[tl.b] = fade_anchors(tl, (const T*)A, side ? +1 : -1);
    if (side == 0) {
        if (tl.rank == 0) {
            if (shift) A[tl.lidx(0)] = bc_ghost(tl, (const T*)A, -1, 1, mode, act, flip, edge, bc_inf, NO_EV);
        } else {
            A[tl.lidx(0)] = tl.remote(A, tl.rank - 1)[tl.lidx(tl.RC)];
        }
    } else {
        if (tl.rank == tl.rank_hi) {
            if (shift) A[tl.ridx(tl.N)] = bc_ghost(tl, (const T*)A, +1, 1, mode, act, flip, edge, bc_inf, NO_EV);
        } else if (tl.rank < tl.rank_hi) {
            const T* up = tl.remote(A, tl.rank + 1);
            for (int h = 1; h <= hi_rows; ++h) A[tl.lidx(tl.RC + h)] = up[tl.lidx(h)];
        }
    }
}

}  // namespace img
