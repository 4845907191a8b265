// Pencil tiles shared by the sweep kernels.
//
// A pencil is one line of cells along the sweep dimension d.  A CTA holds a bundle of Wb pencils
// ("columns") and G rows of each (one cell per thread); a thread-block cluster of CL CTAs covers
// pencils longer than G (rank r holds rows [r*G, (r+1)*G)), so every pencil stays on chip whatever
// its length.  Thread (b, g) owns row g of column b; consecutive threads touch consecutive cells,
// so global loads/stores are coalesced along x for every sweep direction.
//
// Stencil operands live in shared-memory arrays A[row][b] (one per flux array).  A neighbour read
// is one shared load; the row across a CTA boundary is read from the neighbouring cluster rank
// through DSMEM; the rows beyond the pencil ends are boundary-condition ghosts that a few threads
// compute once per stage into ghost slots (shifting/*_shift.m), including the drift of stateful
// edges.  Boundary predicates are per-thread constants, so the common path has no extra work.
#pragma once

#include "common.cuh"

namespace img {

// Geometry of one directional sweep (host-filled).
struct SweepGeom {
    Geom g;
    int d;            // sweep dimension 0..2
    int d1, d2;       // the other two dimensions, in increasing order
    int N;            // pencil length g.n[d]
    long long ncol;   // number of pencils = ncell / N
    int Wb;           // pencils per CTA
    int G;            // rows (threads) per pencil per CTA
    int CL;           // CTAs per cluster along the pencil
    int NT;           // threads per CTA = Wb * G
};

// Ghost slot of one (array, side, column): the ghost value beyond the pencil end and the two fade
// anchors (constant-shifted values at rows 0 and N-1 before damping).
template <typename T>
struct Ghost {
    T g, s0, sN1;
};

template <typename T, int CPT>
struct Tile {
    int b, g, rank, N, Wb, G, CL, d, RC;
    long long col;        // global pencil index
    bool colok;
    long long base;       // linear offset of row 0 of this pencil
    long long sd;         // stride along the sweep
    int coord1, coord2;
    // rows owned by this thread: local row g + k*G, global row rank*RC + g + k*G

    __device__ __forceinline__ void init(const SweepGeom& s) {
        const int t = threadIdx.x;
        if (s.d == 0) { g = t % s.G; b = t / s.G; }
        else { b = t % s.Wb; g = t / s.Wb; }
        rank = (int)(blockIdx.x % (unsigned)s.CL);
        long long bundle = blockIdx.x / (unsigned)s.CL;
        N = s.N;
        Wb = s.Wb;
        G = s.G;
        CL = s.CL;
        d = s.d;
        RC = G * CPT;
        col = bundle * s.Wb + b;
        colok = col < s.ncol;
        long long c = colok ? col : 0;
        coord1 = (int)(c % s.g.n[s.d1]);
        coord2 = (int)(c / s.g.n[s.d1]);
        base = coord1 * sel3(s.d1, s.g.s[0], s.g.s[1], s.g.s[2]) +
               (long long)coord2 * sel3(s.d2, s.g.s[0], s.g.s[1], s.g.s[2]);
        sd = sel3(s.d, s.g.s[0], s.g.s[1], s.g.s[2]);
    }
    __device__ __forceinline__ int lrow(int k) const { return g + k * G; }
    __device__ __forceinline__ int grow(int k) const { return rank * RC + g + k * G; }
    __device__ __forceinline__ bool ok(int k) const { return colok && grow(k) < N; }
    __device__ __forceinline__ long long off(int k) const { return base + (long long)grow(k) * sd; }
    __device__ __forceinline__ int idx(int k) const { return lrow(k) * Wb + b; }
    __device__ __forceinline__ void coords(int k, int& x, int& y, int& z) const {
        int r = grow(k);
        if (d == 0) { x = r; y = coord1; z = coord2; }
        else if (d == 1) { x = coord1; y = r; z = coord2; }
        else { x = coord1; y = coord2; z = r; }
    }
    __device__ __forceinline__ void csync() const {
        if (CL > 1) cg::this_cluster().sync();
        else __syncthreads();
    }
    template <typename U>
    __device__ __forceinline__ U* remote(U* p, int r) const {
        if (CL == 1 || r == rank) return p;
        return cg::this_cluster().map_shared_rank(p, r);
    }
    // Value of array A at global row r of this column (any cluster rank).
    template <typename U>
    __device__ __forceinline__ U row(const U* A, int r) const {
        int rk = r / RC;
        const U* p = remote(const_cast<U*>(A), rk);
        return p[(r - rk * RC) * Wb + b];
    }
    // A.shift(d, -1) and A.shift(d, +1) at row k before fade damping (gs: the array's ghost slots,
    // [side][column]).  The rare cases (pencil end, other cluster rank) are per-row constants.
    template <typename U>
    __device__ __forceinline__ U below(const U* A, const Ghost<U>* gs, int k) const {
        if (grow(k) == 0) return gs[b].g;
        if (lrow(k) == 0) return remote(const_cast<U*>(A), rank - 1)[(RC - 1) * Wb + b];
        return A[idx(k) - Wb];
    }
    template <typename U>
    __device__ __forceinline__ U above(const U* A, const Ghost<U>* gs, int k) const {
        if (grow(k) >= N - 1) return gs[Wb + b].g;   // also rows past the pencil end (idle cells)
        if (lrow(k) == RC - 1) return remote(const_cast<U*>(A), rank + 1)[b];
        return A[idx(k) + Wb];
    }
    // A.shift(d, +2) at row k before fade damping; ghosts at rows N and N+1 in g2[0], g2[1].
    template <typename U>
    __device__ __forceinline__ U above2(const U* A, const U g2[2], int k) const {
        const int r = grow(k) + 2;
        if (r >= N) return r == N ? g2[0] : g2[1];
        const int lr = lrow(k) + 2;
        if (lr >= RC) return remote(const_cast<U*>(A), rank + 1)[(lr - RC) * Wb + b];
        return A[idx(k) + 2 * Wb];
    }
    // Cluster rank that holds the pencil's last row (where its upper ghosts are consumed).
    __device__ __forceinline__ int rank_hi() const { return (N - 1) / RC; }
};

// Fade damping of fade_shift.m:31-44 applied to the constant-shifted value sv at row r of a line of
// N cells: s0 and sN1 are the constant-shifted values at rows 0 and N-1 (the two anchors).
template <typename T>
__device__ __forceinline__ T fade_apply(T sv, int r, int N, const double* fc, int f, T s0, T sN1) {
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

// A.shift(d, n) at row k for n = -1 / +1, fade damping included.
template <typename T, int CPT>
__device__ __forceinline__ T shifted(const Tile<T, CPT>& tl, const T* A, const Ghost<T>* gs, int k, int n, int mode,
                                     const double* fc, int f) {
    T v = n < 0 ? tl.below(A, gs, k) : tl.above(A, gs, k);
    if (mode == BC_FADE) {
        const Ghost<T>& q = gs[(n < 0 ? 0 : tl.Wb) + tl.b];
        v = fade_apply(v, tl.grow(k), tl.N, fc, f, q.s0, q.sN1);
    }
    return v;
}

// "No stored-edge value supplied" marker (stored edges are finite physical values).
constexpr double NO_EV = -1.0e300;

// Ghost of array A beyond the pencil end for one shift call A.shift(d, n): n = -1 (row -1),
// n = +1 (row N) or n = +2 (rows N and N+1, mp = 1 or 2 selects which).  Stateful edges (trans,
// wall) use `ev` when given; otherwise a trans edge is drifted here and written back (the caller is
// the one thread per pencil end and shift call).  Rows are read through tl.row (any cluster rank).
template <typename T, int CPT>
__device__ __forceinline__ T bc_ghost(const Tile<T, CPT>& tl, const T* A, int n, int mp, int mode, int act, int flip,
                                      double* edge, double bc_inf, double ev) {
    const int N = tl.N;
    const bool upper = n > 0;
    const int m = n < 0 ? -n : n;
    switch (mode) {
        case BC_CIRC: return upper ? tl.row(A, mp - 1) : tl.row(A, N - 1);
        case BC_MIRROR: {
            T x = upper ? tl.row(A, N - 1 - mp) : tl.row(A, mp);
            return flip ? -x : x;
        }
        case BC_WALL: return (T)(ev != NO_EV ? ev : edge[tl.col]);
        case BC_TRANS: {
            double y0, y1, y2, cur;
            if (upper) {
                y0 = (double)tl.row(A, trans_pick_upper(N, m, 0));
                y1 = (double)tl.row(A, trans_pick_upper(N, m, 1));
                y2 = (double)tl.row(A, trans_pick_upper(N, m, 2));
                cur = (double)tl.row(A, N - 1);
            } else {
                y0 = (double)tl.row(A, trans_pick_lower(N, m, 0));
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
            return (T)trans_ghost(y0, y1, y2, e, bc_inf, 3.0 + mp, (double)tl.row(A, gpos));
        }
        default: return upper ? tl.row(A, N - 1) : tl.row(A, 0);   // const and fade: constant shift
    }
}

// Fill the ghost slot of array A for one side (n = -1 or +1) of this thread's column: ghost value
// and fade anchors.  Called by exactly one thread per (array, side, column) and stage.
template <typename T, int CPT>
__device__ __forceinline__ void fill_ghost(const Tile<T, CPT>& tl, const T* A, Ghost<T>* gs, int n, int mode, int act,
                                           int flip, double* edge, double bc_inf) {
    Ghost<T> q;
    q.g = bc_ghost(tl, A, n, 1, mode, act, flip, edge, bc_inf, NO_EV);
    const int N = tl.N;
    if (n < 0) { q.s0 = tl.row(A, 0); q.sN1 = tl.row(A, N - 2 < 0 ? 0 : N - 2); }
    else { q.s0 = tl.row(A, N > 1 ? 1 : 0); q.sN1 = tl.row(A, N - 1); }
    gs[(n < 0 ? 0 : tl.Wb) + tl.b] = q;
}

}  // namespace img
