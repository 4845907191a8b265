// Pencil machinery shared by the sweep kernels.
//
// A pencil is one line of cells along the sweep dimension d.  A CTA holds a bundle of Wb
// pencils ("columns"); a thread-block cluster of CL CTAs splits long pencils into CL row ranges,
// so a pencil of any length stays on chip (rank r owns rows [r*RC, (r+1)*RC), RC = G*CPT).
// Each thread owns CPT consecutive cells of one column; values live in registers.  Stencil
// neighbours across thread boundaries and the pencil-end windows that the boundary conditions
// need (rows 0,1,2 and N-3,N-2,N-1) are exchanged through shared memory, and through
// distributed shared memory (map_shared_rank) across the CTAs of a cluster.
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
    int G;            // thread groups per pencil per CTA
    int CL;           // CTAs per cluster along the pencil
    int NT;           // threads per CTA = Wb * G
};

// Per-thread pencil context.
template <typename T, int CPT, int NSLOT, bool HAS2 = false>
struct Pencil {
    const SweepGeom* sg;
    int t, b, g, rank, RC;
    long long col;     // global pencil index (may be >= ncol for idle threads)
    bool colok;
    int r0;            // first row of this thread's segment
    int nv;            // valid rows in the segment (0..CPT)
    long long base;    // linear offset of row 0 of this pencil
    int coord1, coord2;// coordinates of the pencil along d1, d2
    // shared buffers
    T* xf;   // [NSLOT][NT] first value of each thread segment
    T* xs;   // [NSLOT][NT] second value (for shifts by +2)
    T* xl;   // [NSLOT][NT] last valid value
    T* ends; // [NSLOT][Wb][6]

    __device__ void init(const SweepGeom& s, unsigned char* smem_base) {
        sg = &s;
        t = threadIdx.x;
        if (s.d == 0) { g = t % s.G; b = t / s.G; }
        else { b = t % s.Wb; g = t / s.Wb; }
        rank = (int)(blockIdx.x % (unsigned)s.CL);
        long long bundle = blockIdx.x / (unsigned)s.CL;
        RC = s.G * CPT;
        col = bundle * s.Wb + b;
        colok = col < s.ncol;
        r0 = rank * RC + g * CPT;
        int rem = s.N - r0;
        nv = colok ? (rem < 0 ? 0 : (rem > CPT ? CPT : rem)) : 0;
        long long c = colok ? col : 0;
        coord1 = (int)(c % s.g.n[s.d1]);
        coord2 = (int)(c / s.g.n[s.d1]);
        base = coord1 * s.g.s[s.d1] + (long long)coord2 * s.g.s[s.d2];
        T* p = reinterpret_cast<T*>(smem_base);
        xf = p; p += NSLOT * s.NT;
        xs = p; if (HAS2) p += NSLOT * s.NT;
        xl = p; p += NSLOT * s.NT;
        ends = p;
    }
    static __host__ __device__ size_t smem_bytes(int NT, int Wb) {
        return sizeof(T) * ((size_t)(HAS2 ? 3 : 2) * NSLOT * NT + (size_t)NSLOT * Wb * 6);
    }
    __device__ __forceinline__ long long off(int k) const { return base + (long long)(r0 + k) * sg->g.s[sg->d]; }
    __device__ __forceinline__ bool valid(int k) const { return k < nv; }
    __device__ __forceinline__ int row(int k) const { return r0 + k; }
    // cell coordinates (x, y, z) of segment row k
    __device__ __forceinline__ void coords(int k, int& x, int& y, int& z) const {
        int r = r0 + k;
        if (sg->d == 0) { x = r; y = coord1; z = coord2; }
        else if (sg->d == 1) { x = coord1; y = r; z = coord2; }
        else { x = coord1; y = coord2; z = r; }
    }

    __device__ __forceinline__ void csync() const {
        if (sg->CL > 1) cg::this_cluster().sync();
        else __syncthreads();
    }
    __device__ __forceinline__ int tid_of(int bb, int gg) const { return sg->d == 0 ? bb * sg->G + gg : gg * sg->Wb + bb; }
    template <typename U>
    __device__ __forceinline__ U* remote(U* p, int r) const {
        if (sg->CL == 1) return p;
        return cg::this_cluster().map_shared_rank(p, r);
    }

    // Publish array A (this thread's CPT values) into slot s.
    __device__ void publish(int s, const T (&A)[CPT]) {
        int NT = sg->NT;
        xf[s * NT + t] = A[0];
        if (HAS2) xs[s * NT + t] = A[CPT > 1 ? 1 : 0];
        if (nv > 0) xl[s * NT + t] = A[nv - 1];
#pragma unroll
        for (int k = 0; k < CPT; ++k) {
            if (k < nv) {
                int r = r0 + k;
                if (r < 3) ends[(s * sg->Wb + b) * 6 + r] = A[k];
                int u = r - (sg->N - 3);
                if (u >= 0) ends[(s * sg->Wb + b) * 6 + 3 + u] = A[k];
            }
        }
    }
    // Value of the array at global row r of this column (r in 0..2 or N-3..N-1), from the ends buffer.
    __device__ T endv(int s, int r) const {
        int slot = r < 3 ? r : 3 + (r - (sg->N - 3));
        int rk = r / RC;
        T* p = remote(ends, rk);
        return p[(s * sg->Wb + b) * 6 + slot];
    }
    // A at row (r0 + k - 1); requires that row to exist (>= 0).
    __device__ T prev(int s, const T (&A)[CPT], int k) const {
        if (k > 0) return A[k - 1];
        int NT = sg->NT;
        if (g > 0) return xl[s * NT + tid_of(b, g - 1)];
        T* p = remote(xl, rank - 1);
        return p[s * NT + tid_of(b, sg->G - 1)];
    }
    // A at row (r0 + k + 1); requires that row to exist (<= N-1).
    __device__ T next(int s, const T (&A)[CPT], int k) const {
        if (k + 1 < CPT) return A[k + 1];
        int NT = sg->NT;
        if (g + 1 < sg->G) return xf[s * NT + tid_of(b, g + 1)];
        T* p = remote(xf, rank + 1);
        return p[s * NT + tid_of(b, 0)];
    }
    // A at row (r0 + k + 2); requires that row to exist.  Needs CPT >= 2.
    __device__ T next2(int s, const T (&A)[CPT], int k) const {
        if (k + 2 < CPT) return A[k + 2];
        int NT = sg->NT;
        int gg = g + 1, rr = rank;
        if (gg >= sg->G) { gg = 0; rr = rank + 1; }
        int sel = (k + 2) - CPT;   // 0: first of next segment, 1: second
        T* pf = rr == rank ? xf : remote(xf, rr);
        T* ps = rr == rank ? xs : remote(xs, rr);
        return sel == 0 ? pf[s * NT + tid_of(b, gg)] : ps[s * NT + tid_of(b, gg)];
    }
};

// Value of A.shift(d, n)[r] for n = -1 (from_prev) or +1 computed from the const-shifted value
// sv (A[r-1] or A[r+1] with the end row repeated) and the fade damping of fade_shift.m:31-44.
// a0/an1 are the const-shifted values at rows 0 and N-1 (the two fade anchors before damping).
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

}  // namespace img
