// Grid treadmill (treadmill/treadmillGrid.m:14-37) on the device, three launches per call:
//   treadmill_detect_kernel    one CTA per pencil along DIRECTION: mass.shift(X, 1) (with the mass
//                              array's own upper boundary, a trans edge drifting as in the reference),
//                              the forward difference / dGrid, and the first index of its maximum
//                              (NaN skipped, as MATLAB's max does);
//   treadmill_finalize_kernel  one CTA: newIndex = round(mean(mean(indices))) in MATLAB's order (see
//                              there), then `last` on the first call, else dCells = newIndex - last and
//                              the history entry;
//   treadmill_shift_kernel     one CTA per (pencil, primary array): A.array = A.shift(X, dCells) with the
//                              array's own boundary conditions, for any shift distance.
// A pencil is staged in shared memory (the line and its shifted copy), so every boundary rule reads
// the whole line, as the reference's shift functions do.  Not on the hot path: a treadmill run takes
// no CUDA graph and no fused CFL epilogue (the state moves after the last sweep of a step).
#pragma once

#include "pencil.cuh"

namespace img {

constexpr int TREAD_ARRAYS = 8;   // rho, p_x, p_y, p_z, E, B_x, B_y, B_z

struct TreadArgs {
    Geom g;
    int d, d1, d2;                 // DIRECTION - 1 and the two other dimensions (d1 < d2)
    int n1, n2;                    // their extents; pencil col = c1 + n1 * c2
    long long sd, s1, s2;          // strides along d, d1, d2
    void* q[NQ];
    DevTime* tm;
    double dx;                     // DGRID{X}
    int mode[TREAD_ARRAYS][2];     // BC mode of each array's class along d: [array][side]
    int neg[TREAD_ARRAYS];         // the array's component is DIRECTION (mirror / flip negate)
    int act[TREAD_ARRAYS];         // Edges.ACTIVE(DIRECTION) of the array's class (linear-index reading)
    double* edge[TREAD_ARRAYS][2]; // stored edges of the primaries along d (null unless trans / wall)
    const double* fade;
    int fade_f;
    double bc_inf;
    int* idx;                      // per pencil: 1-based index of the maximum
    double* means;                 // first means (n2 values)
    int* hist;                     // TreadmillManager.history
    int hist_cap;
    const void* fade_map;          // point-fade map (null: none) and the arrays it acts on (bits of
    int fade_mask;                 // IMG_FADE_*: 1 rho, 2 momentum, 4 E): the shift's assignment fades them
};

__host__ __device__ inline size_t tread_smem_bytes(int N, size_t elem) { return 2 * (size_t)N * elem; }

__device__ __forceinline__ long long tread_base(const TreadArgs& a, long long col) {
    const long long c2 = col / a.n1, c1 = col - c2 * a.n1;
    return c1 * a.s1 + c2 * a.s2;
}

// out = A.shift(X, n) of one line L of N values (any n; shifting/*_shift.m), by the whole CTA.
// `edge` is the stored edge slot of this line for the side the shift reads (n < 0: lower, else upper,
// as the reference's -sign(n) branches do for n = 0 too); a trans edge drifts once per call.
template <typename T>
__device__ void line_shift(const T* L, T* out, int N, int n, int mode, bool neg, int act, double* edge,
                           const double* fc, int f, double bc_inf) {
    __shared__ double s_edge;
    const int m = n < 0 ? -n : n;
    const bool upper = n >= 0;
    if (mode == BC_TRANS && threadIdx.x == 0) {
        double e = 0.0;
        if (act && edge) {   // transparentEdge: drift toward the current edge cell (Edges.m)
            e = edge_drift(*edge, (double)L[upper ? N - 1 : 0]);
            *edge = e;
        }
        s_edge = e;
    }
    __syncthreads();
    for (int i = threadIdx.x; i < N; i += blockDim.x) {
        T v;
        const bool ghost = m > 0 && (n < 0 ? i < m : i >= N - m);
        if (mode == BC_CIRC) {
            v = L[((i + n) % N + N) % N];
        } else if (mode == BC_MIRROR) {   // mirror_shift.m:23-39
            int src;
            if (n < 0) src = i >= m ? i - m : m - i;
            else src = i < N - m ? i + m : N - 2 - (i - (N - m));
            src = src < 0 ? 0 : (src > N - 1 ? N - 1 : src);   // |n| >= N - 1: the reference's own index error
            v = L[src];
            if (ghost && neg) v = -v;
        } else {
            int src = i + n;
            src = src < 0 ? 0 : (src > N - 1 ? N - 1 : src);
            v = L[src];
            if (ghost) {
                if (mode == BC_FLIP && neg) v = -v;                                     // flip_shift.m
                else if (mode == BC_WALL) v = (T)(edge ? *edge : 0.0);                  // wall_shift.m
                else if (mode == BC_TRANS) {                                            // transparent_shift.m
                    const int k = n < 0 ? i : i - (N - m);
                    const double xe = n < 0 ? 3.0 + (m - k) : 3.0 + (k + 1);
                    const double y1 = (double)L[n < 0 ? trans_pick_lower(N, m, 1) : trans_pick_upper(N, m, 1)];
                    const double y2 = (double)L[n < 0 ? trans_pick_lower(N, m, 2) : trans_pick_upper(N, m, 2)];
                    v = (T)trans_ghost(y1, y2, s_edge, bc_inf, xe, (double)L[i]);
                }
            }
            if (mode == BC_FADE) {   // fade_shift.m: damp the constant shift toward its end rows
                int s0 = n, sN = N - 1 + n;
                s0 = s0 < 0 ? 0 : (s0 > N - 1 ? N - 1 : s0);
                sN = sN < 0 ? 0 : (sN > N - 1 ? N - 1 : sN);
                v = fade_apply(v, i, N, fc, f, L[s0], L[sN]);
            }
        }
        out[i] = v;
    }
    __syncthreads();
}

template <typename T>
__global__ void __launch_bounds__(256) treadmill_detect_kernel(const __grid_constant__ TreadArgs a) {
    extern __shared__ __align__(16) unsigned char smem[];
    if (a.tm->done || a.tm->error) return;
    const int N = a.g.n[a.d];
    T* L = reinterpret_cast<T*>(smem);
    T* S = L + N;
    const long long col = blockIdx.x;
    const long long b = tread_base(a, col);
    const T* rho = reinterpret_cast<const T*>(a.q[Q_RHO]);
    for (int i = threadIdx.x; i < N; i += blockDim.x) L[i] = rho[b + i * a.sd];
    __syncthreads();
    double* e = a.edge[0][1] ? a.edge[0][1] + col : nullptr;
    line_shift<T>(L, S, N, +1, a.mode[0][1], false, a.act[0], e, a.fade, a.fade_f, a.bc_inf);
    // first maximum of (rho.shift(X,1) - rho) / dGrid; NaN never compares larger
    double best = -HUGE_VAL;
    int bi = N;   // no value above -inf yet
    for (int i = threadIdx.x; i < N; i += blockDim.x) {
        const double v = ((double)S[i] - (double)L[i]) / a.dx;
        if (v > best) { best = v; bi = i; }
    }
    // (value, index) pairs: the larger value wins, the smaller index on ties
    __shared__ double sv[8];
    __shared__ int si[8];
    for (int o = 16; o > 0; o >>= 1) {
        const double ov = __shfl_xor_sync(0xffffffffu, best, o);
        const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
        if (ov > best || (ov == best && oi < bi)) { best = ov; bi = oi; }
    }
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) { sv[w] = best; si[w] = bi; }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int k = 1; k < (int)(blockDim.x >> 5); ++k)
            if (sv[k] > best || (sv[k] == best && si[k] < bi)) { best = sv[k]; bi = si[k]; }
        a.idx[col] = (bi >= N ? 0 : bi) + 1;   // nothing above -inf (all NaN): index 1
    }
}

// newIndex = round(mean(mean(I))) for the index array I of size n1 x n2 (the non-swept dimensions, d1
// fastest).  MATLAB's mean runs along the first non-singleton dimension: with n1, n2 > 1 the first mean
// averages along d1 (exact integer sums, one division each), the second sums those means in order and
// divides by n2; with one of them 1 it is one mean over all pencils (a sum in order).  round: halves
// away from zero.
__global__ void treadmill_finalize_kernel(const __grid_constant__ TreadArgs a) {
    if (a.tm->done || a.tm->error) {
        if (threadIdx.x == 0) a.tm->tread_go = 0;
        return;
    }
    const int n1 = a.n1, n2 = a.n2;
    const bool two = n1 > 1 && n2 > 1;
    if (two) {
        for (int c2 = threadIdx.x; c2 < n2; c2 += blockDim.x) {
            long long s = 0;
            for (int c1 = 0; c1 < n1; ++c1) s += a.idx[c1 + (long long)n1 * c2];
            a.means[c2] = (double)s / n1;
        }
    }
    __syncthreads();
    if (threadIdx.x != 0) return;
    double t = 0.0;
    long long cnt;
    if (two) {
        for (int c2 = 0; c2 < n2; ++c2) t += a.means[c2];
        cnt = n2;
    } else {
        cnt = (long long)n1 * n2;
        for (long long k = 0; k < cnt; ++k) t += (double)a.idx[k];
    }
    const int new_index = (int)round(t / (double)cnt);
    DevTime* tm = a.tm;
    if (tm->tread_last < 0) {   // treadmillGrid.m:25-28
        tm->tread_last = new_index;
        tm->tread_go = 0;
        return;
    }
    const int dc = new_index - tm->tread_last;
    tm->tread_dc = dc;
    tm->tread_go = 1;
    if (tm->tread_count < a.hist_cap) a.hist[tm->tread_count] = dc;
    tm->tread_count += 1;
}

template <typename T>
__global__ void __launch_bounds__(256) treadmill_shift_kernel(const __grid_constant__ TreadArgs a) {
    extern __shared__ __align__(16) unsigned char smem[];
    if (!a.tm->tread_go || a.tm->done || a.tm->error) return;
    const int N = a.g.n[a.d];
    const int n = a.tm->tread_dc;
    const int arr = blockIdx.y;
    const int qv = arr == 0 ? Q_RHO : (arr <= 3 ? Q_PX + arr - 1 : (arr == 4 ? Q_E : Q_BX + arr - 5));
    T* A = reinterpret_cast<T*>(a.q[qv]);
    T* L = reinterpret_cast<T*>(smem);
    T* S = L + N;
    const long long col = blockIdx.x;
    const long long b = tread_base(a, col);
    for (int i = threadIdx.x; i < N; i += blockDim.x) L[i] = A[b + i * a.sd];
    __syncthreads();
    const int side = n > 0 ? 1 : 0;   // ImogenArray.shift: edgeshifts{1 + (n > 0)}
    double* slot = a.edge[arr][n >= 0 ? 1 : 0];
    line_shift<T>(L, S, N, n, a.mode[arr][side], a.neg[arr] != 0, a.act[arr], slot ? slot + col : nullptr, a.fade,
                  a.fade_f, a.bc_inf);
    const int fbit = arr == 0 ? 1 : (arr <= 3 ? 2 : (arr == 4 ? 4 : 0));
    const T* F = reinterpret_cast<const T*>(a.fade_map);
    const bool fade = F && (a.fade_mask & fbit);
    for (int i = threadIdx.x; i < N; i += blockDim.x) {
        const long long o = b + i * a.sd;
        A[o] = fade ? point_fade(S[i], F[o]) : S[i];
    }
}

}  // namespace img
