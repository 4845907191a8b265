// C++ FP64 restatement of Imogen's relaxing-TVD fluid + magnet update.
//
// TEST INFRASTRUCTURE ONLY: this is the oracle (the checker).  Only tests/, the smoke check and
// the CPU-baseline / reference arm of bench.py load it; the product library never links it.
//
// Like oracle/np_oracle.py it restates the reference array-at-a-time, one full-array temporary per
// MATLAB expression, so every statement can be read against the MATLAB line it follows (cited
// inline).  The two oracles perform the same IEEE-754 operations in the same order and agree
// bit for bit (checked by tests/test_oracle.py).  Built with -O2 -ffp-contract=off (no FMA
// contraction, no fast-math).  Element-wise loops are OpenMP-parallel over cells; results do not
// depend on the thread count (no reductions other than max, which is exact).
//
// Parity against the MATLAB reference itself is unpinned (MATLAB/Octave are not available); the
// MATLAB builtins it depends on are pinned separately (pchip vs SciPy; the perms tables below
// against oracle/np_oracle.py's restatement of the R2009-era perms algorithm).

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

enum Mode { CIRC = 0, CONST = 1, FADE = 2, MIRROR = 3, TRANS = 4, WALL = 5, FLIP = 6, ZERO = 7, LINEAR = 8, WORMHOLE = 9 };
// FluxArray.fluxType (flux/FluxArray.m:28-35) as zero_shift.m reads it: not a FluxArray, 'fluxr',
// 'fluxl', or another flux type ('flux' of MagnetArray.m:96)
enum FluxType { FT_NONE = 0, FT_FLUXR = 1, FT_FLUXL = 2, FT_FLUX = 3 };
enum Lim { VANLEER = 0, SUPERBEE = 1, MINMOD = 2 };
enum Cls { C_MASS = 0, C_MOM = 1, C_ENER = 2, C_MAG = 3 };

using Vec = std::vector<double>;

// flux.m:17-27 -- the sweep order rows and the matching magnet indices.  FWD = perms([1 2 3]) and
// BWD = perms([3 2 1]) as MATLAB R2009a-R2010b computes them: perms(V) = V(P) over the position
// permutations P = perms(1:3) = 321, 312, 231, 213, 123, 132 (recursive construction with the
// relabelling t(t == i) = n, which leaves the last two rows out of reverse-lexicographic order), so
// BWD = 4 - FWD row by row.
const int FWD[6][3] = {{3, 2, 1}, {3, 1, 2}, {2, 3, 1}, {2, 1, 3}, {1, 2, 3}, {1, 3, 2}};
const int BWD[6][3] = {{1, 2, 3}, {1, 3, 2}, {2, 1, 3}, {2, 3, 1}, {3, 2, 1}, {3, 1, 2}};
const int FWD_MI[3][2] = {{2, 3}, {1, 3}, {1, 2}};
const int BWD_MI[3][2] = {{3, 2}, {3, 1}, {2, 1}};

double msign(double v) { return v > 0 ? 1.0 : (v < 0 ? -1.0 : (v == 0 ? 0.0 : v)); }

// ------------------------------------------------------------------------------------------------
// pchip (MATLAB pchip / Moler pchiptx): harmonic-mean interior slopes, one-sided end slopes.
// ------------------------------------------------------------------------------------------------
void pchip_col(const double* x, int n, const double* y, const double* xi, int m, double* out) {
    std::vector<double> h(n - 1), del(n - 1), d(n);
    for (int k = 0; k < n - 1; ++k) {
        h[k] = x[k + 1] - x[k];
        del[k] = (y[k + 1] - y[k]) / h[k];
    }
    for (int k = 1; k < n - 1; ++k) {
        double w1 = 2 * h[k] + h[k - 1];
        double w2 = h[k] + 2 * h[k - 1];
        if (msign(del[k - 1]) * msign(del[k]) > 0)
            d[k] = (w1 + w2) / (w1 / del[k - 1] + w2 / del[k]);
        else
            d[k] = 0.0;
    }
    auto endslope = [](double h0, double h1, double d0, double d1) {
        double dd = ((2 * h0 + h1) * d0 - h0 * d1) / (h0 + h1);
        if (msign(dd) != msign(d0)) dd = 0.0;
        else if (msign(d0) != msign(d1) && std::fabs(dd) > std::fabs(3 * d0)) dd = 3 * d0;
        return dd;
    };
    d[0] = endslope(h[0], h[1], del[0], del[1]);
    d[n - 1] = endslope(h[n - 2], h[n - 3], del[n - 2], del[n - 3]);
    for (int j = 0; j < m; ++j) {
        int k = int(std::upper_bound(x, x + n, xi[j]) - x) - 1;
        k = std::min(std::max(k, 0), n - 2);
        double s = xi[j] - x[k];
        double c1 = (d[k] + d[k + 1] - 2 * del[k]) / (h[k] * h[k]);
        double c2 = (3 * del[k] - 2 * d[k] - d[k + 1]) / h[k];
        out[j] = ((c1 * s + c2) * s + d[k]) * s + y[k];
    }
}

struct Sim;

// ------------------------------------------------------------------------------------------------
// Edges.m
// ------------------------------------------------------------------------------------------------
struct Edges {
    bool active[2][3] = {{false, false, false}, {false, false, false}};
    Vec store[2][3];
    double tol = 0.005;
};

struct IArr {
    Sim* sim = nullptr;
    int component = 0;   // 0 scalar, 1..3
    int cls = 0;         // BC class
    int ftype = FT_NONE; // FluxArray type (zero_shift.m)
    const Vec* fades = nullptr;   // PointFade map applied at every assignment (readFades; primaries)
    Vec a;
    bool uninit = true;
    Edges edges;
    void set(Vec v);
    void cleanup() { a.clear(); a.shrink_to_fit(); }
    Vec shift(int DIRECT, int n);
    Vec transparent_edge(int dim, bool upper);
};

struct Sim {
    int n[3];
    long long N;
    int ndims;
    double dgrid[3];
    double gamma, cfl, minmass;
    int bc[4][2][3];
    int bc_inf;
    Vec fade_coeff;
    int limiter[3];
    bool fluid_active, magnet_active;
    double time_max;
    int iter_max;
    int update_mode;
    double time = 0, dt = 0;
    int iteration = 1;
    double last_cmax = 0;
    int last_grid_index = 0;
    // ArtificialViscosity (0 empty, 1 neumann_richtmyer, 2 caramana_shashkov_whalen) and Radiation
    // (0 empty, 1 optically_thin) settings (ArtificialViscosity.m:31-57, Radiation.m:32-57)
    int visc_type = 0;
    double visc_lin = 0, visc_quad = 0;
    int rad_type = 0;
    double rad_exp = 0.5, rad_initmax = 0, rad_strength = 1;
    // TreadmillManager (treadmill/TreadmillManager.m): direction (0 inactive), last, history
    int treadmill_dir = 0;
    // one PointFade (ImogenManager.addFades, PointFade.m:29-38): the map and the fluid variables it acts
    // on (bit 0 mass, 1 mom, 2 ener)
    Vec fade_arr;
    int fade_mask = 0;
    int treadmill_last = -1;
    std::vector<int> treadmill_history;

    struct FluidVar { IArr prim, store, store_fluxR, store_fluxL, fluxR, fluxL; };
    struct MagComp {
        IArr prim, cellMag;
        IArr velGrid[4], store[4], store_fluxR[4], wMag[4], flux[4];   // indexed by X (1..3)
        bool isZero = false;
    };
    FluidVar fv[5];   // mass, momx, momy, momz, ener
    MagComp mg[3];

    long long stride(int d) const { return d == 0 ? 1 : (d == 1 ? n[0] : (long long)n[0] * n[1]); }
    long long face(int d) const { return N / n[d]; }

    void init_arr(IArr& A, int comp, int cls) { A.sim = this; A.component = comp; A.cls = cls; }
};

// Extract the face of array a at index idx along dim d, in column-major order of the other dims.
Vec take_face(const Sim& s, const Vec& a, int d, int idx) {
    Vec out(s.face(d));
    int d1 = d == 0 ? 1 : 0, d2 = d == 2 ? 1 : 2;
    long long sd = s.stride(d), s1 = s.stride(d1), s2 = s.stride(d2);
    for (int j = 0; j < s.n[d2]; ++j)
        for (int i = 0; i < s.n[d1]; ++i)
            out[(long long)j * s.n[d1] + i] = a[idx * sd + i * s1 + j * s2];
    return out;
}

void IArr::set(Vec v) {
    if (fades) {   // ImogenArray.applyFades -> PointFade.fadeArray (PointFade.m:46-49), before the edges
        const Vec& A = *fades;
        for (size_t k = 0; k < v.size(); ++k) v[k] = 0.95 * v[k] * A[k] + v[k] * (1 - A[k]);
    }
    a = std::move(v);
    if (uninit) {   // Edges(bcModes, array, 0.005) at first assignment (Edges.m:37-110)
        for (int side = 0; side < 2; ++side)
            for (int d = 0; d < sim->ndims; ++d) {
                int mode = sim->bc[cls][side][d];
                if (mode == TRANS || mode == WALL) {
                    edges.active[side][d] = true;
                    edges.store[side][d] = take_face(*sim, a, d, side == 0 ? 0 : sim->n[d] - 1);
                } else if (mode == FADE) {
                    edges.active[side][d] = true;
                }
            }
        uninit = false;
    }
}

Vec IArr::transparent_edge(int dim, bool upper) {
    // ImogenArray.transparentEdge -> Edges.getEdge (Edges.m:112-137)
    int d = dim - 1, side = upper ? 1 : 0;
    int mode = sim->bc[cls][side][d];
    if (mode == TRANS) {
        Vec ne = take_face(*sim, a, d, upper ? sim->n[d] - 1 : 0);
        Vec& old = edges.store[side][d];
        for (size_t k = 0; k < ne.size(); ++k) {
            double delta = std::min(std::fabs(ne[k] - old[k]), edges.tol);
            bool st = (ne[k] - old[k]) > 0;
            old[k] = old[k] + ((st ? 1.0 : 0.0) - (st ? 0.0 : 1.0)) * delta;
        }
    }
    return edges.store[side][d];
}

// 0-based constant-shift source index (constant_shift.m:21-29)
inline int cidx(int i, int n, int N) { return std::min(std::max(i + n, 0), N - 1); }

Vec IArr::shift(int DIRECT, int n) {
    const Sim& s = *sim;
    int d = DIRECT - 1;
    if (d >= s.ndims) return a;   // ImogenArray.m:159-163 (pShiftEnabled false)
    int mode = s.bc[cls][n > 0 ? 1 : 0][d];
    int Nd = s.n[d];
    int m = std::abs(n);
    long long sd = s.stride(d);
    long long nf = s.face(d);
    int d1 = d == 0 ? 1 : 0, d2 = d == 2 ? 1 : 2;
    long long s1 = s.stride(d1), s2 = s.stride(d2);
    auto base_of = [&](long long f) { return (f % s.n[d1]) * s1 + (f / s.n[d1]) * s2; };
    Vec r(s.N);

    if (mode == CIRC) {   // circ_shift.m:21-29
#pragma omp parallel for schedule(static)
        for (long long f = 0; f < nf; ++f) {
            long long b = base_of(f);
            for (int i = 0; i < Nd; ++i) r[b + i * sd] = a[b + (((i + n) % Nd + Nd) % Nd) * sd];
        }
        return r;
    }
    if (mode == MIRROR) {   // mirror_shift.m:23-39
        bool flip = component == DIRECT;
#pragma omp parallel for schedule(static)
        for (long long f = 0; f < nf; ++f) {
            long long b = base_of(f);
            for (int i = 0; i < Nd; ++i) {
                int src; bool g = false;
                if (n < 0) {
                    if (i >= m) src = i - m; else { src = m - i; g = true; }
                } else {
                    if (i < Nd - m) src = i + m; else { src = Nd - 2 - (i - (Nd - m)); g = true; }
                }
                double v = a[b + (long long)src * sd];
                r[b + i * sd] = (g && flip) ? -v : v;
            }
        }
        return r;
    }
    // constant shift underlies const / trans / wall / fade / flip / zero / wormhole
#pragma omp parallel for schedule(static)
    for (long long f = 0; f < nf; ++f) {
        long long b = base_of(f);
        for (int i = 0; i < Nd; ++i) r[b + i * sd] = a[b + (long long)cidx(i, n, Nd) * sd];
    }
    if (mode == CONST) return r;
    if (mode == FLIP || mode == ZERO) {
        // flip_shift.m:22-40: the ghosts of the constant shift, negated for the component along DIRECT.
        // zero_shift.m:14-46: a FluxArray's ghosts are 0 except on the side where its type keeps the
        // constant shift (fluxl for n < 0, fluxr for n > 0); other arrays take the constant shift.
        bool zero = false;
        if (mode == ZERO) zero = ftype != FT_NONE && !(n < 0 ? ftype == FT_FLUXL : ftype == FT_FLUXR);
        if (mode == FLIP && component != DIRECT) return r;
        if (mode == ZERO && !zero) return r;
        for (long long f = 0; f < nf; ++f) {
            long long b = base_of(f);
            for (int k = 0; k < m; ++k) {
                double& v = r[b + (long long)(n < 0 ? k : Nd - m + k) * sd];
                v = mode == FLIP ? -v : 0.0;
            }
        }
        return r;
    }
    if (mode == WORMHOLE) {
        // wormhole_shift.m:16-61: for n < 0 the first |n| ghosts along DIRECT are the array's own
        // first |n| cells in reverse order along DIRECT and along nextDir = [2 3 1](DIRECT), negated
        // for the component along DIRECT; for n > 0 the constant shift.  (3-D only: in 2-D the
        // reference indexes a third dimension the array does not have.)
        if (n > 0) return r;
        const int dn = (d + 1) % 3;
        const double sg = component == DIRECT ? -1.0 : 1.0;
        for (long long c = 0; c < s.N; ++c) {
            int xyz[3] = {(int)(c % s.n[0]), (int)((c / s.n[0]) % s.n[1]), (int)(c / ((long long)s.n[0] * s.n[1]))};
            if (xyz[d] >= m) continue;
            int src[3] = {xyz[0], xyz[1], xyz[2]};
            src[d] = m - 1 - xyz[d];
            src[dn] = s.n[dn] - 1 - xyz[dn];
            r[c] = sg * a[src[0] + src[1] * s.stride(1) + src[2] * s.stride(2)];
        }
        return r;
    }

    if (mode == WALL) {   // wall_shift.m:12-33
        Vec e = transparent_edge(DIRECT, n >= 0);   // n = 0: dir = -sign(0) takes the else (upper) branch
        for (long long f = 0; f < nf; ++f) {
            long long b = base_of(f);
            for (int k = 0; k < m; ++k) {
                int gi = n < 0 ? k : Nd - m + k;
                r[b + (long long)gi * sd] = e[f];
            }
        }
        return r;
    }
    if (mode == FADE) {   // fade_shift.m:21-45
        int fs = s.bc_inf;
        const Vec& c = s.fade_coeff;
#pragma omp parallel for schedule(static)
        for (long long f = 0; f < nf; ++f) {
            long long b = base_of(f);
            double anchor = r[b];
            for (int i = 0; i < fs; ++i) {
                double& v = r[b + (long long)i * sd];
                v = (1 - c[i]) * v + c[i] * anchor;
            }
            anchor = r[b + (long long)(Nd - 1) * sd];
            for (int k = 0; k < fs; ++k) {
                int i = Nd - fs + k;
                double ck = c[fs - 1 - k];
                double& v = r[b + (long long)i * sd];
                v = (1 - ck) * v + ck * anchor;
            }
        }
        return r;
    }
    // TRANS: transparent_shift.m:23-99
    bool act = edges.active[(DIRECT - 1) % 2][(DIRECT - 1) / 2];   // ACTIVE(DIRECT), linear index
    Vec e;
    if (act) e = transparent_edge(DIRECT, n >= 0);   // n = 0 takes transparent_shift.m's upper branch
    double xk[5] = {1, 2, 3, double(s.bc_inf), double(s.bc_inf + 1)};
    std::vector<double> xe(m), out(m);   // any shift distance (treadmillGrid shifts by many cells)
    for (int k = 0; k < m; ++k) xe[k] = n < 0 ? 3 + (m - k) : 3 + (k + 1);
    for (long long f = 0; f < nf; ++f) {
        long long b = base_of(f);
        double y[5];
        for (int q = 0; q < 3; ++q) {
            int pick = n < 0 ? std::min(3 - q + m, Nd) - 1 : std::max(Nd - (2 - q) - m, 1) - 1;
            y[q] = r[b + (long long)pick * sd];
        }
        y[3] = act ? e[f] : 0.0;
        y[4] = y[3];
        pchip_col(xk, 5, y, xe.data(), m, out.data());
        for (int k = 0; k < m; ++k) {
            int gi = n < 0 ? k : Nd - m + k;
            double orig = a[b + (long long)gi * sd];
            bool t = std::fabs(orig - out[k]) < 1e-4;
            r[b + (long long)gi * sd] = (t ? 0.0 : 1.0) * out[k] + (t ? 1.0 : 0.0) * orig;
        }
    }
    return r;
}

// ------------------------------------------------------------------------------------------------
// Limiters (flux/*Limiter.m): flux.array = flux.array + correction
// ------------------------------------------------------------------------------------------------
void apply_limiter(int lim, IArr& fl, const Vec& dL, const Vec& dR) {
    Vec out(fl.a.size());
    long long N = (long long)out.size();
    if (lim == VANLEER) {
#pragma omp parallel for schedule(static)
        for (long long i = 0; i < N; ++i) {
            double p = dL[i] * dR[i];
            double st = (p > 0 ? p : 0.0) / (dL[i] + dR[i]);
            if (std::isnan(st)) st = 0.0;
            out[i] = fl.a[i] + st;
        }
    } else {
#pragma omp parallel for schedule(static)
        for (long long i = 0; i < N; ++i) {
            double l = dL[i], r = dR[i];
            if (lim == SUPERBEE) {
                double c = std::fabs(l) < std::fabs(r) ? 1.0 : 0.0;
                l = (1 + c) * l;
                r = (2 - c) * r;
            }
            double corr = 0.125 * (msign(l) + msign(r)) * std::fmin(std::fabs(l), std::fabs(r));
            out[i] = fl.a[i] + corr;
        }
    }
    fl.set(std::move(out));
}

// pressure.m:16-66 (modes used on the hot path: totsnd, sound)
void pressure(Sim& s, bool sound_mode, const Vec& rho, const Vec& px, const Vec& py, const Vec& pz,
              const Vec& E, Vec& result, Vec* aux) {
    const double G = s.gamma;
    long long N = s.N;
    result.assign(N, 0.0);
    if (aux) aux->assign(N, 0.0);
    const Vec* cm[3] = {&s.mg[0].cellMag.a, &s.mg[1].cellMag.a, &s.mg[2].cellMag.a};
    bool use[3] = {!s.mg[0].isZero, !s.mg[1].isZero, !s.mg[2].isZero};
#pragma omp parallel for schedule(static)
    for (long long i = 0; i < N; ++i) {
        double vsq = (px[i] * px[i] + py[i] * py[i] + pz[i] * pz[i]) / (rho[i] * rho[i]);
        double msq = 0.0;
        for (int c = 0; c < 3; ++c)
            if (use[c]) msq = msq + (*cm[c])[i] * (*cm[c])[i];
        double r = (G - 1.0) * (E[i] - 0.5 * rho[i] * vsq);
        if (!sound_mode) {
            (*aux)[i] = std::sqrt(std::fabs((G * (r - (G - 1.0) * 0.5 * msq) + 2.0 * msq) / rho[i]));
            r = r + 0.5 * (2.0 - G) * msq;
        } else {
            r = r - (G - 1.0) * 0.5 * msq;
            r = std::sqrt(std::fabs((G * r + 2.0 * msq) / rho[i]));
        }
        result[i] = r < 0 ? 0.0 : r;
    }
}

// pressure('gas') (pressure.m:23-64): (G-1)(E - rho v^2/2) - (G-1) B^2/2, clamped at 0.
Vec gas_pressure(const Sim& s) {
    const double G = s.gamma;
    long long N = s.N;
    Vec out(N);
    const Vec &rho = s.fv[0].prim.a, &px = s.fv[1].prim.a, &py = s.fv[2].prim.a, &pz = s.fv[3].prim.a,
              &E = s.fv[4].prim.a;
    const Vec* cm[3] = {&s.mg[0].cellMag.a, &s.mg[1].cellMag.a, &s.mg[2].cellMag.a};
    bool use[3] = {!s.mg[0].isZero, !s.mg[1].isZero, !s.mg[2].isZero};
    for (long long i = 0; i < N; ++i) {
        double vsq = (px[i] * px[i] + py[i] * py[i] + pz[i] * pz[i]) / (rho[i] * rho[i]);
        double msq = 0.0;
        for (int c = 0; c < 3; ++c)
            if (use[c]) msq = msq + (*cm[c])[i] * (*cm[c])[i];
        double r = (G - 1.0) * (E[i] - 0.5 * rho[i] * vsq);
        r = r - (G - 1.0) * 0.5 * msq;
        out[i] = r < 0 ? 0.0 : r;
    }
    return out;
}

// x^e as NumPy's power computes it (its fast path takes the square root for e = 0.5).
inline double npow(double x, double e) { return e == 0.5 ? std::sqrt(x) : std::pow(x, e); }

// Radiation.solve: opticallyThinSolver (Radiation.m:86-88): strength * rho^(2-exponent) * Pgas^exponent.
Vec radiation_solve(const Sim& s) {
    Vec gas = gas_pressure(s);
    const Vec& rho = s.fv[0].prim.a;
    Vec out(s.N);
    for (long long i = 0; i < s.N; ++i) out[i] = s.rad_strength * npow(rho[i], 2 - s.rad_exp) * npow(gas[i], s.rad_exp);
    return out;
}

// Radiation.initialize (Radiation.m:61-75): strength from the initial state (face-centred B).
void radiation_initialize(Sim& s) {
    if (s.rad_type != 1) {
        s.rad_strength = 0;
        return;
    }
    s.rad_strength = 1;
    Vec un = radiation_solve(s);
    const Vec &rho = s.fv[0].prim.a, &E = s.fv[4].prim.a;
    const Vec *p[3] = {&s.fv[1].prim.a, &s.fv[2].prim.a, &s.fv[3].prim.a};
    const Vec *b[3] = {&s.mg[0].prim.a, &s.mg[1].prim.a, &s.mg[2].prim.a};
    double mn = std::numeric_limits<double>::quiet_NaN();
    for (long long i = 0; i < s.N; ++i) {
        double ke = 0.5 * ((*p[0])[i] * (*p[0])[i] + (*p[1])[i] * (*p[1])[i] + (*p[2])[i] * (*p[2])[i]) / rho[i];
        double me = 0.5 * ((*b[0])[i] * (*b[0])[i] + (*b[1])[i] * (*b[1])[i] + (*b[2])[i] * (*b[2])[i]);
        double r = (E[i] - ke - me) / un[i];
        if (!std::isnan(r) && (std::isnan(mn) || r < mn)) mn = r;   // minFinderND ignores NaN
    }
    s.rad_strength = (s.rad_initmax / 100) * mn;
}

// ArtificialViscosity.cswSoundSpeed (ArtificialViscosity.m:157-190): as in the reference, only the z
// momentum of the velocity-squared sum is divided by rho^2.
Vec csw_sound_speed(Sim& s, IArr* o[5], int X) {
    const double G = s.gamma;
    long long N = s.N;
    Vec snd[2];
    for (int q = 0; q < 2; ++q) {
        int n = q == 0 ? 1 : -1;
        Vec m0 = o[1]->shift(X, n), m1 = o[2]->shift(X, n), m2 = o[3]->shift(X, n), ms = o[0]->shift(X, n);
        Vec b0 = s.mg[0].cellMag.shift(X, n), b1 = s.mg[1].cellMag.shift(X, n), b2 = s.mg[2].cellMag.shift(X, n);
        Vec e = o[4]->shift(X, n), ms2 = o[0]->shift(X, n), ms3 = o[0]->shift(X, n);
        Vec out(N);
        for (long long i = 0; i < N; ++i) {
            double vsq = m0[i] * m0[i] + m1[i] * m1[i] + m2[i] * m2[i] / (ms[i] * ms[i]);
            double msq = b0[i] * b0[i] + b1[i] * b1[i] + b2[i] * b2[i];
            double r = (G - 1.0) * (e[i] - 0.5 * ms2[i] * vsq);
            r = r - (G - 1.0) * 0.5 * msq;
            out[i] = std::sqrt(std::fabs((G * r + 2.0 * msq) / ms3[i]));
        }
        snd[q] = std::move(out);
    }
    Vec res(N);
    for (long long i = 0; i < N; ++i) res[i] = std::fmax(std::fmin(snd[1][i], snd[0][i]), 0.0);
    return res;
}

// ArtificialViscosity.solve (ArtificialViscosity.m:66-148) for the stage objects o (mass, mom x3, ener).
Vec viscosity_solve(Sim& s, IArr* o[5], const Vec& sound, int X) {
    long long N = s.N;
    const double c1 = s.visc_lin, c2 = s.visc_quad, G = s.gamma;
    Vec out(N, 0.0);
    if (s.visc_type == 1) {   // neumannRichtmyerViscosity (:73-77)
        Vec p1 = o[X]->shift(X, 1);
        const Vec &px = o[X]->a, &rho = o[0]->a;
        for (long long i = 0; i < N; ++i) {
            double vm = std::fmin(p1[i] - px[i], 0.0);
            out[i] = vm * (c1 * sound[i] + c2 * vm / rho[i]);
        }
    } else if (s.visc_type == 2) {   // caramanaShashkovWhalenViscosity (:81-148)
        Vec mB = o[0]->shift(X, -1), mC = o[0]->shift(X, 1);
        Vec cs = csw_sound_speed(s, o, X);
        Vec pm2 = o[X]->shift(X, -2), rm2 = o[0]->shift(X, -2);
        Vec pm1 = o[X]->shift(X, -1), rm1 = o[0]->shift(X, -1);
        Vec pp1 = o[X]->shift(X, 1), rp1 = o[0]->shift(X, 1);
        Vec pp2 = o[X]->shift(X, 2), rp2 = o[0]->shift(X, 2);
        const double k1 = c2 * (G + 1), g4 = (G + 1) / 4, k2 = (c2 * c2) * (g4 * g4), k3 = c1 * c1;
        for (long long i = 0; i < N; ++i) {
            double rho = 2 * mC[i] * mB[i] / (mC[i] + mB[i]);
            double v0 = pm2[i] / rm2[i], v1 = pm1[i] / rm1[i], v2 = pp1[i] / rp1[i], v3 = pp2[i] / rp2[i];
            double dv = v2 - v1;
            double rL = (v3 - v2) / (2 * dv), rR = (v1 - v0) / (2 * dv);
            double lim = std::fmax(0.0, std::fmin(std::fmin(0.5 * (rL + rR), std::fmin(2 * rL, 2 * rR)), 1.0));
            double adv = std::fabs(dv);
            out[i] = (dv < 0 ? 1.0 : 0.0) * rho * (k1 * adv / 4 + std::sqrt(k2 * (dv * dv) + k3 * (cs[i] * cs[i]))) *
                     (1 - lim) * adv;
        }
    }
    return out;
}

// wFluidFlux.m:14-44 for the stage objects o (mass, mom x3, ener: primaries or stores)
void w_fluid_flux(Sim& s, IArr* o[5], int X, Vec& freeze, Vec w[5]) {
    int d = X - 1;
    long long N = s.N;
    const Vec* u[5] = {&o[0]->a, &o[1]->a, &o[2]->a, &o[3]->a, &o[4]->a};
    Vec press, sound;
    pressure(s, false, *u[0], *u[1], *u[2], *u[3], *u[4], press, &sound);
    Vec spd_line(s.face(d));
    long long sd = s.stride(d);
    int d1 = d == 0 ? 1 : 0, d2 = d == 2 ? 1 : 2;
    long long s1 = s.stride(d1), s2 = s.stride(d2);
    const Vec& mom_d = *u[1 + d];
    const Vec& rho = *u[0];
#pragma omp parallel for schedule(static)
    for (long long f = 0; f < s.face(d); ++f) {
        long long b = (f % s.n[d1]) * s1 + (f / s.n[d1]) * s2;
        double mx = std::numeric_limits<double>::quiet_NaN();
        for (int i = 0; i < s.n[d]; ++i) {
            long long q = b + i * sd;
            double v = std::fabs(mom_d[q] / rho[q]) + sound[q];
            if (std::isnan(mx) || v > mx) mx = std::isnan(v) ? mx : v;
        }
        spd_line[f] = mx;
    }
    freeze.assign(N, 0.0);
#pragma omp parallel for schedule(static)
    for (long long f = 0; f < s.face(d); ++f) {
        long long b = (f % s.n[d1]) * s1 + (f / s.n[d1]) * s2;
        for (int i = 0; i < s.n[d]; ++i) freeze[b + i * sd] = spd_line[f];
    }
    const Vec* cm[3] = {&s.mg[0].cellMag.a, &s.mg[1].cellMag.a, &s.mg[2].cellMag.a};
    for (int k = 0; k < 5; ++k) w[k].assign(N, 0.0);
    Vec visc = viscosity_solve(s, o, sound, X);   // wFluidFlux.m:24 (0 for the empty solver)
#pragma omp parallel for schedule(static)
    for (long long i = 0; i < N; ++i) {
        double fz = freeze[i];
        double velocity = mom_d[i] / rho[i];
        double press_i = press[i] + visc[i];
        double cx = (*cm[d])[i];
        w[0][i] = (*u[1 + d])[i] / fz;
        double we = velocity * ((*u[4])[i] + press_i) -
                    cx * ((*cm[0])[i] * (*u[1])[i] + (*cm[1])[i] * (*u[2])[i] + (*cm[2])[i] * (*u[3])[i]) / rho[i];
        w[4][i] = we / fz;
        for (int c = 0; c < 3; ++c) {
            double dirv = c == d ? 1.0 : 0.0;
            w[1 + c][i] = (velocity * (*u[1 + c])[i] + press_i * dirv - cx * (*cm[c])[i]) / fz;
        }
    }
}

// relaxingFluid.m:16-73
void relaxing_fluid(Sim& s, int X) {
    long long N = s.N;
    double ff = s.dt / s.dgrid[X - 1];
    Vec freeze, w[5];
    IArr* u[5] = {&s.fv[0].prim, &s.fv[1].prim, &s.fv[2].prim, &s.fv[3].prim, &s.fv[4].prim};
    w_fluid_flux(s, u, X, freeze, w);
    for (int k = 0; k < 5; ++k) {
        auto& v = s.fv[k];
        Vec R(N), L(N);
#pragma omp parallel for schedule(static)
        for (long long i = 0; i < N; ++i) {
            R[i] = 0.5 * (v.prim.a[i] + w[k][i]);
            L[i] = 0.5 * (v.prim.a[i] - w[k][i]);
        }
        v.store_fluxR.set(std::move(R));
        v.store_fluxL.set(std::move(L));
        Vec Rm = v.store_fluxR.shift(X, -1);
        Vec Lp = v.store_fluxL.shift(X, 1);
        Vec st(N);
        const Vec &Ra = v.store_fluxR.a, &La = v.store_fluxL.a;
#pragma omp parallel for schedule(static)
        for (long long i = 0; i < N; ++i)
            st[i] = v.prim.a[i] - 0.5 * ff * freeze[i] * (Ra[i] - Rm[i] + La[i] - Lp[i]);
        v.store.set(std::move(st));
        v.store_fluxR.cleanup();
        v.store_fluxL.cleanup();
    }
    {
        Vec m(N);
        for (long long i = 0; i < N; ++i) m[i] = std::fmax(s.fv[0].store.a[i], s.minmass);   // max ignores NaN
        s.fv[0].store.set(std::move(m));
    }
    IArr* us[5] = {&s.fv[0].store, &s.fv[1].store, &s.fv[2].store, &s.fv[3].store, &s.fv[4].store};
    w_fluid_flux(s, us, X, freeze, w);
    int lim = s.limiter[X - 1];
    for (int k = 0; k < 5; ++k) {
        auto& v = s.fv[k];
        Vec R(N), L(N);
#pragma omp parallel for schedule(static)
        for (long long i = 0; i < N; ++i) {
            R[i] = 0.5 * (v.store.a[i] + w[k][i]);
            L[i] = 0.5 * (v.store.a[i] - w[k][i]);
        }
        v.fluxR.set(std::move(R));
        v.fluxL.set(std::move(L));
        {
            Vec m1 = v.fluxR.shift(X, -1);
            Vec p1 = v.fluxR.shift(X, 1);
            Vec dL(N), dR(N);
            for (long long i = 0; i < N; ++i) { dL[i] = v.fluxR.a[i] - m1[i]; dR[i] = p1[i] - v.fluxR.a[i]; }
            apply_limiter(lim, v.fluxR, dL, dR);
        }
        {
            Vec m1 = v.fluxL.shift(X, -1);
            Vec p1 = v.fluxL.shift(X, 1);
            Vec dL(N), dR(N);
            for (long long i = 0; i < N; ++i) { dL[i] = m1[i] - v.fluxL.a[i]; dR[i] = v.fluxL.a[i] - p1[i]; }
            apply_limiter(lim, v.fluxL, dL, dR);
        }
        Vec Rm = v.fluxR.shift(X, -1);
        Vec Lp = v.fluxL.shift(X, 1);
        Vec nv(N);
        const Vec &Ra = v.fluxR.a, &La = v.fluxL.a;
#pragma omp parallel for schedule(static)
        for (long long i = 0; i < N; ++i)
            nv[i] = v.prim.a[i] - ff * freeze[i] * (Ra[i] - Rm[i] + La[i] - Lp[i]);
        v.prim.set(std::move(nv));
        v.fluxR.cleanup();
        v.fluxL.cleanup();
    }
    {
        Vec m(N);
        for (long long i = 0; i < N; ++i) m[i] = std::fmax(s.fv[0].prim.a[i], s.minmass);
        s.fv[0].prim.set(std::move(m));
    }
}

// relaxingMagnet.m:15-60
void relaxing_magnet(Sim& s, int X, int I, IArr& vg) {
    long long N = s.N;
    auto& m = s.mg[I - 1];
    double ff = 0.5 * s.dt / s.dgrid[X - 1];
    Vec vgp = vg.shift(X, 1);
    Vec vf(N);
    for (long long i = 0; i < N; ++i) vf[i] = (vg.a[i] + vgp[i]) < 0.0 ? 1.0 : 0.0;

    IArr& sfr = m.store_fluxR[X];
    {
        Vec F(N);
        for (long long i = 0; i < N; ++i) F[i] = m.prim.a[i] * vg.a[i];
        sfr.set(std::move(F));
        Vec Fp = sfr.shift(X, 1);
        Vec G(N);
        for (long long i = 0; i < N; ++i) G[i] = sfr.a[i] * (1 - vf[i]) + Fp[i] * vf[i];
        sfr.set(std::move(G));
        Vec Fm = sfr.shift(X, -1);
        Vec st(N);
        for (long long i = 0; i < N; ++i) st[i] = m.prim.a[i] - ff * (sfr.a[i] - Fm[i]);
        m.store[X].set(std::move(st));
    }
    ff = 2 * ff;
    IArr& wm = m.wMag[X];
    {
        Vec W(N);
        for (long long i = 0; i < N; ++i) W[i] = m.store[X].a[i] * vg.a[i];
        wm.set(std::move(W));
    }
    IArr& fx = m.flux[X];
    Vec dFluxR(N), dFluxL(N);
    {
        Vec Wp = wm.shift(X, 1);
        Vec F(N);
        for (long long i = 0; i < N; ++i) F[i] = wm.a[i] * (1 - vf[i]) + Wp[i] * vf[i];
        fx.set(std::move(F));
        Vec Wp1 = wm.shift(X, 1);
        Vec Wp2 = wm.shift(X, 2);
        for (long long i = 0; i < N; ++i) dFluxR[i] = Wp1[i] - (vf[i] * Wp2[i] + (1 - vf[i]) * wm.a[i]);
        Vec Wq1 = wm.shift(X, 1);
        Vec Wm1 = wm.shift(X, -1);
        for (long long i = 0; i < N; ++i) dFluxL[i] = wm.a[i] - (vf[i] * Wq1[i] + (1 - vf[i]) * Wm1[i]);
    }
    apply_limiter(s.limiter[X - 1], fx, dFluxL, dFluxR);
    {
        Vec Fm = fx.shift(X, -1);
        Vec B(N);
        for (long long i = 0; i < N; ++i) B[i] = m.prim.a[i] - ff * (fx.a[i] - Fm[i]);
        m.prim.set(std::move(B));
    }
    ff = s.dt / s.dgrid[I - 1];
    {
        Vec Fp = fx.shift(I, 1);
        Vec C(N);
        for (long long i = 0; i < N; ++i) C[i] = fx.a[i] - Fp[i];
        fx.set(std::move(C));
        Vec Cm = fx.shift(X, -1);
        fx.set(std::move(Cm));
        IArr& bx = s.mg[X - 1].prim;
        Vec B(N);
        for (long long i = 0; i < N; ++i) B[i] = bx.a[i] - ff * fx.a[i];
        bx.set(std::move(B));
    }
}

void update_cell_centered(Sim& s, int c) {   // MagnetArray.m:36-38
    auto& m = s.mg[c - 1];
    Vec sh = m.prim.shift(c, 1);
    Vec out(s.N);
    for (long long i = 0; i < s.N; ++i) out[i] = 0.5 * (m.prim.a[i] + sh[i]);
    m.cellMag.set(std::move(out));
}

// magnetFlux.m:14-31
void magnet_flux(Sim& s, int X, int I1, int I2) {
    long long N = s.N;
    int I = I1;
    for (int q = 0; q < 2; ++q) {
        I = q == 0 ? I1 : I2;
        auto& m = s.mg[I - 1];
        IArr& vg = m.velGrid[X];
        IArr& momX = s.fv[X].prim;
        IArr& mass = s.fv[0].prim;
        Vec pm = momX.shift(I, -1);
        Vec rm = mass.shift(I, -1);
        Vec v(N);
        for (long long i = 0; i < N; ++i) v[i] = (pm[i] + momX.a[i]) / (rm[i] + mass.a[i]);
        vg.set(std::move(v));
        Vec a = vg.shift(X, -1);
        Vec b = vg.shift(X, 1);
        Vec sm(N);
        for (long long i = 0; i < N; ++i) sm[i] = 0.25 * (a[i] + b[i] + 2 * vg.a[i]);
        vg.set(std::move(sm));
        relaxing_magnet(s, X, I, vg);
        vg.cleanup(); m.store[X].cleanup(); m.store_fluxR[X].cleanup(); m.wMag[X].cleanup(); m.flux[X].cleanup();
    }
    update_cell_centered(s, I);
    update_cell_centered(s, X);
}

// flux.m:17-62
void flux(Sim& s, int order) {
    int row = (s.iteration - 1) % 6;
    for (int q = 0; q < 3; ++q) {
        int X = order > 0 ? FWD[row][q] : BWD[row][q];
        if (s.n[X - 1] < 3) continue;
        if (order > 0) {
            if (s.fluid_active) relaxing_fluid(s, X);
            if (s.magnet_active) magnet_flux(s, X, FWD_MI[X - 1][0], FWD_MI[X - 1][1]);
        } else {
            if (s.magnet_active) magnet_flux(s, X, BWD_MI[X - 1][0], BWD_MI[X - 1][1]);
            if (s.fluid_active) relaxing_fluid(s, X);
        }
    }
}

// TimeManager.update (TimeManager.m:55-99); returns 0 or -1 on a CFL error
int time_update(Sim& s, int flux_direction) {
    if (flux_direction > 1 && s.update_mode != 0) return 0;
    double cmax = 1e-2;
    int gi = 0;
    Vec snd;
    pressure(s, true, s.fv[0].prim.a, s.fv[1].prim.a, s.fv[2].prim.a, s.fv[3].prim.a, s.fv[4].prim.a, snd, nullptr);
    for (int i = 0; i < 3; ++i) {
        const Vec& p = s.fv[1 + i].prim.a;
        const Vec& r = s.fv[0].prim.a;
        double c = std::numeric_limits<double>::quiet_NaN();
        for (long long k = 0; k < s.N; ++k) {
            double v = std::fabs(p[k] / r[k]) + snd[k];
            if (!std::isnan(v) && (std::isnan(c) || v > c)) c = v;
        }
        if (c > cmax) { cmax = c; gi = i + 1; }
    }
    s.last_cmax = cmax;
    s.last_grid_index = gi;
    if (gi < 1) return -1;
    s.dt = s.cfl * s.dgrid[gi - 1] / cmax;
    double nt = s.time + (s.update_mode + 1) * s.dt;
    if (nt > s.time_max) {
        s.dt = (s.time_max - s.time) / (s.update_mode + 1);
        nt = s.time_max;
    }
    s.time = nt;
    return 0;
}

bool running(const Sim& s) { return s.iteration <= s.iter_max && s.time < s.time_max; }

// source.m:30 (the radiation sink; gravity is not part of this path)
void source(Sim& s) {
    if (s.rad_type != 1) return;   // the empty solver gives 0
    Vec r = radiation_solve(s);
    Vec e(s.N);
    for (long long k = 0; k < s.N; ++k) e[k] = s.fv[4].prim.a[k] - s.dt * r[k];
    s.fv[4].prim.set(std::move(e));
}

// treadmillGrid (treadmill/treadmillGrid.m:14-37): from iteration 10 on, newIndex = round(mean(mean(
// first index of the largest forward difference of rho along DIRECTION, per pencil))); the first call
// records it as `last`, later calls shift every primary by newIndex - last cells with its own BCs.
void treadmill(Sim& s) {
    const int X = s.treadmill_dir;
    if (X <= 0 || s.iteration < 10) return;
    const int d = X - 1;
    IArr& mass = s.fv[0].prim;
    const Vec sh = mass.shift(X, 1);   // calculate2PtDerivative (ImogenArray.m:190-192)
    const int d1 = d == 0 ? 1 : 0, d2 = d == 2 ? 1 : 2;
    const int n1 = s.n[d1], n2 = s.n[d2], Nd = s.n[d];
    const long long sd = s.stride(d), s1 = s.stride(d1), s2 = s.stride(d2);
    std::vector<double> idx((size_t)n1 * n2);
    for (int c2 = 0; c2 < n2; ++c2)
        for (int c1 = 0; c1 < n1; ++c1) {
            const long long b = c1 * s1 + c2 * s2;
            double best = -HUGE_VAL;
            int bi = 0;
            for (int i = 0; i < Nd; ++i) {   // max(..., [], X): first maximum, NaN skipped
                const double v = (sh[b + i * sd] - mass.a[b + i * sd]) / s.dgrid[d];
                if (v > best) { best = v; bi = i; }
            }
            idx[c1 + (size_t)n1 * c2] = bi + 1;
        }
    // mean(mean(.)): along the first non-singleton remaining dimension, then along the other
    std::vector<double> first;
    if (n1 > 1 && n2 > 1) {
        for (int c2 = 0; c2 < n2; ++c2) {
            double t = 0;
            for (int c1 = 0; c1 < n1; ++c1) t += idx[c1 + (size_t)n1 * c2];
            first.push_back(t / n1);
        }
    } else {
        first = idx;
    }
    double t = 0;
    for (double v : first) t += v;
    const int new_index = (int)std::round(t / (double)first.size());
    if (s.treadmill_last < 0) {
        s.treadmill_last = new_index;
        return;
    }
    const int dc = new_index - s.treadmill_last;
    s.fv[0].prim.set(s.fv[0].prim.shift(X, dc));
    s.fv[4].prim.set(s.fv[4].prim.shift(X, dc));
    for (int i = 0; i < 3; ++i) {
        s.fv[1 + i].prim.set(s.fv[1 + i].prim.shift(X, dc));
        s.mg[i].prim.set(s.mg[i].prim.shift(X, dc));
    }
    s.treadmill_history.push_back(dc);
}

int iterate(Sim& s) {
    for (int i = 1; i <= 2; ++i) {
        if (time_update(s, i) != 0) return -1;
        flux(s, i == 1 ? 1 : -1);
        treadmill(s);
        source(s);
    }
    s.iteration += 1;
    return 0;
}

}  // namespace

extern "C" {

void* orc_create(const int grid[3], const double dgrid[3], double gamma, double cfl, double minmass,
                 const int* bc /*[4][2][3]*/, int bc_infinity, const int limiter[3], int fluid_active,
                 int magnet_active, double time_max, int iter_max, int update_mode) {
    auto* s = new Sim();
    for (int d = 0; d < 3; ++d) { s->n[d] = grid[d]; s->dgrid[d] = dgrid[d]; s->limiter[d] = limiter[d]; }
    s->N = (long long)grid[0] * grid[1] * grid[2];
    s->ndims = grid[2] > 1 ? 3 : 2;
    s->gamma = gamma; s->cfl = cfl; s->minmass = minmass;
    std::memcpy(s->bc, bc, sizeof(s->bc));
    s->bc_inf = bc_infinity;
    {
        int f = bc_infinity;
        double xk[5] = {0, std::ceil(f / 4.0), std::floor(f / 2.0 + 0.5), double(f - 1), double(f)};
        double yk[5] = {1, 1, 0.01, 0, 0};
        std::vector<double> xi(f);
        for (int i = 0; i < f; ++i) xi[i] = i + 1;
        s->fade_coeff.assign(f, 0.0);
        pchip_col(xk, 5, yk, xi.data(), f, s->fade_coeff.data());
    }
    // mirror_shift.m:31-33 and fade_shift.m:34-44 / Edges.m:80-93 index outside short dimensions:
    // the reference stops there, so such settings are rejected.
    for (int c = 0; c < 4; ++c)
        for (int side = 0; side < 2; ++side)
            for (int d = 0; d < s->ndims; ++d) {
                int mode = s->bc[c][side][d];
                // linear_shift.m:20 indexes with the undefined variable `dim` (the reference errors at the
                // first shift); wormhole_shift.m:27-33 indexes a third dimension (2-D grids error at the
                // first lower shift)
                bool bad = mode < 0 || mode > 9 || (mode == MIRROR && grid[d] < 2) ||
                           (mode == FADE && grid[d] < std::max(20, bc_infinity)) || mode == LINEAR ||
                           (mode == WORMHOLE && side == 0 && s->ndims < 3);
                if (bad) { delete s; return nullptr; }
            }
    s->fluid_active = fluid_active != 0;
    s->magnet_active = magnet_active != 0;
    s->time_max = time_max; s->iter_max = iter_max; s->update_mode = update_mode;
    const int cls[5] = {C_MASS, C_MOM, C_MOM, C_MOM, C_ENER};
    const int comp[5] = {0, 1, 2, 3, 0};
    for (int k = 0; k < 5; ++k) {
        auto& v = s->fv[k];
        for (IArr* A : {&v.prim, &v.store, &v.store_fluxR, &v.store_fluxL, &v.fluxR, &v.fluxL})
            s->init_arr(*A, comp[k], cls[k]);
        v.store_fluxR.ftype = v.fluxR.ftype = FT_FLUXR;   // StorageArray.m:69-70, FluidArray.m:104-105
        v.store_fluxL.ftype = v.fluxL.ftype = FT_FLUXL;
    }
    for (int c = 0; c < 3; ++c) {
        auto& m = s->mg[c];
        s->init_arr(m.prim, c + 1, C_MAG);
        s->init_arr(m.cellMag, c + 1, C_MAG);
        for (int X = 1; X <= 3; ++X) {
            for (IArr* A : {&m.velGrid[X], &m.store[X], &m.store_fluxR[X], &m.wMag[X], &m.flux[X]})
                s->init_arr(*A, c + 1, C_MAG);
            m.store_fluxR[X].ftype = FT_FLUXR;   // the store's fluxR (StorageArray.m:70)
            m.flux[X].ftype = FT_FLUX;           // MagnetArray.m:96: fluxType 'flux'
        }
    }
    return s;
}

void orc_destroy(void* p) { delete static_cast<Sim*>(p); }

// Artificial viscosity and radiation settings (before orc_set_state, which initialises the radiation).
void orc_set_physics(void* p, int visc_type, double visc_lin, double visc_quad, int rad_type, double rad_exp,
                     double rad_initmax) {
    Sim& s = *static_cast<Sim*>(p);
    s.visc_type = visc_type;
    s.visc_lin = visc_lin;
    s.visc_quad = visc_quad;
    s.rad_type = rad_type;
    s.rad_exp = rad_exp;
    s.rad_initmax = rad_initmax;
}

int orc_set_state(void* p, const double* mass, const double* mom, const double* ener, const double* mag) {
    Sim& s = *static_cast<Sim*>(p);
    long long N = s.N;
    for (int k = 0; k < 5; ++k) s.fv[k].prim.fades = nullptr;   // the initial assignment is not faded
    s.fv[0].prim.set(Vec(mass, mass + N));
    for (int c = 0; c < 3; ++c) s.fv[1 + c].prim.set(Vec(mom + c * N, mom + (c + 1) * N));
    s.fv[4].prim.set(Vec(ener, ener + N));
    for (int c = 0; c < 3; ++c) {
        s.mg[c].prim.set(Vec(mag + c * N, mag + (c + 1) * N));
        update_cell_centered(s, c + 1);
    }
    for (int c = 0; c < 3; ++c) {
        double sum = 0;
        for (long long i = 0; i < N; ++i) sum += s.mg[c].prim.a[i];
        s.mg[c].isZero = (sum == 0) && !s.magnet_active;
    }
    if (!s.fade_arr.empty()) {   // FluidArray.readFades after the initial assignment (FluidArray.m:54)
        const int bit[5] = {1, 2, 2, 2, 4};
        for (int k = 0; k < 5; ++k)
            if (s.fade_mask & bit[k]) s.fv[k].prim.fades = &s.fade_arr;
    }
    radiation_initialize(s);   // ImogenManager.initialize (imogen.m:46)
    return 0;
}

// PointFade(grid, location, fadeSize).array (classes/PointFade.m:29-38) and the variables it acts on.
void orc_set_fade(void* p, const int location[3], double fade_size, int mask) {
    Sim& s = *static_cast<Sim*>(p);
    s.fade_mask = mask;
    s.fade_arr.assign(s.N, 0.0);
    Vec d(s.N);
    double mx = -HUGE_VAL;
    for (long long c = 0; c < s.N; ++c) {
        const double x = (double)(c % s.n[0]) + 1 - location[0];
        const double y = (double)((c / s.n[0]) % s.n[1]) + 1 - location[1];
        const double z = (double)(c / ((long long)s.n[0] * s.n[1])) + 1 - location[2];
        d[c] = std::max(fade_size * fade_size - (x * x + y * y + z * z), 0.0);
        mx = std::max(mx, d[c]);
    }
    for (long long c = 0; c < s.N; ++c) d[c] = 1 - d[c] / mx;
    const double xk[4] = {-1, 0, 1, 2}, yk[4] = {1, 1, 0, 0};
    pchip_col(xk, 4, yk, d.data(), (int)s.N, s.fade_arr.data());
}

int orc_get_state(void* p, double* mass, double* mom, double* ener, double* mag, double* cellmag) {
    Sim& s = *static_cast<Sim*>(p);
    long long N = s.N;
    if (mass) std::copy(s.fv[0].prim.a.begin(), s.fv[0].prim.a.end(), mass);
    if (ener) std::copy(s.fv[4].prim.a.begin(), s.fv[4].prim.a.end(), ener);
    for (int c = 0; c < 3; ++c) {
        if (mom) std::copy(s.fv[1 + c].prim.a.begin(), s.fv[1 + c].prim.a.end(), mom + c * N);
        if (mag) std::copy(s.mg[c].prim.a.begin(), s.mg[c].prim.a.end(), mag + c * N);
        if (cellmag) std::copy(s.mg[c].cellMag.a.begin(), s.mg[c].cellMag.a.end(), cellmag + c * N);
    }
    return 0;
}

int orc_time_update(void* p, int flux_direction) { return time_update(*static_cast<Sim*>(p), flux_direction); }
int orc_flux(void* p, int order) { flux(*static_cast<Sim*>(p), order); return 0; }
int orc_relaxing_fluid(void* p, int X) { relaxing_fluid(*static_cast<Sim*>(p), X); return 0; }
int orc_magnet_flux(void* p, int X, int I1, int I2) { magnet_flux(*static_cast<Sim*>(p), X, I1, I2); return 0; }
int orc_iterate(void* p) { return iterate(*static_cast<Sim*>(p)); }
void orc_source(void* p) { source(*static_cast<Sim*>(p)); }
void orc_treadmill(void* p) { treadmill(*static_cast<Sim*>(p)); }
void orc_set_treadmill(void* p, int direction) { static_cast<Sim*>(p)->treadmill_dir = direction; }
int orc_treadmill_history(void* p, int* out, int cap) {
    const auto& h = static_cast<Sim*>(p)->treadmill_history;
    for (int i = 0; i < cap && i < (int)h.size(); ++i) out[i] = h[i];
    return (int)h.size();
}
int orc_treadmill_last(void* p) { return static_cast<Sim*>(p)->treadmill_last; }
double orc_radiation_strength(void* p) { return static_cast<Sim*>(p)->rad_strength; }

int orc_run(void* p, int max_iterations) {
    Sim& s = *static_cast<Sim*>(p);
    int n = 0;
    while (running(s) && (max_iterations < 0 || n < max_iterations)) {
        if (iterate(s) != 0) return -1 - n;
        ++n;
    }
    return n;
}

void orc_get_time(void* p, double* time, double* dt, int* iteration) {
    Sim& s = *static_cast<Sim*>(p);
    if (time) *time = s.time;
    if (dt) *dt = s.dt;
    if (iteration) *iteration = s.iteration;
}

void orc_set_time(void* p, double time, double dt, int iteration) {
    Sim& s = *static_cast<Sim*>(p);
    s.time = time; s.dt = dt; s.iteration = iteration;
}

void orc_get_cfl(void* p, double* cmax, int* grid_index) {
    Sim& s = *static_cast<Sim*>(p);
    *cmax = s.last_cmax; *grid_index = s.last_grid_index;
}

// directVec of flux.m:17-27 for an iteration (1-based) and order (+1 forward, -1 backward).
void orc_sweep_order(int order, int iteration, int out[3]) {
    const int row = (iteration - 1) % 6;
    for (int q = 0; q < 3; ++q) out[q] = order > 0 ? FWD[row][q] : BWD[row][q];
}

int orc_pchip(const double* x, int n, const double* y, int ncols, const double* xi, int m, double* out) {
    for (int c = 0; c < ncols; ++c) pchip_col(x, n, y + (long long)c * n, xi, m, out + (long long)c * m);
    return 0;
}

void orc_set_threads(int t) {
#ifdef _OPENMP
    if (t > 0) omp_set_num_threads(t);
#else
    (void)t;
#endif
}

int orc_max_threads() {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

}  // extern "C"
