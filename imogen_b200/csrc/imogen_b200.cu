// Host side of the imogen_b200 C ABI: context, resident state, launch sequencing.
//
// A context owns one grid's state on the device (eleven SoA arrays), its stored edges, scratch for
// the magnet passes and a device-resident TimeManager.  flux()/step() only enqueue kernels on the
// context's stream; the timestep is computed and consumed on the device, so a whole iteration runs
// without a host round trip (and is captured once into a CUDA graph per sweep-order row).
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <functional>
#include <thread>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <ctime>
#include <map>
#include <mutex>
#include <tuple>
#include <string>
#include <vector>

#include "../../include/imogen_b200.h"
#include "cfl.cuh"
#include "treadmill.cuh"

using namespace img;

namespace {

// flux.m:17-27 -- sweep order rows: FWD = perms([1 2 3]), BWD = perms([3 2 1]) as MATLAB
// R2009a-R2010b returns them.  That perms permutes positions and then indexes V (perms(V) = V(P)),
// with P = perms(1:3) = 321, 312, 231, 213, 123, 132 (its recursive relabelling leaves the last two
// rows out of reverse-lexicographic order); so BWD = 4 - FWD, row by row.
const int FWD[6][3] = {{3, 2, 1}, {3, 1, 2}, {2, 3, 1}, {2, 1, 3}, {1, 2, 3}, {1, 3, 2}};
const int BWD[6][3] = {{1, 2, 3}, {1, 3, 2}, {2, 1, 3}, {2, 3, 1}, {3, 2, 1}, {3, 1, 2}};
const int FWD_MI[3][2] = {{2, 3}, {1, 3}, {1, 2}};
const int BWD_MI[3][2] = {{3, 2}, {3, 1}, {2, 1}};

// Launch shape of the pencil kernels for one sweep direction: Wb pencils per CTA, G threads per
// pencil, CPT cells per thread (2, or 4 for long pencils), CL CTAs per cluster.
struct PencilCfg {
    int Wb = 1, G = 32, CL = 1, NT = 32, cpt = 2;
    int nqc = 1;   // magnet chain: transverse components per CTA
    int seg = 0;   // fluid sweep: segment kernel with seg = cpt consecutive cells per thread (G = N / cpt)
};

size_t align256(size_t b) { return (b + 255) & ~size_t(255); }

int pow2ceil(long long v) {
    int p = 1;
    while (p < v) p <<= 1;
    return p;
}

// A small process-wide pool of host threads for the FP64 <-> FP32 conversions of the mixed form's
// host transfers.  run(n, fn) calls fn(0..n-1) on the pool and the calling thread and returns when
// all calls have returned.  Idle workers spin for a short while (transfers come in bursts of calls
// tens of microseconds apart) and then sleep.  One run at a time (callers are serialised).
class HostPool {
  public:
    static HostPool& get() {
        static HostPool* pool = new HostPool();   // never destroyed: workers may sleep at exit
        return *pool;
    }
    int threads() const { return (int)workers_.size() + 1; }
    void run(int n, const std::function<void(int)>& fn) {
        std::lock_guard<std::mutex> serial(run_mu_);
        if (n <= 0) return;
        {
            std::lock_guard<std::mutex> lock(mu_);
            job_.store(&fn);
            total_.store(n);
            next_.store(0);
            finished_.store(0);
            gen_.fetch_add(1);
        }
        cv_.notify_all();
        work();
        while (finished_.load() < n) std::this_thread::yield();
        std::lock_guard<std::mutex> lock(mu_);
        job_.store(nullptr);
    }

  private:
    HostPool() {
        const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
        const int nw = (int)std::min(7u, hw / 2);
        for (int i = 0; i < nw; ++i) workers_.emplace_back([this] { loop(); });
        for (auto& t : workers_) t.detach();
    }
    void work() {
        for (int i; (i = next_.fetch_add(1)) < total_.load();) {
            (*job_.load())(i);
            finished_.fetch_add(1);
        }
    }
    void loop() {
        unsigned long long seen = 0;
        for (;;) {
            const auto t0 = std::chrono::steady_clock::now();
            while (gen_.load() == seen && std::chrono::steady_clock::now() - t0 < std::chrono::microseconds(500))
                std::this_thread::yield();
            if (gen_.load() == seen) {
                std::unique_lock<std::mutex> lock(mu_);
                cv_.wait(lock, [&] { return gen_.load() != seen; });
            }
            std::unique_lock<std::mutex> lock(mu_);
            seen = gen_.load();
            if (!job_.load()) continue;
            lock.unlock();
            work();
        }
    }
    std::vector<std::thread> workers_;
    std::mutex mu_, run_mu_;
    std::condition_variable cv_;
    std::atomic<const std::function<void(int)>*> job_{nullptr};
    std::atomic<int> total_{0}, next_{0}, finished_{0};
    std::atomic<unsigned long long> gen_{0};
};

}  // namespace

// One kernel launch of a context, recorded instead of issued while the context steps as a member of
// a batch (img_batch_*): the batch replays the records of all members as batched launches.
enum OpKind { OP_FLUID, OP_CHAIN, OP_CTCELL, OP_CFL_REDUCE, OP_CFL_FINALIZE };
inline bool pencil_kind(int kind) { return kind == OP_FLUID || kind == OP_CHAIN || kind == OP_CTCELL; }
struct OpRec {
    int kind;
    int elem;                 // 4 (mixed) or 8 (FP64)
    bool mhd;                 // fluid: MHD variant
    PencilLaunch L;           // pencil kernels: this member's launch shape
    unsigned blocks;          // pointwise kernels: this member's block count
    FluidArgs fa;
    MagArgs ma;
    CflArgs ca;
    DevTime* tm;              // cfl finalize
    int check_running;
};

struct img_batch;

struct img_ctx {
    img_config cfg{};
    std::string err;
    int dev = 0;
    size_t elem = 8;            // bytes per state value (8 FP64, 4 mixed)
    Geom g{};
    cudaStream_t stream = nullptr;
    void* slab = nullptr;       // one allocation: state, scratch, edges, tables
    size_t slab_bytes = 0;
    void* q[NQ] = {};
    void* scratch[2] = {};      // F0, F1 (limited fluxes of the magnet chain)
    DevTime* tm = nullptr;
    EdgeTable* edges_dev = nullptr;
    EdgeTable edges_host{};
    double* fade_dev = nullptr;
    double* partial = nullptr;  // totals partials
    int* tread_idx = nullptr;       // treadmill: per-pencil maximum index, first means, history
    double* tread_means = nullptr;
    int* tread_hist = nullptr;
    double* dt_hist = nullptr;      // TimeManager.history (DevTime::dt_hist points here)
    void* fade_map = nullptr;       // PointFade map (T per cell) when a point fade acts on a fluid primary
    int fade_mask = 0;              // IMG_FADE_MASS | MOM | ENER bits in effect
    bool constructing = false;      // img_set_state's uploads (the initial assignment is not faded)
    std::time_t created = 0;        // TimeManager.startTime
    double* stage = nullptr;    // mixed form: FP64 staging buffer of one array for host transfers
    std::vector<double> fade_host;
    int use_b[3] = {1, 1, 1};
    int mhd = 0;
    bool state_set = false;
    bool init_store = true, init_flux = true;   // fluid objects not yet assigned
    bool init_mag[3][3] = {{true, true, true}, {true, true, true}, {true, true, true}};
    bool cfl_valid = false;     // DevTime.maxbits hold the CFL maxima of the current state
    bool pad_cfl = false;       // batch recording: an empty CFL pass where another member needs one
    int iteration = 1;
    int iters_base = 0;
    PencilCfg pcfg[3][3];        // pencil tiling per kernel (0 fluid sweep, 1 magnet chain, 2 magnet CT) and
                                 // direction; the public magnet tiling sets 1 and 2, the autotuner tunes 2 alone
    PencilCfg pcfg_tile[3];      // fluid sweep per direction: the tile-kernel tiling of the launches that the
                                 // segment kernel does not take (stored-edge capture, fade, other ends)
    PencilCfg pcfg_mtile[2][3];  // the same for the magnet chain [0] and CT pass [1] (window kernels)
    // one captured iteration per (cfl_valid at its start, sweep-order row (iteration-1) % 6)
    cudaGraphExec_t graphs[2][6] = {};
    uint64_t graph_launches[2][6] = {};
    bool use_graphs = true;
    DevTime* host_tm = nullptr;  // pinned mirror
    uint64_t launches = 0;       // kernels launched by this context
    cudaStream_t own_stream = nullptr;   // the context's stream (stream is the batch's while a member)
    // mixed form: bulk host transfers in FP32 (copies on xfer_stream, FP64<->FP32 conversions on the
    // host); created at the first bulk transfer
    cudaStream_t xfer_stream = nullptr;
    cudaEvent_t xfer_ev[5] = {};         // [2,3] copy from / to host buffer b done, [4] stream fence
    float* h32 = nullptr;                // two pinned FP32 host buffers of one array each
    img_batch* batch = nullptr;          // batch this context is a member of
    std::vector<OpRec>* rec = nullptr;   // set while the batch records this member's launches
};

namespace {

thread_local std::string g_create_err;

int fail(img_ctx* c, int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    if (c) c->err = buf;
    else g_create_err = buf;
    return code;
}

#define CK(call)                                                                                   \
    do {                                                                                           \
        cudaError_t e_ = (call);                                                                   \
        if (e_ != cudaSuccess) return fail(ctx, IMG_ERR_CUDA, "%s: %s", #call, cudaGetErrorString(e_)); \
    } while (0)

bool active_lin(const img_config& c, int ndims, int cls, int DIRECT) {
    // Edges.ACTIVE(DIRECT) read with a linear index into the 2x3 (side x dim) matrix
    // (transparent_shift.m:42,74): element (side, dim) = ((DIRECT-1) % 2, (DIRECT-1) / 2).
    int side = (DIRECT - 1) % 2, dim = (DIRECT - 1) / 2;
    if (dim >= ndims) return false;
    int m = c.bc_modes[cls][side][dim];
    return m == IMG_BC_TRANS || m == IMG_BC_WALL || m == IMG_BC_FADE;
}

bool stateful(int m) { return m == IMG_BC_TRANS || m == IMG_BC_WALL; }

int obj_class(int o) {
    if (o == OBJ_PRIM_ENER) return CLS_ENER;
    if (o < OBJ_PRIM_MASS) {
        const int cls_of[5] = {CLS_MASS, CLS_MOM, CLS_MOM, CLS_MOM, CLS_ENER};
        return cls_of[(o - OBJ_FLUID) / 4];
    }
    if (o == OBJ_PRIM_MASS) return CLS_MASS;
    if (o < OBJ_PRIM_MAG) return CLS_MOM;
    return CLS_MAG;
}

bool obj_used(const img_config& c, int o) {
    if (o == OBJ_PRIM_ENER) return c.treadmill > 0;   // only treadmillGrid shifts the energy primary
    if (o < OBJ_PRIM_MASS) return c.fluid_active != 0;
    if (o < OBJ_MAG) return true;
    int r = (o - OBJ_MAG) / 4;
    int comp = r / 3, X = r % 3;
    return c.magnet_active && comp != X;
}

// MATLAB pchip on 5 knots (host copy for the fade coefficients of fade_shift.m:31).
// MATLAB pchip(xk, yk, x) (Moler's pchiptx: harmonic-mean interior slopes, one-sided end slopes)
// for a few knots, evaluated at one point (host; the point-fade map).
double pchip_host(const double* xk, const double* yk, int n, double x) {
    std::vector<double> h(n - 1), del(n - 1), d(n);
    auto sg = [](double v) { return v > 0 ? 1.0 : (v < 0 ? -1.0 : 0.0); };
    for (int k = 0; k < n - 1; ++k) { h[k] = xk[k + 1] - xk[k]; del[k] = (yk[k + 1] - yk[k]) / h[k]; }
    for (int k = 1; k < n - 1; ++k) {
        double w1 = 2 * h[k] + h[k - 1], w2 = h[k] + 2 * h[k - 1];
        d[k] = sg(del[k - 1]) * sg(del[k]) > 0 ? (w1 + w2) / (w1 / del[k - 1] + w2 / del[k]) : 0.0;
    }
    auto endslope = [&](double h0, double h1, double d0, double d1) {
        double dd = ((2 * h0 + h1) * d0 - h0 * d1) / (h0 + h1);
        if (sg(dd) != sg(d0)) dd = 0.0;
        else if (sg(d0) != sg(d1) && std::fabs(dd) > std::fabs(3 * d0)) dd = 3 * d0;
        return dd;
    };
    d[0] = endslope(h[0], h[1], del[0], del[1]);
    d[n - 1] = endslope(h[n - 2], h[n - 3], del[n - 2], del[n - 3]);
    int k = 0;
    for (int q = 0; q < n; ++q)
        if (xk[q] <= x) k = q;
    k = std::min(k, n - 2);
    const double s = x - xk[k];
    const double c1 = (d[k] + d[k + 1] - 2 * del[k]) / (h[k] * h[k]);
    const double c2 = (3 * del[k] - 2 * d[k] - d[k + 1]) / h[k];
    return ((c1 * s + c2) * s + d[k]) * s + yk[k];
}

// PointFade(grid, location, fadeSize).array (classes/PointFade.m:29-38): with r the offset of a cell from
// the 1-based location, dist = max(s^2 - |r|^2, 0), the map is pchip([-1 0 1 2], [1 1 0 0], 1 - dist/max).
std::vector<double> point_fade_map(const img_config& c) {
    const long long n = (long long)c.grid[0] * c.grid[1] * c.grid[2];
    std::vector<double> d(n), out(n);
    double mx = -HUGE_VAL;
    const double s = c.fade_size;
    for (long long i = 0; i < n; ++i) {
        const double x = (double)(i % c.grid[0]) + 1 - c.fade_location[0];
        const double y = (double)((i / c.grid[0]) % c.grid[1]) + 1 - c.fade_location[1];
        const double z = (double)(i / ((long long)c.grid[0] * c.grid[1])) + 1 - c.fade_location[2];
        d[i] = std::max(s * s - (x * x + y * y + z * z), 0.0);
        mx = std::max(mx, d[i]);
    }
    const double xk[4] = {-1, 0, 1, 2}, yk[4] = {1, 1, 0, 0};
    for (long long i = 0; i < n; ++i) out[i] = pchip_host(xk, yk, 4, 1 - d[i] / mx);
    return out;
}

std::vector<double> fade_coefficients(int f) {
    double xk[5] = {0, std::ceil(f / 4.0), std::floor(f / 2.0 + 0.5), double(f - 1), double(f)};
    double yk[5] = {1, 1, 0.01, 0, 0};
    double h[4], del[4], d[5];
    auto sg = [](double v) { return v > 0 ? 1.0 : (v < 0 ? -1.0 : 0.0); };
    for (int k = 0; k < 4; ++k) { h[k] = xk[k + 1] - xk[k]; del[k] = (yk[k + 1] - yk[k]) / h[k]; }
    for (int k = 1; k < 4; ++k) {
        double w1 = 2 * h[k] + h[k - 1], w2 = h[k] + 2 * h[k - 1];
        d[k] = sg(del[k - 1]) * sg(del[k]) > 0 ? (w1 + w2) / (w1 / del[k - 1] + w2 / del[k]) : 0.0;
    }
    auto endslope = [&](double h0, double h1, double d0, double d1) {
        double dd = ((2 * h0 + h1) * d0 - h0 * d1) / (h0 + h1);
        if (sg(dd) != sg(d0)) dd = 0.0;
        else if (sg(d0) != sg(d1) && std::fabs(dd) > std::fabs(3 * d0)) dd = 3 * d0;
        return dd;
    };
    d[0] = endslope(h[0], h[1], del[0], del[1]);
    d[4] = endslope(h[3], h[2], del[3], del[2]);
    std::vector<double> out(f);
    for (int j = 0; j < f; ++j) {
        double xv = j + 1;
        int k = 0;
        for (int q = 0; q < 5; ++q)
            if (xk[q] <= xv) k = q;
        k = std::min(k, 3);
        double s = xv - xk[k];
        double c1 = (d[k] + d[k + 1] - 2 * del[k]) / (h[k] * h[k]);
        double c2 = (3 * del[k] - 2 * d[k] - d[k + 1]) / h[k];
        out[j] = ((c1 * s + c2) * s + d[k]) * s + yk[k];
    }
    return out;
}

// Dynamic shared memory per CTA the pencil kernels may use (the opt-in 227 KB, less a margin for
// their static shared memory).
constexpr size_t kPencilSmemLimit = 210 * 1024;
constexpr int kTreadHistCap = 1 << 16;   // treadmill history entries kept on the device
constexpr int kDtHistCap = 1 << 16;      // TimeManager.history entries kept on the device
int dt_hist_cap(const img_config& c) { return std::max(1, std::min(c.iter_max, kDtHistCap)); }

bool tiling_fits(const PencilCfg& p, size_t elem) {
    return (elem == 8 ? fluid_smem_bytes<double>(p.G * p.cpt, p.Wb) : fluid_smem_bytes<float>(p.G * p.cpt, p.Wb)) <=
           kPencilSmemLimit;
}

// Every pencil tiling the kernels accept for direction d (the autotuner's search space): one, two
// or four cells per thread; along x whole-pencil CTAs of up to 256 or 512 threads; along y and z
// 2, 4 or 8 pencils per CTA, or for pencils of at most 16 cells 32..512/G pencils; at most 4 CTAs
// per cluster, and one CTA when pencils sit 32 or more side by side.
std::vector<PencilCfg> pencil_candidates(const Geom& g, int d, size_t elem) {
    const int N = g.n[d];
    const long long ncol = g.ncell / N;
    std::vector<PencilCfg> out;
    auto add1 = [&](int Wb, int G, int CL, int cpt) {
        PencilCfg p;
        p.Wb = Wb;
        p.G = G;
        p.CL = CL;
        p.NT = Wb * G;
        p.cpt = cpt;
        if (CL > 4 || p.NT < 32 || p.NT > 512 || p.NT % 32 || G < 2) return;
        if ((long long)G * cpt * CL < N) return;
        if (d != 0 && Wb >= 32 && CL > 1) return;                 // side-by-side pencils: one CTA
        if (d == 0 && G <= 32 && CL > 1) return;                  // in-warp pencils: one CTA
        if (!tiling_fits(p, elem)) return;
        for (const PencilCfg& q : out)
            if (q.Wb == Wb && q.G == G && q.CL == CL && q.cpt == cpt) return;
        out.push_back(p);
    };
    // each shape also with its pencil spread over twice and four times as many CTAs (less shared
    // memory per CTA, for long FP64 pencils)
    auto add = [&](int Wb, int G, int CL, int cpt) {
        for (; CL <= 4; CL *= 2, G /= 2) {
            add1(Wb, G, CL, cpt);
            const int h = G / 2;
            if (G % 2 || h < 2 || (d == 0 && (h % 32 || h <= 32)) || (d != 0 && (Wb * h) % 32)) break;
        }
    };
    auto up = [](int v, int m) { return (v + m - 1) / m * m; };
    for (int cpt : {1, 2, 4}) {
        const int rows = (N + cpt - 1) / cpt;
        const int G0 = std::max(2, pow2ceil(rows));
        if (d == 0) {
            for (int maxnt : {256, 512}) {
                int G = G0, CL = 1;
                while (G > maxnt) { G >>= 1; CL <<= 1; }
                int Wb = std::max(1, maxnt / G);
                while (Wb > 1 && (long long)Wb / 2 >= ncol && Wb * G > 32) Wb >>= 1;
                if (G > 32 && Wb > 8) continue;   // pencils spanning warps: at most 8 per CTA
                add(Wb, G, CL, cpt);
                // whole warps per pencil without the power-of-two padding (G a multiple of 32)
                if (G > 32) {
                    const int Gt = up((rows + CL - 1) / CL, 32);
                    if (Gt < G) add(Wb, Gt, CL, cpt);
                }
            }
        } else {
            for (int Wb : {2, 4, 8}) {
                int G = std::max(G0, 32 / Wb), CL = 1;
                while (Wb * G > 512) { G >>= 1; CL <<= 1; }
                add(Wb, G, CL, cpt);
                const int Gt = std::max(up((rows + CL - 1) / CL, 32 / Wb), 32 / Wb);
                if (Gt < G) add(Wb, Gt, CL, cpt);
            }
            if (cpt == 1 && G0 <= 16)
                for (int Wb = 32; Wb * G0 <= 512; Wb <<= 1) {
                    if ((long long)Wb / 2 >= ncol && Wb > 32) break;
                    add(Wb, G0, 1, cpt);
                }
        }
    }
    return out;
}

// Segment tilings of the fluid sweep (seg_fluid.cuh): C consecutive cells per thread (2, 3, 4 or 8; 2,
// 3 or 4 in FP64; 2 or 4 with artificial viscosity), the whole pencil in one CTA of NT = Wb * S threads,
// 64 <= NT <= 512, S = N / C threads per pencil.  Along x the S threads of a pencil are consecutive
// lanes: S is a power of two up to 32 or a multiple of 32.  Along y and z Wb >= 4 pencils (a power of
// two) sit side by side, at most 32 of them unless each pencil is one thread's (S = 1).  Along x, for a
// C (2, 4 or 8) with none of these and S = ceil(N / C) >= 64 segments, the cluster forms (seg_fluid.cuh's
// CLU; no artificial viscosity): one pencil per CTA of NT = S rounded up to a multiple of 32 threads,
// or over a cluster of CL = ceil(S / 256) <= 8 CTAs (ceil(S / 512) <= 4) of NT = ceil(S / CL) rounded
// up; where C does not divide N the last segment is ragged (launch_fluid takes these for const ends
// only).
bool seg_cluster_form(const PencilCfg& p, int N) {
    return p.seg && (p.CL > 1 || N % p.seg != 0 || p.NT != p.Wb * p.G);
}

std::vector<PencilCfg> seg_candidates(const Geom& g, int d, size_t elem, bool visc = false) {
    std::vector<PencilCfg> out;
    const int N = g.n[d];
    const long long ncol = g.ncell / N;
    for (int C : {2, 3, 4, 8}) {
        if ((elem == 8 && C == 8) || (visc && (C == 8 || C == 3))) continue;
        const size_t before = out.size();
        auto add_cluster = [&](int S, int CL, int NT) {
            const size_t smem = elem == 8 ? seg_fluid_smem_bytes<double>(NT) : seg_fluid_smem_bytes<float>(NT);
            if (smem > kPencilSmemLimit) return;
            PencilCfg p;
            p.Wb = 1;
            p.G = S;
            p.CL = CL;
            p.NT = NT;
            p.cpt = C;
            p.seg = C;
            out.push_back(p);
        };
        const int Se = N / C;
        const bool exact = N % C == 0 && (d != 0 || Se % 32 == 0 || (Se <= 32 && 32 % Se == 0));
        for (int Wb = d == 0 ? 1 : 4; exact && Wb <= (d != 0 && Se == 1 ? 512 : 32); Wb *= 2) {
            const int NT = Wb * Se;
            if (NT > 512) break;
            if (NT < 64 || NT % 32) continue;
            if (Wb > 1 && (long long)Wb / 2 >= ncol) break;   // more pencil slots than pencils
            const size_t smem = elem == 8 ? seg_fluid_smem_bytes<double>(NT, visc) : seg_fluid_smem_bytes<float>(NT, visc);
            if (smem > kPencilSmemLimit) continue;
            PencilCfg p;
            p.Wb = Wb;
            p.G = Se;
            p.CL = 1;
            p.NT = NT;
            p.cpt = C;
            p.seg = C;
            out.push_back(p);
        }
        if (d != 0 || visc || C == 3 || out.size() > before) continue;
        const int S = (N + C - 1) / C;
        if (S < 64) continue;
        if (S <= 512) add_cluster(S, 1, (S + 31) / 32 * 32);
        for (int cap : {256, 512}) {
            const int CL = (S + cap - 1) / cap;
            if (CL >= 2 && CL <= (cap == 256 ? 8 : 4)) add_cluster(S, CL, ((S + CL - 1) / CL + 31) / 32 * 32);
        }
    }
    return out;
}

// Window tilings of the magnet chain and CT pass (seg_magnet.cuh): C = 2, 3, 4 or 8 consecutive cells per
// thread with C dividing N, S = N / C threads per pencil, the whole pencil in one CTA of NT = Wb * S
// threads (32 <= NT <= 512, a multiple of 32); along y and z Wb >= 4 pencils side by side (up to 64, or
// to the CTA where each pencil is one thread's).  Along x, for a C where no such tiling exists, the
// padded ones: S = ceil(N / C) segments (the last one ragged), NT = Wb * S rounded up to a multiple of
// 32 with the threads past the segments idle, and for S above 256 (512) segments one pencil over a
// cluster of CL = ceil(S / 256) <= 8 CTAs (ceil(S / 512) <= 4) of NT = ceil(S / CL) rounded up.
std::vector<PencilCfg> win_candidates(const Geom& g, int d) {
    std::vector<PencilCfg> out;
    const int N = g.n[d];
    const long long ncol = g.ncell / N;
    auto add = [&](int Wb, int S, int CL, int NT, int C) {
        PencilCfg p;
        p.Wb = Wb;
        p.G = S;
        p.CL = CL;
        p.NT = NT;
        p.cpt = C;
        p.seg = C;
        out.push_back(p);
    };
    for (int C : {2, 3, 4, 8}) {
        const size_t before = out.size();
        if (N % C == 0) {
            const int S = N / C;
            for (int Wb = d == 0 ? 1 : 4; Wb <= (d != 0 && S == 1 ? 512 : 64); Wb *= 2) {
                const int NT = Wb * S;
                if (NT > 512) break;
                if (NT < 32 || NT % 32) continue;
                if (Wb > 1 && (long long)Wb / 2 >= ncol) break;
                add(Wb, S, 1, NT, C);
            }
        }
        if (d != 0 || out.size() > before || C == 3) continue;
        const int S = (N + C - 1) / C;
        for (int Wb = 1; Wb * S <= 512; Wb *= 2) {
            if (Wb > 1 && (long long)Wb / 2 >= ncol) break;
            add(Wb, S, 1, std::max(32, (Wb * S + 31) / 32 * 32), C);
        }
        for (int cap : {256, 512}) {
            const int CL = (S + cap - 1) / cap;
            if (CL < 2 || CL > (cap == 256 ? 8 : 4)) continue;
            add(1, S, CL, ((S + CL - 1) / CL + 31) / 32 * 32, C);
        }
    }
    return out;
}

// Default segment or window tiling among candidates c: 4 cells per thread (along y and z at least 8
// pencils side by side), else whole pencils of one thread each (pencils of 2 to 8 cells across y or z);
// the CTA nearest 256 threads.  nullptr: none of these.
const PencilCfg* default_segments(const std::vector<PencilCfg>& c, int d) {
    const PencilCfg* best = nullptr;
    for (const PencilCfg& p : c) {
        if (p.seg != 4 || (d != 0 && p.Wb < 8)) continue;
        if (!best || std::abs(p.NT - 256) < std::abs(best->NT - 256)) best = &p;
    }
    if (best || d == 0) return best;
    for (const PencilCfg& p : c) {
        if (p.G != 1) continue;
        if (!best || std::abs(p.NT - 256) < std::abs(best->NT - 256)) best = &p;
    }
    return best;
}

// Default magnet tiling: the window kernels where a default window tiling exists, else the tile
// kernels' default.
PencilCfg choose_window(const Geom& g, int d, const PencilCfg& tile) {
    std::vector<PencilCfg> c = win_candidates(g, d);
    const PencilCfg* best = default_segments(c, d);
    return best ? *best : tile;
}

// Default fluid tiling: in the mixed form the segment kernel where a default segment tiling exists
// (default_segments); in FP64, and where none exists, the tile kernels' default (the FP64 segment kernel
// needs more registers than it has; the autotuner may still pick it).
PencilCfg choose_fluid(const Geom& g, int d, size_t elem, const PencilCfg& tile) {
    if (elem == 8) return tile;
    std::vector<PencilCfg> c = seg_candidates(g, d, elem);
    const PencilCfg* best = default_segments(c, d);
    return best ? *best : tile;
}

// Fluid tiling with artificial viscosity: the segment kernel is the only one with the viscous
// exchanges; 4 cells per thread in the mixed form and 2 in FP64 (fewer registers), along y and z at
// least 8 pencils side by side where possible, the CTA nearest 256 threads.  ok = false: no segment
// tiling exists for this pencil length.
PencilCfg choose_fluid_visc(const Geom& g, int d, size_t elem, bool& ok) {
    const int want = elem == 8 ? 2 : 4;
    const PencilCfg* best = nullptr;
    std::vector<PencilCfg> c = seg_candidates(g, d, elem, true);
    auto score = [&](const PencilCfg& p) {
        return (p.seg == want ? 0 : 4096) + ((d != 0 && p.Wb < 8) ? 2048 : 0) + std::abs(p.NT - 256);
    };
    for (const PencilCfg& p : c)
        if (!best || score(p) < score(*best)) best = &p;
    ok = best != nullptr;
    return ok ? *best : PencilCfg{};
}

// Pencil tiling of one sweep direction: one cell per thread where the pencil fits a cluster of at
// most 4 CTAs of 512 threads (2 or 4 cells per thread otherwise).  Along x a CTA holds whole pencil
// segments of up to 512 rows; along y and z it holds 4 adjacent pencils, so each row of the tile is
// 4 contiguous values of x (one 32-byte sector in FP64, half of one in FP32), or, for pencils of at
// most 16 cells, 32 to 256 adjacent pencils.
PencilCfg choose_pencil(const Geom& g, int d, size_t elem) {
    const int N = g.n[d];
    const long long ncol = g.ncell / N;
    const int maxnt = 512;
    PencilCfg p, first;
    bool have_first = false;
    for (int cpt : {1, 2, 4}) {
        int G = std::max(2, pow2ceil((N + cpt - 1) / cpt));
        int CL = 1, Wb;
        if (d == 0) {
            while (G > maxnt) { G >>= 1; CL <<= 1; }
            Wb = std::max(1, 256 / G);
            if (Wb * G < 32) Wb = 32 / G;
            while (Wb > 1 && (long long)Wb / 2 >= ncol && Wb * G > 32) Wb >>= 1;
            if (G > 32) {   // whole warps per pencil, padded to a quarter of the power of two only,
                            // so that pencils of similar length share a launch shape (batching)
                const int rows = (N + cpt - 1) / cpt;
                const int q = std::max(32, G / 4);
                G = ((rows + CL - 1) / CL + q - 1) / q * q;
            }
        } else if (cpt == 1 && G <= 16) {
            // short pencils: many of them side by side, at least a warp of x per row (one CTA
            // holds whole pencils, so the column maximum stays inside the CTA)
            Wb = maxnt / G;
            while (Wb > 32 && (long long)Wb / 2 >= ncol) Wb >>= 1;
        } else {
            Wb = 4;   // 4 pencils: 32 contiguous bytes of x per row in FP64 (16 in FP32)
            G = std::max(G, 32 / Wb);
            while (Wb * G > maxnt) { G >>= 1; CL <<= 1; }
        }
        p.Wb = Wb;
        p.G = G;
        p.CL = CL;
        p.NT = Wb * G;
        p.cpt = cpt;
        // a pencil inside one CTA takes the copy-ghost kernels (no halo jobs) where its BCs allow:
        // the fewest cells per thread that achieve it; otherwise the fewest with a cluster of at
        // most 4 CTAs (clusters of 8 CTAs of these kernels do not schedule)
        if (CL == 1 && tiling_fits(p, elem)) return p;
        if (CL <= 4 && !have_first) {
            first = p;
            have_first = true;
        }
    }
    if (have_first) p = first;
    if (p.CL <= 4 && tiling_fits(p, elem)) return p;
    // too much shared memory per CTA (long FP64 pencils): the accepted tiling with the fewest
    // CTAs per cluster, then the fewest cells per thread, then the most threads
    PencilCfg best = p;
    bool found = false;
    for (const PencilCfg& c : pencil_candidates(g, d, elem)) {
        if (!found || std::make_tuple(c.CL, c.cpt, -c.NT) < std::make_tuple(best.CL, best.cpt, -best.NT)) {
            best = c;
            found = true;
        }
    }
    return best;
}

// Process-wide cache of autotuned tilings, keyed by what decides them: sweep direction, pencil
// length, number of pencils (rounded up to a power of two), precision and physics.  Contexts
// created later with the same key start from the tuned tiling.
using TuneKey = std::tuple<int, int, int, int, int, int, int, int>;
std::mutex g_tune_mu;
std::map<TuneKey, PencilCfg> g_tuned;

TuneKey tune_key(int kind, const Geom& g, int d, size_t elem, const img_config& c) {
    const long long ncol = g.ncell / g.n[d];
    return TuneKey(kind, d, g.n[d], pow2ceil((int)std::min<long long>(ncol, 1 << 30)), (int)elem, c.fluid_active,
                   c.magnet_active, c.viscosity_type);
}

int launch_blocks(long long work, int bs = 256) {
    long long b = (work + bs - 1) / bs;
    return (int)std::max(1LL, std::min(b, 148LL * 16));
}

// Sweep geometry of direction d with the context's pencil tiling (cells per thread CPT).
SweepGeom sweep_geom(const img_ctx* ctx, int d, const PencilCfg& pcf) {
    const int cpt = pcf.cpt;
    SweepGeom s{};
    s.g = ctx->g;
    s.d = d;
    s.d1 = d == 0 ? 1 : 0;
    s.d2 = d == 2 ? 1 : 2;
    s.N = ctx->g.n[d];
    s.ncol = ctx->g.ncell / s.N;
    s.Wb = pcf.Wb;
    s.G = pcf.G;
    s.CL = pcf.CL;
    s.NT = pcf.NT;
    s.RC = pcf.G * cpt;
    s.rank_hi = (s.N - 1) / s.RC;
    s.n1 = ctx->g.n[s.d1];
    s.sd = ctx->g.s[d];
    s.s1 = ctx->g.s[s.d1];
    s.s2 = ctx->g.s[s.d2];
    s.div_lanes = make_fastdiv((unsigned)(d == 0 ? s.G : s.Wb));
    s.div_cl = make_fastdiv((unsigned)s.CL);
    s.div_n1 = make_fastdiv((unsigned)s.n1);
    return s;
}

// A fade BC on sweep direction d for any of the given classes (compiles the fade damping in).
bool fade_on(const img_config& c, int d, int cls_lo, int cls_hi) {
    for (int k = cls_lo; k <= cls_hi; ++k)
        if (c.bc_modes[k][0][d] == IMG_BC_FADE || c.bc_modes[k][1][d] == IMG_BC_FADE) return true;
    return false;
}

// Boundary modes whose ghosts copy an own row of the pencil (fade: the near end row, damped).
bool copy_ghost_mode(int m) { return m == IMG_BC_CIRC || m == IMG_BC_CONST || m == IMG_BC_FADE; }

template <typename T>
PencilLaunch pencil_launch(const img_ctx* ctx, const PencilCfg& pcf, int d, size_t smem, unsigned grid_y, bool fade) {
    const long long ncol = ctx->g.ncell / ctx->g.n[d];
    const long long nb = (ncol + pcf.Wb - 1) / pcf.Wb;
    PencilLaunch L{};
    L.grid_x = (unsigned)(nb * pcf.CL);
    L.grid_y = grid_y;
    L.block = pcf.NT;
    L.smem = smem;
    L.cluster = pcf.CL;
    L.cpt = pcf.cpt;
    L.nqc = pcf.nqc;
    L.fade = fade;
    L.stream = ctx->stream;
    return L;
}

template <typename T>
int launch_fluid(img_ctx* ctx, int d, bool cfl) {
    FluidArgs a{};
    const img_config& c = ctx->cfg;
    // the segment kernel takes the steady sweeps of single-CTA pencils whose ends are circ or const for
    // all fluid classes; stored-edge capture (a run's first sweeps), fade and other ends take the tile
    // kernels
    const bool fade = fade_on(c, d, CLS_MASS, CLS_ENER);
    const bool init = ctx->init_store || ctx->init_flux;
    bool seg_ok = ctx->pcfg[0][d].seg && !init && !fade;
    for (int k = 0; k < 3; ++k)
        for (int side = 0; side < 2; ++side) {
            const int m = c.bc_modes[k][side][d];
            if ((m != IMG_BC_CIRC && m != IMG_BC_CONST) || m != c.bc_modes[CLS_MASS][side][d]) seg_ok = false;
        }
    // with artificial viscosity the tiling is always a segment one and every swept end circ or const
    // (img_create and img_set_tiling see to it), so no stored edge is ever read: the first sweeps too
    const bool visc = c.viscosity_type != IMG_VISC_NONE;
    if (visc) seg_ok = true;
    // a ragged last segment (cluster forms) supports const ends only
    const bool clu = seg_cluster_form(ctx->pcfg[0][d], ctx->g.n[d]);
    if (clu && ctx->g.n[d] % ctx->pcfg[0][d].seg != 0)
        for (int side = 0; side < 2; ++side)
            if (c.bc_modes[CLS_MASS][side][d] != IMG_BC_CONST) seg_ok = false;
    const PencilCfg& pcf = (seg_ok || !ctx->pcfg[0][d].seg) ? ctx->pcfg[0][d] : ctx->pcfg_tile[d];
    a.sg = sweep_geom(ctx, d, pcf);
    for (int v = 0; v < NQ; ++v) a.q[v] = ctx->q[v];
    a.tm = ctx->tm;
    a.gamma = c.gamma;
    a.minmass = c.minmass;
    a.minmass_out = ctx->fade_mask ? -HUGE_VAL : c.minmass;   // the point-fade pass clamps
    a.dx = c.dgrid[d];
    a.limiter = c.limiter[d];
    for (int k = 0; k < 4; ++k) {
        a.mode[k][0] = c.bc_modes[k][0][d];
        a.mode[k][1] = c.bc_modes[k][1][d];
        a.act[k] = active_lin(c, ctx->g.ndims, k, d + 1);
    }
    a.fade = ctx->fade_dev;
    a.fade_f = c.bc_infinity;
    a.bc_inf = c.bc_infinity;
    a.edges = ctx->edges_dev;
    a.init_store = ctx->init_store;
    a.init_flux = ctx->init_flux;
    a.mhd = ctx->mhd;
    for (int k = 0; k < 3; ++k) a.use_b[k] = ctx->use_b[k];
    a.cfl = cfl ? (CFL_ACCUMULATE | (c.nonfinite_check ? CFL_CHECK_NONFINITE : 0)) : 0;
    a.visc = c.viscosity_type;
    if (visc) {   // ArtificialViscosity.m:73-77, 139-147
        const double G = c.gamma, c1 = c.visc_linear, c2 = c.visc_quadratic, g4 = (G + 1) / 4;
        a.vc1 = c1;
        a.vc2 = c2;
        a.vk1 = c2 * (G + 1);
        a.vk2 = (c2 * c2) * (g4 * g4);
        a.vc1sq = c1 * c1;
    }
    PencilLaunch L = pencil_launch<T>(ctx, pcf, d,
                                      pcf.seg ? seg_fluid_smem_bytes<T>(pcf.NT, visc) : fluid_smem_bytes<T>(pcf.G * pcf.cpt, pcf.Wb),
                                      1, fade);
    L.seg = pcf.seg;
    L.clu = seg_cluster_form(pcf, ctx->g.n[d]);
    // copy ghosts: single-CTA pencils, one circ, const or fade mode per side shared by the fluid classes
    L.cg = pcf.CL == 1;
    for (int k = 0; k < 3; ++k)
        for (int side = 0; side < 2; ++side) {
            const int m = a.mode[k][side];
            if (!copy_ghost_mode(m) || m != a.mode[CLS_MASS][side]) L.cg = false;
        }
    L.init = a.init_store || a.init_flux;   // first sweeps: the stored-edge capturing kernel
    if (L.seg) L.cg = true;                  // segment kernels index their ghosts directly
    if (ctx->rec) {
        OpRec r{};
        r.kind = OP_FLUID;
        r.elem = sizeof(T);
        r.mhd = ctx->mhd != 0;
        r.L = L;
        r.fa = a;
        ctx->rec->push_back(r);
        ctx->init_store = false;
        ctx->init_flux = false;
        return IMG_OK;
    }
    cudaError_t le = launch_fluid_sweep<T>(a, L, ctx->mhd != 0);
    if (le != cudaSuccess)
        return fail(ctx, IMG_ERR_CUDA, "fluid sweep launch (dim %d, grid %u, block %u, smem %zu, cluster %d): %s", d,
                    L.grid_x, L.block, L.smem, L.cluster, cudaGetErrorString(le));
    ctx->launches += 1;
    ctx->init_store = false;
    ctx->init_flux = false;
    return IMG_OK;
}

template <typename T>
void fill_mag_args(img_ctx* ctx, int X, int I1, int I2, MagArgs& a) {
    const img_config& c = ctx->cfg;
    int d = X - 1;
    const PencilCfg& pcf = ctx->pcfg[1][d];
    a.sg = sweep_geom(ctx, d, pcf);
    for (int v = 0; v < NQ; ++v) a.q[v] = ctx->q[v];
    a.F[0] = ctx->scratch[0];
    a.F[1] = ctx->scratch[1];
    a.tm = ctx->tm;
    a.X = X;
    a.I[0] = I1;
    a.I[1] = I2;
    a.dx = c.dgrid[d];
    a.limiter = c.limiter[d];
    a.modeX[0] = c.bc_modes[CLS_MAG][0][d];
    a.modeX[1] = c.bc_modes[CLS_MAG][1][d];
    a.modeX_magX[0] = a.modeX[0];
    a.modeX_magX[1] = a.modeX[1];
    a.actX = active_lin(c, ctx->g.ndims, CLS_MAG, X);
    for (int q = 0; q < 2; ++q) {
        int I = q == 0 ? I1 : I2, e = I - 1;
        a.shiftI[q] = e < ctx->g.ndims;
        a.dI[q] = c.dgrid[e];
        for (int s = 0; s < 2; ++s) {
            a.modeI_mass[q][s] = c.bc_modes[CLS_MASS][s][e];
            a.modeI_mom[q][s] = c.bc_modes[CLS_MOM][s][e];
            a.modeI_mag[q][s] = c.bc_modes[CLS_MAG][s][e];
        }
        a.actI_mass[q] = active_lin(c, ctx->g.ndims, CLS_MASS, I);
        a.actI_mom[q] = active_lin(c, ctx->g.ndims, CLS_MOM, I);
        a.actI_mag[q] = active_lin(c, ctx->g.ndims, CLS_MAG, I);
        a.init_mag[q] = ctx->init_mag[I - 1][d];
    }
    a.fade = ctx->fade_dev;
    a.fade_f = c.bc_infinity;
    a.bc_inf = c.bc_infinity;
    a.edges = ctx->edges_dev;
}

template <typename T>
int launch_magnet(img_ctx* ctx, int X, int I1, int I2) {
    MagArgs a{};
    fill_mag_args<T>(ctx, X, I1, I2, a);
    const int d = X - 1;
    // the window kernels take the steady sweeps whose mag-class ends along X and transverse shifts (mass and
    // mom classes below, mag class above, along both I) are circ or const; the rest take the tile kernels
    auto stateless = [](int m) { return m == IMG_BC_CIRC || m == IMG_BC_CONST; };
    bool win_ok = !(a.init_mag[0] || a.init_mag[1]) && stateless(a.modeX[0]) && stateless(a.modeX[1]);
    for (int q = 0; q < 2; ++q)
        win_ok = win_ok && stateless(a.modeI_mass[q][0]) && stateless(a.modeI_mom[q][0]) && stateless(a.modeI_mag[q][1]);
    const PencilCfg& pcf = (win_ok || !ctx->pcfg[1][d].seg) ? ctx->pcfg[1][d] : ctx->pcfg_mtile[0][d];
    const PencilCfg& pcc = (win_ok || !ctx->pcfg[2][d].seg) ? ctx->pcfg[2][d] : ctx->pcfg_mtile[1][d];   // CT: own tiling
    a.sg = sweep_geom(ctx, d, pcf);
    MagArgs ac = a;
    ac.sg = sweep_geom(ctx, d, pcc);
    PencilLaunch L = pencil_launch<T>(ctx, pcf, d, pcf.seg ? 0 : mag_smem_bytes<T>(pcf.G * pcf.cpt, pcf.Wb, pcf.nqc),
                                      pcf.seg ? 1 : 2 / pcf.nqc, fade_on(ctx->cfg, d, CLS_MAG, CLS_MAG));
    PencilLaunch Lc = pencil_launch<T>(ctx, pcc, d, pcc.seg ? 0 : ctcell_smem_bytes<T>(pcc.G * pcc.cpt, pcc.Wb), 1,
                                       fade_on(ctx->cfg, d, CLS_MAG, CLS_MAG));
    L.seg = pcf.seg;
    Lc.seg = pcc.seg;
    // copy ghosts: single-CTA pencils with circ, const or fade mag-class shifts along X
    const bool cg_modes = copy_ghost_mode(a.modeX[0]) && copy_ghost_mode(a.modeX[1]);
    L.cg = pcf.CL == 1 && cg_modes;
    Lc.cg = pcc.CL == 1 && cg_modes;
    L.init = a.init_mag[0] || a.init_mag[1];   // first sweep of (I, X): the stored-edge capturing chain
    if (ctx->rec) {
        OpRec r{};
        r.elem = sizeof(T);
        r.ma = a;
        r.kind = OP_CHAIN;
        r.L = L;
        ctx->rec->push_back(r);
        r.kind = OP_CTCELL;
        r.L = Lc;
        r.ma = ac;
        ctx->rec->push_back(r);
        ctx->init_mag[I1 - 1][d] = false;
        ctx->init_mag[I2 - 1][d] = false;
        return IMG_OK;
    }
    cudaError_t le = launch_mag_chain<T>(a, L);
    if (le != cudaSuccess)
        return fail(ctx, IMG_ERR_CUDA, "magnet chain launch (dim %d, grid %u x 2, block %u, smem %zu, cluster %d): %s", d,
                    L.grid_x, L.block, L.smem, L.cluster, cudaGetErrorString(le));
    le = launch_mag_ctcell<T>(ac, Lc);
    if (le != cudaSuccess)
        return fail(ctx, IMG_ERR_CUDA, "magnet CT launch (dim %d, grid %u, block %u, smem %zu, cluster %d): %s", d,
                    Lc.grid_x, Lc.block, Lc.smem, Lc.cluster, cudaGetErrorString(le));
    ctx->launches += 2;
    ctx->init_mag[I1 - 1][d] = false;
    ctx->init_mag[I2 - 1][d] = false;
    return IMG_OK;
}

template <typename T>
CflArgs cfl_args(img_ctx* ctx) {
    CflArgs a{};
    a.g = ctx->g;
    for (int v = 0; v < NQ; ++v) a.q[v] = ctx->q[v];
    a.tm = ctx->tm;
    a.gamma = ctx->cfg.gamma;
    a.mhd = ctx->mhd;
    for (int k = 0; k < 3; ++k) a.use_b[k] = ctx->use_b[k];
    a.check_nonfinite = ctx->cfg.nonfinite_check != 0;
    a.accumulate = 1;
    a.rad_exp = ctx->cfg.rad_exponent;
    a.fade_map = ctx->fade_map;
    a.fade_ener = (ctx->fade_mask & IMG_FADE_ENER) ? 1 : 0;
    return a;
}

// The CFL maxima pass; with `radiate` the radiation sink first (source.m:30), and with accumulate =
// false the sink alone.
template <typename T>
int launch_cfl_reduce(img_ctx* ctx, bool accumulate = true, bool radiate = false) {
    CflArgs a = cfl_args<T>(ctx);
    a.accumulate = accumulate ? 1 : 0;
    a.radiate = radiate ? 1 : 0;
    if (ctx->rec) {
        if (radiate) return fail(ctx, IMG_ERR_UNSUPPORTED, "radiation in a batched launch");
        OpRec r{};
        r.kind = OP_CFL_REDUCE;
        r.elem = sizeof(T);
        r.ca = a;
        r.blocks = launch_blocks(ctx->g.ncell);
        ctx->rec->push_back(r);
        return IMG_OK;
    }
    cfl_reduce_kernel<T><<<launch_blocks(ctx->g.ncell), 256, 0, ctx->stream>>>(a);
    CK(cudaGetLastError());
    ctx->launches += 1;
    return IMG_OK;
}

// Kernel attributes (dynamic shared memory limits), set once per context so that no attribute call
// happens inside a stream capture, and a schedulability check of every pencil configuration.
template <typename T>
int set_kernel_attributes(img_ctx* ctx) {
    // once per device and precision: every pencil kernel may use the opt-in shared memory maximum
    static std::mutex mu;
    static bool done[64][2] = {};
    {
        std::lock_guard<std::mutex> lock(mu);
        if (ctx->dev < 0 || ctx->dev >= 64) return fail(ctx, IMG_ERR_UNSUPPORTED, "device ordinal %d", ctx->dev);
        bool& dn = done[ctx->dev][sizeof(T) == 8 ? 1 : 0];
        if (!dn) {
            int optin = 0;
            CK(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, ctx->dev));
            for (int cpt : {1, 2, 4}) {
                CK(fluid_attributes<T>(cpt, optin));
                CK(fluid_cluster_attributes<T>(cpt, optin));
                CK(chain_attributes<T>(cpt, optin));
            }
            CK(fluid_seg_attributes<T>(optin));
            CK(cudaFuncSetAttribute(treadmill_detect_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)kPencilSmemLimit));
            CK(cudaFuncSetAttribute(treadmill_shift_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)kPencilSmemLimit));
            dn = true;
        }
    }
    for (int kind = 0; kind < 3; ++kind)
        for (int d = 0; d < 3; ++d) {
            const PencilCfg& p = ctx->pcfg[kind][d];
            if (ctx->g.n[d] < 3 || p.seg) continue;   // segment tilings: one CTA, shared memory checked
            PencilLaunch L = pencil_launch<T>(ctx, p, d, fluid_smem_bytes<T>(p.G * p.cpt, p.Wb), 1, false);
            int nclusters = 0;
            cudaError_t e = fluid_max_clusters<T>(L, &nclusters);
            if (e != cudaSuccess) cudaGetLastError();   // leave no launch error behind for the next call
            if (e != cudaSuccess || nclusters < 1)
                return fail(ctx, IMG_ERR_UNSUPPORTED, "pencil configuration for dim %d (block %d, cluster %d, smem %zu) "
                            "cannot be scheduled: %s", d, p.NT, p.CL, L.smem,
                            e != cudaSuccess ? cudaGetErrorString(e) : "0 active clusters");
        }
    return IMG_OK;
}

// The point-fade pass of one array assignment (var >= 0: img_upload) or of a fluid sweep's assignments.
template <typename T>
int launch_point_fade(img_ctx* ctx, int var) {
    if (ctx->rec) return fail(ctx, IMG_ERR_UNSUPPORTED, "point fades in a batched launch");
    FadeArgs a{};
    a.n = ctx->g.ncell;
    for (int v = 0; v < NQ; ++v) a.q[v] = ctx->q[v];
    a.map = ctx->fade_map;
    a.mask = ctx->fade_mask;
    a.var = var;
    a.minmass = ctx->cfg.minmass;
    a.tm = ctx->tm;
    point_fade_kernel<T><<<launch_blocks(ctx->g.ncell), 256, 0, ctx->stream>>>(a);
    CK(cudaGetLastError());
    ctx->launches += 1;
    return IMG_OK;
}
int point_fade(img_ctx* ctx, int var) {
    return ctx->elem == 8 ? launch_point_fade<double>(ctx, var) : launch_point_fade<float>(ctx, var);
}

// relaxingFluid (fluid/relaxingFluid.m:16-73): the sweep, then with a point fade the pass that fades
// its assignments to the primaries (the sweep leaves rho unclamped for it).
int fluid_sweep(img_ctx* ctx, int X, bool cfl) {
    int rc = ctx->elem == 8 ? launch_fluid<double>(ctx, X - 1, cfl) : launch_fluid<float>(ctx, X - 1, cfl);
    if (rc == IMG_OK && ctx->fade_mask) rc = point_fade(ctx, -1);
    return rc;
}
int magnet_sweep(img_ctx* ctx, int X, int I1, int I2) {
    return ctx->elem == 8 ? launch_magnet<double>(ctx, X, I1, I2) : launch_magnet<float>(ctx, X, I1, I2);
}
int cfl_reduce(img_ctx* ctx) { return ctx->elem == 8 ? launch_cfl_reduce<double>(ctx) : launch_cfl_reduce<float>(ctx); }

// treadmillGrid (treadmill/treadmillGrid.m:14-37): nothing when off or before iteration 10
// (run.time.iteration, known to the host); otherwise the three treadmill kernels.
template <typename T>
int launch_treadmill(img_ctx* ctx) {
    const img_config& c = ctx->cfg;
    if (c.treadmill <= 0 || ctx->iteration < 10) return IMG_OK;
    if (ctx->rec) return fail(ctx, IMG_ERR_UNSUPPORTED, "treadmill in a batched launch");
    const int X = c.treadmill, d = X - 1;
    const Geom& g = ctx->g;
    TreadArgs a{};
    a.g = g;
    a.d = d;
    a.d1 = d == 0 ? 1 : 0;
    a.d2 = d == 2 ? 1 : 2;
    a.n1 = g.n[a.d1];
    a.n2 = g.n[a.d2];
    a.sd = g.s[d];
    a.s1 = g.s[a.d1];
    a.s2 = g.s[a.d2];
    for (int v = 0; v < NQ; ++v) a.q[v] = ctx->q[v];
    a.tm = ctx->tm;
    a.dx = c.dgrid[d];
    const int cls[TREAD_ARRAYS] = {CLS_MASS, CLS_MOM, CLS_MOM, CLS_MOM, CLS_ENER, CLS_MAG, CLS_MAG, CLS_MAG};
    const int comp[TREAD_ARRAYS] = {0, 1, 2, 3, 0, 1, 2, 3};
    const int obj[TREAD_ARRAYS] = {OBJ_PRIM_MASS, OBJ_PRIM_MOM, OBJ_PRIM_MOM + 1, OBJ_PRIM_MOM + 2, OBJ_PRIM_ENER,
                                   OBJ_PRIM_MAG, OBJ_PRIM_MAG + 1, OBJ_PRIM_MAG + 2};
    for (int k = 0; k < TREAD_ARRAYS; ++k) {
        for (int s = 0; s < 2; ++s) {
            a.mode[k][s] = c.bc_modes[cls[k]][s][d];
            a.edge[k][s] = d < g.ndims ? ctx->edges_host.p[obj[k]][d][s] : nullptr;
        }
        a.neg[k] = comp[k] == X;
        a.act[k] = active_lin(c, g.ndims, cls[k], X);
    }
    a.fade = ctx->fade_dev;
    a.fade_f = c.bc_infinity;
    a.bc_inf = c.bc_infinity;
    a.idx = ctx->tread_idx;
    a.means = ctx->tread_means;
    a.hist = ctx->tread_hist;
    a.hist_cap = kTreadHistCap;
    a.fade_map = ctx->fade_map;
    a.fade_mask = ctx->fade_mask;
    const long long ncol = g.ncell / g.n[d];
    const size_t smem = tread_smem_bytes(g.n[d], sizeof(T));
    if (d >= g.ndims) {   // ImogenArray.shift is not enabled along a third dimension of a 2-D grid
        for (int k = 0; k < TREAD_ARRAYS; ++k) a.mode[k][0] = a.mode[k][1] = IMG_BC_CONST;
    }
    treadmill_detect_kernel<T><<<(unsigned)ncol, 256, smem, ctx->stream>>>(a);
    CK(cudaGetLastError());
    treadmill_finalize_kernel<<<1, 256, 0, ctx->stream>>>(a);
    CK(cudaGetLastError());
    treadmill_shift_kernel<T><<<dim3((unsigned)ncol, TREAD_ARRAYS), 256, smem, ctx->stream>>>(a);
    CK(cudaGetLastError());
    ctx->launches += 3;
    return IMG_OK;
}

int treadmill_grid(img_ctx* ctx) { return ctx->elem == 8 ? launch_treadmill<double>(ctx) : launch_treadmill<float>(ctx); }

// source(run, ...) of source.m:1-36 for this path: the radiation sink (source.m:30); nothing
// without radiation.  accumulate: the same pass collects the CFL maxima of the new state for the
// next TimeManager.update.
int source_sink(img_ctx* ctx, bool accumulate) {
    if (ctx->cfg.radiation_type == IMG_RAD_NONE) return IMG_OK;
    return ctx->elem == 8 ? launch_cfl_reduce<double>(ctx, accumulate, true) : launch_cfl_reduce<float>(ctx, accumulate, true);
}

// Radiation.initialize (fluid/Radiation.m:61-75) from the state on the device; tm->rad_minbits holds
// the bits of +inf between calls (set at creation, reset by the finalisation).
template <typename T>
int radiation_initialize(img_ctx* ctx) {
    const CflArgs a = cfl_args<T>(ctx);
    rad_init_kernel<T><<<launch_blocks(ctx->g.ncell), 256, 0, ctx->stream>>>(a);
    CK(cudaGetLastError());
    rad_init_finalize_kernel<<<1, 32, 0, ctx->stream>>>(ctx->tm, ctx->cfg.rad_initial_maximum / 100);
    CK(cudaGetLastError());
    ctx->launches += 2;
    return IMG_OK;
}

// flux.m:17-62 for one half step.  `fuse_cfl`: the final fluid sweep accumulates the CFL maxima.
int do_flux(img_ctx* ctx, int order, bool fuse_cfl) {
    const img_config& c = ctx->cfg;
    int row = (ctx->iteration - 1) % 6;
    int last_fluid = -1;
    for (int q = 0; q < 3; ++q) {
        int X = order > 0 ? FWD[row][q] : BWD[row][q];
        if (ctx->g.n[X - 1] >= 3) last_fluid = q;
    }
    for (int q = 0; q < 3; ++q) {
        int X = order > 0 ? FWD[row][q] : BWD[row][q];
        if (ctx->g.n[X - 1] < 3) continue;
        bool cfl_here = fuse_cfl && order < 0 && q == last_fluid && c.fluid_active;
        int rc;
        if (order > 0) {
            if (c.fluid_active && (rc = fluid_sweep(ctx, X, false)) != IMG_OK) return rc;
            if (c.magnet_active && (rc = magnet_sweep(ctx, X, FWD_MI[X - 1][0], FWD_MI[X - 1][1])) != IMG_OK) return rc;
        } else {
            if (c.magnet_active && (rc = magnet_sweep(ctx, X, BWD_MI[X - 1][0], BWD_MI[X - 1][1])) != IMG_OK) return rc;
            if (c.fluid_active && (rc = fluid_sweep(ctx, X, cfl_here)) != IMG_OK) return rc;
        }
    }
    return IMG_OK;
}

int time_update_async(img_ctx* ctx, int flux_direction) {
    if (flux_direction > 1 && ctx->cfg.update_mode != 0) return IMG_OK;   // TimeManager.m:61-63
    if (!ctx->cfl_valid) {
        int rc = cfl_reduce(ctx);
        if (rc != IMG_OK) return rc;
    } else if (ctx->rec && ctx->pad_cfl) {   // a batch member with valid maxima beside one without
        int rc = ctx->elem == 8 ? launch_cfl_reduce<double>(ctx, false) : launch_cfl_reduce<float>(ctx, false);
        if (rc != IMG_OK) return rc;
    }
    ctx->pad_cfl = false;
    if (ctx->rec) {
        OpRec r{};
        r.kind = OP_CFL_FINALIZE;
        r.elem = (int)ctx->elem;
        r.tm = ctx->tm;
        r.check_running = flux_direction == 1 ? 1 : 0;
        ctx->rec->push_back(r);
        ctx->cfl_valid = false;
        return IMG_OK;
    }
    cfl_finalize_kernel<<<1, 32, 0, ctx->stream>>>(ctx->tm, flux_direction == 1 ? 1 : 0);
    CK(cudaGetLastError());
    ctx->launches += 1;
    ctx->cfl_valid = false;
    return IMG_OK;
}

// One iteration (imogen.m:60-66): time.update(1), flux(+1), time.update(2), flux(-1).
// With radiation each timestep ends with source.m's sink (imogen.m:63-67), whose pass also collects
// the CFL maxima that the next TimeManager.update reads (instead of the last fluid sweep).
// Whether DevTime holds the CFL maxima of the state an iteration leaves: with a per-iteration dt the
// last fluid sweep collects them, or, with radiation, the sink's pass; a treadmill or a point fade changes
// the state after the last sweep, so without radiation nothing collects them.
bool cfl_valid_after_iteration(const img_ctx* ctx) {
    const bool rad = ctx->cfg.radiation_type != IMG_RAD_NONE;
    const bool late = ctx->cfg.treadmill > 0 || ctx->fade_mask;
    return ctx->cfg.update_mode != 0 && ctx->cfg.fluid_active && (rad || !late);
}

// The treadmill (imogen.m:64) moves the state after each flux, so with one the last fluid sweep
// collects no CFL maxima either.
int enqueue_iteration(img_ctx* ctx) {
    int rc;
    const bool per_iter = ctx->cfg.update_mode != 0;
    const bool rad = ctx->cfg.radiation_type != IMG_RAD_NONE;
    const bool tread = ctx->cfg.treadmill > 0 || ctx->fade_mask;   // the state changes after the last sweep
    const bool fl = ctx->cfg.fluid_active != 0;
    if ((rc = time_update_async(ctx, 1)) != IMG_OK) return rc;
    if ((rc = do_flux(ctx, 1, false)) != IMG_OK) return rc;
    if ((rc = treadmill_grid(ctx)) != IMG_OK) return rc;
    if (rad) {
        if ((rc = source_sink(ctx, !per_iter && fl)) != IMG_OK) return rc;
        ctx->cfl_valid = !per_iter && fl;
    }
    if ((rc = time_update_async(ctx, 2)) != IMG_OK) return rc;
    if ((rc = do_flux(ctx, -1, per_iter && !rad && !tread)) != IMG_OK) return rc;
    if ((rc = treadmill_grid(ctx)) != IMG_OK) return rc;
    if (rad && (rc = source_sink(ctx, per_iter && fl)) != IMG_OK) return rc;
    ctx->cfl_valid = cfl_valid_after_iteration(ctx);
    return IMG_OK;
}

int check_dev_error(img_ctx* ctx) {
    CK(cudaMemcpyAsync(ctx->host_tm, ctx->tm, sizeof(DevTime), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    int e = ctx->host_tm->error;
    if (e & DERR_CFL) return fail(ctx, IMG_ERR_CFL, "CFL error: no velocity exceeded the 1e-2 floor (cmax=%g)", ctx->host_tm->cmax);
    if (e & DERR_NONFINITE_DT) return fail(ctx, IMG_ERR_NONFINITE, "non-finite timestep");
    if (e & DERR_NONFINITE_STATE)
        return fail(ctx, IMG_ERR_NONFINITE, "non-finite value in the state (rho, momentum, energy or B)");
    return IMG_OK;
}

int validate(const img_config& c, std::string& why) {
    for (int d = 0; d < 3; ++d) {
        if (c.grid[d] < 1) { why = "grid extents must be >= 1"; return IMG_ERR_ARG; }
        if (!(c.dgrid[d] > 0)) { why = "dGrid must be > 0"; return IMG_ERR_ARG; }
        if (c.limiter[d] < 0 || c.limiter[d] > 2) { why = "unknown flux limiter"; return IMG_ERR_ARG; }
    }
    if (c.precision != IMG_PREC_FP64 && c.precision != IMG_PREC_MIXED) { why = "unknown precision"; return IMG_ERR_ARG; }
    if ((long long)c.grid[0] * c.grid[1] * c.grid[2] >= (1LL << 31)) { why = "grids are limited to < 2^31 cells"; return IMG_ERR_ARG; }
    if (c.bc_infinity < 4) { why = "bcInfinity must be >= 4"; return IMG_ERR_ARG; }
    if (c.viscosity_type < IMG_VISC_NONE || c.viscosity_type > IMG_VISC_CARAMANA_SHASHKOV_WHALEN) {
        why = "unknown artificial viscosity type";
        return IMG_ERR_ARG;
    }
    if (c.radiation_type < IMG_RAD_NONE || c.radiation_type > IMG_RAD_OPTICALLY_THIN) { why = "unknown radiation type"; return IMG_ERR_ARG; }
    if (c.treadmill < 0 || c.treadmill > 3) { why = "treadmill direction must be 0 (off) or 1-3"; return IMG_ERR_ARG; }
    if (c.fade_active & ~31) { why = "unknown point-fade array in fade_active"; return IMG_ERR_ARG; }
    if (c.fade_active) {
        if (!(c.fade_size > 0)) { why = "point fade: fade_size must be > 0"; return IMG_ERR_ARG; }
        for (int d = 0; d < 3; ++d)
            if (c.fade_location[d] < 1 || c.fade_location[d] > c.grid[d]) {
                why = "point fade: fade_location must be a cell of the grid (1-based)";
                return IMG_ERR_ARG;
            }
    }
    if (c.treadmill > 0 &&
        tread_smem_bytes(c.grid[c.treadmill - 1], c.precision == IMG_PREC_FP64 ? 8 : 4) > kPencilSmemLimit) {
        why = "treadmill: the pencils along its direction do not fit one thread block's shared memory";
        return IMG_ERR_UNSUPPORTED;
    }
    if (c.viscosity_type != IMG_VISC_NONE)   // the segment kernel's ends (seg_fluid.cuh)
        for (int d = 0; d < 3; ++d) {
            if (c.grid[d] < 3) continue;
            for (int s = 0; s < 2; ++s) {
                const int m = c.bc_modes[CLS_MASS][s][d];
                bool ok = m == IMG_BC_CIRC || m == IMG_BC_CONST;
                for (int k = 1; k < 4; ++k) ok = ok && c.bc_modes[k][s][d] == m;
                if (!ok) {
                    why = "artificial viscosity needs circ or const ends, the same for mass, momentum, energy and B";
                    return IMG_ERR_UNSUPPORTED;
                }
            }
        }
    int ndims = c.grid[2] > 1 ? 3 : 2;
    for (int k = 0; k < 4; ++k)
        for (int s = 0; s < 2; ++s)
            for (int d = 0; d < ndims; ++d) {
                int m = c.bc_modes[k][s][d];
                if (m < 0 || m > IMG_BC_WORMHOLE) { why = "unknown BC mode"; return IMG_ERR_ARG; }
                if (m == IMG_BC_LINEAR) {   // linear_shift.m:20: `dim` is never defined
                    why = "linear BC: linear_shift.m indexes with the undefined variable 'dim' (the reference stops "
                          "at the first shift)";
                    return IMG_ERR_UNSUPPORTED;
                }
                if (m == IMG_BC_WORMHOLE && s == 0) {   // wormhole_shift.m:16-61, lower side only
                    why = ndims < 3 ? "wormhole BC on a 2-D grid (wormhole_shift.m indexes a third dimension)"
                                    : "lower wormhole BC: the ghosts come from the pencil mirrored along nextDir, "
                                      "which this path does not couple";
                    return IMG_ERR_UNSUPPORTED;
                }
                // mirror_shift.m:31-33 / fade_shift.m:34-44 and Edges.m:80-93 index outside short
                // dimensions: the reference stops with an index error there.
                if (m == IMG_BC_MIRROR && c.grid[d] < 2) { why = "mirror BC on a dimension of extent 1"; return IMG_ERR_UNSUPPORTED; }
                if (m == IMG_BC_FADE && c.grid[d] < std::max(20, c.bc_infinity)) {
                    why = "fade BC on a dimension shorter than max(20, bcInfinity)";
                    return IMG_ERR_UNSUPPORTED;
                }
            }
    return IMG_OK;
}

// Device bytes: state + scratch + edges + tables.
struct Layout {
    size_t state, scratch, tm, table, fade, partial, stage, tread, dthist, fademap, edges, total;
    size_t edge_off[NOBJ][3][2];
};

Layout plan(const img_config& c) {
    Layout L{};
    size_t elem = c.precision == IMG_PREC_FP64 ? 8 : 4;
    long long n = (long long)c.grid[0] * c.grid[1] * c.grid[2];
    size_t arr = align256(n * elem);
    L.state = arr * NQ;
    L.scratch = c.magnet_active ? arr * 2 : 0;
    L.tm = align256(sizeof(DevTime));
    L.table = align256(sizeof(EdgeTable));
    L.fade = align256(sizeof(double) * std::max(1, c.bc_infinity));
    L.partial = align256(sizeof(double) * 2 * 8 * 1024);
    L.stage = elem == 4 ? align256(n * sizeof(double)) : 0;   // FP64 staging of host transfers (mixed)
    if (c.treadmill > 0) {   // per-pencil indices, first means, history
        const long long ncol = n / c.grid[c.treadmill - 1];
        L.tread = align256(sizeof(int) * ncol) + align256(sizeof(double) * ncol) + align256(sizeof(int) * kTreadHistCap);
    }
    int ndims = c.grid[2] > 1 ? 3 : 2;
    size_t off = 0;
    for (int o = 0; o < NOBJ; ++o)
        for (int e = 0; e < 3; ++e)
            for (int s = 0; s < 2; ++s) {
                L.edge_off[o][e][s] = (size_t)-1;
                if (e >= ndims || !obj_used(c, o)) continue;
                if (!stateful(c.bc_modes[obj_class(o)][s][e])) continue;
                L.edge_off[o][e][s] = off;
                off += align256(sizeof(double) * (n / c.grid[e]));
            }
    L.edges = off;
    L.dthist = align256(sizeof(double) * dt_hist_cap(c));
    L.fademap = (c.fade_active & (IMG_FADE_MASS | IMG_FADE_MOM | IMG_FADE_ENER)) ? arr : 0;
    L.total = L.state + L.scratch + L.tm + L.table + L.fade + L.partial + L.stage + L.tread + L.dthist + L.fademap + L.edges;
    return L;
}

// Face of a host FP64 array along dim e at index idx (column-major order of the other dims).
void host_face(const Geom& g, const double* a, int e, int idx, std::vector<double>& out) {
    out.resize(g.ncell / g.n[e]);
    for (int z = 0; z < g.n[2]; ++z)
        for (int y = 0; y < g.n[1]; ++y)
            for (int x = 0; x < g.n[0]; ++x) {
                int c[3] = {x, y, z};
                if (c[e] != idx) continue;
                out[face_index(g, e, x, y, z)] = a[x + (long long)g.n[0] * (y + (long long)g.n[1] * z)];
            }
}

template <typename T>
int cellmag_init(img_ctx* ctx) {
    CellMagInitArgs a{};
    a.g = ctx->g;
    for (int v = 0; v < NQ; ++v) a.q[v] = ctx->q[v];
    for (int c = 0; c < 3; ++c) {
        a.mode_hi[c] = ctx->cfg.bc_modes[CLS_MAG][1][c];
        a.act[c] = active_lin(ctx->cfg, ctx->g.ndims, CLS_MAG, c + 1);
    }
    a.edges = ctx->edges_dev;
    a.fade = ctx->fade_dev;
    a.fade_f = ctx->cfg.bc_infinity;
    a.bc_inf = ctx->cfg.bc_infinity;
    cellmag_init_kernel<T><<<launch_blocks(3 * ctx->g.ncell), 256, 0, ctx->stream>>>(a);
    CK(cudaGetLastError());
    return IMG_OK;
}

}  // namespace

extern "C" {

void img_config_default(img_config* c) {
    std::memset(c, 0, sizeof *c);
    for (int d = 0; d < 3; ++d) { c->grid[d] = 1; c->dgrid[d] = 1.0; c->limiter[d] = IMG_LIM_VANLEER; }
    c->gamma = 5.0 / 3.0;
    c->cfl = 0.7;
    c->minmass = 1e-5;
    c->bc_infinity = 20;
    c->fluid_active = 1;
    c->magnet_active = 0;
    c->time_max = 1e5;
    c->iter_max = 10;
    c->update_mode = 1;
    c->precision = IMG_PREC_FP64;
    c->nonfinite_check = 1;
    c->rad_exponent = 0.5;   // Radiation.m:34
}

size_t img_bytes_required(const img_config* cfg) { return cfg ? plan(*cfg).total : 0; }

int img_create(img_ctx** out, const img_config* cfg) {
    img_ctx* ctx = nullptr;
    if (!out || !cfg) return fail(nullptr, IMG_ERR_ARG, "null argument");
    *out = nullptr;
    std::string why;
    int rc = validate(*cfg, why);
    if (rc != IMG_OK) return fail(nullptr, rc, "%s", why.c_str());
    ctx = new img_ctx();
    ctx->cfg = *cfg;
    ctx->elem = cfg->precision == IMG_PREC_FP64 ? 8 : 4;
    Geom& g = ctx->g;
    for (int d = 0; d < 3; ++d) g.n[d] = cfg->grid[d];
    g.ndims = cfg->grid[2] > 1 ? 3 : 2;
    g.s[0] = 1;
    g.s[1] = g.n[0];
    g.s[2] = (long long)g.n[0] * g.n[1];
    g.ncell = (long long)g.n[0] * g.n[1] * g.n[2];
    // IMOGEN_B200_TILE_KERNELS=1 (read here, at creation): the pencil-tile kernels for every sweep, whatever
    // the default or an earlier autotuning would pick (e.g. to check the segment and window kernels)
    const char* tk = getenv("IMOGEN_B200_TILE_KERNELS");
    const bool tile_only = tk && tk[0] == '1';
    for (int kind = 0; kind < 3; ++kind)
        for (int d = 0; d < 3; ++d) {
            ctx->pcfg[kind][d] = choose_pencil(g, d, ctx->elem);
            if (kind == 0) {
                ctx->pcfg_tile[d] = ctx->pcfg[0][d];
                if (tile_only) continue;
                ctx->pcfg[0][d] = choose_fluid(g, d, ctx->elem, ctx->pcfg_tile[d]);
            } else {
                ctx->pcfg_mtile[kind - 1][d] = ctx->pcfg[kind][d];
                if (tile_only) continue;
                ctx->pcfg[kind][d] = choose_window(g, d, ctx->pcfg_mtile[kind - 1][d]);
            }
            if (kind == 0 && cfg->viscosity_type != IMG_VISC_NONE && g.n[d] >= 3) {
                bool ok = false;
                ctx->pcfg[0][d] = choose_fluid_visc(g, d, ctx->elem, ok);
                if (!ok) {
                    fail(ctx, IMG_ERR_UNSUPPORTED, "artificial viscosity: no one-block segment tiling for dimension %d "
                         "(N = %d)", d + 1, g.n[d]);
                    g_create_err = ctx->err;
                    delete ctx;
                    return IMG_ERR_UNSUPPORTED;
                }
            }
            std::lock_guard<std::mutex> lock(g_tune_mu);
            auto it = g_tuned.find(tune_key(kind, g, d, ctx->elem, *cfg));
            if (it != g_tuned.end()) ctx->pcfg[kind][d] = it->second;
        }

    auto bail = [&](int code) {
        if (ctx->slab) cudaFree(ctx->slab);
        if (ctx->host_tm) cudaFreeHost(ctx->host_tm);
        if (ctx->stream) cudaStreamDestroy(ctx->stream);
        g_create_err = ctx->err;
        delete ctx;
        return code;
    };
    if (cudaGetDevice(&ctx->dev) != cudaSuccess) { fail(ctx, IMG_ERR_CUDA, "no CUDA device"); return bail(IMG_ERR_CUDA); }
    if (cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess) {
        fail(ctx, IMG_ERR_CUDA, "stream creation failed");
        return bail(IMG_ERR_CUDA);
    }
    ctx->own_stream = ctx->stream;
    ctx->created = std::time(nullptr);
    Layout L = plan(*cfg);
    ctx->slab_bytes = L.total;
    if (cudaMalloc(&ctx->slab, L.total) != cudaSuccess) {
        cudaGetLastError();
        fail(ctx, IMG_ERR_NOMEM, "cudaMalloc of %zu bytes failed", L.total);
        return bail(IMG_ERR_NOMEM);
    }
    if (cudaMallocHost(&ctx->host_tm, sizeof(DevTime)) != cudaSuccess) {
        fail(ctx, IMG_ERR_NOMEM, "pinned allocation failed");
        return bail(IMG_ERR_NOMEM);
    }
    char* p = static_cast<char*>(ctx->slab);
    size_t arr = align256(g.ncell * ctx->elem);
    for (int v = 0; v < NQ; ++v) ctx->q[v] = p + v * arr;
    p += L.state;
    if (cfg->magnet_active)
        for (int k = 0; k < 2; ++k) ctx->scratch[k] = p + k * arr;
    p += L.scratch;
    ctx->tm = reinterpret_cast<DevTime*>(p);
    p += L.tm;
    ctx->edges_dev = reinterpret_cast<EdgeTable*>(p);
    p += L.table;
    ctx->fade_dev = reinterpret_cast<double*>(p);
    p += L.fade;
    ctx->partial = reinterpret_cast<double*>(p);
    p += L.partial;
    ctx->stage = L.stage ? reinterpret_cast<double*>(p) : nullptr;
    p += L.stage;
    if (L.tread) {
        const long long ncol = g.ncell / g.n[cfg->treadmill - 1];
        ctx->tread_idx = reinterpret_cast<int*>(p);
        ctx->tread_means = reinterpret_cast<double*>(p + align256(sizeof(int) * ncol));
        ctx->tread_hist = reinterpret_cast<int*>(p + align256(sizeof(int) * ncol) + align256(sizeof(double) * ncol));
    }
    p += L.tread;
    ctx->dt_hist = reinterpret_cast<double*>(p);
    p += L.dthist;
    if (L.fademap) {
        ctx->fade_map = p;
        ctx->fade_mask = cfg->fade_active & (IMG_FADE_MASS | IMG_FADE_MOM | IMG_FADE_ENER);
    }
    p += L.fademap;
    char* edge_base = p;
    for (int o = 0; o < NOBJ; ++o)
        for (int e = 0; e < 3; ++e)
            for (int s = 0; s < 2; ++s)
                ctx->edges_host.p[o][e][s] =
                    L.edge_off[o][e][s] == (size_t)-1 ? nullptr : reinterpret_cast<double*>(edge_base + L.edge_off[o][e][s]);
    if (cudaMemsetAsync(ctx->slab, 0, L.total, ctx->stream) != cudaSuccess ||
        cudaMemcpyAsync(ctx->edges_dev, &ctx->edges_host, sizeof(EdgeTable), cudaMemcpyHostToDevice, ctx->stream) != cudaSuccess) {
        fail(ctx, IMG_ERR_CUDA, "device initialisation failed");
        return bail(IMG_ERR_CUDA);
    }
    ctx->fade_host = fade_coefficients(std::max(1, cfg->bc_infinity));
    DevTime t{};
    t.time = 0;
    t.dt = 0;
    t.time_max = cfg->time_max;
    t.cfl = cfg->cfl;
    for (int d = 0; d < 3; ++d) t.dgrid[d] = cfg->dgrid[d];
    t.update_mode = cfg->update_mode;
    t.rad_minbits = 0xfff0000000000000ull;   // ordered bits of +inf (rad_init_kernel)
    t.tread_last = -1;                       // TreadmillManager.last
    t.dt_hist = ctx->dt_hist;
    t.dt_hist_cap = dt_hist_cap(*cfg);
    *ctx->host_tm = t;
    if (cudaMemcpyAsync(ctx->fade_dev, ctx->fade_host.data(), sizeof(double) * ctx->fade_host.size(), cudaMemcpyHostToDevice,
                        ctx->stream) != cudaSuccess ||
        cudaMemcpyAsync(ctx->tm, ctx->host_tm, sizeof(DevTime), cudaMemcpyHostToDevice, ctx->stream) != cudaSuccess ||
        cudaStreamSynchronize(ctx->stream) != cudaSuccess) {
        fail(ctx, IMG_ERR_CUDA, "device initialisation failed");
        return bail(IMG_ERR_CUDA);
    }
    if (ctx->fade_map) {   // ImogenManager.addFades builds the map from the grid alone (ImogenManager.m:267)
        const std::vector<double> m = point_fade_map(*cfg);
        cudaError_t e;
        if (ctx->elem == 8) {
            e = cudaMemcpy(ctx->fade_map, m.data(), sizeof(double) * m.size(), cudaMemcpyHostToDevice);
        } else {
            const std::vector<float> f(m.begin(), m.end());
            e = cudaMemcpy(ctx->fade_map, f.data(), sizeof(float) * f.size(), cudaMemcpyHostToDevice);
        }
        if (e != cudaSuccess) {
            fail(ctx, IMG_ERR_CUDA, "point-fade map upload failed: %s", cudaGetErrorString(e));
            return bail(IMG_ERR_CUDA);
        }
    }
    {
        const int rc = ctx->elem == 8 ? set_kernel_attributes<double>(ctx) : set_kernel_attributes<float>(ctx);
        if (rc != IMG_OK) return bail(rc);   // IMG_ERR_UNSUPPORTED: a pencil tiling that cannot be scheduled
    }
    *out = ctx;
    return IMG_OK;
}

int img_destroy(img_ctx* ctx) {
    if (!ctx) return IMG_OK;
    if (ctx->batch) img_batch_remove(ctx->batch, ctx);
    cudaStreamSynchronize(ctx->stream);
    for (auto& row : ctx->graphs)
        for (auto& gx : row)
            if (gx) cudaGraphExecDestroy(gx);
    if (ctx->slab) cudaFree(ctx->slab);
    if (ctx->host_tm) cudaFreeHost(ctx->host_tm);
    if (ctx->own_stream) cudaStreamDestroy(ctx->own_stream);
    for (cudaEvent_t e : ctx->xfer_ev)
        if (e) cudaEventDestroy(e);
    if (ctx->xfer_stream) cudaStreamDestroy(ctx->xfer_stream);
    if (ctx->h32) cudaFreeHost(ctx->h32);
    delete ctx;
    return IMG_OK;
}

const char* img_last_error(const img_ctx* ctx) { return ctx ? ctx->err.c_str() : g_create_err.c_str(); }

// Enqueue one host -> device array transfer (no synchronisation).
static int enqueue_upload(img_ctx* ctx, int var, const double* host, size_t n) {
    if (!host || var < 0 || var > IMG_VAR_MAGZ) return fail(ctx, IMG_ERR_ARG, "bad upload argument");
    if (n != (size_t)ctx->g.ncell) return fail(ctx, IMG_ERR_ARG, "upload size %zu != %lld cells", n, ctx->g.ncell);
    if (ctx->elem == 8) {
        CK(cudaMemcpyAsync(ctx->q[var], host, n * 8, cudaMemcpyHostToDevice, ctx->stream));
    } else {   // FP64 values to the staging buffer, rounded to FP32 on the device
        CK(cudaMemcpyAsync(ctx->stage, host, n * 8, cudaMemcpyHostToDevice, ctx->stream));
        f64_to_f32_kernel<<<launch_blocks((long long)(n + 3) / 4), 256, 0, ctx->stream>>>(
            ctx->stage, static_cast<float*>(ctx->q[var]), (long long)n);
        CK(cudaGetLastError());
        ctx->launches += 1;
    }
    ctx->cfl_valid = false;
    return IMG_OK;
}

// Enqueue one device -> host array transfer (no synchronisation).
static int enqueue_download(img_ctx* ctx, int var, double* host, size_t n) {
    if (!host || var < 0 || var >= NQ) return fail(ctx, IMG_ERR_ARG, "bad download argument");
    if (n != (size_t)ctx->g.ncell) return fail(ctx, IMG_ERR_ARG, "download size %zu != %lld cells", n, ctx->g.ncell);
    if (ctx->elem == 8) {
        CK(cudaMemcpyAsync(host, ctx->q[var], n * 8, cudaMemcpyDeviceToHost, ctx->stream));
    } else {   // widened to FP64 on the device, then one copy
        f32_to_f64_kernel<<<launch_blocks((long long)(n + 3) / 4), 256, 0, ctx->stream>>>(
            static_cast<const float*>(ctx->q[var]), ctx->stage, (long long)n);
        CK(cudaGetLastError());
        ctx->launches += 1;
        CK(cudaMemcpyAsync(host, ctx->stage, n * 8, cudaMemcpyDeviceToHost, ctx->stream));
    }
    return IMG_OK;
}

// X.array = value fades a primary the point fade acts on (ImogenArray.m:85), except the initial
// assignment of img_set_state.
static int fade_assigned(img_ctx* ctx, int var) {
    if (!ctx->fade_mask || ctx->constructing) return IMG_OK;
    const int bit = var == IMG_VAR_MASS ? IMG_FADE_MASS
                    : (var >= IMG_VAR_MOMX && var <= IMG_VAR_MOMZ ? IMG_FADE_MOM : (var == IMG_VAR_ENER ? IMG_FADE_ENER : 0));
    return (ctx->fade_mask & bit) ? point_fade(ctx, var) : IMG_OK;
}

int img_upload(img_ctx* ctx, int var, const double* host, size_t n) {
    if (!ctx) return fail(ctx, IMG_ERR_ARG, "null context");
    int rc = enqueue_upload(ctx, var, host, n);
    if (rc != IMG_OK) return rc;
    if ((rc = fade_assigned(ctx, var)) != IMG_OK) return rc;
    CK(cudaStreamSynchronize(ctx->stream));
    return IMG_OK;
}

// Mixed form, several arrays (img_upload_many / img_download_many): FP32 crosses PCIe.  The host
// pool rounds each FP64 array to FP32 (or widens it after the copy) in chunks, into one of two pinned
// FP32 buffers, and the copy of one array overlaps the conversion of the next.  The rounding is IEEE
// round-to-nearest on the host as in the device conversion kernels, so the state holds the same bits
// either way; the caller's arrays need not be pinned.
static int staged_streams(img_ctx* ctx) {
    if (ctx->xfer_stream) return IMG_OK;
    CK(cudaStreamCreateWithFlags(&ctx->xfer_stream, cudaStreamNonBlocking));
    for (cudaEvent_t& e : ctx->xfer_ev) CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    return IMG_OK;
}

static void convert_chunks(size_t n, const std::function<void(size_t, size_t)>& f) {
    HostPool& pool = HostPool::get();
    const size_t chunk = std::max<size_t>(8192, (n + 2 * pool.threads() - 1) / (2 * pool.threads()));
    const int nc = (int)((n + chunk - 1) / chunk);
    pool.run(nc, [&](int c) {
        const size_t a = (size_t)c * chunk;
        f(a, std::min(n, a + chunk));
    });
}

static int staged_transfer(img_ctx* ctx, int count, const int* vars, const double* const* up, double* const* down,
                           size_t n) {
    int rc = staged_streams(ctx);
    if (rc != IMG_OK) return rc;
    if (!ctx->h32) CK(cudaHostAlloc(reinterpret_cast<void**>(&ctx->h32), 2 * n * sizeof(float), cudaHostAllocDefault));
    cudaStream_t ms = ctx->stream, xs = ctx->xfer_stream;
    cudaEvent_t* ev = ctx->xfer_ev;
    float* hb[2] = {ctx->h32, ctx->h32 + n};
    CK(cudaEventRecord(ev[4], ms));        // the stream's earlier work (kernels reading or writing the state)
    CK(cudaStreamWaitEvent(xs, ev[4], 0));
    if (up) {
        for (int i = 0; i < count; ++i) {
            const int b = i & 1;
            if (i >= 2) CK(cudaEventSynchronize(ev[2 + b]));   // buffer b's previous copy is done
            const double* src = up[i];
            float* dst = hb[b];
            convert_chunks(n, [&](size_t a, size_t e) {
                for (size_t j = a; j < e; ++j) dst[j] = (float)src[j];
            });
            CK(cudaMemcpyAsync(ctx->q[vars[i]], dst, n * sizeof(float), cudaMemcpyHostToDevice, xs));
            CK(cudaEventRecord(ev[2 + b], xs));
        }
        ctx->cfl_valid = false;
    } else {
        auto enqueue = [&](int i) -> cudaError_t {
            cudaError_t e = cudaMemcpyAsync(hb[i & 1], ctx->q[vars[i]], n * sizeof(float), cudaMemcpyDeviceToHost, xs);
            return e == cudaSuccess ? cudaEventRecord(ev[2 + (i & 1)], xs) : e;
        };
        for (int i = 0; i < count && i < 2; ++i) CK(enqueue(i));
        for (int i = 0; i < count; ++i) {
            const int b = i & 1;
            CK(cudaEventSynchronize(ev[2 + b]));
            const float* src = hb[b];
            double* dst = down[i];
            convert_chunks(n, [&](size_t a, size_t e) {
                for (size_t j = a; j < e; ++j) dst[j] = (double)src[j];
            });
            if (i + 2 < count) CK(enqueue(i + 2));
        }
    }
    CK(cudaEventRecord(ev[4], xs));        // the caller synchronises the context's stream
    CK(cudaStreamWaitEvent(ms, ev[4], 0));
    return IMG_OK;
}

static bool staged_ok(const img_ctx* ctx, int count, const int* var_ids, size_t n, int nvars) {
    if (ctx->elem != 4 || n != (size_t)ctx->g.ncell) return false;
    for (int i = 0; i < count; ++i)
        if (var_ids[i] < 0 || var_ids[i] >= nvars) return false;
    return true;
}

int img_upload_many(img_ctx* ctx, int count, const int* var_ids, const double* const* hosts, size_t n) {
    if (!ctx || count < 0 || (count && (!var_ids || !hosts))) return fail(ctx, IMG_ERR_ARG, "bad upload argument");
    bool hosts_ok = true;
    for (int i = 0; i < count; ++i) hosts_ok = hosts_ok && hosts[i];
    if (hosts_ok && staged_ok(ctx, count, var_ids, n, IMG_VAR_MAGZ + 1)) {
        int rc = staged_transfer(ctx, count, var_ids, hosts, nullptr, n);
        if (rc != IMG_OK) return rc;
    } else {
        for (int i = 0; i < count; ++i) {
            int rc = enqueue_upload(ctx, var_ids[i], hosts[i], n);
            if (rc != IMG_OK) return rc;
        }
    }
    for (int i = 0; i < count; ++i) {
        int rc = fade_assigned(ctx, var_ids[i]);
        if (rc != IMG_OK) return rc;
    }
    CK(cudaStreamSynchronize(ctx->stream));
    return IMG_OK;
}

int img_download_many(img_ctx* ctx, int count, const int* var_ids, double* const* hosts, size_t n) {
    if (!ctx || count < 0 || (count && (!var_ids || !hosts))) return fail(ctx, IMG_ERR_ARG, "bad download argument");
    bool hosts_ok = true;
    for (int i = 0; i < count; ++i) hosts_ok = hosts_ok && hosts[i];
    if (hosts_ok && staged_ok(ctx, count, var_ids, n, NQ)) {
        int rc = staged_transfer(ctx, count, var_ids, nullptr, hosts, n);
        if (rc != IMG_OK) return rc;
    } else {
        for (int i = 0; i < count; ++i) {
            int rc = enqueue_download(ctx, var_ids[i], hosts[i], n);
            if (rc != IMG_OK) return rc;
        }
    }
    CK(cudaStreamSynchronize(ctx->stream));
    return IMG_OK;
}

int img_download(img_ctx* ctx, int var, double* host, size_t n) {
    if (!ctx) return fail(ctx, IMG_ERR_ARG, "null context");
    int rc = enqueue_download(ctx, var, host, n);
    if (rc != IMG_OK) return rc;
    CK(cudaStreamSynchronize(ctx->stream));
    return IMG_OK;
}

int img_set_state(img_ctx* ctx, const double* mass, const double* mom, const double* ener, const double* mag) {
    if (!ctx || !mass || !mom || !ener || !mag) return fail(ctx, IMG_ERR_ARG, "null state array");
    long long n = ctx->g.ncell;
    int rc;
    ctx->constructing = true;   // FluidArray/MagnetArray construction: no fades on the initial arrays
    struct Done { img_ctx* c; ~Done() { c->constructing = false; } } done{ctx};
    if ((rc = img_upload(ctx, IMG_VAR_MASS, mass, n)) != IMG_OK) return rc;
    for (int c = 0; c < 3; ++c)
        if ((rc = img_upload(ctx, IMG_VAR_MOMX + c, mom + c * n, n)) != IMG_OK) return rc;
    if ((rc = img_upload(ctx, IMG_VAR_ENER, ener, n)) != IMG_OK) return rc;
    for (int c = 0; c < 3; ++c)
        if ((rc = img_upload(ctx, IMG_VAR_MAGX + c, mag + c * n, n)) != IMG_OK) return rc;
    // primary stored edges from the initial condition (Edges.m:37-110 at FluidArray/MagnetArray creation)
    std::vector<double> face;
    const double* prim8[8] = {mass, mom, mom + n, mom + 2 * n, mag, mag + n, mag + 2 * n, ener};
    const int pobj[8] = {OBJ_PRIM_MASS, OBJ_PRIM_MOM, OBJ_PRIM_MOM + 1, OBJ_PRIM_MOM + 2, OBJ_PRIM_MAG, OBJ_PRIM_MAG + 1,
                         OBJ_PRIM_MAG + 2, OBJ_PRIM_ENER};
    for (int k = 0; k < 8; ++k)
        for (int e = 0; e < ctx->g.ndims; ++e)
            for (int s = 0; s < 2; ++s) {
                double* dst = ctx->edges_host.p[pobj[k]][e][s];
                if (!dst) continue;
                host_face(ctx->g, prim8[k], e, s == 0 ? 0 : ctx->g.n[e] - 1, face);
                CK(cudaMemcpyAsync(dst, face.data(), face.size() * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
                CK(cudaStreamSynchronize(ctx->stream));
            }
    // MagnetArray.isZero (MagnetArray.m:44): all-zero component while the magnet is inactive
    ctx->mhd = ctx->cfg.magnet_active ? 1 : 0;
    for (int c = 0; c < 3; ++c) {
        double sum = 0.0;
        for (long long i = 0; i < n; ++i) sum += mag[c * n + i];
        bool isZero = (sum == 0.0) && !ctx->cfg.magnet_active;
        ctx->use_b[c] = !isZero;
        if (!isZero) ctx->mhd = 1;
    }
    if ((rc = ctx->elem == 8 ? cellmag_init<double>(ctx) : cellmag_init<float>(ctx)) != IMG_OK) return rc;
    // Radiation.initialize after the arrays exist (imogen.m:46 -> ImogenManager.initialize)
    if (ctx->cfg.radiation_type != IMG_RAD_NONE &&
        (rc = ctx->elem == 8 ? radiation_initialize<double>(ctx) : radiation_initialize<float>(ctx)) != IMG_OK)
        return rc;
    CK(cudaStreamSynchronize(ctx->stream));
    ctx->state_set = true;
    ctx->cfl_valid = false;
    // new FluidArray/MagnetArray objects: their InitializedArrays take edges at first assignment
    ctx->init_store = ctx->init_flux = true;
    for (auto& r : ctx->init_mag)
        for (auto& v : r) v = true;
    return IMG_OK;
}

int img_time_update(img_ctx* ctx, int flux_direction, double* dt_out, int* dir_out) {
    if (!ctx) return fail(ctx, IMG_ERR_ARG, "null context");
    if (!ctx->state_set) return fail(ctx, IMG_ERR_STATE, "state not set");
    int rc = time_update_async(ctx, flux_direction);
    if (rc != IMG_OK) return rc;
    if (dt_out || dir_out) {
        if ((rc = check_dev_error(ctx)) != IMG_OK) return rc;
        if (dt_out) *dt_out = ctx->host_tm->dt;
        if (dir_out) *dir_out = ctx->host_tm->grid_index;
    }
    return IMG_OK;
}

int img_flux(img_ctx* ctx, int order) {
    if (!ctx) return fail(ctx, IMG_ERR_ARG, "null context");
    if (!ctx->state_set) return fail(ctx, IMG_ERR_STATE, "state not set");
    if (order != 1 && order != -1) return fail(ctx, IMG_ERR_ARG, "%d is not a recognized direction", order);
    ctx->cfl_valid = false;
    return do_flux(ctx, order, false);
}

int img_source(img_ctx* ctx) {
    if (!ctx) return fail(ctx, IMG_ERR_ARG, "null context");
    if (!ctx->state_set) return fail(ctx, IMG_ERR_STATE, "state not set");
    if (ctx->cfg.radiation_type == IMG_RAD_NONE) return IMG_OK;
    ctx->cfl_valid = false;
    return source_sink(ctx, false);
}

int img_treadmill(img_ctx* ctx) {
    if (!ctx) return fail(ctx, IMG_ERR_ARG, "null context");
    if (!ctx->state_set) return fail(ctx, IMG_ERR_STATE, "state not set");
    if (ctx->cfg.treadmill <= 0) return IMG_OK;
    ctx->cfl_valid = false;
    return treadmill_grid(ctx);
}

int img_treadmill_history(img_ctx* ctx, int* out, int cap, int* count, int* last) {
    if (!ctx || (cap > 0 && !out)) return fail(ctx, IMG_ERR_ARG, "null argument");
    CK(cudaMemcpyAsync(ctx->host_tm, ctx->tm, sizeof(DevTime), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    const int n = ctx->host_tm->tread_count;
    const int k = std::min(std::min(cap, n), kTreadHistCap);
    if (k > 0) {
        CK(cudaMemcpyAsync(out, ctx->tread_hist, sizeof(int) * k, cudaMemcpyDeviceToHost, ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
    }
    if (count) *count = n;
    if (last) *last = ctx->host_tm->tread_last;
    return IMG_OK;
}

int img_save_slice(img_ctx* ctx, const char* path, const img_slice_meta* meta) {
    if (!ctx || !path || !meta) return fail(ctx, IMG_ERR_ARG, "null argument");
    if (!ctx->state_set) return fail(ctx, IMG_ERR_STATE, "state not set");
    const long long n = ctx->g.ncell;
    std::vector<double> mass(n), mom(3 * n), ener(n), mag(3 * n);
    int ids[8] = {IMG_VAR_MASS, IMG_VAR_MOMX, IMG_VAR_MOMY, IMG_VAR_MOMZ, IMG_VAR_ENER, IMG_VAR_MAGX, IMG_VAR_MAGY,
                  IMG_VAR_MAGZ};
    double* hosts[8] = {mass.data(), mom.data(), mom.data() + n, mom.data() + 2 * n, ener.data(), mag.data(),
                        mag.data() + n, mag.data() + 2 * n};
    int rc = img_download_many(ctx, 8, ids, hosts, (size_t)n);
    if (rc != IMG_OK) return rc;
    CK(cudaMemcpyAsync(ctx->host_tm, ctx->tm, sizeof(DevTime), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    const DevTime tm = *ctx->host_tm;
    // the save follows the iteration it records: run.time.iteration = iterations completed
    const int iter = ctx->iteration - 1;
    const int nh = std::max(0, std::min(iter, tm.dt_hist_cap));
    std::vector<double> hist(nh);
    if (nh) {
        CK(cudaMemcpyAsync(hist.data(), ctx->dt_hist, sizeof(double) * nh, cudaMemcpyDeviceToHost, ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
    }
    std::vector<int> th(std::min(tm.tread_count, kTreadHistCap));
    if (!th.empty()) {
        CK(cudaMemcpyAsync(th.data(), ctx->tread_hist, sizeof(int) * th.size(), cudaMemcpyDeviceToHost, ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
    }
    img_slice_state st{};
    for (int d = 0; d < 3; ++d) {
        st.grid[d] = ctx->g.n[d];
        st.dgrid[d] = ctx->cfg.dgrid[d];
    }
    st.gamma = ctx->cfg.gamma;
    st.time = tm.time;
    st.iteration = iter;
    st.iter_max = ctx->cfg.iter_max;
    st.time_max = ctx->cfg.time_max;
    st.dt_history = hist.data();
    st.n_history = nh;
    st.magnet_active = ctx->cfg.magnet_active;
    st.mass = mass.data();
    st.mom = mom.data();
    st.ener = ener.data();
    st.mag = mag.data();
    st.treadmill = ctx->cfg.treadmill;
    st.tread_history = th.data();
    st.n_tread = (int)th.size();
    img_slice_meta m = *meta;
    char started[32];
    if (!m.started) {   // datestr(clock) default form, local time
        std::tm lt{};
        localtime_r(&ctx->created, &lt);
        std::strftime(started, sizeof started, "%d-%b-%Y %H:%M:%S", &lt);
        m.started = started;
    }
    rc = img_slice_write(path, &m, &st);
    if (rc != IMG_OK) return fail(ctx, rc, "%s", img_slice_last_error());
    return IMG_OK;
}

int img_load_slice(img_ctx* ctx, const char* path) {
    if (!ctx || !path) return fail(ctx, IMG_ERR_ARG, "null argument");
    int grid[3];
    int rc = img_slice_read(path, grid, nullptr, nullptr, nullptr, nullptr, nullptr);
    if (rc != IMG_OK) return fail(ctx, rc, "%s", img_slice_last_error());
    if (grid[0] != ctx->g.n[0] || grid[1] != ctx->g.n[1] || grid[2] != ctx->g.n[2])
        return fail(ctx, IMG_ERR_ARG, "slice of %dx%dx%d cells, context grid %dx%dx%d", grid[0], grid[1], grid[2],
                    ctx->g.n[0], ctx->g.n[1], ctx->g.n[2]);
    const long long n = ctx->g.ncell;
    std::vector<double> mass(n), mom(3 * n), ener(n), mag(3 * n);
    rc = img_slice_read(path, grid, mass.data(), mom.data(), ener.data(), mag.data(), nullptr);
    if (rc != IMG_OK) return fail(ctx, rc, "%s", img_slice_last_error());
    return img_set_state(ctx, mass.data(), mom.data(), ener.data(), mag.data());
}

int img_radiation_strength(img_ctx* ctx, double* strength) {
    if (!ctx || !strength) return fail(ctx, IMG_ERR_ARG, "null argument");
    CK(cudaMemcpyAsync(ctx->host_tm, ctx->tm, sizeof(DevTime), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    *strength = ctx->host_tm->rad_strength;
    return IMG_OK;
}

int img_fluid_sweep(img_ctx* ctx, int X) {
    if (!ctx || X < 1 || X > 3) return fail(ctx, IMG_ERR_ARG, "bad sweep direction");
    if (!ctx->state_set) return fail(ctx, IMG_ERR_STATE, "state not set");
    if (ctx->g.n[X - 1] < 3) return fail(ctx, IMG_ERR_ARG, "dimension %d has fewer than 3 cells", X);
    ctx->cfl_valid = false;
    return fluid_sweep(ctx, X, false);
}

int img_magnet_sweep(img_ctx* ctx, int X, int I1, int I2) {
    if (!ctx || X < 1 || X > 3 || I1 < 1 || I1 > 3 || I2 < 1 || I2 > 3 || I1 == X || I2 == X || I1 == I2)
        return fail(ctx, IMG_ERR_ARG, "bad magnet sweep indices");
    if (!ctx->state_set) return fail(ctx, IMG_ERR_STATE, "state not set");
    if (!ctx->cfg.magnet_active) return fail(ctx, IMG_ERR_STATE, "magnet is not active");
    ctx->cfl_valid = false;
    return magnet_sweep(ctx, X, I1, I2);
}

// Whether the next iteration's launch sequence is the steady one a graph can replay: every
// InitializedArray has had its first assignment (no edge-capture flags left in the arguments).
static bool steady(const img_ctx* ctx) {
    if (ctx->cfg.treadmill > 0) return false;   // treadmillGrid depends on the host iteration count
    if (ctx->init_store || ctx->init_flux) return !ctx->cfg.fluid_active;
    for (int c = 0; c < 3; ++c)
        for (int X = 0; X < 3; ++X)
            if (c != X && ctx->cfg.magnet_active && ctx->init_mag[c][X] && ctx->g.n[X] >= 3) return false;
    return true;
}

int img_step(img_ctx* ctx) {
    if (!ctx) return fail(ctx, IMG_ERR_ARG, "null context");
    if (!ctx->state_set) return fail(ctx, IMG_ERR_STATE, "state not set");
    int row = (ctx->iteration - 1) % 6;
    if (ctx->use_graphs && steady(ctx)) {
        const int cv = ctx->cfl_valid ? 1 : 0;
        if (!ctx->graphs[cv][row]) {
            uint64_t l0 = ctx->launches;
            CK(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
            int rc = enqueue_iteration(ctx);
            cudaGraph_t graph = nullptr;
            cudaError_t ce = cudaStreamEndCapture(ctx->stream, &graph);
            if (rc != IMG_OK) {
                if (graph) cudaGraphDestroy(graph);
                return rc;
            }
            if (ce != cudaSuccess) return fail(ctx, IMG_ERR_CUDA, "graph capture: %s", cudaGetErrorString(ce));
            cudaGraphExec_t exec = nullptr;
            ce = cudaGraphInstantiate(&exec, graph, 0);
            cudaGraphDestroy(graph);
            if (ce != cudaSuccess) return fail(ctx, IMG_ERR_CUDA, "graph instantiate: %s", cudaGetErrorString(ce));
            ctx->graphs[cv][row] = exec;
            ctx->graph_launches[cv][row] = ctx->launches - l0;
            ctx->launches = l0;   // counted when replayed
        }
        CK(cudaGraphLaunch(ctx->graphs[cv][row], ctx->stream));
        ctx->launches += ctx->graph_launches[cv][row];
        ctx->cfl_valid = cfl_valid_after_iteration(ctx);
        ctx->iteration += 1;
        return IMG_OK;
    }
    int rc = enqueue_iteration(ctx);
    if (rc != IMG_OK) return rc;
    ctx->iteration += 1;
    return IMG_OK;
}

int img_run(img_ctx* ctx, int max_iters, int* iters_done) {
    if (!ctx) return fail(ctx, IMG_ERR_ARG, "null context");
    if (!ctx->state_set) return fail(ctx, IMG_ERR_STATE, "state not set");
    int n = 0, rc;
    while (ctx->iteration <= ctx->cfg.iter_max && (max_iters < 0 || n < max_iters)) {
        // TimeManager.running: time < TIMEMAX (checked on the device copy every iteration)
        if ((rc = check_dev_error(ctx)) != IMG_OK) return rc;
        if (!(ctx->host_tm->time < ctx->host_tm->time_max)) break;
        if ((rc = img_step(ctx)) != IMG_OK) return rc;
        ++n;
    }
    if ((rc = check_dev_error(ctx)) != IMG_OK) return rc;
    if (iters_done) *iters_done = n;
    return IMG_OK;
}

int img_get_time(img_ctx* ctx, double* time, double* dt, int* iteration) {
    if (!ctx) return fail(ctx, IMG_ERR_ARG, "null context");
    int rc = check_dev_error(ctx);
    if (time) *time = ctx->host_tm->time;
    if (dt) *dt = ctx->host_tm->dt;
    if (iteration) *iteration = ctx->iteration;
    return rc;
}

int img_set_time(img_ctx* ctx, double time, double dt, int iteration) {
    if (!ctx) return fail(ctx, IMG_ERR_ARG, "null context");
    CK(cudaMemcpyAsync(ctx->host_tm, ctx->tm, sizeof(DevTime), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    ctx->host_tm->time = time;
    ctx->host_tm->dt = dt;
    ctx->host_tm->done = 0;
    ctx->host_tm->error = 0;
    ctx->host_tm->iters_run = iteration - 1;
    CK(cudaMemcpyAsync(ctx->tm, ctx->host_tm, sizeof(DevTime), cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    ctx->iteration = iteration;
    return IMG_OK;
}

int img_progress(img_ctx* ctx, double* time, int* iterations_run, int* stopped) {
    if (!ctx) return fail(ctx, IMG_ERR_ARG, "null context");
    int rc = check_dev_error(ctx);
    if (time) *time = ctx->host_tm->time;
    if (iterations_run) *iterations_run = ctx->host_tm->iters_run;
    if (stopped) *stopped = ctx->host_tm->done || ctx->iteration > ctx->cfg.iter_max;
    return rc;
}

// ---- checkpoint / resume ------------------------------------------------------------------------
// A checkpoint is the context's whole device slab (state, stored edges, device clock, scratch) plus
// the host-side bookkeeping that decides the next launches (first-assignment flags, CFL validity,
// iteration), behind a header that carries the configuration; it resumes bit for bit in a
// context created with the same configuration.
namespace {
struct CheckpointHeader {
    char magic[8];
    uint32_t version;
    uint32_t header_bytes;
    uint64_t slab_bytes;
    img_config cfg;
    int state_set, init_store, init_flux, cfl_valid, iteration, mhd;
    int init_mag[3][3];
    int use_b[3];
};
const char kCheckpointMagic[8] = {'I', 'M', 'G', 'B', '2', '0', '0', 'C'};
}  // namespace

size_t img_checkpoint_bytes(const img_ctx* ctx) { return ctx ? sizeof(CheckpointHeader) + ctx->slab_bytes : 0; }

int img_checkpoint_save(img_ctx* ctx, void* host, size_t bytes) {
    if (!ctx || !host) return fail(ctx, IMG_ERR_ARG, "null argument");
    if (bytes < img_checkpoint_bytes(ctx)) return fail(ctx, IMG_ERR_ARG, "checkpoint buffer too small");
    CheckpointHeader h{};
    std::memcpy(h.magic, kCheckpointMagic, 8);
    h.version = 1;
    h.header_bytes = sizeof h;
    h.slab_bytes = ctx->slab_bytes;
    h.cfg = ctx->cfg;
    h.state_set = ctx->state_set;
    h.init_store = ctx->init_store;
    h.init_flux = ctx->init_flux;
    h.cfl_valid = ctx->cfl_valid;
    h.iteration = ctx->iteration;
    h.mhd = ctx->mhd;
    for (int i = 0; i < 3; ++i) {
        h.use_b[i] = ctx->use_b[i];
        for (int j = 0; j < 3; ++j) h.init_mag[i][j] = ctx->init_mag[i][j];
    }
    std::memcpy(host, &h, sizeof h);
    CK(cudaMemcpyAsync(static_cast<char*>(host) + sizeof h, ctx->slab, ctx->slab_bytes, cudaMemcpyDeviceToHost,
                       ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return IMG_OK;
}

int img_checkpoint_load(img_ctx* ctx, const void* host, size_t bytes) {
    if (!ctx || !host) return fail(ctx, IMG_ERR_ARG, "null argument");
    if (ctx->batch) return fail(ctx, IMG_ERR_STATE, "cannot load a checkpoint into a batch member");
    CheckpointHeader h;
    if (bytes < sizeof h) return fail(ctx, IMG_ERR_ARG, "checkpoint too short");
    std::memcpy(&h, host, sizeof h);
    if (std::memcmp(h.magic, kCheckpointMagic, 8) || h.version != 1 || h.header_bytes != sizeof h)
        return fail(ctx, IMG_ERR_ARG, "not an imogen_b200 checkpoint of this version");
    if (h.slab_bytes != ctx->slab_bytes || bytes < sizeof h + h.slab_bytes ||
        std::memcmp(&h.cfg, &ctx->cfg, sizeof(img_config)) != 0)
        return fail(ctx, IMG_ERR_ARG, "checkpoint was written by a context with another configuration");
    CK(cudaStreamSynchronize(ctx->stream));
    CK(cudaMemcpyAsync(ctx->slab, static_cast<const char*>(host) + sizeof h, ctx->slab_bytes, cudaMemcpyHostToDevice,
                       ctx->stream));
    // the stored-edge table and the time record hold device addresses: this context's own, not the writer's
    CK(cudaMemcpyAsync(ctx->edges_dev, &ctx->edges_host, sizeof(EdgeTable), cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemcpyAsync(&ctx->tm->dt_hist, &ctx->dt_hist, sizeof(double*), cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    ctx->state_set = h.state_set != 0;
    ctx->init_store = h.init_store != 0;
    ctx->init_flux = h.init_flux != 0;
    ctx->cfl_valid = h.cfl_valid != 0;
    ctx->iteration = h.iteration;
    ctx->mhd = h.mhd;
    for (int i = 0; i < 3; ++i) {
        ctx->use_b[i] = h.use_b[i];
        for (int j = 0; j < 3; ++j) ctx->init_mag[i][j] = h.init_mag[i][j] != 0;
    }
    return check_dev_error(ctx);
}

int img_totals(img_ctx* ctx, double out[8]) {
    if (!ctx || !out) return fail(ctx, IMG_ERR_ARG, "null argument");
    const int nb = 1024;
    void* qp_host[8];
    for (int v = 0; v < 8; ++v) qp_host[v] = ctx->q[v];
    // the pointer table lives in the partial buffer's tail
    void** qp_dev = reinterpret_cast<void**>(ctx->partial + 2 * 8 * nb - 16);
    CK(cudaMemcpyAsync(qp_dev, qp_host, sizeof qp_host, cudaMemcpyHostToDevice, ctx->stream));
    if (ctx->elem == 8) totals_kernel<double><<<nb - 1, 256, 0, ctx->stream>>>(ctx->g, qp_dev, ctx->partial);
    else totals_kernel<float><<<nb - 1, 256, 0, ctx->stream>>>(ctx->g, qp_dev, ctx->partial);
    CK(cudaGetLastError());
    std::vector<double> part(2 * 8 * (nb - 1));
    CK(cudaMemcpyAsync(part.data(), ctx->partial, part.size() * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    for (int v = 0; v < 8; ++v) {
        double S = 0.0, C = 0.0;
        for (int b = 0; b < nb - 1; ++b) {
            double x = part[(b * 8 + v) * 2];
            double t = S + x;
            C += std::fabs(S) >= std::fabs(x) ? (S - t) + x : (x - t) + S;
            S = t;
            C += part[(b * 8 + v) * 2 + 1];
        }
        out[v] = S + C;
    }
    return IMG_OK;
}

}  // extern "C"

// ---- batches: many grids advanced by batched launches ------------------------------------------------
// A batch advances all its member contexts by one iteration per img_batch_step.  The members' own
// launch sequences are recorded (the same host code as img_step, so every member's kernel
// arguments are exactly those of its own launches), and launch k of every member becomes part of
// ONE batched launch (one per group of members that share a launch shape), driven by per-CTA block
// maps and per-member argument blocks in a device arena.  Steady iterations are captured once per
// (CFL-valid, sweep-order row) into a CUDA graph and replayed.  Every member keeps its own time
// step on the device.

struct BatchItem {            // one batched launch
    int kind = 0, elem = 0;
    int op = 0;               // index of the members' launch it batches (the groups of one op run side by side)
    bool mhd = false;
    PencilLaunch L{};         // pencil kernels: the shared shape; grid_x = CTAs of all members
    unsigned blocks = 0;      // pointwise kernels: blocks of all members
    size_t args_off = 0, map_off = 0;
    int nmembers = 0;
    int check_running = 0;
};

struct BatchPlan {            // one recorded iteration of all members
    std::vector<BatchItem> items;
    std::vector<unsigned char> host;
    void* dev = nullptr;
    size_t cap = 0;
    cudaGraphExec_t graph = nullptr;
    void release() {
        if (graph) cudaGraphExecDestroy(graph);
        if (dev) cudaFree(dev);
        graph = nullptr;
        dev = nullptr;
        cap = 0;
        items.clear();
        host.clear();
    }
};

struct img_batch {
    std::string err;
    int dev = 0;
    cudaStream_t stream = nullptr;
    std::vector<img_ctx*> members;
    // Steady plans by phase: every member's sweep-order row advances by one per step, so with fixed
    // membership the batch's launch sequence repeats every 6 steps.  Membership changes clear them.
    BatchPlan cached[6];
    BatchPlan transient[4];          // ring of arenas for plans launched once
    cudaEvent_t transient_done[4] = {};
    int next_transient = 0;
    uint64_t steps = 0;             // steps since the membership last changed
    uint64_t launches = 0;
    int* status_dev = nullptr;      // gathered done/error flags
    DevTime** tms_dev = nullptr;
    size_t status_cap = 0;
    // The launch groups of one op touch disjoint members: all but the first go to side streams forked
    // from and joined back into `stream` around the op, so their tails overlap (parallel graph branches).
    static constexpr int kSide = 4;
    cudaStream_t side[kSide] = {};
    cudaEvent_t fork_ev = nullptr;
    cudaEvent_t join_ev[kSide] = {};
};

namespace {

int bfail(img_batch* b, int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    if (b) b->err = buf;
    return code;
}

#define BCK(call)                                                                                  \
    do {                                                                                           \
        cudaError_t e_ = (call);                                                                   \
        if (e_ != cudaSuccess) return bfail(b, IMG_ERR_CUDA, "%s: %s", #call, cudaGetErrorString(e_)); \
    } while (0)

void clear_plans(img_batch* b) {
    for (auto& p : b->cached) p.release();
    b->steps = 0;
}

// Members must issue the same kinds of launches in the same order: same precision, physics, swept
// dimensions and time update mode (their sweep directions may differ: members that joined at
// other iterations sit at other rows of the sweep-order table, and go to other launch groups).
bool same_signature(const img_ctx* a, const img_ctx* c) {
    if (a->elem != c->elem || a->cfg.fluid_active != c->cfg.fluid_active ||
        a->cfg.magnet_active != c->cfg.magnet_active || a->cfg.update_mode != c->cfg.update_mode ||
        a->dev != c->dev)
        return false;
    for (int d = 0; d < 3; ++d)
        if ((a->g.n[d] >= 3) != (c->g.n[d] >= 3)) return false;
    return true;
}

size_t align16(size_t x) { return (x + 15) & ~(size_t)15; }

template <typename V>
size_t put(std::vector<unsigned char>& h, const V* v, size_t n) {
    size_t off = align16(h.size());
    h.resize(off + n * sizeof(V));
    std::memcpy(h.data() + off, v, n * sizeof(V));
    return off;
}

bool same_shape(const PencilLaunch& x, const PencilLaunch& y) {
    return x.grid_y == y.grid_y && x.block == y.block && x.smem == y.smem && x.cluster == y.cluster &&
           x.cpt == y.cpt && x.nqc == y.nqc && x.fade == y.fade && x.cg == y.cg && x.init == y.init &&
           x.seg == y.seg && x.clu == y.clu;
}

// Turn the members' records into batched launch items and the arena image.
int build_plan(img_batch* b, const std::vector<std::vector<OpRec>>& recs, BatchPlan& plan) {
    plan.items.clear();
    plan.host.clear();
    const size_t nops = recs[0].size();
    const int n = (int)recs.size();
    for (int m = 1; m < n; ++m)
        if (recs[m].size() != nops) return bfail(b, IMG_ERR_STATE, "members recorded different launch sequences");
    std::vector<int> group(n);
    for (size_t k = 0; k < nops; ++k) {
        const int kind = recs[0][k].kind;
        for (int m = 1; m < n; ++m)
            if (recs[m][k].kind != kind) return bfail(b, IMG_ERR_STATE, "members recorded different launch sequences");
        // group members by launch shape (pencil kernels) -- first-appearance order
        std::vector<int> heads;
        for (int m = 0; m < n; ++m) {
            int gi = -1;
            for (int h = 0; h < (int)heads.size() && gi < 0; ++h) {
                const OpRec& a = recs[heads[h]][k];
                const OpRec& c = recs[m][k];
                bool same = a.elem == c.elem && a.mhd == c.mhd;
                if (pencil_kind(kind)) same = same && same_shape(a.L, c.L);
                if (kind == OP_CFL_FINALIZE) same = same && a.check_running == c.check_running;
                if (same) gi = h;
            }
            if (gi < 0) {
                gi = (int)heads.size();
                heads.push_back(m);
            }
            group[m] = gi;
        }
        for (int h = 0; h < (int)heads.size(); ++h) {
            BatchItem it;
            const OpRec& r0 = recs[heads[h]][k];
            it.op = (int)k;
            it.kind = kind;
            it.elem = r0.elem;
            it.mhd = r0.mhd;
            it.L = r0.L;
            it.check_running = r0.check_running;
            std::vector<int> mem;
            for (int m = 0; m < n; ++m)
                if (group[m] == h) mem.push_back(m);
            it.nmembers = (int)mem.size();
            std::vector<BlockMap> map;
            if (kind == OP_CFL_FINALIZE) {
                std::vector<DevTime*> tms;
                for (int m : mem) tms.push_back(recs[m][k].tm);
                it.args_off = put(plan.host, tms.data(), tms.size());
            } else {
                for (int j = 0; j < (int)mem.size(); ++j) {
                    const OpRec& r = recs[mem[j]][k];
                    const int nb = pencil_kind(kind) ? (int)r.L.grid_x : (int)r.blocks;
                    for (int blk = 0; blk < nb; ++blk) map.push_back(BlockMap{j, blk, nb});
                }
                if (kind == OP_FLUID) {
                    std::vector<FluidArgs> v;
                    for (int m : mem) v.push_back(recs[m][k].fa);
                    it.args_off = put(plan.host, v.data(), v.size());
                } else if (kind == OP_CFL_REDUCE) {
                    std::vector<CflArgs> v;
                    for (int m : mem) v.push_back(recs[m][k].ca);
                    it.args_off = put(plan.host, v.data(), v.size());
                } else {
                    std::vector<MagArgs> v;
                    for (int m : mem) v.push_back(recs[m][k].ma);
                    it.args_off = put(plan.host, v.data(), v.size());
                }
                it.map_off = put(plan.host, map.data(), map.size());
                if (pencil_kind(kind)) it.L.grid_x = (unsigned)map.size();
                else it.blocks = (unsigned)map.size();
            }
            it.L.stream = b->stream;
            plan.items.push_back(it);
        }
    }
    if (plan.host.size() > plan.cap) {
        if (plan.dev) BCK(cudaFree(plan.dev));
        plan.dev = nullptr;
        plan.cap = 0;
        BCK(cudaMalloc(&plan.dev, plan.host.size()));
        plan.cap = plan.host.size();
    }
    BCK(cudaMemcpyAsync(plan.dev, plan.host.data(), plan.host.size(), cudaMemcpyHostToDevice, b->stream));
    return IMG_OK;
}

template <typename T>
cudaError_t launch_item(const BatchItem& it, const unsigned char* base, cudaStream_t st) {
    PencilLaunch L = it.L;
    L.stream = st;
    switch (it.kind) {
        case OP_FLUID:
            return launch_fluid_sweep_batch<T>(reinterpret_cast<const FluidArgs*>(base + it.args_off),
                                               reinterpret_cast<const BlockMap*>(base + it.map_off), L, it.mhd);
        case OP_CHAIN:
            return launch_mag_chain_batch<T>(reinterpret_cast<const MagArgs*>(base + it.args_off),
                                             reinterpret_cast<const BlockMap*>(base + it.map_off), L);
        case OP_CTCELL:
            return launch_mag_ctcell_batch<T>(reinterpret_cast<const MagArgs*>(base + it.args_off),
                                              reinterpret_cast<const BlockMap*>(base + it.map_off), L);
        case OP_CFL_REDUCE:
            cfl_reduce_batch_kernel<T><<<it.blocks, 256, 0, st>>>(reinterpret_cast<const CflArgs*>(base + it.args_off),
                                                                 reinterpret_cast<const BlockMap*>(base + it.map_off));
            return cudaGetLastError();
        default:
            cfl_finalize_batch_kernel<<<(it.nmembers + 127) / 128, 128, 0, st>>>(
                reinterpret_cast<DevTime* const*>(base + it.args_off), it.nmembers, it.check_running);
            return cudaGetLastError();
    }
}

int launch_plan(img_batch* b, const BatchPlan& plan) {
    const unsigned char* base = static_cast<const unsigned char*>(plan.dev);
    const size_t n = plan.items.size();
    for (size_t i0 = 0; i0 < n;) {
        size_t i1 = i0 + 1;
        while (i1 < n && plan.items[i1].op == plan.items[i0].op) ++i1;
        const int groups = (int)(i1 - i0);
        const int nside = std::min(groups - 1, img_batch::kSide);
        if (nside > 0) {   // fork: the side streams start after everything before this op
            BCK(cudaEventRecord(b->fork_ev, b->stream));
            for (int j = 0; j < nside; ++j) BCK(cudaStreamWaitEvent(b->side[j], b->fork_ev, 0));
        }
        for (size_t i = i0; i < i1; ++i) {
            const BatchItem& it = plan.items[i];
            const cudaStream_t st = i == i0 ? b->stream : b->side[(i - i0 - 1) % img_batch::kSide];
            cudaError_t e = it.elem == 8 ? launch_item<double>(it, base, st) : launch_item<float>(it, base, st);
            if (e != cudaSuccess)
                return bfail(b, IMG_ERR_CUDA, "batched launch (kind %d, %d members, grid %u): %s", it.kind, it.nmembers,
                             pencil_kind(it.kind) ? it.L.grid_x : it.blocks, cudaGetErrorString(e));
        }
        for (int j = 0; j < nside; ++j) {   // join: the next op starts after every group of this one
            BCK(cudaEventRecord(b->join_ev[j], b->side[j]));
            BCK(cudaStreamWaitEvent(b->stream, b->join_ev[j], 0));
        }
        i0 = i1;
    }
    return IMG_OK;
}

__global__ void batch_status_kernel(DevTime* const* __restrict__ tms, int n, int* __restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = (tms[i]->done ? 1 : 0) | (tms[i]->error ? 2 : 0);
}

}  // namespace

extern "C" {

int img_batch_create(img_batch** out) {
    if (!out) return IMG_ERR_ARG;
    *out = nullptr;
    img_batch* b = new img_batch();
    bool ok = cudaGetDevice(&b->dev) == cudaSuccess &&
              cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) == cudaSuccess &&
              cudaEventCreateWithFlags(&b->fork_ev, cudaEventDisableTiming) == cudaSuccess;
    for (int j = 0; ok && j < img_batch::kSide; ++j)
        ok = cudaStreamCreateWithFlags(&b->side[j], cudaStreamNonBlocking) == cudaSuccess &&
             cudaEventCreateWithFlags(&b->join_ev[j], cudaEventDisableTiming) == cudaSuccess;
    if (!ok) {
        img_batch_destroy(b);
        return IMG_ERR_CUDA;
    }
    *out = b;
    return IMG_OK;
}

static void batch_detach(img_batch* b, img_ctx* m) {
    cudaStreamSynchronize(b->stream);
    m->stream = m->own_stream;
    m->batch = nullptr;
}

int img_batch_destroy(img_batch* b) {
    if (!b) return IMG_OK;
    cudaStreamSynchronize(b->stream);
    for (img_ctx* m : b->members) batch_detach(b, m);
    clear_plans(b);
    for (int i = 0; i < 4; ++i) {
        b->transient[i].release();
        if (b->transient_done[i]) cudaEventDestroy(b->transient_done[i]);
    }
    if (b->status_dev) cudaFree(b->status_dev);
    if (b->tms_dev) cudaFree(b->tms_dev);
    for (int j = 0; j < img_batch::kSide; ++j) {
        if (b->side[j]) cudaStreamDestroy(b->side[j]);
        if (b->join_ev[j]) cudaEventDestroy(b->join_ev[j]);
    }
    if (b->fork_ev) cudaEventDestroy(b->fork_ev);
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
    return IMG_OK;
}

const char* img_batch_last_error(const img_batch* b) { return b ? b->err.c_str() : ""; }

int img_batch_add(img_batch* b, img_ctx* ctx) {
    if (!b || !ctx) return bfail(b, IMG_ERR_ARG, "null argument");
    if (!ctx->state_set) return bfail(b, IMG_ERR_STATE, "member state not set");
    if (ctx->batch) return bfail(b, IMG_ERR_STATE, "context is already a batch member");
    if (ctx->dev != b->dev) return bfail(b, IMG_ERR_ARG, "member is on device %d, batch on %d", ctx->dev, b->dev);
    if (ctx->cfg.viscosity_type != IMG_VISC_NONE || ctx->cfg.radiation_type != IMG_RAD_NONE || ctx->cfg.treadmill > 0 ||
        ctx->fade_mask)
        return bfail(b, IMG_ERR_UNSUPPORTED,
                     "contexts with artificial viscosity, radiation, a treadmill or a point fade do not join batches");
    if (!b->members.empty() && !same_signature(b->members[0], ctx))
        return bfail(b, IMG_ERR_ARG, "member differs from the batch in precision, physics, swept dimensions, "
                     "time update mode or iteration");
    BCK(cudaStreamSynchronize(ctx->own_stream));
    ctx->stream = b->stream;
    ctx->batch = b;
    b->members.push_back(ctx);
    clear_plans(b);
    return IMG_OK;
}

int img_batch_remove(img_batch* b, img_ctx* ctx) {
    if (!b || !ctx || ctx->batch != b) return bfail(b, IMG_ERR_ARG, "not a member of this batch");
    batch_detach(b, ctx);
    b->members.erase(std::find(b->members.begin(), b->members.end(), ctx));
    clear_plans(b);
    return IMG_OK;
}

int img_batch_size(const img_batch* b, int* n) {
    if (!b || !n) return IMG_ERR_ARG;
    *n = (int)b->members.size();
    return IMG_OK;
}

int img_batch_step(img_batch* b) {
    if (!b) return IMG_ERR_ARG;
    if (b->members.empty()) return bfail(b, IMG_ERR_STATE, "empty batch");
    // members past ITERMAX stop (imogen.m:58): their kernels return at once from now on
    static const int one = 1;
    for (img_ctx* m : b->members)
        if (m->iteration > m->cfg.iter_max)
            BCK(cudaMemcpyAsync(&m->tm->done, &one, sizeof(int), cudaMemcpyHostToDevice, b->stream));
    // one launch sequence for all members: where some member's CFL maxima are not valid (a member that
    // just joined), the others record an empty CFL pass in its place (their maxima are left as they are)
    bool all_valid = true;
    for (img_ctx* m : b->members) all_valid = all_valid && m->cfl_valid;
    for (img_ctx* m : b->members) m->pad_cfl = !all_valid && m->cfl_valid;
    bool st = true;
    for (img_ctx* m : b->members) st = st && steady(m) && m->cfl_valid == b->members[0]->cfl_valid;
    const int phase = (int)(b->steps % 6);
    BatchPlan& cp = b->cached[phase];
    if (st && cp.graph) {
        BCK(cudaGraphLaunch(cp.graph, b->stream));
        b->launches += cp.items.size();
        for (img_ctx* m : b->members) {
            m->cfl_valid = cfl_valid_after_iteration(m);
            m->iteration += 1;
        }
        b->steps += 1;
        return IMG_OK;
    }
    std::vector<std::vector<OpRec>> recs(b->members.size());
    for (size_t i = 0; i < b->members.size(); ++i) {
        img_ctx* m = b->members[i];
        m->rec = &recs[i];
        int rc = enqueue_iteration(m);
        m->rec = nullptr;
        if (rc != IMG_OK) return bfail(b, rc, "member %zu: %s", i, m->err.c_str());
    }
    // a steady plan is kept (and captured as a graph) from the second cycle of a membership on,
    // so that a batch whose members change often does not pay for captures it never replays
    const bool keep = st && b->steps >= 6;
    const int tr = b->next_transient;
    BatchPlan& plan = keep ? cp : b->transient[tr];
    if (!keep) {   // wait until this arena's previous launches have finished with it
        if (!b->transient_done[tr]) BCK(cudaEventCreateWithFlags(&b->transient_done[tr], cudaEventDisableTiming));
        else BCK(cudaEventSynchronize(b->transient_done[tr]));
        b->next_transient = (tr + 1) % 4;
    }
    int rc = build_plan(b, recs, plan);
    if (rc != IMG_OK) return rc;
    if (keep) {
        BCK(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
        rc = launch_plan(b, plan);
        cudaGraph_t graph = nullptr;
        cudaError_t ce = cudaStreamEndCapture(b->stream, &graph);
        if (rc != IMG_OK) {
            if (graph) cudaGraphDestroy(graph);
            return rc;
        }
        if (ce != cudaSuccess) return bfail(b, IMG_ERR_CUDA, "graph capture: %s", cudaGetErrorString(ce));
        ce = cudaGraphInstantiate(&plan.graph, graph, 0);
        cudaGraphDestroy(graph);
        if (ce != cudaSuccess) return bfail(b, IMG_ERR_CUDA, "graph instantiate: %s", cudaGetErrorString(ce));
        BCK(cudaGraphLaunch(plan.graph, b->stream));
    } else {
        rc = launch_plan(b, plan);
        if (rc != IMG_OK) return rc;
        BCK(cudaEventRecord(b->transient_done[tr], b->stream));
    }
    b->launches += plan.items.size();
    for (img_ctx* m : b->members) m->iteration += 1;
    b->steps += 1;
    return IMG_OK;
}

// Done/error flags of every member (bit 0: stopped, bit 1: error), after a stream sync.
int img_batch_status(img_batch* b, int* flags, int n) {
    if (!b || !flags || n != (int)b->members.size()) return bfail(b, IMG_ERR_ARG, "bad status buffer");
    if (n == 0) return IMG_OK;
    if ((size_t)n > b->status_cap) {
        if (b->status_dev) cudaFree(b->status_dev);
        if (b->tms_dev) cudaFree(b->tms_dev);
        b->status_dev = nullptr;
        b->tms_dev = nullptr;
        b->status_cap = 0;
        BCK(cudaMalloc(&b->status_dev, sizeof(int) * n));
        BCK(cudaMalloc(&b->tms_dev, sizeof(DevTime*) * n));
        b->status_cap = n;
    }
    std::vector<DevTime*> tms;
    for (img_ctx* m : b->members) tms.push_back(m->tm);
    BCK(cudaMemcpyAsync(b->tms_dev, tms.data(), sizeof(DevTime*) * n, cudaMemcpyHostToDevice, b->stream));
    batch_status_kernel<<<(n + 127) / 128, 128, 0, b->stream>>>(b->tms_dev, n, b->status_dev);
    BCK(cudaGetLastError());
    BCK(cudaMemcpyAsync(flags, b->status_dev, sizeof(int) * n, cudaMemcpyDeviceToHost, b->stream));
    BCK(cudaStreamSynchronize(b->stream));
    for (int i = 0; i < n; ++i)
        if (b->members[i]->iteration > b->members[i]->cfg.iter_max) flags[i] |= 1;
    return IMG_OK;
}

int img_batch_run(img_batch* b, int max_iters, int check_every, int* iters_done) {
    if (!b) return IMG_ERR_ARG;
    if (check_every < 1) check_every = 1;
    std::vector<int> flags(b->members.size());
    int n = 0, rc;
    while (max_iters < 0 || n < max_iters) {
        if (n % check_every == 0) {
            if ((rc = img_batch_status(b, flags.data(), (int)flags.size())) != IMG_OK) return rc;
            bool all = true;
            for (int f : flags) all = all && (f & 1 || f & 2);
            if (all) break;
        }
        if ((rc = img_batch_step(b)) != IMG_OK) return rc;
        ++n;
    }
    if ((rc = img_batch_status(b, flags.data(), (int)flags.size())) != IMG_OK) return rc;
    if (iters_done) *iters_done = n;
    for (size_t i = 0; i < flags.size(); ++i)
        if (flags[i] & 2) {   // report the first failed member's own status (CFL or non-finite)
            int mrc = check_dev_error(b->members[i]);
            return bfail(b, mrc != IMG_OK ? mrc : IMG_ERR_CFL, "member %zu stopped with an error: %s", i,
                         img_last_error(b->members[i]));
        }
    return IMG_OK;
}

int img_batch_get_stream(img_batch* b, void** stream) {
    if (!b || !stream) return IMG_ERR_ARG;
    *stream = (void*)b->stream;
    return IMG_OK;
}

int img_batch_launch_count(const img_batch* b, uint64_t* count) {
    if (!b || !count) return IMG_ERR_ARG;
    *count = b->launches;
    return IMG_OK;
}

// ---- totals with static scratch -------------------------------------------------------------------
// img_totals_static works in a file-scope device array instead of the context's slab: the 1023
// per-block partial pairs (sum, compensation) of 8 variables, the 8 results and the 8-entry pointer
// table: 2*8*1023 + 8 + 8 = 16384 doubles, 128 KiB exactly, whatever the grid size (the reduction is
// a grid-stride loop over a fixed 1023 blocks).  Every call overwrites every slot it later reads, so
// nothing must start at zero.  All contexts of a device share the one array: calls that overlap in
// time (other threads, other streams) race on it and must be serialised by the caller.
namespace {
constexpr int kStaticTotalsBlocks = 1023;
constexpr size_t kStaticTotalsPartial = 2 * 8 * kStaticTotalsBlocks;
constexpr size_t kStaticTotalsDoubles = kStaticTotalsPartial + 8 + 8;
constexpr int kMaxDevices = 64;
}  // namespace

static __device__ __align__(256) double g_static_totals[kStaticTotalsDoubles];
static_assert(sizeof(g_static_totals) == 128 * 1024, "static totals scratch is 128 KiB");

// Address of g_static_totals on the current device, looked up once per device.
static int static_totals_scratch(img_ctx* ctx, double** out) {
    static std::mutex mu;
    static double* addr[kMaxDevices] = {};
    int cur = -1;
    if (cudaGetDevice(&cur) != cudaSuccess) return fail(ctx, IMG_ERR_CUDA, "cudaGetDevice failed");
    if (cur != ctx->dev)
        return fail(ctx, IMG_ERR_ARG, "current device %d is not the context's device %d", cur, ctx->dev);
    if (cur < 0 || cur >= kMaxDevices) return fail(ctx, IMG_ERR_UNSUPPORTED, "device ordinal %d >= %d", cur, kMaxDevices);
    std::lock_guard<std::mutex> lock(mu);
    if (!addr[cur]) {
        void* a = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&a, g_static_totals);
        if (e != cudaSuccess || !a)
            return fail(ctx, IMG_ERR_CUDA, "cudaGetSymbolAddress(static totals scratch): %s", cudaGetErrorString(e));
        addr[cur] = static_cast<double*>(a);
    }
    *out = addr[cur];
    return IMG_OK;
}

int img_totals_static(img_ctx* ctx, double out[8]) {
    if (!ctx || !out) return fail(ctx, IMG_ERR_ARG, "null argument");
    // it copies from a host stack array and synchronises: neither may be captured into a graph
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    CK(cudaStreamIsCapturing(ctx->stream, &cs));
    if (cs != cudaStreamCaptureStatusNone)
        return fail(ctx, IMG_ERR_STATE, "img_totals_static cannot run while the context's stream is captured");
    double* scratch = nullptr;
    int rc = static_totals_scratch(ctx, &scratch);
    if (rc != IMG_OK) return rc;
    double* partial = scratch;
    double* result = scratch + kStaticTotalsPartial;
    void** table = reinterpret_cast<void**>(result + 8);
    void* qp_host[8];
    for (int v = 0; v < 8; ++v) qp_host[v] = ctx->q[v];
    CK(cudaMemcpyAsync(table, qp_host, sizeof qp_host, cudaMemcpyHostToDevice, ctx->stream));
    if (ctx->elem == 8) totals_kernel<double><<<kStaticTotalsBlocks, 256, 0, ctx->stream>>>(ctx->g, table, partial);
    else totals_kernel<float><<<kStaticTotalsBlocks, 256, 0, ctx->stream>>>(ctx->g, table, partial);
    CK(cudaGetLastError());
    totals_finalize_kernel<<<1, 32, 0, ctx->stream>>>(partial, kStaticTotalsBlocks, result);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(out, result, 8 * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return IMG_OK;
}

int img_get_stream(img_ctx* ctx, void** stream) {
    if (!ctx || !stream) return fail(ctx, IMG_ERR_ARG, "null argument");
    *stream = (void*)ctx->stream;
    return IMG_OK;
}

static void drop_graphs(img_ctx* ctx) {
    for (auto& row : ctx->graphs)
        for (auto& gx : row)
            if (gx) {
                cudaGraphExecDestroy(gx);
                gx = nullptr;
            }
}

int img_autotune(img_ctx* ctx, int trials) {
    if (!ctx) return fail(ctx, IMG_ERR_ARG, "null context");
    if (!ctx->state_set) return fail(ctx, IMG_ERR_STATE, "state not set");
    if (ctx->batch) return fail(ctx, IMG_ERR_STATE, "cannot tune a batch member");
    if (trials < 1) trials = 3;
    CK(cudaStreamSynchronize(ctx->stream));
    void* backup = nullptr;
    if (cudaMalloc(&backup, ctx->slab_bytes) != cudaSuccess) {
        cudaGetLastError();
        return fail(ctx, IMG_ERR_NOMEM, "autotune needs a %zu-byte copy of the context", ctx->slab_bytes);
    }
    const bool s_store = ctx->init_store, s_flux = ctx->init_flux, s_cfl = ctx->cfl_valid;
    bool s_mag[3][3];
    std::memcpy(s_mag, ctx->init_mag, sizeof s_mag);
    const uint64_t s_launches = ctx->launches;
    auto restore = [&]() {
        cudaMemcpyAsync(ctx->slab, backup, ctx->slab_bytes, cudaMemcpyDeviceToDevice, ctx->stream);
        ctx->init_store = s_store;
        ctx->init_flux = s_flux;
        ctx->cfl_valid = s_cfl;
        std::memcpy(ctx->init_mag, s_mag, sizeof s_mag);
    };
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    int rc = IMG_OK;
    if (cudaMemcpyAsync(backup, ctx->slab, ctx->slab_bytes, cudaMemcpyDeviceToDevice, ctx->stream) != cudaSuccess ||
        cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess)
        rc = fail(ctx, IMG_ERR_CUDA, "autotune setup failed");
    // each kernel is tuned on its own sweeps: the fluid sweep for the fluid tiling, the magnet sweep
    // for the chain's tiling (the CT on its current one), then the magnet sweep for the CT's tiling
    // with the chain's chosen
    for (int kind = 0; kind < 3 && rc == IMG_OK; ++kind) {
        if (kind == 0 ? !ctx->cfg.fluid_active : !ctx->cfg.magnet_active) continue;
        for (int d = 0; d < 3 && rc == IMG_OK; ++d) {
            if (ctx->g.n[d] < 3) continue;
            PencilCfg best = ctx->pcfg[kind][d];
            float best_ms = 1e30f;
            const bool visc = kind == 0 && ctx->cfg.viscosity_type != IMG_VISC_NONE;   // segment tilings only
            std::vector<PencilCfg> cands = visc ? std::vector<PencilCfg>() : pencil_candidates(ctx->g, d, ctx->elem);
            if (kind == 0)
                for (const PencilCfg& sc : seg_candidates(ctx->g, d, ctx->elem, visc)) cands.push_back(sc);
            if (kind == 1) {   // (window tilings carry both components per thread: no nqc = 2 variant)   // the chain may also take both transverse components per CTA
                const size_t n0 = cands.size();
                for (size_t i = 0; i < n0; ++i)
                    if (cands[i].cpt <= 2) {
                        PencilCfg c2 = cands[i];
                        c2.nqc = 2;
                        cands.push_back(c2);
                    }
            }
            if (kind != 0)
                for (const PencilCfg& wc : win_candidates(ctx->g, d)) cands.push_back(wc);
            for (const PencilCfg& cand : cands) {
                ctx->pcfg[kind][d] = cand;
                if (!cand.seg) {   // segment tilings are one CTA with checked shared memory
                    int ncl = 0;
                    const size_t fs = ctx->elem == 8 ? fluid_smem_bytes<double>(cand.G * cand.cpt, cand.Wb)
                                                     : fluid_smem_bytes<float>(cand.G * cand.cpt, cand.Wb);
                    PencilLaunch L = ctx->elem == 8 ? pencil_launch<double>(ctx, cand, d, fs, 1, false)
                                                    : pencil_launch<float>(ctx, cand, d, fs, 1, false);
                    cudaError_t ce = ctx->elem == 8 ? fluid_max_clusters<double>(L, &ncl) : fluid_max_clusters<float>(L, &ncl);
                    if (ce != cudaSuccess || ncl < 1) {
                        cudaGetLastError();
                        continue;
                    }
                }
                auto sweep = [&]() {
                    return kind == 0 ? fluid_sweep(ctx, d + 1, false)
                                     : magnet_sweep(ctx, d + 1, FWD_MI[d][0], FWD_MI[d][1]);
                };
                bool ok = sweep() == IMG_OK;                                   // warm-up
                ok = ok && cudaEventRecord(e0, ctx->stream) == cudaSuccess;
                for (int t = 0; ok && t < trials; ++t) ok = sweep() == IMG_OK;
                ok = ok && cudaEventRecord(e1, ctx->stream) == cudaSuccess && cudaEventSynchronize(e1) == cudaSuccess;
                float ms = 0.f;
                ok = ok && cudaEventElapsedTime(&ms, e0, e1) == cudaSuccess;
                restore();
                if (!ok) {
                    cudaGetLastError();
                    continue;
                }
                if (ms < best_ms) {
                    best_ms = ms;
                    best = cand;
                }
            }
            ctx->pcfg[kind][d] = best;
            std::lock_guard<std::mutex> lock(g_tune_mu);
            g_tuned[tune_key(kind, ctx->g, d, ctx->elem, ctx->cfg)] = best;
        }
    }
    restore();
    cudaStreamSynchronize(ctx->stream);
    ctx->launches = s_launches;
    drop_graphs(ctx);   // captured with the old tilings
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    cudaFree(backup);
    return rc != IMG_OK ? rc : check_dev_error(ctx);
}

int img_set_tiling(img_ctx* ctx, int dim, const int cfg[7]) {
    if (!ctx || !cfg || dim < 1 || dim > 6) return fail(ctx, IMG_ERR_ARG, "bad tiling argument");
    if (ctx->batch) return fail(ctx, IMG_ERR_STATE, "cannot retile a batch member");
    const int kind = (dim - 1) / 3, d = (dim - 1) % 3;
    const int nqc = cfg[5];
    if (nqc != 1 && !(nqc == 2 && kind == 1 && cfg[4] <= 2))
        return fail(ctx, IMG_ERR_UNSUPPORTED, "two components per CTA: magnet sweeps with at most 2 cells per thread");
    if (cfg[6] && nqc != 1) return fail(ctx, IMG_ERR_UNSUPPORTED, "window tilings carry both components per thread");
    const bool visc = kind == 0 && ctx->cfg.viscosity_type != IMG_VISC_NONE;   // segment tilings only
    std::vector<PencilCfg> cands = visc ? std::vector<PencilCfg>() : pencil_candidates(ctx->g, d, ctx->elem);
    for (const PencilCfg& sc : kind == 0 ? seg_candidates(ctx->g, d, ctx->elem, visc) : win_candidates(ctx->g, d))
        cands.push_back(sc);
    for (PencilCfg c : cands) {
        if (c.Wb != cfg[0] || c.G != cfg[1] || c.CL != cfg[2] || c.NT != cfg[3] || c.cpt != cfg[4] ||
            (c.seg != 0) != (cfg[6] != 0))
            continue;
        c.nqc = nqc;
        if (c.seg) {
            ctx->pcfg[kind][d] = c;
            if (kind == 1) ctx->pcfg[2][d] = c;
            drop_graphs(ctx);
            return IMG_OK;
        }
        int ncl = 0;
        const size_t fs = ctx->elem == 8 ? fluid_smem_bytes<double>(c.G * c.cpt, c.Wb) : fluid_smem_bytes<float>(c.G * c.cpt, c.Wb);
        PencilLaunch L = ctx->elem == 8 ? pencil_launch<double>(ctx, c, d, fs, 1, false) : pencil_launch<float>(ctx, c, d, fs, 1, false);
        cudaError_t e = ctx->elem == 8 ? fluid_max_clusters<double>(L, &ncl) : fluid_max_clusters<float>(L, &ncl);
        if (e != cudaSuccess || ncl < 1) {
            cudaGetLastError();
            return fail(ctx, IMG_ERR_UNSUPPORTED, "tiling cannot be scheduled on this device");
        }
        ctx->pcfg[kind][d] = c;
        if (kind == 1) ctx->pcfg[2][d] = c;   // the public magnet tiling is the chain's and the CT's
        drop_graphs(ctx);
        return IMG_OK;
    }
    return fail(ctx, IMG_ERR_UNSUPPORTED, "not a tiling the kernels accept for this direction");
}

int img_get_tiling(const img_ctx* ctx, int dim, int out[7]) {
    if (!ctx || !out || dim < 1 || dim > 6) return IMG_ERR_ARG;
    const PencilCfg& p = ctx->pcfg[(dim - 1) / 3][(dim - 1) % 3];
    out[0] = p.Wb;
    out[1] = p.G;
    out[2] = p.CL;
    out[3] = p.NT;
    out[4] = p.cpt;
    out[5] = p.nqc;
    out[6] = p.seg ? 1 : 0;
    return IMG_OK;
}

int img_sweep_order(int order, int iteration, int out[3]) {
    if (!out || (order != 1 && order != -1) || iteration < 1) return IMG_ERR_ARG;
    const int row = (iteration - 1) % 6;
    for (int q = 0; q < 3; ++q) out[q] = order > 0 ? FWD[row][q] : BWD[row][q];
    return IMG_OK;
}

int img_launch_count(const img_ctx* ctx, uint64_t* count) {
    if (!ctx || !count) return IMG_ERR_ARG;
    *count = ctx->launches;
    return IMG_OK;
}

int img_sync(img_ctx* ctx) {
    if (!ctx) return fail(ctx, IMG_ERR_ARG, "null context");
    return check_dev_error(ctx);
}

}  // extern "C"
