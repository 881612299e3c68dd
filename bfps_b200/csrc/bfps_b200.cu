// C-ABI implementation of include/bfps_b200.h (single GPU, sm_100a).
//
// The context owns every device buffer; one CUDA stream per context.
// Kernels: passes.cuh (DNS step), particles.cuh (tracers), stats.cuh.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <tuple>
#include <thread>
#include <unordered_map>
#include <vector>

#include "bfps_b200.h"
#include "particles.cuh"
#include "passes.cuh"
#include "pressure.cuh"
#include "stats.cuh"
#include "xpass.cuh"

using namespace bfg;

#define BFG_VERSION "bfps_b200 0.2 (sm_100a)"


struct bfg_ctx {
    int n = 0, nxv = 0, nxp = 0;
    int nsm = 148;           // streaming multiprocessors (persistent grids)
    int smem_optin = 0;      // max dynamic shared memory per block
    int real_bytes = 8;
    int dealias = BFG_SMOOTH;
    int device = 0;
    double dkx = 1, dky = 1, dkz = 1;
    double kM = 0, kM2 = 0, dk = 1, dk2 = 1;
    int nshells = 0;
    std::vector<double> kshell;
    std::vector<int64_t> nshell;
    // physics
    double nu = 0.1;
    int forcing = BFG_FORCING_NONE;
    double famp = 1.0, fk0 = 2.0, fk1 = 4.0;
    int fmode = 1;
    int iteration = 0;
    // device buffers
    void* w0 = nullptr;  // state (cvorticity)
    void* v1 = nullptr;
    void* v2 = nullptr;
    void* wa = nullptr;  // work / cvelocity
    void* wb = nullptr;  // work
    void* ru = nullptr;  // real velocity [z][y][x][3]
    void* tw = nullptr;
    void* filt = nullptr;
    int nfilt = 1;
    void* fac = nullptr;
    double fac_dt = NAN, fac_nu = NAN;
    void* dmember = nullptr;   // this context as a one-element Member<T> array
    std::vector<unsigned char> hmember;  // last uploaded copy
    void* stats_ws = nullptr;  // statistics partial sums
    int* tctr = nullptr;       // tile counters of the persistent passes (self-resetting)
    unsigned long long* dcount = nullptr;  // bfg_check_finite's counter
    size_t stats_ws_bytes = 0;
    size_t field_bytes = 0;
    cudaStream_t stream = nullptr;
    cudaStream_t tstream = nullptr;  // tracers (overlap stages 2-3 of the fluid step)
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    cudaEvent_t ev_ru = nullptr;     // real velocity of this step written
    cudaEvent_t ev_tr = nullptr;     // tracers of this step done
    int64_t launches = 0;
    std::string err;
    // per-kernel profiling (bfg_profile)
    bool prof = false;
    std::vector<cudaEvent_t> prof_ev;  // start/stop pairs
    std::vector<int> prof_kind;
    size_t prof_used = 0;
    double prof_ms[BFG_NKINDS] = {0};
    int64_t prof_n[BFG_NKINDS] = {0};
};

struct bfg_pctx {
    bfg_ctx* ctx = nullptr;
    int64_t n = 0;
    int neighbours = 1, smoothness = 1, nsteps = 1;
    int step_idx = 1;
    int head = 0;
    bool rhs0_zero = true;
    // device state, in cell order; corder = position of each tracer in the
    // order given at creation
    double* pos = nullptr;
    double* hist = nullptr;
    int64_t* corder = nullptr;
    // second copies for the re-sort, and scratch
    double* pos2 = nullptr;
    double* hist2 = nullptr;
    int64_t* corder2 = nullptr;
    double* sample = nullptr;
    unsigned* key = nullptr;
    unsigned* rank = nullptr;
    unsigned* count = nullptr;
    unsigned* offset = nullptr;
    unsigned* perm = nullptr;   // source of each cell-order slot during a sort
    int resort_every = 4;    // 0: never (grids below 256^3 keep u in L2 anyway)
    int loops_since_sort = 0;
    std::vector<int64_t> idx;       // global index of each tracer, creation order
    std::vector<int64_t> by_index;  // creation positions sorted by global index
    bool identity = true;           // idx == 0..n-1
};

// ------------------------------------------------------------ helpers --
static int fail(bfg_ctx* c, int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    if (c) c->err = buf;
    return code;
}

#define CU(call)                                                                      \
    do {                                                                              \
        cudaError_t e_ = (call);                                                      \
        if (e_ != cudaSuccess)                                                        \
            return fail(c, BFG_ECUDA, "%s: %s (%s:%d)", #call, cudaGetErrorString(e_), \
                        __FILE__, __LINE__);                                          \
    } while (0)

static int after_launch(bfg_ctx* c, const char* what) {
    c->launches++;
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail(c, BFG_ECUDA, "launch of %s: %s", what, cudaGetErrorString(e));
    return 0;
}

// ----------------------------------------------------------- profiling --
enum Kind { K_IZ = 0, K_IY = 1, K_X = 2, K_FY = 3, K_FZ = 4, K_KSPACE = 5, K_TRACER = 6, K_STATS = 7 };

static void prof_flush(bfg_ctx* c) {
    if (!c->prof_used) return;
    cudaStreamSynchronize(c->stream);
    if (c->tstream) cudaStreamSynchronize(c->tstream);
    for (size_t i = 0; i < c->prof_used; ++i) {
        float ms = 0.f;
        if (cudaEventElapsedTime(&ms, c->prof_ev[2 * i], c->prof_ev[2 * i + 1]) == cudaSuccess) {
            c->prof_ms[c->prof_kind[i]] += ms;
            c->prof_n[c->prof_kind[i]] += 1;
        }
    }
    c->prof_used = 0;
}

struct Prof {
    bfg_ctx* c;
    cudaStream_t st;
    long slot = -1;
    Prof(bfg_ctx* c_, int kind, cudaStream_t s_ = nullptr) : c(c_), st(s_ ? s_ : c_->stream) {
        if (!c->prof) return;
        if (c->prof_used >= 4096) prof_flush(c);
        if (c->prof_used == c->prof_kind.size()) {
            cudaEvent_t a, b;
            cudaEventCreate(&a);
            cudaEventCreate(&b);
            c->prof_ev.push_back(a);
            c->prof_ev.push_back(b);
            c->prof_kind.push_back(0);
        }
        slot = (long)c->prof_used++;
        c->prof_kind[slot] = kind;
        cudaEventRecord(c->prof_ev[2 * slot], st);
    }
    ~Prof() {
        if (slot >= 0) cudaEventRecord(c->prof_ev[2 * slot + 1], st);
    }
};

static bool is_pow2(int v) { return v > 0 && (v & (v - 1)) == 0; }

// A kernel whose bounded wait on its own bulk copies ran out sets
// g_bfg_wait_status (bulk.cuh); read (and cleared) after the work is done.
static int check_wait_status(bfg_ctx* c) {
    int st = 0;
    CU(cudaMemcpyFromSymbol(&st, g_bfg_wait_status, sizeof(int)));
    if (st) {
        const int zero = 0;
        CU(cudaMemcpyToSymbol(g_bfg_wait_status, &zero, sizeof(int)));
        return fail(c, BFG_ECUDA, "a kernel's wait for its own bulk copies ran out");
    }
    return 0;
}


static KParams kparams(const bfg_ctx* c, double dt) {
    KParams k;
    k.nxv = c->nxv;
    k.nxp = c->nxp;
    k.dkx = c->dkx;
    k.dky = c->dky;
    k.dkz = c->dkz;
    k.kM2 = c->kM2;
    k.dealias = c->dealias;
    k.inv_dk2 = 1.0 / c->dk2;
    k.nfilt = c->nfilt;
    k.forcing = c->forcing;
    k.famp = c->famp;
    k.fk0 = c->fk0;
    k.fk1 = c->fk1;
    k.fmode = c->fmode;
    k.dt = dt;
    return k;
}

// cudaFuncSetAttribute once per kernel and device
template <typename K>
static cudaError_t ensure_smem(K kernel, size_t bytes, int device) {
    // the attribute is a ceiling: only ever raise it (a lower value would
    // reject later launches that need more), and only past the default
    if (bytes <= 48 * 1024) return cudaSuccess;
    static std::mutex mu;
    static std::unordered_map<long long, size_t> done;
    const long long key = (long long)(uintptr_t)(void*)kernel * 64 + device;
    std::lock_guard<std::mutex> lk(mu);
    auto it = done.find(key);
    if (it != done.end() && it->second >= bytes) return cudaSuccess;
    cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)bytes);
    if (e == cudaSuccess) done[key] = bytes;
    return e;
}

static double kwrap_h(int i, int N, double dk) { return dk * (double)(i <= N / 2 ? i : i - N); }

// --------------------------------------------------------- autotuning --
// Column-pass schedule (passes.cuh: 0 or 1) per (device, grid size, real
// bytes, pass kind, members per launch).  The member count is part of the key
// because the better schedule depends on how many tiles one launch holds: a
// lone 64^3 context and a group of sixteen 64^3 ensemble members choose
// differently.  Filled by bfg_autotune (one member), bfg_ens_autotune (each
// size group of an ensemble), bfg_tune_set and, where the environment
// variable BFPS_B200_TUNE_CACHE names a file, by the choices recorded there
// by earlier runs on a device of the same name (one line per choice: device
// name, N, real bytes, pass kind, members, schedule, and the two measured
// times in ms).  Entries not tuned for that exact key use schedule 0.
struct TuneEntry {
    int sched = 0;
    double ms0 = 0, ms1 = 0;
};
static std::mutex g_tune_mu;
using TuneKey = std::tuple<int, int, int, int, int>;  // device, N, real bytes, kind, members
static std::map<TuneKey, TuneEntry> g_tune;
static std::map<int, bool> g_tune_loaded;  // device -> cache file read

static int col_kind(int mode) {
    return (mode == CM_IZ_VEL || mode == CM_IZ_PLAIN || mode == CM_IZ_U) ? K_IZ
           : (mode == CM_Y_INV1 || mode == CM_Y_INV2)                  ? K_IY
           : (mode == CM_Y_FWD1)                                      ? K_FY
                                                                      : K_FZ;
}
static std::string device_name(int dev) {
    cudaDeviceProp p;
    if (cudaGetDeviceProperties(&p, dev) != cudaSuccess) {
        cudaGetLastError();
        return "unknown";
    }
    std::string n = p.name;
    for (char& ch : n)
        if (ch == ' ') ch = '_';
    return n;
}
// read the cache file's entries for this device (g_tune_mu held)
static void tune_load_locked(int dev) {
    if (g_tune_loaded[dev]) return;
    g_tune_loaded[dev] = true;
    const char* path = std::getenv("BFPS_B200_TUNE_CACHE");
    if (!path || !*path) return;
    FILE* f = std::fopen(path, "r");
    if (!f) return;
    const std::string me = device_name(dev);
    char name[256];
    int n, rb, kind, nmem, sched;
    double ms0, ms1;
    while (std::fscanf(f, "%255s %d %d %d %d %d %lf %lf", name, &n, &rb, &kind, &nmem, &sched, &ms0,
                       &ms1) == 8)
        if (me == name && (sched == 0 || sched == 1) && nmem >= 1) {
            TuneEntry& e = g_tune[TuneKey(dev, n, rb, kind, nmem)];
            e.sched = sched;
            e.ms0 = ms0;
            e.ms1 = ms1;
        }
    std::fclose(f);
}
static int tuned_schedule(int dev, int n, int rb, int kind, int nmem) {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    tune_load_locked(dev);
    auto it = g_tune.find(TuneKey(dev, n, rb, kind, nmem));
    return it == g_tune.end() ? 0 : it->second.sched;
}
// Schedule 1 replaces the default only when it is faster by more than a
// margin: the tuner times one launch at a time, and schedule 0 (two CTAs per
// SM) shares the SMs with concurrent launches, where schedule 1 (one CTA
// holding all of an SM's shared memory) keeps every other launch off the
// SMs it runs on.  Near-ties go to schedule 0 (2 %); for the size groups of
// an ensemble that holds several sizes, whose launches run concurrently,
// schedule 1 must be 10 % faster alone (measured on the C4 mix: choices
// made at 2 % lost 1 % of the ensemble step).
constexpr double TUNE_MARGIN = 0.02;
constexpr double TUNE_MARGIN_SHARED = 0.10;

// record measured times (ms[kind * 2 + schedule]) for nmem members per
// launch, the chosen schedule, and append them to the cache file
static void tune_store(int dev, int n, int rb, int nmem, const double* ms,
                       double margin = TUNE_MARGIN) {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    tune_load_locked(dev);
    const char* path = std::getenv("BFPS_B200_TUNE_CACHE");
    FILE* f = (path && *path) ? std::fopen(path, "a") : nullptr;
    const std::string name = device_name(dev);
    for (int kind : {(int)K_IZ, (int)K_IY, (int)K_FY, (int)K_FZ}) {
        TuneEntry e;
        e.ms0 = ms[2 * kind];
        e.ms1 = ms[2 * kind + 1];
        e.sched = e.ms1 < e.ms0 * (1.0 - margin) ? 1 : 0;
        g_tune[TuneKey(dev, n, rb, kind, nmem)] = e;
        if (f)
            std::fprintf(f, "%s %d %d %d %d %d %.6f %.6f\n", name.c_str(), n, rb, kind, nmem, e.sched,
                         e.ms0, e.ms1);
    }
    if (f) std::fclose(f);
}

// ------------------------------------------------------------- engine --
template <typename T, int N>
struct Engine {
    using C = cpx<T>;
    using Mem = Member<T>;

    // one persistent launch of a column pass over nmem members, in the
    // schedule the autotuner chose for this grid, precision, pass and
    // member count
    template <int MODE>
    static int col(bfg_ctx* c, const Mem* mem, int nmem, Roles rl) {
        return tuned_schedule(c->device, N, (int)sizeof(T), col_kind(MODE), nmem) == 1
                   ? col_s<MODE, 1>(c, mem, nmem, rl)
                   : col_s<MODE, 0>(c, mem, nmem, rl);
    }
    template <int MODE, int S>
    static int col_s(bfg_ctx* c, const Mem* mem, int nmem, Roles rl) {
        constexpr int TKX = col_tkx<T, N, MODE, S>();
        constexpr size_t smem = col_smem_bytes<T, N, MODE, S>();
        auto kern = col_pass<T, N, MODE, S>;
        if (smem > (size_t)c->smem_optin)
            return fail(c, BFG_EUNSUP, "column pass needs %zu bytes of shared memory", smem);
        CU(ensure_smem(kern, smem, c->device));
        const int ntx = (N / 2 + 1 + TKX - 1) / TKX;
        const int tiles_per = ntx * N;
        const int ntiles = tiles_per * nmem;
        const int grid = std::min(ntiles, c->nsm * col_ctas<T, N, MODE, S>());
        Prof pr(c, col_kind(MODE));
        // dynamic tile order where a launch has at least 8 tiles per CTA
        int* tctr = ntiles >= 8 * grid ? c->tctr : nullptr;
        kern<<<grid, col_threads<T, N, MODE, S>(), smem, c->stream>>>(mem, rl, (const C*)c->tw, ntx,
                                                                     tiles_per, ntiles, tctr);
        return after_launch(c, "col_pass");
    }

    // bfg_autotune / bfg_ens_autotune: both schedules of each column pass
    // over the nmem members at m (roles that write only the work buffers
    // wa, wb); ms[kind * 2 + schedule] receives the mean launch time
    static int tune(bfg_ctx* c, const Mem* m, int nmem, int reps, double* ms) {
        cudaEvent_t e0 = nullptr, e1 = nullptr;
        if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) {
            if (e0) cudaEventDestroy(e0);
            cudaGetLastError();
            return fail(c, BFG_ECUDA, "cannot create timing events");
        }
        struct Ev {
            cudaEvent_t a, b;
            ~Ev() { cudaEventDestroy(a), cudaEventDestroy(b); }
        } ev{e0, e1};
        auto time_it = [&](auto launch, double* out) -> int {
            int rc = launch();  // warm-up
            if (rc) return rc;
            CU(cudaEventRecord(e0, c->stream));
            for (int r = 0; r < reps; ++r)
                if ((rc = launch())) return rc;
            CU(cudaEventRecord(e1, c->stream));
            CU(cudaEventSynchronize(e1));
            float f = 0.f;
            CU(cudaEventElapsedTime(&f, e0, e1));
            *out = f / reps;
            return 0;
        };
        const Roles r_iz = roles(B_W0, B_NONE, B_WA, B_WB), r_iy = roles(B_WA, B_WB, B_WA, B_WB),
                    r_fy = roles(B_WA, B_NONE, B_WA, B_NONE),
                    r_fz = roles(B_WA, B_NONE, B_WB, B_NONE, B_W0, B_V1, B_W0);
        int rc;
        if ((rc = time_it([&] { return col_s<CM_IZ_VEL, 0>(c, m, nmem, r_iz); }, &ms[2 * K_IZ]))) return rc;
        if ((rc = time_it([&] { return col_s<CM_IZ_VEL, 1>(c, m, nmem, r_iz); }, &ms[2 * K_IZ + 1]))) return rc;
        if ((rc = time_it([&] { return col_s<CM_Y_INV2, 0>(c, m, nmem, r_iy); }, &ms[2 * K_IY]))) return rc;
        if ((rc = time_it([&] { return col_s<CM_Y_INV2, 1>(c, m, nmem, r_iy); }, &ms[2 * K_IY + 1]))) return rc;
        if ((rc = time_it([&] { return col_s<CM_Y_FWD1, 0>(c, m, nmem, r_fy); }, &ms[2 * K_FY]))) return rc;
        if ((rc = time_it([&] { return col_s<CM_Y_FWD1, 1>(c, m, nmem, r_fy); }, &ms[2 * K_FY + 1]))) return rc;
        if ((rc = time_it([&] { return col_s<CM_FZ_RK2, 0>(c, m, nmem, r_fz); }, &ms[2 * K_FZ]))) return rc;
        return time_it([&] { return col_s<CM_FZ_RK2, 1>(c, m, nmem, r_fz); }, &ms[2 * K_FZ + 1]);
    }

    // one persistent launch of a row pass over nmem members
    template <int MODE, bool WRU>
    static int row(bfg_ctx* c, const Mem* mem, int nmem, Roles rl) {
        if constexpr (MODE == RM_NONLIN && sizeof(T) == 4 && N == 512) {
            // FP32 512^3: warp-per-row x pass (xpass.cuh)
            constexpr size_t smem = xw_smem_bytes<N>();
            auto kern = row_nonlin_warp<N, WRU>;
            if (smem > (size_t)c->smem_optin)
                return fail(c, BFG_EUNSUP, "x pass needs %zu bytes of shared memory", smem);
            CU(ensure_smem(kern, smem, c->device));
            const int rows_per = N * N;
            const int nrows = rows_per * nmem;
            const int grid = std::min(c->nsm, (nrows + xw::NWARP - 1) / xw::NWARP);
            Prof pr(c, K_X);
            kern<<<grid, xw::NWARP * 32, smem, c->stream>>>(
                reinterpret_cast<const Member<float>*>(mem), rl,
                reinterpret_cast<const cpx<float>*>(c->tw), rows_per, nrows);
            return after_launch(c, "row_nonlin_warp");
        } else if constexpr (MODE == RM_NONLIN && sizeof(T) == 4 && (N == 64 || N == 128 || N == 256)) {
            // FP32 64^3 - 256^3: warp-group x pass (xpass.cuh)
            constexpr size_t smem = xwg_smem_bytes<N>();
            auto kern = row_nonlin_wg<N, WRU>;
            if (smem > (size_t)c->smem_optin)
                return fail(c, BFG_EUNSUP, "x pass needs %zu bytes of shared memory", smem);
            CU(ensure_smem(kern, smem, c->device));
            constexpr int Q = xwg::Cfg<N>::Q;
            const int rows_per = N * N;
            const int nrows = rows_per * nmem;
            const int nblk = nrows / Q;
            const int grid = std::min(c->nsm, (nblk + xwg::NWARP - 1) / xwg::NWARP);
            Prof pr(c, K_X);
            kern<<<grid, xwg::NWARP * 32, smem, c->stream>>>(
                reinterpret_cast<const Member<float>*>(mem), rl,
                reinterpret_cast<const cpx<float>*>(c->tw), rows_per, nrows);
            return after_launch(c, "row_nonlin_wg");
        } else if constexpr (MODE == RM_NONLIN && rnl_fused<T, N>()) {
            constexpr size_t smem = rnl_smem_bytes<T, N>();
            constexpr int ROWS = rnl_rows<T, N>();
            auto kern = row_nonlin<T, N, WRU>;
            if (smem > (size_t)c->smem_optin)
                return fail(c, BFG_EUNSUP, "row pass needs %zu bytes of shared memory", smem);
            CU(ensure_smem(kern, smem, c->device));
            const int tiles_per = N * N / ROWS;
            const int ntiles = tiles_per * nmem;
            const int grid = std::min(ntiles, c->nsm * rnl_ctas<T, N>());
            Prof pr(c, K_X);
            kern<<<grid, rnl_threads<T, N>(), smem, c->stream>>>(mem, rl, (const C*)c->tw, tiles_per,
                                                         ntiles);
            return after_launch(c, "row_nonlin");
        }
        constexpr size_t smem = row_smem_bytes<T, N, MODE>();
        constexpr int ROWS = row_rows<T, N, MODE>();
        auto kern = row_pass<T, N, MODE, WRU>;
        if (smem > (size_t)c->smem_optin)
            return fail(c, BFG_EUNSUP, "row pass needs %zu bytes of shared memory", smem);
        CU(ensure_smem(kern, smem, c->device));
        const int tiles_per = N * N / ROWS;
        const int ntiles = tiles_per * nmem;
        const int grid = std::min(ntiles, c->nsm * ROW_CTAS);
        Prof pr(c, K_X);
        kern<<<grid, ROW_THREADS, smem, c->stream>>>(mem, rl, (const C*)c->tw, tiles_per, ntiles);
        return after_launch(c, "row_pass");
    }

    static int symmetrize(bfg_ctx* c, const Mem* mem, int nmem, int bufi) {
        Prof pr(c, K_KSPACE);
        symmetrize_kernel<T, N><<<dim3((N * N + 255) / 256, nmem), 256, 0, c->stream>>>(mem, bufi);
        return after_launch(c, "symmetrize");
    }

    // RK stage s of every member: IZ -> IY -> X -> FY -> FZ (with update)
    static int stage(bfg_ctx* c, const Mem* mem, int nmem, int s, bool write_ru) {
        int rc;
        const int src = s == 0 ? B_W0 : (s == 1 ? B_V1 : B_V2);
        if ((rc = col<CM_IZ_VEL>(c, mem, nmem, roles(src, B_NONE, B_WA, B_WB)))) return rc;
        if ((rc = col<CM_Y_INV2>(c, mem, nmem, roles(B_WA, B_WB, B_WA, B_WB)))) return rc;
        if (write_ru)
            rc = row<RM_NONLIN, true>(c, mem, nmem, roles(B_WA, B_WB, B_WA, B_NONE, B_NONE, B_NONE,
                                                          B_NONE, B_RU));
        else
            rc = row<RM_NONLIN, false>(c, mem, nmem, roles(B_WA, B_WB, B_WA, B_NONE));
        if (rc) return rc;
        if ((rc = col<CM_Y_FWD1>(c, mem, nmem, roles(B_WA, B_NONE, B_WA, B_NONE)))) return rc;
        if (s == 0)
            return col<CM_FZ_RK1>(c, mem, nmem, roles(B_WA, B_NONE, B_V1, B_NONE, B_W0, B_NONE, src));
        if (s == 1)
            return col<CM_FZ_RK2>(c, mem, nmem, roles(B_WA, B_NONE, B_V2, B_NONE, B_W0, B_V1, src));
        return col<CM_FZ_RK3>(c, mem, nmem, roles(B_WA, B_NONE, B_W0, B_NONE, B_W0, B_V2, src));
    }

    static int finish_step(bfg_ctx* c, const Mem* mem, int nmem) {
        return symmetrize(c, mem, nmem, B_W0);
    }

    // ---- single-context operations (the context's own member) -------------
    static const Mem* self(bfg_ctx* c) { return (const Mem*)c->dmember; }

    static int velocity_state(bfg_ctx* c) {
        const size_t npts = (size_t)N * N * c->nxv;
        Prof pr(c, K_KSPACE);
        velocity_kernel<T, N><<<(unsigned)((npts + 255) / 256), 256, 0, c->stream>>>(
            kparams(c, 0.0), (const C*)c->w0, (C*)c->wa);
        int rc = after_launch(c, "velocity");
        if (rc) return rc;
        return symmetrize(c, self(c), 1, B_WA);
    }

    static int velocity_rspace(bfg_ctx* c) {
        int rc;
        if ((rc = col<CM_IZ_U>(c, self(c), 1, roles(B_W0, B_NONE, B_WB, B_NONE)))) return rc;
        if ((rc = col<CM_Y_INV1>(c, self(c), 1, roles(B_WB, B_NONE, B_WB, B_NONE)))) return rc;
        return row<RM_C2R, false>(c, self(c), 1, roles(B_WB, B_NONE, B_NONE, B_NONE, B_NONE, B_NONE,
                                                       B_NONE, B_RU));
    }

    static int fixup(bfg_ctx* c) {
        int rc = symmetrize(c, self(c), 1, B_W0);
        if (rc) return rc;
        const size_t npts = (size_t)N * N * c->nxv;
        Prof pr(c, K_KSPACE);
        lowpass_divfree_kernel<T, N><<<(unsigned)((npts + 255) / 256), 256, 0, c->stream>>>(
            kparams(c, 0.0), (C*)c->w0);
        return after_launch(c, "lowpass_divfree");
    }

    // unnormalised C2R of wb (state layout) into ru; uses wa
    static int ift_wb(bfg_ctx* c) {
        int rc;
        if ((rc = col<CM_IZ_PLAIN>(c, self(c), 1, roles(B_WB, B_NONE, B_WA, B_NONE)))) return rc;
        if ((rc = col<CM_Y_INV1>(c, self(c), 1, roles(B_WA, B_NONE, B_WA, B_NONE)))) return rc;
        return row<RM_C2R, false>(c, self(c), 1, roles(B_WA, B_NONE, B_NONE, B_NONE, B_NONE, B_NONE,
                                                       B_NONE, B_RU));
    }
    // unnormalised R2C of ru into wb (state layout); uses wa
    static int dft_ru(bfg_ctx* c) {
        int rc;
        if ((rc = row<RM_R2C, false>(c, self(c), 1, roles(B_NONE, B_NONE, B_WA, B_NONE, B_NONE,
                                                          B_NONE, B_NONE, B_NONE, B_RU))))
            return rc;
        if ((rc = col<CM_Y_FWD1>(c, self(c), 1, roles(B_WA, B_NONE, B_WA, B_NONE)))) return rc;
        return col<CM_FZ_PLAIN>(c, self(c), 1, roles(B_WA, B_NONE, B_WB, B_NONE));
    }

    // real-space products of the velocity in ru into v2 (as reals [z][y][x][3])
    static int products(bfg_ctx* c, int off) {
        const size_t npts = (size_t)N * N * N;
        Prof pr(c, K_KSPACE);
        products_kernel<T><<<(unsigned)((npts + 255) / 256), 256, 0, c->stream>>>(
            (const T*)c->ru, (T*)c->v2, npts, off);
        return after_launch(c, "products");
    }
    // unnormalised R2C of v2 (reals) into wb (state layout); uses wa
    static int dft_v2(bfg_ctx* c) {
        int rc;
        if ((rc = row<RM_R2C, false>(c, self(c), 1, roles(B_NONE, B_NONE, B_WA, B_NONE, B_NONE,
                                                          B_NONE, B_NONE, B_NONE, B_V2))))
            return rc;
        if ((rc = col<CM_Y_FWD1>(c, self(c), 1, roles(B_WA, B_NONE, B_WA, B_NONE)))) return rc;
        return col<CM_FZ_PLAIN>(c, self(c), 1, roles(B_WA, B_NONE, B_WB, B_NONE));
    }
    // vorticity_equation::compute_pressure (vorticity_equation.cpp:441-514)
    // of the current state's velocity: p^ into component 0 of v1; ru holds
    // u(x) afterwards
    static int pressure(bfg_ctx* c) {
        int rc;
        if ((rc = velocity_rspace(c))) return rc;
        const size_t nm = (size_t)N * N * c->nxv;
        for (int off = 0; off < 2; ++off) {
            if ((rc = products(c, off))) return rc;
            if ((rc = dft_v2(c))) return rc;
            Prof pr(c, K_KSPACE);
            pressure_kernel<T, N><<<(unsigned)((nm + 255) / 256), 256, 0, c->stream>>>(
                kparams(c, 0.0), (const T*)c->filt, (const C*)c->wb, (C*)c->v1, off);
            if ((rc = after_launch(c, "pressure"))) return rc;
        }
        return 0;
    }
    // compute_Lagrangian_acceleration (vorticity_equation.cpp:516-578): a^
    // into wb (state layout); u^ of the current state (symmetrised, as
    // compute_velocity does) in wa
    static int acceleration(bfg_ctx* c) {
        int rc;
        if ((rc = pressure(c))) return rc;
        if ((rc = velocity_state(c))) return rc;
        const size_t nm = (size_t)N * N * c->nxv;
        Prof pr(c, K_KSPACE);
        acceleration_kernel<T, N><<<(unsigned)((nm + 255) / 256), 256, 0, c->stream>>>(
            kparams(c, 0.0), c->nu, (const C*)c->wa, (const C*)c->v1, (C*)c->wb);
        return after_launch(c, "acceleration");
    }
    // the acceleration in real space into v2 (reals [z][y][x][3]); uses wa
    static int acceleration_rspace(bfg_ctx* c) {
        int rc;
        if ((rc = acceleration(c))) return rc;
        if ((rc = col<CM_IZ_PLAIN>(c, self(c), 1, roles(B_WB, B_NONE, B_WA, B_NONE)))) return rc;
        if ((rc = col<CM_Y_INV1>(c, self(c), 1, roles(B_WA, B_NONE, B_WA, B_NONE)))) return rc;
        return row<RM_C2R, false>(c, self(c), 1, roles(B_WA, B_NONE, B_NONE, B_NONE, B_NONE, B_NONE,
                                                       B_NONE, B_V2));
    }

    static int stats(bfg_ctx* c, int cfield, double max_est, int nbins, double* spec, double* mom,
                     int64_t* hist);
};

#include "stats_engine.inl"

// runtime dispatch over (T, N)
template <template <typename, int> class F, typename... Args>
static int dispatch(bfg_ctx* c, Args... args) {
    if (c->real_bytes == 4) {
        switch (c->n) {
            case 16: return F<float, 16>::run(c, args...);
            case 32: return F<float, 32>::run(c, args...);
            case 64: return F<float, 64>::run(c, args...);
            case 128: return F<float, 128>::run(c, args...);
            case 256: return F<float, 256>::run(c, args...);
            case 512: return F<float, 512>::run(c, args...);
            case 1024: return F<float, 1024>::run(c, args...);
        }
    } else {
        switch (c->n) {
            case 16: return F<double, 16>::run(c, args...);
            case 32: return F<double, 32>::run(c, args...);
            case 64: return F<double, 64>::run(c, args...);
            case 128: return F<double, 128>::run(c, args...);
            case 256: return F<double, 256>::run(c, args...);
            case 512: return F<double, 512>::run(c, args...);
            case 1024: return F<double, 1024>::run(c, args...);
        }
    }
    return fail(c, BFG_EUNSUP, "grid size %d not supported", c->n);
}

template <typename T, int N>
struct OpStep {
    static int run(bfg_ctx* c, double dt, bfg_pctx* p);
};
template <typename T, int N>
struct OpVelocity {
    static int run(bfg_ctx* c) { return Engine<T, N>::velocity_state(c); }
};
template <typename T, int N>
struct OpVelocityR {
    static int run(bfg_ctx* c) { return Engine<T, N>::velocity_rspace(c); }
};
template <typename T, int N>
struct OpPressure {
    static int run(bfg_ctx* c) { return Engine<T, N>::pressure(c); }
};
template <typename T, int N>
struct OpAccel {
    static int run(bfg_ctx* c) { return Engine<T, N>::acceleration(c); }
};
template <typename T, int N>
struct OpAccelR {
    static int run(bfg_ctx* c) { return Engine<T, N>::acceleration_rspace(c); }
};
template <typename T, int N>
struct OpFixup {
    static int run(bfg_ctx* c) { return Engine<T, N>::fixup(c); }
};
template <typename T, int N>
struct OpIft {
    static int run(bfg_ctx* c) { return Engine<T, N>::ift_wb(c); }
};
template <typename T, int N>
struct OpDft {
    static int run(bfg_ctx* c) { return Engine<T, N>::dft_ru(c); }
};
template <typename T, int N>
struct OpTune {
    static int run(bfg_ctx* c, int reps, double* ms) {
        return Engine<T, N>::tune(c, Engine<T, N>::self(c), 1, reps, ms);
    }
};
template <typename T, int N>
struct OpStats {
    static int run(bfg_ctx* c, int f, double me, int nb, double* s, double* m, int64_t* h) {
        return Engine<T, N>::stats(c, f, me, nb, s, m, h);
    }
};

// ------------------------------------------------------- host tables --
template <typename T>
static std::vector<T> host_twiddles(int N) {
    std::vector<T> t(2 * (size_t)N);
    const long double pi = 3.141592653589793238462643383279502884L;
    for (int m = 0; m < N; ++m) {
        const long double a = 2.0L * pi * (long double)m / (long double)N;
        t[2 * m] = (T)cosl(a);
        t[2 * m + 1] = (T)(-sinl(a));
    }
    return t;
}

static int upload_tables(bfg_ctx* c) {
    const int N = c->n;
    // twiddles exp(-2 pi i m / N)
    if (c->real_bytes == 4) {
        auto t = host_twiddles<float>(N);
        CU(cudaMemcpy(c->tw, t.data(), t.size() * sizeof(float), cudaMemcpyHostToDevice));
    } else {
        auto t = host_twiddles<double>(N);
        CU(cudaMemcpy(c->tw, t.data(), t.size() * sizeof(double), cudaMemcpyHostToDevice));
    }
    // smooth dealias filter keyed by round(k2/dk2), filled in CLOOP order
    // (kspace.cpp:109-137; later writes of a key win)
    std::vector<double> filt;
    if (c->dealias == BFG_SMOOTH) {
        int maxkey = 0;
        for (int y = 0; y < N; ++y)
            for (int z = 0; z < N; ++z)
                for (int x = 0; x < c->nxv; ++x) {
                    const double kx = x * c->dkx, ky = kwrap_h(y, N, c->dky), kz = kwrap_h(z, N, c->dkz);
                    const double k2 = (kx * kx + ky * ky) + kz * kz;
                    maxkey = std::max(maxkey, (int)std::round(k2 / c->dk2));
                }
        filt.assign((size_t)maxkey + 1, 0.0);
        for (int y = 0; y < N; ++y)
            for (int z = 0; z < N; ++z)
                for (int x = 0; x < c->nxv; ++x) {
                    const double kx = x * c->dkx, ky = kwrap_h(y, N, c->dky), kz = kwrap_h(z, N, c->dkz);
                    const double k2 = (kx * kx + ky * ky) + kz * kz;
                    filt[(size_t)std::round(k2 / c->dk2)] = std::exp(-36.0 * std::pow(k2 / c->kM2, 18.));
                }
    } else {
        filt.assign(1, 1.0);
    }
    c->nfilt = (int)filt.size();
    const size_t tb = (size_t)c->real_bytes;
    CU(cudaMalloc(&c->filt, filt.size() * tb));
    if (c->real_bytes == 4) {
        std::vector<float> f(filt.begin(), filt.end());
        CU(cudaMemcpy(c->filt, f.data(), f.size() * 4, cudaMemcpyHostToDevice));
    } else {
        CU(cudaMemcpy(c->filt, filt.data(), filt.size() * 8, cudaMemcpyHostToDevice));
    }
    // shells (kspace.cpp:109-150)
    c->kshell.assign(c->nshells, 0.0);
    c->nshell.assign(c->nshells, 0);
    for (int y = 0; y < N; ++y)
        for (int z = 0; z < N; ++z)
            for (int x = 0; x < c->nxv; ++x) {
                const double kx = x * c->dkx, ky = kwrap_h(y, N, c->dky), kz = kwrap_h(z, N, c->dkz);
                const double k2 = (kx * kx + ky * ky) + kz * kz;
                if (k2 < c->kM2) {
                    const double kn = std::sqrt(k2);
                    const int w = x == 0 ? 1 : 2;
                    c->kshell[(int)(kn / c->dk)] += w * kn;
                    c->nshell[(int)(kn / c->dk)] += w;
                }
            }
    for (int s = 0; s < c->nshells; ++s)
        if (c->nshell[s] != 0) c->kshell[s] /= c->nshell[s];
    return 0;
}

// integrating-factor tables for (nu, dt), per axis
static int ensure_factors(bfg_ctx* c, double dt) {
    if (dt == c->fac_dt && c->nu == c->fac_nu) return 0;
    const int N = c->n, nxv = c->nxv;
    const int nf = nxv + 2 * N;
    std::vector<double> f(3 * (size_t)nf);
    const double mult[3] = {-dt, -dt / 2, dt / 2};
    for (int k = 0; k < 3; ++k) {
        for (int x = 0; x < nxv; ++x) {
            const double kx = x * c->dkx;
            f[k * nf + x] = std::exp(c->nu * kx * kx * mult[k]);
        }
        for (int y = 0; y < N; ++y) {
            const double ky = kwrap_h(y, N, c->dky);
            f[k * nf + nxv + y] = std::exp(c->nu * ky * ky * mult[k]);
        }
        for (int z = 0; z < N; ++z) {
            const double kz = kwrap_h(z, N, c->dkz);
            f[k * nf + nxv + N + z] = std::exp(c->nu * kz * kz * mult[k]);
        }
    }
    if (c->real_bytes == 4) {
        std::vector<float> g(f.begin(), f.end());
        CU(cudaMemcpyAsync(c->fac, g.data(), g.size() * 4, cudaMemcpyHostToDevice, c->stream));
        CU(cudaStreamSynchronize(c->stream));
    } else {
        CU(cudaMemcpyAsync(c->fac, f.data(), f.size() * 8, cudaMemcpyHostToDevice, c->stream));
        CU(cudaStreamSynchronize(c->stream));
    }
    c->fac_dt = dt;
    c->fac_nu = c->nu;
    return 0;
}

// (re)upload this context's Member<T> when parameters or buffers changed
template <typename T>
static int sync_member_t(bfg_ctx* c, double dt) {
    Member<T> m;
    memset(&m, 0, sizeof(m));
    m.kp = kparams(c, dt);
    m.buf[B_W0] = (cpx<T>*)c->w0;
    m.buf[B_V1] = (cpx<T>*)c->v1;
    m.buf[B_V2] = (cpx<T>*)c->v2;
    m.buf[B_WA] = (cpx<T>*)c->wa;
    m.buf[B_WB] = (cpx<T>*)c->wb;
    m.ru = (T*)c->ru;
    m.filt = (const T*)c->filt;
    m.fac = (const T*)c->fac;
    const unsigned char* b = reinterpret_cast<const unsigned char*>(&m);
    if (c->dmember && c->hmember.size() == sizeof(m) && memcmp(c->hmember.data(), b, sizeof(m)) == 0)
        return 0;
    if (!c->dmember) CU(cudaMalloc(&c->dmember, sizeof(m)));
    CU(cudaMemcpyAsync(c->dmember, b, sizeof(m), cudaMemcpyHostToDevice, c->stream));
    CU(cudaStreamSynchronize(c->stream));
    c->hmember.assign(b, b + sizeof(m));
    return 0;
}
static int sync_member(bfg_ctx* c, double dt) {
    if (std::isnan(dt)) dt = 0.0;
    return c->real_bytes == 4 ? sync_member_t<float>(c, dt) : sync_member_t<double>(c, dt);
}

// order the context's main stream after the tracer work queued on the
// second stream (anything that reads or rewrites tracers or ru)
static int join_tracers(bfg_ctx* c) {
    CU(cudaStreamWaitEvent(c->stream, c->ev_tr, 0));
    return 0;
}

static int ensure_ru(bfg_ctx* c) {
    if (c->ru) return 0;
    const size_t bytes = (size_t)c->n * c->n * c->n * 3 * c->real_bytes;
    if (cudaMalloc(&c->ru, bytes) != cudaSuccess) {
        cudaGetLastError();
        return fail(c, BFG_ENOMEM, "cannot allocate %zu bytes for the real velocity", bytes);
    }
    CU(cudaMemset(c->ru, 0, bytes));
    return 0;
}

// ----------------------------------------------------------- tracers --
template <typename T, int NB, int MM>
static int launch_tracers(bfg_ctx* c, const PParams& pp, bfg_pctx* p, double* out,
                          cudaStream_t st, const void* field) {
    const unsigned blocks = (unsigned)((p->n + tracers_per_block<T>() - 1) / tracers_per_block<T>());
    if (blocks == 0) return 0;
    Prof pr(c, K_TRACER, st);
    tracer_kernel<T, NB, MM><<<blocks, TRACER_THREADS, 0, st>>>(
        pp, (const T*)(field ? field : c->ru), p->pos, p->hist, out);
    return after_launch(c, "tracer_kernel");
}

template <typename T>
static int tracers_dispatch(bfg_ctx* c, const PParams& pp, bfg_pctx* p, double* out,
                            cudaStream_t st, const void* field = nullptr) {
#define BFG_TR(NBv, MMv) \
    if (p->neighbours == NBv && p->smoothness == MMv) \
        return launch_tracers<T, NBv, MMv>(c, pp, p, out, st, field);
    BFG_TR(1, 0) BFG_TR(1, 1) BFG_TR(1, 2)
    BFG_TR(2, 0) BFG_TR(2, 1) BFG_TR(2, 2)
    BFG_TR(3, 0) BFG_TR(3, 1) BFG_TR(3, 2)
    BFG_TR(4, 0) BFG_TR(4, 1) BFG_TR(4, 2)
    BFG_TR(5, 0) BFG_TR(5, 1) BFG_TR(5, 2)
#undef BFG_TR
    return fail(c, BFG_EUNSUP, "interpolation (%d, %d) not supported", p->neighbours, p->smoothness);
}

static PParams pparams(const bfg_pctx* p, double dt, int move) {
    const bfg_ctx* c = p->ctx;
    PParams pp;
    pp.n = p->n;
    pp.N = c->n;
    const double dks[3] = {c->dkx, c->dky, c->dkz};
    for (int d = 0; d < 3; ++d) {
        pp.box[d] = 4 * std::acos(0.0) / dks[d];
        pp.hstep[d] = pp.box[d] / (double)c->n;
    }
    pp.nsteps = p->nsteps;
    pp.head = p->head;
    pp.order = std::min(p->step_idx, p->nsteps);
    pp.accum = p->rhs0_zero ? 0 : 1;
    pp.move = move;
    pp.dt = dt;
    return pp;
}

// counting sort of the tracers by (z, y) cell row (tracer_keys / bucket scans /
// tracer_perm / tracer_gather); swaps the state arrays with their second copies
static int tracer_sort(bfg_pctx* p, cudaStream_t st = nullptr) {
    bfg_ctx* c = p->ctx;
    if (!st) st = c->stream;
    if (p->n == 0) return 0;
    const unsigned blocks = (unsigned)((p->n + 255) / 256);
    const int nb = c->n * c->n;
    PParams pp = pparams(p, 0.0, 0);
    Prof pr(c, K_TRACER, st);
    CU(cudaMemsetAsync(p->count, 0, (size_t)nb * sizeof(unsigned), st));
    tracer_keys<<<blocks, 256, 0, st>>>(pp, p->pos, p->key, p->rank, p->count);
    int rc = after_launch(c, "tracer_keys");
    if (rc) return rc;
    // offset holds nb bucket offsets followed by up to 1024 block sums
    const int nblk = (nb + 1023) / 1024;
    unsigned* bsum = p->offset + nb;
    bucket_block_sums<<<nblk, 1024, 0, st>>>(p->count, bsum, nb);
    if ((rc = after_launch(c, "bucket_block_sums"))) return rc;
    bucket_scan_sums<<<1, 1024, 0, st>>>(bsum, nblk);
    if ((rc = after_launch(c, "bucket_scan_sums"))) return rc;
    bucket_scan_blocks<<<nblk, 1024, 0, st>>>(p->count, bsum, p->offset, nb);
    if ((rc = after_launch(c, "bucket_scan_blocks"))) return rc;
    tracer_perm<<<blocks, 256, 0, st>>>(pp, p->key, p->rank, p->offset, p->perm);
    if ((rc = after_launch(c, "tracer_perm"))) return rc;
    tracer_gather<<<blocks, 256, 0, st>>>(pp, p->perm, p->pos, p->hist, p->corder, p->pos2,
                                           p->hist2, p->corder2);
    if ((rc = after_launch(c, "tracer_gather"))) return rc;
    std::swap(p->pos, p->pos2);
    std::swap(p->hist, p->hist2);
    std::swap(p->corder, p->corder2);
    p->loops_since_sort = 0;
    return 0;
}

static int tracer_loop(bfg_pctx* p, double dt, cudaStream_t st = nullptr) {
    bfg_ctx* c = p->ctx;
    if (!st) st = c->stream;
    if (p->resort_every > 0 && p->loops_since_sort >= p->resort_every) {
        int rc = tracer_sort(p, st);
        if (rc) return rc;
    }
    if (p->step_idx > 6 && p->nsteps > 6)
        return fail(c, BFG_EINVAL, "Adams-Bashforth order above 6");
    PParams pp = pparams(p, dt, 1);
    int rc = c->real_bytes == 4 ? tracers_dispatch<float>(c, pp, p, nullptr, st)
                                : tracers_dispatch<double>(c, pp, p, nullptr, st);
    if (rc) return rc;
    // inc_step_idx, shift_rhs_vectors
    p->step_idx += 1;
    p->head = (p->head - 1 + p->nsteps) % p->nsteps;
    p->rhs0_zero = true;
    p->loops_since_sort += 1;
    return 0;
}

template <typename T, int N>
int OpStep<T, N>::run(bfg_ctx* c, double dt, bfg_pctx* p) {
    using E = Engine<T, N>;
    int rc;
    // the previous step's tracers read ru, which stage 1 rewrites
    if (p) CU(cudaStreamWaitEvent(c->stream, c->ev_tr, 0));
    if ((rc = E::stage(c, E::self(c), 1, 0, p != nullptr))) return rc;
    if (p) {
        // tracers on u(t) (written by stage 1).  They run on the main stream:
        // running them beside the persistent passes of stages 2-3 was slower,
        // both sides losing L1/L2 to the other.
        if ((rc = tracer_loop(p, dt, c->stream))) return rc;
        CU(cudaEventRecord(c->ev_tr, c->stream));
    }
    if ((rc = E::stage(c, E::self(c), 1, 1, false))) return rc;
    if ((rc = E::stage(c, E::self(c), 1, 2, false))) return rc;
    return E::finish_step(c, E::self(c), 1);
}

// ================================================================ ABI ==
extern "C" {

const char* bfg_version(void) { return BFG_VERSION; }

const char* bfg_last_error(const bfg_ctx* ctx) { return ctx ? ctx->err.c_str() : "null context"; }

void bfg_ctx_destroy(bfg_ctx* c) {
    if (!c) return;
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    void* bufs[] = {c->w0, c->v1, c->v2, c->wa, c->wb, c->ru, c->tw, c->filt, c->fac, c->stats_ws,
                    c->dmember, c->tctr, c->dcount};
    for (void* b : bufs)
        if (b) cudaFree(b);
    for (cudaEvent_t e : c->prof_ev) cudaEventDestroy(e);
    if (c->tstream) cudaStreamSynchronize(c->tstream);
    if (c->ev_ru) cudaEventDestroy(c->ev_ru);
    if (c->ev_tr) cudaEventDestroy(c->ev_tr);
    if (c->tstream) cudaStreamDestroy(c->tstream);
    if (c->ev0) cudaEventDestroy(c->ev0);
    if (c->ev1) cudaEventDestroy(c->ev1);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
}

int bfg_ctx_create(bfg_ctx** out, int nx, int ny, int nz, double dkx, double dky, double dkz,
                   int real_bytes, int dealias_type, int device) {
    if (!out) return BFG_EINVAL;
    *out = nullptr;
    if (nx != ny || nx != nz) return BFG_EUNSUP;
    if (!is_pow2(nx) || nx < 16 || nx > 1024) return BFG_EUNSUP;
    if (real_bytes != 4 && real_bytes != 8) return BFG_EINVAL;
    if (dealias_type != BFG_SMOOTH && dealias_type != BFG_TWO_THIRDS) return BFG_EINVAL;
    if (!(dkx > 0 && dky > 0 && dkz > 0)) return BFG_EINVAL;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return BFG_ECUDA;
    }
    if (device < 0 || device >= ndev) return BFG_EINVAL;
    bfg_ctx* c = new bfg_ctx();
    c->n = nx;
    c->nxv = nx / 2 + 1;
    c->nxp = nx / 2 + 4;
    c->real_bytes = real_bytes;
    c->dealias = dealias_type;
    c->device = device;
    c->dkx = dkx;
    c->dky = dky;
    c->dkz = dkz;
    // kspace.cpp:75-100 (cubic grid: sizes are (n, n, n/2+1))
    const int s0 = nx, s1 = nx, s2 = nx / 2 + 1;
    double kMx, kMy, kMz;
    if (dealias_type == BFG_TWO_THIRDS) {
        kMx = dkx * ((2 * (s2 - 1)) / 3 - 1);
        kMy = dky * (s0 / 3 - 1);
        kMz = dkz * (s1 / 3 - 1);
    } else {
        kMx = dkx * (s2 - 2);
        kMy = dky * (s0 / 2 - 1);
        kMz = dkz * (s1 / 2 - 1);
    }
    c->kM = std::max(kMx, std::max(kMy, kMz));
    c->kM2 = c->kM * c->kM;
    c->dk = std::min(dkx, std::min(dky, dkz));
    c->dk2 = c->dk * c->dk;
    c->nshells = (int)(c->kM / c->dk) + 2;
    int rc = 0;
    auto bail = [&](int code) {
        bfg_ctx_destroy(c);
        return code;
    };
    if (cudaSetDevice(device) != cudaSuccess) return bail(BFG_ECUDA);
    if (cudaDeviceGetAttribute(&c->nsm, cudaDevAttrMultiProcessorCount, device) != cudaSuccess ||
        cudaDeviceGetAttribute(&c->smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device) !=
            cudaSuccess)
        return bail(BFG_ECUDA);
    if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) return bail(BFG_ECUDA);
    if (cudaStreamCreateWithFlags(&c->tstream, cudaStreamNonBlocking) != cudaSuccess) return bail(BFG_ECUDA);
    cudaEventCreate(&c->ev0);
    cudaEventCreate(&c->ev1);
    cudaEventCreateWithFlags(&c->ev_ru, cudaEventDisableTiming);
    cudaEventCreateWithFlags(&c->ev_tr, cudaEventDisableTiming);
    cudaEventRecord(c->ev_tr, c->tstream);
    const size_t cb = 2 * (size_t)real_bytes;  // bytes per complex
    c->field_bytes = (size_t)nx * nx * c->nxp * 3 * cb;
    void** bufs[] = {&c->w0, &c->v1, &c->v2, &c->wa, &c->wb};
    for (void** b : bufs) {
        if (cudaMalloc(b, c->field_bytes) != cudaSuccess) {
            cudaGetLastError();
            return bail(BFG_ENOMEM);
        }
        if (cudaMemset(*b, 0, c->field_bytes) != cudaSuccess) return bail(BFG_ECUDA);
    }
    if (cudaMalloc(&c->tw, (size_t)nx * cb) != cudaSuccess) return bail(BFG_ENOMEM);
    if (cudaMalloc(&c->tctr, 64) != cudaSuccess || cudaMemset(c->tctr, 0, 64) != cudaSuccess)
        return bail(BFG_ENOMEM);
    if (cudaMalloc(&c->fac, 3 * (size_t)(c->nxv + 2 * nx) * real_bytes) != cudaSuccess)
        return bail(BFG_ENOMEM);
    if ((rc = upload_tables(c))) return bail(rc);
    *out = c;
    return BFG_OK;
}

int bfg_set_physics(bfg_ctx* c, double nu, int forcing_type, double famplitude, double fk0,
                    double fk1, int fmode) {
    if (!c) return BFG_EINVAL;
    if (forcing_type < BFG_FORCING_NONE || forcing_type > BFG_FORCING_KOLMOGOROV)
        return fail(c, BFG_EINVAL, "unknown forcing_type %d", forcing_type);
    if (forcing_type == BFG_FORCING_KOLMOGOROV && (fmode < 0 || fmode >= c->n))
        return fail(c, BFG_EINVAL, "fmode %d outside the grid", fmode);
    c->nu = nu;
    c->forcing = forcing_type;
    c->famp = famplitude;
    c->fk0 = fk0;
    c->fk1 = fk1;
    c->fmode = fmode;
    return 0;
}

int bfg_kspace_info(const bfg_ctx* c, double* kM, double* dk, int* nshells, double* kshell,
                    int64_t* nshell) {
    if (!c) return BFG_EINVAL;
    if (kM) *kM = c->kM;
    if (dk) *dk = c->dk;
    if (nshells) *nshells = c->nshells;
    if (kshell) std::copy(c->kshell.begin(), c->kshell.end(), kshell);
    if (nshell) std::copy(c->nshell.begin(), c->nshell.end(), nshell);
    return 0;
}

// Pitched row copy on the device, 8-byte words: rows of wq words from a
// source of pitch sq to a destination of pitch dq; the zq words after each
// destination row are set to zero.
__global__ void pitch_copy8(const uint2* __restrict__ src, size_t sq, uint2* __restrict__ dst,
                            size_t dq, int wq, int zq, size_t rows) {
    for (size_t r = blockIdx.x; r < rows; r += gridDim.x) {
        for (int k = threadIdx.x; k < wq; k += blockDim.x) dst[r * dq + k] = src[r * sq + k];
        for (int k = threadIdx.x; k < zq; k += blockDim.x) dst[r * dq + wq + k] = make_uint2(0, 0);
    }
}

// Host <-> device field transfer.  The host side is the reference layout;
// the copy itself is one contiguous transfer through the scratch buffer wb
// (pitched host copies run well below the link rate), the change of row
// pitch is a device kernel.
static int field_copy(bfg_ctx* c, int field_id, void* host, bool upload) {
    if (!c || !host) return BFG_EINVAL;
    CU(cudaSetDevice(c->device));
    if (int rj = join_tracers(c)) return rj;
    const size_t cb = 2 * (size_t)c->real_bytes;
    const size_t N = c->n;
    const size_t rows = N * N;
    size_t dpitch, hpitch, width;  // bytes
    void* dev;
    if (field_id == BFG_FIELD_VORTICITY || field_id == BFG_FIELD_VELOCITY) {
        dev = field_id == BFG_FIELD_VORTICITY ? c->w0 : c->wa;
        dpitch = (size_t)c->nxp * 3 * cb;
        hpitch = width = (size_t)c->nxv * 3 * cb;
    } else if (field_id == BFG_FIELD_RVELOCITY) {
        int rc = ensure_ru(c);
        if (rc) return rc;
        const size_t rb = c->real_bytes;
        dev = c->ru;
        dpitch = width = N * 3 * rb;
        hpitch = (N + 2) * 3 * rb;
    } else {
        return fail(c, BFG_EINVAL, "unknown field id %d", field_id);
    }
    const int grid = c->nsm * 8;
    const int wq = (int)(width / 8);
    if (upload) {
        CU(cudaMemcpyAsync(c->wb, host, rows * hpitch, cudaMemcpyHostToDevice, c->stream));
        pitch_copy8<<<grid, 256, 0, c->stream>>>((const uint2*)c->wb, hpitch / 8, (uint2*)dev,
                                                 dpitch / 8, wq, 0, rows);
        CU(cudaGetLastError());
    } else {
        pitch_copy8<<<grid, 256, 0, c->stream>>>((const uint2*)dev, dpitch / 8, (uint2*)c->wb,
                                                 hpitch / 8, wq, (int)((hpitch - width) / 8), rows);
        CU(cudaGetLastError());
        CU(cudaMemcpyAsync(host, c->wb, rows * hpitch, cudaMemcpyDeviceToHost, c->stream));
    }
    CU(cudaStreamSynchronize(c->stream));
    return check_wait_status(c);
}

int bfg_field_upload(bfg_ctx* c, int field_id, const void* host) {
    return field_copy(c, field_id, const_cast<void*>(host), true);
}
int bfg_field_download(bfg_ctx* c, int field_id, void* host) {
    return field_copy(c, field_id, host, false);
}

int bfg_read_checkpoint_fixup(bfg_ctx* c) {
    if (!c) return BFG_EINVAL;
    CU(cudaSetDevice(c->device));
    int rc = sync_member(c, c->fac_dt);
    if (rc) return rc;
    rc = dispatch<OpFixup>(c);
    if (rc) return rc;
    CU(cudaStreamSynchronize(c->stream));
    return 0;
}

int bfg_nsveparticles_step(bfg_ctx* c, bfg_pctx* p, double dt, int nsteps) {
    if (!c || nsteps < 0) return BFG_EINVAL;
    if (p && p->ctx != c) return fail(c, BFG_EINVAL, "tracers belong to another context");
    CU(cudaSetDevice(c->device));
    int rc = ensure_factors(c, dt);
    if (rc) return rc;
    if (p && (rc = ensure_ru(c))) return rc;
    if ((rc = sync_member(c, dt))) return rc;
    CU(cudaEventRecord(c->ev0, c->stream));
    for (int s = 0; s < nsteps; ++s) {
        if ((rc = dispatch<OpStep>(c, dt, p))) return rc;
        c->iteration++;
    }
    if (p) CU(cudaStreamWaitEvent(c->stream, c->ev_tr, 0));
    CU(cudaEventRecord(c->ev1, c->stream));
    return 0;
}

int bfg_step(bfg_ctx* c, double dt, int nsteps) { return bfg_nsveparticles_step(c, nullptr, dt, nsteps); }

int bfg_compute_velocity(bfg_ctx* c) {
    if (!c) return BFG_EINVAL;
    CU(cudaSetDevice(c->device));
    int rc = sync_member(c, c->fac_dt);
    if (rc) return rc;
    rc = dispatch<OpVelocity>(c);
    if (rc) return rc;
    CU(cudaStreamSynchronize(c->stream));
    return 0;
}

int bfg_velocity_rspace(bfg_ctx* c) {
    if (!c) return BFG_EINVAL;
    CU(cudaSetDevice(c->device));
    if (int rj = join_tracers(c)) return rj;
    int rc = ensure_ru(c);
    if (rc) return rc;
    if ((rc = sync_member(c, c->fac_dt))) return rc;
    rc = dispatch<OpVelocityR>(c);
    if (rc) return rc;
    CU(cudaStreamSynchronize(c->stream));
    return 0;
}

// a state-layout device buffer (csrc components per point) to the
// reference host layout with cout components, through the staging buffer
static int download_state(bfg_ctx* c, const void* src, int csrc, int cout, void* host,
                          void* staging) {
    const size_t rows = (size_t)c->n * c->n;
    const size_t n = rows * c->nxv * cout;
    const unsigned blocks = (unsigned)((n + 255) / 256);
    if (c->real_bytes == 4)
        gather_rows_kernel<float><<<blocks, 256, 0, c->stream>>>(
            (const cpx<float>*)src, c->nxp, c->nxv, csrc, cout, (cpx<float>*)staging, rows);
    else
        gather_rows_kernel<double><<<blocks, 256, 0, c->stream>>>(
            (const cpx<double>*)src, c->nxp, c->nxv, csrc, cout, (cpx<double>*)staging, rows);
    int rc = after_launch(c, "gather_rows");
    if (rc) return rc;
    CU(cudaMemcpyAsync(host, staging, n * 2 * c->real_bytes, cudaMemcpyDeviceToHost, c->stream));
    CU(cudaStreamSynchronize(c->stream));
    return 0;
}

int bfg_compute_pressure(bfg_ctx* c, void* host) {
    if (!c) return BFG_EINVAL;
    CU(cudaSetDevice(c->device));
    if (int rj = join_tracers(c)) return rj;
    int rc = ensure_ru(c);
    if (rc) return rc;
    if ((rc = sync_member(c, c->fac_dt))) return rc;
    if ((rc = dispatch<OpPressure>(c))) return rc;
    if (host) return download_state(c, c->v1, 3, 1, host, c->v2);
    CU(cudaStreamSynchronize(c->stream));
    return 0;
}

int bfg_lagrangian_acceleration(bfg_ctx* c, void* host) {
    if (!c) return BFG_EINVAL;
    CU(cudaSetDevice(c->device));
    if (int rj = join_tracers(c)) return rj;
    int rc = ensure_ru(c);
    if (rc) return rc;
    if ((rc = sync_member(c, c->fac_dt))) return rc;
    if ((rc = dispatch<OpAccel>(c))) return rc;
    if (host) return download_state(c, c->wb, 3, 3, host, c->v2);
    CU(cudaStreamSynchronize(c->stream));
    return 0;
}

// host or device memory (unified addressing): cudaMemcpyDefault copies
static bool is_host_memory(const void* p) {
    cudaPointerAttributes at;
    if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
        cudaGetLastError();
        return true;
    }
    return at.type != cudaMemoryTypeDevice && at.type != cudaMemoryTypeManaged;
}

// Caller buffers in device memory may still be written (or read) by work
// the caller queued on other streams; the library's streams do not wait
// for the legacy default stream, so a call that takes such a buffer first
// waits for all work queued on the device.
static int order_after_caller(bfg_ctx* c, const void* a, const void* b) {
    if (is_host_memory(a) && (!b || is_host_memory(b))) return 0;
    CU(cudaDeviceSynchronize());
    return 0;
}

int bfg_ift(bfg_ctx* c, const void* din, void* dout) {
    if (!c || !din || !dout) return BFG_EINVAL;
    CU(cudaSetDevice(c->device));
    if (int rj = join_tracers(c)) return rj;
    if (int ro = order_after_caller(c, din, dout)) return ro;
    int rc = ensure_ru(c);
    if (rc) return rc;
    const size_t N = c->n, cb = 2 * (size_t)c->real_bytes, rb = c->real_bytes;
    if ((rc = sync_member(c, c->fac_dt))) return rc;
    CU(cudaMemcpy2DAsync(c->wb, c->nxp * 3 * cb, din, c->nxv * 3 * cb, c->nxv * 3 * cb, N * N,
                         cudaMemcpyDefault, c->stream));
    if ((rc = dispatch<OpIft>(c))) return rc;
    const bool host_out = is_host_memory(dout);
    if (!host_out)
        CU(cudaMemset2DAsync(dout, (N + 2) * 3 * rb, 0, (N + 2) * 3 * rb, N * N, c->stream));
    CU(cudaMemcpy2DAsync(dout, (N + 2) * 3 * rb, c->ru, N * 3 * rb, N * 3 * rb, N * N,
                         cudaMemcpyDefault, c->stream));
    CU(cudaStreamSynchronize(c->stream));
    if (host_out)  // padding points of every row
        for (size_t r = 0; r < N * N; ++r)
            std::memset(static_cast<char*>(dout) + (r * (N + 2) + N) * 3 * rb, 0, 2 * 3 * rb);
    return 0;
}

int bfg_dft(bfg_ctx* c, const void* din, void* dout) {
    if (!c || !din || !dout) return BFG_EINVAL;
    CU(cudaSetDevice(c->device));
    if (int rj = join_tracers(c)) return rj;
    if (int ro = order_after_caller(c, din, dout)) return ro;
    int rc = ensure_ru(c);
    if (rc) return rc;
    const size_t N = c->n, cb = 2 * (size_t)c->real_bytes, rb = c->real_bytes;
    if ((rc = sync_member(c, c->fac_dt))) return rc;
    CU(cudaMemcpy2DAsync(c->ru, N * 3 * rb, din, (N + 2) * 3 * rb, N * 3 * rb, N * N,
                         cudaMemcpyDefault, c->stream));
    if ((rc = dispatch<OpDft>(c))) return rc;
    CU(cudaMemcpy2DAsync(dout, c->nxv * 3 * cb, c->wb, c->nxp * 3 * cb, c->nxv * 3 * cb, N * N,
                         cudaMemcpyDefault, c->stream));
    CU(cudaStreamSynchronize(c->stream));
    return 0;
}

int bfg_field_ift(bfg_ctx* c, int field_id) {
    if (!c) return BFG_EINVAL;
    if (field_id != BFG_FIELD_VELOCITY)
        return fail(c, BFG_EINVAL, "bfg_field_ift: only the velocity field (%d)", BFG_FIELD_VELOCITY);
    CU(cudaSetDevice(c->device));
    if (int rj = join_tracers(c)) return rj;
    int rc = ensure_ru(c);
    if (rc) return rc;
    if ((rc = sync_member(c, c->fac_dt))) return rc;
    // the transform reads wb and uses wa as scratch: the velocity moves to wb
    CU(cudaMemcpyAsync(c->wb, c->wa, c->field_bytes, cudaMemcpyDeviceToDevice, c->stream));
    if ((rc = dispatch<OpIft>(c))) return rc;
    CU(cudaMemcpyAsync(c->wa, c->wb, c->field_bytes, cudaMemcpyDeviceToDevice, c->stream));
    CU(cudaStreamSynchronize(c->stream));
    return 0;
}

int bfg_field_stats(bfg_ctx* c, const void* field, double max_estimate, int nbins, double* spec,
                    double* mom, int64_t* hist) {
    if (!c || !field || nbins < 1) return BFG_EINVAL;
    CU(cudaSetDevice(c->device));
    if (int rj = join_tracers(c)) return rj;
    if (int ro = order_after_caller(c, field, nullptr)) return ro;
    int rc = sync_member(c, c->fac_dt);
    if (rc) return rc;
    // into v1 (free between steps), re-pitched to the device rows
    const size_t N = c->n, cb = 2 * (size_t)c->real_bytes;
    CU(cudaMemset2DAsync(c->v1, c->nxp * 3 * cb, 0, c->nxp * 3 * cb, N * N, c->stream));
    CU(cudaMemcpy2DAsync(c->v1, c->nxp * 3 * cb, field, c->nxv * 3 * cb, c->nxv * 3 * cb, N * N,
                         cudaMemcpyDefault, c->stream));
    return dispatch<OpStats>(c, (int)B_V1, max_estimate, nbins, spec, mom, hist);
}

int bfg_ctx_reset(bfg_ctx* c) {
    if (!c) return BFG_EINVAL;
    CU(cudaSetDevice(c->device));
    if (int rj = join_tracers(c)) return rj;
    for (void* b : {c->w0, c->v1, c->v2, c->wa, c->wb})
        CU(cudaMemsetAsync(b, 0, c->field_bytes, c->stream));
    c->iteration = 0;
    CU(cudaStreamSynchronize(c->stream));
    return 0;
}

int bfg_get_iteration(const bfg_ctx* c, int* it) {
    if (!c || !it) return BFG_EINVAL;
    *it = c->iteration;
    return 0;
}
int bfg_set_iteration(bfg_ctx* c, int it) {
    if (!c) return BFG_EINVAL;
    c->iteration = it;
    return 0;
}

// bfg_selftest_wait: one warp waits on an mbarrier that nothing arms, with
// a short bound, so the wait runs out and sets the status word
__global__ void wait_selftest_kernel(unsigned limit) {
    __shared__ __align__(8) unsigned long long bar;
    if (threadIdx.x == 0) {
        mbar_init(&bar, 1);
        fence_mbar_init();
    }
    __syncthreads();
    mbar_wait_bounded(&bar, 0, limit);
}

int bfg_selftest_wait(bfg_ctx* c) {
    if (!c) return BFG_EINVAL;
    CU(cudaSetDevice(c->device));
    CU(cudaStreamSynchronize(c->stream));
    wait_selftest_kernel<<<1, 32, 0, c->stream>>>(1u << 12);
    CU(cudaGetLastError());
    CU(cudaStreamSynchronize(c->stream));
    return check_wait_status(c);
}

int bfg_last_step_ms(bfg_ctx* c, double* ms) {
    if (!c || !ms) return BFG_EINVAL;
    CU(cudaSetDevice(c->device));
    CU(cudaEventSynchronize(c->ev1));
    if (int rc = check_wait_status(c)) return rc;
    float f = 0;
    CU(cudaEventElapsedTime(&f, c->ev0, c->ev1));
    *ms = f;
    return 0;
}

int bfg_profile(bfg_ctx* c, int enable) {
    if (!c) return BFG_EINVAL;
    CU(cudaSetDevice(c->device));
    prof_flush(c);
    c->prof = enable != 0;
    if (enable)
        for (int k = 0; k < BFG_NKINDS; ++k) {
            c->prof_ms[k] = 0;
            c->prof_n[k] = 0;
        }
    return 0;
}

int bfg_profile_read(bfg_ctx* c, int kind, double* total_ms, int64_t* launches) {
    if (!c || kind < 0 || kind >= BFG_NKINDS) return BFG_EINVAL;
    CU(cudaSetDevice(c->device));
    prof_flush(c);
    if (total_ms) *total_ms = c->prof_ms[kind];
    if (launches) *launches = c->prof_n[kind];
    return 0;
}

int bfg_kernel_launches(const bfg_ctx* c, int64_t* count) {
    if (!c || !count) return BFG_EINVAL;
    *count = c->launches;
    return 0;
}

int bfg_stats(bfg_ctx* c, double max_velocity_estimate, double max_vorticity_estimate, int nbins,
              double* spec_vel, double* spec_vort, double* mom_vel, double* mom_vort,
              int64_t* hist_vel, int64_t* hist_vort) {
    if (!c || nbins <= 0) return BFG_EINVAL;
    CU(cudaSetDevice(c->device));
    int rc = ensure_ru(c);
    if (rc) return rc;
    // vorticity: state itself; velocity: compute_velocity(cvorticity)
    if ((rc = sync_member(c, c->fac_dt))) return rc;
    if ((rc = dispatch<OpStats>(c, (int)B_W0, max_vorticity_estimate / std::sqrt(3.0),
                                nbins, spec_vort, mom_vort, hist_vort)))
        return rc;
    if ((rc = dispatch<OpVelocity>(c))) return rc;
    if ((rc = dispatch<OpStats>(c, (int)B_WA, max_velocity_estimate / std::sqrt(3.0),
                                nbins, spec_vel, mom_vel, hist_vel)))
        return rc;
    return 0;
}

int bfg_check_finite(bfg_ctx* c, int field_id, int64_t* nonfinite) {
    if (!c || !nonfinite) return BFG_EINVAL;
    CU(cudaSetDevice(c->device));
    if (int rj = join_tracers(c)) return rj;
    const void* dev;
    size_t nvals;
    if (field_id == BFG_FIELD_VORTICITY || field_id == BFG_FIELD_VELOCITY) {
        dev = field_id == BFG_FIELD_VORTICITY ? c->w0 : c->wa;
        nvals = (size_t)c->n * c->n * c->nxp * 3 * 2;  // padding columns hold zeros
    } else if (field_id == BFG_FIELD_RVELOCITY) {
        if (int rc = ensure_ru(c)) return rc;
        dev = c->ru;
        nvals = (size_t)c->n * c->n * c->n * 3;
    } else {
        return fail(c, BFG_EINVAL, "unknown field id %d", field_id);
    }
    if (!c->dcount) CU(cudaMalloc(&c->dcount, sizeof(unsigned long long)));
    CU(cudaMemsetAsync(c->dcount, 0, sizeof(unsigned long long), c->stream));
    if (c->real_bytes == 4)
        nonfinite_kernel<float><<<c->nsm * 8, 256, 0, c->stream>>>((const float*)dev, nvals, c->dcount);
    else
        nonfinite_kernel<double><<<c->nsm * 8, 256, 0, c->stream>>>((const double*)dev, nvals,
                                                                   c->dcount);
    if (int rc = after_launch(c, "nonfinite")) return rc;
    unsigned long long h = 0;
    CU(cudaMemcpyAsync(&h, c->dcount, sizeof(h), cudaMemcpyDeviceToHost, c->stream));
    CU(cudaStreamSynchronize(c->stream));
    *nonfinite = (int64_t)h;
    return 0;
}

static bool col_kind_valid(int kind) {
    return kind == K_IZ || kind == K_IY || kind == K_FY || kind == K_FZ;
}

int bfg_autotune(bfg_ctx* c, int reps) {
    if (!c) return BFG_EINVAL;
    if (reps < 1) reps = 1;
    CU(cudaSetDevice(c->device));
    if (int rj = join_tracers(c)) return rj;
    const double dt = std::isnan(c->fac_dt) ? 1e-3 : c->fac_dt;
    int rc = ensure_factors(c, dt);
    if (rc) return rc;
    if ((rc = sync_member(c, dt))) return rc;
    double ms[2 * BFG_NKINDS] = {0};
    if ((rc = dispatch<OpTune>(c, reps, ms))) return rc;
    tune_store(c->device, c->n, c->real_bytes, 1, ms);
    return 0;
}

int bfg_tune_get(const bfg_ctx* c, int kind, int members, int* schedule, double* ms0, double* ms1) {
    if (!c || !col_kind_valid(kind) || members < 1) return BFG_EINVAL;
    std::lock_guard<std::mutex> lk(g_tune_mu);
    tune_load_locked(c->device);
    auto it = g_tune.find(TuneKey(c->device, c->n, c->real_bytes, kind, members));
    const TuneEntry e = it == g_tune.end() ? TuneEntry() : it->second;
    if (schedule) *schedule = e.sched;
    if (ms0) *ms0 = e.ms0;
    if (ms1) *ms1 = e.ms1;
    return 0;
}

int bfg_tune_set(bfg_ctx* c, int kind, int members, int schedule) {
    if (!c || !col_kind_valid(kind) || members < 1 || (schedule != 0 && schedule != 1))
        return BFG_EINVAL;
    std::lock_guard<std::mutex> lk(g_tune_mu);
    tune_load_locked(c->device);
    g_tune[TuneKey(c->device, c->n, c->real_bytes, kind, members)].sched = schedule;
    return 0;
}

// ------------------------------------------------------------ tracers --
// scatter device-order arrays (width doubles per tracer) into creation order
__global__ void to_creation_order(const double* __restrict__ src, const int64_t* __restrict__ corder,
                                  int64_t n, int width, double* __restrict__ dst) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int64_t d = corder[i];
    for (int w = 0; w < width; ++w) dst[d * width + w] = src[i * width + w];
}
__global__ void iota64(int64_t* a, int64_t n) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) a[i] = i;
}

// device (n, width) array in cell order -> host, global index order
static int fetch_index_order(bfg_pctx* p, const double* dev, int width, double* out) {
    bfg_ctx* c = p->ctx;
    const size_t nw = (size_t)p->n * width;
    if (p->n == 0) return 0;
    const unsigned blocks = (unsigned)((p->n + 255) / 256);
    // pos2 holds n*3 doubles: enough for width <= 3
    to_creation_order<<<blocks, 256, 0, c->stream>>>(dev, p->corder, p->n, width, p->pos2);
    int rc = after_launch(c, "to_creation_order");
    if (rc) return rc;
    if (p->identity) {
        CU(cudaMemcpyAsync(out, p->pos2, nw * 8, cudaMemcpyDeviceToHost, c->stream));
        CU(cudaStreamSynchronize(c->stream));
        return 0;
    }
    std::vector<double> h(nw);
    CU(cudaMemcpyAsync(h.data(), p->pos2, nw * 8, cudaMemcpyDeviceToHost, c->stream));
    CU(cudaStreamSynchronize(c->stream));
    for (int64_t k = 0; k < p->n; ++k)
        for (int w = 0; w < width; ++w) out[k * width + w] = h[p->by_index[k] * width + w];
    return 0;
}

int bfg_particles_create(bfg_ctx* c, bfg_pctx** out, int64_t n, int neighbours, int smoothness,
                         int nsteps, const double* pos, const double* rhs, const int64_t* idx,
                         int step_idx) {
    if (!c || !out || n < 0 || (n > 0 && !pos)) return BFG_EINVAL;
    *out = nullptr;
    if (neighbours < 1 || neighbours > 5 || smoothness < 0 || smoothness > 2)
        return fail(c, BFG_EUNSUP, "interpolation (%d, %d) not supported", neighbours, smoothness);
    if (nsteps < 1 || nsteps > 6)
        return fail(c, BFG_EINVAL, "nsteps %d outside 1..6 (particles_adams_bashforth.hpp:24-28)",
                    nsteps);
    if (step_idx < 1) return fail(c, BFG_EINVAL, "step_idx must be >= 1");
    if (n >= (int64_t)1 << 31) return fail(c, BFG_EUNSUP, "more than 2^31 tracers");
    CU(cudaSetDevice(c->device));
    int rc = ensure_ru(c);
    if (rc) return rc;
    bfg_pctx* p = new bfg_pctx();
    p->ctx = c;
    p->n = n;
    p->neighbours = neighbours;
    p->smoothness = smoothness;
    p->nsteps = nsteps;
    p->step_idx = step_idx;
    p->head = 0;
    p->resort_every = c->n >= 256 ? 4 : 0;
    const size_t n1 = (size_t)std::max<int64_t>(n, 1);
    const size_t nb = n1 * 3 * sizeof(double);
    const size_t nbk = (size_t)c->n * c->n * sizeof(unsigned);
    bool ok = cudaMalloc(&p->pos, nb) == cudaSuccess && cudaMalloc(&p->pos2, nb) == cudaSuccess &&
              cudaMalloc(&p->hist, nb * nsteps) == cudaSuccess &&
              cudaMalloc(&p->hist2, nb * nsteps) == cudaSuccess &&
              cudaMalloc(&p->corder, n1 * 8) == cudaSuccess &&
              cudaMalloc(&p->corder2, n1 * 8) == cudaSuccess &&
              cudaMalloc(&p->sample, nb) == cudaSuccess &&
              cudaMalloc(&p->key, n1 * 4) == cudaSuccess &&
              cudaMalloc(&p->rank, n1 * 4) == cudaSuccess &&
              cudaMalloc(&p->perm, n1 * 4) == cudaSuccess &&
              cudaMalloc(&p->count, nbk) == cudaSuccess &&
              cudaMalloc(&p->offset, nbk + 1024 * sizeof(unsigned)) == cudaSuccess;
    if (!ok) {
        cudaGetLastError();
        bfg_particles_destroy(p);
        return fail(c, BFG_ENOMEM, "cannot allocate tracer state for %lld tracers", (long long)n);
    }
    p->idx.resize((size_t)n);
    for (int64_t i = 0; i < n; ++i) {
        p->idx[i] = idx ? idx[i] : i;
        if (p->idx[i] != i) p->identity = false;
    }
    if (!p->identity) {
        p->by_index.resize((size_t)n);
        for (int64_t i = 0; i < n; ++i) p->by_index[i] = i;
        std::sort(p->by_index.begin(), p->by_index.end(),
                  [&](int64_t a, int64_t b) { return p->idx[a] < p->idx[b]; });
    }
    *out = p;
    rc = bfg_particles_upload(p, pos, rhs, step_idx);
    if (rc) {
        *out = nullptr;
        bfg_particles_destroy(p);
        return rc;
    }
    return 0;
}

void bfg_particles_destroy(bfg_pctx* p) {
    if (!p) return;
    if (p->ctx) {
        cudaSetDevice(p->ctx->device);
        cudaStreamSynchronize(p->ctx->tstream);
        cudaStreamSynchronize(p->ctx->stream);
    }
    void* bufs[] = {p->pos, p->pos2, p->hist, p->hist2, p->corder, p->corder2,
                    p->sample, p->key, p->rank, p->count, p->offset, p->perm};
    for (void* b : bufs)
        if (b) cudaFree(b);
    delete p;
}

int bfg_particles_complete_loop(bfg_pctx* p, double dt) {
    if (!p) return BFG_EINVAL;
    bfg_ctx* c = p->ctx;
    CU(cudaSetDevice(c->device));
    if (int rj = join_tracers(c)) return rj;
    int rc = tracer_loop(p, dt);
    if (rc) return rc;
    CU(cudaStreamSynchronize(c->stream));
    return 0;
}

int bfg_particles_sample_velocity(bfg_pctx* p, double* out) {
    if (!p || !out) return BFG_EINVAL;
    bfg_ctx* c = p->ctx;
    CU(cudaSetDevice(c->device));
    if (int rj = join_tracers(c)) return rj;
    PParams pp = pparams(p, 0.0, 0);
    int rc = c->real_bytes == 4 ? tracers_dispatch<float>(c, pp, p, p->sample, c->stream)
                                : tracers_dispatch<double>(c, pp, p, p->sample, c->stream);
    if (rc) return rc;
    return fetch_index_order(p, p->sample, 3, out);
}

int bfg_particles_sample_acceleration(bfg_pctx* p, double* out) {
    if (!p || !out) return BFG_EINVAL;
    bfg_ctx* c = p->ctx;
    CU(cudaSetDevice(c->device));
    if (int rj = join_tracers(c)) return rj;
    int rc = ensure_ru(c);
    if (rc) return rc;
    if ((rc = sync_member(c, c->fac_dt))) return rc;
    if ((rc = dispatch<OpAccelR>(c))) return rc;
    PParams pp = pparams(p, 0.0, 0);
    rc = c->real_bytes == 4 ? tracers_dispatch<float>(c, pp, p, p->sample, c->stream, c->v2)
                            : tracers_dispatch<double>(c, pp, p, p->sample, c->stream, c->v2);
    if (rc) return rc;
    return fetch_index_order(p, p->sample, 3, out);
}

int bfg_particles_download(bfg_pctx* p, double* pos, double* rhs, int64_t* idx) {
    if (!p) return BFG_EINVAL;
    bfg_ctx* c = p->ctx;
    CU(cudaSetDevice(c->device));
    if (int rj = join_tracers(c)) return rj;
    const size_t n3 = (size_t)p->n * 3;
    int rc;
    if (pos && (rc = fetch_index_order(p, p->pos, 3, pos))) return rc;
    if (rhs) {
        for (int j = 0; j < p->nsteps; ++j) {
            if (j == 0 && p->rhs0_zero) {
                // logically zero slot: zeros through the link (faster than a
                // host fill of the caller's buffer)
                CU(cudaMemsetAsync(p->pos2, 0, n3 * 8, c->stream));
                CU(cudaMemcpyAsync(rhs, p->pos2, n3 * 8, cudaMemcpyDeviceToHost, c->stream));
                CU(cudaStreamSynchronize(c->stream));
                continue;
            }
            const int slot = (p->head + j) % p->nsteps;
            if ((rc = fetch_index_order(p, p->hist + (size_t)slot * n3, 3, rhs + (size_t)j * n3)))
                return rc;
        }
    }
    if (idx) {
        if (p->identity)
            for (int64_t i = 0; i < p->n; ++i) idx[i] = i;
        else
            for (int64_t k = 0; k < p->n; ++k) idx[k] = p->idx[p->by_index[k]];
    }
    return 0;
}

int bfg_particles_upload(bfg_pctx* p, const double* pos, const double* rhs, int step_idx) {
    if (!p || (p->n > 0 && !pos) || step_idx < 1) return BFG_EINVAL;
    bfg_ctx* c = p->ctx;
    CU(cudaSetDevice(c->device));
    if (int rj = join_tracers(c)) return rj;
    const size_t n3 = (size_t)p->n * 3;
    p->head = 0;
    p->step_idx = step_idx;
    if (p->n == 0) return 0;
    // back to creation order, then cell order
    CU(cudaMemcpyAsync(p->pos, pos, n3 * 8, cudaMemcpyHostToDevice, c->stream));
    if (rhs) {
        // rhs[0] as given: the next loop accumulates into it (rhs[0] += u(x),
        // completeLoop's own form; exact when the slot holds zeros)
        CU(cudaMemcpyAsync(p->hist, rhs, n3 * 8 * p->nsteps, cudaMemcpyHostToDevice, c->stream));
        p->rhs0_zero = false;
    } else {
        CU(cudaMemsetAsync(p->hist, 0, n3 * 8 * p->nsteps, c->stream));
        p->rhs0_zero = true;
    }
    iota64<<<(unsigned)((p->n + 255) / 256), 256, 0, c->stream>>>(p->corder, p->n);
    int rc = after_launch(c, "iota64");
    if (rc) return rc;
    if ((rc = tracer_sort(p))) return rc;
    CU(cudaStreamSynchronize(c->stream));
    return 0;
}

int bfg_particles_info(const bfg_pctx* p, int64_t* n, int* nsteps, int* step_idx) {
    if (!p) return BFG_EINVAL;
    if (n) *n = p->n;
    if (nsteps) *nsteps = p->nsteps;
    if (step_idx) *step_idx = p->step_idx;
    return 0;
}

}  // extern "C"

// ======================================================= no-allocation stats ==
// bfg_rspace_stats_noalloc: the real-space moments / histogram reduction of
// field::compute_rspace_stats for callers that cannot call cudaMalloc --
// for example a host whose device memory is already owned or reserved by
// another framework's caching allocator, an application that fixes its
// memory footprint at start-up, or a latency-sensitive loop that cannot
// afford cudaMalloc's implicit device-wide synchronisation.  The caller
// passes the input field and the output arrays; the per-block partial sums
// live in the fixed file-scope device array below instead of in memory the
// library would allocate.  The array exists on every GPU that loads the
// library, for as long as the library stays loaded.

// per-block partial sums: STATS_BLOCKS blocks x NQ doubles = 370 KiB
static __device__ __align__(256) double g_noalloc_partials[STATS_BLOCKS * NQ];

// same reduction as moments_kernel, over a field stored with a padded row
// pitch (the reference real layout (nz, ny, nx+2, 3))
template <typename T>
__global__ void __launch_bounds__(STATS_THREADS)
moments_pitched_kernel(const T* __restrict__ r, int nx, int pitch, size_t npts, double me0,
                       double me1, double me2, double me3, int nbins,
                       double* __restrict__ partial, unsigned long long* __restrict__ hist) {
    extern __shared__ unsigned int shist_p[];  // nbins * 4
    __shared__ double red[STATS_THREADS / 32][NQ];
    for (int i = threadIdx.x; i < nbins * 4; i += blockDim.x) shist_p[i] = 0;
    __syncthreads();
    const double me[4] = {me0, me1, me2, me3};
    double binsize[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) binsize[i] = 2 * me[i] / nbins;
    double mn[4] = {0.0, 0.0, 0.0, me3};
    double mx[4] = {0.0, 0.0, 0.0, 0.0};
    double sm[8][4];
#pragma unroll
    for (int n = 0; n < 8; ++n)
#pragma unroll
        for (int i = 0; i < 4; ++i) sm[n][i] = 0.0;
    for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < npts;
         e += (size_t)gridDim.x * blockDim.x) {
        const size_t x = e % (size_t)nx, rowi = e / (size_t)nx;
        const T* pt = r + (rowi * (size_t)pitch + x) * 3;
        double v[4];
        v[3] = 0.0;
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            v[i] = (double)pt[i];
            v[3] += v[i] * v[i];
        }
        v[3] = sqrt(v[3]);
        {
            const int b = (int)floor(v[3] * 2 / binsize[3]);
            if (b >= 0 && b < nbins) atomicAdd(&shist_p[b * 4 + 3], 1u);
        }
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            const int b = (int)floor((v[i] + me[i]) / binsize[i]);
            if (b >= 0 && b < nbins) atomicAdd(&shist_p[b * 4 + i], 1u);
        }
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            mn[i] = fmin(mn[i], v[i]);
            mx[i] = fmax(mx[i], v[i]);
            double p = 1.0;
#pragma unroll
            for (int n = 0; n < 8; ++n) {
                p = v[i] * p;
                sm[n][i] += p;
            }
        }
    }
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        double a = warp_min(mn[i]);
        double b = warp_max(mx[i]);
        if (lane == 0) {
            red[wid][0 * 4 + i] = a;
            red[wid][9 * 4 + i] = b;
        }
#pragma unroll
        for (int n = 0; n < 8; ++n) {
            double s = warp_sum(sm[n][i]);
            if (lane == 0) red[wid][(n + 1) * 4 + i] = s;
        }
    }
    __syncthreads();
    if (threadIdx.x < NQ) {
        const int q = threadIdx.x;
        double acc = red[0][q];
        for (int w = 1; w < STATS_THREADS / 32; ++w) {
            const double v = red[w][q];
            if (q < 4) acc = fmin(acc, v);
            else if (q >= 36) acc = fmax(acc, v);
            else acc += v;
        }
        partial[(size_t)blockIdx.x * NQ + q] = acc;
    }
    for (int i = threadIdx.x; i < nbins * 4; i += blockDim.x)
        if (shist_p[i]) atomicAdd(&hist[i], (unsigned long long)shist_p[i]);
}

// Device address of g_noalloc_partials in the current device context.  Host
// code cannot use the array's name as a device pointer, so the address is
// looked up (cudaGetSymbolAddress, with the device current) and cached per
// device context: the key is the context's unique id (cuCtxGetId, reached
// through cudaGetDriverEntryPoint so that nothing links libcuda), so a
// device reset, which creates a new context and may load the module at a new
// address, makes the next call look the address up again.  Where the context
// id cannot be read the address is looked up on every call.
typedef int (*CtxGetCurrentFn)(void**);
typedef int (*CtxGetIdFn)(void*, unsigned long long*);
static bool current_ctx_id(unsigned long long* id) {
    static CtxGetCurrentFn get_cur = nullptr;
    static CtxGetIdFn get_id = nullptr;
    static bool tried = false;
    if (!tried) {
        tried = true;
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_cur = (CtxGetCurrentFn)f;
        f = nullptr;
        if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_id = (CtxGetIdFn)f;
        cudaGetLastError();
    }
    if (!get_cur || !get_id) return false;
    void* ctx = nullptr;
    if (get_cur(&ctx) != 0 || !ctx) return false;
    return get_id(ctx, id) == 0;
}

static double* noalloc_partials_on(int device, cudaError_t* err) {
    static std::mutex mu;
    static std::unordered_map<unsigned long long, double*> addr;  // context id -> address
    std::lock_guard<std::mutex> lk(mu);
    unsigned long long id = 0;
    const bool keyed = current_ctx_id(&id);
    if (keyed) {
        auto it = addr.find(id);
        if (it != addr.end()) return it->second;
    }
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_partials);
    if (e != cudaSuccess) {
        cudaGetLastError();  // do not leave the lookup's error pending
        *err = e;
        return nullptr;
    }
    (void)device;
    if (keyed) addr[id] = static_cast<double*>(p);
    return static_cast<double*>(p);
}

extern "C" int bfg_rspace_stats_noalloc(const void* dev_field, int nx, int ny, int nz,
                                        int real_bytes, double max_estimate, int nbins,
                                        double* dev_moments, int64_t* dev_hist, void* stream) {
    if (!dev_field || !dev_moments || !dev_hist) return BFG_EINVAL;
    if (nx < 1 || ny < 1 || nz < 1 || (real_bytes != 4 && real_bytes != 8)) return BFG_EINVAL;
    if (nbins < 1) return BFG_EINVAL;
    if (nbins > BFG_NOALLOC_MAX_BINS) return BFG_EUNSUP;  // shared-memory histogram limit
    int device = 0;
    if (cudaGetDevice(&device) != cudaSuccess) {
        cudaGetLastError();
        return BFG_ECUDA;
    }
    cudaError_t err = cudaSuccess;
    double* partials = noalloc_partials_on(device, &err);
    if (!partials) return BFG_ECUDA;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const size_t npts = (size_t)nx * ny * nz;
    // the reference's padded real layout: rows of 2 (nx/2 + 1) points
    // (field_layout of the in-place R2C buffer), nx + 2 for even nx
    const int pitch = 2 * (nx / 2 + 1);
    // the histogram is accumulated into the caller's output: start it at zero
    if (cudaMemsetAsync(dev_hist, 0, (size_t)nbins * 4 * sizeof(int64_t), s) != cudaSuccess) {
        cudaGetLastError();
        return BFG_ECUDA;
    }
    const double me3 = max_estimate * std::sqrt(3.0);
    const size_t shmem = (size_t)nbins * 4 * sizeof(unsigned int);
    if (real_bytes == 4)
        moments_pitched_kernel<float><<<STATS_BLOCKS, STATS_THREADS, shmem, s>>>(
            static_cast<const float*>(dev_field), nx, pitch, npts, max_estimate, max_estimate,
            max_estimate, me3, nbins, partials, reinterpret_cast<unsigned long long*>(dev_hist));
    else
        moments_pitched_kernel<double><<<STATS_BLOCKS, STATS_THREADS, shmem, s>>>(
            static_cast<const double*>(dev_field), nx, pitch, npts, max_estimate, max_estimate,
            max_estimate, me3, nbins, partials, reinterpret_cast<unsigned long long*>(dev_hist));
    // a failed first launch must not queue the final reduction
    if (cudaGetLastError() != cudaSuccess) return BFG_ECUDA;
    moments_final<<<1, 64, 0, s>>>(partials, STATS_BLOCKS, 1.0 / (double)npts, dev_moments);
    if (cudaGetLastError() != cudaSuccess) return BFG_ECUDA;
    return BFG_OK;
}

// ============================================================== ensembles ==
// Many independent instances advanced together: members of equal grid size
// form a group, and every pass of an RK stage is one persistent launch over
// all members of a group (the tile index decodes to member, then tile).
// The fluid launches of each stage are captured once into CUDA graphs and
// replayed; each member's tracers follow stage 1, which produces its u(t).

struct EnsGroup {
    int n = 0;
    std::vector<int> members;  // indices into bfg_ens::entries
    void* dmem = nullptr;      // Member<T>[members.size()]
    size_t cap = 0;
    bfg_ctx launcher;          // stream / SM count / twiddles / errors for this group's launches
    cudaGraphExec_t graph[3] = {nullptr, nullptr, nullptr};  // stage 1 (+ru), 2, 3 + symmetrize
    int64_t graph_kernels[3] = {0, 0, 0};                       // kernel nodes of each graph
    bool any_tracers = false;
    // each size group runs on its own stream, so the passes of small grids
    // fill the SMs around those of large ones; its own tile counters
    cudaStream_t stream = nullptr;
    cudaEvent_t ev_s1 = nullptr;    // stage 1 (and u(t)) of this step written
    cudaEvent_t ev_done = nullptr;  // this group's last launch of the call
    int* tctr = nullptr;
};

struct bfg_ens {
    int device = 0;
    int real_bytes = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr, ev_ru = nullptr;  // ev_ru: tracers of the step done
    struct Entry {
        bfg_ctx* ctx;
        bfg_pctx* tracers;
        double dt;
    };
    std::vector<Entry> entries;
    std::vector<EnsGroup*> groups;
    // tracer systems advanced by one batched launch (same interpolation, no
    // re-sorting); the others use their own loop
    std::vector<int> batched;   // entry indices
    void* dsets = nullptr;      // TracerSet[batched.size()]
    void* dstart = nullptr;     // int64[batched.size() + 1]: first block of each set
    int64_t nbatched = 0;       // blocks of the batched tracer launch
    bool dirty = true;
    bool use_graphs = true;
    int64_t launches = 0; // kernels launched by bfg_ens_step (graph nodes included)
    std::string err;
};

static int ens_fail(bfg_ens* e, int code, const char* msg) {
    if (e) e->err = msg;
    return code;
}

template <typename T, int NB, int MM>
static int ens_tracers_launch(bfg_ens* e) {
    const unsigned blocks = (unsigned)e->nbatched;  // blocks over all sets
    if (blocks == 0) return 0;
    tracer_batch_kernel<T, NB, MM><<<blocks, TRACER_THREADS, 0, e->stream>>>(
        (const TracerSet*)e->dsets, (const int64_t*)e->dstart, (int)e->batched.size());
    tracer_sets_advance<<<((int)e->batched.size() + 127) / 128, 128, 0, e->stream>>>(
        (TracerSet*)e->dsets, (int)e->batched.size());
    return cudaGetLastError() == cudaSuccess ? 0 : BFG_ECUDA;
}
template <typename T>
static int ens_tracers_dispatch(bfg_ens* e, int nb, int mm) {
#define BFG_ETR(NBv, MMv) \
    if (nb == NBv && mm == MMv) return ens_tracers_launch<T, NBv, MMv>(e);
    BFG_ETR(1, 0) BFG_ETR(1, 1) BFG_ETR(1, 2)
    BFG_ETR(2, 0) BFG_ETR(2, 1) BFG_ETR(2, 2)
    BFG_ETR(3, 0) BFG_ETR(3, 1) BFG_ETR(3, 2)
    BFG_ETR(4, 0) BFG_ETR(4, 1) BFG_ETR(4, 2)
    BFG_ETR(5, 0) BFG_ETR(5, 1) BFG_ETR(5, 2)
#undef BFG_ETR
    return BFG_EUNSUP;
}

static void ens_free_groups(bfg_ens* e) {
    if (e->dsets) cudaFree(e->dsets);
    if (e->dstart) cudaFree(e->dstart);
    e->dsets = e->dstart = nullptr;
    e->batched.clear();
    e->nbatched = 0;
    for (EnsGroup* g : e->groups) {
        if (g->stream) cudaStreamSynchronize(g->stream);
        for (auto& ge : g->graph)
            if (ge) cudaGraphExecDestroy(ge);
        if (g->dmem) cudaFree(g->dmem);
        if (g->tctr) cudaFree(g->tctr);
        if (g->ev_s1) cudaEventDestroy(g->ev_s1);
        if (g->ev_done) cudaEventDestroy(g->ev_done);
        if (g->stream) cudaStreamDestroy(g->stream);
        delete g;
    }
    e->groups.clear();
}

template <typename T>
static Member<T> member_of(bfg_ctx* c, double dt) {
    Member<T> m;
    memset(&m, 0, sizeof(m));
    m.kp = kparams(c, dt);
    m.buf[B_W0] = (cpx<T>*)c->w0;
    m.buf[B_V1] = (cpx<T>*)c->v1;
    m.buf[B_V2] = (cpx<T>*)c->v2;
    m.buf[B_WA] = (cpx<T>*)c->wa;
    m.buf[B_WB] = (cpx<T>*)c->wb;
    m.ru = (T*)c->ru;
    m.filt = (const T*)c->filt;
    m.fac = (const T*)c->fac;
    return m;
}

template <typename T, int N>
struct EnsOps {
    using E = Engine<T, N>;
    static int stage(EnsGroup* g, int s) {
        const Member<T>* mem = (const Member<T>*)g->dmem;
        const int nm = (int)g->members.size();
        int rc = E::stage(&g->launcher, mem, nm, s, s == 0 && g->any_tracers);
        if (rc) return rc;
        if (s == 2) rc = E::finish_step(&g->launcher, mem, nm);
        return rc;
    }
};

template <typename T>
static int ens_group_stage(EnsGroup* g, int s) {
    switch (g->n) {
        case 16: return EnsOps<T, 16>::stage(g, s);
        case 32: return EnsOps<T, 32>::stage(g, s);
        case 64: return EnsOps<T, 64>::stage(g, s);
        case 128: return EnsOps<T, 128>::stage(g, s);
        case 256: return EnsOps<T, 256>::stage(g, s);
        case 512: return EnsOps<T, 512>::stage(g, s);
        case 1024: return EnsOps<T, 1024>::stage(g, s);
    }
    return BFG_EUNSUP;
}

static int ens_stage(bfg_ens* e, EnsGroup* g, int s) {
    return e->real_bytes == 4 ? ens_group_stage<float>(g, s) : ens_group_stage<double>(g, s);
}

// both column-pass schedules timed on a whole size group (one launch over
// all its members, as bfg_ens_step issues them)
template <typename T>
static int ens_group_tune(EnsGroup* g, int reps, double* ms) {
    const Member<T>* mem = (const Member<T>*)g->dmem;
    const int nm = (int)g->members.size();
    switch (g->n) {
        case 16: return Engine<T, 16>::tune(&g->launcher, mem, nm, reps, ms);
        case 32: return Engine<T, 32>::tune(&g->launcher, mem, nm, reps, ms);
        case 64: return Engine<T, 64>::tune(&g->launcher, mem, nm, reps, ms);
        case 128: return Engine<T, 128>::tune(&g->launcher, mem, nm, reps, ms);
        case 256: return Engine<T, 256>::tune(&g->launcher, mem, nm, reps, ms);
        case 512: return Engine<T, 512>::tune(&g->launcher, mem, nm, reps, ms);
        case 1024: return Engine<T, 1024>::tune(&g->launcher, mem, nm, reps, ms);
    }
    return BFG_EUNSUP;
}

// (re)build groups, member arrays and graphs after membership changes
static int ens_prepare(bfg_ens* e) {
    if (!e->dirty) return 0;
    cudaSetDevice(e->device);
    // nothing in flight may still use the descriptors freed here
    if (cudaStreamSynchronize(e->stream) != cudaSuccess)
        return ens_fail(e, BFG_ECUDA, "ensemble stream synchronisation failed");
    ens_free_groups(e);
    std::vector<int> sizes;
    for (auto& en : e->entries)
        if (std::find(sizes.begin(), sizes.end(), en.ctx->n) == sizes.end()) sizes.push_back(en.ctx->n);
    std::sort(sizes.rbegin(), sizes.rend());  // large grids first
    for (int n : sizes) {
        EnsGroup* g = new EnsGroup();
        g->n = n;
        for (int i = 0; i < (int)e->entries.size(); ++i)
            if (e->entries[i].ctx->n == n) g->members.push_back(i);
        bfg_ctx* c0 = e->entries[g->members[0]].ctx;
        g->launcher.n = n;
        g->launcher.nxv = c0->nxv;
        g->launcher.nxp = c0->nxp;
        g->launcher.nsm = c0->nsm;
        g->launcher.smem_optin = c0->smem_optin;
        g->launcher.real_bytes = c0->real_bytes;
        g->launcher.device = c0->device;
        g->launcher.tw = c0->tw;
        e->groups.push_back(g);
        if (cudaStreamCreateWithFlags(&g->stream, cudaStreamNonBlocking) != cudaSuccess ||
            cudaEventCreateWithFlags(&g->ev_s1, cudaEventDisableTiming) != cudaSuccess ||
            cudaEventCreateWithFlags(&g->ev_done, cudaEventDisableTiming) != cudaSuccess ||
            cudaMalloc(&g->tctr, 64) != cudaSuccess || cudaMemset(g->tctr, 0, 64) != cudaSuccess) {
            cudaGetLastError();
            return ens_fail(e, BFG_ECUDA, "cannot create the group's stream, events or counters");
        }
        g->launcher.stream = g->stream;
        g->launcher.tctr = g->tctr;
        for (int i : g->members) g->any_tracers = g->any_tracers || e->entries[i].tracers != nullptr;
        // member descriptors
        std::vector<unsigned char> host;
        for (int i : g->members) {
            auto& en = e->entries[i];
            if (e->real_bytes == 4) {
                Member<float> m = member_of<float>(en.ctx, en.dt);
                host.insert(host.end(), (unsigned char*)&m, (unsigned char*)&m + sizeof(m));
            } else {
                Member<double> m = member_of<double>(en.ctx, en.dt);
                host.insert(host.end(), (unsigned char*)&m, (unsigned char*)&m + sizeof(m));
            }
        }
        if (cudaMalloc(&g->dmem, host.size()) != cudaSuccess) {
            cudaGetLastError();
            return ens_fail(e, BFG_ENOMEM, "cannot allocate member descriptors");
        }
        if (cudaMemcpy(g->dmem, host.data(), host.size(), cudaMemcpyHostToDevice) != cudaSuccess)
            return ens_fail(e, BFG_ECUDA, "member descriptor upload failed");
        g->cap = host.size();
        if (e->use_graphs) {
            for (int s = 0; s < 3; ++s) {
                cudaGraph_t graph = nullptr;
                if (cudaStreamBeginCapture(g->stream, cudaStreamCaptureModeRelaxed) != cudaSuccess)
                    return ens_fail(e, BFG_ECUDA, "stream capture failed to start");
                const int64_t l0 = g->launcher.launches;
                int rc = ens_stage(e, g, s);
                g->graph_kernels[s] = g->launcher.launches - l0;
                cudaError_t ce = cudaStreamEndCapture(g->stream, &graph);
                if (rc || ce != cudaSuccess) {
                    if (graph) cudaGraphDestroy(graph);
                    return ens_fail(e, rc ? rc : BFG_ECUDA,
                                    rc ? g->launcher.err.c_str() : "stream capture failed");
                }
                ce = cudaGraphInstantiate(&g->graph[s], graph, 0);
                cudaGraphDestroy(graph);
                if (ce != cudaSuccess) return ens_fail(e, BFG_ECUDA, "graph instantiation failed");
            }
        }
    }
    // batched tracer sets: every member with tracers on a grid below 256^3
    // whose interpolation matches the first such member
    std::vector<TracerSet> sets;
    std::vector<int64_t> start(1, 0);
    for (int i = 0; i < (int)e->entries.size(); ++i) {
        auto& en = e->entries[i];
        bfg_pctx* p = en.tracers;
        if (!p || p->resort_every != 0 || p->n == 0) continue;
        if (!e->batched.empty()) {
            bfg_pctx* p0 = e->entries[e->batched[0]].tracers;
            if (p->neighbours != p0->neighbours || p->smoothness != p0->smoothness) continue;
        }
        TracerSet ts;
        memset(&ts, 0, sizeof(ts));
        ts.pp = pparams(p, en.dt, 1);
        ts.step_idx = p->step_idx;
        ts.ru = en.ctx->ru;
        ts.pos = p->pos;
        ts.hist = p->hist;
        sets.push_back(ts);
        const int64_t tpb = e->real_bytes == 4 ? tracers_per_block<float>() : tracers_per_block<double>();
        start.push_back(start.back() + (p->n + tpb - 1) / tpb);
        e->batched.push_back(i);
    }
    if (!sets.empty()) {
        if (cudaMalloc(&e->dsets, sets.size() * sizeof(TracerSet)) != cudaSuccess ||
            cudaMalloc(&e->dstart, start.size() * sizeof(int64_t)) != cudaSuccess) {
            cudaGetLastError();
            return ens_fail(e, BFG_ENOMEM, "cannot allocate tracer sets");
        }
        if (cudaMemcpy(e->dsets, sets.data(), sets.size() * sizeof(TracerSet), cudaMemcpyHostToDevice) !=
                cudaSuccess ||
            cudaMemcpy(e->dstart, start.data(), start.size() * sizeof(int64_t), cudaMemcpyHostToDevice) !=
                cudaSuccess)
            return ens_fail(e, BFG_ECUDA, "tracer set upload failed");
        e->nbatched = start.back();
    }
    e->dirty = false;
    return 0;
}

extern "C" {

int bfg_ens_create(bfg_ens** out, int device) {
    if (!out) return BFG_EINVAL;
    *out = nullptr;
    if (cudaSetDevice(device) != cudaSuccess) {
        cudaGetLastError();
        return BFG_ECUDA;
    }
    bfg_ens* e = new bfg_ens();
    e->device = device;
    if (cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete e;
        return BFG_ECUDA;
    }
    cudaEventCreate(&e->ev0);
    cudaEventCreate(&e->ev1);
    cudaEventCreateWithFlags(&e->ev_ru, cudaEventDisableTiming);
    *out = e;
    return 0;
}

void bfg_ens_destroy(bfg_ens* e) {
    if (!e) return;
    cudaSetDevice(e->device);
    cudaStreamSynchronize(e->stream);
    for (auto& en : e->entries) cudaStreamSynchronize(en.ctx->tstream);
    ens_free_groups(e);
    cudaEventDestroy(e->ev0);
    cudaEventDestroy(e->ev1);
    cudaEventDestroy(e->ev_ru);
    cudaStreamDestroy(e->stream);
    delete e;
}

const char* bfg_ens_last_error(const bfg_ens* e) { return e ? e->err.c_str() : "null ensemble"; }

int bfg_ens_add(bfg_ens* e, bfg_ctx* c, bfg_pctx* p, double dt) {
    if (!e || !c || !(dt > 0)) return BFG_EINVAL;
    if (p && p->ctx != c) return ens_fail(e, BFG_EINVAL, "tracers belong to another context");
    if (c->device != e->device) return ens_fail(e, BFG_EINVAL, "member on another device");
    if (e->real_bytes && c->real_bytes != e->real_bytes)
        return ens_fail(e, BFG_EINVAL, "members must share one precision");
    for (auto& en : e->entries)
        if (en.ctx == c) return ens_fail(e, BFG_EINVAL, "context already in the ensemble");
    cudaSetDevice(e->device);
    int rc = ensure_factors(c, dt);
    if (rc) return ens_fail(e, rc, c->err.c_str());
    if ((rc = ensure_ru(c))) return ens_fail(e, rc, c->err.c_str());
    // the member's own streams are idle from here on; the ensemble orders
    // itself after anything still queued there
    if (cudaStreamSynchronize(c->stream) != cudaSuccess || cudaStreamSynchronize(c->tstream) != cudaSuccess)
        return ens_fail(e, BFG_ECUDA, "member stream synchronisation failed");
    e->real_bytes = c->real_bytes;
    e->entries.push_back({c, p, dt});
    e->dirty = true;
    return 0;
}

int bfg_ens_remove(bfg_ens* e, bfg_ctx* c) {
    if (!e || !c) return BFG_EINVAL;
    cudaSetDevice(e->device);
    cudaStreamSynchronize(e->stream);
    for (size_t i = 0; i < e->entries.size(); ++i)
        if (e->entries[i].ctx == c) {
            cudaStreamSynchronize(c->tstream);
            e->entries.erase(e->entries.begin() + i);
            e->dirty = true;
            if (e->entries.empty()) e->real_bytes = 0;
            return 0;
        }
    return ens_fail(e, BFG_EINVAL, "context not in the ensemble");
}

int bfg_ens_count(const bfg_ens* e, int* members) {
    if (!e || !members) return BFG_EINVAL;
    *members = (int)e->entries.size();
    return 0;
}

int bfg_ens_step(bfg_ens* e, int nsteps) {
    if (!e || nsteps < 0) return BFG_EINVAL;
    if (e->entries.empty()) return 0;
    cudaSetDevice(e->device);
    int rc = ens_prepare(e);
    if (rc) return rc;
    // e->stream carries the tracers and orders the call: it starts the
    // groups (ev0), waits for their stage 1 before the tracers, and joins
    // them at the end (ev1)
    for (auto& en : e->entries)
        if (en.tracers) cudaStreamWaitEvent(e->stream, en.ctx->ev_tr, 0);
    if (cudaEventRecord(e->ev0, e->stream) != cudaSuccess ||
        cudaEventRecord(e->ev_ru, e->stream) != cudaSuccess)
        return ens_fail(e, BFG_ECUDA, "event");
    auto launch_stage = [&](EnsGroup* g, int s) -> int {
        const int64_t l0 = g->launcher.launches;
        int r = e->use_graphs ? (cudaGraphLaunch(g->graph[s], g->stream) == cudaSuccess ? 0 : BFG_ECUDA)
                              : ens_stage(e, g, s);
        e->launches += e->use_graphs ? g->graph_kernels[s] : g->launcher.launches - l0;
        return r;
    };
    for (int st = 0; st < nsteps; ++st) {
        // the previous step's tracers read ru, which stage 1 rewrites
        for (EnsGroup* g : e->groups) {
            if (cudaStreamWaitEvent(g->stream, e->ev_ru, 0) != cudaSuccess)
                return ens_fail(e, BFG_ECUDA, "event");
            if ((rc = launch_stage(g, 0))) return ens_fail(e, rc, "stage 1 launch failed");
            if (cudaEventRecord(g->ev_s1, g->stream) != cudaSuccess ||
                cudaStreamWaitEvent(e->stream, g->ev_s1, 0) != cudaSuccess)
                return ens_fail(e, BFG_ECUDA, "event");
        }
        if (!e->batched.empty()) {
            bfg_pctx* p0 = e->entries[e->batched[0]].tracers;
            rc = e->real_bytes == 4 ? ens_tracers_dispatch<float>(e, p0->neighbours, p0->smoothness)
                                    : ens_tracers_dispatch<double>(e, p0->neighbours, p0->smoothness);
            if (rc) return ens_fail(e, rc, "batched tracer launch failed");
            e->launches += 2;
            for (int i : e->batched) {
                // host mirror of tracer_sets_advance
                bfg_pctx* p = e->entries[i].tracers;
                p->step_idx += 1;
                p->head = (p->head - 1 + p->nsteps) % p->nsteps;
                p->rhs0_zero = true;
            }
        }
        for (int i = 0; i < (int)e->entries.size(); ++i) {
            auto& en = e->entries[i];
            if (!en.tracers) continue;
            bfg_ctx* c = en.ctx;
            if (std::find(e->batched.begin(), e->batched.end(), i) == e->batched.end()) {
                const int64_t l0 = c->launches;
                if ((rc = tracer_loop(en.tracers, en.dt, e->stream))) return ens_fail(e, rc, c->err.c_str());
                e->launches += c->launches - l0;
            }
            if (cudaEventRecord(c->ev_tr, e->stream) != cudaSuccess) return ens_fail(e, BFG_ECUDA, "event");
        }
        if (cudaEventRecord(e->ev_ru, e->stream) != cudaSuccess) return ens_fail(e, BFG_ECUDA, "event");
        // stages 2-3 touch neither ru nor the tracer state
        for (EnsGroup* g : e->groups)
            for (int s = 1; s < 3; ++s)
                if ((rc = launch_stage(g, s))) return ens_fail(e, rc, "stage launch failed");
        for (auto& en : e->entries) en.ctx->iteration++;
    }
    for (EnsGroup* g : e->groups)
        if (cudaEventRecord(g->ev_done, g->stream) != cudaSuccess ||
            cudaStreamWaitEvent(e->stream, g->ev_done, 0) != cudaSuccess)
            return ens_fail(e, BFG_ECUDA, "event");
    if (cudaEventRecord(e->ev1, e->stream) != cudaSuccess) return ens_fail(e, BFG_ECUDA, "event");
    // members' own streams follow the ensemble's work
    for (auto& en : e->entries) cudaStreamWaitEvent(en.ctx->stream, e->ev1, 0);
    cudaError_t ce = cudaGetLastError();
    if (ce != cudaSuccess) return ens_fail(e, BFG_ECUDA, cudaGetErrorString(ce));
    return 0;
}

int bfg_ens_autotune(bfg_ens* e, int reps) {
    if (!e) return BFG_EINVAL;
    if (reps < 1) reps = 1;
    if (e->entries.empty()) return 0;
    cudaSetDevice(e->device);
    int rc = ens_prepare(e);
    if (rc) return rc;
    // the groups' streams follow everything the ensemble queued so far
    if (cudaStreamSynchronize(e->stream) != cudaSuccess)
        return ens_fail(e, BFG_ECUDA, "ensemble stream synchronisation failed");
    for (EnsGroup* g : e->groups) {
        double ms[2 * BFG_NKINDS] = {0};
        rc = e->real_bytes == 4 ? ens_group_tune<float>(g, reps, ms) : ens_group_tune<double>(g, reps, ms);
        if (rc) return ens_fail(e, rc, g->launcher.err.c_str());
        tune_store(e->device, g->n, e->real_bytes, (int)g->members.size(), ms,
                   e->groups.size() > 1 ? TUNE_MARGIN_SHARED : TUNE_MARGIN);
    }
    // captured graphs hold the old schedules: rebuild them before the next step
    e->dirty = true;
    return 0;
}

int bfg_ens_last_ms(bfg_ens* e, double* ms) {
    if (!e || !ms) return BFG_EINVAL;
    cudaSetDevice(e->device);
    if (cudaEventSynchronize(e->ev1) != cudaSuccess) return ens_fail(e, BFG_ECUDA, "event sync");
    float f = 0;
    if (cudaEventElapsedTime(&f, e->ev0, e->ev1) != cudaSuccess) return ens_fail(e, BFG_ECUDA, "timing");
    *ms = f;
    return 0;
}

int bfg_ens_wait(bfg_ens* e, double timeout_ms, int* done) {
    if (!e || !done || !(timeout_ms >= 0.0)) return BFG_EINVAL;
    cudaSetDevice(e->device);
    const auto t0 = std::chrono::steady_clock::now();
    for (;;) {
        const cudaError_t q = cudaEventQuery(e->ev1);
        if (q == cudaSuccess) {
            *done = 1;
            return 0;
        }
        if (q != cudaErrorNotReady) return ens_fail(e, BFG_ECUDA, cudaGetErrorString(q));
        const double ms =
            std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        if (ms >= timeout_ms) {
            *done = 0;
            return 0;
        }
        std::this_thread::sleep_for(std::chrono::microseconds(50));
    }
}

int bfg_ens_kernel_launches(const bfg_ens* e, int64_t* count) {
    if (!e || !count) return BFG_EINVAL;
    *count = e->launches;
    return 0;
}

int bfg_ens_use_graphs(bfg_ens* e, int enable) {
    if (!e) return BFG_EINVAL;
    e->use_graphs = enable != 0;
    e->dirty = true;
    return 0;
}

}  // extern "C"
