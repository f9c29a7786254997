// Host-side helpers and state shared by the library's translation units:
// status messages, launch counting, kernel timing records, launch-shape knobs,
// scans and the index-guard check.  State is held in C++17 inline variables,
// so every translation unit sees one copy; helpers are static inline.
#pragma once
#include <mutex>
#include <stddef.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "gw_step_kernels.cuh"
#include "gw_krylov.cuh"

namespace gwh {
using namespace gw;


inline thread_local char g_msg[512];

#define GW_CUDA(call)                                                                         \
    do {                                                                                      \
        cudaError_t e_ = (call);                                                              \
        if (e_ != cudaSuccess) {                                                              \
            snprintf(g_msg, sizeof(g_msg), "%s:%d %s", __FILE__, __LINE__, cudaGetErrorString(e_)); \
            return GW_ECUDA;                                                                  \
        }                                                                                     \
    } while (0)
#define GW_LAUNCHED() GW_CUDA(cudaGetLastError())
#define GW_REQUIRE(cond)                                                      \
    do {                                                                      \
        if (!(cond)) {                                                        \
            snprintf(g_msg, sizeof(g_msg), "invalid argument: %s", #cond);    \
            return GW_EINVAL;                                                 \
        }                                                                     \
    } while (0)

static inline cudaStream_t S(void *s) { return (cudaStream_t)s; }

// -------------------------------------------------------------- optional kernel timing
// When enabled, selected launches are bracketed by CUDA events on their stream;
// gw_profile_read() synchronises and reports per-class totals and the
// algorithmic bytes the host attributed to each launch.
enum ProfClass {
    PC_ASSEMBLE = 0, PC_SPMV, PC_DOTS, PC_UPDATE, PC_NEXT, PC_G2P, PC_ADJ_G2P, PC_ADJ_RES,
    PC_MG_JACOBI, PC_MG_RESID, PC_MG_TRANSFER, PC_MG_SETUP, PC_MG_JACOBI_COARSE, PC_MG_TAIL, PC_COUNT
};
inline const char *kProfNames[PC_COUNT] = {"k_assemble", "k_gm_spmv", "k_gm_dots", "k_gm_update", "k_gm_next", "k_g2p",
                                    "k_adjoint_g2p", "k_adjoint_residual", "k_mg_jacobi (finest level)",
                                    "k_mg_residual", "k_mg_restrict/prolong", "mg_setup",
                                    "k_mg_jacobi (coarse levels)", "k_mg_tail (fused coarse levels)"};
// Event pairs are kept in a pool (created once, reused by later records).
struct ProfRec { int cls; cudaEvent_t a, b; double bytes; bool made; };
inline bool g_prof_on = false;
inline ProfRec *g_prof = nullptr;
inline int g_prof_n = 0, g_prof_cap = 0;
inline double g_prof_ms[PC_COUNT], g_prof_bytes[PC_COUNT];
inline long g_prof_count[PC_COUNT];

namespace {
// A bounded pause of the stream (%globaltimer, at most ns nanoseconds and a
// fixed number of polls): the host queues the next timed launches meanwhile.
__global__ void k_prof_delay(long long ns) {
    long long t0, t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t0));
    for (int i = 0; i < 1000000; ++i) {
        asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
        if (t - t0 >= ns) break;
        __nanosleep(500);
    }
}
}  // namespace

// Brackets one launch (or a short sequence) with events on its stream.  The
// interval [a, b] must not contain host time: when the previous timed launch
// has already finished, the GPU is idle and would start this launch as soon as
// the host submits it, so the submission gap would be timed too.  Then a
// 200-microsecond pause goes in first, and the host queues ahead of the GPU
// again before the interval opens on the device.
struct ProfScope {
    int idx = -1;
    cudaStream_t s;
    ProfScope(int cls, cudaStream_t st, double bytes) : s(st) {
        if (!g_prof_on) return;
        if (g_prof_n == g_prof_cap) {
            int nc = g_prof_cap ? 2 * g_prof_cap : 4096;
            ProfRec *nr = (ProfRec *)realloc(g_prof, sizeof(ProfRec) * nc);
            if (!nr) return;
            for (int i = g_prof_cap; i < nc; ++i) nr[i].made = false;
            g_prof = nr;
            g_prof_cap = nc;
        }
        idx = g_prof_n++;
        ProfRec &r = g_prof[idx];
        r.cls = cls;
        r.bytes = bytes;
        if (!r.made) {
            cudaEventCreate(&r.a);
            cudaEventCreate(&r.b);
            r.made = true;
        }
        if (idx == 0 || cudaEventQuery(g_prof[idx - 1].b) == cudaSuccess) k_prof_delay<<<1, 1, 0, s>>>(200000);
        cudaEventRecord(r.a, s);
    }
    ~ProfScope() {
        if (idx >= 0) cudaEventRecord(g_prof[idx].b, s);
    }
};
// every kernel launch of the library passes its grid size through here, so the
// host can report how many launches a piece of work took (gw_launch_count)
inline int64_t g_launches = 0;
static inline int gw_count_launch(int grid) {
    ++g_launches;
    return grid;
}
static inline int nblk(int64_t n, int t) { return (int)((n + t - 1) / t); }
// The row kernels gather 2x2 and 4x4 blocks and their vectors with 16-byte
// loads: those systems need 16-byte aligned values and vectors.
static inline bool aligned16(const void *p) { return ((uintptr_t)p & 15u) == 0; }
static inline bool vec_ok(const gw_bsr_t *A, const void *u, const void *v) {
    if (A->nf != 2 && A->nf != 4) return true;
    return aligned16(A->vals) && aligned16(u) && aligned16(v);
}

// launch-shape knobs (gw_tune_set): particle CTA, adjoint CTA, warps per CTA
// of the multigrid row kernels, bound of the dense coarsest level
inline int g_tune[GW_TUNE_COUNT] = {256, 128, 8, 160, GW_MG_MAX_LEVELS, 2, 70, 20, 0, 0, 1, 50};
// block-row kernels: kRowsPerWarp rows per warp (groups of kLPR lanes)
static inline int tune_rows_grid(int n_rows) {
    const int w = g_tune[GW_TUNE_ROW_WARPS];
    int b = nblk(n_rows, (int64_t)w * kRowsPerWarp);
    return b < 1 ? 1 : (b > kRedBlocks ? kRedBlocks : b);
}
static inline int tune_rows_block() { return 32 * g_tune[GW_TUNE_ROW_WARPS]; }
static inline int red_grid_rows(int n_rows) {
    int b = nblk(n_rows, (kThreads / 32) * kRowsPerWarp);
    return b < 1 ? 1 : (b > kRedBlocks ? kRedBlocks : b);
}
static inline int red_grid_elems(int64_t n) { int b = nblk(n, kThreads); return b < 1 ? 1 : (b > kRedBlocks ? kRedBlocks : b); }

// Grid of a grid-stride block-row kernel that has no cross-block reduction
// (each row's result is independent of the grid): the CTAs of `block` threads
// the device keeps resident at once, so the rows run in one wave with no
// partly filled last wave, and at most the CTAs the rows need.  The resident
// count comes from the occupancy calculator once per kernel, block size and
// device.
static inline int resident_rows_grid(const void *fn, int block, int n_rows) {
    struct Ent { const void *fn; int block, dev, nb; };
    static Ent cache[256];
    static int n = 0;
    static std::mutex mu;
    int dev = 0;
    (void)cudaGetDevice(&dev);
    int nb = 0;
    {
        std::lock_guard<std::mutex> lk(mu);
        for (int i = 0; i < n; ++i)
            if (cache[i].fn == fn && cache[i].block == block && cache[i].dev == dev) { nb = cache[i].nb; break; }
        if (!nb) {
            int per = 0, sms = 0;
            if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, fn, block, 0) != cudaSuccess || per < 1) per = 1;
            if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms < 1) sms = 1;
            (void)cudaGetLastError();
            nb = per * sms;
            if (n < 256) cache[n++] = {fn, block, dev, nb};
        }
    }
    const int want = nblk(n_rows, (int64_t)(block / 32) * kRowsPerWarp);
    return want < 1 ? 1 : (want < nb ? want : nb);
}

static inline LaunchConst make_lc(const gw_grid_t *g, const gw_material_t *m, const gw_step_t *st) {
    LaunchConst c;
    memset(&c, 0, sizeof(c));
    c.g = *g;
    if (st) c.st = *st;
    if (m) {
        c.mc = make_matconst(*m);
        c.E0 = m->youngs_modulus;
        c.nu = m->poisson_ratio;
    }
    return c;
}

static inline int64_t align256(int64_t b) { return (b + 255) & ~(int64_t)255; }

// -------------------------------------------------------------- exclusive scan
static inline int64_t scan_ws_ints(int64_t n) {
    int64_t total = 0;
    while (n > 1024) {
        const int64_t nb = (n + 1023) / 1024;
        total += 2 * nb + 64;
        n = nb;
    }
    return total + 64;
}

static inline int scan_exclusive(const int *in, int *out, int n, int *ws, cudaStream_t s) {
    if (n <= 0) return GW_OK;
    const int nb = (n + 1023) / 1024;
    int *sums = ws;
    int *sums_scan = ws + nb;
    k_scan_block<<<gw_count_launch(nb), 1024, 0, s>>>(in, out, n, nb > 1 ? sums : nullptr);
    GW_LAUNCHED();
    if (nb > 1) {
        int rc = scan_exclusive(sums, sums_scan, nb, ws + 2 * nb + 64, s);
        if (rc) return rc;
        k_scan_add<<<gw_count_launch(nb), 1024, 0, s>>>(out, n, sums_scan);
        GW_LAUNCHED();
    }
    return GW_OK;
}


static inline int n_cells_of(const gw_grid_t &g) {
    int c = 1;
    for (int k = 0; k < g.dim; ++k) c *= g.n_grid[k];
    return c;
}

inline const char *kGuardNames[GS_COUNT] = {"none", "row_mv column", "coarse flags", "coarse stencil", "pattern fill",
                                     "Galerkin product (coarse block)", "Galerkin product (fine block)",
                                     "smoother setup", "restriction", "prolongation", "dense coarsest level",
                                     "Krylov column counter", "transpose", "assembly scatter", "adjoint scatter",
                                     "block-row map", "fixed-DOF mask", "pre-smoothing"};

// Reads (and clears) the first failed index guard; the stream must be idle or
// the read is ordered after the kernels to check.  Returns GW_ERANGE with the
// site in the message when a guard failed.
static inline int guard_check(cudaStream_t s, const char *where) {
    int site = 0;
    long long value = 0;
    GW_CUDA(cudaMemcpyFromSymbolAsync(&site, g_guard_site, sizeof(int), 0, cudaMemcpyDeviceToHost, s));
    GW_CUDA(cudaMemcpyFromSymbolAsync(&value, g_guard_value, sizeof(long long), 0, cudaMemcpyDeviceToHost, s));
    GW_CUDA(cudaStreamSynchronize(s));
    if (site == 0) return GW_OK;
    const int zero = 0;
    const long long zero_v = 0;
    GW_CUDA(cudaMemcpyToSymbolAsync(g_guard_site, &zero, sizeof(int), 0, cudaMemcpyHostToDevice, s));
    GW_CUDA(cudaMemcpyToSymbolAsync(g_guard_value, &zero_v, sizeof(long long), 0, cudaMemcpyHostToDevice, s));
    GW_CUDA(cudaStreamSynchronize(s));
    snprintf(g_msg, sizeof(g_msg), "%s: index guard failed in %s (value %lld)", where,
             (site > 0 && site < GS_COUNT) ? kGuardNames[site] : "unknown site", value);
    return GW_ERANGE;
}


}  // namespace gwh
