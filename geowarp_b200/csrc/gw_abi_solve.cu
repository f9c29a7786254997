// C ABI, Krylov solvers: BiCGSTAB / CG, restarted GMRES, multigrid-
// preconditioned flexible GMRES, the workspace-free Krylov entry point and
// SpMV (declarations and reference citations in include/geowarp_b200.h).
#include <algorithm>
#include <type_traits>
#include <vector>

#include "gw_host.cuh"
#include "gw_mg.cuh"
#include "gw_mg_tail.cuh"

using namespace gw;
using namespace gwh;

namespace {
struct KWs {
    double *r, *rh, *p, *v, *y, *s, *z, *t, *Minv, *partials;
    KScalars *sc;
};

int64_t krylov_ws_bytes(int64_t n_rows, int nf) {
    const int64_t n = n_rows * nf;
    return 8 * align256(8 * n) + align256(8 * n_rows * nf * nf) + align256(8 * (int64_t)kRedBlocks * 4) +
           align256(sizeof(KScalars));
}

KWs carve(void *ws, int64_t n_rows, int nf) {
    const int64_t n = n_rows * nf;
    char *w = (char *)ws;
    KWs k;
    double **vecs[8] = {&k.r, &k.rh, &k.p, &k.v, &k.y, &k.s, &k.z, &k.t};
    for (int i = 0; i < 8; ++i) { *vecs[i] = (double *)w; w += align256(8 * n); }
    k.Minv = (double *)w; w += align256(8 * n_rows * nf * nf);
    k.partials = (double *)w; w += align256(8 * (int64_t)kRedBlocks * 4);
    k.sc = (KScalars *)w;
    return k;
}

template <int NF, typename VT>
int krylov(const gw_bsr_t *A, int method, int precond, const double *b, double *x, double rtol, int max_iter, void *ws,
           int *iters, double *relres, cudaStream_t s) {
    PtrsA a = make_ptrs(*A);
    KWs k = carve(ws, A->n_rows, NF);
    const int D = (A->mask_words == 1) ? 2 : 3;
    const int nr = A->n_rows;
    if (nr == 0) { *iters = 0; *relres = 0.0; return GW_OK; }
    BicgVecs V;
    V.x = x; V.b = b; V.r = k.r; V.rh = k.rh; V.p = k.p; V.v = k.v; V.y = k.y; V.s = k.s; V.z = k.z; V.t = k.t;
    V.Minv = k.Minv; V.partials = k.partials; V.sc = k.sc;
    GW_CUDA(cudaMemsetAsync(k.sc, 0, sizeof(KScalars), s));
    KScalars h;
    memset(&h, 0, sizeof(h));
    h.max_iter = max_iter;
    GW_CUDA(cudaMemcpyAsync(&k.sc->max_iter, &h.max_iter, sizeof(int), cudaMemcpyHostToDevice, s));
    k_precond_setup<NF, VT><<<gw_count_launch(nblk(nr, kThreads)), kThreads, 0, s>>>(a, D, precond, k.Minv);
    GW_LAUNCHED();
    const int gw_rows = red_grid_rows(nr), ge_rows = red_grid_elems(nr);
    if (method == GW_KRYLOV_CG) k_cg_init<NF, VT><<<gw_count_launch(gw_rows), kThreads, 0, s>>>(a, V, rtol);
    else k_bicg_init<NF, VT><<<gw_count_launch(gw_rows), kThreads, 0, s>>>(a, V, rtol);
    GW_LAUNCHED();
    int chunk = 2;
    for (;;) {
        GW_CUDA(cudaMemcpyAsync(&h, k.sc, sizeof(KScalars), cudaMemcpyDeviceToHost, s));
        GW_CUDA(cudaStreamSynchronize(s));
        if (h.done) break;
        for (int it = 0; it < chunk; ++it) {
            if (method == GW_KRYLOV_CG) {
                k_cg_p<NF><<<gw_count_launch(red_grid_elems((int64_t)nr * NF)), kThreads, 0, s>>>(nr, V);
                k_cg_q<NF, VT><<<gw_count_launch(gw_rows), kThreads, 0, s>>>(a, V);
                k_cg_xr<NF><<<gw_count_launch(ge_rows), kThreads, 0, s>>>(nr, V);
            } else {
                k_bicg_p<NF><<<gw_count_launch(ge_rows), kThreads, 0, s>>>(nr, V);
                k_bicg_v<NF, VT><<<gw_count_launch(gw_rows), kThreads, 0, s>>>(a, V);
                k_bicg_s<NF><<<gw_count_launch(ge_rows), kThreads, 0, s>>>(nr, V);
                k_bicg_t<NF, VT><<<gw_count_launch(gw_rows), kThreads, 0, s>>>(a, V);
                k_bicg_xr<NF><<<gw_count_launch(ge_rows), kThreads, 0, s>>>(nr, V);
            }
        }
        GW_LAUNCHED();
        chunk = chunk < 64 ? chunk * 2 : 64;
    }
    *iters = h.iters;
    *relres = (h.bb > 0.0) ? ::sqrt(h.rr / h.bb) : 0.0;
    const int gc = guard_check(s, "Krylov");
    if (gc) return gc;
    if (h.status == ST_BREAKDOWN) return GW_EBREAKDOWN;
    if (h.status == ST_NAN) return GW_ENAN;
    if (h.rr > h.tol2) return GW_ENOCONV;
    return GW_OK;
}

template <typename VT>
int krylov_nf(const gw_bsr_t *A, int method, int precond, const double *b, double *x, double rtol, int max_iter,
              void *ws, int *iters, double *relres, cudaStream_t s) {
    switch (A->nf) {
        case 1: return krylov<1, VT>(A, method, precond, b, x, rtol, max_iter, ws, iters, relres, s);
        case 2: return krylov<2, VT>(A, method, precond, b, x, rtol, max_iter, ws, iters, relres, s);
        case 3: return krylov<3, VT>(A, method, precond, b, x, rtol, max_iter, ws, iters, relres, s);
        case 4: return krylov<4, VT>(A, method, precond, b, x, rtol, max_iter, ws, iters, relres, s);
        default: return GW_EINVAL;
    }
}
}  // namespace

namespace {
// second Gram-Schmidt passes of the last GMRES solve on this host thread
thread_local int g_last_reorths = 0;
// whether the last GMRES solve on this host thread stopped on stagnation
thread_local int g_last_stalled = 0;

// Restarted GMRES can stagnate for good: the true residual at each cycle start
// stops falling (a preconditioned operator whose field of values contains
// zero, or a preconditioner too weak for the accuracy asked).  A solve whose
// residual fell by less than 10% over the last GW_TUNE_GMRES_STALL restart
// cycles stops there, and returns GW_ENOCONV, instead of running on to
// max_iter: at that rate 650 more cycles would gain less than a factor 4.
// 0 turns the check off.
class StallWatch {
  public:
    StallWatch() : window_(g_tune[GW_TUNE_GMRES_STALL]) {}
    // beta: the true residual norm at the start of a restart cycle
    bool stalled(double beta) {
        if (window_ <= 0) return false;
        hist_.push_back(beta);
        const size_t n = hist_.size();
        return n > (size_t)window_ && beta > 0.9 * hist_[n - 1 - window_];
    }

  private:
    int window_;
    std::vector<double> hist_;
};

// Profiling only: whether column k takes the second Gram-Schmidt pass (read
// after pass 0), so that the timed pass-1 launches are credited with the bytes
// they move.  Timed runs without profiling never read it.
int prof_reorth(GScalars *sc, cudaStream_t s) {
    if (!g_prof_on) return 1;
    int re = 1;
    if (cudaMemcpyAsync(&re, &sc->reorth, sizeof(int), cudaMemcpyDeviceToHost, s) != cudaSuccess) return 1;
    if (cudaStreamSynchronize(s) != cudaSuccess) return 1;
    return re;
}

int64_t gmres_ws_bytes(int64_t n_rows, int nf, int restart) {
    const int64_t n = n_rows * nf;
    return align256(8 * n * (restart + 1)) + 2 * align256(8 * n) + align256(8 * n_rows * nf * nf) +
           align256(8 * (int64_t)kRedBlocks * (kGmresMaxRestart + 1)) + align256(sizeof(GScalars));
}

template <int NF, typename VT>
int gmres(const gw_bsr_t *A, int precond, const double *b, double *x, double rtol, int max_iter, int restart,
          void *ws, int *iters, double *relres, cudaStream_t s) {
    PtrsA a = make_ptrs(*A);
    const int nr = A->n_rows;
    if (nr == 0) { *iters = 0; *relres = 0.0; return GW_OK; }
    const int64_t n = (int64_t)nr * NF;
    char *w = (char *)ws;
    GmresVecs G;
    G.V = (double *)w; w += align256(8 * n * (restart + 1));
    G.w = (double *)w; w += align256(8 * n);
    G.z = (double *)w; w += align256(8 * n);
    G.Minv = (double *)w; w += align256(8 * (int64_t)nr * NF * NF);
    G.partials = (double *)w; w += align256(8 * (int64_t)kRedBlocks * (kGmresMaxRestart + 1));
    G.sc = (GScalars *)w;
    G.x = x; G.b = b; G.n = (size_t)n;
    const size_t head = offsetof(GScalars, H);
    GW_CUDA(cudaMemsetAsync(G.sc, 0, head, s));
    struct { int max_iter, restart; } lim = {max_iter, restart};
    GW_CUDA(cudaMemcpyAsync(&G.sc->max_iter, &lim, sizeof(lim), cudaMemcpyHostToDevice, s));
    const double eta2 = ::pow(10.0, -0.1 * g_tune[GW_TUNE_GS_CANCEL]);
    GW_CUDA(cudaMemcpyAsync(&G.sc->gs_eta2, &eta2, sizeof(double), cudaMemcpyHostToDevice, s));
    const int D = (A->mask_words == 1) ? 2 : 3;
    k_precond_setup<NF, VT><<<gw_count_launch(nblk(nr, kThreads)), kThreads, 0, s>>>(a, D, precond, G.Minv);
    GW_LAUNCHED();
    const int gr = red_grid_rows(nr), ge = red_grid_elems(nr), gv = red_grid_elems(n);
    GScalars h;
    memset(&h, 0, head);
    int first = 1;
    StallWatch stall;
    g_last_stalled = 0;
    for (int cycle = 0; cycle < 1000000; ++cycle) {
        k_gm_residual<NF, VT><<<gw_count_launch(gr), kThreads, 0, s>>>(a, G, first, rtol);
        k_gm_next<NF><<<gw_count_launch(ge), kThreads, 0, s>>>(nr, G, 1);
        GW_LAUNCHED();
        first = 0;
        GW_CUDA(cudaMemcpyAsync(&h, G.sc, head, cudaMemcpyDeviceToHost, s));
        GW_CUDA(cudaStreamSynchronize(s));
        if (h.done) break;
        if (stall.stalled(h.beta)) { g_last_stalled = 1; break; }
        int chunk = 4;
        int kk = 0;  // host-side column estimate (exact until the cycle closes early)
        const double spmv_bytes = (double)A->nnzb * (NF * NF * sizeof(VT) + 4) + 4.0 * (nr + 1) + 16.0 * n;
        for (;;) {
            for (int it = 0; it < chunk; ++it, ++kk) {
                const double vb = 8.0 * n * (kk + 2);
                { ProfScope ps(PC_SPMV, s, spmv_bytes); k_gm_spmv<NF, VT><<<gw_count_launch(gr), kThreads, 0, s>>>(a, G); }
                { ProfScope ps(PC_DOTS, s, vb + 8.0 * n); k_gm_dots<<<gw_count_launch(gv), kThreads, 0, s>>>(G, 0); }
                { ProfScope ps(PC_UPDATE, s, vb + 8.0 * n); k_gm_update<<<gw_count_launch(gv), kThreads, 0, s>>>(G, 0); }
                const int re = prof_reorth(G.sc, s);
                { ProfScope ps(PC_DOTS, s, re ? vb : 0.0); k_gm_dots<<<gw_count_launch(gv), kThreads, 0, s>>>(G, 1); }
                { ProfScope ps(PC_UPDATE, s, re ? vb + 8.0 * n : 0.0); k_gm_update<<<gw_count_launch(gv), kThreads, 0, s>>>(G, 1); }
                { ProfScope ps(PC_NEXT, s, 8.0 * n * 3 + 8.0 * nr * NF * NF); k_gm_next<NF><<<gw_count_launch(ge), kThreads, 0, s>>>(nr, G, 0); }
            }
            GW_LAUNCHED();
            GW_CUDA(cudaMemcpyAsync(&h, G.sc, head, cudaMemcpyDeviceToHost, s));
            GW_CUDA(cudaStreamSynchronize(s));
            if (h.cycle_done) break;
            chunk = chunk < 32 ? chunk * 2 : 32;
        }
        if (h.status) break;
        k_gm_solve_y<<<gw_count_launch(1), 32, 0, s>>>(G.sc);
        k_gm_update_x<NF><<<gw_count_launch(ge), kThreads, 0, s>>>(nr, G);
        GW_LAUNCHED();
    }
    *iters = h.iters;
    g_last_reorths = h.reorths;
    *relres = (h.bnorm > 0.0) ? h.resid / h.bnorm : 0.0;
    const int gc = guard_check(s, "GMRES");
    if (gc) return gc;
    if (h.status == ST_NAN) return GW_ENAN;
    if (h.resid > h.tol) return GW_ENOCONV;
    return GW_OK;
}

template <typename VT>
int gmres_nf(const gw_bsr_t *A, int precond, const double *b, double *x, double rtol, int max_iter, int restart,
             void *ws, int *iters, double *relres, cudaStream_t s) {
    switch (A->nf) {
        case 1: return gmres<1, VT>(A, precond, b, x, rtol, max_iter, restart, ws, iters, relres, s);
        case 2: return gmres<2, VT>(A, precond, b, x, rtol, max_iter, restart, ws, iters, relres, s);
        case 3: return gmres<3, VT>(A, precond, b, x, rtol, max_iter, restart, ws, iters, relres, s);
        case 4: return gmres<4, VT>(A, precond, b, x, rtol, max_iter, restart, ws, iters, relres, s);
        default: return GW_EINVAL;
    }
}
}  // namespace

extern "C" int64_t gw_gmres_workspace_bytes(int32_t n_rows, int32_t nf, int32_t restart) {
    if (restart < 1 || restart > kGmresMaxRestart) return -1;
    return gmres_ws_bytes(n_rows, nf, restart);
}

extern "C" int gw_bsr_gmres_solve(const gw_bsr_t *A, int32_t prec, int32_t precond, const double *b, double *x,
                                  double rtol, int32_t max_iter, int32_t restart, void *workspace, int32_t *iters_host,
                                  double *relres_host, void *stream) {
    GW_REQUIRE(A && b && x && workspace && iters_host && relres_host && max_iter > 0);
    GW_REQUIRE(vec_ok(A, b, x));
    GW_REQUIRE(restart >= 1 && restart <= kGmresMaxRestart);
    int it = 0;
    double rr = 0.0;
    int rc = (prec == GW_PREC_F64)
                 ? gmres_nf<double>(A, precond, b, x, rtol, max_iter, restart, workspace, &it, &rr, S(stream))
                 : gmres_nf<float>(A, precond, b, x, rtol, max_iter, restart, workspace, &it, &rr, S(stream));
    *iters_host = it;
    *relres_host = rr;
    return rc;
}

// ==================================================================== multigrid-preconditioned flexible GMRES
namespace {
// damping of the block-Jacobi smoother (GW_TUNE_MG_OMEGA, in percent)
inline double mg_omega() { return 0.01 * g_tune[GW_TUNE_MG_OMEGA]; }
// smoothing sweeps before / after the coarse correction: two, or one from
// level GW_TUNE_MG_ONE_SWEEP down (fewer launches on the latency-bound coarse
// levels against more Krylov iterations; the autotuner weighs the two)
inline int mg_sweeps(int l) {
    if (l == 0) return g_tune[GW_TUNE_MG_FINE_SWEEPS];
    return l >= g_tune[GW_TUNE_MG_ONE_SWEEP] ? 1 : g_tune[GW_TUNE_MG_SWEEPS];
}

// Bump allocator over the caller's workspace; with p == nullptr it only counts,
// so sizing and carving run the same code.
struct Bump {
    char *p;
    int64_t used;
    void *take(int64_t b) {
        b = align256(b);
        void *r = p ? (void *)(p + used) : nullptr;
        used += b;
        return r;
    }
};

struct MgLevel {
    gw_grid_t g;
    Lat L;
    gw_bsr_t A;             // level 0: the caller's matrix; coarse levels: FP64 in the workspace
    double *Minv, *b, *x, *x2, *r;
    uint8_t *fixed;
    int *tmp, *sws, *blockrow;
    int *child;             // coarse levels: fine rows of the 3^D children of each row (pattern phase)
    int *parent;            // levels with a coarser one: coarse rows of the 2^D parents of each row
    void *pvals;            // level 0: BF16 copy of the fine Jacobian read by the V-cycle (mixed)
    uint8_t *flags;
};
struct MgHier {
    int nl = 0;             // levels holding a matrix; the last one is solved with a dense inverse
    MgLevel lv[kMgMaxLevels];
    double *dM = nullptr, *dInv = nullptr;
    int dn = 0;
};

gw_grid_t coarse_grid(const gw_grid_t &g) {
    gw_grid_t c = g;
    int nn = 1;
    for (int k = 0; k < 3; ++k) {
        if (k < g.dim) {
            c.n_grid[k] = (g.n_grid[k] + 1) / 2;  // fine nodes N -> coarse nodes N/2 + 1
            nn *= c.n_grid[k] + 1;
        } else {
            c.n_grid[k] = 0;
        }
        c.h[k] = 2.0 * g.h[k];
        c.inv_h[k] = 0.5 * g.inv_h[k];
        c.h_nodes[k] = 2.0 * g.h_nodes[k];
    }
    c.n_nodes = nn;
    return c;
}

// Carves (or, with a counting Bump, sizes) every level of the hierarchy at its
// upper bound -- a coarse level holds at most its lattice's node count of rows
// and 5^D blocks per row -- and then the flexible-GMRES vectors.  The hierarchy
// comes first, so its addresses depend only on (grid, n_rows, nf): a plan built
// in a workspace stays valid for any restart length.
struct FlexVecs {
    double *V, *Z, *w, *partials;
    GScalars *sc;
};
void mg_carve_hier(Bump &bp, MgHier &h, const gw_grid_t &g0, int64_t n_rows0, int nf) {
    const int64_t n0 = n_rows0 * nf;
    const int D = g0.dim, mw = D == 2 ? 1 : 4, S = D == 2 ? 25 : 125;
    MgLevel &l0 = h.lv[0];
    l0.g = g0;
    l0.Minv = (double *)bp.take(8 * n_rows0 * nf * nf);
    l0.b = (double *)bp.take(8 * n0);
    l0.x = (double *)bp.take(8 * n0);
    l0.x2 = (double *)bp.take(8 * n0);
    l0.r = (double *)bp.take(8 * n0);
    l0.fixed = (uint8_t *)bp.take(n_rows0);
    const int CN = D == 2 ? 9 : 27, PN = D == 2 ? 4 : 8;
    l0.parent = (int *)bp.take(4 * n_rows0 * PN);
    l0.pvals = bp.take(2 * n_rows0 * S * nf * nf);
    gw_grid_t g = g0;
    int64_t nodes = g0.n_nodes;
    int l = 0;
    // levels carved for the smallest coarsest-level bound a caller may set
    for (; l + 1 < kMgMaxLevels && nodes * nf > kMgCoarseMin; ++l) {
        g = coarse_grid(g);
        nodes = g.n_nodes;
        MgLevel &c = h.lv[l + 1];
        c.g = g;
        c.A.node2row = (int *)bp.take(4 * nodes);
        c.A.row2node = (int *)bp.take(4 * nodes);
        c.A.row_ptr = (int *)bp.take(4 * (nodes + 1));
        c.A.stencil = (uint32_t *)bp.take(4 * nodes * mw);
        c.A.cols = (int *)bp.take(4 * nodes * S);
        c.A.vals = bp.take(8 * nodes * S * nf * nf);
        c.blockrow = (int *)bp.take(4 * nodes * S);
        c.tmp = (int *)bp.take(4 * (nodes + 1));
        c.sws = (int *)bp.take(4 * (scan_ws_ints(nodes + 1) + 64));
        c.flags = (uint8_t *)bp.take(nodes);
        c.Minv = (double *)bp.take(8 * nodes * nf * nf);
        c.b = (double *)bp.take(8 * nodes * nf);
        c.x = (double *)bp.take(8 * nodes * nf);
        c.x2 = (double *)bp.take(8 * nodes * nf);
        c.r = (double *)bp.take(8 * nodes * nf);
        c.fixed = (uint8_t *)bp.take(nodes);
        c.child = (int *)bp.take(4 * nodes * CN);
        c.parent = (int *)bp.take(4 * nodes * PN);
    }
    h.nl = l + 1;  // upper bound; the plan may stop earlier
    h.dM = (double *)bp.take(8 * (int64_t)kMgCoarseMax * kMgCoarseMax);
    h.dInv = (double *)bp.take(8 * (int64_t)kMgCoarseMax * kMgCoarseMax);
}
void mg_carve_flex(Bump &bp, FlexVecs &fv, int64_t n0, int restart) {
    fv.V = (double *)bp.take(8 * n0 * (restart + 1));
    fv.Z = (double *)bp.take(8 * n0 * restart);
    fv.w = (double *)bp.take(8 * n0);
    fv.partials = (double *)bp.take(8 * (int64_t)kRedBlocks * (kGmresMaxRestart + 1));
    fv.sc = (GScalars *)bp.take(sizeof(GScalars));
}

int64_t mg_ws_bytes(const gw_grid_t &g0, int64_t n_rows, int nf, int restart) {
    Bump bp{nullptr, 0};
    MgHier h;
    FlexVecs fv;
    mg_carve_hier(bp, h, g0, n_rows, nf);
    mg_carve_flex(bp, fv, n_rows * nf, restart);
    return bp.used;
}

// Pattern phase: the coarse active sets, row maps, stencils, row pointers and
// columns of every level below A0 (two host reads per coarse level: its row
// count and its block count).  Depends on A0's pattern only.
template <int NF>
int mg_pattern(MgHier &h, const gw_bsr_t *A0, gw_mg_plan_t *plan, cudaStream_t s) {
    const int D = h.lv[0].g.dim, mw = D == 2 ? 1 : 4;
    const int nl_bound = h.nl;
    h.lv[0].L = lat_of(h.lv[0].g);
    h.lv[0].A = *A0;
    int l = 0;
    while (h.lv[l].A.n_rows * NF > g_tune[GW_TUNE_MG_COARSE]) {
        if (l + 1 >= nl_bound) {
            snprintf(g_msg, sizeof(g_msg), "multigrid: coarsest level still has %d unknowns", h.lv[l].A.n_rows * NF);
            return GW_EINVAL;
        }
        MgLevel &f = h.lv[l], &c = h.lv[l + 1];
        c.L = lat_of(c.g);
        const int N = c.g.n_nodes;
        PtrsA fa = make_ptrs(f.A);
        GW_CUDA(cudaMemsetAsync(c.flags, 0, N, s));
        k_mg_coarse_flags<<<gw_count_launch(nblk(f.A.n_rows, kThreads)), kThreads, 0, s>>>(f.L, fa, c.L, c.flags);
        k_flags_to_int<<<gw_count_launch(nblk(N, kThreads)), kThreads, 0, s>>>(c.flags, N, c.tmp);
        GW_LAUNCHED();
        GW_CUDA(cudaMemcpyAsync(c.sws, c.tmp + (N - 1), 4, cudaMemcpyDeviceToDevice, s));
        int rc = scan_exclusive(c.tmp, c.tmp, N, c.sws + 64, s);
        if (rc) return rc;
        k_compact<<<gw_count_launch(nblk(N, kThreads)), kThreads, 0, s>>>(c.flags, c.tmp, N, NF, nullptr,
                                                                          (int *)c.A.node2row, (int *)c.A.row2node, nullptr);
        k_add2<<<gw_count_launch(1), 32, 0, s>>>(c.tmp + (N - 1), c.sws, c.sws + 1);
        GW_LAUNCHED();
        int nrc = 0;
        GW_CUDA(cudaMemcpyAsync(&nrc, c.sws + 1, 4, cudaMemcpyDeviceToHost, s));
        GW_CUDA(cudaStreamSynchronize(s));
        if (nrc <= 0) {
            snprintf(g_msg, sizeof(g_msg), "multigrid: empty coarse level");
            return GW_EINVAL;
        }
        GW_CUDA(cudaMemsetAsync((void *)c.A.stencil, 0, 4 * (size_t)N * mw, s));
        GW_CUDA(cudaMemsetAsync(c.tmp, 0, 4 * ((size_t)nrc + 1), s));
        if (D == 2)
            k_mg_coarse_stencil<2><<<gw_count_launch(nblk(nrc, kThreads)), kThreads, 0, s>>>(
                f.L, fa, c.L, nrc, c.A.row2node, (uint32_t *)c.A.stencil, mw, c.tmp);
        else
            k_mg_coarse_stencil<3><<<gw_count_launch(nblk(nrc, kThreads)), kThreads, 0, s>>>(
                f.L, fa, c.L, nrc, c.A.row2node, (uint32_t *)c.A.stencil, mw, c.tmp);
        GW_LAUNCHED();
        rc = scan_exclusive(c.tmp, (int *)c.A.row_ptr, nrc + 1, c.sws, s);
        if (rc) return rc;
        int nnzb = 0;
        GW_CUDA(cudaMemcpyAsync(&nnzb, c.A.row_ptr + nrc, 4, cudaMemcpyDeviceToHost, s));
        GW_CUDA(cudaStreamSynchronize(s));
        c.A.n_rows = nrc;
        c.A.nf = NF;
        c.A.nnzb = nnzb;
        c.A.mask_words = mw;
        PtrsA ca = make_ptrs(c.A);
        if (D == 2) k_pattern_fill<2><<<gw_count_launch(nblk(nrc, kThreads)), kThreads, 0, s>>>(c.g, ca, (int *)c.A.cols);
        else k_pattern_fill<3><<<gw_count_launch(nblk(nrc, kThreads)), kThreads, 0, s>>>(c.g, ca, (int *)c.A.cols);
        k_mg_blockrow<<<gw_count_launch(nblk(nrc, kThreads)), kThreads, 0, s>>>(c.A.row_ptr, nrc, nnzb, c.blockrow);
        if (D == 2) {
            k_mg_children<2><<<gw_count_launch(nblk(nrc, kThreads)), kThreads, 0, s>>>(f.L, fa, c.L, ca, c.child);
            k_mg_parents<2><<<gw_count_launch(nblk(f.A.n_rows, kThreads)), kThreads, 0, s>>>(f.L, fa, c.L, ca, f.parent);
        } else {
            k_mg_children<3><<<gw_count_launch(nblk(nrc, kThreads)), kThreads, 0, s>>>(f.L, fa, c.L, ca, c.child);
            k_mg_parents<3><<<gw_count_launch(nblk(f.A.n_rows, kThreads)), kThreads, 0, s>>>(f.L, fa, c.L, ca, f.parent);
        }
        GW_LAUNCHED();
        ++l;
    }
    h.nl = l + 1;
    h.dn = h.lv[l].A.n_rows * NF;
    memset(plan, 0, sizeof(*plan));
    plan->levels = h.nl;
    plan->dense_n = h.dn;
    for (int q = 0; q < h.nl; ++q) {
        plan->n_rows[q] = h.lv[q].A.n_rows;
        plan->nnzb[q] = h.lv[q].A.nnzb;
    }
    plan->nf = NF;
    plan->fine_n_rows = A0->n_rows;
    plan->fine_nnzb = A0->nnzb;
    plan->row_ptr = A0->row_ptr;
    plan->cols = A0->cols;
    return GW_OK;
}

// Restores the level sizes a plan recorded into a freshly carved hierarchy.
void mg_apply_plan(MgHier &h, const gw_bsr_t *A0, const gw_mg_plan_t *plan, int nf) {
    const int mw = h.lv[0].g.dim == 2 ? 1 : 4;
    h.nl = plan->levels;
    h.dn = plan->dense_n;
    h.lv[0].L = lat_of(h.lv[0].g);
    h.lv[0].A = *A0;
    for (int q = 1; q < h.nl; ++q) {
        MgLevel &c = h.lv[q];
        c.L = lat_of(c.g);
        c.A.n_rows = plan->n_rows[q];
        c.A.nnzb = plan->nnzb[q];
        c.A.nf = nf;
        c.A.mask_words = mw;
    }
}

// Numeric phase: smoother blocks and fixed-DOF masks of every level, Galerkin
// values of the coarse levels, dense inverse of the coarsest.  No host reads.
template <typename VT>
inline bool mg_bf16_fine() { return std::is_same<VT, float>::value && g_tune[GW_TUNE_MG_BF16] != 0; }

template <int NF, typename VT>
int mg_numeric(MgHier &h, cudaStream_t s) {
    const int D = h.lv[0].g.dim;
    {
        const MgLevel &l0 = h.lv[0];
        PtrsA a0 = make_ptrs(l0.A);
        k_mg_smoother_setup<NF, VT><<<gw_count_launch(nblk(l0.A.n_rows, kThreads)), kThreads, 0, s>>>(a0, D, l0.Minv);
        k_mg_fixed_mask<NF, VT><<<gw_count_launch(nblk(l0.A.n_rows, kThreads)), kThreads, 0, s>>>(a0, l0.fixed);
        GW_LAUNCHED();
    }
    for (int l = 0; l + 1 < h.nl; ++l) {
        MgLevel &f = h.lv[l], &c = h.lv[l + 1];
        PtrsA fa = make_ptrs(f.A), ca = make_ptrs(c.A);
        const int nb = c.A.nnzb;
        if (D == 2) k_mg_rap<2, NF, VT><<<gw_count_launch(nblk(nb, kThreads)), kThreads, 0, s>>>(f.L, fa, f.fixed, c.L, ca, c.blockrow);
        else k_mg_rap<3, NF, VT><<<gw_count_launch(nblk(nb, kThreads)), kThreads, 0, s>>>(f.L, fa, f.fixed, c.L, ca, c.blockrow);
        GW_LAUNCHED();
        const int nrc = c.A.n_rows;
        k_mg_fix_empty_rows<NF, VT><<<gw_count_launch(nblk(nrc, kThreads)), kThreads, 0, s>>>(ca);
        k_mg_smoother_setup<NF, VT><<<gw_count_launch(nblk(nrc, kThreads)), kThreads, 0, s>>>(ca, D, c.Minv);
        k_mg_fixed_mask<NF, VT><<<gw_count_launch(nblk(nrc, kThreads)), kThreads, 0, s>>>(ca, c.fixed);
        GW_LAUNCHED();
    }
    const int l = h.nl - 1;
    const MgLevel &lc = h.lv[l];
    const int n = h.dn;
    GW_CUDA(cudaMemsetAsync(h.dM, 0, 8 * (size_t)n * n, s));
    PtrsA ac = make_ptrs(lc.A);
    k_mg_dense_build<NF, VT><<<gw_count_launch(nblk(lc.A.n_rows, kThreads)), kThreads, 0, s>>>(ac, h.dM, n);
    const size_t smem = 8 * (size_t)n * n;
    GW_CUDA(cudaFuncSetAttribute(k_mg_dense_invert, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 8 * kMgCoarseMax * kMgCoarseMax));
    k_mg_dense_invert<<<gw_count_launch(1), 1024, smem, s>>>(h.dM, h.dInv, n);
    GW_LAUNCHED();
    return GW_OK;
}

template <int NF, typename VT>
void mg_jacobi(const MgHier &h, int l, const double *b, const double *xin, double *xout, int zero, const int *skip,
               cudaStream_t s) {
    const MgLevel &v = h.lv[l];
    PtrsA a = make_ptrs(v.A);
    const int tb = zero ? kThreads : tune_rows_block();
    const bool bf = l == 0 && mg_bf16_fine<VT>();
    if (bf) a.vals = v.pvals;
    const int g = zero ? red_grid_elems(v.A.n_rows)
                       : (bf ? resident_rows_grid((const void *)k_mg_jacobi<NF, __nv_bfloat16>, tb, v.A.n_rows)
                             : resident_rows_grid((const void *)k_mg_jacobi<NF, VT>, tb, v.A.n_rows));
    // algorithmic bytes: b, x_out, Minv; with a previous iterate also x_in and the matrix
    const double vs = 8.0 * v.A.n_rows * NF, mat = (double)v.A.nnzb * (NF * NF * (bf ? 2 : sizeof(VT)) + 4);
    ProfScope ps(l == 0 ? PC_MG_JACOBI : PC_MG_JACOBI_COARSE, s,
                 2 * vs + 8.0 * v.A.n_rows * NF * NF + (zero ? 0.0 : vs + mat));
    if (bf) k_mg_jacobi<NF, __nv_bfloat16><<<gw_count_launch(g), tb, 0, s>>>(a, v.Minv, b, xin, xout, mg_omega(), zero, skip);
    else k_mg_jacobi<NF, VT><<<gw_count_launch(g), tb, 0, s>>>(a, v.Minv, b, xin, xout, mg_omega(), zero, skip);
}

// Largest cluster of the fused coarse tail for this instantiation on the
// current device: 16 CTAs where the device can run such a cluster of it, else
// 8, 0 when neither fits (then every level keeps its own launches).  Queried once
// per device, before any stream capture (gmres_mg calls it first).
template <int D, int NF>
int tail_cluster_size() {
    static int cached[64] = {0};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 0;
    if (cached[dev]) return cached[dev] > 0 ? cached[dev] : 0;
    int size = -1;
    for (int cand : {16, 8}) {
        if (cand > 8 && cudaFuncSetAttribute(k_mg_tail<D, NF>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) !=
                            cudaSuccess)
            continue;
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(cand);
        cfg.blockDim = dim3(kTailThreads);
        cudaLaunchAttribute at;
        at.id = cudaLaunchAttributeClusterDimension;
        at.val.clusterDim.x = cand;
        at.val.clusterDim.y = 1;
        at.val.clusterDim.z = 1;
        cfg.attrs = &at;
        cfg.numAttrs = 1;
        int n = 0;
        if (cudaOccupancyMaxActiveClusters(&n, (void *)k_mg_tail<D, NF>, &cfg) == cudaSuccess && n >= 1) {
            size = cand;
            break;
        }
    }
    (void)cudaGetLastError();  // a refused query leaves no error behind
    cached[dev] = size;
    return size > 0 ? size : 0;
}

template <int NF>
int tail_cluster_size(int D) { return D == 2 ? tail_cluster_size<2, NF>() : tail_cluster_size<3, NF>(); }

// First level of the fused coarse tail (the first coarse level with at most
// GW_TUNE_MG_TAIL rows), or h.nl - 1 when the tail is off or has no level to
// smooth.
template <int NF, typename VT>
int tail_level(const MgHier &h) {
    const int last = h.nl - 1, T = g_tune[GW_TUNE_MG_TAIL];
    // the fused tail reads FP64 coarse operators: FP64 solves only
    if (!std::is_same<VT, double>::value) return last;
    if (T <= 0 || last < 2 || tail_cluster_size<NF>(h.lv[0].g.dim) == 0) return last;
    for (int l = 1; l < last; ++l)
        if (h.lv[l].A.n_rows <= T) return l;
    return last;
}

// Launches levels l0 .. last of the V-cycle as one cluster and returns the
// buffer that holds level l0's result (the same one the per-phase path ends in).
template <int NF>
double *mg_tail(const MgHier &h, int l0, const int *skip, cudaStream_t s) {
    const int last = h.nl - 1, D = h.lv[0].g.dim;
    TailArgs ta;
    memset(&ta, 0, sizeof(ta));
    ta.l0 = l0;
    ta.last = last;
    ta.dInv = h.dInv;
    ta.dn = h.dn;
    ta.omega = mg_omega();
    ta.skip = skip;
    double bytes = 8.0 * h.dn * h.dn;
    for (int l = l0; l <= last; ++l) {
        const MgLevel &v = h.lv[l];
        TailLevel &t = ta.lv[l];
        t.A = make_ptrs(v.A);
        t.L = v.L;
        t.Minv = v.Minv;
        t.b = v.b; t.x = v.x; t.x2 = v.x2; t.r = v.r;
        t.fixed = v.fixed;
        t.sweeps = mg_sweeps(l);
        if (l < last) {
            const double vs = 8.0 * v.A.n_rows * NF, vc = 8.0 * h.lv[l + 1].A.n_rows * NF;
            const double mat = (double)v.A.nnzb * (NF * NF * 8 + 4), minv = 8.0 * v.A.n_rows * NF * NF;
            bytes += (mat + 2 * vs + minv) + (mat + 3 * vs) + (vs + vc) + (2 * vs + vc) + t.sweeps * (mat + 3 * vs + minv);
        }
    }
    // cluster just large enough for two block rows of level l0 per row group
    // (128 groups per CTA), at most what the device runs
    const int cmax = tail_cluster_size<NF>(D), need = (h.lv[l0].A.n_rows + 255) / 256;
    int cl = 1;
    while (cl < need && cl < cmax) cl *= 2;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(cl);
    cfg.blockDim = dim3(kTailThreads);
    cfg.stream = s;
    cudaLaunchAttribute at;
    at.id = cudaLaunchAttributeClusterDimension;
    at.val.clusterDim.x = cl;
    at.val.clusterDim.y = 1;
    at.val.clusterDim.z = 1;
    cfg.attrs = &at;
    cfg.numAttrs = 1;
    {
        ProfScope ps(PC_MG_TAIL, s, bytes);
        gw_count_launch(cl);
        if (D == 2) cudaLaunchKernelEx(&cfg, k_mg_tail<2, NF>, ta);
        else cudaLaunchKernelEx(&cfg, k_mg_tail<3, NF>, ta);
    }
    // the buffer the per-phase path would end level l0 in: x on the way down,
    // alternating with x2 once per sweep
    const int S = mg_sweeps(l0);
    const int swaps = (S >= 2 ? 1 + (S - 2) : S - 1) + S;
    return (swaps & 1) ? h.lv[l0].x2 : h.lv[l0].x;
}

// One V-cycle on h.lv[0].b; returns the buffer that holds the result (the same
// buffer on every call).  Levels from tail_level() down run fused (mg_tail).
template <int NF, typename VT>
double *mg_vcycle(const MgHier &h, const int *skip, cudaStream_t s) {
    const int last = h.nl - 1;
    const int D = h.lv[0].g.dim;
    const int l0 = tail_level<NF, VT>(h);
    double *cur[kMgMaxLevels], *oth[kMgMaxLevels];
    for (int l = 0; l < l0; ++l) {
        const MgLevel &v = h.lv[l], &c = h.lv[l + 1];
        double *x = v.x, *y = v.x2;
        if (mg_sweeps(l) >= 2) {
            // both zero-start sweeps in one launch, into the buffer the
            // second separate sweep would have written
            PtrsA a = make_ptrs(v.A);
            const bool bf = l == 0 && mg_bf16_fine<VT>();
            if (bf) a.vals = v.pvals;
            const double vs = 8.0 * v.A.n_rows * NF;
            const double mat = (double)v.A.nnzb * (NF * NF * (bf ? 2 : sizeof(VT)) + 4);
            ProfScope ps(l == 0 ? PC_MG_JACOBI : PC_MG_JACOBI_COARSE, s, 2 * vs + 8.0 * v.A.n_rows * NF * NF + mat);
            if (bf)
                k_mg_presmooth2<NF, __nv_bfloat16><<<gw_count_launch(resident_rows_grid(
                                                         (const void *)k_mg_presmooth2<NF, __nv_bfloat16>,
                                                         tune_rows_block(), v.A.n_rows)),
                                                     tune_rows_block(), 0, s>>>(a, v.Minv, v.b, y, mg_omega(), skip);
            else
                k_mg_presmooth2<NF, VT><<<gw_count_launch(resident_rows_grid(
                                              (const void *)k_mg_presmooth2<NF, VT>, tune_rows_block(), v.A.n_rows)),
                                          tune_rows_block(), 0, s>>>(a, v.Minv, v.b, y, mg_omega(), skip);
            double *t = x; x = y; y = t;
            for (int it = 2; it < mg_sweeps(l); ++it) {
                mg_jacobi<NF, VT>(h, l, v.b, x, y, 0, skip, s);
                t = x; x = y; y = t;
            }
        } else {
            mg_jacobi<NF, VT>(h, l, v.b, nullptr, x, 1, skip, s);
            for (int it = 1; it < mg_sweeps(l); ++it) {
                mg_jacobi<NF, VT>(h, l, v.b, x, y, 0, skip, s);
                double *t = x; x = y; y = t;
            }
        }
        PtrsA a = make_ptrs(v.A), ca = make_ptrs(c.A);
        const double vs = 8.0 * v.A.n_rows * NF;
        {
        const bool bf = l == 0 && mg_bf16_fine<VT>();
        PtrsA ar = a;
        if (bf) ar.vals = v.pvals;
        ProfScope ps(PC_MG_RESID, s, 3 * vs + (double)v.A.nnzb * (NF * NF * (bf ? 2 : sizeof(VT)) + 4));
        if (bf)
            k_mg_residual<NF, __nv_bfloat16><<<gw_count_launch(resident_rows_grid(
                                                   (const void *)k_mg_residual<NF, __nv_bfloat16>, tune_rows_block(),
                                                   v.A.n_rows)),
                                               tune_rows_block(), 0, s>>>(ar, v.b, x, v.r, skip);
        else
            k_mg_residual<NF, VT><<<gw_count_launch(resident_rows_grid((const void *)k_mg_residual<NF, VT>,
                                                                       tune_rows_block(), v.A.n_rows)),
                                    tune_rows_block(), 0, s>>>(a, v.b, x, v.r, skip);
        }
        ProfScope ps(PC_MG_TRANSFER, s, vs + 8.0 * c.A.n_rows * NF);
        if (D == 2)
            k_mg_restrict_list<2, NF><<<gw_count_launch(nblk(c.A.n_rows, kThreads)), kThreads, 0, s>>>(
                c.A.n_rows, v.A.n_rows, c.child, v.fixed, v.r, c.b, skip);
        else
            k_mg_restrict_list<3, NF><<<gw_count_launch(nblk(c.A.n_rows, kThreads)), kThreads, 0, s>>>(
                c.A.n_rows, v.A.n_rows, c.child, v.fixed, v.r, c.b, skip);
        cur[l] = x;
        oth[l] = y;
    }
    if (l0 < last) {
        cur[l0] = mg_tail<NF>(h, l0, skip, s);
    } else {
        const MgLevel &lc = h.lv[last];
        k_mg_dense_apply<<<gw_count_launch(nblk((int64_t)h.dn * 32, kThreads)), kThreads, 0, s>>>(h.dInv, lc.b, lc.x, h.dn, skip);
        cur[last] = lc.x;
    }
    for (int l = l0 - 1; l >= 0; --l) {
        const MgLevel &v = h.lv[l], &c = h.lv[l + 1];
        PtrsA a = make_ptrs(v.A), ca = make_ptrs(c.A);
        double *x = cur[l], *y = oth[l];
        {
        ProfScope ps(PC_MG_TRANSFER, s, 16.0 * v.A.n_rows * NF + 8.0 * c.A.n_rows * NF);
        if (D == 2)
            k_mg_prolong_list<2, NF><<<gw_count_launch(nblk(v.A.n_rows, kThreads)), kThreads, 0, s>>>(
                v.A.n_rows, c.A.n_rows, v.parent, v.fixed, cur[l + 1], x, skip);
        else
            k_mg_prolong_list<3, NF><<<gw_count_launch(nblk(v.A.n_rows, kThreads)), kThreads, 0, s>>>(
                v.A.n_rows, c.A.n_rows, v.parent, v.fixed, cur[l + 1], x, skip);
        }
        for (int it = 0; it < mg_sweeps(l); ++it) {
            mg_jacobi<NF, VT>(h, l, v.b, x, y, 0, skip, s);
            double *t = x; x = y; y = t;
        }
        cur[l] = x;
    }
    return cur[0];
}

// One Arnoldi step with its V-cycle is ~40 small kernels.  Issuing them one by
// one costs more host time than the GPU spends running them, so the step is
// captured once as a CUDA graph and replayed.  Every kernel argument of the
// step is fixed by the key below (matrix, vectors, workspace, plan), so one
// instantiated graph serves all Newton iterations of a load step.  The graphs
// are held in a small cache (least recently used entry replaced).
struct MgGraphKey {
    int device, nf, vt_bytes, restart, nl, dn, dim, row_warps, one_sweep, sweeps, omega, tail, bf16, fine_sweeps;
    int n_grid[3];
    int n_rows[kMgMaxLevels], nnzb[kMgMaxLevels];
    gw_bsr_t A;
    const void *ws;
    const double *b;
    double *x, *z;
};
struct MgGraphEntry {
    bool valid;
    MgGraphKey key;
    cudaGraphExec_t exec;
    int64_t nodes;
    uint64_t stamp;
};
constexpr int kMgGraphCache = 8;
MgGraphEntry g_mg_graphs[kMgGraphCache];
uint64_t g_mg_graph_clock = 0;
cudaStream_t g_capture_stream[64] = {};

int capture_stream(cudaStream_t *out) {
    int dev = 0;
    GW_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) return GW_EINVAL;
    if (!g_capture_stream[dev]) GW_CUDA(cudaStreamCreateWithFlags(&g_capture_stream[dev], cudaStreamNonBlocking));
    *out = g_capture_stream[dev];
    return GW_OK;
}

template <int NF, typename VT>
void mg_arnoldi_step(const MgHier &h, const PtrsA &a, const GmresVecs &G, double *Z, int gr, int gv, size_t n,
                     const int *skip, cudaStream_t s) {
    k_gm_spmv_keep<NF, VT><<<gw_count_launch(resident_rows_grid((const void *)k_gm_spmv_keep<NF, VT>, kThreads, a.n_rows)),
                             kThreads, 0, s>>>(a, G, Z);
    k_gm_dots<<<gw_count_launch(gv), kThreads, 0, s>>>(G, 0);
    k_gm_update<<<gw_count_launch(gv), kThreads, 0, s>>>(G, 0);
    k_gm_dots<<<gw_count_launch(gv), kThreads, 0, s>>>(G, 1);
    k_gm_update<<<gw_count_launch(gv), kThreads, 0, s>>>(G, 1);
    k_gm_next_flex<<<gw_count_launch(gv), kThreads, 0, s>>>(n, G, 0, h.lv[0].b);
    mg_vcycle<NF, VT>(h, skip, s);
}

// Returns the cached (or newly captured) graph of one Arnoldi step.
template <int NF, typename VT>
int mg_step_graph(const MgHier &h, const gw_grid_t &grid, const gw_bsr_t *A, const GmresVecs &G, double *Z, void *ws,
                  int restart, int gr, int gv, size_t n, const int *skip, cudaGraphExec_t *exec, int64_t *nodes) {
    MgGraphKey k;
    memset(&k, 0, sizeof(k));
    GW_CUDA(cudaGetDevice(&k.device));
    k.nf = NF; k.vt_bytes = sizeof(VT); k.restart = restart; k.nl = h.nl; k.dn = h.dn; k.dim = grid.dim;
    k.row_warps = g_tune[GW_TUNE_ROW_WARPS];
    k.one_sweep = g_tune[GW_TUNE_MG_ONE_SWEEP];
    k.sweeps = g_tune[GW_TUNE_MG_SWEEPS];
    k.omega = g_tune[GW_TUNE_MG_OMEGA];
    k.tail = g_tune[GW_TUNE_MG_TAIL];
    k.bf16 = g_tune[GW_TUNE_MG_BF16];
    k.fine_sweeps = g_tune[GW_TUNE_MG_FINE_SWEEPS];
    for (int q = 0; q < 3; ++q) k.n_grid[q] = grid.n_grid[q];
    for (int q = 0; q < h.nl; ++q) { k.n_rows[q] = h.lv[q].A.n_rows; k.nnzb[q] = h.lv[q].A.nnzb; }
    k.A = *A; k.ws = ws; k.b = G.b; k.x = G.x; k.z = G.z;
    int victim = -1;
    for (int e = 0; e < kMgGraphCache; ++e) {
        MgGraphEntry &ent = g_mg_graphs[e];
        if (ent.valid && memcmp(&ent.key, &k, sizeof(k)) == 0) {
            ent.stamp = ++g_mg_graph_clock;
            *exec = ent.exec;
            *nodes = ent.nodes;
            return GW_OK;
        }
        // an empty slot first, else the least recently used one
        if (victim < 0 || (g_mg_graphs[victim].valid && (!ent.valid || ent.stamp < g_mg_graphs[victim].stamp)))
            victim = e;
    }
    cudaStream_t cs;
    int rc = capture_stream(&cs);
    if (rc) return rc;
    PtrsA a = make_ptrs(*A);
    const int64_t before = g_launches;
    GW_CUDA(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
    mg_arnoldi_step<NF, VT>(h, a, G, Z, gr, gv, n, skip, cs);
    cudaGraph_t graph;
    const cudaError_t ce = cudaStreamEndCapture(cs, &graph);
    const int64_t count = g_launches - before;
    g_launches = before;  // counted when the graph is replayed
    GW_CUDA(ce);
    cudaGraphExec_t ge;
    const cudaError_t ie = cudaGraphInstantiate(&ge, graph, 0);
    cudaGraphDestroy(graph);
    GW_CUDA(ie);
    MgGraphEntry &slot = g_mg_graphs[victim];
    if (slot.valid) GW_CUDA(cudaGraphExecDestroy(slot.exec));
    slot.valid = true;
    slot.key = k;
    slot.exec = ge;
    slot.nodes = count;
    slot.stamp = ++g_mg_graph_clock;
    *exec = ge;
    *nodes = count;
    return GW_OK;
}

template <int NF, typename VT>
int gmres_mg(const gw_grid_t *grid, const gw_bsr_t *A, gw_mg_plan_t *plan_in, const double *b, double *x,
             double rtol, int max_iter, int restart, void *ws, int64_t ws_bytes, int *iters, double *relres,
             cudaStream_t s) {
    const int nr = A->n_rows;
    if (nr == 0) { *iters = 0; *relres = 0.0; return GW_OK; }
    const int64_t n = (int64_t)nr * NF;
    (void)tail_cluster_size<NF>(grid->dim);  // device queries before any stream capture
    {
        const int tb = tune_rows_block();
        (void)resident_rows_grid((const void *)k_mg_jacobi<NF, VT>, tb, 1);
        (void)resident_rows_grid((const void *)k_mg_presmooth2<NF, VT>, tb, 1);
        (void)resident_rows_grid((const void *)k_mg_residual<NF, VT>, tb, 1);
        (void)resident_rows_grid((const void *)k_mg_jacobi<NF, __nv_bfloat16>, tb, 1);
        (void)resident_rows_grid((const void *)k_mg_presmooth2<NF, __nv_bfloat16>, tb, 1);
        (void)resident_rows_grid((const void *)k_mg_residual<NF, __nv_bfloat16>, tb, 1);
        (void)resident_rows_grid((const void *)k_gm_spmv_keep<NF, VT>, kThreads, 1);
    }
    Bump bp{(char *)ws, 0};
    MgHier h;
    FlexVecs fv;
    mg_carve_hier(bp, h, *grid, nr, NF);
    mg_carve_flex(bp, fv, n, restart);
    if (bp.used > ws_bytes) {
        snprintf(g_msg, sizeof(g_msg), "multigrid GMRES: workspace of %lld bytes, %lld needed", (long long)ws_bytes,
                 (long long)bp.used);
        return GW_EINVAL;
    }
    int rc;
    {
        ProfScope ps(PC_MG_SETUP, s, (double)A->nnzb * (NF * NF * sizeof(VT) + 4));
        gw_mg_plan_t local;
        if (plan_in) {
            if (plan_in->workspace != ws || plan_in->nf != NF || plan_in->fine_n_rows != nr ||
                plan_in->fine_nnzb != A->nnzb || plan_in->row_ptr != A->row_ptr || plan_in->cols != A->cols ||
                plan_in->levels < 1 || plan_in->levels > h.nl ||
                plan_in->dense_n != plan_in->n_rows[plan_in->levels - 1] * NF || plan_in->dense_n > kMgCoarseMax) {
                snprintf(g_msg, sizeof(g_msg), "multigrid GMRES: the plan was built for another workspace or pattern");
                return GW_EINVAL;
            }
            mg_apply_plan(h, A, plan_in, NF);
        } else {
            rc = mg_pattern<NF>(h, A, &local, s);
            if (rc) return rc;
        }
        // lag: the previous solve's coarse operators, smoothers and dense
        // inverse are still in the workspace; GMRES itself applies A
        rc = (plan_in && plan_in->lag) ? GW_OK : mg_numeric<NF, VT>(h, s);
        // the V-cycle's BF16 copy of the fine level follows the current A on
        // every solve, lagged or not (the fine level's own rows are never lagged)
        if (!rc && mg_bf16_fine<VT>()) {
            const size_t nv = (size_t)A->nnzb * NF * NF;
            k_to_bf16<<<gw_count_launch(red_grid_elems((int64_t)nv)), kThreads, 0, s>>>(
                (const float *)A->vals, (__nv_bfloat16 *)h.lv[0].pvals, nv);
            GW_LAUNCHED();
        }
    }
    if (rc) return rc;
    PtrsA a = make_ptrs(*A);
    GmresVecs G;
    G.V = fv.V; G.w = fv.w; G.partials = fv.partials; G.sc = fv.sc; G.Minv = nullptr;
    G.x = x; G.b = b; G.n = (size_t)n;
    G.z = nullptr;
    const size_t head = offsetof(GScalars, H);
    GW_CUDA(cudaMemsetAsync(G.sc, 0, head, s));
    struct { int max_iter, restart; } lim = {max_iter, restart};
    GW_CUDA(cudaMemcpyAsync(&G.sc->max_iter, &lim, sizeof(lim), cudaMemcpyHostToDevice, s));
    const double eta2 = ::pow(10.0, -0.1 * g_tune[GW_TUNE_GS_CANCEL]);
    GW_CUDA(cudaMemcpyAsync(&G.sc->gs_eta2, &eta2, sizeof(double), cudaMemcpyHostToDevice, s));
    const int gr = red_grid_rows(nr), gv = red_grid_elems(n);
    const int gk = resident_rows_grid((const void *)k_gm_spmv_keep<NF, VT>, kThreads, nr);
    const int *skip = &G.sc->cycle_done;
    GScalars hs;
    memset(&hs, 0, head);
    int first = 1;
    StallWatch stall;
    g_last_stalled = 0;
    for (int cycle = 0; cycle < 1000000; ++cycle) {
        k_gm_residual<NF, VT><<<gw_count_launch(gr), kThreads, 0, s>>>(a, G, first, rtol);
        k_gm_next_flex<<<gw_count_launch(gv), kThreads, 0, s>>>((size_t)n, G, 1, h.lv[0].b);
        GW_LAUNCHED();
        G.z = mg_vcycle<NF, VT>(h, skip, s);
        GW_LAUNCHED();
        first = 0;
        GW_CUDA(cudaMemcpyAsync(&hs, G.sc, head, cudaMemcpyDeviceToHost, s));
        GW_CUDA(cudaStreamSynchronize(s));
        if (hs.done) break;
        if (stall.stalled(hs.beta)) { g_last_stalled = 1; break; }
        // Arnoldi steps queued before the next host check: the previous
        // solve's iteration count to start with (Newton solves of a step look
        // alike), then the iterations left at the observed convergence rate.
        // Steps queued past convergence still launch their (early-exiting)
        // kernels, so the estimate trims them without adding host reads.
        const int hint = plan_in ? plan_in->last_iters : 0;
        int chunk = hint > 0 ? std::min(std::max(hint, 2), 16) : 4;
        int kk = 0;
        const double spmv_bytes = (double)A->nnzb * (NF * NF * sizeof(VT) + 4) + 4.0 * (nr + 1) + 24.0 * n;
        cudaGraphExec_t step_graph = nullptr;
        int64_t step_nodes = 0;
        if (!g_prof_on) {  // timed runs launch kernel by kernel, bracketed by events
            rc = mg_step_graph<NF, VT>(h, *grid, A, G, fv.Z, ws, restart, gr, gv, (size_t)n, skip, &step_graph,
                                       &step_nodes);
            if (rc) return rc;
        }
        for (;;) {
            for (int it = 0; it < chunk; ++it, ++kk) {
                if (step_graph) {
                    GW_CUDA(cudaGraphLaunch(step_graph, s));
                    g_launches += step_nodes;
                    continue;
                }
                const double vb = 8.0 * n * (kk + 2);
                { ProfScope ps(PC_SPMV, s, spmv_bytes); k_gm_spmv_keep<NF, VT><<<gw_count_launch(gk), kThreads, 0, s>>>(a, G, fv.Z); }
                { ProfScope ps(PC_DOTS, s, vb + 8.0 * n); k_gm_dots<<<gw_count_launch(gv), kThreads, 0, s>>>(G, 0); }
                { ProfScope ps(PC_UPDATE, s, vb + 8.0 * n); k_gm_update<<<gw_count_launch(gv), kThreads, 0, s>>>(G, 0); }
                const int re = prof_reorth(G.sc, s);
                { ProfScope ps(PC_DOTS, s, re ? vb : 0.0); k_gm_dots<<<gw_count_launch(gv), kThreads, 0, s>>>(G, 1); }
                { ProfScope ps(PC_UPDATE, s, re ? vb + 8.0 * n : 0.0); k_gm_update<<<gw_count_launch(gv), kThreads, 0, s>>>(G, 1); }
                { ProfScope ps(PC_NEXT, s, 8.0 * n * 3); k_gm_next_flex<<<gw_count_launch(gv), kThreads, 0, s>>>((size_t)n, G, 0, h.lv[0].b); }
                mg_vcycle<NF, VT>(h, skip, s);
            }
            GW_LAUNCHED();
            GW_CUDA(cudaMemcpyAsync(&hs, G.sc, head, cudaMemcpyDeviceToHost, s));
            GW_CUDA(cudaStreamSynchronize(s));
            if (hs.cycle_done) break;
            int next = chunk < 16 ? chunk * 2 : 16;
            if (hs.k > 0 && hs.beta > 0.0 && hs.resid > 0.0 && hs.resid < hs.beta && hs.tol > 0.0) {
                const double rate = ::pow(hs.resid / hs.beta, 1.0 / hs.k);
                if (rate < 1.0) {
                    const double left = ::ceil(::log(hs.tol / hs.resid) / ::log(rate));
                    next = left < 1.0 ? 1 : (left > 16.0 ? 16 : (int)left);
                }
            }
            chunk = next;
        }
        if (hs.status) break;
        k_gm_solve_y<<<gw_count_launch(1), 32, 0, s>>>(G.sc);
        k_gm_update_x_flex<<<gw_count_launch(gv), kThreads, 0, s>>>((size_t)n, G, fv.Z);
        GW_LAUNCHED();
    }
    *iters = hs.iters;
    g_last_reorths = hs.reorths;
    *relres = (hs.bnorm > 0.0) ? hs.resid / hs.bnorm : 0.0;
    if (plan_in) plan_in->last_iters = hs.iters;
    rc = guard_check(s, "multigrid GMRES");
    if (rc) return rc;
    if (hs.status == ST_NAN) return GW_ENAN;
    if (hs.resid > hs.tol) return GW_ENOCONV;
    return GW_OK;
}

template <typename VT>
int gmres_mg_nf(const gw_grid_t *grid, const gw_bsr_t *A, gw_mg_plan_t *plan, const double *b, double *x,
                double rtol, int max_iter, int restart, void *ws, int64_t ws_bytes, int *iters, double *relres,
                cudaStream_t s) {
    switch (A->nf) {
        case 1: return gmres_mg<1, VT>(grid, A, plan, b, x, rtol, max_iter, restart, ws, ws_bytes, iters, relres, s);
        case 2: return gmres_mg<2, VT>(grid, A, plan, b, x, rtol, max_iter, restart, ws, ws_bytes, iters, relres, s);
        case 3: return gmres_mg<3, VT>(grid, A, plan, b, x, rtol, max_iter, restart, ws, ws_bytes, iters, relres, s);
        case 4: return gmres_mg<4, VT>(grid, A, plan, b, x, rtol, max_iter, restart, ws, ws_bytes, iters, relres, s);
        default: return GW_EINVAL;
    }
}

int mg_check_args(const gw_grid_t *grid, const gw_bsr_t *A) {
    GW_REQUIRE(grid->dim == 2 || grid->dim == 3);
    GW_REQUIRE(A->mask_words == (grid->dim == 2 ? 1 : 4));
    GW_REQUIRE(A->n_rows <= grid->n_nodes);
    GW_REQUIRE(A->nf >= 1 && A->nf <= 4);
    return GW_OK;
}
}  // namespace

extern "C" int64_t gw_gmres_mg_workspace_bytes(const gw_grid_t *grid, int32_t n_rows, int32_t nf, int32_t restart) {
    if (!grid || restart < 1 || restart > kGmresMaxRestart || nf < 1 || nf > 4 || n_rows < 0) return -1;
    return mg_ws_bytes(*grid, n_rows, nf, restart);
}

extern "C" int gw_mg_plan_build(const gw_grid_t *grid, const gw_bsr_t *A, void *workspace, int64_t workspace_bytes,
                                gw_mg_plan_t *plan_host, void *stream) {
    GW_REQUIRE(grid && A && workspace && plan_host);
    int rc = mg_check_args(grid, A);
    if (rc) return rc;
    Bump bp{(char *)workspace, 0};
    MgHier h;
    mg_carve_hier(bp, h, *grid, A->n_rows, A->nf);
    if (bp.used > workspace_bytes) {
        snprintf(g_msg, sizeof(g_msg), "multigrid plan: workspace of %lld bytes, %lld needed",
                 (long long)workspace_bytes, (long long)bp.used);
        return GW_EINVAL;
    }
    cudaStream_t s = S(stream);
    switch (A->nf) {
        case 1: rc = mg_pattern<1>(h, A, plan_host, s); break;
        case 2: rc = mg_pattern<2>(h, A, plan_host, s); break;
        case 3: rc = mg_pattern<3>(h, A, plan_host, s); break;
        default: rc = mg_pattern<4>(h, A, plan_host, s); break;
    }
    if (rc) return rc;
    rc = guard_check(s, "multigrid plan");
    if (rc) return rc;
    plan_host->workspace = workspace;
    return GW_OK;
}

extern "C" int32_t gw_gmres_last_reorths(void) { return g_last_reorths; }
extern "C" int32_t gw_gmres_last_stalled(void) { return g_last_stalled; }

extern "C" int gw_bsr_gmres_mg_solve(const gw_grid_t *grid, const gw_bsr_t *A, int32_t prec,
                                     gw_mg_plan_t *plan_host, const double *b, double *x, double rtol,
                                     int32_t max_iter, int32_t restart, void *workspace, int64_t workspace_bytes,
                                     int32_t *iters_host, double *relres_host, void *stream) {
    GW_REQUIRE(grid && A && b && x && workspace && iters_host && relres_host && max_iter > 0);
    GW_REQUIRE(vec_ok(A, b, x));
    GW_REQUIRE(restart >= 1 && restart <= kGmresMaxRestart);
    int rc = mg_check_args(grid, A);
    if (rc) return rc;
    int it = 0;
    double rr = 0.0;
    rc = (prec == GW_PREC_F64)
             ? gmres_mg_nf<double>(grid, A, plan_host, b, x, rtol, max_iter, restart, workspace, workspace_bytes, &it,
                                   &rr, S(stream))
             : gmres_mg_nf<float>(grid, A, plan_host, b, x, rtol, max_iter, restart, workspace, workspace_bytes, &it,
                                  &rr, S(stream));
    *iters_host = it;
    *relres_host = rr;
    return rc;
}

extern "C" int64_t gw_krylov_workspace_bytes(int32_t n_rows, int32_t nf, int32_t prec) {
    (void)prec;
    return krylov_ws_bytes(n_rows, nf);
}

extern "C" int gw_bsr_krylov_solve(const gw_bsr_t *A, int32_t prec, int32_t method, int32_t precond, const double *b,
                                   double *x, double rtol, int32_t max_iter, void *workspace, int32_t *iters_host,
                                   double *relres_host, void *stream) {
    GW_REQUIRE(A && b && x && workspace && iters_host && relres_host && max_iter > 0);
    GW_REQUIRE(vec_ok(A, b, x));
    int it = 0;
    double rr = 0.0;
    int rc = (prec == GW_PREC_F64)
                 ? krylov_nf<double>(A, method, precond, b, x, rtol, max_iter, workspace, &it, &rr, S(stream))
                 : krylov_nf<float>(A, method, precond, b, x, rtol, max_iter, workspace, &it, &rr, S(stream));
    *iters_host = it;
    *relres_host = rr;
    return rc;
}

// ==================================================================== Krylov without a caller workspace
// For callers that cannot allocate device memory themselves: a host whose own
// memory manager owns the device heap, or a code path where calling cudaMalloc
// is not allowed.  The scratch the BiCGSTAB / CG driver needs lives in one
// file-scope device array, sized for at most kStaticKrylovMaxUnknowns unknowns
// (n_rows * nf); every GPU that loads the library holds it (about 12.6 MB)
// until the process exits.
namespace {
constexpr int64_t kStaticKrylovMaxUnknowns = 131072;
constexpr int64_t align256c(int64_t b) { return (b + 255) & ~(int64_t)255; }
// krylov_ws_bytes at the limit, for the largest block size (nf = 4)
constexpr int64_t kStaticKrylovBytes = 8 * align256c(8 * kStaticKrylovMaxUnknowns) +
                                       align256c(8 * kStaticKrylovMaxUnknowns * 4) +
                                       align256c(8 * (int64_t)kRedBlocks * 4) + align256c(sizeof(KScalars));
static __device__ __align__(256) unsigned char g_krylov_scratch[kStaticKrylovBytes];

constexpr int kMaxStaticDevices = 64;
void *g_krylov_scratch_addr[kMaxStaticDevices] = {};

// Device address of g_krylov_scratch on the current device.  The name is only a
// host-side stand-in, so the address is looked up once per device, with that
// device current, and cached.
int static_krylov_scratch(void **out) {
    int dev = 0;
    GW_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxStaticDevices) {
        snprintf(g_msg, sizeof(g_msg), "gw_bsr_krylov_solve_static: device ordinal %d above %d", dev,
                 kMaxStaticDevices - 1);
        return GW_EINVAL;
    }
    void *p = __atomic_load_n(&g_krylov_scratch_addr[dev], __ATOMIC_ACQUIRE);
    if (!p) {
        GW_CUDA(cudaGetSymbolAddress(&p, g_krylov_scratch));
        __atomic_store_n(&g_krylov_scratch_addr[dev], p, __ATOMIC_RELEASE);
    }
    *out = p;
    return GW_OK;
}
}  // namespace

extern "C" int64_t gw_krylov_static_max_unknowns(void) { return kStaticKrylovMaxUnknowns; }

extern "C" int gw_bsr_krylov_solve_static(const gw_bsr_t *A, int32_t prec, int32_t method, int32_t precond,
                                          const double *b, double *x, double rtol, int32_t max_iter,
                                          int32_t *iters_host, double *relres_host, void *stream) {
    GW_REQUIRE(A && b && x && iters_host && relres_host && max_iter > 0);
    GW_REQUIRE(vec_ok(A, b, x));
    const int64_t unknowns = (int64_t)A->n_rows * A->nf;
    if (A->n_rows < 0 || A->nf < 1 || A->nf > 4 || unknowns > kStaticKrylovMaxUnknowns ||
        krylov_ws_bytes(A->n_rows, A->nf) > kStaticKrylovBytes) {
        snprintf(g_msg, sizeof(g_msg),
                 "gw_bsr_krylov_solve_static: %lld unknowns (n_rows %d x nf %d) exceed the static scratch limit of "
                 "%lld unknowns; use gw_bsr_krylov_solve with a caller workspace",
                 (long long)unknowns, A->n_rows, A->nf, (long long)kStaticKrylovMaxUnknowns);
        return GW_EINVAL;
    }
    void *ws = nullptr;
    const int rs = static_krylov_scratch(&ws);
    if (rs != GW_OK) return rs;
    // the driver clears the scalar block (reduction ticket, flags) on every call
    // and writes every vector before reading it, so the contents a previous call
    // left in the scratch are never used
    int it = 0;
    double rr = 0.0;
    int rc = (prec == GW_PREC_F64)
                 ? krylov_nf<double>(A, method, precond, b, x, rtol, max_iter, ws, &it, &rr, S(stream))
                 : krylov_nf<float>(A, method, precond, b, x, rtol, max_iter, ws, &it, &rr, S(stream));
    *iters_host = it;
    *relres_host = rr;
    return rc;
}

namespace {
template <typename VT>
int spmv_any(const gw_bsr_t *A, const double *x, double *y, bool trans, cudaStream_t s) {
    PtrsA a = make_ptrs(*A);
    const int g = red_grid_rows(A->n_rows);
    if (A->n_rows == 0) return GW_OK;
    if (trans) GW_CUDA(cudaMemsetAsync(y, 0, sizeof(double) * (size_t)A->n_rows * A->nf, s));
#define GW_SPMV_CASE(NF_)                                                  \
    case NF_:                                                              \
        if (trans) k_spmv_t<NF_, VT><<<gw_count_launch(g), kThreads, 0, s>>>(a, x, y);      \
        else k_spmv<NF_, VT><<<gw_count_launch(g), kThreads, 0, s>>>(a, x, y);              \
        break;
    switch (A->nf) {
        GW_SPMV_CASE(1) GW_SPMV_CASE(2) GW_SPMV_CASE(3) GW_SPMV_CASE(4)
        default: return GW_EINVAL;
    }
#undef GW_SPMV_CASE
    GW_LAUNCHED();
    return GW_OK;
}
}  // namespace

extern "C" int gw_bsr_spmv(const gw_bsr_t *A, int32_t prec, const double *x, double *y, void *stream) {
    GW_REQUIRE(A && x && y);
    GW_REQUIRE(vec_ok(A, x, y));
    return prec == GW_PREC_F64 ? spmv_any<double>(A, x, y, false, S(stream)) : spmv_any<float>(A, x, y, false, S(stream));
}

extern "C" int gw_bsr_spmv_t(const gw_bsr_t *A, int32_t prec, const double *x, double *y, void *stream) {
    GW_REQUIRE(A && x && y);
    return prec == GW_PREC_F64 ? spmv_any<double>(A, x, y, true, S(stream)) : spmv_any<float>(A, x, y, true, S(stream));
}