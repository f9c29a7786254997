// C ABI of the engine (declarations and reference citations in
// include/geowarp_b200.h): queries, cell sort, activation, pattern,
// consistent mass, norms, G2P, single-point models, launch knobs and kernel
// timing.  The solvers, the assembly and the adjoint entry points live in
// gw_abi_solve.cu, gw_abi_assemble.cu and gw_abi_adjoint.cu.  This file also
// defines the device globals the kernel headers declare.
#define GW_DEFINE_DEVICE_GLOBALS
#include "gw_host.cuh"
#include "gw_mg.cuh"

using namespace gw;
using namespace gwh;

extern "C" int gw_guard_read(int32_t *site, int64_t *value, void *stream) {
    GW_REQUIRE(site && value);
    int st = 0;
    long long v = 0;
    cudaStream_t s = (cudaStream_t)stream;
    GW_CUDA(cudaMemcpyFromSymbolAsync(&st, g_guard_site, sizeof(int), 0, cudaMemcpyDeviceToHost, s));
    GW_CUDA(cudaMemcpyFromSymbolAsync(&v, g_guard_value, sizeof(long long), 0, cudaMemcpyDeviceToHost, s));
    GW_CUDA(cudaStreamSynchronize(s));
    const int zero = 0;
    const long long zero_v = 0;
    GW_CUDA(cudaMemcpyToSymbolAsync(g_guard_site, &zero, sizeof(int), 0, cudaMemcpyHostToDevice, s));
    GW_CUDA(cudaMemcpyToSymbolAsync(g_guard_value, &zero_v, sizeof(long long), 0, cudaMemcpyHostToDevice, s));
    GW_CUDA(cudaStreamSynchronize(s));
    *site = st;
    *value = v;
    return GW_OK;
}

extern "C" const char *gw_guard_site_name(int32_t site) {
    return (site >= 0 && site < GS_COUNT) ? kGuardNames[site] : "unknown site";
}

// ==================================================================== queries
extern "C" int gw_version(void) { return 1; }

extern "C" const char *gw_status_string(int code) {
    switch (code) {
        case GW_OK: return "ok";
        case GW_EINVAL: return g_msg[0] ? g_msg : "invalid argument";
        case GW_ECUDA: return g_msg[0] ? g_msg : "CUDA error";
        case GW_ENOCONV: return "Krylov solver did not reach the tolerance (iteration cap or GMRES stagnation)";
        case GW_EBREAKDOWN: return "Krylov breakdown";
        case GW_ENAN: return "non-finite value";
        case GW_ERANGE: return g_msg[0] ? g_msg : "index guard failed: a device index was out of range";
        case GW_EMODEL: return "material model not available for this solver kind";
        default: return "unknown status";
    }
}

extern "C" int gw_read_device_status(int32_t *flag_host, void *stream) {
    GW_REQUIRE(flag_host);
    int v = 0;
    GW_CUDA(cudaMemcpyFromSymbolAsync(&v, g_status, sizeof(int), 0, cudaMemcpyDeviceToHost, S(stream)));
    GW_CUDA(cudaStreamSynchronize(S(stream)));
    const int zero = 0;
    GW_CUDA(cudaMemcpyToSymbolAsync(g_status, &zero, sizeof(int), 0, cudaMemcpyHostToDevice, S(stream)));
    GW_CUDA(cudaStreamSynchronize(S(stream)));
    *flag_host = v;
    return GW_OK;
}

// ==================================================================== sort
extern "C" int64_t gw_sort_workspace_bytes(int32_t n) {
    const int64_t nb = (n + kSortTile - 1) / kSortTile;
    return align256(4 * (int64_t)n) * 2 + align256(4 * 256 * nb) + align256(4 * scan_ws_ints(256 * nb));
}

extern "C" int gw_cell_sort(const gw_grid_t *grid, const gw_particles_t *pt, int32_t *keys_out, int32_t *perm_out,
                            void *workspace, void *stream) {
    GW_REQUIRE(grid && pt && keys_out && perm_out && workspace);
    const int n = pt->n;
    if (n == 0) return GW_OK;
    cudaStream_t s = S(stream);
    const int nb = (n + kSortTile - 1) / kSortTile;
    char *w = (char *)workspace;
    int *kalt = (int *)w; w += align256(4 * (int64_t)n);
    int *valt = (int *)w; w += align256(4 * (int64_t)n);
    int *hist = (int *)w; w += align256(4 * 256 * (int64_t)nb);
    int *sws = (int *)w;
    if (grid->dim == 2) k_cell_keys<2><<<gw_count_launch(nblk(n, kThreads)), kThreads, 0, s>>>(*grid, pt->x, pt->lp, n, keys_out, perm_out);
    else k_cell_keys<3><<<gw_count_launch(nblk(n, kThreads)), kThreads, 0, s>>>(*grid, pt->x, pt->lp, n, keys_out, perm_out);
    GW_LAUNCHED();
    const int ncell = n_cells_of(*grid);
    int bits = 1;
    while ((1 << bits) < ncell && bits < 31) ++bits;
    const int passes = (bits + 7) / 8;
    int *kin = keys_out, *vin = perm_out, *kout = kalt, *vout = valt;
    for (int ps = 0; ps < passes; ++ps) {
        const int shift = 8 * ps;
        k_radix_hist<<<gw_count_launch(nb), kThreads, 0, s>>>(kin, n, shift, nb, hist);
        GW_LAUNCHED();
        int rc = scan_exclusive(hist, hist, 256 * nb, sws, s);
        if (rc) return rc;
        k_radix_scatter<<<gw_count_launch(nb), kThreads, 0, s>>>(kin, vin, n, shift, nb, hist, kout, vout);
        GW_LAUNCHED();
        int *t = kin; kin = kout; kout = t;
        t = vin; vin = vout; vout = t;
    }
    if (kin != keys_out) {
        GW_CUDA(cudaMemcpyAsync(keys_out, kin, 4 * (size_t)n, cudaMemcpyDeviceToDevice, s));
        GW_CUDA(cudaMemcpyAsync(perm_out, vin, 4 * (size_t)n, cudaMemcpyDeviceToDevice, s));
    }
    return GW_OK;
}

// ==================================================================== activation / compaction / pattern
extern "C" int gw_p2g_activate(const gw_grid_t *grid, const gw_particles_t *pt, const int32_t *perm,
                               uint8_t *node_active, uint32_t *cell_span_u8, uint8_t *boundary, void *stream) {
    GW_REQUIRE(grid && pt && node_active && cell_span_u8 && boundary);
    if (pt->n == 0) return GW_OK;
    LaunchConst c = make_lc(grid, nullptr, nullptr);
    PtrsP p = make_ptrs(*pt);
    uint32_t *cs = cell_span_u8;
    const int b = nblk(pt->n, kThreads);
    switch (grid->kind) {
        case GW_KIND_SOLID2D: k_activate<GW_KIND_SOLID2D><<<gw_count_launch(b), kThreads, 0, S(stream)>>>(c, p, perm, node_active, cs, boundary); break;
        case GW_KIND_COUPLED2D: k_activate<GW_KIND_COUPLED2D><<<gw_count_launch(b), kThreads, 0, S(stream)>>>(c, p, perm, node_active, cs, boundary); break;
        case GW_KIND_COUPLED3D: k_activate<GW_KIND_COUPLED3D><<<gw_count_launch(b), kThreads, 0, S(stream)>>>(c, p, perm, node_active, cs, boundary); break;
        default: return GW_EINVAL;
    }
    GW_LAUNCHED();
    return GW_OK;
}

extern "C" int gw_touched_nodes(const gw_grid_t *grid, const uint32_t *cell_span, uint8_t *touched, void *stream) {
    GW_REQUIRE(grid && cell_span && touched);
    const int nc = n_cells_of(*grid);
    if (grid->dim == 2) k_touched<2><<<gw_count_launch(nblk(nc, kThreads)), kThreads, 0, S(stream)>>>(*grid, cell_span, nc, touched);
    else k_touched<3><<<gw_count_launch(nblk(nc, kThreads)), kThreads, 0, S(stream)>>>(*grid, cell_span, nc, touched);
    GW_LAUNCHED();
    return GW_OK;
}

extern "C" int64_t gw_scan_workspace_bytes(int32_t n) { return align256(4 * ((int64_t)n + 1)) + align256(4 * (scan_ws_ints((int64_t)n + 1) + 64)); }

extern "C" int gw_compact_rows(const gw_grid_t *grid, const uint8_t *node_active, const uint8_t *boundary,
                               int32_t *node2row, int32_t *row2node, uint8_t *free_mask, int32_t *n_rows_host,
                               void *workspace, void *stream) {
    GW_REQUIRE(grid && node_active && node2row && row2node && n_rows_host && workspace);
    const int n = grid->n_nodes;
    cudaStream_t s = S(stream);
    char *w = (char *)workspace;
    int *tmp = (int *)w; w += align256(4 * ((int64_t)n + 1));
    int *sws = (int *)w;
    k_flags_to_int<<<gw_count_launch(nblk(n, kThreads)), kThreads, 0, s>>>(node_active, n, tmp);
    GW_LAUNCHED();
    int *last = sws;  // [0]: flag of the last node, [1]: number of active nodes
    GW_CUDA(cudaMemcpyAsync(last, tmp + (n - 1), 4, cudaMemcpyDeviceToDevice, s));
    int rc = scan_exclusive(tmp, tmp, n, sws + 64, s);
    if (rc) return rc;
    k_compact<<<gw_count_launch(nblk(n, kThreads)), kThreads, 0, s>>>(node_active, tmp, n, grid->nf, boundary, node2row, row2node,
                                                     free_mask);
    GW_LAUNCHED();
    k_add2<<<gw_count_launch(1), 32, 0, s>>>(tmp + (n - 1), last, last + 1);
    GW_LAUNCHED();
    int tot = 0;
    GW_CUDA(cudaMemcpyAsync(&tot, last + 1, 4, cudaMemcpyDeviceToHost, s));
    GW_CUDA(cudaStreamSynchronize(s));
    *n_rows_host = tot;
    return GW_OK;
}

extern "C" int gw_pattern_count(const gw_grid_t *grid, const uint32_t *cell_span_u8, const int32_t *node2row,
                                const int32_t *row2node, int32_t n_rows, uint32_t *stencil, int32_t *row_ptr,
                                int32_t *nnzb_host, void *workspace, void *stream) {
    GW_REQUIRE(grid && cell_span_u8 && node2row && row2node && stencil && row_ptr && nnzb_host && workspace);
    cudaStream_t s = S(stream);
    const uint32_t *cs = cell_span_u8;
    const int mw = grid->dim == 2 ? 1 : 4;
    GW_CUDA(cudaMemsetAsync(row_ptr, 0, 4 * ((size_t)n_rows + 1), s));
    if (n_rows > 0) {
        if (grid->dim == 2)
            k_pattern_count<2><<<gw_count_launch(nblk(n_rows, kThreads)), kThreads, 0, s>>>(*grid, cs, node2row, row2node, n_rows, mw, stencil, row_ptr);
        else
            k_pattern_count<3><<<gw_count_launch(nblk(n_rows, kThreads)), kThreads, 0, s>>>(*grid, cs, node2row, row2node, n_rows, mw, stencil, row_ptr);
        GW_LAUNCHED();
    }
    int rc = scan_exclusive(row_ptr, row_ptr, n_rows + 1, (int *)workspace, s);
    if (rc) return rc;
    int tot = 0;
    GW_CUDA(cudaMemcpyAsync(&tot, row_ptr + n_rows, 4, cudaMemcpyDeviceToHost, s));
    GW_CUDA(cudaStreamSynchronize(s));
    *nnzb_host = tot;
    return GW_OK;
}

extern "C" int gw_pattern_fill(const gw_grid_t *grid, const gw_bsr_t *A, int32_t *cols, void *stream) {
    GW_REQUIRE(grid && A && cols);
    if (A->n_rows == 0) return GW_OK;
    PtrsA a = make_ptrs(*A);
    if (grid->dim == 2) k_pattern_fill<2><<<gw_count_launch(nblk(A->n_rows, kThreads)), kThreads, 0, S(stream)>>>(*grid, a, cols);
    else k_pattern_fill<3><<<gw_count_launch(nblk(A->n_rows, kThreads)), kThreads, 0, S(stream)>>>(*grid, a, cols);
    GW_LAUNCHED();
    return GW_OK;
}

// ==================================================================== consistent mass
extern "C" int gw_mass_assemble(const gw_grid_t *grid, const gw_particles_t *pt, const int32_t *perm,
                                const gw_step_t *st, const gw_bsr_t *M, double *rhs, void *stream) {
    GW_REQUIRE(grid && pt && perm && st && M && rhs && M->nf == 1);
    cudaStream_t s = S(stream);
    GW_CUDA(cudaMemsetAsync(M->vals, 0, sizeof(double) * (size_t)M->nnzb, s));
    GW_CUDA(cudaMemsetAsync(rhs, 0, sizeof(double) * (size_t)M->n_rows, s));
    LaunchConst c = make_lc(grid, nullptr, st);
    PtrsP p = make_ptrs(*pt);
    PtrsA m = make_ptrs(*M);
    const int b = nblk(pt->n, kThreads);
    if (pt->n > 0) {
        if (grid->kind == GW_KIND_COUPLED2D) k_mass<GW_KIND_COUPLED2D><<<gw_count_launch(b), kThreads, 0, s>>>(c, p, perm, m, rhs);
        else if (grid->kind == GW_KIND_COUPLED3D) k_mass<GW_KIND_COUPLED3D><<<gw_count_launch(b), kThreads, 0, s>>>(c, p, perm, m, rhs);
        else return GW_EINVAL;
        GW_LAUNCHED();
    }
    if (M->n_rows > 0) {
        if (grid->dim == 2) k_mass_fix<2><<<gw_count_launch(nblk(M->n_rows, kThreads)), kThreads, 0, s>>>(m);
        else k_mass_fix<3><<<gw_count_launch(nblk(M->n_rows, kThreads)), kThreads, 0, s>>>(m);
        GW_LAUNCHED();
    }
    return GW_OK;
}

extern "C" int gw_mass_lumped_solve(const gw_bsr_t *M, const double *rhs, double *x, void *stream) {
    GW_REQUIRE(M && rhs && x && M->nf == 1);
    if (M->n_rows == 0) return GW_OK;
    k_mass_lumped<<<gw_count_launch(nblk(M->n_rows, kThreads)), kThreads, 0, S(stream)>>>(make_ptrs(*M), rhs, x);
    GW_LAUNCHED();
    return GW_OK;
}

extern "C" int gw_set_nodal_pressure(const gw_grid_t *grid, const int32_t *mass_row2node, int32_t n_mass_rows,
                                     const double *p_hat, const uint8_t *boundary, const uint8_t *node_active,
                                     double *u_old, double *u_new, void *stream) {
    GW_REQUIRE(grid && mass_row2node && p_hat && boundary && u_old && u_new);
    if (n_mass_rows == 0) return GW_OK;
    k_set_nodal_pressure<<<gw_count_launch(nblk(n_mass_rows, kThreads)), kThreads, 0, S(stream)>>>(
        n_mass_rows, mass_row2node, p_hat, boundary, grid->kind == GW_KIND_COUPLED3D ? node_active : nullptr,
        grid->n_nodes, grid->nf, u_old, u_new);
    GW_LAUNCHED();
    return GW_OK;
}


extern "C" int gw_norm2(const double *v, int32_t n, double *norm_dev, void *workspace, void *stream) {
    GW_REQUIRE(v && norm_dev && workspace);
    double *partials = (double *)workspace;
    unsigned *ticket = (unsigned *)((char *)workspace + align256(8 * kRedBlocks));
    GW_CUDA(cudaMemsetAsync(ticket, 0, sizeof(unsigned), S(stream)));
    k_norm2<<<gw_count_launch(red_grid_elems(n)), kThreads, 0, S(stream)>>>(v, n, partials, ticket, norm_dev);
    GW_LAUNCHED();
    return GW_OK;
}

extern "C" int gw_apply_increment(const gw_bsr_t *A, const double *delta, double *u_full, void *stream) {
    GW_REQUIRE(A && delta && u_full);
    if (A->n_rows == 0) return GW_OK;
    k_apply_increment<<<gw_count_launch(nblk(A->n_rows, kThreads)), kThreads, 0, S(stream)>>>(A->n_rows, A->nf, A->row2node, delta, u_full);
    GW_LAUNCHED();
    return GW_OK;
}

extern "C" int gw_predict_increment(const gw_bsr_t *A, const uint8_t *free_mask, const double *u_prev, double *u_full,
                                    void *stream) {
    GW_REQUIRE(A && free_mask && u_prev && u_full && u_prev != u_full);
    if (A->n_rows == 0) return GW_OK;
    k_predict_increment<<<gw_count_launch(nblk(A->n_rows, kThreads)), kThreads, 0, S(stream)>>>(
        A->n_rows, A->nf, A->row2node, free_mask, u_prev, u_full);
    GW_LAUNCHED();
    return GW_OK;
}

// ==================================================================== G2P
extern "C" int gw_g2p(const gw_grid_t *grid, const gw_step_t *st, const gw_particles_t *pt, const double *u_new,
                      const double *u_old, void *stream) {
    GW_REQUIRE(grid && st && pt && u_new && u_old);
    if (pt->n == 0) return GW_OK;
    LaunchConst c = make_lc(grid, nullptr, st);
    PtrsP p = make_ptrs(*pt);
    const int b = nblk(pt->n, kThreads);
    // algorithmic bytes, each array once: per particle x and lp in and out,
    // F_new and b_new in, F_old and b_old out, pi and the pore pressure; the
    // two nodal solution vectors once per node
    ProfScope ps(PC_G2P, S(stream), (double)pt->n * 8.0 * (4 * grid->dim + 9 * 4 + 3) +
                                        2.0 * 8.0 * grid->nf * (double)grid->n_nodes);
    switch (grid->kind) {
        case GW_KIND_SOLID2D: k_g2p<GW_KIND_SOLID2D><<<gw_count_launch(b), kThreads, 0, S(stream)>>>(c, p, u_new, u_old); break;
        case GW_KIND_COUPLED2D: k_g2p<GW_KIND_COUPLED2D><<<gw_count_launch(b), kThreads, 0, S(stream)>>>(c, p, u_new, u_old); break;
        case GW_KIND_COUPLED3D: k_g2p<GW_KIND_COUPLED3D><<<gw_count_launch(b), kThreads, 0, S(stream)>>>(c, p, u_new, u_old); break;
        default: return GW_EINVAL;
    }
    GW_LAUNCHED();
    return GW_OK;
}

// ==================================================================== single-point models
extern "C" int gw_return_map(const gw_material_t *mat, int32_t n, const double *e_trial, const double *eps_v_total,
                             const double *pi_old, double *pi_new, double *e_out, double *tau_out,
                             double *dtau_de_out, void *stream) {
    GW_REQUIRE(mat && e_trial && e_out && tau_out);
    if (n == 0) return GW_OK;
    MatConst mc = make_matconst(*mat);
    const double nu = mat->poisson_ratio, E = mat->youngs_modulus;
    const double lam = E * nu / ((1.0 + nu) * (1.0 - 2.0 * nu)), mu = E / (2.0 * (1.0 + nu));
    k_return_map<<<gw_count_launch(nblk(n, kThreads)), kThreads, 0, S(stream)>>>(mc, lam, mu, n, e_trial, eps_v_total, pi_old, pi_new,
                                                                e_out, tau_out, dtau_de_out);
    GW_LAUNCHED();
    return GW_OK;
}


extern "C" int64_t gw_launch_count(void) { return g_launches; }

extern "C" int gw_tune_set(int32_t knob, int32_t value) {
    switch (knob) {
        case GW_TUNE_PARTICLE_BLOCK:
        case GW_TUNE_ADJOINT_BLOCK:  // the particle kernels use up to 255 registers: 256 threads at most
            if (value < 32 || value > 256 || value % 32) return GW_EINVAL;
            break;
        case GW_TUNE_ROW_WARPS:
            if (value < 1 || value > 32) return GW_EINVAL;
            break;
        case GW_TUNE_MG_COARSE:
            if (value < kMgCoarseMin || value > kMgCoarseMax) return GW_EINVAL;
            break;
        case GW_TUNE_MG_ONE_SWEEP:
            if (value < 1 || value > kMgMaxLevels) return GW_EINVAL;
            break;
        case GW_TUNE_MG_SWEEPS:
            if (value < 1 || value > 4) return GW_EINVAL;
            break;
        case GW_TUNE_MG_OMEGA:
            if (value < 10 || value > 100) return GW_EINVAL;
            break;
        case GW_TUNE_GS_CANCEL:
            if (value < 0 || value > 300) return GW_EINVAL;
            break;
        case GW_TUNE_MG_TAIL:
            if (value < 0 || value > (1 << 20)) return GW_EINVAL;
            break;
        case GW_TUNE_MG_BF16:
            if (value < 0 || value > 1) return GW_EINVAL;
            break;
        case GW_TUNE_MG_FINE_SWEEPS:
            if (value < 1 || value > 4) return GW_EINVAL;
            break;
        case GW_TUNE_GMRES_STALL:
            if (value < 0 || value > 100000) return GW_EINVAL;
            break;
        default:
            return GW_EINVAL;
    }
    g_tune[knob] = value;
    return GW_OK;
}

extern "C" int32_t gw_tune_get(int32_t knob) { return (knob >= 0 && knob < GW_TUNE_COUNT) ? g_tune[knob] : -1; }

extern "C" int gw_profile_enable(int32_t on) {
    g_prof_on = on != 0;
    return GW_OK;
}

extern "C" int gw_profile_read(int32_t cls, double *ms_total_host, int64_t *launches_host, double *bytes_host) {
    GW_REQUIRE(ms_total_host && launches_host && bytes_host && cls >= 0 && cls < PC_COUNT);
    // fold pending records
    for (int i = 0; i < g_prof_n; ++i) {
        ProfRec &r = g_prof[i];
        GW_CUDA(cudaEventSynchronize(r.b));
        float ms = 0.f;
        GW_CUDA(cudaEventElapsedTime(&ms, r.a, r.b));
        g_prof_ms[r.cls] += ms;
        g_prof_bytes[r.cls] += r.bytes;
        g_prof_count[r.cls] += 1;
    }
    g_prof_n = 0;
    *ms_total_host = g_prof_ms[cls];
    *launches_host = g_prof_count[cls];
    *bytes_host = g_prof_bytes[cls];
    return GW_OK;
}

extern "C" int gw_profile_reset(void) {
    g_prof_n = 0;  // the event pairs stay in the pool
    for (int c = 0; c < PC_COUNT; ++c) { g_prof_ms[c] = 0.0; g_prof_bytes[c] = 0.0; g_prof_count[c] = 0; }
    return GW_OK;
}

extern "C" int gw_profile_count(void) { return PC_COUNT; }

extern "C" const char *gw_profile_name(int32_t cls) { return (cls >= 0 && cls < PC_COUNT) ? kProfNames[cls] : ""; }
