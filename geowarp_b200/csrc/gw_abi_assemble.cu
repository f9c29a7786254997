// C ABI, residual and element-tangent assembly (declarations and reference
// citations in include/geowarp_b200.h): the deterministic cell-coloured
// assembly of the 2D kinds (gw_assemble_sorted) and the atomic one
// (gw_assemble, used for the 3D kind).
#include "gw_host.cuh"
#include "gw_assemble.cuh"

using namespace gw;
using namespace gwh;

namespace {
template <int KIND, typename VT>
void assemble_per_model(const LaunchConst &c, const PtrsP &p, const int *perm, const uint8_t *fm, const double *un,
                        const double *uo, const PtrsA &a, double *R, double *force, int b, cudaStream_t s) {
    const int pb = g_tune[GW_TUNE_PARTICLE_BLOCK];
    switch (c.mc.model) {
        case GW_MODEL_HENCKY: k_assemble<KIND, true, VT, GW_MODEL_HENCKY><<<gw_count_launch(b), pb, 0, s>>>(c, p, perm, fm, un, uo, a, R, force); break;
        case GW_MODEL_J2: k_assemble<KIND, true, VT, GW_MODEL_J2><<<gw_count_launch(b), pb, 0, s>>>(c, p, perm, fm, un, uo, a, R, force); break;
        case GW_MODEL_NEOHOOKEAN: k_assemble<KIND, true, VT, GW_MODEL_NEOHOOKEAN><<<gw_count_launch(b), pb, 0, s>>>(c, p, perm, fm, un, uo, a, R, force); break;
        case GW_MODEL_LINEAR: k_assemble<KIND, true, VT, GW_MODEL_LINEAR><<<gw_count_launch(b), pb, 0, s>>>(c, p, perm, fm, un, uo, a, R, force); break;
        case GW_MODEL_DP: k_assemble<KIND, true, VT, GW_MODEL_DP><<<gw_count_launch(b), pb, 0, s>>>(c, p, perm, fm, un, uo, a, R, force); break;
        default: k_assemble<KIND, true, VT><<<gw_count_launch(b), pb, 0, s>>>(c, p, perm, fm, un, uo, a, R, force); break;
    }
}

template <int KIND>
int launch_assemble(const LaunchConst &c, const PtrsP &p, const int *perm, const uint8_t *fm, const double *un,
                    const double *uo, const gw_bsr_t *A, int prec, double *R, double *force, const PtrsA &a,
                    cudaStream_t s) {
    const int pb = g_tune[GW_TUNE_PARTICLE_BLOCK];
    const int b = nblk(p.n, pb);
    if (p.n > 0) {
        const int D = KindTraits<KIND>::D, NF = KindTraits<KIND>::NF, NS = KindTraits<KIND>::NS;
        // algorithmic bytes, each array once: particle state in (x, lp, F_old,
        // b_old, E) and out (F_new, b_new, sigma), the grid vectors (u_new, u_old,
        // R) and the matrix values
        (void)NS;
        const double per_p = 8.0 * (2 * D + 9 + 9 + 1) + 8.0 * 27;
        const double grid = 8.0 * 3 * (double)A->n_rows * NF;
        const bool want_K = A->vals != nullptr;
        const double mat = want_K ? (double)A->nnzb * NF * NF * (prec == GW_PREC_F64 ? 8 : 4) : 0.0;
        ProfScope ps(PC_ASSEMBLE, s, per_p * p.n + grid + mat);
        if (!want_K) {
            k_assemble<KIND, false, double><<<gw_count_launch(b), pb, 0, s>>>(c, p, perm, fm, un, uo, a, R, force);
        } else if constexpr (KIND == GW_KIND_SOLID2D) {
            // the 2D solid tangent kernel is instantiated per material, so each
            // carries only its own constitutive code (fewer registers and spills)
            if (prec == GW_PREC_F64) assemble_per_model<KIND, double>(c, p, perm, fm, un, uo, a, R, force, b, s);
            else assemble_per_model<KIND, float>(c, p, perm, fm, un, uo, a, R, force, b, s);
        } else {
            if (prec == GW_PREC_F64) k_assemble<KIND, true, double><<<gw_count_launch(b), pb, 0, s>>>(c, p, perm, fm, un, uo, a, R, force);
            else k_assemble<KIND, true, float><<<gw_count_launch(b), pb, 0, s>>>(c, p, perm, fm, un, uo, a, R, force);
        }
        GW_LAUNCHED();
    }
    if (A->vals && A->n_rows > 0) {
        const int D = KindTraits<KIND>::D;
        if (prec == GW_PREC_F64) k_identity_dirichlet<D, double><<<gw_count_launch(nblk(A->n_rows, kThreads)), kThreads, 0, s>>>(a, fm);
        else k_identity_dirichlet<D, float><<<gw_count_launch(nblk(A->n_rows, kThreads)), kThreads, 0, s>>>(a, fm);
        GW_LAUNCHED();
    }
    return GW_OK;
}
}  // namespace

extern "C" int gw_assemble(const gw_grid_t *grid, const gw_material_t *mat, const gw_step_t *st,
                           const gw_particles_t *pt, const int32_t *perm, const uint8_t *free_mask,
                           const double *u_new, const double *u_old, const gw_bsr_t *A, int32_t prec, double *R_rows,
                           double *force, void *stream) {
    GW_REQUIRE(grid && mat && st && pt && perm && free_mask && u_new && u_old && R_rows);
    // the row map is needed for the residual even without a matrix
    GW_REQUIRE(A && A->node2row && (A->n_rows == 0 || A->row2node));
    GW_REQUIRE(mat->model >= 0 && mat->model <= GW_MODEL_NORSAND);
    cudaStream_t s = S(stream);
    LaunchConst c = make_lc(grid, mat, st);
    PtrsP p = make_ptrs(*pt);
    PtrsA a = make_ptrs(*A);
    if (A->vals) {
        GW_REQUIRE(A->row_ptr && A->cols && A->stencil);
        const size_t vb = (prec == GW_PREC_F64 ? 8 : 4) * (size_t)A->nnzb * A->nf * A->nf;
        GW_CUDA(cudaMemsetAsync(A->vals, 0, vb, s));
    }
    GW_CUDA(cudaMemsetAsync(R_rows, 0, sizeof(double) * (size_t)A->n_rows * A->nf, s));
    switch (grid->kind) {
        case GW_KIND_SOLID2D: return launch_assemble<GW_KIND_SOLID2D>(c, p, perm, free_mask, u_new, u_old, A, prec, R_rows, force, a, s);
        case GW_KIND_COUPLED2D: return launch_assemble<GW_KIND_COUPLED2D>(c, p, perm, free_mask, u_new, u_old, A, prec, R_rows, force, a, s);
        case GW_KIND_COUPLED3D: return launch_assemble<GW_KIND_COUPLED3D>(c, p, perm, free_mask, u_new, u_old, A, prec, R_rows, force, a, s);
        default: return GW_EINVAL;
    }
}

// ==================================================================== deterministic (cell-coloured) assembly
namespace {
template <int KIND, typename VT>
int64_t q_record_bytes() { return QRecord<KIND, VT>::BYTES; }

int64_t record_bytes(int kind, int prec) {
    switch (kind) {
        case GW_KIND_SOLID2D: return prec == GW_PREC_F64 ? q_record_bytes<GW_KIND_SOLID2D, double>() : q_record_bytes<GW_KIND_SOLID2D, float>();
        case GW_KIND_COUPLED2D: return prec == GW_PREC_F64 ? q_record_bytes<GW_KIND_COUPLED2D, double>() : q_record_bytes<GW_KIND_COUPLED2D, float>();
        default: return 0;
    }
}

template <int KIND, bool WANT_K, typename VT>
void launch_particle_q(const LaunchConst &c, const PtrsP &p, const int *perm, const double *un, const double *uo,
                       unsigned char *scratch, double *force, cudaStream_t s) {
    const int pb = g_tune[GW_TUNE_PARTICLE_BLOCK];
    const int b = nblk(p.n, pb);
    if constexpr (KIND == GW_KIND_SOLID2D && WANT_K) {
        // one instantiation per material: each carries only its own constitutive code
        switch (c.mc.model) {
            case GW_MODEL_HENCKY: k_particle_q<KIND, WANT_K, VT, GW_MODEL_HENCKY><<<gw_count_launch(b), pb, 0, s>>>(c, p, perm, un, uo, scratch, force); return;
            case GW_MODEL_J2: k_particle_q<KIND, WANT_K, VT, GW_MODEL_J2><<<gw_count_launch(b), pb, 0, s>>>(c, p, perm, un, uo, scratch, force); return;
            case GW_MODEL_NEOHOOKEAN: k_particle_q<KIND, WANT_K, VT, GW_MODEL_NEOHOOKEAN><<<gw_count_launch(b), pb, 0, s>>>(c, p, perm, un, uo, scratch, force); return;
            case GW_MODEL_LINEAR: k_particle_q<KIND, WANT_K, VT, GW_MODEL_LINEAR><<<gw_count_launch(b), pb, 0, s>>>(c, p, perm, un, uo, scratch, force); return;
            case GW_MODEL_DP: k_particle_q<KIND, WANT_K, VT, GW_MODEL_DP><<<gw_count_launch(b), pb, 0, s>>>(c, p, perm, un, uo, scratch, force); return;
            default: break;
        }
    }
    k_particle_q<KIND, WANT_K, VT><<<gw_count_launch(b), pb, 0, s>>>(c, p, perm, un, uo, scratch, force);
}

template <int KIND, bool WANT_K, typename VT>
int assemble_sorted(const LaunchConst &c, const PtrsP &p, const int *perm, const int *keys, const uint8_t *fm,
                    const double *un, const double *uo, const gw_bsr_t *A, double *R, double *force, const PtrsA &a,
                    char *ws, int64_t ws_bytes, cudaStream_t s) {
    const int ncx = c.g.n_grid[0], ncy = c.g.n_grid[1], nc = ncx * ncy;
    // the records written below must fit the caller's workspace (record size
    // of this instantiation, not of another precision)
    const int64_t need = 2 * align256(4 * (int64_t)nc) + (int64_t)QRecord<KIND, VT>::BYTES * p.n;
    if (need > ws_bytes) {
        snprintf(g_msg, sizeof(g_msg), "gw_assemble_sorted: workspace of %lld bytes, %lld needed",
                 (long long)ws_bytes, (long long)need);
        return GW_EINVAL;
    }
    int *cstart = (int *)ws;
    int *cend = (int *)(ws + align256(4 * (int64_t)nc));
    unsigned char *scratch = (unsigned char *)(ws + 2 * align256(4 * (int64_t)nc));
    const int D = KindTraits<KIND>::D, NF = KindTraits<KIND>::NF;
    // algorithmic bytes, each array once: particle state in (x, lp, F_old, b_old,
    // E) and out (F_new, b_new, sigma), the scratch records written and read
    // back, the grid vectors (u_new, u_old, R) and the matrix values
    const double per_p = 8.0 * (2 * D + 9 + 9 + 1) + 8.0 * 27 + 2.0 * QRecord<KIND, VT>::BYTES;
    const double grid = 8.0 * 3 * (double)A->n_rows * NF;
    const double mat = WANT_K ? (double)A->nnzb * NF * NF * sizeof(VT) : 0.0;
    ProfScope ps(PC_ASSEMBLE, s, per_p * p.n + grid + mat);
    GW_CUDA(cudaMemsetAsync(ws, 0, 2 * align256(4 * (int64_t)nc), s));
    k_cell_ranges<<<gw_count_launch(nblk(p.n, kThreads)), kThreads, 0, s>>>(keys, p.n, nc, cstart, cend);
    GW_LAUNCHED();
    launch_particle_q<KIND, WANT_K, VT>(c, p, perm, un, uo, scratch, force, s);
    GW_LAUNCHED();
    // nine colour phases in a fixed order
    for (int ky = 0; ky < 3; ++ky)
        for (int kx = 0; kx < 3; ++kx) {
            const int n3 = ((ncx - kx + 2) / 3) * ((ncy - ky + 2) / 3);
            if (n3 <= 0) continue;
            k_cell_scatter<KIND, WANT_K, VT><<<gw_count_launch(nblk(n3, kScatterWarps)), 32 * kScatterWarps, 0, s>>>(
                c, kx, ky, cstart, cend, scratch, fm, a, R);
        }
    GW_LAUNCHED();
    return GW_OK;
}

template <int KIND>
int assemble_sorted_kind(const LaunchConst &c, const PtrsP &p, const int *perm, const int *keys, const uint8_t *fm,
                         const double *un, const double *uo, const gw_bsr_t *A, int prec, double *R, double *force,
                         const PtrsA &a, char *ws, int64_t ws_bytes, cudaStream_t s) {
    int rc;
    if (p.n > 0) {
        // residual only (A->vals NULL) keeps the record layout of prec: the
        // workspace was sized for it (gw_assemble_workspace_bytes)
        const bool f64 = prec == GW_PREC_F64;
        if (!A->vals)
            rc = f64 ? assemble_sorted<KIND, false, double>(c, p, perm, keys, fm, un, uo, A, R, force, a, ws, ws_bytes, s)
                     : assemble_sorted<KIND, false, float>(c, p, perm, keys, fm, un, uo, A, R, force, a, ws, ws_bytes, s);
        else
            rc = f64 ? assemble_sorted<KIND, true, double>(c, p, perm, keys, fm, un, uo, A, R, force, a, ws, ws_bytes, s)
                     : assemble_sorted<KIND, true, float>(c, p, perm, keys, fm, un, uo, A, R, force, a, ws, ws_bytes, s);
        if (rc) return rc;
    }
    if (A->vals && A->n_rows > 0) {
        if (prec == GW_PREC_F64) k_identity_dirichlet<2, double><<<gw_count_launch(nblk(A->n_rows, kThreads)), kThreads, 0, s>>>(a, fm);
        else k_identity_dirichlet<2, float><<<gw_count_launch(nblk(A->n_rows, kThreads)), kThreads, 0, s>>>(a, fm);
        GW_LAUNCHED();
    }
    return GW_OK;
}
}  // namespace

extern "C" int64_t gw_assemble_workspace_bytes(const gw_grid_t *grid, int32_t n_particles, int32_t prec) {
    if (!grid || n_particles < 0) return -1;
    if (grid->dim != 2) return 0;  // the 3D kind assembles with atomics and needs no workspace
    const int64_t nc = (int64_t)grid->n_grid[0] * grid->n_grid[1];
    return 2 * align256(4 * nc) + align256(record_bytes(grid->kind, prec) * (int64_t)n_particles) + 256;
}

extern "C" int gw_assemble_sorted(const gw_grid_t *grid, const gw_material_t *mat, const gw_step_t *st,
                                  const gw_particles_t *pt, const int32_t *perm, const int32_t *keys,
                                  const uint8_t *free_mask, const double *u_new, const double *u_old, const gw_bsr_t *A,
                                  int32_t prec, double *R_rows, double *force, void *workspace, int64_t workspace_bytes,
                                  void *stream) {
    if (grid && grid->dim == 3)  // no colouring in 3D: the atomic assembly
        return gw_assemble(grid, mat, st, pt, perm, free_mask, u_new, u_old, A, prec, R_rows, force, stream);
    GW_REQUIRE(grid && mat && st && pt && perm && keys && free_mask && u_new && u_old && R_rows && workspace);
    GW_REQUIRE(grid->kind == GW_KIND_SOLID2D || grid->kind == GW_KIND_COUPLED2D);
    GW_REQUIRE(A && A->node2row && (A->n_rows == 0 || A->row2node));
    GW_REQUIRE(mat->model >= 0 && mat->model <= GW_MODEL_NORSAND);
    GW_REQUIRE(((uintptr_t)workspace & 255u) == 0);
    const int64_t need = gw_assemble_workspace_bytes(grid, pt->n, prec);
    if (workspace_bytes < need) {
        snprintf(g_msg, sizeof(g_msg), "gw_assemble_sorted: workspace of %lld bytes, %lld needed",
                 (long long)workspace_bytes, (long long)need);
        return GW_EINVAL;
    }
    cudaStream_t s = S(stream);
    LaunchConst c = make_lc(grid, mat, st);
    PtrsP p = make_ptrs(*pt);
    PtrsA a = make_ptrs(*A);
    if (A->vals) {
        GW_REQUIRE(A->row_ptr && A->cols && A->stencil);
        const size_t vb = (prec == GW_PREC_F64 ? 8 : 4) * (size_t)A->nnzb * A->nf * A->nf;
        GW_CUDA(cudaMemsetAsync(A->vals, 0, vb, s));
    }
    GW_CUDA(cudaMemsetAsync(R_rows, 0, sizeof(double) * (size_t)A->n_rows * A->nf, s));
    char *ws = (char *)workspace;
    if (grid->kind == GW_KIND_SOLID2D)
        return assemble_sorted_kind<GW_KIND_SOLID2D>(c, p, perm, keys, free_mask, u_new, u_old, A, prec, R_rows, force, a, ws, workspace_bytes, s);
    return assemble_sorted_kind<GW_KIND_COUPLED2D>(c, p, perm, keys, free_mask, u_new, u_old, A, prec, R_rows, force, a, ws, workspace_bytes, s);
}
