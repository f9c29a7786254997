// C ABI, residual and element-tangent assembly (declaration and reference
// citation in include/geowarp_b200.h).
#include "gw_host.cuh"

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
