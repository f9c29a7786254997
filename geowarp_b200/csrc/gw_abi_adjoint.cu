// C ABI, adjoint of the 2D solid load step: Jacobian transpose, adjoint G2P
// and adjoint P2G (declarations and reference citations in
// include/geowarp_b200.h).
#include "gw_host.cuh"
#include "gw_adjoint.cuh"

using namespace gw;
using namespace gwh;

namespace {
AdjState make_adj(const gw_adjoint_t &a) {
    AdjState s;
    s.x = a.x; s.lp = a.lp; s.F = a.F; s.b = a.b; s.E = a.E;
    return s;
}
}  // namespace

extern "C" int gw_bsr_transpose(const gw_grid_t *grid, const gw_bsr_t *A, int32_t prec, void *AT_vals, void *stream) {
    GW_REQUIRE(grid && A && AT_vals);
    if (A->n_rows == 0) return GW_OK;
    PtrsA a = make_ptrs(*A);
    cudaStream_t s = S(stream);
    const size_t vb = (prec == GW_PREC_F64 ? 8 : 4) * (size_t)A->nnzb * A->nf * A->nf;
    GW_CUDA(cudaMemsetAsync(AT_vals, 0, vb, s));
    const int b = nblk(A->n_rows, kThreads / 32);
    if (grid->dim == 2) {
        if (prec == GW_PREC_F64) k_bsr_transpose<2, double><<<gw_count_launch(b), kThreads, 0, s>>>(*grid, a, (double *)AT_vals);
        else k_bsr_transpose<2, float><<<gw_count_launch(b), kThreads, 0, s>>>(*grid, a, (float *)AT_vals);
    } else {
        if (prec == GW_PREC_F64) k_bsr_transpose<3, double><<<gw_count_launch(b), kThreads, 0, s>>>(*grid, a, (double *)AT_vals);
        else k_bsr_transpose<3, float><<<gw_count_launch(b), kThreads, 0, s>>>(*grid, a, (float *)AT_vals);
    }
    GW_LAUNCHED();
    return GW_OK;
}

extern "C" int gw_adjoint_g2p(const gw_grid_t *grid, const gw_material_t *mat, const gw_step_t *st,
                              const gw_particles_t *pt, const double *u_new, const double *u_old,
                              const uint8_t *free_mask, const gw_bsr_t *A, const gw_adjoint_t *seed_in,
                              gw_adjoint_t *q_out, double *ubar_rows, void *stream) {
    GW_REQUIRE(grid && mat && st && pt && u_new && u_old && free_mask && A && seed_in && q_out && ubar_rows);
    if (grid->kind != GW_KIND_SOLID2D) return GW_EMODEL;
    if (mat->model == GW_MODEL_NORSAND) return GW_EMODEL;
    cudaStream_t s = S(stream);
    GW_CUDA(cudaMemsetAsync(ubar_rows, 0, sizeof(double) * (size_t)A->n_rows * A->nf, s));
    if (pt->n == 0) return GW_OK;
    LaunchConst c = make_lc(grid, mat, st);
    c.mc.tip_tangent = 0.0;  // exact derivatives of the converged state
    ProfScope ps(PC_ADJ_G2P, s, (double)pt->n * 8.0 * (2 + 2 + 9 + 9 + 1 + 18 + 23 + 2 * 9 * 2));
    const int ab = g_tune[GW_TUNE_ADJOINT_BLOCK];
    const dim3 grd(gw_count_launch(nblk(pt->n, ab))), blk(ab);
    const PtrsP pp = make_ptrs(*pt);
    const PtrsA pa = make_ptrs(*A);
    const AdjState si = make_adj(*seed_in), qo = make_adj(*q_out);
    switch (mat->model) {  // one instantiation per material: see solid2d_vjp
        case GW_MODEL_HENCKY: k_adjoint_g2p<GW_MODEL_HENCKY><<<grd, blk, 0, s>>>(c, pp, u_new, u_old, free_mask, pa, si, qo, ubar_rows); break;
        case GW_MODEL_J2: k_adjoint_g2p<GW_MODEL_J2><<<grd, blk, 0, s>>>(c, pp, u_new, u_old, free_mask, pa, si, qo, ubar_rows); break;
        case GW_MODEL_DP: k_adjoint_g2p<GW_MODEL_DP><<<grd, blk, 0, s>>>(c, pp, u_new, u_old, free_mask, pa, si, qo, ubar_rows); break;
        case GW_MODEL_NEOHOOKEAN: k_adjoint_g2p<GW_MODEL_NEOHOOKEAN><<<grd, blk, 0, s>>>(c, pp, u_new, u_old, free_mask, pa, si, qo, ubar_rows); break;
        case GW_MODEL_LINEAR: k_adjoint_g2p<GW_MODEL_LINEAR><<<grd, blk, 0, s>>>(c, pp, u_new, u_old, free_mask, pa, si, qo, ubar_rows); break;
        default: k_adjoint_g2p<-1><<<grd, blk, 0, s>>>(c, pp, u_new, u_old, free_mask, pa, si, qo, ubar_rows); break;
    }
    GW_LAUNCHED();
    return GW_OK;
}

extern "C" int gw_adjoint_residual(const gw_grid_t *grid, const gw_material_t *mat, const gw_step_t *st,
                                   const gw_particles_t *pt, const double *u_new, const double *u_old,
                                   const uint8_t *free_mask, const gw_bsr_t *A, const double *lambda_rows,
                                   gw_adjoint_t *q_out, void *stream) {
    GW_REQUIRE(grid && mat && st && pt && u_new && u_old && free_mask && A && lambda_rows && q_out);
    if (grid->kind != GW_KIND_SOLID2D) return GW_EMODEL;
    if (mat->model == GW_MODEL_NORSAND) return GW_EMODEL;
    if (pt->n == 0) return GW_OK;
    LaunchConst c = make_lc(grid, mat, st);
    c.mc.tip_tangent = 0.0;  // exact derivatives of the converged residual
    ProfScope ps(PC_ADJ_RES, S(stream), (double)pt->n * 8.0 * (2 + 2 + 9 + 9 + 1 + 23 * 2 + 2 * 9 * 2 + 9 * 2));
    const int ab = g_tune[GW_TUNE_ADJOINT_BLOCK];
    const dim3 grd(gw_count_launch(nblk(pt->n, ab))), blk(ab);
    const PtrsP pp = make_ptrs(*pt);
    const PtrsA pa = make_ptrs(*A);
    const AdjState qo = make_adj(*q_out);
    cudaStream_t s = S(stream);
    switch (mat->model) {  // one instantiation per material: see solid2d_vjp
        case GW_MODEL_HENCKY: k_adjoint_residual<GW_MODEL_HENCKY><<<grd, blk, 0, s>>>(c, pp, u_new, u_old, free_mask, pa, lambda_rows, qo); break;
        case GW_MODEL_J2: k_adjoint_residual<GW_MODEL_J2><<<grd, blk, 0, s>>>(c, pp, u_new, u_old, free_mask, pa, lambda_rows, qo); break;
        case GW_MODEL_DP: k_adjoint_residual<GW_MODEL_DP><<<grd, blk, 0, s>>>(c, pp, u_new, u_old, free_mask, pa, lambda_rows, qo); break;
        case GW_MODEL_NEOHOOKEAN: k_adjoint_residual<GW_MODEL_NEOHOOKEAN><<<grd, blk, 0, s>>>(c, pp, u_new, u_old, free_mask, pa, lambda_rows, qo); break;
        case GW_MODEL_LINEAR: k_adjoint_residual<GW_MODEL_LINEAR><<<grd, blk, 0, s>>>(c, pp, u_new, u_old, free_mask, pa, lambda_rows, qo); break;
        default: k_adjoint_residual<-1><<<grd, blk, 0, s>>>(c, pp, u_new, u_old, free_mask, pa, lambda_rows, qo); break;
    }
    GW_LAUNCHED();
    return GW_OK;
}

// ==================================================================== kernel timing