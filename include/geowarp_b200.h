/*
 * geowarp_b200 — C ABI of the B200-native implicit cpGIMP engine.
 *
 * The reference (choo-group/GeoWarp) has no FFI: its boundary is the Python
 * solver-class API (solvers/quasi_static_solver_2d.py:45-258,
 * solvers/quasi_static_coupled_solver_2d.py:45-313,
 * solvers/quasi_static_coupled_solver_3d.py:56-420) over Warp kernels in
 * mpm/mpm_utils.py, mpm/gimp.py and solvers/sparse_differentiation.py.  Each
 * entry point below replaces one of those Warp launches (or Warp/SciPy library
 * calls) and is cited beside its declaration.  The Python solver classes in
 * geowarp_b200/solvers bind these symbols through ctypes.
 *
 * Conventions
 *  - All pointers are device pointers unless the name ends in _host.
 *  - Memory is owned by the caller; no entry point allocates, except the
 *    caller-sized workspaces passed in explicitly.
 *  - Calls are ordered on the given stream and do not synchronise, except
 *    gw_bsr_krylov_solve (which polls its residual on the host) and the
 *    *_count entry points that return a size.
 *  - Return value: 0 on success, a negative GW_E* code otherwise.
 *  - Particle arrays are indexed by the user's particle id (the reference's
 *    order).  Grid vectors are node-interleaved: value (node, field) at
 *    node*nf + field.  Boundary flags are field-major like the reference's
 *    boundary_flag_array: flag (field, node) at field*n_nodes + node.
 */
#ifndef GEOWARP_B200_H
#define GEOWARP_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------ status codes */
#define GW_OK 0
#define GW_EINVAL -1        /* bad sizes or null pointers                        */
#define GW_ECUDA -2         /* a CUDA launch or API call failed                  */
#define GW_ENOCONV -3       /* Krylov iteration cap (or GMRES stagnation stop)
                               reached before the tolerance                      */
#define GW_EBREAKDOWN -4    /* Krylov breakdown (rho or omega underflow)         */
#define GW_ENAN -5          /* non-finite value detected                         */
#define GW_ERANGE -6        /* a device index guard failed (see gw_guard_read)   */
#define GW_EMODEL -7        /* unknown material model for this solver kind       */

/* ------------------------------------------------------------ enums */
#define GW_KIND_SOLID2D 0   /* quasi_static_solver_2d: unknowns (ux, uy)          */
#define GW_KIND_COUPLED2D 1 /* quasi_static_coupled_solver_2d: (ux, uy, p)        */
#define GW_KIND_COUPLED3D 2 /* quasi_static_coupled_solver_3d: (ux, uy, uz, p)    */

#define GW_MODEL_HENCKY 0   /* 'Hencky elasticity' (mpm/mpm_utils.py:537-542)   */
#define GW_MODEL_J2 1       /* 'J2' (materials/plasticity.py:8-37)                */
#define GW_MODEL_NEOHOOKEAN 2 /* 'Neo-Hookean' (mpm/mpm_utils.py:914-916, 1204-1208) */
#define GW_MODEL_LINEAR 3   /* small-strain linear elasticity (extension)         */
#define GW_MODEL_DP 4       /* Drucker-Prager (triaxial_DruckerPrager.py:119-412) */
#define GW_MODEL_NORSAND 5  /* NorSand (triaxial_NorSand.py:155-400)              */

#define GW_PREC_F64 0       /* plain FP64 everywhere                               */
#define GW_PREC_F32 1       /* FP32 values / FP32 accumulation                     */

#define GW_PRECOND_DIAG 0   /* scalar Jacobi, the reference's ptype='diag'         */
#define GW_PRECOND_BLOCK 1  /* node-block Jacobi (nf x nf inverse)                 */

#define GW_KRYLOV_BICGSTAB 0
#define GW_KRYLOV_CG 1
#define GW_KRYLOV_GMRES 2

/* ------------------------------------------------------------ structs */
typedef struct gw_grid {
    int32_t dim;            /* 2 or 3                                             */
    int32_t kind;           /* GW_KIND_*                                          */
    int32_t nf;             /* unknowns per node: 2, 3 or 4                       */
    int32_t n_grid[3];      /* cells per axis (n_grid_z = 0 in 2D)                */
    int32_t n_nodes;        /* prod(n_grid + 1)                                   */
    int32_t pad0;
    double h[3];            /* cell sizes seen by the shape functions (2D: dx,dx) */
    double inv_h[3];
    double h_nodes[3];      /* cell sizes for nodal positions (pressure BC)       */
    double domain_min[3];   /* lp clipping box (mpm/gimp.py:449-459)              */
    double domain_max[3];
} gw_grid_t;

typedef struct gw_material {
    int32_t model;          /* GW_MODEL_*                                         */
    int32_t dp_tension_cutoff; /* DP: 1 keeps the trial state when P_trial >= 0, as
                                  the reference does (triaxial_DruckerPrager.py:347-349);
                                  0 applies the cone return there too (extension) */
    double youngs_modulus;  /* used when the per-particle E pointer is null       */
    double poisson_ratio;
    double kappa;           /* J2 yield radius                                    */
    double friction_angle;  /* DP, degrees                                        */
    double dilation_angle;  /* DP, degrees                                        */
    double cohesion;        /* DP                                                 */
    double shape_factor;    /* DP hyperbolic smoothing                            */
    /* NorSand (triaxial_NorSand.py:13-43) */
    double ns_kappa, ns_tilde_lambda, ns_M, ns_N, ns_beta, ns_vc0, ns_p0, ns_v0, ns_h;
    double ns_shear_modulus, ns_eps_v0;
    double dp_tip_tangent;  /* DP with dp_tension_cutoff 0 (extension): fraction of the
                               elastic tangent that particles returned to the cone tip
                               contribute to the Jacobian (their exact tangent is zero;
                               0 = exact).  The residual is not changed. */
} gw_material_t;

typedef struct gw_step {
    double current_step;    /* load ramp (step+1)/total_steps                     */
    double total_steps;
    double gravity_mag;
    double point_load[3];
    double traction[3];
    double p_vol, p_rho, PPD;
    double dt, phi_initial, mobility;   /* u-p only                               */
    double lp0;             /* GIMP_lp_initial                                    */
    int32_t has_footing;    /* penalty footing (mpm/mpm_utils.py:1234-1248)       */
    int32_t footing_stable; /* 0: the reference's residual k (z_new - h), a repulsive
                               spring (negative stiffness); 1: k (h - z_new),
                               attractive (extension, for the 2D strip footing) */
    double footing_min[2], footing_max[2];
    double footing_initial_height, footing_incr_disp, penalty_factor;
    int32_t gravity_full;   /* 0: gravity ramped by (step+1)/total_steps as in the
                               reference; 1: full gravity in every load step (extension,
                               for soil that starts from a geostatic stress state) */
    int32_t mobility_law;   /* u-p: 0 constant mobility (the solver classes); 1 the
                               J-dependent mobility of Uzuoka & Borja (2012) Eq. 86,
                               k(J) = k0 (2 mu + lam) J / (mu (1 + J^-2) + (1 - ln J) lam J^-2)
                               (problems/consolidation/large_consolidation_cpGIMP_
                               everything_in_one_script.py:330-338, 740) */
} gw_step_t;

/* Particle state, user order.  x, lp: [N*dim]; F*, b*, sigma: [N*9] row-major
 * 3x3; pressure, pi_*: [N]; flags: uint8 [N]; E: [N] or NULL. */
typedef struct gw_particles {
    int32_t n;
    int32_t pad0;
    double *x, *x0, *lp;
    double *F_old, *F_new, *b_old, *b_new, *sigma;
    double *pressure, *pi_old, *pi_new;
    const uint8_t *ext_flag, *trac_flag, *pbc_flag;
    const double *E;
} gw_particles_t;

/* Block-CSR over active nodes.  Block (r, j) is nf x nf, row-major, at
 * vals[(row_ptr[r] + j)*nf*nf].  cols[] are active-row indices.  With nf = 2
 * or 4 the SpMV and Krylov entry points gather blocks and vectors with
 * 16-byte loads: vals and the FP64 vectors passed to them must be 16-byte
 * aligned (GW_EINVAL otherwise). */
typedef struct gw_bsr {
    int32_t n_rows;
    int32_t nf;
    int32_t nnzb;
    int32_t mask_words;     /* 1 (2D: 5x5 stencil) or 4 (3D: 5x5x5 stencil)       */
    const int32_t *row_ptr; /* [n_rows+1]                                         */
    const int32_t *cols;    /* [nnzb]                                             */
    const int32_t *row2node;/* [n_rows]                                           */
    const int32_t *node2row;/* [n_nodes], -1 for inactive nodes                   */
    const uint32_t *stencil;/* [n_nodes*mask_words] coupled-offset bitmask        */
    void *vals;             /* double or float per precision                      */
} gw_bsr_t;

/* ------------------------------------------------------------ queries */
int gw_version(void);
const char *gw_status_string(int code);
/* Device-side error flag written by kernels (range / NaN); read & clear. */
int gw_read_device_status(int32_t *flag_host, void *stream);
/* Index guards (no counterpart in the reference, whose Warp kernels bounds-check
 * in debug mode only): indices the kernels derive from a column array, a
 * stencil, a coarse transfer list or a Krylov counter, and row-map lookups
 * wherever the kernel knows the node count, are checked before use (the
 * matrix-only kernels -- gw_apply_increment, gw_predict_increment, the
 * preconditioner set-ups -- trust the fine rows' row2node of
 * gw_compact_rows); a failed check skips the access and records the first
 * failing site and value.  The Krylov and multigrid entry points return GW_ERANGE when one
 * fired; gw_guard_read reads and clears the record (site 0: none). */
int gw_guard_read(int32_t *site, int64_t *value, void *stream);
const char *gw_guard_site_name(int32_t site);

/* ------------------------------------------------------------ cell sort
 * Replaces nothing in the reference (which never reorders particles): the
 * cell key is the lower-corner cell of mpm/gimp.py:33-36 and the sort is a
 * stable LSD radix sort, so the order is a deterministic function of keys.
 * keys_out[N], perm_out[N]: perm_out lists user particle ids by (cell, id).
 * workspace: gw_sort_workspace_bytes(n) bytes. */
int64_t gw_sort_workspace_bytes(int32_t n);
int gw_cell_sort(const gw_grid_t *grid, const gw_particles_t *pt, int32_t *keys_out, int32_t *perm_out,
                 void *workspace, void *stream);

/* ------------------------------------------------------------ P2G activation
 * Replaces P2G_2d (mpm/mpm_utils.py:83-136), the activation and pressure-BC
 * parts of P2G_coupled_2d (:138-235) and P2G_coupled_3d (:259-352).
 * node_active[n_nodes] (uint8) and cell_span[n_cells] (uint32 bitmask of
 * per-axis 3-node spans | 0x80 occupied) are OR-accumulated: zero them first.
 * boundary[nf*n_nodes] gets pressure Dirichlet flags for u-p kinds. */
int gw_p2g_activate(const gw_grid_t *grid, const gw_particles_t *pt, const int32_t *perm, uint8_t *node_active,
                    uint32_t *cell_span, uint8_t *boundary, void *stream);

/* Nodes inside the span support of an occupied cell (touched[n_nodes], uint8;
 * zero it first): the row set of the consistent-mass system, i.e. every node
 * the reference's 81/729 mass triplets per particle can reach with a nonzero
 * weight (mpm/mpm_utils.py:237-257, 354-383). */
int gw_touched_nodes(const gw_grid_t *grid, const uint32_t *cell_span, uint8_t *touched, void *stream);

/* Compact active nodes: node2row[n_nodes], row2node[n_nodes] (first n_rows
 * valid), n_rows_host.  Also builds free_mask[n_nodes] (bit f set when DOF
 * (node, f) is active and not a Dirichlet DOF).  Synchronises (returns a size). */
int gw_compact_rows(const gw_grid_t *grid, const uint8_t *node_active, const uint8_t *boundary, int32_t *node2row,
                    int32_t *row2node, uint8_t *free_mask, int32_t *n_rows_host, void *workspace, void *stream);
int64_t gw_scan_workspace_bytes(int32_t n);

/* ------------------------------------------------------------ pattern
 * Replaces the fixed 25/125-slot COO layout of
 * solvers/sparse_differentiation.py:213-401: builds, once per load step, the
 * block-CSR pattern of node pairs that share a particle's support.
 * stencil[n_nodes*mask_words]; row_ptr[n_rows+1]; nnzb_host; then
 * gw_pattern_fill writes cols[nnzb]. */
int gw_pattern_count(const gw_grid_t *grid, const uint32_t *cell_span, const int32_t *node2row, const int32_t *row2node,
                     int32_t n_rows, uint32_t *stencil, int32_t *row_ptr, int32_t *nnzb_host, void *workspace,
                     void *stream);
int gw_pattern_fill(const gw_grid_t *grid, const gw_bsr_t *A, int32_t *cols, void *stream);

/* ------------------------------------------------------------ consistent mass
 * Replaces the consistent-mass triplets of P2G_coupled_2d (mpm_utils.py:237-257)
 * and P2G_coupled_3d (:354-383) plus the host pyamg / Warp BiCGSTAB solve
 * (solvers/quasi_static_coupled_solver_2d.py:287-300,
 *  solvers/quasi_static_coupled_solver_3d.py:409-417): assembles the scalar
 * block-CSR mass matrix M (same pattern, nf = 1, FP64) over all nodes touched
 * by particle supports (mass_node2row) and rhs_b. */
int gw_mass_assemble(const gw_grid_t *grid, const gw_particles_t *pt, const int32_t *perm, const gw_step_t *st,
                     const gw_bsr_t *M, double *rhs, void *stream);
/* Lumped alternative to the consistent-mass solve: p_i = b_i / sum_j M_ij,
 * the P2G_solver_lumped kernel of
 * problems/consolidation/large_consolidation_cpGIMP_everything_in_one_script.py:292-310
 * (the row sum of M is its lumped nodal mass sum_p N_i m_p). */
int gw_mass_lumped_solve(const gw_bsr_t *M, const double *rhs, double *x, void *stream);
/* Writes the projected nodal pressure into the p field of u_old and u_new for
 * non-Dirichlet nodes (and, in 3D, active nodes): P2G_set_nodal_solution(_3d),
 * mpm/mpm_utils.py:387-414. */
int gw_set_nodal_pressure(const gw_grid_t *grid, const int32_t *mass_row2node, int32_t n_mass_rows, const double *p_hat,
                          const uint8_t *boundary, const uint8_t *node_active, double *u_old, double *u_new,
                          void *stream);

/* ------------------------------------------------------------ residual + Jacobian
 * Replaces assemble_residual_2d_hencky / _J2 (mpm/mpm_utils.py:416-780),
 * assemble_residual_coupled_2d_neohookean (:782-1017),
 * assemble_residual_coupled_3d_neohookean (:1020-1294) and the coloured
 * reverse-AD Jacobian (solvers/quasi_static_solver_2d.py:169-198 and
 * solvers/sparse_differentiation.py).  One thread per particle (cell order)
 * evaluates the residual and, when A->vals != NULL, its exact element tangent
 * K = -dR/du, scattered element-by-element into A->vals (precision = prec).
 * A is always required: its row map (node2row) places the residual rows;
 * A->vals == NULL asks for the residual only.
 * R_rows[n_rows*nf] (FP64) receives the masked residual; Dirichlet and
 * inactive DOFs get identity rows (mpm/mpm_utils.py:1299-1341).
 * force_host_accum: device double[1] accumulating the penalty footing force.
 * Writes F_new, b_new, sigma, pi_new (state of this iterate). */
int gw_assemble(const gw_grid_t *grid, const gw_material_t *mat, const gw_step_t *st, const gw_particles_t *pt,
                const int32_t *perm, const uint8_t *free_mask, const double *u_new, const double *u_old,
                const gw_bsr_t *A, int32_t prec, double *R_rows, double *force, void *stream);
/* The same residual and tangent for the 2D kinds, bitwise reproducible: the
 * replacement of the same reference kernels without atomic scatter.  A
 * particle pass (cell-sorted order, perm and the sorted keys of
 * gw_cell_sort) evaluates each particle's stress resultants and their
 * derivatives into workspace records; then one warp per occupied cell sums
 * its particles' contributions in sorted order into R_rows and A->vals, in
 * nine colour phases of cells three apart (disjoint node sets: plain
 * read-modify-writes, no atomics).  Arguments as gw_assemble plus keys (sorted
 * cell keys), workspace (256-byte aligned) of gw_assemble_workspace_bytes;
 * the 3D kind falls back to gw_assemble (atomic scatter) and needs no
 * workspace.  The footing force is still accumulated atomically. */
int64_t gw_assemble_workspace_bytes(const gw_grid_t *grid, int32_t n_particles, int32_t prec);
int gw_assemble_sorted(const gw_grid_t *grid, const gw_material_t *mat, const gw_step_t *st,
                       const gw_particles_t *pt, const int32_t *perm, const int32_t *keys, const uint8_t *free_mask,
                       const double *u_new, const double *u_old, const gw_bsr_t *A, int32_t prec, double *R_rows,
                       double *force, void *workspace, int64_t workspace_bytes, void *stream);

/* ------------------------------------------------------------ Krylov
 * Replaces wp.optim.linear.bicgstab with the 'diag' preconditioner and the
 * host spsolve / pyamg paths (solvers/quasi_static_solver_2d.py:236-256):
 * hand-written BSR SpMV + fused dot/axpy kernels, FP64 inner products.
 * Solves A x = b (x holds the initial guess).  rtol relative to ||b||.
 * workspace: gw_krylov_workspace_bytes(n_rows, nf, prec) bytes.
 * iters_host / relres_host receive the iteration count and final residual. */
int64_t gw_krylov_workspace_bytes(int32_t n_rows, int32_t nf, int32_t prec);
int gw_bsr_krylov_solve(const gw_bsr_t *A, int32_t prec, int32_t method, int32_t precond, const double *b, double *x,
                        double rtol, int32_t max_iter, void *workspace, int32_t *iters_host, double *relres_host,
                        void *stream);
/* gw_bsr_krylov_solve without a workspace argument (no counterpart in the
 * reference).  For callers that cannot call cudaMalloc: a host whose own
 * memory manager owns the device heap, or a path on which allocating device
 * memory is not allowed.  The solver's scratch is a file-scope device array in
 * the library, about 12.6 MB on every GPU that loads it, held until the
 * process exits; the call allocates nothing.  Limit:
 * n_rows * nf <= gw_krylov_static_max_unknowns() (131072); larger systems
 * return GW_EINVAL with a message naming the limit.  The first call on a
 * device looks up the array's device address with that device current (the
 * stream must belong to the current device) and keeps it for the life of the
 * process; make that first call before any stream capture, and do not reset
 * the device (cudaDeviceReset) after it, since the kept address would then be
 * stale.  All calls on a device share the one array: every call
 * clears the part that must start at zero, but calls that overlap on the GPU
 * (other streams, other host threads) race on it and must be serialised by
 * the caller. */
int64_t gw_krylov_static_max_unknowns(void);
int gw_bsr_krylov_solve_static(const gw_bsr_t *A, int32_t prec, int32_t method, int32_t precond, const double *b,
                               double *x, double rtol, int32_t max_iter, int32_t *iters_host, double *relres_host,
                               void *stream);
/* Restarted right-preconditioned GMRES(restart), restart <= 128: the robust
 * solver for the nonsymmetric, indefinite Jacobians (penalty footing, u-p
 * saddle point) on which BiCGSTAB breaks down.  Classical Gram-Schmidt with
 * one re-orthogonalisation; FP64 Krylov basis and inner products.
 * workspace: gw_gmres_workspace_bytes(n_rows, nf, restart) bytes. */
int64_t gw_gmres_workspace_bytes(int32_t n_rows, int32_t nf, int32_t restart);
int gw_bsr_gmres_solve(const gw_bsr_t *A, int32_t prec, int32_t precond, const double *b, double *x, double rtol,
                       int32_t max_iter, int32_t restart, void *workspace, int32_t *iters_host, double *relres_host,
                       void *stream);
/* Flexible GMRES(restart) preconditioned by one geometric-multigrid V-cycle on
 * the background-grid node lattice of `grid` (the grid whose node ids A's
 * row2node/node2row/stencil use).  Replaces the same solver choices as
 * gw_bsr_gmres_solve (solvers/quasi_static_solver_2d.py:236-256; the
 * reference's host pyamg path is the closest counterpart).  Hierarchy:
 * factor-2 coarsening per axis, Galerkin coarse operators P^T A P in the same
 * block-CSR layout and value type as A (sums in FP64; FP32 values when prec is
 * GW_PREC_MIXED), two damped node-block-Jacobi sweeps before and after
 * each coarse correction, an explicit dense inverse on the coarsest level
 * (<= 160 unknowns).  Identity rows of A (Dirichlet DOFs) are excluded from the
 * transfer operators.
 *
 * gw_mg_plan_build: the pattern phase (coarse active sets, stencils, block-CSR
 * patterns), written into the workspace, with the level sizes returned in the
 * host struct *plan_host.  It reads A's pattern only and synchronises twice per
 * coarse level.  A plan stays valid while A keeps its pattern (one load step,
 * and the transpose of its Jacobian, whose pattern is the same) and the same
 * workspace is passed.
 * gw_bsr_gmres_mg_solve: the numeric phase (Galerkin values, smoothers, dense
 * inverse; no host reads) and the solve.  plan_host == NULL builds a plan
 * first.  workspace: at least gw_gmres_mg_workspace_bytes(grid, n_rows, nf,
 * restart) bytes (the plan needs the hierarchy part, which comes first).
 * With plan_host->lag = 1 the numeric phase is skipped: the V-cycle reuses the
 * coarse operators, smoother blocks and coarsest inverse left in the
 * workspace by the previous solve with this plan (a matrix of the same
 * pattern and role, e.g. the previous Newton iterate's Jacobian), while
 * GMRES applies A itself, so the solution is A's; only the preconditioner
 * lags.  The caller must have run one solve with lag = 0 on this plan and
 * workspace first.  A plan is accepted only for the pattern it was built from:
 * the same workspace, row count, block count and row_ptr / cols arrays
 * (GW_EINVAL otherwise).  The solve writes its iteration count to
 * plan_host->last_iters: the next solve with the plan queues that many
 * Arnoldi steps before its first host check (a caller that rebuilds the plan
 * may carry the value over). */
#define GW_MG_MAX_LEVELS 20
typedef struct gw_mg_plan {
    int32_t levels;                     /* levels holding a matrix; the last one is solved densely */
    int32_t dense_n;                    /* unknowns of the coarsest level                          */
    int32_t n_rows[GW_MG_MAX_LEVELS];
    int32_t nnzb[GW_MG_MAX_LEVELS];
    int32_t nf, fine_n_rows, fine_nnzb;
    int32_t lag;                        /* 1: reuse the previous solve's numeric phase (see above)  */
    const void *workspace;              /* the coarse patterns live in this workspace              */
    const void *row_ptr, *cols;         /* pattern arrays of the matrix the plan was built from    */
    int32_t last_iters;                 /* iterations of the last solve with this plan (0: none)    */
    int32_t pad0;
} gw_mg_plan_t;
int64_t gw_gmres_mg_workspace_bytes(const gw_grid_t *grid, int32_t n_rows, int32_t nf, int32_t restart);
int gw_mg_plan_build(const gw_grid_t *grid, const gw_bsr_t *A, void *workspace, int64_t workspace_bytes,
                     gw_mg_plan_t *plan_host, void *stream);
int gw_bsr_gmres_mg_solve(const gw_grid_t *grid, const gw_bsr_t *A, int32_t prec, gw_mg_plan_t *plan_host,
                          const double *b, double *x, double rtol, int32_t max_iter, int32_t restart, void *workspace,
                          int64_t workspace_bytes, int32_t *iters_host, double *relres_host, void *stream);
/* Second (re-orthogonalisation) Gram-Schmidt passes taken by the last
 * gw_bsr_gmres_solve / gw_bsr_gmres_mg_solve on the calling host thread.
 * Both solvers project each new Krylov vector once and repeat the projection
 * only when it cancelled more of the vector's norm than GW_TUNE_GS_CANCEL
 * allows. */
int32_t gw_gmres_last_reorths(void);
/* 1 when the last gw_bsr_gmres_solve / gw_bsr_gmres_mg_solve on the calling
 * host thread stopped on stagnation (GW_ENOCONV before max_iter): its true
 * residual fell by less than 10% over the last GW_TUNE_GMRES_STALL restart
 * cycles.  0 otherwise. */
int32_t gw_gmres_last_stalled(void);
/* y = A x (x, y FP64 of length n_rows*nf; A values in prec). */
int gw_bsr_spmv(const gw_bsr_t *A, int32_t prec, const double *x, double *y, void *stream);
/* y = A^T x. */
int gw_bsr_spmv_t(const gw_bsr_t *A, int32_t prec, const double *x, double *y, void *stream);
/* ||v||_2 of an FP64 vector into norm_dev[0] (device). */
int gw_norm2(const double *v, int32_t n, double *norm_dev, void *workspace, void *stream);
/* u_full[row2node[r]*nf+f] += delta[r*nf+f]: from_increment_to_solution
 * (mpm/mpm_utils.py:1343-1348) restricted to the active rows. */
int gw_apply_increment(const gw_bsr_t *A, const double *delta, double *u_full, void *stream);
/* Newton's starting iterate from the previous load step (no counterpart in the
 * reference, which zeroes the increment at every load step's reset,
 * solvers/quasi_static_solver_2d.py:144-145):
 * u_full[row2node[r]*nf+f] = u_prev[...] on the free DOFs of the active rows
 * (free_mask of gw_compact_rows), 0 on their Dirichlet DOFs.  Nodes outside
 * the active set are not written (u_full is zero there after a reset).
 * u_prev and u_full are node-indexed [n_nodes*nf] and must not alias. */
int gw_predict_increment(const gw_bsr_t *A, const uint8_t *free_mask, const double *u_prev, double *u_full,
                         void *stream);

/* ------------------------------------------------------------ G2P
 * Replaces G2P_2d / G2P_coupled_2d / G2P_coupled_3d (mpm/mpm_utils.py:1351-1590)
 * fused with update_GIMP_lp_2d/3d (mpm/gimp.py:428-507): x += sum N du,
 * F_old <- F_new, b_old <- b_new, pi_old <- pi_new, pressure = sum N p,
 * lp update. */
int gw_g2p(const gw_grid_t *grid, const gw_step_t *st, const gw_particles_t *pt, const double *u_new,
           const double *u_old, void *stream);

/* ------------------------------------------------------------ single-point models
 * Evaluates a return map for n independent principal trial strains (e_trial
 * [n*3]) — the material tests of problems/material_tests/triaxial_*.py.
 * e_out[n*3]; tau_out[n*3] principal Kirchhoff; dtau_de_out[n*9] (may be NULL)
 * the algorithmic tangent d tau_A / d e_trial_B; eps_v_total[n] and pi_old,
 * pi_new (NorSand state) may be NULL for other models. */
int gw_return_map(const gw_material_t *mat, int32_t n, const double *e_trial, const double *eps_v_total,
                  const double *pi_old, double *pi_new, double *e_out, double *tau_out, double *dtau_de_out,
                  void *stream);

/* ------------------------------------------------------------ adjoint (2D solid kind)
 * The reference's only derivative is the Warp-tape gradient of the last
 * residual w.r.t. a scalar Young's modulus at fixed state
 * (solvers/quasi_static_coupled_solver_3d.py:159-165, 323-325).  These entry
 * points give the total derivative of a load step instead: with u* solving
 * R(u; q) = 0 for the particle inputs q = (x, lp, F_old, b_old, E),
 *   q_bar = (d out/d q)^T out_bar + R_q^T lambda,  K^T lambda = (d out/d u)^T out_bar,
 * out = (x_new, lp_new, F_new, b_new) the G2P outputs.  Per-particle arrays:
 * x, lp [N*2]; F, b [N*9]; E [N]. */
typedef struct gw_adjoint {
    double *x, *lp, *F, *b, *E;
} gw_adjoint_t;

/* AT_vals: the values of A^T on A's (symmetric) block pattern. */
int gw_bsr_transpose(const gw_grid_t *grid, const gw_bsr_t *A, int32_t prec, void *AT_vals, void *stream);
/* Adjoint G2P (mpm/mpm_utils.py:1351-1419, mpm/gimp.py:428-462): writes q_out
 * (overwrites) and ubar_rows[n_rows*2] (free DOFs only). pt holds the state at
 * the start of the load step, u_new the converged nodal solution. */
int gw_adjoint_g2p(const gw_grid_t *grid, const gw_material_t *mat, const gw_step_t *st, const gw_particles_t *pt,
                   const double *u_new, const double *u_old, const uint8_t *free_mask, const gw_bsr_t *A,
                   const gw_adjoint_t *seed_in, gw_adjoint_t *q_out, double *ubar_rows, void *stream);
/* Adjoint P2G of the residual (mpm/mpm_utils.py:416-780): q_out += R_q^T lambda. */
int gw_adjoint_residual(const gw_grid_t *grid, const gw_material_t *mat, const gw_step_t *st, const gw_particles_t *pt,
                        const double *u_new, const double *u_old, const uint8_t *free_mask, const gw_bsr_t *A,
                        const double *lambda_rows, gw_adjoint_t *q_out, void *stream);

/* ------------------------------------------------------------ kernel timing
 * Optional CUDA-event timing of the engine's main kernels (off by default):
 * classes 0..12 = k_assemble, k_gm_spmv, k_gm_dots, k_gm_update, k_gm_next,
 * k_g2p, k_adjoint_g2p, k_adjoint_residual, k_mg_jacobi (finest level),
 * k_mg_residual, k_mg_restrict/prolong, mg_setup (the numeric hierarchy
 * build), k_mg_jacobi (coarse levels).  gw_profile_read synchronises and
 * returns the total time, launch count and algorithmic bytes of a class. */
int gw_profile_enable(int32_t on);
/* Number of timing classes (k_assemble ... mg_setup) gw_profile_read accepts. */
int gw_profile_count(void);
int gw_profile_reset(void);
/* Number of kernels the library has launched since it was loaded (host
 * counter; no counterpart in the reference, which launches through Warp). */
int64_t gw_launch_count(void);
int gw_profile_read(int32_t cls, double *ms_total_host, int64_t *launches_host, double *bytes_host);
const char *gw_profile_name(int32_t cls);

/* ------------------------------------------------------------ launch-shape knobs
 * Process-wide settings the autotuner (geowarp_b200/autotune.py) searches per
 * workload on the device it runs on; no counterpart in the reference, whose
 * kernels Warp launches with fixed shapes.  They take effect at the next
 * launch (a changed GW_TUNE_ROW_WARPS recaptures the multigrid step graphs; a
 * changed GW_TUNE_MG_COARSE applies to plans built afterwards).
 *   GW_TUNE_PARTICLE_BLOCK  threads per CTA of the residual/tangent assembly,
 *                           32..256, a multiple of 32 (default 256)
 *   GW_TUNE_ADJOINT_BLOCK   threads per CTA of the adjoint particle kernels,
 *                           32..256, a multiple of 32 (default 128)
 *   GW_TUNE_ROW_WARPS       warps per CTA of the multigrid smoothing and
 *                           residual kernels (four block rows per warp), 1..32
 *                           (default 8)
 *   GW_TUNE_MG_COARSE       most unknowns of the dense coarsest multigrid
 *                           level, 8..160 (default 160)
 *   GW_TUNE_MG_ONE_SWEEP    first multigrid level smoothed by one sweep
 *                           before and after the coarse correction instead of
 *                           GW_TUNE_MG_SWEEPS, 1..20 (default 20: none);
 *                           recaptures the step graphs like GW_TUNE_ROW_WARPS
 *   GW_TUNE_MG_SWEEPS       block-Jacobi sweeps before and after the coarse
 *                           correction on the other levels, 1..4 (default 2)
 *   GW_TUNE_MG_OMEGA        damping of those sweeps in percent, 10..100
 *                           (default 70)
 *   GW_TUNE_GS_CANCEL       GMRES Gram-Schmidt: a second projection pass is
 *                           taken when the first left less than
 *                           10^(-value/10) of the new vector's squared norm,
 *                           0..300 (default 20: below 1/100, i.e. the
 *                           projection removed more than 90% of the norm,
 *                           so a column loses at most ~10 ulp of
 *                           orthogonality; 3: the classical 1/2; 0: always;
 *                           300: never unless non-finite)
 *   GW_TUNE_MG_TAIL         most block rows of a multigrid level run by the
 *                           fused coarse tail: that level and every coarser
 *                           one go through one launch of one thread-block
 *                           cluster with cluster barriers between the
 *                           phases (bitwise the same V-cycle; the cluster
 *                           has 1 to 16 CTAs, two rows of the first tail
 *                           level per 8-lane group), 0..1048576 (default 0:
 *                           one launch per phase); recaptures the step
 *                           graphs.  It pays where the levels are a few
 *                           hundred rows (launch-bound hierarchies)
 *   GW_TUNE_MG_BF16         1: in mixed-precision multigrid solves the V-cycle
 *                           reads a BF16 copy of the fine-level Jacobian (made
 *                           before each solve; GMRES still applies the FP32
 *                           Jacobian), 0: the FP32 Jacobian (default 0);
 *                           changes the preconditioner only, and weakens it on
 *                           ill-conditioned systems solved to small relative
 *                           residuals (plastic footings): for well-conditioned
 *                           ones only; recaptures the step graphs
 *   GW_TUNE_MG_FINE_SWEEPS  block-Jacobi sweeps before and after the coarse
 *                           correction on the finest level, 1..4 (default 1);
 *                           changes the preconditioner; recaptures the step
 *                           graphs
 *   GW_TUNE_GMRES_STALL     restart cycles over which a GMRES solve's true
 *                           residual must fall by 10%, else the solve stops
 *                           with GW_ENOCONV before max_iter, 0..100000
 *                           (default 50; 0: off, run to max_iter)
 * MG_SWEEPS and MG_OMEGA change the preconditioner (Krylov iteration counts),
 * not the solution GMRES converges to; they also recapture the step graphs.
 * GS_CANCEL changes the orthogonality of the Krylov basis and so the
 * iteration count and the attainable accuracy; it is read at each solve.
 * gw_tune_set returns GW_EINVAL outside these ranges; gw_tune_get returns -1
 * for an unknown knob. */
#define GW_TUNE_PARTICLE_BLOCK 0
#define GW_TUNE_ADJOINT_BLOCK 1
#define GW_TUNE_ROW_WARPS 2
#define GW_TUNE_MG_COARSE 3
#define GW_TUNE_MG_ONE_SWEEP 4
#define GW_TUNE_MG_SWEEPS 5
#define GW_TUNE_MG_OMEGA 6
#define GW_TUNE_GS_CANCEL 7
#define GW_TUNE_MG_TAIL 8
#define GW_TUNE_MG_BF16 9
#define GW_TUNE_MG_FINE_SWEEPS 10
#define GW_TUNE_GMRES_STALL 11
#define GW_TUNE_COUNT 12
int gw_tune_set(int32_t knob, int32_t value);
int32_t gw_tune_get(int32_t knob);

#ifdef __cplusplus
}
#endif
#endif /* GEOWARP_B200_H */
