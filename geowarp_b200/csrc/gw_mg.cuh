// Geometric multigrid preconditioner on the background-grid node lattice.
//
// The reference solves each Newton correction with Warp's BiCGSTAB and a
// diagonal preconditioner, or hands it to pyamg / SciPy on the host
// (solvers/quasi_static_solver_2d.py:236-256).  Here the Krylov method is a
// flexible GMRES whose preconditioner is one V-cycle over a hierarchy built
// from the block-CSR Jacobian itself:
//
//   level l+1 lattice: node I sits on fine node 2I (per axis); a fine node with
//     an even coordinate has one parent (weight 1), an odd one two (1/2 each);
//     P is the tensor product of these weights, per field, zero on fixed DOFs;
//   coarse operator: Galerkin A_{l+1} = P^T A_l P in the same 5^D-stencil
//     block-CSR layout (a coarse block (I,J) gathers the fine blocks (i,j) of
//     I's and J's children in a fixed order: deterministic, no atomics);
//   smoother: damped node-block Jacobi; coarsest level (at most 160 unknowns):
//     explicit dense inverse.
//
// Coupled u-p systems (D displacement fields and one pressure field per node)
// are saddle points [[K, B], [B^T, -C]] whose u-p coupling lives off the node
// diagonal (the node's own B entries vanish) and whose pressure block C =
// dt k Laplacian is tiny at small time steps.  Plain node-block Jacobi then
// updates the pressure by r_p / C, which diverges once B^2 / (C K) > 1 (mesh
// Fourier number cv dt / dx^2 below about one).  The smoother therefore
// inverts node blocks whose pressure diagonal is replaced by that of the
// Schur complement with a diagonal K:
//   S_ii = -C_ii - sum_{j != i} sum_g B_i(j,g) B^T(j,g)_i / K(j,g; j,g),
// the diagonal-approximation Schur smoother of SIMPLE-type block methods.
//
// Fixed (Dirichlet) DOFs are recognised from the Jacobian: their rows are
// identity rows (the assembly writes 1 on the diagonal and nothing else).
#pragma once
#include "gw_krylov.cuh"

namespace gw {
namespace {  // internal linkage: each translation unit compiles the kernels it launches

constexpr int kMgMaxLevels = GW_MG_MAX_LEVELS;
// unknowns of the coarsest (dense) level: its n x n FP64 matrix (204,800 bytes
// at 160) is inverted in one CTA's shared memory
constexpr int kMgCoarseMax = 160;
constexpr int kMgCoarseMin = 8;  // smallest coarsest-level bound a caller may set

// lattice node counts of a grid (cells + 1 per axis; 1 on unused axes)
struct Lat {
    int dim, n[3];
};
__host__ __device__ inline Lat lat_of(const gw_grid_t &g) {
    Lat L;
    L.dim = g.dim;
    for (int k = 0; k < 3; ++k) L.n[k] = k < g.dim ? g.n_grid[k] + 1 : 1;
    return L;
}
__device__ __forceinline__ void lat_coords(const Lat &L, int id, int c[3]) {
    c[0] = id % L.n[0];
    const int t = id / L.n[0];
    c[1] = t % L.n[1];
    c[2] = t / L.n[1];
}
__device__ __forceinline__ int lat_id(const Lat &L, const int c[3]) { return c[0] + L.n[0] * (c[1] + L.n[1] * c[2]); }
__host__ __device__ inline int lat_size(const Lat &L) { return L.n[0] * L.n[1] * L.n[2]; }

// 1D prolongation weight of fine coordinate f below coarse coordinate C
__device__ __forceinline__ double p_weight(int f, int C) {
    const int d = f - 2 * C;
    return d == 0 ? 1.0 : ((d == 1 || d == -1) ? 0.5 : 0.0);
}

// ---------------------------------------------------------------- fixed-DOF mask
// bit f of fixed[r]: row (r, f) of A is an identity row
template <int NF, typename VT>
__global__ void k_mg_fixed_mask(PtrsA A, uint8_t *__restrict__ fixed) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= A.n_rows) return;
    const VT *vals = (const VT *)A.vals;
    uint8_t m = 0;
    for (int f = 0; f < NF; ++f) {
        bool id = true;
        bool diag_one = false;
        for (int j = A.row_ptr[r]; j < A.row_ptr[r + 1] && id; ++j) {
            const VT *blk = vals + (size_t)j * NF * NF + f * NF;
            const bool self = A.cols[j] == r;
            for (int g = 0; g < NF; ++g) {
                const double v = (double)blk[g];
                if (self && g == f) diag_one = (v == 1.0);
                else if (v != 0.0) { id = false; break; }
            }
        }
        if (id && diag_one) m |= (uint8_t)(1u << f);
    }
    fixed[r] = m;
}

// ---------------------------------------------------------------- coarse active set
__global__ void k_mg_coarse_flags(Lat Lf, PtrsA Af, Lat Lc, uint8_t *__restrict__ cflag) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= Af.n_rows) return;
    const int node = Af.row2node[r];
    if (!in_range(node, lat_size(Lf), GS_COARSE_FLAGS)) return;
    int c[3];
    lat_coords(Lf, node, c);
    int lo[3], cnt[3];
    for (int k = 0; k < 3; ++k) {
        lo[k] = c[k] >> 1;
        cnt[k] = (k < Lf.dim && (c[k] & 1)) ? 2 : 1;
    }
    for (int a = 0; a < cnt[0]; ++a)
        for (int b = 0; b < cnt[1]; ++b)
            for (int d = 0; d < cnt[2]; ++d) {
                const int C[3] = {lo[0] + a, lo[1] + b, lo[2] + d};
                const int id = lat_id(Lc, C);
                if (in_range(id, lat_size(Lc), GS_COARSE_FLAGS)) cflag[id] = 1;
            }
}

// coarse stencil mask of every coarse row and its block count
template <int D>
__global__ void k_mg_coarse_stencil(Lat Lf, PtrsA Af, Lat Lc, int nc_rows, const int *__restrict__ c_row2node,
                                    uint32_t *__restrict__ c_stencil, int mw, int *__restrict__ c_count) {
    const int R = blockIdx.x * blockDim.x + threadIdx.x;
    if (R >= nc_rows) return;
    const int I = c_row2node[R];
    if (!in_range(I, lat_size(Lc), GS_COARSE_STENCIL)) return;
    int C[3];
    lat_coords(Lc, I, C);
    uint32_t mask[4] = {0u, 0u, 0u, 0u};
    for (int oz = (D == 3 ? -1 : 0); oz <= (D == 3 ? 1 : 0); ++oz)
        for (int oy = -1; oy <= 1; ++oy)
            for (int ox = -1; ox <= 1; ++ox) {
                const int ci[3] = {2 * C[0] + ox, 2 * C[1] + oy, 2 * C[2] + oz};
                bool in = true;
                for (int k = 0; k < D; ++k) in = in && ci[k] >= 0 && ci[k] < Lf.n[k];
                if (!in) continue;
                const int i = lat_id(Lf, ci);
                if (Af.node2row[i] < 0) continue;
                for (int w = 0; w < mw; ++w) {
                    uint32_t m = Af.stencil[(size_t)i * mw + w];
                    while (m) {
                        int bit = w * 32 + __ffs(m) - 1;
                        m &= m - 1u;
                        int cj[3] = {ci[0], ci[1], ci[2]};
                        for (int k = 0; k < D; ++k) {
                            cj[k] += bit % 5 - 2;
                            bit /= 5;
                        }
                        // parents of fine node j, relative to C (always within [-2, 2])
                        int lo[3], cnt[3];
                        for (int k = 0; k < 3; ++k) {
                            lo[k] = (cj[k] >> 1) - C[k];
                            cnt[k] = (k < D && (cj[k] & 1)) ? 2 : 1;
                        }
                        for (int a = 0; a < cnt[0]; ++a)
                            for (int b = 0; b < cnt[1]; ++b)
                                for (int d = 0; d < cnt[2]; ++d) {
                                    const int off[3] = {lo[0] + a, lo[1] + b, lo[2] + d};
                                    bool ok = true;
                                    for (int k = 0; k < D; ++k) ok = ok && in_range(off[k] + 2, 5, GS_COARSE_STENCIL);
                                    if (!ok) continue;
                                    const int ob = offset_bit<D>(off);
                                    mask[ob >> 5] |= 1u << (ob & 31);
                                }
                    }
                }
            }
    int n = 0;
    for (int w = 0; w < mw; ++w) {
        c_stencil[(size_t)I * mw + w] = mask[w];
        n += __popc(mask[w]);
    }
    c_count[R] = n;
}

// block -> row map of a block-CSR (for one-thread-per-block kernels)
__global__ void k_mg_blockrow(const int *__restrict__ row_ptr, int n_rows, int nnzb, int *__restrict__ blockrow) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n_rows) return;
    for (int j = row_ptr[r]; j < row_ptr[r + 1]; ++j)
        if (in_range(j, nnzb, GS_BLOCKROW)) blockrow[j] = r;
}

// ---------------------------------------------------------------- Galerkin product
// One thread per coarse block (I, J): sum over children i of I and j of J,
// in lattice order, of w_i w_j A(i, j) restricted to free DOFs.
template <int D, int NF, typename VT>
__global__ void k_mg_rap(Lat Lf, PtrsA Af, const uint8_t *__restrict__ ffixed, Lat Lc, PtrsA Ac,
                         const int *__restrict__ c_blockrow) {
    const int jb = blockIdx.x * blockDim.x + threadIdx.x;
    if (jb >= Ac.nnzb) return;
    const int R = c_blockrow[jb], Rc = Ac.cols[jb];
    VT *out = (VT *)Ac.vals + (size_t)jb * NF * NF;  // the coarse levels store the fine level's value type
    if (!in_range(R, Ac.n_rows, GS_RAP_COARSE) || !in_range(Rc, Ac.n_rows, GS_RAP_COARSE)) {
        for (int q = 0; q < NF * NF; ++q) out[q] = 0.0;
        return;
    }
    const int I = Ac.row2node[R], J = Ac.row2node[Rc];
    if (!in_range(I, lat_size(Lc), GS_RAP_COARSE) || !in_range(J, lat_size(Lc), GS_RAP_COARSE)) {
        for (int q = 0; q < NF * NF; ++q) out[q] = 0.0;
        return;
    }
    int CI[3], CJ[3];
    lat_coords(Lc, I, CI);
    lat_coords(Lc, J, CJ);
    double acc[NF][NF];
#pragma unroll
    for (int f = 0; f < NF; ++f)
#pragma unroll
        for (int g = 0; g < NF; ++g) acc[f][g] = 0.0;
    const VT *vals = (const VT *)Af.vals;
    for (int iz = (D == 3 ? -1 : 0); iz <= (D == 3 ? 1 : 0); ++iz)
        for (int iy = -1; iy <= 1; ++iy)
            for (int ix = -1; ix <= 1; ++ix) {
                const int ci[3] = {2 * CI[0] + ix, 2 * CI[1] + iy, 2 * CI[2] + iz};
                bool in = true;
                for (int k = 0; k < D; ++k) in = in && ci[k] >= 0 && ci[k] < Lf.n[k];
                if (!in) continue;
                const int i = lat_id(Lf, ci);
                const int fr = Af.node2row[i];
                if (fr < 0 || !in_range(fr, Af.n_rows, GS_RAP_FINE)) continue;
                double wi = 1.0;
                for (int k = 0; k < D; ++k) wi *= p_weight(ci[k], CI[k]);
                const uint8_t fi = ffixed[fr];
                for (int jz = (D == 3 ? -1 : 0); jz <= (D == 3 ? 1 : 0); ++jz)
                    for (int jy = -1; jy <= 1; ++jy)
                        for (int jx = -1; jx <= 1; ++jx) {
                            const int cj[3] = {2 * CJ[0] + jx, 2 * CJ[1] + jy, 2 * CJ[2] + jz};
                            int off[3] = {0, 0, 0};
                            bool ok = true;
                            for (int k = 0; k < D; ++k) {
                                off[k] = cj[k] - ci[k];
                                ok = ok && off[k] >= -2 && off[k] <= 2 && cj[k] >= 0 && cj[k] < Lf.n[k];
                            }
                            if (!ok) continue;
                            const int slot = stencil_slot(Af.stencil, Af.mw, i, offset_bit<D>(off));
                            if (slot < 0) continue;
                            const int fc = Af.node2row[lat_id(Lf, cj)];
                            if (fc < 0 || !in_range(fc, Af.n_rows, GS_RAP_FINE)) continue;
                            const long long fb = (long long)Af.row_ptr[fr] + slot;
                            if (!in_range(fb, Af.nnzb, GS_RAP_FINE)) continue;
                            double wj = 1.0;
                            for (int k = 0; k < D; ++k) wj *= p_weight(cj[k], CJ[k]);
                            const uint8_t fj = ffixed[fc];
                            const VT *blk = vals + (size_t)fb * NF * NF;
                            const double w = wi * wj;
#pragma unroll
                            for (int f = 0; f < NF; ++f) {
                                if ((fi >> f) & 1) continue;
#pragma unroll
                                for (int g = 0; g < NF; ++g)
                                    if (!((fj >> g) & 1)) acc[f][g] += w * (double)blk[f * NF + g];
                            }
                        }
            }
#pragma unroll
    for (int f = 0; f < NF; ++f)
#pragma unroll
        for (int g = 0; g < NF; ++g) out[f * NF + g] = (VT)acc[f][g];
}

// coarse rows that received nothing (every child DOF fixed) become identity rows
template <int NF, typename VT>
__global__ void k_mg_fix_empty_rows(PtrsA A) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= A.n_rows) return;
    VT *vals = (VT *)A.vals;
    int self = -1;
    for (int j = A.row_ptr[r]; j < A.row_ptr[r + 1]; ++j)
        if (A.cols[j] == r) self = j;
    if (self < 0) return;
    for (int f = 0; f < NF; ++f) {
        bool empty = true;
        for (int j = A.row_ptr[r]; j < A.row_ptr[r + 1] && empty; ++j)
            for (int g = 0; g < NF; ++g)
                if (vals[(size_t)j * NF * NF + f * NF + g] != (VT)0) { empty = false; break; }
        if (empty) vals[(size_t)self * NF * NF + f * NF + f] = (VT)1;
    }
}

// ---------------------------------------------------------------- smoother blocks
// Minv of one level: inverse of each node's diagonal block; on u-p systems
// (NF == D + 1) the pressure diagonal first takes the off-node Schur term.
// A row's blocks are stored in stencil-bit order, the bit of offset o being
// sum_k (o_k + 2) 5^k, so the transposed block (j, i) of block (i, j) sits at
// bit (5^D - 1) - bit in row j.
template <int NF, typename VT>
__global__ void k_mg_smoother_setup(PtrsA A, int D, double *__restrict__ Minv) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= A.n_rows) return;
    const int node = A.row2node[r];
    const int top = D == 2 ? 24 : 124;  // 5^D - 1
    const int center = top / 2;
    const int slot = stencil_slot(A.stencil, A.mw, node, center);
    double *out = Minv + (size_t)r * NF * NF;
    if (slot < 0) {
        for (int i = 0; i < NF; ++i)
            for (int j = 0; j < NF; ++j) out[i * NF + j] = (i == j) ? 1.0 : 0.0;
        return;
    }
    const VT *vals = (const VT *)A.vals;
    const VT *blk = vals + ((size_t)A.row_ptr[r] + slot) * NF * NF;
    double M[NF][NF];
    for (int i = 0; i < NF; ++i)
        for (int j = 0; j < NF; ++j) M[i][j] = (double)blk[i * NF + j];
    if (NF == D + 1) {
        constexpr int P = NF - 1;
        double corr = 0.0;
        int s = 0;
        for (int w = 0; w < A.mw; ++w) {
            uint32_t m = A.stencil[(size_t)node * A.mw + w];
            while (m) {
                const int bit = w * 32 + __ffs(m) - 1;
                m &= m - 1u;
                const int k = A.row_ptr[r] + s++;
                if (bit == center) continue;
                if (!in_range(k, A.nnzb, GS_SMOOTHER)) continue;
                const int col = A.cols[k];
                if (!in_range(col, A.n_rows, GS_SMOOTHER)) continue;
                const int nj = A.row2node[col];
                const int tj = stencil_slot(A.stencil, A.mw, nj, top - bit);
                const int dj = stencil_slot(A.stencil, A.mw, nj, center);
                if (tj < 0 || dj < 0) continue;
                if (!in_range((long long)A.row_ptr[col] + (tj > dj ? tj : dj), A.nnzb, GS_SMOOTHER)) continue;
                const VT *b_ij = vals + (size_t)k * NF * NF;
                const VT *b_ji = vals + ((size_t)A.row_ptr[col] + tj) * NF * NF;
                const VT *b_jj = vals + ((size_t)A.row_ptr[col] + dj) * NF * NF;
#pragma unroll
                for (int g = 0; g < P; ++g) {
                    const double kjj = (double)b_jj[g * NF + g];
                    if (kjj != 0.0) corr += (double)b_ij[P * NF + g] * (double)b_ji[g * NF + P] / kjj;
                }
            }
        }
        M[P][P] -= corr;
    }
    invert_block<NF>(M, out);
}

// ---------------------------------------------------------------- cycle kernels
// x_out = x_in + omega Minv (b - A x_in); zero_init: x_in = 0 (x_out = omega Minv b)
template <int NF, typename VT>
__global__ void k_mg_jacobi(PtrsA A, const double *__restrict__ Minv, const double *__restrict__ b,
                            const double *__restrict__ x_in, double *__restrict__ x_out, double omega, int zero_init,
                            const int *__restrict__ skip) {
    if (skip && *skip) return;
    if (zero_init) {
        for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < A.n_rows; r += gridDim.x * blockDim.x) {
            double t[NF], z[NF];
#pragma unroll
            for (int f = 0; f < NF; ++f) t[f] = b[(size_t)r * NF + f];
            apply_minv<NF>(Minv, r, t, z);
#pragma unroll
            for (int f = 0; f < NF; ++f) x_out[(size_t)r * NF + f] = omega * z[f];
        }
        return;
    }
    const int nw = gridDim.x * (blockDim.x >> 5) * kRowsPerWarp;
    for (int rb = (blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5)) * kRowsPerWarp; rb < A.n_rows; rb += nw) {
        const int r = rb + (threadIdx.x & 31) / kLPR;
        double acc[NF];
        row_mv<NF, VT>(A, r, x_in, acc);
        if (r < A.n_rows && (threadIdx.x & (kLPR - 1)) == 0) {
            double t[NF], z[NF];
#pragma unroll
            for (int f = 0; f < NF; ++f) t[f] = b[(size_t)r * NF + f] - acc[f];
            apply_minv<NF>(Minv, r, t, z);
#pragma unroll
            for (int f = 0; f < NF; ++f) x_out[(size_t)r * NF + f] = x_in[(size_t)r * NF + f] + omega * z[f];
        }
    }
}

// Both pre-smoothing sweeps from a zero start in one launch:
//   x1 = omega Minv b,   x_out = x1 + omega Minv (b - A x1),
// with the neighbours' x1 recomputed where they are read (the same
// arithmetic as the separate zero-start sweep, so the result is bitwise the
// same).  The extra Minv and b reads of the neighbours stay in L2; the
// launch and the round trip of x1 through memory are saved.
template <int NF, typename VT>
__global__ void k_mg_presmooth2(PtrsA A, const double *__restrict__ Minv, const double *__restrict__ b,
                                double *__restrict__ x_out, double omega, const int *__restrict__ skip) {
    if (skip && *skip) return;
    const int nw = gridDim.x * (blockDim.x >> 5) * kRowsPerWarp;
    const int lane = threadIdx.x & (kLPR - 1);
    const VT *vals = (const VT *)A.vals;
    for (int rb = (blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5)) * kRowsPerWarp; rb < A.n_rows; rb += nw) {
        const int r = rb + (threadIdx.x & 31) / kLPR;
        double acc[NF];
#pragma unroll
        for (int f = 0; f < NF; ++f) acc[f] = 0.0;
        const int s0 = r < A.n_rows ? A.row_ptr[r] : 0, e0 = r < A.n_rows ? A.row_ptr[r + 1] : 0;
        for (int j = s0 + lane; j < e0; j += kLPR) {
            const int col = A.cols[j];
            if (!in_range(col, A.n_rows, GS_PRESMOOTH)) continue;
            double t[NF], z[NF], bv[NF * NF];
            load_vec<NF>(b + (size_t)col * NF, t);
            load_block<NF, VT>(vals + (size_t)j * NF * NF, bv);
            apply_minv<NF>(Minv, col, t, z);
#pragma unroll
            for (int f = 0; f < NF; ++f)
#pragma unroll
                for (int g = 0; g < NF; ++g) acc[f] += bv[f * NF + g] * (omega * z[g]);
        }
#pragma unroll
        for (int f = 0; f < NF; ++f)
#pragma unroll
            for (int o = kLPR / 2; o > 0; o >>= 1) acc[f] += __shfl_down_sync(0xffffffffu, acc[f], o, kLPR);
        if (r < A.n_rows && lane == 0) {
            double t[NF], z[NF], x1[NF];
#pragma unroll
            for (int f = 0; f < NF; ++f) t[f] = b[(size_t)r * NF + f];
            apply_minv<NF>(Minv, r, t, z);
#pragma unroll
            for (int f = 0; f < NF; ++f) x1[f] = omega * z[f];
#pragma unroll
            for (int f = 0; f < NF; ++f) t[f] = b[(size_t)r * NF + f] - acc[f];
            apply_minv<NF>(Minv, r, t, z);
#pragma unroll
            for (int f = 0; f < NF; ++f) x_out[(size_t)r * NF + f] = x1[f] + omega * z[f];
        }
    }
}

// r = b - A x
template <int NF, typename VT>
__global__ void k_mg_residual(PtrsA A, const double *__restrict__ b, const double *__restrict__ x,
                              double *__restrict__ r_out, const int *__restrict__ skip) {
    if (skip && *skip) return;
    const int nw = gridDim.x * (blockDim.x >> 5) * kRowsPerWarp;
    for (int rb = (blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5)) * kRowsPerWarp; rb < A.n_rows; rb += nw) {
        const int r = rb + (threadIdx.x & 31) / kLPR;
        double acc[NF];
        row_mv<NF, VT>(A, r, x, acc);
        if (r < A.n_rows && (threadIdx.x & (kLPR - 1)) == 0)
#pragma unroll
            for (int f = 0; f < NF; ++f) r_out[(size_t)r * NF + f] = b[(size_t)r * NF + f] - acc[f];
    }
}

// b_c = P^T r_f
template <int D, int NF>
__global__ void k_mg_restrict(Lat Lf, PtrsA Af, const uint8_t *__restrict__ ffixed, Lat Lc, PtrsA Ac,
                              const double *__restrict__ rf, double *__restrict__ bc, const int *__restrict__ skip) {
    if (skip && *skip) return;
    const int R = blockIdx.x * blockDim.x + threadIdx.x;
    if (R >= Ac.n_rows) return;
    const int I = Ac.row2node[R];
    if (!in_range(I, lat_size(Lc), GS_RESTRICT)) return;
    int C[3];
    lat_coords(Lc, I, C);
    double acc[NF];
#pragma unroll
    for (int f = 0; f < NF; ++f) acc[f] = 0.0;
    for (int oz = (D == 3 ? -1 : 0); oz <= (D == 3 ? 1 : 0); ++oz)
        for (int oy = -1; oy <= 1; ++oy)
            for (int ox = -1; ox <= 1; ++ox) {
                const int ci[3] = {2 * C[0] + ox, 2 * C[1] + oy, 2 * C[2] + oz};
                bool in = true;
                for (int k = 0; k < D; ++k) in = in && ci[k] >= 0 && ci[k] < Lf.n[k];
                if (!in) continue;
                const int fr = Af.node2row[lat_id(Lf, ci)];
                if (fr < 0 || !in_range(fr, Af.n_rows, GS_RESTRICT)) continue;
                double w = 1.0;
                for (int k = 0; k < D; ++k) w *= p_weight(ci[k], C[k]);
                const uint8_t fx = ffixed[fr];
#pragma unroll
                for (int f = 0; f < NF; ++f)
                    if (!((fx >> f) & 1)) acc[f] += w * rf[(size_t)fr * NF + f];
            }
#pragma unroll
    for (int f = 0; f < NF; ++f) bc[(size_t)R * NF + f] = acc[f];
}

// x_f += P x_c
template <int D, int NF>
__global__ void k_mg_prolong(Lat Lf, PtrsA Af, const uint8_t *__restrict__ ffixed, Lat Lc, PtrsA Ac,
                             const double *__restrict__ xc, double *__restrict__ xf, const int *__restrict__ skip) {
    if (skip && *skip) return;
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= Af.n_rows) return;
    const int node = Af.row2node[r];
    if (!in_range(node, lat_size(Lf), GS_PROLONG)) return;
    int c[3];
    lat_coords(Lf, node, c);
    int lo[3], cnt[3];
    for (int k = 0; k < 3; ++k) {
        lo[k] = c[k] >> 1;
        cnt[k] = (k < D && (c[k] & 1)) ? 2 : 1;
    }
    double acc[NF];
#pragma unroll
    for (int f = 0; f < NF; ++f) acc[f] = 0.0;
    for (int a = 0; a < cnt[0]; ++a)
        for (int b = 0; b < cnt[1]; ++b)
            for (int d = 0; d < cnt[2]; ++d) {
                const int C[3] = {lo[0] + a, lo[1] + b, lo[2] + d};
                const int cid = lat_id(Lc, C);
                if (!in_range(cid, lat_size(Lc), GS_PROLONG)) continue;
                const int R = Ac.node2row[cid];
                if (R < 0 || !in_range(R, Ac.n_rows, GS_PROLONG)) continue;
                double w = 1.0;
                for (int k = 0; k < D; ++k) w *= p_weight(c[k], C[k]);
#pragma unroll
                for (int f = 0; f < NF; ++f) acc[f] += w * xc[(size_t)R * NF + f];
            }
    const uint8_t fx = ffixed[r];
#pragma unroll
    for (int f = 0; f < NF; ++f)
        if (!((fx >> f) & 1)) xf[(size_t)r * NF + f] += acc[f];
}

// BF16 copy of FP32 block values (the V-cycle's copy of a mixed-precision
// fine level; round to nearest)
__global__ void k_to_bf16(const float *__restrict__ in, __nv_bfloat16 *__restrict__ out, size_t n) {
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        out[i] = __float2bfloat16_rn(in[i]);
}

// ---------------------------------------------------------------- transfer lists
// The transfers above find each child / parent through the lattice
// (row2node, coordinates, node2row) on every V-cycle.  The pattern phase
// resolves those lookups once per load step into row lists, so a V-cycle's
// restriction and prolongation read an index list and then the vector: two
// dependent loads instead of three per child.  The lists keep the loop order
// of k_mg_restrict / k_mg_prolong, so the sums are bitwise the same.

// child[R * 3^D + q]: fine row of child q (q = ox+1 + 3 (oy+1) [+ 9 (oz+1)]) of
// coarse row R, -1 where the child is outside the lattice or inactive
template <int D>
__global__ void k_mg_children(Lat Lf, PtrsA Af, Lat Lc, PtrsA Ac, int *__restrict__ child) {
    constexpr int CN = D == 2 ? 9 : 27;
    const int R = blockIdx.x * blockDim.x + threadIdx.x;
    if (R >= Ac.n_rows) return;
    int *out = child + (size_t)R * CN;
    const int I = Ac.row2node[R];
    if (!in_range(I, lat_size(Lc), GS_RESTRICT)) {
        for (int q = 0; q < CN; ++q) out[q] = -1;
        return;
    }
    int C[3];
    lat_coords(Lc, I, C);
    int q = 0;
    for (int oz = (D == 3 ? -1 : 0); oz <= (D == 3 ? 1 : 0); ++oz)
        for (int oy = -1; oy <= 1; ++oy)
            for (int ox = -1; ox <= 1; ++ox, ++q) {
                const int ci[3] = {2 * C[0] + ox, 2 * C[1] + oy, 2 * C[2] + oz};
                bool in = true;
                for (int k = 0; k < D; ++k) in = in && ci[k] >= 0 && ci[k] < Lf.n[k];
                int fr = -1;
                if (in) {
                    fr = Af.node2row[lat_id(Lf, ci)];
                    if (fr < 0 || !in_range(fr, Af.n_rows, GS_RESTRICT)) fr = -1;
                }
                out[q] = fr;
            }
}

// parent[r * 2^D + q]: coarse rows of fine row r in k_mg_prolong's loop order,
// -1 where that parent is outside the lattice or inactive, -2 past the
// parity count (the weight of every parent is 1 / that count)
template <int D>
__global__ void k_mg_parents(Lat Lf, PtrsA Af, Lat Lc, PtrsA Ac, int *__restrict__ parent) {
    constexpr int PN = D == 2 ? 4 : 8;
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= Af.n_rows) return;
    int *out = parent + (size_t)r * PN;
    for (int q = 0; q < PN; ++q) out[q] = -2;
    const int node = Af.row2node[r];
    if (!in_range(node, lat_size(Lf), GS_PROLONG)) return;
    int c[3];
    lat_coords(Lf, node, c);
    int lo[3], cnt[3];
    for (int k = 0; k < 3; ++k) {
        lo[k] = c[k] >> 1;
        cnt[k] = (k < D && (c[k] & 1)) ? 2 : 1;
    }
    int q = 0;
    for (int a = 0; a < cnt[0]; ++a)
        for (int b = 0; b < cnt[1]; ++b)
            for (int d = 0; d < cnt[2]; ++d, ++q) {
                const int C[3] = {lo[0] + a, lo[1] + b, lo[2] + d};
                const int cid = lat_id(Lc, C);
                int R = -1;
                if (in_range(cid, lat_size(Lc), GS_PROLONG)) {
                    R = Ac.node2row[cid];
                    if (R < 0 || !in_range(R, Ac.n_rows, GS_PROLONG)) R = -1;
                }
                out[q] = R;
            }
}

// b_c = P^T r_f through the child lists
template <int D, int NF>
__global__ void k_mg_restrict_list(int nc, int nf_rows, const int *__restrict__ child,
                                   const uint8_t *__restrict__ ffixed, const double *__restrict__ rf,
                                   double *__restrict__ bc, const int *__restrict__ skip) {
    constexpr int CN = D == 2 ? 9 : 27;
    if (skip && *skip) return;
    const int R = blockIdx.x * blockDim.x + threadIdx.x;
    if (R >= nc) return;
    const int *ch = child + (size_t)R * CN;
    int fr[CN];
#pragma unroll
    for (int q = 0; q < CN; ++q) fr[q] = ch[q];
    double acc[NF];
#pragma unroll
    for (int f = 0; f < NF; ++f) acc[f] = 0.0;
#pragma unroll
    for (int q = 0; q < CN; ++q) {
        if (fr[q] < 0 || !in_range(fr[q], nf_rows, GS_RESTRICT)) continue;
        const int ox = q % 3 - 1, oy = (q / 3) % 3 - 1, oz = q / 9 - 1;
        double w = 1.0;
        w *= ox == 0 ? 1.0 : 0.5;
        w *= oy == 0 ? 1.0 : 0.5;
        if (D == 3) w *= oz == 0 ? 1.0 : 0.5;
        const uint8_t fx = ffixed[fr[q]];
#pragma unroll
        for (int f = 0; f < NF; ++f)
            if (!((fx >> f) & 1)) acc[f] += w * rf[(size_t)fr[q] * NF + f];
    }
#pragma unroll
    for (int f = 0; f < NF; ++f) bc[(size_t)R * NF + f] = acc[f];
}

// x_f += P x_c through the parent lists
template <int D, int NF>
__global__ void k_mg_prolong_list(int n_rows, int nc, const int *__restrict__ parent,
                                  const uint8_t *__restrict__ ffixed, const double *__restrict__ xc,
                                  double *__restrict__ xf, const int *__restrict__ skip) {
    constexpr int PN = D == 2 ? 4 : 8;
    if (skip && *skip) return;
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n_rows) return;
    const int *pa = parent + (size_t)r * PN;
    int R[PN];
#pragma unroll
    for (int q = 0; q < PN; ++q) R[q] = pa[q];
    int cnt = 0;
#pragma unroll
    for (int q = 0; q < PN; ++q) cnt += R[q] != -2;
    const double w = cnt == 1 ? 1.0 : (cnt == 2 ? 0.5 : (cnt == 4 ? 0.25 : 0.125));
    double acc[NF];
#pragma unroll
    for (int f = 0; f < NF; ++f) acc[f] = 0.0;
#pragma unroll
    for (int q = 0; q < PN; ++q) {
        if (R[q] < 0 || !in_range(R[q], nc, GS_PROLONG)) continue;
#pragma unroll
        for (int f = 0; f < NF; ++f) acc[f] += w * xc[(size_t)R[q] * NF + f];
    }
    const uint8_t fx = ffixed[r];
#pragma unroll
    for (int f = 0; f < NF; ++f)
        if (!((fx >> f) & 1)) xf[(size_t)r * NF + f] += acc[f];
}

// ---------------------------------------------------------------- coarsest level
// dense row-major copy of a block-CSR matrix (M zeroed by the caller)
template <int NF, typename VT>
__global__ void k_mg_dense_build(PtrsA A, double *__restrict__ M, int n) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= A.n_rows) return;
    const VT *vals = (const VT *)A.vals;
    for (int j = A.row_ptr[r]; j < A.row_ptr[r + 1]; ++j) {
        const int c = A.cols[j];
        if (!in_range(c, A.n_rows, GS_DENSE) || !in_range((long long)(r + 1) * NF, (long long)n + 1, GS_DENSE)) continue;
        for (int f = 0; f < NF; ++f)
            for (int g = 0; g < NF; ++g)
                M[(size_t)(r * NF + f) * n + c * NF + g] = (double)vals[(size_t)j * NF * NF + f * NF + g];
    }
}

// Inverse of the coarsest operator by in-place Gauss-Jordan elimination with
// partial pivoting, one CTA, the matrix held in dynamic shared memory
// (n <= kMgCoarseMax, n*n doubles).  Step k: swap the pivot row into place,
// divide row k by the pivot p (a_kk := 1/p), and for every other row i with
// f = a_ik subtract f * row k (a_ik := -f/p).  The row interchanges are undone
// at the end by swapping columns in reverse order.  A zero pivot column is
// replaced by a unit pivot, so a singular coarse operator weakens the
// preconditioner instead of producing non-finite values.  Pivot ties go to the
// lowest row: the result is deterministic.
__global__ void k_mg_dense_invert(const double *__restrict__ M, double *__restrict__ Inv, int n) {
    extern __shared__ double a[];
    __shared__ int perm[kMgCoarseMax], colsrc[kMgCoarseMax];
    __shared__ double fk[kMgCoarseMax], prow[kMgCoarseMax], oldk[kMgCoarseMax];
    __shared__ int piv_s, unit_s;
    const int t = threadIdx.x, nt = blockDim.x, lane = t & 31, w = t >> 5;
    for (int q = t; q < n * n; q += nt) a[q] = M[q];
    __syncthreads();
    // elimination threads: column j, row group g of G (each keeps its pivot-row
    // entry in a register; the multipliers fk[i] are broadcast reads)
    const int G = nt / n, j = t % n, g = t / n;
    for (int k = 0; k < n; ++k) {
        // 1. pivot: the first row of largest |a_ik|, i >= k (warp 0)
        if (w == 0) {
            double best = -1.0;
            int bi = k;
            for (int i = k + lane; i < n; i += 32) {
                const double v = fabs(a[i * n + k]);
                if (v > best) { best = v; bi = i; }
            }
            for (int o = 16; o > 0; o >>= 1) {
                const double ov = __shfl_down_sync(0xffffffffu, best, o);
                const int oi = __shfl_down_sync(0xffffffffu, bi, o);
                if (ov > best || (ov == best && oi < bi)) { best = ov; bi = oi; }
            }
            if (lane == 0) {
                const int unit = !(best > 0.0);  // no nonzero pivot: unit pivot in place
                piv_s = unit ? k : bi;
                unit_s = unit;
                perm[k] = piv_s;
            }
        }
        __syncthreads();
        // 2. stage the swapped-in pivot row scaled by 1/pivot, the old row k
        //    (it moves to row p) and column k of the row-swapped matrix
        const int p = piv_s, unit = unit_s;
        const double pinv = 1.0 / (unit ? 1.0 : a[p * n + k]);
        if (t < n) {
            const double rp = (unit && t == k) ? 1.0 : a[p * n + t];
            prow[t] = (t == k) ? pinv : rp * pinv;
            oldk[t] = a[k * n + t];
        } else if (t < 2 * n) {
            const int i = t - n;
            const int src = (i == k) ? p : (i == p ? k : i);
            fk[i] = (unit && i == k) ? 1.0 : a[src * n + k];
        }
        __syncthreads();
        // 3. row k := pivot row; every other row i: a_ij -= fk_i prow_j, a_ik := -fk_i / pivot
        if (g < G) {
            const double pj = prow[j], ok = oldk[j];
            for (int i = g; i < n; i += G) {
                if (i == k) { a[k * n + j] = pj; continue; }
                const double f = fk[i];
                const double v = (i == p) ? ok : a[i * n + j];
                if (j == k) a[i * n + j] = -f * pinv;
                else a[i * n + j] = (f != 0.0) ? v - f * pj : v;
            }
        }
        __syncthreads();
    }
    // undo the row interchanges as column interchanges, last first: compose
    // them into one column map and apply it while writing out
    if (t == 0) {
        for (int q = 0; q < n; ++q) colsrc[q] = q;
        for (int k = n - 1; k >= 0; --k) {
            const int p = perm[k];
            const int tmp = colsrc[k]; colsrc[k] = colsrc[p]; colsrc[p] = tmp;
        }
    }
    __syncthreads();
    for (int q = t; q < n * n; q += nt) {
        const int i = q / n, c = q - i * n;
        Inv[q] = a[i * n + colsrc[c]];
    }
}

// x = Inv b (one warp per row)
__global__ void k_mg_dense_apply(const double *__restrict__ Inv, const double *__restrict__ b, double *__restrict__ x,
                                 int n, const int *__restrict__ skip) {
    if (skip && *skip) return;
    const int nw = gridDim.x * (blockDim.x >> 5) * kRowsPerWarp;
    const int lane = threadIdx.x & 31;
    for (int i = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); i < n; i += nw) {
        double s = 0.0;
        for (int j = lane; j < n; j += 32) s += Inv[(size_t)i * n + j] * b[j];
        for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
        if (lane == 0) x[i] = s;
    }
}

// ---------------------------------------------------------------- flexible GMRES glue
// v_k = w / s -> V[k] and the cycle's right-hand side
__global__ void k_gm_next_flex(size_t n, GmresVecs G, int start, double *__restrict__ mg_b) {
    if (G.sc->cycle_done) return;
    const int k = G.sc->k;
    if (!in_range(k, G.sc->restart + 1, GS_KRYLOV_K)) return;  // V holds restart + 1 vectors
    const double ih = 1.0 / (start ? G.sc->beta : G.sc->wnorm);
    double *vn = G.V + (size_t)k * G.n;
    for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x) {
        const double v = G.w[q] * ih;
        vn[q] = v;
        mg_b[q] = v;
    }
}

// w = A z_k, and z_k -> Z[k] (z is the V-cycle's output)
template <int NF, typename VT>
__global__ void k_gm_spmv_keep(PtrsA A, GmresVecs G, double *__restrict__ Z) {
    if (G.sc->cycle_done) return;
    if (!in_range(G.sc->k, G.sc->restart, GS_KRYLOV_K)) return;  // Z holds restart vectors
    double *zk = Z + (size_t)G.sc->k * G.n;
    const int nw = gridDim.x * (blockDim.x >> 5) * kRowsPerWarp;
    for (int rb = (blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5)) * kRowsPerWarp; rb < A.n_rows; rb += nw) {
        const int r = rb + (threadIdx.x & 31) / kLPR;
        double acc[NF];
        row_mv<NF, VT>(A, r, G.z, acc);
        if (r < A.n_rows && (threadIdx.x & (kLPR - 1)) == 0)
#pragma unroll
            for (int f = 0; f < NF; ++f) {
                G.w[(size_t)r * NF + f] = acc[f];
                zk[(size_t)r * NF + f] = G.z[(size_t)r * NF + f];
            }
    }
}

// x += Z y
__global__ void k_gm_update_x_flex(size_t n, GmresVecs G, const double *__restrict__ Z) {
    const GScalars *sc = G.sc;
    if (sc->done) return;
    const int k = sc->k;
    if (!in_range(k, sc->restart + 1, GS_KRYLOV_K)) return;
    for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x) {
        double s = 0.0;
        for (int i = 0; i < k; ++i) s += sc->y[i] * Z[(size_t)i * n + q];
        G.x[q] += s;
    }
}

}  // namespace
}  // namespace gw
