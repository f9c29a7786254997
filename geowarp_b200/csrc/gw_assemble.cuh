// Deterministic residual and element-tangent assembly for the 2D kinds
// (solid and u-p).  Replaces the per-particle atomic scatter of the
// reference's residual kernels (mpm/mpm_utils.py:586-596, 990-1017: one
// wp.atomic_add per node and field) and of its coloured-AD Jacobian
// (solvers/sparse_differentiation.py:213-401).
//
// Two passes over the particles in cell-sorted order:
//
//  1. k_particle_q (one thread per particle): kinematics, return map and
//     stress, written back as F_new / b_new / sigma like the reference, and
//     the particle's stress resultants Q (FP64) and their derivatives
//     Dm = dQ/dtheta (FP64, or FP32 in mixed precision) with respect to the
//     gathered nodal quantities theta (displacement gradient H, ubar, and for
//     u-p pbar, grad p, dp~).  These go to a scratch record per sorted
//     particle; there is no scatter in this pass.
//
//  2. k_cell_scatter (one warp per occupied cell, nine colour phases): the
//     particles of one cell share their lower corner, so they touch the same
//     3 x 3 nodes.  A warp stages each of its cell's records in shared memory
//     in sorted order and its lanes own the cell's residual entries (slot,
//     field) and element blocks (slot a, slot b), accumulated in registers
//     from per-slot columns shared by the warp.  Cells of one colour (cx mod 3, cy mod 3) are
//     at least three cells apart, so their node sets -- and therefore the
//     residual rows and matrix rows they touch -- are disjoint: the warp adds
//     its sums with plain read-modify-writes, without atomics.  The summation
//     order (phases, cells, particles in sorted order) is fixed, so R and K
//     are bitwise reproducible from run to run.
//
// The residual rows follow residual_rows(): for field j < D
//   r_a[j] = -sum_k G_a[k] Q_U[k][j] + W_a (Q_S g_j + fx_j) + [j = D-1] W_a Q_PEN,
// and for the pressure row (u-p)
//   r_a[D] = W_a Q_M1 + sum_k G_a[k] Q_M2[k] + (W_a - Wavg_a) Q_M3,
// and the element blocks are K_ab = -d r_a / d u_b with
//   d Q_q / d u_b[g] = C_b[q][g] = sum_k Dm[q][TH + k D + g] G_b[k] + [g = D-1] Dm[q][TU] W_b
// (pressure column: Dm[q][TP] W_b + Dm[q][TD] (W_b - Wavg_b) + sum_k Dm[q][TG+k] G_b[k]).
#pragma once
#include "gw_step_kernels.cuh"

namespace gw {
namespace {  // internal linkage: each translation unit compiles the kernels it launches

// Scratch record of one sorted particle: doubles x[D], lp[D], Q[NQ], fx[D]
// (point load and traction per unit weight), then VT Dm[NQ][NT]; padded to 32 bytes.
template <int KIND, typename VT>
struct QRecord {
    typedef Layout<KIND> L;
    static const int D = KindTraits<KIND>::D;
    static const int ND = 3 * D + L::NQ;                 // doubles
    static const int NDM = L::NQ * L::NT;                // tangent entries
    static const int BYTES = ((ND * 8 + NDM * (int)sizeof(VT)) + 31) / 32 * 32;
};

// sorted keys -> [start, end) of every occupied cell (cells without particles keep start = end = 0)
__global__ void k_cell_ranges(const int *__restrict__ keys, int n, int n_cells, int *__restrict__ cstart,
                              int *__restrict__ cend) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const int k = keys[t];
    if (!in_range(k, n_cells, GS_ASSEMBLE)) return;
    if (t == 0 || keys[t - 1] != k) cstart[k] = t;
    if (t == n - 1 || keys[t + 1] != k) cend[k] = t + 1;
}

// Pass 1: one thread per particle in sorted order.
template <int KIND, bool WANT_K, typename VT, int MODEL = -1>
__global__ void __launch_bounds__(kThreads) k_particle_q(LaunchConst c, PtrsP p, const int *__restrict__ perm,
                                                         const double *__restrict__ u_new,
                                                         const double *__restrict__ u_old,
                                                         unsigned char *__restrict__ scratch,
                                                         double *__restrict__ force) {
    typedef KindTraits<KIND> KT;
    typedef Layout<KIND> L;
    typedef QRecord<KIND, VT> RC;
    const int D = KT::D;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= p.n) return;
    const int pid = perm[t];
    double x[D], lp[D], Fo[9], bo[9];
    for (int k = 0; k < D; ++k) { x[k] = p.x[pid * D + k]; lp[k] = p.lp[pid * D + k]; }
    for (int k = 0; k < 9; ++k) { Fo[k] = p.F_old[(size_t)pid * 9 + k]; bo[k] = p.b_old[(size_t)pid * 9 + k]; }
    const double E = p.E ? p.E[pid] : c.E0;
    const double pi_old = p.pi_old ? p.pi_old[pid] : 0.0;
    const double pi_new = p.pi_new ? p.pi_new[pid] : 0.0;
    PState<KIND> s;
    if (!particle_shape<KIND>(c.g, x, lp, s)) atomicOr(&g_status, ST_RANGE);
    particle_gather<KIND>(u_new, u_old, s);
    PEval<KIND> ev;
    particle_eval<KIND, WANT_K, MODEL>(c, s, x, Fo, bo, E, pi_old, pi_new, c.st.p_vol, ev);
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            p.F_new[(size_t)pid * 9 + i * 3 + j] = ev.F_new[i][j];
            p.b_new[(size_t)pid * 9 + i * 3 + j] = ev.b_new[i][j];
            p.sigma[(size_t)pid * 9 + i * 3 + j] = ev.sigma[i][j];
        }
    if (p.pi_new) p.pi_new[pid] = ev.pi_new;
    if (ev.pen_on && force) atomicAdd(force, -ev.pen);
    const double ramp = (c.st.current_step + 1.0) / c.st.total_steps;
    double *rd = (double *)(scratch + (size_t)t * RC::BYTES);
    bool bad = false;
    for (int k = 0; k < D; ++k) {
        rd[k] = x[k];
        rd[D + k] = lp[k];
        double f = (p.ext_flag && p.ext_flag[pid]) ? c.st.point_load[k] * ramp : 0.0;
        if (KIND == GW_KIND_COUPLED2D && p.trac_flag && p.trac_flag[pid]) f += c.st.traction[k] * c.g.h[k] / c.st.PPD;
        rd[2 * D + L::NQ + k] = f;
    }
    for (int q = 0; q < L::NQ; ++q) {
        rd[2 * D + q] = ev.Q[q];
        if (!isfinite(ev.Q[q])) bad = true;
    }
    if (bad) atomicOr(&g_status, ST_NAN);
    if (!WANT_K) return;
    VT *rm = (VT *)(rd + RC::ND);
    for (int q = 0; q < L::NQ; ++q)
        for (int tt = 0; tt < L::NT; ++tt) rm[q * L::NT + tt] = (VT)ev.Dm[q][tt];
}

// Pass 2: one warp per cell of colour (kx, ky); cells (kx + 3i, ky + 3j).
// Per particle of the cell (sorted order) the warp stages the record, two
// lanes evaluate the shape functions of the two axes, nine lanes form the
// slot weights and the columns C_b[q][g] = dQ_q / du_b[g] of the nine slots in
// shared memory, and then every lane adds its residual entries and its whole
// element blocks (a, b) from the shared columns.
constexpr int kScatterWarps = 4;  // warps per CTA
template <int KIND, typename VT>
struct ScatterShared {
    typedef Layout<KIND> L;
    static const int NF = KindTraits<KIND>::NF;
    double W[9], Wavg[9], G[9][2];   // cell-frame slots (0 outside the particle's span)
    double C[9][L::NQ][NF];          // dQ/du of each slot
    double axw[2][3], axg[2][3], axa[2][3];
    int axoff[2], axspan[2];
    unsigned int inspan;              // bit a: cell slot a lies in the particle's span
};

template <int KIND, bool WANT_K, typename VT>
__global__ void __launch_bounds__(32 * kScatterWarps, 6) k_cell_scatter(LaunchConst c, int kx, int ky,
                                                                     const int *__restrict__ cstart,
                                                                     const int *__restrict__ cend,
                                                                     const unsigned char *__restrict__ scratch,
                                                                     const uint8_t *__restrict__ free_mask, PtrsA A,
                                                                     double *__restrict__ R) {
    typedef KindTraits<KIND> KT;
    typedef Layout<KIND> L;
    typedef QRecord<KIND, VT> RC;
    typedef ScatterShared<KIND, VT> SS;
    static_assert(KT::D == 2, "the cell scatter covers the 2D kinds");
    const int D = 2, NF = KT::NF, NS = 9;
    constexpr int NR = NS * NF;             // residual entries of a cell
    constexpr int NB = NS * NS;             // element blocks of a cell
    constexpr int PERB = (NB + 31) / 32;    // blocks per lane
    constexpr int PB = NF == 2 ? 4 : 2;   // particles staged per batch (static shared memory < 48 KB)
    __shared__ __align__(16) unsigned char rec_sh[kScatterWarps][PB][RC::BYTES];
    __shared__ SS ssh[kScatterWarps][PB];
    __shared__ unsigned char inflag[kScatterWarps][PB][NS];
    const int lane = threadIdx.x & 31, wl = threadIdx.x >> 5;
    const int ncx = c.g.n_grid[0], ncy = c.g.n_grid[1];
    const int nx3 = (ncx - kx + 2) / 3, ny3 = (ncy - ky + 2) / 3;
    const int cw = blockIdx.x * kScatterWarps + wl;
    if (cw >= nx3 * ny3) return;  // whole warps only: warp-level syncs below
    const int cx = kx + 3 * (cw % nx3), cy = ky + 3 * (cw / nx3);
    const int cell = cx + cy * ncx;
    const int p0 = cstart[cell], p1 = cend[cell];
    if (p1 <= p0) return;
    const double ramp = (c.st.current_step + 1.0) / c.st.total_steps;
    const double gv = -c.st.gravity_mag * (c.st.gravity_full ? 1.0 : ramp);
    double racc = 0.0;
    double kacc[PERB][NF][NF];
#pragma unroll
    for (int e = 0; e < PERB; ++e)
        for (int f = 0; f < NF; ++f)
            for (int g = 0; g < NF; ++g) kacc[e][f][g] = 0.0;
    unsigned int touched = 0u;  // bit e: block e of this lane received a contribution
    // The cell's particles go in batches of PB: the set-up sections (staging
    // the records, shape functions, slot weights, columns C_b) run for the
    // whole batch at once, one (particle, axis / slot) per lane, and the
    // accumulation then runs over the batch in sorted order, so the sums are
    // those of one particle at a time.
    constexpr int NCH = RC::BYTES / 16;
    for (int t0 = p0; t0 < p1; t0 += PB) {
        const int np = min(PB, p1 - t0);
        for (int k = lane; k < np * NCH; k += 32) {
            const int pp = k / NCH, ch = k % NCH;
            ((uint4 *)rec_sh[wl][pp])[ch] = ((const uint4 *)(scratch + (size_t)(t0 + pp) * RC::BYTES))[ch];
        }
        __syncwarp();
        if (lane < 2 * np) {  // shape functions: one (particle, axis) per lane
            const int pp = lane >> 1, k = lane & 1;
            const double *rd = (const double *)rec_sh[wl][pp];
            SS &s = ssh[wl][pp];
            Axis ax;
            gimp_axis(rd[k], rd[D + k], c.g.h[k], c.g.inv_h[k], ax);
            for (int i = 0; i < 3; ++i) { s.axw[k][i] = ax.w[i]; s.axg[k][i] = ax.gw[i]; s.axa[k][i] = ax.wavg[i]; }
            s.axoff[k] = ax.lower - (k == 0 ? cx : cy);
            s.axspan[k] = ax.span;
        }
        __syncwarp();
        for (int k = lane; k < np * NS; k += 32) {  // cell slot weights (a particle clamped at the grid edge is offset)
            const int pp = k / NS, sl = k % NS;
            SS &s = ssh[wl][pp];
            const int i0 = sl % 3 - s.axoff[0], i1 = sl / 3 - s.axoff[1];
            const bool in = i0 >= 0 && i0 < s.axspan[0] && i1 >= 0 && i1 < s.axspan[1];
            const double w0 = in ? s.axw[0][i0] : 0.0, w1 = in ? s.axw[1][i1] : 0.0;
            s.W[sl] = w0 * w1;
            s.Wavg[sl] = in ? s.axa[0][i0] * s.axa[1][i1] : 0.0;
            s.G[sl][0] = in ? s.axg[0][i0] * w1 : 0.0;
            s.G[sl][1] = in ? w0 * s.axg[1][i1] : 0.0;
            inflag[wl][pp][sl] = in;
        }
        __syncwarp();
        if (lane < np) {
            unsigned int bits = 0u;
            for (int sl = 0; sl < NS; ++sl) bits |= (unsigned int)inflag[wl][lane][sl] << sl;
            ssh[wl][lane].inspan = bits;
        }
        __syncwarp();
        if (WANT_K)
            for (int k = lane; k < np * NS; k += 32) {  // columns of slot b of particle pp
                const int pp = k / NS, b = k % NS;
                SS &s = ssh[wl][pp];
                if (!((s.inspan >> b) & 1u)) continue;
                const VT *Dm = (const VT *)((const double *)rec_sh[wl][pp] + RC::ND);
                const double Wb = s.W[b], Gb0 = s.G[b][0], Gb1 = s.G[b][1];
                for (int q = 0; q < L::NQ; ++q) {
                    const VT *dq = Dm + q * L::NT;
                    s.C[b][q][0] = (double)dq[L::TH + 0] * Gb0 + (double)dq[L::TH + D] * Gb1;
                    s.C[b][q][1] = (double)dq[L::TH + 1] * Gb0 + (double)dq[L::TH + D + 1] * Gb1 + (double)dq[L::TU] * Wb;
                    if (NF > D)
                        s.C[b][q][NF - 1] = (double)dq[L::TP] * Wb + (double)dq[L::TD] * (Wb - s.Wavg[b]) +
                                            (double)dq[L::TG] * Gb0 + (double)dq[L::TG + 1] * Gb1;
                }
            }
        __syncwarp();
        for (int pp = 0; pp < np; ++pp) {
            const SS &s = ssh[wl][pp];
            const double *rd = (const double *)rec_sh[wl][pp];
            const double *Q = rd + 2 * D;
            const double *fx = rd + 2 * D + L::NQ;
            if (lane < NR) {  // residual entry (slot a, field f)
                const int a = lane / NF, f = lane % NF;
                if ((s.inspan >> a) & 1u) {
                    const double Wa = s.W[a];
                    double v;
                    if (f < D) {
                        v = -(s.G[a][0] * Q[L::QU + f] + s.G[a][1] * Q[L::QU + D + f]);
                        v += Wa * (Q[L::QS] * (f == D - 1 ? gv : 0.0) + fx[f]);
                        if (f == D - 1) v += Wa * Q[L::QPEN];
                    } else {
                        v = Wa * Q[L::QM1] + (Wa - s.Wavg[a]) * Q[L::QM3] + s.G[a][0] * Q[L::QM2] + s.G[a][1] * Q[L::QM2 + 1];
                    }
                    racc += v;
                }
            }
            if (WANT_K) {
#pragma unroll
                for (int e = 0; e < PERB; ++e) {
                    const int blk = lane + 32 * e;
                    if (blk >= NB) break;
                    const int a = blk / NS, b = blk % NS;
                    if (!((s.inspan >> a) & 1u) || !((s.inspan >> b) & 1u)) continue;
                    const double Wa = s.W[a], Ga0 = s.G[a][0], Ga1 = s.G[a][1];
#pragma unroll
                    for (int g = 0; g < NF; ++g) {
#pragma unroll
                        for (int f = 0; f < D; ++f) {
                            double v = -(Ga0 * s.C[b][L::QU + f][g] + Ga1 * s.C[b][L::QU + D + f][g]);
                            if (f == D - 1) v += Wa * gv * s.C[b][L::QS][g] + Wa * s.C[b][L::QPEN][g];
                            kacc[e][f][g] -= v;
                        }
                        if (NF > D) {
                            const double v = Wa * s.C[b][L::QM1][g] + (Wa - s.Wavg[a]) * s.C[b][L::QM3][g] +
                                             Ga0 * s.C[b][L::QM2][g] + Ga1 * s.C[b][L::QM2 + 1][g];
                            kacc[e][NF - 1][g] -= v;
                        }
                    }
                    touched |= 1u << e;
                }
            }
        }
        __syncwarp();  // the next batch reuses the staging buffers
    }
    // exclusive writes: no other cell of this colour touches these rows
    if (lane < NR) {
        const int ac = lane / NF, f = lane % NF;
        const int nxi = cx + ac % 3, nyi = cy + ac / 3;
        if (nxi <= ncx && nyi <= ncy) {
            const int node = nxi + nyi * (ncx + 1);
            const uint8_t fm = free_mask[node];
            if ((fm >> f) & 1) {
                const int row = A.node2row[node];
                if (in_range(row, A.n_rows, GS_ASSEMBLE)) {
                    if (!isfinite(racc)) atomicOr(&g_status, ST_NAN);
                    R[(size_t)row * NF + f] += racc;
                }
            }
        }
    }
    if (!WANT_K) return;
    VT *vals = (VT *)A.vals;
#pragma unroll
    for (int e = 0; e < PERB; ++e) {
        if (!((touched >> e) & 1u)) continue;
        const int blk = lane + 32 * e;
        const int ac = blk / NS, bc = blk % NS;
        const int ax = cx + ac % 3, ay = cy + ac / 3, bx = cx + bc % 3, by = cy + bc / 3;
        if (ax > ncx || ay > ncy || bx > ncx || by > ncy) continue;
        const int na = ax + ay * (ncx + 1), nb = bx + by * (ncx + 1);
        const uint8_t fa = free_mask[na], fb = free_mask[nb];
        if (!fa || !fb) continue;
        const int row = A.node2row[na];
        if (!in_range(row, A.n_rows, GS_ASSEMBLE)) continue;
        const int o[3] = {bx - ax, by - ay, 0};
        const int slot = stencil_slot(A.stencil, A.mw, na, offset_bit<2>(o));
        if (slot < 0) { atomicOr(&g_status, ST_RANGE); continue; }
        const long long jb = (long long)A.row_ptr[row] + slot;
        if (!in_range(jb, A.nnzb, GS_ASSEMBLE)) continue;
        VT *dst = vals + (size_t)jb * NF * NF;
#pragma unroll
        for (int f = 0; f < NF; ++f)
#pragma unroll
            for (int g = 0; g < NF; ++g)
                if (((fa >> f) & 1) && ((fb >> g) & 1)) dst[f * NF + g] = (VT)((double)dst[f * NF + g] + kacc[e][f][g]);
    }
}

}  // namespace
}  // namespace gw
