// Fused coarse tail of the multigrid V-cycle.
//
// Below a few thousand block rows a V-cycle level is latency bound: each of
// its kernels (smoothing, residual, restriction, prolongation) runs a chain of
// two or three dependent loads over a few rows per warp, and the launch gap
// between dependent kernels costs as much as the kernel itself.  k_mg_tail
// runs every level from l0 down to the dense coarsest one and back up in ONE
// launch of one thread-block cluster: the phases are separated by cluster
// barriers (hardware barrier.cluster, release/acquire at cluster scope)
// instead of kernel boundaries, and the whole cluster (up to 16 SMs) works on
// each phase.
//
// Every phase does the same per-row arithmetic, in the same order, as the
// separate kernels (k_mg_presmooth2, k_mg_jacobi, k_mg_residual,
// k_mg_restrict, k_mg_prolong, k_mg_dense_apply), and the buffers alternate
// the same way, so the V-cycle's output is bitwise the same with or without
// the fused tail.  Vectors written inside the kernel are read through L2
// (ld.global.cg), never through the non-coherent L1 path.
#pragma once
#include <cooperative_groups.h>

#include "gw_mg.cuh"

namespace gw {
namespace {  // internal linkage: each translation unit compiles the kernels it launches

constexpr int kTailThreads = 1024;

struct TailLevel {
    PtrsA A;  // FP64 values (coarse levels)
    Lat L;
    const double *Minv;
    double *b, *x, *x2, *r;
    const uint8_t *fixed;
    int sweeps;
};

struct TailArgs {
    int l0, last;  // levels l0 .. last-1 are smoothed, level last is solved with the dense inverse
    TailLevel lv[kMgMaxLevels];
    const double *dInv;
    int dn;
    double omega;
    const int *skip;
};

struct ClusterIdx {
    int tid, nthreads, gwarp, nwarps;
};

template <int NF>
__device__ __forceinline__ void ldcg_vec(const double *p, double out[NF]) {
    if constexpr (NF == 2 || NF == 4) {
#pragma unroll
        for (int q = 0; q < NF / 2; ++q) {
            const double2 v = __ldcg(reinterpret_cast<const double2 *>(p) + q);
            out[2 * q] = v.x;
            out[2 * q + 1] = v.y;
        }
    } else {
#pragma unroll
        for (int g = 0; g < NF; ++g) out[g] = __ldcg(p + g);
    }
}

// row_mv<NF, double> with x read through L2
template <int NF>
__device__ __forceinline__ void tail_row_mv(const PtrsA &A, int r, const double *x, double acc[NF]) {
    const int lane = threadIdx.x & (kLPR - 1);
#pragma unroll
    for (int f = 0; f < NF; ++f) acc[f] = 0.0;
    const int s = r < A.n_rows ? A.row_ptr[r] : 0, e = r < A.n_rows ? A.row_ptr[r + 1] : 0;
    const double *vals = (const double *)A.vals;
#pragma unroll 2
    for (int j = s + lane; j < e; j += kLPR) {
        const int col = A.cols[j];
        if (!in_range(col, A.n_rows, GS_ROW_MV)) continue;
        double xv[NF], bv[NF * NF];
        ldcg_vec<NF>(x + (size_t)col * NF, xv);
        load_block<NF, double>(vals + (size_t)j * NF * NF, bv);
#pragma unroll
        for (int f = 0; f < NF; ++f)
#pragma unroll
            for (int g = 0; g < NF; ++g) acc[f] += bv[f * NF + g] * xv[g];
    }
#pragma unroll
    for (int f = 0; f < NF; ++f)
#pragma unroll
        for (int o = kLPR / 2; o > 0; o >>= 1) acc[f] += __shfl_down_sync(0xffffffffu, acc[f], o, kLPR);
}

// x_out = x_in + omega Minv (b - A x_in), or omega Minv b from a zero start
template <int NF>
__device__ void tail_jacobi(const ClusterIdx &ci, const TailLevel &v, const double *b, const double *x_in,
                            double *x_out, double omega, bool zero_init) {
    const PtrsA &A = v.A;
    if (zero_init) {
        for (int r = ci.tid; r < A.n_rows; r += ci.nthreads) {
            double t[NF], z[NF];
#pragma unroll
            for (int f = 0; f < NF; ++f) t[f] = __ldcg(b + (size_t)r * NF + f);
            apply_minv<NF>(v.Minv, r, t, z);
#pragma unroll
            for (int f = 0; f < NF; ++f) x_out[(size_t)r * NF + f] = omega * z[f];
        }
        return;
    }
    const int nw = ci.nwarps * kRowsPerWarp;
    for (int rb = ci.gwarp * kRowsPerWarp; rb < A.n_rows; rb += nw) {
        const int r = rb + (threadIdx.x & 31) / kLPR;
        double acc[NF];
        tail_row_mv<NF>(A, r, x_in, acc);
        if (r < A.n_rows && (threadIdx.x & (kLPR - 1)) == 0) {
            double t[NF], z[NF];
#pragma unroll
            for (int f = 0; f < NF; ++f) t[f] = __ldcg(b + (size_t)r * NF + f) - acc[f];
            apply_minv<NF>(v.Minv, r, t, z);
#pragma unroll
            for (int f = 0; f < NF; ++f) x_out[(size_t)r * NF + f] = __ldcg(x_in + (size_t)r * NF + f) + omega * z[f];
        }
    }
}

// both zero-start sweeps (k_mg_presmooth2)
template <int NF>
__device__ void tail_presmooth2(const ClusterIdx &ci, const TailLevel &v, const double *b, double *x_out,
                                double omega) {
    const PtrsA &A = v.A;
    const int nw = ci.nwarps * kRowsPerWarp;
    const int lane = threadIdx.x & (kLPR - 1);
    const double *vals = (const double *)A.vals;
    for (int rb = ci.gwarp * kRowsPerWarp; rb < A.n_rows; rb += nw) {
        const int r = rb + (threadIdx.x & 31) / kLPR;
        double acc[NF];
#pragma unroll
        for (int f = 0; f < NF; ++f) acc[f] = 0.0;
        const int s0 = r < A.n_rows ? A.row_ptr[r] : 0, e0 = r < A.n_rows ? A.row_ptr[r + 1] : 0;
        for (int j = s0 + lane; j < e0; j += kLPR) {
            const int col = A.cols[j];
            if (!in_range(col, A.n_rows, GS_PRESMOOTH)) continue;
            double t[NF], z[NF], bv[NF * NF];
            ldcg_vec<NF>(b + (size_t)col * NF, t);
            load_block<NF, double>(vals + (size_t)j * NF * NF, bv);
            apply_minv<NF>(v.Minv, col, t, z);
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
            double t[NF], z[NF], x1[NF], bb[NF];
#pragma unroll
            for (int f = 0; f < NF; ++f) bb[f] = __ldcg(b + (size_t)r * NF + f);
            apply_minv<NF>(v.Minv, r, bb, z);
#pragma unroll
            for (int f = 0; f < NF; ++f) x1[f] = omega * z[f];
#pragma unroll
            for (int f = 0; f < NF; ++f) t[f] = bb[f] - acc[f];
            apply_minv<NF>(v.Minv, r, t, z);
#pragma unroll
            for (int f = 0; f < NF; ++f) x_out[(size_t)r * NF + f] = x1[f] + omega * z[f];
        }
    }
}

// r = b - A x
template <int NF>
__device__ void tail_residual(const ClusterIdx &ci, const TailLevel &v, const double *b, const double *x,
                              double *r_out) {
    const PtrsA &A = v.A;
    const int nw = ci.nwarps * kRowsPerWarp;
    for (int rb = ci.gwarp * kRowsPerWarp; rb < A.n_rows; rb += nw) {
        const int r = rb + (threadIdx.x & 31) / kLPR;
        double acc[NF];
        tail_row_mv<NF>(A, r, x, acc);
        if (r < A.n_rows && (threadIdx.x & (kLPR - 1)) == 0)
#pragma unroll
            for (int f = 0; f < NF; ++f) r_out[(size_t)r * NF + f] = __ldcg(b + (size_t)r * NF + f) - acc[f];
    }
}

// b_c = P^T r_f (k_mg_restrict)
template <int D, int NF>
__device__ void tail_restrict(const ClusterIdx &ci, const TailLevel &f, const TailLevel &c, const double *rf,
                              double *bc) {
    const PtrsA &Af = f.A, &Ac = c.A;
    const Lat &Lf = f.L, &Lc = c.L;
    for (int R = ci.tid; R < Ac.n_rows; R += ci.nthreads) {
        const int I = Ac.row2node[R];
        if (!in_range(I, lat_size(Lc), GS_RESTRICT)) continue;
        int C[3];
        lat_coords(Lc, I, C);
        double acc[NF];
#pragma unroll
        for (int q = 0; q < NF; ++q) acc[q] = 0.0;
        for (int oz = (D == 3 ? -1 : 0); oz <= (D == 3 ? 1 : 0); ++oz)
            for (int oy = -1; oy <= 1; ++oy)
                for (int ox = -1; ox <= 1; ++ox) {
                    const int cc[3] = {2 * C[0] + ox, 2 * C[1] + oy, 2 * C[2] + oz};
                    bool in = true;
                    for (int k = 0; k < D; ++k) in = in && cc[k] >= 0 && cc[k] < Lf.n[k];
                    if (!in) continue;
                    const int fr = Af.node2row[lat_id(Lf, cc)];
                    if (fr < 0 || !in_range(fr, Af.n_rows, GS_RESTRICT)) continue;
                    double w = 1.0;
                    for (int k = 0; k < D; ++k) w *= p_weight(cc[k], C[k]);
                    const uint8_t fx = f.fixed[fr];
#pragma unroll
                    for (int q = 0; q < NF; ++q)
                        if (!((fx >> q) & 1)) acc[q] += w * __ldcg(rf + (size_t)fr * NF + q);
                }
#pragma unroll
        for (int q = 0; q < NF; ++q) bc[(size_t)R * NF + q] = acc[q];
    }
}

// x_f += P x_c (k_mg_prolong)
template <int D, int NF>
__device__ void tail_prolong(const ClusterIdx &ci, const TailLevel &f, const TailLevel &c, const double *xc,
                             double *xf) {
    const PtrsA &Af = f.A, &Ac = c.A;
    const Lat &Lf = f.L, &Lc = c.L;
    for (int r = ci.tid; r < Af.n_rows; r += ci.nthreads) {
        const int node = Af.row2node[r];
        if (!in_range(node, lat_size(Lf), GS_PROLONG)) continue;
        int cf[3];
        lat_coords(Lf, node, cf);
        int lo[3], cnt[3];
        for (int k = 0; k < 3; ++k) {
            lo[k] = cf[k] >> 1;
            cnt[k] = (k < D && (cf[k] & 1)) ? 2 : 1;
        }
        double acc[NF];
#pragma unroll
        for (int q = 0; q < NF; ++q) acc[q] = 0.0;
        for (int a = 0; a < cnt[0]; ++a)
            for (int bq = 0; bq < cnt[1]; ++bq)
                for (int d = 0; d < cnt[2]; ++d) {
                    const int C[3] = {lo[0] + a, lo[1] + bq, lo[2] + d};
                    const int cid = lat_id(Lc, C);
                    if (!in_range(cid, lat_size(Lc), GS_PROLONG)) continue;
                    const int R = Ac.node2row[cid];
                    if (R < 0 || !in_range(R, Ac.n_rows, GS_PROLONG)) continue;
                    double w = 1.0;
                    for (int k = 0; k < D; ++k) w *= p_weight(cf[k], C[k]);
#pragma unroll
                    for (int q = 0; q < NF; ++q) acc[q] += w * __ldcg(xc + (size_t)R * NF + q);
                }
        const uint8_t fx = f.fixed[r];
#pragma unroll
        for (int q = 0; q < NF; ++q)
            if (!((fx >> q) & 1)) xf[(size_t)r * NF + q] = __ldcg(xf + (size_t)r * NF + q) + acc[q];
    }
}

// x = Inv b on the coarsest level, one warp per row (k_mg_dense_apply)
__device__ void tail_dense(const ClusterIdx &ci, const double *Inv, const double *b, double *x, int n) {
    const int lane = threadIdx.x & 31;
    for (int i = ci.gwarp; i < n; i += ci.nwarps) {
        double s = 0.0;
        for (int j = lane; j < n; j += 32) s += Inv[(size_t)i * n + j] * __ldcg(b + j);
        for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
        if (lane == 0) x[i] = s;
    }
}

// The V-cycle below level l0 - 1 in one cluster launch (grid = one cluster).
template <int D, int NF>
__global__ void __launch_bounds__(kTailThreads, 1) k_mg_tail(TailArgs a) {
    if (a.skip && *a.skip) return;  // uniform over the cluster: no barrier is left waiting
    namespace cg = cooperative_groups;
    cg::cluster_group cl = cg::this_cluster();
    ClusterIdx ci;
    ci.tid = (int)cl.block_rank() * blockDim.x + threadIdx.x;
    ci.nthreads = (int)cl.num_blocks() * blockDim.x;
    ci.gwarp = ci.tid >> 5;
    ci.nwarps = ci.nthreads >> 5;
    double *cur[kMgMaxLevels], *oth[kMgMaxLevels];
    for (int l = a.l0; l < a.last; ++l) {
        const TailLevel &v = a.lv[l], &c = a.lv[l + 1];
        double *x = v.x, *y = v.x2, *t;
        if (v.sweeps >= 2) {
            tail_presmooth2<NF>(ci, v, v.b, y, a.omega);
            cl.sync();
            t = x; x = y; y = t;
            for (int it = 2; it < v.sweeps; ++it) {
                tail_jacobi<NF>(ci, v, v.b, x, y, a.omega, false);
                cl.sync();
                t = x; x = y; y = t;
            }
        } else {
            tail_jacobi<NF>(ci, v, v.b, nullptr, x, a.omega, true);
            cl.sync();
            for (int it = 1; it < v.sweeps; ++it) {
                tail_jacobi<NF>(ci, v, v.b, x, y, a.omega, false);
                cl.sync();
                t = x; x = y; y = t;
            }
        }
        tail_residual<NF>(ci, v, v.b, x, v.r);
        cl.sync();
        tail_restrict<D, NF>(ci, v, c, v.r, c.b);
        cl.sync();
        cur[l] = x;
        oth[l] = y;
    }
    tail_dense(ci, a.dInv, a.lv[a.last].b, a.lv[a.last].x, a.dn);
    cl.sync();
    cur[a.last] = a.lv[a.last].x;
    for (int l = a.last - 1; l >= a.l0; --l) {
        const TailLevel &v = a.lv[l], &c = a.lv[l + 1];
        double *x = cur[l], *y = oth[l], *t;
        tail_prolong<D, NF>(ci, v, c, cur[l + 1], x);
        cl.sync();
        for (int it = 0; it < v.sweeps; ++it) {
            tail_jacobi<NF>(ci, v, v.b, x, y, a.omega, false);
            cl.sync();
            t = x; x = y; y = t;
        }
        cur[l] = x;
    }
}

}  // namespace
}  // namespace gw
