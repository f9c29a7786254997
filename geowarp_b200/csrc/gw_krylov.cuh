// Preconditioned Krylov solvers on the node-block CSR matrix.
//
// Replaces wp.optim.linear.bicgstab + preconditioner(ptype='diag') and the
// host solvers of solvers/quasi_static_solver_2d.py:236-256.  Every iteration
// is a fixed sequence of fused kernels; inner products are FP64 block
// partials summed in block order by the last block to finish (deterministic),
// which also derives the iteration scalars on the device.  Kernels return
// immediately once the device "done" flag is set, so the host can enqueue
// iterations in chunks and poll the flag once per chunk.
#pragma once
#include <cuda_bf16.h>

#include "gw_kernels.cuh"

namespace gw {
namespace {  // internal linkage: each translation unit compiles the kernels it launches

constexpr int kRedBlocks = 148 * 8;  // grid size of reduction kernels (multiple of the B200 SM count)

struct KScalars {
    double rho, rho_old, alpha, omega, beta;
    double rr, bb, tol2;
    double tmp0, tmp1;
    int done, status, iters, max_iter;
    unsigned ticket;
};

// ---------------------------------------------------------------- block reduction helpers
template <int NV>
__device__ __forceinline__ void block_reduce(double v[NV]) {
    __shared__ double sh[NV][32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
    for (int k = 0; k < NV; ++k) {
        double x = v[k];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
        if (lane == 0) sh[k][w] = x;
    }
    __syncthreads();
    if (w == 0) {
#pragma unroll
        for (int k = 0; k < NV; ++k) {
            double x = lane < nw ? sh[k][lane] : 0.0;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
            v[k] = x;
        }
    }
    __syncthreads();
}

// Writes this block's partials; returns true in the last block, whose v[] then
// holds the grid totals (summed in block order).
template <int NV>
__device__ __forceinline__ bool grid_reduce(double v[NV], double *partials, unsigned *ticket) {
    block_reduce<NV>(v);
    __shared__ bool last;
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < NV; ++k) partials[blockIdx.x * NV + k] = v[k];
        __threadfence();
        const unsigned t = atomicAdd(ticket, 1u);
        last = (t == gridDim.x - 1);
    }
    __syncthreads();
    if (!last) return false;
    __threadfence();
    double acc[NV];
#pragma unroll
    for (int k = 0; k < NV; ++k) acc[k] = 0.0;
    // fixed-order sum: thread t sums partials t, t+B, ... then a block tree
    for (int b = threadIdx.x; b < gridDim.x; b += blockDim.x)
#pragma unroll
        for (int k = 0; k < NV; ++k) acc[k] += ((volatile double *)partials)[b * NV + k];
    block_reduce<NV>(acc);
#pragma unroll
    for (int k = 0; k < NV; ++k) v[k] = acc[k];
    if (threadIdx.x == 0) *ticket = 0u;
    return true;
}

// ---------------------------------------------------------------- SpMV
// Vectorised gathers of one NF x NF block and one NF-vector: 16-byte loads
// for NF = 2 and 4 (block values and vectors 16-byte aligned; the entry
// points check it), scalar loads otherwise.  The values and the order they
// are used in are the same either way.
template <int NF, typename VT>
__device__ __forceinline__ void load_block(const VT *__restrict__ p, double out[NF * NF]) {
#pragma unroll
    for (int i = 0; i < NF * NF; ++i) out[i] = (double)p[i];
}
// BF16 blocks (the multigrid's preconditioner copy of a mixed-precision fine
// level): 2x2 blocks in one 8-byte load, otherwise element by element
template <int NF>
__device__ __forceinline__ void load_block_bf16(const __nv_bfloat16 *__restrict__ p, double out[NF * NF]) {
    if constexpr (NF == 2) {
        const uint2 u = *reinterpret_cast<const uint2 *>(p);
        const __nv_bfloat162 a = *reinterpret_cast<const __nv_bfloat162 *>(&u.x);
        const __nv_bfloat162 b = *reinterpret_cast<const __nv_bfloat162 *>(&u.y);
        out[0] = __low2float(a); out[1] = __high2float(a); out[2] = __low2float(b); out[3] = __high2float(b);
    } else {
#pragma unroll
        for (int i = 0; i < NF * NF; ++i) out[i] = __bfloat162float(p[i]);
    }
}
template <> __device__ __forceinline__ void load_block<1, __nv_bfloat16>(const __nv_bfloat16 *__restrict__ p, double out[1]) { load_block_bf16<1>(p, out); }
template <> __device__ __forceinline__ void load_block<2, __nv_bfloat16>(const __nv_bfloat16 *__restrict__ p, double out[4]) { load_block_bf16<2>(p, out); }
template <> __device__ __forceinline__ void load_block<3, __nv_bfloat16>(const __nv_bfloat16 *__restrict__ p, double out[9]) { load_block_bf16<3>(p, out); }
template <> __device__ __forceinline__ void load_block<4, __nv_bfloat16>(const __nv_bfloat16 *__restrict__ p, double out[16]) { load_block_bf16<4>(p, out); }
template <>
__device__ __forceinline__ void load_block<2, float>(const float *__restrict__ p, double out[4]) {
    const float4 v = *reinterpret_cast<const float4 *>(p);
    out[0] = v.x; out[1] = v.y; out[2] = v.z; out[3] = v.w;
}
template <>
__device__ __forceinline__ void load_block<2, double>(const double *__restrict__ p, double out[4]) {
    const double2 a = reinterpret_cast<const double2 *>(p)[0], b = reinterpret_cast<const double2 *>(p)[1];
    out[0] = a.x; out[1] = a.y; out[2] = b.x; out[3] = b.y;
}
template <>
__device__ __forceinline__ void load_block<4, float>(const float *__restrict__ p, double out[16]) {
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const float4 v = reinterpret_cast<const float4 *>(p)[q];
        out[4 * q] = v.x; out[4 * q + 1] = v.y; out[4 * q + 2] = v.z; out[4 * q + 3] = v.w;
    }
}
template <>
__device__ __forceinline__ void load_block<4, double>(const double *__restrict__ p, double out[16]) {
#pragma unroll
    for (int q = 0; q < 8; ++q) {
        const double2 v = reinterpret_cast<const double2 *>(p)[q];
        out[2 * q] = v.x; out[2 * q + 1] = v.y;
    }
}
template <int NF>
__device__ __forceinline__ void load_vec(const double *__restrict__ p, double out[NF]) {
    if constexpr (NF == 2 || NF == 4) {
#pragma unroll
        for (int q = 0; q < NF / 2; ++q) {
            const double2 v = reinterpret_cast<const double2 *>(p)[q];
            out[2 * q] = v.x; out[2 * q + 1] = v.y;
        }
    } else {
#pragma unroll
        for (int g = 0; g < NF; ++g) out[g] = p[g];
    }
}

// Block rows are processed by groups of kLPR lanes, kRowsPerWarp rows per
// warp in flight: the lanes of a group take consecutive blocks of their row
// (kLPR x 16 bytes per step for 2x2 FP32 blocks: one 128-byte line) and a
// warp keeps four independent row_ptr -> cols -> x load chains going.  Every
// lane of a warp runs the same number of row sweeps (rows at or past n_rows
// are idle groups), so the group shuffles can use the full mask.
constexpr int kLPR = 8;
constexpr int kRowsPerWarp = 32 / kLPR;

// acc = (A x)_r summed over the group (valid in the group's first lane); an
// idle group (r >= n_rows) returns zeros.
template <int NF, typename VT>
__device__ __forceinline__ void row_mv(const PtrsA &A, int r, const double *__restrict__ x, double acc[NF]) {
    const int lane = threadIdx.x & (kLPR - 1);
#pragma unroll
    for (int f = 0; f < NF; ++f) acc[f] = 0.0;
    const int s = r < A.n_rows ? A.row_ptr[r] : 0, e = r < A.n_rows ? A.row_ptr[r + 1] : 0;
    const VT *vals = (const VT *)A.vals;
#pragma unroll 2
    for (int j = s + lane; j < e; j += kLPR) {
        const int col = A.cols[j];
        if (!in_range(col, A.n_rows, GS_ROW_MV)) continue;
        double xv[NF], bv[NF * NF];
        load_vec<NF>(x + (size_t)col * NF, xv);
        load_block<NF, VT>(vals + (size_t)j * NF * NF, bv);
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

template <int NF, typename VT>
__global__ void k_spmv(PtrsA A, const double *__restrict__ x, double *__restrict__ y) {
    const int nw = gridDim.x * (blockDim.x >> 5) * kRowsPerWarp;
    for (int rb = (blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5)) * kRowsPerWarp; rb < A.n_rows; rb += nw) {
        const int r = rb + (threadIdx.x & 31) / kLPR;
        double acc[NF];
        row_mv<NF, VT>(A, r, x, acc);
        if (r < A.n_rows && (threadIdx.x & (kLPR - 1)) == 0)
#pragma unroll
            for (int f = 0; f < NF; ++f) y[(size_t)r * NF + f] = acc[f];
    }
}

// y = A^T x (atomic scatter; used by the adjoint)
template <int NF, typename VT>
__global__ void k_spmv_t(PtrsA A, const double *__restrict__ x, double *__restrict__ y) {
    const int nw = gridDim.x * (blockDim.x >> 5) * kRowsPerWarp;
    const int lane = threadIdx.x & (kLPR - 1);
    const VT *vals = (const VT *)A.vals;
    for (int rb = (blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5)) * kRowsPerWarp; rb < A.n_rows; rb += nw) {
        const int r = rb + (threadIdx.x & 31) / kLPR;
        if (r >= A.n_rows) continue;  // no shuffles below
        double xr[NF];
#pragma unroll
        for (int f = 0; f < NF; ++f) xr[f] = x[(size_t)r * NF + f];
        for (int j = A.row_ptr[r] + lane; j < A.row_ptr[r + 1]; j += kLPR) {
            const int col = A.cols[j];
            if (!in_range(col, A.n_rows, GS_ROW_MV)) continue;
            const VT *blk = vals + (size_t)j * NF * NF;
#pragma unroll
            for (int g = 0; g < NF; ++g) {
                double v = 0.0;
#pragma unroll
                for (int f = 0; f < NF; ++f) v += (double)blk[f * NF + g] * xr[f];
                atomicAdd(&y[(size_t)col * NF + g], v);
            }
        }
    }
}

// ---------------------------------------------------------------- preconditioner
// Inverse of one NF x NF block by Gauss-Jordan with partial pivoting, into
// out (row-major).  A singular block falls back to the inverse of its
// diagonal (zero diagonal entries -> 1).
template <int NF>
__device__ __forceinline__ void invert_block(const double Min[NF][NF], double *__restrict__ out) {
    double M[NF][NF], I[NF][NF];
    for (int i = 0; i < NF; ++i)
        for (int j = 0; j < NF; ++j) { M[i][j] = Min[i][j]; I[i][j] = (i == j) ? 1.0 : 0.0; }
    bool ok = true;
    for (int cidx = 0; cidx < NF; ++cidx) {
        int piv = cidx;
        for (int i = cidx + 1; i < NF; ++i)
            if (fabs(M[i][cidx]) > fabs(M[piv][cidx])) piv = i;
        if (M[piv][cidx] == 0.0) { ok = false; break; }
        for (int j = 0; j < NF; ++j) {
            double t = M[cidx][j]; M[cidx][j] = M[piv][j]; M[piv][j] = t;
            t = I[cidx][j]; I[cidx][j] = I[piv][j]; I[piv][j] = t;
        }
        const double d = 1.0 / M[cidx][cidx];
        for (int j = 0; j < NF; ++j) { M[cidx][j] *= d; I[cidx][j] *= d; }
        for (int i = 0; i < NF; ++i) {
            if (i == cidx) continue;
            const double f = M[i][cidx];
            for (int j = 0; j < NF; ++j) { M[i][j] -= f * M[cidx][j]; I[i][j] -= f * I[cidx][j]; }
        }
    }
    for (int i = 0; i < NF; ++i)
        for (int j = 0; j < NF; ++j) {
            if (ok) out[i * NF + j] = I[i][j];
            else out[i * NF + j] = (i == j) ? (Min[i][i] != 0.0 ? 1.0 / Min[i][i] : 1.0) : 0.0;
        }
}

// Minv: per row an NF x NF block.  mode 0: inverse of the scalar diagonal
// (zero diagonal -> 1, as a Jacobi guard), mode 1: inverse of the diagonal block.
template <int NF, typename VT>
__global__ void k_precond_setup(PtrsA A, int D, int mode, double *__restrict__ Minv) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= A.n_rows) return;
    const int node = A.row2node[r];
    const int off[3] = {0, 0, 0};
    const int bit = D == 2 ? offset_bit<2>(off) : offset_bit<3>(off);
    const int slot = stencil_slot(A.stencil, A.mw, node, bit);
    double *out = Minv + (size_t)r * NF * NF;
    if (slot < 0) {  // no diagonal block: identity preconditioner on this row
        for (int i = 0; i < NF; ++i)
            for (int j = 0; j < NF; ++j) out[i * NF + j] = (i == j) ? 1.0 : 0.0;
        return;
    }
    const VT *blk = (const VT *)A.vals + ((size_t)A.row_ptr[r] + slot) * NF * NF;
    double M[NF][NF];
    for (int i = 0; i < NF; ++i)
        for (int j = 0; j < NF; ++j) M[i][j] = (double)blk[i * NF + j];
    if (mode == 0) {
        for (int i = 0; i < NF; ++i)
            for (int j = 0; j < NF; ++j) out[i * NF + j] = (i == j) ? (M[i][i] != 0.0 ? 1.0 / M[i][i] : 1.0) : 0.0;
        return;
    }
    invert_block<NF>(M, out);
}

template <int NF>
__device__ __forceinline__ void apply_minv(const double *__restrict__ Minv, int r, const double in[NF], double out[NF]) {
    const double *M = Minv + (size_t)r * NF * NF;
#pragma unroll
    for (int i = 0; i < NF; ++i) {
        double v = 0.0;
#pragma unroll
        for (int j = 0; j < NF; ++j) v += M[i * NF + j] * in[j];
        out[i] = v;
    }
}

// ---------------------------------------------------------------- BiCGSTAB
struct BicgVecs {
    double *x, *r, *rh, *p, *v, *y, *s, *z, *t;
    const double *b;
    double *Minv, *partials;
    KScalars *sc;
};

// r = b - A x ; rh = r ; p = v = 0 ; dots (r,r), (b,b)
template <int NF, typename VT>
__global__ void k_bicg_init(PtrsA A, BicgVecs V, double rtol) {
    const int nw = gridDim.x * (blockDim.x >> 5) * kRowsPerWarp;
    double d[2] = {0.0, 0.0};
    for (int rb = (blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5)) * kRowsPerWarp; rb < A.n_rows; rb += nw) {
        const int r = rb + (threadIdx.x & 31) / kLPR;
        double acc[NF];
        row_mv<NF, VT>(A, r, V.x, acc);
        if (r < A.n_rows && (threadIdx.x & (kLPR - 1)) == 0) {
#pragma unroll
            for (int f = 0; f < NF; ++f) {
                const size_t i = (size_t)r * NF + f;
                const double rv = V.b[i] - acc[f];
                V.r[i] = rv; V.rh[i] = rv; V.p[i] = 0.0; V.v[i] = 0.0;
                d[0] += rv * rv;
                d[1] += V.b[i] * V.b[i];
            }
        }
    }
    if (grid_reduce<2>(d, V.partials, &V.sc->ticket) && threadIdx.x == 0) {
        KScalars *sc = V.sc;
        sc->rr = d[0]; sc->bb = d[1];
        sc->rho = d[0]; sc->rho_old = 1.0; sc->alpha = 1.0; sc->omega = 1.0;
        sc->tol2 = rtol * rtol * d[1];
        sc->iters = 0; sc->status = 0;
        sc->done = (d[0] <= sc->tol2 || d[1] == 0.0) ? 1 : 0;
        sc->beta = 0.0;
    }
}

// p = r + beta (p - omega v) ; y = Minv p
template <int NF>
__global__ void k_bicg_p(int n_rows, BicgVecs V) {
    if (V.sc->done) return;
    const double beta = V.sc->beta, omega = V.sc->omega;
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n_rows; r += gridDim.x * blockDim.x) {
        double pv[NF], yv[NF];
#pragma unroll
        for (int f = 0; f < NF; ++f) {
            const size_t i = (size_t)r * NF + f;
            pv[f] = V.r[i] + beta * (V.p[i] - omega * V.v[i]);
            V.p[i] = pv[f];
        }
        apply_minv<NF>(V.Minv, r, pv, yv);
#pragma unroll
        for (int f = 0; f < NF; ++f) V.y[(size_t)r * NF + f] = yv[f];
    }
}

// v = A y ; alpha = rho / (rh, v)
template <int NF, typename VT>
__global__ void k_bicg_v(PtrsA A, BicgVecs V) {
    if (V.sc->done) return;
    const int nw = gridDim.x * (blockDim.x >> 5) * kRowsPerWarp;
    double d[1] = {0.0};
    for (int rb = (blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5)) * kRowsPerWarp; rb < A.n_rows; rb += nw) {
        const int r = rb + (threadIdx.x & 31) / kLPR;
        double acc[NF];
        row_mv<NF, VT>(A, r, V.y, acc);
        if (r < A.n_rows && (threadIdx.x & (kLPR - 1)) == 0)
#pragma unroll
            for (int f = 0; f < NF; ++f) {
                const size_t i = (size_t)r * NF + f;
                V.v[i] = acc[f];
                d[0] += V.rh[i] * acc[f];
            }
    }
    if (grid_reduce<1>(d, V.partials, &V.sc->ticket) && threadIdx.x == 0) {
        KScalars *sc = V.sc;
        if (d[0] == 0.0 || !isfinite(d[0])) { sc->status = ST_BREAKDOWN; sc->done = 1; return; }
        sc->alpha = sc->rho / d[0];
    }
}

// s = r - alpha v ; z = Minv s
template <int NF>
__global__ void k_bicg_s(int n_rows, BicgVecs V) {
    if (V.sc->done) return;
    const double alpha = V.sc->alpha;
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n_rows; r += gridDim.x * blockDim.x) {
        double sv[NF], zv[NF];
#pragma unroll
        for (int f = 0; f < NF; ++f) {
            const size_t i = (size_t)r * NF + f;
            sv[f] = V.r[i] - alpha * V.v[i];
            V.s[i] = sv[f];
        }
        apply_minv<NF>(V.Minv, r, sv, zv);
#pragma unroll
        for (int f = 0; f < NF; ++f) V.z[(size_t)r * NF + f] = zv[f];
    }
}

// t = A z ; omega = (t,s)/(t,t)
template <int NF, typename VT>
__global__ void k_bicg_t(PtrsA A, BicgVecs V) {
    if (V.sc->done) return;
    const int nw = gridDim.x * (blockDim.x >> 5) * kRowsPerWarp;
    double d[3] = {0.0, 0.0, 0.0};
    for (int rb = (blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5)) * kRowsPerWarp; rb < A.n_rows; rb += nw) {
        const int r = rb + (threadIdx.x & 31) / kLPR;
        double acc[NF];
        row_mv<NF, VT>(A, r, V.z, acc);
        if (r < A.n_rows && (threadIdx.x & (kLPR - 1)) == 0)
#pragma unroll
            for (int f = 0; f < NF; ++f) {
                const size_t i = (size_t)r * NF + f;
                V.t[i] = acc[f];
                d[0] += acc[f] * V.s[i];
                d[1] += acc[f] * acc[f];
                d[2] += V.s[i] * V.s[i];
            }
    }
    if (grid_reduce<3>(d, V.partials, &V.sc->ticket) && threadIdx.x == 0) {
        KScalars *sc = V.sc;
        sc->omega = (d[1] != 0.0) ? d[0] / d[1] : 0.0;
        sc->tmp0 = d[2];  // ||s||^2: converged already when below tolerance
    }
}

// x += alpha y + omega z ; r = s - omega t ; rho = (rh, r) ; rr = (r, r)
template <int NF>
__global__ void k_bicg_xr(int n_rows, BicgVecs V) {
    if (V.sc->done) return;
    const double alpha = V.sc->alpha, omega = V.sc->omega;
    double d[2] = {0.0, 0.0};
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n_rows; r += gridDim.x * blockDim.x) {
#pragma unroll
        for (int f = 0; f < NF; ++f) {
            const size_t i = (size_t)r * NF + f;
            V.x[i] += alpha * V.y[i] + omega * V.z[i];
            const double rv = V.s[i] - omega * V.t[i];
            V.r[i] = rv;
            d[0] += V.rh[i] * rv;
            d[1] += rv * rv;
        }
    }
    if (grid_reduce<2>(d, V.partials, &V.sc->ticket) && threadIdx.x == 0) {
        KScalars *sc = V.sc;
        sc->iters += 1;
        sc->rr = d[1];
        if (!isfinite(d[1])) { sc->status = ST_NAN; sc->done = 1; return; }
        if (d[1] <= sc->tol2) { sc->done = 1; return; }
        if (sc->iters >= sc->max_iter) { sc->done = 1; return; }
        if (d[0] == 0.0 || omega == 0.0) { sc->status = ST_BREAKDOWN; sc->done = 1; return; }
        sc->beta = (d[0] / sc->rho) * (sc->alpha / omega);
        sc->rho_old = sc->rho;
        sc->rho = d[0];
    }
}

// ---------------------------------------------------------------- CG (SPD; consistent mass)
// init: r = b - A x ; z = Minv r ; p = z ; rz = (r,z)
template <int NF, typename VT>
__global__ void k_cg_init(PtrsA A, BicgVecs V, double rtol) {
    const int nw = gridDim.x * (blockDim.x >> 5) * kRowsPerWarp;
    double d[3] = {0.0, 0.0, 0.0};
    for (int rb = (blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5)) * kRowsPerWarp; rb < A.n_rows; rb += nw) {
        const int r = rb + (threadIdx.x & 31) / kLPR;
        double acc[NF];
        row_mv<NF, VT>(A, r, V.x, acc);
        if (r < A.n_rows && (threadIdx.x & (kLPR - 1)) == 0) {
            double rv[NF], zv[NF];
#pragma unroll
            for (int f = 0; f < NF; ++f) rv[f] = V.b[(size_t)r * NF + f] - acc[f];
            apply_minv<NF>(V.Minv, r, rv, zv);
#pragma unroll
            for (int f = 0; f < NF; ++f) {
                const size_t i = (size_t)r * NF + f;
                V.r[i] = rv[f]; V.z[i] = zv[f]; V.p[i] = zv[f];
                d[0] += rv[f] * zv[f];
                d[1] += rv[f] * rv[f];
                d[2] += V.b[i] * V.b[i];
            }
        }
    }
    if (grid_reduce<3>(d, V.partials, &V.sc->ticket) && threadIdx.x == 0) {
        KScalars *sc = V.sc;
        sc->rho = d[0]; sc->rr = d[1]; sc->bb = d[2];
        sc->tol2 = rtol * rtol * d[2];
        sc->iters = 0; sc->status = 0; sc->beta = 0.0;
        sc->done = (d[1] <= sc->tol2 || d[2] == 0.0) ? 1 : 0;
    }
}

// p = z + beta p (skipped on the first iteration: beta = 0 and p = z already)
template <int NF>
__global__ void k_cg_p(int n_rows, BicgVecs V) {
    if (V.sc->done) return;
    const double beta = V.sc->beta;
    if (beta == 0.0) return;
    for (size_t i = blockIdx.x * blockDim.x + threadIdx.x; i < (size_t)n_rows * NF; i += gridDim.x * blockDim.x)
        V.p[i] = V.z[i] + beta * V.p[i];
}

// q(=v) = A p ; alpha = rz / (p, q)
template <int NF, typename VT>
__global__ void k_cg_q(PtrsA A, BicgVecs V) {
    if (V.sc->done) return;
    const int nw = gridDim.x * (blockDim.x >> 5) * kRowsPerWarp;
    double d[1] = {0.0};
    for (int rb = (blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5)) * kRowsPerWarp; rb < A.n_rows; rb += nw) {
        const int r = rb + (threadIdx.x & 31) / kLPR;
        double acc[NF];
        row_mv<NF, VT>(A, r, V.p, acc);
        if (r < A.n_rows && (threadIdx.x & (kLPR - 1)) == 0)
#pragma unroll
            for (int f = 0; f < NF; ++f) {
                const size_t i = (size_t)r * NF + f;
                V.v[i] = acc[f];
                d[0] += V.p[i] * acc[f];
            }
    }
    if (grid_reduce<1>(d, V.partials, &V.sc->ticket) && threadIdx.x == 0) {
        KScalars *sc = V.sc;
        if (d[0] == 0.0 || !isfinite(d[0])) { sc->status = ST_BREAKDOWN; sc->done = 1; return; }
        sc->alpha = sc->rho / d[0];
    }
}

// x += alpha p ; r -= alpha q ; z = Minv r ; beta = (r,z)_new / (r,z)
template <int NF>
__global__ void k_cg_xr(int n_rows, BicgVecs V) {
    if (V.sc->done) return;
    const double alpha = V.sc->alpha;
    double d[2] = {0.0, 0.0};
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n_rows; r += gridDim.x * blockDim.x) {
        double rv[NF], zv[NF];
#pragma unroll
        for (int f = 0; f < NF; ++f) {
            const size_t i = (size_t)r * NF + f;
            V.x[i] += alpha * V.p[i];
            rv[f] = V.r[i] - alpha * V.v[i];
            V.r[i] = rv[f];
        }
        apply_minv<NF>(V.Minv, r, rv, zv);
#pragma unroll
        for (int f = 0; f < NF; ++f) {
            V.z[(size_t)r * NF + f] = zv[f];
            d[0] += rv[f] * zv[f];
            d[1] += rv[f] * rv[f];
        }
    }
    if (grid_reduce<2>(d, V.partials, &V.sc->ticket) && threadIdx.x == 0) {
        KScalars *sc = V.sc;
        sc->iters += 1;
        sc->rr = d[1];
        if (!isfinite(d[1])) { sc->status = ST_NAN; sc->done = 1; return; }
        if (d[1] <= sc->tol2 || sc->iters >= sc->max_iter) { sc->done = 1; return; }
        sc->beta = d[0] / sc->rho;
        sc->rho = d[0];
    }
}

// ---------------------------------------------------------------- misc vector kernels
__global__ void k_norm2(const double *__restrict__ v, int n, double *__restrict__ partials, unsigned *ticket,
                        double *__restrict__ out) {
    double d[1] = {0.0};
    for (size_t i = blockIdx.x * blockDim.x + threadIdx.x; i < (size_t)n; i += gridDim.x * blockDim.x) d[0] += v[i] * v[i];
    if (grid_reduce<1>(d, partials, ticket) && threadIdx.x == 0) *out = ::sqrt(d[0]);
}

__global__ void k_apply_increment(int n_rows, int nf, const int *__restrict__ row2node, const double *__restrict__ delta,
                                  double *__restrict__ u) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n_rows) return;
    const int node = row2node[r];
    for (int f = 0; f < nf; ++f) u[(size_t)node * nf + f] += delta[(size_t)r * nf + f];
}

// u[node*nf+f] = u_prev[node*nf+f] on the free DOFs of the active rows (bit f
// of free_mask[node]), 0 on their Dirichlet DOFs; other nodes are not written
__global__ void k_predict_increment(int n_rows, int nf, const int *__restrict__ row2node,
                                    const uint8_t *__restrict__ free_mask, const double *__restrict__ u_prev,
                                    double *__restrict__ u) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n_rows) return;
    const int node = row2node[r];
    const unsigned m = free_mask[node];
    for (int f = 0; f < nf; ++f) {
        const size_t i = (size_t)node * nf + f;
        u[i] = ((m >> f) & 1u) ? u_prev[i] : 0.0;
    }
}

}  // namespace
}  // namespace gw

namespace gw {
namespace {  // internal linkage: each translation unit compiles the kernels it launches

// ---------------------------------------------------------------- restarted GMRES(m)
// Right-preconditioned GMRES with classical Gram-Schmidt and a
// re-orthogonalisation pass when needed.  Column k of the Arnoldi process is
// six kernels:
//   spmv:  w = A z_k                       (z_k = Minv v_k)
//   dots:  h_i = (v_i, w), i <= k, and (w, w)   (pass 0); the last block
//          decides the second pass: ||w - V h||^2 = (w, w) - sum h_i^2 below
//          gs_eta2 (w, w) (by default 1/100: the projection removed more than
//          90% of w's norm) means V h lost more than ~10 ulp of orthogonality
//          and the pass is repeated
//   upd:   w -= V h                        (pass 0)
//   dots:  h2_i = (v_i, w)                 (pass 1, only when needed)
//   upd:   w -= V h2 (only when needed) ; ||w||; last block: Hessenberg
//          column, Givens rotation, residual estimate, cycle/convergence
//          flags, k += 1
//   next:  v_k = w / ||w|| ; z_k = Minv v_k
// The skipped pass reads no basis vector, so an Arnoldi step without strong
// cancellation reads the basis twice instead of four times.
// Robust for the nonsymmetric, indefinite Jacobians of the penalty footing
// and the u-p saddle-point systems, on which BiCGSTAB breaks down.
constexpr int kGmresMaxRestart = 128;

struct GScalars {
    // scalar header first: the host polls only this prefix
    double beta, bnorm, tol, resid, wnorm;
    double gs_eta2;  // second Gram-Schmidt pass below this fraction of ||w||^2 left
    int k;           // completed Arnoldi columns in the current cycle
    int cycle_done, done, status, iters, max_iter, restart;
    unsigned ticket;
    int reorth;      // column k takes the second Gram-Schmidt pass
    int reorths;     // second passes taken in this solve
    double H[kGmresMaxRestart + 1][kGmresMaxRestart];
    double cs[kGmresMaxRestart], sn[kGmresMaxRestart];
    double g[kGmresMaxRestart + 1];
    double y[kGmresMaxRestart];
    double h2[kGmresMaxRestart + 1];
};

struct GmresVecs {
    double *x, *w, *V, *Minv, *partials, *z;
    const double *b;
    GScalars *sc;
    size_t n;  // n_rows * NF (stride of V)
};

// w = r = b - A x ; beta = ||r|| ; first cycle also ||b|| and the tolerance
template <int NF, typename VT>
__global__ void k_gm_residual(PtrsA A, GmresVecs G, int first, double rtol) {
    if (G.sc->done) return;
    const int nw = gridDim.x * (blockDim.x >> 5) * kRowsPerWarp;
    double d[2] = {0.0, 0.0};
    for (int rb = (blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5)) * kRowsPerWarp; rb < A.n_rows; rb += nw) {
        const int r = rb + (threadIdx.x & 31) / kLPR;
        double acc[NF];
        row_mv<NF, VT>(A, r, G.x, acc);
        if (r < A.n_rows && (threadIdx.x & (kLPR - 1)) == 0)
#pragma unroll
            for (int f = 0; f < NF; ++f) {
                const size_t i = (size_t)r * NF + f;
                const double rv = G.b[i] - acc[f];
                G.w[i] = rv;
                d[0] += rv * rv;
                d[1] += G.b[i] * G.b[i];
            }
    }
    if (grid_reduce<2>(d, G.partials, &G.sc->ticket) && threadIdx.x == 0) {
        GScalars *sc = G.sc;
        sc->beta = ::sqrt(d[0]);
        if (first) {
            sc->bnorm = ::sqrt(d[1]);
            sc->tol = rtol * sc->bnorm;
            sc->iters = 0;
            sc->status = 0;
        }
        sc->resid = sc->beta;
        sc->k = 0;
        sc->cycle_done = 0;
        sc->g[0] = sc->beta;
        for (int i = 1; i <= kGmresMaxRestart; ++i) sc->g[i] = 0.0;
        if (!isfinite(sc->beta)) { sc->status = ST_NAN; sc->done = 1; sc->cycle_done = 1; }
        else if (sc->beta <= sc->tol || sc->bnorm == 0.0 || sc->iters >= sc->max_iter) { sc->done = 1; sc->cycle_done = 1; }
    }
}

// v_k = w / s ; z_k = Minv v_k   (s = beta at a cycle start, ||w|| afterwards)
template <int NF>
__global__ void k_gm_next(int n_rows, GmresVecs G, int start) {
    if (G.sc->cycle_done) return;
    const int k = G.sc->k;
    if (!in_range(k, G.sc->restart + 1, GS_KRYLOV_K)) return;
    const double ih = 1.0 / (start ? G.sc->beta : G.sc->wnorm);
    double *vn = G.V + (size_t)k * G.n;
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n_rows; r += gridDim.x * blockDim.x) {
        double v[NF], z[NF];
#pragma unroll
        for (int f = 0; f < NF; ++f) { v[f] = G.w[(size_t)r * NF + f] * ih; vn[(size_t)r * NF + f] = v[f]; }
        apply_minv<NF>(G.Minv, r, v, z);
#pragma unroll
        for (int f = 0; f < NF; ++f) G.z[(size_t)r * NF + f] = z[f];
    }
}

// w = A z_k
template <int NF, typename VT>
__global__ void k_gm_spmv(PtrsA A, GmresVecs G) {
    if (G.sc->cycle_done) return;
    const int nw = gridDim.x * (blockDim.x >> 5) * kRowsPerWarp;
    for (int rb = (blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5)) * kRowsPerWarp; rb < A.n_rows; rb += nw) {
        const int r = rb + (threadIdx.x & 31) / kLPR;
        double acc[NF];
        row_mv<NF, VT>(A, r, G.z, acc);
        if (r < A.n_rows && (threadIdx.x & (kLPR - 1)) == 0)
#pragma unroll
            for (int f = 0; f < NF; ++f) G.w[(size_t)r * NF + f] = acc[f];
    }
}

// (v_i, w) for i <= k; block partials reduced in block order by the last block
// (pass 0 also (w, w) as item k + 1, and the decision on pass 1)
__global__ void k_gm_dots(GmresVecs G, int pass) {
    if (G.sc->cycle_done) return;
    if (pass == 1 && !G.sc->reorth) return;  // uniform over the grid
    const int k = G.sc->k;
    if (!in_range(k, G.sc->restart, GS_KRYLOV_K)) return;  // uniform over the grid: no block takes the ticket
    const int m = pass == 0 ? k + 1 : k;                     // last item (k < restart <= kGmresMaxRestart)
    const size_t n = G.n;
    __shared__ double sh[kGmresMaxRestart + 1];
    __shared__ double wsq;
    __shared__ bool last;
    const size_t per = (n + gridDim.x - 1) / gridDim.x;
    const size_t r0 = (size_t)blockIdx.x * per, r1 = min(n, r0 + per);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
    for (int i = warp; i <= m; i += nwarp) {
        const double *vi = i <= k ? G.V + (size_t)i * n : G.w;
        double s = 0.0;
        for (size_t q = r0 + lane; q < r1; q += 32) s += vi[q] * G.w[q];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
        if (lane == 0) sh[i] = s;
    }
    __syncthreads();
    for (int i = threadIdx.x; i <= m; i += blockDim.x) G.partials[(size_t)blockIdx.x * (kGmresMaxRestart + 1) + i] = sh[i];
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        last = (atomicAdd(&G.sc->ticket, 1u) == gridDim.x - 1);
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    // one warp per basis vector: lanes take the block partials in a fixed
    // stride, then a fixed shuffle tree (deterministic)
    for (int i = warp; i <= m; i += nwarp) {
        double s = 0.0;
        for (int bb = lane; bb < (int)gridDim.x; bb += 32)
            s += ((volatile double *)G.partials)[(size_t)bb * (kGmresMaxRestart + 1) + i];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
        if (lane == 0) {
            if (i > k) wsq = s;
            else if (pass == 0) G.sc->H[i][k] = s;
            else G.sc->h2[i] = s;
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        if (pass == 0) {
            double rem = wsq;
            for (int i = 0; i <= k; ++i) rem -= G.sc->H[i][k] * G.sc->H[i][k];
            const int re = !(rem >= G.sc->gs_eta2 * wsq);  // also when rem or wsq is not finite
            G.sc->reorth = re;
            G.sc->reorths += re;
        }
        G.sc->ticket = 0u;
    }
}

// w -= V c (c = H[.][k] on pass 0, h2 on pass 1).  The pass that ends the
// projection closes column k with ||w||, summed as it writes w: pass 0 when
// k_gm_dots decided against a second pass (pass 1 then has nothing to do),
// pass 1 otherwise.
__global__ void k_gm_update(GmresVecs G, int pass) {
    if (G.sc->cycle_done) return;
    GScalars *sc = G.sc;
    const bool second = sc->reorth;  // set by k_gm_dots pass 0; uniform over the grid
    if (pass == 1 && !second) return;  // before reading k: pass 0 has advanced it
    const int k = sc->k;
    if (!in_range(k, sc->restart, GS_KRYLOV_K)) return;  // uniform over the grid
    const size_t n = G.n;
    __shared__ double coef[kGmresMaxRestart + 1];
    for (int i = threadIdx.x; i <= k; i += blockDim.x) coef[i] = pass == 0 ? sc->H[i][k] : sc->h2[i];
    __syncthreads();
    double d[1] = {0.0};
    for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x) {
        double w = G.w[q];
        for (int i = 0; i <= k; ++i) w -= coef[i] * G.V[(size_t)i * n + q];
        G.w[q] = w;
        d[0] += w * w;
    }
    if (pass == 0 && second) return;  // pass 1 closes the column
    if (grid_reduce<1>(d, G.partials, &sc->ticket) && threadIdx.x == 0) {
        if (pass == 1)
            for (int i = 0; i <= k; ++i) sc->H[i][k] += sc->h2[i];
        const double hn = ::sqrt(d[0]);
        sc->wnorm = hn;
        sc->H[k + 1][k] = hn;
        for (int i = 0; i < k; ++i) {  // previous rotations
            const double a = sc->H[i][k], b2 = sc->H[i + 1][k];
            sc->H[i][k] = sc->cs[i] * a + sc->sn[i] * b2;
            sc->H[i + 1][k] = -sc->sn[i] * a + sc->cs[i] * b2;
        }
        const double a = sc->H[k][k], b2 = sc->H[k + 1][k];
        const double rr = ::sqrt(a * a + b2 * b2);
        double c = 1.0, s = 0.0;
        if (rr > 0.0) { c = a / rr; s = b2 / rr; }
        sc->cs[k] = c;
        sc->sn[k] = s;
        sc->H[k][k] = rr;
        sc->H[k + 1][k] = 0.0;
        sc->g[k + 1] = -s * sc->g[k];
        sc->g[k] = c * sc->g[k];
        sc->resid = fabs(sc->g[k + 1]);
        sc->iters += 1;
        sc->k = k + 1;
        if (!isfinite(sc->resid)) { sc->status = ST_NAN; sc->cycle_done = 1; sc->done = 1; return; }
        if (sc->resid <= sc->tol || hn == 0.0 || k + 1 >= sc->restart || sc->iters >= sc->max_iter) sc->cycle_done = 1;
    }
}

// end of a cycle: y = H^{-1} g by back substitution (one thread)
__global__ void k_gm_solve_y(GScalars *sc) {
    if (threadIdx.x != 0 || blockIdx.x != 0 || sc->done) return;
    const int k = sc->k;
    if (!in_range(k, sc->restart + 1, GS_KRYLOV_K)) return;
    for (int i = k - 1; i >= 0; --i) {
        double s = sc->g[i];
        for (int q = i + 1; q < k; ++q) s -= sc->H[i][q] * sc->y[q];
        sc->y[i] = (sc->H[i][i] != 0.0) ? s / sc->H[i][i] : 0.0;
    }
}

// x += Minv (V y)
template <int NF>
__global__ void k_gm_update_x(int n_rows, GmresVecs G) {
    const GScalars *sc = G.sc;
    if (sc->done) return;
    const int k = sc->k;
    if (!in_range(k, sc->restart + 1, GS_KRYLOV_K)) return;
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n_rows; r += gridDim.x * blockDim.x) {
        double u[NF], z[NF];
#pragma unroll
        for (int f = 0; f < NF; ++f) {
            double s = 0.0;
            for (int i = 0; i < k; ++i) s += sc->y[i] * G.V[(size_t)i * G.n + (size_t)r * NF + f];
            u[f] = s;
        }
        apply_minv<NF>(G.Minv, r, u, z);
#pragma unroll
        for (int f = 0; f < NF; ++f) G.x[(size_t)r * NF + f] += z[f];
    }
}

}  // namespace
}  // namespace gw
