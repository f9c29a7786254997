// Shared kernel-side definitions: particle / matrix pointer bundles, the
// stencil-slot lookup, the device status word and the index guards.
#pragma once
#include "gw_particle.cuh"

namespace gw {

// Device globals shared by every translation unit of the library (relocatable
// device code): defined in the one that sets GW_DEFINE_DEVICE_GLOBALS.
#ifdef GW_DEFINE_DEVICE_GLOBALS
#define GW_DEVICE_GLOBAL __device__
#else
#define GW_DEVICE_GLOBAL extern __device__
#endif
// Device status word: bit 0 range error, bit 1 non-finite value, bit 2 Krylov breakdown.
GW_DEVICE_GLOBAL int g_status;
// first failed index guard (site, value): see in_range below
GW_DEVICE_GLOBAL int g_guard_site;
GW_DEVICE_GLOBAL long long g_guard_value;

namespace {  // internal linkage: each translation unit compiles the kernels it launches

constexpr int ST_RANGE = 1, ST_NAN = 2, ST_BREAKDOWN = 4;

// Index guards.  Indices the kernels compute from a column array, a stencil,
// a coarse transfer list or a Krylov counter, and row-map lookups wherever the
// kernel knows the node count, are checked against the extent of the array
// they address before the access (the matrix-only kernels trust the fine rows'
// row2node written by gw_compact_rows).  A failed check skips the
// access, sets ST_RANGE and records the first failing site and its value
// (gw_guard_read), so a corrupted pattern surfaces as GW_ERANGE on the host
// instead of as a memory fault.
enum GuardSite {
    GS_NONE = 0, GS_ROW_MV, GS_COARSE_FLAGS, GS_COARSE_STENCIL, GS_PATTERN_FILL, GS_RAP_COARSE, GS_RAP_FINE,
    GS_SMOOTHER, GS_RESTRICT, GS_PROLONG, GS_DENSE, GS_KRYLOV_K, GS_TRANSPOSE, GS_ASSEMBLE, GS_ADJOINT,
    GS_BLOCKROW, GS_FIXED, GS_PRESMOOTH, GS_COUNT
};
__device__ __noinline__ void guard_fail(int site, long long v) {
    atomicOr(&g_status, ST_RANGE);
    if (atomicCAS(&g_guard_site, 0, site) == 0) g_guard_value = v;
}
// true when 0 <= i < n; otherwise records the failure
__device__ __forceinline__ bool in_range(long long i, long long n, int site) {
    if ((unsigned long long)i < (unsigned long long)n) return true;
    guard_fail(site, i);
    return false;
}

struct PtrsP {  // particle pointers as seen by kernels
    int n;
    double *x, *lp, *F_old, *F_new, *b_old, *b_new, *sigma, *pressure, *pi_old, *pi_new;
    const uint8_t *ext_flag, *trac_flag, *pbc_flag;
    const double *E;
};

inline PtrsP make_ptrs(const gw_particles_t &p) {
    PtrsP r;
    r.n = p.n;
    r.x = p.x; r.lp = p.lp; r.F_old = p.F_old; r.F_new = p.F_new; r.b_old = p.b_old; r.b_new = p.b_new;
    r.sigma = p.sigma; r.pressure = p.pressure; r.pi_old = p.pi_old; r.pi_new = p.pi_new;
    r.ext_flag = p.ext_flag; r.trac_flag = p.trac_flag; r.pbc_flag = p.pbc_flag; r.E = p.E;
    return r;
}

struct PtrsA {  // block-CSR pointers
    int n_rows, nf, nnzb, mw;
    const int *row_ptr, *cols, *row2node, *node2row;
    const uint32_t *stencil;
    void *vals;
};

inline PtrsA make_ptrs(const gw_bsr_t &a) {
    PtrsA r;
    r.n_rows = a.n_rows; r.nf = a.nf; r.nnzb = a.nnzb; r.mw = a.mask_words;
    r.row_ptr = a.row_ptr; r.cols = a.cols; r.row2node = a.row2node; r.node2row = a.node2row;
    r.stencil = a.stencil; r.vals = a.vals;
    return r;
}

// Position of neighbour offset bit `bit` in the row of node i (popcount of
// lower stencil bits), or -1 when the pattern has no such block.
__device__ __forceinline__ int stencil_slot(const uint32_t *st, int mw, int node, int bit) {
    const uint32_t *m = st + (size_t)node * mw;
    int w = bit >> 5, b = bit & 31;
    if (!((m[w] >> b) & 1u)) return -1;
    int s = 0;
    for (int k = 0; k < w; ++k) s += __popc(m[k]);
    s += __popc(m[w] & ((1u << b) - 1u));
    return s;
}

template <int D>
__device__ __forceinline__ int offset_bit(const int off[3]) {
    int b = 0, m = 1;
    for (int k = 0; k < D; ++k) { b += (off[k] + 2) * m; m *= 5; }
    return b;
}

}  // namespace
}  // namespace gw
