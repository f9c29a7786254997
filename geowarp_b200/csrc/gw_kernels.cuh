// Shared kernel-side definitions.  The library is one translation unit
// (gw_abi.cu includes every kernel header), so device globals live here.
#pragma once
#include "gw_particle.cuh"

namespace gw {

// Device status word: bit 0 range error, bit 1 non-finite value, bit 2 Krylov breakdown.
__device__ int g_status;
constexpr int ST_RANGE = 1, ST_NAN = 2, ST_BREAKDOWN = 4;

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

}  // namespace gw
