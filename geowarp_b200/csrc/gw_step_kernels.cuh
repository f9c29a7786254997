// Load-step kernels: cell sort, P2G activation, row compaction, block-CSR
// pattern, residual + element-tangent assembly, consistent mass, G2P.
#pragma once
#include "gw_kernels.cuh"

namespace gw {
namespace {  // internal linkage: each translation unit compiles the kernels it launches

constexpr int kThreads = 256;
constexpr int kSortTile = 2048;
constexpr int kSortWarps = kThreads / 32;

__device__ __forceinline__ unsigned lanemask_lt() {
    unsigned m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// ================================================================ scan (exclusive, int32)
// Each block scans 1024 elements and emits its total; the host recurses on
// the block totals and adds them back.
__global__ void k_scan_block(const int *__restrict__ in, int *__restrict__ out, int n, int *__restrict__ sums) {
    __shared__ int ws[32];
    const int i = blockIdx.x * 1024 + threadIdx.x;
    int v = (i < n) ? in[i] : 0;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) ws[w] = x;
    __syncthreads();
    if (w == 0) {
        int s = ws[lane];
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            int y = __shfl_up_sync(0xffffffffu, s, o);
            if (lane >= o) s += y;
        }
        ws[lane] = s;
    }
    __syncthreads();
    const int incl = x + (w > 0 ? ws[w - 1] : 0);
    if (i < n) out[i] = incl - v;
    if (threadIdx.x == 1023 && sums) sums[blockIdx.x] = incl;
}

// *out = *a + *b (one thread): the total of an exclusive scan from its last
// element and the last input flag
__global__ void k_add2(const int *a, const int *b, int *out) {
    if (threadIdx.x == 0 && blockIdx.x == 0) *out = *a + *b;
}

__global__ void k_scan_add(int *__restrict__ out, int n, const int *__restrict__ offs) {
    const int i = blockIdx.x * 1024 + threadIdx.x;
    if (i < n && blockIdx.x > 0) out[i] += offs[blockIdx.x];
}

// ================================================================ cell sort
template <int D>
__global__ void k_cell_keys(gw_grid_t g, const double *__restrict__ x, const double *__restrict__ lp, int n,
                            int *__restrict__ keys, int *__restrict__ idx) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    int key = 0, stride = 1;
    for (int k = 0; k < D; ++k) {
        int c = cell_of(x[p * D + k] - lp[p * D + k], g.inv_h[k]);
        c = c < 0 ? 0 : (c >= g.n_grid[k] ? g.n_grid[k] - 1 : c);
        key += c * stride;
        stride *= g.n_grid[k];
    }
    keys[p] = key;
    idx[p] = p;
}

__global__ void k_radix_hist(const int *__restrict__ keys, int n, int shift, int nblocks, int *__restrict__ hist) {
    __shared__ int cnt[256];
    for (int i = threadIdx.x; i < 256; i += blockDim.x) cnt[i] = 0;
    __syncthreads();
    const int base = blockIdx.x * kSortTile;
    const int end = min(base + kSortTile, n);
    for (int i = base + threadIdx.x; i < end; i += blockDim.x) atomicAdd(&cnt[(keys[i] >> shift) & 255], 1);
    __syncthreads();
    for (int d = threadIdx.x; d < 256; d += blockDim.x) hist[d * nblocks + blockIdx.x] = cnt[d];
}

// Stable scatter: ranks inside a chunk come from warp match + per-warp counts,
// so equal digits keep their input order.
__global__ void k_radix_scatter(const int *__restrict__ kin, const int *__restrict__ vin, int n, int shift, int nblocks,
                                const int *__restrict__ offs, int *__restrict__ kout, int *__restrict__ vout) {
    __shared__ int running[256];
    __shared__ int wcnt[kSortWarps][256];
    __shared__ int total[256];
    for (int d = threadIdx.x; d < 256; d += blockDim.x) running[d] = offs[d * nblocks + blockIdx.x];
    const int base = blockIdx.x * kSortTile;
    const int end = min(base + kSortTile, n);
    const int w = threadIdx.x >> 5;
    for (int chunk = base; chunk < end; chunk += blockDim.x) {
        for (int k = threadIdx.x; k < kSortWarps * 256; k += blockDim.x) (&wcnt[0][0])[k] = 0;
        __syncthreads();
        const int i = chunk + threadIdx.x;
        const bool valid = i < end;
        const int key = valid ? kin[i] : 0;
        const int digit = valid ? ((key >> shift) & 255) : 256;
        const unsigned peers = __match_any_sync(0xffffffffu, digit);
        const int wrank = __popc(peers & lanemask_lt());
        if (valid && wrank == 0) wcnt[w][digit] = __popc(peers);
        __syncthreads();
        for (int d = threadIdx.x; d < 256; d += blockDim.x) {
            int s = 0;
            for (int q = 0; q < kSortWarps; ++q) {
                int c = wcnt[q][d];
                wcnt[q][d] = s;
                s += c;
            }
            total[d] = s;
        }
        __syncthreads();
        if (valid) {
            const int pos = running[digit] + wcnt[w][digit] + wrank;
            kout[pos] = key;
            vout[pos] = vin[i];
        }
        __syncthreads();
        for (int d = threadIdx.x; d < 256; d += blockDim.x) running[d] += total[d];
        __syncthreads();
    }
}

// ================================================================ activation
template <int KIND>
__global__ void k_activate(LaunchConst c, PtrsP p, const int *__restrict__ perm, uint8_t *__restrict__ node_active,
                           uint32_t *__restrict__ cell_span, uint8_t *__restrict__ boundary) {
    typedef KindTraits<KIND> KT;
    const int D = KT::D, NS = KT::NS;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= p.n) return;
    const int pid = perm ? perm[t] : t;
    double x[D], lp[D];
    for (int k = 0; k < D; ++k) { x[k] = p.x[pid * D + k]; lp[k] = p.lp[pid * D + k]; }
    PState<KIND> s;
    if (!particle_shape<KIND>(c.g, x, lp, s)) atomicOr(&g_status, ST_RANGE);
    // cell span bits (bit k: 3-node span along axis k; 0x80: occupied)
    int cell = 0, stride = 1;
    uint32_t bits = 0x80u;
    for (int k = 0; k < D; ++k) {
        int cc = s.sh.ax[k].lower;
        cc = cc < 0 ? 0 : (cc >= c.g.n_grid[k] ? c.g.n_grid[k] - 1 : cc);
        cell += cc * stride;
        stride *= c.g.n_grid[k];
        if (s.sh.ax[k].span == 3) bits |= 1u << k;
    }
    atomicOr(&cell_span[cell], bits);
    const double thr = (KIND == GW_KIND_COUPLED2D) ? 1e-6 : 1e-7;
    for (int a = 0; a < NS; ++a) {
        const int id = s.nid[a];
        if (id < 0) continue;
        if (KIND == GW_KIND_SOLID2D) {  // mpm/mpm_utils.py:115-136
            if (s.sh.in_span(a)) node_active[id] = 1;
        } else {
            // 2D loops over the span (mpm_utils.py:209-223); 3D over all 27 (:327-347)
            if (KIND == GW_KIND_COUPLED2D && !s.sh.in_span(a)) continue;
            if (s.sh.W(a) > thr) node_active[id] = 1;
        }
    }
    if (KT::UP && p.pbc_flag && p.pbc_flag[pid]) {  // pressure Dirichlet above flagged particles
        const int v = D - 1;
        for (int a = 0; a < NS; ++a) {
            const int id = s.nid[a];
            if (id < 0) continue;
            if (KIND == GW_KIND_COUPLED2D && !s.sh.in_span(a)) continue;
            const double node_v = (double)(s.sh.ax[v].lower + s.sh.idx(a, v)) * c.g.h_nodes[v];
            if (node_v >= x[v]) boundary[(size_t)D * c.g.n_nodes + id] = 1;
        }
    }
}

// nodes inside the span support of an occupied cell (rows of the mass system)
template <int D>
__global__ void k_touched(gw_grid_t g, const uint32_t *__restrict__ cell_span, int n_cells, uint8_t *__restrict__ touched) {
    const int cidx = blockIdx.x * blockDim.x + threadIdx.x;
    if (cidx >= n_cells) return;
    const uint32_t cs = cell_span[cidx];
    if (!(cs & 0x80u)) return;
    int cc[3] = {0, 0, 0};
    int r = cidx;
    for (int k = 0; k < D; ++k) { cc[k] = r % g.n_grid[k]; r /= g.n_grid[k]; }
    const int NS = D == 2 ? 9 : 27;
    for (int a = 0; a < NS; ++a) {
        int id = 0;
        bool ok = true;
        for (int k = 0; k < D; ++k) {
            const int o = k == 0 ? a % 3 : (k == 1 ? (a / 3) % 3 : a / 9);
            const int span = 2 + ((cs >> k) & 1);
            if (o >= span) { ok = false; break; }
            const int nk = cc[k] + o;
            if (nk > g.n_grid[k]) { ok = false; break; }
            id += nk * node_stride(g, k);
        }
        if (ok) touched[id] = 1;
    }
}

__global__ void k_flags_to_int(const uint8_t *__restrict__ f, int n, int *__restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = f[i] ? 1 : 0;
}

__global__ void k_compact(const uint8_t *__restrict__ flags, const int *__restrict__ scan, int n, int nf,
                          const uint8_t *__restrict__ boundary, int *__restrict__ node2row, int *__restrict__ row2node,
                          uint8_t *__restrict__ free_mask) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const bool on = flags[i] != 0;
    node2row[i] = on ? scan[i] : -1;
    if (on) row2node[scan[i]] = i;
    if (free_mask) {
        uint8_t m = 0;
        if (on)
            for (int f = 0; f < nf; ++f)
                if (!boundary[(size_t)f * n + i]) m |= (uint8_t)(1u << f);
        free_mask[i] = m;
    }
}

// ================================================================ pattern
template <int D>
__global__ void k_pattern_count(gw_grid_t g, const uint32_t *__restrict__ cell_span, const int *__restrict__ node2row,
                                const int *__restrict__ row2node, int n_rows, int mw, uint32_t *__restrict__ stencil,
                                int *__restrict__ counts) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n_rows) return;
    const int node = row2node[r];
    if (!in_range(node, g.n_nodes, GS_PATTERN_FILL)) {
        counts[r] = 0;
        return;
    }
    int ic[3] = {0, 0, 0};
    {
        int q = node;
        for (int k = 0; k < D; ++k) { ic[k] = q % (g.n_grid[k] + 1); q /= (g.n_grid[k] + 1); }
    }
    uint32_t m[4] = {0u, 0u, 0u, 0u};
    const int NC = D == 2 ? 9 : 27;
    for (int co = 0; co < NC; ++co) {
        int cc[3], cidx = 0, cstride = 1;
        bool ok = true;
        for (int k = 0; k < D; ++k) {
            const int o = k == 0 ? co % 3 : (k == 1 ? (co / 3) % 3 : co / 9);
            cc[k] = ic[k] - o;
            if (cc[k] < 0 || cc[k] >= g.n_grid[k]) { ok = false; break; }
            cidx += cc[k] * cstride;
            cstride *= g.n_grid[k];
        }
        if (!ok) continue;
        const uint32_t cs = cell_span[cidx];
        if (!(cs & 0x80u)) continue;
        int span[3];
        for (int k = 0; k < D; ++k) {
            span[k] = 2 + ((cs >> k) & 1);
            if (ic[k] - cc[k] >= span[k]) ok = false;
        }
        if (!ok) continue;
        for (int jo = 0; jo < NC; ++jo) {
            int off[3] = {0, 0, 0}, jid = 0;
            bool okj = true;
            for (int k = 0; k < D; ++k) {
                const int o = k == 0 ? jo % 3 : (k == 1 ? (jo / 3) % 3 : jo / 9);
                if (o >= span[k]) { okj = false; break; }
                const int jk = cc[k] + o;
                if (jk > g.n_grid[k]) { okj = false; break; }
                off[k] = jk - ic[k];
                jid += jk * node_stride(g, k);
            }
            if (!okj || node2row[jid] < 0) continue;
            const int bit = offset_bit<D>(off);
            m[bit >> 5] |= 1u << (bit & 31);
        }
    }
    int cnt = 0;
    for (int w = 0; w < mw; ++w) {
        stencil[(size_t)node * mw + w] = m[w];
        cnt += __popc(m[w]);
    }
    counts[r] = cnt;
}

template <int D>
__global__ void k_pattern_fill(gw_grid_t g, PtrsA A, int *__restrict__ cols) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= A.n_rows) return;
    const int node = A.row2node[r];
    if (!in_range(node, g.n_nodes, GS_PATTERN_FILL)) return;
    int pos = A.row_ptr[r];
    const int end = A.row_ptr[r + 1];
    for (int w = 0; w < A.mw; ++w) {
        uint32_t m = A.stencil[(size_t)node * A.mw + w];
        while (m) {
            const int b = __ffs(m) - 1;
            m &= m - 1u;
            int bit = w * 32 + b;
            int jid = node;
            for (int k = 0; k < D; ++k) {
                const int o = bit % 5 - 2;
                bit /= 5;
                jid += o * node_stride(g, k);
            }
            if (!in_range(pos, end, GS_PATTERN_FILL)) return;
            const int col = in_range(jid, g.n_nodes, GS_PATTERN_FILL) ? A.node2row[jid] : 0;
            cols[pos++] = in_range(col, A.n_rows, GS_PATTERN_FILL) ? col : 0;
        }
    }
}

// ================================================================ residual + element tangent
template <int KIND, bool WANT_K, typename VT, int MODEL = -1>
__global__ void __launch_bounds__(kThreads) k_assemble(LaunchConst c, PtrsP p, const int *__restrict__ perm,
                                                       const uint8_t *__restrict__ free_mask,
                                                       const double *__restrict__ u_new,
                                                       const double *__restrict__ u_old, PtrsA A,
                                                       double *__restrict__ R, double *__restrict__ force) {
    typedef KindTraits<KIND> KT;
    typedef Layout<KIND> L;
    const int D = KT::D, NF = KT::NF, NS = KT::NS;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= p.n) return;
    const int pid = perm[t];
    double x[D], lp[D], Fo[9], bo[9];
    for (int k = 0; k < D; ++k) { x[k] = p.x[pid * D + k]; lp[k] = p.lp[pid * D + k]; }
    for (int k = 0; k < 9; ++k) { Fo[k] = p.F_old[(size_t)pid * 9 + k]; bo[k] = p.b_old[(size_t)pid * 9 + k]; }
    const double E = p.E ? p.E[pid] : c.E0;
    const double pi_old = p.pi_old ? p.pi_old[pid] : 0.0;
    const double pi_new = p.pi_new ? p.pi_new[pid] : 0.0;
    const double V0 = c.st.p_vol;

    PState<KIND> s;
    if (!particle_shape<KIND>(c.g, x, lp, s)) atomicOr(&g_status, ST_RANGE);
    particle_gather<KIND>(u_new, u_old, s);
    PEval<KIND> ev;
    particle_eval<KIND, WANT_K, MODEL>(c, s, x, Fo, bo, E, pi_old, pi_new, V0, ev);

    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            p.F_new[(size_t)pid * 9 + i * 3 + j] = ev.F_new[i][j];
            p.b_new[(size_t)pid * 9 + i * 3 + j] = ev.b_new[i][j];
            p.sigma[(size_t)pid * 9 + i * 3 + j] = ev.sigma[i][j];
        }
    if (p.pi_new) p.pi_new[pid] = ev.pi_new;

    const double ramp = (c.st.current_step + 1.0) / c.st.total_steps;
    double fext[D], ftr[D];
    for (int k = 0; k < D; ++k) {
        fext[k] = (p.ext_flag && p.ext_flag[pid]) ? c.st.point_load[k] * ramp : 0.0;
        ftr[k] = (p.trac_flag && p.trac_flag[pid]) ? c.st.traction[k] * c.g.h[k] / c.st.PPD : 0.0;
    }
    bool bad = false;
    for (int a = 0; a < NS; ++a) {
        const int id = s.nid[a];
        if (id < 0) continue;
        const uint8_t fm = free_mask[id];
        if (!fm) continue;
        const int row = A.node2row[id];
        if (!in_range(row, A.n_rows, GS_ASSEMBLE)) continue;
        double r[NF];
        residual_rows<KIND>(c, s, ev, a, fext, ftr, V0, r);
        for (int f = 0; f < NF; ++f)
            if ((fm >> f) & 1) {
                if (!isfinite(r[f])) bad = true;
                atomicAdd(&R[(size_t)row * NF + f], r[f]);
            }
    }
    if (ev.pen_on && force) atomicAdd(force, -ev.pen);
    if (bad) atomicOr(&g_status, ST_NAN);
    if (!WANT_K) return;

    for (int k = 0; k < D; ++k)
        if (s.sh.ax[k].lower < 0 || s.sh.ax[k].lower >= c.g.n_grid[k]) { atomicOr(&g_status, ST_RANGE); return; }
    VT *vals = (VT *)A.vals;
    const double gv = -c.st.gravity_mag * (c.st.gravity_full ? 1.0 : ramp);
    for (int b = 0; b < NS; ++b) {
        const int idb = s.nid[b];
        if (idb < 0 || !s.sh.in_span(b)) continue;
        const uint8_t fmb = free_mask[idb];
        if (!fmb) continue;
        const double Wb = s.sh.W(b), Wab = s.sh.Wavg(b);
        double Gb[D];
        for (int k = 0; k < D; ++k) Gb[k] = s.sh.G(b, k);
        // C_b = (dQ/dtheta) B_b
        double C[L::NQ][NF];
        for (int q = 0; q < L::NQ; ++q) {
            for (int gcol = 0; gcol < D; ++gcol) {
                double v = 0.0;
                for (int k = 0; k < D; ++k) v += ev.Dm[q][L::TH + k * D + gcol] * Gb[k];
                if (gcol == D - 1) v += ev.Dm[q][L::TU] * Wb;
                C[q][gcol] = v;
            }
            if (KT::UP) {
                double v = ev.Dm[q][L::TP] * Wb + ev.Dm[q][L::TD] * (Wb - Wab);
                for (int k = 0; k < D; ++k) v += ev.Dm[q][L::TG + k] * Gb[k];
                C[q][D] = v;
            }
        }
        for (int a = 0; a < NS; ++a) {
            const int ida = s.nid[a];
            if (ida < 0 || !s.sh.in_span(a)) continue;
            const uint8_t fma = free_mask[ida];
            if (!fma) continue;
            const int row = A.node2row[ida];
            if (!in_range(row, A.n_rows, GS_ASSEMBLE)) continue;
            int off[3] = {0, 0, 0};
            for (int k = 0; k < D; ++k) off[k] = s.sh.idx(b, k) - s.sh.idx(a, k);
            const int slot = stencil_slot(A.stencil, A.mw, ida, offset_bit<D>(off));
            if (slot < 0) { atomicOr(&g_status, ST_RANGE); continue; }
            const long long jb = (long long)A.row_ptr[row] + slot;
            if (!in_range(jb, A.nnzb, GS_ASSEMBLE)) continue;
            VT *blk = vals + (size_t)jb * NF * NF;
            const double Wa_ = s.sh.W(a), Waa = s.sh.Wavg(a);
            double Ga[D];
            for (int k = 0; k < D; ++k) Ga[k] = s.sh.G(a, k);
            for (int f = 0; f < NF; ++f) {
                if (!((fma >> f) & 1)) continue;
                for (int gcol = 0; gcol < NF; ++gcol) {
                    if (!((fmb >> gcol) & 1)) continue;
                    double v;
                    if (f < D) {
                        v = 0.0;
                        for (int i = 0; i < D; ++i) v -= Ga[i] * C[L::QU + i * D + f][gcol];
                        if (f == D - 1) v += Wa_ * gv * C[L::QS][gcol] + Wa_ * C[L::QPEN][gcol];
                    } else {
                        v = Wa_ * C[L::QM1][gcol] + (Wa_ - Waa) * C[L::QM3][gcol];
                        for (int i = 0; i < D; ++i) v += Ga[i] * C[L::QM2 + i][gcol];
                    }
                    atomicAdd(&blk[f * NF + gcol], (VT)(-v));
                }
            }
        }
    }
}

// identity on Dirichlet DOFs of active nodes (mpm/mpm_utils.py:1299-1341)
template <int D, typename VT>
__global__ void k_identity_dirichlet(PtrsA A, const uint8_t *__restrict__ free_mask) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= A.n_rows) return;
    const int node = A.row2node[r];
    const int off[3] = {0, 0, 0};
    const int slot = stencil_slot(A.stencil, A.mw, node, offset_bit<D>(off));
    if (slot < 0) { atomicOr(&g_status, ST_RANGE); return; }
    VT *blk = (VT *)A.vals + ((size_t)A.row_ptr[r] + slot) * A.nf * A.nf;
    const uint8_t fm = free_mask ? free_mask[node] : 0xffu;
    for (int f = 0; f < A.nf; ++f)
        if (!((fm >> f) & 1)) blk[f * A.nf + f] = VT(1);
}

// ================================================================ consistent mass
// Lumped projection: p_i = b_i / sum_j M_ij (the row sum is the lumped nodal
// mass sum_p N_i m_p by the partition of unity); rows without mass get 0.
__global__ void k_mass_lumped(PtrsA M, const double *__restrict__ rhs, double *__restrict__ x) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= M.n_rows) return;
    const double *vals = (const double *)M.vals;
    double m = 0.0;
    for (int j = M.row_ptr[r]; j < M.row_ptr[r + 1]; ++j) m += vals[j];
    x[r] = (m != 0.0) ? rhs[r] / m : 0.0;
}

template <int KIND>
__global__ void k_mass(LaunchConst c, PtrsP p, const int *__restrict__ perm, PtrsA M, double *__restrict__ rhs) {
    typedef KindTraits<KIND> KT;
    const int D = KT::D, NS = KT::NS;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= p.n) return;
    const int pid = perm[t];
    double x[D], lp[D];
    for (int k = 0; k < D; ++k) { x[k] = p.x[pid * D + k]; lp[k] = p.lp[pid * D + k]; }
    PState<KIND> s;
    particle_shape<KIND>(c.g, x, lp, s);
    const double m = c.st.p_vol * c.st.p_rho;
    const double pp = p.pressure[pid];
    double wsum = 0.0;
    for (int b = 0; b < NS; ++b)
        if (s.nid[b] >= 0) wsum += s.sh.W(b);
    double *vals = (double *)M.vals;
    for (int a = 0; a < NS; ++a) {
        const int ida = s.nid[a];
        if (ida < 0 || !s.sh.in_span(a)) continue;
        const int row = M.node2row[ida];
        if (row < 0) continue;
        const double Wa_ = s.sh.W(a);
        atomicAdd(&rhs[row], Wa_ * wsum * m * pp);  // sum_b W_a W_b m p (mpm_utils.py:254)
        for (int b = 0; b < NS; ++b) {
            const int idb = s.nid[b];
            if (idb < 0 || !s.sh.in_span(b)) continue;
            if (M.node2row[idb] < 0) continue;
            int off[3] = {0, 0, 0};
            for (int k = 0; k < D; ++k) off[k] = s.sh.idx(b, k) - s.sh.idx(a, k);
            const int slot = stencil_slot(M.stencil, M.mw, ida, offset_bit<D>(off));
            if (slot < 0) { atomicOr(&g_status, ST_RANGE); continue; }
            atomicAdd(&vals[(size_t)M.row_ptr[row] + slot], Wa_ * s.sh.W(b) * m);
        }
    }
}

// rows of M with a zero diagonal (no mass) become identity: p_hat = 0 there
template <int D>
__global__ void k_mass_fix(PtrsA M) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= M.n_rows) return;
    const int node = M.row2node[r];
    const int off[3] = {0, 0, 0};
    const int slot = stencil_slot(M.stencil, M.mw, node, offset_bit<D>(off));
    if (slot < 0) return;
    double *v = (double *)M.vals + (size_t)M.row_ptr[r] + slot;
    if (*v == 0.0) *v = 1.0;
}

__global__ void k_set_nodal_pressure(int n_rows, const int *__restrict__ row2node, const double *__restrict__ p_hat,
                                     const uint8_t *__restrict__ boundary, const uint8_t *__restrict__ node_active,
                                     int n_nodes, int nf, double *__restrict__ u_old, double *__restrict__ u_new) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n_rows) return;
    const int node = row2node[r];
    const int pf = nf - 1;
    if (boundary[(size_t)pf * n_nodes + node]) return;
    if (node_active && !node_active[node]) return;  // 3D variant (mpm_utils.py:412)
    u_old[(size_t)node * nf + pf] = p_hat[r];
    u_new[(size_t)node * nf + pf] = p_hat[r];
}

// ================================================================ G2P + lp update
template <int KIND>
__global__ void k_g2p(LaunchConst c, PtrsP p, const double *__restrict__ u_new, const double *__restrict__ u_old) {
    typedef KindTraits<KIND> KT;
    const int D = KT::D, NF = KT::NF, NS = KT::NS;
    const int pid = blockIdx.x * blockDim.x + threadIdx.x;
    if (pid >= p.n) return;
    double x[D], lp[D];
    for (int k = 0; k < D; ++k) { x[k] = p.x[pid * D + k]; lp[k] = p.lp[pid * D + k]; }
    PState<KIND> s;
    particle_shape<KIND>(c.g, x, lp, s);
    double du[D], pn = 0.0;
    for (int k = 0; k < D; ++k) du[k] = 0.0;
    for (int a = 0; a < NS; ++a) {
        const int id = s.nid[a];
        if (id < 0) continue;
        const double W = s.sh.W(a);
        for (int k = 0; k < D; ++k) du[k] += W * (u_new[(size_t)id * NF + k] - u_old[(size_t)id * NF + k]);
        if (KT::UP) pn += W * u_new[(size_t)id * NF + D];
    }
    double F[9];
    for (int k = 0; k < 9; ++k) {
        F[k] = p.F_new[(size_t)pid * 9 + k];
        p.F_old[(size_t)pid * 9 + k] = F[k];
        p.b_old[(size_t)pid * 9 + k] = p.b_new[(size_t)pid * 9 + k];
    }
    if (p.pi_old && p.pi_new) p.pi_old[pid] = p.pi_new[pid];
    for (int k = 0; k < D; ++k) x[k] += du[k];
    for (int k = 0; k < D; ++k) p.x[pid * D + k] = x[k];
    if (KT::UP) p.pressure[pid] = pn;
    // lp update, Charlton et al. 2017 Eqs. 38-39 (mpm/gimp.py:440-462)
    for (int k = 0; k < D; ++k) {
        const double U = ::sqrt(F[0 * 3 + k] * F[0 * 3 + k] + F[1 * 3 + k] * F[1 * 3 + k] + F[2 * 3 + k] * F[2 * 3 + k]);
        double v = c.st.lp0 * U;
        if (x[k] - v < c.g.domain_min[k]) v = x[k] - c.g.domain_min[k] - 1e-6;
        if (x[k] + v > c.g.domain_max[k]) v = c.g.domain_max[k] - x[k] - 1e-6;
        p.lp[pid * D + k] = v;
    }
}

// ================================================================ single-point return maps
__global__ void k_return_map(MatConst mc, double lam, double mu, int n, const double *__restrict__ etr,
                             const double *__restrict__ evt, const double *__restrict__ pi_old,
                             double *__restrict__ pi_new, double *__restrict__ e_out, double *__restrict__ tau_out,
                             double *__restrict__ dtau_out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double e[3] = {etr[3 * i], etr[3 * i + 1], etr[3 * i + 2]};
    double tau[3], dt[3][4], eo[3];
    double pn = pi_new ? pi_new[i] : 0.0;
    principal_model<double>(mc, lam, mu, e, evt ? evt[i] : 0.0, pi_old ? pi_old[i] : 0.0, pn, tau, dt, eo,
                            dtau_out != nullptr);
    if (pi_new) pi_new[i] = pn;
    for (int k = 0; k < 3; ++k) {
        e_out[3 * i + k] = eo[k];
        tau_out[3 * i + k] = tau[k];
        if (dtau_out)
            for (int l = 0; l < 3; ++l) dtau_out[9 * i + 3 * k + l] = dt[k][l];
    }
}

}  // namespace
}  // namespace gw
