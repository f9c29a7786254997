// cpGIMP shape functions: per-axis weights of the convected particle domain.
// Same formulas as mpm/gimp.py:25-193 (Coombs et al. section 2.4.2) and the
// cell-averaged weights used for PPP stabilisation; lp update after Charlton
// et al. 2017 (mpm/gimp.py:428-507).  Cell indices are always computed in
// FP64 so that cell keys and connectivity are bit-identical in every
// precision mode.
#pragma once
#include "gw_math.cuh"

namespace gw {
namespace {  // internal linkage: each translation unit compiles the kernels it launches

struct Axis {
    int lower;    // lower-corner cell (node index of slot 0)
    int span;     // 2 or 3 nodes touched
    double w[3], gw[3], wavg[3];
};

// int(c*inv + 1e-8) with C truncation, as mpm/gimp.py:34-36.
GW_HD int cell_of(double c, double inv) { return (int)(c * inv + 1e-8); }

GW_HD void gimp_axis(double xp, double lp, double d, double inv_d, Axis &ax) {
    const int lower = cell_of(xp - lp, inv_d);
    const int upper = cell_of(xp + lp, inv_d);
    const int base = cell_of(xp, inv_d);
    ax.lower = lower;
    if (upper == lower) {
        const double fx = xp * inv_d - (double)base;
        ax.span = 2;
        ax.w[0] = 1.0 - fx; ax.w[1] = fx; ax.w[2] = 0.0;
        ax.gw[0] = -inv_d; ax.gw[1] = inv_d; ax.gw[2] = 0.0;
        ax.wavg[0] = 0.5; ax.wavg[1] = 0.5; ax.wavg[2] = 0.0;
    } else {
        ax.span = 3;
        const double x0 = (double)lower * d;
        const double x1 = ((double)lower + 1.0) * d;
        const double x2 = ((double)lower + 2.0) * d;
        const double a0 = fabs(xp - x0), a2 = fabs(xp - x2);
        const double t0 = d + lp - a0, t2 = d + lp - a2;
        const double dl = d * lp;
        ax.w[0] = t0 * t0 / (4.0 * dl);
        ax.gw[0] = (-t0 / (2.0 * dl) * (xp - x0)) / a0;  // same association as the reference
        ax.w[1] = 1.0 - ((xp - x1) * (xp - x1) + lp * lp) / (2.0 * dl);
        ax.gw[1] = -(xp - x1) / dl;
        ax.w[2] = t2 * t2 / (4.0 * dl);
        ax.gw[2] = (-t2 / (2.0 * dl) * (xp - x2)) / a2;
        ax.wavg[0] = t0 / (4.0 * lp);
        ax.wavg[1] = 0.5;
        ax.wavg[2] = t2 / (4.0 * lp);
    }
}

// Slot a of the 3^D local nodes: a = i + 3 j (+ 9 k).
template <int D>
struct Shape {
    Axis ax[D];
    GW_HD int idx(int a, int k) const { return k == 0 ? a % 3 : (k == 1 ? (a / 3) % 3 : a / 9); }
    GW_HD bool in_span(int a) const {
        for (int k = 0; k < D; ++k)
            if (idx(a, k) >= ax[k].span) return false;
        return true;
    }
    GW_HD double W(int a) const {
        double r = 1.0;
        for (int k = 0; k < D; ++k) r *= ax[k].w[idx(a, k)];
        return r;
    }
    GW_HD double Wavg(int a) const {
        double r = 1.0;
        for (int k = 0; k < D; ++k) r *= ax[k].wavg[idx(a, k)];
        return r;
    }
    // reference gradient (weight_GRAD), component c
    GW_HD double G(int a, int c) const {
        double r = 1.0;
        for (int k = 0; k < D; ++k) r *= (k == c) ? ax[k].gw[idx(a, k)] : ax[k].w[idx(a, k)];
        return r;
    }
};

}  // namespace
}  // namespace gw
