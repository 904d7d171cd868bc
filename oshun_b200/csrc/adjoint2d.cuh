// Transpose of the RK4-stage right-hand side for any grid (1D or 2D, any
// m0): F'(s)^T c at one stage state s, gathered per source point.  The
// forward is Actions::Adv as the stage kernels compute it (stage_pipe.cuh
// couple_src3 / couple_f00_row, field_update): for a source harmonic
// (s, M) with values f, momentum stencils G, H (wG/wH/wG00 of
// adjoint_math.h, the reference's ends), x/y differences dx, dy (times v),
//   (s+1, M)    += ex_g Ex G + ax_p dx          (s-1, M)    += ex_h Ex H + ax_m dx
//   (s+1, M+1)  += em_g (Ey - i Ez) G + ay_pp dy   (s-1, M+1) += em_h (Ey - i Ez) H + ay_mp dy
//   (s,   M+1)  += (Bz + i By)/2 f
//   (s-1, M-1)  += ep_h (Ey + i Ez) H + ay_mm dy   (s+1, M-1) += ep_g (Ey + i Ez) G + ay_pm dy
//   (s,   M-1)  += b_m (Bz - i By) f              (s,   M)   += -i M Bx f
// (G terms see E = 0 at p = 0 for s >= 1; m = 0 targets keep the real part;
// targets beyond the truncation are dropped; CLEAN_LOW_PC zeroes the slope
// of l >= 2 below p = min(l-1, 80)); the f00 source feeds (1, 0) and (1, 1)
// through G00 with the full E; dE/dt = J + curl B, dB/dt = -curl E with the
// current of f10 and f11.  The transpose of a complex coupling a f is
// conj(a) applied to the target cotangent; of a centred difference, minus
// the difference.  State and cotangent vectors use the plane layout: the
// f00 plane, the l >= 1 planes, the 6 field planes.
#pragma once

#include "adjoint_math.h"
#include "oshun_internal.h"

namespace oshun {
namespace adj2 {

struct Grid2 {
    int np, nx, ny, l0, m0, nplanes;
    long long cells, pstride;
    const double* invp;     // 1/p
    const double* vr;       // p/gamma
    const double* wj;       // current quadrature weight
    const CoefLM* coef;     // [(l0+1)(m0+1)]
    const int* plane_of;    // [(l0+1)(m0+1)]: plane of Re f_lm (l >= 1)
    double g00_s, g00_inv, g00_gr;
    double idx, idy;        // -1/(2 dx), -1/(2 dy)
};

struct Cx {
    double r, i;
};
__device__ __forceinline__ double re_conj(Cx c, Cx t) { return c.r * t.r + c.i * t.i; }   // Re(conj(c) t)
// conj(a) * b
__device__ __forceinline__ Cx conjmul(Cx a, Cx b) { return {a.r * b.r + a.i * b.i, a.r * b.i - a.i * b.r}; }

__device__ __forceinline__ bool masked(int t, int p) { return t >= 2 && p < (t - 1 < 80 ? t - 1 : 80); }
__device__ __forceinline__ bool exists(const Grid2& g, int t, int mt) {
    return t >= 0 && t <= g.l0 && mt >= 0 && mt <= (t < g.m0 ? t : g.m0);
}
// harmonic (l, m) of plane-layout vector v at (cell, p): f00 real, m = 0 real
__device__ __forceinline__ Cx harm(const Grid2& g, const double* v, int l, int m, long long cell, int p) {
    if (l == 0) return {v[cell * g.np + p], 0.0};
    const long long q = g.plane_of[l * (g.m0 + 1) + m];
    const double* b = v + (1 + q) * g.pstride + cell * g.np + p;
    return {b[0], m > 0 ? b[g.pstride] : 0.0};
}
// a target's slope cotangent: zero for a dropped target or a cleaned point
__device__ __forceinline__ Cx cot(const Grid2& g, const double* c, int t, int mt, long long cell, int p) {
    if (!exists(g, t, mt) || masked(t, p)) return {0.0, 0.0};
    return harm(g, c, t, mt, cell, p);
}
// field k (Ex Ey Ez Bx By Bz) of v at a cell
__device__ __forceinline__ double fld(const Grid2& g, const double* v, int k, long long cell) {
    return v[(1 + (long long)g.nplanes) * g.pstride + (long long)k * g.cells + cell];
}

// neighbours of a cell (periodic in x and y)
struct Nbr {
    long long xm, xp, ym, yp;
};
__device__ __forceinline__ Nbr nbr(const Grid2& g, long long cell) {
    const long long y = cell / g.nx, x = cell - y * g.nx;
    Nbr n;
    n.xm = y * g.nx + (x == 0 ? g.nx - 1 : x - 1);
    n.xp = y * g.nx + (x == g.nx - 1 ? 0 : x + 1);
    n.ym = (y == 0 ? g.ny - 1 : y - 1) * (long long)g.nx + x;
    n.yp = (y == g.ny - 1 ? 0 : y + 1) * (long long)g.nx + x;
    return n;
}

// G / H / G00 of source (s, M) of s-vector sv at (cell, p)
__device__ __forceinline__ Cx stencil(const Grid2& g, const double* sv, int s, int M, long long cell, int p, bool isH) {
    const int np = g.np;
    Cx acc{0.0, 0.0};
    const CoefLM& c = g.coef[s * (g.m0 + 1) + M];
    const double ipx = g.invp[p] * c.invpax;
    for (int k = (p > 0 ? p - 1 : 0); k <= (p + 1 < np ? p + 1 : np - 1); ++k) {
        double w;
        if (s == 0) w = adj::wG00<double>(p, k, np, g.g00_s, g.g00_inv, g.g00_gr);
        else if (isH) w = adj::wH<double>(p, k, np, ipx, c.hp0);
        else w = adj::wG<double>(p, k, np, ipx, c.gfac);
        if (w != 0.0) {
            const Cx f = harm(g, sv, s, M, cell, k);
            acc.r += w * f.r;
            acc.i += w * f.i;
        }
    }
    return acc;
}

// cotangent of source (s, M) at (cell, k), and this point's share of the
// cell's field cotangents (added to cF[6])
__device__ inline Cx vjp_source(const Grid2& g, const double* sv, const double* c, int s, int M, long long cell, int k,
                         double* cF) {
    const CoefLM& cf = g.coef[s * (g.m0 + 1) + M];
    const Nbr n = nbr(g, cell);
    const double Ex = fld(g, sv, 0, cell), Ey = fld(g, sv, 1, cell), Ez = fld(g, sv, 2, cell);
    const double Bx = fld(g, sv, 3, cell), By = fld(g, sv, 4, cell), Bz = fld(g, sv, 5, cell);
    const int np = g.np;
    const double v = g.vr[k];
    const bool has_y = g.ny > 1;
    Cx out{0.0, 0.0};
    auto add = [&](Cx a) { out.r += a.r; out.i += a.i; };
    // a G (or H) term: target (t, mt) += a(p) X(p), X the momentum stencil; a(p)
    // the complex field factor (p = 0 sees Eg = 0 for G when s >= 1)
    auto pterm = [&](int t, int mt, bool isH, double coef, double fr, double fi) {
        if (!exists(g, t, mt)) return;
        for (int p = (k > 0 ? k - 1 : 0); p <= (k + 1 < np ? k + 1 : np - 1); ++p) {
            if (masked(t, p)) continue;
            double w;
            if (s == 0) w = adj::wG00<double>(p, k, np, g.g00_s, g.g00_inv, g.g00_gr);
            else if (isH) w = adj::wH<double>(p, k, np, g.invp[p] * cf.invpax, cf.hp0);
            else w = adj::wG<double>(p, k, np, g.invp[p] * cf.invpax, cf.gfac);
            if (w == 0.0) continue;
            const Cx a{coef * fr, coef * fi};
            const Cx ct = cot(g, c, t, mt, cell, p);
            const Cx u = conjmul(a, ct);
            out.r += w * u.r;
            out.i += w * u.i;
        }
    };
    // an x (or y) difference term: target (t, mt) += coef v (f[n-] - f[n+])
    auto dterm = [&](int t, int mt, double coef, bool ydir) {
        if (!exists(g, t, mt) || masked(t, k) || coef == 0.0) return;
        const long long np_ = ydir ? n.yp : n.xp, nm_ = ydir ? n.ym : n.xm;
        const Cx cp = cot(g, c, t, mt, np_, k), cm = cot(g, c, t, mt, nm_, k);
        out.r += coef * v * (cp.r - cm.r);
        out.i += coef * v * (cp.i - cm.i);
    };
    // a pointwise term: target (t, mt) += a f
    auto fterm = [&](int t, int mt, double ar, double ai) {
        if (!exists(g, t, mt) || masked(t, k)) return;
        add(conjmul(Cx{ar, ai}, cot(g, c, t, mt, cell, k)));
    };
    // the field cotangents of this point (p = k): Re(conj(c_t) dT/dF)
    const Cx f = harm(g, sv, s, M, cell, k);
    const Cx G = stencil(g, sv, s, M, cell, k, false);
    const Cx H = s >= 1 ? stencil(g, sv, s, M, cell, k, true) : Cx{0.0, 0.0};
    const double gmask = (s >= 1 && k == 0) ? 0.0 : 1.0;   // G terms see E = 0 at p = 0
    auto fcot = [&](int t, int mt) -> Cx {
        if (!exists(g, t, mt) || masked(t, k)) return Cx{0.0, 0.0};
        return cot(g, c, t, mt, cell, k);
    };

    // (s+1, M): ex_g Ex G + ax_p dx
    pterm(s + 1, M, false, cf.ex_g, Ex, 0.0);
    dterm(s + 1, M, cf.ax_p, false);
    { const Cx ct = fcot(s + 1, M); cF[0] += gmask * re_conj(ct, Cx{cf.ex_g * G.r, cf.ex_g * G.i}); }
    if (s >= 1) {
        // (s-1, M): ex_h Ex H + ax_m dx
        pterm(s - 1, M, true, cf.ex_h, Ex, 0.0);
        dterm(s - 1, M, cf.ax_m, false);
        const Cx ct = fcot(s - 1, M);
        cF[0] += re_conj(ct, Cx{cf.ex_h * H.r, cf.ex_h * H.i});
    }
    if (M + 1 <= g.m0) {
        // (s+1, M+1): em_g (Ey - i Ez) G + ay_pp dy
        pterm(s + 1, M + 1, false, cf.em_g, Ey, -Ez);
        if (has_y) dterm(s + 1, M + 1, cf.ay_pp, true);
        { const Cx ct = fcot(s + 1, M + 1);
          cF[1] += gmask * re_conj(ct, Cx{cf.em_g * G.r, cf.em_g * G.i});
          cF[2] += gmask * re_conj(ct, Cx{cf.em_g * G.i, -cf.em_g * G.r}); }          // -i G
        if (s >= 1) {
            // (s-1, M+1): em_h (Ey - i Ez) H + ay_mp dy
            pterm(s - 1, M + 1, true, cf.em_h, Ey, -Ez);
            if (has_y) dterm(s - 1, M + 1, cf.ay_mp, true);
            const Cx ct = fcot(s - 1, M + 1);
            cF[1] += re_conj(ct, Cx{cf.em_h * H.r, cf.em_h * H.i});
            cF[2] += re_conj(ct, Cx{cf.em_h * H.i, -cf.em_h * H.r});
            // (s, M+1): (Bz + i By)/2 f
            fterm(s, M + 1, 0.5 * Bz, 0.5 * By);
            const Cx cb = fcot(s, M + 1);
            cF[5] += re_conj(cb, Cx{0.5 * f.r, 0.5 * f.i});
            cF[4] += re_conj(cb, Cx{-0.5 * f.i, 0.5 * f.r});                           // i f / 2
        }
    }
    if (M >= 1) {
        // (s-1, M-1): ep_h (Ey + i Ez) H + ay_mm dy
        pterm(s - 1, M - 1, true, cf.ep_h, Ey, Ez);
        if (has_y) dterm(s - 1, M - 1, cf.ay_mm, true);
        { const Cx ct = fcot(s - 1, M - 1);
          cF[1] += re_conj(ct, Cx{cf.ep_h * H.r, cf.ep_h * H.i});
          cF[2] += re_conj(ct, Cx{-cf.ep_h * H.i, cf.ep_h * H.r}); }                  // i H
        // (s+1, M-1): ep_g (Ey + i Ez) G + ay_pm dy
        pterm(s + 1, M - 1, false, cf.ep_g, Ey, Ez);
        if (has_y) dterm(s + 1, M - 1, cf.ay_pm, true);
        { const Cx ct = fcot(s + 1, M - 1);
          cF[1] += gmask * re_conj(ct, Cx{cf.ep_g * G.r, cf.ep_g * G.i});
          cF[2] += gmask * re_conj(ct, Cx{-cf.ep_g * G.i, cf.ep_g * G.r}); }
        // (s, M-1): b_m (Bz - i By) f
        fterm(s, M - 1, cf.b_m * Bz, -cf.b_m * By);
        { const Cx ct = fcot(s, M - 1);
          cF[5] += re_conj(ct, Cx{cf.b_m * f.r, cf.b_m * f.i});
          cF[4] += re_conj(ct, Cx{cf.b_m * f.i, -cf.b_m * f.r}); }                    // -i f b_m
        // (s, M): -i M Bx f
        fterm(s, M, 0.0, -(double)M * Bx);
        { const Cx ct = fcot(s, M);
          cF[3] += re_conj(ct, Cx{(double)M * f.i, -(double)M * f.r}); }             // -i M f
    }
    return out;
}

}  // namespace adj2

// F'(s)^T c for any grid (adjoint.cu stage_vjp2_kernel)
cudaError_t launch_stage_vjp2(const adj2::Grid2& g, const double* s, const double* c, double* out, cudaStream_t st);

}  // namespace oshun
