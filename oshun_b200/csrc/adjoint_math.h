// Adjoint (vector-Jacobian products) of one small step of the 1D1P path with
// m0 = 0 (harmonics f_l(x, p), l = 0..l0, and E_x) and tridiagonal implicit
// collisions, in FP64.  Plain C++ usable from host and device code: the CUDA
// kernels (adjoint.cu) and the CPU derivative tests share it.
//
// The forward operators are the ones of the CUDA path (stage_pipe.cuh,
// collide.cu), restated here in the form the adjoint needs:
//   RHS F (Actions::Adv, OSHUN-1/def-Actions.cpp:73-94) for m0 = 0 in 1D:
//     slope_t(x,p) = E_x(x) [ex_g(t-1) G_{t-1}(p) + ex_h(t+1) H_{t+1}(p)]
//                    + ax_p(t-1) v(p) (f_{t-1}(x-1,p) - f_{t-1}(x+1,p))
//                    + ax_m(t+1) v(p) (f_{t+1}(x-1,p) - f_{t+1}(x+1,p)),
//     zeroed for p < min(t-1, 80) when t >= 2 (CLEAN_LOW_PC); G_l, H_l the
//     momentum stencils of MakeGH/G00 (def-VlasovMax.cpp:496-535) with the
//     reference's ends; dE_x/dt = J_x = sum_p wj(p) f_1(x,p) (the other five
//     fields never reach f or E_x when m0 = 0, so their cotangents are zero);
//   collision step (Explicit_EC_FP::loop, def-FokkerPlanck.cpp:590-625, then
//     Implicit_FLM_step::reset_coeff/advance, :808-1035): nsub RK4 substeps of
//     the e-e slope on f00, then (I - Dt C_l(f00)) f_l^new = f_l for l >= 1
//     with the tridiagonal C_l of reset_coeff, solved by Thomas.
#pragma once

#include <math.h>

#ifdef __CUDACC__
#define OSHUN_HD __host__ __device__
#else
#define OSHUN_HD
#endif

namespace oshun {
namespace adj {

constexpr double kPi = 3.14159265358979323846;

// per-l coupling coefficients of m = 0 (the CoefLM fields the 1D path uses)
struct Coef1 {
    double ex_g, ex_h, ax_p, ax_m, gfac, invpax, hp0;
};

// ---------------------------------------------------------------------------
// momentum stencils: weight of f(k) in G_l(p) and H_l(p).  T is the
// arithmetic type of the stage transpose (double; float for the FP32 bulk
// form); the data stay FP64 and are rounded to T where they are read.
// ---------------------------------------------------------------------------
// G for l >= 1 (0 at p = 0), dr = f(p-1) - f(p+1) with the reference's ends
template <typename T = double>
OSHUN_HD inline T wG(int p, int k, int np, T ipx, T gfac) {
    if (p == 0) return T(0);
    if (p < np - 1) {
        if (k == p - 1) return T(1) + gfac;
        if (k == p + 1) return -(T(1) + gfac);
        if (k == p) return ipx;
        return T(0);
    }
    if (k == p - 1) return T(1) + gfac;
    if (k == p) return ipx - (T(1) + gfac);
    return T(0);
}
// H for l >= 1: H(0) = hp0 f(1)
template <typename T = double>
OSHUN_HD inline T wH(int p, int k, int np, T ipx, T hp0) {
    if (p == 0) return k == 1 ? hp0 : T(0);
    if (p < np - 1) {
        if (k == p - 1) return T(1);
        if (k == p + 1) return T(-1);
        if (k == p) return ipx;
        return T(0);
    }
    if (k == p - 1) return T(1);
    if (k == p) return ipx - T(1);
    return T(0);
}
// G00 of f00: f(p-1) - f(p+1) with the reference's ends, the p = 0
// extrapolation (f(1) - f00x) g00_gr, f00x = (f(0) - f(1) g00_s) g00_inv
template <typename T = double>
OSHUN_HD inline T wG00(int p, int k, int np, T g00_s, T g00_inv, T g00_gr) {
    if (p == 0) {
        if (k == 0) return -g00_gr * g00_inv;
        if (k == 1) return g00_gr * (T(1) + g00_inv * g00_s);
        return T(0);
    }
    if (p < np - 1) {
        if (k == p - 1) return T(1);
        if (k == p + 1) return T(-1);
        return T(0);
    }
    if (k == p - 1) return T(1);
    if (k == p) return T(-1);
    return T(0);
}

// the stencils applied to one row f[0..np)
template <typename T = double>
OSHUN_HD inline T applyG(const double* f, int p, int np, T ipx, T gfac) {
    T s = T(0);
    for (int k = (p > 0 ? p - 1 : 0); k <= (p + 1 < np ? p + 1 : np - 1); ++k) s += wG<T>(p, k, np, ipx, gfac) * (T)f[k];
    return s;
}
template <typename T = double>
OSHUN_HD inline T applyH(const double* f, int p, int np, T ipx, T hp0) {
    T s = T(0);
    for (int k = (p > 0 ? p - 1 : 0); k <= (p + 1 < np ? p + 1 : np - 1); ++k) s += wH<T>(p, k, np, ipx, hp0) * (T)f[k];
    return s;
}
template <typename T = double>
OSHUN_HD inline T applyG00(const double* f, int p, int np, T gs, T gi, T gg) {
    T s = T(0);
    for (int k = (p > 0 ? p - 1 : 0); k <= (p + 1 < np ? p + 1 : np - 1); ++k)
        s += wG00<T>(p, k, np, gs, gi, gg) * (T)f[k];
    return s;
}

OSHUN_HD inline bool clean_masked(int t, int p) { return t >= 2 && p < (t - 1 < 80 ? t - 1 : 80); }

// grid and coefficients of one 1D problem (device or host pointers)
struct Grid1 {
    int np, nx, l0;
    const double* invp;    // 1/p
    const double* vr;      // p/gamma
    const double* wj;      // current quadrature weight
    const Coef1* coef;     // [l0+1]
    double g00_s, g00_inv, g00_gr;
};

// state layout: f[l][x][p] (l = 0..l0) then E_x[x]
OSHUN_HD inline const double* row(const double* f, const Grid1& g, int l, int x) {
    return f + ((long long)l * g.nx + x) * g.np;
}

// F at one (x, p) for every target t (slope[t]); the E_x slope is the cell's J_x
OSHUN_HD inline void rhs_point(const Grid1& g, const double* f, const double* Ex, int x, int p, double* slope) {
    const int np = g.np, nx = g.nx;
    const int xm = x == 0 ? nx - 1 : x - 1, xp = x == nx - 1 ? 0 : x + 1;
    const double E = Ex[x], v = g.vr[p];
    for (int t = 0; t <= g.l0; ++t) {
        double s = 0.0;
        if (t >= 1) {
            const int src = t - 1;
            const Coef1& c = g.coef[src];
            const double* fr = row(f, g, src, x);
            if (src == 0) s += E * c.ex_g * applyG00(fr, p, np, g.g00_s, g.g00_inv, g.g00_gr);
            else s += E * c.ex_g * applyG(fr, p, np, g.invp[p] * c.invpax, c.gfac);
            s += c.ax_p * v * (row(f, g, src, xm)[p] - row(f, g, src, xp)[p]);
        }
        if (t + 1 <= g.l0) {
            const int src = t + 1;
            const Coef1& c = g.coef[src];
            const double* fr = row(f, g, src, x);
            s += E * c.ex_h * applyH(fr, p, np, g.invp[p] * c.invpax, c.hp0);
            s += c.ax_m * v * (row(f, g, src, xm)[p] - row(f, g, src, xp)[p]);
        }
        slope[t] = clean_masked(t, p) ? 0.0 : s;
    }
}

// cotangent of f_s(x, k) from the slope cotangents cf[t][x][p] (masked
// points carry no cotangent) and the E_x slope cotangent cE[x]
template <typename T = double>
OSHUN_HD inline T vjp_f(const Grid1& g, const double* Ex, const double* cf, const double* cE, int s, int x, int k) {
    const int np = g.np, nx = g.nx;
    const int xm = x == 0 ? nx - 1 : x - 1, xp = x == nx - 1 ? 0 : x + 1;
    const Coef1& c = g.coef[s];
    const T E = (T)Ex[x];
    T acc = T(0);
    const int plo = k > 0 ? k - 1 : 0, phi = k + 1 < np ? k + 1 : np - 1;
    if (s + 1 <= g.l0) {   // source of target s+1 through G and x advection
        const int t = s + 1;
        const double* ct = row(cf, g, t, x);
        for (int p = plo; p <= phi; ++p) {
            if (clean_masked(t, p)) continue;
            const T w = s == 0 ? wG00<T>(p, k, np, (T)g.g00_s, (T)g.g00_inv, (T)g.g00_gr)
                               : wG<T>(p, k, np, (T)(g.invp[p] * c.invpax), (T)c.gfac);
            acc += E * (T)c.ex_g * w * (T)ct[p];
        }
        const T cxp = clean_masked(t, k) ? T(0) : (T)row(cf, g, t, xp)[k];
        const T cxm = clean_masked(t, k) ? T(0) : (T)row(cf, g, t, xm)[k];
        acc += (T)c.ax_p * (T)g.vr[k] * (cxp - cxm);
    }
    if (s >= 1) {          // source of target s-1 through H and x advection
        const int t = s - 1;
        const double* ct = row(cf, g, t, x);
        for (int p = plo; p <= phi; ++p) {
            if (clean_masked(t, p)) continue;
            acc += E * (T)c.ex_h * wH<T>(p, k, np, (T)(g.invp[p] * c.invpax), (T)c.hp0) * (T)ct[p];
        }
        const T cxp = clean_masked(t, k) ? T(0) : (T)row(cf, g, t, xp)[k];
        const T cxm = clean_masked(t, k) ? T(0) : (T)row(cf, g, t, xm)[k];
        acc += (T)c.ax_m * (T)g.vr[k] * (cxp - cxm);
    }
    if (s == 1) acc += (T)g.wj[k] * (T)cE[x];
    return acc;
}

// one momentum point's share of the E_x(x) cotangent
template <typename T = double>
OSHUN_HD inline T vjp_E_point(const Grid1& g, const double* f, const double* cf, int x, int p) {
    const int np = g.np;
    T acc = T(0);
    for (int s = 0; s <= g.l0; ++s) {
        const Coef1& c = g.coef[s];
        const double* fr = row(f, g, s, x);
        if (s + 1 <= g.l0 && !clean_masked(s + 1, p)) {
            const T G = s == 0 ? applyG00<T>(fr, p, np, (T)g.g00_s, (T)g.g00_inv, (T)g.g00_gr)
                               : applyG<T>(fr, p, np, (T)(g.invp[p] * c.invpax), (T)c.gfac);
            acc += (T)c.ex_g * G * (T)row(cf, g, s + 1, x)[p];
        }
        if (s >= 1 && !clean_masked(s - 1, p))
            acc += (T)c.ex_h * applyH<T>(fr, p, np, (T)(g.invp[p] * c.invpax), (T)c.hp0) * (T)row(cf, g, s - 1, x)[p];
    }
    return acc;
}

// ---------------------------------------------------------------------------
// collision step of one cell
// ---------------------------------------------------------------------------
struct CollTables {
    int np, NB;
    const double *vr, *U4, *U4m1, *U2, *U2m1, *U1, *U1m1, *U3, *Qn, *Pn, *V5, *V7;
    double density_np, Zeta, c_kpre, kpre;
};

// Coulomb logarithms (def-FokkerPlanck.cpp:41-95) and their derivatives
OSHUN_HD inline double log_ee_d(double ne, double Te, double dens, double* d_ne, double* d_Te) {
    *d_ne = 0.0;
    *d_Te = 0.0;
    if (ne > 0.000000001) {
        const double T = Te / (3.0 * ne) * 511000, n = ne * dens;
        const double lT = log(T), ln = log(n);
        const double sq = sqrt(0.00001 + 0.0625 * (lT - 2.0) * (lT - 2.0));
        const double v = 23.5 - 0.5 * ln + 1.25 * lT - sq;
        if (v > 2.0) {
            const double dv_dlT = 1.25 - 0.0625 * (lT - 2.0) / sq;
            *d_Te = dv_dlT / Te;
            *d_ne = -dv_dlT / ne - 0.5 / ne;
            return v;
        }
    }
    return 2.0;
}
OSHUN_HD inline double zlog_ei_d(double ne, double Te, double dens, double Z, double* d_ne, double* d_Te) {
    *d_ne = 0.0;
    *d_Te = 0.0;
    if (ne > 0.0000001) {
        const double T = Te / (3.0 * ne) * 511000, n = ne * dens;
        const double v = 24.0 - 0.5 * log(n) + log(T);
        if (v > 2.0) {
            *d_Te = Z / Te;
            *d_ne = Z * (-1.0 / ne - 0.5 / ne);
            return v * Z;
        }
    }
    return 2.0 * Z;
}

// the three cumulative integrals of f (I4 with U4, I2 with U2 forward; J1 with U1 backward)
OSHUN_HD inline void scans(const CollTables& T, const double* f, double* I4, double* I2, double* J1) {
    const int n = T.np;
    I4[0] = 0.0;
    I2[0] = 0.0;
    for (int k = 1; k < n; ++k) {
        I4[k] = I4[k - 1] + (T.U4[k] * f[k] + T.U4m1[k] * f[k - 1]);
        I2[k] = I2[k - 1] + (T.U2[k] * f[k] + T.U2m1[k] * f[k - 1]);
    }
    J1[n - 1] = 0.0;
    for (int k = n - 2; k >= 0; --k) J1[k] = J1[k + 1] + (T.U1[k + 1] * f[k + 1] + T.U1m1[k + 1] * f[k]);
}
// their transpose: cotangents of I4, I2, J1 -> cotangent of f (added)
OSHUN_HD inline void scans_T(const CollTables& T, const double* lI4, const double* lI2, const double* lJ1, double* lf) {
    const int n = T.np;
    double r4 = 0.0, r2 = 0.0;
    for (int i = n - 1; i >= 1; --i) {   // term i enters I4[k], I2[k] for every k >= i
        r4 += lI4[i];
        r2 += lI2[i];
        lf[i] += r4 * T.U4[i] + r2 * T.U2[i];
        lf[i - 1] += r4 * T.U4m1[i] + r2 * T.U2m1[i];
    }
    double r1 = 0.0;
    for (int i = 1; i <= n - 1; ++i) {   // term i enters J1[k] for every k <= i-1
        r1 += lJ1[i - 1];
        lf[i] += r1 * T.U1[i];
        lf[i - 1] += r1 * T.U1m1[i];
    }
}

// e-e slope (EE_isotropic_conserva::Getslope, def-FokkerPlanck.cpp:192-267);
// w: 5 np doubles of work space
OSHUN_HD inline void ee_slope(const CollTables& T, const double* f, double* fh, double* w) {
    const int n = T.np;
    double *I4 = w, *I2 = w + n, *J1 = w + 2 * n, *G = w + 3 * n, *D = w + 4 * n;
    scans(T, f, I4, I2, J1);
    double dn, dT;
    const double lnee = log_ee_d(4.0 * kPi * I2[n - 1], 4.0 * kPi * I4[n - 1], T.density_np, &dn, &dT);
    const double v0s = T.vr[0] * T.vr[0], v1s = T.vr[1] * T.vr[1];
    for (int k = 0; k < n; ++k) {
        if (k < T.NB) {
            const double f00 = (f[0] - f[1] * v0s / v1s) / (1.0 - v0s / v1s);
            const double v3 = T.U3[k], v5 = T.V5[k], v7 = T.V7[k];
            const double i2s = f00 * v3 / 3.0 + (f[1] - f00) * v5 / v1s * 0.2;
            const double i4s = f00 * v5 * 0.2 + (f[1] - f00) * v7 / (v1s * 7.0);
            G[k] = f[k] * i4s + (v3 * f[k] - 3.0 * i2s) * J1[k];
        } else {
            G[k] = (I4[k] + T.U3[k] * J1[k]) * f[k] - 3.0 * I2[k] * J1[k];
        }
    }
    for (int k = 0; k < n; ++k) D[k] = (k < n - 1) ? (G[k] - G[k + 1]) * T.Pn[k] : G[k];
    const double norm = T.c_kpre * lnee;
    for (int k = 0; k < n; ++k) {
        const double r = k == 0 ? ((-G[0]) * (2.0 / v0s) - D[0]) * T.Qn[0] : T.Qn[k] * (D[k - 1] - D[k]);
        fh[k] = r * norm;
    }
}
// transpose of the slope's derivative at f: mu (cotangent of fh) -> lf (added);
// w: 13 np doubles of work space
OSHUN_HD inline void ee_slope_T(const CollTables& T, const double* f, const double* mu, double* lf, double* w) {
    const int n = T.np;
    double *I4 = w, *I2 = w + n, *J1 = w + 2 * n, *G = w + 3 * n, *D = w + 4 * n;
    double *lG = w + 5 * n, *lD = w + 6 * n, *lI4 = w + 7 * n, *lI2 = w + 8 * n, *lJ1 = w + 9 * n;
    double* raw = w + 10 * n;
    scans(T, f, I4, I2, J1);
    double dn, dT;
    const double lnee = log_ee_d(4.0 * kPi * I2[n - 1], 4.0 * kPi * I4[n - 1], T.density_np, &dn, &dT);
    const double v0s = T.vr[0] * T.vr[0], v1s = T.vr[1] * T.vr[1];
    const double r = v0s / v1s;
    const double f00 = (f[0] - f[1] * r) / (1.0 - r);
    for (int k = 0; k < n; ++k) {
        if (k < T.NB) {
            const double v3 = T.U3[k], v5 = T.V5[k], v7 = T.V7[k];
            const double i2s = f00 * v3 / 3.0 + (f[1] - f00) * v5 / v1s * 0.2;
            const double i4s = f00 * v5 * 0.2 + (f[1] - f00) * v7 / (v1s * 7.0);
            G[k] = f[k] * i4s + (v3 * f[k] - 3.0 * i2s) * J1[k];
        } else {
            G[k] = (I4[k] + T.U3[k] * J1[k]) * f[k] - 3.0 * I2[k] * J1[k];
        }
    }
    for (int k = 0; k < n; ++k) D[k] = (k < n - 1) ? (G[k] - G[k + 1]) * T.Pn[k] : G[k];
    for (int k = 0; k < n; ++k)
        raw[k] = k == 0 ? ((-G[0]) * (2.0 / v0s) - D[0]) * T.Qn[0] : T.Qn[k] * (D[k - 1] - D[k]);
    const double norm = T.c_kpre * lnee;
    double l_norm = 0.0;
    for (int k = 0; k < n; ++k) { lG[k] = 0.0; lD[k] = 0.0; lI4[k] = 0.0; lI2[k] = 0.0; lJ1[k] = 0.0; }
    for (int k = 0; k < n; ++k) {
        l_norm += mu[k] * raw[k];
        const double lr = mu[k] * norm;
        if (k == 0) {
            lG[0] += -lr * T.Qn[0] * (2.0 / v0s);
            lD[0] += -lr * T.Qn[0];
        } else {
            lD[k - 1] += lr * T.Qn[k];
            lD[k] -= lr * T.Qn[k];
        }
    }
    for (int k = 0; k < n; ++k) {
        if (k < n - 1) {
            lG[k] += lD[k] * T.Pn[k];
            lG[k + 1] -= lD[k] * T.Pn[k];
        } else {
            lG[k] += lD[k];
        }
    }
    double l_f00 = 0.0, l_f1 = 0.0;
    for (int k = 0; k < n; ++k) {
        const double lg = lG[k];
        if (k < T.NB) {
            const double v3 = T.U3[k], v5 = T.V5[k], v7 = T.V7[k];
            const double i2s = f00 * v3 / 3.0 + (f[1] - f00) * v5 / v1s * 0.2;
            const double i4s = f00 * v5 * 0.2 + (f[1] - f00) * v7 / (v1s * 7.0);
            lf[k] += lg * (i4s + v3 * J1[k]);
            const double l_i4s = lg * f[k];
            const double l_i2s = -3.0 * lg * J1[k];
            lJ1[k] += lg * (v3 * f[k] - 3.0 * i2s);
            l_f00 += l_i2s * (v3 / 3.0 - v5 / v1s * 0.2) + l_i4s * (v5 * 0.2 - v7 / (v1s * 7.0));
            l_f1 += l_i2s * (v5 / v1s * 0.2) + l_i4s * (v7 / (v1s * 7.0));
        } else {
            lI4[k] += lg * f[k];
            lJ1[k] += lg * (T.U3[k] * f[k] - 3.0 * I2[k]);
            lf[k] += lg * (I4[k] + T.U3[k] * J1[k]);
            lI2[k] += -3.0 * lg * J1[k];
        }
    }
    lf[0] += l_f00 / (1.0 - r);
    lf[1] += l_f1 - l_f00 * r / (1.0 - r);
    const double l_lnee = l_norm * T.c_kpre;
    lI2[n - 1] += l_lnee * dn * 4.0 * kPi;
    lI4[n - 1] += l_lnee * dT * 4.0 * kPi;
    scans_T(T, lI4, lI2, lJ1, lf);
}

// one RK4 substep of the e-e slope: f <- f + h/6 (k1 + 2 k2 + 2 k3 + k4);
// w: 8 np doubles
OSHUN_HD inline void ee_rk4(const CollTables& T, double* f, double h, double* w) {
    const int n = T.np;
    double *s = w, *k = w + n, *acc = w + 2 * n, *sw = w + 3 * n;
    for (int i = 0; i < n; ++i) acc[i] = 0.0;
    const double c_in[4] = {0.0, 0.5 * h, 0.5 * h, h}, c_out[4] = {h / 6.0, h / 3.0, h / 3.0, h / 6.0};
    for (int st = 0; st < 4; ++st) {
        for (int i = 0; i < n; ++i) s[i] = f[i] + (st == 0 ? 0.0 : c_in[st] * k[i]);
        ee_slope(T, s, k, sw);
        for (int i = 0; i < n; ++i) acc[i] += c_out[st] * k[i];
    }
    for (int i = 0; i < n; ++i) f[i] += acc[i];
}
// its transpose at f: lam (cotangent of the substep's output, in place) ->
// cotangent of its input; w: 20 np doubles
OSHUN_HD inline void ee_rk4_T(const CollTables& T, const double* f, double* lam, double h, double* w) {
    const int n = T.np;
    double *S = w, *K = w + 4 * n, *c = w + 8 * n, *a = w + 9 * n, *lout = w + 10 * n, *sw = w + 11 * n;
    // stage inputs s1..s4 and slopes
    const double c_in[4] = {0.0, 0.5 * h, 0.5 * h, h};
    for (int st = 0; st < 4; ++st) {
        for (int i = 0; i < n; ++i) S[st * n + i] = f[i] + (st == 0 ? 0.0 : c_in[st] * K[(st - 1) * n + i]);
        ee_slope(T, S + st * n, K + st * n, sw);
    }
    for (int i = 0; i < n; ++i) lout[i] = lam[i];
    // cotangents of k4 .. k1 (see the RK4 transpose of the stage)
    const double w_out[4] = {h / 6.0, h / 3.0, h / 3.0, h / 6.0};
    for (int i = 0; i < n; ++i) a[i] = 0.0;
    for (int st = 3; st >= 0; --st) {
        const double w_next = st < 3 ? c_in[st + 1] : 0.0;
        for (int i = 0; i < n; ++i) c[i] = w_out[st] * lout[i] + w_next * a[i];
        for (int i = 0; i < n; ++i) a[i] = 0.0;
        ee_slope_T(T, S + st * n, c, a, sw);
        for (int i = 0; i < n; ++i) lam[i] += a[i];
    }
}

// tridiagonal coefficients of reset_coeff from f00 (tridiagonal mode);
// out: ta, tb, tc, scat (np each); w: 3 np
OSHUN_HD inline void reset_coeff(const CollTables& T, const double* f, double Dt, double* ta, double* tb, double* tc,
                                 double* scat, double* w) {
    const int n = T.np;
    double *I2 = w, *I0 = w + n, *J1 = w + 2 * n;
    scans(T, f, I2, I0, J1);
    const double Tt = I2[n - 1] * (4.0 * kPi), N = I0[n - 1] * (4.0 * kPi);
    double d1, d2, d3, d4;
    const double lnee = log_ee_d(N, Tt, T.density_np, &d1, &d2);
    const double zl = zlog_ei_d(N, Tt, T.density_np, T.Zeta, &d3, &d4);
    const double scale = (-1.0) * lnee * T.kpre * Dt;
    const double* vr = T.vr;
    for (int k = 0; k < n; ++k) {
        const double i2 = I2[k] * (4.0 * kPi) / (vr[k] * vr[k]);
        const double i0 = I0[k] * (4.0 * kPi);
        const double j1m = J1[k] * (4.0 * kPi * vr[k]);
        const double t1 = i0 + (2.0 * j1m - i2) / 3.0;
        const double t2 = (i2 + j1m) / 3.0;
        scat[k] = (((k == 0) ? 0.0 : t1 * lnee) + zl * N) / T.U3[k] * (T.kpre * Dt);
        ta[k] = tb[k] = tc[k] = 0.0;
        if (k == 0) {
            tb[k] = 8.0 * kPi * f[0] * scale;
        } else if (k < n - 1) {
            const double Dm = 1.0 / (vr[k] * 0.5 * (vr[k + 1] - vr[k - 1]) * (vr[k] - vr[k - 1]));
            const double Dp = 1.0 / (vr[k] * 0.5 * (vr[k + 1] - vr[k - 1]) * (vr[k + 1] - vr[k]));
            const double S2 = 1.0 / (vr[k] * vr[k] * (vr[k + 1] - vr[k - 1]));
            tb[k] = (8.0 * kPi * f[k] - t2 * (Dm + Dp)) * scale;
            ta[k] = (t2 * Dm - t1 * S2) * scale;
            tc[k] = (t2 * Dp + t1 * S2) * scale;
        }
    }
}
// transpose: cotangents of ta, tb, tc, scat -> cotangent of f (added); w: 6 np
OSHUN_HD inline void reset_coeff_T(const CollTables& T, const double* f, double Dt, const double* la,
                                   const double* lb, const double* lc, const double* ls, double* lf, double* w) {
    const int n = T.np;
    double *I2 = w, *I0 = w + n, *J1 = w + 2 * n, *lI2 = w + 3 * n, *lI0 = w + 4 * n, *lJ1 = w + 5 * n;
    scans(T, f, I2, I0, J1);
    const double Tt = I2[n - 1] * (4.0 * kPi), N = I0[n - 1] * (4.0 * kPi);
    double le_dN, le_dT, zl_dN, zl_dT;
    const double lnee = log_ee_d(N, Tt, T.density_np, &le_dN, &le_dT);
    const double zl = zlog_ei_d(N, Tt, T.density_np, T.Zeta, &zl_dN, &zl_dT);
    const double scale = (-1.0) * lnee * T.kpre * Dt;
    const double* vr = T.vr;
    double l_scale = 0.0, l_lnee = 0.0, l_zl = 0.0, l_N = 0.0;
    for (int k = 0; k < n; ++k) { lI2[k] = 0.0; lI0[k] = 0.0; lJ1[k] = 0.0; }
    for (int k = 0; k < n; ++k) {
        const double i2 = I2[k] * (4.0 * kPi) / (vr[k] * vr[k]);
        const double i0 = I0[k] * (4.0 * kPi);
        const double j1m = J1[k] * (4.0 * kPi * vr[k]);
        const double t1 = i0 + (2.0 * j1m - i2) / 3.0;
        const double t2 = (i2 + j1m) / 3.0;
        double l_t1 = 0.0, l_t2 = 0.0;
        const double K = T.kpre * Dt / T.U3[k];
        if (k > 0) {
            l_t1 += ls[k] * K * lnee;
            l_lnee += ls[k] * K * t1;
        }
        l_zl += ls[k] * K * N;
        l_N += ls[k] * K * zl;
        if (k == 0) {
            lf[0] += lb[0] * 8.0 * kPi * scale;
            l_scale += lb[0] * 8.0 * kPi * f[0];
        } else if (k < n - 1) {
            const double Dm = 1.0 / (vr[k] * 0.5 * (vr[k + 1] - vr[k - 1]) * (vr[k] - vr[k - 1]));
            const double Dp = 1.0 / (vr[k] * 0.5 * (vr[k + 1] - vr[k - 1]) * (vr[k + 1] - vr[k]));
            const double S2 = 1.0 / (vr[k] * vr[k] * (vr[k + 1] - vr[k - 1]));
            lf[k] += lb[k] * 8.0 * kPi * scale;
            l_t2 += (-lb[k] * (Dm + Dp) + la[k] * Dm + lc[k] * Dp) * scale;
            l_t1 += (-la[k] * S2 + lc[k] * S2) * scale;
            l_scale += lb[k] * (8.0 * kPi * f[k] - t2 * (Dm + Dp)) + la[k] * (t2 * Dm - t1 * S2) +
                       lc[k] * (t2 * Dp + t1 * S2);
        }
        // t1 = i0 + (2 j1m - i2)/3, t2 = (i2 + j1m)/3
        const double l_i0 = l_t1;
        const double l_j1m = 2.0 / 3.0 * l_t1 + l_t2 / 3.0;
        const double l_i2 = -l_t1 / 3.0 + l_t2 / 3.0;
        lI2[k] += l_i2 * (4.0 * kPi) / (vr[k] * vr[k]);
        lI0[k] += l_i0 * (4.0 * kPi);
        lJ1[k] += l_j1m * (4.0 * kPi * vr[k]);
    }
    l_lnee += l_scale * (-1.0) * T.kpre * Dt;
    l_N += l_lnee * le_dN + l_zl * zl_dN;
    const double l_T = l_lnee * le_dT + l_zl * zl_dT;
    lI0[n - 1] += l_N * (4.0 * kPi);
    lI2[n - 1] += l_T * (4.0 * kPi);
    scans_T(T, lI2, lI0, lJ1, lf);
}

// matrix of order l: rows i: a_i x_{i-1} + b_i x_i + c_i x_{i+1}
OSHUN_HD inline double diag_l(const double* tb, const double* scat, int l, int i) {
    const double ll1 = l * ((-0.5) * (l + 1.0));
    return (i == 0 && l > 1 ? 0.0 : tb[i]) + (1.0 - ll1 * scat[i]);
}
// x = A^{-1} d (Thomas, TridiagonalSolve def-Nmethods.cpp:142-167); w: np
OSHUN_HD inline void thomas(const double* a, const double* tb, const double* c, const double* scat, int l, int n,
                            const double* d, double* x, double* w) {
    double* cp = w;
    double b = diag_l(tb, scat, l, 0);
    cp[0] = c[0] / b;
    x[0] = d[0] / b;
    for (int i = 1; i < n; ++i) {
        b = diag_l(tb, scat, l, i) - cp[i - 1] * a[i];
        cp[i] = c[i] / b;
        x[i] = (d[i] - x[i - 1] * a[i]) / b;
    }
    for (int i = n - 2; i >= 0; --i) x[i] = x[i] - cp[i] * x[i + 1];
}
// y = A^{-T} r: the transposed system has sub-diagonal c_{i-1}, super-diagonal a_{i+1}
OSHUN_HD inline void thomas_T(const double* a, const double* tb, const double* c, const double* scat, int l, int n,
                              const double* r, double* y, double* w) {
    double* cp = w;
    double b = diag_l(tb, scat, l, 0);
    cp[0] = (n > 1 ? a[1] : 0.0) / b;
    y[0] = r[0] / b;
    for (int i = 1; i < n; ++i) {
        b = diag_l(tb, scat, l, i) - cp[i - 1] * c[i - 1];
        cp[i] = (i + 1 < n ? a[i + 1] : 0.0) / b;
        y[i] = (r[i] - y[i - 1] * c[i - 1]) / b;
    }
    for (int i = n - 2; i >= 0; --i) y[i] = y[i] - cp[i] * y[i + 1];
}

// Work space (doubles) of one cell's collision forward and adjoint
OSHUN_HD inline long long coll_ws(int np, int l0, int nsub) {
    return (long long)np * (40 + 3 * (long long)l0 + (long long)nsub + 1);
}

// forward collision step of one cell: f00 (np) and f_l (l = 1..l0, np each)
// in place; ee/eb select the e-e substeps and the implicit solves
OSHUN_HD inline void collide_cell(const CollTables& T, int l0, double* f00, double* fl, long long lstride, int ee,
                                  int eb, int nsub, double hsub, double Dt, double* w) {
    const int n = T.np;
    if (ee)
        for (int s = 0; s < nsub; ++s) ee_rk4(T, f00, hsub, w);
    if (!eb) return;
    double *ta = w + 8 * n, *tb = w + 9 * n, *tc = w + 10 * n, *sc = w + 11 * n, *x = w + 12 * n, *tw = w + 13 * n;
    reset_coeff(T, f00, Dt, ta, tb, tc, sc, tw);
    for (int l = 1; l <= l0; ++l) {
        double* d = fl + (long long)(l - 1) * lstride;
        thomas(ta, tb, tc, sc, l, n, d, x, tw);
        for (int i = 0; i < n; ++i) d[i] = x[i];
    }
}

// adjoint of collide_cell at its input (f00_in, fl_in): lam00 / laml hold the
// cotangents of the outputs and receive those of the inputs
OSHUN_HD inline void collide_cell_T(const CollTables& T, int l0, const double* f00_in, const double* fl_in,
                                    long long lstride, int ee, int eb, int nsub, double hsub, double Dt,
                                    double* lam00, double* laml, long long lamstride, double* w) {
    const int n = T.np;
    double* fstart = w;                       // (nsub + 1) np: f00 at each substep start, then after e-e
    double* g = fstart + (long long)nsub * n; // f00 after the e-e substeps
    double* rest = g + n;
    for (int i = 0; i < n; ++i) g[i] = f00_in[i];
    if (ee)
        for (int s = 0; s < nsub; ++s) {
            for (int i = 0; i < n; ++i) fstart[(long long)s * n + i] = g[i];
            ee_rk4(T, g, hsub, rest);
        }
    if (eb) {
        double *ta = rest, *tb = rest + n, *tc = rest + 2 * n, *sc = rest + 3 * n;
        double *la = rest + 4 * n, *lb = rest + 5 * n, *lc = rest + 6 * n, *ls = rest + 7 * n;
        double *x = rest + 8 * n, *y = rest + 9 * n, *tw = rest + 10 * n;
        reset_coeff(T, g, Dt, ta, tb, tc, sc, tw);
        for (int i = 0; i < n; ++i) { la[i] = 0.0; lb[i] = 0.0; lc[i] = 0.0; ls[i] = 0.0; }
        for (int l = 1; l <= l0; ++l) {
            const double ll1 = l * ((-0.5) * (l + 1.0));
            thomas(ta, tb, tc, sc, l, n, fl_in + (long long)(l - 1) * lstride, x, tw);
            double* lam = laml + (long long)(l - 1) * lamstride;
            thomas_T(ta, tb, tc, sc, l, n, lam, y, tw);
            for (int i = 0; i < n; ++i) {
                // dA/d(coefficients): row i holds a_i, b_i, c_i
                if (i >= 1) la[i] += -y[i] * x[i - 1];
                if (i + 1 < n) lc[i] += -y[i] * x[i + 1];
                const double lbi = -y[i] * x[i];
                if (!(i == 0 && l > 1)) lb[i] += lbi;
                ls[i] += -ll1 * lbi;
            }
            for (int i = 0; i < n; ++i) lam[i] = y[i];
        }
        reset_coeff_T(T, g, Dt, la, lb, lc, ls, lam00, tw);
    }
    if (ee)
        for (int s = nsub - 1; s >= 0; --s) ee_rk4_T(T, fstart + (long long)s * n, lam00, hsub, rest);
}

}  // namespace adj
}  // namespace oshun
