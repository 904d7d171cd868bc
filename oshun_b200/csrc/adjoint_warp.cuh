// Warp-cooperative form of the collision step's transpose (adjoint_math.h
// collide_cell_T): one warp per cell, the work space in shared memory.  The
// pointwise loops run lane-strided, the cumulative integrals and their
// transposes are warp scans over contiguous runs of p per lane, the scalar
// sums are warp reductions, and the Thomas solves run on lane 0.  The
// arithmetic is the serial form's up to the order of the sums.
#pragma once

#include "adjoint_math.h"

namespace oshun {
namespace adjw {

using adj::CollTables;
constexpr unsigned kAll = 0xffffffffu;

__device__ __forceinline__ int lane_id() { return threadIdx.x & 31; }

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(kAll, v, off);
    return v;
}

// out[k] = sum_{i <= k} t(i) (forward) or sum_{i >= k} t(i) (backward), k < n;
// each lane sums a contiguous run, the run totals are scanned across the warp
template <bool FWD, class F>
__device__ void warp_cumsum(int n, F t, double* out) {
    const int lane = lane_id();
    const int E = (n + 31) >> 5;
    const int b = min(lane * E, n), e = min(b + E, n);
    double run = 0.0;
    for (int k = b; k < e; ++k) {
        const double v = t(k);
        out[k] = v;
        run += v;
    }
    double s = run;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        const double u = FWD ? __shfl_up_sync(kAll, s, off) : __shfl_down_sync(kAll, s, off);
        if (FWD ? lane >= off : lane + off < 32) s += u;
    }
    double r = FWD ? __shfl_up_sync(kAll, s, 1) : __shfl_down_sync(kAll, s, 1);
    if (FWD ? lane == 0 : lane == 31) r = 0.0;
    if (FWD) {
        for (int k = b; k < e; ++k) { r += out[k]; out[k] = r; }
    } else {
        for (int k = e - 1; k >= b; --k) { r += out[k]; out[k] = r; }
    }
    __syncwarp();
}

// the three cumulative integrals (adj::scans)
__device__ void scans(const CollTables& T, const double* f, double* I4, double* I2, double* J1) {
    const int n = T.np;
    warp_cumsum<true>(n, [&](int k) { return k >= 1 ? T.U4[k] * f[k] + T.U4m1[k] * f[k - 1] : 0.0; }, I4);
    warp_cumsum<true>(n, [&](int k) { return k >= 1 ? T.U2[k] * f[k] + T.U2m1[k] * f[k - 1] : 0.0; }, I2);
    warp_cumsum<false>(n, [&](int k) { return k + 1 < n ? T.U1[k + 1] * f[k + 1] + T.U1m1[k + 1] * f[k] : 0.0; },
                       J1);
}

// transpose (adj::scans_T): r4_i = sum_{j >= i} lI4_j, r2 likewise (i >= 1),
// r1_i = sum_{j < i} lJ1_j; w: 3 np
__device__ void scans_T(const CollTables& T, const double* lI4, const double* lI2, const double* lJ1, double* lf,
                        double* w) {
    const int n = T.np;
    double *R4 = w, *R2 = w + n, *R1 = w + 2 * n;
    warp_cumsum<false>(n, [&](int k) { return lI4[k]; }, R4);
    warp_cumsum<false>(n, [&](int k) { return lI2[k]; }, R2);
    warp_cumsum<true>(n, [&](int k) { return lJ1[k]; }, R1);   // R1[k] = sum_{j <= k}: r1_i = R1[i-1]
    for (int k = lane_id(); k < n; k += 32) {
        double a = 0.0;
        if (k >= 1) a += R4[k] * T.U4[k] + R2[k] * T.U2[k] + R1[k - 1] * T.U1[k];
        if (k + 1 < n) a += R4[k + 1] * T.U4m1[k + 1] + R2[k + 1] * T.U2m1[k + 1] + R1[k] * T.U1m1[k + 1];
        lf[k] += a;
    }
    __syncwarp();
}

// G of the e-e flux at k (adj::ee_slope)
__device__ __forceinline__ double ee_G(const CollTables& T, const double* f, const double* I4, const double* I2,
                                       const double* J1, int k, double f00, double v1s) {
    if (k < T.NB) {
        const double v3 = T.U3[k], v5 = T.V5[k], v7 = T.V7[k];
        const double i2s = f00 * v3 / 3.0 + (f[1] - f00) * v5 / v1s * 0.2;
        const double i4s = f00 * v5 * 0.2 + (f[1] - f00) * v7 / (v1s * 7.0);
        return f[k] * i4s + (v3 * f[k] - 3.0 * i2s) * J1[k];
    }
    return (I4[k] + T.U3[k] * J1[k]) * f[k] - 3.0 * I2[k] * J1[k];
}

// e-e slope (adj::ee_slope); w: 5 np
__device__ void ee_slope(const CollTables& T, const double* f, double* fh, double* w) {
    const int n = T.np;
    double *I4 = w, *I2 = w + n, *J1 = w + 2 * n, *G = w + 3 * n, *D = w + 4 * n;
    adjw::scans(T, f, I4, I2, J1);
    double dn, dT;
    const double lnee = adj::log_ee_d(4.0 * adj::kPi * I2[n - 1], 4.0 * adj::kPi * I4[n - 1], T.density_np, &dn, &dT);
    const double v0s = T.vr[0] * T.vr[0], v1s = T.vr[1] * T.vr[1];
    const double f00 = (f[0] - f[1] * v0s / v1s) / (1.0 - v0s / v1s);
    for (int k = lane_id(); k < n; k += 32) G[k] = ee_G(T, f, I4, I2, J1, k, f00, v1s);
    __syncwarp();
    for (int k = lane_id(); k < n; k += 32) D[k] = (k < n - 1) ? (G[k] - G[k + 1]) * T.Pn[k] : G[k];
    __syncwarp();
    const double norm = T.c_kpre * lnee;
    for (int k = lane_id(); k < n; k += 32) {
        const double r = k == 0 ? ((-G[0]) * (2.0 / v0s) - D[0]) * T.Qn[0] : T.Qn[k] * (D[k - 1] - D[k]);
        fh[k] = r * norm;
    }
    __syncwarp();
}

// transpose of the slope's derivative at f: mu -> lf (added); w: 16 np
__device__ void ee_slope_T(const CollTables& T, const double* f, const double* mu, double* lf, double* w) {
    const int n = T.np;
    const int lane = lane_id();
    double *I4 = w, *I2 = w + n, *J1 = w + 2 * n, *G = w + 3 * n, *D = w + 4 * n;
    double *lG = w + 5 * n, *lD = w + 6 * n, *lI4 = w + 7 * n, *lI2 = w + 8 * n, *lJ1 = w + 9 * n;
    double* raw = w + 10 * n;
    double* sw = w + 13 * n;
    adjw::scans(T, f, I4, I2, J1);
    double dn, dT;
    const double lnee = adj::log_ee_d(4.0 * adj::kPi * I2[n - 1], 4.0 * adj::kPi * I4[n - 1], T.density_np, &dn, &dT);
    const double v0s = T.vr[0] * T.vr[0], v1s = T.vr[1] * T.vr[1];
    const double r = v0s / v1s;
    const double f00 = (f[0] - f[1] * r) / (1.0 - r);
    for (int k = lane; k < n; k += 32) G[k] = ee_G(T, f, I4, I2, J1, k, f00, v1s);
    __syncwarp();
    for (int k = lane; k < n; k += 32) D[k] = (k < n - 1) ? (G[k] - G[k + 1]) * T.Pn[k] : G[k];
    __syncwarp();
    const double norm = T.c_kpre * lnee;
    double part = 0.0;
    for (int k = lane; k < n; k += 32) {
        raw[k] = k == 0 ? ((-G[0]) * (2.0 / v0s) - D[0]) * T.Qn[0] : T.Qn[k] * (D[k - 1] - D[k]);
        part += mu[k] * raw[k];
    }
    const double l_norm = warp_sum(part);
    // lD_k = -lr_k Qn_k + lr_{k+1} Qn_{k+1}, lr = mu * norm
    for (int k = lane; k < n; k += 32) {
        double v = -(mu[k] * norm) * T.Qn[k];
        if (k + 1 < n) v += (mu[k + 1] * norm) * T.Qn[k + 1];
        lD[k] = v;
    }
    __syncwarp();
    for (int k = lane; k < n; k += 32) {
        double v = (k < n - 1) ? lD[k] * T.Pn[k] : lD[k];
        if (k >= 1) v -= lD[k - 1] * T.Pn[k - 1];
        if (k == 0) v += -(mu[0] * norm) * T.Qn[0] * (2.0 / v0s);
        lG[k] = v;
    }
    __syncwarp();
    double l_f00 = 0.0, l_f1 = 0.0;
    for (int k = lane; k < n; k += 32) {
        const double lg = lG[k];
        double li4 = 0.0, li2 = 0.0, lj1;
        if (k < T.NB) {
            const double v3 = T.U3[k], v5 = T.V5[k], v7 = T.V7[k];
            const double i2s = f00 * v3 / 3.0 + (f[1] - f00) * v5 / v1s * 0.2;
            const double i4s = f00 * v5 * 0.2 + (f[1] - f00) * v7 / (v1s * 7.0);
            lf[k] += lg * (i4s + v3 * J1[k]);
            const double l_i4s = lg * f[k];
            const double l_i2s = -3.0 * lg * J1[k];
            lj1 = lg * (v3 * f[k] - 3.0 * i2s);
            l_f00 += l_i2s * (v3 / 3.0 - v5 / v1s * 0.2) + l_i4s * (v5 * 0.2 - v7 / (v1s * 7.0));
            l_f1 += l_i2s * (v5 / v1s * 0.2) + l_i4s * (v7 / (v1s * 7.0));
        } else {
            li4 = lg * f[k];
            lj1 = lg * (T.U3[k] * f[k] - 3.0 * I2[k]);
            lf[k] += lg * (I4[k] + T.U3[k] * J1[k]);
            li2 = -3.0 * lg * J1[k];
        }
        lI4[k] = li4;
        lI2[k] = li2;
        lJ1[k] = lj1;
    }
    l_f00 = warp_sum(l_f00);
    l_f1 = warp_sum(l_f1);
    __syncwarp();
    if (lane == 0) {
        lf[0] += l_f00 / (1.0 - r);
        lf[1] += l_f1 - l_f00 * r / (1.0 - r);
        const double l_lnee = l_norm * T.c_kpre;
        lI2[n - 1] += l_lnee * dn * 4.0 * adj::kPi;
        lI4[n - 1] += l_lnee * dT * 4.0 * adj::kPi;
    }
    __syncwarp();
    adjw::scans_T(T, lI4, lI2, lJ1, lf, sw);
}

// one RK4 substep (adj::ee_rk4); w: 8 np
__device__ void ee_rk4(const CollTables& T, double* f, double h, double* w) {
    const int n = T.np;
    double *s = w, *k = w + n, *acc = w + 2 * n, *sw = w + 3 * n;
    for (int i = lane_id(); i < n; i += 32) acc[i] = 0.0;
    const double c_in[4] = {0.0, 0.5 * h, 0.5 * h, h}, c_out[4] = {h / 6.0, h / 3.0, h / 3.0, h / 6.0};
    for (int st = 0; st < 4; ++st) {
        for (int i = lane_id(); i < n; i += 32) s[i] = f[i] + (st == 0 ? 0.0 : c_in[st] * k[i]);
        __syncwarp();
        adjw::ee_slope(T, s, k, sw);
        for (int i = lane_id(); i < n; i += 32) acc[i] += c_out[st] * k[i];
        __syncwarp();
    }
    for (int i = lane_id(); i < n; i += 32) f[i] += acc[i];
    __syncwarp();
}

// its transpose (adj::ee_rk4_T); w: 27 np
__device__ void ee_rk4_T(const CollTables& T, const double* f, double* lam, double h, double* w) {
    const int n = T.np;
    double *S = w, *K = w + 4 * n, *c = w + 8 * n, *a = w + 9 * n, *lout = w + 10 * n, *sw = w + 11 * n;
    const double c_in[4] = {0.0, 0.5 * h, 0.5 * h, h};
    for (int st = 0; st < 4; ++st) {
        for (int i = lane_id(); i < n; i += 32) S[st * n + i] = f[i] + (st == 0 ? 0.0 : c_in[st] * K[(st - 1) * n + i]);
        __syncwarp();
        adjw::ee_slope(T, S + st * n, K + st * n, sw);
    }
    for (int i = lane_id(); i < n; i += 32) { lout[i] = lam[i]; a[i] = 0.0; }
    __syncwarp();
    const double w_out[4] = {h / 6.0, h / 3.0, h / 3.0, h / 6.0};
    for (int st = 3; st >= 0; --st) {
        const double w_next = st < 3 ? c_in[st + 1] : 0.0;
        for (int i = lane_id(); i < n; i += 32) { c[i] = w_out[st] * lout[i] + w_next * a[i]; }
        __syncwarp();
        for (int i = lane_id(); i < n; i += 32) a[i] = 0.0;
        __syncwarp();
        adjw::ee_slope_T(T, S + st * n, c, a, sw);
        for (int i = lane_id(); i < n; i += 32) lam[i] += a[i];
        __syncwarp();
    }
}

// tridiagonal coefficients of reset_coeff (adj::reset_coeff); w: 3 np
__device__ void reset_coeff(const CollTables& T, const double* f, double Dt, double* ta, double* tb, double* tc,
                            double* scat, double* w) {
    const int n = T.np;
    double *I2 = w, *I0 = w + n, *J1 = w + 2 * n;
    adjw::scans(T, f, I2, I0, J1);
    const double Tt = I2[n - 1] * (4.0 * adj::kPi), N = I0[n - 1] * (4.0 * adj::kPi);
    double d1, d2, d3, d4;
    const double lnee = adj::log_ee_d(N, Tt, T.density_np, &d1, &d2);
    const double zl = adj::zlog_ei_d(N, Tt, T.density_np, T.Zeta, &d3, &d4);
    const double scale = (-1.0) * lnee * T.kpre * Dt;
    const double* vr = T.vr;
    for (int k = lane_id(); k < n; k += 32) {
        const double i2 = I2[k] * (4.0 * adj::kPi) / (vr[k] * vr[k]);
        const double i0 = I0[k] * (4.0 * adj::kPi);
        const double j1m = J1[k] * (4.0 * adj::kPi * vr[k]);
        const double t1 = i0 + (2.0 * j1m - i2) / 3.0;
        const double t2 = (i2 + j1m) / 3.0;
        scat[k] = (((k == 0) ? 0.0 : t1 * lnee) + zl * N) / T.U3[k] * (T.kpre * Dt);
        double a = 0.0, b = 0.0, c = 0.0;
        if (k == 0) {
            b = 8.0 * adj::kPi * f[0] * scale;
        } else if (k < n - 1) {
            const double Dm = 1.0 / (vr[k] * 0.5 * (vr[k + 1] - vr[k - 1]) * (vr[k] - vr[k - 1]));
            const double Dp = 1.0 / (vr[k] * 0.5 * (vr[k + 1] - vr[k - 1]) * (vr[k + 1] - vr[k]));
            const double S2 = 1.0 / (vr[k] * vr[k] * (vr[k + 1] - vr[k - 1]));
            b = (8.0 * adj::kPi * f[k] - t2 * (Dm + Dp)) * scale;
            a = (t2 * Dm - t1 * S2) * scale;
            c = (t2 * Dp + t1 * S2) * scale;
        }
        ta[k] = a; tb[k] = b; tc[k] = c;
    }
    __syncwarp();
}

// its transpose (adj::reset_coeff_T): cotangents of ta, tb, tc, scat -> lf (added); w: 9 np
__device__ void reset_coeff_T(const CollTables& T, const double* f, double Dt, const double* la, const double* lb,
                              const double* lc, const double* ls, double* lf, double* w) {
    const int n = T.np;
    const int lane = lane_id();
    double *I2 = w, *I0 = w + n, *J1 = w + 2 * n, *lI2 = w + 3 * n, *lI0 = w + 4 * n, *lJ1 = w + 5 * n;
    double* sw = w + 6 * n;
    adjw::scans(T, f, I2, I0, J1);
    const double Tt = I2[n - 1] * (4.0 * adj::kPi), N = I0[n - 1] * (4.0 * adj::kPi);
    double le_dN, le_dT, zl_dN, zl_dT;
    const double lnee = adj::log_ee_d(N, Tt, T.density_np, &le_dN, &le_dT);
    const double zl = adj::zlog_ei_d(N, Tt, T.density_np, T.Zeta, &zl_dN, &zl_dT);
    const double scale = (-1.0) * lnee * T.kpre * Dt;
    const double* vr = T.vr;
    double l_scale = 0.0, l_lnee = 0.0, l_zl = 0.0, l_N = 0.0;
    for (int k = lane; k < n; k += 32) {
        const double i2 = I2[k] * (4.0 * adj::kPi) / (vr[k] * vr[k]);
        const double i0 = I0[k] * (4.0 * adj::kPi);
        const double j1m = J1[k] * (4.0 * adj::kPi * vr[k]);
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
            lf[0] += lb[0] * 8.0 * adj::kPi * scale;
            l_scale += lb[0] * 8.0 * adj::kPi * f[0];
        } else if (k < n - 1) {
            const double Dm = 1.0 / (vr[k] * 0.5 * (vr[k + 1] - vr[k - 1]) * (vr[k] - vr[k - 1]));
            const double Dp = 1.0 / (vr[k] * 0.5 * (vr[k + 1] - vr[k - 1]) * (vr[k + 1] - vr[k]));
            const double S2 = 1.0 / (vr[k] * vr[k] * (vr[k + 1] - vr[k - 1]));
            lf[k] += lb[k] * 8.0 * adj::kPi * scale;
            l_t2 += (-lb[k] * (Dm + Dp) + la[k] * Dm + lc[k] * Dp) * scale;
            l_t1 += (-la[k] * S2 + lc[k] * S2) * scale;
            l_scale += lb[k] * (8.0 * adj::kPi * f[k] - t2 * (Dm + Dp)) + la[k] * (t2 * Dm - t1 * S2) +
                       lc[k] * (t2 * Dp + t1 * S2);
        }
        const double l_i0 = l_t1;
        const double l_j1m = 2.0 / 3.0 * l_t1 + l_t2 / 3.0;
        const double l_i2 = -l_t1 / 3.0 + l_t2 / 3.0;
        lI2[k] = l_i2 * (4.0 * adj::kPi) / (vr[k] * vr[k]);
        lI0[k] = l_i0 * (4.0 * adj::kPi);
        lJ1[k] = l_j1m * (4.0 * adj::kPi * vr[k]);
    }
    l_scale = warp_sum(l_scale);
    l_lnee = warp_sum(l_lnee);
    l_zl = warp_sum(l_zl);
    l_N = warp_sum(l_N);
    __syncwarp();
    if (lane == 0) {
        l_lnee += l_scale * (-1.0) * T.kpre * Dt;
        l_N += l_lnee * le_dN + l_zl * zl_dN;
        const double l_T = l_lnee * le_dT + l_zl * zl_dT;
        lI0[n - 1] += l_N * (4.0 * adj::kPi);
        lI2[n - 1] += l_T * (4.0 * adj::kPi);
    }
    __syncwarp();
    adjw::scans_T(T, lI2, lI0, lJ1, lf, sw);
}

// Thomas solves on lane 0 (adj::thomas, adj::thomas_T); w: np
__device__ void thomas(const double* a, const double* tb, const double* c, const double* scat, int l, int n,
                       const double* d, double* x, double* w) {
    if (lane_id() == 0) adj::thomas(a, tb, c, scat, l, n, d, x, w);
    __syncwarp();
}
__device__ void thomas_T(const double* a, const double* tb, const double* c, const double* scat, int l, int n,
                         const double* r, double* y, double* w) {
    if (lane_id() == 0) adj::thomas_T(a, tb, c, scat, l, n, r, y, w);
    __syncwarp();
}

// Work space of collide_cell_T below (doubles): the substep starts, the
// post-e-e f00 and 27 np of scratch
__host__ __device__ inline long long coll_ws(int np, int nsub) { return (long long)np * (nsub + 1 + 27); }

// the collided planes of a cell: for each l >= 1 the planes of m <= min(l,
// mmax) (Re, and Im for m > 0), all sharing the l matrix; plane q of the
// cell is at base + q * stride
struct CellPlanes {
    const int* plane_of;   // [(l0+1)(m0+1)]: plane of Re f_lm
    int m0, mmax;
};

// adj::collide_cell_T on one warp: lam00 / laml hold the cotangents of the
// outputs and receive those of the inputs.  Without `P` (plane_of null) the
// planes are f_l, l = 1..l0, lstride apart (m0 = 0); with it, every
// collided plane of each l (lstride, lamstride: the plane strides)
__device__ void collide_cell_T(const CollTables& T, int l0, const double* f00_in, const double* fl_in,
                               long long lstride, int ee, int eb, int nsub, double hsub, double Dt, double* lam00,
                               double* laml, long long lamstride, double* w, const CellPlanes P = {nullptr, 0, 0}) {
    const int n = T.np;
    const int lane = lane_id();
    double* fstart = w;
    double* g = fstart + (long long)nsub * n;
    double* rest = g + n;
    for (int i = lane; i < n; i += 32) g[i] = f00_in[i];
    __syncwarp();
    if (ee)
        for (int s = 0; s < nsub; ++s) {
            for (int i = lane; i < n; i += 32) fstart[(long long)s * n + i] = g[i];
            __syncwarp();
            adjw::ee_rk4(T, g, hsub, rest);
        }
    if (eb) {
        double *ta = rest, *tb = rest + n, *tc = rest + 2 * n, *sc = rest + 3 * n;
        double *la = rest + 4 * n, *lb = rest + 5 * n, *lc = rest + 6 * n, *ls = rest + 7 * n;
        double *x = rest + 8 * n, *y = rest + 9 * n, *tw = rest + 10 * n;
        adjw::reset_coeff(T, g, Dt, ta, tb, tc, sc, tw);
        for (int i = lane; i < n; i += 32) { la[i] = 0.0; lb[i] = 0.0; lc[i] = 0.0; ls[i] = 0.0; }
        __syncwarp();
        for (int l = 1; l <= l0; ++l) {
            const double ll1 = l * ((-0.5) * (l + 1.0));
            const int mtop = P.plane_of ? (l < P.mmax ? l : P.mmax) : 0;
            for (int m = 0; m <= mtop; ++m)
                for (int comp = 0; comp < (m > 0 ? 2 : 1); ++comp) {
                    const long long q =
                        P.plane_of ? (long long)P.plane_of[l * (P.m0 + 1) + m] + comp : (long long)(l - 1);
                    thomas(ta, tb, tc, sc, l, n, fl_in + q * lstride, x, tw);
                    double* lam = laml + q * lamstride;
                    thomas_T(ta, tb, tc, sc, l, n, lam, y, tw);
                    for (int i = lane; i < n; i += 32) {
                        if (i >= 1) la[i] += -y[i] * x[i - 1];
                        if (i + 1 < n) lc[i] += -y[i] * x[i + 1];
                        const double lbi = -y[i] * x[i];
                        if (!(i == 0 && l > 1)) lb[i] += lbi;
                        ls[i] += -ll1 * lbi;
                    }
                    __syncwarp();
                    for (int i = lane; i < n; i += 32) lam[i] = y[i];
                    __syncwarp();
                }
        }
        adjw::reset_coeff_T(T, g, Dt, la, lb, lc, ls, lam00, tw);
    }
    if (ee)
        for (int s = nsub - 1; s >= 0; --s) adjw::ee_rk4_T(T, fstart + (long long)s * n, lam00, hsub, rest);
}

}  // namespace adjw
}  // namespace oshun
