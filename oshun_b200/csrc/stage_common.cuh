// Device pieces shared by the RK4-stage kernels: the RK epilogue and the
// couplings of one source harmonic (l = s, m) into the accumulators of target
// rows s-1, s, s+1 (see vlasov.cu for the list and the reference lines).
#pragma once

#include "oshun_internal.h"

namespace oshun {

// Roundings spelled out: the RK updates and the field updates run in several
// kernels (single-problem, batched, global-load), and a product the compiler
// fused into an add in one and not in another would make their results
// differ in the last bit
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float add_rn(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ double add_rn(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float fma_rn(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ double fma_rn(double a, double b, double c) { return __fma_rn(a, b, c); }

// out/B/A are base pointers (out may be null: stage 4 has no next input)
template <typename TS>
__device__ __forceinline__ void rk_update(int mode, int first, double c1, double c2, TS* out, const TS* B, TS* A,
                                          long long i, TS k) {
    if (mode == 1) { out[i] = k; return; }
    const TS t = mul_rn(k, (TS)c1);
    const TS b = B[i];
    if (out) out[i] = add_rn(b, t);
    A[i] = fma_rn(t, (TS)c2, first ? b : A[i]);
}

// Couplings of source (s, m) at one momentum point.  fr/fi: value, frm/frp
// (fim/fip): p-1/p+1 neighbours, dxr/dxi = v (f[x-1]-f[x+1]), dyr/dyi likewise
// in y.  R[0..2] / I[0..2] are the target rows s-1, s, s+1.
template <int MC, typename TS>
__device__ __forceinline__ void couple(TS (&ar)[3][MC + 1], TS (&ai)[3][MC + 1], const int m, const int s,
                                       const CoefLM& c, const TS fr, const TS fi, const TS frm, const TS frp,
                                       const TS fim, const TS fip, const TS dxr, const TS dxi, const TS dyr,
                                       const TS dyi, const bool has_y, const int p, const int np, const TS invp,
                                       const TS ex, const TS ey, const TS ez, const TS bx, const TS by, const TS bz,
                                       const double g00_s, const double g00_inv, const double g00_gr) {
    // G and H (MakeGH / G00), Dp f = f[p-1] - f[p+1], 0 at p0, f[np-2]-f[np-1] at the end
    TS Gr, Gi, Hr, Hi;
    const TS dr = (p == 0) ? TS(0) : (p == np - 1 ? frm - fr : frm - frp);
    const TS di = (p == 0) ? TS(0) : (p == np - 1 ? fim - fi : fim - fip);
    if (s == 0) {
        Gr = dr; Gi = 0; Hr = 0; Hi = 0;
        if (p == 0) {
            const TS f00x = (fr - frp * (TS)g00_s) * (TS)g00_inv;
            Gr = (frp - f00x) * (TS)g00_gr;
        }
    } else {
        const TS ipx = invp * (TS)c.invpax;
        const TS gf = (TS)c.gfac;
        Hr = fr * ipx + dr; Hi = fi * ipx + di;
        Gr = dr * gf + Hr;  Gi = di * gf + Hi;
        if (p == 0) {
            const TS hp0 = (TS)c.hp0;
            Gr = 0; Gi = 0; Hr = frp * hp0; Hi = fip * hp0;
        }
    }
    const int mp = m + 1 <= MC ? m + 1 : MC;
    const int mm = m >= 1 ? m - 1 : 0;
    // E field
    {
        const TS cg = (TS)c.ex_g * ex, ch = (TS)c.ex_h * ex;
        ar[2][m] += cg * Gr; ai[2][m] += cg * Gi;
        ar[0][m] += ch * Hr; ai[0][m] += ch * Hi;
        if (m + 1 <= MC) {
            const TS eg = (TS)c.em_g, eh = (TS)c.em_h;
            ar[2][mp] += eg * (ey * Gr + ez * Gi); ai[2][mp] += eg * (ey * Gi - ez * Gr);
            ar[0][mp] += eh * (ey * Hr + ez * Hi); ai[0][mp] += eh * (ey * Hi - ez * Hr);
        }
        if (m >= 1) {
            const TS ph = (TS)c.ep_h, pg = (TS)c.ep_g;
            ar[0][mm] += ph * (ey * Hr - ez * Hi);
            ar[2][mm] += pg * (ey * Gr - ez * Gi);
            if (m >= 2) {
                ai[0][mm] += ph * (ey * Hi + ez * Hr);
                ai[2][mm] += pg * (ey * Gi + ez * Gr);
            }
        }
    }
    // B field
    {
        if (m + 1 <= MC) {
            ar[1][mp] += TS(0.5) * (bz * fr - by * fi);
            ai[1][mp] += TS(0.5) * (bz * fi + by * fr);
        }
        if (m >= 1) {
            const TS mb = (TS)m * bx;
            ar[1][m] += mb * fi; ai[1][m] += -(mb * fr);
            const TS cb = (TS)c.b_m;
            ar[1][mm] += cb * (bz * fr + by * fi);
            if (m >= 2) ai[1][mm] += cb * (bz * fi - by * fr);
        }
    }
    // x advection
    {
        const TS xp = (TS)c.ax_p, xm = (TS)c.ax_m;
        ar[2][m] += xp * dxr; ai[2][m] += xp * dxi;
        ar[0][m] += xm * dxr; ai[0][m] += xm * dxi;
    }
    // y advection
    if (has_y) {
        if (m + 1 <= MC) {
            const TS pp = (TS)c.ay_pp, mp_ = (TS)c.ay_mp;
            ar[2][mp] += pp * dyr; ai[2][mp] += pp * dyi;
            ar[0][mp] += mp_ * dyr; ai[0][mp] += mp_ * dyi;
        }
        if (m >= 1) {
            const TS ym_ = (TS)c.ay_mm, yp_ = (TS)c.ay_pm;
            ar[0][mm] += ym_ * dyr; ar[2][mm] += yp_ * dyr;
            if (m >= 2) { ai[0][mm] += ym_ * dyi; ai[2][mm] += yp_ * dyi; }
        }
    }
}

template <int MC, typename TS>
__device__ __forceinline__ void rotate_rows(TS (&ar)[3][MC + 1], TS (&ai)[3][MC + 1]) {
#pragma unroll
    for (int m = 0; m <= MC; ++m) {
        ar[0][m] = ar[1][m]; ai[0][m] = ai[1][m];
        ar[1][m] = ar[2][m]; ai[1][m] = ai[2][m];
        ar[2][m] = 0;        ai[2][m] = 0;
    }
}

}  // namespace oshun
