// Moments of the distribution on the device: the output quantities of
// Parallel_Output::nonrelativistic_moments (OSHUN-1/def-Parallel.cpp:1677-2258)
// for every cell, so that a diagnostic step copies numx*numy floats per
// moment instead of the whole state.
//
// The reference accumulates each moment in a Matrix2D<float>: every term is a
// double expression added to the float running value (float += double
// rounds the double sum to float), and the scalings are float multiplies by
// constants rounded to float.  moments_cell_kernel keeps that order of
// operations (p from 0 upwards, the same grouping of each product), so the
// results agree with the reference's to a few float ulps (the remaining
// differences come from the host's and the device's pow, sqrt and log).
//
// One warp per 32 cells: each needed momentum row of the 32 cells is staged
// through shared memory with coalesced loads, then each lane sums its cell's
// row in order.  A second kernel takes the x and y differences of <v^2>^2
// for the heat conductivities Kx, Ky.
#include <float.h>

#include "oshun_internal.h"

namespace oshun {
namespace {

constexpr int kMomWarps = 4;   // warps (32 cells each) per CTA

template <typename TP>
__device__ __forceinline__ double plane_at(const void* planes, long long q, long long pstride, long long i) {
    return (double)reinterpret_cast<const TP*>(planes)[q * pstride + i];
}

// float += double, as Matrix2D<float>(i,j) += <double expression>
__device__ __forceinline__ float fadd_d(float acc, double t) { return __double2float_rn(__dadd_rn((double)acc, t)); }

template <typename TP>
__global__ void __launch_bounds__(32 * kMomWarps) moments_cell_kernel(const MomentArgs a) {
    extern __shared__ double srow[];   // [warps][32][np + 1]
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int n = a.np, ld = n + 1;
    double* rows = srow + (size_t)warp * 32 * ld;
    const long long cell0 = ((long long)blockIdx.x * kMomWarps + warp) * 32;
    if (cell0 >= a.cells) return;
    const long long cell = cell0 + lane;
    const bool valid = cell < a.cells;
    const double* pr = a.pr;
    const double* ig = a.invgamma;
    const double dx = a.dp;
    const double p0 = pr[0], pl = pr[n - 1];
    const double q = a.p0p1_sq, iq = a.inv_mp0p1_sq;

    // stage one momentum row of the warp's 32 cells (plane q, -1 = f00, -2 = absent)
    auto stage = [&](const int which) {
        __syncwarp();
        const int nc = (int)min(32LL, a.cells - cell0);
        for (int idx = lane; idx < 32 * n; idx += 32) {
            const int c = idx / n, p = idx - c * n;
            double v = 0.0;
            if (c < nc && which != -2) {
                const long long i = (cell0 + c) * n + p;
                v = which == -1 ? a.f00[i]
                                : plane_at<TP>(a.planes, which, a.pstride, i) + (a.pl_ref ? a.pl_ref[(long long)which * n + p] : 0.0);
            }
            rows[c * ld + p] = v;
        }
        __syncwarp();
    };
    const double* my = rows + (size_t)lane * ld;
    auto f = [&](int ip) { return my[ip]; };

    // ---- density (def-Parallel.cpp:1700-1728) ----
    stage(-1);
    // ends F0(0)*pr(0)*pr(0), interior pr*pr*F0: (f p) p and (p p) f
    float dens = __double2float_rn(__dmul_rn(__dmul_rn(f(0), p0), p0));
    dens = fadd_d(dens, __dmul_rn(__dmul_rn(f(n - 1), pl), pl));
    dens = __double2float_rn(__dmul_rn((double)dens, 0.5));
    for (int ip = 1; ip < n - 1; ++ip) dens = fadd_d(dens, __dmul_rn(__dmul_rn(pr[ip], pr[ip]), f(ip)));
    double c0 = __dmul_rn(__ddiv_rn(f(1), 5.0), q);
    c0 = __dadd_rn(c0, __dmul_rn(__dmul_rn(__dsub_rn(f(0), __dmul_rn(f(1), q)), iq),
                                 __dsub_rn(1.0 / 3.0, __dmul_rn(1.0 / 5.0, q))));
    c0 = __dmul_rn(c0, __dmul_rn(__dmul_rn(p0, __ddiv_rn(p0, dx)), p0));
    dens = fadd_d(dens, c0);
    dens = __fmul_rn(dens, a.s_dens);
    if ((double)dens < 4.0 * FLT_EPSILON) dens = 1.0f;

    // ---- moment_1: f00 with p^4/gamma^2 (def-Parallel.cpp:1810-1832) ----
    float m1;
    {
        m1 = __double2float_rn(__dmul_rn(__dmul_rn(f(0), a.pow4[0]), a.ig2[0]));
        m1 = fadd_d(m1, __dmul_rn(__dmul_rn(f(n - 1), a.pow4[n - 1]), a.ig2[n - 1]));
        m1 = __double2float_rn(__dmul_rn((double)m1, 0.5));
        for (int ip = 1; ip < n - 1; ++ip) m1 = fadd_d(m1, __dmul_rn(__dmul_rn(a.pow4[ip], a.ig2[ip]), f(ip)));
        double c = __dmul_rn(__ddiv_rn(f(1), 7.0), q);
        c = __dadd_rn(c, __dmul_rn(__dmul_rn(__dsub_rn(f(0), __dmul_rn(f(1), q)), iq),
                                   __dsub_rn(1.0 / 5.0, __dmul_rn(1.0 / 7.0, q))));
        c = __dmul_rn(c, __dmul_rn(a.pow4[0], __ddiv_rn(p0, dx)));
        m1 = fadd_d(m1, c);
        m1 = __fmul_rn(m1, a.s_v1);   // 4 pi/3 dp, as for Vx
    }

    // f_l1-type velocity integral: ends and interior with p^k/gamma^j, the p0
    // term f(1) p0^(k+2)/(dx p1 (k+2)) (def-Parallel.cpp:1738-1756, 2106-2124)
    auto vel_int = [&](const double* powk, const double* igj, const double corr) {
        float v = __double2float_rn(__dmul_rn(__dmul_rn(f(0), powk[0]), igj[0]));
        v = fadd_d(v, __dmul_rn(__dmul_rn(f(n - 1), powk[n - 1]), igj[n - 1]));
        v = __double2float_rn(__dmul_rn((double)v, 0.5));
        for (int ip = 1; ip < n - 1; ++ip) v = fadd_d(v, __dmul_rn(__dmul_rn(powk[ip], igj[ip]), f(ip)));
        v = fadd_d(v, __dmul_rn(f(1), corr));
        return v;
    };
    // l = 2 integrals: no p = 0 end, p^4/gamma^2 (def-Parallel.cpp:1836-1848)
    auto l2_int = [&](const bool sq_form) {
        float v = 0.0f;
        v = fadd_d(v, __dmul_rn(__dmul_rn(f(n - 1), a.pow4[n - 1]), a.ig2[n - 1]));
        v = __double2float_rn(__dmul_rn((double)v, 0.5));
        for (int ip = 1; ip < n - 1; ++ip) {
            // VxVz writes invgamma*invgamma where the others write pow(invgamma, 2)
            const double w = sq_form ? __dmul_rn(__dmul_rn(a.pow4[ip], ig[ip]), ig[ip])
                                     : __dmul_rn(a.pow4[ip], a.ig2[ip]);
            v = fadd_d(v, __dmul_rn(w, f(ip)));
        }
        return v;
    };

    // ---- Vx, Vy (f10, Re f11) ----
    stage(a.q10);
    float vx = a.q10 >= 0 ? vel_int(a.pow3, ig, a.corr5) : 0.0f;
    vx = __fmul_rn(vx, a.s_v1);
    vx = __fdiv_rn(vx, dens);
    float qx2 = 0.0f;
    if (a.q10 >= 0) {
        qx2 = vel_int(a.pow5, a.ig3, a.corr7);
        qx2 = __fmul_rn(qx2, a.s_v1);
    }
    stage(a.q11);
    float vy = a.q11 >= 0 ? vel_int(a.pow3, ig, a.corr5) : 0.0f;
    vy = __fmul_rn(vy, a.s_v2);
    vy = __fdiv_rn(vy, dens);
    float qy2 = 0.0f;
    if (a.q11 >= 0) {
        qy2 = vel_int(a.pow5, a.ig3, a.corr7);
        qy2 = __fmul_rn(qy2, a.s_v2);
    }

    // ---- VxVx, VyVy, VzVz (f00, f20) ----
    stage(a.q20);
    float m2 = a.q20 >= 0 ? l2_int(false) : 0.0f;
    float vyvy_raw = m2;                      // the reference's VyVy integrates f20 again
    m2 = __fmul_rn(m2, a.s_m2);
    float vxvx = __fadd_rn(m1, m2);
    vxvx = __fdiv_rn(vxvx, dens);
    m2 = __fmul_rn(m2, 0.5f);
    m1 = __fsub_rn(m1, m2);
    float vyvy = __fmul_rn(vyvy_raw, a.s_vyvy);
    m2 = vyvy;
    vyvy = __fadd_rn(vyvy, m1);
    vyvy = __fdiv_rn(vyvy, dens);
    float vzvz = __fsub_rn(m1, m2);
    vzvz = __fdiv_rn(vzvz, dens);

    // ---- VxVy (Re f21), VxVz (Im f21), VyVz (Im f22) ----
    stage(a.q21);
    float vxvy = a.q21 >= 0 ? l2_int(false) : 0.0f;
    vxvy = __fdiv_rn(__fmul_rn(vxvy, a.s_vxvy), dens);
    stage(a.q21 >= 0 ? a.q21 + 1 : -2);
    float vxvz = a.q21 >= 0 ? l2_int(true) : 0.0f;
    vxvz = __fdiv_rn(__fmul_rn(vxvz, a.s_vxvz), dens);
    stage(a.q22 >= 0 ? a.q22 + 1 : -2);
    float vyvz = a.q22 >= 0 ? l2_int(false) : 0.0f;
    vyvz = __fdiv_rn(__fmul_rn(vyvz, a.s_vyvz), dens);

    // ---- <v^2>, T, P, ND, nu (def-Parallel.cpp:2024-2083) ----
    float vsq = 0.0f;
    vsq = __fadd_rn(vsq, vxvx);
    vsq = __fadd_rn(vsq, vyvy);
    vsq = __fadd_rn(vsq, vzvz);
    vsq = __fsub_rn(vsq, __fmul_rn(vx, vx));
    vsq = __fsub_rn(vsq, __fmul_rn(vy, vy));
    const float tev = __fmul_rn(vsq, 170880.776f);
    // the reference scales <v^2> to eV for the temperature output and back
    // (def-Parallel.cpp:2039-2045); what follows uses the round-tripped value
    const float vsq_out = vsq;
    vsq = __fmul_rn(tev, (float)(1.0 / 170880.776));
    const float pre = __fmul_rn(__fmul_rn(vsq, a.s_pre), dens);
    const double t3 = pow(__dmul_rn((double)vsq, 170880.776), 3.0);
    const float nd = __double2float_rn(__dmul_rn(1.72e+9, sqrt(__ddiv_rn(t3, __dmul_rn(a.density_np, (double)dens)))));
    float lnei = __double2float_rn(__dadd_rn(__dsub_rn(24.0, __dmul_rn(0.5, log(__dmul_rn(a.density_np, (double)dens)))),
                                             log(__dmul_rn((double)vsq, 170880.776))));
    lnei = __double2float_rn(__dmul_rn((double)lnei, a.Zeta));
    const float nu = __double2float_rn(__ddiv_rn(__dmul_rn(a.nu_pre, (double)lnei), (double)nd));

    // ---- Qx, Qy (def-Parallel.cpp:2089-2224) ----
    auto heat = [&](const float v, const float vv_x, const float vv_y, const float mom) {
        float Q = 0.0f;
        Q = __fsub_rn(Q, __fmul_rn(v, __fadd_rn(__fadd_rn(vxvx, vyvy), vzvz)));
        const float s1 = __fadd_rn(__fmul_rn(vv_x, vx), __fmul_rn(vv_y, vy));
        Q = __double2float_rn(__dsub_rn((double)Q, __dmul_rn(2.0, (double)s1)));
        const float s2 = __fadd_rn(__fmul_rn(vx, vx), __fmul_rn(vy, vy));
        Q = __double2float_rn(__dadd_rn((double)Q, __dmul_rn(__dmul_rn(2.0, (double)s2), (double)v)));
        Q = __fmul_rn(Q, dens);
        Q = __fadd_rn(Q, mom);
        return __fmul_rn(Q, 0.5f);
    };
    const float qx = heat(vx, vxvx, vxvy, qx2);
    const float qy = heat(vy, vxvy, vyvy, qy2);

    if (valid) {
        const long long C = a.cells;
        float* o = a.out;
        o[kMomN * C + cell] = dens;
        o[kMomVx * C + cell] = vx;
        o[kMomVy * C + cell] = vy;
        o[kMomVxVx * C + cell] = vxvx;
        o[kMomVyVy * C + cell] = vyvy;
        o[kMomVzVz * C + cell] = vzvz;
        o[kMomVxVy * C + cell] = vxvy;
        o[kMomVxVz * C + cell] = vxvz;
        o[kMomVyVz * C + cell] = vyvz;
        o[kMomVsq * C + cell] = vsq_out;
        o[kMomT * C + cell] = tev;
        o[kMomP * C + cell] = pre;
        o[kMomND * C + cell] = nd;
        o[kMomNu * C + cell] = nu;
        o[kMomQx * C + cell] = qx;
        o[kMomQy * C + cell] = qy;
        o[kMomCount * C + cell] = vsq;   // scratch plane: round-tripped <v^2> for the conductivities
    }
}

// Heat conductivities from the centred difference of <v^2>^2, with the edge
// cells taking their neighbour's value (def-Parallel.cpp:2140-2166, 2205-2231)
__global__ void moments_conductivity_kernel(const MomentArgs a) {
    const long long cell = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (cell >= a.cells) return;
    const int nx = a.nx, ny = a.ny;
    const int y = (int)(cell / nx), x = (int)(cell - (long long)y * nx);
    const long long C = a.cells;
    const float* o = a.out;
    // <v^2> after the eV round trip, left in the scratch plane by moments_cell_kernel
    auto sq = [&](int xx, int yy) {
        const float v = o[kMomCount * C + (long long)yy * nx + xx];
        return __fmul_rn(v, v);
    };
    auto kappa = [&](float d, float scale, float Q) {
        float c = __fmul_rn(d, scale);
        c = __fmul_rn(c, o[kMomN * C + cell]);
        c = __fdiv_rn(c, o[kMomNu * C + cell]);
        c = __fmul_rn(c, (float)(-1.0 / 18.0));
        if ((double)c < 4.0 * FLT_MIN && (double)c > -4.0 * FLT_MIN) c = 1.0f;
        return __fdiv_rn(Q, c);
    };
    float dxs = 0.0f, dys = 0.0f;
    if (nx >= 3) {
        const int xa = x == 0 ? 1 : (x == nx - 1 ? nx - 2 : x);
        dxs = __fsub_rn(sq(xa - 1, y), sq(xa + 1, y));
    }
    if (ny >= 3) {
        const int ya = y == 0 ? 1 : (y == ny - 1 ? ny - 2 : y);
        dys = __fsub_rn(sq(x, ya - 1), sq(x, ya + 1));
    }
    a.out[kMomKx * C + cell] = kappa(dxs, a.s_kx, o[kMomQx * C + cell]);
    a.out[kMomKy * C + cell] = kappa(dys, a.s_ky, o[kMomQy * C + cell]);
}

}  // namespace

cudaError_t launch_moments(const MomentArgs& a, int planes_fp32, cudaStream_t s) {
    const long long groups = (a.cells + 31) / 32;
    const long long blocks = (groups + kMomWarps - 1) / kMomWarps;
    const size_t smem = sizeof(double) * (size_t)kMomWarps * 32 * (a.np + 1);
    const void* fn = planes_fp32 ? (const void*)moments_cell_kernel<float> : (const void*)moments_cell_kernel<double>;
    cudaError_t e = ensure_dyn_smem(fn, smem);
    if (e != cudaSuccess) return e;
    if (planes_fp32)
        moments_cell_kernel<float><<<(unsigned)blocks, 32 * kMomWarps, smem, s>>>(a);
    else
        moments_cell_kernel<double><<<(unsigned)blocks, 32 * kMomWarps, smem, s>>>(a);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    moments_conductivity_kernel<<<(unsigned)((a.cells + 255) / 256), 256, 0, s>>>(a);
    return cudaGetLastError();
}

}  // namespace oshun
