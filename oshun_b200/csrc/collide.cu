// Fokker-Planck collision step, one CTA per configuration-space cell
// (grid-stride over cells), all arithmetic in FP64:
//
//   1. f00 e-e, Explicit_EC_FP::loop (OSHUN-1/def-FokkerPlanck.cpp:590-625):
//      nsub RK4 substeps (RungeKutta4_ee::advance, :518-553) of Bell's
//      number/energy conserving operator (EE_isotropic_conserva::Getslope,
//      :192-267).  Warp 0 runs it; the cumulative integrals I4, I2 (forward)
//      and J1 (backward) are warp scans over lane-owned runs of the p axis.
//   2. Coefficients of the implicit f_lm step from the new f00,
//      Implicit_FLM_step::reset_coeff (:808-939): I2, I0, J_{-1} scans,
//      Coulomb logarithms, scattering term, the tridiagonal Alpha_Tri,
//      f00 derivatives.  Computed once per cell for every l (the reference
//      computes them in both f1_loop and flm_loop with the same f00).
//   3. (I - Dt C_l) f_lm^{n+1} = f_lm^n for every collided plane,
//      Implicit_FLM_step::advance (:943-1035):
//      tridiagonal: the cell's planes are staged through shared memory in
//        chunks and each thread runs the reference's Thomas recursion
//        (TridiagonalSolve, OSHUN-1/def-Nmethods.cpp:142-167) on one plane;
//      dense: per l the np x np matrix is assembled in a per-CTA global
//        workspace and each warp runs the reference's Gauss-Seidel
//        (def-Nmethods.cpp:44-136: dominance test, <= 5 sweeps, prefix
//        convergence rule) on one complex right-hand side.
#include <float.h>

#include "oshun_internal.h"

namespace oshun {
namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr int kCollideThreads = 128;

// The three cumulative integrals of one f on one warp, interleaved:
//   I4[k] = sum_{i=1..k} U4[i] f[i] + U4m1[i] f[i-1]
//   I2[k] = sum_{i=1..k} U2[i] f[i] + U2m1[i] f[i-1]
//   J1[k] = sum_{i=k+1..n-1} U1[i] f[i] + U1m1[i] f[i-1]
// Each lane sums a contiguous run of k, keeping each term in the output
// arrays (the I4 and I2 terms at their k, the J1 term of i at i - 1, all
// inside the lane's own run), the lanes' run totals are combined by a warp
// scan, and the lane then accumulates its run again from the scanned start
// out of the kept terms; the three chains are independent and interleaved.
template <class T4, class T2, class T1>
__device__ void warp_cumsum3(double* I4, double* I2, double* J1, int n, T4 t4, T2 t2, T1 t1) {
    const int lane = threadIdx.x & 31;
    const int E = (n + 31) >> 5;
    const int b = min(lane * E, n), e = min(b + E, n);
    double l4 = 0.0, l2 = 0.0, l1 = 0.0;
    for (int k = b; k < e; ++k) {
        if (k > 0) {
            const double v4 = t4(k), v2 = t2(k);
            l4 += v4; l2 += v2;
            I4[k] = v4; I2[k] = v2;
        }
        if (k + 1 <= n - 1) {
            const double v1 = t1(k + 1);
            l1 += v1;
            J1[k] = v1;
        }
    }
    double s4 = l4, s2 = l2, s1 = l1;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        const double v4 = __shfl_up_sync(kFull, s4, off);
        const double v2 = __shfl_up_sync(kFull, s2, off);
        const double v1 = __shfl_down_sync(kFull, s1, off);
        if (lane >= off) { s4 += v4; s2 += v2; }
        if (lane + off < 32) s1 += v1;
    }
    double r4 = __shfl_up_sync(kFull, s4, 1), r2 = __shfl_up_sync(kFull, s2, 1);
    double r1 = __shfl_down_sync(kFull, s1, 1);
    if (lane == 0) { r4 = 0.0; r2 = 0.0; }
    if (lane == 31) r1 = 0.0;
    for (int k = b; k < e; ++k) {
        if (k > 0) { r4 += I4[k]; r2 += I2[k]; }
        I4[k] = r4;
        I2[k] = r2;
    }
    for (int k = e - 1; k >= b; --k) {
        if (k + 1 <= n - 1) r1 += J1[k];
        J1[k] = r1;
    }
    __syncwarp();
}

// Coulomb logarithms, NRL formulary as coded in OSHUN-1/def-FokkerPlanck.cpp:41-95
__device__ double log_ee(double ne, double Te, double density_np) {
    if (ne > 0.000000001) {
        Te /= (3.0 * ne);
        Te *= 511000;
        ne *= density_np;
        Te = log(Te);
        ne = log(ne);
        const double v = 23.5 - 0.5 * ne + 1.25 * Te - sqrt(0.00001 + 0.0625 * (Te - 2.0) * (Te - 2.0));
        if (v > 2.0) return v;
    }
    return 2.0;
}
__device__ double zlog_ei(double ne, double Te, double density_np, double Zeta) {
    if (ne > 0.0000001) {
        Te /= (3.0 * ne);
        Te *= 511000;
        ne *= density_np;
        Te = log(Te);
        ne = log(ne);
        const double v = 24.0 - 0.5 * ne + Te;
        if (v > 2.0) return v * Zeta;
    }
    return 2.0 * Zeta;
}

// The planes hold f - ref when a momentum profile is given (FP32 split):
// f of plane q at momentum point p, and the stored value of f.
// (FP64 planes hold f itself: no profile is read for them.)
// The profile row of plane q when the plane keeps one (FP32 planes), else null:
// looked up once per plane, so the plane loops branch once per plane
template <typename TP>
__device__ __forceinline__ const float* ref_row(const CollideArgs& a, long long q) {
    if constexpr (sizeof(TP) == sizeof(float)) return (a.pl_ref32 && __ldg(a.pl_keep + q)) ? a.pl_ref32 + q * a.np : nullptr;
    return nullptr;
}
template <typename TP>
__device__ __forceinline__ double ref_at(const CollideArgs& a, long long q, int p) {
    if constexpr (sizeof(TP) == sizeof(float))
        return (a.pl_ref32 && __ldg(a.pl_keep + q)) ? (double)__ldg(a.pl_ref32 + q * a.np + p) : 0.0;
    return 0.0;
}

struct Smem {
    double *f, *f0, *f1, *fh, *I4, *I2, *J1;            // e-e work (np each)
    double *tri_a, *tri_b, *tri_c, *scat, *df0, *ddf0;  // implicit coefficients (np each)
    double* sc;                                          // scalars: [0] dense-term scale
    double* chunk;                                       // staged planes / solver scratch
};

constexpr int kSmemArrays = 13;
constexpr int kSmemScalars = 4;

__device__ Smem carve(double* base, int np) {
    Smem s;
    s.f = base; s.f0 = base + np; s.f1 = base + 2 * np; s.fh = base + 3 * np;
    s.I4 = base + 4 * np; s.I2 = base + 5 * np; s.J1 = base + 6 * np;
    s.tri_a = base + 7 * np; s.tri_b = base + 8 * np; s.tri_c = base + 9 * np;
    s.scat = base + 10 * np; s.df0 = base + 11 * np; s.ddf0 = base + 12 * np;
    s.sc = base + kSmemArrays * np;
    s.chunk = s.sc + kSmemScalars;
    return s;
}

// e-e substeps and implicit step of one collision call: from the arguments,
// or, when a device clock is given, by the reference's clock arithmetic for a
// step ending at the clock's t (Explicit_EC_FP::loop, def-FokkerPlanck.cpp:
// 598-599; Euler_Backward, :1277, 1297), as collide_params does on the host
struct StepP {
    int nsub;
    double hsub, Dt;
};
__device__ __forceinline__ StepP step_params(const CollideArgs& a) {
    StepP p{a.nsub, a.hsub, a.Dt};
    if (a.clock) {
        const double t = a.clock[0], t_ee = a.clock[1], t_eb = a.clock[2];
        p.nsub = (int)((t - t_ee) / a.small_dt) + 1;
        p.hsub = (t - t_ee) / (double)p.nsub;
        p.Dt = t - t_eb;
    }
    return p;
}

// EE_isotropic_conserva::Getslope on warp 0: fh = C_ee(fin)
__device__ void ee_slope(const CollideArgs& a, const Smem& s, const double* fin, double* fh) {
    const int n = a.np;
    const int lane = threadIdx.x & 31;
    warp_cumsum3(s.I4, s.I2, s.J1, n, [&](int k) { return a.U4[k] * fin[k] + a.U4m1[k] * fin[k - 1]; },
                 [&](int k) { return a.U2[k] * fin[k] + a.U2m1[k] * fin[k - 1]; },
                 [&](int i) { return a.U1[i] * fin[i] + a.U1m1[i] * fin[i - 1]; });
    const double lnee = log_ee(4.0 * M_PI * s.I2[n - 1], 4.0 * M_PI * s.I4[n - 1], a.density_np);
    const double* vr = a.vr;
    const double v0s = vr[0] * vr[0], v1s = vr[1] * vr[1];
    // flux G_n (stored in I4); the first NB cells use the parabolic fit near v = 0
    for (int k = lane; k < n; k += 32) {
        double g;
        if (k < a.NB) {
            const double f00 = (fin[0] - fin[1] * v0s / v1s) / (1.0 - v0s / v1s);
            // v^3, v^5, v^7 tabulated on the host with the same pow() the reference calls
            const double v3 = a.U3[k], v5 = a.V5[k], v7 = a.V7[k];
            const double i2s = f00 * v3 / 3.0 + (fin[1] - f00) * v5 / v1s * 0.2;
            const double i4s = f00 * v5 * 0.2 + (fin[1] - f00) * v7 / (v1s * 7.0);
            g = fin[k] * i4s + (v3 * fin[k] - 3.0 * i2s) * s.J1[k];
        } else {
            double i2 = s.I2[k] * s.J1[k];
            i2 *= -3.0;
            double i4 = s.I4[k] + a.U3[k] * s.J1[k];
            i4 *= fin[k];
            g = i4 + i2;
        }
        s.I4[k] = g;
    }
    __syncwarp();
    // D_k = (G_k - G_{k+1}) P_k for k < n-1, D_{n-1} = G_{n-1}   (kept in I2)
    for (int k = lane; k < n; k += 32) s.I2[k] = (k < n - 1) ? (s.I4[k] - s.I4[k + 1]) * a.Pn[k] : s.I4[k];
    __syncwarp();
    const double norm = a.c_kpre * lnee;
    for (int k = lane; k < n; k += 32) {
        double v;
        if (k == 0) {
            v = (-1.0) * s.I4[0];
            v *= 2.0 / v0s;
            v -= s.I2[0];
            v *= a.Qn[0];
        } else {
            v = a.Qn[k] * (s.I2[k - 1] - s.I2[k]);
        }
        fh[k] = v * norm;
    }
    __syncwarp();
}

// Implicit_FLM_step::reset_coeff on warp 0 (f = f00 of the cell in smem)
__device__ void flm_reset(const CollideArgs& a, const Smem& s, const double* f) {
    const StepP sp = step_params(a);
    const int n = a.np;
    const int lane = threadIdx.x & 31;
    const double* vr = a.vr;
    double* I2 = s.I4;   // reuse the e-e work arrays
    double* I0 = s.I2;
    double* J1m = s.J1;
    warp_cumsum3(I2, I0, J1m, n, [&](int k) { return a.U4[k] * f[k] + a.U4m1[k] * f[k - 1]; },
                 [&](int k) { return a.U2[k] * f[k] + a.U2m1[k] * f[k - 1]; },
                 [&](int i) { return a.U1[i] * f[i] + a.U1m1[i] * f[i - 1]; });
    const double I2_temperature = I2[n - 1] * (4.0 * M_PI);
    const double I0_density = I0[n - 1] * (4.0 * M_PI);
    const double lnee = log_ee(I0_density, I2_temperature, a.density_np);
    const double zlnei = zlog_ei(I0_density, I2_temperature, a.density_np, a.Zeta);
    const double scale = (-1.0) * lnee * a.kpre * sp.Dt;
    if (lane == 0) s.sc[0] = scale;
    for (int k = lane; k < n; k += 32) {
        double i2 = I2[k] * (4.0 * M_PI);
        i2 /= vr[k] * vr[k];
        const double i0 = I0[k] * (4.0 * M_PI);
        const double j1m = J1m[k] * (4.0 * M_PI * vr[k]);
        const double t1 = i0 + (2.0 * j1m - i2) / 3.0;
        const double t2 = (i2 + j1m) / 3.0;
        double sc = (k == 0) ? 0.0 : t1 * lnee;
        sc += zlnei * I0_density;
        sc /= a.U3[k];
        sc *= a.kpre * sp.Dt;
        s.scat[k] = sc;
        double ta = 0.0, tb = 0.0, tc = 0.0;
        if (k == 0) {
            tb = 8.0 * M_PI * f[0] * scale;
        } else if (k < n - 1) {
            const double IvDnDm1 = 1.0 / (vr[k] * 0.5 * (vr[k + 1] - vr[k - 1]) * (vr[k] - vr[k - 1]));
            const double IvDnDp1 = 1.0 / (vr[k] * 0.5 * (vr[k + 1] - vr[k - 1]) * (vr[k + 1] - vr[k]));
            const double Ivsq2Dn = 1.0 / (vr[k] * vr[k] * (vr[k + 1] - vr[k - 1]));
            tb = (8.0 * M_PI * f[k] - t2 * (IvDnDm1 + IvDnDp1)) * scale;
            ta = (t2 * IvDnDm1 - t1 * Ivsq2Dn) * scale;
            tc = (t2 * IvDnDp1 + t1 * Ivsq2Dn) * scale;
        }
        s.tri_a[k] = ta; s.tri_b[k] = tb; s.tri_c[k] = tc;
        // raw -df/dv at n-1/2 (finished below); f0 is free once the e-e step is done
        s.f0[k] = (k >= 1) ? (f[k - 1] - f[k]) / (vr[k] - vr[k - 1]) : 0.0;
    }
    __syncwarp();
    for (int k = lane; k < n; k += 32) {
        double df, ddf;
        if (k == 0) {
            const double f00 = (f[0] - (vr[0] * vr[0] / (vr[1] * vr[1])) * f[1]) / (1.0 - (vr[0] * vr[0]) / (vr[1] * vr[1]));
            ddf = 2.0 * (f[1] - f00) / (vr[1] * vr[1]);
            df = ddf * vr[0];
        } else if (k < n - 1) {
            df = (f[k + 1] - f[k - 1]) / (vr[k + 1] - vr[k - 1]);
            ddf = (s.f0[k] - s.f0[k + 1]) / (0.5 * (vr[k + 1] - vr[k - 1]));
        } else {
            df = 0.0;
            ddf = s.f0[k];
        }
        if (k < n - 1) { df /= vr[k] * vr[k]; ddf /= 2.0 * vr[k]; }
        s.df0[k] = df;
        s.ddf0[k] = ddf;
    }
    __syncwarp();
}

template <typename TP>
__device__ void tridiagonal_chunks(const CollideArgs& a, const Smem& s, long long cell) {
    TP* planes = reinterpret_cast<TP*>(a.planes);
    const int* plane_l = a.plane_l;
    const int* plane_m = a.plane_m;
    const int nplanes = a.nplanes;
    const int n = a.np, ld = n + 1;
    for (int q0 = 0; q0 < nplanes; q0 += a.chunk) {
        const int nq = min(a.chunk, nplanes - q0);
        // stage: d column of plane j at chunk[j*2*ld], c' column at chunk[j*2*ld + ld]
        for (int idx = threadIdx.x; idx < nq * n; idx += blockDim.x) {
            const int j = idx / n, p = idx - j * n;
            s.chunk[(long long)j * 2 * ld + p] =
                (double)planes[(long long)(q0 + j) * a.pstride + cell * n + p] + ref_at<TP>(a, q0 + j, p);
        }
        __syncthreads();
        for (int j = threadIdx.x; j < nq; j += blockDim.x) {
            const int q = q0 + j;
            const int l = plane_l[q], m = plane_m[q];
            if (l < 1 || m > a.mmax_coll || (l == 1 ? !a.do_l1 : !a.do_lm)) continue;
            double* d = s.chunk + (long long)j * 2 * ld;
            double* c = d + ld;
            const double ll1 = l * ((-0.5) * (l + 1.0));
            // Thomas, TridiagonalSolve (def-Nmethods.cpp:150-166)
            double b0 = (l > 1 ? 0.0 : s.tri_b[0]) + (1.0 - ll1 * s.scat[0]);
            c[0] = s.tri_c[0] / b0;
            d[0] /= b0;
            for (int i = 1; i < n; ++i) {
                const double bi = s.tri_b[i] + (1.0 - ll1 * s.scat[i]);
                const double id = 1.0 / (bi - c[i - 1] * s.tri_a[i]);
                c[i] = s.tri_c[i] * id;
                d[i] = (d[i] - d[i - 1] * s.tri_a[i]) * id;
            }
            for (int i = n - 2; i > -1; --i) d[i] = d[i] - c[i] * d[i + 1];
        }
        __syncthreads();
        for (int idx = threadIdx.x; idx < nq * n; idx += blockDim.x) {
            const int j = idx / n, p = idx - j * n;
            const int q = q0 + j;
            const int l = plane_l[q], m = plane_m[q];
            if (l < 1 || m > a.mmax_coll || (l == 1 ? !a.do_l1 : !a.do_lm)) continue;
            planes[(long long)q * a.pstride + cell * n + p] = (TP)(s.chunk[(long long)j * 2 * ld + p] - ref_at<TP>(a, q, p));
        }
        __syncthreads();
    }
}

// dense path: assemble Alpha for harmonic order el in the CTA workspace
__device__ void dense_assemble(const CollideArgs& a, const Smem& s, double* A, int el) {
    const int n = a.np;
    const double* vr = a.vr;
    const double LL = el;
    const double A1 = (LL + 1.0) * (LL + 2.0) / ((2.0 * LL + 1.0) * (2.0 * LL + 3.0));
    const double A2 = (-1.0) * (LL - 1.0) * LL / ((2.0 * LL + 1.0) * (2.0 * LL - 1.0));
    const double B1 = (-1.0) * (0.5 * LL * (LL + 1.0) + (LL + 1.0)) / ((2.0 * LL + 1.0) * (2.0 * LL + 3.0));
    const double B2 = ((-0.5) * LL * (LL + 1.0) + (LL + 2.0)) / ((2.0 * LL + 1.0) * (2.0 * LL + 3.0));
    const double B3 = (0.5 * LL * (LL + 1.0) + (LL - 1.0)) / ((2.0 * LL + 1.0) * (2.0 * LL - 1.0));
    const double B4 = (0.5 * LL * (LL + 1.0) - LL) / ((2.0 * LL + 1.0) * (2.0 * LL - 1.0));
    const double ll1 = el * ((-0.5) * (el + 1.0));
    const double sc = s.sc[0];  // (-1) lnee kpre Dt (def-FokkerPlanck.cpp:973)
    for (long long idx = threadIdx.x; idx < (long long)n * n; idx += blockDim.x) {
        const int i = (int)(idx / n), j = (int)(idx - (long long)i * n);
        double v = 0.0;
        if (i == j) v = s.tri_b[i];
        else if (j == i - 1) v = s.tri_a[i];
        else if (j == i + 1) v = s.tri_c[i];
        if (i == 0 && j == 0 && el > 1) v = 0.0;
        if (i < n - 1 && j < n - 1) {
            double t1 = A1 * s.ddf0[i] + B1 * s.df0[i]; t1 *= sc;
            double t2 = A1 * s.ddf0[i] + B2 * s.df0[i]; t2 *= sc;
            double t3 = A2 * s.ddf0[i] + B3 * s.df0[i]; t3 *= sc;
            double t4 = A2 * s.ddf0[i] + B4 * s.df0[i]; t4 *= sc;
            // same accumulation order as the reference row loop (def-FokkerPlanck.cpp:981-998)
            if (j == 0) {
                v += t1 * (2.0 * M_PI * pow(vr[0] / vr[i], el + 2) * vr[0] * vr[0] * (vr[1] - vr[0]));
                v += t3 * (2.0 * M_PI * pow(vr[0] / vr[i], el) * vr[0] * vr[0] * (vr[1] - vr[0]));
            }
            if (j >= 1 && j < i) {
                v += t1 * (2.0 * M_PI * pow(vr[j] / vr[i], el + 2) * vr[j] * vr[j] * (vr[j + 1] - vr[j - 1]));
                v += t3 * (2.0 * M_PI * pow(vr[j] / vr[i], el) * vr[j] * vr[j] * (vr[j + 1] - vr[j - 1]));
            }
            if (j == i) {
                // the reference reads vr[-1] at i = 0 (def-FokkerPlanck.cpp:989-990), a
                // denormal malloc header word; 0 here
                const double vlow = i > 0 ? vr[i - 1] : 0.0;
                v += t1 * (2.0 * M_PI * vr[i] * vr[i] * (vr[i] - vlow));
                v += t3 * (2.0 * M_PI * vr[i] * vr[i] * (vr[i] - vlow));
                v += t2 * (2.0 * M_PI * vr[i] * vr[i] * (vr[i + 1] - vr[i]));
                v += t4 * (2.0 * M_PI * vr[i] * vr[i] * (vr[i + 1] - vr[i]));
            }
            if (j > i) {
                v += t2 * (2.0 * M_PI * pow(vr[j] / vr[i], -el - 1) * vr[j] * vr[j] * (vr[j + 1] - vr[j - 1]));
                v += t4 * (2.0 * M_PI * pow(vr[j] / vr[i], -el + 1) * vr[j] * vr[j] * (vr[j + 1] - vr[j - 1]));
            }
        }
        if (i == j) v += 1.0 - ll1 * s.scat[i];
        A[idx] = v;
    }
}

// Gauss_Seidel on one warp; x: complex (re at xr, im at xi) in smem, initial
// guess = b.  Returns false (x untouched) when the dominance test fails.
__device__ void dense_gauss_seidel(const double* A, int n, const double* inv, double* xr, double* xi,
                                   const double* br, const double* bi, double* ovr, double* ovi) {
    const int lane = threadIdx.x & 31;
    const double tol = 1.0e-1;
    int iteration = 0, conv = 0;
    while ((iteration++ < 5) && (conv < n)) {
        for (int k = lane; k < n; k += 32) { ovr[k] = xr[k]; ovi[k] = xi[k]; }
        __syncwarp();
        for (int i = 0; i < n; ++i) {
            const double* row = A + (long long)i * n;
            double sr = 0.0, si = 0.0;
            for (int j = lane; j < n; j += 32) {
                if (j == i) continue;
                const double aij = row[j];
                sr += aij * xr[j];
                si += aij * xi[j];
            }
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) {
                sr += __shfl_xor_sync(kFull, sr, off);
                si += __shfl_xor_sync(kFull, si, off);
            }
            if (lane == 0) {
                xr[i] = inv[i] * (br[i] - sr);
                xi[i] = inv[i] * (bi[i] - si);
            }
            __syncwarp();
        }
        // prefix convergence test |dx_i| < tol |x_i + 20 DBL_MIN|
        conv = n;
        for (int base = 0; base < n; base += 32) {
            const int k = base + lane;
            bool ok = true;
            if (k < n) {
                const double dr = ovr[k] - xr[k], di = ovi[k] - xi[k];
                ok = hypot(dr, di) < tol * hypot(xr[k] + 20.0 * DBL_MIN, xi[k]);
            }
            const unsigned bad = __ballot_sync(kFull, !ok);
            if (bad) { conv = base + __ffs(bad) - 1; break; }
        }
        __syncwarp();
    }
}

template <typename TP>
__device__ void dense_solves(const CollideArgs& a, const Smem& s, long long cell, double* A, double* scratch) {
    TP* planes = reinterpret_cast<TP*>(a.planes);
    const int* plane_of = a.plane_of;
    const int n = a.np;
    const int warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    // per warp: x re/im, b re/im, old re/im (6n); shared: inv diag (n), dominance flag
    double* inv = scratch;
    int* dominant = reinterpret_cast<int*>(scratch + n);
    double* wbase = scratch + n + 2 + warp * 6 * n;
    double *xr = wbase, *xi = wbase + n, *br = wbase + 2 * n, *bi = wbase + 3 * n, *ovr = wbase + 4 * n,
           *ovi = wbase + 5 * n;
    for (int el = 1; el <= a.l0; ++el) {
        if (el == 1 ? !a.do_l1 : !a.do_lm) continue;
        dense_assemble(a, s, A, el);
        __syncthreads();
        if (threadIdx.x == 0) *dominant = 1;
        __syncthreads();
        // dominance: sequential signed row sums as in the reference
        for (int i = threadIdx.x; i < n; i += blockDim.x) {
            double row = 0.0;
            for (int j = 0; j < n; ++j) row += A[(long long)i * n + j];
            if (!(row < 2.0 * A[(long long)i * n + i])) atomicExch(dominant, 0);
            inv[i] = 1.0 / A[(long long)i * n + i];
        }
        __syncthreads();
        const int mtop = min(el, a.mmax_coll);
        if (*dominant) {
            for (int m = warp; m <= mtop; m += nwarps) {
                const long long q = plane_of[el * (a.m0 + 1) + m];
                const TP* pr_ = planes + q * a.pstride + cell * n;
                const TP* pi_ = planes + (q + 1) * a.pstride + cell * n;
                for (int k = threadIdx.x & 31; k < n; k += 32) {
                    br[k] = (double)pr_[k] + ref_at<TP>(a, q, k);
                    bi[k] = m > 0 ? (double)pi_[k] + ref_at<TP>(a, q + 1, k) : 0.0;
                    xr[k] = br[k];
                    xi[k] = bi[k];
                }
                __syncwarp();
                dense_gauss_seidel(A, n, inv, xr, xi, br, bi, ovr, ovi);
                TP* wr = planes + q * a.pstride + cell * n;
                TP* wi = planes + (q + 1) * a.pstride + cell * n;
                for (int k = threadIdx.x & 31; k < n; k += 32) {
                    wr[k] = (TP)(xr[k] - ref_at<TP>(a, q, k));
                    if (m > 0) wi[k] = (TP)(xi[k] - ref_at<TP>(a, q + 1, k));
                }
                __syncwarp();
            }
        } else if (threadIdx.x == 0) {
            atomicOr(a.status, 1);
            atomicAdd(a.status + 1, mtop + 1);
        }
        __syncthreads();
    }
}

// Opt-in backward-Euler e-e step (OSHUN_FLAG_IMPLICIT_EE; not a reference
// scheme) on one warp, f00 of the cell in s.f.  The explicit operator of
// EE_isotropic_conserva (def-FokkerPlanck.cpp:201-267) is
//   C(f)_k = c_kpre lnee Qn_k (D_{k-1} - D_k),  D_k = P_k (G_k - G_{k+1}),
//   G_j = A_j f_j - B_j  (A = I4 + v^3 J1, B = 3 I2 J1; the low-v fit's
//   i4s, i2s for j < NB); row 0 Qn_0 (-(2/v_0^2) G_0 - D_0), D_{n-1} = G_{n-1}.
// One step g - D C(g) = f over the whole e-e interval D, by Picard sweeps,
// each a tridiagonal solve with the coefficients of the previous iterate x
// (the first from f): on each face the B difference becomes a drag on g,
// B_{k+1} - B_k = gam_k ((1 - w) g_k + w g_{k+1}), gam_k = (B_{k+1} - B_k) /
// ((1 - w) x_k + w x_{k+1}), w = 1/2, or 0 / 1 (upwind) where 1/2 would give
// the face a coefficient of the wrong sign; likewise B_0 = (B_0 / x_0) g_0.
// Every sweep's matrix is then an M-matrix (f stays positive for any D),
// and at convergence (g = x) the operator is the explicit one exactly, so
// the step converges to the explicit scheme as D -> 0.
// face k (between points k and k+1): D_k = al g_k + be g_{k+1} + cs; the
// B difference stays explicit (cs) where the iterate is not positive there
__device__ __forceinline__ void ee_face(double Ak, double Ak1, double Bk, double Bk1, double xk, double xk1,
                                        double P, double& al, double& be, double& cs) {
    const double dB = Bk1 - Bk;
    const double h = 0.5 * (xk + xk1);
    cs = 0.0;
    if (!(h > 0.0)) { al = P * Ak; be = -P * Ak1; cs = P * dB; return; }
    double w = 0.5;
    double gam = dB / h;
    if (Ak + 0.5 * gam < 0.0) w = 1.0;
    else if (0.5 * gam > Ak1) w = 0.0;
    if (w != 0.5) {
        const double hw = (1.0 - w) * xk + w * xk1;
        if (!(hw > 0.0)) { al = P * Ak; be = -P * Ak1; cs = P * dB; return; }
        gam = dB / hw;
    }
    al = P * (Ak + gam * (1.0 - w));
    be = P * (gam * w - Ak1);
}
__device__ void ee_implicit_step(const CollideArgs& a, const Smem& s) {
    const StepP sp = step_params(a);
    const double D = a.clock ? (a.clock[0] - a.clock[1]) : sp.hsub * (double)sp.nsub;
    const int n = a.np;
    const int lane = threadIdx.x & 31;
    const double* vr = a.vr;
    const double v0s = vr[0] * vr[0], v1s = vr[1] * vr[1];
    double* x = s.f1;    // iterate
    double* A = s.f0;    // A_j, then the Thomas c'
    double* B = s.fh;    // B_j
    double* al = s.tri_a;
    double* be = s.tri_c;
    double* tb = s.tri_b;
    double* cs = s.scat;   // explicit face parts
    for (int k = lane; k < n; k += 32) x[k] = s.f[k];
    __syncwarp();
    for (int sweep = 0; sweep < a.ee_implicit; ++sweep) {
        warp_cumsum3(s.I4, s.I2, s.J1, n, [&](int k) { return a.U4[k] * x[k] + a.U4m1[k] * x[k - 1]; },
                     [&](int k) { return a.U2[k] * x[k] + a.U2m1[k] * x[k - 1]; },
                     [&](int i) { return a.U1[i] * x[i] + a.U1m1[i] * x[i - 1]; });
        const double lnee = log_ee(4.0 * M_PI * s.I2[n - 1], 4.0 * M_PI * s.I4[n - 1], a.density_np);
        const double dn = D * a.c_kpre * lnee;
        const double fz = (x[0] - x[1] * v0s / v1s) / (1.0 - v0s / v1s);
        for (int k = lane; k < n; k += 32) {
            const double j1 = s.J1[k], v3 = a.U3[k];
            double i4 = s.I4[k], i2 = s.I2[k];
            if (k < a.NB) {
                i2 = fz * v3 / 3.0 + (x[1] - fz) * a.V5[k] / v1s * 0.2;
                i4 = fz * a.V5[k] * 0.2 + (x[1] - fz) * a.V7[k] / (v1s * 7.0);
            }
            A[k] = i4 + v3 * j1;
            B[k] = 3.0 * i2 * j1;
        }
        __syncwarp();
        for (int k = lane; k < n - 1; k += 32)
            ee_face(A[k], A[k + 1], B[k], B[k + 1], x[k], x[k + 1], a.Pn[k], al[k], be[k], cs[k]);
        __syncwarp();
        const bool imp0 = x[0] > 0.0;
        const double a0 = imp0 ? A[0] - B[0] / x[0] : A[0];
        const double b0 = imp0 ? 0.0 : B[0];
        double* rhs = s.I2;   // free once A and B are formed
        for (int k = lane; k < n; k += 32) {
            const double q = a.Qn[k];
            double d0, c0;
            if (k == 0) { d0 = -q * ((2.0 / v0s) * a0 + al[0]); c0 = q * ((2.0 / v0s) * b0 - cs[0]); }
            else if (k < n - 1) { d0 = q * (be[k - 1] - al[k]); c0 = q * (cs[k - 1] - cs[k]); }
            else { d0 = q * (be[k - 1] - A[k]); c0 = q * cs[k - 1]; }
            tb[k] = 1.0 - dn * d0;
            rhs[k] = s.f[k] + dn * c0;
        }
        __syncwarp();
        if (lane == 0) {
            // Thomas: sub-diagonal -dn Qn_k al_{k-1}, super-diagonal dn Qn_k be_k;
            // c' into A, d' then the solution into x
            double sup = dn * a.Qn[0] * be[0];
            double cp = sup / tb[0];
            double dp = rhs[0] / tb[0];
            A[0] = cp; x[0] = dp;
            for (int k = 1; k < n; ++k) {
                const double sub = -dn * a.Qn[k] * al[k - 1];
                sup = k < n - 1 ? dn * a.Qn[k] * be[k] : 0.0;
                const double id = 1.0 / (tb[k] - sub * cp);
                cp = sup * id;
                dp = (rhs[k] - sub * dp) * id;
                A[k] = cp; x[k] = dp;
            }
            for (int k = n - 2; k >= 0; --k) x[k] -= A[k] * x[k + 1];
        }
        __syncwarp();
    }
    for (int k = lane; k < n; k += 32) s.f[k] = x[k];
    __syncwarp();
}

// e-e RK4 substeps of Explicit_EC_FP::loop on one warp (f00 of the cell in s.f)
__device__ void ee_substeps(const CollideArgs& a, const Smem& s) {
    const StepP sp = step_params(a);
    const int n = a.np;
    const int lane = threadIdx.x & 31;
    for (int sub = 0; sub < sp.nsub; ++sub) {
        const double h = sp.hsub;
        for (int k = lane; k < n; k += 32) { s.f0[k] = s.f[k]; s.f1[k] = s.f[k]; }
        __syncwarp();
        ee_slope(a, s, s.f1, s.fh);
        for (int k = lane; k < n; k += 32) {
            double t = s.fh[k] * (0.5 * h);
            s.f1[k] += t; t *= 1.0 / 3.0; s.f[k] += t;
        }
        __syncwarp();
        ee_slope(a, s, s.f1, s.fh);
        for (int k = lane; k < n; k += 32) {
            s.f1[k] = s.f0[k];
            double t = s.fh[k] * (0.5 * h);
            s.f1[k] += t; t *= 2.0 / 3.0; s.f[k] += t;
        }
        __syncwarp();
        ee_slope(a, s, s.f1, s.fh);
        for (int k = lane; k < n; k += 32) {
            double t = s.fh[k] * h;
            s.f0[k] += t; t *= 1.0 / 3.0; s.f[k] += t;
        }
        __syncwarp();
        ee_slope(a, s, s.f0, s.fh);
        for (int k = lane; k < n; k += 32) s.f[k] += s.fh[k] * (h / 6.0);
        __syncwarp();
    }
}

// The same substeps with the four slopes from one call site of ee_slope:
// one inlined copy of its scans and logarithms instead of four, for the lane
// kernels of short rows (the stage updates are the ones above)
__device__ void ee_substeps_one_site(const CollideArgs& a, const Smem& s) {
    const StepP sp = step_params(a);
    const int n = a.np;
    const int lane = threadIdx.x & 31;
    for (int sub = 0; sub < sp.nsub; ++sub) {
        const double h = sp.hsub;
        for (int k = lane; k < n; k += 32) { s.f0[k] = s.f[k]; s.f1[k] = s.f[k]; }
        __syncwarp();
        for (int st = 0; st < 4; ++st) {
            ee_slope(a, s, st == 3 ? s.f0 : s.f1, s.fh);
            if (st == 0) {
                for (int k = lane; k < n; k += 32) {
                    double t = s.fh[k] * (0.5 * h);
                    s.f1[k] += t; t *= 1.0 / 3.0; s.f[k] += t;
                }
            } else if (st == 1) {
                for (int k = lane; k < n; k += 32) {
                    s.f1[k] = s.f0[k];
                    double t = s.fh[k] * (0.5 * h);
                    s.f1[k] += t; t *= 2.0 / 3.0; s.f[k] += t;
                }
            } else if (st == 2) {
                for (int k = lane; k < n; k += 32) {
                    double t = s.fh[k] * h;
                    s.f0[k] += t; t *= 1.0 / 3.0; s.f[k] += t;
                }
            } else {
                for (int k = lane; k < n; k += 32) s.f[k] += s.fh[k] * (h / 6.0);
            }
            __syncwarp();
        }
    }
}

// the backward-Euler e-e step alone, one warp per cell (the collision
// kernels then run with do_ee = 0)
__global__ void __launch_bounds__(32) ee_implicit_kernel(const CollideArgs a) {
    extern __shared__ double smem[];
    const int n = a.np;
    const Smem s = carve(smem, n);
    const int lane = threadIdx.x & 31;
    for (long long cell = blockIdx.x; cell < a.cells; cell += gridDim.x) {
        for (int k = lane; k < n; k += 32) s.f[k] = a.f00[cell * n + k];
        __syncwarp();
        ee_implicit_step(a, s);
        for (int k = lane; k < n; k += 32) a.f00[cell * n + k] = s.f[k];
        __syncwarp();
    }
}

__global__ void __launch_bounds__(kCollideThreads) collide_kernel(const CollideArgs a) {
    extern __shared__ double smem[];
    const int n = a.np;
    Smem s = carve(smem, n);
    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    for (long long cell = blockIdx.x; cell < a.cells; cell += gridDim.x) {
        // f00 of the cell
        for (int k = threadIdx.x; k < n; k += blockDim.x) s.f[k] = a.f00[cell * n + k];
        __syncthreads();
        if (warp == 0 && a.do_ee) {
            ee_substeps(a, s);
            for (int k = lane; k < n; k += 32) a.f00[cell * n + k] = s.f[k];
        }
        if (a.do_l1 || a.do_lm) {
            if (warp == 0) flm_reset(a, s, s.f);
            __syncthreads();
            if (a.if_tridiagonal) {
                if (a.planes_fp32) tridiagonal_chunks<float>(a, s, cell);
                else tridiagonal_chunks<double>(a, s, cell);
            } else {
                double* A = a.dense_ws + (long long)blockIdx.x * n * n;
                if (a.planes_fp32) dense_solves<float>(a, s, cell, A, s.chunk);
                else dense_solves<double>(a, s, cell, A, s.chunk);
            }
        }
        __syncthreads();
    }
}

__device__ __forceinline__ bool collided(const CollideArgs& a, int l, int m) {
    return l >= 1 && m <= a.mmax_coll && (l == 1 ? a.do_l1 : a.do_lm);
}

// Tridiagonal collision step, one warp per cell (1-warp CTAs, one CTA per
// cell), no CTA-wide barriers:
//   1. f00 e-e substeps, reset_coeff, and the Thomas pivots of every l --
//      c'_i and 1/(b_i - c'_{i-1} a_i), with b_0 kept for the reference's
//      d_0/b_0 -- one lane per l (TridiagonalSolve, def-Nmethods.cpp:152-159).
//   2. every collided plane of the cell: the row is loaded coalesced into
//      shared memory and both recurrences of TridiagonalSolve run with lanes
//      over momentum.  Each lane owns a contiguous run of p; the value
//      entering its run comes from a warp scan of the affine maps
//      d'_i = (d_i - a_i d'_{i-1}) id_i (forward) and x_i = d'_i - c'_i x_{i+1}
//      (backward); inside the run the lane applies the reference's recursion.
template <typename TP>
__global__ void __launch_bounds__(32) collide_warp_kernel(const CollideArgs a) {
    extern __shared__ double smem[];
    const int n = a.np;
    const int l0 = a.l0;
    const int lane = threadIdx.x & 31;
    TP* planes = reinterpret_cast<TP*>(a.planes);
    const bool solve = a.do_l1 || a.do_lm;
    Smem s = carve(smem, n);
    double* cp = s.chunk;                    // [l0][n]
    double* idv = cp + (size_t)l0 * n;       // [l0][n]
    double* row = idv + (size_t)l0 * n;      // [n]
    const int E = (n + 31) >> 5;
    const int rb = min(lane * E, n), re = min(rb + E, n);

    for (long long cell = blockIdx.x; cell < a.cells; cell += gridDim.x) {
        for (int k = lane; k < n; k += 32) s.f[k] = a.f00[cell * n + k];
        __syncwarp();
        if (a.do_ee) {
            ee_substeps(a, s);
            for (int k = lane; k < n; k += 32) a.f00[cell * n + k] = s.f[k];
        }
        if (!solve) continue;
        flm_reset(a, s, s.f);
        for (int l = 1 + lane; l <= l0; l += 32) {
            if (!(l == 1 ? a.do_l1 : a.do_lm)) continue;
            const double ll1 = l * ((-0.5) * (l + 1.0));
            double* cpl = cp + (size_t)(l - 1) * n;
            double* idl = idv + (size_t)(l - 1) * n;
            const double b0 = (l > 1 ? 0.0 : s.tri_b[0]) + (1.0 - ll1 * s.scat[0]);
            double cprev = s.tri_c[0] / b0;
            cpl[0] = cprev;
            idl[0] = b0;
            for (int i = 1; i < n; ++i) {
                const double bi = s.tri_b[i] + (1.0 - ll1 * s.scat[i]);
                const double id = 1.0 / (bi - cprev * s.tri_a[i]);
                cprev = s.tri_c[i] * id;
                cpl[i] = cprev;
                idl[i] = id;
            }
        }
        __syncwarp();
        const double* tri_a = s.tri_a;
        for (int q = 0; q < a.nplanes; ++q) {
            const int l = a.plane_l[q], m = a.plane_m[q];
            if (!collided(a, l, m)) continue;
            const double* cpl = cp + (size_t)(l - 1) * n;
            const double* idl = idv + (size_t)(l - 1) * n;
            TP* g = planes + (long long)q * a.pstride + cell * n;
            for (int k = lane; k < n; k += 32) row[k] = (double)g[k] + ref_at<TP>(a, q, k);
            __syncwarp();
            // forward: compose this lane's maps x -> A x + B over [rb, re)
            double A = 1.0, B = 0.0;
            for (int i = rb; i < re; ++i) {
                double Ai, Bi;
                if (i == 0) { Ai = 0.0; Bi = row[0] / idl[0]; }
                else { Ai = -(tri_a[i] * idl[i]); Bi = row[i] * idl[i]; }
                B = Ai * B + Bi;
                A = Ai * A;
            }
            // inclusive scan of the maps over the lanes (earlier lanes first)
#pragma unroll
            for (int off = 1; off < 32; off <<= 1) {
                const double Ap = __shfl_up_sync(kFull, A, off), Bp = __shfl_up_sync(kFull, B, off);
                if (lane >= off) { B = A * Bp + B; A = A * Ap; }
            }
            double din = __shfl_up_sync(kFull, B, 1);   // d' just before this lane's run
            if (rb < re) {
                double d = din;
                for (int i = rb; i < re; ++i) {
                    if (i == 0) d = row[0] / idl[0];
                    else d = (row[i] - d * tri_a[i]) * idl[i];
                    row[i] = d;
                }
            }
            __syncwarp();
            // backward: x_i = d'_i - c'_i x_{i+1}, x_{n-1} = d'_{n-1}
            A = 1.0; B = 0.0;
            for (int i = re - 1; i >= rb; --i) {
                double Ai, Bi;
                if (i == n - 1) { Ai = 0.0; Bi = row[i]; }
                else { Ai = -cpl[i]; Bi = row[i]; }
                B = Ai * B + Bi;
                A = Ai * A;
            }
#pragma unroll
            for (int off = 1; off < 32; off <<= 1) {
                const double Ap = __shfl_down_sync(kFull, A, off), Bp = __shfl_down_sync(kFull, B, off);
                if (lane + off < 32) { B = A * Bp + B; A = A * Ap; }
            }
            double xin = __shfl_down_sync(kFull, B, 1);  // x just after this lane's run
            if (rb < re) {
                double x = xin;
                for (int i = re - 1; i >= rb; --i) {
                    if (i == n - 1) x = row[i];
                    else x = row[i] - cpl[i] * x;
                    row[i] = x;
                }
            }
            __syncwarp();
            for (int k = lane; k < n; k += 32) g[k] = (TP)(row[k] - ref_at<TP>(a, q, k));
            __syncwarp();
        }
    }
}

// Tridiagonal collision step for nump <= 32 E, one warp per cell (1-warp
// CTAs, grid-stride over cells), rows in registers:
//   1. f00 e-e substeps and reset_coeff as above.
//   2. per collided l, the Thomas pivots of each lane's run of p (c'_i and
//      1/(b_i - c'_{i-1} a_i), 1/b_0 at i = 0; TridiagonalSolve,
//      def-Nmethods.cpp:152-159) from a warp scan of the pivot recurrence
//      (lane_pivots); then the collided planes of that l in batches of P: lane j holds p in
//      [jE, jE+E) of each row in registers (the next batch's rows are loaded
//      while this one is solved).  Both recurrences of TridiagonalSolve --
//      d'_i = (d_i - a_i d'_{i-1}) / (b_i - c'_{i-1} a_i) forward,
//      x_i = d'_i - c'_i x_{i+1} backward -- are affine maps of the previous
//      value.  Each lane composes its run, a warp scan gives the value entering
//      the run, and the lane applies the recursion inside its run.  The maps'
//      multipliers depend on l only, so their composition and scan are done
//      once per l and only the offsets are scanned per plane.
// Shared memory (doubles): 4 scalars, tri_a, tri_b, tri_c, scat, then the
// e-e/reset work arrays (the pivots stay in registers, per l).
__device__ Smem carve_lane(double* base, int np) {
    Smem s;
    s.sc = base;
    s.tri_a = base + 4; s.tri_b = s.tri_a + np; s.tri_c = s.tri_b + np; s.scat = s.tri_c + np;
    s.df0 = s.scat + np; s.ddf0 = s.df0 + np;
    s.f = s.ddf0 + np; s.f0 = s.f + np; s.f1 = s.f0 + np; s.fh = s.f1 + np;
    s.I4 = s.fh + np; s.I2 = s.I4 + np; s.J1 = s.I2 + np;
    s.chunk = nullptr;
    return s;
}
__host__ __device__ inline size_t lane_smem_doubles(int np, int /*l0*/) {
    return 4 + 13 * (size_t)np;   // scalars, tri_a/b/c, scat, e-e and reset work arrays
}

// Thomas pivots of harmonic order l for this lane's run of p, c'_i and
// 1/(b_i - c'_{i-1} a_i), with b_i = tri_b_i + 1 - ll1 scat_i (tri_b_0 left
// out for l > 1), as TridiagonalSolve forms them (def-Nmethods.cpp:152-159).
// c'_i = c_i / (b_i - a_i c'_{i-1}) is a linear-fractional map of c'_{i-1},
// the 2x2 matrix [[0, c_i], [-a_i, b_i]] acting on (c'_{i-1}, 1): each lane
// composes its run's matrices, a warp scan of the products (rescaled by
// powers of two, which leaves the maps unchanged) gives the value entering
// the run, and the lane applies the recursion inside its run.  No per-l
// table is kept, so a cell needs 4 + 13 np doubles of shared memory.
struct M22 {
    double a, b, c, d;
};
__device__ __forceinline__ M22 m22_mul(const M22& x, const M22& y) {
    return M22{fma(x.a, y.a, x.b * y.c), fma(x.a, y.b, x.b * y.d), fma(x.c, y.a, x.d * y.c),
               fma(x.c, y.b, x.d * y.d)};
}
__device__ __forceinline__ M22 m22_rescale(M22 x) {
    const double mx = fmax(fmax(fabs(x.a), fabs(x.b)), fmax(fabs(x.c), fabs(x.d)));
    const int ex = (int)((__double_as_longlong(mx) >> 52) & 0x7ff);
    if (mx > 0.0 && ex > 0 && ex < 0x7ff) {
        const double sc = __longlong_as_double((long long)(2046 - ex) << 52);   // 2^(1023 - ex)
        x.a *= sc; x.b *= sc; x.c *= sc; x.d *= sc;
    }
    return x;
}
template <int E>
__device__ __forceinline__ void lane_pivots(const Smem& s, const int l, const int n, const int i0, double (&cp)[E],
                                            double (&id)[E]) {
    const int lane = threadIdx.x & 31;
    const double ll1 = l * ((-0.5) * (l + 1.0));
    double b[E];
    M22 m{1.0, 0.0, 0.0, 1.0};
#pragma unroll
    for (int e = 0; e < E; ++e) {
        const int i = i0 + e;
        b[e] = 1.0;
        if (i < n) {
            b[e] = (i == 0 && l > 1 ? 0.0 : s.tri_b[i]) + (1.0 - ll1 * s.scat[i]);
            m = m22_mul(M22{0.0, s.tri_c[i], -s.tri_a[i], b[e]}, m);
        }
    }
    m = m22_rescale(m);
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        const M22 o{__shfl_up_sync(kFull, m.a, off), __shfl_up_sync(kFull, m.b, off),
                    __shfl_up_sync(kFull, m.c, off), __shfl_up_sync(kFull, m.d, off)};
        if (lane >= off) m = m22_rescale(m22_mul(m, o));
    }
    const double xb = __shfl_up_sync(kFull, m.b, 1), xd = __shfl_up_sync(kFull, m.d, 1);
    double cprev = lane == 0 ? 0.0 : xb / xd;
#pragma unroll
    for (int e = 0; e < E; ++e) {
        const int i = i0 + e;
        if (i < n) {
            if (i == 0) {
                id[e] = 1.0 / b[e];
                cprev = s.tri_c[0] / b[e];
            } else {
                id[e] = 1.0 / (b[e] - cprev * s.tri_a[i]);
                cprev = s.tri_c[i] * id[e];
            }
            cp[e] = cprev;
        } else {
            id[e] = 0.0;
            cp[e] = 0.0;
        }
    }
}

template <typename TP, int E, int P>
__device__ __forceinline__ void collide_lane_cell(const CollideArgs& a, const long long cell, double* smem) {
    const int n = a.np;
    const int l0 = a.l0;
    const int lane = threadIdx.x & 31;
    TP* planes = reinterpret_cast<TP*>(a.planes);
    const bool solve = a.do_l1 || a.do_lm;
    const Smem s = carve_lane(smem, n);
    const int i0 = lane * E;   // first p of this lane's run

    // plane batches: l, first plane, count (planes of one l are consecutive)
    auto batch_first = [&](int& l, int& j) {
        l = 1; j = 0;
        while (l <= l0 && !collided(a, l, 0)) ++l;
    };
    auto batch_next = [&](int& l, int& j) {
        const int nq = 1 + 2 * min(min(l, a.m0), a.mmax_coll);
        j += P;
        if (j < nq) return;
        j = 0;
        do { ++l; } while (l <= l0 && !collided(a, l, 0));
    };
    // a batch's rows as stored: the next batch's loads stay in flight during
    // this batch's solve in the storage type (FP32 planes take half the
    // registers of their FP64 values) ...
    auto load_raw = [&](long long cell, int l, int j, TP (&r)[P][E]) {
        if (l > l0) return;
        const int nq = 1 + 2 * min(min(l, a.m0), a.mmax_coll);
        const long long q0 = a.plane_of[l * (a.m0 + 1)] + j;
#pragma unroll
        for (int b = 0; b < P; ++b) {
            const TP* g = planes + (q0 + b) * a.pstride + cell * n;
#pragma unroll
            for (int e = 0; e < E; ++e) r[b][e] = (j + b < nq && i0 + e < n) ? g[i0 + e] : TP(0);
        }
    };
    // ... and widened to FP64, the plane's profile added, when the batch is solved
    auto widen = [&](int l, int j, const TP (&r)[P][E], double (&d)[P][E]) {
        const int nq = 1 + 2 * min(min(l, a.m0), a.mmax_coll);
        const long long q0 = a.plane_of[l * (a.m0 + 1)] + j;
#pragma unroll
        for (int b = 0; b < P; ++b) {
#pragma unroll
            for (int e = 0; e < E; ++e) d[b][e] = (double)r[b][e];
            const float* rp = (j + b < nq) ? ref_row<TP>(a, q0 + b) : nullptr;
            if (rp) {
#pragma unroll
                for (int e = 0; e < E; ++e)
                    if (i0 + e < n) d[b][e] += (double)__ldg(rp + i0 + e);
            }
        }
    };

    TP raw[P][E];
    double cur[P][E];
    {
        int bl, bj;
        batch_first(bl, bj);
        if (solve) load_raw(cell, bl, bj, raw);   // in flight during the e-e step
        for (int k = lane; k < n; k += 32) s.f[k] = a.f00[cell * n + k];
        __syncwarp();
        if (a.do_ee) {
            if constexpr (E <= 3) ee_substeps_one_site(a, s);
            else ee_substeps(a, s);
            for (int k = lane; k < n; k += 32) a.f00[cell * n + k] = s.f[k];
        }
        if (!solve) return;
        flm_reset(a, s, s.f);
        // this lane's tri_a (forward multiplier -a_i id_i)
        double ta[E];
#pragma unroll
        for (int e = 0; e < E; ++e) ta[e] = (i0 + e < n) ? s.tri_a[i0 + e] : 0.0;

        int cl = -1;   // l of the per-l constants below
        double id[E], cp[E], Af[5], Ab[5];
        if (bl <= l0) widen(bl, bj, raw, cur);
        while (bl <= l0) {
            const int l = bl, j = bl <= l0 ? bj : 0;
            const int nq = 1 + 2 * min(min(l, a.m0), a.mmax_coll);
            int nl = bl, nj = bj;
            batch_next(nl, nj);
            if (nl <= l0) load_raw(cell, nl, nj, raw);
            if (l != cl) {
                // per-l constants: pivots of this lane's run and the scan multipliers
                cl = l;
                lane_pivots<E>(s, l, n, i0, cp, id);
                double A = 1.0, B = 1.0;
#pragma unroll
                for (int e = 0; e < E; ++e) {
                    const int i = i0 + e;
                    if (i < n) A = (i == 0) ? 0.0 : A * (-(ta[e] * id[e]));
                }
#pragma unroll
                for (int e = E - 1; e >= 0; --e) {
                    const int i = i0 + e;
                    if (i < n) B = (i == n - 1) ? 0.0 : B * (-cp[e]);
                }
#pragma unroll
                for (int k = 0, off = 1; k < 5; ++k, off <<= 1) {
                    Af[k] = A;
                    Ab[k] = B;
                    const double Ap = __shfl_up_sync(kFull, A, off);
                    const double Bp = __shfl_down_sync(kFull, B, off);
                    if (lane >= off) A *= Ap;
                    if (lane + off < 32) B *= Bp;
                }
            }
            // forward: run offsets, scan, recursion inside the run
            double Bf[P];
#pragma unroll
            for (int b = 0; b < P; ++b) {
                double B = 0.0;
#pragma unroll
                for (int e = 0; e < E; ++e) {
                    const int i = i0 + e;
                    if (i < n) B = (i == 0) ? cur[b][e] * id[e] : (cur[b][e] - B * ta[e]) * id[e];
                }
                Bf[b] = B;
            }
#pragma unroll
            for (int k = 0, off = 1; k < 5; ++k, off <<= 1) {
#pragma unroll
                for (int b = 0; b < P; ++b) {
                    const double Bp = __shfl_up_sync(kFull, Bf[b], off);
                    if (lane >= off) Bf[b] += Af[k] * Bp;
                }
            }
#pragma unroll
            for (int b = 0; b < P; ++b) {
                double d = __shfl_up_sync(kFull, Bf[b], 1);
#pragma unroll
                for (int e = 0; e < E; ++e) {
                    const int i = i0 + e;
                    if (i < n) {
                        d = (i == 0) ? cur[b][e] * id[e] : (cur[b][e] - d * ta[e]) * id[e];
                        cur[b][e] = d;
                    }
                }
            }
            // backward
            double Bb[P];
#pragma unroll
            for (int b = 0; b < P; ++b) {
                double B = 0.0;
#pragma unroll
                for (int e = E - 1; e >= 0; --e) {
                    const int i = i0 + e;
                    if (i < n) B = (i == n - 1) ? cur[b][e] : cur[b][e] - cp[e] * B;
                }
                Bb[b] = B;
            }
#pragma unroll
            for (int k = 0, off = 1; k < 5; ++k, off <<= 1) {
#pragma unroll
                for (int b = 0; b < P; ++b) {
                    const double Bp = __shfl_down_sync(kFull, Bb[b], off);
                    if (lane + off < 32) Bb[b] += Ab[k] * Bp;
                }
            }
            const long long q0 = a.plane_of[l * (a.m0 + 1)] + j;
#pragma unroll
            for (int b = 0; b < P; ++b) {
                double x = __shfl_down_sync(kFull, Bb[b], 1);
                TP* g = planes + (q0 + b) * a.pstride + cell * n;
                const float* rp = (j + b < nq) ? ref_row<TP>(a, q0 + b) : nullptr;
#pragma unroll
                for (int e = E - 1; e >= 0; --e) {
                    const int i = i0 + e;
                    if (i < n) {
                        x = (i == n - 1) ? cur[b][e] : cur[b][e] - cp[e] * x;
                        if (j + b < nq) g[i] = (TP)(rp ? x - (double)__ldg(rp + i) : x);
                    }
                }
            }
            if (nl <= l0) widen(nl, nj, raw, cur);
            bl = nl; bj = nj;
        }
        __syncwarp();
    }
}

// rows of up to 96 points (E <= 3) leave 12.3 KB of shared memory per cell:
// the kernel is held to 128 registers so that 16 cells are resident per SM
template <int E>
constexpr int lane_min_blocks() { return E <= 3 ? 16 : 1; }
template <typename TP, int E, int P>
__global__ void __launch_bounds__(32, lane_min_blocks<E>()) collide_lane_kernel(const CollideArgs a) {
    extern __shared__ double smem[];
    for (long long cell = blockIdx.x; cell < a.cells; cell += gridDim.x) collide_lane_cell<TP, E, P>(a, cell, smem);
}

// batched form: work item = (problem, cell); the problems share E
template <typename TP, int E, int P>
__global__ void __launch_bounds__(32) collide_lane_batch_kernel(const CollideBatch b) {
    extern __shared__ double smem[];
    for (long long it = blockIdx.x; it < b.nitems; it += gridDim.x) {
        const int2 w = b.items[it];
        collide_lane_cell<TP, E, P>(b.probs[w.x], (long long)w.y, smem);
        __syncwarp();
    }
}

// chunked batched form: a CTA of W warps takes W cells of one problem (one
// cell per warp) and first stages the problem's twelve velocity tables (vr,
// U4, U4m1, U2, U2m1, U1, U1m1, U3, Qn, Pn, v^5, v^7: contiguous from vr) and
// its arguments in shared memory, so the e-e slopes and the coefficient
// build read them there instead of from L2
constexpr int kArgsDoubles = (int)((sizeof(CollideArgs) + 15) / 16 * 2);
template <typename TP, int E, int P>
__global__ void __launch_bounds__(256, 1) collide_lane_chunk_kernel(const CollideBatch b) {
    extern __shared__ __align__(16) double smem[];
    CollideArgs* sa = reinterpret_cast<CollideArgs*>(smem);
    double* tab = smem + kArgsDoubles;
    double* work = tab + b.tab_doubles;
    const int warp = threadIdx.x >> 5;
    for (long long ch = blockIdx.x; ch < b.nchunks; ch += gridDim.x) {
        const int4 c = b.chunks[ch];
        const CollideArgs& ga = b.probs[c.x];
        const int np = ga.np;
        if (threadIdx.x == 0) *sa = ga;
        for (int i = threadIdx.x; i < 12 * np; i += blockDim.x) tab[i] = ga.vr[i];
        __syncthreads();
        if (threadIdx.x == 0) {
            sa->vr = tab; sa->U4 = tab + np; sa->U4m1 = tab + 2 * np; sa->U2 = tab + 3 * np;
            sa->U2m1 = tab + 4 * np; sa->U1 = tab + 5 * np; sa->U1m1 = tab + 6 * np; sa->U3 = tab + 7 * np;
            sa->Qn = tab + 8 * np; sa->Pn = tab + 9 * np; sa->V5 = tab + 10 * np; sa->V7 = tab + 11 * np;
        }
        __syncthreads();
        if (warp < c.z) collide_lane_cell<TP, E, P>(*sa, (long long)c.y + warp, work + (size_t)warp * b.cell_doubles);
        __syncthreads();
    }
}

}  // namespace

cudaError_t launch_ee_implicit(const CollideArgs& a, cudaStream_t st) {
    const size_t smem = ((size_t)kSmemArrays * a.np + kSmemScalars) * sizeof(double);
    {
        const cudaError_t e = ensure_dyn_smem((const void*)ee_implicit_kernel, smem);
        if (e != cudaSuccess) return e;
    }
    const long long blocks = a.cells < (1ll << 30) ? a.cells : (1ll << 30);
    ee_implicit_kernel<<<(unsigned)blocks, 32, smem, st>>>(a);
    return cudaGetLastError();
}

size_t collide_smem_bytes(int np, int chunk, int if_tridiagonal) {
    size_t base = ((size_t)kSmemArrays * np + kSmemScalars) * sizeof(double);
    size_t extra;
    if (if_tridiagonal) extra = (size_t)chunk * 2 * (np + 1) * sizeof(double);
    else extra = ((size_t)np + 2 + (size_t)(kCollideThreads / 32) * 6 * np) * sizeof(double);
    return base + extra;
}

int collide_max_chunk(int np, size_t smem_budget) {
    size_t base = ((size_t)kSmemArrays * np + kSmemScalars) * sizeof(double);
    if (smem_budget <= base) return 0;
    size_t per = (size_t)2 * (np + 1) * sizeof(double);
    return (int)((smem_budget - base) / per);
}

int collide_threads() { return kCollideThreads; }

cudaError_t launch_collide(const CollideArgs& a, cudaStream_t st, size_t smem, int blocks) {
    {
        const cudaError_t e = ensure_dyn_smem((const void*)collide_kernel, smem);
        if (e != cudaSuccess) return e;
    }
    collide_kernel<<<blocks, kCollideThreads, smem, st>>>(a);
    return cudaGetLastError();
}

size_t collide_tri_smem_per_cell(int np, int l0) {
    if (np <= 256) return lane_smem_doubles(np, l0) * sizeof(double);
    return ((size_t)kSmemArrays * np + kSmemScalars + 2 * (size_t)l0 * np + np) * sizeof(double);
}

namespace {
template <typename TP, int E>
cudaError_t launch_lane(const CollideArgs& a, cudaStream_t st, int blocks, size_t smem) {
    // planes per batch: two row sets of P x E doubles stay in registers
    constexpr int P = E <= 2 ? 4 : (E <= 4 ? 2 : 1);
    {
        const cudaError_t e = ensure_dyn_smem((const void*)collide_lane_kernel<TP, E, P>, smem);
        if (e != cudaSuccess) return e;
    }
    collide_lane_kernel<TP, E, P><<<blocks, 32, smem, st>>>(a);
    return cudaGetLastError();
}
template <typename TP>
cudaError_t launch_lane_e(const CollideArgs& a, cudaStream_t st, int blocks, size_t smem) {
    switch ((a.np + 31) / 32) {
        case 1: return launch_lane<TP, 1>(a, st, blocks, smem);
        case 2: return launch_lane<TP, 2>(a, st, blocks, smem);
        case 3: return launch_lane<TP, 3>(a, st, blocks, smem);
        case 4: return launch_lane<TP, 4>(a, st, blocks, smem);
        case 5: return launch_lane<TP, 5>(a, st, blocks, smem);
        case 6: return launch_lane<TP, 6>(a, st, blocks, smem);
        case 7: return launch_lane<TP, 7>(a, st, blocks, smem);
        case 8: return launch_lane<TP, 8>(a, st, blocks, smem);
        default: return cudaErrorInvalidValue;
    }
}
}  // namespace

namespace {
template <typename TP, int E>
cudaError_t launch_lane_batch(const CollideBatch& b, cudaStream_t st, size_t smem) {
    constexpr int P = E <= 2 ? 4 : (E <= 4 ? 2 : 1);
    {
        const cudaError_t e = ensure_dyn_smem((const void*)collide_lane_batch_kernel<TP, E, P>, smem);
        if (e != cudaSuccess) return e;
    }
    const long long blocks = b.nitems < (1ll << 30) ? b.nitems : (1ll << 30);
    if (blocks < 1) return cudaSuccess;
    collide_lane_batch_kernel<TP, E, P><<<(unsigned)blocks, 32, smem, st>>>(b);
    return cudaGetLastError();
}
template <typename TP>
cudaError_t launch_lane_batch_e(const CollideBatch& b, int E, cudaStream_t st, size_t smem) {
    switch (E) {
        case 1: return launch_lane_batch<TP, 1>(b, st, smem);
        case 2: return launch_lane_batch<TP, 2>(b, st, smem);
        case 3: return launch_lane_batch<TP, 3>(b, st, smem);
        case 4: return launch_lane_batch<TP, 4>(b, st, smem);
        case 5: return launch_lane_batch<TP, 5>(b, st, smem);
        case 6: return launch_lane_batch<TP, 6>(b, st, smem);
        case 7: return launch_lane_batch<TP, 7>(b, st, smem);
        case 8: return launch_lane_batch<TP, 8>(b, st, smem);
        default: return cudaErrorInvalidValue;
    }
}

__global__ void clock_advance_batch_kernel(double* clocks, const double* dt, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) clocks[3 * i] += dt[i];
}
__global__ void clock_commit_batch_kernel(double* clocks, const int* collide, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n && (!collide || collide[i])) { clocks[3 * i + 1] = clocks[3 * i]; clocks[3 * i + 2] = clocks[3 * i]; }
}
}  // namespace

size_t collide_chunk_smem(int warps, int tab_doubles, int cell_doubles) {
    return sizeof(double) * ((size_t)kArgsDoubles + (size_t)tab_doubles + (size_t)warps * cell_doubles);
}

namespace {
template <typename TP, int E>
cudaError_t launch_lane_chunk(const CollideBatch& b, cudaStream_t st) {
    constexpr int P = E <= 2 ? 4 : (E <= 4 ? 2 : 1);
    const size_t smem = collide_chunk_smem(b.warps, b.tab_doubles, b.cell_doubles);
    {
        const cudaError_t e = ensure_dyn_smem((const void*)collide_lane_chunk_kernel<TP, E, P>, smem);
        if (e != cudaSuccess) return e;
    }
    const long long blocks = b.nchunks < (1ll << 30) ? b.nchunks : (1ll << 30);
    if (blocks < 1) return cudaSuccess;
    collide_lane_chunk_kernel<TP, E, P><<<(unsigned)blocks, 32 * b.warps, smem, st>>>(b);
    return cudaGetLastError();
}
template <typename TP, int E>
int regs_of(int chunked) {
    constexpr int P = E <= 2 ? 4 : (E <= 4 ? 2 : 1);
    cudaFuncAttributes fa{};
    const cudaError_t e = chunked ? cudaFuncGetAttributes(&fa, collide_lane_chunk_kernel<TP, E, P>)
                                  : cudaFuncGetAttributes(&fa, collide_lane_batch_kernel<TP, E, P>);
    return e == cudaSuccess ? fa.numRegs : 255;
}
template <typename TP>
int regs_e(int E, int chunked) {
    switch (E) {
        case 1: return regs_of<TP, 1>(chunked);
        case 2: return regs_of<TP, 2>(chunked);
        case 3: return regs_of<TP, 3>(chunked);
        case 4: return regs_of<TP, 4>(chunked);
        case 5: return regs_of<TP, 5>(chunked);
        case 6: return regs_of<TP, 6>(chunked);
        case 7: return regs_of<TP, 7>(chunked);
        case 8: return regs_of<TP, 8>(chunked);
        default: return 255;
    }
}
template <typename TP>
cudaError_t launch_lane_chunk_e(const CollideBatch& b, int E, cudaStream_t st) {
    switch (E) {
        case 1: return launch_lane_chunk<TP, 1>(b, st);
        case 2: return launch_lane_chunk<TP, 2>(b, st);
        case 3: return launch_lane_chunk<TP, 3>(b, st);
        case 4: return launch_lane_chunk<TP, 4>(b, st);
        case 5: return launch_lane_chunk<TP, 5>(b, st);
        case 6: return launch_lane_chunk<TP, 6>(b, st);
        case 7: return launch_lane_chunk<TP, 7>(b, st);
        case 8: return launch_lane_chunk<TP, 8>(b, st);
        default: return cudaErrorInvalidValue;
    }
}
}  // namespace

int collide_batch_regs(int E, int planes_fp32, int chunked) {
    return planes_fp32 ? regs_e<float>(E, chunked) : regs_e<double>(E, chunked);
}

cudaError_t launch_collide_batch(const CollideBatch& b, int E, int planes_fp32, size_t smem, cudaStream_t st) {
    if (b.nchunks > 0) return planes_fp32 ? launch_lane_chunk_e<float>(b, E, st) : launch_lane_chunk_e<double>(b, E, st);
    if (planes_fp32) return launch_lane_batch_e<float>(b, E, st, smem);
    return launch_lane_batch_e<double>(b, E, st, smem);
}
cudaError_t launch_clock_advance(double* clocks, const double* dt, int n, cudaStream_t st) {
    clock_advance_batch_kernel<<<(n + 127) / 128, 128, 0, st>>>(clocks, dt, n);
    return cudaGetLastError();
}
cudaError_t launch_clock_commit(double* clocks, const int* collide, int n, cudaStream_t st) {
    clock_commit_batch_kernel<<<(n + 127) / 128, 128, 0, st>>>(clocks, collide, n);
    return cudaGetLastError();
}

cudaError_t launch_collide_tri(const CollideArgs& a, cudaStream_t st, int /*cells_per_cta*/, int blocks) {
    const size_t smem = collide_tri_smem_per_cell(a.np, a.l0);
    if (a.np <= 256) {
        if (a.planes_fp32) return launch_lane_e<float>(a, st, blocks, smem);
        return launch_lane_e<double>(a, st, blocks, smem);
    }
    if (a.planes_fp32) {
        const cudaError_t e = ensure_dyn_smem((const void*)collide_warp_kernel<float>, smem);
        if (e != cudaSuccess) return e;
        collide_warp_kernel<float><<<blocks, 32, smem, st>>>(a);
    } else {
        const cudaError_t e = ensure_dyn_smem((const void*)collide_warp_kernel<double>, smem);
        if (e != cudaSuccess) return e;
        collide_warp_kernel<double><<<blocks, 32, smem, st>>>(a);
    }
    return cudaGetLastError();
}

}  // namespace oshun
