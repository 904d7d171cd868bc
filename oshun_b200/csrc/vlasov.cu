// Fused RHS + RK4-stage kernels: Actions::Adv (OSHUN-1/def-Actions.cpp:73-94)
// evaluated on one stage input and folded straight into the stage update of
// Runge_Kutta_4::advance_p1 (OSHUN-1/def-RK.cpp:110-145).
//
// Work decomposition.  One thread owns one (cell, p) point of every harmonic.
// Each thread walks the source harmonics row by row (l = 0..l0, all m of a
// row unrolled) and scatters every coupling of source (l,m) into register
// accumulators of the only target rows it can reach, l-1, l and l+1.  After
// source row l has passed, target row l-1 has all of its terms; it is
// RK-updated and written at once, so the slope never touches HBM.  Per stage
// and plane HBM sees one read of the stage input, the reads of Y0 and Y and
// the writes of the next stage input and Y: 3/5/5/3 words over the four
// stages.
//
// This file holds the global-load variant (any nump <= 1024): momentum
// neighbours by warp shuffles, rows wider than 256 swept in chunks.  The
// bulk-copy pipelined variant for nump <= 256 is in stage_pipe.cu; the
// launcher below takes it whenever the shape fits.
//
// Couplings, per source (l,m), G/H as in MakeGH/G00
// (OSHUN-1/def-VlasovMax.cpp:496-535), Dp = f[p-1]-f[p+1] with the reference's
// ends (OSHUN-1/def-State.cpp:359-380):
//   E field (Exyz, def-VlasovMax.cpp:346-491):
//     Ex G -> (l+1,m), Ex H -> (l-1,m), Em G -> (l+1,m+1), Em H -> (l-1,m+1),
//     Ep H -> (l-1,m-1), Ep G -> (l+1,m-1) (real part only when m = 1)
//   B field (Bxyz, def-VlasovMax.cpp:597-644):
//     (Bz+iBy)/2 f -> (l,m+1), -i m Bx f -> (l,m), (Bz-iBy) f -> (l,m-1)
//   advection (Axy, def-VlasovMax.cpp:834-951), v = p/gamma:
//     x: -> (l+1,m), (l-1,m);  y: -> (l+1,m+1), (l-1,m+1), (l-1,m-1), (l+1,m-1)
//   current (Jxyz, def-VlasovMax.cpp:680-745): FP64 quadrature of f10, f11
//   Ampere/Faraday (def-VlasovMax.cpp:979-1035) on the cell's neighbours
//   CLEAN_LOW_PC (def-Actions.cpp:240-253): slope of l >= 2 zeroed for
//   p < min(l-1, 80)
#include "stage_common.cuh"

namespace oshun {
namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr int kMaxCellsPerCta = 8;
constexpr int kPChunk = 256;

template <typename T>
__device__ __forceinline__ T ld(const T* p) { return __ldg(p); }

// ---------------------------------------------------------------------------
// field epilogue: J reduction result + Ampere/Faraday, RK update of 6 fields
// ---------------------------------------------------------------------------
// hside: bit 0 the x-1 neighbour, bit 1 the x+1 neighbour comes from the
// x halo columns (row y)
template <typename TS>
__device__ __forceinline__ void field_update(const StageArgs<TS>& a, long long cell, long long cxm, long long cxp,
                                             long long cym, long long cyp, double Jx, double Jyr, double Jyi,
                                             int hside, long long y) {
    const TS* F = a.fld_in;
    const long long C = a.cells;
    const TS idx = (TS)a.idx, idy = (TS)a.idy;
    auto xm = [&](int k) { return (hside & 1) ? hx_field(a, 0, k, y) : ld(F + k * C + cxm); };
    auto xp = [&](int k) { return (hside & 2) ? hx_field(a, 1, k, y) : ld(F + k * C + cxp); };
    TS dEx = 0, dEy = 0, dEz = 0, dBx = 0, dBy = 0, dBz = 0;
    if (a.parts & kPartAmpere) {
        // J: Ex += Jx, Ey += Re J11, Ez += -Im J11 with J11 = 2 * (f11 quadrature)
        dEx = fma_rn(idy, ld(F + 5 * C + cym) - ld(F + 5 * C + cyp), (TS)Jx);
        dEy = fma_rn(-idx, xm(5) - xp(5), (TS)(2.0 * Jyr));
        dEz = fma_rn(idx, xm(4) - xp(4), fma_rn(-idy, ld(F + 3 * C + cym) - ld(F + 3 * C + cyp), (TS)(-(2.0 * Jyi))));
    }
    if (a.parts & kPartFaraday) {
        dBx = mul_rn(-idy, ld(F + 2 * C + cym) - ld(F + 2 * C + cyp));
        dBy = mul_rn(idx, xm(2) - xp(2));
        dBz = fma_rn(-idx, xm(1) - xp(1), mul_rn(idy, ld(F + 0 * C + cym) - ld(F + 0 * C + cyp)));
    }
    rk_update(a.mode, a.first, a.c1, a.c2, a.fld_out, a.fld_B, a.fld_A, 0 * C + cell, dEx);
    rk_update(a.mode, a.first, a.c1, a.c2, a.fld_out, a.fld_B, a.fld_A, 1 * C + cell, dEy);
    rk_update(a.mode, a.first, a.c1, a.c2, a.fld_out, a.fld_B, a.fld_A, 2 * C + cell, dEz);
    rk_update(a.mode, a.first, a.c1, a.c2, a.fld_out, a.fld_B, a.fld_A, 3 * C + cell, dBx);
    rk_update(a.mode, a.first, a.c1, a.c2, a.fld_out, a.fld_B, a.fld_A, 4 * C + cell, dBy);
    rk_update(a.mode, a.first, a.c1, a.c2, a.fld_out, a.fld_B, a.fld_A, 5 * C + cell, dBz);
}

// RK epilogue of target row t at one (cell, p) point
template <int MC, typename TS>
__device__ __forceinline__ void row_epilogue(const StageArgs<TS>& a, const int* plane_of, int t, int p, bool pv,
                                             long long o, TS (&R)[MC + 1], TS (&I)[MC + 1]) {
    const int nzero = (t >= 2 && (a.parts & kPartClean)) ? min(t - 1, 80) : 0;
    const int mstride = a.m0 + 1;
#pragma unroll
    for (int m = 0; m <= MC; ++m) {
        if (m > a.m0 || m > t) continue;
        TS kr = R[m], ki = I[m];
        if (p < nzero) { kr = 0; ki = 0; }
        if (!pv) continue;
        if (t == 0) {
            rk_update<double>(a.mode, a.first, a.c1, a.c2, a.f00_out, a.f00_B, a.f00_A, o, (double)kr);
        } else {
            const long long q = plane_of[t * mstride + m];
            rk_update(a.mode, a.first, a.c1, a.c2, a.pl_out, a.pl_B, a.pl_A, q * a.pstride + o, kr);
            if (m > 0) rk_update(a.mode, a.first, a.c1, a.c2, a.pl_out, a.pl_B, a.pl_A, (q + 1) * a.pstride + o, ki);
        }
    }
}

// ---------------------------------------------------------------------------
// variant 1: global loads
// ---------------------------------------------------------------------------
template <int MC, typename TS>
__global__ void __launch_bounds__(256) rk_stage_kernel(const StageArgs<TS> a) {
    __shared__ double sj[3][kMaxCellsPerCta][kPChunk / 32];

    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const long long cell = (long long)blockIdx.x * blockDim.y + threadIdx.y;
    const bool cv = cell < a.cells;
    const int np = a.np;
    const int mstride = a.m0 + 1;

    long long cx = 0, cyy = 0;
    if (cv) { cx = cell % a.nx; cyy = cell / a.nx; }
    const long long cxm = cyy * a.nx + (cx == 0 ? a.nx - 1 : cx - 1);
    const long long cxp = cyy * a.nx + (cx == a.nx - 1 ? 0 : cx + 1);
    const long long cym = (cyy == 0 ? a.ny - 1 : cyy - 1) * (long long)a.nx + cx;
    const long long cyp = (cyy == a.ny - 1 ? 0 : cyy + 1) * (long long)a.nx + cx;
    const bool has_y = a.ny > 1;

    TS ex = 0, ey = 0, ez = 0, bx = 0, by = 0, bz = 0;
    if (cv) {
        // the couplings of the parts not evaluated see a zero field
        if (a.parts & kPartEx) ex = ld(a.fld_in + cell);
        if (a.parts & kPartEy) ey = ld(a.fld_in + a.cells + cell);
        if (a.parts & kPartEz) ez = ld(a.fld_in + 2 * a.cells + cell);
        if (a.parts & kPartB) {
            bx = ld(a.fld_in + 3 * a.cells + cell);
            by = ld(a.fld_in + 4 * a.cells + cell);
            bz = ld(a.fld_in + 5 * a.cells + cell);
        }
    }
    const bool adv = (a.parts & kPartAdv) != 0;

    double jx = 0.0, jyr = 0.0, jyi = 0.0;

    for (int pbase = 0; pbase < np; pbase += blockDim.x) {
        const int p = pbase + threadIdx.x;
        const bool pv = cv && p < np;
        const long long o = cell * np + p;
        const long long oxm = cxm * np + p, oxp = cxp * np + p;
        const long long oym = cym * np + p, oyp = cyp * np + p;
        const TS invp = pv ? (TS)ld(a.inv_pr + p) : TS(0);
        const TS vr = (pv && adv) ? (TS)ld(a.vr + p) : TS(0);
        const double wj = pv ? ld(a.wj + p) : 0.0;

        TS ar[3][MC + 1], ai[3][MC + 1];
#pragma unroll
        for (int r = 0; r < 3; ++r)
#pragma unroll
            for (int m = 0; m <= MC; ++m) { ar[r][m] = 0; ai[r][m] = 0; }

        for (int s = 0; s <= a.l0; ++s) {
#pragma unroll
            for (int m = 0; m <= MC; ++m) {
                if (m > a.m0 || m > s) continue;
                const CoefLM c = a.coef[s * mstride + m];
                const TS* src = nullptr;
                if (s > 0) src = a.pl_in + (long long)ld(a.plane_of + s * mstride + m) * a.pstride;
                auto load = [&](long long off, int comp) -> TS {
                    if (s == 0) return (TS)ld(a.f00_in + off);
                    return ld(src + comp * a.pstride + off);
                };
                // f itself (the stored value plus the plane's momentum profile, if any) at momentum
                // index pp of this cell; the x and y differences below act on the stored values alone
                const TS* ref = (s > 0 && a.pl_ref) ? a.pl_ref + (long long)ld(a.plane_of + s * mstride + m) * np
                                                    : nullptr;
                auto loadf = [&](long long off, int comp, int pp) -> TS {
                    const TS v = load(off, comp);
                    return ref ? v + ld(ref + comp * np + pp) : v;
                };
                TS fr = pv ? loadf(o, 0, p) : TS(0);
                TS fi = (m > 0 && pv) ? loadf(o, 1, p) : TS(0);
                TS frm = __shfl_up_sync(kFull, fr, 1), frp = __shfl_down_sync(kFull, fr, 1);
                TS fim = TS(0), fip = TS(0);
                if (m > 0) { fim = __shfl_up_sync(kFull, fi, 1); fip = __shfl_down_sync(kFull, fi, 1); }
                if (pv && lane == 0 && p > 0) {
                    frm = loadf(o - 1, 0, p - 1);
                    if (m > 0) fim = loadf(o - 1, 1, p - 1);
                }
                if (pv && lane == 31 && p + 1 < np) {
                    frp = loadf(o + 1, 0, p + 1);
                    if (m > 0) fip = loadf(o + 1, 1, p + 1);
                }
                // x neighbours: the halo columns at the edges of an x slab or a mirrored grid
                auto loadx = [&](int side, int comp) -> TS {
                    const bool edge = a.hx && (side ? cx == a.nx - 1 : cx == 0);
                    if (!edge) return load(side ? oxp : oxm, comp);
                    if (s == 0) return (TS)ld(hx_f00(a, side, cyy) + p);
                    return ld(hx_plane(a, side, (long long)ld(a.plane_of + s * mstride + m) + comp, cyy) + p);
                };
                const TS dxr = pv ? (loadx(0, 0) - loadx(1, 0)) * vr : TS(0);
                const TS dxi = (m > 0 && pv) ? (loadx(0, 1) - loadx(1, 1)) * vr : TS(0);
                TS dyr = 0, dyi = 0;
                if (has_y) {
                    dyr = pv ? (load(oym, 0) - load(oyp, 0)) * vr : TS(0);
                    dyi = (m > 0 && pv) ? (load(oym, 1) - load(oyp, 1)) * vr : TS(0);
                }
                couple<MC, TS>(ar, ai, m, s, c, fr, fi, frm, frp, fim, fip, dxr, dxi, dyr, dyi, has_y, p, np, invp,
                               ex, ey, ez, bx, by, bz, a.g00_s, a.g00_inv, a.g00_gr);
                if (s == 1) {
                    if (m == 0) jx += wj * (double)fr;
                    else if (m == 1) { jyr += wj * (double)fr; jyi += wj * (double)fi; }
                }
            }
            if (s >= 1) row_epilogue<MC, TS>(a, a.plane_of, s - 1, p, pv, o, ar[0], ai[0]);
            rotate_rows<MC, TS>(ar, ai);
        }
        row_epilogue<MC, TS>(a, a.plane_of, a.l0, p, pv, o, ar[0], ai[0]);
    }

    // per-cell current: warp sums, then warps in order (deterministic)
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        jx += __shfl_xor_sync(kFull, jx, off);
        jyr += __shfl_xor_sync(kFull, jyr, off);
        jyi += __shfl_xor_sync(kFull, jyi, off);
    }
    if (lane == 0) {
        sj[0][threadIdx.y][warp] = jx;
        sj[1][threadIdx.y][warp] = jyr;
        sj[2][threadIdx.y][warp] = jyi;
    }
    __syncthreads();
    if (threadIdx.x != 0 || !cv) return;
    double Jx = 0.0, Jyr = 0.0, Jyi = 0.0;
    const int nw = (min(np, (int)blockDim.x) + 31) >> 5;
    for (int w = 0; w < nw; ++w) { Jx += sj[0][threadIdx.y][w]; Jyr += sj[1][threadIdx.y][w]; Jyi += sj[2][threadIdx.y][w]; }
    const int hside = a.hx ? ((cx == 0 ? 1 : 0) | (cx == a.nx - 1 ? 2 : 0)) : 0;
    field_update(a, cell, cxm, cxp, cym, cyp, Jx, Jyr, Jyi, hside, cyy);
}

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------
template <typename TS, int MC>
cudaError_t launch_mc(const StageArgs<TS>& a, cudaStream_t s) {
    const int np_pad = ((a.np + 31) / 32) * 32;
    const int tx = np_pad < kPChunk ? np_pad : kPChunk;
    int cpb = kPChunk / tx;
    if (cpb > kMaxCellsPerCta) cpb = kMaxCellsPerCta;
    if (cpb < 1) cpb = 1;
    const long long blocks = (a.cells + cpb - 1) / cpb;
    rk_stage_kernel<MC, TS><<<dim3((unsigned)blocks), dim3(tx, cpb), 0, s>>>(a);
    return cudaGetLastError();
}

template <typename TS>
cudaError_t launch_stage(const StageArgs<TS>& a, int mc, cudaStream_t s) {
    // the pipelined kernel where the shape fits it (the full right-hand side),
    // else the global-load kernel
    if (a.parts == kPartAll) {
        const cudaError_t e = launch_stage_pipe<TS>(a, mc, s);
        if (e != cudaErrorNotSupported) return e;
        (void)cudaGetLastError();
    }
    switch (mc) {
        case 0: return launch_mc<TS, 0>(a, s);
        case 1: return launch_mc<TS, 1>(a, s);
        case 2: return launch_mc<TS, 2>(a, s);
        case 3: return launch_mc<TS, 3>(a, s);
        case 4: return launch_mc<TS, 4>(a, s);
        case 6: return launch_mc<TS, 6>(a, s);
        case 8: return launch_mc<TS, 8>(a, s);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace

cudaError_t launch_stage_fp64(const StageArgs<double>& a, int mc, cudaStream_t s) {
    return launch_stage<double>(a, mc, s);
}
cudaError_t launch_stage_fp32(const StageArgs<float>& a, int mc, cudaStream_t s) {
    return launch_stage<float>(a, mc, s);
}

}  // namespace oshun
