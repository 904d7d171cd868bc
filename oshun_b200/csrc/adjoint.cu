// Adjoint kernels of one small step of the 1D path with m0 = 0 (FP64), over
// the math of adjoint_math.h:
//   stage_vjp_kernel   F'(s)^T c for one RK4 stage state s (FP64 or FP32
//                      arithmetic on FP64 vectors): one CTA per cell,
//                      one thread per momentum point computes the cotangent
//                      of every f_l(x, p) (transposed G/H stencils, x
//                      advection, current) and its share of the E_x(x)
//                      cotangent, summed over the CTA in a fixed order;
//   collide_adj_kernel the collision step's transpose (reverse sweep through
//                      the e-e RK4 substeps, the transposed Thomas solves and
//                      the dependence of the tridiagonal coefficients on f00),
//                      one warp per cell (adjoint_warp.cuh: lane-parallel
//                      maps, warp scans for the cumulative integrals and
//                      their transposes, Thomas on lane 0), the cell's work
//                      space in shared memory where it fits, else in global
//                      memory;
//   rk_combine_kernel  the linear combinations of the RK4 transpose.
// State vectors use the plane layout: f00 plane, the l >= 1 planes, the 6
// field planes (for m0 = 0 and numy = 1: f[l][x][p] then E_x[x], ...).
#include "adjoint2d.cuh"
#include "adjoint_math.h"
#include "adjoint_warp.cuh"
#include "oshun_internal.h"

namespace oshun {
namespace {

using adj::Coef1;
using adj::CollTables;
using adj::Grid1;

// T: arithmetic of the transpose (double; float for the FP32 bulk form),
// the vectors stay FP64
template <typename T>
__global__ void stage_vjp_kernel(const Grid1 g, const double* __restrict__ s, const double* __restrict__ c,
                                 double* __restrict__ out) {
    const int x = blockIdx.x;
    const int k = threadIdx.x;
    const long long fsz = (long long)(g.l0 + 1) * g.nx * g.np;
    const double* Ex = s + fsz;          // field 0 of the state
    const double* cE = c + fsz;          // cotangent of the E_x slope
    __shared__ double red[8];
    double e = 0.0;
    if (k < g.np) {
        for (int l = 0; l <= g.l0; ++l)
            out[((long long)l * g.nx + x) * g.np + k] = (double)adj::vjp_f<T>(g, Ex, c, cE, l, x, k);
        e = (double)adj::vjp_E_point<T>(g, s, c, x, k);
    }
    // E_x cotangent: warp sums, then warps in order
    for (int off = 16; off > 0; off >>= 1) e += __shfl_xor_sync(0xffffffffu, e, off);
    if ((k & 31) == 0) red[k >> 5] = e;
    __syncthreads();
    if (k == 0) {
        double tot = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) tot += red[w];
        out[fsz + x] = tot;
        for (int f = 1; f < 6; ++f) out[fsz + (long long)f * g.nx + x] = 0.0;
    }
}

// F'(s)^T c for any grid (adjoint2d.cuh): one CTA per cell, one thread per
// momentum point gathers the cotangent of every source harmonic at its
// point; the cell's field cotangents are summed over the CTA in a fixed
// order, then the transposes of the current and of Ampere/Faraday added
__global__ void stage_vjp2_kernel(const adj2::Grid2 g, const double* __restrict__ s, const double* __restrict__ c,
                                  double* __restrict__ out) {
    const long long cell = blockIdx.x;
    const int k = threadIdx.x;
    __shared__ double red[6][8];
    double cF[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    if (k < g.np) {
        const double cdEx = adj2::fld(g, c, 0, cell), cdEy = adj2::fld(g, c, 1, cell), cdEz = adj2::fld(g, c, 2, cell);
        for (int l = 0; l <= g.l0; ++l)
            for (int M = 0; M <= (l < g.m0 ? l : g.m0); ++M) {
                adj2::Cx v = adj2::vjp_source(g, s, c, l, M, cell, k, cF);
                // the current: dEx = sum wj Re f10, dEy = 2 sum wj Re f11, dEz = -2 sum wj Im f11
                if (l == 1 && M == 0) v.r += g.wj[k] * cdEx;
                if (l == 1 && M == 1) { v.r += 2.0 * g.wj[k] * cdEy; v.i += -2.0 * g.wj[k] * cdEz; }
                if (l == 0) {
                    out[cell * g.np + k] = v.r;
                } else {
                    const long long q = g.plane_of[l * (g.m0 + 1) + M];
                    out[(1 + q) * g.pstride + cell * g.np + k] = v.r;
                    if (M > 0) out[(2 + q) * g.pstride + cell * g.np + k] = v.i;
                }
            }
    }
    const int lane = k & 31, warp = k >> 5;
#pragma unroll
    for (int f = 0; f < 6; ++f) {
        double v = cF[f];
        for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
        if (lane == 0) red[f][warp] = v;
    }
    __syncthreads();
    if (k == 0) {
        double F[6];
        for (int f = 0; f < 6; ++f) {
            F[f] = 0.0;
            for (int w = 0; w < (int)(blockDim.x >> 5); ++w) F[f] += red[f][w];
        }
        const adj2::Nbr n = adj2::nbr(g, cell);
        auto C = [&](int f, long long cc) { return adj2::fld(g, c, f, cc); };
        F[0] += g.idy * (C(5, n.yp) - C(5, n.ym));
        F[1] += -g.idx * (C(5, n.xp) - C(5, n.xm));
        F[2] += -g.idy * (C(3, n.yp) - C(3, n.ym)) + g.idx * (C(4, n.xp) - C(4, n.xm));
        F[3] += -g.idy * (C(2, n.yp) - C(2, n.ym));
        F[4] += g.idx * (C(2, n.xp) - C(2, n.xm));
        F[5] += g.idy * (C(0, n.yp) - C(0, n.ym)) - g.idx * (C(1, n.xp) - C(1, n.xm));
        double* of = out + (1 + (long long)g.nplanes) * g.pstride;
        for (int f = 0; f < 6; ++f) of[(long long)f * g.cells + cell] = F[f];
    }
}

// FP64 state vector <-> the FP32 planes and fields of an FP32-split handle
__global__ void to_fp32_kernel(const double* __restrict__ src, float* __restrict__ dst, long long n) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        dst[i] = (float)src[i];
}
__global__ void to_fp64_kernel(const float* __restrict__ src, double* __restrict__ dst, long long n) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        dst[i] = (double)src[i];
}

__global__ void __launch_bounds__(32) collide_adj_kernel(const CollTables T, const int l0, const double* __restrict__ y,
                                                         double* __restrict__ lam, const int ee, const int eb,
                                                         const int nsub, const double hsub, const double Dt,
                                                         double* __restrict__ ws, const long long wsz,
                                                         const int smem_ws, const long long pstride,
                                                         const adjw::CellPlanes P) {
    extern __shared__ double sws[];
    const long long x = blockIdx.x;
    const int np = T.np;
    double* w = smem_ws ? sws : ws + x * wsz;
    adjw::collide_cell_T(T, l0, y + x * np, y + pstride + x * np, pstride, ee, eb, nsub, hsub, Dt, lam + x * np,
                         lam + pstride + x * np, pstride, w, P);
}

// out = a0 * v0 + a1 * v1 (+ a2 * v2)
__global__ void rk_combine_kernel(double* out, const double* v0, double a0, const double* v1, double a1,
                                  const double* v2, double a2, long long n) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        double r = a0 * v0[i] + a1 * v1[i];
        if (v2) r += a2 * v2[i];
        out[i] = r;
    }
}

}  // namespace

cudaError_t launch_stage_vjp(const Grid1& g, const double* s, const double* c, double* out, cudaStream_t st,
                             bool fp32) {
    const int threads = ((g.np + 31) / 32) * 32;
    if (threads > 256) return cudaErrorInvalidValue;
    if (fp32) stage_vjp_kernel<float><<<g.nx, threads, 0, st>>>(g, s, c, out);
    else stage_vjp_kernel<double><<<g.nx, threads, 0, st>>>(g, s, c, out);
    return cudaGetLastError();
}

cudaError_t launch_convert(const double* src, float* dst, long long n, cudaStream_t st) {
    long long b = (n + 255) / 256;
    if (b > 148 * 8) b = 148 * 8;
    if (b < 1) return cudaSuccess;
    to_fp32_kernel<<<(unsigned)b, 256, 0, st>>>(src, dst, n);
    return cudaGetLastError();
}
cudaError_t launch_convert(const float* src, double* dst, long long n, cudaStream_t st) {
    long long b = (n + 255) / 256;
    if (b > 148 * 8) b = 148 * 8;
    if (b < 1) return cudaSuccess;
    to_fp64_kernel<<<(unsigned)b, 256, 0, st>>>(src, dst, n);
    return cudaGetLastError();
}

cudaError_t launch_collide_adj(const CollTables& T, int l0, int nx, const double* y, double* lam, int ee, int eb,
                               int nsub, double hsub, double Dt, double* ws, long long wsz, cudaStream_t st,
                               const int* plane_of, int m0, int mmax) {
    // wsz: the serial form's work space per cell (adj::coll_ws), at least the warp form's
    const long long need = adjw::coll_ws(T.np, nsub);
    if (need > wsz) return cudaErrorInvalidValue;
    const long long pstride = (long long)nx * T.np;   // nx: the cells of the grid
    const adjw::CellPlanes P{plane_of, m0, mmax};
    const size_t smem = sizeof(double) * (size_t)need;
    if (smem <= 200 * 1024) {
        const cudaError_t e = ensure_dyn_smem((const void*)collide_adj_kernel, smem);
        if (e != cudaSuccess) return e;
        collide_adj_kernel<<<nx, 32, smem, st>>>(T, l0, y, lam, ee, eb, nsub, hsub, Dt, ws, wsz, 1, pstride, P);
    } else {
        collide_adj_kernel<<<nx, 32, 0, st>>>(T, l0, y, lam, ee, eb, nsub, hsub, Dt, ws, wsz, 0, pstride, P);
    }
    return cudaGetLastError();
}

cudaError_t launch_stage_vjp2(const adj2::Grid2& g, const double* s, const double* c, double* out, cudaStream_t st) {
    const int threads = ((g.np + 31) / 32) * 32;
    if (threads > 256) return cudaErrorInvalidValue;
    stage_vjp2_kernel<<<(unsigned)g.cells, threads, 0, st>>>(g, s, c, out);
    return cudaGetLastError();
}

cudaError_t launch_rk_combine(double* out, const double* v0, double a0, const double* v1, double a1, const double* v2,
                              double a2, long long n, cudaStream_t st) {
    long long b = (n + 255) / 256;
    if (b > 148 * 8) b = 148 * 8;
    rk_combine_kernel<<<(unsigned)b, 256, 0, st>>>(out, v0, a0, v1, a1, v2, a2, n);
    return cudaGetLastError();
}

}  // namespace oshun
