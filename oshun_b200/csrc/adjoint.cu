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
                                                         const int smem_ws, const long long pstride) {
    extern __shared__ double sws[];
    const long long x = blockIdx.x;
    const int np = T.np;
    double* w = smem_ws ? sws : ws + x * wsz;
    adjw::collide_cell_T(T, l0, y + x * np, y + pstride + x * np, pstride, ee, eb, nsub, hsub, Dt, lam + x * np,
                         lam + pstride + x * np, pstride, w);
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
                               int nsub, double hsub, double Dt, double* ws, long long wsz, cudaStream_t st) {
    // wsz: the serial form's work space per cell (adj::coll_ws), at least the warp form's
    const long long need = adjw::coll_ws(T.np, nsub);
    if (need > wsz) return cudaErrorInvalidValue;
    const long long pstride = (long long)nx * T.np;
    const size_t smem = sizeof(double) * (size_t)need;
    if (smem <= 200 * 1024) {
        const cudaError_t e = ensure_dyn_smem((const void*)collide_adj_kernel, smem);
        if (e != cudaSuccess) return e;
        collide_adj_kernel<<<nx, 32, smem, st>>>(T, l0, y, lam, ee, eb, nsub, hsub, Dt, ws, wsz, 1, pstride);
    } else {
        collide_adj_kernel<<<nx, 32, 0, st>>>(T, l0, y, lam, ee, eb, nsub, hsub, Dt, ws, wsz, 0, pstride);
    }
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
