// Per-cell pieces of the implicit electric field, Implicit_E_Field::advance
// (OSHUN-1/def-ImplicitE.cpp:471-676): the current of the probe states, the
// current Ampere's law asks for, the probe amplitudes and the 3x3 solve of
// the finite-difference conductivity tensor.  The probe states themselves
// come from the stage kernel (restricted coupling tables) and the collision
// kernel; the host drives the sequence (abi.cu, oshun_rk2_imp_step).
//
// Every field and current is real in the reference (its complex arithmetic
// carries zero imaginary parts), so the kernels work on real numbers with the
// reference's order of operations.
#include <float.h>

#include "oshun_internal.h"

namespace oshun {
namespace {

// Current_xyz::calculate_J (def-ImplicitE.cpp:125-185) of one cell.  The
// reference halves the end points of its trapezoid through a one-index
// access, jayx(ix) *= 0.5, that addresses row y = 0 of its guarded array
// (def-ImplicitE.cpp:143, 166), so every interior cell sums its momentum
// row with unhalved ends: S = w0 f0 + w_{n-1} f_{n-1} + sum_{0<i<n-1} w_i f_i,
// J = c (dp S + small w1 f1) with w = p^3/gamma, c = -4 pi/3 (f10) or
// -8 pi/3 (f11; Jy = Re, Jz = -Im).
template <typename TP>
__global__ void implicit_current_kernel(const ImplicitArgs a, const int set, double* J) {
    const long long cell = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (cell >= a.cells) return;
    const int n = a.np;
    const double* w = a.p3og;
    const TP* pl = reinterpret_cast<const TP*>(a.planes[set]);
    // f of plane q at momentum point i: the stored value plus the plane's profile, if any
    auto row_sum = [&](const int q) {
        const TP* g = pl + (long long)q * a.pstride + cell * n;
        const double* r = a.pl_ref ? a.pl_ref + (long long)q * n : nullptr;
        auto f = [&](int i) { return (double)g[i] + (r ? r[i] : 0.0); };
        double s = f(0) * w[0];
        s = s + f(n - 1) * w[n - 1];
        for (int i = 1; i < n - 1; ++i) s = s + f(i) * w[i];
        s = s * a.dp;
        s = s + a.small * (f(1) * w[1]);
        return s;
    };
    J[cell] = row_sum(a.q10) * a.c4;
    if (a.q11 >= 0) {
        const double re = row_sum(a.q11) * a.c8;
        const double im = row_sum(a.q11 + 1) * a.c8;
        J[a.cells + cell] = re;
        J[2 * a.cells + cell] = -im;
    } else {
        J[a.cells + cell] = 0.0;
        J[2 * a.cells + cell] = 0.0;
    }
}

// Implicit_E_Field::Ampere (def-ImplicitE.cpp:724-752): JN = rot B from
// centred differences of the B field scaled first (tmp = B idy; tmp.Dy())
template <typename TS>
__global__ void implicit_ampere_kernel(const ImplicitArgs a, const TS* F, double* JN) {
    const long long cell = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (cell >= a.cells) return;
    const int nx = a.nx, ny = a.ny;
    const int y = (int)(cell / nx), x = (int)(cell - (long long)y * nx);
    const long long C = a.cells;
    const long long xm = (long long)y * nx + (x == 0 ? nx - 1 : x - 1), xp = (long long)y * nx + (x == nx - 1 ? 0 : x + 1);
    const long long ym = (long long)(y == 0 ? ny - 1 : y - 1) * nx + x, yp = (long long)(y == ny - 1 ? 0 : y + 1) * nx + x;
    const double idx = a.idx, idy = a.idy, midx = -1.0 * a.idx, midy = -1.0 * a.idy;
    const TS* Bx = F + 3 * C;
    const TS* By = F + 4 * C;
    const TS* Bz = F + 5 * C;
    JN[cell] = (double)Bz[ym] * idy - (double)Bz[yp] * idy;
    JN[C + cell] = (double)Bz[xm] * midx - (double)Bz[xp] * midx;
    double jz = (double)Bx[ym] * midy - (double)Bx[yp] * midy;
    jz = jz + ((double)By[xm] * idx - (double)By[xp] * idx);
    JN[2 * C + cell] = jz;
}

// Implicit_E_Field::FindDE (def-ImplicitE.cpp:694-720): the probe amplitude
// sqrt(Ex^2 + Ey^2 + Ez^2) LargeEps + Eps, the same for the three components
template <typename TS>
__global__ void implicit_find_de_kernel(const ImplicitArgs a, const TS* F, double* DE) {
    const long long cell = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (cell >= a.cells) return;
    const long long C = a.cells;
    const double ex = (double)F[cell], ey = (double)F[C + cell], ez = (double)F[2 * C + cell];
    double d = ex * ex;
    d = d + ey * ey;
    d = d + ez * ez;
    d = sqrt(d);
    d = d * a.large_eps;
    d = d + a.eps;
    DE[cell] = d;
    DE[C + cell] = d;
    DE[2 * C + cell] = d;
}

// one probe's field: component `comp` = DE, the others and B zero (the
// reference sets Y.EMF().E_comp() = DE before each probe; the restricted
// coupling table of that probe reads only that component)
template <typename TS>
__global__ void implicit_probe_field_kernel(const ImplicitArgs a, const double* DE, const int comp, TS* FE) {
    const long long cell = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (cell >= a.cells) return;
    const long long C = a.cells;
    for (int f = 0; f < 6; ++f) FE[f * C + cell] = f == comp ? (TS)DE[comp * C + cell] : TS(0);
}

// The conductivity-tensor solve of one attempt (def-ImplicitE.cpp:543-600):
// sgm_ij = (J(E_j)_i - J0_i) / DE_j, clm = JN - J0, E = Cramer's rule
// (Det33 and Detx/y/z33, def-Nmethods.cpp:215-253) where |det| > 6 DBL_MIN,
// else the cell counts a zero determinant and its DEx, DEy grow by 2 and 1.3
// for the next attempt.  1D (if_implicit1D): Ex = DEx J0x / (J0x - J(Ex)x).
__global__ void implicit_solve_kernel(const ImplicitArgs a, const double* J0, const double* JX, const double* JY,
                                      const double* JZ, const double* JN, double* DE, double* EN, int* zeros) {
    const long long cell = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (cell >= a.cells) return;
    const long long C = a.cells;
    if (a.one_d) {
        EN[cell] = DE[cell] * J0[cell] / (J0[cell] - JX[cell]);
        EN[C + cell] = 0.0;
        EN[2 * C + cell] = 0.0;
        return;
    }
    double A[3][3], D[3];
    const double* Jp[3] = {JX, JY, JZ};
    for (int j = 0; j < 3; ++j)
        for (int i = 0; i < 3; ++i) A[i][j] = (Jp[j][i * C + cell] - J0[i * C + cell]) / DE[j * C + cell];
    for (int i = 0; i < 3; ++i) D[i] = JN[i * C + cell] - J0[i * C + cell];
    const double det = A[0][0] * (A[1][1] * A[2][2] - A[2][1] * A[1][2]) -
                       A[1][0] * (A[0][1] * A[2][2] - A[2][1] * A[0][2]) +
                       A[2][0] * (A[0][1] * A[1][2] - A[1][1] * A[0][2]);
    if (fabs(det) > 6.0 * DBL_MIN) {
        const double dx = D[0] * (A[1][1] * A[2][2] - A[2][1] * A[1][2]) -
                          D[1] * (A[0][1] * A[2][2] - A[2][1] * A[0][2]) +
                          D[2] * (A[0][1] * A[1][2] - A[1][1] * A[0][2]);
        const double dy = A[0][0] * (D[1] * A[2][2] - D[2] * A[1][2]) -
                          A[1][0] * (D[0] * A[2][2] - D[2] * A[0][2]) +
                          A[2][0] * (D[0] * A[1][2] - D[1] * A[0][2]);
        const double dz = A[0][0] * (A[1][1] * D[2] - A[2][1] * D[1]) -
                          A[1][0] * (A[0][1] * D[2] - A[2][1] * D[0]) +
                          A[2][0] * (A[0][1] * D[1] - A[1][1] * D[0]);
        EN[cell] = dx / det;
        EN[C + cell] = dy / det;
        EN[2 * C + cell] = dz / det;
    } else {
        atomicAdd(zeros, 1);
        DE[cell] *= 2;
        DE[C + cell] *= 1.3;
        EN[cell] = 0.0;
        EN[C + cell] = 0.0;
        EN[2 * C + cell] = 0.0;
    }
}

// Y.EMF().E = EN (def-ImplicitE.cpp:662-664)
template <typename TS>
__global__ void implicit_set_e_kernel(const ImplicitArgs a, const double* EN, TS* F) {
    const long long cell = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (cell >= a.cells) return;
    for (int i = 0; i < 3; ++i) F[i * a.cells + cell] = (TS)EN[i * a.cells + cell];
}

unsigned grid(long long n) { return (unsigned)((n + 127) / 128); }

}  // namespace

cudaError_t launch_implicit_current(const ImplicitArgs& a, int set, double* J, cudaStream_t s) {
    if (a.fp32) implicit_current_kernel<float><<<grid(a.cells), 128, 0, s>>>(a, set, J);
    else implicit_current_kernel<double><<<grid(a.cells), 128, 0, s>>>(a, set, J);
    return cudaGetLastError();
}
cudaError_t launch_implicit_ampere(const ImplicitArgs& a, const void* fields, double* JN, cudaStream_t s) {
    if (a.fp32) implicit_ampere_kernel<float><<<grid(a.cells), 128, 0, s>>>(a, (const float*)fields, JN);
    else implicit_ampere_kernel<double><<<grid(a.cells), 128, 0, s>>>(a, (const double*)fields, JN);
    return cudaGetLastError();
}
cudaError_t launch_implicit_find_de(const ImplicitArgs& a, const void* fields, double* DE, cudaStream_t s) {
    if (a.fp32) implicit_find_de_kernel<float><<<grid(a.cells), 128, 0, s>>>(a, (const float*)fields, DE);
    else implicit_find_de_kernel<double><<<grid(a.cells), 128, 0, s>>>(a, (const double*)fields, DE);
    return cudaGetLastError();
}
cudaError_t launch_implicit_probe_field(const ImplicitArgs& a, const double* DE, int comp, void* FE, cudaStream_t s) {
    if (a.fp32) implicit_probe_field_kernel<float><<<grid(a.cells), 128, 0, s>>>(a, DE, comp, (float*)FE);
    else implicit_probe_field_kernel<double><<<grid(a.cells), 128, 0, s>>>(a, DE, comp, (double*)FE);
    return cudaGetLastError();
}
cudaError_t launch_implicit_solve(const ImplicitArgs& a, const double* J0, const double* JX, const double* JY,
                                  const double* JZ, const double* JN, double* DE, double* EN, int* zeros,
                                  cudaStream_t s) {
    implicit_solve_kernel<<<grid(a.cells), 128, 0, s>>>(a, J0, JX, JY, JZ, JN, DE, EN, zeros);
    return cudaGetLastError();
}
cudaError_t launch_implicit_set_e(const ImplicitArgs& a, const double* EN, void* fields, cudaStream_t s) {
    if (a.fp32) implicit_set_e_kernel<float><<<grid(a.cells), 128, 0, s>>>(a, EN, (float*)fields);
    else implicit_set_e_kernel<double><<<grid(a.cells), 128, 0, s>>>(a, EN, (double*)fields);
    return cudaGetLastError();
}

}  // namespace oshun
