// x halo columns of a grid (the reference's x boundary handling,
// OSHUN-1/def-Parallel.cpp):
//   * mirrored x boundaries (Node_Communications::sameNode_mirror_X,
//     :1160-1206): the guard next to an edge column holds that column with
//     the sign (-1)^(l+m) on f_lm and -1 on Ey, Ez and Bx;
//   * an x slab of a grid split over ranks (Neighbor_Communications,
//     :3040-3129): the guards hold the neighbours' edge columns, exchanged
//     by the caller before each RK4 stage.
// Both fill the halo column sets the stage kernels read for the x-1
// neighbour of column 0 (side 0) and the x+1 neighbour of column nx-1
// (side 1); one side holds f00 [ny][np] (FP64), the l >= 1 planes
// [nplanes][ny][np] and the fields [6][ny], each part 256-byte aligned.
#include "oshun_internal.h"

namespace oshun {
namespace {

// the edge column x0 of one state set into one side's column set, times
// the mirror signs when `mirror`
template <typename TS>
__global__ void halo_column_kernel(const double* __restrict__ f00, const TS* __restrict__ pl,
                                   const TS* __restrict__ fld, HaloGrid g, int x0, unsigned char* __restrict__ out,
                                   int mirror) {
    const long long n00 = (long long)g.ny * g.np;
    const long long npl = (long long)g.nplanes * n00;
    const long long nf = 6LL * g.ny;
    double* o00 = reinterpret_cast<double*>(out);
    TS* opl = reinterpret_cast<TS*>(out + g.off_pl);
    TS* ofl = reinterpret_cast<TS*>(out + g.off_fld);
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n00 + npl + nf;
         i += (long long)gridDim.x * blockDim.x) {
        if (i < n00) {
            const long long y = i / g.np, p = i - y * g.np;
            o00[i] = f00[(y * g.nx + x0) * g.np + p];                  // l = m = 0: sign +1
        } else if (i < n00 + npl) {
            const long long j = i - n00;
            const long long q = j / n00, r = j - q * n00;
            const long long y = r / g.np, p = r - y * g.np;
            TS v = pl[q * g.pstride + (y * g.nx + x0) * g.np + p];
            if (mirror && ((g.plane_l[q] + g.plane_m[q]) & 1)) v = -v;   // (-1)^(l+m)
            opl[j] = v;
        } else {
            const long long j = i - n00 - npl;
            const int k = (int)(j / g.ny);
            const long long y = j - (long long)k * g.ny;
            TS v = fld[(long long)k * g.cells + y * g.nx + x0];
            if (mirror && (k == 1 || k == 2 || k == 3)) v = -v;           // Ey, Ez, Bx
            ofl[j] = v;
        }
    }
}

template <typename TS>
cudaError_t columns(const double* f00, const void* pl, const void* fld, const HaloGrid& g, int x0, void* out,
                    int mirror, cudaStream_t st) {
    const long long n = (long long)g.ny * g.np * (1 + g.nplanes) + 6LL * g.ny;
    long long b = (n + 255) / 256;
    if (b > 148 * 8) b = 148 * 8;
    halo_column_kernel<TS><<<(unsigned)b, 256, 0, st>>>(f00, (const TS*)pl, (const TS*)fld, g, x0,
                                                         (unsigned char*)out, mirror);
    return cudaGetLastError();
}

}  // namespace

cudaError_t launch_halo_column(const double* f00, const void* pl, const void* fld, const HaloGrid& g, bool fp32,
                               int x0, void* out, int mirror, cudaStream_t st) {
    if (fp32) return columns<float>(f00, pl, fld, g, x0, out, mirror, st);
    return columns<double>(f00, pl, fld, g, x0, out, mirror, st);
}

cudaError_t launch_halo_columns(const double* f00, const void* pl, const void* fld, const HaloGrid& g, bool fp32,
                                void* side0, void* side1, int mirror, cudaStream_t st) {
    const cudaError_t e = launch_halo_column(f00, pl, fld, g, fp32, 0, side0, mirror, st);
    if (e != cudaSuccess) return e;
    return launch_halo_column(f00, pl, fld, g, fp32, g.nx - 1, side1, mirror, st);
}

}  // namespace oshun
