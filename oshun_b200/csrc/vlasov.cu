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
// Two variants:
//   rk_stage_tma_kernel (nump <= 256, rows of 16-byte multiples): a CTA owns
//     `tx` consecutive cells of one y row.  A producer warp streams each
//     source harmonic's tile -- the cells, their x neighbours and their
//     y-1/y+1 neighbour segments, all momentum points -- into a ring of
//     shared-memory slots with bulk async copies (cp.async.bulk, full/empty
//     mbarriers), kDepth harmonics ahead of the compute, and the RK
//     epilogue's Y0/Y rows into a double-buffered row stage one row ahead.
//     The consumer warps read the stencil (p +- 1, x +- 1, y +- 1) and the
//     epilogue operands from shared memory; their only global accesses are
//     the stores.
//   rk_stage_kernel (any nump <= 1024): the same arithmetic with global loads
//     and warp shuffles for p +- 1; momentum rows wider than 256 are swept in
//     chunks.
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
constexpr int kDepth = 10;
constexpr long long kWaitLimit = 1ll << 22;   // mbarrier try_wait rounds before giving up

template <typename T>
__device__ __forceinline__ T ld(const T* p) { return __ldg(p); }

// ---------------------------------------------------------------------------
// field epilogue: J reduction result + Ampere/Faraday, RK update of 6 fields
// ---------------------------------------------------------------------------
template <typename TS>
__device__ __forceinline__ void field_update(const StageArgs<TS>& a, long long cell, long long cxm, long long cxp,
                                             long long cym, long long cyp, double Jx, double Jyr, double Jyi) {
    const TS* F = a.fld_in;
    const long long C = a.cells;
    const TS idx = (TS)a.idx, idy = (TS)a.idy;
    // J: Ex += Jx, Ey += Re J11, Ez += -Im J11 with J11 = 2 * (f11 quadrature)
    TS dEx = (TS)Jx;
    TS dEy = (TS)(2.0 * Jyr);
    TS dEz = (TS)(-(2.0 * Jyi));
    dEx += idy * (ld(F + 5 * C + cym) - ld(F + 5 * C + cyp));
    dEy += -idx * (ld(F + 5 * C + cxm) - ld(F + 5 * C + cxp));
    dEz += -idy * (ld(F + 3 * C + cym) - ld(F + 3 * C + cyp));
    dEz += idx * (ld(F + 4 * C + cxm) - ld(F + 4 * C + cxp));
    TS dBx = -idy * (ld(F + 2 * C + cym) - ld(F + 2 * C + cyp));
    TS dBy = idx * (ld(F + 2 * C + cxm) - ld(F + 2 * C + cxp));
    TS dBz = idy * (ld(F + 0 * C + cym) - ld(F + 0 * C + cyp));
    dBz += -idx * (ld(F + 1 * C + cxm) - ld(F + 1 * C + cxp));
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
    const int nzero = t >= 2 ? min(t - 1, 80) : 0;
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
        ex = ld(a.fld_in + cell);
        ey = ld(a.fld_in + a.cells + cell);
        ez = ld(a.fld_in + 2 * a.cells + cell);
        bx = ld(a.fld_in + 3 * a.cells + cell);
        by = ld(a.fld_in + 4 * a.cells + cell);
        bz = ld(a.fld_in + 5 * a.cells + cell);
    }

    double jx = 0.0, jyr = 0.0, jyi = 0.0;

    for (int pbase = 0; pbase < np; pbase += blockDim.x) {
        const int p = pbase + threadIdx.x;
        const bool pv = cv && p < np;
        const long long o = cell * np + p;
        const long long oxm = cxm * np + p, oxp = cxp * np + p;
        const long long oym = cym * np + p, oyp = cyp * np + p;
        const TS invp = pv ? (TS)ld(a.inv_pr + p) : TS(0);
        const TS vr = pv ? (TS)ld(a.vr + p) : TS(0);
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
                TS fr = pv ? load(o, 0) : TS(0);
                TS fi = (m > 0 && pv) ? load(o, 1) : TS(0);
                TS frm = __shfl_up_sync(kFull, fr, 1), frp = __shfl_down_sync(kFull, fr, 1);
                TS fim = TS(0), fip = TS(0);
                if (m > 0) { fim = __shfl_up_sync(kFull, fi, 1); fip = __shfl_down_sync(kFull, fi, 1); }
                if (pv && lane == 0 && p > 0) {
                    frm = load(o - 1, 0);
                    if (m > 0) fim = load(o - 1, 1);
                }
                if (pv && lane == 31 && p + 1 < np) {
                    frp = load(o + 1, 0);
                    if (m > 0) fip = load(o + 1, 1);
                }
                const TS dxr = pv ? (load(oxm, 0) - load(oxp, 0)) * vr : TS(0);
                const TS dxi = (m > 0 && pv) ? (load(oxm, 1) - load(oxp, 1)) * vr : TS(0);
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
    field_update(a, cell, cxm, cxp, cym, cyp, Jx, Jyr, Jyi);
}

// ---------------------------------------------------------------------------
// variant 2: warp-specialised bulk-copy pipeline through shared memory
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
// bounded wait for the phase with this parity; false when the limit ran out
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
    const uint32_t addr = smem_u32(bar);
    for (long long i = 0; i < kWaitLimit; ++i) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred P1;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, P1;\n\t}"
            : "=r"(done)
            : "r"(addr), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}
// global -> shared bulk copy completing on `bar`; 16-byte aligned, size % 16 == 0
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}
__device__ __forceinline__ void consumer_sync(int nthreads) {
    asm volatile("bar.sync 1, %0;" ::"r"(nthreads) : "memory");
}

__host__ __device__ inline size_t align_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

// shared-memory layout of the pipelined kernel (host and device agree)
struct TmaLayout {
    size_t off_coef, off_plane, off_seq, off_sj, off_flag, off_slots, slot_bytes, off_rows, row_arr_bytes, total;
    int seg_cells;
};
// barriers at offset 0: full[kDepth], empty[kDepth], rowfull[2], rowempty[2]
__host__ __device__ inline TmaLayout tma_layout(int ncoef, int nh, int tx, int np, bool has_y, int elem_bytes,
                                               int m0) {
    TmaLayout L;
    L.seg_cells = tx + 2 + (has_y ? 2 * tx : 0);
    L.off_coef = 256;
    L.off_plane = align_up(L.off_coef + sizeof(CoefLM) * (size_t)ncoef, 16);
    L.off_seq = align_up(L.off_plane + sizeof(int) * (size_t)ncoef, 16);
    L.off_sj = align_up(L.off_seq + sizeof(int) * (size_t)nh, 16);
    L.off_flag = align_up(L.off_sj + sizeof(double) * 3 * (size_t)tx * 8, 16);
    L.off_slots = align_up(L.off_flag + 16, 128);
    L.slot_bytes = align_up((size_t)2 * L.seg_cells * np * elem_bytes, 128);
    L.off_rows = L.off_slots + kDepth * L.slot_bytes;
    size_t row0 = (size_t)tx * np * 8;
    size_t rowl = (size_t)(1 + 2 * m0) * tx * np * elem_bytes;
    L.row_arr_bytes = align_up(row0 > rowl ? row0 : rowl, 128);
    L.total = L.off_rows + 2 * 2 * L.row_arr_bytes;   // [buffer][B, A]
    return L;
}

template <int MC, typename TS, int MAXT>
__global__ void __launch_bounds__(MAXT, 1) rk_stage_tma_kernel(const StageArgs<TS> a) {
    extern __shared__ __align__(128) unsigned char smem[];
    const int np = a.np, nx = a.nx, ny = a.ny;
    const int np_pad = (np + 31) & ~31;
    const bool has_y = ny > 1;
    const int tx = (int)(blockDim.x - 32) / np_pad;
    const int nct = np_pad * tx;                       // consumer threads
    const int ncw = nct >> 5;                          // consumer warps
    const int mstride = a.m0 + 1;
    const int ncoef = (a.l0 + 1) * mstride;
    const TmaLayout L = tma_layout(ncoef, a.nh, tx, np, has_y, (int)sizeof(TS), a.m0);
    uint64_t* full = reinterpret_cast<uint64_t*>(smem);
    uint64_t* empty = full + kDepth;
    uint64_t* rowfull = empty + kDepth;
    uint64_t* rowempty = rowfull + 2;
    CoefLM* scoef = reinterpret_cast<CoefLM*>(smem + L.off_coef);
    int* splane = reinterpret_cast<int*>(smem + L.off_plane);
    int* sseq = reinterpret_cast<int*>(smem + L.off_seq);
    double* sj = reinterpret_cast<double*>(smem + L.off_sj);
    unsigned char* slots = smem + L.off_slots;
    unsigned char* rows = smem + L.off_rows;
    const bool need_B = a.mode != 1;
    const bool need_A = a.mode != 1 && !a.first;

    const int tid = threadIdx.x;
    const int tiles_x = (nx + tx - 1) / tx;
    const int y = blockIdx.x / tiles_x;
    const int x0 = (blockIdx.x - y * tiles_x) * tx;
    const int txv = min(tx, nx - x0);
    const long long row = (long long)y * nx;
    const long long rym = (long long)(y == 0 ? ny - 1 : y - 1) * nx;
    const long long ryp = (long long)(y == ny - 1 ? 0 : y + 1) * nx;

    // tables to shared memory, barriers
    {
        const double* src = reinterpret_cast<const double*>(a.coef);
        double* dst = reinterpret_cast<double*>(scoef);
        const int nd = ncoef * (int)(sizeof(CoefLM) / sizeof(double));
        for (int i = tid; i < nd; i += blockDim.x) dst[i] = src[i];
        for (int i = tid; i < ncoef; i += blockDim.x) splane[i] = a.plane_of[i];
        for (int i = tid; i < a.nh; i += blockDim.x) sseq[i] = a.seq[i];
        if (tid == 0) {
            for (int k = 0; k < kDepth; ++k) { mbar_init(full + k, 1); mbar_init(empty + k, ncw); }
            for (int k = 0; k < 2; ++k) { mbar_init(rowfull + k, 1); mbar_init(rowempty + k, ncw); }
            asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        }
    }
    __syncthreads();

    // ---------------- producer warp -----------------------------------------
    if (tid >= nct) {
        if (tid != nct) return;
        const long long xm_cell = row + (x0 == 0 ? nx - 1 : x0 - 1);
        const long long xp_cell = row + ((x0 + txv) % nx);
        int issued = 0;
        bool ok = true;
        auto fill_source = [&](int s, int m) {
            const int idx = issued;
            const int slot = idx % kDepth, j = idx / kDepth;
            if (j >= 1 && !mbar_wait(empty + slot, (uint32_t)((j - 1) & 1))) { ok = false; return; }
            unsigned char* dst = slots + (size_t)slot * L.slot_bytes;
            const unsigned char* src;
            int esz, ncomp;
            if (s == 0) {
                src = reinterpret_cast<const unsigned char*>(a.f00_in);
                esz = 8; ncomp = 1;
            } else {
                const long long q = splane[s * mstride + m];
                src = reinterpret_cast<const unsigned char*>(a.pl_in + q * a.pstride);
                esz = (int)sizeof(TS); ncomp = m > 0 ? 2 : 1;
            }
            const uint32_t bpc = (uint32_t)np * esz;   // bytes per cell
            const uint32_t ncell = txv + 2 + (has_y ? 2 * txv : 0);
            mbar_expect_tx(full + slot, ncomp * ncell * bpc);
            for (int comp = 0; comp < ncomp; ++comp) {
                unsigned char* cb = dst + (size_t)comp * L.seg_cells * bpc;
                const unsigned char* pb = src + (size_t)comp * a.pstride * esz;
                bulk_g2s(cb, pb + (size_t)xm_cell * bpc, bpc, full + slot);
                bulk_g2s(cb + bpc, pb + (size_t)(row + x0) * bpc, txv * bpc, full + slot);
                bulk_g2s(cb + (size_t)(txv + 1) * bpc, pb + (size_t)xp_cell * bpc, bpc, full + slot);
                if (has_y) {
                    bulk_g2s(cb + (size_t)(tx + 2) * bpc, pb + (size_t)(rym + x0) * bpc, txv * bpc, full + slot);
                    bulk_g2s(cb + (size_t)(2 * tx + 2) * bpc, pb + (size_t)(ryp + x0) * bpc, txv * bpc, full + slot);
                }
            }
            ++issued;
        };
        int rows_issued = 0;
        auto fill_row = [&](int t) {
            const int rb = t & 1, k = t >> 1;
            if (k >= 1 && !mbar_wait(rowempty + rb, (uint32_t)((k - 1) & 1))) { ok = false; return; }
            unsigned char* base = rows + (size_t)rb * 2 * L.row_arr_bytes;
            uint32_t bytes = 0;
            const uint32_t nb = (need_B ? 1 : 0) + (need_A ? 1 : 0);
            if (t == 0) {
                bytes = nb * (uint32_t)txv * np * 8;
            } else {
                int np_row = 0;
                for (int m = 0; m <= min(t, a.m0); ++m) np_row += m > 0 ? 2 : 1;
                bytes = nb * (uint32_t)np_row * txv * np * (uint32_t)sizeof(TS);
            }
            mbar_expect_tx(rowfull + rb, bytes);
            if (t == 0) {
                const uint32_t b = (uint32_t)txv * np * 8;
                if (need_B) bulk_g2s(base, a.f00_B + (row + x0) * np, b, rowfull + rb);
                if (need_A) bulk_g2s(base + L.row_arr_bytes, a.f00_A + (row + x0) * np, b, rowfull + rb);
            } else {
                const uint32_t b = (uint32_t)txv * np * sizeof(TS);
                int kk = 0;
                for (int m = 0; m <= min(t, a.m0); ++m) {
                    const long long q = splane[t * mstride + m];
                    for (int comp = 0; comp < (m > 0 ? 2 : 1); ++comp, ++kk) {
                        const long long off = (q + comp) * a.pstride + (row + x0) * np;
                        const size_t d = (size_t)kk * tx * np * sizeof(TS);
                        if (need_B) bulk_g2s(base + d, a.pl_B + off, b, rowfull + rb);
                        if (need_A) bulk_g2s(base + L.row_arr_bytes + d, a.pl_A + off, b, rowfull + rb);
                    }
                }
            }
            ++rows_issued;
        };
        for (int s = 0; s <= a.l0 && ok; ++s) {
            if (need_B && s >= 1) fill_row(s - 1);
            for (int m = 0; m <= min(s, a.m0) && ok; ++m) fill_source(s, m);
        }
        if (ok && need_B) fill_row(a.l0);
        if (!ok) {
            atomicOr(a.err, 16);
            // bounded drain of every copy that may still be in flight
            for (int idx = max(0, issued - kDepth); idx < issued; ++idx)
                mbar_wait(full + (idx % kDepth), (uint32_t)((idx / kDepth) & 1));
            for (int t = max(0, rows_issued - 2); t < rows_issued; ++t)
                mbar_wait(rowfull + (t & 1), (uint32_t)((t >> 1) & 1));
        }
        return;
    }

    // ---------------- consumer warps ----------------------------------------
    const int c = tid / np_pad, p = tid - c * np_pad;
    const int lane = tid & 31;
    const bool cv = c < txv;
    const bool pv = cv && p < np;
    const int xc = x0 + (cv ? c : 0);
    const long long cell = row + xc;
    const long long cxm = row + (xc == 0 ? nx - 1 : xc - 1);
    const long long cxp = row + (xc == nx - 1 ? 0 : xc + 1);
    const long long cym = rym + xc, cyp = ryp + xc;

    TS ex = 0, ey = 0, ez = 0, bx = 0, by = 0, bz = 0;
    if (cv) {
        ex = ld(a.fld_in + cell);
        ey = ld(a.fld_in + a.cells + cell);
        ez = ld(a.fld_in + 2 * a.cells + cell);
        bx = ld(a.fld_in + 3 * a.cells + cell);
        by = ld(a.fld_in + 4 * a.cells + cell);
        bz = ld(a.fld_in + 5 * a.cells + cell);
    }
    const TS invp = pv ? (TS)ld(a.inv_pr + p) : TS(0);
    const TS vr = pv ? (TS)ld(a.vr + p) : TS(0);
    const double wj = pv ? ld(a.wj + p) : 0.0;
    const long long o = cell * np + p;

    TS ar[3][MC + 1], ai[3][MC + 1];
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int m = 0; m <= MC; ++m) { ar[r][m] = 0; ai[r][m] = 0; }
    double jx = 0.0, jyr = 0.0, jyi = 0.0;
    bool dead = false;   // a wait ran out: skip all further work and writes

    // RK epilogue of target row t from the staged Y0/Y rows
    auto epilogue = [&](int t) {
        const int rb = t & 1;
        if (need_B && !dead && !mbar_wait(rowfull + rb, (uint32_t)((t >> 1) & 1))) {
            atomicOr(a.err, 16);
            dead = true;
        }
        if (!dead) {
            const unsigned char* base = rows + (size_t)rb * 2 * L.row_arr_bytes;
            const int nzero = t >= 2 ? min(t - 1, 80) : 0;
            int kk = 0;
#pragma unroll
            for (int m = 0; m <= MC; ++m) {
                if (m > a.m0 || m > t) continue;
                TS kr = ar[0][m], ki = ai[0][m];
                if (p < nzero) { kr = 0; ki = 0; }
                if (pv) {
                    if (t == 0) {
                        const double* Bs = reinterpret_cast<const double*>(base) + c * np + p;
                        const double* As = reinterpret_cast<const double*>(base + L.row_arr_bytes) + c * np + p;
                        double* Ag = a.f00_A + o;
                        if (a.mode == 1) {
                            a.f00_out[o] = (double)kr;
                        } else {
                            const double tt = (double)kr * a.c1;
                            const double b = *Bs;
                            if (a.f00_out) a.f00_out[o] = b + tt;
                            *Ag = (a.first ? b : *As) + tt * a.c2;
                        }
                    } else {
                        const long long q = splane[t * mstride + m];
                        for (int comp = 0; comp < (m > 0 ? 2 : 1); ++comp) {
                            const TS k = comp ? ki : kr;
                            const size_t d = (size_t)(kk + comp) * tx * np + c * np + p;
                            const long long g = (q + comp) * a.pstride + o;
                            if (a.mode == 1) {
                                a.pl_out[g] = k;
                            } else {
                                const TS tt = k * (TS)a.c1;
                                const TS b = reinterpret_cast<const TS*>(base)[d];
                                if (a.pl_out) a.pl_out[g] = b + tt;
                                a.pl_A[g] = (a.first ? b : reinterpret_cast<const TS*>(base + L.row_arr_bytes)[d]) +
                                            tt * (TS)a.c2;
                            }
                        }
                    }
                }
                kk += m > 0 ? 2 : 1;
            }
        }
        __syncwarp();
        if (need_B && lane == 0) mbar_arrive(rowempty + rb);
    };

    // consume source harmonic `id` (already landed) of order (s, m)
    auto consume = [&](const int s, const int m, const int id) {
        const unsigned char* sb = slots + (size_t)(id % kDepth) * L.slot_bytes;
        const int seg = L.seg_cells * np;
        auto rd = [&](int comp, int cs, int pp) -> TS {
            if constexpr (sizeof(TS) == 8) {
                return reinterpret_cast<const TS*>(sb)[comp * seg + cs * np + pp];
            } else {
                if (s == 0) return (TS)reinterpret_cast<const double*>(sb)[cs * np + pp];
                return reinterpret_cast<const TS*>(sb)[comp * seg + cs * np + pp];
            }
        };
        TS fr = 0, fi = 0, frm = 0, frp = 0, fim = 0, fip = 0, dxr = 0, dxi = 0, dyr = 0, dyi = 0;
        if (pv) {
            fr = rd(0, 1 + c, p);
            if (p > 0) frm = rd(0, 1 + c, p - 1);
            if (p + 1 < np) frp = rd(0, 1 + c, p + 1);
            dxr = (rd(0, c, p) - rd(0, c + 2, p)) * vr;
            if (has_y) dyr = (rd(0, tx + 2 + c, p) - rd(0, 2 * tx + 2 + c, p)) * vr;
            if (m > 0) {
                fi = rd(1, 1 + c, p);
                if (p > 0) fim = rd(1, 1 + c, p - 1);
                if (p + 1 < np) fip = rd(1, 1 + c, p + 1);
                dxi = (rd(1, c, p) - rd(1, c + 2, p)) * vr;
                if (has_y) dyi = (rd(1, tx + 2 + c, p) - rd(1, 2 * tx + 2 + c, p)) * vr;
            }
        }
        // 128-bit broadcast loads of the coupling table entry
        CoefLM cc;
        {
            const double2* src2 = reinterpret_cast<const double2*>(scoef + s * mstride + m);
            double2* dst2 = reinterpret_cast<double2*>(&cc);
#pragma unroll
            for (int k = 0; k < (int)(sizeof(CoefLM) / sizeof(double2)); ++k) dst2[k] = src2[k];
        }
        couple<MC, TS>(ar, ai, m, s, cc, fr, fi, frm, frp, fim, fip, dxr, dxi, dyr, dyi, has_y, p, np, invp, ex,
                       ey, ez, bx, by, bz, a.g00_s, a.g00_inv, a.g00_gr);
        if (s == 1) {
            if (m == 0) jx += wj * (double)fr;
            else if (m == 1) { jyr += wj * (double)fr; jyi += wj * (double)fi; }
        }
    };

    // harmonics are consumed in pairs behind one wait, so the compiler can
    // interleave the two instruction streams
    int idx = 0;
    for (int s = 0; s <= a.l0; ++s) {
        const int mtop = min(s, a.m0);
#pragma unroll
        for (int mp = 0; mp <= MC; mp += 2) {
            if (mp > mtop) continue;
            const bool two = (mp + 1 <= MC) && (mp + 1 <= mtop);
            if (!dead && !mbar_wait(full + (idx % kDepth), (uint32_t)((idx / kDepth) & 1))) {
                atomicOr(a.err, 16);
                dead = true;
            }
            if (two && !dead && !mbar_wait(full + ((idx + 1) % kDepth), (uint32_t)(((idx + 1) / kDepth) & 1))) {
                atomicOr(a.err, 16);
                dead = true;
            }
            if (!dead) {
                consume(s, mp, idx);
                if (mp + 1 <= MC) {
                    if (two) consume(s, mp + 1, idx + 1);
                }
            }
            __syncwarp();
            if (lane == 0) {                          // this warp is done with the slot(s)
                mbar_arrive(empty + (idx % kDepth));
                if (two) mbar_arrive(empty + ((idx + 1) % kDepth));
            }
            idx += two ? 2 : 1;
        }
        if (s >= 1) epilogue(s - 1);
        rotate_rows<MC, TS>(ar, ai);
    }
    epilogue(a.l0);

    // per-cell current: warp sums, then warps in order (deterministic)
    const int warp_in_cell = p >> 5;
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        jx += __shfl_xor_sync(kFull, jx, off);
        jyr += __shfl_xor_sync(kFull, jyr, off);
        jyi += __shfl_xor_sync(kFull, jyi, off);
    }
    if (lane == 0) {
        sj[(0 * tx + c) * 8 + warp_in_cell] = jx;
        sj[(1 * tx + c) * 8 + warp_in_cell] = jyr;
        sj[(2 * tx + c) * 8 + warp_in_cell] = jyi;
    }
    consumer_sync(nct);
    if (p != 0 || !cv || dead) return;
    double Jx = 0.0, Jyr = 0.0, Jyi = 0.0;
    const int nw = np_pad >> 5;
    for (int w = 0; w < nw; ++w) {
        Jx += sj[(0 * tx + c) * 8 + w];
        Jyr += sj[(1 * tx + c) * 8 + w];
        Jyi += sj[(2 * tx + c) * 8 + w];
    }
    field_update(a, cell, cxm, cxp, cym, cyp, Jx, Jyr, Jyi);
}

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------
template <typename TS, int MC>
cudaError_t launch_mc(const StageArgs<TS>& a, cudaStream_t s) {
    const int np_pad = ((a.np + 31) / 32) * 32;
    // bulk copies move whole momentum rows: 16-byte multiples for every plane type
    const bool tma_ok = (a.np * (int)sizeof(TS)) % 16 == 0 && (a.np * 8) % 16 == 0 && np_pad <= kPChunk &&
                        a.seq != nullptr;
    if (tma_ok) {
        // consumer threads <= 192 keep the block at 7 warps (255 registers per thread)
        int tx = np_pad <= 192 ? 192 / np_pad : 1;
        if (tx > kMaxCellsPerCta) tx = kMaxCellsPerCta;
        if (tx > a.nx) tx = a.nx;
        const int ncoef = (a.l0 + 1) * (a.m0 + 1);
        const TmaLayout L = tma_layout(ncoef, a.nh, tx, a.np, a.ny > 1, (int)sizeof(TS), a.m0);
        if (L.total <= 227 * 1024) {
            const long long blocks = (long long)a.ny * ((a.nx + tx - 1) / tx);
            const int threads = np_pad * tx + 32;
            if (threads <= 224) {
                static size_t attr = 0;
                if (L.total > attr) {
                    cudaError_t e = cudaFuncSetAttribute(rk_stage_tma_kernel<MC, TS, 224>,
                                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L.total);
                    if (e != cudaSuccess) return e;
                    attr = L.total;
                }
                rk_stage_tma_kernel<MC, TS, 224><<<dim3((unsigned)blocks), dim3(threads), L.total, s>>>(a);
            } else {
                static size_t attr = 0;
                if (L.total > attr) {
                    cudaError_t e = cudaFuncSetAttribute(rk_stage_tma_kernel<MC, TS, 288>,
                                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L.total);
                    if (e != cudaSuccess) return e;
                    attr = L.total;
                }
                rk_stage_tma_kernel<MC, TS, 288><<<dim3((unsigned)blocks), dim3(threads), L.total, s>>>(a);
            }
            return cudaGetLastError();
        }
    }
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
