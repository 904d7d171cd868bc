// Pipelined RK4-stage kernel (nump <= 256, momentum rows of 16-byte
// multiples): Actions::Adv (OSHUN-1/def-Actions.cpp:73-94) on one stage input
// folded into the stage update of Runge_Kutta_4::advance_p1
// (OSHUN-1/def-RK.cpp:110-145).
//
// One resident CTA per SM walks tiles of `tx` consecutive cells of one y row
// (tiles blockIdx.x, blockIdx.x + gridDim.x, ...); one consumer thread owns
// one (cell, p) point of every harmonic of the tile and keeps register
// accumulators of the three target rows a source row reaches (l-1, l, l+1).
// Two producer warps feed shared memory with bulk async copies
// (cp.async.bulk, completion on mbarriers; every wait sleeps in
// mbarrier.try_wait and gives up after 1 s), running ahead across tile
// boundaries:
//   * the source warp streams each source harmonic's tile -- the cells, their
//     x neighbours and their y-1/y+1 segments, every momentum point -- into a
//     ring of kDepth slots, in (l, m) order;
//   * the row warp streams the RK epilogue operands (Y0 and Y of the target
//     row about to complete) into a double-buffered row stage.
// The consumers read every stencil operand from shared memory through
// per-thread offsets fixed at kernel start; the momentum-edge rules are
// folded into those offsets (the p+1 offset of the last point is the point
// itself, the p-1 offset of the first point is the point itself) and the
// G/H rules at p = 0 into zeroed field copies and one select, so the
// per-source code has no data-dependent branches.  Their only global
// accesses are the epilogue stores.
//
// Couplings of source (l, m) at one momentum point, with G/H as in
// MakeGH/G00 (OSHUN-1/def-VlasovMax.cpp:496-535) and the reference's Dp ends
// (OSHUN-1/def-State.cpp:359-380):
//   E (def-VlasovMax.cpp:346-491): Ex G -> (l+1,m), Ex H -> (l-1,m),
//     Em G -> (l+1,m+1), Em H -> (l-1,m+1), Ep H -> (l-1,m-1),
//     Ep G -> (l+1,m-1), real part only into m = 0;
//   B (def-VlasovMax.cpp:597-644): (Bz+iBy)/2 f -> (l,m+1), -i m Bx f -> (l,m),
//     (Bz-iBy) f -> (l,m-1);
//   advection (def-VlasovMax.cpp:834-951): x -> (l+-1,m), y -> (l+-1,m+-1);
//   current (def-VlasovMax.cpp:680-745) from f10, f11; Ampere/Faraday
//   (def-VlasovMax.cpp:979-1035); CLEAN_LOW_PC (def-Actions.cpp:240-253).
#include <type_traits>
#include <utility>

#include "stage_common.cuh"

namespace oshun {
namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr int kDepth = 10;                    // source slots in the ring
constexpr uint32_t kSuspendNs = 20000;         // sleep hint of one mbarrier try_wait
constexpr unsigned long long kWaitNs = 1000000000ull;   // a pipeline wait gives up after 1 s
constexpr int kMaxTx = 8;

template <typename T>
__device__ __forceinline__ T ldg(const T* p) { return __ldg(p); }

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
__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
__device__ __forceinline__ bool mbar_try(uint32_t addr, uint32_t parity) {
    uint32_t done;
    // the thread sleeps in the wait until the phase completes or kSuspendNs pass
    asm volatile(
        "{\n\t.reg .pred P1;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2, %3;\n\t"
        "selp.u32 %0, 1, 0, P1;\n\t}"
        : "=r"(done)
        : "r"(addr), "r"(parity), "r"(kSuspendNs)
        : "memory");
    return done != 0;
}
// bounded wait for the phase with this parity; false after kWaitNs
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
    const uint32_t addr = smem_u32(bar);
    if (mbar_try(addr, parity)) return true;
    const unsigned long long t0 = global_ns();
    for (;;) {
        if (mbar_try(addr, parity)) return true;
        if (global_ns() - t0 > kWaitNs) return false;
    }
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

// coupling table entry in the arithmetic type (CoefLM converted)
template <typename TS>
struct alignas(16) CoefT {
    TS ex_g, ex_h, em_g, em_h, ep_h, ep_g, ax_p, ax_m, ay_pp, ay_mp, ay_mm, ay_pm, b_m, gfac, invpax, hp0;
};

// shared-memory layout (host and device agree)
struct PipeLayout {
    size_t off_coef, off_plane, off_sj, off_slots, slot_bytes, off_rows, row_arr_bytes, total;
    int seg_cells;
};
// barriers at offset 0: full[kDepth], empty[kDepth], rowfull[2], rowempty[2]
__host__ __device__ inline PipeLayout pipe_layout(int ncoef, int tx, int np, bool has_y, int elem_bytes, int m0) {
    PipeLayout L;
    L.seg_cells = tx + 2 + (has_y ? 2 * tx : 0);
    L.off_coef = 256;
    L.off_plane = align_up(L.off_coef + (size_t)16 * elem_bytes * ncoef, 16);
    L.off_sj = align_up(L.off_plane + sizeof(int) * (size_t)ncoef, 16);
    L.off_slots = align_up(L.off_sj + sizeof(double) * 2 * 3 * (size_t)tx * 8, 128);
    // a slot holds one harmonic: Re and Im planes of the TS type, or the FP64 f00 plane
    const size_t plane_part = (size_t)2 * L.seg_cells * np * elem_bytes;
    const size_t f00_part = (size_t)L.seg_cells * np * 8;
    L.slot_bytes = align_up(plane_part > f00_part ? plane_part : f00_part, 128);
    L.off_rows = L.off_slots + kDepth * L.slot_bytes;
    const size_t row0 = (size_t)tx * np * 8;
    const size_t rowl = (size_t)(1 + 2 * m0) * tx * np * elem_bytes;
    L.row_arr_bytes = align_up(row0 > rowl ? row0 : rowl, 128);
    L.total = L.off_rows + 2 * 2 * L.row_arr_bytes;   // [buffer][B, A]
    return L;
}

// per-thread element offsets of the stencil operands inside a slot
struct Nb {
    int ctr, pm, pp, xm, xp, ym, yp;
};

// per-thread constants of the coupling arithmetic
template <typename TS>
struct Th {
    TS ex, ey, ez;          // E at the cell
    TS exg, eyg, ezg;       // E for the G terms: 0 at p = 0, where G = 0 for l >= 1
    TS bx, by, bz, hby, hbz;
    TS invp, vr;
    bool is0;               // p == 0: H = f[1] hp0
};

template <int N, typename F, int... I>
__device__ __forceinline__ void static_for_impl(F&& f, std::integer_sequence<int, I...>) {
    (f(std::integral_constant<int, I>{}), ...);
}
// f(integral_constant<int, 0>) ... f(integral_constant<int, N-1>)
template <int N, typename F>
__device__ __forceinline__ void static_for(F&& f) {
    static_for_impl<N>(f, std::make_integer_sequence<int, N>{});
}

// couplings of source (s, M), s >= 1, into target rows s-1 (R[0]), s (R[1]), s+1 (R[2])
template <int MC, int M, typename TS>
__device__ __forceinline__ void couple_src(TS (&R)[3][MC + 1], TS (&I)[3][MC + 1], const CoefT<TS>& c,
                                           const TS* __restrict__ sb, const int seg, const Nb& nb,
                                           const Th<TS>& th) {
    constexpr bool UP = M + 1 <= MC;
    constexpr bool DN = M >= 1;
    const TS ipx = th.invp * c.invpax;
    const TS fr = sb[nb.ctr], frm = sb[nb.pm], frp = sb[nb.pp];
    const TS dxr = (sb[nb.xm] - sb[nb.xp]) * th.vr;
    const TS dyr = (sb[nb.ym] - sb[nb.yp]) * th.vr;
    const TS dr = frm - frp;
    const TS Hnr = fr * ipx + dr;
    const TS Gr = dr * c.gfac + Hnr;
    const TS Hr = th.is0 ? frp * c.hp0 : Hnr;
    TS fi = 0, Gi = 0, Hi = 0, dxi = 0, dyi = 0;
    if constexpr (DN) {
        const TS* __restrict__ si = sb + seg;
        fi = si[nb.ctr];
        const TS fim = si[nb.pm], fip = si[nb.pp];
        dxi = (si[nb.xm] - si[nb.xp]) * th.vr;
        dyi = (si[nb.ym] - si[nb.yp]) * th.vr;
        const TS di = fim - fip;
        const TS Hni = fi * ipx + di;
        Gi = di * c.gfac + Hni;
        Hi = th.is0 ? fip * c.hp0 : Hni;
    }
    // Ex and x advection: (s+1, M), (s-1, M)
    {
        const TS cg = c.ex_g * th.exg, ch = c.ex_h * th.ex;
        R[2][M] += cg * Gr + c.ax_p * dxr;
        R[0][M] += ch * Hr + c.ax_m * dxr;
        if constexpr (DN) {
            I[2][M] += cg * Gi + c.ax_p * dxi;
            I[0][M] += ch * Hi + c.ax_m * dxi;
        }
    }
    if constexpr (UP) {
        // Em G -> (s+1, M+1), Em H -> (s-1, M+1), y advection, (Bz + iBy)/2 f -> (s, M+1)
        const TS gy = c.em_g * th.eyg, gz = c.em_g * th.ezg;
        const TS hy = c.em_h * th.ey, hz = c.em_h * th.ez;
        R[2][M + 1] += gy * Gr + gz * Gi + c.ay_pp * dyr;
        I[2][M + 1] += gy * Gi - gz * Gr + c.ay_pp * dyi;
        R[0][M + 1] += hy * Hr + hz * Hi + c.ay_mp * dyr;
        I[0][M + 1] += hy * Hi - hz * Hr + c.ay_mp * dyi;
        R[1][M + 1] += th.hbz * fr - th.hby * fi;
        I[1][M + 1] += th.hbz * fi + th.hby * fr;
    }
    if constexpr (DN) {
        // Ep H -> (s-1, M-1), Ep G -> (s+1, M-1), y advection, -i M Bx f -> (s, M),
        // (Bz - iBy) f -> (s, M-1); only real parts into m = 0
        const TS py = c.ep_h * th.ey, pz = c.ep_h * th.ez;
        const TS qy = c.ep_g * th.eyg, qz = c.ep_g * th.ezg;
        const TS cz = c.b_m * th.bz, cy = c.b_m * th.by;
        const TS mb = TS(M) * th.bx;
        R[0][M - 1] += py * Hr - pz * Hi + c.ay_mm * dyr;
        R[2][M - 1] += qy * Gr - qz * Gi + c.ay_pm * dyr;
        R[1][M - 1] += cz * fr + cy * fi;
        R[1][M] += mb * fi;
        I[1][M] -= mb * fr;
        if constexpr (M >= 2) {
            I[0][M - 1] += py * Hi + pz * Hr + c.ay_mm * dyi;
            I[2][M - 1] += qy * Gi + qz * Gr + c.ay_pm * dyi;
            I[1][M - 1] += cz * fi - cy * fr;
        }
    }
}

// couplings of the f00 source into row 1 (R[2]); G00 at p = 0 from the
// extrapolated f00(p=0) (OSHUN-1/def-VlasovMax.cpp:520-535)
template <int MC, typename TS>
__device__ __forceinline__ void couple_f00(TS (&R)[3][MC + 1], TS (&I)[3][MC + 1], const CoefT<TS>& c,
                                           const double* __restrict__ sb, const Nb& nb, const Th<TS>& th,
                                           const double g00_s, const double g00_inv, const double g00_gr) {
    const TS fr = (TS)sb[nb.ctr], frm = (TS)sb[nb.pm], frp = (TS)sb[nb.pp];
    const TS dxr = (TS)(sb[nb.xm] - sb[nb.xp]) * th.vr;
    const TS dyr = (TS)(sb[nb.ym] - sb[nb.yp]) * th.vr;
    TS Gr = frm - frp;
    if (th.is0) {
        const TS f00x = (fr - frp * (TS)g00_s) * (TS)g00_inv;
        Gr = (frp - f00x) * (TS)g00_gr;
    }
    const TS cg = c.ex_g * th.ex;
    R[2][0] += cg * Gr + c.ax_p * dxr;
    if constexpr (MC >= 1) {
        const TS gy = c.em_g * th.ey, gz = c.em_g * th.ez;
        R[2][1] += gy * Gr + c.ay_pp * dyr;
        I[2][1] -= gz * Gr;
    }
}

template <int MC, typename TS>
__device__ __forceinline__ void rotate(TS (&R)[3][MC + 1], TS (&I)[3][MC + 1]) {
#pragma unroll
    for (int m = 0; m <= MC; ++m) {
        R[0][m] = R[1][m]; I[0][m] = I[1][m];
        R[1][m] = R[2][m]; I[1][m] = I[2][m];
        R[2][m] = 0;       I[2][m] = 0;
    }
}

// field epilogue: J reduction result + Ampere/Faraday, RK update of 6 fields
template <typename TS>
__device__ __forceinline__ void field_update(const StageArgs<TS>& a, long long cell, long long cxm, long long cxp,
                                             long long cym, long long cyp, double Jx, double Jyr, double Jyi) {
    const TS* F = a.fld_in;
    const long long C = a.cells;
    const TS idx = (TS)a.idx, idy = (TS)a.idy;
    TS dEx = (TS)Jx;
    TS dEy = (TS)(2.0 * Jyr);
    TS dEz = (TS)(-(2.0 * Jyi));
    dEx += idy * (ldg(F + 5 * C + cym) - ldg(F + 5 * C + cyp));
    dEy += -idx * (ldg(F + 5 * C + cxm) - ldg(F + 5 * C + cxp));
    dEz += -idy * (ldg(F + 3 * C + cym) - ldg(F + 3 * C + cyp));
    dEz += idx * (ldg(F + 4 * C + cxm) - ldg(F + 4 * C + cxp));
    TS dBx = -idy * (ldg(F + 2 * C + cym) - ldg(F + 2 * C + cyp));
    TS dBy = idx * (ldg(F + 2 * C + cxm) - ldg(F + 2 * C + cxp));
    TS dBz = idy * (ldg(F + 0 * C + cym) - ldg(F + 0 * C + cyp));
    dBz += -idx * (ldg(F + 1 * C + cxm) - ldg(F + 1 * C + cxp));
    rk_update(a.mode, a.first, a.c1, a.c2, a.fld_out, a.fld_B, a.fld_A, 0 * C + cell, dEx);
    rk_update(a.mode, a.first, a.c1, a.c2, a.fld_out, a.fld_B, a.fld_A, 1 * C + cell, dEy);
    rk_update(a.mode, a.first, a.c1, a.c2, a.fld_out, a.fld_B, a.fld_A, 2 * C + cell, dEz);
    rk_update(a.mode, a.first, a.c1, a.c2, a.fld_out, a.fld_B, a.fld_A, 3 * C + cell, dBx);
    rk_update(a.mode, a.first, a.c1, a.c2, a.fld_out, a.fld_B, a.fld_A, 4 * C + cell, dBy);
    rk_update(a.mode, a.first, a.c1, a.c2, a.fld_out, a.fld_B, a.fld_A, 5 * C + cell, dBz);
}

// RK update of one target row's planes from its slopes and the staged Y0 (Bs)
// and Y (As); the stage form is decided once per row
template <int MC, typename TS>
__device__ __forceinline__ void store_row(const StageArgs<TS>& a, const int mtop, const bool zero,
                                          const TS (&R)[MC + 1], const TS (&I)[MC + 1], TS* __restrict__ out,
                                          TS* __restrict__ A, const TS* __restrict__ Bs, const TS* __restrict__ As,
                                          const int rstride) {
    const long long ps = a.pstride;
    auto k_of = [&](int m, int comp) -> TS { return zero ? TS(0) : (comp ? I[m] : R[m]); };
    if (a.mode == 1) {
        static_for<MC + 1>([&](auto mcst) {
            constexpr int m = decltype(mcst)::value;
            constexpr int kk = m == 0 ? 0 : 2 * m - 1;
            if (m > mtop) return;
            out[kk * ps] = k_of(m, 0);
            if constexpr (m > 0) out[(kk + 1) * ps] = k_of(m, 1);
        });
        return;
    }
    const TS c1 = (TS)a.c1, c2 = (TS)a.c2;
    const bool first = a.first, has_out = out != nullptr;
    static_for<MC + 1>([&](auto mcst) {
        constexpr int m = decltype(mcst)::value;
        constexpr int kk = m == 0 ? 0 : 2 * m - 1;
        if (m > mtop) return;
#pragma unroll
        for (int comp = 0; comp < (m > 0 ? 2 : 1); ++comp) {
            const int k = kk + comp;
            const TS t = k_of(m, comp) * c1;
            const TS b = Bs[k * rstride];
            if (has_out) out[k * ps] = b + t;
            A[k * ps] = (first ? b : As[k * rstride]) + t * c2;
        }
    });
}

template <int MC, typename TS, int MAXT>
__global__ void __launch_bounds__(MAXT, 1) rk_stage_pipe_kernel(const StageArgs<TS> a) {
    extern __shared__ __align__(128) unsigned char smem[];
    const int np = a.np, nx = a.nx, ny = a.ny;
    const int np_pad = (np + 31) & ~31;
    const bool has_y = ny > 1;
    const int tx = (int)(blockDim.x - 64) / np_pad;
    const int nct = np_pad * tx;                       // consumer threads
    const int ncw = nct >> 5;                          // consumer warps
    const int mstride = a.m0 + 1;
    const int ncoef = (a.l0 + 1) * mstride;
    const PipeLayout L = pipe_layout(ncoef, tx, np, has_y, (int)sizeof(TS), a.m0);
    uint64_t* full = reinterpret_cast<uint64_t*>(smem);
    uint64_t* empty = full + kDepth;
    uint64_t* rowfull = empty + kDepth;
    uint64_t* rowempty = rowfull + 2;
    CoefT<TS>* scoef = reinterpret_cast<CoefT<TS>*>(smem + L.off_coef);
    int* splane = reinterpret_cast<int*>(smem + L.off_plane);
    double* sj = reinterpret_cast<double*>(smem + L.off_sj);   // [2 tiles][3][tx][8 warps]
    unsigned char* slots = smem + L.off_slots;
    unsigned char* rows = smem + L.off_rows;
    const bool need_B = a.mode != 1;
    const bool need_A = a.mode != 1 && !a.first;

    const int tid = threadIdx.x;
    const int tiles_x = (nx + tx - 1) / tx;
    const int ntiles = tiles_x * ny;
    // persistent CTAs: tiles blockIdx.x, blockIdx.x + gridDim.x, ...

    // tables to shared memory (coefficients in the arithmetic type), barriers
    {
        const double* src = reinterpret_cast<const double*>(a.coef);
        TS* dst = reinterpret_cast<TS*>(scoef);
        const int nd = ncoef * 16;
        for (int i = tid; i < nd; i += blockDim.x) dst[i] = (TS)src[i];
        for (int i = tid; i < ncoef; i += blockDim.x) splane[i] = a.plane_of[i];
        if (tid == 0) {
            for (int k = 0; k < kDepth; ++k) { mbar_init(full + k, 1); mbar_init(empty + k, ncw); }
            for (int k = 0; k < 2; ++k) { mbar_init(rowfull + k, 1); mbar_init(rowempty + k, ncw); }
            asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        }
    }
    __syncthreads();

    // ---------------- producer warps ----------------------------------------
    if (tid >= nct) {
        if ((tid & 31) != 0) return;
        if (tid == nct) {
            // source warp: every harmonic of the stage input, (l, m) order, tile after tile
            int issued = 0;
            bool ok = true;
            for (int tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x) {
                const int y = tile / tiles_x;
                const int x0 = (tile - y * tiles_x) * tx;
                const int txv = min(tx, nx - x0);
                const long long row = (long long)y * nx;
                const long long rym = (long long)(y == 0 ? ny - 1 : y - 1) * nx;
                const long long ryp = (long long)(y == ny - 1 ? 0 : y + 1) * nx;
                const long long xm_cell = row + (x0 == 0 ? nx - 1 : x0 - 1);
                const long long xp_cell = row + ((x0 + txv) % nx);
                const uint32_t ncell = txv + 2 + (has_y ? 2 * txv : 0);
                for (int s = 0; s <= a.l0 && ok; ++s) {
                    for (int m = 0; m <= min(s, a.m0); ++m) {
                        const int slot = issued % kDepth, j = issued / kDepth;
                        if (j >= 1 && !mbar_wait(empty + slot, (uint32_t)((j - 1) & 1))) { ok = false; break; }
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
                        mbar_expect_tx(full + slot, ncomp * ncell * bpc);
                        for (int comp = 0; comp < ncomp; ++comp) {
                            unsigned char* cb = dst + (size_t)comp * L.seg_cells * bpc;
                            const unsigned char* pb = src + (size_t)comp * a.pstride * esz;
                            bulk_g2s(cb, pb + (size_t)xm_cell * bpc, bpc, full + slot);
                            bulk_g2s(cb + bpc, pb + (size_t)(row + x0) * bpc, txv * bpc, full + slot);
                            bulk_g2s(cb + (size_t)(txv + 1) * bpc, pb + (size_t)xp_cell * bpc, bpc, full + slot);
                            if (has_y) {
                                bulk_g2s(cb + (size_t)(tx + 2) * bpc, pb + (size_t)(rym + x0) * bpc, txv * bpc,
                                         full + slot);
                                bulk_g2s(cb + (size_t)(2 * tx + 2) * bpc, pb + (size_t)(ryp + x0) * bpc, txv * bpc,
                                         full + slot);
                            }
                        }
                        ++issued;
                    }
                }
            }
            if (!ok) {
                atomicOr(a.err, 16);
                // bounded drain of every copy that may still be in flight
                for (int idx = max(0, issued - kDepth); idx < issued; ++idx)
                    mbar_wait(full + (idx % kDepth), (uint32_t)((idx / kDepth) & 1));
            }
        } else if (tid == nct + 32 && need_B) {
            // row warp: Y0 (and Y) of each target row, up to two rows ahead of its epilogue
            int issued = 0;
            bool ok = true;
            for (int tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x) {
                const int y = tile / tiles_x;
                const int x0 = (tile - y * tiles_x) * tx;
                const int txv = min(tx, nx - x0);
                const long long base_cell = (long long)y * nx + x0;
                for (int t = 0; t <= a.l0; ++t) {
                    const int rb = issued & 1, k = issued >> 1;
                    if (k >= 1 && !mbar_wait(rowempty + rb, (uint32_t)((k - 1) & 1))) { ok = false; break; }
                    unsigned char* base = rows + (size_t)rb * 2 * L.row_arr_bytes;
                    const uint32_t nb = need_A ? 2 : 1;
                    if (t == 0) {
                        const uint32_t b = (uint32_t)txv * np * 8;
                        mbar_expect_tx(rowfull + rb, nb * b);
                        bulk_g2s(base, a.f00_B + base_cell * np, b, rowfull + rb);
                        if (need_A) bulk_g2s(base + L.row_arr_bytes, a.f00_A + base_cell * np, b, rowfull + rb);
                    } else {
                        const int np_row = 1 + 2 * min(t, a.m0);
                        const uint32_t b = (uint32_t)txv * np * sizeof(TS);
                        mbar_expect_tx(rowfull + rb, nb * np_row * b);
                        const long long q0 = splane[t * mstride];
                        for (int kk = 0; kk < np_row; ++kk) {
                            const long long off = (q0 + kk) * a.pstride + base_cell * np;
                            const size_t d = (size_t)kk * tx * np * sizeof(TS);
                            bulk_g2s(base + d, a.pl_B + off, b, rowfull + rb);
                            if (need_A) bulk_g2s(base + L.row_arr_bytes + d, a.pl_A + off, b, rowfull + rb);
                        }
                    }
                    ++issued;
                }
            }
            if (!ok) {
                atomicOr(a.err, 16);
                for (int t = max(0, issued - 2); t < issued; ++t)
                    mbar_wait(rowfull + (t & 1), (uint32_t)((t >> 1) & 1));
            }
        }
        return;
    }

    // ---------------- consumer warps ----------------------------------------
    const int c = tid / np_pad, p = tid - c * np_pad;
    const int lane = tid & 31;
    const bool pin = p < np;
    // invalid threads read a valid point (finite data) and store nothing
    const int pc = pin ? p : 0;
    const int seg = L.seg_cells * np;
    const int rstride = tx * np;            // plane stride inside a staged row
    const double wj_p = pin ? ldg(a.wj + p) : 0.0;
    const TS invp = (TS)ldg(a.inv_pr + pc);
    const TS vr = (TS)ldg(a.vr + pc);

    bool dead = false;   // a wait ran out: skip all further work and writes
    int slot = 0;
    uint32_t phase = 0;
    int rows_used = 0;
    int tile_iter = 0;

    auto acquire = [&]() {
        if (!dead && !mbar_wait(full + slot, phase)) {
            atomicOr(a.err, 16);
            dead = true;
        }
    };
    auto release = [&]() {
        __syncwarp();
        if (lane == 0) mbar_arrive(empty + slot);
        if (++slot == kDepth) { slot = 0; phase ^= 1u; }
    };

    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x, ++tile_iter) {
        const int y = tile / tiles_x;
        const int x0 = (tile - y * tiles_x) * tx;
        const int txv = min(tx, nx - x0);
        const bool cv = c < txv;
        const bool pv = cv && pin;
        const int cc = cv ? c : 0;
        const long long row = (long long)y * nx;
        const long long rym = (long long)(y == 0 ? ny - 1 : y - 1) * nx;
        const long long ryp = (long long)(y == ny - 1 ? 0 : y + 1) * nx;
        const int xc = x0 + cc;
        const long long cell = row + xc;

        Nb nb;
        nb.ctr = (1 + cc) * np + pc;
        nb.pm = nb.ctr - (pc > 0 ? 1 : 0);
        nb.pp = nb.ctr + (pc < np - 1 ? 1 : 0);
        nb.xm = cc * np + pc;
        nb.xp = (cc + 2) * np + pc;
        nb.ym = has_y ? (tx + 2 + cc) * np + pc : nb.ctr;
        nb.yp = has_y ? (2 * tx + 2 + cc) * np + pc : nb.ctr;
        const int roff = cc * np + pc;          // this point inside a staged row

        Th<TS> th;
        th.ex = ldg(a.fld_in + cell);
        th.ey = ldg(a.fld_in + a.cells + cell);
        th.ez = ldg(a.fld_in + 2 * a.cells + cell);
        th.bx = ldg(a.fld_in + 3 * a.cells + cell);
        th.by = ldg(a.fld_in + 4 * a.cells + cell);
        th.bz = ldg(a.fld_in + 5 * a.cells + cell);
        th.is0 = pc == 0;
        th.exg = th.is0 ? TS(0) : th.ex;
        th.eyg = th.is0 ? TS(0) : th.ey;
        th.ezg = th.is0 ? TS(0) : th.ez;
        th.hby = TS(0.5) * th.by;
        th.hbz = TS(0.5) * th.bz;
        th.invp = invp;
        th.vr = vr;
        const double wj = pv ? wj_p : 0.0;
        const long long o = cell * np + pc;

        TS R[3][MC + 1], I[3][MC + 1];
#pragma unroll
        for (int r = 0; r < 3; ++r)
#pragma unroll
            for (int m = 0; m <= MC; ++m) { R[r][m] = 0; I[r][m] = 0; }
        double jx = 0.0, jyr = 0.0, jyi = 0.0;

        // RK epilogue of target row t from the staged Y0/Y rows
        auto epilogue = [&](const int t) {
            const int rb = rows_used & 1;
            if (need_B && !dead && !mbar_wait(rowfull + rb, (uint32_t)((rows_used >> 1) & 1))) {
                atomicOr(a.err, 16);
                dead = true;
            }
            if (!dead && pv) {
                const unsigned char* base = rows + (size_t)rb * 2 * L.row_arr_bytes;
                if (t == 0) {
                    const double k = (double)R[0][0];
                    if (a.mode == 1) {
                        a.f00_out[o] = k;
                    } else {
                        const double tt = k * a.c1;
                        const double b = reinterpret_cast<const double*>(base)[roff];
                        if (a.f00_out) a.f00_out[o] = b + tt;
                        a.f00_A[o] = (a.first ? b : reinterpret_cast<const double*>(base + L.row_arr_bytes)[roff]) +
                                     tt * a.c2;
                    }
                } else {
                    const bool zero = p < (t >= 2 ? min(t - 1, 80) : 0);
                    const long long g0 = (long long)splane[t * mstride] * a.pstride + o;
                    store_row<MC, TS>(a, min(t, a.m0), zero, R[0], I[0], a.pl_out ? a.pl_out + g0 : nullptr,
                                      a.pl_A + g0, reinterpret_cast<const TS*>(base) + roff,
                                      reinterpret_cast<const TS*>(base + L.row_arr_bytes) + roff, rstride);
                }
            }
            __syncwarp();
            if (need_B && lane == 0) mbar_arrive(rowempty + rb);
            ++rows_used;
        };

        // source row 0: f00
        acquire();
        if (!dead) {
            const double* sb = reinterpret_cast<const double*>(slots + (size_t)slot * L.slot_bytes);
            couple_f00<MC, TS>(R, I, scoef[0], sb, nb, th, a.g00_s, a.g00_inv, a.g00_gr);
        }
        release();
        rotate<MC, TS>(R, I);

        for (int s = 1; s <= a.l0; ++s) {
            const CoefT<TS>* crow = scoef + s * mstride;
            const int mtop = min(s, a.m0);
            static_for<MC + 1>([&](auto mcst) {
                constexpr int m = decltype(mcst)::value;
                if (m > mtop) return;
                acquire();
                if (!dead) {
                    const TS* sb = reinterpret_cast<const TS*>(slots + (size_t)slot * L.slot_bytes);
                    couple_src<MC, m, TS>(R, I, crow[m], sb, seg, nb, th);
                    if constexpr (m <= 1) {
                        if (s == 1) {
                            if constexpr (m == 0) {
                                jx += wj * (double)sb[nb.ctr];
                            } else {
                                jyr += wj * (double)sb[nb.ctr];
                                jyi += wj * (double)sb[seg + nb.ctr];
                            }
                        }
                    }
                }
                release();
            });
            epilogue(s - 1);
            rotate<MC, TS>(R, I);
        }
        epilogue(a.l0);

        // per-cell current: warp sums, then warps in order (deterministic);
        // the partial sums of consecutive tiles alternate between two buffers
        double* sjt = sj + (size_t)(tile_iter & 1) * 3 * tx * 8;
        const int warp_in_cell = p >> 5;
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) {
            jx += __shfl_xor_sync(kFull, jx, off);
            jyr += __shfl_xor_sync(kFull, jyr, off);
            jyi += __shfl_xor_sync(kFull, jyi, off);
        }
        if (lane == 0) {
            sjt[(0 * tx + c) * 8 + warp_in_cell] = jx;
            sjt[(1 * tx + c) * 8 + warp_in_cell] = jyr;
            sjt[(2 * tx + c) * 8 + warp_in_cell] = jyi;
        }
        consumer_sync(nct);
        if (p == 0 && cv && !dead) {
            double Jx = 0.0, Jyr = 0.0, Jyi = 0.0;
            const int nw = np_pad >> 5;
            for (int w = 0; w < nw; ++w) {
                Jx += sjt[(0 * tx + c) * 8 + w];
                Jyr += sjt[(1 * tx + c) * 8 + w];
                Jyi += sjt[(2 * tx + c) * 8 + w];
            }
            const long long cxm = row + (xc == 0 ? nx - 1 : xc - 1);
            const long long cxp = row + (xc == nx - 1 ? 0 : xc + 1);
            field_update(a, cell, cxm, cxp, rym + xc, ryp + xc, Jx, Jyr, Jyi);
        }
        if (dead) break;
    }
}

int sm_count() {
    static int n[64] = {0};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 148;
    if (n[dev] == 0) {
        int v = 0;
        if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || v <= 0) v = 148;
        n[dev] = v;
    }
    return n[dev];
}

template <int MC, typename TS, int MAXT>
cudaError_t launch_pipe(const StageArgs<TS>& a, int tx, const PipeLayout& L, cudaStream_t s) {
    static size_t attr = 0;
    if (L.total > attr) {
        cudaError_t e = cudaFuncSetAttribute(rk_stage_pipe_kernel<MC, TS, MAXT>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L.total);
        if (e != cudaSuccess) return e;
        attr = L.total;
    }
    const int np_pad = ((a.np + 31) / 32) * 32;
    const long long tiles = (long long)a.ny * ((a.nx + tx - 1) / tx);
    // one resident CTA per SM, each walking tiles blockIdx.x + k gridDim.x
    const long long blocks = tiles < sm_count() ? tiles : sm_count();
    rk_stage_pipe_kernel<MC, TS, MAXT><<<dim3((unsigned)blocks), dim3(np_pad * tx + 64), L.total, s>>>(a);
    return cudaGetLastError();
}

template <typename TS, int MC>
cudaError_t pipe_mc(const StageArgs<TS>& a, cudaStream_t s) {
    const int np_pad = ((a.np + 31) / 32) * 32;
    // bulk copies move whole momentum rows: 16-byte multiples for every plane type
    if ((a.np * (int)sizeof(TS)) % 16 != 0 || np_pad > 256) return cudaErrorNotSupported;
    // consumer threads <= 192: 8 warps with the producers, 255 registers per thread
    int tx = np_pad <= 192 ? 192 / np_pad : 1;
    if (tx > kMaxTx) tx = kMaxTx;
    if (tx > a.nx) tx = a.nx;
    const int ncoef = (a.l0 + 1) * (a.m0 + 1);
    const PipeLayout L = pipe_layout(ncoef, tx, a.np, a.ny > 1, (int)sizeof(TS), a.m0);
    if (L.total > 227 * 1024) return cudaErrorNotSupported;
    if (np_pad * tx <= 192) return launch_pipe<MC, TS, 256>(a, tx, L, s);
    return launch_pipe<MC, TS, 320>(a, tx, L, s);
}

}  // namespace

// the pipelined stage for m0 <= MC; cudaErrorNotSupported when the shape
// does not fit it (the caller then uses the global-load kernel)
template <typename TS>
cudaError_t launch_stage_pipe(const StageArgs<TS>& a, int mc, cudaStream_t s) {
    if (a.seq == nullptr) return cudaErrorNotSupported;
    switch (mc) {
        case 0: return pipe_mc<TS, 0>(a, s);
        case 1: return pipe_mc<TS, 1>(a, s);
        case 2: return pipe_mc<TS, 2>(a, s);
        case 3: return pipe_mc<TS, 3>(a, s);
        case 4: return pipe_mc<TS, 4>(a, s);
        case 6: return pipe_mc<TS, 6>(a, s);
        case 8: return pipe_mc<TS, 8>(a, s);
        default: return cudaErrorNotSupported;
    }
}
template cudaError_t launch_stage_pipe<double>(const StageArgs<double>&, int, cudaStream_t);
template cudaError_t launch_stage_pipe<float>(const StageArgs<float>&, int, cudaStream_t);

}  // namespace oshun
