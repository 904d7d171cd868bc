// Pipelined RK4-stage kernel (nump <= 256, momentum rows of 16-byte
// multiples): Actions::Adv (OSHUN-1/def-Actions.cpp:73-94) on one stage input
// folded into the stage update of Runge_Kutta_4::advance_p1
// (OSHUN-1/def-RK.cpp:110-145).
//
// Two kernels share the helpers of this header: rk_stage_tile_kernel
// (stage_pipe.cu) for one problem, and rk_stage_pipe_kernel (below, launched
// from stage_batch.cu) for a batch of problems, whose tiles
// carry their problem's descriptor in the header of their first copy.
//
// One resident CTA per SM walks tiles of `tx` consecutive cells of one y row
// (tiles blockIdx.x, blockIdx.x + gridDim.x, ...); one consumer thread owns
// one (cell, p) point of every harmonic of the tile and keeps register
// accumulators of the three target rows a source row reaches (l-1, l, l+1).
// Two producer warps feed shared memory with bulk async copies
// (cp.async.bulk, completion on mbarriers; every wait polls
// mbarrier.test_wait and gives up after 1 s), running ahead across tile
// boundaries:
//   * the source warp streams each source harmonic's tile -- the cells, their
//     x neighbours and their y-1/y+1 segments, every momentum point -- into a
//     ring of source slots (up to kMaxDepth), in (l, m) order;
//   * the row warp streams the RK epilogue operands (Y0 and Y of the target
//     row about to complete) into a double-buffered row stage (and, in the
//     single-problem kernel, each tile's six field values with its row 0).
// The consumers read every stencil operand from shared memory through
// per-thread offsets fixed per tile; the momentum-edge rules are folded into
// those offsets (the p+1 offset of the last point is the point itself, the
// p-1 offset of the first point is the point itself) and the G/H rules at
// p = 0 into zeroed field copies and one select, so the per-source code has
// no data-dependent branches.  The consumer warps share no barrier: each
// writes its per-warp sums of the current to a per-cell array, and a field
// kernel (stage_fields_kernel / stage_fields_batch_kernel) adds them in warp
// order and updates E and B after the stage.
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
#pragma once

#include <type_traits>
#include <utility>

#include "stage_common.cuh"

namespace oshun {
namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr int kDepth = 10;                    // source slots in the ring (batched kernel; default)
constexpr int kMaxDepth = 12;                 // ring slots the barrier area holds
constexpr unsigned long long kWaitNs = 1000000000ull;   // a pipeline wait gives up after 1 s
constexpr int kMaxTx = 8;
constexpr size_t kSmemMax = 227 * 1024;          // dynamic shared memory of one CTA
constexpr size_t kSmemHalf = (228 * 1024 - 2 * 1024) / 2;   // each of two CTAs on one SM (1 KB reserved each)

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
    // a non-blocking test of the phase (the caller polls with a time bound);
    // it timed 0.7 % faster per stage than a try_wait that may suspend the thread
    asm volatile(
        "{\n\t.reg .pred P1;\n\t"
        "mbarrier.test_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, P1;\n\t}"
        : "=r"(done)
        : "r"(addr), "r"(parity)
        : "memory");
    return done != 0;
}
// bounded wait for the phase with this parity; false after limit_ns
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity,
                                          const unsigned long long limit_ns = kWaitNs) {
    const uint32_t addr = smem_u32(bar);
    if (mbar_try(addr, parity)) return true;
    const unsigned long long t0 = global_ns();
    for (;;) {
        if (mbar_try(addr, parity)) return true;
        if (global_ns() - t0 > limit_ns) return false;
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

__host__ __device__ inline size_t align_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

// coupling table entry in the arithmetic type (CoefLM converted)
template <typename TS>
struct alignas(16) CoefT {
    TS ex_g, ex_h, em_g, em_h, ep_h, ep_g, ax_p, ax_m, ay_pp, ay_mp, ay_mm, ay_pm, b_m, gfac, invpax, hp0;
};

// shared-memory layout (host and device agree)
struct PipeLayout {
    size_t off_coef, off_plane, off_fld, fld_stride, off_slots, slot_bytes, off_rows, row_arr_bytes, total;
    size_t rowl_arr_bytes, off_f00, f00_arr_bytes;   // single-problem kernel's row stage
    int seg_cells;
    int depth;   // slots in the source ring (<= kMaxDepth)
};
// barriers at offset 0: full[kMaxDepth], empty[kMaxDepth], rowfull[2], rowempty[2],
// f00full, f00empty
static_assert((2 * kMaxDepth + 6) * sizeof(uint64_t) <= 256, "barrier area");
__host__ __device__ inline PipeLayout pipe_layout(int ncoef, int tx, int np, bool has_y, int elem_bytes, int m0,
                                                 int depth = kDepth) {
    PipeLayout L;
    L.seg_cells = tx + 2 + (has_y ? 2 * tx : 0);
    L.off_coef = 256;
    L.off_plane = align_up(L.off_coef + (size_t)16 * elem_bytes * ncoef, 16);
    // fields of the tile's cells (single-problem kernel), [2 tiles][6 fields]:
    // each the 16-byte aligned span of memory holding the tile's values
    L.off_fld = align_up(L.off_plane + sizeof(int) * (size_t)ncoef, 16);
    L.fld_stride = align_up((size_t)tx * elem_bytes + 32, 16);
    L.off_slots = align_up(L.off_fld + 2 * 6 * L.fld_stride, 128);
    // a slot holds one harmonic: Re and Im planes of the TS type (Re alone
    // when m0 = 0: every source is real), or the FP64 f00 plane
    const size_t plane_part = (size_t)(m0 > 0 ? 2 : 1) * L.seg_cells * np * elem_bytes;
    const size_t f00_part = (size_t)L.seg_cells * np * 8;
    L.slot_bytes = align_up(plane_part > f00_part ? plane_part : f00_part, 128);
    L.depth = depth;
    L.off_rows = L.off_slots + (size_t)depth * L.slot_bytes;
    const size_t row0 = (size_t)tx * np * 8;
    const size_t rowl = (size_t)(1 + 2 * m0) * tx * np * elem_bytes;
    // batched kernel: every target row, f00 included, passes the double-buffered row stage
    L.row_arr_bytes = align_up(row0 > rowl ? row0 : rowl, 128);
    // single-problem kernel: rows l >= 1 pass the double-buffered stage
    // [buffer][B, A]; the f00 row (and the tile's fields) have their own
    // buffer [B, A], refilled for the next tile once row 0 is stored, so
    // they arrive a whole tile ahead instead of at the tile boundary
    L.rowl_arr_bytes = align_up(rowl, 128);
    L.f00_arr_bytes = align_up(row0, 128);
    L.off_f00 = L.off_rows + 2 * 2 * L.rowl_arr_bytes;
    L.total = L.off_f00 + 2 * L.f00_arr_bytes;
    return L;
}

// per-thread element offsets of the stencil operands inside a slot
struct Nb {
    int ctr, pm, pp, xm, xp, ym, yp;
    int p, p_m, p_p;   // momentum index of the point and of its p-1, p+1 operands (edge rules applied)
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

// Slope accumulators of one target row.  FP64: Re and Im arrays.  FP32:
// (Re, Im) pairs, which the paired FP32 FMA of sm_100 (__ffma2_rn) updates
// in one instruction; the Im half of m = 0 is carried along and never stored.
template <int MC>
struct AccD {
    double R[MC + 1], I[MC + 1];
};
template <int MC>
struct AccF {
    float2 V[MC + 1];
};
template <typename TS, int MC>
struct AccOf {
    using type = AccD<MC>;
};
template <int MC>
struct AccOf<float, MC> {
    using type = AccF<MC>;
};
template <typename TS, int MC>
using Acc = typename AccOf<TS, MC>::type;

template <int MC>
__device__ __forceinline__ double acc_re(const AccD<MC>& a, int m) { return a.R[m]; }
template <int MC>
__device__ __forceinline__ double acc_im(const AccD<MC>& a, int m) { return a.I[m]; }
template <int MC>
__device__ __forceinline__ float acc_re(const AccF<MC>& a, int m) { return a.V[m].x; }
template <int MC>
__device__ __forceinline__ float acc_im(const AccF<MC>& a, int m) { return a.V[m].y; }
template <int MC>
__device__ __forceinline__ void acc_zero(AccD<MC>& a) {
#pragma unroll
    for (int m = 0; m <= MC; ++m) { a.R[m] = 0.0; a.I[m] = 0.0; }
}
template <int MC>
__device__ __forceinline__ void acc_zero(AccF<MC>& a) {
#pragma unroll
    for (int m = 0; m <= MC; ++m) a.V[m] = make_float2(0.f, 0.f);
}

// couplings of source (s, M), s >= 1, into target rows s-1 (R0, I0), s (R1, I1), s+1 (R2, I2)
template <int MC, int M, typename TS>
__device__ __forceinline__ void couple_src3_ri(TS (&R0)[MC + 1], TS (&R1)[MC + 1], TS (&R2)[MC + 1],
                                            TS (&I0)[MC + 1], TS (&I1)[MC + 1], TS (&I2)[MC + 1],
                                            const CoefT<TS>& c, const TS* __restrict__ sb, const int seg,
                                            const Nb& nb, const Th<TS>& th) {
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
        R2[M] += cg * Gr + c.ax_p * dxr;
        R0[M] += ch * Hr + c.ax_m * dxr;
        if constexpr (DN) {
            I2[M] += cg * Gi + c.ax_p * dxi;
            I0[M] += ch * Hi + c.ax_m * dxi;
        }
    }
    if constexpr (UP) {
        // Em G -> (s+1, M+1), Em H -> (s-1, M+1), y advection, (Bz + iBy)/2 f -> (s, M+1)
        const TS gy = c.em_g * th.eyg, gz = c.em_g * th.ezg;
        const TS hy = c.em_h * th.ey, hz = c.em_h * th.ez;
        if constexpr (DN) {
            R2[M + 1] += gy * Gr + gz * Gi + c.ay_pp * dyr;
            I2[M + 1] += gy * Gi - gz * Gr + c.ay_pp * dyi;
            R0[M + 1] += hy * Hr + hz * Hi + c.ay_mp * dyr;
            I0[M + 1] += hy * Hi - hz * Hr + c.ay_mp * dyi;
            R1[M + 1] += th.hbz * fr - th.hby * fi;
            I1[M + 1] += th.hbz * fi + th.hby * fr;
        } else {
            // an m = 0 source is real: its imaginary terms are zero
            R2[M + 1] += gy * Gr + c.ay_pp * dyr;
            I2[M + 1] -= gz * Gr;
            R0[M + 1] += hy * Hr + c.ay_mp * dyr;
            I0[M + 1] -= hz * Hr;
            R1[M + 1] += th.hbz * fr;
            I1[M + 1] += th.hby * fr;
        }
    }
    if constexpr (DN) {
        // Ep H -> (s-1, M-1), Ep G -> (s+1, M-1), y advection, -i M Bx f -> (s, M),
        // (Bz - iBy) f -> (s, M-1); only real parts into m = 0
        const TS py = c.ep_h * th.ey, pz = c.ep_h * th.ez;
        const TS qy = c.ep_g * th.eyg, qz = c.ep_g * th.ezg;
        const TS cz = c.b_m * th.bz, cy = c.b_m * th.by;
        const TS mb = TS(M) * th.bx;
        R0[M - 1] += py * Hr - pz * Hi + c.ay_mm * dyr;
        R2[M - 1] += qy * Gr - qz * Gi + c.ay_pm * dyr;
        R1[M - 1] += cz * fr + cy * fi;
        R1[M] += mb * fi;
        I1[M] -= mb * fr;
        if constexpr (M >= 2) {
            I0[M - 1] += py * Hi + pz * Hr + c.ay_mm * dyi;
            I2[M - 1] += qy * Gi + qz * Gr + c.ay_pm * dyi;
            I1[M - 1] += cz * fi - cy * fr;
        }
    }
}

// couplings of the f00 source into row 1 (R2, I2); G00 at p = 0 from the
// extrapolated f00(p=0) (OSHUN-1/def-VlasovMax.cpp:520-535)
template <int MC, typename TS>
__device__ __forceinline__ void couple_f00_row(TS (&R2)[MC + 1], TS (&I2)[MC + 1], const CoefT<TS>& c,
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
    R2[0] += cg * Gr + c.ax_p * dxr;
    if constexpr (MC >= 1) {
        const TS gy = c.em_g * th.ey, gz = c.em_g * th.ez;
        R2[1] += gy * Gr + c.ay_pp * dyr;
        I2[1] -= gz * Gr;
    }
}

// the couplings on the accumulator types: FP64 through the Re/Im arrays
template <int MC, int M>
__device__ __forceinline__ void couple_src3(AccD<MC>& A0, AccD<MC>& A1, AccD<MC>& A2, const CoefT<double>& c,
                                            const double* __restrict__ sb, const int seg, const Nb& nb,
                                            const Th<double>& th, const double* /*ref: FP64 planes hold f*/,
                                            const int /*np*/) {
    couple_src3_ri<MC, M, double>(A0.R, A1.R, A2.R, A0.I, A1.I, A2.I, c, sb, seg, nb, th);
}
template <int MC>
__device__ __forceinline__ void couple_f00(AccD<MC>& A2, const CoefT<double>& c, const double* __restrict__ sb,
                                           const Nb& nb, const Th<double>& th, const double g00_s,
                                           const double g00_inv, const double g00_gr) {
    couple_f00_row<MC, double>(A2.R, A2.I, c, sb, nb, th, g00_s, g00_inv, g00_gr);
}

__device__ __forceinline__ float2 bc2(float v) { return make_float2(v, v); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }

// FP32: the same couplings on (Re, Im) pairs.  With F = (fr, fi) and
// F' = (fi, -fr), a complex coupling (a + i b) F adds a F + b F'; the
// m = 0 sources (M = 0) carry Im = 0.
// The planes hold f - ref (ref: the plane's momentum profile, null for
// none): the x and y differences act on the stored deviation alone, the
// momentum stencil and the value itself on f = ref + deviation.
template <int MC, int M>
__device__ __forceinline__ void couple_src3(AccF<MC>& A0, AccF<MC>& A1, AccF<MC>& A2, const CoefT<float>& c,
                                            const float* __restrict__ sb, const int seg, const Nb& nb,
                                            const Th<float>& th, const float* __restrict__ ref, const int np) {
    constexpr bool UP = M + 1 <= MC;
    constexpr bool DN = M >= 1;
    const float2 m1 = bc2(-1.f);
    const float2 vr = bc2(th.vr);
    float2 f, fm, fp, xm, xp, ym, yp;
    f.x = sb[nb.ctr]; fm.x = sb[nb.pm]; fp.x = sb[nb.pp];
    xm.x = sb[nb.xm]; xp.x = sb[nb.xp]; ym.x = sb[nb.ym]; yp.x = sb[nb.yp];
    if constexpr (DN) {
        const float* __restrict__ si = sb + seg;
        f.y = si[nb.ctr]; fm.y = si[nb.pm]; fp.y = si[nb.pp];
        xm.y = si[nb.xm]; xp.y = si[nb.xp]; ym.y = si[nb.ym]; yp.y = si[nb.yp];
    } else {
        f.y = 0.f; fm.y = 0.f; fp.y = 0.f; xm.y = 0.f; xp.y = 0.f; ym.y = 0.f; yp.y = 0.f;
    }
    if (ref) {
        f.x += __ldg(ref + nb.p); fm.x += __ldg(ref + nb.p_m); fp.x += __ldg(ref + nb.p_p);
        if constexpr (DN) {
            f.y += __ldg(ref + np + nb.p); fm.y += __ldg(ref + np + nb.p_m); fp.y += __ldg(ref + np + nb.p_p);
        }
    }
    const float2 dx = __fmul2_rn(fma2(xp, m1, xm), vr);   // (f(x-1) - f(x+1)) v
    const float2 dy = __fmul2_rn(fma2(yp, m1, ym), vr);
    const float2 d = fma2(fp, m1, fm);                    // f(p-1) - f(p+1)
    const float2 Hn = fma2(f, bc2(th.invp * c.invpax), d);
    const float2 G = fma2(d, bc2(c.gfac), Hn);
    const float2 H = th.is0 ? __fmul2_rn(fp, bc2(c.hp0)) : Hn;
    // Ex and x advection: (s+1, M), (s-1, M)
    A2.V[M] = fma2(bc2(c.ex_g * th.exg), G, fma2(bc2(c.ax_p), dx, A2.V[M]));
    A0.V[M] = fma2(bc2(c.ex_h * th.ex), H, fma2(bc2(c.ax_m), dx, A0.V[M]));
    if constexpr (UP || DN) {
        const float2 Gs = make_float2(G.y, -G.x), Hs = make_float2(H.y, -H.x), Fs = make_float2(f.y, -f.x);
        if constexpr (UP) {
            // Em G -> (s+1, M+1), Em H -> (s-1, M+1), y advection, (Bz + iBy)/2 f -> (s, M+1)
            A2.V[M + 1] = fma2(bc2(c.em_g * th.eyg), G,
                               fma2(bc2(c.em_g * th.ezg), Gs, fma2(bc2(c.ay_pp), dy, A2.V[M + 1])));
            A0.V[M + 1] = fma2(bc2(c.em_h * th.ey), H,
                               fma2(bc2(c.em_h * th.ez), Hs, fma2(bc2(c.ay_mp), dy, A0.V[M + 1])));
            A1.V[M + 1] = fma2(bc2(th.hbz), f, fma2(bc2(-th.hby), Fs, A1.V[M + 1]));
        }
        if constexpr (DN) {
            // Ep H -> (s-1, M-1), Ep G -> (s+1, M-1), y advection, (Bz - iBy) f -> (s, M-1),
            // -i M Bx f -> (s, M); the Im halves of m = 0 targets are never stored
            A0.V[M - 1] = fma2(bc2(c.ep_h * th.ey), H,
                               fma2(bc2(-(c.ep_h * th.ez)), Hs, fma2(bc2(c.ay_mm), dy, A0.V[M - 1])));
            A2.V[M - 1] = fma2(bc2(c.ep_g * th.eyg), G,
                               fma2(bc2(-(c.ep_g * th.ezg)), Gs, fma2(bc2(c.ay_pm), dy, A2.V[M - 1])));
            A1.V[M - 1] = fma2(bc2(c.b_m * th.bz), f, fma2(bc2(c.b_m * th.by), Fs, A1.V[M - 1]));
            A1.V[M] = fma2(bc2(float(M) * th.bx), Fs, A1.V[M]);
        }
    }
}
template <int MC>
__device__ __forceinline__ void couple_f00(AccF<MC>& A2, const CoefT<float>& c, const double* __restrict__ sb,
                                           const Nb& nb, const Th<float>& th, const double g00_s,
                                           const double g00_inv, const double g00_gr) {
    float R2[MC + 1], I2[MC + 1];
#pragma unroll
    for (int m = 0; m <= MC; ++m) { R2[m] = A2.V[m].x; I2[m] = A2.V[m].y; }
    couple_f00_row<MC, float>(R2, I2, c, sb, nb, th, g00_s, g00_inv, g00_gr);
#pragma unroll
    for (int m = 0; m <= MC; ++m) A2.V[m] = make_float2(R2[m], I2[m]);
}

// field epilogue: J reduction result + Ampere/Faraday, RK update of 6 fields
// hside: bit 0 the x-1 neighbour, bit 1 the x+1 neighbour comes from the
// x halo columns (row y)
template <typename TS>
__device__ __forceinline__ void field_update(const StageArgs<TS>& a, long long cell, long long cxm, long long cxp,
                                             long long cym, long long cyp, double Jx, double Jyr, double Jyi,
                                             int hside = 0, long long y = 0) {
    const TS* F = a.fld_in;
    const long long C = a.cells;
    const TS idx = (TS)a.idx, idy = (TS)a.idy;
    auto xm = [&](int k) { return (hside & 1) ? hx_field(a, 0, k, y) : ldg(F + k * C + cxm); };
    auto xp = [&](int k) { return (hside & 2) ? hx_field(a, 1, k, y) : ldg(F + k * C + cxp); };
    const TS dEx = fma_rn(idy, ldg(F + 5 * C + cym) - ldg(F + 5 * C + cyp), (TS)Jx);
    const TS dEy = fma_rn(-idx, xm(5) - xp(5), (TS)(2.0 * Jyr));
    const TS dEz = fma_rn(idx, xm(4) - xp(4),
                          fma_rn(-idy, ldg(F + 3 * C + cym) - ldg(F + 3 * C + cyp), (TS)(-(2.0 * Jyi))));
    const TS dBx = mul_rn(-idy, ldg(F + 2 * C + cym) - ldg(F + 2 * C + cyp));
    const TS dBy = mul_rn(idx, xm(2) - xp(2));
    const TS dBz = fma_rn(-idx, xm(1) - xp(1), mul_rn(idy, ldg(F + 0 * C + cym) - ldg(F + 0 * C + cyp)));
    rk_update(a.mode, a.first, a.c1, a.c2, a.fld_out, a.fld_B, a.fld_A, 0 * C + cell, dEx);
    rk_update(a.mode, a.first, a.c1, a.c2, a.fld_out, a.fld_B, a.fld_A, 1 * C + cell, dEy);
    rk_update(a.mode, a.first, a.c1, a.c2, a.fld_out, a.fld_B, a.fld_A, 2 * C + cell, dEz);
    rk_update(a.mode, a.first, a.c1, a.c2, a.fld_out, a.fld_B, a.fld_A, 3 * C + cell, dBx);
    rk_update(a.mode, a.first, a.c1, a.c2, a.fld_out, a.fld_B, a.fld_A, 4 * C + cell, dBy);
    rk_update(a.mode, a.first, a.c1, a.c2, a.fld_out, a.fld_B, a.fld_A, 5 * C + cell, dBz);
}

// E and B of one cell from the per-warp current partial sums of the stage
// kernel: the warps of the cell in order (deterministic), then field_update
template <typename TS>
__device__ __forceinline__ void fields_cell(const StageArgs<TS>& a, const long long cell, const int nw) {
    const int nx = a.nx, ny = a.ny;
    const int y = (int)(cell / nx), xc = (int)(cell - (long long)y * nx);
    const long long row = (long long)y * nx;
    const long long rym = (long long)(y == 0 ? ny - 1 : y - 1) * nx;
    const long long ryp = (long long)(y == ny - 1 ? 0 : y + 1) * nx;
    const double* jc = a.jw + cell * 24;
    double Jx = 0.0, Jyr = 0.0, Jyi = 0.0;
    for (int w = 0; w < nw; ++w) {
        Jx += jc[w];
        Jyr += jc[8 + w];
        Jyi += jc[16 + w];
    }
    const long long cxm = row + (xc == 0 ? nx - 1 : xc - 1);
    const long long cxp = row + (xc == nx - 1 ? 0 : xc + 1);
    const int hside = a.hx ? ((xc == 0 ? 1 : 0) | (xc == nx - 1 ? 2 : 0)) : 0;
    field_update(a, cell, cxm, cxp, rym + xc, ryp + xc, Jx, Jyr, Jyi, hside, y);
}

// the field step of every problem of a batch: one CTA per problem
template <typename TS>
__global__ void __launch_bounds__(128) stage_fields_batch_kernel(const unsigned char* __restrict__ probs,
                                                                 const int desc_bytes) {
    const StageArgs<TS>& a = *reinterpret_cast<const StageArgs<TS>*>(probs + (size_t)blockIdx.x * desc_bytes);
    const int nw = (a.np + 31) >> 5;
    for (long long cell = threadIdx.x; cell < a.cells; cell += blockDim.x) fields_cell(a, cell, nw);
}

// RK update of one target row's planes from its slopes and the staged Y0 (Bs)
// and Y (As); the stage form is decided once per row
template <int MC, typename TS>
__device__ __forceinline__ void store_row(const StageArgs<TS>& a, const int mtop, const bool zero,
                                          const Acc<TS, MC>& K, TS* __restrict__ out,
                                          TS* __restrict__ A, const TS* __restrict__ Bs, const TS* __restrict__ As,
                                          const int rstride) {
    const long long ps = a.pstride;
    auto k_of = [&](int m, int comp) -> TS { return zero ? TS(0) : (comp ? acc_im(K, m) : acc_re(K, m)); };
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
            const TS t = mul_rn(k_of(m, comp), c1);
            const TS b = Bs[k * rstride];
            if (has_out) out[k * ps] = add_rn(b, t);
            A[k * ps] = fma_rn(t, c2, first ? b : As[k * rstride]);
        }
    });
}

__host__ __device__ inline int tile_cells(int np, int nx, int nc, int tx_cap) {
    const int np_pad = (np + 31) & ~31;
    int tx = nc / np_pad;
    if (tx > tx_cap) tx = tx_cap;
    if (tx > nx) tx = nx;
    return tx < 1 ? 1 : tx;
}

// shared-memory plan of one launch (host and device agree)
struct SmemPlan {
    size_t off_cur, off_coef, off_plane, off_slots, slot_stride, hdr, off_rows, row_arr_bytes, total;
};
// barriers at offset 0: full[kDepth], empty[kDepth], rowfull[kRowMax], rowempty[kRowMax]
constexpr int kRowMax = 8;
constexpr int kMaxConsumerWarps = 10;   // batched launches: at most 320 consumer threads
template <typename TS>
__host__ __device__ inline SmemPlan smem_plan(bool batch, int hdr_bytes, int ncoef, size_t slot_bytes,
                                              size_t row_arr_bytes, int row_depth = 2) {
    SmemPlan P;
    P.hdr = batch ? (size_t)hdr_bytes : 0;
    P.off_cur = 512;                                   // batch: each consumer warp's copy of its item's header
    P.off_coef = P.off_cur + kMaxConsumerWarps * P.hdr;   // single problem: coupling table, plane map
    P.off_plane = align_up(P.off_coef + (batch ? 0 : sizeof(CoefT<TS>) * (size_t)ncoef), 16);
    P.off_slots = align_up(P.off_plane + (batch ? 0 : sizeof(int) * (size_t)ncoef), 128);
    P.slot_stride = align_up(P.hdr + slot_bytes, 128);
    P.off_rows = P.off_slots + kDepth * P.slot_stride;
    P.row_arr_bytes = row_arr_bytes;
    P.total = P.off_rows + (size_t)row_depth * 2 * row_arr_bytes;   // [buffer][B, A]
    return P;
}

// resident CTAs per SM the batched kernel is compiled for: two when the
// accumulators are few (m0 <= 1, the 1D batches) and the CTA has at most
// 10 warps, so that one CTA's tile start and end latencies overlap the
// other's work (two 12-warp CTAs would leave 80 registers a thread)
template <int MC, int MAXT>
constexpr int batch_min_blocks() { return (MC <= 1 && MAXT <= 320) ? 2 : 1; }

// a1: the launch's kernel parameter (its error word receives pipeline
// timeouts); every item's own descriptor arrives with its first slot
template <int MC, typename TS, int MAXT>
__global__ void __launch_bounds__(MAXT, batch_min_blocks<MC, MAXT>())
    rk_stage_pipe_kernel(const StageArgs<TS> a1, const BatchWork bw) {
    extern __shared__ __align__(128) unsigned char smem[];
    const int tid = threadIdx.x;
    const int nc = (int)blockDim.x - 64;               // consumer threads
    const int ncw = nc >> 5;                           // consumer warps
    const SmemPlan P = smem_plan<TS>(true, bw.hdr_bytes, 0, bw.slot_bytes, bw.row_arr_bytes, bw.row_depth);
    const int nitems = bw.nitems;
    uint64_t* full = reinterpret_cast<uint64_t*>(smem);
    uint64_t* empty = full + kDepth;
    uint64_t* rowfull = empty + kDepth;
    uint64_t* rowempty = rowfull + kRowMax;
    // staged-row ring depth: a batch of few harmonics per row needs rows further ahead
    const int RD = bw.row_depth;
    unsigned char* slots = smem + P.off_slots;
    unsigned char* rows = smem + P.off_rows;

    // barriers
    if (tid == 0) {
        for (int k = 0; k < kDepth; ++k) { mbar_init(full + k, 1); mbar_init(empty + k, ncw); }
        for (int k = 0; k < RD; ++k) { mbar_init(rowfull + k, 1); mbar_init(rowempty + k, ncw); }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();

    auto item_pid = [&](int it) -> int { return bw.items[it].x; };
    auto item_tile = [&](int it) -> int { return bw.items[it].y; };
    auto load_desc = [&](int pid) -> StageArgs<TS> {
        return *reinterpret_cast<const StageArgs<TS>*>(bw.probs + (size_t)pid * bw.desc_bytes);
    };

    // ---------------- producer warps ----------------------------------------
    if (tid >= nc) {
        if ((tid & 31) != 0) return;
        const bool src_warp = tid == nc;
        if (!src_warp && a1.mode == 1) return;   // the slope-only form reads no Y0/Y rows
        int issued = 0;
        bool ok = true;
        int it = blockIdx.x;
        StageArgs<TS> an;
        if (it < nitems) an = load_desc(item_pid(it));
        for (; it < nitems && ok; it += gridDim.x) {
            const StageArgs<TS> a = an;
            const int pid = item_pid(it), tile = item_tile(it);
            if (it + (int)gridDim.x < nitems) an = load_desc(item_pid(it + gridDim.x));   // next item, early
            const int np = a.np, nx = a.nx, ny = a.ny;
            const bool has_y = ny > 1;
            const int mstride = a.m0 + 1;
            const int tx = tile_cells(np, nx, nc, bw.tx_cap);
            const int tiles_x = (nx + tx - 1) / tx;
            const int y = tile / tiles_x;
            const int x0 = (tile - y * tiles_x) * tx;
            const int txv = min(tx, nx - x0);
            const long long row = (long long)y * nx;
            const int seg_cells = tx + 2 + (has_y ? 2 * tx : 0);
            if (src_warp) {
                // every harmonic of the stage input, (l, m) order
                const long long rym = (long long)(y == 0 ? ny - 1 : y - 1) * nx;
                const long long ryp = (long long)(y == ny - 1 ? 0 : y + 1) * nx;
                const long long xm_cell = row + (x0 == 0 ? nx - 1 : x0 - 1);
                const long long xp_cell = row + ((x0 + txv) % nx);
                // the x-stencil segment is one contiguous run unless it wraps
                const bool x_contig = x0 > 0 && x0 + txv < nx;
                const uint32_t ncell = txv + 2 + (has_y ? 2 * txv : 0);
                bool first = true;
                // planes are stored in (l, m) order, Re then Im: the stream's running count is the plane
                long long q = 0;
                for (int s = 0; s <= a.l0 && ok; ++s) {
                    for (int m = 0; m <= min(s, a.m0); ++m) {
                        const int slot = issued % kDepth, j = issued / kDepth;
                        if (j >= 1 && !mbar_wait(empty + slot, (uint32_t)((j - 1) & 1))) { ok = false; break; }
                        unsigned char* sbase = slots + (size_t)slot * P.slot_stride;
                        unsigned char* dst = sbase + P.hdr;
                        const unsigned char* src;
                        int esz, ncomp;
                        if (s == 0) {
                            src = reinterpret_cast<const unsigned char*>(a.f00_in);
                            esz = 8; ncomp = 1;
                        } else {
                            src = reinterpret_cast<const unsigned char*>(a.pl_in + q * a.pstride);
                            esz = (int)sizeof(TS); ncomp = m > 0 ? 2 : 1;
                            q += ncomp;
                        }
                        const uint32_t bpc = (uint32_t)np * esz;   // bytes per cell
                        uint32_t bytes = ncomp * ncell * bpc;
                        if (first) bytes += (uint32_t)bw.desc_bytes;
                        mbar_expect_tx(full + slot, bytes);
                        if (first)
                            bulk_g2s(sbase, bw.probs + (size_t)pid * bw.desc_bytes, (uint32_t)bw.desc_bytes,
                                     full + slot);
                        first = false;
                        for (int comp = 0; comp < ncomp; ++comp) {
                            unsigned char* cb = dst + (size_t)comp * seg_cells * bpc;
                            const unsigned char* pb = src + (size_t)comp * a.pstride * esz;
                            if (x_contig) {
                                bulk_g2s(cb, pb + (size_t)xm_cell * bpc, (txv + 2) * bpc, full + slot);
                            } else {
                                bulk_g2s(cb, pb + (size_t)xm_cell * bpc, bpc, full + slot);
                                bulk_g2s(cb + bpc, pb + (size_t)(row + x0) * bpc, txv * bpc, full + slot);
                                bulk_g2s(cb + (size_t)(txv + 1) * bpc, pb + (size_t)xp_cell * bpc, bpc, full + slot);
                            }
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
            } else {
                // row warp: Y0 (and Y) of each target row, up to RD rows ahead of its epilogue
                const bool need_A = !a.first;
                // Y0 enters only through the stage output and the first stage's Y
                const bool need_Y0 = a.first || a.f00_out != nullptr;
                const long long base_cell = row + x0;
                long long q0 = 0;   // first plane of row t (planes in (l, m) order)
                for (int t = 0; t <= a.l0; ++t) {
                    const int rb = issued % RD, k = issued / RD;
                    if (k >= 1 && !mbar_wait(rowempty + rb, (uint32_t)((k - 1) & 1))) { ok = false; break; }
                    unsigned char* base = rows + (size_t)rb * 2 * P.row_arr_bytes;
                    const uint32_t nb = (need_Y0 ? 1 : 0) + (need_A ? 1 : 0);
                    if (t == 0) {
                        const uint32_t b = (uint32_t)txv * np * 8;
                        mbar_expect_tx(rowfull + rb, nb * b);
                        if (need_Y0) bulk_g2s(base, a.f00_B + base_cell * np, b, rowfull + rb);
                        if (need_A) bulk_g2s(base + P.row_arr_bytes, a.f00_A + base_cell * np, b, rowfull + rb);
                    } else {
                        const int np_row = 1 + 2 * min(t, a.m0);
                        const uint32_t b = (uint32_t)txv * np * sizeof(TS);
                        mbar_expect_tx(rowfull + rb, nb * np_row * b);
                        for (int kk = 0; kk < np_row; ++kk) {
                            const long long off = (q0 + kk) * a.pstride + base_cell * np;
                            const size_t d = (size_t)kk * tx * np * sizeof(TS);
                            if (need_Y0) bulk_g2s(base + d, a.pl_B + off, b, rowfull + rb);
                            if (need_A) bulk_g2s(base + P.row_arr_bytes + d, a.pl_A + off, b, rowfull + rb);
                        }
                        q0 += np_row;
                    }
                    ++issued;
                }
            }
        }
        if (!ok) {
            atomicOr(a1.err, 16);
            // bounded drain of every copy that may still be in flight
            if (src_warp) {
                for (int idx = max(0, issued - kDepth); idx < issued; ++idx)
                    mbar_wait(full + (idx % kDepth), (uint32_t)((idx / kDepth) & 1));
            } else {
                for (int t = max(0, issued - RD); t < issued; ++t)
                    mbar_wait(rowfull + (t % RD), (uint32_t)((t / RD) & 1));
            }
        }
        return;
    }

    // ---------------- consumer warps ----------------------------------------
    const int lane = tid & 31;
    bool dead = false;   // a wait ran out: skip all further work and writes
    int slot = 0;
    uint32_t phase = 0;
    int rows_used = 0;
    int* err = a1.err;

    auto acquire = [&]() {
        if (!dead && !mbar_wait(full + slot, phase)) {
            atomicOr(err, 16);
            dead = true;
        }
    };
    auto release = [&]() {
        __syncwarp();
        if (lane == 0) mbar_arrive(empty + slot);
        if (++slot == kDepth) { slot = 0; phase ^= 1u; }
    };

    // one item: its tile of its problem (a = the kernel parameter for a
    // single problem, so that every field read stays a parameter read)
    auto item = [&](const StageArgs<TS>& a, const CoefT<TS>* scoef, const int* splane, const int tile) {
        const int np = a.np, nx = a.nx, ny = a.ny;
        const int np_pad = (np + 31) & ~31;
        const bool has_y = ny > 1;
        const int mstride = a.m0 + 1;
        const bool need_B = a.mode != 1;
        const bool need_A = a.mode != 1 && !a.first;
        const int tx = tile_cells(np, nx, nc, bw.tx_cap);
        const int seg_cells = tx + 2 + (has_y ? 2 * tx : 0);
        const int tiles_x = (nx + tx - 1) / tx;
        const int y = tile / tiles_x;
        const int x0 = (tile - y * tiles_x) * tx;
        const int txv = min(tx, nx - x0);
        const int c = tid / np_pad, p = tid - c * np_pad;
        const bool cv = c < txv;
        const bool pin = p < np;
        const bool pv = cv && pin;
        // invalid threads read a valid point (finite data) and store nothing
        const int cc = cv ? c : 0, pc = pin ? p : 0;
        const int xc = x0 + cc;
        const long long cell = (long long)y * nx + xc;

        Nb nb;
        nb.ctr = (1 + cc) * np + pc;
        nb.pm = nb.ctr - (pc > 0 ? 1 : 0);
        nb.pp = nb.ctr + (pc < np - 1 ? 1 : 0);
        nb.xm = cc * np + pc;
        nb.xp = (cc + 2) * np + pc;
        nb.ym = has_y ? (tx + 2 + cc) * np + pc : nb.ctr;
        nb.yp = has_y ? (2 * tx + 2 + cc) * np + pc : nb.ctr;
        nb.p = pc;
        nb.p_m = pc - (pc > 0 ? 1 : 0);
        nb.p_p = pc + (pc < np - 1 ? 1 : 0);
        const int seg = seg_cells * np;
        const int rstride = tx * np;            // plane stride inside a staged row
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
        th.invp = (TS)ldg(a.inv_pr + pc);
        th.vr = (TS)ldg(a.vr + pc);
        const double wj = pv ? ldg(a.wj + p) : 0.0;
        const long long o = cell * np + pc;

        Acc<TS, MC> A[3];
        acc_zero(A[0]);
        acc_zero(A[1]);
        acc_zero(A[2]);
        double jx = 0.0, jyr = 0.0, jyi = 0.0;

        // RK epilogue of target row t (slopes Rt, It) from the staged Y0/Y rows
        auto epilogue = [&](const int t, const Acc<TS, MC>& At) {
            const int rb = rows_used % RD;
            if (need_B && !dead && !mbar_wait(rowfull + rb, (uint32_t)((rows_used / RD) & 1))) {
                atomicOr(err, 16);
                dead = true;
            }
            if (!dead && pv) {
                const unsigned char* base = rows + (size_t)rb * 2 * P.row_arr_bytes;
                if (t == 0) {
                    const double k = (double)acc_re(At, 0);
                    if (a.mode == 1) {
                        a.f00_out[o] = k;
                    } else {
                        const double tt = mul_rn(k, a.c1);
                        const double b = reinterpret_cast<const double*>(base)[roff];
                        if (a.f00_out) a.f00_out[o] = add_rn(b, tt);
                        a.f00_A[o] = fma_rn(tt, a.c2,
                                            a.first ? b : reinterpret_cast<const double*>(base + P.row_arr_bytes)[roff]);
                    }
                } else {
                    const bool zero = p < (t >= 2 ? min(t - 1, 80) : 0);
                    const long long g0 = (long long)splane[t * mstride] * a.pstride + o;
                    store_row<MC, TS>(a, min(t, a.m0), zero, At, a.pl_out ? a.pl_out + g0 : nullptr,
                                      a.pl_A + g0, reinterpret_cast<const TS*>(base) + roff,
                                      reinterpret_cast<const TS*>(base + P.row_arr_bytes) + roff, rstride);
                }
            }
            __syncwarp();
            if (need_B && lane == 0) mbar_arrive(rowempty + rb);
            ++rows_used;
        };

        // target row t is in A[0] (row s-1), A[1] (row s) or A[2] (row s+1) while source row s is added
        // source row 0: f00 (already acquired) into row 1
        if (!dead) {
            const double* sb = reinterpret_cast<const double*>(slots + (size_t)slot * P.slot_stride + P.hdr);
            couple_f00<MC>(A[1], scoef[0], sb, nb, th, a.g00_s, a.g00_inv, a.g00_gr);
        }
        release();

        // source row s into target rows s-1 (A[0]), s (A[1]), s+1 (A[2]); then row s-1 is stored
        auto source_row = [&](const int s) {
            const CoefT<TS>* crow = scoef + s * mstride;
            const int mtop = min(s, a.m0);
            static_for<MC + 1>([&](auto mcst) {
                constexpr int m = decltype(mcst)::value;
                if (m > mtop) return;
                acquire();
                if (!dead) {
                    const TS* sb = reinterpret_cast<const TS*>(slots + (size_t)slot * P.slot_stride + P.hdr);
                    const long long qs = splane[s * mstride + m];
                    const TS* ref = (a.pl_ref && __ldg(a.pl_keep + qs)) ? a.pl_ref + qs * np : nullptr;
                    couple_src3<MC, m>(A[0], A[1], A[2], crow[m], sb, seg, nb, th, ref, np);
                    if constexpr (m <= 1) {
                        if (s == 1) {
                            // the current of f = ref + stored deviation
                            const double r0 = ref ? (double)ref[pc] : 0.0;
                            if constexpr (m == 0) {
                                jx += wj * ((double)sb[nb.ctr] + r0);
                            } else {
                                const double r1 = ref ? (double)ref[np + pc] : 0.0;
                                jyr += wj * ((double)sb[nb.ctr] + r0);
                                jyi += wj * ((double)sb[seg + nb.ctr] + r1);
                            }
                        }
                    }
                }
                release();
            });
            epilogue(s - 1, A[0]);
        };
        // the rows move down one accumulator after each source row (one copy
        // of the source-row code keeps the loop within the instruction cache)
        for (int s = 1; s <= a.l0; ++s) {
            source_row(s);
            A[0] = A[1];
            A[1] = A[2];
            acc_zero(A[2]);
        }
        epilogue(a.l0, A[0]);

        // per-cell current: warp sums to the problem's partial-sum array;
        // the batched field kernel adds the warps of a cell in order
        const int warp_in_cell = p >> 5;
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) {
            jx += __shfl_xor_sync(kFull, jx, off);
            jyr += __shfl_xor_sync(kFull, jyr, off);
            jyi += __shfl_xor_sync(kFull, jyi, off);
        }
        if (lane == 0 && cv && !dead) {
            double* jc = a.jw + cell * 24 + warp_in_cell;
            jc[0] = jx;
            jc[8] = jyr;
            jc[16] = jyi;
        }
    };

    for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
        const int tile = item_tile(it);
        // the item's first slot (f00) carries the batch header; every consumer
        // warp keeps its own copy, so no barrier joins the warps.  A wait
        // that ran out here leaves no descriptor to read: the warp stops
        // before item() touches any descriptor field.
        acquire();
        if (dead) break;
        unsigned char* cur = smem + P.off_cur + (size_t)(tid >> 5) * P.hdr;
        {
            const float4* s4 = reinterpret_cast<const float4*>(slots + (size_t)slot * P.slot_stride);
            float4* d4 = reinterpret_cast<float4*>(cur);
            for (int i = lane; i < (int)(P.hdr / 16); i += 32) d4[i] = s4[i];
        }
        __syncwarp();
        // the coupling table and the plane map stay in global memory (L1-resident)
        const StageArgs<TS>& ab = *reinterpret_cast<const StageArgs<TS>*>(cur);
        item(ab, reinterpret_cast<const CoefT<TS>*>(ab.coef_ts), ab.plane_of, tile);
        if (dead) break;
    }
}

template <int MC, typename TS, int MAXT>
cudaError_t launch_pipe(const StageArgs<TS>& a, const BatchWork& bw, int threads, size_t smem, long long nitems,
                        cudaStream_t s) {
    {
        const cudaError_t e = ensure_dyn_smem((const void*)rk_stage_pipe_kernel<MC, TS, MAXT>, smem);
        if (e != cudaSuccess) return e;
    }
    // persistent CTAs, as many as are resident at once, each walking items
    // blockIdx.x + k gridDim.x
    int per_sm = 1;
    {
        cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, rk_stage_pipe_kernel<MC, TS, MAXT>,
                                                                      threads, smem);
        if (e != cudaSuccess || per_sm < 1) per_sm = 1;
    }
    const long long cap = (long long)per_sm * sm_count();
    const long long blocks = nitems < cap ? nitems : cap;
    if (blocks < 1) return cudaSuccess;
    rk_stage_pipe_kernel<MC, TS, MAXT><<<dim3((unsigned)blocks), dim3(threads), smem, s>>>(a, bw);
    return cudaGetLastError();
}

}  // namespace
}  // namespace oshun
