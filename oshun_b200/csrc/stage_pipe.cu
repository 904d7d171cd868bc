// Launchers of the pipelined RK4-stage kernel for one problem.  The helpers
// (pipeline waits, bulk copies, couplings, epilogue) and the description of
// the pipeline are in stage_pipe.cuh; this file holds the single-problem
// kernel, whose argument struct stays in the parameter space throughout (the
// batched kernel in stage_pipe.cuh reads it from each tile's header).
#include "stage_pipe.cuh"

namespace oshun {
namespace {

// CTAs per SM the kernel is compiled for: two for m0 = 0 (few accumulators,
// 80 registers a thread, half-size ring slots) and at most 384 threads, so
// that one CTA's tile starts and ends overlap the other's work
template <int MC, int MAXT>
constexpr int tile_min_blocks() { return (MC == 0 && MAXT <= 384) ? 2 : 1; }

template <int MC, typename TS, int MAXT>
__global__ void __launch_bounds__(MAXT, tile_min_blocks<MC, MAXT>())
    rk_stage_tile_kernel(const StageArgs<TS> a, const int D) {
    extern __shared__ __align__(128) unsigned char smem[];
    const int np = a.np, nx = a.nx, ny = a.ny;
    const int np_pad = (np + 31) & ~31;
    const bool has_y = ny > 1;
    const int tx = (int)(blockDim.x - 64) / np_pad;
    const int nct = np_pad * tx;                       // consumer threads
    const int ncw = nct >> 5;                          // consumer warps
    const int mstride = a.m0 + 1;
    const int ncoef = (a.l0 + 1) * mstride;
    const PipeLayout L = pipe_layout(ncoef, tx, np, has_y, (int)sizeof(TS), a.m0, D);
    uint64_t* full = reinterpret_cast<uint64_t*>(smem);
    uint64_t* empty = full + kMaxDepth;
    uint64_t* rowfull = empty + kMaxDepth;
    uint64_t* rowempty = rowfull + 2;
    uint64_t* f0full = rowempty + 2;
    uint64_t* f0empty = f0full + 1;
    CoefT<TS>* scoef = reinterpret_cast<CoefT<TS>*>(smem + L.off_coef);
    int* splane = reinterpret_cast<int*>(smem + L.off_plane);
    unsigned char* sfld = smem + L.off_fld;    // [2 tiles][6]: the spans holding the tile's E and B
    unsigned char* slots = smem + L.off_slots;
    unsigned char* rows = smem + L.off_rows;          // rows l >= 1: [2 buffers][B, A]
    unsigned char* f0row = smem + L.off_f00;          // the f00 row: [B, A]
    const bool need_B = a.mode != 1;
    const bool need_A = a.mode != 1 && !a.first;
    // Y0 enters the update only through the stage output and the first
    // stage's Y = Y0 + ...; the last stage (no output) reads none
    const bool need_Y0 = need_B && (a.first || a.f00_out != nullptr);

    const int tid = threadIdx.x;
    const unsigned long long wlim = a.wait_ns;   // every pipeline wait gives up after this
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
            for (int k = 0; k < D; ++k) { mbar_init(full + k, 1); mbar_init(empty + k, ncw); }
            for (int k = 0; k < 2; ++k) { mbar_init(rowfull + k, 1); mbar_init(rowempty + k, ncw); }
            mbar_init(f0full, 1);
            mbar_init(f0empty, ncw);
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
            bool ok = true, injected = false;
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
                // the x-stencil segment is one contiguous run unless it wraps
                const bool x_contig = x0 > 0 && x0 + txv < nx;
                for (int s = 0; s <= a.l0 && ok; ++s) {
                    for (int m = 0; m <= min(s, a.m0); ++m) {
                        const int slot = issued % D, j = issued / D;
                        if (issued == a.withhold && blockIdx.x == 0) {
                            // fault injection (tests): this copy and every later one is
                            // withheld, so the consumers' waits for it run out
                            injected = true;
                            ok = false;
                            break;
                        }
                        if (j >= 1 && !mbar_wait(empty + slot, (uint32_t)((j - 1) & 1), wlim)) { ok = false; break; }
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
                            if (x_contig) {
                                bulk_g2s(cb, pb + (size_t)xm_cell * bpc, (txv + 2) * bpc, full + slot);
                            } else {
                                // the edge neighbours come from the x halo columns when the
                                // grid has them (an x slab, or mirrored x boundaries)
                                auto halo = [&](int side) -> const unsigned char* {
                                    if (s == 0) return reinterpret_cast<const unsigned char*>(hx_f00(a, side, y));
                                    const long long q = splane[s * mstride + m];
                                    return reinterpret_cast<const unsigned char*>(hx_plane(a, side, q + comp, y));
                                };
                                const unsigned char* sxm = (a.hx && x0 == 0) ? halo(0) : pb + (size_t)xm_cell * bpc;
                                const unsigned char* sxp =
                                    (a.hx && x0 + txv == nx) ? halo(1) : pb + (size_t)xp_cell * bpc;
                                bulk_g2s(cb, sxm, bpc, full + slot);
                                bulk_g2s(cb + bpc, pb + (size_t)(row + x0) * bpc, txv * bpc, full + slot);
                                bulk_g2s(cb + (size_t)(txv + 1) * bpc, sxp, bpc, full + slot);
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
            }
            if (!ok) {
                if (!injected) atomicOr(a.err, 16);
                // bounded drain of every copy that may still be in flight
                for (int idx = max(0, issued - D); idx < issued; ++idx)
                    mbar_wait(full + (idx % D), (uint32_t)((idx / D) & 1), wlim);
            }
        } else if (tid == nct + 32 && need_B) {
            // row warp, per tile: the f00 row (Y0 and Y) with the tile's fields
            // into the f00 buffer, a tile ahead of its use; then Y0 (and Y) of
            // each target row l >= 1, up to two rows ahead of its epilogue
            int issued = 0;      // rows l >= 1
            int f0_issued = 0;   // f00 rows (one per tile)
            bool ok = true;
            const uint32_t nb = (need_Y0 ? 1 : 0) + (need_A ? 1 : 0);
            for (int tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x) {
                const int y = tile / tiles_x;
                const int x0 = (tile - y * tiles_x) * tx;
                const int txv = min(tx, nx - x0);
                const long long base_cell = (long long)y * nx + x0;
                // the buffer is free once every consumer warp has stored the
                // previous tile's row 0 (and so has read that tile's fields)
                if (f0_issued >= 1 && !mbar_wait(f0empty, (uint32_t)((f0_issued - 1) & 1), wlim)) {
                    ok = false;
                    break;
                }
                {
                    // the tile's fields: per field one bulk copy of the 16-byte
                    // aligned span holding its txv values (a span never leaves the
                    // allocation's pages); then Y0 and Y of the f00 row
                    unsigned char* fd = sfld + (size_t)(f0_issued & 1) * 6 * L.fld_stride;
                    const unsigned char* fsrc[6];
                    uint32_t fsz[6], ftot = 0;
#pragma unroll
                    for (int f = 0; f < 6; ++f) {
                        const uintptr_t lo = reinterpret_cast<uintptr_t>(a.fld_in + f * a.cells + base_cell);
                        const uintptr_t hi = lo + (uintptr_t)txv * sizeof(TS);
                        fsrc[f] = reinterpret_cast<const unsigned char*>(lo & ~(uintptr_t)15);
                        fsz[f] = (uint32_t)(((hi + 15) & ~(uintptr_t)15) - (lo & ~(uintptr_t)15));
                        ftot += fsz[f];
                    }
                    const uint32_t b = (uint32_t)txv * np * 8;
                    mbar_expect_tx(f0full, nb * b + ftot);
#pragma unroll
                    for (int f = 0; f < 6; ++f) bulk_g2s(fd + (size_t)f * L.fld_stride, fsrc[f], fsz[f], f0full);
                    if (need_Y0) bulk_g2s(f0row, a.f00_B + base_cell * np, b, f0full);
                    if (need_A) bulk_g2s(f0row + L.f00_arr_bytes, a.f00_A + base_cell * np, b, f0full);
                    ++f0_issued;
                }
                for (int t = 1; t <= a.l0; ++t) {
                    const int rb = issued & 1, k = issued >> 1;
                    if (k >= 1 && !mbar_wait(rowempty + rb, (uint32_t)((k - 1) & 1), wlim)) { ok = false; break; }
                    unsigned char* base = rows + (size_t)rb * 2 * L.rowl_arr_bytes;
                    const int np_row = 1 + 2 * min(t, a.m0);
                    const uint32_t b = (uint32_t)txv * np * sizeof(TS);
                    mbar_expect_tx(rowfull + rb, nb * np_row * b);
                    const long long q0 = splane[t * mstride];
                    for (int kk = 0; kk < np_row; ++kk) {
                        const long long off = (q0 + kk) * a.pstride + base_cell * np;
                        const size_t d = (size_t)kk * tx * np * sizeof(TS);
                        if (need_Y0) bulk_g2s(base + d, a.pl_B + off, b, rowfull + rb);
                        if (need_A) bulk_g2s(base + L.rowl_arr_bytes + d, a.pl_A + off, b, rowfull + rb);
                    }
                    ++issued;
                }
            }
            if (!ok) {
                atomicOr(a.err, 16);
                // bounded drain of the copies that may still be in flight
                for (int t = max(0, issued - 2); t < issued; ++t)
                    mbar_wait(rowfull + (t & 1), (uint32_t)((t >> 1) & 1), wlim);
                if (f0_issued >= 1) mbar_wait(f0full, (uint32_t)((f0_issued - 1) & 1), wlim);
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
        if (!dead && !mbar_wait(full + slot, phase, wlim)) {
            atomicOr(a.err, 16);
            dead = true;
        }
    };
    auto release = [&]() {
        __syncwarp();
        if (lane == 0) mbar_arrive(empty + slot);
        if (++slot == D) { slot = 0; phase ^= 1u; }
    };

    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x, ++tile_iter) {
        const int y = tile / tiles_x;
        const int x0 = (tile - y * tiles_x) * tx;
        const int txv = min(tx, nx - x0);
        const bool cv = c < txv;
        const bool pv = cv && pin;
        const int cc = cv ? c : 0;
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
        const int roff = cc * np + pc;          // this point inside a staged row

        Th<TS> th;
        if (need_B) {
            // the row warp staged this tile's fields with its f00 row
            if (!dead && !mbar_wait(f0full, (uint32_t)(tile_iter & 1), wlim)) {
                atomicOr(a.err, 16);
                dead = true;
            }
            // field f of this cell: its span's start is the aligned-down address
            const unsigned char* fb = sfld + (size_t)(tile_iter & 1) * 6 * L.fld_stride;
            const long long c0 = (long long)y * nx + x0;
            auto fval = [&](int f) -> TS {
                const uintptr_t addr = reinterpret_cast<uintptr_t>(a.fld_in + f * a.cells + c0);
                return reinterpret_cast<const TS*>(fb + (size_t)f * L.fld_stride + (addr & 15))[cc];
            };
            th.ex = fval(0); th.ey = fval(1); th.ez = fval(2);
            th.bx = fval(3); th.by = fval(4); th.bz = fval(5);
        } else {
            th.ex = ldg(a.fld_in + cell);
            th.ey = ldg(a.fld_in + a.cells + cell);
            th.ez = ldg(a.fld_in + 2 * a.cells + cell);
            th.bx = ldg(a.fld_in + 3 * a.cells + cell);
            th.by = ldg(a.fld_in + 4 * a.cells + cell);
            th.bz = ldg(a.fld_in + 5 * a.cells + cell);
        }
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

        Acc<TS, MC> A[3];
        acc_zero(A[0]);
        acc_zero(A[1]);
        acc_zero(A[2]);
        double jx = 0.0, jyr = 0.0, jyi = 0.0;

        // RK epilogue of target row t (slopes Rt, It) from the staged Y0/Y rows
        auto epilogue = [&](const int t, const Acc<TS, MC>& At) {
            if (t == 0) {
                // the f00 buffer: its wait was the tile's first
                if (!dead && pv) {
                    const double k = (double)acc_re(At, 0);
                    if (a.mode == 1) {
                        a.f00_out[o] = k;
                    } else {
                        const double* fb = reinterpret_cast<const double*>(f0row);
                        const double tt = mul_rn(k, a.c1);
                        const double b = fb[roff];
                        if (a.f00_out) a.f00_out[o] = add_rn(b, tt);
                        a.f00_A[o] = fma_rn(
                            tt, a.c2, a.first ? b : reinterpret_cast<const double*>(f0row + L.f00_arr_bytes)[roff]);
                    }
                }
                __syncwarp();
                if (need_B && lane == 0) mbar_arrive(f0empty);
                return;
            }
            const int rb = rows_used & 1;
            if (need_B && !dead && !mbar_wait(rowfull + rb, (uint32_t)((rows_used >> 1) & 1), wlim)) {
                atomicOr(a.err, 16);
                dead = true;
            }
            if (!dead && pv) {
                const unsigned char* base = rows + (size_t)rb * 2 * L.rowl_arr_bytes;
                const bool zero = p < (t >= 2 ? min(t - 1, 80) : 0);
                const long long g0 = (long long)splane[t * mstride] * a.pstride + o;
                store_row<MC, TS>(a, min(t, a.m0), zero, At, a.pl_out ? a.pl_out + g0 : nullptr, a.pl_A + g0,
                                  reinterpret_cast<const TS*>(base) + roff,
                                  reinterpret_cast<const TS*>(base + L.rowl_arr_bytes) + roff, rstride);
            }
            __syncwarp();
            if (need_B && lane == 0) mbar_arrive(rowempty + rb);
            ++rows_used;
        };

        // source row 0: f00 into row 1
        acquire();
        if (!dead) {
            const double* sb = reinterpret_cast<const double*>(slots + (size_t)slot * L.slot_bytes);
            couple_f00<MC>(A[1], scoef[0], sb, nb, th, a.g00_s, a.g00_inv, a.g00_gr);
        }
        release();

        // source row s, K = s % 3
        // source row s into target rows s-1 (A[0]), s (A[1]), s+1 (A[2]); then row s-1 is stored
        auto source_row = [&](const int s) {
            const CoefT<TS>* crow = scoef + s * mstride;
            const int mtop = min(s, a.m0);
            static_for<MC + 1>([&](auto mcst) {
                constexpr int m = decltype(mcst)::value;
                if (m > mtop) return;
                acquire();
                if (!dead) {
                    const TS* sb = reinterpret_cast<const TS*>(slots + (size_t)slot * L.slot_bytes);
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
        // A[0], A[1], A[2] hold target rows s-1, s, s+1 while source row s is
        // added; then row s-1 is stored and the rows move down one accumulator.
        // One copy of the source-row code (not one per row position) keeps the
        // consumer loop small enough for the instruction cache.
        for (int s = 1; s <= a.l0; ++s) {
            source_row(s);
            A[0] = A[1];
            A[1] = A[2];
            acc_zero(A[2]);
        }
        epilogue(a.l0, A[0]);

        // per-cell current: warp sums to global; stage_fields_kernel adds the
        // warps of a cell in order (deterministic) and updates E and B.  No
        // barrier joins the consumer warps: a warp whose wait ran out stops on
        // its own and the others' waits end by their own limits.
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
        if (dead) break;
    }
}

// E and B of every cell from the current partial sums of the stage kernel
// (Ampere and Faraday with centred differences, then the RK update)
template <typename TS>
__global__ void __launch_bounds__(256) stage_fields_kernel(const StageArgs<TS> a, const int nw) {
    const long long cell = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (cell < a.cells) fields_cell(a, cell, nw);
}

template <int MC, typename TS, int MAXT>
cudaError_t launch_tile(const StageArgs<TS>& a, int tx, const PipeLayout& L, cudaStream_t s) {
    {
        const cudaError_t e = ensure_dyn_smem((const void*)rk_stage_tile_kernel<MC, TS, MAXT>, L.total);
        if (e != cudaSuccess) return e;
    }
    const int np_pad = ((a.np + 31) / 32) * 32;
    const long long tiles = (long long)a.ny * ((a.nx + tx - 1) / tx);
    // as many CTAs as are resident at once (one per SM, two for the m0 = 0
    // form when its shared memory allows), each walking tiles blockIdx.x + k gridDim.x
    int per_sm = 1;
    if (tile_min_blocks<MC, MAXT>() > 1) {
        const cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(
            &per_sm, rk_stage_tile_kernel<MC, TS, MAXT>, np_pad * tx + 64, L.total);
        if (e != cudaSuccess || per_sm < 1) { (void)cudaGetLastError(); per_sm = 1; }
        if (per_sm > tile_min_blocks<MC, MAXT>()) per_sm = tile_min_blocks<MC, MAXT>();
    }
    const long long resident = (long long)sm_count() * per_sm;
    const long long blocks = tiles < resident ? tiles : resident;
    rk_stage_tile_kernel<MC, TS, MAXT><<<dim3((unsigned)blocks), dim3(np_pad * tx + 64), L.total, s>>>(a, L.depth);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    stage_fields_kernel<TS><<<dim3((unsigned)((a.cells + 255) / 256)), dim3(256), 0, s>>>(a, np_pad >> 5);
    return cudaGetLastError();
}

template <typename TS, int MC>
cudaError_t pipe_mc(const StageArgs<TS>& a, cudaStream_t s) {
    const int np_pad = ((a.np + 31) / 32) * 32;
    // bulk copies move whole momentum rows: 16-byte multiples for every plane type
    if ((a.np * (int)sizeof(TS)) % 16 != 0 || np_pad > 256) return cudaErrorNotSupported;
    // The kernel is latency-bound: more consumer warps per SM pay even when
    // the register cap makes the accumulators spill a little.  Registers are
    // granted per SM sub-partition, so a CTA of 9-12 warps costs 12 warps'
    // worth: 168 registers a thread; 13-16 warps: 128.  Consumer threads:
    //   m0 <= 1, or FP32 with m0 <= 6           up to 448 (16 warps)
    //   FP64 with m0 <= 6, FP32 with m0 >= 7    up to 320 (12 warps)
    //   FP64 with m0 >= 7 (spills at 168)       up to 192 (8 warps, 255)
    constexpr bool f32 = sizeof(TS) == 4;
    // m0 = 0: up to 320 consumer threads, two CTAs per SM (tile_min_blocks)
    constexpr int budget = MC == 0 ? 320 : (MC <= 1 || (f32 && MC <= 6)) ? 448 : (f32 || MC <= 6) ? 320 : 192;
    int tx = budget >= np_pad ? budget / np_pad : 1;
    if (tx > kMaxTx) tx = kMaxTx;
    if (tx > a.nx) tx = a.nx;
    // at least one tile per SM where the grid has the cells for it
    const long long cells = (long long)a.nx * a.ny;
    const long long per_sm = cells / sm_count();
    if (tx > per_sm) tx = per_sm > 1 ? (int)per_sm : 1;
    const int ncoef = (a.l0 + 1) * (a.m0 + 1);
    // the deepest source ring that fits `cap` (4 slots at least), else fewer cells a tile
    auto plan = [&](size_t cap, PipeLayout& L, int& t) -> bool {
        t = tx;
        for (;;) {
            int depth = kDepth;
            L = pipe_layout(ncoef, t, a.np, a.ny > 1, (int)sizeof(TS), a.m0, depth);
            while (L.total > cap && depth > 4)
                L = pipe_layout(ncoef, t, a.np, a.ny > 1, (int)sizeof(TS), a.m0, --depth);
            if (L.total <= cap || t == 1) break;
            --t;
        }
        return L.total <= cap;
    };
    // m0 = 0: half an SM's shared memory, so that two CTAs share it, when
    // that still leaves 4 slots; otherwise the whole of it
    PipeLayout L;
    int txp = tx;
    if (!(MC == 0 && plan(kSmemHalf, L, txp)) && !plan(kSmemMax, L, txp)) return cudaErrorNotSupported;
    tx = txp;
    const int threads = np_pad * tx + 64;
    if (threads <= 256) return launch_tile<MC, TS, 256>(a, tx, L, s);
    if (threads <= 384) return launch_tile<MC, TS, 384>(a, tx, L, s);
    if constexpr (budget == 448) return launch_tile<MC, TS, 512>(a, tx, L, s);
    return cudaErrorNotSupported;
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
