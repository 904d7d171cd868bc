// Launchers of the pipelined RK4-stage kernel for one problem (the kernel
// and its description are in stage_pipe.cuh).
#include "stage_pipe.cuh"

namespace oshun {
namespace {

template <typename TS, int MC>
cudaError_t pipe_mc(const StageArgs<TS>& a, cudaStream_t s) {
    const int np_pad = ((a.np + 31) / 32) * 32;
    // bulk copies move whole momentum rows: 16-byte multiples for every plane type
    if ((a.np * (int)sizeof(TS)) % 16 != 0 || np_pad > 256) return cudaErrorNotSupported;
    // consumer threads <= 192: 8 warps with the producers, 255 registers per thread
    const int nc = np_pad <= 192 ? (192 / np_pad) * np_pad : np_pad;
    const int tx = tile_cells(a.np, a.nx, nc, kMaxTx);
    const int ncoef = (a.l0 + 1) * (a.m0 + 1);
    const PipeLayout L = pipe_layout(ncoef, tx, a.np, a.ny > 1, (int)sizeof(TS), a.m0);
    const SmemPlan P = smem_plan<TS>(false, 0, ncoef, L.slot_bytes, L.row_arr_bytes);
    if (P.total > 227 * 1024) return cudaErrorNotSupported;
    BatchWork bw = {};
    bw.tx_cap = tx;
    const long long tiles = (long long)a.ny * ((a.nx + tx - 1) / tx);
    const int threads = np_pad * tx + 64;
    if (threads <= 256) return launch_pipe<MC, TS, 256, false>(a, bw, threads, P.total, tiles, s);
    return launch_pipe<MC, TS, 320, false>(a, bw, threads, P.total, tiles, s);
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
