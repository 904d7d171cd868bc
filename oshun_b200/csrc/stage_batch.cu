// Launcher of the pipelined RK4-stage kernel over a batch of independent
// problems (the kernel is in stage_pipe.cuh): one persistent launch walks the
// (problem, tile) list of every problem of the batch.
#include "stage_pipe.cuh"

namespace oshun {
namespace {

template <typename TS, int MC>
cudaError_t batch_mc(const StageArgs<TS>& a1, const BatchWork& bw, int nc, cudaStream_t s) {
    const SmemPlan P = smem_plan<TS>(true, bw.hdr_bytes, 0, bw.slot_bytes, bw.row_arr_bytes, bw.row_depth);
    if (P.total > kSmemMax) return cudaErrorNotSupported;
    const int threads = nc + 64;
    // 9-12 warps are granted 12 warps' registers (168 a thread), so one
    // instantiation covers 257-384 threads; with m0 <= 1 a 320-thread CTA is
    // compiled for two per SM (102 registers)
    cudaError_t e = cudaErrorNotSupported;
    if (threads <= 256) {
        e = launch_pipe<MC, TS, 256>(a1, bw, threads, P.total, bw.nitems, s);
    } else if constexpr (MC <= 1) {
        if (threads <= 320) e = launch_pipe<MC, TS, 320>(a1, bw, threads, P.total, bw.nitems, s);
        else if (threads <= 384) e = launch_pipe<MC, TS, 384>(a1, bw, threads, P.total, bw.nitems, s);
    } else if (threads <= 384) {
        e = launch_pipe<MC, TS, 384>(a1, bw, threads, P.total, bw.nitems, s);
    }
    if (e != cudaSuccess) return e;
    // E and B of every problem from the stage's current partial sums
    stage_fields_batch_kernel<TS><<<dim3((unsigned)bw.nprobs), dim3(128), 0, s>>>(bw.probs, bw.desc_bytes);
    return cudaGetLastError();
}

}  // namespace

size_t stage_batch_smem(const BatchWork& bw, int elem_bytes) {
    return elem_bytes == 4 ? smem_plan<float>(true, bw.hdr_bytes, 0, bw.slot_bytes, bw.row_arr_bytes, bw.row_depth).total
                           : smem_plan<double>(true, bw.hdr_bytes, 0, bw.slot_bytes, bw.row_arr_bytes, bw.row_depth).total;
}

void stage_batch_sizes(int np, int nx, int ny, int l0, int m0, int nc, int tx_cap, int elem_bytes, int* tx,
                       size_t* slot_bytes, size_t* row_arr_bytes) {
    *tx = tile_cells(np, nx, nc, tx_cap);
    const PipeLayout L = pipe_layout((l0 + 1) * (m0 + 1), *tx, np, ny > 1, elem_bytes, m0);
    *slot_bytes = L.slot_bytes;
    *row_arr_bytes = L.row_arr_bytes;
}

int stage_batch_coef_bytes(int elem_bytes) {
    return elem_bytes == 4 ? (int)sizeof(CoefT<float>) : (int)sizeof(CoefT<double>);
}

// nc consumer threads per CTA (a multiple of 32, <= 320); m0 of every problem <= mc
template <typename TS>
cudaError_t launch_stage_batch(const StageArgs<TS>& a1, const BatchWork& bw, int mc, int nc, cudaStream_t s) {
    if (nc < 32 || nc > 320 || nc % 32) return cudaErrorInvalidValue;
    switch (mc) {
        case 0: return batch_mc<TS, 0>(a1, bw, nc, s);
        case 1: return batch_mc<TS, 1>(a1, bw, nc, s);
        case 2: return batch_mc<TS, 2>(a1, bw, nc, s);
        case 3: return batch_mc<TS, 3>(a1, bw, nc, s);
        case 4: return batch_mc<TS, 4>(a1, bw, nc, s);
        case 6: return batch_mc<TS, 6>(a1, bw, nc, s);
        case 8: return batch_mc<TS, 8>(a1, bw, nc, s);
        default: return cudaErrorNotSupported;
    }
}
template cudaError_t launch_stage_batch<double>(const StageArgs<double>&, const BatchWork&, int, int, cudaStream_t);
template cudaError_t launch_stage_batch<float>(const StageArgs<float>&, const BatchWork&, int, int, cudaStream_t);

}  // namespace oshun
