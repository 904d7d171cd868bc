// oshun_collide_flm_noalloc: the implicit f_lm collision step on caller-owned
// device planes, allocating no device memory.
//
// Some callers cannot call cudaMalloc inside their time loop: applications
// that hand all device memory to their own pool at start-up, or foreign
// runtimes driving this library through the C ABI whose memory is owned by
// the host program.  For them this entry point keeps every piece of scratch
// the collision kernel needs -- its velocity-grid tables, plane maps, status
// word and, in the dense (Gauss-Seidel) mode, the per-CTA np x np matrix
// workspace -- in one file-scope __device__ array of kScratchBytes.  Every
// GPU that loads the library holds that array until the process exits.
//
// The kernel is the collision kernel of collide.cu (launch_collide), the
// staged-chunk / dense Gauss-Seidel variant, run with do_ee = 0 and both f1
// and f_lm steps; only the source of its scratch differs.  A small kernel
// writes the velocity tables and plane maps into the array first, so the
// call stages nothing in host memory.
//
// Set-up: the first call on a device, with that device current, looks up
// the device address of the array (cudaGetSymbolAddress) and caches it; make
// that first call before any stream capture.  All calls share the array and
// it keeps the last call's contents, so calls that overlap on the GPU (two
// streams, or two threads) race on it: serialise them.
#include <cmath>
#include <cstring>
#include <mutex>
#include <string>

#include "oshun_internal.h"

namespace oshun {
namespace {

constexpr size_t kScratchBytes = 32ull << 20;   // 32 MiB
constexpr int kMaxDevices = 64;
constexpr int kMaxL0 = 64;

static __device__ __align__(256) unsigned char g_scratch[kScratchBytes];

std::mutex g_setup_mutex;
void* g_scratch_ptr[kMaxDevices] = {nullptr};

// byte offsets inside the scratch array
constexpr size_t kOffStatus = 0;      // 4 ints
constexpr size_t kOffTables = 256;    // 12 * np doubles
size_t off_ints(int np) { return kOffTables + ((size_t)12 * np * sizeof(double) + 255) / 256 * 256; }
size_t off_dense(int np, int ncoef, int nplanes) {
    return off_ints(np) + (((size_t)ncoef + 2 * (size_t)nplanes) * sizeof(int) + 255) / 256 * 256;
}

// The velocity-grid tables of the collision operators
// (OSHUN-1/def-FokkerPlanck.cpp:143-172, 790-803) and the plane maps, built
// on the device straight into the scratch array, so the call keeps no host
// staging buffer alive after it returns.  The arithmetic mirrors the handle's
// host-side tables operation by operation (no contracted multiply-adds).
__global__ void __launch_bounds__(256) noalloc_tables_kernel(double* V, int* plane_of, int* plane_l, int* plane_m,
                                                             int* status, int np, int l0, int m0, double pmin,
                                                             double pmax) {
    const int t = threadIdx.x;
    if (t < 4) status[t] = 0;   // the status word starts at zero every call
    const double step = __ddiv_rn(__dsub_rn(pmax, pmin), (double)(np - 1));
    double* vr = V;
    for (int i = t; i < np; i += blockDim.x) {
        const double p = __dadd_rn(__dmul_rn((double)i, step), pmin);
        vr[i] = __ddiv_rn(p, __dsqrt_rn(__dadd_rn(1.0, __dmul_rn(p, p))));
    }
    __syncthreads();
    for (int i = t; i < np; i += blockDim.x) {
        const double v = vr[i];
        if (i >= 1) {
            const double w = vr[i - 1];
            const double dv = __dsub_rn(v, w);
            V[np + i] = __dmul_rn(__dmul_rn(0.5, pow(v, 4.0)), dv);
            V[2 * np + i] = __dmul_rn(__dmul_rn(0.5, pow(w, 4.0)), dv);
            V[3 * np + i] = __dmul_rn(__dmul_rn(__dmul_rn(0.5, v), v), dv);
            V[4 * np + i] = __dmul_rn(__dmul_rn(__dmul_rn(0.5, w), w), dv);
            V[5 * np + i] = __dmul_rn(__dmul_rn(0.5, v), dv);
            V[6 * np + i] = __dmul_rn(__dmul_rn(0.5, w), dv);
        } else {
            for (int k = 1; k <= 6; ++k) V[k * np] = 0.0;
        }
        V[7 * np + i] = pow(v, 3.0);
        V[10 * np + i] = pow(v, 5.0);
        V[11 * np + i] = pow(v, 7.0);
        if (i == 0)
            V[8 * np] = __ddiv_rn(1.0, __ddiv_rn(__dmul_rn(__dmul_rn(vr[0], vr[0]), vr[1]), 2.0));
        else if (i < np - 1)
            V[8 * np + i] = __ddiv_rn(1.0, __ddiv_rn(__dmul_rn(__dmul_rn(v, v), __dsub_rn(vr[i + 1], vr[i - 1])), 2.0));
        else
            V[8 * np + i] = 0.0;
        if (i < np - 1)
            V[9 * np + i] = __ddiv_rn(1.0, __dmul_rn(__ddiv_rn(__dsub_rn(vr[i + 1], v), 2.0), __dadd_rn(vr[i + 1], v)));
        else
            V[9 * np + i] = 0.0;
    }
    // plane maps (the handle's plane order: l >= 1, m <= min(l, m0), Re then Im)
    if (t == 0) {
        const int ncoef = (l0 + 1) * (m0 + 1);
        for (int i = 0; i < ncoef; ++i) plane_of[i] = -1;
        int q = 0;
        for (int l = 1; l <= l0; ++l)
            for (int m = 0; m <= (l < m0 ? l : m0); ++m) {
                plane_of[l * (m0 + 1) + m] = q;
                for (int k = 0; k < (m > 0 ? 2 : 1); ++k) {
                    plane_l[q] = l;
                    plane_m[q] = m;
                    ++q;
                }
            }
    }
}

}  // namespace
}  // namespace oshun

using namespace oshun;

extern "C" int oshun_collide_flm_noalloc(const oshun_cfg* cfg, double* f00, double* planes, double Dt,
                                         void* stream, long long* nondominant, int* flags) {
    if (!cfg || !f00 || !planes) { set_error("NULL argument"); return OSHUN_ERR_ARG; }
    const oshun_cfg& c = *cfg;
    if (c.precision != OSHUN_FP64) { set_error("noalloc collision step: FP64 planes only"); return OSHUN_ERR_UNSUPPORTED; }
    if (c.l0 < 1 || c.m0 < 0 || c.m0 > c.l0 || c.nump < 3 || c.numx < 1 || c.numy < 1 || !(c.pmax > c.pmin) ||
        !(c.pmin > 0.0) || !(c.density_np > 0.0)) {
        set_error("noalloc collision step: bad configuration");
        return OSHUN_ERR_ARG;
    }
    if (c.l0 > kMaxL0 || c.m0 > kMaxM0 || c.nump > kMaxNp) {
        set_error("noalloc collision step: needs l0 <= 64, m0 <= 8, nump <= 1024");
        return OSHUN_ERR_UNSUPPORTED;
    }
    const int np = c.nump, l0 = c.l0, m0 = c.m0;
    const long long cells = (long long)c.numx * c.numy;
    const int ncoef = (l0 + 1) * (m0 + 1);
    int nplanes = 0;
    for (int l = 1; l <= l0; ++l)
        for (int m = 0; m <= (l < m0 ? l : m0); ++m) nplanes += m > 0 ? 2 : 1;

    // size check against the fixed scratch
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess || dev >= kMaxDevices) { set_error("noalloc collision step: no usable device"); return OSHUN_ERR_NO_DEVICE; }
    int nsm = 0, smem_optin = 0;
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    cudaDeviceGetAttribute(&smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    const size_t budget = (size_t)smem_optin < (size_t)200 * 1024 ? (size_t)smem_optin : (size_t)200 * 1024;
    const size_t dense_off = off_dense(np, ncoef, nplanes);
    int blocks, chunk = 0;
    size_t smem;
    if (c.if_tridiagonal) {
        chunk = collide_max_chunk(np, budget);
        if (chunk < 1) { set_error("noalloc collision step: nump too large for shared memory"); return OSHUN_ERR_UNSUPPORTED; }
        if (chunk > nplanes) chunk = nplanes > 0 ? nplanes : 1;
        smem = collide_smem_bytes(np, chunk, 1);
        blocks = (int)(cells < (long long)nsm * 16 ? cells : (long long)nsm * 16);
        if (dense_off > kScratchBytes) { set_error("noalloc collision step: tables exceed the 32 MiB scratch"); return OSHUN_ERR_UNSUPPORTED; }
    } else {
        smem = collide_smem_bytes(np, 0, 0);
        if (smem > budget) { set_error("noalloc collision step: nump too large for the dense path"); return OSHUN_ERR_UNSUPPORTED; }
        const size_t per_block = (size_t)np * np * sizeof(double);
        if (dense_off + per_block > kScratchBytes) {
            set_error("noalloc collision step: one np x np workspace exceeds the 32 MiB scratch");
            return OSHUN_ERR_UNSUPPORTED;
        }
        long long fit = (long long)((kScratchBytes - dense_off) / per_block);
        long long want = cells < (long long)nsm * 4 ? cells : (long long)nsm * 4;
        blocks = (int)(fit < want ? fit : want);
    }

    // one-time set-up per device: the device address of the scratch array
    void* base;
    {
        std::lock_guard<std::mutex> lock(g_setup_mutex);
        if (!g_scratch_ptr[dev]) {
            void* ptr = nullptr;
            e = cudaGetSymbolAddress(&ptr, g_scratch);
            if (e != cudaSuccess || !ptr) {
                set_error(std::string("noalloc collision step: cudaGetSymbolAddress: ") + cudaGetErrorString(e));
                return OSHUN_ERR_CUDA;
            }
            g_scratch_ptr[dev] = ptr;
        }
        base = g_scratch_ptr[dev];
    }
    unsigned char* sb = static_cast<unsigned char*>(base);
    cudaStream_t st = static_cast<cudaStream_t>(stream);

    double* dV = reinterpret_cast<double*>(sb + kOffTables);
    int* dI = reinterpret_cast<int*>(sb + off_ints(np));
    int* dstatus = reinterpret_cast<int*>(sb + kOffStatus);
#define CKN(call)                                                                             \
    do {                                                                                      \
        cudaError_t e_ = (call);                                                              \
        if (e_ != cudaSuccess) {                                                              \
            set_error(std::string("noalloc collision step: ") + #call + ": " + cudaGetErrorString(e_)); \
            return OSHUN_ERR_CUDA;                                                            \
        }                                                                                     \
    } while (0)
    noalloc_tables_kernel<<<1, 256, 0, st>>>(dV, dI, dI + ncoef, dI + ncoef + nplanes, dstatus, np, l0, m0, c.pmin,
                                             c.pmax);
    CKN(cudaGetLastError());
    const double kRe = 2.8179402894e-13;
    const double kp = std::sqrt(4.0 * M_PI * c.density_np * kRe);

    CollideArgs a;
    std::memset(&a, 0, sizeof(a));
    a.f00 = f00;
    a.planes = planes;
    a.planes_fp32 = 0;
    a.plane_of = dI; a.plane_l = dI + ncoef; a.plane_m = dI + ncoef + nplanes;
    a.nplanes = nplanes;
    a.cells = cells; a.pstride = cells * np;
    a.np = np; a.l0 = l0; a.m0 = m0;
    a.mmax_coll = c.if_implicit1D ? 0 : m0;
    a.do_ee = 0; a.do_l1 = 1; a.do_lm = 1;
    a.if_tridiagonal = c.if_tridiagonal;
    a.nsub = 0; a.hsub = 0.0; a.Dt = Dt;
    a.NB = c.NB_algorithms;
    a.density_np = c.density_np; a.Zeta = c.Zeta;
    a.c_kpre = 4.0 * M_PI / 3.0 * kRe * kp;
    a.kpre = kRe * kp;
    a.vr = dV; a.U4 = dV + np; a.U4m1 = dV + 2 * np; a.U2 = dV + 3 * np; a.U2m1 = dV + 4 * np;
    a.U1 = dV + 5 * np; a.U1m1 = dV + 6 * np; a.U3 = dV + 7 * np; a.Qn = dV + 8 * np; a.Pn = dV + 9 * np;
    a.V5 = dV + 10 * np; a.V7 = dV + 11 * np;
    a.chunk = chunk;
    a.dense_ws = c.if_tridiagonal ? nullptr : reinterpret_cast<double*>(sb + dense_off);
    a.status = dstatus;
    CKN(launch_collide(a, st, smem, blocks));
    if (nondominant || flags) {
        // NaN/Inf in the result planes sets bit 1; then wait for the stream
        // and report the status word (a read-back that a stream capture
        // cannot hold: refused while the stream is capturing)
        cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
        CKN(cudaStreamIsCapturing(st, &cs));
        if (cs != cudaStreamCaptureStatusNone) {
            set_error("noalloc collision step: nondominant/flags read back the status; pass NULL while capturing");
            return OSHUN_ERR_UNSUPPORTED;
        }
        CKN(launch_nan_check(f00, planes, 0, cells * np, (long long)nplanes * cells * np, nullptr, 0, dstatus, st));
        int h_status[2] = {0, 0};
        CKN(cudaMemcpyAsync(h_status, dstatus, sizeof(int) * 2, cudaMemcpyDeviceToHost, st));
        CKN(cudaStreamSynchronize(st));
        if (nondominant) *nondominant = h_status[1];
        if (flags) *flags = h_status[0];
        if (h_status[0] & 2) {
            set_error("noalloc collision step: NaN/Inf in the result planes");
            return OSHUN_ERR_NUMERIC;
        }
    }
#undef CKN
    return OSHUN_OK;
}
