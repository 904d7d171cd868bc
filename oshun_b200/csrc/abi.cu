// C ABI of liboshun_b200 (include/oshun_b200.h): handle lifetime, operator
// tables, state transfer, the RK4 step driver, the collision driver and the
// captured-graph step loop.
//
// Device state (per handle):
//   f00 plane      FP64 [numy][numx][nump]
//   planes         every l >= 1 harmonic as 1 (m = 0) or 2 (m > 0, Re then Im)
//                  real planes [numy][numx][nump], harmonics in ind(l,m) order;
//                  FP64, or FP32 in OSHUN_FP32_SPLIT
//   fields         6 real planes [numy][numx] (Ex Ey Ez Bx By Bz)
// m = 0 harmonics and the fields are stored real: every reference operator
// keeps them real (the couplings into m = 0 take real parts,
// OSHUN-1/def-VlasovMax.cpp:386,394,614,878), so their imaginary parts are
// identically zero.
//
// Four copies of the state rotate through an RK4 step (Runge_Kutta_4 keeps
// Y, Y0, Y1, Yh; def-RK.cpp:56): set `cur` is Y0 (stage-1 input), set `nxt`
// is the accumulator Y that becomes the new state, sets 2 and 3 carry the
// stage inputs.  `cur` and `nxt` swap after each step.
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstddef>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "adjoint2d.cuh"
#include "oshun_internal.h"

namespace oshun {

static thread_local std::string g_last_error;
void set_error(const std::string& msg) { g_last_error = msg; }

cudaError_t ensure_dyn_smem(const void* func, size_t bytes) {
    static std::mutex mu;
    static std::vector<std::pair<std::pair<const void*, int>, size_t>> set;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    std::lock_guard<std::mutex> lk(mu);
    for (auto& kv : set)
        if (kv.first.first == func && kv.first.second == dev) {
            if (bytes <= kv.second) return cudaSuccess;
            e = cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
            if (e == cudaSuccess) kv.second = bytes;
            return e;
        }
    e = cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    if (e == cudaSuccess) set.push_back({{func, dev}, bytes});
    return e;
}

int sm_count() {
    static std::mutex mu;
    static int n[64] = {0};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 148;
    std::lock_guard<std::mutex> lk(mu);
    if (n[dev] == 0) {
        int v = 0;
        if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || v <= 0) v = 148;
        n[dev] = v;
    }
    return n[dev];
}

namespace {

struct Clock {
    double t, t_ee, t_eb;
};

// ---- small kernels ---------------------------------------------------------

// case layout (complex128 per harmonic) -> planes; flags nonzero imaginary
// parts of m = 0 harmonics and fields
template <typename TS>
__global__ void scatter_kernel(const double2* __restrict__ src, double* f00, TS* planes, TS* fields,
                               const int* __restrict__ hplane, long long pstride, int nh, long long cells,
                               int* flag, const double* __restrict__ ref, int np) {
    const long long total = (long long)nh * pstride + 6 * cells;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        const double2 v = src[i];
        if (i < (long long)nh * pstride) {
            const int h = (int)(i / pstride);
            const long long off = i - (long long)h * pstride;
            const int q = hplane[h];
            if (q < 0) {                               // f00
                f00[off] = v.x;
                if (v.y != 0.0) *flag = 1;
            } else if (q >= 0 && hplane[nh + h]) {     // m > 0: Re, Im
                const int p = (int)(off % np);
                planes[(long long)q * pstride + off] = (TS)(ref ? v.x - ref[(long long)q * np + p] : v.x);
                planes[(long long)(q + 1) * pstride + off] = (TS)(ref ? v.y - ref[(long long)(q + 1) * np + p] : v.y);
            } else {
                const int p = (int)(off % np);
                planes[(long long)q * pstride + off] = (TS)(ref ? v.x - ref[(long long)q * np + p] : v.x);
                if (v.y != 0.0) *flag = 1;
            }
        } else {
            const long long j = i - (long long)nh * pstride;
            fields[j] = (TS)v.x;
            if (v.y != 0.0) *flag = 1;
        }
    }
}

template <typename TS>
__global__ void gather_kernel(double2* __restrict__ dst, const double* f00, const TS* planes, const TS* fields,
                              const int* __restrict__ hplane, long long pstride, int nh, long long cells,
                              const double* __restrict__ ref, int np) {
    const long long total = (long long)nh * pstride + 6 * cells;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        double2 v;
        if (i < (long long)nh * pstride) {
            const int h = (int)(i / pstride);
            const long long off = i - (long long)h * pstride;
            const int q = hplane[h];
            const int p = (int)(off % np);
            auto val = [&](long long qq) {
                return (double)planes[qq * pstride + off] + (ref ? ref[qq * np + p] : 0.0);
            };
            if (q < 0) v = make_double2(f00[off], 0.0);
            else if (hplane[nh + h]) v = make_double2(val(q), val(q + 1));
            else v = make_double2(val(q), 0.0);
        } else {
            v = make_double2((double)fields[i - (long long)nh * pstride], 0.0);
        }
        dst[i] = v;
    }
}

// FP32 split: the momentum profile each l >= 1 plane is stored relative to,
// the average over the cells of the uploaded state.  Partial sums over
// chunks of cells, then the chunks in order (deterministic); the profile is
// rounded to the plane type so that the stored deviation and every reader
// (stage, collision, moments, download) use one value.
constexpr int kProfChunks = 64;
// A plane keeps its profile only where the cell average carries at least
// this share of the plane's sum of squares (a large, nearly uniform
// harmonic); elsewhere the profile is zero and its loads are skipped.
constexpr double kProfileShare = 0.01;
__global__ void profile_partial_kernel(const double2* __restrict__ src, const int* __restrict__ hplane,
                                       long long cells, int np, double2* part, double2* part_sq) {
    const int h = blockIdx.x, ch = blockIdx.y;
    if (hplane[h] < 0) return;   // f00 is FP64
    const long long c0 = cells * ch / kProfChunks, c1 = cells * (ch + 1) / kProfChunks;
    for (int p = threadIdx.x; p < np; p += blockDim.x) {
        double sr = 0.0, si = 0.0, qr = 0.0, qi = 0.0;
        for (long long c = c0; c < c1; ++c) {
            const double2 v = src[((long long)h * cells + c) * np + p];
            sr += v.x;
            si += v.y;
            qr += v.x * v.x;
            qi += v.y * v.y;
        }
        part[((long long)h * kProfChunks + ch) * np + p] = make_double2(sr, si);
        part_sq[((long long)h * kProfChunks + ch) * np + p] = make_double2(qr, qi);
    }
}
// per harmonic (one CTA each): keep the profile if the cell average's sum of
// squares is at least kProfileShare of the harmonic's, else zero it
template <typename TS>
__global__ void profile_keep_kernel(const double2* __restrict__ part_sq, const int* __restrict__ hplane, int nh,
                                    long long cells, int np, double* ref64, TS* refts, int* keep) {
    const int h = blockIdx.x;
    const int q = hplane[h];
    if (q < 0) return;
    const bool cplx = hplane[nh + h] != 0;
    __shared__ double red[2][32];
    double mean = 0.0, tot = 0.0;
    for (int p = threadIdx.x; p < np; p += blockDim.x) {
        const double r = ref64[(long long)q * np + p];
        mean += r * r;
        double t = 0.0;
        for (int ch = 0; ch < kProfChunks; ++ch) {
            const double2 v = part_sq[((long long)h * kProfChunks + ch) * np + p];
            t += v.x + (cplx ? v.y : 0.0);
        }
        tot += t;
        if (cplx) {
            const double ri = ref64[(long long)(q + 1) * np + p];
            mean += ri * ri;
        }
    }
    for (int off = 16; off > 0; off >>= 1) {
        mean += __shfl_xor_sync(0xffffffffu, mean, off);
        tot += __shfl_xor_sync(0xffffffffu, tot, off);
    }
    if ((threadIdx.x & 31) == 0) { red[0][threadIdx.x >> 5] = mean; red[1][threadIdx.x >> 5] = tot; }
    __syncthreads();
    if (threadIdx.x == 0) {
        double m = 0.0, t = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) { m += red[0][w]; t += red[1][w]; }
        red[0][0] = (m * (double)cells >= kProfileShare * t && m > 0.0) ? 1.0 : 0.0;
    }
    __syncthreads();
    const bool k = red[0][0] != 0.0;
    if (threadIdx.x == 0) { keep[q] = k; if (cplx) keep[q + 1] = k; }
    if (!k)
        for (int p = threadIdx.x; p < np; p += blockDim.x) {
            ref64[(long long)q * np + p] = 0.0;
            refts[(long long)q * np + p] = TS(0);
            if (cplx) { ref64[(long long)(q + 1) * np + p] = 0.0; refts[(long long)(q + 1) * np + p] = TS(0); }
        }
}
template <typename TS>
__global__ void profile_final_kernel(const double2* __restrict__ part, const int* __restrict__ hplane, int nh,
                                     long long cells, int np, double* ref64, TS* refts) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < (long long)nh * np;
         i += (long long)gridDim.x * blockDim.x) {
        const int h = (int)(i / np), p = (int)(i - (long long)h * np);
        const int q = hplane[h];
        if (q < 0) continue;
        double sr = 0.0, si = 0.0;
        for (int ch = 0; ch < kProfChunks; ++ch) {
            const double2 v = part[((long long)h * kProfChunks + ch) * np + p];
            sr += v.x;
            si += v.y;
        }
        const TS r = (TS)(sr / (double)cells);
        ref64[(long long)q * np + p] = (double)r;
        refts[(long long)q * np + p] = r;
        if (hplane[nh + h]) {
            const TS ri = (TS)(si / (double)cells);
            ref64[(long long)(q + 1) * np + p] = (double)ri;
            refts[(long long)(q + 1) * np + p] = ri;
        }
    }
}

__global__ void clock_advance_kernel(Clock* c, double dt) { c->t += dt; }
__global__ void clock_set_kernel(Clock* c, double t, double t_ee, double t_eb) {
    c->t = t; c->t_ee = t_ee; c->t_eb = t_eb;
}
__global__ void clock_commit_kernel(Clock* c, int ee, int eb) {
    if (ee) c->t_ee = c->t;
    if (eb) c->t_eb = c->t;
}

template <typename T>
__global__ void nan_kernel(const T* x, long long n, int* status) {
    bool bad = false;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        if (!isfinite((double)x[i])) bad = true;
    if (__syncthreads_or(bad) && threadIdx.x == 0) atomicOr(status, 2);
}

int grid_for(long long n, int threads) {
    long long b = (n + threads - 1) / threads;
    if (b > 148 * 16) b = 148 * 16;
    if (b < 1) b = 1;
    return (int)b;
}

}  // namespace

cudaError_t launch_nan_check(const double* f00, const void* planes, int planes_fp32, long long n_f00,
                             long long n_planes, const void* fields, long long n_fields, int* status,
                             cudaStream_t s) {
    nan_kernel<double><<<grid_for(n_f00, 256), 256, 0, s>>>(f00, n_f00, status);
    if (planes_fp32) {
        if (n_planes) nan_kernel<float><<<grid_for(n_planes, 256), 256, 0, s>>>((const float*)planes, n_planes, status);
        nan_kernel<float><<<grid_for(n_fields, 256), 256, 0, s>>>((const float*)fields, n_fields, status);
    } else {
        if (n_planes) nan_kernel<double><<<grid_for(n_planes, 256), 256, 0, s>>>((const double*)planes, n_planes, status);
        nan_kernel<double><<<grid_for(n_fields, 256), 256, 0, s>>>((const double*)fields, n_fields, status);
    }
    return cudaGetLastError();
}

}  // namespace oshun

using namespace oshun;

struct oshun_ctx {
    oshun_cfg cfg;
    int nh = 0, nplanes = 0, mc = 0;
    long long cells = 0, pstride = 0;
    bool fp32 = false;
    size_t ts = 8;
    int dev = 0;

    double* f00[4] = {nullptr, nullptr, nullptr, nullptr};
    void* pl[4] = {nullptr, nullptr, nullptr, nullptr};
    void* fld[4] = {nullptr, nullptr, nullptr, nullptr};
    int cur = 0;

    // fault injection for tests (oshun_debug_inject_stage_timeout): armed for
    // the next oshun_rk4_step, active only while that step's stages launch
    bool inject_armed = false, inject_active = false;
    int inject_withhold = -1;
    unsigned long long inject_wait_ns = 1000000000ull;

    CoefLM* d_coef = nullptr;
    int* d_plane_of = nullptr;   // [(l0+1)*(m0+1)]
    std::vector<int> plane_of_host;   // the same map on the host
    int* d_plane_l = nullptr;    // [nplanes]
    int* d_plane_m = nullptr;    // [nplanes]
    int* d_hplane = nullptr;     // [2*nh]: plane of Re (or -1 for f00), complex flag
    int* d_seq = nullptr;        // [nh]: source harmonics in stream order, l | (m << 16)
    double* d_ptab = nullptr;    // inv_pr, vr, wj
    double* d_vtab = nullptr;    // vr, U4, U4m1, U2, U2m1, U1, U1m1, U3, Qn, Pn, v^5, v^7
    double* d_dense_ws = nullptr;
    int dense_blocks = 0;
    int* d_status = nullptr;
    double* d_jw = nullptr;      // [cells][3][8] current partial sums of the pipelined stage
    Clock* d_clock = nullptr;
    double2* d_stage = nullptr;  // host-layout staging for transfers and slopes
    std::vector<CoefLM> coef_host;   // the coupling table on the host
    // FP32 split: the l >= 1 planes store f minus a momentum profile per plane
    // (the cell average at upload), FP64 and plane-type copies [nplanes][np]
    bool use_profile = false;
    double* d_ref64 = nullptr;
    void* d_ref_ts = nullptr;
    double2* d_refpart = nullptr;   // per-chunk sums, then per-chunk sums of squares
    int* d_refkeep = nullptr;       // [nplanes]: the plane keeps a nonzero profile
    // implicit electric field (built on first use): coupling tables of
    // ImpEx, ImpEx1D, ImpEy/z and Exyz1D; J0, J(DEx), J(DEy), J(DEz), JN, DE,
    // EN ([3][cells] each) and p^3/gamma; the probe field; the zero count
    CoefLM* d_coef_imp[4] = {nullptr, nullptr, nullptr, nullptr};
    double* d_imp = nullptr;
    void* d_fe = nullptr;
    int* d_zeros = nullptr;
    int imp_zeros = 0;           // cells left with a zero determinant by the last implicit-E solve
    bool imp_zero_seen = false;  // some implicit-E solve since the last status read left one
    double* d_mom_tab = nullptr; // moments: p, 1/gamma, pow tables [7][np] (built on first use)
    float* d_mom = nullptr;      // moments: [kMomCount + 1][cells] (the last plane is scratch)
    // x boundary (OSHUN_XB_*) and the x halo column sets of the next stage's input
    int xb = 0;
    unsigned char* d_hx = nullptr;
    long long hx_side = 0, hx_pl = 0, hx_fld = 0;
    int stage_next = 1;          // the RK4 stage oshun_step_stage runs next (1..4)

    cudaStream_t stream = nullptr;
    bool own_stream = false;
    cudaGraphExec_t graph[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};  // [parity][collisions]
    bool graphs_ok = true;

    // host mirrors of the clocks (the reference's Runge_Kutta_4::t, Explicit_EC_FP::t, Euler_Backward::t)
    double t = 0.0, t_ee = 0.0, t_eb = 0.0;

    int collide_chunk = 0;
    size_t collide_smem = 0;
    int collide_blocks = 0;
    int tri_cpc = 0;       // cells per CTA of the tridiagonal collision kernel (0: staged-chunk kernel)
    int tri_blocks = 0;

    // constants
    double dp = 0, idx = 0, idy = 0, g00_s = 0, g00_inv = 0, g00_gr = 0, c_kpre = 0, kpre = 0;

    template <typename TS>
    StageArgs<TS> stage_args(int in_set, int out_set, int mode) const;
};

namespace {

#define CK(call)                                                                      \
    do {                                                                              \
        cudaError_t e_ = (call);                                                      \
        if (e_ != cudaSuccess) {                                                      \
            set_error(std::string(#call) + ": " + cudaGetErrorString(e_));            \
            return OSHUN_ERR_CUDA;                                                    \
        }                                                                             \
    } while (0)

double axis_point(int i, int n, double lo, double hi) {
    const double step = (hi - lo) / (double)(n - 1);
    return (double)i * step + lo;
}
double local_dx(int nglob, double lo, double hi) {
    const double dg = axis_point(1, nglob, lo, hi) - axis_point(0, nglob, lo, hi);
    const double x0 = axis_point(0, nglob, lo, hi) - 4.0 * dg;
    const double x1 = x0 + dg;
    return x1 - x0;
}

int num_harmonics(int l0, int m0) { return ((m0 + 1) * (2 * l0 - m0 + 2)) / 2; }

int ind(int l, int m, int m0) {
    return (l < m0 + 1) ? (l * (l + 1)) / 2 + m : l * (m0 + 1) - (m0 * (m0 + 1)) / 2 + m;
}

const double kRe = 2.8179402894e-13;  // classical electron radius in cm (def-FokkerPlanck.cpp:136)

// Reference y-advection chain factor for m >= 2 (OSHUN-1/def-VlasovMax.cpp:901-946):
// the loop multiplier is divided by C1[m+1] where C1[l-1] is meant (line 918) and
// carries into the next m.  Returned factor multiplies every y coupling of (l,m).
double yadv_chain(int l, int m, int l0, int m0, double idy, bool keep) {
    if (!keep || m < 2) return 1.0;
    auto C1 = [&](int ll) { return (-0.5) * idy / (2.0 * ll + 1.0); };
    double R = 1.0;
    for (int mm = 2; mm <= m; ++mm) {
        if (mm == m0) return R;
        if (mm + 1 >= l0) {
            if (mm == m) return R;
            continue;
        }
        double q = R, at_l = R;
        for (int ll = mm + 2; ll <= l0 - 1; ++ll) {
            if (ll > mm + 2) q = q * (C1(ll - 1) / C1(mm + 1));
            if (mm == m && ll == l) at_l = q;
        }
        if (mm == m) {
            if (l <= mm + 1) return R;
            if (l == l0) return q;
            return at_l;
        }
        R = q;
    }
    return R;
}

int validate(const oshun_cfg* c) {
    if (!c) { set_error("cfg is NULL"); return OSHUN_ERR_ARG; }
    if (c->l0 < 1 || c->m0 < 0 || c->m0 > c->l0) { set_error("need 1 <= l0 and 0 <= m0 <= l0"); return OSHUN_ERR_ARG; }
    if (c->m0 > kMaxM0) { set_error("m0 above the compiled maximum of 8"); return OSHUN_ERR_UNSUPPORTED; }
    if (c->nump < 3 || c->nump > kMaxNp) { set_error("need 3 <= nump <= 1024"); return OSHUN_ERR_ARG; }
    if (c->numx < 1 || c->numy < 1) { set_error("need numx, numy >= 1"); return OSHUN_ERR_ARG; }
    if (c->numx < 2 && c->numy < 2) { set_error("need at least two cells"); return OSHUN_ERR_ARG; }
    if (!(c->pmax > c->pmin) || !(c->pmin > 0.0)) { set_error("need 0 < pmin < pmax"); return OSHUN_ERR_ARG; }
    if (!(c->xmax > c->xmin) || (c->numy > 1 && !(c->ymax > c->ymin))) { set_error("bad x/y extent"); return OSHUN_ERR_ARG; }
    if (!(c->dt > 0.0) || !(c->small_dt > 0.0)) { set_error("need dt > 0 and small_dt > 0"); return OSHUN_ERR_ARG; }
    if (!(c->density_np > 0.0)) { set_error("need density_np > 0"); return OSHUN_ERR_ARG; }
    if (c->precision != OSHUN_FP64 && c->precision != OSHUN_FP32_SPLIT) { set_error("bad precision"); return OSHUN_ERR_ARG; }
    return OSHUN_OK;
}

int pick_mc(int m0) {
    const int caps[] = {0, 1, 2, 3, 4, 6, 8};
    for (int c : caps)
        if (c >= m0) return c;
    return -1;
}

}  // namespace

template <typename TS>
StageArgs<TS> oshun_ctx::stage_args(int in_set, int out_set, int mode) const {
    StageArgs<TS> a;
    std::memset(&a, 0, sizeof(a));
    a.f00_in = f00[in_set]; a.pl_in = (const TS*)pl[in_set]; a.fld_in = (const TS*)fld[in_set];
    a.pl_ref = use_profile ? (const TS*)d_ref_ts : nullptr;
    a.pl_keep = use_profile ? d_refkeep : nullptr;
    if (xb != OSHUN_XB_PERIODIC) { a.hx = d_hx; a.hx_side = hx_side; a.hx_pl = hx_pl; a.hx_fld = hx_fld; }
    a.coef = d_coef; a.plane_of = d_plane_of;
    a.inv_pr = d_ptab; a.vr = d_ptab + cfg.nump; a.wj = d_ptab + 2 * cfg.nump;
    a.cells = cells; a.pstride = pstride;
    a.np = cfg.nump; a.nx = cfg.numx; a.ny = cfg.numy; a.l0 = cfg.l0; a.m0 = cfg.m0;
    a.mode = mode;
    a.g00_s = g00_s; a.g00_inv = g00_inv; a.g00_gr = g00_gr;
    a.idx = idx; a.idy = idy;
    a.seq = d_seq; a.nh = nh; a.err = d_status;
    a.parts = kPartAll;
    a.wait_ns = inject_active ? inject_wait_ns : 1000000000ull;
    a.withhold = inject_active ? inject_withhold : -1;
    a.jw = d_jw;
    (void)out_set;
    return a;
}

namespace {

int build_tables(oshun_ctx* h) {
    const oshun_cfg& c = h->cfg;
    const int np = c.nump, l0 = c.l0, m0 = c.m0;
    std::vector<double> pr(np), inv_pr(np), vr(np);
    for (int i = 0; i < np; ++i) {
        pr[i] = axis_point(i, np, c.pmin, c.pmax);
        inv_pr[i] = 1.0 / pr[i];
        vr[i] = pr[i] / std::sqrt(1.0 + pr[i] * pr[i]);
    }
    const double dp = pr[1] - pr[0];
    h->dp = dp;
    h->idx = -1.0 / (2.0 * local_dx(c.numx, c.xmin, c.xmax));
    h->idy = c.numy > 1 ? -1.0 / (2.0 * local_dx(c.numy, c.ymin, c.ymax)) : 0.0;
    const double p0 = pr[0], p1 = pr[1];
    h->g00_s = p0 * p0 / (p1 * p1);
    h->g00_inv = 1.0 / (1.0 - h->g00_s);
    h->g00_gr = -4.0 * dp * p0 / (p1 * p1);

    // current quadrature (Current ctor and Jxyz, def-VlasovMax.cpp:670-712)
    std::vector<double> wj(np);
    double small = p0;
    small *= small; small *= small; small *= p0; small *= 0.2; small *= 1.0 / p1;
    for (int i = 0; i < np; ++i) {
        const double q = pr[i];
        const double p3og = (q * q) * (q / std::sqrt(1.0 + q * q));
        double w = (i == 0 || i == np - 1) ? 0.5 * dp * p3og : dp * p3og;
        if (i == 1) w += small * p3og;
        wj[i] = w * (4.0 * M_PI / 3.0);
    }

    // coupling tables
    const bool keep_chain = !(c.flags & OSHUN_FLAG_FIX_YADV_CHAIN);
    std::vector<CoefLM> coef((size_t)(l0 + 1) * (m0 + 1));
    std::memset(coef.data(), 0, sizeof(CoefLM) * coef.size());
    auto exists = [&](int l, int m) { return l >= 0 && l <= l0 && m >= 0 && m <= m0 && m <= l; };
    const double hdp = 0.5 / dp, qdp = 0.25 / dp;
    for (int l = 0; l <= l0; ++l)
        for (int m = 0; m <= std::min(l, m0); ++m) {
            CoefLM& k = coef[(size_t)l * (m0 + 1) + m];
            const double L = l, M = m;
            // E field (ElectricField ctor, def-VlasovMax.cpp:97-140)
            const double A1 = (l == 0) ? -1.0 * hdp : (L + 1.0 - M) * L / ((2.0 * L + 1.0) * (L + 1.0)) * hdp;
            const double A2 = -(L + M) / (2.0 * L + 1.0) * hdp;
            const double C1 = (l == 0) ? -qdp : qdp * L / ((2.0 * L + 1.0) * (L + 1.0));
            const double C3 = qdp / (2.0 * L + 1.0);
            const double B1 = (-hdp) * L * L / (2.0 * L + 1.0);
            const double B2 = (-hdp) * L * (L + 1.0) / (2.0 * L + 1.0);
            const double C2 = (-qdp) * L * (L - M + 2.0) * (L - M + 1.0) / ((2.0 * L + 1.0) * (L + 1.0));
            const double C4 = (-qdp) * (L + M - 1.0) * (L + M) / (2.0 * L + 1.0);
            k.ex_g = exists(l + 1, m) ? A1 : 0.0;
            k.ex_h = exists(l - 1, m) ? A2 : 0.0;
            k.em_g = exists(l + 1, m + 1) ? C1 : 0.0;
            k.em_h = exists(l - 1, m + 1) ? C3 : 0.0;
            if (m == 1) {
                k.ep_h = exists(l - 1, 0) ? B2 : 0.0;
                k.ep_g = exists(l + 1, 0) ? B1 : 0.0;
            } else if (m >= 2) {
                k.ep_h = exists(l - 1, m - 1) ? C4 : 0.0;
                k.ep_g = exists(l + 1, m - 1) ? C2 : 0.0;
            }
            // advection (Spatial_Advection ctor, def-VlasovMax.cpp:775-826)
            const double ix = h->idx, iy = h->idy;
            k.ax_p = exists(l + 1, m) ? ix * (-1.0) * (L - M + 1.0) / (2.0 * L + 1.0) : 0.0;
            k.ax_m = exists(l - 1, m) ? ix * (-1.0) * (L + M) / (2.0 * L + 1.0) : 0.0;
            if (c.numy > 1) {
                const double q = yadv_chain(l, m, l0, m0, iy, keep_chain);
                const double yC1 = (-0.5) * iy / (2.0 * L + 1.0);
                const double yC3 = -yC1;
                const double yB1 = iy * (L + 1.0) * L / (2.0 * L + 1.0);
                const double yB2 = -yB1;
                const double yC2 = iy * 0.5 * (L + 2.0 - M) * (L - M + 1.0) / (2.0 * L + 1.0);
                const double yC4 = iy * (-0.5) * (L + M - 1.0) * (L + M) / (2.0 * L + 1.0);
                k.ay_pp = exists(l + 1, m + 1) ? q * yC1 : 0.0;
                k.ay_mp = exists(l - 1, m + 1) ? q * yC3 : 0.0;
                if (m == 1) {
                    k.ay_mm = exists(l - 1, 0) ? yB2 : 0.0;
                    k.ay_pm = exists(l + 1, 0) ? yB1 : 0.0;
                } else if (m >= 2) {
                    k.ay_mm = exists(l - 1, m - 1) ? q * yC4 : 0.0;
                    k.ay_pm = exists(l + 1, m - 1) ? q * yC2 : 0.0;
                }
            }
            // B field (MagneticField ctor, def-VlasovMax.cpp:563-589)
            if (m == 1) k.b_m = -L * (L + 1.0);
            else if (m >= 2) k.b_m = (-0.5) * (L + 1.0 - M) * (L + M);
            // G/H (MakeGH, def-VlasovMax.cpp:496-515; Hp0, :145-147)
            if (l >= 1) {
                k.gfac = -(2.0 * L + 1.0) / L;
                k.invpax = -2.0 * (L + 1.0) * dp;
                double hp = 1.0 / p0;
                for (int kk = 1; kk <= l; ++kk) hp = hp * (p0 / p1) * (2.0 * kk + 1.0) / (2.0 * kk - 1);
                k.hp0 = hp * (-2.0 * dp);
            }
        }

    // plane maps
    std::vector<int> plane_of((size_t)(l0 + 1) * (m0 + 1), -1), plane_l, plane_m;
    std::vector<int> hplane(2 * (size_t)h->nh, 0);
    int q = 0;
    for (int l = 0; l <= l0; ++l)
        for (int m = 0; m <= std::min(l, m0); ++m) {
            const int hi = ind(l, m, m0);
            if (l == 0) { hplane[hi] = -1; continue; }
            plane_of[(size_t)l * (m0 + 1) + m] = q;
            hplane[hi] = q;
            hplane[h->nh + hi] = m > 0 ? 1 : 0;
            const int ncomp = m > 0 ? 2 : 1;
            for (int k = 0; k < ncomp; ++k) { plane_l.push_back(l); plane_m.push_back(m); }
            q += ncomp;
        }
    h->nplanes = q;

    // velocity grid of the collision operators (def-FokkerPlanck.cpp:143-172, 790-803)
    std::vector<double> vt((size_t)12 * np, 0.0);
    double* V = vt.data();
    for (int i = 0; i < np; ++i) V[i] = vr[i];
    for (int i = 1; i < np; ++i) {
        const double dv = vr[i] - vr[i - 1];
        V[np + i] = 0.5 * std::pow(vr[i], 4) * dv;
        V[2 * np + i] = 0.5 * std::pow(vr[i - 1], 4) * dv;
        V[3 * np + i] = 0.5 * vr[i] * vr[i] * dv;
        V[4 * np + i] = 0.5 * vr[i - 1] * vr[i - 1] * dv;
        V[5 * np + i] = 0.5 * vr[i] * dv;
        V[6 * np + i] = 0.5 * vr[i - 1] * dv;
    }
    for (int i = 0; i < np; ++i) {
        V[7 * np + i] = std::pow(vr[i], 3);
        V[10 * np + i] = std::pow(vr[i], 5);
        V[11 * np + i] = std::pow(vr[i], 7);
    }
    V[8 * np + 0] = 1.0 / ((vr[0] * vr[0] * vr[1]) / 2.0);
    for (int i = 1; i < np - 1; ++i) V[8 * np + i] = 1.0 / (vr[i] * vr[i] * (vr[i + 1] - vr[i - 1]) / 2.0);
    for (int i = 0; i < np - 1; ++i) V[9 * np + i] = 1.0 / ((vr[i + 1] - vr[i]) / 2.0 * (vr[i + 1] + vr[i]));
    const double kp = std::sqrt(4.0 * M_PI * c.density_np * kRe);
    h->c_kpre = 4.0 * M_PI / 3.0 * kRe * kp;
    h->kpre = kRe * kp;

    std::vector<double> ptab((size_t)3 * np);
    for (int i = 0; i < np; ++i) { ptab[i] = inv_pr[i]; ptab[np + i] = vr[i]; ptab[2 * np + i] = wj[i]; }

    CK(cudaMalloc(&h->d_coef, sizeof(CoefLM) * coef.size()));
    CK(cudaMemcpy(h->d_coef, coef.data(), sizeof(CoefLM) * coef.size(), cudaMemcpyHostToDevice));
    h->coef_host = coef;
    // padded to 16 bytes: batched launches bulk-copy the map
    const size_t plane_bytes = (sizeof(int) * plane_of.size() + 15) / 16 * 16;
    CK(cudaMalloc(&h->d_plane_of, plane_bytes));
    CK(cudaMemset(h->d_plane_of, 0xff, plane_bytes));
    CK(cudaMemcpy(h->d_plane_of, plane_of.data(), sizeof(int) * plane_of.size(), cudaMemcpyHostToDevice));
    h->plane_of_host = plane_of;
    const size_t npl = std::max<size_t>(1, plane_l.size());
    CK(cudaMalloc(&h->d_plane_l, sizeof(int) * npl));
    CK(cudaMalloc(&h->d_plane_m, sizeof(int) * npl));
    if (!plane_l.empty()) {
        CK(cudaMemcpy(h->d_plane_l, plane_l.data(), sizeof(int) * plane_l.size(), cudaMemcpyHostToDevice));
        CK(cudaMemcpy(h->d_plane_m, plane_m.data(), sizeof(int) * plane_m.size(), cudaMemcpyHostToDevice));
    }
    std::vector<int> seq;
    for (int l = 0; l <= l0; ++l)
        for (int m = 0; m <= std::min(l, m0); ++m) seq.push_back(l | (m << 16));
    CK(cudaMalloc(&h->d_seq, sizeof(int) * seq.size()));
    CK(cudaMemcpy(h->d_seq, seq.data(), sizeof(int) * seq.size(), cudaMemcpyHostToDevice));
    CK(cudaMalloc(&h->d_hplane, sizeof(int) * hplane.size()));
    CK(cudaMemcpy(h->d_hplane, hplane.data(), sizeof(int) * hplane.size(), cudaMemcpyHostToDevice));
    CK(cudaMalloc(&h->d_ptab, sizeof(double) * ptab.size()));
    CK(cudaMemcpy(h->d_ptab, ptab.data(), sizeof(double) * ptab.size(), cudaMemcpyHostToDevice));
    CK(cudaMalloc(&h->d_vtab, sizeof(double) * vt.size()));
    CK(cudaMemcpy(h->d_vtab, vt.data(), sizeof(double) * vt.size(), cudaMemcpyHostToDevice));
    return OSHUN_OK;
}

int launch_stage(oshun_ctx* h, int in_set, int B_set, int A_set, int out_set, int mode, int first, double c1,
                 double c2) {
    cudaError_t e;
    if (h->fp32) {
        StageArgs<float> a = h->stage_args<float>(in_set, out_set, mode);
        a.f00_B = h->f00[B_set]; a.pl_B = (const float*)h->pl[B_set]; a.fld_B = (const float*)h->fld[B_set];
        a.f00_A = h->f00[A_set]; a.pl_A = (float*)h->pl[A_set]; a.fld_A = (float*)h->fld[A_set];
        if (out_set >= 0) { a.f00_out = h->f00[out_set]; a.pl_out = (float*)h->pl[out_set]; a.fld_out = (float*)h->fld[out_set]; }
        a.first = first; a.c1 = c1; a.c2 = c2;
        e = launch_stage_fp32(a, h->mc, h->stream);
    } else {
        StageArgs<double> a = h->stage_args<double>(in_set, out_set, mode);
        a.f00_B = h->f00[B_set]; a.pl_B = (const double*)h->pl[B_set]; a.fld_B = (const double*)h->fld[B_set];
        a.f00_A = h->f00[A_set]; a.pl_A = (double*)h->pl[A_set]; a.fld_A = (double*)h->fld[A_set];
        if (out_set >= 0) { a.f00_out = h->f00[out_set]; a.pl_out = (double*)h->pl[out_set]; a.fld_out = (double*)h->fld[out_set]; }
        a.first = first; a.c1 = c1; a.c2 = c2;
        e = launch_stage_fp64(a, h->mc, h->stream);
    }
    if (e != cudaSuccess) { set_error(std::string("rk stage launch: ") + cudaGetErrorString(e)); return OSHUN_ERR_CUDA; }
    return OSHUN_OK;
}

HaloGrid halo_grid(const oshun_ctx* h) {
    HaloGrid g;
    g.nx = h->cfg.numx; g.ny = h->cfg.numy; g.np = h->cfg.nump; g.nplanes = h->nplanes;
    g.pstride = h->pstride; g.cells = h->cells;
    g.off_pl = h->hx_pl; g.off_fld = h->hx_fld;
    g.plane_l = h->d_plane_l; g.plane_m = h->d_plane_m;
    return g;
}

// the halo columns of set `set` from its own edge columns: mirrored x
// boundaries (sameNode_mirror_X, def-Parallel.cpp:1160-1206)
int fill_mirror(oshun_ctx* h, int set) {
    if (h->xb != OSHUN_XB_MIRROR) return OSHUN_OK;
    CK(launch_halo_columns(h->f00[set], h->pl[set], h->fld[set], halo_grid(h), h->fp32, h->d_hx,
                           h->d_hx + h->hx_side, 1, h->stream));
    return OSHUN_OK;
}

// RK4 stage k (1..4) of Runge_Kutta_4::advance_p1 (def-RK.cpp:116-142) on set
// cur: inputs cur, Sa, Sb, Sa; the fourth writes the step's result to cur ^ 1
int stage_input(const oshun_ctx* h, int k) { return k == 1 ? h->cur : (k == 3 ? 3 : 2); }
int enqueue_stage(oshun_ctx* h, int k) {
    const double dt = h->cfg.dt;
    const int B = h->cur, A = h->cur ^ 1, Sa = 2, Sb = 3;
    int rc = fill_mirror(h, stage_input(h, k));
    if (rc) return rc;
    switch (k) {
        case 1: return launch_stage(h, B, B, A, Sa, 0, 1, 0.5 * dt, 1.0 / 3.0);
        case 2: return launch_stage(h, Sa, B, A, Sb, 0, 0, 0.5 * dt, 2.0 / 3.0);
        case 3: return launch_stage(h, Sb, B, A, Sa, 0, 0, dt, 1.0 / 3.0);
        default: return launch_stage(h, Sa, B, A, -1, 0, 0, dt / 6.0, 1.0);
    }
}

// Runge_Kutta_4::advance_p1 on set cur -> set cur ^ 1
int enqueue_rk4(oshun_ctx* h) {
    int rc;
    for (int k = 1; k <= 4; ++k)
        if ((rc = enqueue_stage(h, k))) return rc;
    return OSHUN_OK;
}

CollideArgs collide_args(oshun_ctx* h, int do_ee, int do_l1, int do_lm, int nsub, double hsub, double Dt,
                         int set = -1) {
    CollideArgs a;
    std::memset(&a, 0, sizeof(a));
    const oshun_cfg& c = h->cfg;
    const int np = c.nump;
    if (set < 0) set = h->cur;
    a.f00 = h->f00[set];
    a.planes = h->pl[set];
    a.pl_ref = h->use_profile ? h->d_ref64 : nullptr;
    a.pl_ref32 = h->use_profile ? (const float*)h->d_ref_ts : nullptr;
    a.pl_keep = h->use_profile ? h->d_refkeep : nullptr;
    a.planes_fp32 = h->fp32 ? 1 : 0;
    a.plane_of = h->d_plane_of; a.plane_l = h->d_plane_l; a.plane_m = h->d_plane_m;
    a.nplanes = h->nplanes;
    a.cells = h->cells; a.pstride = h->pstride;
    a.np = np; a.l0 = c.l0; a.m0 = c.m0;
    a.mmax_coll = c.if_implicit1D ? 0 : c.m0;
    a.do_ee = do_ee; a.do_l1 = do_l1; a.do_lm = do_lm;
    a.if_tridiagonal = c.if_tridiagonal;
    a.nsub = nsub; a.hsub = hsub; a.Dt = Dt;
    a.ee_implicit = (c.flags & OSHUN_FLAG_IMPLICIT_EE) ? kEeImplicitSweeps : 0;
    a.NB = c.NB_algorithms;
    a.density_np = c.density_np; a.Zeta = c.Zeta;
    a.c_kpre = h->c_kpre; a.kpre = h->kpre;
    const double* V = h->d_vtab;
    a.vr = V; a.U4 = V + np; a.U4m1 = V + 2 * np; a.U2 = V + 3 * np; a.U2m1 = V + 4 * np;
    a.U1 = V + 5 * np; a.U1m1 = V + 6 * np; a.U3 = V + 7 * np; a.Qn = V + 8 * np; a.Pn = V + 9 * np;
    a.V5 = V + 10 * np; a.V7 = V + 11 * np;
    a.chunk = h->collide_chunk;
    a.dense_ws = h->d_dense_ws;
    a.status = h->d_status;
    return a;
}

int launch_collide_args(oshun_ctx* h, const CollideArgs& a0) {
    cudaError_t e;
    CollideArgs a = a0;
    if (a.do_ee && a.ee_implicit > 0) {
        // the backward-Euler e-e step in its own launch, then the f_lm solves
        e = launch_ee_implicit(a, h->stream);
        if (e != cudaSuccess) { set_error(std::string("e-e launch: ") + cudaGetErrorString(e)); return OSHUN_ERR_CUDA; }
        a.do_ee = 0;
        if (!a.do_l1 && !a.do_lm) return OSHUN_OK;
    }
    if (h->tri_cpc > 0)
        e = launch_collide_tri(a, h->stream, h->tri_cpc, h->tri_blocks);
    else
        e = launch_collide(a, h->stream, h->collide_smem, h->collide_blocks);
    if (e != cudaSuccess) { set_error(std::string("collide launch: ") + cudaGetErrorString(e)); return OSHUN_ERR_CUDA; }
    return OSHUN_OK;
}

int enqueue_collide(oshun_ctx* h, int do_ee, int do_l1, int do_lm, int nsub, double hsub, double Dt) {
    return launch_collide_args(h, collide_args(h, do_ee, do_l1, do_lm, nsub, hsub, Dt));
}

// One small step of the reference's main loop (main.cpp:77-107) on the device
// clock, graph-capturable: RK4 on set cur, t += dt, then (collisions) the e-e
// substeps and the implicit f1/f_lm solves with nsub, hsub, Dt from the
// device clock, t_ee = t_eb = t.  Flips h->cur.
int enqueue_step_device(oshun_ctx* h, int collisions) {
    int rc = enqueue_rk4(h);
    if (rc) return rc;
    h->cur ^= 1;
    clock_advance_kernel<<<1, 1, 0, h->stream>>>(h->d_clock, h->cfg.dt);
    CK(cudaGetLastError());
    if (collisions) {
        CollideArgs a = collide_args(h, 1, 1, 1, 0, 0.0, 0.0);
        a.clock = reinterpret_cast<const double*>(h->d_clock);
        a.small_dt = h->cfg.small_dt;
        if ((rc = launch_collide_args(h, a))) return rc;
        clock_commit_kernel<<<1, 1, 0, h->stream>>>(h->d_clock, 1, 1);
        CK(cudaGetLastError());
    }
    return OSHUN_OK;
}

// the reference's clock arithmetic for one small step ending at t_new
void collide_params(const oshun_ctx* h, double t_new, int* nsub, double* hsub, double* Dt) {
    *nsub = (int)((t_new - h->t_ee) / h->cfg.small_dt) + 1;   // def-FokkerPlanck.cpp:598-599
    *hsub = (t_new - h->t_ee) / (double)(*nsub);
    *Dt = t_new - h->t_eb;                                     // def-FokkerPlanck.cpp:1277,1297
}

// ---- implicit electric field: Runge_Kutta_2_Imp and Implicit_E_Field ----

// The coupling tables of the implicit actions, subsets of the explicit E
// couplings (same closed-form coefficients):
//   [0] ImpEx    Ex G from (0,0) (1,0) (1,1), Ex H from (1,0) (2,0) (3,0) (2,1) (3,1)
//                (ElectricField::Implicit_Ex, def-VlasovMax.cpp:157-198)
//   [1] ImpEx1D  the m = 0 part of [0] (Implicit_Ex1D, :202-228)
//   [2] ImpEy/z  every E_+- coupling into l <= 2 (Implicit_Eyz, :233-292)
//   [3] Exyz1D   Ex couplings among m = 0 harmonics (Exyz1D, :299-341)
int build_implicit(oshun_ctx* h) {
    const oshun_cfg& c = h->cfg;
    const int l0 = c.l0, m0 = c.m0, np = c.nump;
    auto keep = [&](int l, int m, int which) {
        CoefLM k{};
        const CoefLM& e = h->coef_host[(size_t)l * (m0 + 1) + m];
        k.gfac = e.gfac; k.invpax = e.invpax; k.hp0 = e.hp0;
        auto in = [&](std::initializer_list<std::pair<int, int>> lst) {
            for (auto& q : lst)
                if (q.first == l && q.second == m) return true;
            return false;
        };
        switch (which) {
            case 0:
                if (in({{0, 0}, {1, 0}, {1, 1}})) k.ex_g = e.ex_g;
                if (in({{1, 0}, {2, 0}, {3, 0}, {2, 1}, {3, 1}})) k.ex_h = e.ex_h;
                break;
            case 1:
                if (in({{0, 0}, {1, 0}})) k.ex_g = e.ex_g;
                if (in({{1, 0}, {2, 0}, {3, 0}})) k.ex_h = e.ex_h;
                break;
            case 2:
                if (in({{0, 0}, {1, 0}, {1, 1}})) k.em_g = e.em_g;
                if (in({{2, 0}, {3, 0}, {3, 1}})) k.em_h = e.em_h;
                if (in({{1, 1}, {2, 1}, {3, 1}, {2, 2}, {3, 2}}) || (m0 > 2 && l == 3 && m == 3)) k.ep_h = e.ep_h;
                if (in({{1, 1}})) k.ep_g = e.ep_g;
                break;
            default:
                if (m == 0) { k.ex_g = e.ex_g; k.ex_h = e.ex_h; }
                break;
        }
        return k;
    };
    for (int which = 0; which < 4; ++which) {
        std::vector<CoefLM> t((size_t)(l0 + 1) * (m0 + 1));
        std::memset(t.data(), 0, sizeof(CoefLM) * t.size());
        for (int l = 0; l <= l0; ++l)
            for (int m = 0; m <= std::min(l, m0); ++m) t[(size_t)l * (m0 + 1) + m] = keep(l, m, which);
        CK(cudaMalloc(&h->d_coef_imp[which], sizeof(CoefLM) * t.size()));
        CK(cudaMemcpy(h->d_coef_imp[which], t.data(), sizeof(CoefLM) * t.size(), cudaMemcpyHostToDevice));
    }
    // p^3/gamma of Current_xyz (def-ImplicitE.cpp:59-69)
    std::vector<double> w(np);
    for (int i = 0; i < np; ++i) {
        const double p = axis_point(i, np, c.pmin, c.pmax);
        w[i] = (p * p) * (p / std::sqrt(1.0 + p * p));
    }
    CK(cudaMalloc(&h->d_imp, sizeof(double) * ((size_t)21 * h->cells + np)));
    CK(cudaMemcpy(h->d_imp + 21 * h->cells, w.data(), sizeof(double) * np, cudaMemcpyHostToDevice));
    CK(cudaMalloc(&h->d_fe, h->ts * 6 * (size_t)h->cells));
    CK(cudaMalloc(&h->d_zeros, sizeof(int)));
    return OSHUN_OK;
}

ImplicitArgs implicit_args(const oshun_ctx* h) {
    const oshun_cfg& c = h->cfg;
    ImplicitArgs a;
    std::memset(&a, 0, sizeof(a));
    for (int i = 0; i < 4; ++i) a.planes[i] = h->pl[i];
    a.pl_ref = h->use_profile ? h->d_ref64 : nullptr;
    a.cells = h->cells; a.pstride = h->pstride;
    a.np = c.nump; a.nx = c.numx; a.ny = c.numy;
    a.q10 = h->plane_of_host[(size_t)(c.m0 + 1)];
    a.q11 = c.m0 >= 1 ? h->plane_of_host[(size_t)(c.m0 + 1) + 1] : -1;
    a.fp32 = h->fp32 ? 1 : 0;
    a.one_d = c.if_implicit1D ? 1 : 0;
    a.p3og = h->d_imp + 21 * h->cells;
    const double p0 = axis_point(0, c.nump, c.pmin, c.pmax), p1 = axis_point(1, c.nump, c.pmin, c.pmax);
    double small = p0;
    small *= small; small *= small; small *= p0; small *= 0.2; small *= 1.0 / p1;
    a.dp = h->dp; a.small = small;
    a.c4 = (-4.0) * M_PI / 3.0;
    a.c8 = (-8.0) * M_PI / 3.0;
    a.idx = h->idx; a.idy = h->idy;
    a.eps = 16.0 * DBL_EPSILON;
    a.large_eps = std::sqrt(a.eps);
    return a;
}

// one stage launch of a partial right-hand side (the implicit actions)
int launch_stage_part(oshun_ctx* h, int in_set, int B_set, int A_set, int out_set, int first, double c1, double c2,
                      int parts, const CoefLM* coef, const void* fld_in) {
    cudaError_t e;
    if (h->fp32) {
        StageArgs<float> a = h->stage_args<float>(in_set, out_set, 0);
        a.f00_B = h->f00[B_set]; a.pl_B = (const float*)h->pl[B_set]; a.fld_B = (const float*)h->fld[B_set];
        a.f00_A = h->f00[A_set]; a.pl_A = (float*)h->pl[A_set]; a.fld_A = (float*)h->fld[A_set];
        if (out_set >= 0) { a.f00_out = h->f00[out_set]; a.pl_out = (float*)h->pl[out_set]; a.fld_out = (float*)h->fld[out_set]; }
        a.first = first; a.c1 = c1; a.c2 = c2; a.parts = parts; a.coef = coef;
        if (fld_in) a.fld_in = (const float*)fld_in;
        e = launch_stage_fp32(a, h->mc, h->stream);
    } else {
        StageArgs<double> a = h->stage_args<double>(in_set, out_set, 0);
        a.f00_B = h->f00[B_set]; a.pl_B = (const double*)h->pl[B_set]; a.fld_B = (const double*)h->fld[B_set];
        a.f00_A = h->f00[A_set]; a.pl_A = (double*)h->pl[A_set]; a.fld_A = (double*)h->fld[A_set];
        if (out_set >= 0) { a.f00_out = h->f00[out_set]; a.pl_out = (double*)h->pl[out_set]; a.fld_out = (double*)h->fld[out_set]; }
        a.first = first; a.c1 = c1; a.c2 = c2; a.parts = parts; a.coef = coef;
        if (fld_in) a.fld_in = (const double*)fld_in;
        e = launch_stage_fp64(a, h->mc, h->stream);
    }
    if (e != cudaSuccess) { set_error(std::string("rk2 stage launch: ") + cudaGetErrorString(e)); return OSHUN_ERR_CUDA; }
    return OSHUN_OK;
}

// One Runge_Kutta_2_Imp update (def-RK.cpp:463-493 and the advance_IE*
// forms, :515-588) from set S into set T through set U:
//   Y0 = Y; Yh = F(Y0) h; Y0 += Yh; Yh *= 0.5; Y += Yh; Yh = F(Y0) h/2; Y += Yh
int enqueue_rk2(oshun_ctx* h, int S, int T, int U, int parts, const CoefLM* coef, const void* fld_in) {
    const double dt = h->cfg.dt;
    int rc = launch_stage_part(h, S, S, T, U, 1, dt, 0.5, parts, coef, fld_in);
    if (rc) return rc;
    return launch_stage_part(h, U, S, T, -1, 0, 0.5 * dt, 1.0, parts, coef, fld_in);
}

// Implicit_E_Field::advance (def-ImplicitE.cpp:471-676) on set cur at RK time t
int enqueue_implicit_e(oshun_ctx* h) {
    int rc;
    if (!h->d_imp && (rc = build_implicit(h))) return rc;
    const ImplicitArgs ia = implicit_args(h);
    const long long C = h->cells;
    double* J0 = h->d_imp;
    double* JX = J0 + 3 * C;
    double* JY = J0 + 6 * C;
    double* JZ = J0 + 9 * C;
    double* JN = J0 + 12 * C;
    double* DE = J0 + 15 * C;
    double* EN = J0 + 18 * C;
    const int S = h->cur, W = h->cur ^ 1, U = 3;
    const bool one_d = ia.one_d != 0;
    int nsub; double hsub, Dt;
    collide_params(h, h->t, &nsub, &hsub, &Dt);
    // Euler_Backward::advance_1 of a probe state, then its current
    auto collide_and_current = [&](double* J) -> int {
        int r = launch_collide_args(h, collide_args(h, 0, 1, 0, nsub, hsub, Dt, W));
        if (r) return r;
        CK(launch_implicit_current(ia, W, J, h->stream));
        return OSHUN_OK;
    };
    CK(launch_implicit_find_de(ia, h->fld[S], DE, h->stream));
    int zeros = 0;
    for (int attempt = 0; attempt < 4; ++attempt) {
        CK(cudaMemsetAsync(h->d_zeros, 0, sizeof(int), h->stream));
        // E = 0: the probe state is the state itself (its f00 and l = 1 planes)
        CK(cudaMemcpyAsync(h->f00[W], h->f00[S], sizeof(double) * h->pstride, cudaMemcpyDeviceToDevice, h->stream));
        const int q1 = ia.q10, n1 = ia.q11 >= 0 ? 3 : 1;
        CK(cudaMemcpyAsync((char*)h->pl[W] + h->ts * (size_t)q1 * h->pstride,
                           (const char*)h->pl[S] + h->ts * (size_t)q1 * h->pstride,
                           h->ts * (size_t)n1 * h->pstride, cudaMemcpyDeviceToDevice, h->stream));
        if ((rc = collide_and_current(J0))) return rc;
        // the probes: E = DE in one component, its RK2 effect on l <= 2, collisions, current
        const int ncomp = one_d ? 1 : 3;
        double* Jp[3] = {JX, JY, JZ};
        for (int comp = 0; comp < ncomp; ++comp) {
            CK(launch_implicit_probe_field(ia, DE, comp, h->d_fe, h->stream));
            const CoefLM* tab = comp == 0 ? h->d_coef_imp[one_d ? 1 : 0] : h->d_coef_imp[2];
            const int part = comp == 0 ? kPartEx : (comp == 1 ? kPartEy : kPartEz);
            if ((rc = enqueue_rk2(h, S, W, U, part, tab, h->d_fe))) return rc;
            if ((rc = collide_and_current(Jp[comp]))) return rc;
        }
        if (!one_d) CK(launch_implicit_ampere(ia, h->fld[S], JN, h->stream));
        CK(launch_implicit_solve(ia, J0, JX, JY, JZ, JN, DE, EN, h->d_zeros, h->stream));
        CK(cudaMemcpyAsync(&zeros, h->d_zeros, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
        CK(cudaStreamSynchronize(h->stream));
        if (zeros == 0) break;
    }
    CK(launch_implicit_set_e(ia, EN, h->fld[S], h->stream));
    h->imp_zeros = zeros;
    if (zeros > 0) h->imp_zero_seen = true;   // status bit 2 until the word is read
    return OSHUN_OK;
}

void free_ctx(oshun_ctx* h) {
    for (int p = 0; p < 2; ++p)
        for (int c = 0; c < 2; ++c)
            if (h->graph[p][c]) cudaGraphExecDestroy(h->graph[p][c]);
    for (int i = 0; i < 4; ++i) { cudaFree(h->f00[i]); cudaFree(h->pl[i]); cudaFree(h->fld[i]); }
    cudaFree(h->d_coef); cudaFree(h->d_plane_of); cudaFree(h->d_plane_l); cudaFree(h->d_plane_m);
    cudaFree(h->d_hplane); cudaFree(h->d_seq); cudaFree(h->d_ptab); cudaFree(h->d_vtab); cudaFree(h->d_dense_ws);
    cudaFree(h->d_status); cudaFree(h->d_clock); cudaFree(h->d_stage); cudaFree(h->d_jw);
    cudaFree(h->d_mom_tab); cudaFree(h->d_mom);
    cudaFree(h->d_ref64); cudaFree(h->d_ref_ts); cudaFree(h->d_refpart); cudaFree(h->d_refkeep); cudaFree(h->d_hx);
    for (int i = 0; i < 4; ++i) cudaFree(h->d_coef_imp[i]);
    cudaFree(h->d_imp); cudaFree(h->d_fe); cudaFree(h->d_zeros);
    if (h->own_stream && h->stream) cudaStreamDestroy(h->stream);
    delete h;
}

}  // namespace

namespace {
// nsteps small steps on the device clock, queued on the handle's stream
// without waiting (one captured graph per state parity)
int enqueue_steps(oshun_ctx* h, int nsteps, int collisions) {
    for (int s = 0; s < nsteps; ++s) {
        // one graph per state parity: RK4 stages, clocks, collision step
        cudaGraphExec_t& g = h->graph[h->cur][collisions];
        if (!g && h->graphs_ok) {
            const int cur0 = h->cur;
            cudaGraph_t graph = nullptr;
            bool ok = cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeRelaxed) == cudaSuccess;
            int rc = ok ? enqueue_step_device(h, collisions) : OSHUN_OK;
            h->cur = cur0;
            if (ok) ok = cudaStreamEndCapture(h->stream, &graph) == cudaSuccess && rc == OSHUN_OK;
            if (ok) ok = cudaGraphInstantiate(&g, graph, 0) == cudaSuccess;
            if (graph) cudaGraphDestroy(graph);
            if (!ok) {
                // capture unavailable on this stream: plain launches from now on
                (void)cudaGetLastError();
                if (g) { cudaGraphExecDestroy(g); g = nullptr; }
                h->graphs_ok = false;
                if (rc) return rc;
            }
        }
        if (g) {
            CK(cudaGraphLaunch(g, h->stream));
            h->cur ^= 1;
        } else {
            int rc = enqueue_step_device(h, collisions);
            if (rc) return rc;
        }
        h->t += h->cfg.dt;
        if (collisions) {
            h->t_ee = h->t;
            h->t_eb = h->t;
        }
    }
    return OSHUN_OK;
}

}  // namespace

extern "C" {

int oshun_abi_version(void) { return OSHUN_ABI_VERSION; }
const char* oshun_last_error(void) { return g_last_error.c_str(); }

int oshun_create(const oshun_cfg* cfg, oshun_handle* out) {
    if (!out) { set_error("out is NULL"); return OSHUN_ERR_ARG; }
    *out = nullptr;
    int rc = validate(cfg);
    if (rc) return rc;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1) { set_error("no CUDA device"); return OSHUN_ERR_NO_DEVICE; }
    int dev = 0;
    CK(cudaGetDevice(&dev));
    cudaDeviceProp prop;
    CK(cudaGetDeviceProperties(&prop, dev));
    if (prop.major != 10) { set_error("liboshun_b200 is built for sm_100a (B200)"); return OSHUN_ERR_NO_DEVICE; }

    oshun_ctx* h = new oshun_ctx();
    h->cfg = *cfg;
    h->dev = dev;
    h->nh = num_harmonics(cfg->l0, cfg->m0);
    h->mc = pick_mc(cfg->m0);
    h->cells = (long long)cfg->numx * cfg->numy;
    h->pstride = h->cells * cfg->nump;
    h->fp32 = cfg->precision == OSHUN_FP32_SPLIT;
    h->ts = h->fp32 ? 4 : 8;
    h->t = h->t_ee = h->t_eb = cfg->t0;
    auto fail = [&](int code) { free_ctx(h); return code; };
#define CKF(call)                                                                  \
    do {                                                                           \
        cudaError_t e_ = (call);                                                   \
        if (e_ != cudaSuccess) {                                                   \
            set_error(std::string(#call) + ": " + cudaGetErrorString(e_));         \
            return fail(OSHUN_ERR_CUDA);                                           \
        }                                                                          \
    } while (0)
    if ((rc = build_tables(h))) return fail(rc);
    for (int i = 0; i < 4; ++i) {
        CKF(cudaMalloc(&h->f00[i], sizeof(double) * h->pstride));
        CKF(cudaMalloc(&h->pl[i], h->ts * std::max<long long>(1, (long long)h->nplanes * h->pstride)));
        CKF(cudaMalloc(&h->fld[i], h->ts * 6 * h->cells));
        CKF(cudaMemset(h->f00[i], 0, sizeof(double) * h->pstride));
        CKF(cudaMemset(h->pl[i], 0, h->ts * std::max<long long>(1, (long long)h->nplanes * h->pstride)));
        CKF(cudaMemset(h->fld[i], 0, h->ts * 6 * h->cells));
    }
    CKF(cudaMalloc(&h->d_status, sizeof(int) * 4));
    CKF(cudaMemset(h->d_status, 0, sizeof(int) * 4));
    CKF(cudaMalloc(&h->d_jw, sizeof(double) * 24 * h->cells));
    CKF(cudaMemset(h->d_jw, 0, sizeof(double) * 24 * h->cells));
    if (h->fp32) {
        // the FP32 planes are stored relative to a momentum profile per plane
        const size_t nr = (size_t)std::max(1, h->nplanes) * cfg->nump;
        h->use_profile = true;
        CKF(cudaMalloc(&h->d_ref64, sizeof(double) * nr));
        CKF(cudaMemset(h->d_ref64, 0, sizeof(double) * nr));
        CKF(cudaMalloc(&h->d_ref_ts, sizeof(float) * nr));
        CKF(cudaMemset(h->d_ref_ts, 0, sizeof(float) * nr));
        CKF(cudaMalloc(&h->d_refpart, 2 * sizeof(double2) * (size_t)h->nh * kProfChunks * cfg->nump));
        CKF(cudaMalloc(&h->d_refkeep, sizeof(int) * (size_t)std::max(1, h->nplanes)));
        CKF(cudaMemset(h->d_refkeep, 0, sizeof(int) * (size_t)std::max(1, h->nplanes)));
    }
    CKF(cudaMalloc(&h->d_clock, sizeof(Clock)));
    Clock ck{h->t, h->t_ee, h->t_eb};
    CKF(cudaMemcpy(h->d_clock, &ck, sizeof(Clock), cudaMemcpyHostToDevice));
    CKF(cudaMalloc(&h->d_stage, sizeof(double2) * ((size_t)h->nh * h->pstride + 6 * h->cells)));
    CKF(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
    h->own_stream = true;

    // collision launch shape
    const int np = cfg->nump;
    int smem_optin = 0;
    CKF(cudaDeviceGetAttribute(&smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    const size_t budget = std::min<size_t>((size_t)smem_optin, 200 * 1024);
    if (cfg->if_tridiagonal) {
        int chunk = collide_max_chunk(np, budget);
        if (chunk < 1) { set_error("nump too large for the collision kernel's shared memory"); return fail(OSHUN_ERR_UNSUPPORTED); }
        chunk = std::min(chunk, std::max(1, h->nplanes));
        h->collide_chunk = chunk;
        h->collide_smem = collide_smem_bytes(np, chunk, 1);
        h->collide_blocks = (int)std::min<long long>(h->cells, (long long)prop.multiProcessorCount * 16);
        // one warp per cell: one 1-warp CTA per cell (grid-stride beyond 2^30 cells)
        const size_t per_cell = collide_tri_smem_per_cell(np, cfg->l0);
        if (per_cell <= budget) {
            h->tri_cpc = 1;
            h->tri_blocks = (int)std::min<long long>(h->cells, 1ll << 30);
        }
    } else {
        h->collide_smem = collide_smem_bytes(np, 0, 0);
        if (h->collide_smem > budget) { set_error("nump too large for the dense collision path"); return fail(OSHUN_ERR_UNSUPPORTED); }
        h->collide_blocks = (int)std::min<long long>(h->cells, (long long)prop.multiProcessorCount * 4);
        h->dense_blocks = h->collide_blocks;
        CKF(cudaMalloc(&h->d_dense_ws, sizeof(double) * (size_t)np * np * h->dense_blocks));
    }
#undef CKF
    *out = h;
    return OSHUN_OK;
}

int oshun_destroy(oshun_handle h) {
    if (!h) return OSHUN_ERR_ARG;
    cudaStreamSynchronize(h->stream);
    free_ctx(h);
    return OSHUN_OK;
}

int oshun_set_stream(oshun_handle h, void* stream) {
    if (!h) return OSHUN_ERR_ARG;
    CK(cudaStreamSynchronize(h->stream));
    if (h->own_stream) { cudaStreamDestroy(h->stream); h->own_stream = false; }
    for (int p = 0; p < 2; ++p)
        for (int c = 0; c < 2; ++c)
            if (h->graph[p][c]) { cudaGraphExecDestroy(h->graph[p][c]); h->graph[p][c] = nullptr; }
    h->graphs_ok = true;
    if (stream) {
        h->stream = (cudaStream_t)stream;
    } else {
        CK(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
        h->own_stream = true;
    }
    return OSHUN_OK;
}

int oshun_synchronize(oshun_handle h) {
    if (!h) return OSHUN_ERR_ARG;
    CK(cudaStreamSynchronize(h->stream));
    return OSHUN_OK;
}

int oshun_upload(oshun_handle h, const double* harmonics, const double* fields) {
    if (!h || !harmonics || !fields) { set_error("NULL argument"); return OSHUN_ERR_ARG; }
    const size_t nb_h = sizeof(double2) * (size_t)h->nh * h->pstride;
    const size_t nb_f = sizeof(double2) * 6 * (size_t)h->cells;
    CK(cudaMemcpyAsync(h->d_stage, harmonics, nb_h, cudaMemcpyHostToDevice, h->stream));
    CK(cudaMemcpyAsync((char*)h->d_stage + nb_h, fields, nb_f, cudaMemcpyHostToDevice, h->stream));
    CK(cudaMemsetAsync(h->d_status + 2, 0, sizeof(int), h->stream));
    const long long total = (long long)h->nh * h->pstride + 6 * h->cells;
    const int set = h->cur;
    const int np = h->cfg.nump;
    if (h->use_profile) {
        double2* part_sq = h->d_refpart + (size_t)h->nh * kProfChunks * np;
        profile_partial_kernel<<<dim3((unsigned)h->nh, kProfChunks), 128, 0, h->stream>>>(
            h->d_stage, h->d_hplane, h->cells, np, h->d_refpart, part_sq);
        profile_final_kernel<float><<<grid_for((long long)h->nh * np, 128), 128, 0, h->stream>>>(
            h->d_refpart, h->d_hplane, h->nh, h->cells, np, h->d_ref64, (float*)h->d_ref_ts);
        profile_keep_kernel<float><<<(unsigned)h->nh, 128, 0, h->stream>>>(part_sq, h->d_hplane, h->nh, h->cells, np,
                                                                            h->d_ref64, (float*)h->d_ref_ts,
                                                                            h->d_refkeep);
        CK(cudaGetLastError());
    }
    const double* ref = h->use_profile ? h->d_ref64 : nullptr;
    if (h->fp32)
        scatter_kernel<float><<<grid_for(total, 256), 256, 0, h->stream>>>(
            h->d_stage, h->f00[set], (float*)h->pl[set], (float*)h->fld[set], h->d_hplane, h->pstride, h->nh,
            h->cells, h->d_status + 2, ref, np);
    else
        scatter_kernel<double><<<grid_for(total, 256), 256, 0, h->stream>>>(
            h->d_stage, h->f00[set], (double*)h->pl[set], (double*)h->fld[set], h->d_hplane, h->pstride, h->nh,
            h->cells, h->d_status + 2, ref, np);
    CK(cudaGetLastError());
    int flag = 0;
    CK(cudaMemcpyAsync(&flag, h->d_status + 2, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    if (flag) { set_error("an m=0 harmonic or a field has a nonzero imaginary part"); return OSHUN_ERR_NONREAL; }
    return OSHUN_OK;
}

// with_profile: the set holds a state (stored relative to the planes'
// profile); a slope is gathered as it is
static int gather_to_host(oshun_handle h, int set, double* harmonics, double* fields, bool with_profile = true) {
    const long long total = (long long)h->nh * h->pstride + 6 * h->cells;
    const double* ref = (with_profile && h->use_profile) ? h->d_ref64 : nullptr;
    if (h->fp32)
        gather_kernel<float><<<grid_for(total, 256), 256, 0, h->stream>>>(
            h->d_stage, h->f00[set], (const float*)h->pl[set], (const float*)h->fld[set], h->d_hplane, h->pstride,
            h->nh, h->cells, ref, h->cfg.nump);
    else
        gather_kernel<double><<<grid_for(total, 256), 256, 0, h->stream>>>(
            h->d_stage, h->f00[set], (const double*)h->pl[set], (const double*)h->fld[set], h->d_hplane,
            h->pstride, h->nh, h->cells, ref, h->cfg.nump);
    CK(cudaGetLastError());
    const size_t nb_h = sizeof(double2) * (size_t)h->nh * h->pstride;
    const size_t nb_f = sizeof(double2) * 6 * (size_t)h->cells;
    CK(cudaMemcpyAsync(harmonics, h->d_stage, nb_h, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaMemcpyAsync(fields, (char*)h->d_stage + nb_h, nb_f, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return OSHUN_OK;
}

int oshun_download(oshun_handle h, double* harmonics, double* fields) {
    if (!h || !harmonics || !fields) { set_error("NULL argument"); return OSHUN_ERR_ARG; }
    return gather_to_host(h, h->cur, harmonics, fields);
}

int oshun_rhs(oshun_handle h, double* slope_harmonics, double* slope_fields) {
    if (!h || !slope_harmonics || !slope_fields) { set_error("NULL argument"); return OSHUN_ERR_ARG; }
    // slope written to set 2 (scratch), in plane layout
    int rc = fill_mirror(h, h->cur);
    if (rc) return rc;
    rc = launch_stage(h, h->cur, h->cur, h->cur, 2, 1, 0, 1.0, 1.0);
    if (rc) return rc;
    return gather_to_host(h, 2, slope_harmonics, slope_fields, false);
}

static int refuse_halo(oshun_handle h) {
    if (h->xb == OSHUN_XB_HALO) {
        set_error("an x slab (OSHUN_XB_HALO) steps stage by stage: oshun_step_stage, with the halo "
                  "columns loaded before each stage");
        return OSHUN_ERR_UNSUPPORTED;
    }
    return OSHUN_OK;
}

int oshun_rk4_step(oshun_handle h) {
    if (!h) return OSHUN_ERR_ARG;
    if (int rc = refuse_halo(h)) return rc;
    h->inject_active = h->inject_armed;
    h->inject_armed = false;
    int rc = enqueue_rk4(h);
    h->inject_active = false;
    if (rc) return rc;
    h->cur ^= 1;
    h->t += h->cfg.dt;
    clock_advance_kernel<<<1, 1, 0, h->stream>>>(h->d_clock, h->cfg.dt);
    CK(cudaGetLastError());
    return OSHUN_OK;
}

int oshun_collide_ee(oshun_handle h, double t_new) {
    if (!h) return OSHUN_ERR_ARG;
    int nsub; double hsub, Dt;
    collide_params(h, t_new, &nsub, &hsub, &Dt);
    int rc = enqueue_collide(h, 1, 0, 0, nsub, hsub, Dt);
    if (rc) return rc;
    h->t_ee = t_new;
    Clock ck{h->t, h->t_ee, h->t_eb};
    CK(cudaMemcpyAsync(h->d_clock, &ck, sizeof(Clock), cudaMemcpyHostToDevice, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return OSHUN_OK;
}

int oshun_collide_f1(oshun_handle h, double t_new) {
    if (!h) return OSHUN_ERR_ARG;
    int nsub; double hsub, Dt;
    collide_params(h, t_new, &nsub, &hsub, &Dt);
    return enqueue_collide(h, 0, 1, 0, nsub, hsub, Dt);
}

int oshun_collide_flm(oshun_handle h, double t_new) {
    if (!h) return OSHUN_ERR_ARG;
    int nsub; double hsub, Dt;
    collide_params(h, t_new, &nsub, &hsub, &Dt);
    int rc = enqueue_collide(h, 0, 0, 1, nsub, hsub, Dt);
    if (rc) return rc;
    h->t_eb = t_new;
    Clock ck{h->t, h->t_ee, h->t_eb};
    CK(cudaMemcpyAsync(h->d_clock, &ck, sizeof(Clock), cudaMemcpyHostToDevice, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return OSHUN_OK;
}

int oshun_step(oshun_handle h, int nsteps, int collisions) {
    if (!h || nsteps < 0) return OSHUN_ERR_ARG;
    if (int rc = refuse_halo(h)) return rc;
    collisions = collisions ? 1 : 0;
    Clock ck{h->t, h->t_ee, h->t_eb};
    CK(cudaMemcpyAsync(h->d_clock, &ck, sizeof(Clock), cudaMemcpyHostToDevice, h->stream));
    if (int rc = enqueue_steps(h, nsteps, collisions)) return rc;
    CK(cudaStreamSynchronize(h->stream));
    return OSHUN_OK;
}

int oshun_set_x_boundary(oshun_handle h, int mode) {
    if (!h) return OSHUN_ERR_ARG;
    if (mode != OSHUN_XB_PERIODIC && mode != OSHUN_XB_MIRROR && mode != OSHUN_XB_HALO) {
        set_error("x boundary: OSHUN_XB_PERIODIC, OSHUN_XB_MIRROR or OSHUN_XB_HALO");
        return OSHUN_ERR_ARG;
    }
    if (mode != OSHUN_XB_PERIODIC && h->fp32) {
        // FP32 planes hold deviations from this grid's own momentum profile
        set_error("mirrored and slab x boundaries run in FP64");
        return OSHUN_ERR_UNSUPPORTED;
    }
    if (mode != OSHUN_XB_PERIODIC && !h->d_hx) {
        const long long ts = h->fp32 ? 4 : 8;
        auto al = [](long long b) { return (b + 255) / 256 * 256; };
        const long long ny = h->cfg.numy, np = h->cfg.nump;
        h->hx_pl = al(ny * np * 8);
        h->hx_fld = h->hx_pl + al((long long)h->nplanes * ny * np * ts);
        h->hx_side = h->hx_fld + al(6 * ny * ts);
        CK(cudaMalloc(&h->d_hx, 2 * h->hx_side));
        CK(cudaMemset(h->d_hx, 0, 2 * h->hx_side));
    }
    if (mode != h->xb) {
        // the captured step graphs hold the old boundary's launches
        CK(cudaStreamSynchronize(h->stream));
        for (auto& row : h->graph)
            for (auto& g : row)
                if (g) { cudaGraphExecDestroy(g); g = nullptr; }
    }
    h->xb = mode;
    h->stage_next = 1;
    return OSHUN_OK;
}

int oshun_halo_bytes(oshun_handle h, long long* bytes) {
    if (!h || !bytes) return OSHUN_ERR_ARG;
    if (h->xb == OSHUN_XB_PERIODIC) { set_error("periodic x boundaries have no halo columns"); return OSHUN_ERR_ARG; }
    *bytes = h->hx_side;
    return OSHUN_OK;
}

int oshun_halo_pack(oshun_handle h, void* left_edge, void* right_edge) {
    if (!h || !left_edge || !right_edge) return OSHUN_ERR_ARG;
    if (h->xb != OSHUN_XB_HALO) { set_error("oshun_halo_pack needs OSHUN_XB_HALO"); return OSHUN_ERR_ARG; }
    const int set = stage_input(h, h->stage_next);
    CK(launch_halo_columns(h->f00[set], h->pl[set], h->fld[set], halo_grid(h), h->fp32, left_edge, right_edge, 0,
                           h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return OSHUN_OK;
}

int oshun_halo_unpack(oshun_handle h, const void* from_left, const void* from_right) {
    if (!h || !from_left || !from_right) return OSHUN_ERR_ARG;
    if (h->xb != OSHUN_XB_HALO) { set_error("oshun_halo_unpack needs OSHUN_XB_HALO"); return OSHUN_ERR_ARG; }
    CK(cudaMemcpyAsync(h->d_hx, from_left, h->hx_side, cudaMemcpyDeviceToDevice, h->stream));
    CK(cudaMemcpyAsync(h->d_hx + h->hx_side, from_right, h->hx_side, cudaMemcpyDeviceToDevice, h->stream));
    return OSHUN_OK;
}

int oshun_halo_mirror_side(oshun_handle h, int side) {
    if (!h || (side != 0 && side != 1)) return OSHUN_ERR_ARG;
    if (h->xb != OSHUN_XB_HALO) { set_error("oshun_halo_mirror_side needs OSHUN_XB_HALO"); return OSHUN_ERR_ARG; }
    const int set = stage_input(h, h->stage_next);
    CK(launch_halo_column(h->f00[set], h->pl[set], h->fld[set], halo_grid(h), h->fp32,
                          side == 0 ? 0 : h->cfg.numx - 1, h->d_hx + (side ? h->hx_side : 0), 1, h->stream));
    return OSHUN_OK;
}

int oshun_step_stage(oshun_handle h, int k, int collisions) {
    if (!h) return OSHUN_ERR_ARG;
    if (k != h->stage_next) { set_error("stages run in order 1, 2, 3, 4"); return OSHUN_ERR_ARG; }
    int rc = enqueue_stage(h, k);
    if (rc) return rc;
    if (k < 4) {
        h->stage_next = k + 1;
        CK(cudaStreamSynchronize(h->stream));
        return OSHUN_OK;
    }
    h->stage_next = 1;
    h->cur ^= 1;
    h->t += h->cfg.dt;
    clock_advance_kernel<<<1, 1, 0, h->stream>>>(h->d_clock, h->cfg.dt);
    CK(cudaGetLastError());
    if (collisions) {
        int nsub; double hsub, Dt;
        collide_params(h, h->t, &nsub, &hsub, &Dt);
        if ((rc = enqueue_collide(h, 1, 1, 1, nsub, hsub, Dt))) return rc;
        clock_commit_kernel<<<1, 1, 0, h->stream>>>(h->d_clock, 1, 1);
        CK(cudaGetLastError());
        h->t_ee = h->t;
        h->t_eb = h->t;
    }
    CK(cudaStreamSynchronize(h->stream));
    return OSHUN_OK;
}

int oshun_rk2_imp_step(oshun_handle h, int nsteps, int mask) {
    if (!h || nsteps < 0) return OSHUN_ERR_ARG;
    if (h->xb != OSHUN_XB_PERIODIC) {
        set_error("the implicit-E step runs with periodic x boundaries");
        return OSHUN_ERR_UNSUPPORTED;
    }
    if (mask < 0 || mask > 63) { set_error("mask: bits 1, 2, 4, 8, 16, 32"); return OSHUN_ERR_ARG; }
    if (!h->d_imp) {
        const int rc = build_implicit(h);
        if (rc) return rc;
    }
    int rc;
    for (int s = 0; s < nsteps; ++s) {
        if (mask & 1) {
            // Runge_Kutta_2_Imp::advance_p1: Adv1 = advection + B + Faraday (def-Actions.cpp:117-133)
            if ((rc = enqueue_rk2(h, h->cur, h->cur ^ 1, 3, kPartB | kPartAdv | kPartFaraday, h->d_coef, nullptr)))
                return rc;
            h->cur ^= 1;
            h->t += h->cfg.dt;
        }
        if (mask & 2) {
            int nsub; double hsub, Dt;
            collide_params(h, h->t, &nsub, &hsub, &Dt);
            if ((rc = enqueue_collide(h, 1, 0, 0, nsub, hsub, Dt))) return rc;
            h->t_ee = h->t;
        }
        if (mask & 16) {
            if ((rc = enqueue_implicit_e(h))) return rc;
            if (h->imp_zeros > 8) {
                set_error("implicit E: zero determinant in " + std::to_string(h->imp_zeros) +
                          " cells after 4 attempts (the reference stops here)");
                return OSHUN_ERR_NUMERIC;
            }
        }
        if (mask & 32) {
            // advance_p2: Adv2 = the new E's couplings + CLEAN_LOW_PC (def-Actions.cpp:137-160)
            const bool one_d = h->cfg.if_implicit1D != 0;
            const int parts = (one_d ? kPartEx : (kPartEx | kPartEy | kPartEz)) | kPartClean;
            if ((rc = enqueue_rk2(h, h->cur, h->cur ^ 1, 3, parts, one_d ? h->d_coef_imp[3] : h->d_coef, nullptr)))
                return rc;
            h->cur ^= 1;
        }
        if (mask & 12) {
            int nsub; double hsub, Dt;
            collide_params(h, h->t, &nsub, &hsub, &Dt);
            if ((mask & 4) && (rc = enqueue_collide(h, 0, 1, 0, nsub, hsub, Dt))) return rc;
            if (mask & 8) {
                if ((rc = enqueue_collide(h, 0, 0, 1, nsub, hsub, Dt))) return rc;
                h->t_eb = h->t;
            }
        }
    }
    Clock ck{h->t, h->t_ee, h->t_eb};
    CK(cudaMemcpyAsync(h->d_clock, &ck, sizeof(Clock), cudaMemcpyHostToDevice, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return OSHUN_OK;
}

int oshun_plane_profile(oshun_handle h, const double** profile) {
    if (!h || !profile) { set_error("NULL argument"); return OSHUN_ERR_ARG; }
    *profile = h->use_profile ? h->d_ref64 : nullptr;
    return OSHUN_OK;
}

int oshun_get_config(oshun_handle h, oshun_cfg* cfg) {
    if (!h || !cfg) { set_error("NULL argument"); return OSHUN_ERR_ARG; }
    *cfg = h->cfg;
    return OSHUN_OK;
}

int oshun_moments(oshun_handle h, float* out) {
    if (!h || !out) { set_error("NULL argument"); return OSHUN_ERR_ARG; }
    const oshun_cfg& c = h->cfg;
    const int np = c.nump;
    if (!h->d_mom) {
        // momentum tables with the host's pow(), the function the reference
        // calls (def-Parallel.cpp:1693-1696, 1741-1750, 1815-1823, 2107-2118)
        std::vector<double> t((size_t)7 * np);
        for (int i = 0; i < np; ++i) {
            const double p = axis_point(i, np, c.pmin, c.pmax);
            const double ig = 1.0 / std::sqrt(1.0 + p * p);
            t[i] = p;
            t[np + i] = ig;
            t[2 * np + i] = std::pow(ig, 2);
            t[3 * np + i] = std::pow(ig, 3);
            t[4 * np + i] = std::pow(p, 3);
            t[5 * np + i] = std::pow(p, 4);
            t[6 * np + i] = std::pow(p, 5);
        }
        CK(cudaMalloc(&h->d_mom_tab, sizeof(double) * t.size()));
        CK(cudaMemcpy(h->d_mom_tab, t.data(), sizeof(double) * t.size(), cudaMemcpyHostToDevice));
        CK(cudaMalloc(&h->d_mom, sizeof(float) * (kMomCount + 1) * h->cells));
    }
    MomentArgs a;
    std::memset(&a, 0, sizeof(a));
    a.f00 = h->f00[h->cur];
    a.planes = h->pl[h->cur];
    a.pl_ref = h->use_profile ? h->d_ref64 : nullptr;
    a.cells = h->cells; a.pstride = h->pstride;
    a.np = np; a.nx = c.numx; a.ny = c.numy;
    auto plane = [&](int l, int m) {
        return (l <= c.l0 && m <= c.m0) ? (int)(h->plane_of_host[(size_t)l * (c.m0 + 1) + m]) : -2;
    };
    a.q10 = plane(1, 0); a.q11 = plane(1, 1); a.q20 = plane(2, 0); a.q21 = plane(2, 1); a.q22 = plane(2, 2);
    const double* T = h->d_mom_tab;
    a.pr = T; a.invgamma = T + np; a.ig2 = T + 2 * np; a.ig3 = T + 3 * np;
    a.pow3 = T + 4 * np; a.pow4 = T + 5 * np; a.pow5 = T + 6 * np;
    const double p0 = axis_point(0, np, c.pmin, c.pmax), p1 = axis_point(1, np, c.pmin, c.pmax);
    const double dp = p1 - p0;
    a.dp = dp;
    a.p0p1_sq = p0 * p0 / (p1 * p1);
    a.inv_mp0p1_sq = 1.0 / (1.0 - a.p0p1_sq);
    a.corr5 = std::pow(p0, 5) / (dp * p1 * 5.0);
    a.corr7 = std::pow(p0, 7) / (dp * p1 * 7.0);
    a.density_np = c.density_np; a.Zeta = c.Zeta;
    a.nu_pre = std::sqrt(2.0 / M_PI) / 9.0;
    a.s_dens = (float)(4.0 * M_PI * dp);
    a.s_v1 = (float)((4.0 * M_PI / 3.0) * dp);
    a.s_v2 = (float)((8.0 * M_PI / 3.0) * dp);
    a.s_m2 = (float)(8.0 * M_PI / 15.0 * dp);
    a.s_vyvy = (float)(16.0 * M_PI / 5.0 * dp);
    a.s_vxvy = (float)(8.0 * M_PI / 5.0 * dp);
    a.s_vxvz = (float)(-(8.0 * M_PI / 5.0) * dp);
    a.s_vyvz = (float)(-(16.0 * M_PI / 5.0) * dp);
    a.s_pre = (float)(2.73785179e-19 * c.density_np);
    a.s_kx = (float)(0.5 / (axis_point(0, c.numx, c.xmin, c.xmax) - axis_point(1, c.numx, c.xmin, c.xmax)));
    a.s_ky = c.numy > 1 ? (float)(0.5 / (axis_point(0, c.numy, c.ymin, c.ymax) - axis_point(1, c.numy, c.ymin, c.ymax)))
                        : 0.0f;
    a.out = h->d_mom;
    CK(launch_moments(a, h->fp32 ? 1 : 0, h->stream));
    CK(cudaMemcpyAsync(out, h->d_mom, sizeof(float) * kMomCount * h->cells, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return OSHUN_OK;
}

int oshun_debug_inject_stage_timeout(oshun_handle h, int withhold_copy, double wait_seconds) {
    if (!h) return OSHUN_ERR_ARG;
    if (withhold_copy < 0 || !(wait_seconds >= 1e-4 && wait_seconds <= 1.0)) {
        set_error("need withhold_copy >= 0 and 1e-4 <= wait_seconds <= 1");
        return OSHUN_ERR_ARG;
    }
    h->inject_armed = true;
    h->inject_withhold = withhold_copy;
    h->inject_wait_ns = (unsigned long long)(wait_seconds * 1e9);
    return OSHUN_OK;
}

int oshun_time(oshun_handle h, double* t) {
    if (!h || !t) return OSHUN_ERR_ARG;
    *t = h->t;
    return OSHUN_OK;
}

int oshun_status_flags(oshun_handle h, int* flags, long long* count) {
    if (!h) return OSHUN_ERR_ARG;
    const long long nf = h->pstride, npl = (long long)h->nplanes * h->pstride, nfl = 6 * h->cells;
    CK(launch_nan_check(h->f00[h->cur], h->pl[h->cur], h->fp32, nf, npl, h->fld[h->cur], nfl, h->d_status, h->stream));
    int st[2] = {0, 0};
    CK(cudaMemcpyAsync(st, h->d_status, sizeof(int) * 2, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaMemsetAsync(h->d_status, 0, sizeof(int) * 2, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    if (flags) *flags = st[0] | (h->imp_zero_seen ? 4 : 0);
    if (count) *count = st[1];
    h->imp_zero_seen = false;
    return OSHUN_OK;
}

int oshun_device_state(oshun_handle h, void** f00, void** planes, void** fields, size_t* planes_bytes,
                       size_t* fields_bytes) {
    if (!h) return OSHUN_ERR_ARG;
    if (f00) *f00 = h->f00[h->cur];
    if (planes) *planes = h->pl[h->cur];
    if (fields) *fields = h->fld[h->cur];
    if (planes_bytes) *planes_bytes = h->ts * (size_t)h->nplanes * h->pstride;
    if (fields_bytes) *fields_bytes = h->ts * 6 * (size_t)h->cells;
    return OSHUN_OK;
}

int oshun_plane_index(oshun_handle h, int l, int m, int* plane) {
    if (!h || !plane || l < 0 || l > h->cfg.l0 || m < 0 || m > h->cfg.m0 || m > l) return OSHUN_ERR_ARG;
    if (l == 0) { *plane = -1; return OSHUN_OK; }
    int q = 0;
    for (int ll = 1; ll <= h->cfg.l0; ++ll)
        for (int mm = 0; mm <= std::min(ll, h->cfg.m0); ++mm) {
            if (ll == l && mm == m) { *plane = q; return OSHUN_OK; }
            q += mm > 0 ? 2 : 1;
        }
    return OSHUN_ERR_ARG;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Batches of independent problems (no counterpart in the reference, whose
// runs are one problem per process): every problem keeps its own handle
// (state sets, tables, clocks); one step of the batch is one captured graph of
//   4 x batched RK4 stage launch (one persistent kernel each, over the
//       (problem, tile) list of the whole batch),
//   device clock advance,
//   per group of problems with equal ceil(nump/32) and on the same side of
//       8 resident collision CTAs per SM: one batched collision launch over
//       their (problem, cell) list,
//   device clock commit.
// The stage tiles (consumer threads per CTA, cells per tile) are chosen by
// oshun_batch_autotune, which times each candidate on the batch itself.
// ---------------------------------------------------------------------------
struct oshun_batch_ctx {
    std::vector<oshun_ctx*> P;
    std::vector<int> collide;       // per problem: collision step on
    bool fp32 = false;
    int mc = 0;                     // template class of the largest m0
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    // the collision groups run side by side on the batch's stream and these
    // two, forked after the clock advance and joined before the clock commit
    // (groups touch disjoint problems; a group held to few resident CTAs per
    // SM by its shared memory leaves room for another group's CTAs)
    cudaStream_t side[2] = {nullptr, nullptr};
    cudaEvent_t ev_fork = nullptr, ev_join[2] = {nullptr, nullptr};
    int cur = 0;                    // parity of every problem's state sets
    int nc = 192, tx_cap = 8;       // stage tiles
    // stage launches
    int desc_bytes = 0, ncoef_max = 0, hdr_bytes = 0;
    unsigned char* d_desc = nullptr;   // [2 parities][4 stages][n] descriptors
    void* d_coef_ts = nullptr;         // coupling tables in the arithmetic type
    int2* d_items = nullptr;
    int nitems = 0;
    size_t slot_bytes = 0, row_arr_bytes = 0;
    int row_depth = 2;
    std::vector<unsigned char> h_a1[2][4];   // kernel parameter of each launch (a problem's descriptor)
    // collision launches
    struct Group {
        int E = 0;
        size_t smem = 0;
        int4* d_chunks = nullptr;   // chunked form (CTAs of `warps` cells of one problem), or none
        long long nchunks = 0;
        int warps = 0, tab_doubles = 0;
        CollideArgs* d_args[2] = {nullptr, nullptr};   // per parity
        int2* d_items = nullptr;
        long long nitems = 0;
    };
    std::vector<Group> groups;
    double* d_clocks = nullptr;   // [n][t, t_ee, t_eb]
    double* d_dt = nullptr;       // [n]
    int* d_collide = nullptr;     // [n]
    int* d_status = nullptr;      // pipeline status of the batched launches
    cudaGraphExec_t graph[2] = {nullptr, nullptr};
    bool graphs_ok = true;
};

namespace {

void batch_drop_graphs(oshun_batch_ctx* b) {
    for (int c = 0; c < 2; ++c)
        if (b->graph[c]) { cudaGraphExecDestroy(b->graph[c]); b->graph[c] = nullptr; }
}

void free_batch(oshun_batch_ctx* b) {
    batch_drop_graphs(b);
    for (oshun_ctx* h : b->P)
        if (h) free_ctx(h);
    for (auto& g : b->groups) { cudaFree(g.d_args[0]); cudaFree(g.d_args[1]); cudaFree(g.d_items); cudaFree(g.d_chunks); }
    cudaFree(b->d_desc); cudaFree(b->d_coef_ts); cudaFree(b->d_items);
    cudaFree(b->d_clocks); cudaFree(b->d_dt); cudaFree(b->d_collide); cudaFree(b->d_status);
    for (int i = 0; i < 2; ++i) {
        if (b->side[i]) cudaStreamDestroy(b->side[i]);
        if (b->ev_join[i]) cudaEventDestroy(b->ev_join[i]);
    }
    if (b->ev_fork) cudaEventDestroy(b->ev_fork);
    if (b->own_stream && b->stream) cudaStreamDestroy(b->stream);
    delete b;
}

// descriptor of RK4 stage k (Runge_Kutta_4::advance_p1, def-RK.cpp:116-142)
// of problem h for state parity c, as launch_stage builds it
template <typename TS>
StageArgs<TS> batch_stage_args(const oshun_ctx* h, int c, int k, const void* coef_ts) {
    const double dt = h->cfg.dt;
    const int B = c, A = c ^ 1, Sa = 2, Sb = 3;
    const int in_set[4] = {B, Sa, Sb, Sa}, out_set[4] = {Sa, Sb, Sa, -1};
    const double c1[4] = {0.5 * dt, 0.5 * dt, dt, dt / 6.0}, c2[4] = {1.0 / 3.0, 2.0 / 3.0, 1.0 / 3.0, 1.0};
    StageArgs<TS> a = h->stage_args<TS>(in_set[k], out_set[k], 0);
    a.f00_B = h->f00[B]; a.pl_B = (const TS*)h->pl[B]; a.fld_B = (const TS*)h->fld[B];
    a.f00_A = h->f00[A]; a.pl_A = (TS*)h->pl[A]; a.fld_A = (TS*)h->fld[A];
    if (out_set[k] >= 0) {
        a.f00_out = h->f00[out_set[k]]; a.pl_out = (TS*)h->pl[out_set[k]]; a.fld_out = (TS*)h->fld[out_set[k]];
    }
    a.first = k == 0; a.c1 = c1[k]; a.c2 = c2[k];
    a.coef_ts = coef_ts;
    return a;
}

// (problem, tile) list for the current tiles, heaviest tiles first, so that
// the persistent CTAs' round-robin shares are even
int batch_build_items(oshun_batch_ctx* b) {
    const int esz = b->fp32 ? 4 : 8;
    struct It { double cost; int p, tile; };
    std::vector<It> items;
    size_t slot = 0, rowb = 0;
    for (int i = 0; i < (int)b->P.size(); ++i) {
        const oshun_cfg& c = b->P[i]->cfg;
        if (((c.nump + 31) / 32) * 32 > b->nc) {
            set_error("batch stage threads below a problem's padded nump");
            return OSHUN_ERR_UNSUPPORTED;
        }
        int tx;
        size_t sb, rb;
        stage_batch_sizes(c.nump, c.numx, c.numy, c.l0, c.m0, b->nc, b->tx_cap, esz, &tx, &sb, &rb);
        slot = std::max(slot, sb);
        rowb = std::max(rowb, rb);
        const int tiles = c.numy * ((c.numx + tx - 1) / tx);
        const double cost = (double)b->P[i]->nh * (double)(((c.nump + 31) / 32) * 32) * tx;
        for (int t = 0; t < tiles; ++t) items.push_back({cost, i, t});
    }
    // staged-row ring: as deep as 24 KB of rows allow, 2..8 rows
    b->row_depth = (int)std::max<size_t>(2, std::min<size_t>(8, (24 * 1024) / std::max<size_t>(1, 2 * rowb)));
    BatchWork bw{};
    bw.hdr_bytes = b->hdr_bytes; bw.slot_bytes = (int)slot; bw.row_arr_bytes = (int)rowb;
    bw.row_depth = b->row_depth;
    if (stage_batch_smem(bw, esz) > 227 * 1024) {
        set_error("batch tiles do not fit in shared memory (lower the cells per tile)");
        return OSHUN_ERR_UNSUPPORTED;
    }
    std::stable_sort(items.begin(), items.end(), [](const It& x, const It& y) { return x.cost > y.cost; });
    std::vector<int2> h(items.size());
    for (size_t k = 0; k < items.size(); ++k) h[k] = make_int2(items[k].p, items[k].tile);
    cudaFree(b->d_items);
    b->d_items = nullptr;
    CK(cudaMalloc(&b->d_items, sizeof(int2) * std::max<size_t>(1, h.size())));
    CK(cudaMemcpy(b->d_items, h.data(), sizeof(int2) * h.size(), cudaMemcpyHostToDevice));
    b->nitems = (int)h.size();
    b->slot_bytes = slot;
    b->row_arr_bytes = rowb;
    return OSHUN_OK;
}

BatchWork batch_work(const oshun_batch_ctx* b, int c, int k) {
    BatchWork bw{};
    bw.probs = b->d_desc + ((size_t)(c * 4 + k) * b->P.size()) * b->desc_bytes;
    bw.items = b->d_items;
    bw.nitems = b->nitems;
    bw.tx_cap = b->tx_cap;
    bw.desc_bytes = b->desc_bytes;
    bw.ncoef_max = b->ncoef_max;
    bw.hdr_bytes = b->hdr_bytes;
    bw.slot_bytes = (int)b->slot_bytes;
    bw.row_arr_bytes = (int)b->row_arr_bytes;
    bw.row_depth = b->row_depth;
    bw.nprobs = (int)b->P.size();
    return bw;
}

// one step of every problem for state parity c (graph-capturable)
int batch_enqueue_step(oshun_batch_ctx* b, int c) {
    const int n = (int)b->P.size();
    for (int k = 0; k < 4; ++k) {
        const BatchWork bw = batch_work(b, c, k);
        cudaError_t e;
        if (b->fp32)
            e = launch_stage_batch<float>(*reinterpret_cast<const StageArgs<float>*>(b->h_a1[c][k].data()), bw, b->mc,
                                          b->nc, b->stream);
        else
            e = launch_stage_batch<double>(*reinterpret_cast<const StageArgs<double>*>(b->h_a1[c][k].data()), bw,
                                           b->mc, b->nc, b->stream);
        if (e != cudaSuccess) { set_error(std::string("batched stage launch: ") + cudaGetErrorString(e)); return OSHUN_ERR_CUDA; }
    }
    CK(launch_clock_advance(b->d_clocks, b->d_dt, n, b->stream));
    // fork: each group goes to the least loaded of the three streams, largest
    // first (load = cells x ceil(nump/32)); join before the clock commit
    CK(cudaEventRecord(b->ev_fork, b->stream));
    for (int i = 0; i < 2; ++i) CK(cudaStreamWaitEvent(b->side[i], b->ev_fork, 0));
    std::vector<int> order(b->groups.size());
    for (size_t i = 0; i < order.size(); ++i) order[i] = (int)i;
    auto load_of = [&](int i) { return (double)b->groups[i].nitems * b->groups[i].E; };
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return load_of(x) > load_of(y); });
    double load[3] = {0.0, 0.0, 0.0};
    cudaStream_t lanes[3] = {b->stream, b->side[0], b->side[1]};
    cudaError_t e = cudaSuccess;
    for (int gi : order) {
        const auto& g = b->groups[gi];
        const int li = (int)(std::min_element(load, load + 3) - load);
        load[li] += load_of(gi);
        CollideBatch cb{g.d_args[c ^ 1], g.d_items, g.nitems, g.d_chunks, g.nchunks, g.warps, g.tab_doubles,
                        (int)(g.smem / sizeof(double))};   // the new state is parity c^1
        e = launch_collide_batch(cb, g.E, b->fp32 ? 1 : 0, g.smem, lanes[li]);
        if (e != cudaSuccess) break;
    }
    for (int i = 0; i < 2; ++i) {
        CK(cudaEventRecord(b->ev_join[i], b->side[i]));
        CK(cudaStreamWaitEvent(b->stream, b->ev_join[i], 0));
    }
    if (e != cudaSuccess) { set_error(std::string("batched collision launch: ") + cudaGetErrorString(e)); return OSHUN_ERR_CUDA; }
    CK(launch_clock_commit(b->d_clocks, b->d_collide, n, b->stream));
    return OSHUN_OK;
}

int batch_upload_clocks(oshun_batch_ctx* b) {
    std::vector<double> ck(3 * b->P.size());
    for (size_t i = 0; i < b->P.size(); ++i) {
        ck[3 * i] = b->P[i]->t; ck[3 * i + 1] = b->P[i]->t_ee; ck[3 * i + 2] = b->P[i]->t_eb;
    }
    CK(cudaMemcpyAsync(b->d_clocks, ck.data(), sizeof(double) * ck.size(), cudaMemcpyHostToDevice, b->stream));
    CK(cudaStreamSynchronize(b->stream));
    return OSHUN_OK;
}

// host mirrors of the clocks after one step (the same arithmetic as the device)
void batch_advance_host(oshun_batch_ctx* b) {
    b->cur ^= 1;
    for (size_t i = 0; i < b->P.size(); ++i) {
        oshun_ctx* h = b->P[i];
        h->cur = b->cur;
        h->t += h->cfg.dt;
        if (b->collide[i]) { h->t_ee = h->t; h->t_eb = h->t; }
    }
}

int batch_steps_plain(oshun_batch_ctx* b, int nsteps) {
    for (int s = 0; s < nsteps; ++s) {
        int rc = batch_enqueue_step(b, b->cur);
        if (rc) return rc;
        batch_advance_host(b);
    }
    return OSHUN_OK;
}

}  // namespace

extern "C" {

int oshun_batch_create(const oshun_cfg* cfgs, int n, const int* collide, oshun_batch* out) {
    if (!out || !cfgs || n < 1) { set_error("bad batch arguments"); return OSHUN_ERR_ARG; }
    *out = nullptr;
    oshun_batch_ctx* b = new oshun_batch_ctx();
    auto fail = [&](int code) { free_batch(b); return code; };
#define CKB(call)                                                                  \
    do {                                                                           \
        cudaError_t e_ = (call);                                                   \
        if (e_ != cudaSuccess) {                                                   \
            set_error(std::string(#call) + ": " + cudaGetErrorString(e_));         \
            return fail(OSHUN_ERR_CUDA);                                           \
        }                                                                          \
    } while (0)
    b->fp32 = cfgs[0].precision == OSHUN_FP32_SPLIT;
    CKB(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking));
    b->own_stream = true;
    for (int i = 0; i < 2; ++i) {
        CKB(cudaStreamCreateWithFlags(&b->side[i], cudaStreamNonBlocking));
        CKB(cudaEventCreateWithFlags(&b->ev_join[i], cudaEventDisableTiming));
    }
    CKB(cudaEventCreateWithFlags(&b->ev_fork, cudaEventDisableTiming));
    const int esz = b->fp32 ? 4 : 8;
    int m0max = 0;
    for (int i = 0; i < n; ++i) {
        const oshun_cfg& c = cfgs[i];
        if (c.precision != cfgs[0].precision) { set_error("a batch has one precision"); return fail(OSHUN_ERR_ARG); }
        if (((c.nump + 31) / 32) * 32 > 256 || (c.nump * esz) % 16 != 0) {
            set_error("batched problems need nump <= 256 with nump * element size a multiple of 16 bytes");
            return fail(OSHUN_ERR_UNSUPPORTED);
        }
        const int col = collide ? (collide[i] != 0) : 1;
        if (col && !c.if_tridiagonal) { set_error("batched collision steps are tridiagonal"); return fail(OSHUN_ERR_UNSUPPORTED); }
        if (col && (c.flags & OSHUN_FLAG_IMPLICIT_EE)) {
            set_error("batched collision steps use the explicit e-e substeps");
            return fail(OSHUN_ERR_UNSUPPORTED);
        }
        oshun_handle h = nullptr;
        int rc = oshun_create(&c, &h);
        if (rc) return fail(rc);
        b->P.push_back(h);
        b->collide.push_back(col);
        if ((rc = oshun_set_stream(h, b->stream))) return fail(rc);
        m0max = std::max(m0max, c.m0);
        b->ncoef_max = std::max(b->ncoef_max, (c.l0 + 1) * (c.m0 + 1));
    }
    b->mc = pick_mc(m0max);
    b->desc_bytes = (int)((std::max(sizeof(StageArgs<float>), sizeof(StageArgs<double>)) + 15) / 16 * 16);
    const int cbytes = stage_batch_coef_bytes(esz);
    b->hdr_bytes = b->desc_bytes;

    // coupling tables in the arithmetic type
    std::vector<size_t> coff(n);
    size_t ctot = 0;
    for (int i = 0; i < n; ++i) {
        coff[i] = ctot;
        ctot += (size_t)cbytes * (b->P[i]->cfg.l0 + 1) * (b->P[i]->cfg.m0 + 1);
    }
    CKB(cudaMalloc(&b->d_coef_ts, ctot));
    {
        std::vector<unsigned char> hc(ctot);
        for (int i = 0; i < n; ++i) {
            const int nco = (b->P[i]->cfg.l0 + 1) * (b->P[i]->cfg.m0 + 1);
            std::vector<double> dc((size_t)nco * 16);
            CKB(cudaMemcpy(dc.data(), b->P[i]->d_coef, sizeof(double) * dc.size(), cudaMemcpyDeviceToHost));
            for (size_t k = 0; k < dc.size(); ++k) {
                if (b->fp32) { const float v = (float)dc[k]; std::memcpy(&hc[coff[i] + 4 * k], &v, 4); }
                else std::memcpy(&hc[coff[i] + 8 * k], &dc[k], 8);
            }
        }
        CKB(cudaMemcpy(b->d_coef_ts, hc.data(), ctot, cudaMemcpyHostToDevice));
    }
    // stage descriptors [parity][stage][problem] and the launches' parameters
    CKB(cudaMalloc(&b->d_status, sizeof(int) * 4));
    CKB(cudaMemset(b->d_status, 0, sizeof(int) * 4));
    {
        std::vector<unsigned char> hd((size_t)8 * n * b->desc_bytes, 0);
        for (int c = 0; c < 2; ++c)
            for (int k = 0; k < 4; ++k)
                for (int i = 0; i < n; ++i) {
                    unsigned char* dst = &hd[((size_t)(c * 4 + k) * n + i) * b->desc_bytes];
                    const void* ct = (const unsigned char*)b->d_coef_ts + coff[i];
                    if (b->fp32) {
                        StageArgs<float> a = batch_stage_args<float>(b->P[i], c, k, ct);
                        std::memcpy(dst, &a, sizeof(a));
                    } else {
                        StageArgs<double> a = batch_stage_args<double>(b->P[i], c, k, ct);
                        std::memcpy(dst, &a, sizeof(a));
                    }
                    if (i == 0) {
                        b->h_a1[c][k].assign(dst, dst + b->desc_bytes);
                        // pipeline timeouts of a batched launch land in the batch's status word
                        int* st = b->d_status;
                        const size_t off = b->fp32 ? offsetof(StageArgs<float>, err) : offsetof(StageArgs<double>, err);
                        std::memcpy(b->h_a1[c][k].data() + off, &st, sizeof(st));
                    }
                }
        CKB(cudaMalloc(&b->d_desc, hd.size()));
        CKB(cudaMemcpy(b->d_desc, hd.data(), hd.size(), cudaMemcpyHostToDevice));
    }
    // default tiles: 192 consumer threads, or 256 when a momentum row needs them
    int pad_max = 32;
    for (oshun_ctx* h : b->P) pad_max = std::max(pad_max, ((h->cfg.nump + 31) / 32) * 32);
    b->nc = pad_max <= 192 ? 192 : 256;
    int rc = OSHUN_ERR_UNSUPPORTED;
    for (int tx : {8, 4, 2, 1}) {   // the widest tiles whose plan fits in shared memory
        b->tx_cap = tx;
        if ((rc = batch_build_items(b)) == OSHUN_OK) break;
    }
    if (rc) return fail(rc);
    // device clocks and per-problem steps
    CKB(cudaMalloc(&b->d_clocks, sizeof(double) * 3 * n));
    CKB(cudaMalloc(&b->d_dt, sizeof(double) * n));
    CKB(cudaMalloc(&b->d_collide, sizeof(int) * n));
    {
        std::vector<double> dt(n);
        for (int i = 0; i < n; ++i) dt[i] = b->P[i]->cfg.dt;
        CKB(cudaMemcpy(b->d_dt, dt.data(), sizeof(double) * n, cudaMemcpyHostToDevice));
        CKB(cudaMemcpy(b->d_collide, b->collide.data(), sizeof(int) * n, cudaMemcpyHostToDevice));
    }
    // collision groups by ceil(nump / 32) and, within one nump class, by
    // whether a cell's shared memory allows at least 8 resident one-warp CTAs
    // per SM (the pivots of every l take 2 l0 nump doubles), so that a few
    // problems with large l0 do not set the footprint of all the others;
    // descriptors per state parity, (problem, cell) items
    auto ctas_per_sm = [](size_t smem) {
        const size_t k = (size_t)228 * 1024 / (smem + 1024);   // 1 KB reserved per CTA
        return (int)std::min<size_t>(16, std::max<size_t>(1, k));
    };
    for (int E = 1; E <= 8; ++E)
    for (int wide = 1; wide >= 0; --wide) {
        oshun_batch_ctx::Group g;
        g.E = E;
        std::vector<CollideArgs> args[2];
        std::vector<int2> items;
        for (int i = 0; i < n; ++i) {
            oshun_ctx* h = b->P[i];
            if (!b->collide[i] || (h->cfg.nump + 31) / 32 != E) continue;
            if ((ctas_per_sm(collide_tri_smem_per_cell(h->cfg.nump, h->cfg.l0)) >= 8) != (wide == 1)) continue;
            const int local = (int)args[0].size();
            for (int c = 0; c < 2; ++c) {
                const int cur0 = h->cur;
                h->cur = c;
                CollideArgs a = collide_args(h, 1, 1, 1, 0, 0.0, 0.0);
                h->cur = cur0;
                a.clock = b->d_clocks + 3 * i;
                a.small_dt = h->cfg.small_dt;
                args[c].push_back(a);
            }
            g.smem = std::max(g.smem, collide_tri_smem_per_cell(h->cfg.nump, h->cfg.l0));
            for (long long cell = 0; cell < h->cells; ++cell) items.push_back(make_int2(local, (int)cell));
        }
        if (items.empty()) continue;
        // chunked form where it keeps at least as many warps resident: CTAs of
        // W cells of one problem share the problem's velocity tables in shared
        // memory (per SM: 228 KB of shared memory with 1 KB reserved per CTA,
        // 64 K registers granted in 256-register units per warp, 32 CTAs)
        {
            int npmax = 0;
            for (const auto& a : args[0]) npmax = std::max(npmax, a.np);
            const size_t tab = 12 * (size_t)npmax, celld = g.smem / sizeof(double);
            auto resident = [](size_t bytes, int W, int regs) {
                const int by_smem = (int)((size_t)228 * 1024 / (bytes + 1024));
                const int per_warp = (regs * 32 + 255) / 256 * 256;
                const int by_regs = 65536 / (per_warp * W);
                return W * std::min(std::min(by_smem, by_regs), 32);
            };
            const int f32 = b->fp32 ? 1 : 0;
            const int plain = resident(g.smem, 1, collide_batch_regs(E, f32, 0));
            const int rchunk = collide_batch_regs(E, f32, 1);
            int bestW = 0, bestWarps = 0;
            for (int W = 1; W <= 8; ++W) {
                const size_t bytes = collide_chunk_smem(W, (int)tab, (int)celld);
                if (bytes > (size_t)227 * 1024) break;
                const int warps = resident(bytes, W, rchunk);
                if (warps >= bestWarps) { bestWarps = warps; bestW = W; }
            }
            if (bestW > 0 && bestWarps >= plain) {
                std::vector<int4> chunks;
                for (size_t k = 0; k < items.size();) {
                    const int p = items[k].x, c0 = items[k].y;
                    int cnt = 0;
                    while (k < items.size() && items[k].x == p && cnt < bestW) { ++k; ++cnt; }
                    chunks.push_back(make_int4(p, c0, cnt, 0));
                }
                g.warps = bestW;
                g.tab_doubles = (int)tab;
                g.nchunks = (long long)chunks.size();
                CKB(cudaMalloc(&g.d_chunks, sizeof(int4) * chunks.size()));
                CKB(cudaMemcpy(g.d_chunks, chunks.data(), sizeof(int4) * chunks.size(), cudaMemcpyHostToDevice));
            }
        }
        b->groups.push_back(g);
        auto& gg = b->groups.back();
        gg.nitems = (long long)items.size();
        for (int c = 0; c < 2; ++c) {
            CKB(cudaMalloc(&gg.d_args[c], sizeof(CollideArgs) * args[c].size()));
            CKB(cudaMemcpy(gg.d_args[c], args[c].data(), sizeof(CollideArgs) * args[c].size(), cudaMemcpyHostToDevice));
        }
        CKB(cudaMalloc(&gg.d_items, sizeof(int2) * items.size()));
        CKB(cudaMemcpy(gg.d_items, items.data(), sizeof(int2) * items.size(), cudaMemcpyHostToDevice));
    }
#undef CKB
    if ((rc = batch_upload_clocks(b))) return fail(rc);
    *out = b;
    return OSHUN_OK;
}

int oshun_batch_destroy(oshun_batch b) {
    if (!b) return OSHUN_ERR_ARG;
    cudaStreamSynchronize(b->stream);
    free_batch(b);
    return OSHUN_OK;
}

int oshun_batch_set_stream(oshun_batch b, void* stream) {
    if (!b) return OSHUN_ERR_ARG;
    CK(cudaStreamSynchronize(b->stream));
    batch_drop_graphs(b);
    b->graphs_ok = true;
    cudaStream_t next = (cudaStream_t)stream;
    if (!next) CK(cudaStreamCreateWithFlags(&next, cudaStreamNonBlocking));
    // the problems move first: oshun_set_stream waits on their current (the old) stream
    for (oshun_ctx* h : b->P) {
        int rc = oshun_set_stream(h, next);
        if (rc) return rc;
    }
    if (b->own_stream) cudaStreamDestroy(b->stream);
    b->stream = next;
    b->own_stream = stream == nullptr;
    return OSHUN_OK;
}

int oshun_batch_size(oshun_batch b, int* n) {
    if (!b || !n) return OSHUN_ERR_ARG;
    *n = (int)b->P.size();
    return OSHUN_OK;
}

int oshun_batch_problem(oshun_batch b, int i, oshun_handle* h) {
    if (!b || !h || i < 0 || i >= (int)b->P.size()) return OSHUN_ERR_ARG;
    *h = b->P[i];
    return OSHUN_OK;
}

int oshun_batch_upload(oshun_batch b, int i, const double* harmonics, const double* fields) {
    if (!b || i < 0 || i >= (int)b->P.size()) return OSHUN_ERR_ARG;
    return oshun_upload(b->P[i], harmonics, fields);
}

int oshun_batch_download(oshun_batch b, int i, double* harmonics, double* fields) {
    if (!b || i < 0 || i >= (int)b->P.size()) return OSHUN_ERR_ARG;
    return oshun_download(b->P[i], harmonics, fields);
}

int oshun_batch_set_tiles(oshun_batch b, int stage_threads, int tile_cells) {
    if (!b || stage_threads < 32 || stage_threads > 320 || stage_threads % 32 || tile_cells < 1 || tile_cells > 8)
        return OSHUN_ERR_ARG;
    CK(cudaStreamSynchronize(b->stream));
    const int nc0 = b->nc, tx0 = b->tx_cap;
    b->nc = stage_threads;
    b->tx_cap = tile_cells;
    int rc = batch_build_items(b);
    if (rc) {
        const std::string why = g_last_error;
        b->nc = nc0; b->tx_cap = tx0;
        batch_build_items(b);
        set_error(why);
        return rc;
    }
    batch_drop_graphs(b);
    return OSHUN_OK;
}

int oshun_batch_get_tiles(oshun_batch b, int* stage_threads, int* tile_cells) {
    if (!b) return OSHUN_ERR_ARG;
    if (stage_threads) *stage_threads = b->nc;
    if (tile_cells) *tile_cells = b->tx_cap;
    return OSHUN_OK;
}

int oshun_batch_step(oshun_batch b, int nsteps) {
    if (!b || nsteps < 0) return OSHUN_ERR_ARG;
    int rc = batch_upload_clocks(b);
    if (rc) return rc;
    for (int s = 0; s < nsteps; ++s) {
        cudaGraphExec_t& g = b->graph[b->cur];
        if (!g && b->graphs_ok) {
            cudaGraph_t graph = nullptr;
            bool ok = cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeRelaxed) == cudaSuccess;
            rc = ok ? batch_enqueue_step(b, b->cur) : OSHUN_OK;
            if (ok) ok = cudaStreamEndCapture(b->stream, &graph) == cudaSuccess && rc == OSHUN_OK;
            if (ok) ok = cudaGraphInstantiate(&g, graph, 0) == cudaSuccess;
            if (graph) cudaGraphDestroy(graph);
            if (!ok) {
                (void)cudaGetLastError();
                if (g) { cudaGraphExecDestroy(g); g = nullptr; }
                b->graphs_ok = false;
                if (rc) return rc;
            }
        }
        if (g) {
            CK(cudaGraphLaunch(g, b->stream));
            batch_advance_host(b);
        } else if ((rc = batch_steps_plain(b, 1))) {
            return rc;
        }
    }
    CK(cudaStreamSynchronize(b->stream));
    return OSHUN_OK;
}

int oshun_batch_status(oshun_batch b, int* flags) {
    if (!b) return OSHUN_ERR_ARG;
    int st = 0;
    CK(cudaMemcpyAsync(&st, b->d_status, sizeof(int), cudaMemcpyDeviceToHost, b->stream));
    CK(cudaStreamSynchronize(b->stream));
    int any = st;
    for (oshun_ctx* h : b->P) {
        int f = 0;
        int rc = oshun_status_flags(h, &f, nullptr);
        if (rc) return rc;
        any |= f;
    }
    if (flags) *flags = any;
    return OSHUN_OK;
}

// Times every stage tiling candidate -- consumer threads per CTA x cells per
// tile -- on `steps` steps of the batch itself (after one untimed step) and
// keeps the fastest.  The state and the clocks are restored after each trial.
int oshun_batch_autotune(oshun_batch b, int steps, int* stage_threads, int* tile_cells, double* ms_per_step) {
    if (!b || steps < 1) return OSHUN_ERR_ARG;
    CK(cudaStreamSynchronize(b->stream));
    const int n = (int)b->P.size();
    std::vector<void*> bak(3 * n, nullptr);
    int rc = OSHUN_OK;
    // copy every problem's current set to (save) or from (restore) the backup
    auto save_restore = [&](bool save) -> int {
        for (int i = 0; i < n; ++i) {
            oshun_ctx* h = b->P[i];
            void* live[3] = {h->f00[b->cur], h->pl[b->cur], h->fld[b->cur]};
            const size_t sz[3] = {sizeof(double) * h->pstride,
                                  h->ts * std::max<long long>(1, (long long)h->nplanes * h->pstride),
                                  h->ts * 6 * h->cells};
            for (int k = 0; k < 3; ++k) {
                if (save) {
                    if (!bak[3 * i + k]) CK(cudaMalloc(&bak[3 * i + k], sz[k]));
                    CK(cudaMemcpyAsync(bak[3 * i + k], live[k], sz[k], cudaMemcpyDeviceToDevice, b->stream));
                } else {
                    CK(cudaMemcpyAsync(live[k], bak[3 * i + k], sz[k], cudaMemcpyDeviceToDevice, b->stream));
                }
            }
        }
        return OSHUN_OK;
    };
    const int cur0 = b->cur;
    std::vector<double> t0(n), tee0(n), teb0(n);
    for (int i = 0; i < n; ++i) { t0[i] = b->P[i]->t; tee0[i] = b->P[i]->t_ee; teb0[i] = b->P[i]->t_eb; }
    auto reset_clocks = [&]() {
        b->cur = cur0;
        for (int i = 0; i < n; ++i) {
            b->P[i]->cur = cur0; b->P[i]->t = t0[i]; b->P[i]->t_ee = tee0[i]; b->P[i]->t_eb = teb0[i];
        }
        return batch_upload_clocks(b);
    };
    rc = save_restore(true);
    if (!rc) {
        const int nc_c[] = {128, 192, 256, 320};
        const int tx_c[] = {1, 2, 4, 8};
        int best_nc = b->nc, best_tx = b->tx_cap;
        double best = 1e300;
        cudaEvent_t e0, e1;
        cudaEventCreate(&e0);
        cudaEventCreate(&e1);
        for (int nc : nc_c) {
            for (int tx : tx_c) {
                b->nc = nc;
                b->tx_cap = tx;
                if (batch_build_items(b) != OSHUN_OK) { (void)cudaGetLastError(); continue; }
                if ((rc = batch_steps_plain(b, 1))) break;
                cudaEventRecord(e0, b->stream);
                if ((rc = batch_steps_plain(b, steps))) break;
                cudaEventRecord(e1, b->stream);
                cudaEventSynchronize(e1);
                float ms = 0.f;
                cudaEventElapsedTime(&ms, e0, e1);
                if (ms / steps < best) { best = ms / steps; best_nc = nc; best_tx = tx; }
                if ((rc = save_restore(false))) break;
                if ((rc = reset_clocks())) break;
            }
            if (rc) break;
        }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        b->nc = best_nc;
        b->tx_cap = best_tx;
        const int rc2 = batch_build_items(b);
        if (!rc) rc = rc2;
        if (!rc) rc = save_restore(false);
        if (!rc) rc = reset_clocks();
        batch_drop_graphs(b);
        if (stage_threads) *stage_threads = best_nc;
        if (tile_cells) *tile_cells = best_tx;
        if (ms_per_step) *ms_per_step = best;
    }
    cudaStreamSynchronize(b->stream);
    for (void* p : bak) cudaFree(p);
    return rc;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Adjoint of the small step, 1D with m0 = 0, FP64 (no counterpart in the
// reference, which has no derivatives).  oshun_adjoint_forward runs one step
// of the production path on caller-owned device vectors; oshun_adjoint_vjp
// recomputes that step's RK4 stage states with the production stage kernels
// and applies the transposes of adjoint.cu:
//   lambda_1 = cotangent of the step's output;
//   collision step transpose (if collisions) at the RK4 output y1;
//   RK4 transpose, s1..s4 the stage inputs, h the step:
//     a4 = F'(s4)^T (h/6 l), a3 = F'(s3)^T (h/3 l + h a4),
//     a2 = F'(s2)^T (h/3 l + h/2 a3), a1 = F'(s1)^T (h/6 l + h/2 a2),
//     lambda_0 = l + a1 + a2 + a3 + a4.
// ---------------------------------------------------------------------------
struct oshun_adj_ctx {
    oshun_ctx* h = nullptr;
    long long n = 0;                 // doubles of one state vector
    double *s2 = nullptr, *s3 = nullptr, *s4 = nullptr, *y1 = nullptr;
    double *lam1 = nullptr, *c = nullptr, *a = nullptr, *acc = nullptr;
    adj::Coef1* d_coef1 = nullptr;
    bool general = false;            // a 2D grid or m0 > 0: the general stage transpose
    double* ws = nullptr;
    long long ws_cap = 0;            // doubles
    bool async = false;              // a caller's stream is set: calls are queued on it and do not wait
};

namespace {

// FP64 state vector <-> handle set; an FP32-split handle rounds the planes
// and fields to FP32 on the way in (f00 stays FP64)
int adj_copy_in(oshun_ctx* h, int set, const double* y) {
    const size_t pb = sizeof(double) * h->pstride;
    const long long npl = (long long)h->nplanes * h->pstride;
    const double* yf = y + (1 + (long long)h->nplanes) * h->pstride;
    CK(cudaMemcpyAsync(h->f00[set], y, pb, cudaMemcpyDeviceToDevice, h->stream));
    if (h->fp32) {
        CK(launch_convert(y + h->pstride, (float*)h->pl[set], npl, h->stream));
        CK(launch_convert(yf, (float*)h->fld[set], 6 * h->cells, h->stream));
    } else {
        CK(cudaMemcpyAsync(h->pl[set], y + h->pstride, pb * h->nplanes, cudaMemcpyDeviceToDevice, h->stream));
        CK(cudaMemcpyAsync(h->fld[set], yf, sizeof(double) * 6 * h->cells, cudaMemcpyDeviceToDevice, h->stream));
    }
    return OSHUN_OK;
}
int adj_copy_out(oshun_ctx* h, int set, double* y) {
    const size_t pb = sizeof(double) * h->pstride;
    const long long npl = (long long)h->nplanes * h->pstride;
    double* yf = y + (1 + (long long)h->nplanes) * h->pstride;
    CK(cudaMemcpyAsync(y, h->f00[set], pb, cudaMemcpyDeviceToDevice, h->stream));
    if (h->fp32) {
        CK(launch_convert((const float*)h->pl[set], y + h->pstride, npl, h->stream));
        CK(launch_convert((const float*)h->fld[set], yf, 6 * h->cells, h->stream));
    } else {
        CK(cudaMemcpyAsync(y + h->pstride, h->pl[set], pb * h->nplanes, cudaMemcpyDeviceToDevice, h->stream));
        CK(cudaMemcpyAsync(yf, h->fld[set], sizeof(double) * 6 * h->cells, cudaMemcpyDeviceToDevice, h->stream));
    }
    return OSHUN_OK;
}

void free_adj(oshun_adj_ctx* a) {
    if (a->h) free_ctx(a->h);
    cudaFree(a->s2); cudaFree(a->s3); cudaFree(a->s4); cudaFree(a->y1);
    cudaFree(a->lam1); cudaFree(a->c); cudaFree(a->a); cudaFree(a->acc);
    cudaFree(a->d_coef1); cudaFree(a->ws);
    delete a;
}

adj::Grid1 adj_grid(const oshun_adj_ctx* a) {
    const oshun_ctx* h = a->h;
    adj::Grid1 g;
    g.np = h->cfg.nump; g.nx = h->cfg.numx; g.l0 = h->cfg.l0;
    g.invp = h->d_ptab; g.vr = h->d_ptab + h->cfg.nump; g.wj = h->d_ptab + 2 * h->cfg.nump;
    g.coef = a->d_coef1;
    g.g00_s = h->g00_s; g.g00_inv = h->g00_inv; g.g00_gr = h->g00_gr;
    return g;
}

adj2::Grid2 adj_grid2(const oshun_ctx* h) {
    adj2::Grid2 g;
    g.np = h->cfg.nump; g.nx = h->cfg.numx; g.ny = h->cfg.numy; g.l0 = h->cfg.l0; g.m0 = h->cfg.m0;
    g.nplanes = h->nplanes;
    g.cells = h->cells; g.pstride = h->pstride;
    g.invp = h->d_ptab; g.vr = h->d_ptab + h->cfg.nump; g.wj = h->d_ptab + 2 * h->cfg.nump;
    g.coef = h->d_coef; g.plane_of = h->d_plane_of;
    g.g00_s = h->g00_s; g.g00_inv = h->g00_inv; g.g00_gr = h->g00_gr;
    g.idx = h->idx; g.idy = h->idy;
    return g;
}

adj::CollTables adj_tables(const oshun_ctx* h) {
    adj::CollTables T;
    const int np = h->cfg.nump;
    const double* V = h->d_vtab;
    T.np = np; T.NB = h->cfg.NB_algorithms;
    T.vr = V; T.U4 = V + np; T.U4m1 = V + 2 * np; T.U2 = V + 3 * np; T.U2m1 = V + 4 * np;
    T.U1 = V + 5 * np; T.U1m1 = V + 6 * np; T.U3 = V + 7 * np; T.Qn = V + 8 * np; T.Pn = V + 9 * np;
    T.V5 = V + 10 * np; T.V7 = V + 11 * np;
    T.density_np = h->cfg.density_np; T.Zeta = h->cfg.Zeta; T.c_kpre = h->c_kpre; T.kpre = h->kpre;
    return T;
}

}  // namespace

extern "C" {

int oshun_adjoint_create(const oshun_cfg* cfg, oshun_adjoint* out) {
    if (!out || !cfg) { set_error("NULL argument"); return OSHUN_ERR_ARG; }
    *out = nullptr;
    if (!cfg->if_tridiagonal || ((cfg->nump + 31) / 32) * 32 > 256) {
        set_error("the adjoint covers tridiagonal collisions and nump <= 256");
        return OSHUN_ERR_UNSUPPORTED;
    }
    const bool general = cfg->numy > 1 || cfg->m0 > 0;
    if (general && cfg->precision != OSHUN_FP64) {
        set_error("the FP32 bulk adjoint covers 1D runs with m0 = 0");
        return OSHUN_ERR_UNSUPPORTED;
    }
    if (cfg->flags & OSHUN_FLAG_IMPLICIT_EE) {
        set_error("the adjoint transposes the explicit e-e substeps, not the implicit e-e step");
        return OSHUN_ERR_UNSUPPORTED;
    }
    oshun_adj_ctx* a = new oshun_adj_ctx();
    int rc = oshun_create(cfg, &a->h);
    if (rc) { delete a; return rc; }
    oshun_ctx* h = a->h;
    // FP32 bulk: the handle's planes hold f itself (the trajectory comes in as FP64 vectors)
    h->use_profile = false;
    a->n = (1 + (long long)h->nplanes) * h->pstride + 6 * h->cells;
    auto fail = [&](int code) { free_adj(a); return code; };
    double** bufs[] = {&a->s2, &a->s3, &a->s4, &a->y1, &a->lam1, &a->c, &a->a, &a->acc};
    for (double** b : bufs)
        if (cudaMalloc(b, sizeof(double) * a->n) != cudaSuccess) { set_error("cudaMalloc failed"); return fail(OSHUN_ERR_CUDA); }
    a->general = general;
    if (general) {
        *out = a;
        return OSHUN_OK;
    }
    const int l0 = cfg->l0;
    std::vector<double> cf((size_t)(l0 + 1) * 16);
    std::vector<adj::Coef1> c1(l0 + 1);
    if (cudaMemcpy(cf.data(), h->d_coef, sizeof(double) * cf.size(), cudaMemcpyDeviceToHost) != cudaSuccess) {
        set_error("coefficient copy failed");
        return fail(OSHUN_ERR_CUDA);
    }
    for (int l = 0; l <= l0; ++l) {
        const CoefLM* k = reinterpret_cast<const CoefLM*>(cf.data()) + l;
        c1[l] = adj::Coef1{k->ex_g, k->ex_h, k->ax_p, k->ax_m, k->gfac, k->invpax, k->hp0};
    }
    if (cudaMalloc(&a->d_coef1, sizeof(adj::Coef1) * c1.size()) != cudaSuccess ||
        cudaMemcpy(a->d_coef1, c1.data(), sizeof(adj::Coef1) * c1.size(), cudaMemcpyHostToDevice) != cudaSuccess) {
        set_error("coefficient upload failed");
        return fail(OSHUN_ERR_CUDA);
    }
    *out = a;
    return OSHUN_OK;
}

int oshun_adjoint_destroy(oshun_adjoint a) {
    if (!a) return OSHUN_ERR_ARG;
    cudaStreamSynchronize(a->h->stream);
    free_adj(a);
    return OSHUN_OK;
}

int oshun_adjoint_set_stream(oshun_adjoint a, void* stream) {
    if (!a) return OSHUN_ERR_ARG;
    const int rc = oshun_set_stream(a->h, stream);
    a->async = rc == OSHUN_OK && stream != nullptr;
    return rc;
}

int oshun_adjoint_state_size(oshun_adjoint a, long long* n) {
    if (!a || !n) return OSHUN_ERR_ARG;
    *n = a->n;
    return OSHUN_OK;
}

int oshun_adjoint_forward(oshun_adjoint a, const double* y, double* y_next, int collisions, double t, double t_ee,
                          double t_eb) {
    if (!a || !y || !y_next) return OSHUN_ERR_ARG;
    oshun_ctx* h = a->h;
    int rc = adj_copy_in(h, h->cur, y);
    if (rc) return rc;
    h->t = t; h->t_ee = t_ee; h->t_eb = t_eb;
    if (a->async) {
        // queued on the caller's stream: the clock set by a kernel, no wait
        clock_set_kernel<<<1, 1, 0, h->stream>>>(h->d_clock, t, t_ee, t_eb);
        CK(cudaGetLastError());
        if ((rc = enqueue_steps(h, 1, collisions ? 1 : 0))) return rc;
        return adj_copy_out(h, h->cur, y_next);
    }
    if ((rc = oshun_step(h, 1, collisions))) return rc;
    if ((rc = adj_copy_out(h, h->cur, y_next))) return rc;
    CK(cudaStreamSynchronize(h->stream));
    return OSHUN_OK;
}

int oshun_adjoint_vjp(oshun_adjoint a, const double* y, const double* lam_next, double* lam, int collisions, double t,
                      double t_ee, double t_eb) {
    if (!a || !y || !lam_next || !lam) return OSHUN_ERR_ARG;
    oshun_ctx* h = a->h;
    const double dt = h->cfg.dt;
    const int B = h->cur, A = h->cur ^ 1, Sa = 2, Sb = 3;
    int rc;
    // stage inputs of the step (the production stage kernels)
    if ((rc = adj_copy_in(h, B, y))) return rc;
    if ((rc = launch_stage(h, B, B, A, Sa, 0, 1, 0.5 * dt, 1.0 / 3.0))) return rc;
    if ((rc = adj_copy_out(h, Sa, a->s2))) return rc;
    if ((rc = launch_stage(h, Sa, B, A, Sb, 0, 0, 0.5 * dt, 2.0 / 3.0))) return rc;
    if ((rc = adj_copy_out(h, Sb, a->s3))) return rc;
    if ((rc = launch_stage(h, Sb, B, A, Sa, 0, 0, dt, 1.0 / 3.0))) return rc;
    if ((rc = adj_copy_out(h, Sa, a->s4))) return rc;
    if ((rc = launch_stage(h, Sa, B, A, -1, 0, 0, dt / 6.0, 1.0))) return rc;
    if ((rc = adj_copy_out(h, A, a->y1))) return rc;
    CK(cudaMemcpyAsync(a->lam1, lam_next, sizeof(double) * a->n, cudaMemcpyDeviceToDevice, h->stream));
    // collision step transpose at y1
    if (collisions) {
        const double t_new = t + dt;
        const int nsub = (int)((t_new - t_ee) / h->cfg.small_dt) + 1;   // def-FokkerPlanck.cpp:598-599
        const double hsub = (t_new - t_ee) / (double)nsub;
        const double Dt = t_new - t_eb;
        const long long wsz = adj::coll_ws(h->cfg.nump, h->cfg.l0, nsub);
        if (wsz * h->cells > a->ws_cap) {
            CK(cudaStreamSynchronize(h->stream));
            cudaFree(a->ws);
            a->ws = nullptr;
            CK(cudaMalloc(&a->ws, sizeof(double) * wsz * h->cells));
            a->ws_cap = wsz * h->cells;
        }
        const int mmax = h->cfg.if_implicit1D ? 0 : h->cfg.m0;
        CK(launch_collide_adj(adj_tables(h), h->cfg.l0, (int)h->cells, a->y1, a->lam1, 1, 1, nsub, hsub, Dt, a->ws,
                              wsz, h->stream, a->general ? h->d_plane_of : nullptr, h->cfg.m0, mmax));
    }
    // RK4 transpose
    const adj::Grid1 g = adj_grid(a);
    const adj2::Grid2 g2 = adj_grid2(h);
    const long long n = a->n;
    CK(cudaMemcpyAsync(a->acc, a->lam1, sizeof(double) * n, cudaMemcpyDeviceToDevice, h->stream));
    const double* S[4] = {y, a->s2, a->s3, a->s4};
    const double w_out[4] = {dt / 6.0, dt / 3.0, dt / 3.0, dt / 6.0};
    const double w_in[4] = {0.0, 0.5 * dt, 0.5 * dt, dt};   // weight of k_{i-1} in s_i
    for (int st = 3; st >= 0; --st) {
        if (st == 3) CK(launch_rk_combine(a->c, a->lam1, w_out[3], a->lam1, 0.0, nullptr, 0.0, n, h->stream));
        else CK(launch_rk_combine(a->c, a->lam1, w_out[st], a->a, w_in[st + 1], nullptr, 0.0, n, h->stream));
        if (a->general) CK(launch_stage_vjp2(g2, S[st], a->c, a->a, h->stream));
        else CK(launch_stage_vjp(g, S[st], a->c, a->a, h->stream, h->fp32));
        CK(launch_rk_combine(a->acc, a->acc, 1.0, a->a, 1.0, nullptr, 0.0, n, h->stream));
    }
    CK(cudaMemcpyAsync(lam, a->acc, sizeof(double) * n, cudaMemcpyDeviceToDevice, h->stream));
    if (!a->async) CK(cudaStreamSynchronize(h->stream));
    return OSHUN_OK;
}

}  // extern "C"
