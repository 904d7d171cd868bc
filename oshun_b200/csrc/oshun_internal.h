// Internal declarations shared by the CUDA translation units of liboshun_b200.
#pragma once

#include "adjoint_math.h"
#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "oshun_b200.h"

namespace oshun {

// Largest m0 the RK-stage kernel is compiled for; each instantiation keeps
// 3 x (MC+1) complex accumulators per thread.
constexpr int kMaxM0 = 8;
// Largest nump (threads of one cell row are one CTA dimension).
constexpr int kMaxNp = 1024;
// Picard sweeps of the opt-in backward-Euler e-e step (OSHUN_FLAG_IMPLICIT_EE)
constexpr int kEeImplicitSweeps = 3;

// Coupling coefficients of one source harmonic (l,m).  Each names the target
// it feeds; a coefficient of a target that does not exist is 0 and the
// target slot is never stored.  16-byte aligned, 128 bytes: the kernels copy
// entries with 128-bit loads and stores.
struct alignas(16) CoefLM {
    double ex_g, ex_h;      // Ex*G -> (l+1,m),   Ex*H -> (l-1,m)
    double em_g, em_h;      // Em*G -> (l+1,m+1), Em*H -> (l-1,m+1)   Em = Ey - i Ez
    double ep_h, ep_g;      // Ep*H -> (l-1,m-1), Ep*G -> (l+1,m-1)   Ep = Ey + i Ez (Re if m = 1)
    double ax_p, ax_m;      // x advection -> (l+1,m), (l-1,m)
    double ay_pp, ay_mp;    // y advection -> (l+1,m+1), (l-1,m+1)
    double ay_mm, ay_pm;    // y advection -> (l-1,m-1), (l+1,m-1)   (Re if m = 1)
    double b_m;             // (Bz - i By) f -> (l,m-1)               (Re if m = 1)
    double gfac;            // G = Dp f * gfac + H,  gfac = -(2l+1)/l
    double invpax;          // H = f * invpax/p + Dp f, invpax = -2(l+1) dp
    double hp0;             // H at the p0 cell = f(p1) * hp0
};
static_assert(sizeof(CoefLM) == 128 && alignof(CoefLM) == 16, "CoefLM layout");

// Parts of the right-hand side a stage launch evaluates.  Actions::Adv
// (def-Actions.cpp:73-94) is every part; the implicit-E actions
// (Implicit_Actions, def-Actions.cpp:117-218) are subsets: Adv1 = B +
// advection + Faraday, Adv2 = E + CLEAN_LOW_PC, ImpEx/y/z = one E component
// with a restricted coupling table.
enum : int {
    kPartEx = 1, kPartEy = 2, kPartEz = 4,   // E couplings, per component of the stage-input field
    kPartB = 8,                              // B couplings
    kPartAdv = 16,                           // x and y advection
    kPartAmpere = 32,                        // dE/dt: current and rot B
    kPartFaraday = 64,                       // dB/dt: -rot E
    kPartClean = 128,                        // CLEAN_LOW_PC on the slope
    kPartAll = 255
};

// Arguments of one fused RHS + RK4 stage launch.  TS is the storage and
// arithmetic type of the l >= 1 planes and the fields; f00 is always FP64.
template <typename TS>
struct StageArgs {
    const double* f00_in; const TS* pl_in; const TS* fld_in;   // stage input (F is evaluated here)
    // FP32 split: the l >= 1 planes store f minus this momentum profile of
    // each plane ([nplanes][np]); null: the planes store f
    const TS* pl_ref;
    const int* pl_keep;   // [nplanes]: 0 where the plane's profile is zero (its loads are skipped)
    const double* f00_B;  const TS* pl_B;  const TS* fld_B;    // step base Y0
    double* f00_A;        TS* pl_A;        TS* fld_A;          // RK accumulator Y
    double* f00_out;      TS* pl_out;      TS* fld_out;        // next stage input (or the slope)
    const CoefLM* coef;   // [(l0+1)*(m0+1)]
    const int* plane_of;  // [(l0+1)*(m0+1)]: plane of Re f_lm (l >= 1), -1 otherwise
    const double* inv_pr; // 1/p
    const double* vr;     // p/gamma
    const double* wj;     // current quadrature weight (4 pi/3 included)
    long long cells;      // numx*numy
    long long pstride;    // cells*nump (elements per plane)
    int np, nx, ny, l0, m0;
    int mode;             // 0: RK stage; 1: write the slope to *_out
    int first;            // stage 1: A = B + t*c2 instead of A += t*c2
    double c1, c2;        // t = k*c1; out = B + t; A (+)= t*c2
    double g00_s, g00_inv, g00_gr;   // p0 extrapolation of f00 for G00
    double idx, idy;      // -1/(2dx), -1/(2dy)
    // bulk-copy pipelined variant
    const int* seq;       // [nh]: source harmonics in stream order, s | (m << 16)
    int nh;
    int* err;             // error word (bit 4: a pipeline wait timed out)
    unsigned long long wait_ns;   // a pipeline wait gives up after this many ns (single-problem kernel)
    int parts;            // kPart* bits of the RHS evaluated (kPartAll: Actions::Adv); any other
                          // set runs the global-load kernel (the implicit-E actions)
    int withhold;         // fault injection for tests: CTA 0's source producer skips this copy (-1: none)
    const void* coef_ts;  // coupling table in the arithmetic type (batched launches)
    double* jw;           // [cells][3][8]: per-warp partial sums of Jx, Re Jy, Im Jy (single-problem pipeline)
    // x halo columns of the stage input (null: periodic in x).  Side 0 is the
    // x-1 neighbour of column 0, side 1 the x+1 neighbour of column nx-1;
    // one side (hx_side bytes apart): f00 [ny][np] FP64, at hx_pl the l >= 1
    // planes [nplanes][ny][np], at hx_fld the fields [6][ny]
    const unsigned char* hx;
    long long hx_side, hx_pl, hx_fld;
};

template <typename TS>
__device__ __forceinline__ const double* hx_f00(const StageArgs<TS>& a, int side, long long y) {
    return reinterpret_cast<const double*>(a.hx + side * a.hx_side) + y * a.np;
}
template <typename TS>
__device__ __forceinline__ const TS* hx_plane(const StageArgs<TS>& a, int side, long long q, long long y) {
    return reinterpret_cast<const TS*>(a.hx + side * a.hx_side + a.hx_pl) + (q * a.ny + y) * a.np;
}
template <typename TS>
__device__ __forceinline__ TS hx_field(const StageArgs<TS>& a, int side, int k, long long y) {
    return reinterpret_cast<const TS*>(a.hx + side * a.hx_side + a.hx_fld)[(long long)k * a.ny + y];
}

struct CollideArgs {
    double* f00;          // FP64 f00 plane (in/out)
    void* planes;         // l >= 1 planes (double or float)
    int planes_fp32;
    const double* pl_ref; // [nplanes][np] momentum profile the planes are stored relative to (null: none)
    const float* pl_ref32;   // the same profile in FP32 (it is FP32-rounded: the values are equal)
    const int* pl_keep;      // [nplanes]: 0 where the plane's profile is zero
    const int* plane_of;  // [(l0+1)*(m0+1)]
    const int* plane_l;   // [nplanes]: l of each plane
    const int* plane_m;   // [nplanes]: m of each plane
    int nplanes;
    long long cells, pstride;
    int np, l0, m0, mmax_coll;   // harmonics m <= min(l, mmax_coll) are collided
    int do_ee, do_l1, do_lm;
    int if_tridiagonal;
    int nsub;             // e-e RK4 substeps
    int ee_implicit;      // > 0: the e-e step is the backward-Euler one (launch_ee_implicit), this many sweeps
    double hsub;          // e-e substep
    double Dt;            // implicit step
    int NB;
    double density_np, Zeta;
    double c_kpre, kpre;  // 4pi/3 re kp, re kp
    // velocity grid tables [np]
    const double *vr, *U4, *U4m1, *U2, *U2m1, *U1, *U1m1, *U3, *Qn, *Pn, *V5, *V7;
    int chunk;            // planes staged per pass (tridiagonal path)
    double* dense_ws;     // dense path: np*np doubles per block
    int* status;          // [0] flags, [1] non-dominant count
    // when set, nsub/hsub/Dt come from this device clock {t, t_ee, t_eb} at
    // kernel start (the reference's clock arithmetic, see collide_params)
    const double* clock;
    double small_dt;
};

// x halo column sets (halo.cu): grid sizes and one side's layout
struct HaloGrid {
    int nx, ny, np, nplanes;
    long long pstride, cells;
    long long off_pl, off_fld;      // byte offsets of the planes and fields in one side
    const int *plane_l, *plane_m;   // [nplanes]
};
// the edge columns x = 0 and x = nx-1 of one state set into side0 / side1
// (times the mirror signs when `mirror`)
cudaError_t launch_halo_columns(const double* f00, const void* pl, const void* fld, const HaloGrid& g, bool fp32,
                                void* side0, void* side1, int mirror, cudaStream_t st);
// one column x0 into one side's column set
cudaError_t launch_halo_column(const double* f00, const void* pl, const void* fld, const HaloGrid& g, bool fp32,
                               int x0, void* out, int mirror, cudaStream_t st);

// opt-in backward-Euler e-e step (a.ee_implicit sweeps), one warp per cell
cudaError_t launch_ee_implicit(const CollideArgs& a, cudaStream_t st);

// batched collision launch: CollideArgs per problem, (problem, cell) work items
struct CollideBatch {
    const CollideArgs* probs;
    const int2* items;
    long long nitems;
    // chunked form: CTAs of `warps` warps, one chunk (problem, first cell,
    // cells) per CTA, the problem's velocity tables staged in shared memory
    const int4* chunks;
    long long nchunks;
    int warps;
    int tab_doubles;    // 12 x the group's largest nump
    int cell_doubles;   // work space of one cell
};

// launchers (return cudaError_t)
// pipelined stage kernel (stage_pipe.cu); cudaErrorNotSupported when the shape does not fit
template <typename TS>
cudaError_t launch_stage_pipe(const StageArgs<TS>& a, int mc, cudaStream_t s);
cudaError_t launch_stage_fp64(const StageArgs<double>& a, int mc, cudaStream_t s);
// The work of one stage launch: a list of tiles, either of one problem (the
// kernel parameter) or of a batch of problems (`probs` holds one StageArgs per
// problem, `items` the (problem, tile) pairs).  In a batch the first bulk copy
// of each tile also brings the problem's descriptor into the slot's header.
struct BatchWork {
    const unsigned char* probs;   // StageArgs<TS>[nprob], desc_bytes apart
    const int2* items;            // (problem, tile)
    int nitems;
    int tx_cap;                   // cells per tile at most
    int desc_bytes;               // sizeof(StageArgs<TS>) rounded to 16
    int ncoef_max;                // largest (l0+1)(m0+1) of the batch
    int hdr_bytes;                // slot header: the descriptor
    int slot_bytes, row_arr_bytes;   // largest slot / staged-row array of the batch
    int row_depth;                // staged-row ring depth (2..8)
    int nprobs;                   // problems of the batch
};
// batched stage kernel (stage_batch.cu); nc consumer threads per CTA
template <typename TS>
cudaError_t launch_stage_batch(const StageArgs<TS>& a1, const BatchWork& bw, int mc, int nc, cudaStream_t s);
size_t stage_batch_smem(const BatchWork& bw, int elem_bytes);
void stage_batch_sizes(int np, int nx, int ny, int l0, int m0, int nc, int tx_cap, int elem_bytes, int* tx,
                       size_t* slot_bytes, size_t* row_arr_bytes);
int stage_batch_coef_bytes(int elem_bytes);
cudaError_t launch_stage_fp32(const StageArgs<float>& a, int mc, cudaStream_t s);
cudaError_t launch_collide(const CollideArgs& a, cudaStream_t s, size_t smem_bytes, int blocks);
size_t collide_smem_bytes(int np, int chunk, int if_tridiagonal);
int collide_max_chunk(int np, size_t smem_budget);
int collide_threads();
size_t collide_tri_smem_per_cell(int np, int l0);
// adjoint kernels of the 1D m0 = 0 step (adjoint.cu; types in adjoint_math.h)
cudaError_t launch_stage_vjp(const adj::Grid1& g, const double* s, const double* c, double* out, cudaStream_t st,
                             bool fp32);
// FP64 state vector <-> FP32 planes/fields (the FP32 bulk adjoint)
cudaError_t launch_convert(const double* src, float* dst, long long n, cudaStream_t st);
cudaError_t launch_convert(const float* src, double* dst, long long n, cudaStream_t st);
cudaError_t launch_collide_adj(const adj::CollTables& T, int l0, int nx, const double* y, double* lam, int ee, int eb,
                               int nsub, double hsub, double Dt, double* ws, long long wsz, cudaStream_t st,
                               const int* plane_of = nullptr, int m0 = 0, int mmax = 0);
cudaError_t launch_rk_combine(double* out, const double* v0, double a0, const double* v1, double a1, const double* v2,
                              double a2, long long n, cudaStream_t st);
// tridiagonal collision step of a batch whose problems share E = ceil(np/32) <= 8
cudaError_t launch_collide_batch(const CollideBatch& b, int E, int planes_fp32, size_t smem, cudaStream_t s);
// shared memory of one chunked batched-collision CTA
size_t collide_chunk_smem(int warps, int tab_doubles, int cell_doubles);
// registers per thread of the batched collision kernel for this E (chunked or one cell per CTA)
int collide_batch_regs(int E, int planes_fp32, int chunked);
// device clocks {t, t_ee, t_eb} of n problems: t += dt; after a collision step t_ee = t_eb = t
cudaError_t launch_clock_advance(double* clocks, const double* dt, int n, cudaStream_t s);
cudaError_t launch_clock_commit(double* clocks, const int* collide, int n, cudaStream_t s);
cudaError_t launch_collide_tri(const CollideArgs& a, cudaStream_t s, int cells_per_cta, int blocks);
cudaError_t launch_nan_check(const double* f00, const void* planes, int planes_fp32, long long n_f00,
                             long long n_planes, const void* fields, long long n_fields, int* status,
                             cudaStream_t s);

// Moments of Parallel_Output::nonrelativistic_moments (moments.cu); output
// planes [kMomCount][numy][numx] in this order (the public oshun_moment enum)
enum { kMomN = 0, kMomVx, kMomVy, kMomVxVx, kMomVyVy, kMomVzVz, kMomVxVy, kMomVxVz, kMomVyVz, kMomVsq, kMomT, kMomP,
       kMomND, kMomNu, kMomQx, kMomKx, kMomQy, kMomKy, kMomCount };
struct MomentArgs {
    const double* f00;    // FP64 f00 plane
    const void* planes;   // l >= 1 planes (double or float)
    const double* pl_ref; // [nplanes][np] momentum profile the planes are stored relative to (null: none)
    long long cells, pstride;
    int np, nx, ny;
    int q10, q11, q20, q21, q22;   // plane of Re f_lm, -2 when the harmonic is absent
    // momentum tables [np]: p, 1/gamma, and the host's pow() of the reference's moments
    const double *pr, *invgamma, *ig2, *ig3, *pow3, *pow4, *pow5;
    double dp, p0p1_sq, inv_mp0p1_sq, corr5, corr7;
    double density_np, Zeta, nu_pre;
    // scalings rounded to float as Matrix2D<float> *= <double> does
    float s_dens, s_v1, s_v2, s_m2, s_vyvy, s_vxvy, s_vxvz, s_vyvz, s_pre, s_kx, s_ky;
    float* out;           // [kMomCount + 1][cells]: the moments, then a scratch plane
};
cudaError_t launch_moments(const MomentArgs& a, int planes_fp32, cudaStream_t s);

// Implicit electric field (implicit_e.cu): per-cell kernels of
// Implicit_E_Field::advance; the probe states come from the stage and
// collision kernels
struct ImplicitArgs {
    const void* planes[4];   // l >= 1 planes of each state set (double or float)
    const double* pl_ref;    // [nplanes][np] momentum profile the planes are stored relative to (null: none)
    long long cells, pstride;
    int np, nx, ny;
    int q10, q11;            // planes of f10 and Re f11 (-1: absent)
    int fp32;
    int one_d;               // if_implicit1D: Ex alone, no Ampere
    const double* p3og;      // p^3/gamma [np]
    double dp, small, c4, c8;   // quadrature step, p0 correction, -4 pi/3, -8 pi/3
    double idx, idy;         // -1/(2 dx), -1/(2 dy)
    double eps, large_eps;   // 16 DBL_EPSILON and its square root
};
cudaError_t launch_implicit_current(const ImplicitArgs& a, int set, double* J, cudaStream_t s);
cudaError_t launch_implicit_ampere(const ImplicitArgs& a, const void* fields, double* JN, cudaStream_t s);
cudaError_t launch_implicit_find_de(const ImplicitArgs& a, const void* fields, double* DE, cudaStream_t s);
cudaError_t launch_implicit_probe_field(const ImplicitArgs& a, const double* DE, int comp, void* FE, cudaStream_t s);
cudaError_t launch_implicit_solve(const ImplicitArgs& a, const double* J0, const double* JX, const double* JY,
                                  const double* JZ, const double* JN, double* DE, double* EN, int* zeros,
                                  cudaStream_t s);
cudaError_t launch_implicit_set_e(const ImplicitArgs& a, const double* EN, void* fields, cudaStream_t s);

void set_error(const std::string& msg);

// Raises a kernel's dynamic shared-memory limit to `bytes` on the current
// device.  The attribute is per device, so the size already set is cached
// per (kernel, device), under a lock (launchers may run on several threads).
cudaError_t ensure_dyn_smem(const void* func, size_t bytes);
// SM count of the current device (148 when the query fails)
int sm_count();

}  // namespace oshun
