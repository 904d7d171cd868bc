/* oshun_b200 — C ABI of the B200 (sm_100a) implementation of OSHUN's
 * per-time-step hot path: the RK4 Vlasov-Maxwell stage on the spherical-
 * harmonic distribution f_lm(p,x,y) and the Fokker-Planck collision step.
 *
 * Plain C linkage, plain pointers and sizes.  Every entry point returns an
 * oshun_status code; none throws or exits.  Each entry point names the
 * reference interface it replaces (paths are within the OSHUN repository).
 *
 * Host data layout (the reference's storage order without guard cells):
 *   harmonics: complex128, [Nh][numy][numx][nump], harmonic index ind(l,m)
 *              (OSHUN-1/def-State.cpp:420-427), Nh = (m0+1)(2 l0-m0+2)/2
 *              (OSHUN-1/def-State.cpp:417), p fastest
 *              (OSHUN-1/matrices.h:714-716)
 *   fields:    complex128, [6][numy][numx] in the order Ex Ey Ez Bx By Bz
 *              (OSHUN-1/decl-state.h:120-125)
 * Boundaries are periodic in x and y; the reference's RKLevel = 4 guard
 * cells are not stored (a periodic stencil gives the same interior values,
 * OSHUN-1/def-Input.cpp:156-164).
 */
#ifndef OSHUN_B200_H
#define OSHUN_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define OSHUN_ABI_VERSION 1

typedef enum oshun_status {
    OSHUN_OK = 0,
    OSHUN_ERR_ARG = 1,          /* bad pointer, size or configuration value */
    OSHUN_ERR_UNSUPPORTED = 2,  /* configuration outside the compiled range */
    OSHUN_ERR_CUDA = 3,         /* a CUDA runtime call failed (see oshun_last_error) */
    OSHUN_ERR_NONREAL = 4,      /* upload: an m=0 harmonic or a field has an imaginary part */
    OSHUN_ERR_NUMERIC = 5,      /* a step produced NaN/Inf (see oshun_status_flags) */
    OSHUN_ERR_NO_DEVICE = 6     /* no CUDA device, or not an sm_100 device */
} oshun_status;

typedef enum oshun_precision {
    OSHUN_FP64 = 0,       /* every operator in IEEE FP64: the drop-in */
    OSHUN_FP32_SPLIT = 1  /* f_lm (l >= 1), fields and their arithmetic in FP32 (the planes
                             stored relative to an FP64 momentum profile, see
                             oshun_plane_profile); f00, the Rosenbluth integrals, the
                             collision solves and the current reduction in FP64 */
} oshun_precision;

/* flags */
#define OSHUN_FLAG_FIX_YADV_CHAIN 0x1  /* drop the reference's y-advection coefficient
                                          factor C1[l-1]/C1[m+1] that OSHUN-1 carries for
                                          m >= 2 (def-VlasovMax.cpp:916-946) */
#define OSHUN_FLAG_IMPLICIT_EE 0x2     /* opt-in, not in the reference: the f00 e-e step
                                          as one backward-Euler step over the whole
                                          interval (three Picard sweeps of a per-cell
                                          tridiagonal solve of the same discrete flux
                                          operator) instead of the explicit RK4
                                          substeps of Explicit_EC_FP::loop
                                          (def-FokkerPlanck.cpp:590-625) */

/* Run configuration: the input-deck fields the hot path reads
 * (OSHUN-1/decl-input.h:59-138, derived values as in
 * OSHUN-1/def-Input.cpp:79,156-164,313-334). */
typedef struct oshun_cfg {
    int l0, m0;              /* harmonic truncation, 0 <= m0 <= l0 */
    int nump, numx, numy;    /* interior cells; numy = 1 for a 1D run */
    double pmin, pmax;       /* p_i = i (pmax-pmin)/(nump-1) + pmin (matrices.h:860-866) */
    double xmin, xmax;       /* dx = (xmax-xmin)/(numx-1) (the reference's xglob axis) */
    double ymin, ymax;       /* dy likewise; unused when numy = 1 */
    double dt;               /* RK4 step h (Runge_Kutta_4 ctor, def-RK.cpp:60-61) */
    double t0;               /* start time of the RK, e-e and implicit clocks */
    double small_dt;         /* bound on the f00 e-e substep (def-FokkerPlanck.cpp:598) */
    int NB_algorithms;       /* low-v cells of the e-e flux (def-FokkerPlanck.cpp:241) */
    int if_tridiagonal;      /* 1: Thomas solve; 0: dense matrix + Gauss-Seidel */
    int if_implicit1D;       /* 1: implicit collisions on m = 0 only (f1_loop1D/flm_loop1D) */
    double density_np;       /* electron density in 1/cm^3 (Coulomb logarithms) */
    double Zeta;             /* ion charge */
    int precision;           /* oshun_precision */
    int flags;               /* OSHUN_FLAG_* */
} oshun_cfg;

typedef struct oshun_ctx* oshun_handle;

/* ---- lifetime ---------------------------------------------------------- */

/* Allocates the device state for cfg and builds the operator tables.
 * Replaces the construction of Stat, Runge_Kutta_4, Explicit_EC_FP and
 * Euler_Backward (OSHUN-1/main.cpp:147-199; def-State.cpp:533-538;
 * def-RK.cpp:49-62; def-FokkerPlanck.cpp:568-585, 1258-1266). */
int oshun_create(const oshun_cfg* cfg, oshun_handle* out);
int oshun_destroy(oshun_handle h);

/* Runs the handle's work on this cudaStream_t (passed as void*; NULL = the
 * handle's own stream). */
int oshun_set_stream(oshun_handle h, void* stream);
int oshun_synchronize(oshun_handle h);

/* ---- state transfer ------------------------------------------------------ */

/* Host -> device copy of the state.  Replaces filling a Stat
 * (Setup_Y::initialize, OSHUN-1/def-Setup.cpp:293-471, or
 * Restart_Facility::Read, def-Export.cpp:733-766).  m = 0 harmonics and the
 * fields must be real (OSHUN_ERR_NONREAL otherwise): every reference operator
 * maps real m = 0 harmonics and real fields to real values. */
int oshun_upload(oshun_handle h, const double* harmonics, const double* fields);
/* Device -> host copy of the state (replaces reading Stat, e.g.
 * Restart_Facility::Write, def-Export.cpp:768-836). */
int oshun_download(oshun_handle h, double* harmonics, double* fields);

/* ---- operators ------------------------------------------------------------ */

/* slope = Actions::Adv(state) (OSHUN-1/def-Actions.cpp:73-94): E-field,
 * current, Ampere, advection, B-field, Faraday, CLEAN_LOW_PC.  Writes the
 * slope to host buffers in the state layout; the state is unchanged. */
int oshun_rhs(oshun_handle h, double* slope_harmonics, double* slope_fields);

/* One RK4 step of h = cfg.dt: Runge_Kutta_4::advance_p1
 * (OSHUN-1/def-RK.cpp:110-145).  Advances the RK clock. */
int oshun_rk4_step(oshun_handle h);

/* Explicit_EC_FP::loop(t_new) (OSHUN-1/def-FokkerPlanck.cpp:590-625): f00
 * e-e collisions, floor((t_new - t_ee)/small_dt)+1 RK4 substeps per cell. */
int oshun_collide_ee(oshun_handle h, double t_new);

/* Euler_Backward::advance_1(t_new) (OSHUN-1/def-FokkerPlanck.cpp:1270-1286):
 * implicit step of f10 (and f11 in 2D) over t_new - t_eb. */
int oshun_collide_f1(oshun_handle h, double t_new);
/* Euler_Backward::advance_lm(t_new) (OSHUN-1/def-FokkerPlanck.cpp:1290-1304):
 * implicit step of every f_lm with l >= 2; sets t_eb = t_new. */
int oshun_collide_flm(oshun_handle h, double t_new);

/* nsteps of the reference's small-step sequence (OSHUN-1/main.cpp:77-107):
 * rk4.advance_p1; ee.loop(t); eb.advance_1(t); eb.advance_lm(t).  Runs as a
 * CUDA graph once captured.  `collisions` = 0 skips the collision calls. */
int oshun_step(oshun_handle h, int nsteps, int collisions);

/* ---- x boundaries and x slabs -------------------------------------------- */

/* The reference's x boundary of a grid (input deck bndX, OSHUN-1/
 * def-Parallel.cpp:1115-1135) and its split over ranks in x
 * (Parallel_Environment::Neighbor_Communications, :3040-3129):
 *   OSHUN_XB_PERIODIC  (default) sameNode_periodic_X, :1138-1158;
 *   OSHUN_XB_MIRROR    sameNode_mirror_X (:1160-1206): the guard next to an
 *                      edge column is that column, times (-1)^(l+m) on f_lm
 *                      and -1 on Ey, Ez and Bx (every l; the reference leaves
 *                      the l = l0 guards as they are);
 *   OSHUN_XB_HALO      the grid is one x slab of a larger grid: the x-1
 *                      neighbour of column 0 and the x+1 neighbour of column
 *                      numx-1 are halo columns the caller loads before every
 *                      RK4 stage (oshun_halo_pack on each rank, the exchange
 *                      with the left and right ranks, oshun_halo_unpack), and
 *                      the step runs stage by stage (oshun_step_stage).
 * FP64 only for MIRROR and HALO; y stays periodic. */
#define OSHUN_XB_PERIODIC 0
#define OSHUN_XB_MIRROR 1
#define OSHUN_XB_HALO 2
int oshun_set_x_boundary(oshun_handle h, int mode);
/* bytes of one halo column set (one edge column: f00 [numy][nump] FP64, the
 * l >= 1 planes [nplanes][numy][nump], the fields [6][numy], each part
 * 256-byte aligned) */
int oshun_halo_bytes(oshun_handle h, long long* bytes);
/* the next stage's input columns x = 0 -> left_edge and x = numx-1 ->
 * right_edge (device buffers of oshun_halo_bytes each; the left one goes to
 * the left neighbour, the right one to the right neighbour) */
int oshun_halo_pack(oshun_handle h, void* left_edge, void* right_edge);
/* the neighbours' columns: from_left = the left rank's right_edge, from_right
 * = the right rank's left_edge (device buffers) */
int oshun_halo_unpack(oshun_handle h, const void* from_left, const void* from_right);
/* the halo of side 0 (left) or 1 (right) as a mirrored boundary of the next
 * stage's input (the end ranks of a slab split with bndX = 1:
 * Node_Communications::mirror_bound_Xleft/right, def-Parallel.cpp:964-1031,
 * called at :3058, 3075) */
int oshun_halo_mirror_side(oshun_handle h, int side);
/* RK4 stage k (1..4, in order) of the small step; stage 4 completes the RK4
 * step (Runge_Kutta_4::advance_p1) and, with `collisions`, runs the e-e and
 * implicit f_lm steps of oshun_step. */
int oshun_step_stage(oshun_handle h, int k, int collisions);

/* nsteps of the reference's small step with the implicit electric field
 * (OSHUN-1/main.cpp:77-107 with implicit_E; Runge_Kutta_2_Imp, def-RK.cpp:
 * 399-588; Implicit_E_Field, def-ImplicitE.cpp:471-676), cfg.dt the RK2 step h.
 * mask selects the calls of each step, in this order (63 = the whole step):
 *    1  rk.advance_p1   RK2 of advection, B and Faraday (Implicit_Actions::Adv1)
 *    2  ee.loop(t)      f00 e-e collisions
 *   16  em.advance      the implicit E: probes of the collisional plasma's
 *                       response to DE = sqrt(eps)|E| + eps in each component
 *                       (their RK2 effect on l <= 2 and the f1 solve), the
 *                       finite-difference conductivity tensor and a 3x3 solve
 *                       per cell for the E whose current matches rot B (1D,
 *                       if_implicit1D: Ex with zero current), up to 4 attempts
 *   32  rk.advance_p2   RK2 of the new E's couplings (Adv2) and CLEAN_LOW_PC
 *    4  eb.advance_1(t) implicit f1 collisions
 *    8  eb.advance_lm(t) implicit f_lm collisions
 * The probe's finite differences amplify rounding by about 1/sqrt(16 eps):
 * results agree with the reference to the reference's own sensitivity to a
 * 1-ulp change of its input (about 1e-8 relative).  Returns OSHUN_ERR_NUMERIC
 * where the reference exits (a zero determinant left in more than 8 cells). */
int oshun_rk2_imp_step(oshun_handle h, int nsteps, int mask);

/* ---- queries -------------------------------------------------------------- */

/* RK clock (Runge_Kutta_4::time, OSHUN-1/def-RK.cpp:76). */
int oshun_time(oshun_handle h, double* t);
/* Status word: bit 0 = a Gauss-Seidel solve found its matrix not diagonally
 * dominant and kept f (the reference's WARNING, def-FokkerPlanck.cpp:1027-1030);
 * bit 1 = NaN/Inf in the state (checked by this call); bit 2 = an implicit-E
 * solve left cells with a zero determinant after its 4 attempts (the
 * reference's WARNING, def-ImplicitE.cpp:666-669); bit 4 = a pipeline wait
 * of a stage launch gave up (that launch returned without finishing: the state
 * is undefined).  *count = skipped solves since the last call.  Reading clears
 * the word. */
int oshun_status_flags(oshun_handle h, int* flags, long long* count);
/* Device pointers of the state planes for zero-copy use: the f00 plane
 * (FP64, [numy][numx][nump]), the other planes (see oshun_plane_index), the
 * 6 field planes; sizes in bytes. */
int oshun_device_state(oshun_handle h, void** f00, void** planes, void** fields,
                       size_t* planes_bytes, size_t* fields_bytes);
/* Plane index of the real part of harmonic (l,m) in `planes` (the imaginary
 * part, m > 0, follows it), or -1 for (0,0), which lives in `f00`. */
int oshun_plane_index(oshun_handle h, int l, int m, int* plane);
/* OSHUN_FP32_SPLIT: the l >= 1 planes hold f minus a momentum profile per
 * plane, the average over the cells of the state at its last upload
 * (rounded to FP32), so that the x and y differences of a harmonic with a
 * large, nearly uniform part act on its small deviation and FP32 storage
 * keeps that deviation's precision.  *profile = the device array
 * [nplanes][nump] (FP64 values), or NULL in OSHUN_FP64 and in batches. */
int oshun_plane_profile(oshun_handle h, const double** profile);
/* The configuration the handle was created with. */
int oshun_get_config(oshun_handle h, oshun_cfg* cfg);

/* ---- moments on the device -------------------------------------------------- */

/* Parallel_Output::nonrelativistic_moments (OSHUN-1/def-Parallel.cpp:1677-2258)
 * for every cell, computed on the device from the current state; out receives
 * OSHUN_NUM_MOMENTS float planes [numy][numx] in the order below (the
 * reference's Matrix2D<float> results in its normalised units; N is the
 * density those moments divide by, 1 where it is below 4 FLT_EPSILON).  The
 * reference's float accumulation order is kept, so results agree with its
 * output files to a few float ulps.  Harmonics the run does not carry
 * (f11, f2m for small l0, m0) count as zero.  Kx (Ky) needs numx (numy) >= 3;
 * with fewer cells the derivative of <v^2>^2 is taken as zero. */
enum oshun_moment {
    OSHUN_MOM_N = 0, OSHUN_MOM_VX, OSHUN_MOM_VY, OSHUN_MOM_VXVX, OSHUN_MOM_VYVY, OSHUN_MOM_VZVZ,
    OSHUN_MOM_VXVY, OSHUN_MOM_VXVZ, OSHUN_MOM_VYVZ, OSHUN_MOM_VSQ, OSHUN_MOM_T_EV, OSHUN_MOM_P_MBAR,
    OSHUN_MOM_ND, OSHUN_MOM_NU, OSHUN_MOM_QX, OSHUN_MOM_KX, OSHUN_MOM_QY, OSHUN_MOM_KY, OSHUN_NUM_MOMENTS
};
int oshun_moments(oshun_handle h, float* out);

/* ---- restart files ---------------------------------------------------------- */

/* The reference's restart files, byte for byte (Restart_Facility::Write/Read,
 * OSHUN-1/def-Export.cpp:733-836): <prefix>_<rank:06>_<step:03>.dat (prefix
 * NULL = "RESTART/re", the reference's), the Stat written raw with
 * guard_cells (the deck's RKLevel) guard cells per side: every harmonic in
 * ind(l,m) order as complex128 [numy+2g][numx+2g][nump], then the 6 fields as
 * complex128 [numy+2g][numx+2g].  Guards hold the periodic image of the
 * interior, as the reference leaves them after each step
 * (def-Parallel.cpp:1138-1158, 1229-1248); a 1D run (numy = 1) has 1 + 2g
 * rows, each holding the interior row.  Reading takes the interior cells (and
 * uploads them: OSHUN_ERR_NONREAL as oshun_upload).  A periodic image needs
 * numx (and numy > 1) >= guard_cells.
 * The pack/unpack forms convert between host buffers in the oshun_download
 * layout and a file image; they need no device. */
long long oshun_restart_bytes(const oshun_cfg* cfg, int guard_cells);
int oshun_restart_pack(const oshun_cfg* cfg, int guard_cells, const double* harmonics, const double* fields,
                       double* image);
int oshun_restart_unpack(const oshun_cfg* cfg, int guard_cells, const double* image, double* harmonics,
                         double* fields);
int oshun_restart_write(oshun_handle h, const char* prefix, int rank, int re_step, int guard_cells);
int oshun_restart_read(oshun_handle h, const char* prefix, int rank, int re_step, int guard_cells);

/* ---- batches of independent problems -------------------------------------- */

/* No counterpart in the reference, whose runs are one problem per process
 * (the loop over runs a caller would write around main_loop).  A batch holds
 * n independent problems of one precision, any mix of l0, m0 <= 8, nump <=
 * 256 (nump x element size a multiple of 16 bytes), numx, numy and dt, each
 * with its own state and clocks.  oshun_batch_step advances every problem by
 * one small step of its own dt per step (oshun_step's sequence) with one
 * captured CUDA graph per step: four persistent stage launches over the
 * (problem, tile) list of the whole batch and one collision launch per group
 * of problems with equal ceil(nump/32).  collide[i] = 0 (or collide = NULL
 * for all on) skips problem i's collision calls; collisional problems need
 * if_tridiagonal = 1. */
typedef struct oshun_batch_ctx* oshun_batch;
int oshun_batch_create(const oshun_cfg* cfgs, int n, const int* collide, oshun_batch* out);
int oshun_batch_destroy(oshun_batch b);
/* Runs the batch's work on this cudaStream_t (NULL = the batch's own stream);
 * the captured graphs are rebuilt on the next step. */
int oshun_batch_set_stream(oshun_batch b, void* stream);
int oshun_batch_size(oshun_batch b, int* n);
/* the handle of problem i (owned by the batch; its queries and transfers work,
 * its stream is the batch's) */
int oshun_batch_problem(oshun_batch b, int i, oshun_handle* h);
int oshun_batch_upload(oshun_batch b, int i, const double* harmonics, const double* fields);
int oshun_batch_download(oshun_batch b, int i, double* harmonics, double* fields);
int oshun_batch_step(oshun_batch b, int nsteps);
/* OR of every problem's status word (oshun_status_flags) and bit 4 = a
 * pipeline wait of a batched launch ran out. */
int oshun_batch_status(oshun_batch b, int* flags);
/* Stage tiles: consumer threads per CTA (32..320, a multiple of 32, at least
 * the widest padded nump of the batch) and cells per tile at most (1..8). */
int oshun_batch_set_tiles(oshun_batch b, int stage_threads, int tile_cells);
int oshun_batch_get_tiles(oshun_batch b, int* stage_threads, int* tile_cells);
/* Autotuner: times every tile candidate (stage threads 128/192/256/320 x cells
 * per tile 1/2/4/8) on `steps` steps of the batch itself, keeps the fastest
 * and restores the state and clocks; returns the choice and its ms/step. */
int oshun_batch_autotune(oshun_batch b, int steps, int* stage_threads, int* tile_cells, double* ms_per_step);

/* ---- adjoint of the small step ------------------------------------------- */

/* No counterpart in the reference, which computes no derivatives.  For any
 * grid (1D or 2D, any m0) with tridiagonal collisions and nump <= 256, in
 * FP64; for 1D runs with m0 = 0 also the FP32 bulk form (precision
 * OSHUN_FP32_SPLIT: the forward steps keep the l >= 1 planes and fields in
 * FP32, and the stage transposes run in FP32 arithmetic; f00, the collision
 * transposes and the cotangent vectors stay FP64).  The flag
 * OSHUN_FLAG_IMPLICIT_EE is refused.  The entry points give the
 * vector-Jacobian product of one small step (oshun_step's sequence: RK4
 * Vlasov-Maxwell step, then, with `collisions`, the e-e substeps and the
 * implicit f_lm solves).  State vectors are device arrays of
 * oshun_adjoint_state_size doubles in the plane layout: the f00 plane, the
 * l >= 1 planes (oshun_plane_index; [numy][numx][nump] each), the 6 field
 * planes.  (t, t_ee, t_eb) are the
 * RK, e-e and implicit clocks before the step (Runge_Kutta_4::t,
 * Explicit_EC_FP::t, Euler_Backward::t): they fix the step's e-e substeps
 * and implicit step as in the forward.  For 1D runs with m0 = 0 the
 * cotangents of the fields other than E_x come back zero: they never act on
 * f or E_x there. */
typedef struct oshun_adj_ctx* oshun_adjoint;
int oshun_adjoint_create(const oshun_cfg* cfg, oshun_adjoint* out);
int oshun_adjoint_destroy(oshun_adjoint a);
/* Without a stream set, oshun_adjoint_forward and oshun_adjoint_vjp run on
 * the handle's own stream and return when their results are written.  With a
 * caller's stream set (non-null), both are queued on that stream and return
 * without waiting: the caller orders its own reads and writes of the vectors
 * on the same stream.  A null stream restores the waiting form. */
int oshun_adjoint_set_stream(oshun_adjoint a, void* stream);
int oshun_adjoint_state_size(oshun_adjoint a, long long* n);
/* y_next = step(y) through the production kernels */
int oshun_adjoint_forward(oshun_adjoint a, const double* y, double* y_next, int collisions, double t, double t_ee,
                          double t_eb);
/* lam = (d step / d y)^T lam_next at y (stage states recomputed from y) */
int oshun_adjoint_vjp(oshun_adjoint a, const double* y, const double* lam_next, double* lam, int collisions, double t,
                      double t_ee, double t_eb);

/* ---- allocation-free collision step --------------------------------------- */

/* No counterpart in the reference.  The implicit f_lm collision step (the work
 * of oshun_collide_f1 followed by oshun_collide_flm, over Dt) on device planes
 * the caller owns, for callers that cannot allocate device memory in their
 * time loop (an application that gives all device memory to its own pool at
 * start-up, or a foreign runtime that owns every device buffer).  The call
 * allocates nothing: its tables and, in the dense Gauss-Seidel mode, its
 * matrix workspace live in a fixed 32 MiB __device__ array that every GPU
 * loading the library holds until exit.
 *   cfg        the run configuration; precision must be OSHUN_FP64; limits
 *              l0 <= 64, m0 <= 8, nump <= 1024 and one nump x nump FP64
 *              matrix within the 32 MiB (OSHUN_ERR_UNSUPPORTED beyond them)
 *   f00        device pointer, FP64 f00 plane [numy][numx][nump] (read)
 *   planes     device pointer, the l >= 1 planes in the layout of
 *              oshun_device_state / oshun_plane_index, FP64 (read/written)
 *   Dt         implicit step (Euler_Backward's t_new - t)
 *   stream     cudaStream_t (NULL: the default stream)
 *   nondominant  optional out: the number of Gauss-Seidel solves skipped as
 *              not diagonally dominant
 *   flags      optional out: the status word of oshun_status_flags (bit 0 =
 *              a skipped solve, bit 1 = NaN/Inf in the result planes)
 * Without nondominant and flags the call only enqueues work on the stream.
 * With either, it also checks the result planes for NaN/Inf, waits for the
 * stream, stores the outputs and returns OSHUN_ERR_NUMERIC when bit 1 is set.
 * The first call on a device looks up the array's device address; make it
 * before any stream capture.  Later calls can be captured with nondominant
 * and flags NULL (their read-back is refused, OSHUN_ERR_UNSUPPORTED, while
 * the stream captures).  Every call shares the array and it keeps the
 * last call's contents: calls that overlap on the GPU race on it. */
int oshun_collide_flm_noalloc(const oshun_cfg* cfg, double* f00, double* planes, double Dt, void* stream,
                              long long* nondominant, int* flags);

/* ---- fault injection for tests -------------------------------------------- */

/* No counterpart in the reference.  Arms a failure of the pipelined stage
 * kernel for the next oshun_rk4_step only (the captured step graphs of
 * oshun_step never carry it): in each of that step's four stage launches the
 * first CTA's source producer stops before its withhold_copy-th bulk copy, so
 * the consumers waiting for that copy give up after wait_seconds (1e-4 to 1)
 * instead of the default 1 s.  The launches return, bit 4 of the status word
 * is set (oshun_status_flags) and the state is undefined until the next
 * oshun_upload; the handle stays usable.  No GPU fault is involved: every
 * wait of the kernel is bounded and every copy issued is waited for. */
int oshun_debug_inject_stage_timeout(oshun_handle h, int withhold_copy, double wait_seconds);

/* Human-readable message of the last error on this thread. */
const char* oshun_last_error(void);
int oshun_abi_version(void);

#ifdef __cplusplus
}
#endif
#endif
