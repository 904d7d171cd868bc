/* CPU restatement of the OSHUN-1 hot path (test infrastructure only).
 *
 * This is the checker the CUDA path is compared against; nothing in the
 * product links it.  It restates, in closed form and on a periodic grid
 * without guard cells, the reference's
 *   Actions::Adv            (OSHUN-1/def-Actions.cpp:73-94)
 *   Runge_Kutta_4           (OSHUN-1/def-RK.cpp:110-145)
 *   Explicit_EC_FP::loop    (OSHUN-1/def-FokkerPlanck.cpp:590-625)
 *   Euler_Backward          (OSHUN-1/def-FokkerPlanck.cpp:1270-1304)
 * Parity of this restatement is pinned against the reference's own code
 * (oracle/_ref/oshun_ref) and against the golden cases in tests/golden.
 *
 * Data layout: the case layout of oracle/ref_harness/harness.cpp — every
 * harmonic complex128 [numy][numx][nump] in ind(l,m) order
 * (OSHUN-1/def-State.cpp:420-427), then 6 complex128 fields [numy][numx]
 * (Ex, Ey, Ez, Bx, By, Bz). */
#ifndef OSHUN_ORACLE_H
#define OSHUN_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct oo_deck {
    int l0, m0, nump, numx, numy, NB_algorithms, if_tridiagonal, if_implicit1D;
    double pmin, pmax, xmin, xmax, ymin, ymax, dt, small_dt, density_np, Zeta;
} oo_deck;

/* keep (1, default) or drop (0) the reference's y-advection coefficient
 * chain factor for m >= 2 (see oo_yadv_factor in oshun_oracle.c) */
void oo_set_yadv_chain(int keep);

/* e-e step of later oo_steps calls: 0 (default) the reference's explicit RK4
 * substeps; sweeps > 0 the opt-in backward-Euler step with that many Picard
 * sweeps (OSHUN_FLAG_IMPLICIT_EE of the CUDA path) */
void oo_set_ee_implicit(int sweeps);

/* x boundaries of later calls: 0 periodic (default), 1 mirrored
 * (sameNode_mirror_X: (-1)^(l+m) on f_lm, -1 on Ey, Ez, Bx, every l) */
void oo_set_mirror_x(int on);

long oo_state_doubles(const oo_deck* d);

/* slope = Actions::Adv(state) */
int oo_rhs(const oo_deck* d, const double* state, double* slope);

/* nsteps of the main loop order; mask bits: 1 RK4, 2 e-e f00, 4 f1 implicit,
 * 8 flm (l>=2) implicit.  Returns 0, or -1 on a bad deck. */
int oo_steps(const oo_deck* d, double* state, int nsteps, int mask);

/* Gauss-Seidel solves skipped as not diagonally dominant by the last
 * oo_steps call (the reference prints a warning and keeps f,
 * OSHUN-1/def-FokkerPlanck.cpp:1027-1030) */
long oo_nondominant_count(void);

#ifdef __cplusplus
}
#endif
#endif
