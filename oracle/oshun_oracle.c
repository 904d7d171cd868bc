/* CPU restatement of the OSHUN-1 hot path — TEST INFRASTRUCTURE ONLY.
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load
 * this file's library, and only as the checker.  The product (liboshun_b200)
 * never links or calls it.  See oshun_oracle.h for the data layout.
 *
 * Parity is pinned by tests/test_oracle_vs_reference.py (this code against
 * the reference's own sources built as oracle/_ref/oshun_ref) and by the
 * golden cases in tests/golden (generated by the reference build).
 *
 * The reference spreads every operator over whole-array passes with in-place
 * coefficient ratio chains.  Here each coupling is written once, in closed
 * form, as "source harmonic (l,m) -> target harmonic (l', m') with
 * coefficient c".  The per-line citations below name the reference lines each
 * coupling follows.  Rounding differs from the reference at the 1e-16 level;
 * the tests hold this file to 1e-12 relative L2 per harmonic. */
#include "oshun_oracle.h"

#include <complex.h>
#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

typedef double complex cplx;

static int g_keep_chain = 1;
static long g_nondominant = 0;

void oo_set_yadv_chain(int keep) { g_keep_chain = keep ? 1 : 0; }
/* mirrored x boundaries (Node_Communications::sameNode_mirror_X,
 * def-Parallel.cpp:1160-1206): the neighbour beyond an edge column is that
 * column, times (-1)^(l+m) on f_lm and -1 on Ey, Ez, Bx (every l) */
static int g_mirror_x = 0;
void oo_set_mirror_x(int on) { g_mirror_x = on ? 1 : 0; }
long oo_nondominant_count(void) { return g_nondominant; }

/* ------------------------------------------------------------------------ */
/* grid                                                                      */
/* ------------------------------------------------------------------------ */

typedef struct {
    const oo_deck* d;
    int l0, m0, np, nx, ny, nh;
    long cells, hsize;
    int* ind;          /* (l0+1)*(m0+1), -1 where (l,m) does not exist */
    double* pr;        /* momentum axis */
    double* vr;        /* p / gamma */
    double dp, idx, idy;
} Grid;

/* Axis(n, lo, hi): a_i = i*(hi-lo)/(n-1) + lo; dx() = a_1 - a_0
 * (OSHUN-1/matrices.h:860-866, 880) */
static double axis_point(int i, int n, double lo, double hi) {
    double step = (hi - lo) / (double)(n - 1);
    return (double)i * step + lo;
}
static double axis_dx(int n, double lo, double hi) {
    return axis_point(1, n, lo, hi) - axis_point(0, n, lo, hi);
}
/* local axis = global axis shifted by RKLevel=4 guard cells, built by
 * repeated addition (OSHUN-1/def-Input.cpp:322-325) */
static double local_dx(int nglob, double lo, double hi) {
    double dg = axis_dx(nglob, lo, hi);
    double x0 = axis_point(0, nglob, lo, hi) - 4.0 * dg;
    double x1 = x0 + dg;
    return x1 - x0;
}

static int grid_init(Grid* g, const oo_deck* d) {
    memset(g, 0, sizeof(*g));
    if (d->l0 < 0 || d->m0 < 0 || d->m0 > d->l0 || d->nump < 3 || d->numx < 1 || d->numy < 1)
        return -1;
    g->d = d;
    g->l0 = d->l0; g->m0 = d->m0;
    g->np = d->nump; g->nx = d->numx; g->ny = d->numy;
    g->nh = ((d->m0 + 1) * (2 * d->l0 - d->m0 + 2)) / 2;
    g->cells = (long)g->nx * g->ny;
    g->hsize = g->cells * g->np;
    g->ind = (int*)malloc(sizeof(int) * (g->l0 + 1) * (g->m0 + 1));
    g->pr = (double*)malloc(sizeof(double) * g->np);
    g->vr = (double*)malloc(sizeof(double) * g->np);
    /* ind(l,m) of OSHUN-1/def-State.cpp:420-427 */
    for (int l = 0; l <= g->l0; ++l)
        for (int m = 0; m <= g->m0; ++m) {
            int v = -1;
            if (m <= l) v = (l < g->m0 + 1) ? (l * (l + 1)) / 2 + m
                                            : l * (g->m0 + 1) - (g->m0 * (g->m0 + 1)) / 2 + m;
            g->ind[l * (g->m0 + 1) + m] = v;
        }
    for (int i = 0; i < g->np; ++i) {
        g->pr[i] = axis_point(i, g->np, d->pmin, d->pmax);
        g->vr[i] = g->pr[i] / sqrt(1.0 + g->pr[i] * g->pr[i]);
    }
    g->dp = g->pr[1] - g->pr[0];
    g->idx = -1.0 / (2.0 * local_dx(g->nx, d->xmin, d->xmax));
    /* a 1D case runs the reference with 4 identical global y cells; its y
     * spacing never enters (every y difference vanishes) */
    g->idy = -1.0 / (2.0 * local_dx(g->ny == 1 ? 4 : g->ny, d->ymin, d->ymax));
    return 0;
}

static void grid_free(Grid* g) {
    free(g->ind); free(g->pr); free(g->vr);
}

static int IND(const Grid* g, int l, int m) {
    if (l < 0 || l > g->l0 || m < 0 || m > g->m0 || m > l) return -1;
    return g->ind[l * (g->m0 + 1) + m];
}

long oo_state_doubles(const oo_deck* d) {
    long nh = ((d->m0 + 1) * (2 * d->l0 - d->m0 + 2)) / 2;
    long cells = (long)d->numx * d->numy;
    return 2 * (nh * cells * d->nump + 6 * cells);
}

/* periodic neighbours */
static long cell_xm(const Grid* g, long c) { long x = c % g->nx, y = c / g->nx; return y * g->nx + (x + g->nx - 1) % g->nx; }
static long cell_xp(const Grid* g, long c) { long x = c % g->nx, y = c / g->nx; return y * g->nx + (x + 1) % g->nx; }
static long cell_ym(const Grid* g, long c) { long x = c % g->nx, y = c / g->nx; return ((y + g->ny - 1) % g->ny) * g->nx + x; }
static long cell_yp(const Grid* g, long c) { long x = c % g->nx, y = c / g->nx; return ((y + 1) % g->ny) * g->nx + x; }

/* ------------------------------------------------------------------------ */
/* coupling coefficients                                                     */
/* ------------------------------------------------------------------------ */

/* E-field tables, ElectricField ctor (OSHUN-1/def-VlasovMax.cpp:97-147) */
static double eA1(const Grid* g, int l, int m) {
    if (l == 0) return -1.0 * (0.5 / g->dp);
    return (l + 1.0 - m) * l / ((2.0 * l + 1.0) * (l + 1.0)) * (0.5 / g->dp);
}
static double eA2(const Grid* g, int l, int m) { return -(l + m + 0.0) / (2.0 * l + 1.0) * (0.5 / g->dp); }
static double eB1(const Grid* g, int l) { return (-0.5 / g->dp) * l * l / (2.0 * l + 1.0); }
static double eB2(const Grid* g, int l) { return (-0.5 / g->dp) * l * (l + 1.0) / (2.0 * l + 1.0); }
static double eC1(const Grid* g, int l) {
    if (l == 0) return -0.25 / g->dp;
    return (0.25 / g->dp) * l / ((2.0 * l + 1.0) * (l + 1.0));
}
static double eC3(const Grid* g, int l) { return (0.25 / g->dp) / (2.0 * l + 1.0); }
static double eC2(const Grid* g, int l, int m) {
    return (-0.25 / g->dp) * l * (l - m + 2.0) * (l - m + 1.0) / ((2.0 * l + 1.0) * (l + 1.0));
}
static double eC4(const Grid* g, int l, int m) {
    return (-0.25 / g->dp) * (l + m - 1.0) * (l + m) / (2.0 * l + 1.0);
}
/* p0-cell extrapolation of H (def-VlasovMax.cpp:145-147) */
static double eHp0(const Grid* g, int l) {
    double h = 1.0 / g->pr[0];
    for (int k = 1; k <= l; ++k) h = h * (g->pr[0] / g->pr[1]) * (2.0 * k + 1.0) / (2.0 * k - 1);
    return h * (-2.0 * g->dp);
}

/* advection tables, Spatial_Advection ctor (def-VlasovMax.cpp:775-826) */
static double xA1(const Grid* g, int l, int m) { return g->idx * (-1.0) * (l - m + 1.0) / (2.0 * l + 1.0); }
static double xA2(const Grid* g, int l, int m) { return g->idx * (-1.0) * (l + m + 0.0) / (2.0 * l + 1.0); }
static double yB1(const Grid* g, int l) { return g->idy * (l + 1.0) * l / (2.0 * l + 1.0); }
static double yB2(const Grid* g, int l) { return -yB1(g, l); }
static double yC1(const Grid* g, int l) { return (-0.5) * g->idy / (2.0 * l + 1.0); }
static double yC3(const Grid* g, int l) { return -yC1(g, l); }
static double yC2(const Grid* g, int l, int m) { return g->idy * 0.5 * (l + 2.0 - m) * (l - m + 1.0) / (2.0 * l + 1.0); }
static double yC4(const Grid* g, int l, int m) { return g->idy * (-0.5) * (l + m - 1.0) * (l + m) / (2.0 * l + 1.0); }

/* The reference's y advection for m >= 2 walks one running multiplier
 * through its l loop and divides by C1[m+1] where C1[l-1] is meant
 * (OSHUN-1/def-VlasovMax.cpp:916-921); the multiplier also carries over into
 * the next m (def-VlasovMax.cpp:924-927, 936-946).  For parity the same factor
 * multiplies every y-advection coupling of source (l,m), m >= 2:
 *   m in [2, m0-1]:  l = m, m+1: R_m;   l in [m+2, l0-1]: q_l with q_{m+2}=R_m,
 *                    q_l = q_{l-1} C1[l-1]/C1[m+1];   l = l0: q_{l0-1};
 *                    R_{m+1} = (factor at l0) if m+1 < l0 else R_m;
 *   m = m0:          R_m0 for every l;   R_2 = 1. */
static double yadv_factor(const Grid* g, int l, int m) {
    if (!g_keep_chain || m < 2) return 1.0;
    double R = 1.0;
    for (int mm = 2; mm <= m; ++mm) {
        if (mm == g->m0) return R;               /* the m0 block */
        if (mm + 1 >= g->l0) {                   /* no l >= m+2 in this m */
            if (mm == m) return R;
            continue;
        }
        double q = R, at_l = R;
        for (int ll = mm + 2; ll <= g->l0 - 1; ++ll) {
            if (ll > mm + 2) q = q * (yC1(g, ll - 1) / yC1(g, mm + 1));
            if (mm == m && ll == l) at_l = q;
        }
        /* at l0 the factor is the last q (R when the loop was empty) */
        if (mm == m) {
            if (l <= mm + 1) return R;
            if (l == g->l0) return q;
            return at_l;
        }
        R = q;
    }
    return R;
}

/* ------------------------------------------------------------------------ */
/* RHS = Actions::Adv (def-Actions.cpp:73-94)                                */
/* ------------------------------------------------------------------------ */

static void addto(cplx* S, const Grid* g, int l, int m, long k, cplx v) {
    int h = IND(g, l, m);
    if (h >= 0) S[h * g->hsize + k] += v;
}
static void addto_re(cplx* S, const Grid* g, int l, int m, long k, cplx v) {
    int h = IND(g, l, m);
    if (h >= 0) S[h * g->hsize + k] += creal(v);
}

/* G and H of one harmonic: MakeGH (def-VlasovMax.cpp:496-515), G00
 * (def-VlasovMax.cpp:519-535), with the p-difference Dp
 * (def-State.cpp:359-380): f[p-1]-f[p+1] inside, 0 at p0,
 * f[np-2]-f[np-1] at the last cell. */
static void make_gh(const Grid* g, int l, const cplx* f, cplx* G, cplx* H) {
    const int np = g->np;
    const double p0 = g->pr[0], p1 = g->pr[1];
    const double hp0 = l > 0 ? eHp0(g, l) : 0.0;
    for (long c = 0; c < g->cells; ++c) {
        const cplx* fc = f + c * np;
        cplx* Gc = G + c * np;
        cplx* Hc = H + c * np;
        for (int p = 0; p < np; ++p) {
            cplx dpf;
            if (p == 0) dpf = 0.0;
            else if (p == np - 1) dpf = fc[np - 2] - fc[np - 1];
            else dpf = fc[p - 1] - fc[p + 1];
            if (l == 0) {
                Gc[p] = dpf;
                Hc[p] = 0.0;
            } else {
                double invpax = (1.0 / g->pr[p]) * (-2.0 * (l + 1.0) * g->dp);
                cplx h = fc[p] * invpax + dpf;
                Hc[p] = h;
                Gc[p] = dpf * (-(2.0 * l + 1.0) / l) + h;
            }
        }
        if (l == 0) {
            double s = p0 * p0 / (p1 * p1);
            double inv = 1.0 / (1.0 - s);
            double gr = -4.0 * g->dp * p0 / (p1 * p1);
            cplx f00 = (fc[0] - fc[1] * s) * inv;
            Gc[0] = (fc[1] - f00) * gr;
        } else {
            Gc[0] = 0.0;
            Hc[0] = fc[1] * hp0;
        }
    }
}

static void rhs(const Grid* g, const cplx* Y, cplx* S) {
    const int np = g->np;
    const long hs = g->hsize, cells = g->cells;
    memset(S, 0, sizeof(cplx) * (g->nh * hs + 6 * cells));
    const cplx* F = Y + g->nh * hs;          /* fields of the input */
    cplx* dF = S + g->nh * hs;               /* field slopes */
    const cplx *Ex = F, *Ey = F + cells, *Ez = F + 2 * cells;
    const cplx *Bx = F + 3 * cells, *By = F + 4 * cells, *Bz = F + 5 * cells;
    cplx* G = (cplx*)malloc(sizeof(cplx) * hs);
    cplx* H = (cplx*)malloc(sizeof(cplx) * hs);

    for (int l = 0; l <= g->l0; ++l) {
        for (int m = 0; m <= (l < g->m0 ? l : g->m0); ++m) {
            const cplx* f = Y + IND(g, l, m) * hs;
            make_gh(g, l, f, G, H);
            for (long c = 0; c < cells; ++c) {
                /* Em = Ey - i Ez, Ep = Ey + i Ez (def-VlasovMax.cpp:351-353);
                 * B- = Bz - i By, B+ = (Bz + i By)/2 (def-VlasovMax.cpp:602-607) */
                const cplx ex = Ex[c], em = Ey[c] - I * Ez[c], ep = Ey[c] + I * Ez[c];
                const cplx bx = Bx[c], bm = Bz[c] - I * By[c], bp = (Bz[c] + I * By[c]) * 0.5;
                /* advection neighbours */
                const long xc = c % g->nx;
                const double sgn = ((l + m) & 1) ? -1.0 : 1.0;
                const int mxm = g_mirror_x && xc == 0, mxp = g_mirror_x && xc == g->nx - 1;
                const cplx* fxm = f + (mxm ? c : cell_xm(g, c)) * np;
                const cplx* fxp = f + (mxp ? c : cell_xp(g, c)) * np;
                const double sxm = mxm ? sgn : 1.0, sxp = mxp ? sgn : 1.0;
                const cplx* fym = f + cell_ym(g, c) * np;
                const cplx* fyp = f + cell_yp(g, c) * np;
                const double qy = yadv_factor(g, l, m);
                for (int p = 0; p < np; ++p) {
                    const long k = c * np + p;
                    const cplx gv = G[k], hv = H[k], fv = f[k];
                    /* E-field coupling, Exyz (def-VlasovMax.cpp:346-491) */
                    if (l < g->l0) addto(S, g, l + 1, m, k, eA1(g, l, m) * ex * gv);
                    if (l >= 1 && l - 1 >= m) addto(S, g, l - 1, m, k, eA2(g, l, m) * ex * hv);
                    if (m + 1 <= g->m0) {
                        if (l < g->l0) addto(S, g, l + 1, m + 1, k, eC1(g, l) * em * gv);
                        if (l >= 1 && m + 1 <= l - 1) addto(S, g, l - 1, m + 1, k, eC3(g, l) * em * hv);
                    }
                    if (m == 1) {
                        addto_re(S, g, l - 1, 0, k, eB2(g, l) * ep * hv);
                        if (l < g->l0) addto_re(S, g, l + 1, 0, k, eB1(g, l) * ep * gv);
                    } else if (m >= 2) {
                        addto(S, g, l - 1, m - 1, k, eC4(g, l, m) * ep * hv);
                        if (l < g->l0) addto(S, g, l + 1, m - 1, k, eC2(g, l, m) * ep * gv);
                    }
                    /* B-field rotation, Bxyz (def-VlasovMax.cpp:597-644) */
                    if (m + 1 <= g->m0 && m + 1 <= l) addto(S, g, l, m + 1, k, bp * fv);
                    if (m >= 1) addto(S, g, l, m, k, (-I * (double)m) * bx * fv);
                    if (m == 1) addto_re(S, g, l, 0, k, (-(double)l * (l + 1.0)) * bm * fv);
                    else if (m >= 2) addto(S, g, l, m - 1, k, (-0.5 * (l + 1.0 - m) * (l + m)) * bm * fv);
                    /* x advection (def-VlasovMax.cpp:842-853), Dx f = f[x-1]-f[x+1]
                     * (matrices.h:813-820) */
                    const cplx dxf = (sxm * fxm[p] - sxp * fxp[p]) * g->vr[p];
                    if (l < g->l0) addto(S, g, l + 1, m, k, xA1(g, l, m) * dxf);
                    if (l >= 1 && l - 1 >= m) addto(S, g, l - 1, m, k, xA2(g, l, m) * dxf);
                    /* y advection (def-VlasovMax.cpp:857-947) */
                    if (g->ny > 1) {
                        const cplx dyf = (fym[p] - fyp[p]) * g->vr[p];
                        if (m + 1 <= g->m0) {
                            if (l < g->l0) addto(S, g, l + 1, m + 1, k, qy * yC1(g, l) * dyf);
                            if (l >= 1 && m + 1 <= l - 1) addto(S, g, l - 1, m + 1, k, qy * yC3(g, l) * dyf);
                        }
                        if (m == 1) {
                            addto_re(S, g, l - 1, 0, k, yB2(g, l) * dyf);
                            if (l < g->l0) addto_re(S, g, l + 1, 0, k, yB1(g, l) * dyf);
                        } else if (m >= 2) {
                            addto(S, g, l - 1, m - 1, k, qy * yC4(g, l, m) * dyf);
                            if (l < g->l0) addto(S, g, l + 1, m - 1, k, qy * yC2(g, l, m) * dyf);
                        }
                    }
                }
            }
        }
    }
    free(G);
    free(H);

    /* current, Current::Jxyz (def-VlasovMax.cpp:670-745): trapezoid in p of
     * f*p^3/gamma plus the 0..p0 correction small*f(p1) */
    {
        const double p0 = g->pr[0], p1 = g->pr[1];
        double small = p0;
        small *= small; small *= small; small *= p0; small *= 0.2; small *= 1.0 / p1;
        double* p3og = (double*)malloc(sizeof(double) * np);
        for (int p = 0; p < np; ++p) {
            double q = g->pr[p];
            p3og[p] = (q * q) * (q / sqrt(1.0 + q * q));
        }
        for (int which = 0; which < 2; ++which) {
            int h = IND(g, 1, which);
            if (h < 0) continue;
            const cplx* f = Y + h * hs;
            for (long c = 0; c < cells; ++c) {
                const cplx* fc = f + c * np;
                cplx j = fc[0] * p3og[0];
                j += fc[np - 1] * p3og[np - 1];
                j *= 0.5;
                for (int p = 1; p < np - 1; ++p) j += fc[p] * p3og[p];
                j *= g->dp;
                j += small * (fc[1] * p3og[1]);
                if (which == 0) {
                    j *= 4.0 * M_PI / 3.0;
                    dF[c] += j;
                } else {
                    j *= 8.0 * M_PI / 3.0;
                    dF[cells + c] += creal(j);          /* Ey += Re J */
                    dF[2 * cells + c] += -cimag(j);     /* Ez += -Im J */
                }
            }
        }
        free(p3og);
    }

    /* Ampere and Faraday, MaxwellEq (def-VlasovMax.cpp:979-1035):
     * idx*Dx g = (g[x+1]-g[x-1])/(2dx) */
    for (long c = 0; c < cells; ++c) {
        const long ym = cell_ym(g, c), yp = cell_yp(g, c);
        const long xc = c % g->nx;
        const int mxm = g_mirror_x && xc == 0, mxp = g_mirror_x && xc == g->nx - 1;
        const long xm = mxm ? c : cell_xm(g, c), xp = mxp ? c : cell_xp(g, c);
        const double sm = mxm ? -1.0 : 1.0, sp = mxp ? -1.0 : 1.0;   /* Ey, Ez flip at a mirror */
        cplx dEx = 0, dEy = 0, dEz = 0, dBx = 0, dBy = 0, dBz = 0;
        dEx += g->idy * (Bz[ym] - Bz[yp]);
        dEy += -g->idx * (Bz[xm] - Bz[xp]);
        dEz += -g->idy * (Bx[ym] - Bx[yp]);
        dEz += g->idx * (By[xm] - By[xp]);
        dBx += -g->idy * (Ez[ym] - Ez[yp]);
        dBy += g->idx * (sm * Ez[xm] - sp * Ez[xp]);
        dBz += g->idy * (Ex[ym] - Ex[yp]);
        dBz += -g->idx * (sm * Ey[xm] - sp * Ey[xp]);
        dF[c] += dEx; dF[cells + c] += dEy; dF[2 * cells + c] += dEz;
        dF[3 * cells + c] += dBx; dF[4 * cells + c] += dBy; dF[5 * cells + c] += dBz;
    }

    /* CLEAN_LOW_PC: zero the slope below p cell min(l-1, 80) for l >= 1
     * (def-Actions.cpp:240-253) */
    for (int l = 2; l <= g->l0; ++l)
        for (int m = 0; m <= (l < g->m0 ? l : g->m0); ++m) {
            cplx* s = S + IND(g, l, m) * hs;
            int nz = (l - 1) < 80 ? (l - 1) : 80;
            for (long c = 0; c < cells; ++c)
                for (int p = 0; p < nz && p < np; ++p) s[c * np + p] = 0.0;
        }
}

int oo_rhs(const oo_deck* d, const double* state, double* slope) {
    Grid g;
    if (grid_init(&g, d)) return -1;
    rhs(&g, (const cplx*)state, (cplx*)slope);
    grid_free(&g);
    return 0;
}

/* ------------------------------------------------------------------------ */
/* RK4, Runge_Kutta_4::advance_p1 (def-RK.cpp:110-145)                       */
/* ------------------------------------------------------------------------ */

static void rk4(const Grid* g, cplx* Y, double h) {
    const long n = g->nh * g->hsize + 6 * g->cells;
    cplx* Y0 = (cplx*)malloc(sizeof(cplx) * n);
    cplx* Y1 = (cplx*)malloc(sizeof(cplx) * n);
    cplx* K = (cplx*)malloc(sizeof(cplx) * n);
    memcpy(Y0, Y, sizeof(cplx) * n);
    memcpy(Y1, Y, sizeof(cplx) * n);
    rhs(g, Y1, K);
    for (long i = 0; i < n; ++i) { K[i] *= 0.5 * h; Y1[i] += K[i]; K[i] *= 1.0 / 3.0; Y[i] += K[i]; }
    rhs(g, Y1, K);
    for (long i = 0; i < n; ++i) { Y1[i] = Y0[i]; K[i] *= 0.5 * h; Y1[i] += K[i]; K[i] *= 2.0 / 3.0; Y[i] += K[i]; }
    rhs(g, Y1, K);
    for (long i = 0; i < n; ++i) { K[i] *= h; Y0[i] += K[i]; K[i] *= 1.0 / 3.0; Y[i] += K[i]; }
    rhs(g, Y0, K);
    for (long i = 0; i < n; ++i) { K[i] *= h / 6.0; Y[i] += K[i]; }
    free(Y0); free(Y1); free(K);
}

/* ------------------------------------------------------------------------ */
/* Coulomb logarithms (def-FokkerPlanck.cpp:41-95)                           */
/* ------------------------------------------------------------------------ */

static double log_ee(const oo_deck* d, double ne, double Te) {
    if (ne > 0.000000001) {
        Te /= (3.0 * ne);
        Te *= 511000;
        ne *= d->density_np;
        Te = log(Te);
        ne = log(ne);
        double v = 23.5 - 0.5 * ne + 1.25 * Te - sqrt(0.00001 + 0.0625 * (Te - 2.0) * (Te - 2.0));
        if (v > 2.0) return v;
    }
    return 2.0;
}

static double zlog_ei(const oo_deck* d, double ne, double Te) {
    if (ne > 0.0000001) {
        Te /= (3.0 * ne);
        Te *= 511000;
        ne *= d->density_np;
        Te = log(Te);
        ne = log(ne);
        double v = 24.0 - 0.5 * ne + Te;
        if (v > 2.0) return v * d->Zeta;
    }
    return 2.0 * d->Zeta;
}

static const double RE_CLASSICAL = 2.8179402894e-13;

/* velocity-grid weights shared by the e-e and f_lm operators
 * (def-FokkerPlanck.cpp:143-157, 790-803) */
typedef struct {
    int n;
    double *vr, *U4, *U4m1, *U2, *U2m1, *U1, *U1m1, *U3, *Qn, *Pn;
} VGrid;

static void vgrid_init(VGrid* v, const Grid* g) {
    const int n = g->np;
    v->n = n;
    double* buf = (double*)calloc((size_t)10 * n, sizeof(double));
    v->vr = buf; v->U4 = buf + n; v->U4m1 = buf + 2 * n; v->U2 = buf + 3 * n; v->U2m1 = buf + 4 * n;
    v->U1 = buf + 5 * n; v->U1m1 = buf + 6 * n; v->U3 = buf + 7 * n; v->Qn = buf + 8 * n; v->Pn = buf + 9 * n;
    for (int i = 0; i < n; ++i) v->vr[i] = g->vr[i];
    const double* vr = v->vr;
    for (int i = 1; i < n; ++i) {
        double dv = vr[i] - vr[i - 1];
        v->U4[i] = 0.5 * pow(vr[i], 4) * dv;
        v->U4m1[i] = 0.5 * pow(vr[i - 1], 4) * dv;
        v->U2[i] = 0.5 * vr[i] * vr[i] * dv;
        v->U2m1[i] = 0.5 * vr[i - 1] * vr[i - 1] * dv;
        v->U1[i] = 0.5 * vr[i] * dv;
        v->U1m1[i] = 0.5 * vr[i - 1] * dv;
    }
    for (int i = 0; i < n; ++i) v->U3[i] = pow(vr[i], 3);
    v->Qn[0] = 1.0 / ((vr[0] * vr[0] * vr[1]) / 2.0);
    for (int i = 1; i < n - 1; ++i) v->Qn[i] = 1.0 / (vr[i] * vr[i] * (vr[i + 1] - vr[i - 1]) / 2.0);
    for (int i = 0; i < n - 1; ++i) v->Pn[i] = 1.0 / ((vr[i + 1] - vr[i]) / 2.0 * (vr[i + 1] + vr[i]));
}
static void vgrid_free(VGrid* v) { free(v->vr); }

/* ------------------------------------------------------------------------ */
/* f00 e-e: EE_isotropic_conserva (def-FokkerPlanck.cpp:107-267),            */
/* RungeKutta4_ee (:518-553), Explicit_EC_FP::loop (:590-625)                */
/* ------------------------------------------------------------------------ */

typedef struct {
    const oo_deck* d;
    const VGrid* v;
    double c_kpre;
    double *I4, *I2, *J1;
} EE;

static double ee_G(const EE* e, int n, const double* f) {
    const double* vr = e->v->vr;
    double f00 = (f[0] - f[1] * (vr[0] * vr[0]) / (vr[1] * vr[1])) / (1.0 - (vr[0] * vr[0]) / (vr[1] * vr[1]));
    double i2s = f00 * pow(vr[n], 3) / 3.0 + (f[1] - f00) * pow(vr[n], 5) / (vr[1] * vr[1]) * 0.2;
    double i4s = f00 * pow(vr[n], 5) * 0.2 + (f[1] - f00) * pow(vr[n], 7) / (vr[1] * vr[1] * 7.0);
    return f[n] * i4s + (pow(vr[n], 3) * f[n] - 3.0 * i2s) * e->J1[n];
}

static void ee_slope(EE* e, const double* f, double* fh) {
    const VGrid* v = e->v;
    const int n = v->n;
    double *I4 = e->I4, *I2 = e->I2, *J1 = e->J1;
    I4[0] = 0;
    for (int k = 1; k < n; ++k) { I4[k] = v->U4[k] * f[k] + v->U4m1[k] * f[k - 1]; I4[k] += I4[k - 1]; }
    I2[0] = 0;
    for (int k = 1; k < n; ++k) { I2[k] = v->U2[k] * f[k] + v->U2m1[k] * f[k - 1]; I2[k] += I2[k - 1]; }
    J1[n - 1] = 0;
    for (int k = n - 2; k > -1; --k) { J1[k] = v->U1[k + 1] * f[k + 1] + v->U1m1[k + 1] * f[k]; J1[k] += J1[k + 1]; }
    double lnee = log_ee(e->d, 4.0 * M_PI * I2[n - 1], 4.0 * M_PI * I4[n - 1]);
    /* flux G_n = f_n (I4 + v^3 J1) - 3 J1 I2 */
    for (int k = 0; k < n; ++k) {
        I2[k] *= J1[k];
        I2[k] *= -3.0;
        I4[k] += v->U3[k] * J1[k];
        I4[k] *= f[k];
        I4[k] += I2[k];
    }
    /* parabolic f near v=0 for the first NB cells */
    for (int k = 0; k < e->d->NB_algorithms && k < n; ++k) I4[k] = ee_G(e, k, f);
    /* flux differences */
    fh[0] = (-1.0) * I4[0];
    for (int k = 0; k < n - 1; ++k) I4[k] -= I4[k + 1];
    fh[0] *= 2.0 / (v->vr[0] * v->vr[0]);
    for (int k = 0; k < n - 1; ++k) I4[k] *= v->Pn[k];
    fh[0] -= I4[0];
    for (int k = 0; k < n - 1; ++k) I4[k] -= I4[k + 1];
    fh[0] *= v->Qn[0];
    for (int k = 0; k < n - 1; ++k) fh[k + 1] = v->Qn[k + 1] * I4[k];
    for (int k = 0; k < n; ++k) fh[k] *= e->c_kpre * lnee;
}

static void collide_ee(const Grid* g, const VGrid* v, cplx* Y, double hstep, int nsub) {
    const int n = g->np;
    EE e;
    e.d = g->d; e.v = v;
    double kp = sqrt(4.0 * M_PI * g->d->density_np * RE_CLASSICAL);
    e.c_kpre = 4.0 * M_PI / 3.0 * RE_CLASSICAL * kp;
    double* buf = (double*)calloc((size_t)8 * n, sizeof(double));
    e.I4 = buf; e.I2 = buf + n; e.J1 = buf + 2 * n;
    double *f = buf + 3 * n, *f0 = buf + 4 * n, *f1 = buf + 5 * n, *fh = buf + 6 * n;
    cplx* f00 = Y + IND(g, 0, 0) * g->hsize;
    for (long c = 0; c < g->cells; ++c) {
        for (int p = 0; p < n; ++p) f[p] = creal(f00[c * n + p]);
        for (int s = 0; s < nsub; ++s) {
            const double h = hstep;
            for (int p = 0; p < n; ++p) { f0[p] = f[p]; f1[p] = f[p]; }
            ee_slope(&e, f1, fh);
            for (int p = 0; p < n; ++p) { fh[p] *= 0.5 * h; f1[p] += fh[p]; fh[p] *= 1.0 / 3.0; f[p] += fh[p]; }
            ee_slope(&e, f1, fh);
            for (int p = 0; p < n; ++p) { f1[p] = f0[p]; fh[p] *= 0.5 * h; f1[p] += fh[p]; fh[p] *= 2.0 / 3.0; f[p] += fh[p]; }
            ee_slope(&e, f1, fh);
            for (int p = 0; p < n; ++p) { fh[p] *= h; f0[p] += fh[p]; fh[p] *= 1.0 / 3.0; f[p] += fh[p]; }
            ee_slope(&e, f0, fh);
            for (int p = 0; p < n; ++p) { fh[p] *= h / 6.0; f[p] += fh[p]; }
        }
        for (int p = 0; p < n; ++p) f00[c * n + p] = f[p];   /* imaginary part -> 0 */
    }
    free(buf);
}

/* Opt-in backward-Euler e-e step (not a reference scheme; the checker of
 * OSHUN_FLAG_IMPLICIT_EE).  The explicit operator of ee_slope is
 *   C(f)_k = c_kpre lnee Qn_k (D_{k-1} - D_k),  D_k = P_k (G_k - G_{k+1}),
 *   G_j = A_j f_j - B_j  (A = I4 + v^3 J1, B = 3 I2 J1; the low-v fit's
 *   i4s, i2s for j < NB), row 0: Qn_0 (-(2/v_0^2) G_0 - D_0), D_{n-1} = G_{n-1}.
 * One step g - D C(g) = f over the whole interval D is solved by Picard
 * sweeps, each a tridiagonal solve with the coefficients from the previous
 * iterate x (the first from f): on each face the B difference becomes a drag
 * on g, B_{k+1} - B_k = gam_k ((1 - w) g_k + w g_{k+1}) with
 * gam_k = (B_{k+1} - B_k) / ((1 - w) x_k + w x_{k+1}), w = 1/2, or 0 / 1
 * (upwind) where 1/2 would give the face a coefficient of the wrong sign;
 * likewise B_0 = (B_0 / x_0) g_0.  So every sweep's matrix is an M-matrix
 * (the step keeps f positive for any D) and at convergence (g = x) the
 * operator is the explicit one exactly: the step converges to the explicit
 * scheme as D -> 0 and moves number and energy as it does. */
static int g_ee_sweeps = 0;
void oo_set_ee_implicit(int sweeps) { g_ee_sweeps = sweeps > 0 ? sweeps : 0; }

/* face k (between points k and k+1): D_k = al g_k + be g_{k+1} + cs; the
 * B difference stays explicit (cs) where the iterate is not positive there */
static void ee_face(double Ak, double Ak1, double Bk, double Bk1, double xk, double xk1, double P,
                    double* al, double* be, double* cs) {
    const double dB = Bk1 - Bk;
    const double h = 0.5 * (xk + xk1);
    *cs = 0.0;
    if (!(h > 0.0)) {
        *al = P * Ak; *be = -P * Ak1; *cs = P * dB;
        return;
    }
    double w = 0.5;
    double gam = dB / h;
    if (Ak + 0.5 * gam < 0.0) w = 1.0;          /* gam < 0: all of it on g_{k+1} */
    else if (0.5 * gam > Ak1) w = 0.0;          /* gam > 0: all of it on g_k */
    if (w != 0.5) {
        const double hw = (1.0 - w) * xk + w * xk1;
        if (!(hw > 0.0)) { *al = P * Ak; *be = -P * Ak1; *cs = P * dB; return; }
        gam = dB / hw;
    }
    *al = P * (Ak + gam * (1.0 - w));
    *be = P * (gam * w - Ak1);
}

static void collide_ee_be(const Grid* g, const VGrid* v, cplx* Y, double D, int sweeps) {
    const int n = g->np;
    const double* vr = v->vr;
    const double v0s = vr[0] * vr[0], v1s = vr[1] * vr[1];
    double kp = sqrt(4.0 * M_PI * g->d->density_np * RE_CLASSICAL);
    const double c_kpre = 4.0 * M_PI / 3.0 * RE_CLASSICAL * kp;
    double* buf = (double*)calloc((size_t)13 * n, sizeof(double));
    double *I4 = buf, *I2 = buf + n, *J1 = buf + 2 * n, *f = buf + 3 * n, *x = buf + 4 * n;
    double *A = buf + 5 * n, *B = buf + 6 * n, *al = buf + 7 * n, *be = buf + 8 * n;
    double *tb = buf + 9 * n, *r = buf + 10 * n, *cp = buf + 11 * n, *cs = buf + 12 * n;
    cplx* f00 = Y + IND(g, 0, 0) * g->hsize;
    for (long c = 0; c < g->cells; ++c) {
        for (int p = 0; p < n; ++p) { f[p] = creal(f00[c * n + p]); x[p] = f[p]; }
        for (int sw = 0; sw < sweeps; ++sw) {
            I4[0] = 0; I2[0] = 0; J1[n - 1] = 0;
            for (int k = 1; k < n; ++k) I4[k] = I4[k - 1] + (v->U4[k] * x[k] + v->U4m1[k] * x[k - 1]);
            for (int k = 1; k < n; ++k) I2[k] = I2[k - 1] + (v->U2[k] * x[k] + v->U2m1[k] * x[k - 1]);
            for (int k = n - 2; k >= 0; --k) J1[k] = J1[k + 1] + (v->U1[k + 1] * x[k + 1] + v->U1m1[k + 1] * x[k]);
            const double lnee = log_ee(g->d, 4.0 * M_PI * I2[n - 1], 4.0 * M_PI * I4[n - 1]);
            const double dn = D * c_kpre * lnee;
            const double fz = (x[0] - x[1] * v0s / v1s) / (1.0 - v0s / v1s);
            for (int k = 0; k < n; ++k) {
                double i4 = I4[k], i2 = I2[k];
                const double v3 = pow(vr[k], 3);
                if (k < g->d->NB_algorithms) {
                    i2 = fz * v3 / 3.0 + (x[1] - fz) * pow(vr[k], 5) / v1s * 0.2;
                    i4 = fz * pow(vr[k], 5) * 0.2 + (x[1] - fz) * pow(vr[k], 7) / (v1s * 7.0);
                }
                A[k] = i4 + v3 * J1[k];
                B[k] = 3.0 * i2 * J1[k];
            }
            for (int k = 0; k < n - 1; ++k)
                ee_face(A[k], A[k + 1], B[k], B[k + 1], x[k], x[k + 1], v->Pn[k], al + k, be + k, cs + k);
            /* rows of M = I - dn W': sub -dn Qn al_{k-1}, diagonal, super dn Qn be_k
             * (as in Thomas below); the explicit parts go to the right-hand side */
            const int imp0 = x[0] > 0.0;
            const double a0 = imp0 ? A[0] - B[0] / x[0] : A[0];
            const double b0 = imp0 ? 0.0 : B[0];
            for (int k = 0; k < n; ++k) {
                const double q = v->Qn[k];
                double d0, c0;
                if (k == 0) { d0 = -q * ((2.0 / v0s) * a0 + al[0]); c0 = q * ((2.0 / v0s) * b0 - cs[0]); }
                else if (k < n - 1) { d0 = q * (be[k - 1] - al[k]); c0 = q * (cs[k - 1] - cs[k]); }
                else { d0 = q * (be[k - 1] - A[k]); c0 = q * cs[k - 1]; }
                tb[k] = 1.0 - dn * d0;
                r[k] = f[k] + dn * c0;
            }
            /* Thomas: sub_k = -dn Qn_k al_{k-1}, super_k = dn Qn_k be_k */
            {
                double sup = dn * v->Qn[0] * be[0];
                cp[0] = sup / tb[0];
                x[0] = r[0] / tb[0];
                for (int k = 1; k < n; ++k) {
                    const double sub = -dn * v->Qn[k] * al[k - 1];
                    sup = k < n - 1 ? dn * v->Qn[k] * be[k] : 0.0;
                    const double id = 1.0 / (tb[k] - sub * cp[k - 1]);
                    cp[k] = sup * id;
                    x[k] = (r[k] - sub * x[k - 1]) * id;
                }
                for (int k = n - 2; k >= 0; --k) x[k] -= cp[k] * x[k + 1];
            }
        }
        for (int p = 0; p < n; ++p) f00[c * n + p] = x[p];
    }
    free(buf);
}

/* ------------------------------------------------------------------------ */
/* implicit f_lm: Implicit_FLM_step (def-FokkerPlanck.cpp:757-1035)          */
/* ------------------------------------------------------------------------ */

typedef struct {
    const oo_deck* d;
    const VGrid* v;
    double kpre, Dt, lnee, zlnei;
    double *I2, *I0, *J1m, *TriI1, *TriI2, *Scat, *df0, *ddf0;
    double *tri_a, *tri_b, *tri_c;   /* Alpha_Tri: sub, diagonal, super */
} FLM;

static void flm_reset(FLM* s, const double* f, double Dt) {
    const VGrid* v = s->v;
    const double* vr = v->vr;
    const int n = v->n;
    s->Dt = Dt;
    double *I2 = s->I2, *I0 = s->I0, *J1m = s->J1m;
    I2[0] = 0;
    for (int k = 1; k < n; ++k) { I2[k] = v->U4[k] * f[k] + v->U4m1[k] * f[k - 1]; I2[k] += I2[k - 1]; }
    for (int k = 0; k < n; ++k) I2[k] *= 4.0 * M_PI;
    double I2_temperature = I2[n - 1];
    for (int k = 0; k < n; ++k) I2[k] /= vr[k] * vr[k];
    I0[0] = 0;
    for (int k = 1; k < n; ++k) { I0[k] = v->U2[k] * f[k] + v->U2m1[k] * f[k - 1]; I0[k] += I0[k - 1]; }
    for (int k = 0; k < n; ++k) I0[k] *= 4.0 * M_PI;
    double I0_density = I0[n - 1];
    J1m[n - 1] = 0;
    for (int k = n - 2; k > -1; --k) { J1m[k] = v->U1[k + 1] * f[k + 1] + v->U1m1[k + 1] * f[k]; J1m[k] += J1m[k + 1]; }
    for (int k = 0; k < n; ++k) J1m[k] *= 4.0 * M_PI * vr[k];

    s->lnee = log_ee(s->d, I0_density, I2_temperature);
    s->zlnei = zlog_ei(s->d, I0_density, I2_temperature);

    for (int i = 0; i < n; ++i) {
        s->TriI1[i] = I0[i] + (2.0 * J1m[i] - I2[i]) / 3.0;
        s->TriI2[i] = (I2[i] + J1m[i]) / 3.0;
    }
    for (int i = 0; i < n; ++i) s->Scat[i] = s->TriI1[i] * s->lnee;
    s->Scat[0] = 0.0;
    for (int i = 0; i < n; ++i) {
        s->Scat[i] += s->zlnei * I0_density;
        s->Scat[i] /= pow(vr[i], 3);
        s->Scat[i] *= s->kpre * Dt;
    }
    const double scale = (-1.0) * s->lnee * s->kpre * Dt;
    for (int i = 0; i < n; ++i) { s->tri_a[i] = 0; s->tri_b[i] = 0; s->tri_c[i] = 0; }
    s->tri_b[0] = 8.0 * M_PI * f[0] * scale;
    for (int i = 1; i < n - 1; ++i) {
        double IvDnDm1 = 1.0 / (vr[i] * 0.5 * (vr[i + 1] - vr[i - 1]) * (vr[i] - vr[i - 1]));
        double IvDnDp1 = 1.0 / (vr[i] * 0.5 * (vr[i + 1] - vr[i - 1]) * (vr[i + 1] - vr[i]));
        double Ivsq2Dn = 1.0 / (vr[i] * vr[i] * (vr[i + 1] - vr[i - 1]));
        s->tri_b[i] = (8.0 * M_PI * f[i] - s->TriI2[i] * (IvDnDm1 + IvDnDp1)) * scale;
        s->tri_a[i] = (s->TriI2[i] * IvDnDm1 - s->TriI1[i] * Ivsq2Dn) * scale;
        s->tri_c[i] = (s->TriI2[i] * IvDnDp1 + s->TriI1[i] * Ivsq2Dn) * scale;
    }
    /* derivatives of f00 */
    double *df0 = s->df0, *ddf0 = s->ddf0;
    for (int k = 0; k < n; ++k) { df0[k] = 0; ddf0[k] = 0; }
    for (int k = 1; k < n - 1; ++k) { df0[k] = f[k + 1] - f[k - 1]; df0[k] /= vr[k + 1] - vr[k - 1]; }
    for (int k = 1; k < n; ++k) { ddf0[k] = f[k - 1] - f[k]; ddf0[k] /= vr[k] - vr[k - 1]; }
    for (int k = 1; k < n - 1; ++k) { ddf0[k] -= ddf0[k + 1]; ddf0[k] /= 0.5 * (vr[k + 1] - vr[k - 1]); }
    double f00 = (f[0] - ((vr[0] * vr[0]) / (vr[1] * vr[1])) * f[1]) / (1.0 - (vr[0] * vr[0]) / (vr[1] * vr[1]));
    ddf0[0] = 2.0 * (f[1] - f00) / (vr[1] * vr[1]);
    df0[0] = ddf0[0] * vr[0];
    for (int k = 0; k < n - 1; ++k) { df0[k] /= vr[k] * vr[k]; ddf0[k] /= 2.0 * vr[k]; }
}

/* Thomas_Tridiagonal / TridiagonalSolve (def-Nmethods.cpp:142-207) */
static void thomas(int n, const double* a_in, const double* b, const double* c_in, const cplx* d_in, cplx* x) {
    double* c = (double*)malloc(sizeof(double) * n);
    cplx* d = (cplx*)malloc(sizeof(cplx) * n);
    for (int i = 0; i < n; ++i) { c[i] = c_in[i]; d[i] = d_in[i]; }
    c[0] /= b[0];
    d[0] /= b[0];
    for (int i = 1; i < n; ++i) {
        double id = 1.0 / (b[i] - c[i - 1] * a_in[i]);
        c[i] *= id;
        d[i] -= d[i - 1] * a_in[i];
        d[i] *= id;
    }
    x[n - 1] = d[n - 1];
    for (int i = n - 2; i > -1; --i) { x[i] = d[i]; x[i] -= c[i] * x[i + 1]; }
    free(c); free(d);
}

/* Gauss_Seidel (def-Nmethods.cpp:44-136): returns 0 when the diagonal
 * dominance test fails (x untouched) */
static int gauss_seidel(int n, const double* A, const cplx* b, cplx* xk) {
    const double tol = 1.0e-1;
    const int MAXiter = 5;
    for (int i = 0; i < n; ++i) {
        double row = 0.0;
        for (int j = 0; j < n; ++j) row += A[(long)i * n + j];
        if (!(row < 2.0 * A[(long)i * n + i])) return 0;
    }
    double* inv = (double*)malloc(sizeof(double) * n);
    cplx* xold = (cplx*)malloc(sizeof(cplx) * n);
    for (int i = 0; i < n; ++i) inv[i] = 1.0 / A[(long)i * n + i];
    int iteration = 0, conv = 0;
    while ((iteration++ < MAXiter) && (conv < n)) {
        for (int i = 0; i < n; ++i) xold[i] = xk[i];
        for (int i = 0; i < n; ++i) {
            cplx sigma = 0.0;
            for (int j = 0; j < i; ++j) sigma += A[(long)i * n + j] * xk[j];
            for (int j = i + 1; j < n; ++j) sigma += A[(long)i * n + j] * xk[j];
            xk[i] = inv[i] * (b[i] - sigma);
        }
        for (int i = 0; i < n; ++i) xold[i] -= xk[i];
        conv = 0;
        while (conv < n && cabs(xold[conv]) < tol * cabs(xk[conv] + 20.0 * DBL_MIN)) ++conv;
    }
    free(inv); free(xold);
    return 1;
}

/* one implicit solve (I - Dt C_l) f_new = f for harmonic order el */
static void flm_advance(FLM* s, cplx* fin, int el, double* A, cplx* fout) {
    const VGrid* v = s->v;
    const double* vr = v->vr;
    const int n = v->n;
    const double scale = (-1.0) * s->lnee * s->kpre * s->Dt;
    const double ll1 = el * (-0.5 * (el + 1.0));
    for (int i = 0; i < n; ++i) fout[i] = fin[i];
    if (s->d->if_tridiagonal) {
        double *a = (double*)malloc(sizeof(double) * n), *b = (double*)malloc(sizeof(double) * n),
               *c = (double*)malloc(sizeof(double) * n);
        for (int i = 0; i < n; ++i) { a[i] = s->tri_a[i]; b[i] = s->tri_b[i]; c[i] = s->tri_c[i]; }
        if (el > 1) b[0] = 0.0;
        for (int i = 0; i < n; ++i) b[i] += 1.0 - ll1 * s->Scat[i];
        a[0] = 0.0;
        c[n - 1] = 0.0;
        thomas(n, a, b, c, fin, fout);
        free(a); free(b); free(c);
    } else {
        for (long k = 0; k < (long)n * n; ++k) A[k] = 0.0;
        A[0] = s->tri_b[0];
        for (int i = 1; i < n - 1; ++i) {
            A[(long)i * n + i] = s->tri_b[i];
            A[(long)i * n + i - 1] = s->tri_a[i];
            A[(long)i * n + i + 1] = s->tri_c[i];
        }
        if (el > 1) A[0] = 0.0;
        const double LL = el;
        const double A1 = (LL + 1.0) * (LL + 2.0) / ((2.0 * LL + 1.0) * (2.0 * LL + 3.0));
        const double A2 = (-1.0) * (LL - 1.0) * LL / ((2.0 * LL + 1.0) * (2.0 * LL - 1.0));
        const double B1 = (-1.0) * (0.5 * LL * (LL + 1.0) + (LL + 1.0)) / ((2.0 * LL + 1.0) * (2.0 * LL + 3.0));
        const double B2 = ((-0.5) * LL * (LL + 1.0) + (LL + 2.0)) / ((2.0 * LL + 1.0) * (2.0 * LL + 3.0));
        const double B3 = (0.5 * LL * (LL + 1.0) + (LL - 1.0)) / ((2.0 * LL + 1.0) * (2.0 * LL - 1.0));
        const double B4 = (0.5 * LL * (LL + 1.0) - LL) / ((2.0 * LL + 1.0) * (2.0 * LL - 1.0));
        for (int i = 0; i < n - 1; ++i) {
            double t1 = A1 * s->ddf0[i] + B1 * s->df0[i]; t1 *= scale;
            double t2 = A1 * s->ddf0[i] + B2 * s->df0[i]; t2 *= scale;
            double t3 = A2 * s->ddf0[i] + B3 * s->df0[i]; t3 *= scale;
            double t4 = A2 * s->ddf0[i] + B4 * s->df0[i]; t4 *= scale;
            double* row = A + (long)i * n;
            row[0] += t1 * (2.0 * M_PI * pow(vr[0] / vr[i], el + 2) * vr[0] * vr[0] * (vr[1] - vr[0]));
            row[0] += t3 * (2.0 * M_PI * pow(vr[0] / vr[i], el) * vr[0] * vr[0] * (vr[1] - vr[0]));
            for (int j = 1; j < i; ++j) {
                row[j] += t1 * (2.0 * M_PI * pow(vr[j] / vr[i], el + 2) * vr[j] * vr[j] * (vr[j + 1] - vr[j - 1]));
                row[j] += t3 * (2.0 * M_PI * pow(vr[j] / vr[i], el) * vr[j] * vr[j] * (vr[j + 1] - vr[j - 1]));
            }
            /* the reference reads vr[i-1] at i = 0, one element before the
             * array (def-FokkerPlanck.cpp:989-990); with glibc's allocator
             * that word is the chunk header, a denormal of order 1e-320,
             * so it is taken as 0 here */
            const double vlow = i > 0 ? vr[i - 1] : 0.0;
            row[i] += t1 * (2.0 * M_PI * vr[i] * vr[i] * (vr[i] - vlow));
            row[i] += t3 * (2.0 * M_PI * vr[i] * vr[i] * (vr[i] - vlow));
            row[i] += t2 * (2.0 * M_PI * vr[i] * vr[i] * (vr[i + 1] - vr[i]));
            row[i] += t4 * (2.0 * M_PI * vr[i] * vr[i] * (vr[i + 1] - vr[i]));
            for (int j = i + 1; j < n - 1; ++j) {
                row[j] += t2 * (2.0 * M_PI * pow(vr[j] / vr[i], -el - 1) * vr[j] * vr[j] * (vr[j + 1] - vr[j - 1]));
                row[j] += t4 * (2.0 * M_PI * pow(vr[j] / vr[i], -el + 1) * vr[j] * vr[j] * (vr[j + 1] - vr[j - 1]));
            }
        }
        for (int i = 0; i < n; ++i) A[(long)i * n + i] += 1.0 - ll1 * s->Scat[i];
        if (!gauss_seidel(n, A, fin, fout)) ++g_nondominant;
    }
    for (int i = 0; i < n; ++i) fin[i] = fout[i];
}

static void collide_flm(const Grid* g, const VGrid* v, cplx* Y, double Dt, int do_l1, int do_lm) {
    const int n = g->np;
    FLM s;
    memset(&s, 0, sizeof(s));
    s.d = g->d; s.v = v;
    s.kpre = RE_CLASSICAL * sqrt(4.0 * M_PI * g->d->density_np * RE_CLASSICAL);
    double* buf = (double*)calloc((size_t)12 * n, sizeof(double));
    s.I2 = buf; s.I0 = buf + n; s.J1m = buf + 2 * n; s.TriI1 = buf + 3 * n; s.TriI2 = buf + 4 * n;
    s.Scat = buf + 5 * n; s.df0 = buf + 6 * n; s.ddf0 = buf + 7 * n;
    s.tri_a = buf + 8 * n; s.tri_b = buf + 9 * n; s.tri_c = buf + 10 * n;
    double* f00 = buf + 11 * n;
    double* A = g->d->if_tridiagonal ? NULL : (double*)malloc(sizeof(double) * n * n);
    cplx* fc = (cplx*)malloc(sizeof(cplx) * n);
    cplx* fout = (cplx*)malloc(sizeof(cplx) * n);
    /* 1D loops touch m = 0 only (def-FokkerPlanck.cpp:1069-1108, 1156-1198);
     * the 2D loops m <= 1 for l = 1 and m <= min(m0, l) above
     * (def-FokkerPlanck.cpp:1112-1151, 1202-1244) */
    const int mmax = g->d->if_implicit1D ? 0 : g->m0;
    for (long c = 0; c < g->cells; ++c) {
        const cplx* h00 = Y + IND(g, 0, 0) * g->hsize + c * n;
        for (int p = 0; p < n; ++p) f00[p] = creal(h00[p]);
        flm_reset(&s, f00, Dt);
        for (int l = 1; l <= g->l0; ++l) {
            if ((l == 1 && !do_l1) || (l > 1 && !do_lm)) continue;
            for (int m = 0; m <= (l < mmax ? l : mmax); ++m) {
                cplx* h = Y + IND(g, l, m) * g->hsize + c * n;
                for (int p = 0; p < n; ++p) fc[p] = h[p];
                flm_advance(&s, fc, l, A, fout);
                for (int p = 0; p < n; ++p) h[p] = fc[p];
            }
        }
    }
    free(buf); free(A); free(fc); free(fout);
}

/* ------------------------------------------------------------------------ */
/* the main loop order (OSHUN-1/main.cpp:77-107)                             */
/* ------------------------------------------------------------------------ */

int oo_steps(const oo_deck* d, double* state, int nsteps, int mask) {
    Grid g;
    if (grid_init(&g, d)) return -1;
    VGrid v;
    vgrid_init(&v, &g);
    cplx* Y = (cplx*)state;
    g_nondominant = 0;
    double t = 0.0, t_ee = 0.0, t_eb = 0.0;
    for (int s = 0; s < nsteps; ++s) {
        t += d->dt;
        if (mask & 1) rk4(&g, Y, d->dt);
        if (mask & 2) {
            int nsub = (int)((t - t_ee) / d->small_dt) + 1;
            double hh = (t - t_ee) / (double)nsub;
            if (g_ee_sweeps > 0) collide_ee_be(&g, &v, Y, t - t_ee, g_ee_sweeps);
            else collide_ee(&g, &v, Y, hh, nsub);
            t_ee = t;
        }
        if (mask & 12) collide_flm(&g, &v, Y, t - t_eb, (mask & 4) != 0, (mask & 8) != 0);
        if (mask & 8) t_eb = t;
    }
    vgrid_free(&v);
    grid_free(&g);
    return 0;
}
