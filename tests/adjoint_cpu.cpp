// CPU entry points over the adjoint math of oshun_b200/csrc/adjoint_math.h,
// for the derivative tests (test_adjoint_cpu.py): the same forward and
// transpose code the CUDA adjoint kernels run, called from ctypes.
#include <vector>

#include "../oshun_b200/csrc/adjoint_math.h"

using namespace oshun::adj;

namespace {
CollTables tables(int np, int NB, const double* tab, double dens, double Z, double ckpre, double kpre) {
    CollTables T;
    T.np = np; T.NB = NB;
    T.vr = tab; T.U4 = tab + np; T.U4m1 = tab + 2 * np; T.U2 = tab + 3 * np; T.U2m1 = tab + 4 * np;
    T.U1 = tab + 5 * np; T.U1m1 = tab + 6 * np; T.U3 = tab + 7 * np; T.Qn = tab + 8 * np; T.Pn = tab + 9 * np;
    T.V5 = tab + 10 * np; T.V7 = tab + 11 * np;
    T.density_np = dens; T.Zeta = Z; T.c_kpre = ckpre; T.kpre = kpre;
    return T;
}
Grid1 grid(int np, int nx, int l0, const double* ptab, const double* coef, const double* g00) {
    Grid1 g;
    g.np = np; g.nx = nx; g.l0 = l0;
    g.invp = ptab; g.vr = ptab + np; g.wj = ptab + 2 * np;
    g.coef = reinterpret_cast<const Coef1*>(coef);
    g.g00_s = g00[0]; g.g00_inv = g00[1]; g.g00_gr = g00[2];
    return g;
}
}  // namespace

extern "C" {

void ac_collide(int np, int NB, const double* tab, double dens, double Z, double ckpre, double kpre, int l0,
                double* f00, double* fl, int ee, int eb, int nsub, double hsub, double Dt) {
    const CollTables T = tables(np, NB, tab, dens, Z, ckpre, kpre);
    std::vector<double> w(coll_ws(np, l0, nsub));
    collide_cell(T, l0, f00, fl, np, ee, eb, nsub, hsub, Dt, w.data());
}

void ac_collide_T(int np, int NB, const double* tab, double dens, double Z, double ckpre, double kpre, int l0,
                  const double* f00, const double* fl, int ee, int eb, int nsub, double hsub, double Dt,
                  double* lam00, double* laml) {
    const CollTables T = tables(np, NB, tab, dens, Z, ckpre, kpre);
    std::vector<double> w(coll_ws(np, l0, nsub));
    collide_cell_T(T, l0, f00, fl, np, ee, eb, nsub, hsub, Dt, lam00, laml, np, w.data());
}

// F of the whole state: f[l][x][p], Ex[x] -> slope_f, slope_E
void ac_rhs(int np, int nx, int l0, const double* ptab, const double* coef, const double* g00, const double* f,
            const double* Ex, double* sf, double* sE) {
    const Grid1 g = grid(np, nx, l0, ptab, coef, g00);
    std::vector<double> s(l0 + 1);
    for (int x = 0; x < nx; ++x) {
        double J = 0.0;
        for (int p = 0; p < np; ++p) {
            rhs_point(g, f, Ex, x, p, s.data());
            for (int t = 0; t <= l0; ++t) sf[((long long)t * nx + x) * np + p] = s[t];
            J += g.wj[p] * f[((long long)1 * nx + x) * np + p];
        }
        sE[x] = J;
    }
}

// F'(f, Ex)^T (cf, cE) -> (lf, lE)
void ac_vjp(int np, int nx, int l0, const double* ptab, const double* coef, const double* g00, const double* f,
            const double* Ex, const double* cf, const double* cE, double* lf, double* lE) {
    const Grid1 g = grid(np, nx, l0, ptab, coef, g00);
    for (int x = 0; x < nx; ++x) {
        double e = 0.0;
        for (int k = 0; k < np; ++k) {
            for (int s = 0; s <= l0; ++s) lf[((long long)s * nx + x) * np + k] = vjp_f(g, Ex, cf, cE, s, x, k);
            e += vjp_E_point(g, f, cf, x, k);
        }
        lE[x] = e;
    }
}

}  // extern "C"
