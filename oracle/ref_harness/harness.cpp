// CPU checker driver around the reference's own hot-path code.
//
// Test infrastructure only.  Linked with the unmodified reference sources
// (OSHUN-1/def-State.cpp, def-VlasovMax.cpp, def-Actions.cpp, def-RK.cpp,
// def-FokkerPlanck.cpp, def-Nmethods.cpp) and deck.cpp into
// oracle/_ref/oshun_ref.  It replaces the reference's main_loop
// (OSHUN-1/main.cpp:40-134) with a deck read from a case file, runs the
// requested operators on a `Stat` with 4 guard cells, refreshes the periodic
// guards the way Node_Communications::sameNode_periodic_X/Y does
// (OSHUN-1/def-Parallel.cpp:1138-1158, 1229-1248) and writes the interior
// back out.
//
// usage: oshun_ref IN.case OUT.case OP [OP ...]
//   rhs              slope of Actions::Adv (def-Actions.cpp:73-94) of the input
//   step:N[:MASK]    N time steps of the main loop order (main.cpp:77-107):
//                    MASK bit 1 rk4.advance_p1, 2 ee.loop, 4 eb.advance_1,
//                    8 eb.advance_lm; default 15
//   istep:N[:MASK]   N time steps of the implicit-E main loop (main.cpp:77-107
//                    with implicit_E): MASK bit 1 Runge_Kutta_2_Imp::advance_p1,
//                    2 ee.loop, 16 Implicit_E_Field::advance (def-ImplicitE.cpp:
//                    471-676), 32 advance_p2, 4 eb.advance_1, 8 eb.advance_lm;
//                    default 63
//   time             print the wall time of the step loops to stdout
//   restart_write:R:S  Restart_Facility::Write(R, S, Y) (def-Export.cpp:768-800):
//                    RESTART/re_<R>_<S>.dat in the working directory
//   restart_read:R:S   Restart_Facility::Read(R, S, Y) (def-Export.cpp:733-766)
//   moments:S        Parallel_Output::nonrelativistic_moments(S, Y)
//                    (def-Parallel.cpp:1677-2258) with every moment output on:
//                    OUTPUT/MOM/<name>/... text files in the working directory
// The restart and moment ops also link def-Export.cpp, def-Output.cpp and
// def-Parallel.cpp (single rank, the MPI stand-in of mpi.h here).
//
// Case file (little-endian), shared with oracle/oshun_oracle.c and the tests:
//   char magic[4] = "OSHC"; int32 version = 1;
//   int32 l0, m0, nump, numx, numy, NB_algorithms, if_tridiagonal, if_implicit1D;
//   float64 pmin, pmax, xmin, xmax, ymin, ymax, dt, small_dt, density_np, Zeta;
//   complex128 harmonics[Nh][numy][numx][nump]  (index ind(l,m) of
//              def-State.cpp:420-427, interior cells only)
//   complex128 fields[6][numy][numx]            (Ex, Ey, Ez, Bx, By, Bz)
// The reference's periodic guard copy (def-Parallel.cpp:1138-1158, 1229-1248)
// is a periodic image only when a direction holds at least RKLevel = 4
// interior cells, so cases need numx >= 4 and numy >= 4; a 1D case
// (numy == 1) runs the reference with 4 identical y rows.
#include <iostream>
#include <vector>
#include <valarray>
#include <complex>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <sys/time.h>
#include <math.h>
#include <float.h>

#include "matrices.h"
#include "decl-input.h"
#include "decl-state.h"
#include "decl-vlasovmax.h"
#include "decl-actions.h"
#include "decl-RK.h"
#include "decl-nmethods.h"
#include "decl-fokkerplanck.h"
#include <fstream>
#include <sstream>
#include <mpi.h>
#include "decl-implicitE.h"
#include "decl-output.h"
#include "decl-export.h"
#include "decl-parallel.h"
#include "deck.h"

namespace {

struct CaseHead {
    int l0, m0, nump, numx, numy, NB, tri, imp1d;
    double pmin, pmax, xmin, xmax, ymin, ymax, dt, small_dt, density_np, Zeta;
};

const int NBC = 4;

int num_harmonics(int l0, int m0) { return ((m0 + 1) * (2 * l0 - m0 + 2)) / 2; }

double now_s() {
    struct timeval tv;
    gettimeofday(&tv, 0);
    return tv.tv_sec + 1e-6 * tv.tv_usec;
}

bool read_case(const char* path, CaseHead& h, std::vector<double>& data) {
    FILE* f = std::fopen(path, "rb");
    if (!f) return false;
    char magic[4];
    int version;
    bool ok = std::fread(magic, 1, 4, f) == 4 && std::memcmp(magic, "OSHC", 4) == 0 &&
              std::fread(&version, 4, 1, f) == 1 && version == 1;
    int iv[8];
    double dv[10];
    ok = ok && std::fread(iv, 4, 8, f) == 8 && std::fread(dv, 8, 10, f) == 10;
    if (ok) {
        h.l0 = iv[0]; h.m0 = iv[1]; h.nump = iv[2]; h.numx = iv[3]; h.numy = iv[4];
        h.NB = iv[5]; h.tri = iv[6]; h.imp1d = iv[7];
        h.pmin = dv[0]; h.pmax = dv[1]; h.xmin = dv[2]; h.xmax = dv[3];
        h.ymin = dv[4]; h.ymax = dv[5]; h.dt = dv[6]; h.small_dt = dv[7];
        h.density_np = dv[8]; h.Zeta = dv[9];
        size_t cells = size_t(h.numx) * h.numy;
        size_t n = 2 * (size_t(num_harmonics(h.l0, h.m0)) * h.nump * cells + 6 * cells);
        data.resize(n);
        ok = std::fread(&data[0], 8, n, f) == n;
    }
    std::fclose(f);
    return ok;
}

bool write_case(const char* path, const CaseHead& h, const std::vector<double>& data) {
    FILE* f = std::fopen(path, "wb");
    if (!f) return false;
    int version = 1;
    int iv[8] = {h.l0, h.m0, h.nump, h.numx, h.numy, h.NB, h.tri, h.imp1d};
    double dv[10] = {h.pmin, h.pmax, h.xmin, h.xmax, h.ymin, h.ymax,
                     h.dt, h.small_dt, h.density_np, h.Zeta};
    bool ok = std::fwrite("OSHC", 1, 4, f) == 4 && std::fwrite(&version, 4, 1, f) == 1 &&
              std::fwrite(iv, 4, 8, f) == 8 && std::fwrite(dv, 8, 10, f) == 10 &&
              std::fwrite(&data[0], 8, data.size(), f) == data.size();
    std::fclose(f);
    return ok;
}

// interior (case) -> guarded Stat; y rows of a 1D case are duplicated
void load_state(Stat& Y, const CaseHead& h, const std::vector<double>& d) {
    const int nh = num_harmonics(h.l0, h.m0);
    const int ny_ref = Y.SH(0).numy() - 2 * NBC;
    size_t k = 0;
    for (int i = 0; i < nh; ++i)
        for (int iy = 0; iy < h.numy; ++iy)
            for (int ix = 0; ix < h.numx; ++ix)
                for (int ip = 0; ip < h.nump; ++ip, k += 2) {
                    std::complex<double> v(d[k], d[k + 1]);
                    for (int r = iy; r < ny_ref; r += h.numy)
                        Y.SH(i)(ip, ix + NBC, r + NBC) = v;
                }
    for (int i = 0; i < 6; ++i)
        for (int iy = 0; iy < h.numy; ++iy)
            for (int ix = 0; ix < h.numx; ++ix, k += 2) {
                std::complex<double> v(d[k], d[k + 1]);
                for (int r = iy; r < ny_ref; r += h.numy)
                    Y.FLD(i)(ix + NBC, r + NBC) = v;
            }
}

void store_state(Stat& Y, const CaseHead& h, std::vector<double>& d) {
    const int nh = num_harmonics(h.l0, h.m0);
    size_t k = 0;
    for (int i = 0; i < nh; ++i)
        for (int iy = 0; iy < h.numy; ++iy)
            for (int ix = 0; ix < h.numx; ++ix)
                for (int ip = 0; ip < h.nump; ++ip, k += 2) {
                    std::complex<double> v = Y.SH(i)(ip, ix + NBC, iy + NBC);
                    d[k] = v.real(); d[k + 1] = v.imag();
                }
    for (int i = 0; i < 6; ++i)
        for (int iy = 0; iy < h.numy; ++iy)
            for (int ix = 0; ix < h.numx; ++ix, k += 2) {
                std::complex<double> v = Y.FLD(i)(ix + NBC, iy + NBC);
                d[k] = v.real(); d[k + 1] = v.imag();
            }
}

// periodic guard refresh: x first, then whole rows (guards included) in y
void refresh_guards(Stat& Y) {
    const int nh = Y.DF().dim();
    const int np = Y.SH(0).nump(), nx = Y.SH(0).numx(), ny = Y.SH(0).numy();
    const int ix_in = nx - 2 * NBC, iy_in = ny - 2 * NBC;
    for (int i = 0; i < nh; ++i) {
        SHarmonic& s = Y.SH(i);
        for (int iy = 0; iy < ny; ++iy)
            for (int g = 0; g < NBC; ++g)
                for (int ip = 0; ip < np; ++ip) {
                    s(ip, g, iy) = s(ip, g + ix_in, iy);
                    s(ip, nx - NBC + g, iy) = s(ip, NBC + g, iy);
                }
        for (int g = 0; g < NBC; ++g)
            for (int ix = 0; ix < nx; ++ix)
                for (int ip = 0; ip < np; ++ip) {
                    s(ip, ix, g) = s(ip, ix, g + iy_in);
                    s(ip, ix, ny - NBC + g) = s(ip, ix, NBC + g);
                }
    }
    for (int i = 0; i < 6; ++i) {
        Field2D& fl = Y.FLD(i);
        for (int iy = 0; iy < ny; ++iy)
            for (int g = 0; g < NBC; ++g) {
                fl(g, iy) = fl(g + ix_in, iy);
                fl(nx - NBC + g, iy) = fl(NBC + g, iy);
            }
        for (int g = 0; g < NBC; ++g)
            for (int ix = 0; ix < nx; ++ix) {
                fl(ix, g) = fl(ix, g + iy_in);
                fl(ix, ny - NBC + g) = fl(ix, NBC + g);
            }
    }
}

}  // namespace

int main(int argc, char** argv) {
    if (argc < 4) {
        std::fprintf(stderr, "usage: oshun_ref IN.case OUT.case OP [OP ...]\n");
        return 2;
    }
    CaseHead h;
    std::vector<double> data;
    if (!read_case(argv[1], h, data)) {
        std::fprintf(stderr, "oshun_ref: cannot read case %s\n", argv[1]);
        return 2;
    }
    if (h.numx < NBC || (h.numy != 1 && h.numy < NBC)) {
        std::fprintf(stderr, "oshun_ref: periodic guards need numx, numy >= %d (or numy == 1)\n", NBC);
        return 3;
    }
    if (h.l0 < 3 || h.m0 < 2 || h.m0 > h.l0) {
        // OSHUN-1's explicit operators index SH(l0>=3, m0>=2) unconditionally
        // (def-Input.cpp:73, def-VlasovMax.cpp:346-491).
        std::fprintf(stderr, "oshun_ref: the reference needs l0>=3 and 2<=m0<=l0 (got %d,%d)\n",
                     h.l0, h.m0);
        return 3;
    }

    g_deck.l0 = h.l0; g_deck.m0 = h.m0; g_deck.nump = h.nump;
    g_deck.numx_glob = h.numx;
    g_deck.numy_glob = h.numy == 1 ? NBC : h.numy;
    g_deck.xmin = h.xmin; g_deck.xmax = h.xmax;
    g_deck.ymin = h.ymin; g_deck.ymax = h.ymax;
    g_deck.pmin = h.pmin; g_deck.pmax = h.pmax;
    // num_h = int(dt_out/CLF)+1 = 1 and h = dt_out (def-RK.cpp:60-61)
    g_deck.clf_dp = 2.0 * h.dt;
    g_deck.n_outsteps = 1;
    g_deck.t_stop = h.dt;
    g_deck.small_dt = h.small_dt;
    g_deck.NB_algorithms = h.NB;
    g_deck.if_tridiagonal = h.tri;
    g_deck.if_implicit1D = h.imp1d;
    g_deck.density_np = h.density_np;
    g_deck.Zeta = h.Zeta;

    Inputdata::IN();
    Stat Y;
    Y = std::complex<double>(0.0, 0.0);
    load_state(Y, h, data);
    refresh_guards(Y);

    double elapsed = 0.0;
    bool print_time = false;
    for (int a = 3; a < argc; ++a) {
        std::string op(argv[a]);
        if (op == "time") {
            print_time = true;
        } else if (op == "rhs") {
            Stat Yh(Y);
            Actions act(Yh);
            act.Adv(Y);
            Y = Yh;
        } else if (op.compare(0, 5, "step:") == 0) {
            int nsteps = 0, mask = 15;
            if (std::sscanf(op.c_str() + 5, "%d:%d", &nsteps, &mask) < 1) {
                std::fprintf(stderr, "oshun_ref: bad op %s\n", op.c_str());
                return 2;
            }
            Runge_Kutta_4 rk(Y, 0);
            Explicit_EC_FP ee(Y, 0);
            Euler_Backward eb(Y, 0);
            double t0 = now_s();
            double tnew = 0.0;  // accumulated like Runge_Kutta_4's t += h (def-RK.cpp:142)
            for (int s = 0; s < nsteps; ++s) {
                tnew += h.dt;
                if (mask & 1) rk.advance_p1();
                if (mask & 2) ee.loop(tnew);
                if (mask & 4) eb.advance_1(tnew);
                if (mask & 8) eb.advance_lm(tnew);
                refresh_guards(Y);
            }
            elapsed += now_s() - t0;
        } else if (op.compare(0, 6, "istep:") == 0) {
            int nsteps = 0, mask = 63;
            if (std::sscanf(op.c_str() + 6, "%d:%d", &nsteps, &mask) < 1) {
                std::fprintf(stderr, "oshun_ref: bad op %s\n", op.c_str());
                return 2;
            }
            Runge_Kutta_2_Imp rk(Y, 0);
            Explicit_EC_FP ee(Y, 0);
            Euler_Backward eb(Y, 0);
            Electric_Field_Methods::Implicit_E_Field em(Y, 0);
            double t0 = now_s();
            for (int s = 0; s < nsteps; ++s) {
                if (mask & 1) rk.advance_p1();
                refresh_guards(Y);   // the single-node image of Neighbor_ImplicitE_Communications
                if (mask & 2) ee.loop(rk.time());
                if (mask & 16) em.advance(&rk, &eb);
                if (mask & 32) rk.advance_p2();
                if (mask & 4) eb.advance_1(rk.time());
                if (mask & 8) eb.advance_lm(rk.time());
                refresh_guards(Y);
            }
            elapsed += now_s() - t0;
        } else if (op.compare(0, 14, "restart_write:") == 0 || op.compare(0, 13, "restart_read:") == 0) {
            const bool wr = op[8] == 'w';
            int rank = 0, re_step = 0;
            if (std::sscanf(op.c_str() + (wr ? 14 : 13), "%d:%d", &rank, &re_step) != 2) {
                std::fprintf(stderr, "oshun_ref: bad op %s\n", op.c_str());
                return 2;
            }
            Restart_Facility re;
            if (wr) re.Write(rank, re_step, Y);
            else re.Read(rank, re_step, Y);
        } else if (op.compare(0, 8, "moments:") == 0) {
            int mstep = 0;
            if (std::sscanf(op.c_str() + 8, "%d", &mstep) != 1) {
                std::fprintf(stderr, "oshun_ref: bad op %s\n", op.c_str());
                return 2;
            }
            Parallel_Output po;
            po.nonrelativistic_moments((size_t)mstep, Y);
        } else {
            std::fprintf(stderr, "oshun_ref: unknown op %s\n", op.c_str());
            return 2;
        }
    }
    store_state(Y, h, data);
    if (!write_case(argv[2], h, data)) {
        std::fprintf(stderr, "oshun_ref: cannot write %s\n", argv[2]);
        return 2;
    }
    if (print_time) std::printf("elapsed_s=%.9f\n", elapsed);
    return 0;
}
