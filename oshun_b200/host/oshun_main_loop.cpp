// The reference's small-step loop (OSHUN-1/main.cpp:77-107) driven through
// the C++ host layer (oshun.hpp) and the C ABI, on a case file.
//
// usage: oshun_main_loop IN.case OUT.case NSTEPS [MASK]
//   MASK bits: 1 rk.advance_p1, 2 ee.loop, 4 eb.advance_1, 8 eb.advance_lm
//   (default 15).  The case format is the one of oracle/ref_harness:
//   "OSHC", int32 version 1, int32 l0 m0 nump numx numy NB_algorithms
//   if_tridiagonal if_implicit1D, float64 pmin pmax xmin xmax ymin ymax dt
//   small_dt density_np Zeta, complex128 harmonics then 6 complex128 fields.
#include <complex>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "oshun.hpp"

namespace {

bool read_case(const char* path, oshun_cfg& cfg, std::vector<std::complex<double>>& f,
               std::vector<std::complex<double>>& fields) {
    FILE* fp = std::fopen(path, "rb");
    if (!fp) return false;
    char magic[4];
    int version = 0, iv[8];
    double dv[10];
    bool ok = std::fread(magic, 1, 4, fp) == 4 && std::memcmp(magic, "OSHC", 4) == 0 &&
              std::fread(&version, 4, 1, fp) == 1 && version == 1 && std::fread(iv, 4, 8, fp) == 8 &&
              std::fread(dv, 8, 10, fp) == 10;
    if (ok) {
        std::memset(&cfg, 0, sizeof(cfg));
        cfg.l0 = iv[0]; cfg.m0 = iv[1]; cfg.nump = iv[2]; cfg.numx = iv[3]; cfg.numy = iv[4];
        cfg.NB_algorithms = iv[5]; cfg.if_tridiagonal = iv[6]; cfg.if_implicit1D = iv[7];
        cfg.pmin = dv[0]; cfg.pmax = dv[1]; cfg.xmin = dv[2]; cfg.xmax = dv[3]; cfg.ymin = dv[4];
        cfg.ymax = dv[5]; cfg.dt = dv[6]; cfg.small_dt = dv[7]; cfg.density_np = dv[8]; cfg.Zeta = dv[9];
        cfg.t0 = 0.0; cfg.precision = OSHUN_FP64; cfg.flags = 0;
        const std::size_t nf = oshun_b200::num_harmonics(cfg.l0, cfg.m0) * cfg.numy * cfg.numx * cfg.nump;
        f.resize(nf);
        fields.resize(6u * cfg.numy * cfg.numx);
        ok = std::fread(f.data(), 16, nf, fp) == nf && std::fread(fields.data(), 16, fields.size(), fp) == fields.size();
    }
    std::fclose(fp);
    return ok;
}

bool write_case(const char* path, const char* like, const std::vector<std::complex<double>>& f,
                const std::vector<std::complex<double>>& fields) {
    // header copied from the input case
    FILE* in = std::fopen(like, "rb");
    if (!in) return false;
    unsigned char head[120];
    const bool okh = std::fread(head, 1, sizeof(head), in) == sizeof(head);
    std::fclose(in);
    if (!okh) return false;
    FILE* fp = std::fopen(path, "wb");
    if (!fp) return false;
    const bool ok = std::fwrite(head, 1, sizeof(head), fp) == sizeof(head) &&
                    std::fwrite(f.data(), 16, f.size(), fp) == f.size() &&
                    std::fwrite(fields.data(), 16, fields.size(), fp) == fields.size();
    std::fclose(fp);
    return ok;
}

}  // namespace

int main(int argc, char** argv) {
    if (argc < 4) {
        std::fprintf(stderr, "usage: oshun_main_loop IN.case OUT.case NSTEPS [MASK]\n");
        return 2;
    }
    oshun_cfg cfg;
    std::vector<std::complex<double>> f, fields;
    if (!read_case(argv[1], cfg, f, fields)) {
        std::fprintf(stderr, "cannot read %s\n", argv[1]);
        return 2;
    }
    const int nsteps = std::atoi(argv[3]);
    const int mask = argc > 4 ? std::atoi(argv[4]) : 15;
    try {
        oshun_b200::State Y(cfg);
        Y.upload(f, fields);
        // dt_out = h: one small step per output step, as the checker decks use
        oshun_b200::Runge_Kutta_4 rk(Y, 0, cfg.dt);
        oshun_b200::Explicit_EC_FP ee(Y);
        oshun_b200::Euler_Backward eb(Y);
        double tnew = 0.0;
        for (int s = 0; s < nsteps; ++s) {
            if (mask & 1) {
                rk.advance_p1();
                tnew = rk.time();
            } else {
                tnew += cfg.dt;
            }
            if (mask & 2) ee.loop(tnew);
            rk.advance_p2();
            if (mask & 4) eb.advance_1(tnew);
            if (mask & 8) eb.advance_lm(tnew);
        }
        Y.download(f, fields);
    } catch (const oshun_b200::Error& e) {
        std::fprintf(stderr, "oshun_main_loop: %s (status %d)\n", e.what(), e.code());
        return 3;
    }
    if (!write_case(argv[2], argv[1], f, fields)) {
        std::fprintf(stderr, "cannot write %s\n", argv[2]);
        return 2;
    }
    return 0;
}
