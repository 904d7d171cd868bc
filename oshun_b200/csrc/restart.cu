// Restart files in the reference's byte layout: Restart_Facility::Write and
// ::Read (OSHUN-1/def-Export.cpp:733-836), file name adj_name
// (def-Export.cpp:804-836): <prefix>_<rank, 6 digits>_<step, 3 digits>.dat.
//
// The file is the reference's Stat written raw, guard cells included: every
// harmonic in ind(l,m) order (DF order, def-State.cpp:420-427) as
// complex<double>[numy+2g][numx+2g][nump] (p fastest, matrices.h:714-716),
// then the six fields Ex..Bz as complex<double>[numy+2g][numx+2g].  g is the
// deck's RKLevel.  After every small step the reference refreshes the guards
// with the periodic image of the interior (main.cpp:107,
// Node_Communications::sameNode_periodic_X/Y, def-Parallel.cpp:1138-1158,
// 1229-1248), which is what the packer writes: x index i of the guarded grid
// holds interior cell (i - g) mod numx, and y likewise.  A 1D run (numy = 1)
// has 1 + 2g rows in the reference; its y copy moves rows through the guards
// one step at a time, so they hold earlier steps' rows there; no operator of
// a 1D run reads them, and the packer writes the current interior row into
// every one.  Reading takes the interior cells only.
//
// Host code only: packing works on host buffers in the oshun_download layout,
// and the handle entry points download or upload through the C ABI.
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "oshun_internal.h"

namespace oshun {
namespace {

constexpr int kMaxGuard = 64;

int num_harm(const oshun_cfg& c) { return ((c.m0 + 1) * (2 * c.l0 - c.m0 + 2)) / 2; }

// guarded grid of this configuration; 0 when g does not fit
struct Guarded {
    long long nxt, nyt;
};
int guarded(const oshun_cfg* cfg, int g, Guarded* out) {
    if (!cfg) { set_error("cfg is NULL"); return OSHUN_ERR_ARG; }
    const oshun_cfg& c = *cfg;
    if (c.l0 < 0 || c.m0 < 0 || c.m0 > c.l0 || c.nump < 1 || c.numx < 1 || c.numy < 1) {
        set_error("restart: bad configuration");
        return OSHUN_ERR_ARG;
    }
    if (g < 0 || g > kMaxGuard) { set_error("restart: need 0 <= guard_cells <= 64"); return OSHUN_ERR_ARG; }
    // the periodic image of the guard copy needs g interior cells (1D: y has one row)
    if (c.numx < g || (c.numy > 1 && c.numy < g)) {
        set_error("restart: the periodic guard image needs numx (and numy > 1) >= guard_cells");
        return OSHUN_ERR_UNSUPPORTED;
    }
    out->nxt = c.numx + 2LL * g;
    out->nyt = c.numy + 2LL * g;
    return OSHUN_OK;
}

long long wrap(long long i, long long n) { return ((i % n) + n) % n; }

std::string file_name(const char* prefix, int rank, int re_step) {
    char buf[64];
    std::snprintf(buf, sizeof(buf), "_%06d_%03d.dat", rank, re_step);
    return std::string(prefix ? prefix : "RESTART/re") + buf;
}

}  // namespace
}  // namespace oshun

using namespace oshun;

extern "C" {

long long oshun_restart_bytes(const oshun_cfg* cfg, int guard_cells) {
    Guarded G;
    if (guarded(cfg, guard_cells, &G) != OSHUN_OK) return -1;
    const long long cells = G.nxt * G.nyt;
    return 16LL * ((long long)num_harm(*cfg) * cfg->nump * cells + 6 * cells);
}

int oshun_restart_pack(const oshun_cfg* cfg, int guard_cells, const double* harmonics, const double* fields,
                       double* image) {
    Guarded G;
    const int rc = guarded(cfg, guard_cells, &G);
    if (rc) return rc;
    if (!harmonics || !fields || !image) { set_error("NULL argument"); return OSHUN_ERR_ARG; }
    const oshun_cfg& c = *cfg;
    const long long np = c.nump, nx = c.numx, ny = c.numy, g = guard_cells;
    const int nh = num_harm(c);
    double* o = image;
    for (int h = 0; h < nh; ++h)
        for (long long yt = 0; yt < G.nyt; ++yt) {
            const long long y = ny > 1 ? wrap(yt - g, ny) : 0;
            for (long long xt = 0; xt < G.nxt; ++xt) {
                const long long x = wrap(xt - g, nx);
                std::memcpy(o, harmonics + 2 * (((long long)h * ny + y) * nx + x) * np, sizeof(double) * 2 * np);
                o += 2 * np;
            }
        }
    for (int f = 0; f < 6; ++f)
        for (long long yt = 0; yt < G.nyt; ++yt) {
            const long long y = ny > 1 ? wrap(yt - g, ny) : 0;
            for (long long xt = 0; xt < G.nxt; ++xt) {
                const long long x = wrap(xt - g, nx);
                o[0] = fields[2 * ((f * ny + y) * nx + x)];
                o[1] = fields[2 * ((f * ny + y) * nx + x) + 1];
                o += 2;
            }
        }
    return OSHUN_OK;
}

int oshun_restart_unpack(const oshun_cfg* cfg, int guard_cells, const double* image, double* harmonics,
                         double* fields) {
    Guarded G;
    const int rc = guarded(cfg, guard_cells, &G);
    if (rc) return rc;
    if (!harmonics || !fields || !image) { set_error("NULL argument"); return OSHUN_ERR_ARG; }
    const oshun_cfg& c = *cfg;
    const long long np = c.nump, nx = c.numx, ny = c.numy, g = guard_cells;
    const int nh = num_harm(c);
    const long long hstride = G.nyt * G.nxt * np * 2;
    for (int h = 0; h < nh; ++h)
        for (long long y = 0; y < ny; ++y)
            for (long long x = 0; x < nx; ++x)
                std::memcpy(harmonics + 2 * (((long long)h * ny + y) * nx + x) * np,
                            image + h * hstride + 2 * ((y + g) * G.nxt + (x + g)) * np, sizeof(double) * 2 * np);
    const double* fimg = image + nh * hstride;
    for (int f = 0; f < 6; ++f)
        for (long long y = 0; y < ny; ++y)
            for (long long x = 0; x < nx; ++x) {
                const double* s = fimg + 2 * ((f * G.nyt + y + g) * G.nxt + (x + g));
                fields[2 * ((f * ny + y) * nx + x)] = s[0];
                fields[2 * ((f * ny + y) * nx + x) + 1] = s[1];
            }
    return OSHUN_OK;
}

int oshun_restart_write(oshun_handle h, const char* prefix, int rank, int re_step, int guard_cells) {
    if (!h) { set_error("NULL handle"); return OSHUN_ERR_ARG; }
    if (rank < 0 || re_step < 0) { set_error("restart: need rank, re_step >= 0"); return OSHUN_ERR_ARG; }
    oshun_cfg c;
    int rc = oshun_get_config(h, &c);
    if (rc) return rc;
    const long long bytes = oshun_restart_bytes(&c, guard_cells);
    if (bytes < 0) return OSHUN_ERR_ARG;
    const long long cells = (long long)c.numx * c.numy;
    std::vector<double> f(2 * (size_t)num_harm(c) * c.nump * cells), fl(2 * 6 * (size_t)cells);
    if ((rc = oshun_download(h, f.data(), fl.data()))) return rc;
    std::vector<double> img((size_t)(bytes / 8));
    if ((rc = oshun_restart_pack(&c, guard_cells, f.data(), fl.data(), img.data()))) return rc;
    const std::string name = file_name(prefix, rank, re_step);
    FILE* fp = std::fopen(name.c_str(), "wb");
    if (!fp) { set_error("restart: cannot open " + name + " for writing"); return OSHUN_ERR_ARG; }
    const bool ok = std::fwrite(img.data(), 1, (size_t)bytes, fp) == (size_t)bytes;
    if (std::fclose(fp) != 0 || !ok) { set_error("restart: short write to " + name); return OSHUN_ERR_ARG; }
    return OSHUN_OK;
}

int oshun_restart_read(oshun_handle h, const char* prefix, int rank, int re_step, int guard_cells) {
    if (!h) { set_error("NULL handle"); return OSHUN_ERR_ARG; }
    if (rank < 0 || re_step < 0) { set_error("restart: need rank, re_step >= 0"); return OSHUN_ERR_ARG; }
    oshun_cfg c;
    int rc = oshun_get_config(h, &c);
    if (rc) return rc;
    const long long bytes = oshun_restart_bytes(&c, guard_cells);
    if (bytes < 0) return OSHUN_ERR_ARG;
    const std::string name = file_name(prefix, rank, re_step);
    FILE* fp = std::fopen(name.c_str(), "rb");
    if (!fp) { set_error("restart: cannot open " + name); return OSHUN_ERR_ARG; }
    std::vector<double> img((size_t)(bytes / 8));
    const bool ok = std::fread(img.data(), 1, (size_t)bytes, fp) == (size_t)bytes;
    const bool at_end = ok && std::fgetc(fp) == EOF;
    std::fclose(fp);
    if (!ok || !at_end) {
        set_error("restart: " + name + " does not hold " + std::to_string(bytes) +
                  " bytes (configuration or guard cells differ)");
        return OSHUN_ERR_ARG;
    }
    const long long cells = (long long)c.numx * c.numy;
    std::vector<double> f(2 * (size_t)num_harm(c) * c.nump * cells), fl(2 * 6 * (size_t)cells);
    if ((rc = oshun_restart_unpack(&c, guard_cells, img.data(), f.data(), fl.data()))) return rc;
    return oshun_upload(h, f.data(), fl.data());
}

}  // extern "C"
