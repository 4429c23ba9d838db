// Host-only file surface of the reference: the .ini readers, start_*.txt
// initial conditions, S_/DM_ binary snapshots and LIE_0.bin.  No device work.
//
// Formats follow the reference's readers and writers (cited per function);
// the parsers check what they read and report KHRR_ERR_IO instead of the
// reference's exit(0) on a missing file.
#include <charconv>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "khrr.h"

namespace {

constexpr double kPi = 3.14159265358979;  // common.cuh:7 (DEG2RAD uses it)

struct File {
    FILE* f = nullptr;
    File(const char* path, const char* mode) : f(path ? std::fopen(path, mode) : nullptr) {}
    ~File() {
        if (f) std::fclose(f);
    }
    explicit operator bool() const { return f != nullptr; }
};

// One ini value line: the value(s) per `fmt`, then the rest of the line (the
// comment) is consumed, as the reference's "%... %[^\n]" patterns do.
bool skip_rest(FILE* f) {
    int ch;
    while ((ch = std::fgetc(f)) != EOF && ch != '\n') {
    }
    return true;
}

bool read_int(FILE* f, int* v) {
    if (std::fscanf(f, "%d", v) != 1) return false;
    return skip_rest(f);
}

bool read_double(FILE* f, double* v) {
    if (std::fscanf(f, "%lf", v) != 1) return false;
    return skip_rest(f);
}

// Whole text file into memory.
bool slurp(const char* path, std::string& out) {
    File fl(path, "rb");
    if (!fl) return false;
    std::fseek(fl.f, 0, SEEK_END);
    const long sz = std::ftell(fl.f);
    std::fseek(fl.f, 0, SEEK_SET);
    if (sz < 0) return false;
    out.resize(static_cast<size_t>(sz));
    return sz == 0 || std::fread(out.data(), 1, out.size(), fl.f) == out.size();
}

// Number scanner over a text buffer (whitespace separated).
struct Scanner {
    const char* p;
    const char* e;
    void ws() {
        while (p < e && (*p == ' ' || *p == '\t' || *p == '\n' || *p == '\r')) ++p;
    }
    bool num(double* v) {
        ws();
        if (p >= e) return false;
        if (*p == '+') ++p;
        auto r = std::from_chars(p, e, *v);
        if (r.ec != std::errc()) return false;
        p = r.ptr;
        return true;
    }
    bool num(long long* v) {
        ws();
        if (p >= e) return false;
        if (*p == '+') ++p;
        auto r = std::from_chars(p, e, *v);
        if (r.ec != std::errc()) return false;
        p = r.ptr;
        return true;
    }
};

}  // namespace

extern "C" {

khrr_status khrr_read_galaxies_ini(const char* path, khrr_galaxy* out, int max, int* count) {
    if (!path || !count || max < 0 || (max > 0 && !out)) return KHRR_ERR_INVALID_ARG;
    File fl(path, "r");
    if (!fl) return KHRR_ERR_IO;
    FILE* f = fl.f;
    int n = 0;
    if (!read_int(f, &n) || n < 0) return KHRR_ERR_IO;
    for (int k = 0; k < n; ++k) {
        int id = 0, ns = 0, nd = 0;
        double ms = 0, md = 0, es = 0, ed = 0, a = 0, c[3] = {0, 0, 0}, v[3] = {0, 0, 0};
        if (!read_int(f, &id)) return KHRR_ERR_IO;
        if (std::fscanf(f, "%d,%d", &ns, &nd) != 2 || !skip_rest(f)) return KHRR_ERR_IO;
        if (std::fscanf(f, "%lf,%lf", &ms, &md) != 2 || !skip_rest(f)) return KHRR_ERR_IO;
        if (std::fscanf(f, "%lf,%lf", &es, &ed) != 2 || !skip_rest(f)) return KHRR_ERR_IO;
        if (!read_double(f, &a)) return KHRR_ERR_IO;
        if (std::fscanf(f, "%lf,%lf,%lf", &c[0], &c[1], &c[2]) != 3 || !skip_rest(f)) return KHRR_ERR_IO;
        if (std::fscanf(f, "%lf,%lf,%lf", &v[0], &v[1], &v[2]) != 3 || !skip_rest(f)) return KHRR_ERR_IO;
        if (k < max) {
            khrr_galaxy& g = out[k];
            // GalaxyProperties::get_n_*_particles: a massless component has no bodies.
            g.n_star = ms > 0.0 ? ns : 0;
            g.n_dark = md > 0.0 ? nd : 0;
            g.m_star = ms;
            g.m_dark = md;
            g.eps_star = es;
            g.eps_dark = ed;
            g.angle_deg = a;
            for (int q = 0; q < 3; ++q) {
                g.centre[q] = c[q];
                g.vel[q] = v[q];
            }
        }
    }
    *count = n;
    return KHRR_OK;
}

khrr_status khrr_read_start_nbody_ini(const char* path, int* i_cont, double* tmax, double* dt_save) {
    if (!path || !i_cont || !tmax || !dt_save) return KHRR_ERR_INVALID_ARG;
    File fl(path, "r");
    if (!fl) return KHRR_ERR_IO;
    if (!read_int(fl.f, i_cont) || !read_double(fl.f, tmax) || !read_double(fl.f, dt_save)) return KHRR_ERR_IO;
    return KHRR_OK;
}

khrr_status khrr_read_gr_par_ini(const char* path, khrr_field_params* field, double* eps, double* dtgrav,
                                 double* K_m, double* K_r) {
    if (!path) return KHRR_ERR_INVALID_ARG;
    File fl(path, "r");
    if (!fl) return KHRR_ERR_IO;
    double v[10];
    for (double& x : v)
        if (!read_double(fl.f, &x)) return KHRR_ERR_IO;
    if (field) *field = khrr_field_params{v[0], v[1], v[2], v[3], v[4], v[5]};
    if (eps) *eps = v[6];
    if (dtgrav) *dtgrav = v[7];
    if (K_m) *K_m = v[8];
    if (K_r) *K_r = v[9];
    return KHRR_OK;
}

khrr_status khrr_read_gpus_ini(const char* path, int* ngpu, int* devices, int max) {
    if (!path || !ngpu || max < 0 || (max > 0 && !devices)) return KHRR_ERR_INVALID_ARG;
    File fl(path, "r");
    if (!fl) return KHRR_ERR_IO;
    if (!read_int(fl.f, ngpu) || *ngpu < 0) return KHRR_ERR_IO;
    for (int k = 0; k < *ngpu; ++k) {
        int d = 0;
        if (!read_int(fl.f, &d)) return KHRR_ERR_IO;
        if (k < max) devices[k] = d;
    }
    return KHRR_OK;
}

khrr_status khrr_read_start_txt(const char* path, int64_t max, double* pos, double* vel, int64_t* n, double* t) {
    if (!path || !n || max < 0 || (max > 0 && (!pos || !vel))) return KHRR_ERR_INVALID_ARG;
    std::string buf;
    if (!slurp(path, buf)) return KHRR_ERR_IO;
    Scanner sc{buf.data(), buf.data() + buf.size()};
    long long hdr = 0;
    double tt = 0.0;
    if (!sc.num(&hdr) || !sc.num(&tt)) return KHRR_ERR_IO;
    const int64_t want = hdr < max ? hdr : max;
    for (int64_t i = 0; i < want; ++i) {
        double r[6];
        for (double& x : r)
            if (!sc.num(&x)) return KHRR_ERR_IO;
        for (int q = 0; q < 3; ++q) {
            pos[3 * i + q] = r[q];
            vel[3 * i + q] = r[3 + q];
        }
    }
    *n = want;
    if (t) *t = tt;
    return KHRR_OK;
}

khrr_status khrr_write_start_txt(const char* path, int64_t n, const double* pos, const double* vel, double t) {
    if (!path || n < 0 || (n > 0 && (!pos || !vel))) return KHRR_ERR_INVALID_ARG;
    File fl(path, "w");
    if (!fl) return KHRR_ERR_IO;
    std::fprintf(fl.f, "%lld %f\n", static_cast<long long>(n), t);
    for (int64_t i = 0; i < n; ++i)
        std::fprintf(fl.f, "%.17g %.17g %.17g %.17g %.17g %.17g\n", pos[3 * i], pos[3 * i + 1], pos[3 * i + 2],
                     vel[3 * i], vel[3 * i + 1], vel[3 * i + 2]);
    return std::ferror(fl.f) ? KHRR_ERR_IO : KHRR_OK;
}

khrr_status khrr_write_snapshot(const char* path, int32_t count, double t, const double* pos, const double* vel) {
    if (!path || count < 0 || (count > 0 && (!pos || !vel))) return KHRR_ERR_INVALID_ARG;
    File fl(path, "wb");
    if (!fl) return KHRR_ERR_IO;
    std::vector<double> rec(6 * static_cast<size_t>(count));
    for (int32_t i = 0; i < count; ++i)
        for (int q = 0; q < 3; ++q) {
            rec[6 * static_cast<size_t>(i) + q] = pos[3 * i + q];
            rec[6 * static_cast<size_t>(i) + 3 + q] = vel[3 * i + q];
        }
    if (std::fwrite(&count, sizeof count, 1, fl.f) != 1 || std::fwrite(&t, sizeof t, 1, fl.f) != 1 ||
        std::fwrite(rec.data(), sizeof(double), rec.size(), fl.f) != rec.size())
        return KHRR_ERR_IO;
    return KHRR_OK;
}

khrr_status khrr_read_snapshot(const char* path, int64_t max, double* pos, double* vel, int32_t* count, double* t) {
    if (!path || !count || max < 0 || (max > 0 && (!pos || !vel))) return KHRR_ERR_INVALID_ARG;
    File fl(path, "rb");
    if (!fl) return KHRR_ERR_IO;
    int32_t c = 0;
    double tt = 0.0;
    if (std::fread(&c, sizeof c, 1, fl.f) != 1 || std::fread(&tt, sizeof tt, 1, fl.f) != 1 || c < 0)
        return KHRR_ERR_IO;
    const int64_t want = c < max ? c : max;
    std::vector<double> rec(6 * static_cast<size_t>(want));
    if (std::fread(rec.data(), sizeof(double), rec.size(), fl.f) != rec.size()) return KHRR_ERR_IO;
    for (int64_t i = 0; i < want; ++i)
        for (int q = 0; q < 3; ++q) {
            pos[3 * i + q] = rec[6 * static_cast<size_t>(i) + q];
            vel[3 * i + q] = rec[6 * static_cast<size_t>(i) + 3 + q];
        }
    *count = c;
    if (t) *t = tt;
    return KHRR_OK;
}

khrr_status khrr_write_lie0(const char* path, const khrr_lie* lie0) {
    if (!path || !lie0) return KHRR_ERR_INVALID_ARG;
    File fl(path, "wb");
    if (!fl) return KHRR_ERR_IO;
    double rec[9] = {lie0->L[0], lie0->L[1], lie0->L[2], lie0->Imp[0], lie0->Imp[1], lie0->Imp[2], lie0->E, 0.0, 0.0};
    return std::fwrite(rec, sizeof(double), 9, fl.f) == 9 ? KHRR_OK : KHRR_ERR_IO;
}

khrr_status khrr_read_lie0(const char* path, khrr_lie* lie0) {
    if (!path || !lie0) return KHRR_ERR_INVALID_ARG;
    File fl(path, "rb");
    if (!fl) return KHRR_ERR_IO;
    double rec[7];
    if (std::fread(rec, sizeof(double), 7, fl.f) != 7) return KHRR_ERR_IO;
    std::memset(lie0, 0, sizeof *lie0);
    for (int q = 0; q < 3; ++q) {
        lie0->L[q] = rec[q];
        lie0->Imp[q] = rec[3 + q];
    }
    lie0->E = rec[6];
    return KHRR_OK;
}

khrr_status khrr_load_initial_conditions(const char* dir, const khrr_galaxy* g, int ngal, int64_t max, double* pos,
                                         double* vel, double* mass, double* eps2, int64_t* n, int64_t* n_star_total) {
    if (!dir || !g || ngal < 0 || !n || !pos || !vel || !mass || !eps2) return KHRR_ERR_INVALID_ARG;
    int64_t total = 0, stars = 0;
    for (int k = 0; k < ngal; ++k) {
        if (g[k].n_star < 0 || g[k].n_dark < 0) return KHRR_ERR_INVALID_ARG;
        total += g[k].n_star + g[k].n_dark;
        stars += g[k].n_star;
    }
    if (total > max) return KHRR_ERR_INVALID_ARG;
    int64_t at = 0;
    // Stars of every galaxy, then dark matter of every galaxy (nbody.cu:1318-1417).
    for (int comp = 0; comp < 2; ++comp) {
        for (int k = 0; k < ngal; ++k) {
            const int64_t cnt = comp == 0 ? g[k].n_star : g[k].n_dark;
            if (cnt == 0) continue;
            const std::string path = std::string(dir) + (comp == 0 ? "/start_S" : "/start_DM") + std::to_string(k) + ".txt";
            int64_t got = 0;
            khrr_status st = khrr_read_start_txt(path.c_str(), cnt, pos + 3 * at, vel + 3 * at, &got, nullptr);
            if (st != KHRR_OK) return st;
            if (got != cnt) return KHRR_ERR_IO;
            const double rad = kPi / 180.0 * g[k].angle_deg;  // DEG2RAD * angle
            const double m = (comp == 0 ? g[k].m_star : g[k].m_dark) / static_cast<double>(cnt);
            const double e = comp == 0 ? g[k].eps_star : g[k].eps_dark;
            for (int64_t i = at; i < at + cnt; ++i) {
                double* p = pos + 3 * i;
                double* v = vel + 3 * i;
                // nbody.cu:1342-1358: z uses the x just overwritten (a shear for alpha != 0).
                p[0] = g[k].centre[0] + p[0] * std::cos(rad) + p[2] * std::sin(rad);
                p[1] += g[k].centre[1];
                p[2] = g[k].centre[2] + p[2] * std::cos(rad) - p[0] * std::sin(rad);
                v[0] = g[k].vel[0] + v[0] * std::cos(rad) + v[2] * std::sin(rad);
                v[1] += g[k].vel[1];
                v[2] = g[k].vel[2] + v[2] * std::cos(rad) - v[0] * std::sin(rad);
                mass[i] = m;
                eps2[i] = e * e;
            }
            at += cnt;
        }
    }
    *n = total;
    if (n_star_total) *n_star_total = stars;
    return KHRR_OK;
}

}  // extern "C"
