// khrr_nbody: the reference's program (run(), nbody/src/nbody.cu:1010-1711)
// on libkhrr.  Reads the same data/nbody/ini files, writes the same bin/ and
// out/ files, and runs the time loop on the GPU through the C ABI.
//
//   khrr_nbody [--data DIR] [--device K] [--compat-accumulate] [--no-mesh]
//              [--mesh-nx N] [--mesh-dx D] [--wave] [--wave-fp32] [--cic]
//              [--wave-setup ITERS] [--kernel auto|pair|one-sided|fp64] [--quiet]
//
// --kernel picks the direct-sum force kernel: auto (default) times the
// candidates on the initial state (khrr_autotune), pair is the symmetric
// kernel (each unordered pair once for both bodies), one-sided the kernel
// that evaluates every ordered pair, fp64 the direct sum in FP64 (the
// reference's own precision, KHRR_FP64; about a fifth of the pair kernel's
// rate).
//
// --wave selects the reference's Wave solver (NBodySolver::Wave, compiled in
// the reference but switched off at nbody.cu:1132): forces and potentials
// from the damped-wave mesh field (setup ITERS iterations, default 20000,
// then (int)(dtgrav / dt_wave) per step), the FP64 stencil and NGP deposit
// unless --wave-fp32 / --cic; phi/ cuts then show that field (nbody.cu:1485,
// 1666).
//
// DIR defaults to $KHRR_DATA or ./data/nbody (the reference's BASE_PATH,
// target_dir.h.in:5-9); inputs come from DIR/ini, outputs go to DIR/bin and
// DIR/out.  Deliberate differences from the reference, each a fix of a defect:
//  * the step force overwrites the previous one (the reference never resets
//    acct_, nbody.cu:1559-1566); --compat-accumulate restores the literal loop;
//  * restart (i_cont > 0) reads S_/DM_ snapshots by the names they are written
//    under ("{:5}") and reads the dark matter too (nbody.cu:1251, 1274);
//  * the potential of a save comes out of the last step's force pass (the
//    positions after the corrector are the predicted ones the force used),
//    instead of a second O(N^2) PHI_kernel pass;
//  * the readme's E(t).dat, imp(t).dat, LL(t).dat, Lz(t).dat and
//    time_frame.dat are written next to the code's CSV logs.
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <filesystem>
#include <format>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "khrr.h"

namespace fs = std::filesystem;

namespace {

struct Options {
    std::string data;
    int device = -1;
    bool compat = false;
    bool mesh = true;
    int mesh_nx = 200;     // nbody.cu:1134
    double mesh_dx = 0.2;  // nbody.cu:1135
    bool wave = false;
    bool wave_fp32 = false;
    bool cic = false;
    int wave_setup = 20000;  // _iterations_to_setup, nbody.cu:1143
    std::string kernel = "auto";
    bool quiet = false;
};

[[noreturn]] void die(const std::string& msg) {
    std::fprintf(stderr, "Error: %s\n", msg.c_str());
    std::exit(1);
}

void check(khrr_status st, khrr_ctx* ctx, const char* what) {
    if (st != KHRR_OK)
        die(std::format("{} failed: {} ({})", what, khrr_status_name(st), ctx ? khrr_last_error(ctx) : ""));
}

// ostream's default double formatting, as the reference's CSV rows use it.
std::string g6(double v) {
    std::ostringstream s;
    s << v;
    return s.str();
}

struct Lie {
    double L[3], Imp[3], E;
};

// One save frame's conservation output (result(), nbody.cu:763-960).
struct Writer {
    fs::path bin, out;
    bool quiet;
    Lie lie0{};
    std::chrono::steady_clock::time_point start = std::chrono::steady_clock::now();

    void rows(const char* csv, const char* dat, const char* header, int it, const std::string& row) const {
        const auto mode = it == 0 ? std::ios::out : std::ios::app;
        std::ofstream c(out / csv, mode), d(out / dat, mode);
        if (it == 0) c << header << std::endl;
        c << row << std::endl;
        std::string sp = row;
        for (size_t k = 0; (k = sp.find(", ", k)) != std::string::npos;) sp.replace(k, 2, " ");
        d << sp << std::endl;
    }

    void result(khrr_ctx* ctx, const std::vector<double>& pos, const std::vector<double>& vel, int64_t ns,
                int64_t nn, int it, double t, long long it_all) {
        if (it > 1 && it % 10 == 0) {
            check(khrr_write_snapshot((bin / std::format("S_{:5}.bin", it)).string().c_str(), static_cast<int32_t>(ns),
                                      t, pos.data(), vel.data()),
                  nullptr, "snapshot");
            if (nn > ns)
                check(khrr_write_snapshot((bin / std::format("DM_{:5}.bin", it)).string().c_str(),
                                          static_cast<int32_t>(nn - ns), t, pos.data() + 3 * ns, vel.data() + 3 * ns),
                      nullptr, "snapshot");
        }
        khrr_lie v{};
        check(khrr_conservation(ctx, &v), ctx, "conservation");
        if (it == 0) {
            for (int q = 0; q < 3; ++q) {
                lie0.L[q] = v.L[q];
                lie0.Imp[q] = v.Imp[q];
            }
            lie0.E = v.E;
            khrr_lie l0{};
            for (int q = 0; q < 3; ++q) {
                l0.L[q] = v.L[q];
                l0.Imp[q] = v.Imp[q];
            }
            l0.E = v.E;
            check(khrr_write_lie0((bin / "LIE_0.bin").string().c_str(), &l0), nullptr, "LIE_0.bin");
        }
        const double LL = std::sqrt(v.L[0] * v.L[0] + v.L[1] * v.L[1] + v.L[2] * v.L[2]);
        const double LL0 = std::sqrt(lie0.L[0] * lie0.L[0] + lie0.L[1] * lie0.L[1] + lie0.L[2] * lie0.L[2]);
        const double imp = std::sqrt(v.Imp[0] * v.Imp[0] + v.Imp[1] * v.Imp[1] + v.Imp[2] * v.Imp[2]);
        const double imp0 =
            std::sqrt(lie0.Imp[0] * lie0.Imp[0] + lie0.Imp[1] * lie0.Imp[1] + lie0.Imp[2] * lie0.Imp[2]);
        if (!quiet) {
            std::printf("           ***Star***\n R_max = %g  Z_max = %g \n", v.R_max, v.Z_max);
            std::printf("Vr_max = %g  Vfi_max = %g  Vz_max = %g \n", v.Vr_max, v.Vfi_max, v.Vz_max);
            std::printf("           ***Conservation Laws***\n");
            std::printf("----Imp0--- = %g; %g; %g  \n", lie0.Imp[0], lie0.Imp[1], lie0.Imp[2]);
            std::printf("----dImp--- = %g; %g; %g  \n", v.Imp[0] - lie0.Imp[0], v.Imp[1] - lie0.Imp[1],
                        v.Imp[2] - lie0.Imp[2]);
            std::printf("Lz = %g  dLz = %g \n", v.L[2], v.L[2] / lie0.L[2] - 1.0);
            std::printf("LL = %g  dLL = %g \n", LL, LL / LL0 - 1.0);
            std::printf("E = %g  dE = %g \n", v.E, v.E / lie0.E - 1.0);
        }
        const std::string pre = std::format("{}, ", it_all) + g6(t) + ", ";
        rows("Lz(t).csv", "Lz(t).dat", "it, t, Lz, Lz_rel_err, Lz_rel_err_magnitude", it,
             pre + std::format("{:.15f}", v.L[2]) + ", " + g6(v.L[2] / lie0.L[2] - 1.0) + ", " +
                 g6(std::fabs(v.L[2] / lie0.L[2] - 1.0)));
        rows("LL(t).csv", "LL(t).dat", "it, t, LL, LL_rel_err, LL_rel_err_magnitude", it,
             pre + std::format("{:.15f}", LL) + ", " + g6(LL / LL0 - 1.0) + ", " + g6(std::fabs(LL / LL0 - 1.0)));
        rows("Imp(t).csv", "imp(t).dat", "it, t, Imp, Imp_abs_err, Imp_rel_err, Imp_rel_err_magnitude", it,
             pre + std::format("{:.15f}", imp) + ", " + g6(imp - imp0) + ", " + g6(imp / imp0 - 1.0) + ", " +
                 g6(std::fabs(imp / imp0 - 1.0)));
        rows("E(t).csv", "E(t).dat", "it, t, E, E_rel_err, E_rel_err_magnitude, Ek, Ep", it,
             pre + std::format("{:.15f}", v.E) + ", " + g6(v.E / lie0.E - 1.0) + ", " +
                 g6(std::fabs(v.E / lie0.E - 1.0)) + ", " + g6(0.5 * v.Ek) + ", " + g6(0.5 * v.Ep));
    }
};

Options parse(int argc, char** argv) {
    Options o;
    if (const char* e = std::getenv("KHRR_DATA")) o.data = e;
    if (o.data.empty()) o.data = "data/nbody";
    for (int i = 1; i < argc; ++i) {
        const std::string a = argv[i];
        auto next = [&]() -> std::string {
            if (i + 1 >= argc) die("missing value after " + a);
            return argv[++i];
        };
        if (a == "--data") o.data = next();
        else if (a == "--device") o.device = std::stoi(next());
        else if (a == "--compat-accumulate") o.compat = true;
        else if (a == "--no-mesh") o.mesh = false;
        else if (a == "--mesh-nx") o.mesh_nx = std::stoi(next());
        else if (a == "--mesh-dx") o.mesh_dx = std::stod(next());
        else if (a == "--wave") o.wave = true;
        else if (a == "--wave-fp32") o.wave_fp32 = true;
        else if (a == "--cic") o.cic = true;
        else if (a == "--wave-setup") o.wave_setup = std::stoi(next());
        else if (a == "--kernel") {
            o.kernel = next();
            if (o.kernel != "auto" && o.kernel != "pair" && o.kernel != "one-sided" && o.kernel != "fp64")
                die("--kernel takes auto, pair, one-sided or fp64");
        }
        else if (a == "--quiet") o.quiet = true;
        else die("unknown argument " + a);
    }
    return o;
}

}  // namespace

int main(int argc, char** argv) {
    const Options opt = parse(argc, argv);
    const fs::path base(opt.data), ini = base / "ini", bin = base / "bin", out = base / "out";
    std::error_code ec;

    // ---- inputs (nbody.cu:1030-1106) ----
    std::vector<khrr_galaxy> gal(256);
    int ngal = 0;
    if (khrr_read_galaxies_ini((ini / "__start_galaxies.ini").string().c_str(), gal.data(), 256, &ngal) != KHRR_OK)
        die("can't read galaxy properties file: " + (ini / "__start_galaxies.ini").string());
    if (ngal < 1 || ngal > 256) die("no galaxy properties read");
    gal.resize(ngal);
    int device = 0;
    {
        int ngpu = 0, devs[8] = {0};
        const fs::path gp = ini / "__GPUs.ini";
        if (fs::exists(gp)) {
            if (khrr_read_gpus_ini(gp.string().c_str(), &ngpu, devs, 8) != KHRR_OK) die("can't read " + gp.string());
            if (ngpu != 1) die(std::format("__GPUs.ini asks for {} GPUs; this program runs on one", ngpu));
            device = devs[0];
        }
    }
    if (opt.device >= 0) device = opt.device;
    int i_cont = 0;
    double tmax = 0.0, dtsave = 0.0;
    if (khrr_read_start_nbody_ini((ini / "__start_nbody.ini").string().c_str(), &i_cont, &tmax, &dtsave) != KHRR_OK)
        die("can't read __start_nbody.ini");
    khrr_field_params field{};
    double eps = 0.0, dtgrav = 0.0, K_m = 0.0, K_r = 0.0;
    if (khrr_read_gr_par_ini((ini / "__gr_par.ini").string().c_str(), &field, &eps, &dtgrav, &K_m, &K_r) != KHRR_OK)
        die("can't read __gr_par.ini");
    if (!(dtgrav > 0.0) || !(dtsave > 0.0)) die("dtgrav and dt_save must be > 0");
    const int is_grav = static_cast<int>(dtsave / dtgrav + 0.5);  // nbody.cu:1108
    if (is_grav < 1) die("dt_save shorter than half a time step");

    int64_t ns = 0, nn = 0;
    for (const auto& g : gal) {
        ns += g.n_star;
        nn += g.n_star + g.n_dark;
    }
    if (nn < 1) die("no bodies");
    std::printf("galaxies count: %d\ntotal particles: %lld\nstar particles: %lld\ndark particles: %lld\n", ngal,
                static_cast<long long>(nn), static_cast<long long>(ns), static_cast<long long>(nn - ns));
    std::printf("i_cont: %d\ntmax: %f\ndtsave %f\ndtgrav\t= %lf\n", i_cont, tmax, dtsave, dtgrav);

    fs::create_directories(bin, ec);
    fs::create_directories(out, ec);
    std::vector<double> pos(3 * nn), vel(3 * nn), acc(3 * nn), mass(nn), eps2(nn), phi(nn);
    double t = 0.0, tsave = 0.0, tgrav = 0.0;
    int it = 1, itt = 1, ittg = 0, itg = 1;
    Writer w{bin, out, opt.quiet};

    if (i_cont > 0) {
        // Restart (nbody.cu:1247-1314) with the snapshot names as written.
        std::vector<double> p(3 * nn), v(3 * nn);
        int32_t cnt = 0;
        double ts = 0.0;
        if (khrr_read_snapshot((bin / std::format("S_{:5}.bin", i_cont)).string().c_str(), ns, pos.data(), vel.data(),
                               &cnt, &ts) != KHRR_OK ||
            cnt != ns)
            die(std::format("can't read star snapshot S_{:5}.bin", i_cont));
        t = ts;
        if (nn > ns &&
            (khrr_read_snapshot((bin / std::format("DM_{:5}.bin", i_cont)).string().c_str(), nn - ns, pos.data() + 3 * ns,
                                vel.data() + 3 * ns, &cnt, &ts) != KHRR_OK ||
             cnt != nn - ns))
            die(std::format("can't read dark-matter snapshot DM_{:5}.bin", i_cont));
        int64_t at = 0;
        for (int comp = 0; comp < 2; ++comp)
            for (const auto& g : gal) {
                const int64_t c = comp == 0 ? g.n_star : g.n_dark;
                const double m = c ? (comp == 0 ? g.m_star : g.m_dark) / static_cast<double>(c) : 0.0;
                const double e = comp == 0 ? g.eps_star : g.eps_dark;
                for (int64_t i = at; i < at + c; ++i) {
                    mass[i] = m;
                    eps2[i] = e * e;
                }
                at += c;
            }
        it = static_cast<int>(t / dtsave);
        khrr_lie l0{};
        if (khrr_read_lie0((bin / "LIE_0.bin").string().c_str(), &l0) != KHRR_OK) die("can't read LIE_0.bin");
        for (int q = 0; q < 3; ++q) {
            w.lie0.L[q] = l0.L[q];
            w.lie0.Imp[q] = l0.Imp[q];
        }
        w.lie0.E = l0.E;
        ++it;
        itg = static_cast<int>(t / dtgrav) + 1;
        tsave = t + dtsave;
        tgrav = t + dtgrav;
        std::printf("Start time = %f  it = %d\n", t, it);
    } else {
        int64_t got = 0, got_s = 0;
        khrr_status st = khrr_load_initial_conditions(ini.string().c_str(), gal.data(), ngal, nn, pos.data(), vel.data(),
                                                      mass.data(), eps2.data(), &got, &got_s);
        if (st != KHRR_OK || got != nn) die("can't read the start_S*/start_DM* initial conditions in " + ini.string());
        tsave = dtsave;
        tgrav = dtgrav;
        t = 0.0;
    }

    // ---- device state and setup forces (nbody.cu:1428-1486) ----
    khrr_ctx* ctx = nullptr;
    if (khrr_create(device, &ctx) != KHRR_OK) die(std::format("no usable sm_100 device {}", device));
    if (field.Mh != 0.0 || field.Mb != 0.0) check(khrr_set_external_field(ctx, &field), ctx, "external field");
    check(khrr_upload_state(ctx, nn, pos.data(), vel.data(), mass.data(), eps2.data(), 1, nullptr), ctx, "upload");
    if (!opt.wave && opt.kernel == "auto") {
        check(khrr_autotune(ctx, nullptr), ctx, "autotune");
    } else if (opt.kernel == "pair") {
        const khrr_tuning pair{128, 8, 128, 0, 2};
        check(khrr_set_tuning(ctx, &pair), ctx, "tuning");
    }
    // Mesh of the save-time binning and of the Wave solver (nbody.cu:1134-1143).
    const int NX = opt.mesh_nx;
    const double L = 0.5 * NX * opt.mesh_dx;
    khrr_mesh mesh{};
    for (int q = 0; q < 3; ++q) {
        mesh.lo[q] = -L;
        mesh.cell[q] = opt.mesh_dx;
        mesh.grid[q] = NX;
    }
    int solver_flag = 0;
    if (opt.wave) {
        khrr_mesh_solver ms{};
        const double c_wave = 4574.337022617616;  // nbody.cu:1137
        ms.wave.nx = NX;
        ms.wave.dx = opt.mesh_dx;
        ms.wave.c = c_wave;
        ms.wave.dt = 0.5 * opt.mesh_dx / (c_wave * std::sqrt(3.0));
        ms.wave.diss_base = 0.1;
        ms.wave.diss_extra = 0.01;
        ms.wave.sim_l = L;
        ms.wave.bc_l = L / 10.;
        ms.assign = opt.cic ? KHRR_ASSIGN_CIC : KHRR_ASSIGN_NGP;
        ms.fp64 = opt.wave_fp32 ? 0 : 1;
        ms.iters_per_step = static_cast<int>(dtgrav / ms.wave.dt);  // calc_acceleration_by_grid's int argument
        ms.setup_iters = opt.wave_setup;
        if (ms.iters_per_step < 1) die("dtgrav is shorter than one wave step");
        std::printf("Wave eq iterations: %d\n", ms.iters_per_step);
        check(khrr_set_mesh_solver(ctx, &ms), ctx, "mesh solver");
        solver_flag = KHRR_MESH;
    } else if (opt.kernel == "fp64") {
        solver_flag = KHRR_FP64;
    }
    std::vector<double> cell_phi(opt.mesh || opt.wave ? static_cast<size_t>(NX) * NX * NX : 0);
    auto print_cell_phi = [&](int iter) {
        const fs::path dir = out / "phi";
        fs::create_directories(dir, ec);
        std::ofstream s(dir / std::format("phi_{:5}.csv", iter));
        s << "x, phi" << std::endl;
        const int IY = NX / 2, IZ = NX / 2;
        for (int i = 0; i < NX; ++i) {
            const double x = -L + i * opt.mesh_dx;
            const size_t at = static_cast<size_t>(i) + static_cast<size_t>(IY) * NX + static_cast<size_t>(IZ) * NX * NX;
            s << std::format("{}, {:.7f}", x, cell_phi[at]) << std::endl;
        }
    };

    const auto t_setup = std::chrono::steady_clock::now();
    check(khrr_forces(ctx, KHRR_ACC | KHRR_PHI | solver_flag), ctx, "setup forces");
    if (opt.wave) {
        check(khrr_mesh_solver_phi(ctx, cell_phi.data()), ctx, "mesh field");
        print_cell_phi(0);
    }
    check(khrr_synchronize(ctx), ctx, "setup");
    std::printf("time for setup: %g seconds \n",
                std::chrono::duration<double>(std::chrono::steady_clock::now() - t_setup).count());
    if (it == 1) {
        std::printf("***Start result t=0***\n");
        check(khrr_download_state(ctx, pos.data(), vel.data(), acc.data(), phi.data()), ctx, "download");
        w.result(ctx, pos, vel, ns, nn, 0, 0.0, 0);
    }

    // ---- time loop (nbody.cu:1518-1709) ----
    // The Wave branch zeroes acct_ every step (nbody.cu:1542): nothing to accumulate.
    const int flags_compat = opt.compat && !opt.wave ? KHRR_COMPAT_ACCUMULATE : 0;
    int it_grav = 0;
    long long total_steps = 0;
    double gpu_time = 0.0;
    auto t_frame = std::chrono::steady_clock::now();
    bool running = true;
    while (running) {
        // Steps until the next save or the end, with the reference's counters.
        int k = 0;
        bool save = false;
        do {
            ++ittg;
            ++itg;
            t = tgrav;
            tgrav = itg * dtgrav;
            ++it_grav;
            ++k;
            if (it_grav >= is_grav) {
                save = true;
                break;
            }
            ++itt;
        } while (t < tmax);
        check(khrr_step(ctx, dtgrav, k, flags_compat | solver_flag | (save ? KHRR_PHI : 0)), ctx, "step");
        total_steps += k;
        if (save) {
            tsave = tgrav;
            if (opt.wave) {
                check(khrr_mesh_solver_phi(ctx, cell_phi.data()), ctx, "mesh field");
            } else if (opt.mesh) {  // the Nbody branch's save-time binning (nbody.cu:1601-1634)
                check(khrr_bin(ctx, &mesh, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr), ctx, "binning");
                check(khrr_bin_cell_phi(ctx, 0, cell_phi.data()), ctx, "cell phi");
            }
            check(khrr_download_state(ctx, pos.data(), vel.data(), acc.data(), phi.data()), ctx, "download");
            const auto now = std::chrono::steady_clock::now();
            const double frame_s = std::chrono::duration<double>(now - t_frame).count();
            t_frame = now;
            gpu_time += frame_s;
            std::printf("--------------------------------------------------------------------------------\n");
            std::printf("<Time_frame> = %.3f s, frame = %d, iter = %d, iter_g = %d\n", gpu_time, it, itt, ittg);
            std::printf("Time = (%g,  %g) ---  dt = (%g,  %g)\n", t, tgrav - dtgrav, dtsave / itt, dtgrav);
            if (opt.mesh || opt.wave) print_cell_phi(itt * it);
            {
                // sample.csv: body 1 (nbody.cu:1668-1699).
                std::ofstream s(out / "sample.csv", it == 1 ? std::ios::out : std::ios::app);
                if (it == 1) s << "it, t, i, r, fi, z, acc, phi, ax, ay, az" << std::endl;
                const int64_t i = nn > 1 ? 1 : 0;
                const double x = pos[3 * i], y = pos[3 * i + 1], z = pos[3 * i + 2];
                const double ax = acc[3 * i], ay = acc[3 * i + 1], az = acc[3 * i + 2];
                s << it * itt << ", " << t << ", " << i << ", " << std::sqrt(x * x + y * y) << ", " << std::atan2(y, x)
                  << ", " << z << ", " << std::sqrt(ax * ax + ay * ay + az * az) << ", " << phi[i] << ", " << ax << ", "
                  << ay << ", " << az << std::endl;
            }
            w.result(ctx, pos, vel, ns, nn, it, t, static_cast<long long>(it) * itt);
            {
                // time_frame.dat (readme.md:51-53): iterations, model time, compute time, 0, compute time.
                std::ofstream s(out / "time_frame.dat", std::ios::app);
                s << total_steps << " " << t << " " << gpu_time << " 0 " << gpu_time << std::endl;
            }
            tsave += dtsave;
            ++it;
            itt = 0;
            ittg = 0;
            it_grav = 0;
            ++itt;
        }
        running = t < tmax;
    }
    khrr_destroy(ctx);
    std::printf("done: %lld steps, t = %g\n", total_steps, t);
    return 0;
}
