// C ABI of the p2mesh path: kernel-level entry points (the reference's
// pointers and layouts) and the context-level pipeline khrr_bin /
// khrr_wave_solve.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "khrr.h"
#include "khrr_internal.h"
#include "khrr_runtime.h"

using namespace khrr;

namespace {

constexpr double kPi = 3.14159265358979;  // the reference's PI (common.cuh:7)

// The reference's cell id can exceed the cell count for some non-cubic grids
// (iz is clamped to gy - 1 and the y stride is gz); such meshes are refused.
khrr_status check_mesh(khrr_ctx* c, const khrr_mesh* m, MeshGeom* g, int64_t* ncells) {
    if (!m) return c->fail(KHRR_ERR_INVALID_ARG, "null mesh");
    for (int k = 0; k < 3; ++k) {
        if (m->grid[k] < 1) return c->fail(KHRR_ERR_INVALID_ARG, "grid[%d] must be >= 1", k);
        if (!(m->cell[k] > 0.0) || !std::isfinite(m->cell[k]) || !std::isfinite(m->lo[k]))
            return c->fail(KHRR_ERR_INVALID_ARG, "mesh origin / cell size must be finite, cell > 0");
        g->lo[k] = m->lo[k];
        g->cs[k] = m->cell[k];
        g->g[k] = m->grid[k];
    }
    const int64_t gx = m->grid[0], gy = m->grid[1], gz = m->grid[2];
    const int64_t C = gx * gy * gz;
    if (C > 0x7fffffffLL) return c->fail(KHRR_ERR_INVALID_ARG, "too many cells");
    const int64_t max_id = (gy - 1) * gx * gy + (gy - 1) * gz + (gx - 1);
    if (max_id >= C) return c->fail(KHRR_ERR_INVALID_ARG, "grid shape gives cell ids beyond the mesh");
    *ncells = C;
    return KHRR_OK;
}

WaveConsts wave_consts(const khrr_wave_params* p) {
    WaveConsts w{};
    w.nx = p->nx;
    w.dx = p->dx;
    w.dt = p->dt;
    w.c = p->c;
    w.diss_base = p->diss_base;
    w.diss_extra = p->diss_extra;
    w.sim_l = p->sim_l;
    w.bc_l = p->bc_l;
    return w;
}

khrr_status check_wave(khrr_ctx* c, const khrr_wave_params* p) {
    if (!p) return c->fail(KHRR_ERR_INVALID_ARG, "null wave parameters");
    if (p->nx < 3 || p->nx > 2048) return c->fail(KHRR_ERR_INVALID_ARG, "nx must be in [3, 2048]");
    if (!(p->dx > 0.0) || !(p->dt > 0.0) || !(p->c > 0.0))
        return c->fail(KHRR_ERR_INVALID_ARG, "dx, dt and c must be > 0");
    return KHRR_OK;
}

// Per-axis sponge terms of wave_diss_iteration (wave-kernel.cuh:32-60) in
// FP64, rounded once to FP32; the x test compares against -(L - bc).
void sponge_tables(const khrr_wave_params* p, std::vector<float>& t) {
    const int nx = p->nx;
    const double L = p->sim_l - p->bc_l;
    t.assign(3 * static_cast<size_t>(nx), 0.0f);
    for (int i = 0; i < nx; ++i) {
        const double x = i * p->dx;
        double sx = 0.0, sy = 0.0;
        if (x > -L) sx = p->diss_extra * std::fabs(x - L) * std::fabs(x - L);
        else if (x < -L) sx = p->diss_extra * std::fabs(x + L) * std::fabs(x + L);
        if (x > L) sy = p->diss_extra * std::fabs(x - L) * std::fabs(x - L);
        else if (x < -L) sy = p->diss_extra * std::fabs(x + L) * std::fabs(x + L);
        t[i] = static_cast<float>(sx);
        t[nx + i] = static_cast<float>(sy);
        t[2 * nx + i] = static_cast<float>(sy);  // the z test is the y test
    }
}

WaveF32 wave_f32(const khrr_wave_params* p, const float* tab) {
    WaveF32 w{};
    const double C = p->c, DT = p->dt, DX = p->dx;
    const double K = C * C * (DT * DT) / (DX * DX);
    w.nx = p->nx;
    w.diss_base = static_cast<float>(p->diss_base);
    w.cdt_half = static_cast<float>(C * DT * 0.5);
    w.K = static_cast<float>(K);
    w.A = static_cast<float>(2.0 * (1.0 - 3.0 * K));
    w.S = static_cast<float>(-(C * C) * (DT * DT) * (4.0 * kPi) / (DX * DX * DX));
    w.sx = tab;
    w.sy = tab + p->nx;
    w.sz = tab + 2 * p->nx;
    return w;
}

}  // namespace

extern "C" {

khrr_status khrr_assign_particles_to_cells(khrr_ctx* c, const double* pos, int64_t n, const khrr_mesh* mesh,
                                           int* particle_cell_info, int* cell_info, int* cell_count,
                                           const double* mass, double* cell_mass) {
    if (!c) return KHRR_ERR_INVALID_ARG;
    MeshGeom g;
    int64_t C = 0;
    khrr_status st = check_mesh(c, mesh, &g, &C);
    if (st != KHRR_OK) return st;
    if (n < 0 || (n > 0 && (!pos || !particle_cell_info || !cell_info)) || (cell_mass && !mass))
        return c->fail(KHRR_ERR_INVALID_ARG, "bad binning arguments");
    int* counter = cell_count ? cell_count : cell_info;
    const int cstride = cell_count ? 1 : 2;
    int* count2 = cell_count ? cell_info : nullptr;
    return c->cuda(launch_assign(pos, n, g, reinterpret_cast<int2*>(particle_cell_info), counter, cstride, count2, 2,
                                 mass, cell_mass, c->stream),
                   "assign");
}

khrr_status khrr_compute_prefix_sums(khrr_ctx* c, int* cell_info, int* max_pbc, int64_t ncells, int mode) {
    if (!c) return KHRR_ERR_INVALID_ARG;
    if (ncells < 1 || ncells > 0x7fffffffLL || !cell_info || !max_pbc ||
        (mode != KHRR_SCAN_REFERENCE && mode != KHRR_SCAN_EXCLUSIVE))
        return c->fail(KHRR_ERR_INVALID_ARG, "bad prefix-sum arguments");
    if (reinterpret_cast<uintptr_t>(cell_info) % 16)
        return c->fail(KHRR_ERR_INVALID_ARG, "cell_info must be 16-byte aligned");
    khrr_status st = c->cuda(c->mtmp.ensure(static_cast<size_t>(scan_scratch_ints(ncells))), "alloc");
    if (st != KHRR_OK) return st;
    return c->cuda(launch_scan(cell_info, true, ncells, max_pbc, nullptr, mode == KHRR_SCAN_REFERENCE, c->mtmp.p,
                               c->stream),
                   "prefix sums");
}

khrr_status khrr_cell_phi(khrr_ctx* c, const double* phi, const int* particle_cell_info, const int* cell_info,
                          int64_t n, double* cell_phi) {
    if (!c) return KHRR_ERR_INVALID_ARG;
    if (n < 0 || (n > 0 && (!phi || !particle_cell_info || !cell_info || !cell_phi)))
        return c->fail(KHRR_ERR_INVALID_ARG, "bad cell-phi arguments");
    return c->cuda(launch_cell_phi(phi, reinterpret_cast<const int2*>(particle_cell_info), cell_info, 2, n, cell_phi,
                                   c->stream),
                   "cell phi");
}

khrr_status khrr_wave_iteration(khrr_ctx* c, double* phi_new, const double* phi, const double* phi_old,
                                const double* cell_mass, const khrr_wave_params* p) {
    if (!c) return KHRR_ERR_INVALID_ARG;
    khrr_status st = check_wave(c, p);
    if (st != KHRR_OK) return st;
    if (!phi_new || !phi || !phi_old || !cell_mass) return c->fail(KHRR_ERR_INVALID_ARG, "null mesh array");
    return c->cuda(launch_wave_f64(phi_new, phi, phi_old, cell_mass, wave_consts(p), c->stream), "wave iteration");
}

khrr_status khrr_acc_field(khrr_ctx* c, double* cell_acc, double* cell_acc_abs, const double* cell_phi, int nx,
                           double dx) {
    if (!c) return KHRR_ERR_INVALID_ARG;
    if (nx < 2 || nx > 2048 || !cell_acc || !cell_phi || !(dx > 0.0))
        return c->fail(KHRR_ERR_INVALID_ARG, "bad acc_field arguments");
    return c->cuda(launch_acc_field(cell_acc, cell_acc_abs, cell_phi, nx, dx, c->stream), "acc_field");
}

khrr_status khrr_apply_cells_to_particles(khrr_ctx* c, double* particle_acc, double* particle_value,
                                          const double* cell_acc, const double* cell_value,
                                          const int* particle_cell_info, int64_t n) {
    if (!c) return KHRR_ERR_INVALID_ARG;
    if (n < 0 || (n > 0 && !particle_cell_info) || (particle_acc && !cell_acc) || (particle_value && !cell_value))
        return c->fail(KHRR_ERR_INVALID_ARG, "bad gather arguments");
    return c->cuda(launch_apply(particle_acc, particle_value, cell_acc, cell_value,
                                reinterpret_cast<const int2*>(particle_cell_info), n, c->stream),
                   "gather");
}

khrr_status khrr_bin(khrr_ctx* c, const khrr_mesh* mesh, int* cell_id, int* id_in_cell, int* count, int* start,
                     int* start_ref, double* cell_mass) {
    if (!c) return KHRR_ERR_INVALID_ARG;
    if (!c->has_state) return c->fail(KHRR_ERR_STATE, "no state uploaded");
    MeshGeom g;
    int64_t C = 0;
    khrr_status st = check_mesh(c, mesh, &g, &C);
    if (st != KHRR_OK) return st;
    cudaStream_t s = c->stream;
    const size_t np = static_cast<size_t>(c->npad);
    if ((st = c->cuda(c->pci.ensure(np), "alloc")) != KHRR_OK) return st;
    if ((st = c->cuda(c->mtmp.ensure(2 * np), "alloc")) != KHRR_OK) return st;
    for (DevBuf<int>* b : {&c->mcount, &c->mstart})
        if ((st = c->cuda(b->ensure(static_cast<size_t>(C)), "alloc")) != KHRR_OK) return st;
    if ((st = c->cuda(c->maxpbc.ensure(static_cast<size_t>(scan_block_count(C))), "alloc")) != KHRR_OK) return st;
    if ((st = c->cuda(c->cell_mass.ensure(static_cast<size_t>(C)), "alloc")) != KHRR_OK) return st;
    cudaMemsetAsync(c->mcount.p, 0, static_cast<size_t>(C) * sizeof(int), s);
    cudaMemsetAsync(c->cell_mass.p, 0, static_cast<size_t>(C) * sizeof(double), s);
    // Every system's real bodies go to the one mesh (ghosts stay out).
    for (size_t k = 0; k < c->cnt.size(); ++k) {
        const int64_t o = c->poff[k];
        if ((st = c->cuda(launch_assign(c->pos.p + 3 * o, c->cnt[k], g, c->pci.p + o, c->mcount.p, 1, nullptr, 0,
                                        c->mass.p + o, c->cell_mass.p, s),
                          "assign")) != KHRR_OK)
            return st;
    }
    if ((st = c->cuda(c->mscan.ensure(static_cast<size_t>(scan_scratch_ints(C))), "alloc")) != KHRR_OK) return st;
    if ((st = c->cuda(launch_scan(c->mcount.p, false, C, c->maxpbc.p, c->mstart.p, false, c->mscan.p, s), "scan")) !=
        KHRR_OK)
        return st;
    c->mesh = g;
    c->ncells = C;
    c->has_bin = true;
    if (cell_id || id_in_cell) {
        if ((st = c->cuda(launch_deinterleave(c->pci.p, c->npad, c->mtmp.p, c->mtmp.p + np, s), "deinterleave")) !=
            KHRR_OK)
            return st;
        for (size_t k = 0; k < c->cnt.size() && st == KHRR_OK; ++k) {
            const size_t o = static_cast<size_t>(c->off[k]), q = static_cast<size_t>(c->poff[k]);
            const size_t m = static_cast<size_t>(c->cnt[k]) * sizeof(int);
            if (cell_id) st = c->cuda(cudaMemcpyAsync(cell_id + o, c->mtmp.p + q, m, cudaMemcpyDeviceToHost, s), "download");
            if (id_in_cell && st == KHRR_OK)
                st = c->cuda(cudaMemcpyAsync(id_in_cell + o, c->mtmp.p + np + q, m, cudaMemcpyDeviceToHost, s), "download");
        }
        if (st != KHRR_OK) return st;
    }
    const size_t cb = static_cast<size_t>(C) * sizeof(int);
    if (count && (st = c->cuda(cudaMemcpyAsync(count, c->mcount.p, cb, cudaMemcpyDeviceToHost, s), "download")) != KHRR_OK)
        return st;
    if (start && (st = c->cuda(cudaMemcpyAsync(start, c->mstart.p, cb, cudaMemcpyDeviceToHost, s), "download")) != KHRR_OK)
        return st;
    // The reference's start_id view is a function of maxPBC alone (the total
    // of all earlier 512-cell blocks): expanded on the host when asked for.
    std::vector<int> mp;
    if (start_ref) {
        mp.resize(static_cast<size_t>(scan_block_count(C)));
        if ((st = c->cuda(cudaMemcpyAsync(mp.data(), c->maxpbc.p, mp.size() * sizeof(int), cudaMemcpyDeviceToHost, s),
                          "download")) != KHRR_OK)
            return st;
    }
    if (cell_mass && (st = c->cuda(cudaMemcpyAsync(cell_mass, c->cell_mass.p, static_cast<size_t>(C) * sizeof(double),
                                                   cudaMemcpyDeviceToHost, s),
                                   "download")) != KHRR_OK)
        return st;
    if ((st = khrr_synchronize(c)) != KHRR_OK) return st;
    if (start_ref)
        for (int64_t cell = 0; cell < C; ++cell) start_ref[cell] = cell >= 512 ? mp[cell / 512 - 1] : 0;
    return KHRR_OK;
}

khrr_status khrr_bin_cell_phi(khrr_ctx* c, int reset, double* cell_phi) {
    if (!c) return KHRR_ERR_INVALID_ARG;
    if (!c->has_bin) return c->fail(KHRR_ERR_STATE, "no binned bodies (call khrr_bin first)");
    const size_t C = static_cast<size_t>(c->ncells);
    khrr_status st;
    cudaStream_t s = c->stream;
    if (reset || c->cell_phi_cells != c->ncells) {  // a new mesh starts from zero
        if ((st = c->cuda(c->cell_phi.ensure(C), "alloc")) != KHRR_OK) return st;
        cudaMemsetAsync(c->cell_phi.p, 0, C * sizeof(double), s);
        c->cell_phi_cells = c->ncells;
    }
    for (size_t k = 0; k < c->cnt.size(); ++k) {
        const int64_t o = c->poff[k];
        if ((st = c->cuda(launch_cell_phi(c->phi.p + o, c->pci.p + o, c->mcount.p, 1, c->cnt[k], c->cell_phi.p, s),
                          "cell phi")) != KHRR_OK)
            return st;
    }
    if (cell_phi &&
        (st = c->cuda(cudaMemcpyAsync(cell_phi, c->cell_phi.p, C * sizeof(double), cudaMemcpyDeviceToHost, s),
                      "download")) != KHRR_OK)
        return st;
    return khrr_synchronize(c);
}

khrr_status khrr_wave_solve(khrr_ctx* c, const khrr_wave_params* p, double tol, int max_iter, int check_every,
                            int cold, int* iters, double* resid, float* phi_out) {
    if (!c) return KHRR_ERR_INVALID_ARG;
    khrr_status st = check_wave(c, p);
    if (st != KHRR_OK) return st;
    if (!c->has_bin) return c->fail(KHRR_ERR_STATE, "no binned masses (call khrr_bin first)");
    const int64_t nx = p->nx;
    const int64_t C = nx * nx * nx;
    if (C != c->ncells) return c->fail(KHRR_ERR_INVALID_ARG, "nx^3 differs from the binned mesh");
    if (max_iter < 1 || check_every < 1) return c->fail(KHRR_ERR_INVALID_ARG, "max_iter and check_every must be >= 1");
    cudaStream_t s = c->stream;
    const size_t cz = static_cast<size_t>(C);
    if (c->wave_nx != p->nx) {
        for (auto& kv : c->wave_graphs) {
            cudaGraphExecDestroy(kv.second.exec);
            cudaGraphDestroy(kv.second.graph);
        }
        c->wave_graphs.clear();
        if ((st = c->cuda(c->wave_phi.ensure(3 * cz), "alloc")) != KHRR_OK) return st;
        if ((st = c->cuda(c->wave_mass.ensure(cz), "alloc")) != KHRR_OK) return st;
        if ((st = c->cuda(c->wave_tab.ensure(3 * static_cast<size_t>(nx)), "alloc")) != KHRR_OK) return st;
        if ((st = c->cuda(c->wave_resid.ensure(2), "alloc")) != KHRR_OK) return st;
        c->wave_nx = p->nx;
        c->wave_warm = false;
    }
    std::vector<float> tab;
    sponge_tables(p, tab);
    if ((st = c->cuda(cudaMemcpyAsync(c->wave_tab.p, tab.data(), tab.size() * sizeof(float), cudaMemcpyHostToDevice, s),
                      "upload")) != KHRR_OK)
        return st;
    if ((st = c->cuda(launch_to_float(c->cell_mass.p, c->wave_mass.p, C, s), "mass to float")) != KHRR_OK) return st;
    if (cold || !c->wave_warm) {
        cudaMemsetAsync(c->wave_phi.p, 0, 3 * cz * sizeof(float), s);
        c->wave_rot = 0;
    }
    const WaveF32 w = wave_f32(p, c->wave_tab.p);
    // Graph of one chunk of `check_every` iterations starting at a rotation;
    // the last iteration of the chunk reduces the residual.
    auto chunk_graph = [&](int k, int rot, StepGraph** out) -> khrr_status {
        const auto key = std::make_pair(k, rot);
        auto it = c->wave_graphs.find(key);
        if (it != c->wave_graphs.end()) {
            *out = &it->second;
            return KHRR_OK;
        }
        StepGraph g{};
        khrr_status e = c->cuda(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal), "begin capture");
        if (e != KHRR_OK) return e;
        cudaMemsetAsync(c->wave_resid.p, 0, 2 * sizeof(double), s);
        int r = rot;
        for (int i = 0; i < k; ++i) {
            float* old = c->wave_phi.p + static_cast<size_t>(r) * cz;
            float* cur = c->wave_phi.p + static_cast<size_t>((r + 1) % 3) * cz;
            float* nxt = c->wave_phi.p + static_cast<size_t>((r + 2) % 3) * cz;
            launch_wave_f32(nxt, cur, old, c->wave_mass.p, w, i == k - 1 ? c->wave_resid.p : nullptr, s);
            r = (r + 1) % 3;
        }
        cudaGraph_t graph = nullptr;
        if ((e = c->cuda(cudaStreamEndCapture(s, &graph), "end capture")) != KHRR_OK) return e;
        g.graph = graph;
        if ((e = c->cuda(cudaGraphInstantiate(&g.exec, graph, 0), "graph instantiate")) != KHRR_OK) {
            cudaGraphDestroy(graph);
            return e;
        }
        *out = &c->wave_graphs.emplace(key, g).first->second;
        return KHRR_OK;
    };
    // Tables and constants are baked into the graphs: rebuild them per call.
    for (auto& kv : c->wave_graphs) {
        cudaGraphExecDestroy(kv.second.exec);
        cudaGraphDestroy(kv.second.graph);
    }
    c->wave_graphs.clear();
    int done = 0;
    double rel = INFINITY;
    while (done < max_iter) {
        const int k = std::min(check_every, max_iter - done);
        StepGraph* g = nullptr;
        if ((st = chunk_graph(k, c->wave_rot, &g)) != KHRR_OK) return st;
        if ((st = c->cuda(cudaGraphLaunch(g->exec, s), "wave graph")) != KHRR_OK) return st;
        double r2[2];
        if ((st = c->cuda(cudaMemcpyAsync(r2, c->wave_resid.p, sizeof r2, cudaMemcpyDeviceToHost, s), "download")) !=
            KHRR_OK)
            return st;
        if ((st = c->cuda(cudaStreamSynchronize(s), "wave sync")) != KHRR_OK) return st;
        done += k;
        c->wave_rot = (c->wave_rot + k) % 3;
        rel = r2[1] > 0.0 ? std::sqrt(r2[0] / r2[1]) : (r2[0] > 0.0 ? INFINITY : 0.0);
        if (rel < tol) break;
    }
    c->wave_warm = true;
    if (iters) *iters = done;
    if (resid) *resid = rel;
    if (phi_out) {
        const float* cur = c->wave_phi.p + static_cast<size_t>((c->wave_rot + 1) % 3) * cz;
        if ((st = c->cuda(cudaMemcpyAsync(phi_out, cur, cz * sizeof(float), cudaMemcpyDeviceToHost, s), "download")) !=
            KHRR_OK)
            return st;
        if ((st = c->cuda(cudaStreamSynchronize(s), "sync")) != KHRR_OK) return st;
    }
    return KHRR_OK;
}

}  // extern "C"
