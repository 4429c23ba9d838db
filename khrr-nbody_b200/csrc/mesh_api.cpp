// C ABI of the p2mesh path: kernel-level entry points (the reference's
// pointers and layouts) and the context-level pipeline khrr_bin /
// khrr_wave_solve.
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>
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
        g->rcs[k] = 1.0 / m->cell[k];  // IEEE division: the correctly rounded reciprocal
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

// cuTensorMapEncodeTiled through the runtime's driver entry point (the
// library does not link libcuda directly).
PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
    static const PFN_cuTensorMapEncodeTiled_v12000 fn = [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            p = nullptr;
        return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    }();
    return fn;
}

// One nx^3 float field as a 3-D tensor with bx x by x 1 boxes (the planes the
// tensor-copy stencils stream); outside coordinates read as zero.
bool make_box_map(CUtensorMap* m, const float* base, int nx, unsigned bx, unsigned by) {
    const auto enc = tensor_map_encoder();
    if (!enc) return false;
    const cuuint64_t n = static_cast<cuuint64_t>(nx);
    const cuuint64_t dims[3] = {n, n, n};
    const cuuint64_t strides[2] = {n * 4, n * n * 4};
    const cuuint32_t box[3] = {bx, by, 1};
    const cuuint32_t elem[3] = {1, 1, 1};
    return enc(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<float*>(base), dims, strides, box, elem,
               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// Maps of the four ring buffers and the mass for the tensor-copy stencils,
// made only when KHRR_WAVE_TMA selects one (read at every solve set-up):
// 1 = the warp-specialised one-step kernel, 2 = the two-step kernel for
// pairs of iterations; unset or 0 = the cache-fed one-step kernel, which
// measured fastest on the 128^3 mesh (10.4 us per iteration against 16.4 and
// 13.1) and within noise of both on 256^3.  The tensor-copy kernels need
// 16-byte row strides (nx % 4 == 0) and a mesh at least one box wide.
void make_wave_maps(WaveMaps* w, float* ring, const float* mass, int nx, unsigned* sync) {
    w->ok = false;
    // The shared-memory-resident stencil (nx = 128) unless KHRR_WAVE_RESIDENT=0.
    const char* r = std::getenv("KHRR_WAVE_RESIDENT");
    w->sync = sync;
    w->resident = sync && !(r && std::atoi(r) == 0) && wave_resident_available(nx);
    const char* e = std::getenv("KHRR_WAVE_TMA");
    const int mode = e ? std::atoi(e) : 0;
    if ((mode != 1 && mode != 2) || nx % 4 != 0 || nx < 40) return;
    const size_t cz = static_cast<size_t>(nx) * nx * nx;
    for (int b = 0; b < 4; ++b)
        if (!make_box_map(&w->ring[b], ring + b * cz, nx, 40, 12) ||
            !make_box_map(&w->halo[b], ring + b * cz, nx, 40, 10) ||
            !make_box_map(&w->tile[b], ring + b * cz, nx, 32, 8))
            return;
    if (!make_box_map(&w->mass, mass, nx, 40, 12) || !make_box_map(&w->tile_mass, mass, nx, 32, 8)) return;
    w->two_step = mode == 2;
    w->ok = true;
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
    khrr::NvtxRange nvtx_range("khrr_bin");
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
    if ((st = c->call_start()) != KHRR_OK) return st;
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
    if ((st = c->call_stop()) != KHRR_OK) return st;
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
    khrr::NvtxRange nvtx_range("khrr_bin_cell_phi");
    if (!c) return KHRR_ERR_INVALID_ARG;
    if (!c->has_bin) return c->fail(KHRR_ERR_STATE, "no binned bodies (call khrr_bin first)");
    const size_t C = static_cast<size_t>(c->ncells);
    khrr_status st;
    cudaStream_t s = c->stream;
    if ((st = c->call_start()) != KHRR_OK) return st;
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
    if ((st = c->call_stop()) != KHRR_OK) return st;
    if (cell_phi &&
        (st = c->cuda(cudaMemcpyAsync(cell_phi, c->cell_phi.p, C * sizeof(double), cudaMemcpyDeviceToHost, s),
                      "download")) != KHRR_OK)
        return st;
    return khrr_synchronize(c);
}

khrr_status khrr_wave_solve(khrr_ctx* c, const khrr_wave_params* p, double tol, int max_iter, int check_every,
                            int cold, int* iters, double* resid, float* phi_out) {
    khrr::NvtxRange nvtx_range("khrr_wave_solve");
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
        if ((st = c->cuda(c->wave_phi.ensure(4 * cz), "alloc")) != KHRR_OK) return st;
        if ((st = c->cuda(c->wave_mass.ensure(cz), "alloc")) != KHRR_OK) return st;
        if ((st = c->cuda(c->wave_tab.ensure(3 * static_cast<size_t>(nx)), "alloc")) != KHRR_OK) return st;
        if ((st = c->cuda(c->wave_resid.ensure(2), "alloc")) != KHRR_OK) return st;
        if ((st = c->cuda(c->wave_sync.ensure(static_cast<size_t>(nx) + 1), "alloc")) != KHRR_OK) return st;
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
        cudaMemsetAsync(c->wave_phi.p, 0, 4 * cz * sizeof(float), s);
        c->wave_rot = kRingStart;
    }
    const WaveF32 w = wave_f32(p, c->wave_tab.p);
    make_wave_maps(&c->wave_maps, c->wave_phi.p, c->wave_mass.p, p->nx, c->wave_sync.p);
    // Graph of one chunk of `check_every` iterations starting at a ring state;
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
        enqueue_wave_f32(c->wave_phi.p, C, c->wave_mass.p, w, k, rot, c->wave_resid.p, s, &c->wave_maps,
                         c->errflag.p);
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
        if ((st = c->check_device_flag()) != KHRR_OK) return st;
        done += k;
        c->wave_rot = ring_after_f32(c->wave_rot, k);
        rel = r2[1] > 0.0 ? std::sqrt(r2[0] / r2[1]) : (r2[0] > 0.0 ? INFINITY : 0.0);
        if (rel < tol) break;
    }
    c->wave_warm = true;
    if (iters) *iters = done;
    if (resid) *resid = rel;
    if (phi_out) {
        const float* cur = c->wave_phi.p + static_cast<size_t>(c->wave_rot % 4) * cz;
        if ((st = c->cuda(cudaMemcpyAsync(phi_out, cur, cz * sizeof(float), cudaMemcpyDeviceToHost, s), "download")) !=
            KHRR_OK)
            return st;
        if ((st = c->cuda(cudaStreamSynchronize(s), "sync")) != KHRR_OK) return st;
    }
    return KHRR_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Cloud-in-cell, the counting sort, and the mesh-force solver.
// ---------------------------------------------------------------------------
namespace {

khrr_status check_cubic(khrr_ctx* c, const khrr_mesh* m, MeshGeom* g, int64_t* ncells) {
    khrr_status st = check_mesh(c, m, g, ncells);
    if (st != KHRR_OK) return st;
    if (m->grid[0] != m->grid[1] || m->grid[1] != m->grid[2])
        return c->fail(KHRR_ERR_INVALID_ARG, "cloud-in-cell needs a cubic mesh");
    return KHRR_OK;
}

}  // namespace

khrr_status khrr_probe_resident_wave(khrr_ctx* c, double seconds) {
    khrr::NvtxRange nvtx_range("khrr_probe_resident_wave");
    if (!c) return KHRR_ERR_INVALID_ARG;
    if (!(seconds > 0.0) || seconds > 10.0) return c->fail(KHRR_ERR_INVALID_ARG, "seconds must be in (0, 10]");
    constexpr int nx = 128;
    if (!wave_resident_available(nx))
        return c->fail(KHRR_ERR_UNSUPPORTED, "the resident 128^3 stencil does not run on this device");
    khrr_status st = c->check_device_flag();  // report (and clear) anything raised earlier first
    if (st != KHRR_OK) return st;
    // A zero field on scratch buffers of the probe's own (the context's
    // solver state is not touched), four iterations, brick 0 withholding
    // its counter.
    const size_t cz = static_cast<size_t>(nx) * nx * nx;
    DevBuf<float> ring, mass, tab;
    DevBuf<unsigned> sync;
    if ((st = c->cuda(ring.ensure(4 * cz), "alloc")) != KHRR_OK || (st = c->cuda(mass.ensure(cz), "alloc")) != KHRR_OK ||
        (st = c->cuda(tab.ensure(3 * nx), "alloc")) != KHRR_OK || (st = c->cuda(sync.ensure(nx + 1), "alloc")) != KHRR_OK)
        return st;
    cudaStream_t s = c->stream;
    cudaMemsetAsync(ring.p, 0, 4 * cz * sizeof(float), s);
    cudaMemsetAsync(mass.p, 0, cz * sizeof(float), s);
    cudaMemsetAsync(tab.p, 0, 3 * nx * sizeof(float), s);
    WaveF32 w{};
    w.nx = nx;
    w.sx = tab.p;
    w.sy = tab.p + nx;
    w.sz = tab.p + 2 * nx;
    if ((st = c->cuda(launch_wave_resident(ring.p, static_cast<int64_t>(cz), mass.p, w, 4, 1, nullptr, sync.p,
                                           c->errflag.p, s, static_cast<unsigned long long>(seconds * 1e9), 0),
                      "resident wave probe")) != KHRR_OK)
        return st;
    return c->check_device_flag();  // synchronises before the scratch is freed
}

khrr_status khrr_cic_deposit(khrr_ctx* c, const double* pos, const double* mass, int64_t n, const khrr_mesh* mesh,
                             double* cell_mass) {
    khrr::NvtxRange nvtx_range("khrr_cic_deposit");
    if (!c) return KHRR_ERR_INVALID_ARG;
    MeshGeom g;
    int64_t C = 0;
    khrr_status st = check_cubic(c, mesh, &g, &C);
    if (st != KHRR_OK) return st;
    if (n < 0 || (n > 0 && (!pos || !mass || !cell_mass))) return c->fail(KHRR_ERR_INVALID_ARG, "bad deposit arguments");
    return c->cuda(launch_cic_deposit(pos, mass, n, g, cell_mass, c->stream), "cic deposit");
}

khrr_status khrr_cic_gather(khrr_ctx* c, const double* pos, int64_t n, const khrr_mesh* mesh, const double* cell_acc,
                            const double* cell_value, double* particle_acc, double* particle_value) {
    khrr::NvtxRange nvtx_range("khrr_cic_gather");
    if (!c) return KHRR_ERR_INVALID_ARG;
    MeshGeom g;
    int64_t C = 0;
    khrr_status st = check_cubic(c, mesh, &g, &C);
    if (st != KHRR_OK) return st;
    if (n < 0 || (n > 0 && !pos) || (particle_acc && !cell_acc) || (particle_value && !cell_value))
        return c->fail(KHRR_ERR_INVALID_ARG, "bad gather arguments");
    return c->cuda(launch_cic_gather(pos, n, g, cell_acc, cell_value, particle_acc, particle_value, c->stream),
                   "cic gather");
}

khrr_status khrr_sort_by_cell(khrr_ctx* c, int* order) {
    khrr::NvtxRange nvtx_range("khrr_sort_by_cell");
    if (!c) return KHRR_ERR_INVALID_ARG;
    if (!c->has_bin) return c->fail(KHRR_ERR_STATE, "no binned bodies (call khrr_bin first)");
    if (c->n > 0x7fffffffLL) return c->fail(KHRR_ERR_INVALID_ARG, "more bodies than int32 indices");
    khrr_status st;
    if ((st = c->cuda(c->morder.ensure(static_cast<size_t>(c->n)), "alloc")) != KHRR_OK) return st;
    if ((st = c->call_start()) != KHRR_OK) return st;
    for (size_t k = 0; k < c->cnt.size(); ++k)
        if ((st = c->cuda(launch_scatter_order(c->pci.p + c->poff[k], c->mstart.p, c->cnt[k],
                                               static_cast<int>(c->off[k]), c->morder.p, c->stream),
                          "scatter")) != KHRR_OK)
            return st;
    if ((st = c->call_stop()) != KHRR_OK) return st;
    if (order && (st = c->cuda(cudaMemcpyAsync(order, c->morder.p, static_cast<size_t>(c->n) * sizeof(int),
                                               cudaMemcpyDeviceToHost, c->stream),
                               "download")) != KHRR_OK)
        return st;
    return khrr_synchronize(c);
}

khrr_status khrr_set_mesh_solver(khrr_ctx* c, const khrr_mesh_solver* p) {
    khrr::NvtxRange nvtx_range("khrr_set_mesh_solver");
    if (!c) return KHRR_ERR_INVALID_ARG;
    MeshSolver& M = c->msolver;
    M.drop_graphs();
    if (!p) {
        M.on = false;
        return KHRR_OK;
    }
    khrr_status st = check_wave(c, &p->wave);
    if (st != KHRR_OK) return st;
    if (p->assign != KHRR_ASSIGN_NGP && p->assign != KHRR_ASSIGN_CIC)
        return c->fail(KHRR_ERR_INVALID_ARG, "assign must be KHRR_ASSIGN_NGP or KHRR_ASSIGN_CIC");
    if (p->iters_per_step < 1 || p->setup_iters < 0)
        return c->fail(KHRR_ERR_INVALID_ARG, "iters_per_step must be >= 1 and setup_iters >= 0");
    const int nx = p->wave.nx;
    const double L = 0.5 * nx * p->wave.dx;  // _domain_l = 0.5 * _nx * _dx (nbody.cu:1136)
    khrr_mesh m{{-L, -L, -L}, {p->wave.dx, p->wave.dx, p->wave.dx}, {nx, nx, nx}};
    MeshGeom g;
    int64_t C = 0;
    if ((st = check_mesh(c, &m, &g, &C)) != KHRR_OK) return st;
    const size_t cz = static_cast<size_t>(C);
    if ((st = c->cuda(M.cell_mass.ensure(cz), "alloc")) != KHRR_OK) return st;
    if ((st = c->cuda(M.cell_acc.ensure(3 * cz), "alloc")) != KHRR_OK) return st;
    if (p->fp64) {
        if ((st = c->cuda(M.phi64.ensure(4 * cz), "alloc")) != KHRR_OK) return st;
    } else {
        if ((st = c->cuda(M.phi32.ensure(4 * cz), "alloc")) != KHRR_OK) return st;
        if ((st = c->cuda(M.mass32.ensure(cz), "alloc")) != KHRR_OK) return st;
        if ((st = c->cuda(M.tab.ensure(3 * static_cast<size_t>(nx)), "alloc")) != KHRR_OK) return st;
        std::vector<float> tab;
        sponge_tables(&p->wave, tab);
        if ((st = c->cuda(cudaMemcpyAsync(M.tab.p, tab.data(), tab.size() * sizeof(float), cudaMemcpyHostToDevice,
                                          c->stream),
                          "upload")) != KHRR_OK)
            return st;
        if ((st = c->cuda(M.sync.ensure(static_cast<size_t>(nx) + 1), "alloc")) != KHRR_OK) return st;
        make_wave_maps(&M.maps, M.phi32.p, M.mass32.p, nx, M.sync.p);
    }
    M.cfg = *p;
    M.geom = g;
    M.cells = C;
    M.rot = kRingStart;
    M.on = true;
    // The field starts at zero, as the reference's freshly allocated arrays.
    if (p->fp64) cudaMemsetAsync(M.phi64.p, 0, 4 * cz * sizeof(double), c->stream);
    else cudaMemsetAsync(M.phi32.p, 0, 4 * cz * sizeof(float), c->stream);
    return khrr_synchronize(c);
}

khrr_status khrr_mesh_solver_phi(khrr_ctx* c, double* cell_phi) {
    if (!c || !cell_phi) return KHRR_ERR_INVALID_ARG;
    MeshSolver& M = c->msolver;
    if (!M.on) return c->fail(KHRR_ERR_STATE, "no mesh solver set");
    const size_t cz = static_cast<size_t>(M.cells);
    const size_t cur = static_cast<size_t>(M.rot % 4) * cz;
    khrr_status st;
    if (M.cfg.fp64) {
        st = c->cuda(cudaMemcpyAsync(cell_phi, M.phi64.p + cur, cz * sizeof(double), cudaMemcpyDeviceToHost, c->stream),
                     "download");
        if (st != KHRR_OK) return st;
        return khrr_synchronize(c);
    }
    std::vector<float> f(cz);
    if ((st = c->cuda(cudaMemcpyAsync(f.data(), M.phi32.p + cur, cz * sizeof(float), cudaMemcpyDeviceToHost, c->stream),
                      "download")) != KHRR_OK)
        return st;
    if ((st = khrr_synchronize(c)) != KHRR_OK) return st;
    for (size_t i = 0; i < cz; ++i) cell_phi[i] = f[i];
    return KHRR_OK;
}

// Per-body buffers of the solver, sized for the uploaded layout.
khrr_status khrr_ctx::mesh_ensure_layout() {
    MeshSolver& M = msolver;
    // All bodies share the one mesh: several independent systems would
    // attract each other through it.
    if (cnt.size() != 1) return fail(KHRR_ERR_INVALID_ARG, "the mesh solver runs one system (got %zu)", cnt.size());
    if (M.layout_poff == poff && M.layout_cnt == cnt && M.ns.p) return KHRR_OK;
    const size_t np = static_cast<size_t>(npad);
    khrr_status st;
    if ((st = cuda(M.pci.ensure(np), "alloc")) != KHRR_OK) return st;
    if ((st = cuda(M.part.ensure(np), "alloc")) != KHRR_OK) return st;
    if ((st = cuda(M.ns.ensure(np), "alloc")) != KHRR_OK) return st;
    std::vector<unsigned char> ns(np, 0);
    for (size_t k = 0; k < cnt.size(); ++k)
        std::fill(ns.begin() + poff[k], ns.begin() + poff[k] + cnt[k], static_cast<unsigned char>(1));
    if ((st = cuda(cudaMemcpyAsync(M.ns.p, ns.data(), np, cudaMemcpyHostToDevice, stream), "upload")) != KHRR_OK)
        return st;
    cudaMemsetAsync(M.part.p, 0, np * sizeof(double4), stream);
    if ((st = cuda(cudaStreamSynchronize(stream), "sync")) != KHRR_OK) return st;  // ns outlives the call
    M.layout_poff = poff;
    M.layout_cnt = cnt;
    M.drop_graphs();
    return KHRR_OK;
}

// calc_acceleration_by_grid (nbody.cu:183-285) at positions x: deposit, `iters`
// stencil iterations from ring state rot0, gradient, gather into M.part.
khrr_status khrr_ctx::mesh_enqueue_force(const double* x, int iters, int rot0) {
    MeshSolver& M = msolver;
    const khrr_mesh_solver& P = M.cfg;
    const size_t cz = static_cast<size_t>(M.cells);
    const bool cic = P.assign == KHRR_ASSIGN_CIC;
    cudaStream_t s = stream;
    khrr_status st;
    if ((st = cuda(cudaMemsetAsync(M.cell_mass.p, 0, cz * sizeof(double), s), "memset")) != KHRR_OK) return st;
    for (size_t k = 0; k < cnt.size(); ++k) {
        const int64_t o = poff[k];
        cudaError_t e = cic ? launch_cic_deposit(x + 3 * o, mass.p + o, cnt[k], M.geom, M.cell_mass.p, s)
                            : launch_assign_cells(x + 3 * o, cnt[k], M.geom, M.pci.p + o, mass.p + o, M.cell_mass.p, s);
        if ((st = cuda(e, "deposit")) != KHRR_OK) return st;
    }
    const int nx = P.wave.nx;
    int r = rot0;
    if (P.fp64) {
        const WaveConsts w = wave_consts(&P.wave);
        for (int i = 0; i < iters; ++i, r = ring_step1(r)) {
            int f0, f1;
            ring_free(r, f0, f1);
            double* old = M.phi64.p + static_cast<size_t>(r / 4) * cz;
            double* cur = M.phi64.p + static_cast<size_t>(r % 4) * cz;
            double* nxt = M.phi64.p + static_cast<size_t>(f0) * cz;
            if ((st = cuda(launch_wave_f64(nxt, cur, old, M.cell_mass.p, w, s), "wave")) != KHRR_OK) return st;
        }
        const double* cur = M.phi64.p + static_cast<size_t>(r % 4) * cz;
        if ((st = cuda(launch_acc_field(M.cell_acc.p, nullptr, cur, nx, P.wave.dx, s), "acc_field")) != KHRR_OK)
            return st;
        for (size_t k = 0; k < cnt.size(); ++k) {
            const int64_t o = poff[k];
            if ((st = cuda(launch_mesh_gather(x + 3 * o, M.pci.p + o, cnt[k], M.geom, cic, M.cell_acc.p, nullptr, cur,
                                              M.part.p + o, s),
                           "gather")) != KHRR_OK)
                return st;
        }
        return KHRR_OK;
    }
    if ((st = cuda(launch_to_float(M.cell_mass.p, M.mass32.p, M.cells, s), "mass to float")) != KHRR_OK) return st;
    const WaveF32 w = wave_f32(&P.wave, M.tab.p);
    if ((st = cuda(enqueue_wave_f32(M.phi32.p, M.cells, M.mass32.p, w, iters, r, nullptr, s, &M.maps, errflag.p),
                   "wave")) != KHRR_OK)
        return st;
    r = ring_after_f32(r, iters);
    const float* cur = M.phi32.p + static_cast<size_t>(r % 4) * cz;
    if ((st = cuda(launch_acc_field_f32(M.cell_acc.p, cur, nx, P.wave.dx, s), "acc_field")) != KHRR_OK) return st;
    for (size_t k = 0; k < cnt.size(); ++k) {
        const int64_t o = poff[k];
        if ((st = cuda(launch_mesh_gather(x + 3 * o, M.pci.p + o, cnt[k], M.geom, cic, M.cell_acc.p, cur, nullptr,
                                          M.part.p + o, s),
                       "gather")) != KHRR_OK)
            return st;
    }
    return KHRR_OK;
}

namespace {

StepArgs mesh_step_args(khrr_ctx* c, double dt) {
    StepArgs a{};
    a.pos = c->pos.p;
    a.vel = c->vel.p;
    a.acc = c->acc.p;
    a.post = c->post.p;
    a.velt = c->velt.p;
    a.acct = c->acct.p;
    a.mass = c->mass.p;
    a.phi = c->phi.p;
    a.shadow = c->shadow();
    a.part = c->msolver.part.p;
    a.npad = c->npad;
    a.nsplit = c->msolver.ns.p;
    a.n = c->npad;
    a.dt = dt;
    a.field = c->field;
    return a;
}

}  // namespace

// Setup evaluation (nbody.cu:1449-1472): the field from zero, setup_iters
// iterations, at the current positions.
khrr_status khrr_ctx::mesh_forces(int flags) {
    MeshSolver& M = msolver;
    if (!M.on) return fail(KHRR_ERR_STATE, "KHRR_MESH without a mesh solver (khrr_set_mesh_solver)");
    khrr_status st = mesh_ensure_layout();
    if (st != KHRR_OK) return st;
    const size_t cz = static_cast<size_t>(M.cells);
    if (M.cfg.fp64) cudaMemsetAsync(M.phi64.p, 0, 4 * cz * sizeof(double), stream);
    else cudaMemsetAsync(M.phi32.p, 0, 4 * cz * sizeof(float), stream);
    if ((st = mesh_enqueue_force(pos.p, M.cfg.setup_iters, kRingStart)) != KHRR_OK) return st;
    M.rot = M.cfg.fp64 ? ring_after_f64(kRingStart, M.cfg.setup_iters) : ring_after_f32(kRingStart, M.cfg.setup_iters);
    StepArgs sa = mesh_step_args(this, 0.0);
    sa.want_phi = (flags & KHRR_PHI) ? 1 : 0;
    if ((st = cuda(launch_collect(sa, (flags & KHRR_ACC) != 0, false, stream), "collect")) != KHRR_OK) return st;
    predicted = false;
    return KHRR_OK;
}

// Steps in Wave mode (nbody.cu:1521-1589): predictor, the mesh force at the
// predicted positions (acct_ zeroed first, nbody.cu:1542, so there is no
// accumulation), corrector fused with the next predictor; one graph per
// (dt, ring rotation, phi).
khrr_status khrr_ctx::mesh_step(double dt, int nsteps, int flags) {
    MeshSolver& M = msolver;
    if (!M.on) return fail(KHRR_ERR_STATE, "KHRR_MESH without a mesh solver (khrr_set_mesh_solver)");
    khrr_status st = mesh_ensure_layout();
    if (st != KHRR_OK) return st;
    if (!predicted || pred_dt != dt) {
        if ((st = cuda(launch_predictor(mesh_step_args(this, dt), stream), "predictor")) != KHRR_OK) return st;
    }
    const bool phi_last = (flags & KHRR_PHI) != 0;
    const int iters = M.cfg.iters_per_step;
    uint64_t dt_bits;
    std::memcpy(&dt_bits, &dt, sizeof dt_bits);
    for (int k = 0; k < nsteps; ++k) {
        const bool phi_now = phi_last && k == nsteps - 1;
        const auto key = std::make_tuple(dt_bits, M.rot, phi_now);
        auto it = M.graphs.find(key);
        if (it == M.graphs.end()) {
            StepGraph g{};
            if ((st = cuda(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal), "begin capture")) !=
                KHRR_OK)
                return st;
            khrr_status est = mesh_enqueue_force(post.p, iters, M.rot);
            if (est == KHRR_OK) {
                StepArgs sa = mesh_step_args(this, dt);
                sa.want_phi = phi_now ? 1 : 0;
                sa.predict_next = 1;
                est = cuda(launch_corrector(sa, stream), "corrector");
            }
            cudaGraph_t graph = nullptr;
            cudaError_t ce = cudaStreamEndCapture(stream, &graph);
            if (est != KHRR_OK) {
                if (graph) cudaGraphDestroy(graph);
                return est;
            }
            if ((st = cuda(ce, "end capture")) != KHRR_OK) return st;
            g.graph = graph;
            if ((st = cuda(cudaGraphInstantiate(&g.exec, graph, 0), "graph instantiate")) != KHRR_OK) {
                cudaGraphDestroy(graph);
                return st;
            }
            it = M.graphs.emplace(key, g).first;
        }
        if ((st = cuda(cudaGraphLaunch(it->second.exec, stream), "graph launch")) != KHRR_OK) return st;
        M.rot = M.cfg.fp64 ? ring_after_f64(M.rot, iters) : ring_after_f32(M.rot, iters);
    }
    predicted = true;
    pred_dt = dt;
    return KHRR_OK;
}
