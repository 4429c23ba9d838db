// Host-side context of libkhrr (the object behind the opaque khrr_ctx*).
#pragma once

#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include <cstdint>
#include <map>
#include <string>
#include <tuple>
#include <utility>
#include <vector>

#include "khrr.h"
#include "khrr_internal.h"

namespace khrr {

// An NVTX range over one library call, shown by Nsight Systems as a named
// phase (header-only NVTX v3; without a tool attached it costs a few ns).
struct NvtxRange {
    explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
    NvtxRange(const NvtxRange&) = delete;
    NvtxRange& operator=(const NvtxRange&) = delete;
};

// Grow-only device allocation.
template <class T>
struct DevBuf {
    T* p = nullptr;
    size_t n = 0;
    DevBuf() = default;
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    ~DevBuf() { release(); }
    cudaError_t ensure(size_t count) {
        if (count <= n && p) return cudaSuccess;
        release();
        cudaError_t e = cudaMalloc(reinterpret_cast<void**>(&p), (count ? count : 1) * sizeof(T));
        if (e != cudaSuccess) {
            p = nullptr;
            n = 0;
            return e;
        }
        n = count;
        return cudaSuccess;
    }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
    }
};

// The force-pass work queue for one layout of systems and one kernel shape.
struct ForcePlan {
    bool valid = false;
    int threads = 0, ipt = 0, jt = 0, split_req = -1, ctas = 0;
    std::vector<WorkItem> items;
    std::vector<int> sys_item_begin;  // plain plans: items of system k
    std::vector<int> sys_split;       // j chunks per system
    int nslots = 1;
    DevBuf<WorkItem> d_items;
    DevBuf<unsigned char> d_nsplit;
    // The symmetric pair kernel's queue (pair plans; FP64 plans with f64_pair).
    bool pair = false;
    bool f64_pair = false;  // FP64 plan: the symmetric FP64 kernel on pair_items
    std::vector<PairItem> pair_items;
    DevBuf<PairItem> d_pair_items;
    ForcePlan() = default;
    ForcePlan(const ForcePlan&) = delete;
    ForcePlan& operator=(const ForcePlan&) = delete;
};

void plan_force_items(const std::vector<int64_t>& poff, const std::vector<int64_t>& cnt, int itile,
                      int jt, int ctas, int forced_split, bool plain, ForcePlan& out);
// The symmetric pair kernel's blocks: per system the padded indices
// P_k = b_0 < b_1 < ... < b_nb = P_{k+1}, each block at most kPairBlock
// bodies starting at a multiple of kPad.
using PairBlocks = std::vector<std::vector<int64_t>>;
// 1024-body blocks over each system's padded range (the last may be shorter).
PairBlocks pair_blocks_fixed(const std::vector<int64_t>& poff);
// Runs of 128-body tiles of one mass (tile_mass[tile]), cut at 1024 bodies.
PairBlocks pair_blocks_by_mass(const std::vector<int64_t>& poff, const std::vector<float>& tile_mass);
// The pair kernel's items: block rows cut into chunks of `chunk` blocks (0 =
// chosen from the CTA count), costliest first.
void plan_pair_items(const PairBlocks& blocks, const std::vector<int64_t>& cnt, int ctas, int chunk,
                     ForcePlan& out);

// Force paths of the state API: the batched FP32 kernels (pair or one-sided,
// per the tuning), the plain one-launch-per-system FP32 baseline (KHRR_PLAIN)
// and the FP64 direct sum (KHRR_FP64).
enum ForceMode { kModeBatched = 0, kModePlain = 1, kModeF64 = 2 };

struct StepGraph {
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    cudaGraphNode_t ev0 = nullptr, ev1 = nullptr;  // event-record nodes around the force pass
};

// The mesh-force solver (khrr_set_mesh_solver): its mesh, field ring and
// per-body gather slot, and the step graphs per (dt, ring state, phi).
struct MeshSolver {
    bool on = false;
    khrr_mesh_solver cfg{};
    MeshGeom geom{};
    int64_t cells = 0;
    DevBuf<double> cell_mass, phi64, cell_acc;  // C, 4 C (field ring), 3 C
    DevBuf<float> mass32, phi32, tab;           // C, 4 C (field ring), 3 nx
    DevBuf<int2> pci;                           // npad
    DevBuf<double4> part;                       // npad: {acc, -phi} per body
    WaveMaps maps;                              // tensor maps of phi32 / mass32
    DevBuf<unsigned> sync;                      // nx + 1 plane counters of the resident stencil
    DevBuf<unsigned char> ns;                   // npad: 1 for real bodies, 0 for ghosts
    std::vector<int64_t> layout_poff, layout_cnt;  // the layout pci/part/ns were sized for
    int rot = kRingStart;                       // ring state: 4 * (phi^{n-1} buffer) + phi^n buffer
    std::map<std::tuple<uint64_t, int, bool>, StepGraph> graphs;
    void drop_graphs() {
        for (auto& kv : graphs) {
            if (kv.second.exec) cudaGraphExecDestroy(kv.second.exec);
            if (kv.second.graph) cudaGraphDestroy(kv.second.graph);
        }
        graphs.clear();
    }
};

}  // namespace khrr

struct khrr_ctx {
    int device = 0;
    int sm_count = 0;
    cudaStream_t own = nullptr, stream = nullptr;
    std::string err;

    // State layout.
    bool has_state = false;
    int64_t n = 0, npad = 0;
    std::vector<int64_t> off, poff, cnt;  // real offsets, padded offsets, counts per system
    khrr::DevBuf<double> pos, vel, acc, post, velt, acct, mass, eps2, phi;
    khrr::DevBuf<float> shadow_buf;  // SoA FP32 shadow, 5 x npad
    khrr::DevBuf<double4> part;
    khrr::DevBuf<unsigned long long> fx;  // the pair kernel's fixed-point sums, kFxComps x npad
    khrr::DevBuf<khrr::FxScale> fx_scale; // their scale per 128-body tile
    std::vector<khrr::FxScale> fx_scales; // host copy (kept alive until the upload's copies complete)
    khrr::DevBuf<unsigned> queue, errflag;
    khrr::DevBuf<double> cons_blocks, scratch;
    bool uniform = false;
    float h_uniform = 0.0f;
    bool tile_uniform_mass = false;     // every 128-body tile of the layout has one mass
    khrr::DevBuf<float> tile_mass;      // that mass per tile (FP32)
    bool block_uniform_mass = false;    // every pair block has one mass (the pair kernel's block-mass form)
    khrr::PairBlocks pair_blocks;       // the pair kernel's blocks of the layout
    khrr::FieldConsts field{};
    khrr_tuning tuning{128, 4, 128, 0, 1};
    khrr::ForcePlan plan_batched, plan_plain, plan_fp64;
    bool predicted = false;
    double pred_dt = 0.0;
    std::map<std::tuple<uint64_t, int, bool, bool>, khrr::StepGraph> graphs;  // (dt, mode, phi, compat)

    // Kernel-level entry points: their own shadow, partials and plan.
    khrr::DevBuf<float> kshadow, kishadow;
    khrr::DevBuf<double4> kpart;
    khrr::DevBuf<unsigned long long> kfx;  // the pair kernel's sums (pos_i == pos_j under the pair tuning)
    khrr::DevBuf<khrr::FxScale> kscale;    // their tile scales
    khrr::DevBuf<double> ktile_hmin, ktile_msum;  // classification scratch per tile
    khrr::DevBuf<float> ktile_mass;   // per-tile masses (block-mass form)
    khrr::DevBuf<unsigned> kflags;    // classification of the caller's arrays
    float kh_uniform = 0.0f;          // 0.5 eps2[0] when the softenings are all equal
    khrr::ForcePlan kplan;
    int64_t kplan_n = -1;

    // Mesh pipeline (khrr_bin / khrr_wave_solve).
    bool has_bin = false;
    khrr::MeshGeom mesh{};
    int64_t ncells = 0;
    khrr::DevBuf<int2> pci;                              // per padded body: {cell, slot}
    khrr::DevBuf<int> mcount, mstart, maxpbc, mscan, mtmp;  // mscan: scan block/tile totals
    khrr::DevBuf<int> morder;                            // khrr_sort_by_cell: n body indices
    khrr::DevBuf<double> cell_mass, cell_phi, wave_resid;
    int64_t cell_phi_cells = 0;                          // mesh size the cell_phi sums belong to
    khrr::DevBuf<float> wave_phi, wave_mass, wave_tab;   // 4 C (field ring), C, 3 nx
    int wave_nx = 0;
    int wave_rot = khrr::kRingStart;                     // ring state: 4 * (phi^{n-1} buffer) + phi^n buffer
    khrr::WaveMaps wave_maps;                            // tensor maps of wave_phi / wave_mass
    khrr::DevBuf<unsigned> wave_sync;                    // nx + 1 plane counters of the resident stencil
    bool wave_warm = false;
    std::map<std::pair<int, int>, khrr::StepGraph> wave_graphs;  // (chunk, rotation)

    // Mesh-force solver (KHRR_MESH).
    khrr::MeshSolver msolver;

    // Timing.
    bool timing = false;
    cudaEvent_t ph0 = nullptr, ph1 = nullptr;  // placeholders captured in graphs
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> ev_pool;
    size_t ev_used = 0;
    int64_t timed_launches = 0;
    double timed_pairs = 0.0;
    // Device time of the last synchronising mesh call (khrr_call_timing):
    // events before its first and after its last kernel.
    cudaEvent_t call0 = nullptr, call1 = nullptr;
    bool call_timed = false;
    std::map<const void*, int> occupancy;

    khrr_status fail(khrr_status s, const char* fmt, ...);
    khrr_status cuda(cudaError_t e, const char* what);
    khrr_status check_device_flag();
    int resident_ctas(const khrr::ForceVariant* v);
    const khrr::ForceVariant* variant(bool unif, bool acc, bool phi) const;
    bool pair_mode() const;  // the tuning asks for the pair kernel (any layout of the state admits it)
    khrr::ForcePlan& plan_for(int mode) {
        return mode == khrr::kModePlain ? plan_plain : (mode == khrr::kModeF64 ? plan_fp64 : plan_batched);
    }
    khrr_status ensure_plan(int mode);
    void drop_graphs();
    khrr::ForceArgs force_args(const khrr::ForcePlan& p, int item_begin, int item_end);
    // x: the FP64 positions the forces are wanted at (read by the FP64 kernel;
    // the FP32 kernels read the shadow packed from them).
    khrr_status enqueue_force(int mode, bool acc, bool phi, bool events, const double* x);
    khrr::StepArgs step_args(const khrr::ForcePlan& p, double dt);
    khrr::Shadow shadow() { return khrr::shadow_at(shadow_buf.p, npad); }
    khrr_status enqueue_step(double dt, int mode, bool phi_now, bool compat);
    khrr_status get_step_graph(double dt, int mode, bool phi_now, bool compat, khrr::StepGraph** out);
    khrr_status timing_pair(cudaEvent_t* e0, cudaEvent_t* e1);
    khrr_status call_start();  // with timing on: event before the call's first kernel
    khrr_status call_stop();   // with timing on: event after its last kernel
    double pairs_per_pass() const;
    khrr_status force_mode(int flags, int* mode);  // KHRR_PLAIN / KHRR_FP64 -> ForceMode
    // Mesh-force solver (mesh_api.cpp).
    khrr_status mesh_ensure_layout();
    khrr_status mesh_enqueue_force(const double* x, int iters, int rot0);
    khrr_status mesh_forces(int flags);
    khrr_status mesh_step(double dt, int nsteps, int flags);
};
