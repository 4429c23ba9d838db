// Internal declarations shared by the CUDA kernels (*.cu) and the host
// runtime (*.cpp) of libkhrr.  Not part of the public ABI (include/khrr.h).
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>

namespace khrr {

// Bodies of each system are padded on the device to a multiple of this with
// zero-mass "ghost" bodies, so every j tile is whole and 16-byte aligned.
constexpr int kPad = 128;
// Error codes a kernel can raise through the context's device flag word.
constexpr unsigned kErrTimeout = 1u;

// One unit of force work: a tile of i bodies against a chunk of j bodies of
// the same system.  Indices are padded device indices.
struct WorkItem {
    int i_begin;  // first i body of the tile
    int i_end;    // end of the system's real bodies (tile entries past it are skipped)
    int j_begin;  // first j body of the chunk (multiple of the j tile)
    int j_end;    // end of the chunk (multiple of the j tile)
    int slot;     // partial-sum slot this chunk writes
    int sys;      // system index
    int pad0;     // i bodies in the tile (planner's cost estimate only)
    int pad1;
};

// FP32 shadow of a body set in structure-of-arrays form (padded length each):
// x, y, z, m and h = eps^2 / 2.  The force kernel streams j tiles of every
// array with bulk copies (16-byte aligned: j tiles start at multiples of 128).
struct Shadow {
    float* x;
    float* y;
    float* z;
    float* m;
    float* h;
};

inline Shadow shadow_at(float* base, int64_t npad) {
    return Shadow{base, base + npad, base + 2 * npad, base + 3 * npad, base + 4 * npad};
}

// Arguments of one force-kernel launch.
struct ForceArgs {
    Shadow j;                // the j (source) bodies
    Shadow i;                // the i (target) bodies; equal to j unless the sets differ
    const WorkItem* items;   // work queue
    int n_items;
    unsigned* queue;         // next-item counter (zeroed before each launch)
    double4* part;           // partial sums [slot][npad]: ax, ay, az, sum m/r
    long long npad;          // slot stride
    float h_uniform;         // 0.5 * eps2 when every body shares it
    const float* tile_mass;  // mass of each 128-body j tile (tile-mass kernels only)
    unsigned* err;           // device error flag word
};

// One compiled force-kernel instance.  pair: the symmetric kernel (pair.cu),
// launched with PairArgs; its tile_mass means one mass per kPairBlock block.
struct ForceVariant {
    int threads, i_per_thread, j_tile, stages;
    bool packed, uniform_eps, acc, phi, tile_mass;
    const void* fn;
    size_t smem;
    bool pair = false;
};

// ---- the symmetric pair kernel (pair.cu) --------------------------------------
constexpr int kPairThreads = 128;                          // threads per CTA
constexpr int kPairBodies = 8;                             // i bodies per thread
constexpr int kPairBlock = kPairThreads * kPairBodies;     // bodies per block (1024)
constexpr int kPairTile = 128;                             // j bodies per shared-memory tile

// One unit of symmetric work: the i block [i_begin, i_end) against the j
// bodies [j_begin, j_end) of later blocks of the same system (the first
// chunk of a row starts with the i block itself, [j_begin, diag_end), which
// is evaluated one-sided).  Padded device indices; j bounds are multiples of
// kPairTile.  real_end ends the system's real bodies: sums of the ghosts
// past it are not accumulated.
struct PairItem {
    int i_begin;
    int i_end;
    int j_begin;
    int j_end;
    int diag_end;  // == j_begin when the chunk holds no tile of the i block
    int real_end;  // end of the system's real bodies
    int cost;      // planner's estimate (i bodies x j bodies / 1024)
    int pad;
};

// The pair kernel's results are 64-bit fixed-point sums: every partial (an
// FP32 sum) is scaled by a power of two and rounded to an integer, then added
// with an integer atomic into its body's accumulator.  Integer addition is
// associative, so the totals do not depend on the order the partials arrive
// in (bitwise reproducible), and the accumulators take 32 bytes per body
// (components ax, ay, az, sum m/r; [component][npad]).  The scale of a
// 128-body tile keeps every possible sum of its bodies below 2^61
// (fx_scale): for a body i, |a_i| <= sum_j m_j max_d d / (d^2 + H)^{3/2}
// = 0.3849 M / H with H = h_i + h_j >= h_i + h_min, and
// |sum m/r| <= M / sqrt(h_i + h_min).
constexpr int kFxComps = 4;
struct FxScale {
    double acc, phi;          // 2^E: partial -> integer
    double inv_acc, inv_phi;  // 2^-E: integer -> value
};
// Scale of one tile from its smallest h = eps^2 / 2, the system's smallest h
// and the system's total |mass|.
FxScale fx_scale(double h_tile_min, double h_sys_min, double mass_sys);

struct PairArgs {
    Shadow sh;               // the bodies (i and j are the same set)
    const PairItem* items;
    int n_items;
    unsigned* queue;         // next-item counter (zeroed before each launch)
    unsigned long long* fx;  // fixed-point sums [kFxComps][npad] (zeroed before each launch)
    long long npad;          // component stride
    const FxScale* scale;    // per 128-body tile
    float h_uniform;         // 0.5 * eps2 when every body shares it
    const float* tile_mass;  // mass per 128-body tile (block-mass kernels)
    unsigned* err;           // device error flag word
};

int pair_variant_count();
const ForceVariant* pair_variant(int idx);
const ForceVariant* find_pair_variant(bool unif, bool acc, bool phi, bool block_mass);
cudaError_t launch_pair(const ForceVariant* v, const PairArgs& a, int grid, cudaStream_t s);
// Fixed-point sums -> acc[i] (+)= a_i and/or phi[i] (-)= sum m/r, i < n (FP64).
cudaError_t launch_reduce_pair_fx(const unsigned long long* fx, long long npad, const FxScale* scale, int64_t n,
                                  double* acc, double* phi, bool overwrite, cudaStream_t s);
// Caller's arrays -> tile_mass (first mass of each 128 tile), the tile
// scales of the fixed-point sums, and *flags &= ~1 unless every 1024 block is
// real bodies of one mass, &= ~2 unless every softening equals eps2[0], &= ~4
// unless every softening is positive (the pair kernel's condition; set *flags
// to ~0 first).  tile_hmin, tile_msum: scratch of one double per tile.
cudaError_t launch_classify(const double* mass, const double* eps2, int64_t n, float* tile_mass, double* tile_hmin,
                            double* tile_msum, FxScale* scale, unsigned* flags, cudaStream_t s);

// Derived constants of the analytic halo/bulge field (dev_fex operands).
struct FieldConsts {
    double a, b, Rb, Mb, Rh2, con, const1, Mh_inf;
    int enabled;
};

FieldConsts make_field(double Mh, double a, double Rh, double Mb, double b, double Rb);

// ---- force.cu ---------------------------------------------------------------
int force_variant_count();
const ForceVariant* force_variant(int idx);
// tile_mass: the variant that factors each j tile's single mass out of the
// tile sum (compiled for the packed shapes only).
const ForceVariant* find_force_variant(int threads, int ipt, int jt, bool packed, bool unif,
                                       bool acc, bool phi, bool tile_mass = false);
cudaError_t launch_force(const ForceVariant* v, const ForceArgs& a, int grid, cudaStream_t s);
// The plain baseline: one system (shadow offset to it, n real bodies, npad
// padded) in one launch, one i body per thread; writes partial slot 0.
cudaError_t launch_plain_force(const Shadow& sh, int n, int npad, double4* out, bool acc, bool phi,
                               cudaStream_t s);
// FP64 AoS positions -> padded FP32 SoA shadow (x, y, z, m, eps2 / 2).
cudaError_t launch_pack(const double* pos, const double* mass, const double* eps2, int64_t n,
                        int64_t npad, const Shadow& sh, cudaStream_t s);
// Partials -> out[i] (+)= sum_s part[s][i] (xyz) and/or phi[i] (-)= ...
cudaError_t launch_reduce_partials(const double4* part, long long npad, int nslots, int64_t n,
                                   double* acc, double* phi, bool overwrite, cudaStream_t s);
cudaError_t launch_fp32_probe(float* out, int iters, int grid, int block, cudaStream_t s);
// One CTA waiting (bounded, limit_ns) on an mbarrier nothing completes: the
// timeout path of every bounded wait, raising kErrTimeout in *err.
cudaError_t launch_wait_probe(unsigned* err, unsigned long long limit_ns, cudaStream_t s);
// FP64 direct sum for sampled targets: tgt[k] is a padded index, [jb[k], je[k])
// its system's padded body range; out4[k] = (ax, ay, az, phi).
cudaError_t launch_fp64_sample(const double* pos, const double* mass, const double* eps2,
                               const int64_t* tgt, const int64_t* jb, const int64_t* je, int64_t nt,
                               double* out4, cudaStream_t s);

// ---- force64.cu: the FP64 direct sum (KHRR_FP64) ------------------------------
constexpr int kF64ITile = 512;  // i bodies per work item (128 threads x 4)
struct F64Args {
    const double* pos;      // positions the forces are wanted at, AoS double3 [npad]
    const double* mass;     // [npad]
    const double* eps2;     // [npad]
    const WorkItem* items;  // work queue (plan_force_items with kF64ITile, j tiles of kPad)
    int n_items;
    unsigned* queue;        // next-item counter (zeroed before each launch)
    double4* part;          // partial sums [slot][npad]: ax, ay, az, sum m/r
    long long npad;
};
cudaError_t launch_fp64_force(const F64Args& a, bool acc, bool phi, int grid, cudaStream_t s);
int fp64_force_ctas(int sm_count);  // resident CTAs of the FP64 kernel on the device
// The symmetric FP64 pass on the pair kernel's plan: sums (ax, ay, az,
// sum m/r per body, zeroed before the launch) accumulated with FP64 atomics.
struct F64PairArgs {
    const double* pos;      // AoS double3 [npad]
    const double* mass;     // [npad]
    const double* eps2;     // [npad]
    const PairItem* items;  // plan_pair_items over 1024-body blocks
    int n_items;
    unsigned* queue;        // next-item counter (zeroed before each launch)
    double4* sums;          // [npad]
};
cudaError_t launch_fp64_pair(const F64PairArgs& a, bool acc, bool phi, int grid, cudaStream_t s);
int fp64_pair_ctas(int sm_count);

// ---- integrate.cu -----------------------------------------------------------
struct StepArgs {
    double* pos;          // x(t)           [npad] double3
    double* vel;          // v(t)
    double* acc;          // a(t) without the external field (acc0)
    double* post;         // predicted x*
    double* velt;         // predicted v*
    double* acct;         // force workspace of the literal reference loop
    const double* mass;   // [npad]
    double* phi;          // [npad] potential (written when want_phi)
    Shadow shadow;        // FP32 shadow: x, y, z rewritten with the predicted positions
    const double4* part;  // force partials [slot][npad]
    long long npad;
    const unsigned char* nsplit;  // partial slots per body
    const unsigned long long* fx;   // the pair kernel's fixed-point sums [kFxComps][npad] (replace part when set)
    const FxScale* fx_scale;        // their scales per 128-body tile
    int64_t n;            // padded count
    double dt;
    FieldConsts field;
    int compat_accumulate;
    int want_phi;
    int predict_next;
};
cudaError_t launch_predictor(const StepArgs& a, cudaStream_t s);
cudaError_t launch_corrector(const StepArgs& a, cudaStream_t s);
// Reduce partials into acc/phi of the state (khrr_forces).
cudaError_t launch_collect(const StepArgs& a, bool want_acc, bool accumulate, cudaStream_t s);
// The reference kernel-level integrator (kernelNbody_integTime semantics).
cudaError_t launch_integ_time(const double* acc, double* pos_t, double* vel_t, const double* pos,
                              const double* vel, double dt, int istep, double* acc0, int64_t n,
                              const FieldConsts& f, cudaStream_t s);
// FP64 conservation sums over bodies (ghosts have zero mass and contribute
// nothing to the sums; they sit at the origin with zero velocity).
cudaError_t launch_conservation(const double* pos, const double* vel, const double* mass,
                                const double* phi, int64_t n, double* block_out, int nblocks,
                                double* out16, cudaStream_t s);
int conservation_blocks(int64_t n);

// ---- mesh.cu ------------------------------------------------------------------
struct MeshGeom {
    double lo[3];
    double cs[3];
    double rcs[3];  // 1 / cs, correctly rounded (the cell divisions use it)
    int g[3];
};
struct WaveConsts {
    int nx;
    double dx, dt, c, diss_base, diss_extra, sim_l, bc_l;
};
// FP32 stencil constants: per-axis sponge tables (device arrays of nx) and
// cdt_half = c dt / 2, K = c^2 dt^2 / dx^2, A = 2 (1 - 3K), S = -c^2 dt^2 4 pi / dx^3.
struct WaveF32 {
    int nx;
    float diss_base, cdt_half, K, A, S;
    const float* sx;
    const float* sy;
    const float* sz;
};
// Bins n bodies: slots from counter (stride counter_stride); count2 (may be
// NULL) receives the same counts; cell_mass (may be NULL) the mass deposit.
cudaError_t launch_assign(const double* pos, int64_t n, const MeshGeom& m, int2* pci, int* counter,
                          int counter_stride, int* count2, int count2_stride, const double* mass, double* cell_mass,
                          cudaStream_t s);
int64_t scan_block_count(int64_t ncells);
int64_t scan_scratch_ints(int64_t ncells);
// Counts -> maxpbc (scan_block_count entries: inclusive scan of 512-cell block
// totals) and starts: the true exclusive scan, or with ref_view the
// reference's start_id (total of earlier 512-cell blocks).  pair: count points
// at {count, start_id} pairs and the starts go to the .start_id fields (16-byte
// aligned); else counts and starts are plain int arrays (start 16-byte
// aligned).  scratch: scan_scratch_ints(ncells) ints.
cudaError_t launch_scan(int* count, bool pair, int64_t ncells, int* maxpbc, int* start, bool ref_view, int* scratch,
                        cudaStream_t s);
cudaError_t launch_cell_phi(const double* phi, const int2* pci, const int* count, int cstride, int64_t n,
                            double* cell_phi, cudaStream_t s);
cudaError_t launch_wave_f64(double* phi_new, const double* phi, const double* phi_old, const double* mass,
                            const WaveConsts& w, cudaStream_t s);
cudaError_t launch_wave_f32(float* phi_new, const float* phi, const float* phi_old, const float* mass,
                            const WaveF32& w, double* resid, cudaStream_t s);
// The four-buffer field ring of the FP32 solver: state = 4 * old + cur; a
// single iteration writes the lower free buffer (state -> 4 * cur + f0), a
// pair writes f0 and f1 (state -> 4 * f0 + f1).
constexpr int kRingStart = 1;  // old = buffer 0, cur = buffer 1
inline void ring_free(int st, int& f0, int& f1) {
    const int o = st / 4, c = st % 4;
    int f[2], n = 0;
    for (int b = 0; b < 4; ++b)
        if (b != o && b != c) f[n++] = b;
    f0 = f[0];
    f1 = f[1];
}
inline int ring_step1(int st) {
    int f0, f1;
    ring_free(st, f0, f1);
    return 4 * (st % 4) + f0;
}
inline int ring_step2(int st) {
    int f0, f1;
    ring_free(st, f0, f1);
    return 4 * f0 + f1;
}
// k FP32 iterations: pairs, then a single one when k is odd.
inline int ring_after_f32(int st, int k) {
    for (int i = 0; i < k / 2; ++i) st = ring_step2(st);
    return k % 2 ? ring_step1(st) : st;
}
inline int ring_after_f64(int st, int k) {
    for (int i = 0; i < k; ++i) st = ring_step1(st);
    return st;
}
// Tensor maps (40 x 12 x 1 float boxes) of the four ring buffers and the
// FP32 mass of one nx^3 mesh, for the tensor-copy stencil; ok is false when
// they do not exist (nx % 4 != 0, or no driver entry point), and the stencil
// then loads through the cache instead.
struct WaveMaps {
    CUtensorMap ring[4];             // 40 x 12 boxes (two-step kernel)
    CUtensorMap mass;
    CUtensorMap halo[4];             // 40 x 10 boxes: phi with its x/y halo (one-step kernel)
    CUtensorMap tile[4], tile_mass;  // 32 x 8 boxes: phi^{n-1} and mass (one-step kernel)
    bool ok = false;
    bool two_step = false;           // pairs of iterations through the two-step kernel
    // The shared-memory-resident kernel (nx = 128): nx + 1 words for its 128
    // brick counters and abort word.
    bool resident = false;
    unsigned* sync = nullptr;
};
// Whether the shared-memory-resident FP32 stencil runs for this mesh edge on
// the current device (nx = 128, one 221 KB CTA per 128 x 16 x 8 brick, all
// co-resident).
bool wave_resident_available(int nx);
// k FP32 iterations of the ring in one cooperative launch with the field
// resident in shared memory, bit-identical to k launch_wave_f32 iterations and
// leaving the ring in the state enqueue_wave_f32 leaves it; sync: nx + 1
// counters (zeroed here); bounded waits (limit_ns each) report into err.
// withhold: a brick that never publishes its counter (the failure probe;
// -1 otherwise).
cudaError_t launch_wave_resident(float* ring, int64_t cells, const float* mass, const WaveF32& w, int k, int st,
                                 double* resid, unsigned* sync, unsigned* err, cudaStream_t s,
                                 unsigned long long limit_ns = 2000000000ull, int withhold = -1);
// One FP32 iteration fed by tensor copies (wave1_tma_kernel), bit-identical
// to launch_wave_f32.
cudaError_t launch_wave1_tma(float* phi_new, const CUtensorMap& phi, const CUtensorMap& phi_old,
                             const CUtensorMap& mass, const WaveF32& w, double* resid, unsigned* err, cudaStream_t s);
// Two FP32 iterations in one launch fed by tensor copies (wave2_tma_kernel):
// out1 = phi^{n+1}, out2 = phi^{n+2}, bit-identical to two launch_wave_f32
// calls; resid (may be NULL) sums (phi^{n+2} - phi^{n+1})^2 and (phi^{n+2})^2.
// out1 and out2 must differ from the buffers of phi and phi_old.
cudaError_t launch_wave2_tma(float* out1, float* out2, const CUtensorMap& phi, const CUtensorMap& phi_old,
                             const CUtensorMap& mass, const WaveF32& w, double* resid, unsigned* err, cudaStream_t s);
// Enqueues k FP32 iterations on the ring (4 buffers of cells floats) from
// state st; resid (may be NULL) is reduced by the last one.  With maps
// (resident, nx = 128) and err, all k run in one shared-memory-resident
// launch; else with maps (ok) the pairs run through the tensor-copy kernel.
// Bounded waits of both report into err.
cudaError_t enqueue_wave_f32(float* ring, int64_t cells, const float* mass, const WaveF32& w, int k, int st,
                             double* resid, cudaStream_t s, const WaveMaps* maps = nullptr, unsigned* err = nullptr);
cudaError_t launch_acc_field(double* cell_acc, double* cell_acc_abs, const double* phi, int nx, double dx,
                             cudaStream_t s);
cudaError_t launch_apply(double* pacc, double* pval, const double* cacc, const double* cval, const int2* pci,
                         int64_t n, cudaStream_t s);
cudaError_t launch_deinterleave(const int2* pci, int64_t n, int* a, int* b, cudaStream_t s);
cudaError_t launch_to_float(const double* src, float* dst, int64_t n, cudaStream_t s);

// Cloud-in-cell: trilinear weights about cell centres (u = (x - lo)/cs - 1/2,
// cells floor(u) and floor(u) + 1 per axis, corners outside the mesh dropped),
// cell ids as the binning's.  The deposit adds m w into cell_mass (FP64
// atomics); the gather writes acc = sum w cell_acc and value = sum w
// cell_value (either output may be NULL), corners in z, y, x order.
cudaError_t launch_cic_deposit(const double* pos, const double* mass, int64_t n, const MeshGeom& m,
                               double* cell_mass, cudaStream_t s);
cudaError_t launch_cic_gather(const double* pos, int64_t n, const MeshGeom& m, const double* cell_acc,
                              const double* cell_value, double* pacc, double* pval, cudaStream_t s);
// Counting sort: order[start[cell_i] + slot_i] = base + i for the n bodies of pci.
cudaError_t launch_scatter_order(const int2* pci, const int* start, int64_t n, int base, int* order, cudaStream_t s);
// Mesh-force gather into one partial slot per body: part[i] = {acc, -phi} of
// the body's cell (NGP, from pci) or CIC-interpolated (from pos); phi is the
// mesh potential in FP32 or FP64 (exactly one of phi32 / phi64 non-NULL).
cudaError_t launch_mesh_gather(const double* pos, const int2* pci, int64_t n, const MeshGeom& m, bool cic,
                               const double* cell_acc, const float* phi32, const double* phi64, double4* part,
                               cudaStream_t s);
// acc_field on an FP32 potential (differences formed in FP64, exact).
cudaError_t launch_acc_field_f32(double* cell_acc, const float* phi, int nx, double dx, cudaStream_t s);
// Binning without slots: pci[i] = {cell, 0} and the NGP mass deposit.
cudaError_t launch_assign_cells(const double* pos, int64_t n, const MeshGeom& m, int2* pci, const double* mass,
                                double* cell_mass, cudaStream_t s);

}  // namespace khrr
