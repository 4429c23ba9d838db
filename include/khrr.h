/*
 * khrr.h - C ABI of the B200 (sm_100a) KHRR-NBody hot path.
 *
 * The reference (KHRR-NBody) has no plugin layer: its driver nbody/src/nbody.cu
 * calls __global__ kernels directly through its RR helper
 * (CuCall(kernel, grid, block)(args...)), passing raw device pointers in the
 * reference's layouts (double3 AoS positions, double masses/eps^2,
 * CellInfo/ParticleCellInfo int pairs) and scalars through __constant__
 * DataBlock / WaveEqData.  This header is the drop-in boundary for that path:
 *
 *  - kernel-level entry points (khrr_accel, khrr_phi, khrr_integ_time, ...)
 *    take the same device pointers, layouts and accumulate semantics as the
 *    reference kernel each one replaces (cited per function);
 *  - a simulation-level API (khrr_upload_state / khrr_step / ...) owns the
 *    device state for the reference's time loop, in one or many systems;
 *  - host-only I/O functions read and write the reference's files.
 *
 * Conventions: every function returns khrr_status (no exceptions cross the
 * ABI); khrr_last_error() describes the last failure on a context.  Device
 * work is enqueued on the context's stream (khrr_set_stream to use another);
 * host pointers are borrowed for the duration of the call.  One context per
 * host thread.  Plain C types only.
 */
#ifndef KHRR_H
#define KHRR_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define KHRR_ABI_VERSION 1

typedef enum khrr_status {
    KHRR_OK = 0,
    KHRR_ERR_INVALID_ARG = 1,  /* bad pointer, size or parameter            */
    KHRR_ERR_NOT_MULTIPLE = 2, /* size violates a documented multiple        */
    KHRR_ERR_CUDA = 3,         /* CUDA runtime error (see khrr_last_error)   */
    KHRR_ERR_IO = 4,           /* file missing, unreadable or malformed      */
    KHRR_ERR_TIMEOUT = 5,      /* a bounded device wait gave up              */
    KHRR_ERR_STATE = 6,        /* call out of order (e.g. step before upload)*/
    KHRR_ERR_OOM = 7,          /* device allocation failed                   */
    KHRR_ERR_UNSUPPORTED = 8,  /* no device / wrong architecture             */
    KHRR_ERR_TOO_LARGE = 9     /* n exceeds the fixed scratch of khrr_accel_noalloc */
} khrr_status;

typedef struct khrr_ctx khrr_ctx;

/* Force-evaluation flags. */
enum {
    KHRR_ACC = 1,               /* accelerations (ACCEL_kernel)                   */
    KHRR_PHI = 2,               /* potentials (PHI_kernel), fused in the same pass */
    KHRR_COMPAT_ACCUMULATE = 4, /* reference time loop: the step force is added to
                                   the previous step's (nbody.cu:1559-1566 never
                                   zeroes acct_); default overwrites             */
    KHRR_PLAIN = 8,             /* baseline: the conventional FP32 kernel (one i
                                   body per thread, shared-memory j tiles), one
                                   launch per system                              */
    KHRR_OVERWRITE = 16,        /* kernel-level calls: overwrite instead of +=    */
    KHRR_MESH = 32,             /* khrr_forces / khrr_step: forces from the mesh
                                   solver (khrr_set_mesh_solver), the reference's
                                   Wave mode, instead of the direct sum          */
    KHRR_FP64 = 64              /* khrr_forces / khrr_step: the direct sum in FP64,
                                   the reference's precision (ACCEL_kernel and
                                   PHI_kernel with real = double; each unordered
                                   pair evaluated once, or with the environment
                                   variable KHRR_FP64_ONESIDED=1 every ordered
                                   pair), at about 30 % of the FP32 pair
                                   kernel's rate: the comparator for accuracy
                                   and energy drift                              */
};

/* Analytic halo + bulge parameters (__gr_par.ini lines 1-6); the derived
 * constants are computed as nbody/src/nbody.cu:1111-1120 does. */
typedef struct khrr_field_params {
    double Mh, a, Rh, Mb, b, Rb;
} khrr_field_params;

/* Conservation diagnostics of result() (nbody/src/nbody.cu:797-833), reduced
 * on the GPU in FP64.  Ek and Ep are the raw sums; E = (Ek + Ep) / 2. */
typedef struct khrr_lie {
    double L[3];
    double Imp[3];
    double Ek, Ep, E;
    double R_max, Z_max, Vr_max, Vfi_max, Vz_max;
} khrr_lie;

/* Force-kernel shape: threads per CTA, i bodies per thread, j-tile size,
 * j_split = number of j chunks per system (0 = chosen automatically), and
 * packed = 1 for the packed-FP32 (f32x2, two j bodies per instruction) inner
 * loop, 0 for the scalar one.  packed = 2 selects the symmetric pair kernel
 * (shape {128, 8, 128}): each unordered pair of a system is evaluated once
 * and applied to both bodies, the softening term (eps_i^2 + eps_j^2)/2 being
 * symmetric; j_split is then its chunk of 1024-body blocks per work item
 * (0 = chosen automatically).  It serves the state API and khrr_accel /
 * khrr_phi calls with pos_i == pos_j; other calls run the packed 128 x 4
 * one-sided kernel. */
typedef struct khrr_tuning {
    int threads;
    int i_per_thread;
    int j_tile;
    int j_split;
    int packed;
} khrr_tuning;

/* ---- library / context ---------------------------------------------------- */
int khrr_abi_version(void);
const char* khrr_status_name(khrr_status s);
/* Creates a context on CUDA device `device` (a B200, sm_100). */
khrr_status khrr_create(int device, khrr_ctx** out);
void khrr_destroy(khrr_ctx* ctx);
const char* khrr_last_error(const khrr_ctx* ctx);
/* The context's stream (cudaStream_t) and a way to replace it (NULL restores
 * the context's own stream). */
void* khrr_get_stream(khrr_ctx* ctx);
khrr_status khrr_set_stream(khrr_ctx* ctx, void* stream);
khrr_status khrr_synchronize(khrr_ctx* ctx);

/* ---- kernel-level entry points (device pointers) ------------------------ */
/* ACCEL_kernel (nbody-kernel.cuh:89-142): acc[i] += sum_j m_j d/(d^2 +
 * (eps2_i + eps2_j)/2)^{3/2}, d = pos_j[j] - pos_i[i], over i, j < n
 * (KHRR_OVERWRITE: acc = sum).  pos_*, acc: n double3 (AoS xyz); mass_j,
 * eps2_j: n doubles.  Pair terms in FP32 with compensated sums; any n >= 0 (0: nothing to do)
 * (the reference needs n % 512 == 0). */
khrr_status khrr_accel(khrr_ctx* ctx, double* acc, const double* pos_i, const double* pos_j,
                       const double* mass_j, const double* eps2_j, int64_t n, int flags);
/* PHI_kernel (nbody-kernel.cuh:43-86): phi[i] -= sum_j m_j/sqrt(d^2 +
 * (eps2_i + eps2_j)/2), j = i included (KHRR_OVERWRITE: phi = -sum). */
khrr_status khrr_phi(khrr_ctx* ctx, double* phi, const double* pos_i, const double* pos_j,
                     const double* mass_j, const double* eps2_j, int64_t n, int flags);
/* kernelNbody_integTime (nbody-kernel.cuh:144-193), FP64, with the context's
 * external field: istep 0 = predictor, 1 = corrector; same argument roles. */
khrr_status khrr_integ_time(khrr_ctx* ctx, const double* acc, double* pos_t, double* vel_t,
                            const double* pos, const double* vel, double dt, int istep,
                            double t, double* acc0, int64_t n);

/* ---- p2mesh: binning, prefix sums, deposits, wave stencil, gather ------- */
/* Mesh geometry (WaveEqData.domainMin / cellSize / gridSize, common.cuh:57-61). */
typedef struct khrr_mesh {
    double lo[3];
    double cell[3];
    int grid[3];
} khrr_mesh;

/* Wave-equation constants (WaveEqData, common.cuh:62-71; values as
 * nbody/src/nbody.cu:1134-1143 derives them: dt = 0.5 dx / (c sqrt 3),
 * sim_l = nx dx / 2, bc_l = sim_l / 10). */
typedef struct khrr_wave_params {
    int nx;
    double dx, dt, c, diss_base, diss_extra, sim_l, bc_l;
} khrr_wave_params;

enum {
    KHRR_SCAN_REFERENCE = 0, /* start_id = total of all earlier 512-cell blocks (the reference) */
    KHRR_SCAN_EXCLUSIVE = 1  /* start_id = exclusive prefix sum of the counts (a true scan)     */
};

/* assignParticlesToCells (p2mesh-kernel.cuh:11-57), fused with
 * computeCellMassesUnsorted (:126-137) when mass and cell_mass are given.
 * pos: n double3; particle_cell_info: n x {cell_id, id_in_cell} (int pairs);
 * cell_info: C x {count, start_id}; cell_count: C (the reference's slot
 * counter, may be NULL); cell_mass: C (may be NULL).  Counts and masses are
 * accumulated into, as in the reference (its driver zeroes them first,
 * nbody.cu:149-153).  Cell indices follow the reference bit for bit
 * (IEEE FP64 division, truncation, clamps, iz clamped to gridSize.y - 1,
 * id = iz*gx*gy + iy*gz + ix); id_in_cell is a valid slot order within each
 * cell (atomics, as in the reference). */
khrr_status khrr_assign_particles_to_cells(khrr_ctx* ctx, const double* pos, int64_t n,
                                           const khrr_mesh* mesh, int* particle_cell_info,
                                           int* cell_info, int* cell_count, const double* mass,
                                           double* cell_mass);
/* computePrefixSums + adjustGlobalPrefixSums (p2mesh-kernel.cuh:62-123):
 * reads cell_info.count, writes cell_info.start_id (per mode) and max_pbc
 * (ceil(ncells/512) ints: inclusive prefix of 512-cell block totals, the
 * array the reference leaves in its second argument). */
khrr_status khrr_compute_prefix_sums(khrr_ctx* ctx, int* cell_info, int* max_pbc, int64_t ncells,
                                     int mode);
/* computeCellPhiUnsorted (p2mesh-kernel.cuh:152-167): cell_phi[c] += phi_i /
 * count[c] for every body (accumulates, as the reference does). */
khrr_status khrr_cell_phi(khrr_ctx* ctx, const double* phi, const int* particle_cell_info,
                          const int* cell_info, int64_t n, double* cell_phi);
/* wave_diss_iteration (wave-kernel.cuh:5-103), FP64: one leap-frog step of
 * the damped wave equation on the nx^3 mesh (faces held at 0). */
khrr_status khrr_wave_iteration(khrr_ctx* ctx, double* phi_new, const double* phi,
                                const double* phi_old, const double* cell_mass,
                                const khrr_wave_params* p);
/* acc_field (p2mesh-kernel.cuh:169-225) over the whole nx^3 mesh (the
 * reference's 1-D launch leaves most cells unset; this covers all of them):
 * cell_acc = -grad(phi) / dx (central, one-sided on faces), nx^3 double3;
 * cell_acc_abs (nx^3, may be NULL) = |cell_acc|. */
khrr_status khrr_acc_field(khrr_ctx* ctx, double* cell_acc, double* cell_acc_abs,
                           const double* cell_phi, int nx, double dx);
/* apply_acceleration_to_particles + apply_cell_to_particles
 * (p2mesh-kernel.cuh:227-254): NGP gather; either output may be NULL. */
khrr_status khrr_apply_cells_to_particles(khrr_ctx* ctx, double* particle_acc,
                                          double* particle_value, const double* cell_acc,
                                          const double* cell_value,
                                          const int* particle_cell_info, int64_t n);

/* Context-level mesh pipeline on the uploaded positions: bin, scan (both
 * views), deposit masses; results stay on the device for khrr_wave_solve and
 * are copied to any non-NULL host array (n or C entries). */
khrr_status khrr_bin(khrr_ctx* ctx, const khrr_mesh* mesh, int* cell_id, int* id_in_cell,
                     int* count, int* start, int* start_ref, double* cell_mass);
/* Damped-wave Poisson solve on the last khrr_bin's masses (mesh: p->nx^3,
 * same geometry): FP32 stencil, the residual |phi_new - phi|_2 / |phi_new|_2
 * reduced in FP64 every check_every iterations; stops below tol or after
 * max_iter.  Starts from the previous solve's field (warm start) unless
 * cold != 0.  phi_out (nx^3 floats, may be NULL) receives the field. */
khrr_status khrr_wave_solve(khrr_ctx* ctx, const khrr_wave_params* p, double tol, int max_iter,
                            int check_every, int cold, int* iters, double* resid,
                            float* phi_out);

/* Potential per cell of the last khrr_bin: cell_phi[c] += phi_i / count[c]
 * over the uploaded bodies (computeCellPhiUnsorted, p2mesh-kernel.cuh:152-167)
 * with phi from the last KHRR_PHI evaluation.  The sums persist in the
 * context and accumulate over calls, as the reference's cell_phi_curr_ does
 * (nbody.cu:1628-1634); reset != 0 clears them first.  cell_phi (host, C,
 * may be NULL) receives the sums. */
khrr_status khrr_bin_cell_phi(khrr_ctx* ctx, int reset, double* cell_phi);

/* ---- p2mesh beyond the reference's NGP path ------------------------------ */
/* Mass assignment schemes of the mesh solver and the CIC entry points. */
enum {
    KHRR_ASSIGN_NGP = 0, /* nearest grid point: the reference's cell of each body */
    KHRR_ASSIGN_CIC = 1  /* cloud in cell: trilinear weights about cell centres     */
};

/* Cloud-in-cell deposit (no counterpart in the reference, whose deposit is
 * NGP, computeCellMassesUnsorted, p2mesh-kernel.cuh:126-137): each body
 * spreads its mass over the 8 cells around u = (x - lo)/cell - 1/2 with
 * weights (1 - f, f) per axis (f = u - floor(u)); corners outside the mesh
 * are dropped.  Device pointers: pos n double3, mass n, cell_mass C
 * (accumulated into, FP64 atomics).  Cubic meshes only. */
khrr_status khrr_cic_deposit(khrr_ctx* ctx, const double* pos, const double* mass, int64_t n,
                             const khrr_mesh* mesh, double* cell_mass);
/* Cloud-in-cell interpolation, the gather matching khrr_cic_deposit (the
 * reference's NGP gathers are apply_acceleration_to_particles /
 * apply_cell_to_particles, p2mesh-kernel.cuh:227-254): particle_acc (n
 * double3) = sum w cell_acc (C double3), particle_value (n) = sum w
 * cell_value (C); either output may be NULL. */
khrr_status khrr_cic_gather(khrr_ctx* ctx, const double* pos, int64_t n, const khrr_mesh* mesh,
                            const double* cell_acc, const double* cell_value,
                            double* particle_acc, double* particle_value);
/* The int32 cell-index prefix-sum sort of the last khrr_bin (the reference
 * computes start_id and id_in_cell, p2mesh-kernel.cuh:11-123, but never
 * reorders): order[start[cell_i] + id_in_cell_i] = i, bodies numbered as
 * uploaded (all systems).  Within a cell bodies follow their slot, the
 * atomic order of id_in_cell.  order (host, n ints) may be NULL: the order
 * then stays on the device only. */
khrr_status khrr_sort_by_cell(khrr_ctx* ctx, int* order);

/* The mesh-force solver: the reference's Wave mode (nbody.cu:1449-1472 at
 * setup, 1540-1558 per step; it is compiled there but switched off by
 * solver = NBodySolver::Nbody, nbody.cu:1132).  The mesh is the wave grid:
 * wave.nx^3 cells of size wave.dx over [-nx dx/2, nx dx/2]^3.  Per force
 * evaluation: zero and deposit the masses (NGP, the reference's, or CIC) at
 * the positions the force is wanted at, run `iters_per_step` stencil
 * iterations continuing from the previous field (the reference's
 * (int)(dtgrav / dt_wave)), take -grad(phi) (acc_field with its 3-D launch)
 * and gather acceleration and potential to the bodies.  khrr_forces with
 * KHRR_MESH starts from a zero field and runs `setup_iters` iterations (the
 * reference's 20000).  fp64 != 0 runs the reference's FP64 stencil, else the
 * FP32 one.  NULL switches the solver off. */
typedef struct khrr_mesh_solver {
    khrr_wave_params wave;
    int assign;          /* KHRR_ASSIGN_NGP or KHRR_ASSIGN_CIC */
    int fp64;
    int iters_per_step;
    int setup_iters;
} khrr_mesh_solver;
khrr_status khrr_set_mesh_solver(khrr_ctx* ctx, const khrr_mesh_solver* solver);
/* The mesh solver's potential field (nx^3, host, FP64; from the FP32 field
 * when fp64 == 0), e.g. for the reference's print_cell_phi cuts. */
khrr_status khrr_mesh_solver_phi(khrr_ctx* ctx, double* cell_phi);

/* ---- drop-in file surface (host only; no device work) ------------------- */
/* One entry of __start_galaxies.ini (GalaxyProperties, parse.cuh:19-62).
 * n_star / n_dark are the bodies the reference loads: a component of zero
 * mass has none (parse.cuh:33-42); the per-body mass is M / n. */
typedef struct khrr_galaxy {
    int n_star, n_dark;
    double m_star, m_dark;
    double eps_star, eps_dark;
    double angle_deg;
    double centre[3];
    double vel[3];
} khrr_galaxy;

/* read_galaxy_properties (parse.cuh:320-367): the galaxy count, then per
 * galaxy its id, "Ns,Ndm", "Ms,Mdm", "eps_s,eps_dm", alpha, "X,Y,Z",
 * "Vx,Vy,Vz", each value followed by a comment to the end of the line. */
khrr_status khrr_read_galaxies_ini(const char* path, khrr_galaxy* out, int max, int* count);
/* read_start_info (nbody.cu:961-984): i_cont, tmax, dt_save. */
khrr_status khrr_read_start_nbody_ini(const char* path, int* i_cont, double* tmax, double* dt_save);
/* __gr_par.ini (nbody.cu:1080-1106): Mh, a, Rh, Mb, b, Rb, eps, dtgrav, K_m,
 * K_r (any output pointer may be NULL). */
khrr_status khrr_read_gr_par_ini(const char* path, khrr_field_params* field, double* eps, double* dtgrav,
                                 double* K_m, double* K_r);
/* __GPUs.ini: nGPU then nGPU device ids, one per line. */
khrr_status khrr_read_gpus_ini(const char* path, int* ngpu, int* devices, int max);
/* start_S{k}.txt / start_DM{k}.txt (nbody.cu:1331-1341): "N t" then N lines
 * "x y z vx vy vz".  Reads up to max bodies (n = bodies read). */
khrr_status khrr_read_start_txt(const char* path, int64_t max, double* pos, double* vel, int64_t* n,
                                double* t);
khrr_status khrr_write_start_txt(const char* path, int64_t n, const double* pos, const double* vel,
                                 double t);
/* S_/DM_ snapshots (print_particles_bin, nbody.cu:726-755): int32 count,
 * f64 t, count x {x y z vx vy vz} f64, little-endian, no padding. */
khrr_status khrr_write_snapshot(const char* path, int32_t count, double t, const double* pos,
                                const double* vel);
khrr_status khrr_read_snapshot(const char* path, int64_t max, double* pos, double* vel, int32_t* count,
                               double* t);
/* LIE_0.bin (nbody.cu:844-848): L0 (3 f64), Imp0 (3 f64), E0 (f64) and 16
 * padding bytes (the reference writes E0 with sizeof(double3); written as
 * zeros here).  The reader fills L, Imp and E. */
khrr_status khrr_write_lie0(const char* path, const khrr_lie* lie0);
khrr_status khrr_read_lie0(const char* path, khrr_lie* lie0);
/* The initial-condition load of run() (nbody.cu:1315-1421): for every galaxy
 * with stars, start_S{k}.txt from dir, then for every galaxy with dark
 * matter start_DM{k}.txt; each body placed by the galaxy's tilt and shift
 * exactly as the reference does (including its use of the already updated x
 * for z, a shear for alpha != 0), masses M/n and eps2 = eps^2.  Layout: the
 * stars of all galaxies, then the dark matter of all galaxies.  n and
 * n_star_total receive the counts. */
khrr_status khrr_load_initial_conditions(const char* dir, const khrr_galaxy* g, int ngal, int64_t max,
                                         double* pos, double* vel, double* mass, double* eps2, int64_t* n,
                                         int64_t* n_star_total);

/* Largest n khrr_accel_noalloc accepts. */
#define KHRR_NOALLOC_MAX_BODIES 32768
/* khrr_accel without any device allocation.  This entry point has no
 * counterpart in the reference.  It exists for callers that cannot allocate
 * device memory on their call path: a host program that fixes its device
 * memory budget at start-up (cudaMalloc can synchronize the device and can
 * fail under memory pressure mid-run), or a plugin host that only hands out
 * device pointers it already owns.  It needs no context: the caller passes
 * the inputs, the output and a stream (cudaStream_t, NULL = legacy default).
 * Same arguments and semantics as khrr_accel (acc += sum, or acc = sum with
 * KHRR_OVERWRITE), for 1 <= n <= KHRR_NOALLOC_MAX_BODIES; larger n returns
 * KHRR_ERR_TOO_LARGE before any device work.
 * Scratch: one file-scope device array of about 9.3 MiB (shadow positions,
 * work items, partial sums, a queue counter and an error flag), which every
 * GPU that loads the library holds until the process exits.  The first call
 * on a device looks up that array's device address (with the device current)
 * and sets the kernel's attributes, so make the first call before any stream
 * capture; if that set-up fails, the call returns the error and the next call
 * tries it again.  All calls share the array and the counter and flag are
 * cleared on every call, so calls whose GPU work overlaps (on different
 * streams or host threads) race: serialize them on one stream.  The call only
 * enqueues work; it returns without synchronizing, so a failure on the device
 * cannot be its return value: if one of the kernel's bounded waits gives up
 * (about 2 s without a copy completing), every entry of acc[0 .. 3n) is set
 * to NaN instead of the sums, in either mode. */
khrr_status khrr_accel_noalloc(double* acc, const double* pos_i, const double* pos_j,
                               const double* mass_j, const double* eps2_j, int64_t n,
                               int flags, void* stream);

/* ---- simulation-level API (context-owned device state) ------------------ */
/* External field for all later integration; NULL disables it. */
khrr_status khrr_set_external_field(khrr_ctx* ctx, const khrr_field_params* p);
/* Uploads n bodies: pos, vel (n x 3, AoS), mass and eps2 (n).  Systems are
 * independent (no mutual gravity): nsys >= 1 ranges given by sys_offsets
 * (nsys + 1 increasing offsets, first 0, last n); sys_offsets NULL = one
 * system.  Resets acc/phi to zero (call khrr_forces for a(t0)).  Every eps2
 * must be > 0 (KHRR_ERR_INVALID_ARG otherwise).  The arrays are checked
 * while their copies to the device are in flight, so an upload that fails
 * after its argument checks leaves the context without state: entry points
 * that need one return KHRR_ERR_STATE until the next successful upload. */
khrr_status khrr_upload_state(khrr_ctx* ctx, int64_t n, const double* pos, const double* vel,
                              const double* mass, const double* eps2, int nsys,
                              const int64_t* sys_offsets);
/* Copies the state back; any pointer may be NULL.  acc excludes the external
 * field (the reference's acc0); phi is from the last KHRR_PHI evaluation. */
khrr_status khrr_download_state(khrr_ctx* ctx, double* pos, double* vel, double* acc,
                                double* phi);
/* Sets a(t) (n x 3, without the external field) after an upload, e.g. when a
 * run resumes with known accelerations; the next khrr_step uses it. */
khrr_status khrr_set_accelerations(khrr_ctx* ctx, const double* acc);
/* FP64 direct sum on the GPU for nt sampled bodies (indices into the uploaded
 * order) over their own system, at the current positions: the accuracy
 * reference each run reports against.  acc: nt x 3, phi: nt (either NULL). */
khrr_status khrr_accel_fp64_sample(khrr_ctx* ctx, const int64_t* targets, int64_t nt, double* acc,
                                   double* phi);
/* Forces at the current positions (KHRR_ACC and/or KHRR_PHI; KHRR_PLAIN or
 * KHRR_FP64; KHRR_MESH). */
khrr_status khrr_forces(khrr_ctx* ctx, int flags);
/* nsteps predictor -> force -> corrector steps of size dt (nbody.cu:1525-1582),
 * replayed from a CUDA graph.  flags: KHRR_PHI evaluates the potential at the
 * new positions in the last step's force pass; KHRR_COMPAT_ACCUMULATE;
 * KHRR_PLAIN (per-system launches) or KHRR_FP64 (the FP64 direct sum);
 * KHRR_MESH. */
khrr_status khrr_step(khrr_ctx* ctx, double dt, int nsteps, int flags);
/* L, Imp, Ek, Ep, E and maxima over all bodies (uses the last phi). */
khrr_status khrr_conservation(khrr_ctx* ctx, khrr_lie* out);

/* Force-kernel shape; khrr_autotune times the candidates on the current
 * state and caches the winner per body count in cache_path (NULL = no cache). */
khrr_status khrr_set_tuning(khrr_ctx* ctx, const khrr_tuning* t);
khrr_status khrr_get_tuning(khrr_ctx* ctx, khrr_tuning* t);
khrr_status khrr_autotune(khrr_ctx* ctx, const char* cache_path);

/* Device timing of the force kernel: when enabled, every force launch is
 * bracketed by CUDA events on the launching stream; khrr_force_timing returns
 * (after a synchronize) the summed milliseconds and the launch count since the
 * last call, and the pair interactions those launches computed. */
khrr_status khrr_enable_timing(khrr_ctx* ctx, int enable);
khrr_status khrr_force_timing(khrr_ctx* ctx, double* ms, int64_t* launches,
                              double* interactions);
/* Device time of the last khrr_bin, khrr_bin_cell_phi or khrr_sort_by_cell
 * made with timing enabled: the milliseconds between CUDA events recorded on
 * the context's stream before the call's first kernel and after its last one,
 * so neither the downloads to the caller's buffers nor the host-side
 * synchronisation that ends the call are included.  (No reference
 * counterpart: the reference times nothing on the mesh path.)  Returns
 * KHRR_ERR_STATE when no such call was timed. */
khrr_status khrr_call_timing(khrr_ctx* ctx, double* ms);
/* Pair interactions one force pass computes on the uploaded state
 * (sum over systems of n_k^2, j = i counted as the reference does). */
khrr_status khrr_pair_count(khrr_ctx* ctx, double* pairs);
/* FP32 FMA throughput probe: a dependent-chain FMA kernel on all SMs;
 * returns TFLOP/s (2 flops per FMA) measured with CUDA events. */
khrr_status khrr_fp32_probe(khrr_ctx* ctx, double* tflops);
/* Failure-path check (the reference has no failure detection; main only
 * catches host exceptions, nbody.cu:1713-1721): runs one kernel that waits,
 * through the same bounded wait as the force and stencil kernels, on a
 * barrier nothing completes.  It gives up after `seconds` (0 < s <= 10),
 * raises the context's device error flag and returns; this call then reports
 * KHRR_ERR_TIMEOUT with the message a stalled copy gives, and clears the
 * flag.  The context stays usable.  No fault, trap or unbounded loop is
 * involved. */
khrr_status khrr_probe_bounded_wait(khrr_ctx* ctx, double seconds);
/* The same check for the cooperative 128^3 stencil, whose CTAs wait on one
 * another's counters: four iterations on a zero field in scratch buffers of
 * its own, with brick 0 never publishing its counter and every wait limited
 * to `seconds` (0 < s <= 10).  Its neighbours give up and raise the device
 * error flag and the kernel's abort word, every other CTA's wait ends on
 * that word, and the launch completes; the call reports KHRR_ERR_TIMEOUT and
 * clears the flag, and the context stays usable.  KHRR_ERR_UNSUPPORTED where
 * the resident stencil cannot run (it needs 128 co-resident 221 KB CTAs). */
khrr_status khrr_probe_resident_wave(khrr_ctx* ctx, double seconds);

#ifdef __cplusplus
}
#endif
#endif /* KHRR_H */
