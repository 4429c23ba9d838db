// oracle/_ref: the reference's own FP64 kernels, compiled for the host.
//
// TEST INFRASTRUCTURE ONLY.  This translation unit includes the reference's
// unmodified kernel headers (nbody/include/nbody-kernel.cuh,
// p2mesh-kernel.cuh, wave-kernel.cuh) through refshim/ and exposes them with a
// C ABI so the tests can (a) pin the oracle restatement and (b) time the
// reference's arithmetic on the host cores as the CPU baseline.  Nothing here
// is linked into the product library.
#include <omp.h>

#include <cstdint>

#include "cuda_runtime.h"
#include "ref_launch.h"

#include "nbody-kernel.cuh"
#include "p2mesh-kernel.cuh"
#include "wave-kernel.cuh"

thread_local shim_dim3 threadIdx{0, 0, 0};
thread_local shim_dim3 blockIdx{0, 0, 0};
thread_local shim_dim3 blockDim{1, 1, 1};
thread_local shim_dim3 gridDim{1, 1, 1};

static inline unsigned blocks_for(int64_t n, unsigned b) { return (unsigned)((n + b - 1) / b); }

extern "C" {

// Host constants of the analytic halo/bulge field, as nbody/src/nbody.cu:1111-1120
// computes them before uploading DataBlock (nbody.cu:1205-1220).
void ref_set_field(double Mh, double a, double Rh, double Mb, double b, double Rb,
                   int ns, int nn) {
    const double Rh2 = 3.0 * Rh;
    const double rcore1 = Rh / a;
    const double rbcore1 = 1.0 / b;
    const double rbcore2 = rbcore1 * rbcore1;
    const double root1 = std::sqrt(1.0 + (Rb * Rb) * rbcore2);
    const double con = Mh / (rcore1 - std::atan(rcore1));
    const double const1 = Mb / (b * std::log(Rb * rbcore1 + root1) - Rb / root1);
    const double c_phi_h = con / a * (0.5 * std::log(Rh2 * Rh2 / a / a + 1.0) + std::atan(Rh2 / a) * a / Rh2) + Mh / Rh2;
    const double c_phi_b = Mb / Rb - const1 * std::log(Rb / b + root1) / Rb;
    const double Mh_inf = Mh * (Rh2 / a - std::atan(Rh2 / a)) / (rcore1 - std::atan(rcore1));
    dd.Ns = ns;
    dd.NN = nn;
    dd.Mh = Mh;
    dd.Mh_inf = Mh_inf;
    dd.a = a;
    dd.Rh = Rh;
    dd.Mb = Mb;
    dd.b = b;
    dd.Rb = Rb;
    dd.Rh2 = Rh2;
    dd.con = con;
    dd.const1 = const1;
    dd.c_phi_h = c_phi_h;
    dd.c_phi_b = c_phi_b;
    dd.eps2 = 0.0;
}

// Derived field constants as set by ref_set_field: Rh2, con, const1, Mh_inf.
void ref_get_field_consts(double* out4) {
    out4[0] = dd.Rh2;
    out4[1] = dd.con;
    out4[2] = dd.const1;
    out4[3] = dd.Mh_inf;
}

// dev_fex (nbody-kernel.cuh:8-40) for n positions (AoS xyz).
void ref_fex(int64_t n, const double* pos, double* out) {
    const double3* p = reinterpret_cast<const double3*>(pos);
#pragma omp parallel for
    for (int64_t i = 0; i < n; ++i) {
        double3 f = dev_fex(p[i], 0.0);
        out[3 * i + 0] = f.x;
        out[3 * i + 1] = f.y;
        out[3 * i + 2] = f.z;
    }
}

// ACCEL_kernel (nbody-kernel.cuh:89-142) for the listed target bodies, run as
// gridDim = n, blockDim = 1: the j order (0..n-1) is the kernel's own.
// acc has n entries (AoS xyz) and is accumulated into (acc += f), as the
// kernel does; targets == nullptr means all bodies.
void ref_accel(int64_t n, const double* pos, const double* mass, const double* eps2,
               int64_t nt, const int64_t* targets, double* acc) {
    dd.NN = (int)n;
    const double3* p = reinterpret_cast<const double3*>(pos);
    double3* a = reinterpret_cast<double3*>(acc);
    const int64_t count = targets ? nt : n;
#pragma omp parallel for schedule(dynamic, 1)
    for (int64_t k = 0; k < count; ++k) {
        const int64_t i = targets ? targets[k] : k;
        threadIdx = shim_dim3{0, 0, 0};
        blockIdx = shim_dim3{(unsigned)i, 0, 0};
        blockDim = shim_dim3{1, 1, 1};
        gridDim = shim_dim3{(unsigned)n, 1, 1};
        ACCEL_kernel(a, p, p, mass, eps2);
    }
}

// kernelNbody_integTime (nbody-kernel.cuh:144-193); one thread per body.
void ref_integ(int64_t n, const double* acc, double* pos_t, double* vel_t,
               const double* pos, const double* vel, double dt, int istep, double t,
               double* acc0) {
    launch_grid(shim_make_dim3((unsigned)n), shim_make_dim3(1), true, [&] {
        kernelNbody_integTime(reinterpret_cast<const double3*>(acc),
                              reinterpret_cast<double3*>(pos_t),
                              reinterpret_cast<double3*>(vel_t),
                              reinterpret_cast<const double3*>(pos),
                              reinterpret_cast<const double3*>(vel), dt, istep, t,
                              reinterpret_cast<double3*>(acc0));
    });
}

// WaveEqData upload (common.cuh:57-72; values set at nbody/src/nbody.cu:1222-1234).
void ref_set_mesh(double minx, double miny, double minz, double csx, double csy, double csz,
                  int gx, int gy, int gz, int nx_wave, double dx_wave, double dt_wave,
                  double c_wave, double diss_base, double diss_extra, double sim_l,
                  double bc_l) {
    wave_eq_data_.domainMin = make_double3(minx, miny, minz);
    wave_eq_data_.domainMax = make_double3(-minx, -miny, -minz);
    wave_eq_data_.cellSize = make_double3(csx, csy, csz);
    wave_eq_data_.gridSize = make_int3(gx, gy, gz);
    wave_eq_data_.nx_wave = nx_wave;
    wave_eq_data_.dx_wave = dx_wave;
    wave_eq_data_.dt_wave = dt_wave;
    wave_eq_data_.c_wave = c_wave;
    wave_eq_data_.diss_base = diss_base;
    wave_eq_data_.diss_extra = diss_extra;
    wave_eq_data_.sim_l = sim_l;
    wave_eq_data_.bc_l = bc_l;
}

// assignParticlesToCells (p2mesh-kernel.cuh:11-57), 512-thread blocks, run in
// launch order on one thread so the atomic slots come out in body order.
// pci: n x {cell_id, id_in_cell}; cell_info: C x {count, start_id}; count: C.
// All outputs must be zeroed by the caller (nbody.cu:149-153 does set_zero).
void ref_assign(int64_t n, const double* pos, int* pci, int* cell_info, int* count) {
    launch_grid(shim_make_dim3(blocks_for(n, 512)), shim_make_dim3(512), false, [&] {
        assignParticlesToCells(reinterpret_cast<const double3*>(pos),
                               reinterpret_cast<ParticleCellInfo*>(pci),
                               reinterpret_cast<CellInfo*>(cell_info), count, (int)n);
    });
}

// adjustGlobalPrefixSums (p2mesh-kernel.cuh:110-123).
void ref_adjust(int64_t ncells, int* cell_info, const int* maxpbc) {
    launch_grid(shim_make_dim3(blocks_for(ncells, 512)), shim_make_dim3(512), true, [&] {
        adjustGlobalPrefixSums(reinterpret_cast<CellInfo*>(cell_info), maxpbc, (int)ncells);
    });
}

// computeCellMassesUnsorted (p2mesh-kernel.cuh:126-137), in body order.
void ref_cell_masses(int64_t n, const double* mass, int* pci, double* cell_mass) {
    launch_grid(shim_make_dim3(blocks_for(n, 512)), shim_make_dim3(512), false, [&] {
        computeCellMassesUnsorted(mass, reinterpret_cast<ParticleCellInfo*>(pci), cell_mass,
                                  (int)n);
    });
}

// computeCellPhiUnsorted (p2mesh-kernel.cuh:152-167), in body order.
void ref_cell_phi(int64_t n, const double* phi, const int* pci, const int* cell_info,
                  double* cell_phi) {
    launch_grid(shim_make_dim3(blocks_for(n, 512)), shim_make_dim3(512), false, [&] {
        computeCellPhiUnsorted(phi, reinterpret_cast<const ParticleCellInfo*>(pci),
                               reinterpret_cast<const CellInfo*>(cell_info), cell_phi, (int)n);
    });
}

// wave_diss_iteration (wave-kernel.cuh:5-103) on the nx^3 mesh set by
// ref_set_mesh, 8^3-thread blocks as nbody/src/nbody.cu:217-236 launches it.
void ref_wave(double* phi_new, const double* phi, const double* phi_old, const double* mass) {
    const int nx = wave_eq_data_.nx_wave;
    const unsigned b = blocks_for(nx, 8);
    launch_grid(shim_make_dim3(b, b, b), shim_make_dim3(8, 8, 8), true,
                [&] { wave_diss_iteration(phi_new, phi, phi_old, mass); });
}

// acc_field (p2mesh-kernel.cuh:169-225) with a 3-D launch covering the mesh
// (the reference launches it 1-D, which leaves most cells unset); nx % 8 == 0.
void ref_acc_field(int nx, double dx, const double* cell_phi, double* cell_acc,
                   double* cell_acc_abs) {
    const unsigned b = blocks_for(nx, 8);
    launch_grid(shim_make_dim3(b, b, b), shim_make_dim3(8, 8, 8), true, [&] {
        acc_field(reinterpret_cast<double3*>(cell_acc), cell_acc_abs, cell_phi, nx, dx);
    });
}

// apply_acceleration_to_particles / apply_cell_to_particles (p2mesh-kernel.cuh:227-254).
void ref_apply_acc(int64_t n, double* particle_acc, const double* cell_acc, int* pci) {
    launch_grid(shim_make_dim3(blocks_for(n, 512)), shim_make_dim3(512), true, [&] {
        apply_acceleration_to_particles(reinterpret_cast<double3*>(particle_acc),
                                        reinterpret_cast<const double3*>(cell_acc),
                                        reinterpret_cast<ParticleCellInfo*>(pci), (int)n);
    });
}

void ref_apply_cell(int64_t n, double* particle_value, const double* cell_value, int* pci) {
    launch_grid(shim_make_dim3(blocks_for(n, 512)), shim_make_dim3(512), true, [&] {
        apply_cell_to_particles(particle_value, cell_value,
                                reinterpret_cast<ParticleCellInfo*>(pci), (int)n);
    });
}

int ref_max_threads(void) { return omp_get_max_threads(); }

}  // extern "C"
