// oracle/_ref: reference kernels that need real block barriers.
//
// TEST INFRASTRUCTURE ONLY.  PHI_kernel (nbody-kernel.cuh:43-86),
// ACCEL_kernel (:89-142) and computePrefixSums (p2mesh-kernel.cuh:62-105)
// cooperate through __shared__ memory and __syncthreads(); here every CUDA
// block runs as an OpenMP team of blockDim threads with a team barrier, so
// their block semantics (including the reference's partial scan, D2) are
// reproduced exactly.  Small sizes only: each block is a 512-thread team.
#define KHRR_SHIM_TEAM 1
#include <omp.h>

#include <cstdint>

#include "cuda_runtime.h"
#include "ref_launch.h"

#include "nbody-kernel.cuh"
#include "p2mesh-kernel.cuh"

extern "C" {

// PHI_kernel with the reference launch <<<n/512, 512>>> (nbody.cu:1468);
// phi (n) is accumulated into (phi -= sum); n % 512 == 0.
int ref_phi_team(int64_t n, const double* pos, const double* mass, const double* eps2,
                 double* phi) {
    if (n % BLOCK_SIZE) return -1;
    const double3* p = reinterpret_cast<const double3*>(pos);
    launch_team(shim_make_dim3((unsigned)(n / BLOCK_SIZE)), shim_make_dim3(BLOCK_SIZE),
                [&] { PHI_kernel(phi, p, p, mass, eps2); });
    return 0;
}

// ACCEL_kernel with the reference launch <<<n/512, 512>>> (nbody.cu:1475);
// acc (n x 3) is accumulated into; n % 512 == 0.
int ref_accel_team(int64_t n, const double* pos, const double* mass, const double* eps2,
                   double* acc) {
    if (n % BLOCK_SIZE) return -1;
    dd.NN = (int)n;
    const double3* p = reinterpret_cast<const double3*>(pos);
    launch_team(shim_make_dim3((unsigned)(n / BLOCK_SIZE)), shim_make_dim3(BLOCK_SIZE),
                [&] { ACCEL_kernel(reinterpret_cast<double3*>(acc), p, p, mass, eps2); });
    return 0;
}

// computePrefixSums with <<<ceil(C/512), 512>>> (nbody.cu:165); maxpbc has
// ceil(C/512) entries and must be zeroed by the caller.
void ref_prefix_team(int64_t ncells, int* cell_info, int* maxpbc) {
    const unsigned nb = (unsigned)((ncells + BLOCK_SIZE - 1) / BLOCK_SIZE);
    launch_team(shim_make_dim3(nb), shim_make_dim3(BLOCK_SIZE), [&] {
        computePrefixSums(reinterpret_cast<CellInfo*>(cell_info), maxpbc, (int)ncells);
    });
}

}  // extern "C"
