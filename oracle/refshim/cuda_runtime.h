// Host-compilation shim for the reference's CUDA kernel headers.
//
// TEST INFRASTRUCTURE ONLY.  This header lets the reference's unmodified
// kernel headers (nbody/include/{common,nbody-kernel,p2mesh-kernel,
// wave-kernel}.cuh) compile as plain host C++ so that oracle/_ref can run the
// reference's own arithmetic on the CPU.  It supplies the few CUDA vector
// types and qualifiers those headers use; it is never linked into the product.
//
// Two execution models are selected by the including translation unit:
//   KHRR_SHIM_TEAM     one OpenMP team per CUDA block, one OpenMP thread per
//                      CUDA thread; __syncthreads() is an OpenMP barrier and
//                      __shared__ arrays are function statics shared by the
//                      team (exact block semantics, used for barrier kernels).
//   (default)          independent threads: every "block" runs on its own
//                      OpenMP worker, __shared__ arrays are thread-local and
//                      __syncthreads() is a no-op (valid for kernels launched
//                      with blockDim = 1, e.g. ACCEL_kernel per target body).
#pragma once
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>

struct double2 { double x, y; };
struct double3 { double x, y, z; };
struct int3 { int x, y, z; };
struct shim_dim3 { unsigned x, y, z; };

inline double2 make_double2(double x, double y) { return double2{x, y}; }
inline double3 make_double3(double x, double y, double z) { return double3{x, y, z}; }
inline int3 make_int3(int x, int y, int z) { return int3{x, y, z}; }

// Launch coordinates, one copy per host thread (defined in ref_launch.cpp).
extern thread_local shim_dim3 threadIdx, blockIdx, blockDim, gridDim;

// Qualifiers: everything the headers define gets internal linkage, so that
// several translation units (FP64, FP32, team mode) can each include them.
#define __global__ static
#define __device__ static
#define __host__
#define __constant__ static
#define __forceinline__ inline

#ifdef KHRR_SHIM_TEAM
#define __shared__ static
#define __syncthreads() _Pragma("omp barrier")
#else
#define __shared__ static thread_local
#define __syncthreads() ((void)0)
#endif

static inline int atomicAdd(int* addr, int v) {
    return __atomic_fetch_add(addr, v, __ATOMIC_SEQ_CST);
}

static inline double atomicAdd(double* addr, double v) {
    uint64_t* p = reinterpret_cast<uint64_t*>(addr);
    uint64_t old_bits = __atomic_load_n(p, __ATOMIC_SEQ_CST);
    for (;;) {
        double old_val;
        std::memcpy(&old_val, &old_bits, sizeof(double));
        double new_val = old_val + v;
        uint64_t new_bits;
        std::memcpy(&new_bits, &new_val, sizeof(double));
        if (__atomic_compare_exchange_n(p, &old_bits, new_bits, false,
                                        __ATOMIC_SEQ_CST, __ATOMIC_SEQ_CST))
            return old_val;
    }
}
