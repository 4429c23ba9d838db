// oracle/_ref: the reference's ACCEL_kernel with its `real` type set to float.
//
// TEST INFRASTRUCTURE ONLY.  The reference has no FP32 kernel; "the
// reference's own FP32 kernel" is nbody-kernel.cuh:89-142 with real/real3
// mapped to float types.  common.cuh hard-codes `#define real double`, so the
// token `double` itself is redefined to `float` while the headers are read.
// The literal 0.5 in the kernel stays a double literal, exactly as it would in
// a CUDA build with real = float.
#include <omp.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>

#define double float
#include "cuda_runtime.h"
#include "ref_launch.h"
#include "nbody-kernel.cuh"
#undef double

extern "C" {

// ACCEL_kernel (nbody-kernel.cuh:89-142) in FP32 for the listed targets, run as
// gridDim = n, blockDim = 1 (j order 0..n-1).  Inputs are converted from
// double; out (nt x 3) receives the FP32 sum (overwrite semantics).
void ref_accel_f32(int64_t n, const double* pos, const double* mass, const double* eps2,
                   int64_t nt, const int64_t* targets, double* out) {
    dd.NN = (int)n;
    double3* p = new double3[n];  // shim double3 holds floats in this unit
    float* m = new float[n];
    float* e = new float[n];
    for (int64_t i = 0; i < n; ++i) {
        p[i].x = (float)pos[3 * i + 0];
        p[i].y = (float)pos[3 * i + 1];
        p[i].z = (float)pos[3 * i + 2];
        m[i] = (float)mass[i];
        e[i] = (float)eps2[i];
    }
    const int64_t count = targets ? nt : n;
#pragma omp parallel
    {
        double3* acc_one = new double3[n];
#pragma omp for schedule(dynamic, 1)
        for (int64_t k = 0; k < count; ++k) {
            const int64_t i = targets ? targets[k] : k;
            acc_one[i].x = acc_one[i].y = acc_one[i].z = 0.0f;
            threadIdx = shim_dim3{0, 0, 0};
            blockIdx = shim_dim3{(unsigned)i, 0, 0};
            blockDim = shim_dim3{1, 1, 1};
            gridDim = shim_dim3{(unsigned)n, 1, 1};
            ACCEL_kernel(acc_one, p, p, m, e);
            out[3 * k + 0] = acc_one[i].x;
            out[3 * k + 1] = acc_one[i].y;
            out[3 * k + 2] = acc_one[i].z;
        }
        delete[] acc_one;
    }
    delete[] p;
    delete[] m;
    delete[] e;
}

}  // extern "C"
