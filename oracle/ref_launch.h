// Host launch emulation for the reference kernels (TEST INFRASTRUCTURE ONLY).
//
// The reference kernels compiled through refshim/ read threadIdx/blockIdx/
// blockDim/gridDim from thread-local globals.  These helpers set them and run
// the kernel body the way a CUDA launch would:
//   launch_grid  - every thread of every block, blocks in parallel (OpenMP),
//                  threads of a block in order; valid for kernels with no
//                  __syncthreads().  parallel=false runs everything on the
//                  calling thread in launch order (deterministic atomics).
//   launch_team  - one OpenMP team of blockDim threads per block, blocks in
//                  order; needs a translation unit built with KHRR_SHIM_TEAM
//                  so that __syncthreads() is a team barrier.
#pragma once
#include <omp.h>

#include <cstdio>
#include <cstdlib>

#include "cuda_runtime.h"

inline shim_dim3 shim_make_dim3(unsigned x, unsigned y = 1, unsigned z = 1) {
    return shim_dim3{x, y, z};
}

template <class F>
void launch_grid(shim_dim3 grid, shim_dim3 block, bool parallel, F body) {
    const long nblocks = (long)grid.x * grid.y * grid.z;
    const long nthr = (long)block.x * block.y * block.z;
    auto run_block = [&](long b) {
        blockIdx = shim_dim3{(unsigned)(b % grid.x), (unsigned)((b / grid.x) % grid.y),
                             (unsigned)(b / ((long)grid.x * grid.y))};
        blockDim = block;
        gridDim = grid;
        for (long t = 0; t < nthr; ++t) {
            threadIdx = shim_dim3{(unsigned)(t % block.x), (unsigned)((t / block.x) % block.y),
                                  (unsigned)(t / ((long)block.x * block.y))};
            body();
        }
    };
    if (parallel) {
#pragma omp parallel for schedule(dynamic, 4)
        for (long b = 0; b < nblocks; ++b) run_block(b);
    } else {
        for (long b = 0; b < nblocks; ++b) run_block(b);
    }
}

template <class F>
void launch_team(shim_dim3 grid, shim_dim3 block, F body) {
    const int nthr = (int)(block.x * block.y * block.z);
    omp_set_dynamic(0);
    const long nblocks = (long)grid.x * grid.y * grid.z;
    for (long b = 0; b < nblocks; ++b) {
        int bad = 0;
#pragma omp parallel num_threads(nthr) shared(bad)
        {
            if (omp_get_num_threads() != nthr) {
#pragma omp atomic write
                bad = 1;
            } else {
                const unsigned t = (unsigned)omp_get_thread_num();
                threadIdx = shim_dim3{t % block.x, (t / block.x) % block.y, t / (block.x * block.y)};
                blockIdx = shim_dim3{(unsigned)(b % grid.x), (unsigned)((b / grid.x) % grid.y),
                                     (unsigned)(b / ((long)grid.x * grid.y))};
                blockDim = block;
                gridDim = grid;
                body();
            }
        }
        if (bad) {
            std::fprintf(stderr, "launch_team: OpenMP refused a team of %d threads\n", nthr);
            std::abort();
        }
    }
}
