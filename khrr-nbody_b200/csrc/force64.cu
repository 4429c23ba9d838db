// FP64 direct-sum gravity on sm_100a: the reference's own precision for
// ACCEL_kernel (nbody-kernel.cuh:89-142) and PHI_kernel (nbody-kernel.cuh:43-86),
// behind the state API (KHRR_FP64).  Every run reports its FP32 forces and
// its energy drift against this path.
//
// Work decomposition: the one-sided kernel's queue of WorkItems (system, i
// tile of 512 bodies, j chunk), pulled by a persistent grid with one atomic
// per item; each item writes its FP64 sums to its partial slot, which the
// corrector adds in FP64.
//
// Per item: 128 threads hold 4 i bodies each (FP64 position, softening and
// sums in registers); the chunk's j bodies pass through a double-buffered
// shared-memory tile of 128 (x, y, z, m, eps^2/2 as doubles), the next tile
// loaded into registers while the current one is evaluated, one barrier per
// tile.  Per pair: d (3 sub), r^2 = h_i + h_j + d.d (1 add, 3 fma), r^-1 =
// rsqrt (CUDA's double-precision function), m r^-3 (3 mul), the sums (3 fma,
// + 1 fma for the potential).  FP64-pipe bound: B200 runs FP64 at half the
// FP32 rate.
//
// Terms: the softening enters as (eps2_i + eps2_j) / 2, the self pair gives
// zero acceleration and m / eps to the potential, ghosts (zero mass) give
// nothing: the reference's sums, evaluated in IEEE double.
#include <cstdint>

#include "khrr_internal.h"

namespace khrr {
namespace {

#ifndef KHRR_F64_NT
#define KHRR_F64_NT 128
#endif
constexpr int NT = KHRR_F64_NT;   // threads per CTA
constexpr int K = kF64ITile / NT;  // i bodies per thread
constexpr int JT = 128;            // j bodies per shared-memory tile
constexpr int FP = (JT + NT - 1) / NT;  // j bodies each thread stages per tile
static_assert(NT * K == kF64ITile && JT == kPad && (JT % NT == 0 || NT % JT == 0), "tile shapes");

constexpr int kMinCtas = NT >= 128 ? 512 / NT : 4;  // resident CTAs per SM the registers aim at

template <bool ACC, bool PHI>
__global__ void __launch_bounds__(NT, kMinCtas) fp64_force_kernel(const F64Args a) {
    __shared__ double sx[2][JT], sy[2][JT], sz[2][JT], sm[2][JT], sh[2][JT];
    __shared__ int s_item;
    const int tid = threadIdx.x;
    for (;;) {
        if (tid == 0) s_item = static_cast<int>(atomicAdd(a.queue, 1u));
        __syncthreads();
        const int it = s_item;
        if (it >= a.n_items) break;
        const WorkItem w = a.items[it];

        double xi[K], yi[K], zi[K], hi[K], ax[K], ay[K], az[K], ph[K];
#pragma unroll
        for (int k = 0; k < K; ++k) {
            const int i = w.i_begin + k * NT + tid;
            const bool in = i < w.i_end;
            xi[k] = in ? a.pos[3 * static_cast<int64_t>(i)] : 0.0;
            yi[k] = in ? a.pos[3 * static_cast<int64_t>(i) + 1] : 0.0;
            zi[k] = in ? a.pos[3 * static_cast<int64_t>(i) + 2] : 0.0;
            hi[k] = in ? 0.5 * a.eps2[i] : 1.0;
            ax[k] = ay[k] = az[k] = ph[k] = 0.0;
        }

        const int ntiles = (w.j_end - w.j_begin) / JT;
        // Register copy of the next tile's bodies tid, tid + NT, ... (< JT).
        double nx[FP], ny[FP], nz[FP], nm[FP], nh[FP];
        auto fetch = [&](int t) {
#pragma unroll
            for (int q = 0; q < FP; ++q) {
                const int jj = tid + q * NT;
                if (jj >= JT) break;
                const int64_t j = w.j_begin + static_cast<int64_t>(t) * JT + jj;
                nx[q] = a.pos[3 * j];
                ny[q] = a.pos[3 * j + 1];
                nz[q] = a.pos[3 * j + 2];
                nm[q] = a.mass[j];
                nh[q] = 0.5 * a.eps2[j];
            }
        };
        fetch(0);
        for (int t = 0; t < ntiles; ++t) {
            const int b = t & 1;
#pragma unroll
            for (int q = 0; q < FP; ++q) {
                const int jj = tid + q * NT;
                if (jj >= JT) break;
                sx[b][jj] = nx[q];
                sy[b][jj] = ny[q];
                sz[b][jj] = nz[q];
                sm[b][jj] = nm[q];
                sh[b][jj] = nh[q];
            }
            __syncthreads();
            if (t + 1 < ntiles) fetch(t + 1);
#pragma unroll 2
            for (int jj = 0; jj < JT; ++jj) {
                const double xj = sx[b][jj], yj = sy[b][jj], zj = sz[b][jj], mj = sm[b][jj], hj = sh[b][jj];
#pragma unroll
                for (int k = 0; k < K; ++k) {
                    const double dx = xj - xi[k], dy = yj - yi[k], dz = zj - zi[k];
                    double r2 = hi[k] + hj;
                    r2 = fma(dx, dx, r2);
                    r2 = fma(dy, dy, r2);
                    r2 = fma(dz, dz, r2);
                    const double inv = rsqrt(r2);
                    if (ACC) {
                        const double k3 = mj * (inv * inv * inv);
                        ax[k] = fma(dx, k3, ax[k]);
                        ay[k] = fma(dy, k3, ay[k]);
                        az[k] = fma(dz, k3, az[k]);
                    }
                    if (PHI) ph[k] = fma(mj, inv, ph[k]);
                }
            }
        }
        double4* out = a.part + static_cast<long long>(w.slot) * a.npad;
#pragma unroll
        for (int k = 0; k < K; ++k) {
            const int i = w.i_begin + k * NT + tid;
            if (i < w.i_end) out[i] = make_double4(ax[k], ay[k], az[k], ph[k]);
        }
        // Every thread is done with the item (and s_item) before the next pull.
        __syncthreads();
    }
}

}  // namespace

cudaError_t launch_fp64_force(const F64Args& a, bool acc, bool phi, int grid, cudaStream_t s) {
    if (a.n_items < 1) return cudaSuccess;
    if (acc && phi) fp64_force_kernel<true, true><<<grid, NT, 0, s>>>(a);
    else if (acc) fp64_force_kernel<true, false><<<grid, NT, 0, s>>>(a);
    else fp64_force_kernel<false, true><<<grid, NT, 0, s>>>(a);
    return cudaGetLastError();
}

int fp64_force_ctas(int sm_count) {
    int occ = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fp64_force_kernel<true, true>, NT, 0) != cudaSuccess ||
        occ < 1)
        occ = 1;
    return occ * sm_count;
}

}  // namespace khrr
