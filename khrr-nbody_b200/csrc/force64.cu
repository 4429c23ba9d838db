// FP64 direct-sum gravity on sm_100a: the reference's own precision for
// ACCEL_kernel (nbody-kernel.cuh:89-142) and PHI_kernel (nbody-kernel.cuh:43-86),
// behind the state API (KHRR_FP64).  Every run reports its FP32 forces and
// its energy drift against this path.
//
// Two forms.  fp64_pair_kernel (the default; below) evaluates each unordered
// pair once for both bodies on the FP32 pair kernel's plan.  fp64_force_kernel
// (KHRR_FP64_ONESIDED=1) evaluates every ordered pair: the one-sided
// kernel's queue of WorkItems (system, i tile of 512 bodies, j chunk),
// pulled by a persistent grid with one atomic per item; each item writes its
// FP64 sums to its partial slot, which the corrector adds in FP64.
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

// The symmetric form of the same sums (the default FP64 pass): every
// unordered pair of a system evaluated once for both bodies, on the FP32
// pair kernel's work plan (1024-body blocks, a block row cut into chunks,
// the block's own tiles one-sided).  A CTA holds its i block in registers
// (256 threads x 4 bodies) and streams the chunk's j tiles of 128 bodies
// through a double-buffered shared-memory tile; the reaction on a j body is
// summed across a warp by handing it from lane to lane (lane l evaluates
// body (l + s) mod 32 of a 32-body sub-chunk at step s and passes its running
// reaction to lane l - 1), then across the 8 warps in shared memory, and
// added with FP64 atomics into the body's sums (one partial slot), as are
// the i block's sums at the item's end.  Per unordered pair: d (3 sub),
// r^2 (1 add, 3 fma), rsqrt, r^-3 (2 mul), m_j r^-3 and m_i r^-3 (2 mul),
// the two sides (6 fma; +2 fma for the potential).  The sums are FP64
// throughout; their order differs from the reference's j loop (and between
// runs, through the atomics) only at the level of FP64 rounding.
#ifndef KHRR_F64P_NT
#define KHRR_F64P_NT 256
#endif
#ifndef KHRR_F64P_UNROLL
#define KHRR_F64P_UNROLL 2
#endif
#ifndef KHRR_F64P_CTAS
#define KHRR_F64P_CTAS 2
#endif
constexpr int PNT = KHRR_F64P_NT;         // threads per CTA
constexpr int kF64PUnroll = KHRR_F64P_UNROLL;
constexpr int PK = kPairBlock / PNT;      // i bodies per thread (4)
constexpr int PJT = kPairTile;            // j bodies per tile (128)
constexpr int PW = PNT / 32;              // warps (8)
static_assert(PNT * PK == kPairBlock && PJT == 128 && PJT % 32 == 0 && PNT >= PJT, "pair shapes");

template <bool ACC, bool PHI>
__global__ void __launch_bounds__(PNT, KHRR_F64P_CTAS) fp64_pair_kernel(const F64PairArgs a) {
    constexpr int NC = (ACC ? 3 : 0) + (PHI ? 1 : 0), CP = NC - 1;
    __shared__ double tx[2][PJT], ty[2][PJT], tz[2][PJT], tm[2][PJT], th[2][PJT];
    __shared__ double jw[PW][NC][PJT];
    __shared__ int s_item;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int src = (lane + 1) & 31;
    for (;;) {
        if (tid == 0) s_item = static_cast<int>(atomicAdd(a.queue, 1u));
        __syncthreads();
        const int it = s_item;
        if (it >= a.n_items) break;
        const PairItem w = a.items[it];
        // The i bodies (index i_begin + k PNT + tid); lanes past the block's
        // end have no mass (and a positive softening term).
        double xi[PK], yi[PK], zi[PK], hi[PK], mi[PK], ai[NC][PK];
#pragma unroll
        for (int k = 0; k < PK; ++k) {
            const int64_t i = w.i_begin + k * PNT + tid;
            const bool in = i < w.i_end;
            xi[k] = in ? a.pos[3 * i] : 0.0;
            yi[k] = in ? a.pos[3 * i + 1] : 0.0;
            zi[k] = in ? a.pos[3 * i + 2] : 0.0;
            hi[k] = in ? 0.5 * a.eps2[i] : 1.0;
            mi[k] = in ? a.mass[i] : 0.0;
#pragma unroll
            for (int c = 0; c < NC; ++c) ai[c][k] = 0.0;
        }
        const int ntiles = (w.j_end - w.j_begin) / PJT;
        // Register copy of the next tile's body tid (threads < PJT).
        double nx = 0.0, ny = 0.0, nz = 0.0, nm = 0.0, nh = 0.0;
        auto fetch = [&](int t) {
            if (tid < PJT) {
                const int64_t j = w.j_begin + static_cast<int64_t>(t) * PJT + tid;
                nx = a.pos[3 * j];
                ny = a.pos[3 * j + 1];
                nz = a.pos[3 * j + 2];
                nm = a.mass[j];
                nh = 0.5 * a.eps2[j];
            }
        };
        fetch(0);
        for (int t = 0; t < ntiles; ++t) {
            const int b = t & 1;
            if (tid < PJT) {
                tx[b][tid] = nx;
                ty[b][tid] = ny;
                tz[b][tid] = nz;
                tm[b][tid] = nm;
                th[b][tid] = nh;
            }
            __syncthreads();  // the tile is staged; the last tile's reactions were read
            if (t + 1 < ntiles) fetch(t + 1);
            const int jt0 = w.j_begin + t * PJT;
            const bool sym = jt0 >= w.diag_end;
#pragma unroll 1
            for (int c0 = 0; c0 < PJT; c0 += 32) {
                double r[NC];
#pragma unroll
                for (int c = 0; c < NC; ++c) r[c] = 0.0;
#pragma unroll kF64PUnroll
                for (int s = 0; s < 32; ++s) {
                    const int j = c0 + ((lane + s) & 31);
                    const double xj = tx[b][j], yj = ty[b][j], zj = tz[b][j], mj = tm[b][j], hj = th[b][j];
#pragma unroll
                    for (int k = 0; k < PK; ++k) {
                        const double dx = xj - xi[k], dy = yj - yi[k], dz = zj - zi[k];
                        double r2 = hi[k] + hj;
                        r2 = fma(dx, dx, r2);
                        r2 = fma(dy, dy, r2);
                        r2 = fma(dz, dz, r2);
                        const double inv = rsqrt(r2);
                        if (ACC) {
                            const double i3 = inv * inv * inv;
                            const double fi = mj * i3;
                            ai[0][k] = fma(dx, fi, ai[0][k]);
                            ai[1][k] = fma(dy, fi, ai[1][k]);
                            ai[2][k] = fma(dz, fi, ai[2][k]);
                            if (sym) {
                                const double fj = mi[k] * i3;
                                r[0] = fma(dx, fj, r[0]);
                                r[1] = fma(dy, fj, r[1]);
                                r[2] = fma(dz, fj, r[2]);
                            }
                        }
                        if (PHI) {
                            ai[CP][k] = fma(mj, inv, ai[CP][k]);
                            if (sym) r[CP] = fma(mi[k], inv, r[CP]);
                        }
                    }
                    if (sym) {
#pragma unroll
                        for (int c = 0; c < NC; ++c) r[c] = __shfl_sync(0xffffffffu, r[c], src);
                    }
                }
                if (sym) {
#pragma unroll
                    for (int c = 0; c < NC; ++c) jw[warp][c][c0 + lane] = r[c];
                }
            }
            if (sym) {
                __syncthreads();  // every warp's reactions of the tile are in jw
                if (tid < PJT) {
                    const int64_t j = jt0 + tid;
                    if (j < w.real_end) {
                        double s4[NC];
#pragma unroll
                        for (int c = 0; c < NC; ++c) {
                            double v = 0.0;
#pragma unroll
                            for (int q = 0; q < PW; ++q) v += jw[q][c][tid];
                            s4[c] = v;
                        }
                        // The reaction on j is minus the sum of m_i d / r^3
                        // (d = x_j - x_i); the potential's sum keeps its sign.
                        if (ACC) {
                            atomicAdd(&a.sums[j].x, -s4[0]);
                            atomicAdd(&a.sums[j].y, -s4[1]);
                            atomicAdd(&a.sums[j].z, -s4[2]);
                        }
                        if (PHI) atomicAdd(&a.sums[j].w, s4[CP]);
                    }
                }
            }
        }
#pragma unroll
        for (int k = 0; k < PK; ++k) {
            const int64_t i = w.i_begin + k * PNT + tid;
            if (i < w.i_end && i < w.real_end) {
                if (ACC) {
                    atomicAdd(&a.sums[i].x, ai[0][k]);
                    atomicAdd(&a.sums[i].y, ai[1][k]);
                    atomicAdd(&a.sums[i].z, ai[2][k]);
                }
                if (PHI) atomicAdd(&a.sums[i].w, ai[CP][k]);
            }
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

cudaError_t launch_fp64_pair(const F64PairArgs& a, bool acc, bool phi, int grid, cudaStream_t s) {
    if (a.n_items < 1) return cudaSuccess;
    if (acc && phi) fp64_pair_kernel<true, true><<<grid, PNT, 0, s>>>(a);
    else if (acc) fp64_pair_kernel<true, false><<<grid, PNT, 0, s>>>(a);
    else fp64_pair_kernel<false, true><<<grid, PNT, 0, s>>>(a);
    return cudaGetLastError();
}

int fp64_pair_ctas(int sm_count) {
    int occ = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fp64_pair_kernel<true, true>, PNT, 0) != cudaSuccess ||
        occ < 1)
        occ = 1;
    return occ * sm_count;
}

int fp64_force_ctas(int sm_count) {
    int occ = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fp64_force_kernel<true, true>, NT, 0) != cudaSuccess ||
        occ < 1)
        occ = 1;
    return occ * sm_count;
}

}  // namespace khrr
