// p2mesh on sm_100a: binning, prefix sums, deposits, the damped-wave Poisson
// stencil, the mesh gradient and the NGP gather.
//
// Replaces assignParticlesToCells, computePrefixSums, adjustGlobalPrefixSums,
// computeCellMassesUnsorted, computeCellPhiUnsorted, acc_field and the
// apply_* gathers (p2mesh-kernel.cuh:11-254) and wave_diss_iteration
// (wave-kernel.cuh:5-103).  All of it is HBM (or L2) bound integer/FP64/FP32
// streaming; nothing here is reshaped for tensor cores.
//
// Binning: the cell of a body is the reference's (IEEE FP64 division,
// truncation toward zero, clamps, including the iz clamp to gridSize.y - 1 and
// the id iz*gx*gy + iy*gz + ix).  Slots come from atomics aggregated per warp:
// lanes of a warp that hit the same cell take consecutive slots with one
// atomic (__match_any_sync), and their masses are summed by the group leader
// before one FP64 atomic, so dense cells cost one atomic per warp instead of
// one per body.
//
// Scan: single pass over 4096-cell tiles in three launches (tile/block totals,
// one CTA scanning the 512-cell block totals, per-tile downsweep).  The
// inclusive block-total scan is exactly the reference's maxPBC array, and the
// reference's start_id (the total of earlier 512-cell blocks, its in-block
// scan being discarded) is read off it; the true exclusive scan is produced
// alongside.
//
// This file is built without FMA contraction: the FP64 kernels evaluate the
// reference's expressions in IEEE double; the FP32 stencil uses explicit fmaf.
#include <cmath>
#include <cstdint>

#include "khrr_internal.h"

namespace khrr {
namespace {

constexpr double kPi = 3.14159265358979;  // the reference's PI (common.cuh:7)

int grid_for(int64_t n, int block) {
    int64_t g = (n + block - 1) / block;
    if (g > 148 * 32) g = 148 * 32;
    if (g < 1) g = 1;
    return static_cast<int>(g);
}

// Cell coordinate of one axis: (int)((p - lo) / cs) clamped to [0, g - 1],
// with the CUDA conversion's behaviour for quotients outside the int range.
__device__ __forceinline__ int cell_axis(double p, double lo, double cs, int g) {
    const double q = (p - lo) / cs;
    if (q >= static_cast<double>(g - 1)) return g - 1;
    if (q > -1.0) return static_cast<int>(q);
    return 0;
}

__global__ void assign_kernel(const double* __restrict__ pos, int64_t n, const MeshGeom m, int2* __restrict__ pci,
                              int* __restrict__ counter, int counter_stride, int* __restrict__ count2,
                              int count2_stride, const double* __restrict__ mass, double* __restrict__ cell_mass) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int ix = cell_axis(pos[3 * i], m.lo[0], m.cs[0], m.g[0]);
    const int iy = cell_axis(pos[3 * i + 1], m.lo[1], m.cs[1], m.g[1]);
    const int iz = cell_axis(pos[3 * i + 2], m.lo[2], m.cs[2], m.g[1]);
    const int c = iz * m.g[0] * m.g[1] + iy * m.g[2] + ix;

    const unsigned lane = threadIdx.x & 31u;
    const unsigned peers = __match_any_sync(__activemask(), c);
    const unsigned leader = __ffs(peers) - 1u;
    const int rank = __popc(peers & ((1u << lane) - 1u));
    int base = 0;
    if (lane == leader) {
        const int k = __popc(peers);
        base = atomicAdd(&counter[static_cast<int64_t>(c) * counter_stride], k);
        if (count2) atomicAdd(&count2[static_cast<int64_t>(c) * count2_stride], k);
    }
    base = __shfl_sync(peers, base, leader);
    pci[i] = make_int2(c, base + rank);

    if (cell_mass) {
        // Group sum in lane order, then one FP64 atomic per group.
        double s = 0.0;
        unsigned rest = peers;
        const double mi = mass[i];
        while (rest) {
            const int src = __ffs(rest) - 1;
            const double v = __shfl_sync(peers, mi, src);
            s += v;
            rest &= rest - 1u;
        }
        if (lane == leader) atomicAdd(&cell_mass[c], s);
    }
}

// ---- prefix sums -----------------------------------------------------------
constexpr int kScanThreads = 512;
constexpr int kScanPer = 8;                              // cells per thread
constexpr int kScanTile = kScanThreads * kScanPer;       // 4096 cells
constexpr int kRefBlock = 512;                           // the reference's BLOCK_SIZE
constexpr int kBlocksPerTile = kScanTile / kRefBlock;    // 8

__device__ __forceinline__ int warp_sum(int v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Totals of the 512-cell blocks of one 4096-cell tile.
__global__ void scan_block_totals_kernel(const int* __restrict__ count, int stride, int64_t ncells,
                                         int* __restrict__ block_tot) {
    const int64_t t = blockIdx.x;
    const int tid = threadIdx.x;
    const int64_t c0 = t * kScanTile + static_cast<int64_t>(tid) * kScanPer;
    int s = 0;
#pragma unroll
    for (int k = 0; k < kScanPer; ++k) {
        const int64_t c = c0 + k;
        if (c < ncells) s += count[c * stride];
    }
    // 64 threads = one 512-cell block = two warps.
    s = warp_sum(s);
    __shared__ int ws[kScanThreads / 32];
    if ((tid & 31) == 0) ws[tid >> 5] = s;
    __syncthreads();
    if (tid < kBlocksPerTile) {
        const int64_t b = t * kBlocksPerTile + tid;
        if (b * kRefBlock < ncells) block_tot[b] = ws[2 * tid] + ws[2 * tid + 1];
    }
}

// One CTA: inclusive scan of the block totals (in place) = maxPBC.
__global__ void scan_blocks_kernel(int* __restrict__ tot, int64_t nb) {
    constexpr int T = 1024;
    __shared__ int part[T];
    const int tid = threadIdx.x;
    const int64_t per = (nb + T - 1) / T;
    const int64_t b0 = tid * per;
    int s = 0;
    for (int64_t b = b0; b < b0 + per && b < nb; ++b) s += tot[b];
    part[tid] = s;
    __syncthreads();
    for (int o = 1; o < T; o <<= 1) {  // Hillis-Steele inclusive scan of thread totals
        const int v = tid >= o ? part[tid - o] : 0;
        __syncthreads();
        part[tid] += v;
        __syncthreads();
    }
    int run = tid ? part[tid - 1] : 0;
    for (int64_t b = b0; b < b0 + per && b < nb; ++b) {
        run += tot[b];
        tot[b] = run;
    }
}

// Per tile: exclusive in-tile scan + tile offset -> the true start of every
// cell; the reference view from maxPBC.
__global__ void scan_downsweep_kernel(const int* __restrict__ count, int cstride, int64_t ncells,
                                      const int* __restrict__ maxpbc, int* __restrict__ start, int sstride,
                                      int* __restrict__ start_ref, int rstride) {
    const int64_t t = blockIdx.x;
    const int tid = threadIdx.x;
    const int64_t c0 = t * kScanTile + static_cast<int64_t>(tid) * kScanPer;
    int v[kScanPer];
    int s = 0;
#pragma unroll
    for (int k = 0; k < kScanPer; ++k) {
        const int64_t c = c0 + k;
        v[k] = c < ncells ? count[c * cstride] : 0;
        s += v[k];
    }
    // Exclusive scan of the 512 thread totals.
    const int lane = tid & 31, w = tid >> 5;
    int incl = s;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += y;
    }
    __shared__ int wsum[kScanThreads / 32];
    if (lane == 31) wsum[w] = incl;
    __syncthreads();
    if (w == 0) {
        int x = lane < kScanThreads / 32 ? wsum[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        if (lane < kScanThreads / 32) wsum[lane] = x;
    }
    __syncthreads();
    const int tile_off = t > 0 ? maxpbc[t * kBlocksPerTile - 1] : 0;
    int run = tile_off + (w > 0 ? wsum[w - 1] : 0) + (incl - s);
#pragma unroll
    for (int k = 0; k < kScanPer; ++k) {
        const int64_t c = c0 + k;
        if (c < ncells) {
            if (start) start[c * sstride] = run;
            if (start_ref) {
                const int64_t b = c / kRefBlock;
                start_ref[c * rstride] = b > 0 ? maxpbc[b - 1] : 0;
            }
        }
        run += v[k];
    }
}

// computeCellPhiUnsorted: cell_phi[c] += phi_i / count[c].
__global__ void cell_phi_kernel(const double* __restrict__ phi, const int2* __restrict__ pci,
                                const int* __restrict__ count, int cstride, int64_t n, double* __restrict__ cell_phi) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int c = pci[i].x;
    atomicAdd(&cell_phi[c], phi[i] / count[static_cast<int64_t>(c) * cstride]);
}

// ---- wave stencil --------------------------------------------------------------
__device__ __forceinline__ int64_t at3(int x, int y, int z, int nx) {
    return static_cast<int64_t>(x) + static_cast<int64_t>(y) * nx + static_cast<int64_t>(z) * nx * nx;
}

// Sponge of wave-kernel.cuh:32-60 (coordinates ix*dx, not centred; the x
// test compares against -(L - bc)).
__device__ __forceinline__ double wave_diss(const WaveConsts& W, int ix, int iy, int iz) {
    const double x = ix * W.dx, y = iy * W.dx, z = iz * W.dx;
    const double L = W.sim_l - W.bc_l;
    double d = W.diss_base;
    if (x > -L) d += W.diss_extra * fabs(x - L) * fabs(x - L);
    else if (x < -L) d += W.diss_extra * fabs(x + L) * fabs(x + L);
    if (y > L) d += W.diss_extra * fabs(y - L) * fabs(y - L);
    else if (y < -L) d += W.diss_extra * fabs(y + L) * fabs(y + L);
    if (z > L) d += W.diss_extra * fabs(z - L) * fabs(z - L);
    else if (z < -L) d += W.diss_extra * fabs(z + L) * fabs(z + L);
    return d;
}

// wave_diss_iteration in FP64, the reference's expressions.
__global__ void wave_f64_kernel(double* __restrict__ phi_new, const double* __restrict__ phi,
                                const double* __restrict__ phi_old, const double* __restrict__ mass,
                                const WaveConsts W) {
    const int NX = W.nx;
    const int ix = blockIdx.x * blockDim.x + threadIdx.x;
    const int iy = blockIdx.y * blockDim.y + threadIdx.y;
    const int iz = blockIdx.z;
    if (ix >= NX || iy >= NX || iz >= NX) return;
    const int64_t at = at3(ix, iy, iz, NX);
    if (ix == 0 || ix == NX - 1 || iy == 0 || iy == NX - 1 || iz == 0 || iz == NX - 1) {
        phi_new[at] = 0.0;
        return;
    }
    const double DX = W.dx, C = W.c, DT = W.dt;
    const double rho = mass[at] / (DX * DX * DX);
    const double f = 4 * kPi * 1.0 * rho;
    const double diss = wave_diss(W, ix, iy, iz);
    const double Q = diss * C * DT * 0.5;
    const double Wt = 1 + Q;
    const double K = C * C * (DT * DT) / (DX * DX);
    const double KM = K / Wt;
    const double KF = -(C * C) * (DT * DT) / Wt;
    const double KA = 2 * (1. - 3 * K) / Wt;
    const double KO = (Q - 1.) / Wt;
    phi_new[at] = phi[at3(ix - 1, iy, iz, NX)] * KM + phi[at3(ix + 1, iy, iz, NX)] * KM +
                  phi[at3(ix, iy - 1, iz, NX)] * KM + phi[at3(ix, iy + 1, iz, NX)] * KM +
                  phi[at3(ix, iy, iz - 1, NX)] * KM + phi[at3(ix, iy, iz + 1, NX)] * KM + phi[at] * KA +
                  phi_old[at] * KO + f * KF;
}

// The same step in FP32 storage and arithmetic.  The sponge is separable,
// diss = base + sx[ix] + sy[iy] + sz[iz] (per-axis tables built in FP64 on the
// host); per cell: Q = diss c dt / 2, w = 1 / (1 + Q), and
//   phi_new = nb K w + phi (2 (1 - 3K)) w + phi_old (Q - 1) w + mass S w,
// with nb the six-neighbour sum and S = -c^2 dt^2 4 pi / dx^3.  With resid,
// sum (phi_new - phi)^2 and sum phi_new^2 are accumulated in FP64.
__global__ void wave_f32_kernel(float* __restrict__ phi_new, const float* __restrict__ phi,
                                const float* __restrict__ phi_old, const float* __restrict__ mass,
                                const WaveF32 W, double* __restrict__ resid) {
    const int NX = W.nx;
    const int ix = blockIdx.x * blockDim.x + threadIdx.x;
    const int iy = blockIdx.y * blockDim.y + threadIdx.y;
    const int iz = blockIdx.z;
    double d2 = 0.0, n2 = 0.0;
    if (ix < NX && iy < NX) {
        const int64_t at = at3(ix, iy, iz, NX);
        float out = 0.0f;
        const float c0 = phi[at];
        if (!(ix == 0 || ix == NX - 1 || iy == 0 || iy == NX - 1 || iz == 0 || iz == NX - 1)) {
            const int64_t sy = NX, sz = static_cast<int64_t>(NX) * NX;
            const float nb = ((phi[at - 1] + phi[at + 1]) + (phi[at - sy] + phi[at + sy])) + (phi[at - sz] + phi[at + sz]);
            const float diss = ((W.diss_base + W.sx[ix]) + W.sy[iy]) + W.sz[iz];
            const float Q = diss * W.cdt_half;
            const float w = 1.0f / (1.0f + Q);
            out = fmaf(nb, W.K * w, fmaf(c0, W.A * w, fmaf(phi_old[at], (Q - 1.0f) * w, mass[at] * (W.S * w))));
        }
        phi_new[at] = out;
        if (resid) {
            const double dd = static_cast<double>(out) - static_cast<double>(c0);
            d2 = dd * dd;
            n2 = static_cast<double>(out) * static_cast<double>(out);
        }
    }
    if (resid) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            d2 += __shfl_xor_sync(0xffffffffu, d2, o);
            n2 += __shfl_xor_sync(0xffffffffu, n2, o);
        }
        if ((threadIdx.x & 31) == 0) {
            atomicAdd(&resid[0], d2);
            atomicAdd(&resid[1], n2);
        }
    }
}

// acc_field (p2mesh-kernel.cuh:169-225) with a 3-D launch over the mesh.
__global__ void acc_field_kernel(double* __restrict__ cell_acc, double* __restrict__ cell_acc_abs,
                                 const double* __restrict__ phi, int NX, double DX) {
    const int ix = blockIdx.x * blockDim.x + threadIdx.x;
    const int iy = blockIdx.y * blockDim.y + threadIdx.y;
    const int iz = blockIdx.z;
    if (ix >= NX || iy >= NX) return;
    const int64_t at = at3(ix, iy, iz, NX);
    double d[3];
    if (ix == 0) d[0] = phi[at3(ix + 1, iy, iz, NX)] - phi[at];
    else if (ix == NX - 1) d[0] = phi[at] - phi[at3(ix - 1, iy, iz, NX)];
    else d[0] = 0.5 * (phi[at3(ix + 1, iy, iz, NX)] - phi[at3(ix - 1, iy, iz, NX)]);
    if (iy == 0) d[1] = phi[at3(ix, iy + 1, iz, NX)] - phi[at];
    else if (iy == NX - 1) d[1] = phi[at] - phi[at3(ix, iy - 1, iz, NX)];
    else d[1] = 0.5 * (phi[at3(ix, iy + 1, iz, NX)] - phi[at3(ix, iy - 1, iz, NX)]);
    if (iz == 0) d[2] = phi[at3(ix, iy, iz + 1, NX)] - phi[at];
    else if (iz == NX - 1) d[2] = phi[at] - phi[at3(ix, iy, iz - 1, NX)];
    else d[2] = 0.5 * (phi[at3(ix, iy, iz + 1, NX)] - phi[at3(ix, iy, iz - 1, NX)]);
    const double coef = -1. / DX;
    d[0] *= coef;
    d[1] *= coef;
    d[2] *= coef;
    cell_acc[3 * at] = d[0];
    cell_acc[3 * at + 1] = d[1];
    cell_acc[3 * at + 2] = d[2];
    if (cell_acc_abs) cell_acc_abs[at] = sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
}

__global__ void apply_kernel(double* __restrict__ pacc, double* __restrict__ pval, const double* __restrict__ cacc,
                             const double* __restrict__ cval, const int2* __restrict__ pci, int64_t n) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int64_t c = pci[i].x;
    if (pacc) {
        pacc[3 * i] = cacc[3 * c];
        pacc[3 * i + 1] = cacc[3 * c + 1];
        pacc[3 * i + 2] = cacc[3 * c + 2];
    }
    if (pval) pval[i] = cval[c];
}

__global__ void to_float_kernel(const double* __restrict__ src, float* __restrict__ dst, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        dst[i] = static_cast<float>(src[i]);
}

__global__ void deinterleave_kernel(const int2* __restrict__ pci, int64_t n, int* __restrict__ a, int* __restrict__ b) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int2 v = pci[i];
    a[i] = v.x;
    b[i] = v.y;
}

}  // namespace

cudaError_t launch_assign(const double* pos, int64_t n, const MeshGeom& m, int2* pci, int* counter,
                          int counter_stride, int* count2, int count2_stride, const double* mass, double* cell_mass,
                          cudaStream_t s) {
    if (n < 1) return cudaSuccess;
    assign_kernel<<<static_cast<unsigned>((n + 255) / 256), 256, 0, s>>>(pos, n, m, pci, counter, counter_stride,
                                                                           count2, count2_stride, mass, cell_mass);
    return cudaGetLastError();
}

int64_t scan_block_count(int64_t ncells) { return (ncells + kRefBlock - 1) / kRefBlock; }

cudaError_t launch_scan(const int* count, int cstride, int64_t ncells, int* maxpbc, int* start, int sstride,
                        int* start_ref, int rstride, cudaStream_t s) {
    if (ncells < 1) return cudaSuccess;
    const int64_t tiles = (ncells + kScanTile - 1) / kScanTile;
    scan_block_totals_kernel<<<static_cast<unsigned>(tiles), kScanThreads, 0, s>>>(count, cstride, ncells, maxpbc);
    scan_blocks_kernel<<<1, 1024, 0, s>>>(maxpbc, scan_block_count(ncells));
    scan_downsweep_kernel<<<static_cast<unsigned>(tiles), kScanThreads, 0, s>>>(count, cstride, ncells, maxpbc, start,
                                                                              sstride, start_ref, rstride);
    return cudaGetLastError();
}

cudaError_t launch_cell_phi(const double* phi, const int2* pci, const int* count, int cstride, int64_t n,
                            double* cell_phi, cudaStream_t s) {
    if (n < 1) return cudaSuccess;
    cell_phi_kernel<<<static_cast<unsigned>((n + 255) / 256), 256, 0, s>>>(phi, pci, count, cstride, n, cell_phi);
    return cudaGetLastError();
}

cudaError_t launch_wave_f64(double* phi_new, const double* phi, const double* phi_old, const double* mass,
                            const WaveConsts& w, cudaStream_t s) {
    const dim3 block(32, 8), grid((w.nx + 31) / 32, (w.nx + 7) / 8, w.nx);
    wave_f64_kernel<<<grid, block, 0, s>>>(phi_new, phi, phi_old, mass, w);
    return cudaGetLastError();
}

cudaError_t launch_wave_f32(float* phi_new, const float* phi, const float* phi_old, const float* mass,
                            const WaveF32& w, double* resid, cudaStream_t s) {
    const dim3 block(32, 8), grid((w.nx + 31) / 32, (w.nx + 7) / 8, w.nx);
    wave_f32_kernel<<<grid, block, 0, s>>>(phi_new, phi, phi_old, mass, w, resid);
    return cudaGetLastError();
}

cudaError_t launch_acc_field(double* cell_acc, double* cell_acc_abs, const double* phi, int nx, double dx,
                             cudaStream_t s) {
    const dim3 block(32, 8), grid((nx + 31) / 32, (nx + 7) / 8, nx);
    acc_field_kernel<<<grid, block, 0, s>>>(cell_acc, cell_acc_abs, phi, nx, dx);
    return cudaGetLastError();
}

cudaError_t launch_apply(double* pacc, double* pval, const double* cacc, const double* cval, const int2* pci,
                         int64_t n, cudaStream_t s) {
    if (n < 1) return cudaSuccess;
    apply_kernel<<<static_cast<unsigned>((n + 255) / 256), 256, 0, s>>>(pacc, pval, cacc, cval, pci, n);
    return cudaGetLastError();
}

cudaError_t launch_to_float(const double* src, float* dst, int64_t n, cudaStream_t s) {
    if (n < 1) return cudaSuccess;
    to_float_kernel<<<grid_for(n, 256), 256, 0, s>>>(src, dst, n);
    return cudaGetLastError();
}

cudaError_t launch_deinterleave(const int2* pci, int64_t n, int* a, int* b, cudaStream_t s) {
    if (n < 1) return cudaSuccess;
    deinterleave_kernel<<<static_cast<unsigned>((n + 255) / 256), 256, 0, s>>>(pci, n, a, b);
    return cudaGetLastError();
}

}  // namespace khrr
