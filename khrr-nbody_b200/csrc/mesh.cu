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
// the id iz*gx*gy + iy*gz + ix).  Slots and the mass deposit come from one
// atomic each per body (fused in one pass over the bodies).
//
// Scan: 4096-cell tiles in three launches (tile totals with 16-byte loads,
// one CTA scanning the tile totals, per-tile downsweep with 16-byte stores
// that also yields the 512-cell block totals).  The inclusive block-total scan is exactly the reference's maxPBC
// array, and the reference's start_id (the total of earlier 512-cell blocks,
// its in-block scan being discarded) is read off it; the true exclusive scan
// is the other mode.  (A one-launch scan with decoupled look-back measured
// slower at 256^3: 75 us against 48 us for the three launches.)
//
// This file is built without FMA contraction: the FP64 kernels evaluate the
// reference's expressions in IEEE double; the FP32 stencil uses explicit fmaf.
#include <algorithm>
#include <cmath>
#include <cstdint>

#include "async_copy.cuh"
#include "khrr_internal.h"
#include "wave_bricks.h"

namespace khrr {
namespace {

constexpr double kPi = 3.14159265358979;  // the reference's PI (common.cuh:7)

int grid_for(int64_t n, int block) {
    int64_t g = (n + block - 1) / block;
    if (g > 148 * 32) g = 148 * 32;
    if (g < 1) g = 1;
    return static_cast<int>(g);
}

// a / b, correctly rounded, from y = RN(1/b): Markstein's correction step
// (P. Markstein, "Computation of elementary functions on the IBM RISC
// System/6000 processor", IBM J. Res. Develop. 34(1), 1990; see also
// Muller et al., "Handbook of Floating-Point Arithmetic", ch. 4): q = RN(a y)
// is within an ulp of a/b, r = a - b q is exact in one fma, and RN(q + r y)
// is RN(a/b).  Several quotients over one denominator then share one
// correctly rounded reciprocal (__drcp_rn).  Checked bitwise against the IEEE
// division on 1.7e10 quotients (the stencil's operand ranges and random
// operands over 64 binary orders of magnitude): no difference.
__device__ __forceinline__ double div_rn(double a, double b, double y) {
    const double q = __dmul_rn(a, y);
    const double r = fma(-b, q, a);
    return fma(r, y, q);
}

// Cell coordinate of one axis: (int)((p - lo) / cs) clamped to [0, g - 1],
// with the CUDA conversion's behaviour for quotients outside the int range.
// The quotient is the IEEE one, from the mesh's correctly rounded reciprocal
// rcs = RN(1 / cs) (div_rn: three FP64 operations instead of a division).
__device__ __forceinline__ int cell_axis(double p, double lo, double cs, double rcs, int g) {
    const double q = div_rn(p - lo, cs, rcs);
    if (q >= static_cast<double>(g - 1)) return g - 1;
    if (q > -1.0) return static_cast<int>(q);
    return 0;
}

// The reference's cell id (p2mesh-kernel.cuh:25-40): iz clamps to g[1] - 1 and
// the y stride is g[2].
__device__ __forceinline__ int cell_of(const double* __restrict__ p, const MeshGeom& m) {
    const int ix = cell_axis(p[0], m.lo[0], m.cs[0], m.rcs[0], m.g[0]);
    const int iy = cell_axis(p[1], m.lo[1], m.cs[1], m.rcs[1], m.g[1]);
    const int iz = cell_axis(p[2], m.lo[2], m.cs[2], m.rcs[2], m.g[1]);
    return iz * m.g[0] * m.g[1] + iy * m.g[2] + ix;
}

// kAssignPer bodies per thread (strided by the block size, so loads stay
// coalesced): their slot atomics are independent and go out back to back,
// so a thread waits for all of them once instead of once per body.
#ifndef KHRR_ASSIGN_PER
#define KHRR_ASSIGN_PER 4
#endif
constexpr int kAssignPer = KHRR_ASSIGN_PER;

__global__ void assign_kernel(const double* __restrict__ pos, int64_t n, const MeshGeom m, int2* __restrict__ pci,
                              int* __restrict__ counter, int counter_stride, int* __restrict__ count2,
                              int count2_stride, const double* __restrict__ mass, double* __restrict__ cell_mass) {
    const int64_t base = blockIdx.x * (int64_t)blockDim.x * kAssignPer + threadIdx.x;
    int c[kAssignPer], slot[kAssignPer];
#pragma unroll
    for (int k = 0; k < kAssignPer; ++k) {
        const int64_t i = base + static_cast<int64_t>(k) * blockDim.x;
        c[k] = i < n ? cell_of(pos + 3 * i, m) : 0;
    }
    // The mass deposit first: its reductions return nothing, so they are on
    // their way while the slot atomics below wait for their values.
    if (cell_mass) {
#pragma unroll
        for (int k = 0; k < kAssignPer; ++k) {
            const int64_t i = base + static_cast<int64_t>(k) * blockDim.x;
            if (i < n) atomicAdd(&cell_mass[c[k]], mass[i]);
        }
    }
    // One atomic per body, as the reference does: bodies arrive in no
    // spatial order, so warp-level aggregation finds almost no shared cells
    // and its match/shuffle traffic costs more than it saves.
#pragma unroll
    for (int k = 0; k < kAssignPer; ++k) {
        const int64_t i = base + static_cast<int64_t>(k) * blockDim.x;
        slot[k] = i < n ? atomicAdd(&counter[static_cast<int64_t>(c[k]) * counter_stride], 1) : 0;
    }
#pragma unroll
    for (int k = 0; k < kAssignPer; ++k) {
        const int64_t i = base + static_cast<int64_t>(k) * blockDim.x;
        if (i >= n) continue;
        if (count2) atomicAdd(&count2[static_cast<int64_t>(c[k]) * count2_stride], 1);
        pci[i] = make_int2(c[k], slot[k]);
    }
}

// Cells and the NGP mass deposit only (the mesh-force step needs no slots).
__global__ void assign_cells_kernel(const double* __restrict__ pos, int64_t n, const MeshGeom m,
                                    int2* __restrict__ pci, const double* __restrict__ mass,
                                    double* __restrict__ cell_mass) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int c = cell_of(pos + 3 * i, m);
    pci[i] = make_int2(c, 0);
    atomicAdd(&cell_mass[c], mass[i]);
}

// The prefix-sum sort: each body lands at start[cell] + slot.
__global__ void scatter_order_kernel(const int2* __restrict__ pci, const int* __restrict__ start, int64_t n, int base,
                                     int* __restrict__ order) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int2 v = pci[i];
    order[start[v.x] + v.y] = base + static_cast<int>(i);
}

// ---- prefix sums -----------------------------------------------------------
// Counts are read, and starts written, 16 bytes at a time: each thread owns 8
// consecutive cells (stride 1: two int4; the reference's {count, start_id}
// pairs: four int4).  Tiles of 4096 cells = 8 of the reference's 512-cell
// blocks.
constexpr int kScanThreads = 512;
constexpr int kScanPer = 8;                              // cells per thread
constexpr int kScanTile = kScanThreads * kScanPer;       // 4096 cells
constexpr int kRefBlock = 512;                           // the reference's BLOCK_SIZE
constexpr int kBlocksPerTile = kScanTile / kRefBlock;    // 8
constexpr int kThreadsPerBlock = kRefBlock / kScanPer;   // 64

__device__ __forceinline__ int warp_sum(int v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// The 8 counts of a thread; cells past ncells read as 0.  PAIR: the counts
// are the .x of {count, start_id} pairs.
template <bool PAIR>
__device__ __forceinline__ void load8(const int* __restrict__ count, int64_t c0, int64_t ncells, int (&v)[kScanPer]) {
    if (c0 + kScanPer <= ncells) {
        if (PAIR) {
            const int4* p = reinterpret_cast<const int4*>(count + 2 * c0);
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const int4 a = p[q];
                v[2 * q] = a.x;
                v[2 * q + 1] = a.z;
            }
        } else {
            const int4* p = reinterpret_cast<const int4*>(count + c0);
            const int4 a = p[0], b = p[1];
            v[0] = a.x, v[1] = a.y, v[2] = a.z, v[3] = a.w;
            v[4] = b.x, v[5] = b.y, v[6] = b.z, v[7] = b.w;
        }
    } else {
#pragma unroll
        for (int k = 0; k < kScanPer; ++k) v[k] = c0 + k < ncells ? count[(c0 + k) * (PAIR ? 2 : 1)] : 0;
    }
}

// K1: per tile, the total of its counts.
template <bool PAIR>
__global__ void __launch_bounds__(kScanThreads) scan_totals_kernel(const int* __restrict__ count, int64_t ncells,
                                                                   int* __restrict__ tile_tot) {
    const int64_t t = blockIdx.x;
    const int tid = threadIdx.x;
    int v[kScanPer];
    load8<PAIR>(count, t * kScanTile + static_cast<int64_t>(tid) * kScanPer, ncells, v);
    int s = 0;
#pragma unroll
    for (int k = 0; k < kScanPer; ++k) s += v[k];
    s = warp_sum(s);
    __shared__ int ws[kScanThreads / 32];
    if ((tid & 31) == 0) ws[tid >> 5] = s;
    __syncthreads();
    if (tid == 0) {
        int tot = 0;
#pragma unroll
        for (int w = 0; w < kScanThreads / 32; ++w) tot += ws[w];
        tile_tot[t] = tot;
    }
}

// K2 (one CTA): tile totals -> exclusive tile offsets, in place.  Chunks of
// 1024 x kTilesPer tiles: each thread sums its kTilesPer consecutive totals,
// the 1024 thread sums are scanned with warp shuffles and one pass over the
// 32 warp sums (two barriers per chunk), and the chunks follow with a
// running carry (one chunk covers 4096 tiles = 16.8 M cells, a 256^3 mesh).
constexpr int kTilesPer = 4;
__global__ void __launch_bounds__(1024) scan_tiles_kernel(int* __restrict__ tile, int64_t ntiles) {
    constexpr int T = 1024;
    __shared__ int wsum[T / 32];
    __shared__ int s_total;
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    const int64_t chunk = static_cast<int64_t>(T) * kTilesPer;
    int carry = 0;
    for (int64_t c0 = 0; c0 < ntiles; c0 += chunk) {
        const int64_t e0 = c0 + static_cast<int64_t>(tid) * kTilesPer;
        int v[kTilesPer];
        int sum = 0;
#pragma unroll
        for (int k = 0; k < kTilesPer; ++k) {
            v[k] = e0 + k < ntiles ? tile[e0 + k] : 0;
            sum += v[k];
        }
        int incl = sum;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += y;
        }
        if (lane == 31) wsum[w] = incl;
        __syncthreads();
        if (w == 0) {
            int x = wsum[lane];
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int y = __shfl_up_sync(0xffffffffu, x, o);
                if (lane >= o) x += y;
            }
            wsum[lane] = x;
            if (lane == 31) s_total = x;
        }
        __syncthreads();
        int run = carry + (w > 0 ? wsum[w - 1] : 0) + (incl - sum);
#pragma unroll
        for (int k = 0; k < kTilesPer; ++k) {
            if (e0 + k < ntiles) tile[e0 + k] = run;
            run += v[k];
        }
        carry += s_total;
        __syncthreads();  // wsum and s_total are rewritten by the next chunk
    }
}

// K3: per tile, maxPBC for its blocks (inclusive block-total scan), the true
// exclusive start of every cell and/or the reference's start_id view, all
// from the tile's own scan and its offset (no other global reads).
template <bool PAIR>
__global__ void __launch_bounds__(kScanThreads) scan_downsweep_kernel(int* __restrict__ count, int64_t ncells,
                                                                      const int* __restrict__ tile_off,
                                                                      int* __restrict__ maxpbc, int* __restrict__ start,
                                                                      bool ref_view) {
    const int64_t t = blockIdx.x;
    const int tid = threadIdx.x;
    const int64_t c0 = t * kScanTile + static_cast<int64_t>(tid) * kScanPer;
    const int toff = tile_off[t];  // in flight while the tile is scanned
    int v[kScanPer];
    load8<PAIR>(count, c0, ncells, v);
    int s = 0;
#pragma unroll
    for (int k = 0; k < kScanPer; ++k) s += v[k];
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
    // A 512-cell block is two warps (256 cells each): the inclusive prefix
    // through block b ends at warp 2b + 1.
    if (tid < kBlocksPerTile) {
        const int64_t b = t * kBlocksPerTile + tid;
        if (b * kRefBlock < ncells) maxpbc[b] = toff + wsum[2 * tid + 1];
    }
    int out[kScanPer];
    if (ref_view) {
        // The reference's start_id: the total of all earlier 512-cell blocks.
        const int blk = tid / kThreadsPerBlock;
        const int r = toff + (blk > 0 ? wsum[2 * blk - 1] : 0);
#pragma unroll
        for (int k = 0; k < kScanPer; ++k) out[k] = r;
    } else {
        int run = toff + (w > 0 ? wsum[w - 1] : 0) + (incl - s);
#pragma unroll
        for (int k = 0; k < kScanPer; ++k) {
            out[k] = run;
            run += v[k];
        }
    }
    if (c0 + kScanPer <= ncells) {
        if (PAIR) {
            int4* p = reinterpret_cast<int4*>(count + 2 * c0);
#pragma unroll
            for (int q = 0; q < 4; ++q) p[q] = make_int4(v[2 * q], out[2 * q], v[2 * q + 1], out[2 * q + 1]);
        } else {
            int4* p = reinterpret_cast<int4*>(start + c0);
            p[0] = make_int4(out[0], out[1], out[2], out[3]);
            p[1] = make_int4(out[4], out[5], out[6], out[7]);
        }
    } else {
#pragma unroll
        for (int k = 0; k < kScanPer; ++k) {
            if (c0 + k >= ncells) break;
            if (PAIR) count[2 * (c0 + k) + 1] = out[k];
            else start[c0 + k] = out[k];
        }
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


// wave_diss_iteration in FP64, the reference's expressions term for term
// (same bits as the literal per-cell kernel): kWZ consecutive z cells of one
// (x, y) column per thread with every load issued up front, K computed once
// per thread, and the five per-cell divisions (rho and the four coefficients
// over Wt) through shared correctly rounded reciprocals: 1.41x the literal
// kernel at 256^3.
template <int kWZ>
__global__ void __launch_bounds__(256) wave_f64_kernel(double* __restrict__ phi_new, const double* __restrict__ phi,
                                                       const double* __restrict__ phi_old,
                                                       const double* __restrict__ mass, const WaveConsts W) {
    const int NX = W.nx;
    const int ix = blockIdx.x * 32 + threadIdx.x, iy = blockIdx.y * 8 + threadIdx.y;
    const int zb = blockIdx.z * kWZ;
    if (ix >= NX || iy >= NX) return;
    const int64_t sy = NX, sz = static_cast<int64_t>(NX) * NX;
    const int64_t col = static_cast<int64_t>(iy) * NX + ix;
    const int64_t dxm = ix > 0 ? 1 : 0, dxp = ix < NX - 1 ? 1 : 0;
    const int64_t dym = iy > 0 ? sy : 0, dyp = iy < NX - 1 ? sy : 0;
    double c[kWZ + 2];
    double xm[kWZ], xp[kWZ], ym[kWZ], yp[kWZ], po[kWZ], ms[kWZ];
#pragma unroll
    for (int u = 0; u < kWZ + 2; ++u) c[u] = phi[min(max(zb - 1 + u, 0), NX - 1) * sz + col];
#pragma unroll
    for (int u = 0; u < kWZ; ++u) {
        const int64_t at = min(zb + u, NX - 1) * sz + col;
        xm[u] = phi[at - dxm];
        xp[u] = phi[at + dxp];
        ym[u] = phi[at - dym];
        yp[u] = phi[at + dyp];
        po[u] = phi_old[at];
        ms[u] = mass[at];
    }
    const bool edge_xy = ix == 0 || ix == NX - 1 || iy == 0 || iy == NX - 1;
    const double DX = W.dx, C = W.c, DT = W.dt;
    const double D3 = DX * DX * DX;
    const double yD3 = __drcp_rn(D3);
    const double K = C * C * (DT * DT) / (DX * DX);
    const double KFn = -(C * C) * (DT * DT);
    const double KAn = 2 * (1. - 3 * K);
#pragma unroll
    for (int u = 0; u < kWZ; ++u) {
        const int z = zb + u;
        if (z >= NX) break;
        double out = 0.0;
        if (!(edge_xy || z == 0 || z == NX - 1)) {
            const double rho = div_rn(ms[u], D3, yD3);
            const double f = 4 * kPi * 1.0 * rho;
            const double diss = wave_diss(W, ix, iy, z);
            const double Q = diss * C * DT * 0.5;
            const double Wt = 1 + Q;
            const double yW = __drcp_rn(Wt);
            const double KM = div_rn(K, Wt, yW);
            const double KF = div_rn(KFn, Wt, yW);
            const double KA = div_rn(KAn, Wt, yW);
            const double KO = div_rn(Q - 1., Wt, yW);
            out = xm[u] * KM + xp[u] * KM + ym[u] * KM + yp[u] * KM + c[u] * KM + c[u + 2] * KM + c[u + 1] * KA +
                  po[u] * KO + f * KF;
        }
        phi_new[z * sz + col] = out;
    }
}

// The FP32 form of the step.  The sponge is separable,
// diss = base + sx[ix] + sy[iy] + sz[iz] (per-axis tables built in FP64 on the
// host); per cell: Q = diss c dt / 2, w = 1 / (1 + Q), and
//   phi_new = nb K w + phi (2 (1 - 3K)) w + phi_old (Q - 1) w + mass S w,
// with nb the six-neighbour sum and S = -c^2 dt^2 4 pi / dx^3.  With resid,
// sum (phi_new - phi)^2 and sum phi_new^2 are accumulated in FP64.
// Each thread computes kWZ consecutive z cells of one (x, y) column: the
// column's phi values are loaded once and shared as z neighbours, and all
// other loads (x/y neighbours, phi_old, mass) are issued up front, so a warp
// keeps many requests in flight (no barriers, no shared memory).  kWZ = 8 on
// large meshes, 4 on small ones (more CTAs).
// CTA shape in x (a multiple of 32: each warp is one x row segment) and y.
#ifndef KHRR_WAVE_WX
#define KHRR_WAVE_WX 32
#endif
#ifndef KHRR_WAVE_WY
#define KHRR_WAVE_WY 8
#endif
constexpr int kWX = KHRR_WAVE_WX, kWY = KHRR_WAVE_WY;


static_assert(kWX % 32 == 0 && kWX * kWY <= 1024, "whole warps along x");

template <int kWZ>
__global__ void __launch_bounds__(kWX * kWY) wave_f32_kernel(float* __restrict__ phi_new, const float* __restrict__ phi,
                                                             const float* __restrict__ phi_old,
                                                             const float* __restrict__ mass, const WaveF32 W,
                                                             double* __restrict__ resid) {
    const int NX = W.nx;
    const int ix = blockIdx.x * kWX + threadIdx.x, iy = blockIdx.y * kWY + threadIdx.y;
    const int zb = blockIdx.z * kWZ;
    const int64_t sy = NX, sz = static_cast<int64_t>(NX) * NX;
    double d2 = 0.0, n2 = 0.0;
    // Programmatic dependent launch: the next step's grid may be scheduled
    // while this one drains; every grid waits here until the previous one
    // has completed and its writes are visible (a no-op without a
    // programmatic dependency).
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    asm volatile("griddepcontrol.wait;" ::: "memory");
    if (ix < NX && iy < NX) {
        const int64_t col = static_cast<int64_t>(iy) * NX + ix;
        // Neighbour offsets clamped into the mesh, so every load below is
        // unconditional and in bounds (face cells discard their values).
        const int64_t dxm = ix > 0 ? 1 : 0, dxp = ix < NX - 1 ? 1 : 0;
        const int64_t dym = iy > 0 ? sy : 0, dyp = iy < NX - 1 ? sy : 0;
        float c[kWZ + 2];  // phi at z = zb - 1 .. zb + kWZ (clamped into the mesh)
        float xm[kWZ], xp[kWZ], ym[kWZ], yp[kWZ], po[kWZ], ms[kWZ];
#pragma unroll
        for (int u = 0; u < kWZ + 2; ++u) {
            const int z = min(max(zb - 1 + u, 0), NX - 1);
            c[u] = phi[z * sz + col];
        }
#pragma unroll
        for (int u = 0; u < kWZ; ++u) {
            const int64_t at = min(zb + u, NX - 1) * sz + col;
            xm[u] = phi[at - dxm];
            xp[u] = phi[at + dxp];
            ym[u] = phi[at - dym];
            yp[u] = phi[at + dyp];
            po[u] = phi_old[at];
            ms[u] = mass[at];
        }
        const bool edge_xy = ix == 0 || ix == NX - 1 || iy == 0 || iy == NX - 1;
        const float sxy = (W.diss_base + W.sx[ix]) + W.sy[iy];
#pragma unroll
        for (int u = 0; u < kWZ; ++u) {
            const int z = zb + u;
            if (z >= NX) break;
            const int64_t at = z * sz + col;
            float out = 0.0f;
            if (!(edge_xy || z == 0 || z == NX - 1)) {
                const float nb = ((xm[u] + xp[u]) + (ym[u] + yp[u])) + (c[u] + c[u + 2]);
                const float diss = sxy + W.sz[z];
                const float Q = diss * W.cdt_half;
                const float w = __frcp_rn(1.0f + Q);  // correctly rounded: the bits of 1.0f / (1.0f + Q)
                out = fmaf(nb, W.K * w, fmaf(c[u + 1], W.A * w, fmaf(po[u], (Q - 1.0f) * w, ms[u] * (W.S * w))));
            }
            phi_new[at] = out;
            if (resid) {
                const double dd = static_cast<double>(out) - static_cast<double>(c[u + 1]);
                d2 += dd * dd;
                n2 += static_cast<double>(out) * static_cast<double>(out);
            }
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

// The same step with four consecutive x cells per thread (nx % 4 == 0):
// every row access is one 16-byte load or store, so a warp moves 512
// contiguous bytes per access and issues a quarter of the load instructions.
// The x neighbours come from the float4 itself and, across threads, by warp
// shuffles (a warp covers 128 consecutive x cells); lanes 0 and 31 load the
// one cell beyond their warp's span.  Threads past the mesh in x read
// clamped addresses (for the shuffles) and store nothing.  Per cell the
// arithmetic is wave_f32_kernel's, so the bits are the same.
constexpr int kW4X = 32, kW4Y = 8;  // threads: 128 x cells x 8 rows

__device__ __forceinline__ float f4c(const float4& v, int k) { return k == 0 ? v.x : k == 1 ? v.y : k == 2 ? v.z : v.w; }

template <int kWZ>
__global__ void __launch_bounds__(kW4X * kW4Y) wave_f32x4_kernel(float* __restrict__ phi_new, const float* __restrict__ phi,
                                                                 const float* __restrict__ phi_old,
                                                                 const float* __restrict__ mass, const WaveF32 W,
                                                                 double* __restrict__ resid) {
    const int NX = W.nx;
    const int ix0 = (blockIdx.x * kW4X + threadIdx.x) * 4, iy = blockIdx.y * kW4Y + threadIdx.y;
    const int zb = blockIdx.z * kWZ;
    const int lane = threadIdx.x;  // kW4X == 32: one warp per x row segment
    const int64_t sy = NX, sz = static_cast<int64_t>(NX) * NX;
    double d2 = 0.0, n2 = 0.0;
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    asm volatile("griddepcontrol.wait;" ::: "memory");
    if (iy < NX) {  // whole warps share iy: the shuffles below see every lane
        const bool xin = ix0 < NX;
        const int xc = xin ? ix0 : NX - 4;  // clamped for the loads
        const int64_t col = static_cast<int64_t>(iy) * NX + xc;
        const int64_t dym = iy > 0 ? sy : 0, dyp = iy < NX - 1 ? sy : 0;
        const int64_t dxm = xc > 0 ? 1 : 0, dxp = xc + 4 < NX ? 4 : 3;  // the cells beyond the float4
        float4 c[kWZ + 2];  // phi at z = zb - 1 .. zb + kWZ (clamped)
        float4 ym[kWZ], yp[kWZ], po[kWZ], ms[kWZ];
        float xl[kWZ], xr[kWZ];  // lanes 0 / 31: phi at xc - 1 / xc + 4
#pragma unroll
        for (int u = 0; u < kWZ + 2; ++u) {
            const int z = min(max(zb - 1 + u, 0), NX - 1);
            c[u] = *reinterpret_cast<const float4*>(phi + z * sz + col);
        }
#pragma unroll
        for (int u = 0; u < kWZ; ++u) {
            const int64_t at = min(zb + u, NX - 1) * sz + col;
            ym[u] = *reinterpret_cast<const float4*>(phi + at - dym);
            yp[u] = *reinterpret_cast<const float4*>(phi + at + dyp);
            po[u] = *reinterpret_cast<const float4*>(phi_old + at);
            ms[u] = *reinterpret_cast<const float4*>(mass + at);
            xl[u] = lane == 0 ? phi[at - dxm] : 0.0f;
            xr[u] = lane == 31 ? phi[at + dxp] : 0.0f;
        }
        const float4 sx4 = *reinterpret_cast<const float4*>(W.sx + xc);
        const float sy1 = W.sy[iy];
        const bool edge_y = iy == 0 || iy == NX - 1;
#pragma unroll
        for (int u = 0; u < kWZ; ++u) {
            const int z = zb + u;
            const float4 cc = c[u + 1];
            // x neighbours of the end cells from the adjacent lanes
            float left = __shfl_up_sync(0xffffffffu, cc.w, 1);
            float right = __shfl_down_sync(0xffffffffu, cc.x, 1);
            if (lane == 0) left = xl[u];
            if (lane == 31) right = xr[u];
            if (z >= NX || !xin) continue;
            const int64_t at = z * sz + col;
            float out[4];
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                const int ix = xc + k;
                float o = 0.0f;
                if (!(edge_y || ix == 0 || ix == NX - 1 || z == 0 || z == NX - 1)) {
                    const float xm = k == 0 ? left : f4c(cc, k - 1);
                    const float xp = k == 3 ? right : f4c(cc, k + 1);
                    const float nb = ((xm + xp) + (f4c(ym[u], k) + f4c(yp[u], k))) + (f4c(c[u], k) + f4c(c[u + 2], k));
                    const float diss = ((W.diss_base + f4c(sx4, k)) + sy1) + W.sz[z];
                    const float Q = diss * W.cdt_half;
                    const float w = __frcp_rn(1.0f + Q);  // correctly rounded: the bits of 1.0f / (1.0f + Q)
                    o = fmaf(nb, W.K * w,
                             fmaf(f4c(cc, k), W.A * w, fmaf(f4c(po[u], k), (Q - 1.0f) * w, f4c(ms[u], k) * (W.S * w))));
                }
                out[k] = o;
                if (resid) {
                    const double dd = static_cast<double>(o) - static_cast<double>(f4c(cc, k));
                    d2 += dd * dd;
                    n2 += static_cast<double>(o) * static_cast<double>(o);
                }
            }
            *reinterpret_cast<float4*>(phi_new + at) = make_float4(out[0], out[1], out[2], out[3]);
        }
    }
    if (resid) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            d2 += __shfl_xor_sync(0xffffffffu, d2, o);
            n2 += __shfl_xor_sync(0xffffffffu, n2, o);
        }
        if (lane == 0) {
            atomicAdd(&resid[0], d2);
            atomicAdd(&resid[1], n2);
        }
    }
}

// Two leap-frog steps per launch (temporal blocking), fed by tensor copies.
// A CTA owns a 32 x 8 column tile and TZ planes of it and marches up in z.
// Thread 0 streams, plane by plane, three 40 x 12 boxes (phi^n, phi^{n-1},
// mass at x0-4 .. x0+35, y0-2 .. y0+9; outside the mesh they read as zero)
// into a kTmaD-stage shared-memory ring on mbarriers, up to kTmaD planes ahead
// of the stencil, which then reads only shared memory.  At each plane the
// CTA first computes phi^{n+1} on the tile extended by one cell in x and y
// (34 x 10 = 340 points, one per thread and a second for threads 0..83) into
// a 4-plane shared ring, then phi^{n+2} one plane below on its own 32 x 8
// points.  Per cell the arithmetic is exactly wave_f32_kernel's, so two
// launches of that kernel and one of this give identical bits.  It reads
// phi^n, phi^{n-1} and the mass once and writes phi^{n+1} (own tile) and
// phi^{n+2}: 20 bytes per cell for two iterations instead of 32.  out1 and
// out2 must be buffers this launch does not read (neighbouring CTAs still
// read phi^{n-1} and phi^n).  Plane q of a CTA is z0-2+q; step 1 at plane
// zs = z0-1+j reads planes j, j+1, j+2 and step 2 at zs-1 reads plane j, so
// after iteration j's barrier plane j-1 is free and its stage takes plane
// j-1+kTmaD.  Needs nx % 4 == 0 (16-byte row strides) and nx >= 40.
constexpr int kT2X = 32, kT2Y = 8;
constexpr int kT2EX = kT2X + 2, kT2EY = kT2Y + 2;
constexpr int kT2E = kT2EX * kT2EY;           // 340 first-step points per plane
constexpr int kT2Threads = kT2X * kT2Y;       // 256
constexpr int kTmaD = 6;
constexpr int kTmaBX = 40, kTmaBY = 12;
constexpr unsigned kTmaBoxBytes = kTmaBX * kTmaBY * 4u;

// One stencil update (wave_f32_kernel's expression) or 0 on faces and
// outside the mesh.
__device__ __forceinline__ float wave1_point(const WaveF32& W, float sxy, bool edge_xy, int z, float xm, float xp,
                                             float ym, float yp, float zm, float c, float zp, float po, float ms) {
    if (edge_xy || z <= 0 || z >= W.nx - 1) return 0.0f;
    const float nb = ((xm + xp) + (ym + yp)) + (zm + zp);
    const float diss = sxy + W.sz[z];
    const float Q = diss * W.cdt_half;
    const float w = __frcp_rn(1.0f + Q);  // correctly rounded: the bits of 1.0f / (1.0f + Q)
    return fmaf(nb, W.K * w, fmaf(c, W.A * w, fmaf(po, (Q - 1.0f) * w, ms * (W.S * w))));
}

// A first-step point of the extended tile: its box offset, sponge and edge flag.
struct Wave2Pt {
    int box;  // offset in a 40 x 12 box
    int e;    // index in the 34 x 10 extended plane
    float sxy;
    bool edge;
};

__device__ __forceinline__ Wave2Pt wave2_point(const WaveF32& W, int e, int x0, int y0) {
    const int NX = W.nx;
    const int ex = e % kT2EX, ey = e / kT2EX;
    const int gx = x0 - 1 + ex, gy = y0 - 1 + ey;
    const int cx = min(max(gx, 0), NX - 1), cy = min(max(gy, 0), NX - 1);
    Wave2Pt p;
    p.box = (ey + 1) * kTmaBX + (ex + 3);  // extended point (ex, ey) sits at box (ex + 3, ey + 1)
    p.e = e;
    p.sxy = (W.diss_base + W.sx[cx]) + W.sy[cy];
    p.edge = gx <= 0 || gx >= NX - 1 || gy <= 0 || gy >= NX - 1;
    return p;
}

__device__ __forceinline__ float wave2_step1(const WaveF32& W, const Wave2Pt& p, int zs, const float* __restrict__ a,
                                             const float* __restrict__ b, const float* __restrict__ c,
                                             const float* __restrict__ pm, const float* __restrict__ ms) {
    const int o = p.box;
    return wave1_point(W, p.sxy, p.edge, zs, b[o - 1], b[o + 1], b[o - kTmaBX], b[o + kTmaBX], a[o], b[o], c[o],
                       pm[o], ms[o]);
}

template <int TZ>
__global__ void __launch_bounds__(kT2Threads) wave2_tma_kernel(float* __restrict__ out1, float* __restrict__ out2,
                                                              const __grid_constant__ CUtensorMap tp0,
                                                              const __grid_constant__ CUtensorMap tpm,
                                                              const __grid_constant__ CUtensorMap tms,
                                                              const WaveF32 W, double* __restrict__ resid,
                                                              unsigned* __restrict__ err) {
    __shared__ alignas(128) float ring[kTmaD][3][kTmaBY * kTmaBX];
    __shared__ float s1[4][kT2E];
    __shared__ alignas(8) uint64_t full[kTmaD];
    const int NX = W.nx;
    const int tid = threadIdx.x;
    const int x0 = blockIdx.x * kT2X, y0 = blockIdx.y * kT2Y, z0 = blockIdx.z * TZ;
    const int zend = min(z0 + TZ, NX);
    const int P = zend - z0 + 4;  // planes z0-2 .. zend+1

    if (tid == 0) {
        for (int s = 0; s < kTmaD; ++s) mbar_init(&full[s], 1);
        fence_mbar_init();
    }
    __syncthreads();
    auto issue = [&](int q) {
        const int s = q % kTmaD, z = z0 - 2 + q;
        mbar_arrive_expect_tx(&full[s], 3 * kTmaBoxBytes);
        tensor_copy_3d_g2s(ring[s][0], &tp0, x0 - 4, y0 - 2, z, &full[s]);
        tensor_copy_3d_g2s(ring[s][1], &tpm, x0 - 4, y0 - 2, z, &full[s]);
        tensor_copy_3d_g2s(ring[s][2], &tms, x0 - 4, y0 - 2, z, &full[s]);
    };
    if (tid == 0)
        for (int q = 0; q < kTmaD && q < P; ++q) issue(q);

    // First-step points of this thread (the second one for tid < 84).
    const Wave2Pt p1 = wave2_point(W, tid, x0, y0);
    const bool has2 = tid + kT2Threads < kT2E;
    const Wave2Pt p2 = wave2_point(W, has2 ? tid + kT2Threads : tid, x0, y0);
    // Own second-step point.
    const int tx = tid % kT2X, ty = tid / kT2X;
    const int ox = x0 + tx, oy = y0 + ty;
    const bool own_in = ox < NX && oy < NX;
    const bool own_edge = ox <= 0 || ox >= NX - 1 || oy <= 0 || oy >= NX - 1;
    const float own_sxy =
        (W.diss_base + W.sx[min(max(ox, 0), NX - 1)]) + W.sy[min(max(oy, 0), NX - 1)];
    const int oe = (ty + 1) * kT2EX + (tx + 1);  // own point in the extended plane
    const int ob = (ty + 2) * kTmaBX + (tx + 4);  // and in a box
    const int64_t col = static_cast<int64_t>(oy) * NX + ox;
    const int64_t plane = static_cast<int64_t>(NX) * NX;

    bool ok = mbar_wait_bounded(&full[0], 0u) && mbar_wait_bounded(&full[1 % kTmaD], 0u);
    double d2 = 0.0, n2 = 0.0;
    for (int j = 0; j + 2 < P; ++j) {
        const int zs = z0 - 1 + j;
        const int q2 = j + 2;
        if (ok) ok = mbar_wait_bounded(&full[q2 % kTmaD], static_cast<unsigned>((q2 / kTmaD) & 1));
        if (ok) {
            const float* a = ring[j % kTmaD][0];        // phi^n at zs - 1
            const float* b = ring[(j + 1) % kTmaD][0];  // phi^n at zs
            const float* c = ring[q2 % kTmaD][0];       // phi^n at zs + 1
            const float* pm = ring[(j + 1) % kTmaD][1];
            const float* ms = ring[(j + 1) % kTmaD][2];
            float* dst = s1[j % 4];
            dst[p1.e] = wave2_step1(W, p1, zs, a, b, c, pm, ms);
            if (has2) dst[p2.e] = wave2_step1(W, p2, zs, a, b, c, pm, ms);
        }
        if (__syncthreads_or(!ok)) {
            if (tid == 0) {
                atomicOr(err, kErrTimeout);
                // Let copies still in flight into this CTA's ring land:
                // planes [0, issued) have been issued so far.
                const int issued = min(P, max(kTmaD, j - 1 + kTmaD));
                for (int q = j; q < issued; ++q)
                    (void)mbar_wait_bounded(&full[q % kTmaD], static_cast<unsigned>((q / kTmaD) & 1));
            }
            return;
        }
        // Plane j - 1 was last read before this barrier: refill its stage.
        if (tid == 0 && j >= 1 && j - 1 + kTmaD < P) {
            fence_proxy_async();
            issue(j - 1 + kTmaD);
        }
        // Second step at plane k = zs - 1 from first-step planes k-1, k, k+1.
        const int k = zs - 1;
        if (j >= 2 && own_in) {
            const float* lo = s1[(j + 2) % 4];  // plane k - 1
            const float* pl = s1[(j + 3) % 4];  // plane k
            const float* hi = s1[j % 4];        // plane k + 1
            const float c1 = pl[oe];
            float o2 = 0.0f;
            if (!(own_edge || k <= 0 || k >= NX - 1)) {
                const float old = ring[j % kTmaD][0][ob], mk = ring[j % kTmaD][2][ob];
                const float nb = ((pl[oe - 1] + pl[oe + 1]) + (pl[oe - kT2EX] + pl[oe + kT2EX])) + (lo[oe] + hi[oe]);
                const float diss = own_sxy + W.sz[k];
                const float Q = diss * W.cdt_half;
                const float w = __frcp_rn(1.0f + Q);
                o2 = fmaf(nb, W.K * w, fmaf(c1, W.A * w, fmaf(old, (Q - 1.0f) * w, mk * (W.S * w))));
            }
            const int64_t at = k * plane + col;
            out1[at] = c1;
            out2[at] = o2;
            if (resid) {
                const double dd = static_cast<double>(o2) - static_cast<double>(c1);
                d2 += dd * dd;
                n2 += static_cast<double>(o2) * static_cast<double>(o2);
            }
        }
    }
    if (resid) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            d2 += __shfl_xor_sync(0xffffffffu, d2, o);
            n2 += __shfl_xor_sync(0xffffffffu, n2, o);
        }
        if ((tid & 31) == 0) {
            atomicAdd(&resid[0], d2);
            atomicAdd(&resid[1], n2);
        }
    }
}

// One leap-frog step fed by tensor copies, warp-specialised.  A CTA owns a
// 32 x 8 column tile and TZ planes of it.  Warp 8 (one lane) is the
// producer: plane by plane it copies phi^n with its x/y halo (a 40 x 10 box
// at x0-4, y0-1), phi^{n-1} and the mass (32 x 8 boxes at x0, y0) into a
// kW1D-stage ring, waiting on each stage's "empty" barrier before reuse.
// Warps 0..7 are consumers, one output point per thread: output plane z
// reads phi^n at z-1, z, z+1 (stages i, i+1, i+2 for z = z0+i) and
// phi^{n-1}, mass at z (stage i+1), then releases stage i.  No CTA-wide
// barrier after set-up: warps drift up to kW1D planes apart and each waits
// only for its data.  Per cell the arithmetic is wave_f32_kernel's (same
// bits).  Needs nx % 4 == 0 and nx >= 40.
constexpr int kW1D = 8;
constexpr int kW1Consumers = 8;                 // warps
constexpr int kW1PhiFloats = 40 * 10;           // phi box
constexpr int kW1PhiPad = 416;                  // 1664 bytes: keeps the next box 128-byte aligned
constexpr int kW1TileFloats = 32 * 8;           // phi^{n-1} and mass boxes
constexpr int kW1StageFloats = kW1PhiPad + 2 * kW1TileFloats;
constexpr unsigned kW1StageBytes = (kW1PhiFloats + 2 * kW1TileFloats) * 4u;

template <int TZ>
__global__ void __launch_bounds__((kW1Consumers + 1) * 32) wave1_tma_kernel(float* __restrict__ phi_new,
                                                                           const __grid_constant__ CUtensorMap tphi,
                                                                           const __grid_constant__ CUtensorMap told,
                                                                           const __grid_constant__ CUtensorMap tmass,
                                                                           const WaveF32 W, double* __restrict__ resid,
                                                                           unsigned* __restrict__ err) {
    __shared__ alignas(128) float ring[kW1D][kW1StageFloats];
    __shared__ alignas(8) uint64_t full[kW1D], empty[kW1D];
    const int NX = W.nx;
    const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
    const int x0 = blockIdx.x * 32, y0 = blockIdx.y * 8, z0 = blockIdx.z * TZ;
    const int zend = min(z0 + TZ, NX);
    const int P = zend - z0 + 2;  // planes z0-1 .. zend: plane q is z0-1+q

    if (threadIdx.x == 0) {
        for (int s = 0; s < kW1D; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], kW1Consumers);
        }
        fence_mbar_init();
    }
    __syncthreads();

    if (warp == kW1Consumers) {  // producer
        if (lane != 0) return;
        bool ok = true;
        int issued = 0;
        for (int q = 0; q < P; ++q) {
            const int s = q % kW1D;
            if (q >= kW1D) {
                ok = mbar_wait_bounded(&empty[s], static_cast<unsigned>((q / kW1D - 1) & 1));
                if (!ok) break;
                fence_proxy_async();
            }
            const int z = z0 - 1 + q;
            float* st = ring[s];
            mbar_arrive_expect_tx(&full[s], kW1StageBytes);
            tensor_copy_3d_g2s(st, &tphi, x0 - 4, y0 - 1, z, &full[s]);
            tensor_copy_3d_g2s(st + kW1PhiPad, &told, x0, y0, z, &full[s]);
            tensor_copy_3d_g2s(st + kW1PhiPad + kW1TileFloats, &tmass, x0, y0, z, &full[s]);
            issued = q + 1;
        }
        if (!ok) atomicOr(err, kErrTimeout);
        // No copy may still be in flight when the CTA exits.
        for (int q = max(0, issued - kW1D); q < issued; ++q)
            (void)mbar_wait_bounded(&full[q % kW1D], static_cast<unsigned>((q / kW1D) & 1));
        return;
    }

    // Consumers: thread (lane, warp) owns point (x0 + lane, y0 + warp).
    const int ox = x0 + lane, oy = y0 + warp;
    const bool own_in = ox < NX && oy < NX;
    const bool edge_xy = ox <= 0 || ox >= NX - 1 || oy <= 0 || oy >= NX - 1;
    const float sxy = (W.diss_base + W.sx[min(max(ox, 0), NX - 1)]) + W.sy[min(max(oy, 0), NX - 1)];
    const int pb = (warp + 1) * 40 + (lane + 4);  // point in the phi box
    const int tb = warp * 32 + lane;              // point in the 32 x 8 boxes
    const int64_t plane = static_cast<int64_t>(NX) * NX;
    const int64_t col = static_cast<int64_t>(oy) * NX + ox;
    double d2 = 0.0, n2 = 0.0;
    bool ok = mbar_wait_bounded(&full[0], 0u) && mbar_wait_bounded(&full[1], 0u);
    for (int i = 0; ok && i + 2 < P; ++i) {
        const int q2 = i + 2;
        ok = mbar_wait_bounded(&full[q2 % kW1D], static_cast<unsigned>((q2 / kW1D) & 1));
        if (!ok) break;
        const int z = z0 + i;
        const float* a = ring[i % kW1D];
        const float* b = ring[(i + 1) % kW1D];
        const float* c = ring[q2 % kW1D];
        const float cc = b[pb];
        const float out = wave1_point(W, sxy, edge_xy, z, b[pb - 1], b[pb + 1], b[pb - 40], b[pb + 40], a[pb], cc,
                                      c[pb], b[kW1PhiPad + tb], b[kW1PhiPad + kW1TileFloats + tb]);
        __syncwarp();
        if (lane == 0) mbar_arrive(&empty[i % kW1D]);  // this warp is done with plane i
        if (own_in) {
            phi_new[z * plane + col] = out;
            if (resid) {
                const double dd = static_cast<double>(out) - static_cast<double>(cc);
                d2 += dd * dd;
                n2 += static_cast<double>(out) * static_cast<double>(out);
            }
        }
    }
    if (!ok) atomicOr(err, kErrTimeout);
    if (resid) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            d2 += __shfl_xor_sync(0xffffffffu, d2, o);
            n2 += __shfl_xor_sync(0xffffffffu, n2, o);
        }
        if (lane == 0) {
            atomicAdd(&resid[0], d2);
            atomicAdd(&resid[1], n2);
        }
    }
}

// k FP32 iterations in one launch with the field resident in shared memory
// (nx = 128: the 128^3 mesh of the two-galaxy encounter).  The mesh is cut
// into 128 bricks of 128 (x) x 16 (y) x 8 (z) cells, one CTA each, for the
// whole launch: phi^n of the brick in shared memory (two buffers,
// alternating by iteration), phi^{n-1} and the mass term in registers, the
// sponge factor w = 1/(1 + Q) of every cell in shared memory.  A warp owns 8
// of the brick's 128 rows of 128 x cells, four consecutive cells per lane
// (16-byte shared and global accesses; x neighbours from the float4 and by
// shuffles).  An iteration first updates the brick's 84 interior rows, whose
// neighbours all lie in the brick, while the neighbour bricks finish the
// previous iteration; then it waits for them, stages the 48 rows of theirs
// that touch it (y - 1, y + 1, z - 1, z + 1 faces; 24 KB) from global memory
// into shared memory, and updates its 44 face rows, which it writes to the
// ring buffer the one-launch-per-iteration path would write.  The last
// iteration writes the whole brick, and the interior rows of phi^{k-1}
// follow it, so the ring ends in the state of the per-iteration path (its
// two current buffers; the other two are free).  Bricks are exchanged
// through per-brick counters: after iteration t a CTA sets flag[b] = t + 1
// (release); before the face rows of iteration t (t >= 1) it waits for its
// (up to four) neighbours' flags >= t.  That wait also keeps every CTA at
// most one iteration ahead of its neighbours, so a ring buffer's face rows
// are overwritten only once the neighbours have finished the iteration that
// read them (the buffer holds phi^{t-2} or older when iteration t writes
// phi^{t+1}); interior rows are read by no other CTA.  Every wait is bounded
// (2 s of wall time); a CTA that gives up sets err (kErrTimeout) and
// flag[kRzBricks] (abort), and every other wait ends on that flag.  The grid
// is one CTA per brick, launched cooperatively so all of them are resident.
// Per cell the arithmetic is wave_f32_kernel's, in its order, so the bits
// are the same; the residual of the last iteration is formed after the loop
// from the two shared buffers it leaves, summed per warp and added with one
// FP64 atomic pair per warp (its last bits depend on the order).
//
// Measured on the encounter's mesh (CUDA events, same GPU, 1000-iteration
// solve / Wave-mode step of 507 iterations): 5.6 us per iteration, 2.91 ms
// per step, against 7.07 us / 3.39 ms for one plane per CTA (two 64 KB
// neighbour planes read and the whole plane written per CTA and iteration)
// and 10.4 us with one launch per iteration.  Steps on the way: bricks with
// the face rows read straight from global memory 8.5 us (each warp's loads
// serialised behind its z carry); halos staged in shared memory 7.2 us;
// interior rows before the wait 6.7 us; the residual moved out of the loop
// (no FP64 branch in it) 5.6 us.
// Brick geometry, row map and halo rows: wave_bricks.h.
constexpr size_t kRzSmem = (3 * static_cast<size_t>(kRzBrick) + kRzHalo) * sizeof(float);  // 221,184 B

__device__ __forceinline__ unsigned ld_acquire_gpu(const unsigned* p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void st_release_gpu(unsigned* p, unsigned v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Free buffers f0 < f1 of the four-buffer ring besides o and c.
__device__ __forceinline__ void ring_free_dev(int o, int c, int& f0, int& f1) {
    int f[2], n = 0;
#pragma unroll
    for (int b = 0; b < 4; ++b)
        if (b != o && b != c && n < 2) f[n++] = b;
    f0 = f[0];
    f1 = f[1];
}

__global__ void __launch_bounds__(kRzThreads, 1) wave_resident_kernel(float* __restrict__ ring, int64_t cz,
                                                                      const float* __restrict__ mass,
                                                                      const WaveF32 W, int k, int st,
                                                                      double* __restrict__ resid,
                                                                      unsigned* __restrict__ flag,
                                                                      unsigned* __restrict__ err,
                                                                      unsigned long long limit_ns, int withhold) {
    extern __shared__ __align__(16) float rz_smem[];
    float* sphi = rz_smem;                  // [2][brick]: phi^n by iteration parity
    float* sw = rz_smem + 2 * kRzBrick;     // [brick]: w = 1 / (1 + Q)
    float* shalo = sw + kRzBrick;           // [48 rows]: y halos by zl, then z halos by yl
    const int b = blockIdx.x, by = b % kRzBricksY, bz = b / kRzBricksY;
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    const int y0 = by * kRzBY, z0 = bz * kRzBZ;
    const int x0 = 4 * lane;  // the lane's cells x0 .. x0 + 3 of each of its rows
    constexpr int kSRow = kRzBY * kRzNX;  // shared stride of zl
    // Row (yl, zl): shared index (zl * BY + yl) * nx + x0, global index
    // (z0 + zl) * nx^2 + (y0 + yl) * nx + x0.
    auto sidx = [&](int yl, int zl) { return (zl * kRzBY + yl) * kRzNX + x0; };
    auto gidx = [&](int yl, int zl) {
        return static_cast<int64_t>(z0 + zl) * kRzPlane + static_cast<int64_t>(y0 + yl) * kRzNX + x0;
    };
    float sxb[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) sxb[j] = W.diss_base + W.sx[x0 + j];
    int old = st / 4, cur = st % 4;

    float po[kRzCells], msw[kRzCells];  // per slot: phi^{n-1}; mass times S w
#pragma unroll
    for (int i = 0; i < kRzSlots; ++i) {
        int yl, zl;
        rz_row(wid, i, yl, zl);
        const int s = sidx(yl, zl);
        const int64_t g = gidx(yl, zl);
        const float4 m4 = *reinterpret_cast<const float4*>(mass + g);
        const float4 o4 = *reinterpret_cast<const float4*>(ring + old * cz + g);
        const float4 c4 = *reinterpret_cast<const float4*>(ring + cur * cz + g);
        const float mj[4] = {m4.x, m4.y, m4.z, m4.w}, oj[4] = {o4.x, o4.y, o4.z, o4.w};
        const float sy = W.sy[y0 + yl], sz = W.sz[z0 + zl];
        float wj[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const float sxy = sxb[j] + sy;
            const float diss = sxy + sz;
            const float Q = diss * W.cdt_half;
            wj[j] = __frcp_rn(1.0f + Q);
            msw[4 * i + j] = mj[j] * (W.S * wj[j]);
            po[4 * i + j] = oj[j];
        }
        *reinterpret_cast<float4*>(sw + s) = make_float4(wj[0], wj[1], wj[2], wj[3]);
        *reinterpret_cast<float4*>(sphi + s) = c4;
    }
    __syncthreads();  // the brick's phi^n and w are in shared memory
    const int pairs = k / 2;
    int pending = 0;
    __shared__ int s_abort;
    for (int t = 0; t < k; ++t) {
        // This iteration's output buffer, as enqueue_wave_f32 sequences them:
        // pairs write the two free buffers f0 then f1, an odd last one f0.
        int ob;
        if (t < 2 * pairs && (t & 1)) {
            ob = pending;
        } else {
            int f0, f1;
            ring_free_dev(old, cur, f0, f1);
            ob = f0;
            pending = f1;
        }
        const float* rd = sphi + (t & 1) * kRzBrick;
        float* wr = sphi + ((t + 1) & 1) * kRzBrick;
        float* out_g = ring + ob * cz;
        const bool last = t == k - 1;
        // One row: every load from shared memory and unconditional (the
        // neighbour row is in the brick or in the staged halo: a warp-uniform
        // address choice; face cells discard the value).
        auto row = [&](int i) {
            int yl, zl;
            rz_row(wid, i, yl, zl);
            const int y = y0 + yl, z = z0 + zl;
            const int s = sidx(yl, zl);
            const float* pzm = zl > 0 ? rd + s - kSRow : shalo + rz_halo_zm(yl) * kRzNX + x0;
            const float* pzp = zl < kRzBZ - 1 ? rd + s + kSRow : shalo + rz_halo_zp(yl) * kRzNX + x0;
            const float* pym = yl > 0 ? rd + s - kRzNX : shalo + rz_halo_ym(zl) * kRzNX + x0;
            const float* pyp = yl < kRzBY - 1 ? rd + s + kRzNX : shalo + rz_halo_yp(zl) * kRzNX + x0;
            const float4 c4 = *reinterpret_cast<const float4*>(rd + s);
            const float4 zm4 = *reinterpret_cast<const float4*>(pzm);
            const float4 zp4 = *reinterpret_cast<const float4*>(pzp);
            const float4 ym4 = *reinterpret_cast<const float4*>(pym);
            const float4 yp4 = *reinterpret_cast<const float4*>(pyp);
            const float4 w4 = *reinterpret_cast<const float4*>(sw + s);
            float left = __shfl_up_sync(0xffffffffu, c4.w, 1);
            float right = __shfl_down_sync(0xffffffffu, c4.x, 1);
            if (lane == 0) left = c4.x;    // x = 0 is a face
            if (lane == 31) right = c4.w;  // x = nx - 1 is a face
            const float cj[4] = {c4.x, c4.y, c4.z, c4.w};
            const float xm[4] = {left, c4.x, c4.y, c4.z}, xp[4] = {c4.y, c4.z, c4.w, right};
            const float ym[4] = {ym4.x, ym4.y, ym4.z, ym4.w}, yp[4] = {yp4.x, yp4.y, yp4.z, yp4.w};
            const float zmj[4] = {zm4.x, zm4.y, zm4.z, zm4.w}, zpj[4] = {zp4.x, zp4.y, zp4.z, zp4.w};
            const float wj[4] = {w4.x, w4.y, w4.z, w4.w};
            const bool rface = y == 0 || y == kRzNX - 1 || z == 0 || z == kRzNX - 1;
            const float sy = __ldg(W.sy + y), sz = __ldg(W.sz + z);
            float oj[4];
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const int u = 4 * i + j;
                const float nb = ((xm[j] + xp[j]) + (ym[j] + yp[j])) + (zmj[j] + zpj[j]);
                const float sxy = sxb[j] + sy;
                const float diss = sxy + sz;
                const float Q = diss * W.cdt_half;
                const float w = wj[j];
                const float val = fmaf(nb, W.K * w, fmaf(cj[j], W.A * w, fmaf(po[u], (Q - 1.0f) * w, msw[u])));
                const bool face = rface || (lane == 0 && j == 0) || (lane == 31 && j == 3);
                oj[j] = face ? 0.0f : val;
                po[u] = cj[j];
            }
            const float4 o4 = make_float4(oj[0], oj[1], oj[2], oj[3]);
            *reinterpret_cast<float4*>(wr + s) = o4;
            // Face rows every iteration (the neighbours read them), interior
            // rows on the last one.
            if (last || !rz_interior_slot(wid, i)) *reinterpret_cast<float4*>(out_g + gidx(yl, zl)) = o4;
        };
        // Interior rows first: they need nothing from the neighbours, so they
        // run while the neighbours finish the previous iteration.
#pragma unroll
        for (int i = 0; i < kRzSlots; ++i)
            if (rz_interior_slot(wid, i)) row(i);
        if (tid == 0) {
            int abort = 0;
            if (t > 0) {
                // All counters in flight together; the abort flag and the
                // clock only every 64th poll.  A missing neighbour (a mesh
                // face) is stood in for by the brick's own counter (>= t).
                const unsigned* fn[4] = {flag + rz_neighbour(b, 0), flag + rz_neighbour(b, 1),
                                         flag + rz_neighbour(b, 2), flag + rz_neighbour(b, 3)};
                const unsigned need = static_cast<unsigned>(t);
                auto ready = [&]() {
                    const unsigned a0 = ld_acquire_gpu(fn[0]), a1 = ld_acquire_gpu(fn[1]);
                    const unsigned a2 = ld_acquire_gpu(fn[2]), a3 = ld_acquire_gpu(fn[3]);
                    return a0 >= need && a1 >= need && a2 >= need && a3 >= need;
                };
                if (!ready()) {
                    const uint64_t t0 = global_ns();
                    for (unsigned spin = 1;; ++spin) {
                        if (ready()) break;
                        if ((spin & 63u) == 0u) {
                            if (ld_acquire_gpu(flag + kRzBricks) != 0u) {
                                abort = 1;
                                break;
                            }
                            if (global_ns() - t0 > limit_ns) {
                                atomicOr(err, kErrTimeout);
                                st_release_gpu(flag + kRzBricks, 1u);
                                abort = 1;
                                break;
                            }
                        }
                    }
                }
            }
            s_abort = abort;
        }
        __syncthreads();
        if (s_abort) return;  // uniform across the CTA; no barrier follows
        // The 48 rows of the neighbour bricks this brick reads, staged in
        // shared memory: three independent 16-byte loads per thread through
        // L2 (ld.cg: the neighbours rewrote them since this CTA last read the
        // buffer); rows outside the mesh are zeros (only face cells, whose
        // value is discarded, would read them).
        const float* gcur = ring + cur * cz;
#pragma unroll
        for (int r = 0; r < kRzHaloVec / kRzThreads; ++r) {
            const int q = tid + r * kRzThreads, hr = q >> 5, hx = 4 * (q & 31);
            int gy, gz;
            rz_halo_source(hr, by, bz, gy, gz);
            float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
            if (gy >= 0 && gy < kRzNX && gz >= 0 && gz < kRzNX)
                v = __ldcg(reinterpret_cast<const float4*>(gcur + static_cast<int64_t>(gz) * kRzPlane +
                                                           static_cast<int64_t>(gy) * kRzNX + hx));
            *reinterpret_cast<float4*>(shalo + hr * kRzNX + hx) = v;
        }
        __syncthreads();
#pragma unroll
        for (int i = 0; i < kRzSlots; ++i)
            if (!rz_interior_slot(wid, i)) row(i);
        __syncthreads();  // the brick is written (shared and global); rd and the halo are free
        // The barrier orders the CTA's stores before thread 0's release.
        // (withhold: the failure probe's brick that never publishes, so its
        // neighbours' waits run out; -1 in every solve)
        if (tid == 0 && b != withhold) st_release_gpu(flag + b, static_cast<unsigned>(t + 1));
        old = cur;
        cur = ob;
    }
    // phi^{k-1} (now in po) of the interior rows, which no neighbour reads:
    // its face rows were written by iteration k - 2 (for k = 1 the buffer is
    // the input, whole).
    if (k >= 2) {
        float* og = ring + old * cz;
#pragma unroll
        for (int i = 0; i < kRzSlots; ++i) {
            if (!rz_interior_slot(wid, i)) continue;
            int yl, zl;
            rz_row(wid, i, yl, zl);
            *reinterpret_cast<float4*>(og + gidx(yl, zl)) =
                make_float4(po[4 * i], po[4 * i + 1], po[4 * i + 2], po[4 * i + 3]);
        }
    }
    if (resid) {
        // The residual of the last iteration from the two shared buffers it
        // leaves: phi^k (written) and phi^{k-1} (read).
        const float* pk = sphi + (k & 1) * kRzBrick;
        const float* pk1 = sphi + ((k - 1) & 1) * kRzBrick;
        double d2 = 0.0, n2 = 0.0;
#pragma unroll
        for (int i = 0; i < kRzSlots; ++i) {
            int yl, zl;
            rz_row(wid, i, yl, zl);
            const int s = sidx(yl, zl);
            const float4 a4 = *reinterpret_cast<const float4*>(pk + s);
            const float4 c4 = *reinterpret_cast<const float4*>(pk1 + s);
            const float aj[4] = {a4.x, a4.y, a4.z, a4.w}, cj[4] = {c4.x, c4.y, c4.z, c4.w};
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const double dd = static_cast<double>(aj[j]) - static_cast<double>(cj[j]);
                d2 += dd * dd;
                n2 += static_cast<double>(aj[j]) * static_cast<double>(aj[j]);
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            d2 += __shfl_xor_sync(0xffffffffu, d2, o);
            n2 += __shfl_xor_sync(0xffffffffu, n2, o);
        }
        if (lane == 0) {
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

// ---- cloud-in-cell ----------------------------------------------------------
// One axis: u = (p - lo)/cs - 1/2 in cell-centre units; corners floor(u) and
// floor(u) + 1 with weights 1 - f and f.  Far-away (and NaN) coordinates map
// to corners that are both outside the mesh.
struct CicAxis {
    int i0;
    double w[2];
};

__device__ __forceinline__ CicAxis cic_axis(double p, double lo, double cs, double rcs, int g) {
    const double u = div_rn(p - lo, cs, rcs) - 0.5;
    const double fl = floor(u);
    CicAxis a;
    a.i0 = fl >= -1.0 ? (fl <= static_cast<double>(g) ? static_cast<int>(fl) : g) : -2;
    const double f = u - fl;
    a.w[0] = 1.0 - f;
    a.w[1] = f;
    return a;
}

__global__ void cic_deposit_kernel(const double* __restrict__ pos, const double* __restrict__ mass, int64_t n,
                                   const MeshGeom m, double* __restrict__ cell_mass) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const CicAxis ax = cic_axis(pos[3 * i], m.lo[0], m.cs[0], m.rcs[0], m.g[0]);
    const CicAxis ay = cic_axis(pos[3 * i + 1], m.lo[1], m.cs[1], m.rcs[1], m.g[1]);
    const CicAxis az = cic_axis(pos[3 * i + 2], m.lo[2], m.cs[2], m.rcs[2], m.g[2]);
    const double mi = mass[i];
#pragma unroll
    for (int c = 0; c < 2; ++c) {
        const int z = az.i0 + c;
        if (z < 0 || z >= m.g[2]) continue;
#pragma unroll
        for (int b = 0; b < 2; ++b) {
            const int y = ay.i0 + b;
            if (y < 0 || y >= m.g[1]) continue;
#pragma unroll
            for (int a = 0; a < 2; ++a) {
                const int x = ax.i0 + a;
                if (x < 0 || x >= m.g[0]) continue;
                const double w = (ax.w[a] * ay.w[b]) * az.w[c];
                atomicAdd(&cell_mass[static_cast<int64_t>(z) * m.g[0] * m.g[1] + static_cast<int64_t>(y) * m.g[2] + x],
                          mi * w);
            }
        }
    }
}

// Interpolation back to a body: acc (3 per cell) and a scalar field in FP32
// or FP64; sums in z, y, x corner order.
template <class T>
__device__ __forceinline__ void cic_interp(const double* __restrict__ p, const MeshGeom& m,
                                           const double* __restrict__ cacc, const T* __restrict__ cval, double (&acc)[3],
                                           double& val) {
    const CicAxis ax = cic_axis(p[0], m.lo[0], m.cs[0], m.rcs[0], m.g[0]);
    const CicAxis ay = cic_axis(p[1], m.lo[1], m.cs[1], m.rcs[1], m.g[1]);
    const CicAxis az = cic_axis(p[2], m.lo[2], m.cs[2], m.rcs[2], m.g[2]);
    acc[0] = acc[1] = acc[2] = 0.0;
    val = 0.0;
#pragma unroll
    for (int c = 0; c < 2; ++c) {
        const int z = az.i0 + c;
        if (z < 0 || z >= m.g[2]) continue;
#pragma unroll
        for (int b = 0; b < 2; ++b) {
            const int y = ay.i0 + b;
            if (y < 0 || y >= m.g[1]) continue;
#pragma unroll
            for (int a = 0; a < 2; ++a) {
                const int x = ax.i0 + a;
                if (x < 0 || x >= m.g[0]) continue;
                const double w = (ax.w[a] * ay.w[b]) * az.w[c];
                const int64_t id = static_cast<int64_t>(z) * m.g[0] * m.g[1] + static_cast<int64_t>(y) * m.g[2] + x;
                if (cacc) {
                    acc[0] += w * cacc[3 * id];
                    acc[1] += w * cacc[3 * id + 1];
                    acc[2] += w * cacc[3 * id + 2];
                }
                if (cval) val += w * static_cast<double>(cval[id]);
            }
        }
    }
}

__global__ void cic_gather_kernel(const double* __restrict__ pos, int64_t n, const MeshGeom m,
                                  const double* __restrict__ cacc, const double* __restrict__ cval,
                                  double* __restrict__ pacc, double* __restrict__ pval) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    double a[3], v;
    cic_interp(pos + 3 * i, m, pacc ? cacc : nullptr, pval ? cval : nullptr, a, v);
    if (pacc) {
        pacc[3 * i] = a[0];
        pacc[3 * i + 1] = a[1];
        pacc[3 * i + 2] = a[2];
    }
    if (pval) pval[i] = v;
}

// The mesh-force gather into the corrector's partial slot: {acc, -phi}, so
// the corrector's phi = 0 - (-phi) is the mesh potential (apply_acceleration_
// to_particles and apply_cell_to_particles, p2mesh-kernel.cuh:227-254).
template <bool CIC, class T>
__global__ void mesh_gather_kernel(const double* __restrict__ pos, const int2* __restrict__ pci, int64_t n,
                                   const MeshGeom m, const double* __restrict__ cacc, const T* __restrict__ phi,
                                   double4* __restrict__ part) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    double a[3], v;
    if (CIC) {
        cic_interp(pos + 3 * i, m, cacc, phi, a, v);
    } else {
        const int64_t c = pci[i].x;
        a[0] = cacc[3 * c];
        a[1] = cacc[3 * c + 1];
        a[2] = cacc[3 * c + 2];
        v = static_cast<double>(phi[c]);
    }
    part[i] = make_double4(a[0], a[1], a[2], -v);
}

// acc_field on an FP32 potential: the float differences are exact in FP64.
__global__ void acc_field_f32_kernel(double* __restrict__ cell_acc, const float* __restrict__ phi, int NX, double DX) {
    const int ix = blockIdx.x * blockDim.x + threadIdx.x;
    const int iy = blockIdx.y * blockDim.y + threadIdx.y;
    const int iz = blockIdx.z;
    if (ix >= NX || iy >= NX) return;
    const int64_t at = at3(ix, iy, iz, NX);
    const double p0 = phi[at];
    double d[3];
    if (ix == 0) d[0] = static_cast<double>(phi[at3(ix + 1, iy, iz, NX)]) - p0;
    else if (ix == NX - 1) d[0] = p0 - static_cast<double>(phi[at3(ix - 1, iy, iz, NX)]);
    else d[0] = 0.5 * (static_cast<double>(phi[at3(ix + 1, iy, iz, NX)]) - static_cast<double>(phi[at3(ix - 1, iy, iz, NX)]));
    if (iy == 0) d[1] = static_cast<double>(phi[at3(ix, iy + 1, iz, NX)]) - p0;
    else if (iy == NX - 1) d[1] = p0 - static_cast<double>(phi[at3(ix, iy - 1, iz, NX)]);
    else d[1] = 0.5 * (static_cast<double>(phi[at3(ix, iy + 1, iz, NX)]) - static_cast<double>(phi[at3(ix, iy - 1, iz, NX)]));
    if (iz == 0) d[2] = static_cast<double>(phi[at3(ix, iy, iz + 1, NX)]) - p0;
    else if (iz == NX - 1) d[2] = p0 - static_cast<double>(phi[at3(ix, iy, iz - 1, NX)]);
    else d[2] = 0.5 * (static_cast<double>(phi[at3(ix, iy, iz + 1, NX)]) - static_cast<double>(phi[at3(ix, iy, iz - 1, NX)]));
    const double coef = -1. / DX;
    cell_acc[3 * at] = d[0] * coef;
    cell_acc[3 * at + 1] = d[1] * coef;
    cell_acc[3 * at + 2] = d[2] * coef;
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
    assign_kernel<<<static_cast<unsigned>((n + 256 * kAssignPer - 1) / (256 * kAssignPer)), 256, 0, s>>>(
        pos, n, m, pci, counter, counter_stride, count2, count2_stride, mass, cell_mass);
    return cudaGetLastError();
}

int64_t scan_block_count(int64_t ncells) { return (ncells + kRefBlock - 1) / kRefBlock; }

int64_t scan_scratch_ints(int64_t ncells) { return (ncells + kScanTile - 1) / kScanTile; }

cudaError_t launch_scan(int* count, bool pair, int64_t ncells, int* maxpbc, int* start, bool ref_view, int* scratch,
                        cudaStream_t s) {
    if (ncells < 1) return cudaSuccess;
    const int64_t tiles = (ncells + kScanTile - 1) / kScanTile;
    int* tile_tot = scratch;
    const unsigned g = static_cast<unsigned>(tiles);
    if (pair) scan_totals_kernel<true><<<g, kScanThreads, 0, s>>>(count, ncells, tile_tot);
    else scan_totals_kernel<false><<<g, kScanThreads, 0, s>>>(count, ncells, tile_tot);
    scan_tiles_kernel<<<1, 1024, 0, s>>>(tile_tot, tiles);
    if (pair) scan_downsweep_kernel<true><<<g, kScanThreads, 0, s>>>(count, ncells, tile_tot, maxpbc, start, ref_view);
    else scan_downsweep_kernel<false><<<g, kScanThreads, 0, s>>>(count, ncells, tile_tot, maxpbc, start, ref_view);
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
    // One cell per thread: the FP64 update is bound by its FP64 arithmetic,
    // so occupancy (48 registers) beats more cells per thread (measured at
    // 256^3: 151.7 us per iteration against 155.9 for 2 and 169.3 for 4).
    const dim3 block(32, 8), grid((w.nx + 31) / 32, (w.nx + 7) / 8, w.nx);
    wave_f64_kernel<1><<<grid, block, 0, s>>>(phi_new, phi, phi_old, mass, w);
    return cudaGetLastError();
}

cudaError_t launch_wave_f32(float* phi_new, const float* phi, const float* phi_old, const float* mass,
                            const WaveF32& w, double* resid, cudaStream_t s) {
    // Launched with programmatic stream serialization: a chain of steps
    // overlaps each grid's launch with the previous grid's tail (measured
    // ~2 % on the 507-step Wave-mode chain at 128^3; same bits).
    cudaLaunchConfig_t cfg = {};
    cfg.blockDim = dim3(kWX, kWY);
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    // Kernel choice, measured (us per iteration, 128^3 / 256^3): one cell per
    // thread with 4 / 8 z planes 12.5 / 71.8; four x cells per thread with 2 z
    // planes 12.0 / 72.3 (with 4 planes 12.8 / 79.6).
    if (w.nx < 192 && w.nx % 4 == 0 && w.nx >= 8) {
        cfg.blockDim = dim3(kW4X, kW4Y);
        cfg.gridDim = dim3((w.nx + 4 * kW4X - 1) / (4 * kW4X), (w.nx + kW4Y - 1) / kW4Y, (w.nx + 1) / 2);
        return cudaLaunchKernelEx(&cfg, wave_f32x4_kernel<2>, phi_new, phi, phi_old, mass, w, resid);
    }
    if (w.nx >= 192) {
        cfg.gridDim = dim3((w.nx + kWX - 1) / kWX, (w.nx + kWY - 1) / kWY, (w.nx + 7) / 8);
        return cudaLaunchKernelEx(&cfg, wave_f32_kernel<8>, phi_new, phi, phi_old, mass, w, resid);
    }
    cfg.gridDim = dim3((w.nx + kWX - 1) / kWX, (w.nx + kWY - 1) / kWY, (w.nx + 3) / 4);
    return cudaLaunchKernelEx(&cfg, wave_f32_kernel<4>, phi_new, phi, phi_old, mass, w, resid);
}

bool wave_resident_available(int nx) {
    if (nx != kRzNX) return false;
    static const bool ok = [] {
        int dev = 0, sms = 0, coop = 0, occ = 0;
        if (cudaGetDevice(&dev) != cudaSuccess ||
            cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
            cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev) != cudaSuccess || !coop)
            return false;
        if (cudaFuncSetAttribute(wave_resident_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 static_cast<int>(kRzSmem)) != cudaSuccess ||
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, wave_resident_kernel, kRzThreads, kRzSmem) !=
                cudaSuccess)
            return false;
        return occ >= 1 && static_cast<int64_t>(occ) * sms >= kRzBricks;
    }();
    return ok;
}

cudaError_t launch_wave_resident(float* ring, int64_t cells, const float* mass, const WaveF32& w, int k, int st,
                                 double* resid, unsigned* sync, unsigned* err, cudaStream_t s,
                                 unsigned long long limit_ns, int withhold) {
    if (k < 1) return cudaSuccess;
    cudaError_t e = cudaMemsetAsync(sync, 0, (kRzBricks + 1) * sizeof(unsigned), s);
    if (e != cudaSuccess) return e;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(kRzBricks);
    cfg.blockDim = dim3(kRzThreads);
    cfg.dynamicSmemBytes = kRzSmem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, wave_resident_kernel, ring, cells, mass, w, k, st, resid, sync, err, limit_ns,
                              withhold);
}

cudaError_t enqueue_wave_f32(float* ring, int64_t cells, const float* mass, const WaveF32& w, int k, int st,
                             double* resid, cudaStream_t s, const WaveMaps* maps, unsigned* err) {
    const size_t cz = static_cast<size_t>(cells);
    if (maps && maps->resident && maps->sync && err && w.nx == kRzNX)
        return launch_wave_resident(ring, cells, mass, w, k, st, resid, maps->sync, err, s);
    const bool tma = maps && maps->ok && err;
    // One iteration: buffer `out` from phi^n in `cur` and phi^{n-1} in `old`.
    auto single = [&](int old, int cur, int out, double* r) {
        if (tma)
            return launch_wave1_tma(ring + out * cz, maps->halo[cur], maps->tile[old], maps->tile_mass, w, r, err, s);
        return launch_wave_f32(ring + out * cz, ring + cur * cz, ring + old * cz, mass, w, r, s);
    };
    for (int i = 0; i + 1 < k; i += 2) {
        int f0, f1;
        ring_free(st, f0, f1);
        double* r = i + 2 == k ? resid : nullptr;
        cudaError_t e;
        if (tma && maps->two_step) {
            e = launch_wave2_tma(ring + f0 * cz, ring + f1 * cz, maps->ring[st % 4], maps->ring[st / 4], maps->mass, w,
                                 r, err, s);
        } else {  // two single steps: phi^{n+1} into f0, phi^{n+2} into f1
            e = single(st / 4, st % 4, f0, nullptr);
            if (e == cudaSuccess) e = single(st % 4, f0, f1, r);
        }
        if (e != cudaSuccess) return e;
        st = ring_step2(st);
    }
    if (k % 2) {
        int f0, f1;
        ring_free(st, f0, f1);
        cudaError_t e = single(st / 4, st % 4, f0, resid);
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

cudaError_t launch_wave1_tma(float* phi_new, const CUtensorMap& phi, const CUtensorMap& phi_old,
                             const CUtensorMap& mass, const WaveF32& w, double* resid, unsigned* err, cudaStream_t s) {
    const dim3 block((kW1Consumers + 1) * 32);
    if (w.nx >= 192) {
        const dim3 grid((w.nx + 31) / 32, (w.nx + 7) / 8, (w.nx + 31) / 32);
        wave1_tma_kernel<32><<<grid, block, 0, s>>>(phi_new, phi, phi_old, mass, w, resid, err);
    } else {
        const dim3 grid((w.nx + 31) / 32, (w.nx + 7) / 8, (w.nx + 15) / 16);
        wave1_tma_kernel<16><<<grid, block, 0, s>>>(phi_new, phi, phi_old, mass, w, resid, err);
    }
    return cudaGetLastError();
}

cudaError_t launch_wave2_tma(float* out1, float* out2, const CUtensorMap& phi, const CUtensorMap& phi_old,
                             const CUtensorMap& mass, const WaveF32& w, double* resid, unsigned* err, cudaStream_t s) {
    const dim3 block(kT2Threads);
    if (w.nx >= 192) {
        const dim3 grid((w.nx + kT2X - 1) / kT2X, (w.nx + kT2Y - 1) / kT2Y, (w.nx + 31) / 32);
        wave2_tma_kernel<32><<<grid, block, 0, s>>>(out1, out2, phi, phi_old, mass, w, resid, err);
    } else {
        const dim3 grid((w.nx + kT2X - 1) / kT2X, (w.nx + kT2Y - 1) / kT2Y, (w.nx + 15) / 16);
        wave2_tma_kernel<16><<<grid, block, 0, s>>>(out1, out2, phi, phi_old, mass, w, resid, err);
    }
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

cudaError_t launch_cic_deposit(const double* pos, const double* mass, int64_t n, const MeshGeom& m,
                               double* cell_mass, cudaStream_t s) {
    if (n < 1) return cudaSuccess;
    cic_deposit_kernel<<<static_cast<unsigned>((n + 255) / 256), 256, 0, s>>>(pos, mass, n, m, cell_mass);
    return cudaGetLastError();
}

cudaError_t launch_cic_gather(const double* pos, int64_t n, const MeshGeom& m, const double* cell_acc,
                              const double* cell_value, double* pacc, double* pval, cudaStream_t s) {
    if (n < 1) return cudaSuccess;
    cic_gather_kernel<<<static_cast<unsigned>((n + 255) / 256), 256, 0, s>>>(pos, n, m, cell_acc, cell_value, pacc,
                                                                               pval);
    return cudaGetLastError();
}

cudaError_t launch_scatter_order(const int2* pci, const int* start, int64_t n, int base, int* order, cudaStream_t s) {
    if (n < 1) return cudaSuccess;
    scatter_order_kernel<<<static_cast<unsigned>((n + 255) / 256), 256, 0, s>>>(pci, start, n, base, order);
    return cudaGetLastError();
}

cudaError_t launch_mesh_gather(const double* pos, const int2* pci, int64_t n, const MeshGeom& m, bool cic,
                               const double* cell_acc, const float* phi32, const double* phi64, double4* part,
                               cudaStream_t s) {
    if (n < 1) return cudaSuccess;
    const unsigned g = static_cast<unsigned>((n + 255) / 256);
    if (cic) {
        if (phi32) mesh_gather_kernel<true, float><<<g, 256, 0, s>>>(pos, pci, n, m, cell_acc, phi32, part);
        else mesh_gather_kernel<true, double><<<g, 256, 0, s>>>(pos, pci, n, m, cell_acc, phi64, part);
    } else {
        if (phi32) mesh_gather_kernel<false, float><<<g, 256, 0, s>>>(pos, pci, n, m, cell_acc, phi32, part);
        else mesh_gather_kernel<false, double><<<g, 256, 0, s>>>(pos, pci, n, m, cell_acc, phi64, part);
    }
    return cudaGetLastError();
}

cudaError_t launch_acc_field_f32(double* cell_acc, const float* phi, int nx, double dx, cudaStream_t s) {
    const dim3 block(32, 8), grid((nx + 31) / 32, (nx + 7) / 8, nx);
    acc_field_f32_kernel<<<grid, block, 0, s>>>(cell_acc, phi, nx, dx);
    return cudaGetLastError();
}

cudaError_t launch_assign_cells(const double* pos, int64_t n, const MeshGeom& m, int2* pci, const double* mass,
                                double* cell_mass, cudaStream_t s) {
    if (n < 1) return cudaSuccess;
    assign_cells_kernel<<<static_cast<unsigned>((n + 255) / 256), 256, 0, s>>>(pos, n, m, pci, mass, cell_mass);
    return cudaGetLastError();
}

}  // namespace khrr
