// Geometry of the resident 128^3 FP32 stencil (wave_resident_kernel in
// mesh.cu): the mesh cut into 128 bricks of 128 (x) x 16 (y) x 8 (z) cells,
// one CTA each; a warp of a brick owns 8 of its 128 rows of 128 x cells; the
// 48 rows of the four neighbour bricks that touch the brick are staged in
// shared memory each iteration.  Host and device code both include this
// file: the kernel uses it, and a CPU check (tests/wave_bricks_check.cpp)
// verifies that the row map, the halo rows and the neighbour counters fit
// together.
#pragma once

#ifdef __CUDACC__
#define KHRR_HD __host__ __device__ __forceinline__
#else
#define KHRR_HD inline
#endif

namespace khrr {

constexpr int kRzNX = 128;                                   // mesh edge
constexpr int kRzBY = 16, kRzBZ = 8;                         // brick rows in y and z
constexpr int kRzBricksY = kRzNX / kRzBY;                    // 8
constexpr int kRzBricks = kRzBricksY * (kRzNX / kRzBZ);      // 128
constexpr int kRzThreads = 32 * kRzBY;                       // 16 warps
constexpr int kRzSlots = kRzBY * kRzBZ / (kRzThreads / 32);  // rows per warp (8)
constexpr int kRzCells = 4 * kRzSlots;                       // cells per thread
constexpr int kRzPlane = kRzNX * kRzNX;
constexpr int kRzBrick = kRzNX * kRzBY * kRzBZ;              // 16,384 cells
constexpr int kRzHaloRows = 2 * kRzBZ + 2 * kRzBY;           // 48
constexpr int kRzHalo = kRzHaloRows * kRzNX;                 // the neighbour rows read, 6,144 cells
constexpr int kRzHaloVec = kRzHalo / 4;
static_assert(kRzHaloVec % kRzThreads == 0, "whole halo loads per thread");
static_assert(kRzNX == 4 * 32 && kRzNX % kRzBY == 0 && kRzNX % kRzBZ == 0, "a warp covers a row, four cells per lane");
static_assert(kRzBricks <= kRzNX, "the counters (nx + 1 words, allocated by the mesh set-up) cover the bricks and the abort flag");

// The brick's rows: 84 interior rows (1 <= yl <= 14, 1 <= zl <= 6), which no
// neighbour reads and whose neighbours all lie in the brick, and 44 face rows
// (yl in {0, 15} or zl in {0, 7}).  Warp w owns 8 rows for the whole launch:
// slots 0-4 are interior rows w + 16 m; slot 5 is interior row 80 + (w - 12)
// for w >= 12 and face row w for w < 12; slots 6, 7 are face rows
// w + 16 (m + [w < 12]).  Face row f: zl = 0 for f < 16, zl = 7 for f >= 28,
// otherwise zl = 1 + (f - 16) / 2 at yl = 0 or 15.
static_assert(kRzBY == 16 && kRzBZ == 8 && kRzSlots == 8, "the row map below is written for 16 x 8 rows, 16 warps");
KHRR_HD bool rz_interior_slot(int w, int i) { return i < 5 || (i == 5 && w >= 12); }

KHRR_HD void rz_row(int w, int i, int& yl, int& zl) {
    if (rz_interior_slot(w, i)) {
        const int ii = i < 5 ? w + 16 * i : 80 + (w - 12);
        zl = 1 + ii / 14;
        yl = 1 + ii % 14;
    } else {
        const int f = w + 16 * (i - (w < 12 ? 5 : 6));
        if (f < 16) {
            zl = 0;
            yl = f;
        } else if (f >= 28) {
            zl = kRzBZ - 1;
            yl = f - 28;
        } else {
            zl = 1 + (f - 16) / 2;
            yl = (f - 16) & 1 ? kRzBY - 1 : 0;
        }
    }
}

// Staged halo rows, by index in the halo area: the y - 1 row of plane zl at
// zl, the y + BY row at BZ + zl, the z - 1 row of column yl at 2 BZ + yl and
// the z + BZ row at 2 BZ + BY + yl.
KHRR_HD int rz_halo_ym(int zl) { return zl; }
KHRR_HD int rz_halo_yp(int zl) { return kRzBZ + zl; }
KHRR_HD int rz_halo_zm(int yl) { return 2 * kRzBZ + yl; }
KHRR_HD int rz_halo_zp(int yl) { return 2 * kRzBZ + kRzBY + yl; }

// The mesh row (gy, gz) that halo row hr of brick (by, bz) is loaded from
// (outside the mesh for a brick on a mesh face: then it is zeros).
KHRR_HD void rz_halo_source(int hr, int by, int bz, int& gy, int& gz) {
    const int y0 = by * kRzBY, z0 = bz * kRzBZ;
    if (hr < 2 * kRzBZ) {
        gy = hr < kRzBZ ? y0 - 1 : y0 + kRzBY;
        gz = z0 + (hr % kRzBZ);
    } else {
        const int h = hr - 2 * kRzBZ;
        gy = y0 + (h % kRzBY);
        gz = h < kRzBY ? z0 - 1 : z0 + kRzBZ;
    }
}

// Neighbour bricks whose counters a brick waits on: y - 1, y + 1, z - 1,
// z + 1; a missing one (a mesh face) is the brick itself.
KHRR_HD int rz_neighbour(int b, int k) {
    const int by = b % kRzBricksY, bz = b / kRzBricksY;
    switch (k) {
        case 0: return by > 0 ? b - 1 : b;
        case 1: return by < kRzBricksY - 1 ? b + 1 : b;
        case 2: return bz > 0 ? b - kRzBricksY : b;
        default: return bz * kRzBZ + kRzBZ < kRzNX ? b + kRzBricksY : b;
    }
}

}  // namespace khrr
