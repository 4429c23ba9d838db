// Host-side check of the resident 128^3 stencil's geometry (wave_bricks.h,
// the header the kernel itself uses), run on the CPU by
// tests/test_wave_bricks.py:
//   * the 16 warps x 8 slots of a brick cover its 128 rows exactly once, and
//     a slot is an interior slot exactly when its row has all four neighbour
//     rows inside the brick;
//   * the bricks tile the mesh's 128 x 128 rows exactly once, and every
//     shared-memory offset a row uses lies inside the brick buffer;
//   * every neighbour row a face row reads from the staged halo is loaded
//     from the right mesh row, that row belongs to the brick whose counter
//     is waited on, and its owner writes it every iteration (it is a face row
//     there); rows beyond a mesh face belong to no brick and the wait stands
//     in the brick itself;
//   * the staging loop loads each of the 48 halo rows' 32 float4s once;
//   * the neighbour relation is symmetric (a brick waits on the bricks that
//     wait on it).
// Prints "ok" or the first violation.
#include <cstdio>
#include <vector>

#include "wave_bricks.h"

using namespace khrr;

namespace {

int bad(const char* what, int a, int b, int c) {
    std::printf("FAIL %s (%d, %d, %d)\n", what, a, b, c);
    return 1;
}

// The brick owning mesh row (y, z), or -1 outside the mesh.
int owner(int y, int z) {
    if (y < 0 || y >= kRzNX || z < 0 || z >= kRzNX) return -1;
    return (z / kRzBZ) * kRzBricksY + y / kRzBY;
}

bool face_row_in_owner(int y, int z) {
    const int yl = y % kRzBY, zl = z % kRzBZ;
    for (int w = 0; w < kRzThreads / 32; ++w)
        for (int i = 0; i < kRzSlots; ++i) {
            int a, c;
            rz_row(w, i, a, c);
            if (a == yl && c == zl) return !rz_interior_slot(w, i);
        }
    return false;
}

// The halo row a face row reads for one direction: its index must be in
// range, loaded from (ey, ez), owned by the brick waited on (k).
int check_halo(int b, int hr, int ey, int ez, int k) {
    const int by = b % kRzBricksY, bz = b / kRzBricksY;
    if (hr < 0 || hr >= kRzHaloRows) return bad("halo index out of range", b, hr, k);
    int gy, gz;
    rz_halo_source(hr, by, bz, gy, gz);
    if (gy != ey || gz != ez) return bad("halo row loaded from the wrong mesh row", b, hr, k);
    const int o = owner(gy, gz);
    const int nb = rz_neighbour(b, k);
    if (o < 0) return nb == b ? 0 : bad("a mesh face waits on another brick", b, hr, k);
    if (o != nb) return bad("halo row owned by a brick that is not waited on", b, hr, k);
    if (!face_row_in_owner(gy, gz)) return bad("halo row is not written every iteration by its owner", b, hr, k);
    return 0;
}

}  // namespace

int main() {
    std::vector<int> mesh_rows(kRzNX * kRzNX, 0);
    for (int b = 0; b < kRzBricks; ++b) {
        const int by = b % kRzBricksY, bz = b / kRzBricksY;
        const int y0 = by * kRzBY, z0 = bz * kRzBZ;
        std::vector<int> seen(kRzBY * kRzBZ, 0);
        for (int w = 0; w < kRzThreads / 32; ++w)
            for (int i = 0; i < kRzSlots; ++i) {
                int yl, zl;
                rz_row(w, i, yl, zl);
                if (yl < 0 || yl >= kRzBY || zl < 0 || zl >= kRzBZ) return bad("row outside the brick", b, w, i);
                if (seen[zl * kRzBY + yl]++) return bad("row owned twice", b, w, i);
                const bool interior = yl > 0 && yl < kRzBY - 1 && zl > 0 && zl < kRzBZ - 1;
                if (interior != rz_interior_slot(w, i)) return bad("interior slot flag", b, w, i);
                for (int x0 = 0; x0 < kRzNX; x0 += 4) {
                    const int s = (zl * kRzBY + yl) * kRzNX + x0;
                    if (s < 0 || s + 4 > kRzBrick) return bad("shared offset outside the brick", b, w, i);
                }
                mesh_rows[(z0 + zl) * kRzNX + y0 + yl]++;
                if (interior) continue;
                // neighbours outside the brick come from the halo
                if (zl == 0 && check_halo(b, rz_halo_zm(yl), y0 + yl, z0 - 1, 2)) return 1;
                if (zl == kRzBZ - 1 && check_halo(b, rz_halo_zp(yl), y0 + yl, z0 + kRzBZ, 3)) return 1;
                if (yl == 0 && check_halo(b, rz_halo_ym(zl), y0 - 1, z0 + zl, 0)) return 1;
                if (yl == kRzBY - 1 && check_halo(b, rz_halo_yp(zl), y0 + kRzBY, z0 + zl, 1)) return 1;
            }
        for (int k = 0; k < 4; ++k) {
            const int a = rz_neighbour(b, k);
            if (a < 0 || a >= kRzBricks) return bad("neighbour out of range", b, k, a);
            if (a != b && rz_neighbour(a, k ^ 1) != b) return bad("neighbour relation not symmetric", b, k, a);
        }
    }
    for (int r = 0; r < kRzNX * kRzNX; ++r)
        if (mesh_rows[r] != 1) return bad("mesh row not covered exactly once", r, mesh_rows[r], 0);
    std::vector<int> staged(kRzHaloRows * 32, 0);
    for (int tid = 0; tid < kRzThreads; ++tid)
        for (int r = 0; r < kRzHaloVec / kRzThreads; ++r) {
            const int q = tid + r * kRzThreads, hr = q >> 5;
            if (hr >= kRzHaloRows) return bad("staging load past the halo", tid, r, hr);
            staged[hr * 32 + (q & 31)]++;
        }
    for (int v = 0; v < kRzHaloRows * 32; ++v)
        if (staged[v] != 1) return bad("halo float4 not staged exactly once", v, staged[v], 0);
    std::printf("ok\n");
    return 0;
}
