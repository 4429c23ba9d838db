// Host-side check of the symmetric pair kernel's work plan (plan_pair_items
// in libkhrr), run on the CPU by tests/test_pair_plan.py.  For a layout of
// systems, with 1024-body blocks or with the blocks the block-mass form uses
// (runs of equal-mass 128-body tiles, here two components per system with the
// first a third of the bodies rounded down to whole tiles), it replays every
// item as the kernel executes it:
//   * evaluations, per ordered pair of 128-body tiles: the item's tiles of
//     its own block ([j_begin, diag_end)) once, (i tile, j tile); every later
//     tile twice, (i, j) and (j, i).  Every ordered pair of tiles of the same
//     system must be evaluated exactly once, and none across systems.
//   * sums: the i block's sums over the chunk go to the block's real bodies,
//     each symmetric tile's reactions to the tile's real bodies (both into
//     the bodies' fixed-point accumulators).  real_end must be the end of the
//     item's system's real bodies, so ghosts receive nothing, and every real
//     body must receive sums.
// Prints "ok <items>" per layout, or the first violation.
#include <cstdint>
#include <cstdio>
#include <algorithm>
#include <cstdlib>
#include <string>
#include <vector>

#include "khrr_runtime.h"

using namespace khrr;

namespace {

int fail(const std::string& what, long long a, long long b) {
    std::printf("FAIL %s (%lld, %lld)\n", what.c_str(), a, b);
    return 1;
}

int check(const std::vector<int64_t>& cnt, int ctas, int chunk, bool by_mass) {
    std::vector<int64_t> poff(cnt.size() + 1, 0);
    for (size_t k = 0; k < cnt.size(); ++k) poff[k + 1] = poff[k] + (cnt[k] + kPad - 1) / kPad * kPad;
    const int64_t npad = poff.back(), ntiles = npad / kPad;
    PairBlocks blocks = pair_blocks_fixed(poff);
    if (by_mass) {
        std::vector<float> tm(static_cast<size_t>(ntiles));
        for (size_t k = 0; k < cnt.size(); ++k) {
            const int64_t first = cnt[k] / 3 / kPad * kPad;
            for (int64_t t = poff[k] / kPad; t < poff[k + 1] / kPad; ++t)
                tm[t] = (t * kPad - poff[k] < first) ? 1.0f : 0.25f;
        }
        blocks = pair_blocks_by_mass(poff, tm);
        for (size_t k = 0; k < cnt.size(); ++k)
            for (size_t b = 0; b + 1 < blocks[k].size(); ++b) {
                const int64_t lo = blocks[k][b], hi = blocks[k][b + 1];
                if (hi - lo > kPairBlock || lo % kPad) return fail("bad block", lo, hi);
                for (int64_t t = lo / kPad; t < hi / kPad; ++t)
                    if (tm[t] != tm[lo / kPad]) return fail("block with two masses", lo, t);
            }
    }
    ForcePlan p;
    plan_pair_items(blocks, cnt, ctas, chunk, p);

    std::vector<int> sys_of_tile(ntiles);
    for (size_t k = 0; k < cnt.size(); ++k)
        for (int64_t t = poff[k] / kPad; t < poff[k + 1] / kPad; ++t) sys_of_tile[t] = static_cast<int>(k);
    std::vector<unsigned char> cover(static_cast<size_t>(ntiles * ntiles), 0);
    std::vector<int> received(static_cast<size_t>(npad), 0);
    auto hit = [&](int64_t a, int64_t b) { return ++cover[static_cast<size_t>(a * ntiles + b)] > 1; };

    for (const PairItem& w : p.pair_items) {
        if (w.i_begin % kPad || w.j_begin % kPad || w.j_end % kPad || w.i_end % kPad || w.diag_end % kPad)
            return fail("unaligned item", w.i_begin, w.j_begin);
        if (w.i_end - w.i_begin > kPairBlock || w.i_end <= w.i_begin || w.j_end <= w.j_begin)
            return fail("bad item extent", w.i_begin, w.i_end);
        if (w.diag_end != w.j_begin && !(w.j_begin == w.i_begin && w.diag_end == w.i_end))
            return fail("own-block tiles must be the item's i block", w.j_begin, w.diag_end);
        for (int64_t ti = w.i_begin / kPad; ti < w.i_end / kPad; ++ti)
            for (int64_t tj = w.j_begin / kPad; tj < w.j_end / kPad; ++tj) {
                if (sys_of_tile[ti] != sys_of_tile[tj]) return fail("pair across systems", ti, tj);
                if (hit(ti, tj)) return fail("ordered tile pair evaluated twice", ti, tj);
                if (tj * kPad >= w.diag_end && hit(tj, ti)) return fail("reverse tile pair evaluated twice", tj, ti);
            }
        const int64_t sys = sys_of_tile[w.i_begin / kPad];
        if (w.real_end != poff[sys] + cnt[sys]) return fail("real_end is not the system's real end", w.real_end, sys);
        for (int64_t i = w.i_begin; i < std::min<int64_t>(w.i_end, w.real_end); ++i) ++received[i];
        for (int64_t j = w.diag_end; j < std::min<int64_t>(w.j_end, w.real_end); ++j) ++received[j];
    }
    for (int64_t a = 0; a < ntiles; ++a)
        for (int64_t b = 0; b < ntiles; ++b) {
            const bool same = sys_of_tile[a] == sys_of_tile[b];
            if (cover[static_cast<size_t>(a * ntiles + b)] != (same ? 1 : 0)) return fail("tile pair not covered", a, b);
        }
    for (size_t k = 0; k < cnt.size(); ++k)
        for (int64_t i = poff[k]; i < poff[k] + cnt[k]; ++i)
            if (received[i] < 1) return fail("real body without sums", i, received[i]);
    std::printf("ok %zu\n", p.pair_items.size());
    return 0;
}

}  // namespace

// Arguments: fixed|mass ctas chunk n_0 [n_1 ...]
int main(int argc, char** argv) {
    if (argc < 5) {
        std::printf("usage: %s fixed|mass ctas chunk n0 [n1 ...]\n", argv[0]);
        return 2;
    }
    const bool by_mass = std::string(argv[1]) == "mass";
    const int ctas = std::atoi(argv[2]), chunk = std::atoi(argv[3]);
    std::vector<int64_t> cnt;
    for (int a = 4; a < argc; ++a) cnt.push_back(std::atoll(argv[a]));
    return check(cnt, ctas, chunk, by_mass);
}
