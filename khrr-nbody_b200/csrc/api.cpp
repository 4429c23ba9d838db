// Host runtime behind include/khrr.h: contexts, device state layout, work
// planning for the force pass, CUDA-graph time steps and device timing.
//
// Device layout (per context).  Bodies of system k occupy the padded index
// range [P_k, P_k + round_up(n_k, kPad)); the tail of each range holds
// zero-mass ghost bodies at the origin.  FP64 state is AoS double3 (the
// reference's layout, so uploads and downloads are straight copies): pos,
// vel, acc (a(t) without the external field), post/velt (predicted), acct
// (force workspace of the literal reference loop), mass, eps2, phi.  The force
// kernels read the FP32 structure-of-arrays shadow (x, y, z, m, eps2 / 2); the
// one-sided kernel writes FP64 partials part[slot][body], the symmetric pair
// kernel adds into 64-bit fixed-point sums fx[component][body].
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdlib>
#include <cstdio>
#include <cstring>
#include <map>
#include <string>
#include <thread>
#include <tuple>
#include <vector>

#include "khrr.h"
#include "khrr_internal.h"
#include "khrr_runtime.h"

using namespace khrr;

// ---------------------------------------------------------------------------
// helpers
// ---------------------------------------------------------------------------
namespace {

int64_t round_up(int64_t v, int64_t m) { return (v + m - 1) / m * m; }

// One 128-body tile of the caller's arrays (a system's tiles start at its
// first body; its last one may be partial): whether every softening is
// positive and equal to eps2[0], whether every mass equals the tile's first,
// the smallest h = eps2 / 2 and the sum of |m|.
struct TileScan {
    int64_t begin, end;
    int sys;
    bool pos_eps, same_eps, same_mass;
    double hmin, msum;
};

void scan_tile(const double* mass, const double* eps2, double e0, TileScan& t) {
    const double m0 = mass[t.begin];
    bool pos = true, same_e = true, same_m = true;
    double h = 1e300, s[4] = {0.0, 0.0, 0.0, 0.0};
    for (int64_t i = t.begin; i < t.end; ++i) {
        const double e = eps2[i], m = mass[i];
        pos &= e > 0.0;
        same_e &= e == e0;
        same_m &= m == m0;
        h = std::min(h, e);
        s[(i - t.begin) & 3] += std::fabs(m);  // four running sums, added pairwise
    }
    t.pos_eps = pos;
    t.same_eps = same_e;
    t.same_mass = same_m;
    t.hmin = 0.5 * h;
    t.msum = (s[0] + s[1]) + (s[2] + s[3]);
}

// All tiles of an upload.  The tiles are independent, so a large upload
// splits them over host threads; each tile's result is the same whatever the
// split.
std::vector<TileScan> scan_state_tiles(const double* mass, const double* eps2, const std::vector<int64_t>& off) {
    std::vector<TileScan> tiles;
    const int nsys = static_cast<int>(off.size()) - 1;
    tiles.reserve(static_cast<size_t>(off[nsys] / kPad + nsys));
    for (int k = 0; k < nsys; ++k)
        for (int64_t b = off[k]; b < off[k + 1]; b += kPad)
            tiles.push_back(TileScan{b, std::min(b + kPad, off[k + 1]), k, false, false, false, 0.0, 0.0});
    const double e0 = eps2[0];
    const unsigned hw = std::thread::hardware_concurrency();
    const int nthreads = off[nsys] < (int64_t(1) << 17) ? 1 : static_cast<int>(std::clamp(hw, 1u, 8u));
    const size_t per = (tiles.size() + nthreads - 1) / nthreads;
    auto work = [&](int r) {
        const size_t t1 = std::min(tiles.size(), (r + 1) * per);
        for (size_t t = r * per; t < t1; ++t) scan_tile(mass, eps2, e0, tiles[t]);
    };
    std::vector<std::thread> pool;
    int started = 1;
    try {
        for (; started < nthreads; ++started) pool.emplace_back(work, started);
    } catch (...) {
        // No more threads: the ranges not started run here.
    }
    for (int r = started; r < nthreads; ++r) work(r);
    work(0);
    for (std::thread& th : pool) th.join();
    return tiles;
}

}  // namespace

khrr_status khrr_ctx::fail(khrr_status s, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    std::vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    err = buf;
    return s;
}

khrr_status khrr_ctx::cuda(cudaError_t e, const char* what) {
    if (e == cudaSuccess) return KHRR_OK;
    if (e == cudaErrorMemoryAllocation)
        return fail(KHRR_ERR_OOM, "%s: %s", what, cudaGetErrorString(e));
    return fail(KHRR_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

khrr_status khrr_ctx::check_device_flag() {
    unsigned flag = 0;
    cudaError_t e = cudaMemcpyAsync(&flag, errflag.p, sizeof flag, cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) return cuda(e, "device error flag");
    if (flag & kErrTimeout) {
        cudaMemsetAsync(errflag.p, 0, sizeof(unsigned), stream);
        return fail(KHRR_ERR_TIMEOUT, "a kernel gave up a bounded wait (an asynchronous copy or a neighbour plane)");
    }
    return KHRR_OK;
}

int khrr_ctx::resident_ctas(const ForceVariant* v) {
    auto it = occupancy.find(v->fn);
    if (it != occupancy.end()) return it->second * sm_count;
    int occ = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, v->fn, v->threads, v->smem) != cudaSuccess ||
        occ < 1)
        occ = 1;
    occupancy[v->fn] = occ;
    return occ * sm_count;
}

// The pair kernel's sums take 32 bytes per body whatever the layout, and the
// state's softenings are positive (checked at upload), which the fixed-point
// bounds need: the tuning alone decides.
bool khrr_ctx::pair_mode() const { return tuning.packed == 2 && has_state; }

// The state's kernel: the symmetric pair kernel when the tuning asks for it
// (packed = 2) and the layout admits it; else the tile-mass form where the
// layout allows it and the shape has one, else the general form.
const ForceVariant* khrr_ctx::variant(bool unif, bool acc, bool phi) const {
    if (tuning.packed == 2) {
        if (pair_mode()) return find_pair_variant(unif, acc, phi, block_uniform_mass);
        if (tile_uniform_mass)
            if (const ForceVariant* v = find_force_variant(128, 4, 128, true, unif, acc, phi, true)) return v;
        return find_force_variant(128, 4, 128, true, unif, acc, phi, false);
    }
    const bool packed = tuning.packed != 0;
    if (tile_uniform_mass)
        if (const ForceVariant* v =
                find_force_variant(tuning.threads, tuning.i_per_thread, tuning.j_tile, packed, unif, acc, phi, true))
            return v;
    return find_force_variant(tuning.threads, tuning.i_per_thread, tuning.j_tile, packed, unif, acc, phi, false);
}

// ---------------------------------------------------------------------------
// work planning
// ---------------------------------------------------------------------------
namespace khrr {

// Splits of the j range for one system so that the persistent grid stays busy:
// with one system, the split that best fills the last wave of items; with
// several, a split per system that brings every item near a common cost, the
// items then run longest first.
void plan_force_items(const std::vector<int64_t>& poff, const std::vector<int64_t>& cnt, int itile,
                      int jt, int ctas, int forced_split, bool plain, ForcePlan& out) {
    out.items.clear();
    out.sys_item_begin.assign(cnt.size() + 1, 0);
    out.sys_split.assign(cnt.size(), 1);
    out.nslots = 1;
    const size_t nsys = cnt.size();
    std::vector<int> split(nsys, 1);
    double total_cost = 0.0;
    for (size_t k = 0; k < nsys; ++k) {
        const int64_t np = round_up(cnt[k], kPad);
        const int64_t nit = (cnt[k] + itile - 1) / itile;
        total_cost += static_cast<double>(nit) * itile * np;
    }
    for (size_t k = 0; k < nsys; ++k) {
        const int64_t np = round_up(cnt[k], kPad);
        const int tiles = static_cast<int>(np / jt);
        const int64_t nit = (cnt[k] + itile - 1) / itile;
        int s = 1;
        if (plain) {
            s = 1;
        } else if (forced_split > 0) {
            s = std::min(forced_split, tiles);
        } else if (nsys == 1) {
            // Best last-wave fill; chunks of at least 8 tiles; ties -> fewer chunks.
            double best = -1.0;
            const int smax = std::max(1, std::min(64, tiles / 8));
            for (int c = 1; c <= smax; ++c) {
                const double items = static_cast<double>(nit) * c;
                const double rounds = std::ceil(items / ctas);
                const double eff = items / (rounds * ctas);
                if (eff > best + 1e-9) {
                    best = eff;
                    s = c;
                }
                if (eff > 0.985) break;
            }
        } else {
            const double target = total_cost / (static_cast<double>(ctas) * 6.0);
            const double row = static_cast<double>(itile) * np;
            s = static_cast<int>(std::lround(row / std::max(target, 1.0)));
            s = std::max(1, std::min({s, tiles, 64}));
        }
        split[k] = s;
        out.sys_split[k] = s;
        out.nslots = std::max(out.nslots, s);
    }
    for (size_t k = 0; k < nsys; ++k) {
        out.sys_item_begin[k] = static_cast<int>(out.items.size());
        const int64_t np = round_up(cnt[k], kPad);
        const int tiles = static_cast<int>(np / jt);
        const int s = split[k];
        for (int64_t ib = 0; ib < cnt[k]; ib += itile) {
            for (int c = 0; c < s; ++c) {
                WorkItem w{};
                w.i_begin = static_cast<int>(poff[k] + ib);
                w.i_end = static_cast<int>(poff[k] + cnt[k]);
                w.j_begin = static_cast<int>(poff[k] + static_cast<int64_t>(c) * tiles / s * jt);
                w.j_end = static_cast<int>(poff[k] + static_cast<int64_t>(c + 1) * tiles / s * jt);
                w.slot = c;
                w.sys = static_cast<int>(k);
                w.pad0 = static_cast<int>(std::min<int64_t>(itile, cnt[k] - ib));  // i bodies in the tile
                out.items.push_back(w);
            }
        }
    }
    out.sys_item_begin[nsys] = static_cast<int>(out.items.size());
    if (!plain && nsys > 1) {
        std::stable_sort(out.items.begin(), out.items.end(), [](const WorkItem& a, const WorkItem& b) {
            const int64_t ca = static_cast<int64_t>(a.pad0) * (a.j_end - a.j_begin);
            const int64_t cb = static_cast<int64_t>(b.pad0) * (b.j_end - b.j_begin);
            return ca > cb;
        });
    }
}

PairBlocks pair_blocks_fixed(const std::vector<int64_t>& poff) {
    PairBlocks out(poff.size() - 1);
    for (size_t k = 0; k + 1 < poff.size(); ++k) {
        for (int64_t b = poff[k]; b < poff[k + 1]; b += kPairBlock) out[k].push_back(b);
        out[k].push_back(poff[k + 1]);
    }
    return out;
}

PairBlocks pair_blocks_by_mass(const std::vector<int64_t>& poff, const std::vector<float>& tile_mass) {
    PairBlocks out(poff.size() - 1);
    for (size_t k = 0; k + 1 < poff.size(); ++k) {
        int64_t start = poff[k];
        out[k].push_back(start);
        for (int64_t t = poff[k] + kPad; t < poff[k + 1]; t += kPad)
            if (t - start == kPairBlock || tile_mass[t / kPad] != tile_mass[start / kPad]) {
                start = t;
                out[k].push_back(start);
            }
        out[k].push_back(poff[k + 1]);
    }
    return out;
}

// Block row b of a system with nb blocks holds the block pairs (b, J), J >= b,
// cut into chunks of C blocks.  A body of block b receives the reactions of
// blocks 0..b-1 and its own row's chunk sums, all added into its fixed-point
// accumulators.  C is the largest chunk (up to 32 blocks) that still gives
// the persistent grid about 16 items per CTA; items run costliest first.
void plan_pair_items(const PairBlocks& blocks, const std::vector<int64_t>& cnt, int ctas, int chunk,
                     ForcePlan& out) {
    out.pair_items.clear();
    const size_t nsys = cnt.size();
    double block_pairs = 0.0;
    for (const auto& bb : blocks) {
        const double nb = static_cast<double>(bb.size() - 1);
        block_pairs += nb * (nb + 1.0) / 2.0;
    }
    int C = chunk;
    if (C <= 0) C = static_cast<int>(std::clamp(block_pairs / (16.0 * std::max(ctas, 1)), 1.0, 32.0));
    out.nslots = 1;
    for (size_t k = 0; k < nsys; ++k) {
        const std::vector<int64_t>& bb = blocks[k];
        const int64_t nb = static_cast<int64_t>(bb.size()) - 1, real_end = bb[0] + cnt[k];
        for (int64_t b = 0; b < nb; ++b) {
            const int64_t ib = bb[b], ie = bb[b + 1];
            const int64_t nch = (nb - b + C - 1) / C;
            for (int64_t u = 0; u < nch; ++u) {
                const int64_t Jb = b + u * C, Je = std::min(Jb + C, nb);
                PairItem it{};
                it.i_begin = static_cast<int>(ib);
                it.i_end = static_cast<int>(ie);
                it.j_begin = static_cast<int>(bb[Jb]);
                it.j_end = static_cast<int>(bb[Je]);
                it.diag_end = u == 0 ? it.i_end : it.j_begin;
                it.real_end = static_cast<int>(real_end);
                it.cost = static_cast<int>((ie - ib) * (it.j_end - it.j_begin) / kPairBlock);
                out.pair_items.push_back(it);
            }
        }
    }
    std::stable_sort(out.pair_items.begin(), out.pair_items.end(),
                     [](const PairItem& a, const PairItem& b) { return a.cost > b.cost; });
}

}  // namespace khrr

khrr_status khrr_ctx::ensure_plan(int mode) {
    ForcePlan& p = plan_for(mode);
    const bool plain = mode == kModePlain;
    khrr_status st;
    if (mode == kModeF64) {
        // The symmetric FP64 kernel on the pair plan over 1024-body blocks
        // (one partial slot per body, FP64 atomics), or with
        // KHRR_FP64_ONESIDED=1 the one-sided kernel's queue: 512-body i
        // tiles, 128-body j tiles, the j split that fills the last wave of
        // its resident CTAs.
        const char* e = std::getenv("KHRR_FP64_ONESIDED");
        const bool sym = !(e && std::atoi(e) == 1);
        const int ctas = sym ? fp64_pair_ctas(sm_count) : fp64_force_ctas(sm_count);
        if (p.valid && p.ctas == ctas && p.f64_pair == sym) return KHRR_OK;
        if (sym) {
            plan_pair_items(pair_blocks_fixed(poff), cnt, ctas, 0, p);
            p.nslots = 1;
            p.sys_split.assign(cnt.size(), 1);
            if ((st = cuda(p.d_pair_items.ensure(p.pair_items.size()), "alloc items")) != KHRR_OK) return st;
            if ((st = cuda(cudaMemcpyAsync(p.d_pair_items.p, p.pair_items.data(),
                                           p.pair_items.size() * sizeof(PairItem), cudaMemcpyHostToDevice, stream),
                           "upload items")) != KHRR_OK)
                return st;
        } else {
            plan_force_items(poff, cnt, kF64ITile, kPad, ctas, 0, false, p);
            if ((st = cuda(p.d_items.ensure(p.items.size()), "alloc items")) != KHRR_OK) return st;
            if ((st = cuda(cudaMemcpyAsync(p.d_items.p, p.items.data(), p.items.size() * sizeof(WorkItem),
                                           cudaMemcpyHostToDevice, stream),
                           "upload items")) != KHRR_OK)
                return st;
        }
        p.pair = false;
        p.f64_pair = sym;
        p.threads = sym ? kPairBlock / 4 : 128;
        p.ipt = sym ? 4 : kF64ITile / 128;
        p.jt = kPad;
        p.split_req = 0;
        p.ctas = ctas;
        std::vector<unsigned char> ns(static_cast<size_t>(npad), 0);
        for (size_t k = 0; k < cnt.size(); ++k)
            std::fill(ns.begin() + poff[k], ns.begin() + poff[k] + cnt[k], static_cast<unsigned char>(p.sys_split[k]));
        if ((st = cuda(p.d_nsplit.ensure(ns.size()), "alloc nsplit")) != KHRR_OK) return st;
        if ((st = cuda(cudaMemcpyAsync(p.d_nsplit.p, ns.data(), ns.size(), cudaMemcpyHostToDevice, stream),
                       "upload nsplit")) != KHRR_OK)
            return st;
        if ((st = cuda(part.ensure(static_cast<size_t>(p.nslots) * npad), "alloc partials")) != KHRR_OK) return st;
        if ((st = cuda(cudaStreamSynchronize(stream), "plan sync")) != KHRR_OK) return st;
        p.valid = true;
        drop_graphs();  // captured graphs may hold the old queue or partial buffer
        return KHRR_OK;
    }
    // The plan depends on the kernel shape only; acceleration and potential
    // passes of that shape share it (the grid follows each kernel's occupancy).
    const ForceVariant* v = variant(uniform, true, false);
    if (!v) return fail(KHRR_ERR_INVALID_ARG, "no force kernel for the current tuning");
    const int ctas = resident_ctas(v);
    if (!plain && v->pair) {
        if (p.valid && p.pair && p.split_req == tuning.j_split && p.ctas == ctas) return KHRR_OK;
        plan_pair_items(pair_blocks, cnt, ctas, tuning.j_split, p);
        p.pair = true;
        p.threads = v->threads;
        p.ipt = v->i_per_thread;
        p.jt = v->j_tile;
        p.split_req = tuning.j_split;
        p.ctas = ctas;
        if ((st = cuda(p.d_pair_items.ensure(p.pair_items.size()), "alloc items")) != KHRR_OK) return st;
        if ((st = cuda(cudaMemcpyAsync(p.d_pair_items.p, p.pair_items.data(), p.pair_items.size() * sizeof(PairItem),
                                       cudaMemcpyHostToDevice, stream),
                       "upload items")) != KHRR_OK)
            return st;
        if ((st = cuda(fx.ensure(static_cast<size_t>(kFxComps) * npad), "alloc fixed-point sums")) != KHRR_OK)
            return st;
        if ((st = cuda(cudaStreamSynchronize(stream), "plan sync")) != KHRR_OK) return st;
        p.valid = true;
        drop_graphs();
        return KHRR_OK;
    }
    if (p.valid && !p.pair && p.threads == v->threads && p.ipt == v->i_per_thread && p.jt == v->j_tile &&
        p.split_req == tuning.j_split && p.ctas == ctas)
        return KHRR_OK;
    plan_force_items(poff, cnt, v->threads * v->i_per_thread, v->j_tile, ctas, tuning.j_split, plain, p);
    p.pair = false;
    p.threads = v->threads;
    p.ipt = v->i_per_thread;
    p.jt = v->j_tile;
    p.split_req = tuning.j_split;
    p.ctas = ctas;
    if ((st = cuda(p.d_items.ensure(p.items.size()), "alloc items")) != KHRR_OK) return st;
    if ((st = cuda(cudaMemcpyAsync(p.d_items.p, p.items.data(), p.items.size() * sizeof(WorkItem),
                                   cudaMemcpyHostToDevice, stream),
                   "upload items")) != KHRR_OK)
        return st;
    // Partial slots per body: the system's split for real bodies, 0 for ghosts.
    std::vector<unsigned char> ns(static_cast<size_t>(npad), 0);
    for (size_t k = 0; k < cnt.size(); ++k)
        std::fill(ns.begin() + poff[k], ns.begin() + poff[k] + cnt[k],
                  static_cast<unsigned char>(p.sys_split[k]));
    if ((st = cuda(p.d_nsplit.ensure(ns.size()), "alloc nsplit")) != KHRR_OK) return st;
    if ((st = cuda(cudaMemcpyAsync(p.d_nsplit.p, ns.data(), ns.size(), cudaMemcpyHostToDevice, stream),
                   "upload nsplit")) != KHRR_OK)
        return st;
    if ((st = cuda(part.ensure(static_cast<size_t>(p.nslots) * npad), "alloc partials")) != KHRR_OK)
        return st;
    if ((st = cuda(cudaStreamSynchronize(stream), "plan sync")) != KHRR_OK) return st;
    p.valid = true;
    drop_graphs();
    return KHRR_OK;
}

void khrr_ctx::drop_graphs() {
    for (auto& kv : graphs) {
        if (kv.second.exec) cudaGraphExecDestroy(kv.second.exec);
        if (kv.second.graph) cudaGraphDestroy(kv.second.graph);
    }
    graphs.clear();
    for (auto& kv : wave_graphs) {
        if (kv.second.exec) cudaGraphExecDestroy(kv.second.exec);
        if (kv.second.graph) cudaGraphDestroy(kv.second.graph);
    }
    wave_graphs.clear();
    msolver.drop_graphs();
}

// ---------------------------------------------------------------------------
// force pass + step enqueue
// ---------------------------------------------------------------------------
ForceArgs khrr_ctx::force_args(const ForcePlan& p, int item_begin, int item_end) {
    ForceArgs a{};
    a.j = shadow();
    a.i = a.j;
    a.items = p.d_items.p + item_begin;
    a.n_items = item_end - item_begin;
    a.queue = queue.p;
    a.part = part.p;
    a.npad = npad;
    a.h_uniform = h_uniform;
    a.tile_mass = tile_mass.p;
    a.err = errflag.p;
    return a;
}

khrr_status khrr_ctx::enqueue_force(int mode, bool acc, bool phi, bool events, const double* x) {
    const bool plain = mode == kModePlain;
    const ForceVariant* v = variant(uniform, acc, phi);
    if (!v) return fail(KHRR_ERR_INVALID_ARG, "no force kernel for the current tuning");
    khrr_status st = ensure_plan(mode);
    if (st != KHRR_OK) return st;
    ForcePlan& p = plan_for(mode);
    const int ctas = mode == kModeF64 ? p.ctas : resident_ctas(v);
    // External records become event-record nodes when captured into a graph;
    // khrr_step points them at fresh timing events before each replay.
    if (events && (st = cuda(cudaEventRecordWithFlags(ph0, stream, cudaEventRecordExternal), "event")) != KHRR_OK)
        return st;
    if (mode == kModeF64 && p.f64_pair) {
        if ((st = cuda(cudaMemsetAsync(queue.p, 0, sizeof(unsigned), stream), "queue reset")) != KHRR_OK) return st;
        if ((st = cuda(cudaMemsetAsync(part.p, 0, sizeof(double4) * npad, stream), "sums reset")) != KHRR_OK)
            return st;
        F64PairArgs a{};
        a.pos = x;
        a.mass = mass.p;
        a.eps2 = eps2.p;
        a.items = p.d_pair_items.p;
        a.n_items = static_cast<int>(p.pair_items.size());
        a.queue = queue.p;
        a.sums = part.p;
        if ((st = cuda(launch_fp64_pair(a, acc, phi, std::min(a.n_items, ctas), stream), "FP64 pair kernel")) !=
            KHRR_OK)
            return st;
    } else if (mode == kModeF64) {
        if ((st = cuda(cudaMemsetAsync(queue.p, 0, sizeof(unsigned), stream), "queue reset")) != KHRR_OK) return st;
        F64Args a{};
        a.pos = x;
        a.mass = mass.p;
        a.eps2 = eps2.p;
        a.items = p.d_items.p;
        a.n_items = static_cast<int>(p.items.size());
        a.queue = queue.p;
        a.part = part.p;
        a.npad = npad;
        if ((st = cuda(launch_fp64_force(a, acc, phi, std::min(a.n_items, ctas), stream), "FP64 force kernel")) !=
            KHRR_OK)
            return st;
    } else if (plain) {
        // The conventional baseline: one launch per system, one i body per thread.
        for (size_t k = 0; k < cnt.size(); ++k) {
            Shadow sh = shadow();
            const int64_t o = poff[k];
            sh.x += o;
            sh.y += o;
            sh.z += o;
            sh.m += o;
            sh.h += o;
            if ((st = cuda(launch_plain_force(sh, static_cast<int>(cnt[k]), static_cast<int>(poff[k + 1] - o),
                                              part.p + o, acc, phi, stream),
                           "plain force kernel")) != KHRR_OK)
                return st;
        }
    } else if (p.pair) {
        if (!v->pair) return fail(KHRR_ERR_INVALID_ARG, "no pair kernel for this output set");
        if ((st = cuda(cudaMemsetAsync(queue.p, 0, sizeof(unsigned), stream), "queue reset")) != KHRR_OK) return st;
        if ((st = cuda(cudaMemsetAsync(fx.p, 0, sizeof(unsigned long long) * kFxComps * npad, stream),
                       "sums reset")) != KHRR_OK)
            return st;
        PairArgs a{};
        a.sh = shadow();
        a.items = p.d_pair_items.p;
        a.n_items = static_cast<int>(p.pair_items.size());
        a.queue = queue.p;
        a.fx = fx.p;
        a.npad = npad;
        a.scale = fx_scale.p;
        a.h_uniform = h_uniform;
        a.tile_mass = tile_mass.p;
        a.err = errflag.p;
        if ((st = cuda(launch_pair(v, a, std::min(a.n_items, ctas), stream), "pair force kernel")) != KHRR_OK)
            return st;
    } else {
        if ((st = cuda(cudaMemsetAsync(queue.p, 0, sizeof(unsigned), stream), "queue reset")) != KHRR_OK) return st;
        const int e = static_cast<int>(p.items.size());
        if ((st = cuda(launch_force(v, force_args(p, 0, e), std::min(e, ctas), stream), "force kernel")) != KHRR_OK)
            return st;
    }
    if (events && (st = cuda(cudaEventRecordWithFlags(ph1, stream, cudaEventRecordExternal), "event")) != KHRR_OK)
        return st;
    return KHRR_OK;
}

StepArgs khrr_ctx::step_args(const ForcePlan& p, double dt) {
    StepArgs a{};
    a.pos = pos.p;
    a.vel = vel.p;
    a.acc = acc.p;
    a.post = post.p;
    a.velt = velt.p;
    a.acct = acct.p;
    a.mass = mass.p;
    a.phi = phi.p;
    a.shadow = shadow();
    a.part = part.p;
    a.npad = npad;
    a.nsplit = p.d_nsplit.p;
    a.fx = p.pair ? fx.p : nullptr;
    a.fx_scale = fx_scale.p;
    a.n = npad;
    a.dt = dt;
    a.field = field;
    return a;
}

khrr_status khrr_ctx::enqueue_step(double dt, int mode, bool phi_now, bool compat) {
    const bool plain = mode == kModePlain;
    khrr_status st = enqueue_force(mode, true, phi_now, true, post.p);
    if (st != KHRR_OK) return st;
    ForcePlan& p = plan_for(mode);
    StepArgs sa = step_args(p, dt);
    sa.compat_accumulate = compat ? 1 : 0;
    sa.want_phi = phi_now ? 1 : 0;
    sa.predict_next = 1;
    if (!plain) return cuda(launch_corrector(sa, stream), "corrector");
    // Baseline path: one launch per system for the integrator as well.
    for (size_t k = 0; k < cnt.size(); ++k) {
        StepArgs s = sa;
        const int64_t o = poff[k];
        s.pos += 3 * o;
        s.vel += 3 * o;
        s.acc += 3 * o;
        s.post += 3 * o;
        s.velt += 3 * o;
        s.acct += 3 * o;
        s.mass += o;
        s.phi += o;
        s.shadow = shadow_at(shadow_buf.p, npad);
        s.shadow.x += o;
        s.shadow.y += o;
        s.shadow.z += o;
        s.shadow.m += o;
        s.shadow.h += o;
        s.part += o;
        s.nsplit += o;
        s.n = round_up(cnt[k], kPad);
        if ((st = cuda(launch_corrector(s, stream), "corrector")) != KHRR_OK) return st;
    }
    return KHRR_OK;
}

khrr_status khrr_ctx::get_step_graph(double dt, int mode, bool phi_now, bool compat, StepGraph** out) {
    // Plans first: their uploads must not happen inside a capture.
    khrr_status st = ensure_plan(mode);
    if (st != KHRR_OK) return st;
    uint64_t dt_bits;
    std::memcpy(&dt_bits, &dt, sizeof dt_bits);
    const auto key = std::make_tuple(dt_bits, mode, phi_now, compat);
    auto it = graphs.find(key);
    if (it != graphs.end()) {
        *out = &it->second;
        return KHRR_OK;
    }
    StepGraph g{};
    if ((st = cuda(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal), "begin capture")) != KHRR_OK)
        return st;
    khrr_status est = enqueue_step(dt, mode, phi_now, compat);
    cudaGraph_t graph = nullptr;
    cudaError_t ce = cudaStreamEndCapture(stream, &graph);
    if (est != KHRR_OK) {
        if (graph) cudaGraphDestroy(graph);
        return est;
    }
    if ((st = cuda(ce, "end capture")) != KHRR_OK) return st;
    g.graph = graph;
    size_t nn = 0;
    cudaGraphGetNodes(graph, nullptr, &nn);
    std::vector<cudaGraphNode_t> nodes(nn);
    cudaGraphGetNodes(graph, nodes.data(), &nn);
    for (cudaGraphNode_t node : nodes) {
        cudaGraphNodeType t;
        cudaGraphNodeGetType(node, &t);
        if (t != cudaGraphNodeTypeEventRecord) continue;
        cudaEvent_t e = nullptr;
        cudaGraphEventRecordNodeGetEvent(node, &e);
        if (e == ph0) g.ev0 = node;
        if (e == ph1) g.ev1 = node;
    }
    if ((st = cuda(cudaGraphInstantiate(&g.exec, graph, 0), "graph instantiate")) != KHRR_OK) {
        cudaGraphDestroy(graph);
        return st;
    }
    auto ins = graphs.emplace(key, g);
    *out = &ins.first->second;
    return KHRR_OK;
}

khrr_status khrr_ctx::timing_pair(cudaEvent_t* e0, cudaEvent_t* e1) {
    if (ev_used == ev_pool.size()) {
        cudaEvent_t a, b;
        khrr_status st;
        if ((st = cuda(cudaEventCreate(&a), "event create")) != KHRR_OK) return st;
        if ((st = cuda(cudaEventCreate(&b), "event create")) != KHRR_OK) return st;
        ev_pool.emplace_back(a, b);
    }
    *e0 = ev_pool[ev_used].first;
    *e1 = ev_pool[ev_used].second;
    ++ev_used;
    return KHRR_OK;
}

khrr_status khrr_ctx::call_start() {
    call_timed = false;
    if (!timing) return KHRR_OK;
    khrr_status st;
    if (!call0 && (st = cuda(cudaEventCreate(&call0), "event create")) != KHRR_OK) return st;
    if (!call1 && (st = cuda(cudaEventCreate(&call1), "event create")) != KHRR_OK) return st;
    return cuda(cudaEventRecord(call0, stream), "event");
}

khrr_status khrr_ctx::call_stop() {
    if (!timing || !call0 || !call1) return KHRR_OK;
    khrr_status st = cuda(cudaEventRecord(call1, stream), "event");
    if (st == KHRR_OK) call_timed = true;
    return st;
}

khrr_status khrr_ctx::force_mode(int flags, int* mode) {
    const bool plain = (flags & KHRR_PLAIN) != 0, f64 = (flags & KHRR_FP64) != 0;
    if (plain && f64) return fail(KHRR_ERR_INVALID_ARG, "KHRR_PLAIN and KHRR_FP64 exclude each other");
    *mode = plain ? kModePlain : (f64 ? kModeF64 : kModeBatched);
    return KHRR_OK;
}

double khrr_ctx::pairs_per_pass() const {
    double s = 0.0;
    for (int64_t c : cnt) s += static_cast<double>(c) * static_cast<double>(c);
    return s;
}

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
extern "C" {

int khrr_abi_version(void) { return KHRR_ABI_VERSION; }

const char* khrr_status_name(khrr_status s) {
    switch (s) {
        case KHRR_OK: return "KHRR_OK";
        case KHRR_ERR_INVALID_ARG: return "KHRR_ERR_INVALID_ARG";
        case KHRR_ERR_NOT_MULTIPLE: return "KHRR_ERR_NOT_MULTIPLE";
        case KHRR_ERR_CUDA: return "KHRR_ERR_CUDA";
        case KHRR_ERR_IO: return "KHRR_ERR_IO";
        case KHRR_ERR_TIMEOUT: return "KHRR_ERR_TIMEOUT";
        case KHRR_ERR_STATE: return "KHRR_ERR_STATE";
        case KHRR_ERR_OOM: return "KHRR_ERR_OOM";
        case KHRR_ERR_UNSUPPORTED: return "KHRR_ERR_UNSUPPORTED";
        case KHRR_ERR_TOO_LARGE: return "KHRR_ERR_TOO_LARGE";
    }
    return "KHRR_ERR_UNKNOWN";
}

khrr_status khrr_create(int device, khrr_ctx** out) {
    if (!out) return KHRR_ERR_INVALID_ARG;
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return KHRR_ERR_UNSUPPORTED;
    if (device < 0 || device >= ndev) return KHRR_ERR_INVALID_ARG;
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) return KHRR_ERR_CUDA;
    if (prop.major != 10) return KHRR_ERR_UNSUPPORTED;  // built for sm_100a only
    if (cudaSetDevice(device) != cudaSuccess) return KHRR_ERR_CUDA;
    khrr_ctx* c = new khrr_ctx();
    c->device = device;
    c->sm_count = prop.multiProcessorCount;
    if (cudaStreamCreateWithFlags(&c->own, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreate(&c->ph0) != cudaSuccess || cudaEventCreate(&c->ph1) != cudaSuccess ||
        c->queue.ensure(1) != cudaSuccess || c->errflag.ensure(1) != cudaSuccess ||
        c->scratch.ensure(64) != cudaSuccess) {
        khrr_destroy(c);
        return KHRR_ERR_CUDA;
    }
    c->stream = c->own;
    cudaMemset(c->queue.p, 0, sizeof(unsigned));
    cudaMemset(c->errflag.p, 0, sizeof(unsigned));
    for (int i = 0; i < force_variant_count() + pair_variant_count(); ++i) {
        const ForceVariant* v = i < force_variant_count() ? force_variant(i) : pair_variant(i - force_variant_count());
        if (cudaFuncSetAttribute(v->fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 static_cast<int>(v->smem)) != cudaSuccess) {
            khrr_destroy(c);
            return KHRR_ERR_CUDA;
        }
        c->resident_ctas(v);  // caches the occupancy (no queries during captures)
    }
    if (cudaDeviceSynchronize() != cudaSuccess) {
        khrr_destroy(c);
        return KHRR_ERR_CUDA;
    }
    *out = c;
    return KHRR_OK;
}

void khrr_destroy(khrr_ctx* c) {
    if (!c) return;
    cudaSetDevice(c->device);
    if (c->own) cudaStreamSynchronize(c->own);
    c->drop_graphs();
    for (auto& e : c->ev_pool) {
        cudaEventDestroy(e.first);
        cudaEventDestroy(e.second);
    }
    if (c->call0) cudaEventDestroy(c->call0);
    if (c->call1) cudaEventDestroy(c->call1);
    if (c->ph0) cudaEventDestroy(c->ph0);
    if (c->ph1) cudaEventDestroy(c->ph1);
    if (c->own) cudaStreamDestroy(c->own);
    delete c;  // device buffers free themselves
}

const char* khrr_last_error(const khrr_ctx* c) { return c ? c->err.c_str() : "null context"; }

void* khrr_get_stream(khrr_ctx* c) { return c ? static_cast<void*>(c->stream) : nullptr; }

khrr_status khrr_set_stream(khrr_ctx* c, void* stream) {
    if (!c) return KHRR_ERR_INVALID_ARG;
    cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : c->own;
    if (s != c->stream) {
        cudaStreamSynchronize(c->stream);
        c->stream = s;
        c->drop_graphs();
    }
    return KHRR_OK;
}

khrr_status khrr_synchronize(khrr_ctx* c) {
    if (!c) return KHRR_ERR_INVALID_ARG;
    khrr_status st = c->cuda(cudaStreamSynchronize(c->stream), "synchronize");
    if (st != KHRR_OK) return st;
    return c->check_device_flag();
}

khrr_status khrr_set_external_field(khrr_ctx* c, const khrr_field_params* p) {
    if (!c) return KHRR_ERR_INVALID_ARG;
    if (p) {
        if (!(p->a > 0.0) || !(p->b > 0.0) || !(p->Rh > 0.0) || !(p->Rb > 0.0))
            return c->fail(KHRR_ERR_INVALID_ARG, "field scale lengths a, b, Rh, Rb must be > 0");
        c->field = make_field(p->Mh, p->a, p->Rh, p->Mb, p->b, p->Rb);
    } else {
        c->field = FieldConsts{};
    }
    c->drop_graphs();
    c->predicted = false;
    return KHRR_OK;
}

khrr_status khrr_upload_state(khrr_ctx* c, int64_t n, const double* pos, const double* vel,
                              const double* mass, const double* eps2, int nsys,
                              const int64_t* sys_offsets) {
    khrr::NvtxRange nvtx_range("khrr_upload_state");
    if (!c) return KHRR_ERR_INVALID_ARG;
    if (n < 1 || !pos || !vel || !mass || !eps2) return c->fail(KHRR_ERR_INVALID_ARG, "bad state arrays");
    if (nsys < 1 || (nsys > 1 && !sys_offsets)) return c->fail(KHRR_ERR_INVALID_ARG, "bad system count");
    std::vector<int64_t> off(static_cast<size_t>(nsys) + 1);
    if (sys_offsets) {
        for (int k = 0; k <= nsys; ++k) off[k] = sys_offsets[k];
    } else {
        off[0] = 0;
        off[1] = n;
    }
    if (off[0] != 0 || off[nsys] != n) return c->fail(KHRR_ERR_INVALID_ARG, "system offsets must span [0, n]");
    for (int k = 0; k < nsys; ++k)
        if (off[k + 1] <= off[k]) return c->fail(KHRR_ERR_INVALID_ARG, "system %d is empty", k);
    std::vector<int64_t> cnt(static_cast<size_t>(nsys)), poff(static_cast<size_t>(nsys) + 1);
    int64_t p = 0;
    for (int k = 0; k < nsys; ++k) {
        cnt[k] = off[k + 1] - off[k];
        poff[k] = p;
        p += round_up(cnt[k], kPad);
    }
    poff[nsys] = p;
    if (p > (int64_t(1) << 30)) return c->fail(KHRR_ERR_INVALID_ARG, "too many bodies");
    cudaSetDevice(c->device);
    const bool same_offsets = c->has_state && c->off == off;
    // From here on the device arrays are rewritten: whatever the outcome, the
    // previous state is gone, and a failed upload leaves the context without
    // state.
    c->has_state = false;
    c->predicted = false;
    c->off = off;
    c->cnt = cnt;
    c->poff = poff;
    c->n = n;
    c->npad = p;
    const size_t np = static_cast<size_t>(p);
    khrr_status st;
    for (DevBuf<double>* b : {&c->pos, &c->vel, &c->acc, &c->post, &c->velt, &c->acct})
        if ((st = c->cuda(b->ensure(3 * np), "alloc state")) != KHRR_OK) return st;
    for (DevBuf<double>* b : {&c->mass, &c->eps2, &c->phi})
        if ((st = c->cuda(b->ensure(np), "alloc state")) != KHRR_OK) return st;
    if ((st = c->cuda(c->shadow_buf.ensure(5 * np), "alloc shadow")) != KHRR_OK) return st;
    if ((st = c->cuda(c->tile_mass.ensure(np / kPad), "alloc tile masses")) != KHRR_OK) return st;
    if ((st = c->cuda(c->fx_scale.ensure(np / kPad), "alloc tile scales")) != KHRR_OK) return st;
    cudaStream_t s = c->stream;
    for (DevBuf<double>* b : {&c->pos, &c->vel, &c->acc, &c->post, &c->velt, &c->acct})
        cudaMemsetAsync(b->p, 0, 3 * np * sizeof(double), s);
    for (DevBuf<double>* b : {&c->mass, &c->phi}) cudaMemsetAsync(b->p, 0, np * sizeof(double), s);
    // eps2 of ghosts = eps2 of their system's first body (positive); the real
    // bodies' values are copied straight from the caller's array below.
    std::vector<double> ghost_eps2(np - static_cast<size_t>(n));
    for (int k = 0, g = 0; k < nsys; ++k) {
        const int64_t pad = poff[k + 1] - poff[k] - cnt[k];
        std::fill(ghost_eps2.begin() + g, ghost_eps2.begin() + g + pad, eps2[off[k]]);
        g += static_cast<int>(pad);
    }
    // The copies first: the scan of the caller's masses and softenings below
    // runs on the host while they are in flight.
    st = KHRR_OK;
    for (int k = 0, g = 0; k < nsys && st == KHRR_OK; ++k) {
        const size_t o = static_cast<size_t>(off[k]), q = static_cast<size_t>(poff[k]);
        const size_t m = static_cast<size_t>(cnt[k]);
        const size_t pad = static_cast<size_t>(poff[k + 1]) - q - m;
        st = c->cuda(cudaMemcpyAsync(c->eps2.p + q, eps2 + o, m * sizeof(double), cudaMemcpyHostToDevice, s), "upload");
        if (st == KHRR_OK && pad)
            st = c->cuda(cudaMemcpyAsync(c->eps2.p + q + m, ghost_eps2.data() + g, pad * sizeof(double),
                                         cudaMemcpyHostToDevice, s),
                         "upload");
        g += static_cast<int>(pad);
        if (st != KHRR_OK) break;
        st = c->cuda(cudaMemcpyAsync(c->pos.p + 3 * q, pos + 3 * o, 3 * m * sizeof(double), cudaMemcpyHostToDevice, s), "upload");
        if (st == KHRR_OK)
            st = c->cuda(cudaMemcpyAsync(c->vel.p + 3 * q, vel + 3 * o, 3 * m * sizeof(double), cudaMemcpyHostToDevice, s), "upload");
        if (st == KHRR_OK)
            st = c->cuda(cudaMemcpyAsync(c->mass.p + q, mass + o, m * sizeof(double), cudaMemcpyHostToDevice, s), "upload");
    }
    if (st != KHRR_OK) {
        cudaStreamSynchronize(s);  // no copy may still read the caller's arrays
        return st;
    }
    const std::vector<TileScan> tiles = scan_state_tiles(mass, eps2, off);
    for (size_t t = 0; t < tiles.size(); ++t) {
        if (tiles[t].pos_eps) continue;
        cudaStreamSynchronize(s);
        for (int64_t i = tiles[t].begin; i < tiles[t].end; ++i)
            if (!(eps2[i] > 0.0)) return c->fail(KHRR_ERR_INVALID_ARG, "eps2[%lld] must be > 0", (long long)i);
    }
    // Per system its total |mass| (tile sums in tile order) and smallest
    // h = eps2 / 2; per padded 128-body tile the first mass; whether every
    // softening equals eps2[0] and whether every tile has one mass (and no
    // ghosts).
    bool uniform_new = true, tile_uniform = true;
    std::vector<double> sys_msum(static_cast<size_t>(nsys), 0.0), sys_hmin(static_cast<size_t>(nsys), 1e300);
    std::vector<float> tm(np / kPad, 0.0f);
    for (const TileScan& t : tiles) {
        uniform_new = uniform_new && t.same_eps;
        tile_uniform = tile_uniform && t.same_mass && t.end - t.begin == kPad;
        sys_msum[t.sys] += t.msum;
        sys_hmin[t.sys] = std::min(sys_hmin[t.sys], t.hmin);
        tm[(poff[t.sys] + t.begin - off[t.sys]) / kPad] = static_cast<float>(mass[t.begin]);
    }
    const bool same_layout = same_offsets && c->uniform == uniform_new &&
                             c->h_uniform == static_cast<float>(0.5 * eps2[0]);
    c->uniform = uniform_new;
    c->h_uniform = static_cast<float>(0.5 * eps2[0]);
    // One mass per 128-body tile (and no ghosts) lets the kernel factor the
    // mass out of each tile sum; the reference's layouts have it (component
    // counts are multiples of 1024).
    if (tile_uniform != c->tile_uniform_mass) c->drop_graphs();
    c->tile_uniform_mass = tile_uniform;
    // The pair kernel's blocks: with one mass per tile, runs of equal-mass
    // tiles cut at 1024 bodies (one mass per block: the block-mass form);
    // otherwise 1024-body blocks.
    PairBlocks blocks = tile_uniform ? pair_blocks_by_mass(poff, tm) : pair_blocks_fixed(poff);
    if (tile_uniform != c->block_uniform_mass || blocks != c->pair_blocks) {
        c->plan_batched.valid = false;
        c->drop_graphs();
    }
    c->block_uniform_mass = tile_uniform;
    c->pair_blocks = std::move(blocks);
    // Scales of the pair kernel's fixed-point sums per 128-body tile, from the
    // tile's smallest h = eps2 / 2, its system's smallest h and total |mass|
    // (real bodies; ghosts carry the system's first softening and no sums).
    c->fx_scales.assign(tm.size(), FxScale{1.0, 1.0, 1.0, 1.0});
    for (const TileScan& t : tiles)
        c->fx_scales[(poff[t.sys] + t.begin - off[t.sys]) / kPad] =
            fx_scale(t.hmin, sys_hmin[t.sys], sys_msum[t.sys]);
    st = c->cuda(cudaMemcpyAsync(c->fx_scale.p, c->fx_scales.data(), tm.size() * sizeof(FxScale),
                                 cudaMemcpyHostToDevice, s),
                 "upload");
    if (st == KHRR_OK)
        st = c->cuda(cudaMemcpyAsync(c->tile_mass.p, tm.data(), tm.size() * sizeof(float), cudaMemcpyHostToDevice, s),
                     "upload");
    if (st == KHRR_OK)
        st = c->cuda(launch_pack(c->pos.p, c->mass.p, c->eps2.p, c->npad, c->npad, c->shadow(), s), "pack");
    // The host vectors above are sources of the copies: wait for them either way.
    const khrr_status sync = c->cuda(cudaStreamSynchronize(s), "upload sync");
    if (st != KHRR_OK) return st;
    if (sync != KHRR_OK) return sync;
    if (!same_layout) {
        c->plan_batched.valid = false;
        c->plan_plain.valid = false;
        c->plan_fp64.valid = false;
        c->drop_graphs();
    }
    c->has_state = true;
    return KHRR_OK;
}

khrr_status khrr_set_accelerations(khrr_ctx* c, const double* acc) {
    if (!c) return KHRR_ERR_INVALID_ARG;
    if (!c->has_state) return c->fail(KHRR_ERR_STATE, "no state uploaded");
    if (!acc) return c->fail(KHRR_ERR_INVALID_ARG, "null acc");
    khrr_status st = KHRR_OK;
    for (size_t k = 0; k < c->cnt.size() && st == KHRR_OK; ++k) {
        const size_t o = static_cast<size_t>(c->off[k]), q = static_cast<size_t>(c->poff[k]);
        st = c->cuda(cudaMemcpyAsync(c->acc.p + 3 * q, acc + 3 * o, 3 * static_cast<size_t>(c->cnt[k]) * sizeof(double),
                                     cudaMemcpyHostToDevice, c->stream),
                     "upload acc");
    }
    c->predicted = false;
    return st;
}

khrr_status khrr_accel_fp64_sample(khrr_ctx* c, const int64_t* targets, int64_t nt, double* acc, double* phi) {
    if (!c) return KHRR_ERR_INVALID_ARG;
    if (!c->has_state) return c->fail(KHRR_ERR_STATE, "no state uploaded");
    if (nt < 1 || !targets) return c->fail(KHRR_ERR_INVALID_ARG, "no targets");
    std::vector<int64_t> h(3 * static_cast<size_t>(nt));
    for (int64_t k = 0; k < nt; ++k) {
        const int64_t t = targets[k];
        if (t < 0 || t >= c->n) return c->fail(KHRR_ERR_INVALID_ARG, "target %lld out of range", (long long)t);
        const size_t sys = static_cast<size_t>(std::upper_bound(c->off.begin(), c->off.end(), t) - c->off.begin()) - 1;
        h[k] = c->poff[sys] + (t - c->off[sys]);
        h[nt + k] = c->poff[sys];
        h[2 * nt + k] = c->poff[sys] + c->cnt[sys];
    }
    DevBuf<int64_t> d;
    DevBuf<double> out;
    khrr_status st;
    if ((st = c->cuda(d.ensure(h.size()), "alloc")) != KHRR_OK) return st;
    if ((st = c->cuda(out.ensure(4 * static_cast<size_t>(nt)), "alloc")) != KHRR_OK) return st;
    if ((st = c->cuda(cudaMemcpyAsync(d.p, h.data(), h.size() * sizeof(int64_t), cudaMemcpyHostToDevice, c->stream),
                      "upload targets")) != KHRR_OK)
        return st;
    if ((st = c->cuda(launch_fp64_sample(c->pos.p, c->mass.p, c->eps2.p, d.p, d.p + nt, d.p + 2 * nt, nt, out.p,
                                         c->stream),
                      "fp64 sample")) != KHRR_OK)
        return st;
    std::vector<double> o(4 * static_cast<size_t>(nt));
    if ((st = c->cuda(cudaMemcpyAsync(o.data(), out.p, o.size() * sizeof(double), cudaMemcpyDeviceToHost, c->stream),
                      "download")) != KHRR_OK)
        return st;
    if ((st = khrr_synchronize(c)) != KHRR_OK) return st;
    for (int64_t k = 0; k < nt; ++k) {
        if (acc)
            for (int q = 0; q < 3; ++q) acc[3 * k + q] = o[4 * k + q];
        if (phi) phi[k] = o[4 * k + 3];
    }
    return KHRR_OK;
}

khrr_status khrr_download_state(khrr_ctx* c, double* pos, double* vel, double* acc, double* phi) {
    khrr::NvtxRange nvtx_range("khrr_download_state");
    if (!c) return KHRR_ERR_INVALID_ARG;
    if (!c->has_state) return c->fail(KHRR_ERR_STATE, "no state uploaded");
    cudaStream_t s = c->stream;
    khrr_status st = KHRR_OK;
    for (size_t k = 0; k < c->cnt.size() && st == KHRR_OK; ++k) {
        const size_t o = static_cast<size_t>(c->off[k]), q = static_cast<size_t>(c->poff[k]);
        const size_t m = static_cast<size_t>(c->cnt[k]);
        if (pos) st = c->cuda(cudaMemcpyAsync(pos + 3 * o, c->pos.p + 3 * q, 3 * m * sizeof(double), cudaMemcpyDeviceToHost, s), "download");
        if (vel && st == KHRR_OK) st = c->cuda(cudaMemcpyAsync(vel + 3 * o, c->vel.p + 3 * q, 3 * m * sizeof(double), cudaMemcpyDeviceToHost, s), "download");
        if (acc && st == KHRR_OK) st = c->cuda(cudaMemcpyAsync(acc + 3 * o, c->acc.p + 3 * q, 3 * m * sizeof(double), cudaMemcpyDeviceToHost, s), "download");
        if (phi && st == KHRR_OK) st = c->cuda(cudaMemcpyAsync(phi + o, c->phi.p + q, m * sizeof(double), cudaMemcpyDeviceToHost, s), "download");
    }
    if (st != KHRR_OK) return st;
    return khrr_synchronize(c);
}

khrr_status khrr_forces(khrr_ctx* c, int flags) {
    khrr::NvtxRange nvtx_range("khrr_forces");
    if (!c) return KHRR_ERR_INVALID_ARG;
    if (!c->has_state) return c->fail(KHRR_ERR_STATE, "no state uploaded");
    const bool want_acc = (flags & KHRR_ACC) != 0, want_phi = (flags & KHRR_PHI) != 0;
    if (!want_acc && !want_phi) return c->fail(KHRR_ERR_INVALID_ARG, "flags select nothing");
    if (flags & KHRR_MESH) return c->mesh_forces(flags);
    int mode;
    if (khrr_status st = c->force_mode(flags, &mode); st != KHRR_OK) return st;
    const bool plain = mode == kModePlain;
    cudaStream_t s = c->stream;
    khrr_status st;
    // Shadow of the current positions (a previous step leaves the predicted ones).
    if ((st = c->cuda(launch_pack(c->pos.p, c->mass.p, c->eps2.p, c->npad, c->npad, c->shadow(), s),
                      "pack")) != KHRR_OK)
        return st;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (c->timing && (st = c->timing_pair(&e0, &e1)) != KHRR_OK) return st;
    if (e0) cudaEventRecord(e0, s);
    if ((st = c->enqueue_force(mode, want_acc, want_phi, false, c->pos.p)) != KHRR_OK) return st;
    if (e1) cudaEventRecord(e1, s);
    if (c->timing) {
        c->timed_launches += plain ? static_cast<int64_t>(c->cnt.size()) : 1;
        c->timed_pairs += c->pairs_per_pass();
    }
    ForcePlan& p = c->plan_for(mode);
    StepArgs sa = c->step_args(p, 0.0);
    sa.want_phi = want_phi ? 1 : 0;
    if ((st = c->cuda(launch_collect(sa, want_acc, (flags & KHRR_COMPAT_ACCUMULATE) != 0, s), "collect")) != KHRR_OK)
        return st;
    c->predicted = false;
    return KHRR_OK;
}

khrr_status khrr_step(khrr_ctx* c, double dt, int nsteps, int flags) {
    khrr::NvtxRange nvtx_range("khrr_step");
    if (!c) return KHRR_ERR_INVALID_ARG;
    if (!c->has_state) return c->fail(KHRR_ERR_STATE, "no state uploaded");
    if (nsteps < 0 || !std::isfinite(dt)) return c->fail(KHRR_ERR_INVALID_ARG, "bad step arguments");
    if (nsteps == 0) return KHRR_OK;
    if (flags & KHRR_MESH) return c->mesh_step(dt, nsteps, flags);
    int mode;
    if (khrr_status st = c->force_mode(flags, &mode); st != KHRR_OK) return st;
    const bool plain = mode == kModePlain;
    const bool compat = (flags & KHRR_COMPAT_ACCUMULATE) != 0;
    const bool phi_last = (flags & KHRR_PHI) != 0;
    khrr_status st;
    cudaStream_t s = c->stream;
    if (!c->predicted || c->pred_dt != dt) {
        StepArgs sa = c->step_args(c->plan_for(mode), dt);
        if ((st = c->cuda(launch_predictor(sa, s), "predictor")) != KHRR_OK) return st;
    }
    for (int k = 0; k < nsteps; ++k) {
        const bool phi_now = phi_last && k == nsteps - 1;
        StepGraph* g = nullptr;
        if ((st = c->get_step_graph(dt, mode, phi_now, compat, &g)) != KHRR_OK) return st;
        if (!g->ev0 || !g->ev1) return c->fail(KHRR_ERR_CUDA, "step graph lacks its timing event nodes");
        cudaEvent_t e0 = c->ph0, e1 = c->ph1;
        if (c->timing && (st = c->timing_pair(&e0, &e1)) != KHRR_OK) return st;
        if ((st = c->cuda(cudaGraphExecEventRecordNodeSetEvent(g->exec, g->ev0, e0), "graph event")) != KHRR_OK ||
            (st = c->cuda(cudaGraphExecEventRecordNodeSetEvent(g->exec, g->ev1, e1), "graph event")) != KHRR_OK)
            return st;
        if ((st = c->cuda(cudaGraphLaunch(g->exec, s), "graph launch")) != KHRR_OK) return st;
        if (c->timing) {
            c->timed_launches += plain ? static_cast<int64_t>(c->cnt.size()) : 1;
            c->timed_pairs += c->pairs_per_pass();
        }
    }
    c->predicted = true;
    c->pred_dt = dt;
    return KHRR_OK;
}

khrr_status khrr_conservation(khrr_ctx* c, khrr_lie* out) {
    khrr::NvtxRange nvtx_range("khrr_conservation");
    if (!c || !out) return KHRR_ERR_INVALID_ARG;
    if (!c->has_state) return c->fail(KHRR_ERR_STATE, "no state uploaded");
    const int nb = conservation_blocks(c->npad);
    khrr_status st;
    if ((st = c->cuda(c->cons_blocks.ensure(static_cast<size_t>(nb) * 16), "alloc")) != KHRR_OK) return st;
    if ((st = c->cuda(launch_conservation(c->pos.p, c->vel.p, c->mass.p, c->phi.p, c->npad, c->cons_blocks.p,
                                          nb, c->scratch.p, c->stream),
                      "conservation")) != KHRR_OK)
        return st;
    double v[16];
    if ((st = c->cuda(cudaMemcpyAsync(v, c->scratch.p, sizeof v, cudaMemcpyDeviceToHost, c->stream), "download")) !=
        KHRR_OK)
        return st;
    if ((st = khrr_synchronize(c)) != KHRR_OK) return st;
    for (int k = 0; k < 3; ++k) {
        out->L[k] = v[k];
        out->Imp[k] = v[3 + k];
    }
    out->Ek = v[6];
    out->Ep = v[7];
    out->E = v[8];
    out->R_max = v[9];
    out->Z_max = v[10];
    out->Vr_max = v[11];
    out->Vfi_max = v[12];
    out->Vz_max = v[13];
    return KHRR_OK;
}

khrr_status khrr_set_tuning(khrr_ctx* c, const khrr_tuning* t) {
    if (!c || !t) return KHRR_ERR_INVALID_ARG;
    khrr_tuning n = *t;
    if (n.j_tile == 0) n.j_tile = 128;
    if (n.packed == 2) {
        if (n.threads != kPairThreads || n.i_per_thread != kPairBodies || n.j_tile != kPairTile)
            return c->fail(KHRR_ERR_INVALID_ARG, "the pair kernel (packed=2) has threads=%d i_per_thread=%d j_tile=%d",
                           kPairThreads, kPairBodies, kPairTile);
    } else if (n.packed != 0 && n.packed != 1) {
        return c->fail(KHRR_ERR_INVALID_ARG, "packed must be 0, 1 or 2");
    } else if (!find_force_variant(n.threads, n.i_per_thread, n.j_tile, n.packed != 0, false, true, false))
        return c->fail(KHRR_ERR_INVALID_ARG,
                       "no compiled force kernel with threads=%d i_per_thread=%d j_tile=%d packed=%d", n.threads,
                       n.i_per_thread, n.j_tile, n.packed);
    if (n.j_split < 0 || n.j_split > 255) return c->fail(KHRR_ERR_INVALID_ARG, "j_split must be in [0, 255]");
    c->tuning = n;
    c->plan_batched.valid = false;
    c->plan_plain.valid = false;
    c->drop_graphs();
    return KHRR_OK;
}

khrr_status khrr_get_tuning(khrr_ctx* c, khrr_tuning* t) {
    if (!c || !t) return KHRR_ERR_INVALID_ARG;
    *t = c->tuning;
    return KHRR_OK;
}

khrr_status khrr_enable_timing(khrr_ctx* c, int enable) {
    if (!c) return KHRR_ERR_INVALID_ARG;
    c->timing = enable != 0;
    c->ev_used = 0;
    c->timed_launches = 0;
    c->timed_pairs = 0.0;
    return KHRR_OK;
}

khrr_status khrr_call_timing(khrr_ctx* c, double* ms) {
    if (!c || !ms) return KHRR_ERR_INVALID_ARG;
    if (!c->call_timed)
        return c->fail(KHRR_ERR_STATE, "no timed call (enable timing, then khrr_bin, khrr_bin_cell_phi or khrr_sort_by_cell)");
    khrr_status st = c->cuda(cudaEventSynchronize(c->call1), "synchronize");
    if (st != KHRR_OK) return st;
    float t = 0.0f;
    if ((st = c->cuda(cudaEventElapsedTime(&t, c->call0, c->call1), "elapsed")) != KHRR_OK) return st;
    *ms = t;
    return KHRR_OK;
}

khrr_status khrr_force_timing(khrr_ctx* c, double* ms, int64_t* launches, double* interactions) {
    if (!c) return KHRR_ERR_INVALID_ARG;
    khrr_status st = c->cuda(cudaStreamSynchronize(c->stream), "synchronize");
    if (st != KHRR_OK) return st;
    double total = 0.0;
    for (size_t k = 0; k < c->ev_used; ++k) {
        float t = 0.0f;
        if ((st = c->cuda(cudaEventElapsedTime(&t, c->ev_pool[k].first, c->ev_pool[k].second), "elapsed")) != KHRR_OK)
            return st;
        total += t;
    }
    if (ms) *ms = total;
    if (launches) *launches = c->timed_launches;
    if (interactions) *interactions = c->timed_pairs;
    c->ev_used = 0;
    c->timed_launches = 0;
    c->timed_pairs = 0.0;
    return KHRR_OK;
}

khrr_status khrr_pair_count(khrr_ctx* c, double* pairs) {
    if (!c || !pairs) return KHRR_ERR_INVALID_ARG;
    if (!c->has_state) return c->fail(KHRR_ERR_STATE, "no state uploaded");
    *pairs = c->pairs_per_pass();
    return KHRR_OK;
}

khrr_status khrr_fp32_probe(khrr_ctx* c, double* tflops) {
    if (!c || !tflops) return KHRR_ERR_INVALID_ARG;
    const int block = 256, grid = c->sm_count * 8, iters = 4096;
    cudaEvent_t a, b;
    khrr_status st;
    if ((st = c->cuda(cudaEventCreate(&a), "event")) != KHRR_OK) return st;
    if ((st = c->cuda(cudaEventCreate(&b), "event")) != KHRR_OK) return st;
    float* out = reinterpret_cast<float*>(c->scratch.p);
    launch_fp32_probe(out, iters / 8, grid, block, c->stream);  // warm-up
    cudaEventRecord(a, c->stream);
    st = c->cuda(launch_fp32_probe(out, iters, grid, block, c->stream), "probe");
    cudaEventRecord(b, c->stream);
    float ms = 0.0f;
    if (st == KHRR_OK) st = c->cuda(cudaEventSynchronize(b), "probe sync");
    if (st == KHRR_OK) st = c->cuda(cudaEventElapsedTime(&ms, a, b), "probe time");
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    if (st != KHRR_OK) return st;
    const double fmas = static_cast<double>(grid) * block * iters * 16.0 * 8.0;
    *tflops = 2.0 * fmas / (ms * 1e-3) / 1e12;
    return KHRR_OK;
}

khrr_status khrr_probe_bounded_wait(khrr_ctx* c, double seconds) {
    if (!c) return KHRR_ERR_INVALID_ARG;
    if (!(seconds > 0.0) || seconds > 10.0) return c->fail(KHRR_ERR_INVALID_ARG, "seconds must be in (0, 10]");
    khrr_status st = c->check_device_flag();  // report (and clear) anything raised earlier first
    if (st != KHRR_OK) return st;
    if ((st = c->cuda(launch_wait_probe(c->errflag.p, static_cast<unsigned long long>(seconds * 1e9), c->stream),
                      "wait probe")) != KHRR_OK)
        return st;
    return c->check_device_flag();
}

}  // extern "C"
