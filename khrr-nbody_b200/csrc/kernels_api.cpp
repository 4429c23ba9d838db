// Kernel-level entry points of include/khrr.h (device pointers in the
// reference's layouts) and the force-kernel autotuner.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "khrr.h"
#include "khrr_internal.h"
#include "khrr_runtime.h"

using namespace khrr;

namespace {

int64_t round_up(int64_t v, int64_t m) { return (v + m - 1) / m * m; }

// The pair kernel's plan, tile scales and fixed-point sums for one system of
// n bodies (the same set as i and j).  The caller's masses and softenings are
// classified on the device first (one 4-byte read-back, which waits for the
// stream's earlier work): whole 1024 blocks of one mass select the
// block-mass form, equal softenings the uniform form; a softening <= 0 leaves
// the pass to the one-sided kernel (*vout = NULL), since the fixed-point
// bounds need positive softenings.
khrr_status prepare_pair_pass(khrr_ctx* c, const double* mass, const double* eps2, int64_t n, int64_t npad,
                              bool acc, bool phi, const ForceVariant** vout) {
    *vout = nullptr;
    khrr_status st;
    const size_t ntiles = static_cast<size_t>(npad / kPad);
    if ((st = c->cuda(c->ktile_mass.ensure(ntiles), "alloc")) != KHRR_OK ||
        (st = c->cuda(c->ktile_hmin.ensure(ntiles), "alloc")) != KHRR_OK ||
        (st = c->cuda(c->ktile_msum.ensure(ntiles), "alloc")) != KHRR_OK ||
        (st = c->cuda(c->kscale.ensure(ntiles), "alloc")) != KHRR_OK ||
        (st = c->cuda(c->kflags.ensure(1), "alloc")) != KHRR_OK)
        return st;
    cudaStream_t s = c->stream;
    unsigned flags = 0;
    double e0 = 0.0;
    if ((st = c->cuda(cudaMemsetAsync(c->kflags.p, 0xff, sizeof(unsigned), s), "flags")) != KHRR_OK ||
        (st = c->cuda(launch_classify(mass, eps2, n, c->ktile_mass.p, c->ktile_hmin.p, c->ktile_msum.p, c->kscale.p,
                                      c->kflags.p, s),
                      "classify")) != KHRR_OK ||
        (st = c->cuda(cudaMemcpyAsync(&flags, c->kflags.p, sizeof flags, cudaMemcpyDeviceToHost, s), "flags")) !=
            KHRR_OK ||
        (st = c->cuda(cudaMemcpyAsync(&e0, eps2, sizeof e0, cudaMemcpyDeviceToHost, s), "flags")) != KHRR_OK ||
        (st = c->cuda(cudaStreamSynchronize(s), "classify sync")) != KHRR_OK)
        return st;
    if (!(flags & 4u)) return KHRR_OK;  // a softening <= 0: one-sided kernel
    const bool unif = (flags & 2u) != 0, block_mass = (flags & 1u) != 0 && n % kPairBlock == 0;
    c->kh_uniform = static_cast<float>(0.5 * e0);
    const ForceVariant* v = find_pair_variant(unif, acc, phi, block_mass);
    const ForceVariant* vplan = find_pair_variant(false, true, false, false);
    if (!v || !vplan) return c->fail(KHRR_ERR_INVALID_ARG, "no pair kernel for this output set");
    ForcePlan& p = c->kplan;
    const int ctas = c->resident_ctas(vplan);
    if (!p.valid || !p.pair || c->kplan_n != n || p.split_req != c->tuning.j_split || p.ctas != ctas) {
        std::vector<int64_t> cnt{n};
        plan_pair_items(pair_blocks_fixed({0, npad}), cnt, ctas, c->tuning.j_split, p);
        p.pair = true;
        p.threads = v->threads;
        p.ipt = v->i_per_thread;
        p.jt = v->j_tile;
        p.split_req = c->tuning.j_split;
        p.ctas = ctas;
        if ((st = c->cuda(p.d_pair_items.ensure(p.pair_items.size()), "alloc")) != KHRR_OK) return st;
        if ((st = c->cuda(cudaMemcpy(p.d_pair_items.p, p.pair_items.data(), p.pair_items.size() * sizeof(PairItem),
                                     cudaMemcpyHostToDevice),
                          "upload items")) != KHRR_OK)
            return st;
        p.valid = true;
        c->kplan_n = n;
    }
    if ((st = c->cuda(c->kfx.ensure(static_cast<size_t>(kFxComps) * npad), "alloc fixed-point sums")) != KHRR_OK)
        return st;
    *vout = v;
    return KHRR_OK;
}

// Shadow + plan + partials for a one-system pass over n bodies given by
// device pointers; returns the variant to launch (the pair kernel when the
// tuning asks for it and i and j are the same set).
khrr_status prepare_kernel_pass(khrr_ctx* c, const double* pos_i, const double* pos_j,
                                const double* mass_j, const double* eps2_j, int64_t n, bool acc,
                                bool phi, const ForceVariant** vout) {
    if (n < 1 || n > (int64_t(1) << 30)) return c->fail(KHRR_ERR_INVALID_ARG, "n out of range");
    if (!pos_i || !pos_j || !mass_j || !eps2_j) return c->fail(KHRR_ERR_INVALID_ARG, "null device pointer");
    const int64_t npad = round_up(n, kPad);
    khrr_status st;
    if (c->tuning.packed == 2 && pos_i == pos_j) {
        if ((st = c->cuda(c->kshadow.ensure(5 * static_cast<size_t>(npad)), "alloc")) != KHRR_OK) return st;
        if ((st = prepare_pair_pass(c, mass_j, eps2_j, n, npad, acc, phi, vout)) != KHRR_OK) return st;
        if (*vout)
            return c->cuda(launch_pack(pos_j, mass_j, eps2_j, n, npad, shadow_at(c->kshadow.p, npad), c->stream),
                           "pack");
    }
    // The one-sided kernel (i and j may be different sets); the pair tuning
    // maps to its packed 128 x 4 shape.
    const bool pair_tuning = c->tuning.packed == 2;
    const int threads = pair_tuning ? 128 : c->tuning.threads;
    const int ipt = pair_tuning ? 4 : c->tuning.i_per_thread;
    const int jt = pair_tuning ? 128 : c->tuning.j_tile;
    const bool packed = c->tuning.packed != 0;
    const ForceVariant* v = find_force_variant(threads, ipt, jt, packed, false, acc, phi);
    const ForceVariant* vplan = find_force_variant(threads, ipt, jt, packed, false, true, false);
    if (!v || !vplan) return c->fail(KHRR_ERR_INVALID_ARG, "no force kernel for the current tuning");
    if ((st = c->cuda(c->kshadow.ensure(5 * static_cast<size_t>(npad)), "alloc")) != KHRR_OK) return st;
    ForcePlan& p = c->kplan;
    const int ctas = c->resident_ctas(vplan);
    if (!p.valid || p.pair || c->kplan_n != n || p.threads != v->threads || p.ipt != v->i_per_thread ||
        p.split_req != c->tuning.j_split || p.ctas != ctas) {
        std::vector<int64_t> poff{0, npad}, cnt{n};
        plan_force_items(poff, cnt, v->threads * v->i_per_thread, v->j_tile, ctas, c->tuning.j_split, false, p);
        p.pair = false;
        p.threads = v->threads;
        p.ipt = v->i_per_thread;
        p.jt = v->j_tile;
        p.split_req = c->tuning.j_split;
        p.ctas = ctas;
        if ((st = c->cuda(p.d_items.ensure(p.items.size()), "alloc")) != KHRR_OK) return st;
        if ((st = c->cuda(cudaMemcpy(p.d_items.p, p.items.data(), p.items.size() * sizeof(WorkItem),
                                     cudaMemcpyHostToDevice),
                          "upload items")) != KHRR_OK)
            return st;
        p.valid = true;
        c->kplan_n = n;
    }
    if ((st = c->cuda(c->kpart.ensure(static_cast<size_t>(p.nslots) * npad), "alloc partials")) != KHRR_OK)
        return st;
    cudaStream_t s = c->stream;
    if ((st = c->cuda(launch_pack(pos_j, mass_j, eps2_j, n, npad, shadow_at(c->kshadow.p, npad), s), "pack")) !=
        KHRR_OK)
        return st;
    if (pos_i != pos_j) {
        if ((st = c->cuda(c->kishadow.ensure(5 * static_cast<size_t>(npad)), "alloc")) != KHRR_OK) return st;
        if ((st = c->cuda(launch_pack(pos_i, mass_j, eps2_j, n, npad, shadow_at(c->kishadow.p, npad), s), "pack")) !=
            KHRR_OK)
            return st;
    }
    *vout = v;
    return KHRR_OK;
}

khrr_status run_kernel_pass(khrr_ctx* c, const ForceVariant* v, bool distinct_i) {
    ForcePlan& p = c->kplan;
    const int64_t npad = round_up(c->kplan_n, kPad);
    if (v->pair) {
        PairArgs a{};
        a.sh = shadow_at(c->kshadow.p, npad);
        a.items = p.d_pair_items.p;
        a.n_items = static_cast<int>(p.pair_items.size());
        a.queue = c->queue.p;
        a.fx = c->kfx.p;
        a.npad = npad;
        a.scale = c->kscale.p;
        a.h_uniform = c->kh_uniform;
        a.tile_mass = c->ktile_mass.p;
        a.err = c->errflag.p;
        cudaStream_t s = c->stream;
        cudaEvent_t e0 = nullptr, e1 = nullptr;
        khrr_status st;
        if (c->timing && (st = c->timing_pair(&e0, &e1)) != KHRR_OK) return st;
        if ((st = c->cuda(cudaMemsetAsync(c->queue.p, 0, sizeof(unsigned), s), "queue reset")) != KHRR_OK) return st;
        if ((st = c->cuda(cudaMemsetAsync(c->kfx.p, 0, sizeof(unsigned long long) * kFxComps * npad, s),
                          "sums reset")) != KHRR_OK)
            return st;
        if (e0) cudaEventRecord(e0, s);
        if ((st = c->cuda(launch_pair(v, a, std::min(a.n_items, c->resident_ctas(v)), s), "pair force kernel")) !=
            KHRR_OK)
            return st;
        if (e1) cudaEventRecord(e1, s);
        if (c->timing) {
            c->timed_launches += 1;
            c->timed_pairs += static_cast<double>(c->kplan_n) * static_cast<double>(c->kplan_n);
        }
        return KHRR_OK;
    }
    ForceArgs a{};
    a.j = shadow_at(c->kshadow.p, npad);
    a.i = distinct_i ? shadow_at(c->kishadow.p, npad) : a.j;
    a.items = p.d_items.p;
    a.n_items = static_cast<int>(p.items.size());
    a.queue = c->queue.p;
    a.part = c->kpart.p;
    a.npad = npad;
    a.h_uniform = 0.0f;
    a.err = c->errflag.p;
    cudaStream_t s = c->stream;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    khrr_status st;
    if (c->timing && (st = c->timing_pair(&e0, &e1)) != KHRR_OK) return st;
    if ((st = c->cuda(cudaMemsetAsync(c->queue.p, 0, sizeof(unsigned), s), "queue reset")) != KHRR_OK) return st;
    if (e0) cudaEventRecord(e0, s);
    const int grid = std::min(a.n_items, c->resident_ctas(v));
    if ((st = c->cuda(launch_force(v, a, grid, s), "force kernel")) != KHRR_OK) return st;
    if (e1) cudaEventRecord(e1, s);
    if (c->timing) {
        c->timed_launches += 1;
        c->timed_pairs += static_cast<double>(c->kplan_n) * static_cast<double>(c->kplan_n);
    }
    return KHRR_OK;
}

}  // namespace

extern "C" {

khrr_status khrr_accel(khrr_ctx* c, double* acc, const double* pos_i, const double* pos_j,
                       const double* mass_j, const double* eps2_j, int64_t n, int flags) {
    khrr::NvtxRange nvtx_range("khrr_accel");
    if (!c) return KHRR_ERR_INVALID_ARG;
    if (n == 0) return KHRR_OK;  // nothing to do, as a launch of zero blocks
    if (!acc) return c->fail(KHRR_ERR_INVALID_ARG, "null acc");
    const ForceVariant* v = nullptr;
    khrr_status st = prepare_kernel_pass(c, pos_i, pos_j, mass_j, eps2_j, n, true, false, &v);
    if (st != KHRR_OK) return st;
    if ((st = run_kernel_pass(c, v, pos_i != pos_j)) != KHRR_OK) return st;
    if (v->pair)
        return c->cuda(launch_reduce_pair_fx(c->kfx.p, round_up(n, kPad), c->kscale.p, n, acc, nullptr,
                                             (flags & KHRR_OVERWRITE) != 0, c->stream),
                       "reduce sums");
    return c->cuda(launch_reduce_partials(c->kpart.p, round_up(n, kPad), c->kplan.nslots, n, acc, nullptr,
                                          (flags & KHRR_OVERWRITE) != 0, c->stream),
                   "reduce partials");
}

khrr_status khrr_phi(khrr_ctx* c, double* phi, const double* pos_i, const double* pos_j,
                     const double* mass_j, const double* eps2_j, int64_t n, int flags) {
    khrr::NvtxRange nvtx_range("khrr_phi");
    if (!c) return KHRR_ERR_INVALID_ARG;
    if (n == 0) return KHRR_OK;
    if (!phi) return c->fail(KHRR_ERR_INVALID_ARG, "null phi");
    const ForceVariant* v = nullptr;
    khrr_status st = prepare_kernel_pass(c, pos_i, pos_j, mass_j, eps2_j, n, false, true, &v);
    if (st != KHRR_OK) return st;
    if ((st = run_kernel_pass(c, v, pos_i != pos_j)) != KHRR_OK) return st;
    if (v->pair)
        return c->cuda(launch_reduce_pair_fx(c->kfx.p, round_up(n, kPad), c->kscale.p, n, nullptr, phi,
                                             (flags & KHRR_OVERWRITE) != 0, c->stream),
                       "reduce sums");
    return c->cuda(launch_reduce_partials(c->kpart.p, round_up(n, kPad), c->kplan.nslots, n, nullptr, phi,
                                          (flags & KHRR_OVERWRITE) != 0, c->stream),
                   "reduce partials");
}

khrr_status khrr_integ_time(khrr_ctx* c, const double* acc, double* pos_t, double* vel_t,
                            const double* pos, const double* vel, double dt, int istep, double t,
                            double* acc0, int64_t n) {
    (void)t;  // the reference passes t to dev_fex, which ignores it (static field)
    if (!c) return KHRR_ERR_INVALID_ARG;
    if (n == 0) return KHRR_OK;
    if (n < 0 || !acc || !pos_t || !vel_t || !pos || !vel || (istep == 1 && !acc0) || (istep != 0 && istep != 1))
        return c->fail(KHRR_ERR_INVALID_ARG, "bad integrator arguments");
    return c->cuda(launch_integ_time(acc, pos_t, vel_t, pos, vel, dt, istep, acc0, n, c->field, c->stream),
                   "integrator");
}

// Autotuner: every compiled kernel shape is timed on a force pass over the
// uploaded state (automatic j split), the fastest kept; the winner is cached
// per state key ("npad:nsys:uniform") in a small JSON object file.
khrr_status khrr_autotune(khrr_ctx* c, const char* cache_path) {
    khrr::NvtxRange nvtx_range("khrr_autotune");
    if (!c) return KHRR_ERR_INVALID_ARG;
    if (!c->has_state) return c->fail(KHRR_ERR_STATE, "no state uploaded");
    char key[96];
    std::snprintf(key, sizeof key, "%lld:%zu:%d", static_cast<long long>(c->npad), c->cnt.size(),
                  c->uniform ? 1 : 0);
    std::string text;
    if (cache_path) {
        std::ifstream in(cache_path);
        std::stringstream ss;
        ss << in.rdbuf();
        text = ss.str();
        const std::string needle = std::string("\"") + key + "\": [";
        const size_t at = text.find(needle);
        if (at != std::string::npos) {
            khrr_tuning t{};
            if (std::sscanf(text.c_str() + at + needle.size(), "%d, %d, %d, %d, %d", &t.threads, &t.i_per_thread,
                            &t.j_tile, &t.j_split, &t.packed) == 5 &&
                khrr_set_tuning(c, &t) == KHRR_OK)
                return KHRR_OK;
        }
    }
    const bool was_timing = c->timing;
    const khrr_tuning keep = c->tuning;
    khrr_tuning best = keep;
    double best_ms = 1e300;
    // {threads, i bodies per thread, packed, j_split}; packed 2 is the
    // symmetric pair kernel, whose j_split is its chunk of blocks per item
    const int shapes[][4] = {{128, 8, 2, 0}, {128, 8, 2, 4}, {128, 8, 2, 12}, {128, 2, 1, 0}, {128, 4, 1, 0},
                             {256, 2, 1, 0}, {256, 4, 1, 0}, {128, 4, 0, 0},  {128, 8, 0, 0}, {256, 4, 0, 0},
                             {256, 8, 0, 0}};
    for (const auto& sh : shapes) {
        khrr_tuning t{sh[0], sh[1], 128, sh[3], sh[2]};
        if (khrr_set_tuning(c, &t) != KHRR_OK) continue;
        khrr_enable_timing(c, 0);
        khrr_status st = khrr_forces(c, KHRR_ACC);  // warm-up (plans, caches)
        khrr_enable_timing(c, 1);
        for (int r = 0; r < 2 && st == KHRR_OK; ++r) st = khrr_forces(c, KHRR_ACC);
        double ms = 0.0;
        int64_t launches = 0;
        if (st == KHRR_OK) st = khrr_force_timing(c, &ms, &launches, nullptr);
        if (st != KHRR_OK) {
            khrr_enable_timing(c, was_timing);
            khrr_set_tuning(c, &keep);
            return st;
        }
        const double per = launches > 0 ? ms / static_cast<double>(launches) : ms;
        if (per < best_ms) {
            best_ms = per;
            best = t;
        }
    }
    khrr_enable_timing(c, was_timing);
    khrr_status st = khrr_set_tuning(c, &best);
    if (st != KHRR_OK) return st;
    if (cache_path) {
        // Append (or start) the JSON object.
        std::string entry = std::string("\"") + key + "\": [" + std::to_string(best.threads) + ", " +
                            std::to_string(best.i_per_thread) + ", " + std::to_string(best.j_tile) + ", " +
                            std::to_string(best.j_split) + ", " + std::to_string(best.packed) + "]";
        std::string out;
        const size_t close = text.rfind('}');
        if (close == std::string::npos || text.find('{') == std::string::npos) {
            out = "{\n " + entry + "\n}\n";
        } else {
            std::string head = text.substr(0, close);
            while (!head.empty() && (head.back() == '\n' || head.back() == ' ')) head.pop_back();
            out = head + (head.back() == '{' ? "\n " : ",\n ") + entry + "\n}\n";
        }
        std::ofstream o(cache_path);
        if (!o) return c->fail(KHRR_ERR_IO, "cannot write autotune cache %s", cache_path);
        o << out;
    }
    return KHRR_OK;
}

}  // extern "C"
