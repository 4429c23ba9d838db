// Symmetric direct-sum gravity on sm_100a: every unordered pair of bodies of a
// system is evaluated once and applied to both bodies (Newton's third law).
// The sums are those of ACCEL_kernel (nbody-kernel.cuh:89-142) and PHI_kernel
// (nbody-kernel.cuh:43-86); the reference's softening term
// 0.5 (eps2_i + eps2_j) is symmetric in i and j, so one r^-3 serves both.
//
// Decomposition.  A system's padded bodies form blocks of at most
// kPairBlock = 1024 (whole 128-body tiles; with one mass per tile, runs of
// equal-mass tiles, so every block has one mass).  Block row b is the block
// pairs (b, J), J >= b, cut into chunks of C blocks, one PairItem each.  A CTA
// holds the
// bodies of block b in registers (8 per thread, 128 threads) and streams the
// chunk's j bodies through a 3-stage ring of 128-body shared-memory tiles
// filled by cp.async.bulk (no multicast) completing on mbarriers.  Tiles of
// block b itself are evaluated one-sided (every ordered pair once, i side
// only).  Tiles of J > b are evaluated symmetrically: the i side accumulates
// in registers, and the reaction on each j body, summed over the CTA's i
// bodies, is one FP32 partial added to the body's sums.
//
// Results: 64-bit fixed-point sums, one accumulator per body and component
// (ax, ay, az, sum m/r).  Each (i block, symmetric j tile) adds the reactions
// on the tile's 128 bodies, summed over the CTA's 1024 i bodies, and each item
// adds the i block's sums over its chunk; a partial is scaled by its tile's
// power of two, rounded to an integer and added with an integer atomic
// (red.global.add.u64).  Integer addition is associative, so the totals do
// not depend on the order in which CTAs finish: the result is bitwise
// reproducible, and the accumulators take 32 bytes per body, independent of
// the number of blocks.  The corrector converts them back to FP64.
//
// The reaction sum across a warp.  The tile's 128 j bodies form four 32-body
// sub-chunks, taken two at a time.  At step s (0..31) lane l evaluates body
// r = (l + s) mod 32 of both sub-chunks against its 8 i bodies, adds the
// results to the pair of running reactions it holds for those two bodies and
// hands the pair to lane l - 1 (shuffles); after 32 steps lane l holds the
// reactions of the bodies r = l summed over the warp's 256 i bodies.  The four
// warps' sums meet in shared memory (double-buffered by tile parity) and one
// thread per j body adds them and accumulates the partial.
//
// Inner loop: packed f32x2 instructions over the two j bodies of a step
// against one i body (its coordinates duplicated in both lanes once per
// item): d (3 add), r^2 (3 fma), two MUFU.RSQ, r^-3 (2 mul), i side (3 fma),
// j side (3 fma) = 14 f32x2 instructions per two pair evaluations, that is 14
// FP32 operations per evaluation of an unordered pair and 7 per interaction,
// against 11 per interaction for the one-sided kernel.  When every block has one
// mass (and no ghosts) the masses are factored out of both sums; otherwise
// m_j and m_i enter per pair (2 more multiplies).
//
// Accuracy: the i-side partials (two halves of 64 terms per tile, over up to
// eight tiles with accelerations only, one with the potential) fold into
// compensated (hi + lo) running sums kept in shared memory; a reaction partial
// is a sum of 1024 terms in three levels (8 i bodies, 32 lanes, 4 warps).
#include <cstdint>

#include "async_copy.cuh"
#include "khrr_internal.h"

namespace khrr {
namespace {

__device__ __forceinline__ float rsqrt_approx(float x) {
    float y;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

__device__ __forceinline__ void two_sum_into(float& hi, float& lo, float p) {
    const float s = hi + p;
    const float bp = s - hi;
    const float e = (hi - (s - bp)) + (p - bp);
    hi = s;
    lo += e;
}

__device__ __forceinline__ float2 f2(float a, float b) { return make_float2(a, b); }

// A partial (FP32) as a fixed-point integer: times the power of two s,
// rounded to the nearest integer (exact for |v s| >= 2^24).
__device__ __forceinline__ long long to_fx(float v, double s) {
    return __double2ll_rn(static_cast<double>(v) * s);
}

// Integer atomic add without return (red.global.add.u64): two's complement
// makes the unsigned add a signed one.
__device__ __forceinline__ void fx_add(unsigned long long* p, long long v) {
    atomicAdd(p, static_cast<unsigned long long>(v));
}

__device__ __forceinline__ float2 shfl2(float2 v, int src) {
    return f2(__shfl_sync(0xffffffffu, v.x, src), __shfl_sync(0xffffffffu, v.y, src));
}

constexpr int kBarBytes = 128;
constexpr int NT = kPairThreads;  // threads per CTA
constexpr int K = kPairBodies;    // i bodies per thread
constexpr int JT = kPairTile;     // j bodies per tile
constexpr int STAGES = 3;
constexpr int W = NT / 32;        // warps
static_assert(NT * K == kPairBlock, "block = threads x bodies per thread");
static_assert(JT == NT, "one thread per j body writes the reaction partials");
static_assert(JT % 64 == 0 && JT == kPad, "tiles are whole sub-chunk pairs and padding units");

// Unroll of the 32-step loop, measured at 786k bodies: 2 for accelerations
// (149.6 ms per pass against 153.1 for 1 and 151.2 for 4), 1 with the
// potential (168.9 ms against 171.1 for 2 and 175.4 for 4).
#ifndef KHRR_PAIR_UNROLL
#define KHRR_PAIR_UNROLL 2
#endif
constexpr int kSUnroll = KHRR_PAIR_UNROLL;
// Tiles per fold of the acceleration-only variants' i-side partials,
// measured at 786k bodies (ms per pass; relative RMS error vs FP64 on 8192
// targets at 786k / 2.1M): 2: 149.7-150.3, 3.64e-8 / 6.44e-8; 8: 148.3,
// 3.76e-8 / 6.48e-8; 32: 148.0, 4.77e-8 / 6.78e-8; 256 (item ends only):
// 147.9, 2.26e-7 / 1.54e-7.
#ifndef KHRR_PAIR_FOLD
#define KHRR_PAIR_FOLD 8
#endif
constexpr int kFoldEvery = KHRR_PAIR_FOLD;
constexpr int kSUnrollPhi = 1;

constexpr unsigned kUnif = 1;   // every body has the same softening: no h array
constexpr unsigned kAcc = 2;    // accumulate accelerations
constexpr unsigned kPhi = 4;    // accumulate potentials
constexpr unsigned kBMass = 8;  // one mass per block: masses factored out
// Lanes past a short block's end, in the block-mass form, sit this far away:
// r^-3 underflows to exactly 0, so they add nothing to the accelerations'
// reactions, and r^-1 (< 6e-19) adds nothing visible to the potentials'.
constexpr float kFar = 1.0e18f;

template <unsigned F>
struct PairShape {
    static constexpr bool UNIF = F & kUnif, ACC = F & kAcc, PHI = F & kPhi, BMASS = F & kBMass;
    static constexpr int NC = (ACC ? 3 : 0) + (PHI ? 1 : 0);
    static constexpr int NCOMP = 3 + (BMASS ? 0 : 1) + (UNIF ? 0 : 1);  // x, y, z, [m], [h]
    static constexpr int kOffM = 3, kOffH = BMASS ? 3 : 4;
    static constexpr unsigned kTileBytes = NCOMP * JT * 4u;
    static constexpr int kJwFloats = W * NC * JT;       // one parity of the reaction buffer
    static constexpr int kRunFloats = 2 * NC * K * NT;  // (hi, lo) running sums
    static constexpr size_t kSmem =
        kBarBytes + (size_t)STAGES * kTileBytes + (2 * (size_t)kJwFloats + kRunFloats) * 4;
};

// One tile against the lane's K i bodies.  SYM adds the reactions (written
// to jw[warp][comp][j]); without it the tile is the i block itself and only
// the i side is summed.  ai[c][k] keeps the i-side sums of the two lanes (the
// two sub-chunks) apart.
template <unsigned F, bool SYM>
__device__ __forceinline__ void pair_tile(const float* __restrict__ tile, float* __restrict__ jw,
                                          const float2 (&nx)[K], const float2 (&ny)[K], const float2 (&nz)[K],
                                          const float2 (&hi)[K], const float2 (&mi)[K], float2 e2,
                                          float2 (&ai)[PairShape<F>::NC][K], int lane, int warp) {
    using S = PairShape<F>;
    constexpr bool UNIF = S::UNIF, ACC = S::ACC, PHI = S::PHI, BMASS = S::BMASS;
    constexpr int NC = S::NC, CP = NC - 1;  // CP: the potential's component
    const float* X = tile;
    const float* Y = tile + JT;
    const float* Z = tile + 2 * JT;
    const float* M = tile + S::kOffM * JT;
    const float* H = tile + S::kOffH * JT;
    const int src = (lane + 1) & 31;
    constexpr int kU = PHI ? kSUnrollPhi : kSUnroll;
#pragma unroll 1
    for (int c0 = 0; c0 < JT / 32; c0 += 2) {
        float2 rx = f2(0.f, 0.f), ry = rx, rz = rx, rp = rx;  // reactions held by this lane
#pragma unroll kU
        for (int s = 0; s < 32; ++s) {
            const int ja = c0 * 32 + ((lane + s) & 31), jb = ja + 32;
            const float2 X2 = f2(X[ja], X[jb]), Y2 = f2(Y[ja], Y[jb]), Z2 = f2(Z[ja], Z[jb]);
            const float2 M2 = BMASS ? f2(1.f, 1.f) : f2(M[ja], M[jb]);
            const float2 H2 = UNIF ? f2(0.f, 0.f) : f2(H[ja], H[jb]);
#pragma unroll
            for (int k = 0; k < K; ++k) {
                const float2 dx = __fadd2_rn(X2, nx[k]);
                const float2 dy = __fadd2_rn(Y2, ny[k]);
                const float2 dz = __fadd2_rn(Z2, nz[k]);
                float2 r2 = UNIF ? e2 : __fadd2_rn(H2, hi[k]);
                r2 = __ffma2_rn(dx, dx, r2);
                r2 = __ffma2_rn(dy, dy, r2);
                r2 = __ffma2_rn(dz, dz, r2);
                const float2 inv = f2(rsqrt_approx(r2.x), rsqrt_approx(r2.y));
                if (ACC) {
                    const float2 i3 = __fmul2_rn(inv, __fmul2_rn(inv, inv));
                    const float2 fi = BMASS ? i3 : __fmul2_rn(M2, i3);
                    ai[0][k] = __ffma2_rn(dx, fi, ai[0][k]);
                    ai[1][k] = __ffma2_rn(dy, fi, ai[1][k]);
                    ai[2][k] = __ffma2_rn(dz, fi, ai[2][k]);
                    if (SYM) {
                        const float2 fj = BMASS ? i3 : __fmul2_rn(mi[k], i3);
                        rx = __ffma2_rn(dx, fj, rx);
                        ry = __ffma2_rn(dy, fj, ry);
                        rz = __ffma2_rn(dz, fj, rz);
                    }
                }
                if (PHI) {
                    ai[CP][k] = BMASS ? __fadd2_rn(ai[CP][k], inv) : __ffma2_rn(M2, inv, ai[CP][k]);
                    if (SYM) rp = BMASS ? __fadd2_rn(rp, inv) : __ffma2_rn(mi[k], inv, rp);
                }
            }
            if (SYM) {
                // Hand the reactions to the lane that evaluates their bodies next.
                if (ACC) {
                    rx = shfl2(rx, src);
                    ry = shfl2(ry, src);
                    rz = shfl2(rz, src);
                }
                if (PHI) rp = shfl2(rp, src);
            }
        }
        if (SYM) {
            // After 32 steps: the reactions of j = c0 * 32 + lane and of j + 32.
            float* w = jw + warp * NC * JT + c0 * 32 + lane;
            if (ACC) {
                w[0] = rx.x;
                w[32] = rx.y;
                w[JT] = ry.x;
                w[JT + 32] = ry.y;
                w[2 * JT] = rz.x;
                w[2 * JT + 32] = rz.y;
            }
            if (PHI) {
                w[CP * JT] = rp.x;
                w[CP * JT + 32] = rp.y;
            }
        }
    }
}

// Resident CTAs per SM the register allocation aims at: three (168
// registers), the uniform block-mass force + potential variant included (171
// ms per pass at 786k bodies against 178 ms at two); the other force +
// potential variants carry per-body masses or softenings as well and run at
// two rather than spill.
#ifndef KHRR_PAIR_ACC_CTAS
#define KHRR_PAIR_ACC_CTAS 3
#endif
template <unsigned F>
constexpr int pair_min_blocks() {
    if ((F & kAcc) && !(F & kPhi)) return KHRR_PAIR_ACC_CTAS;
    return ((F & kAcc) && (F & kPhi) && !((F & kUnif) && (F & kBMass))) ? 2 : 3;
}

template <unsigned F>
__global__ void __launch_bounds__(NT, (pair_min_blocks<F>())) pair_kernel(const PairArgs a) {
    using S = PairShape<F>;
    constexpr bool UNIF = S::UNIF, ACC = S::ACC, PHI = S::PHI, BMASS = S::BMASS;
    constexpr int NC = S::NC, NCOMP = S::NCOMP, CP = NC - 1;
    static_assert(NC > 0, "nothing to accumulate");

    extern __shared__ __align__(128) unsigned char smem_raw[];
    uint64_t* full = reinterpret_cast<uint64_t*>(smem_raw);
    float* ring = reinterpret_cast<float*>(smem_raw + kBarBytes);  // [STAGES][NCOMP][JT]
    float* jwbuf = ring + STAGES * NCOMP * JT;                      // [2][W][NC][JT]
    float* runs = jwbuf + 2 * S::kJwFloats;                         // [2][NC][K][NT]: hi, lo
    __shared__ int s_item;

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (tid == 0) {
#pragma unroll
        for (int s = 0; s < STAGES; ++s) mbar_init(&full[s], 1);
        fence_mbar_init();
    }
    __syncthreads();

    auto issue = [&](int stage, int jstart) {  // elected thread only
        float* dst = ring + stage * NCOMP * JT;
        mbar_arrive_expect_tx(&full[stage], S::kTileBytes);
        bulk_copy_g2s(dst, a.sh.x + jstart, JT * 4u, &full[stage]);
        bulk_copy_g2s(dst + JT, a.sh.y + jstart, JT * 4u, &full[stage]);
        bulk_copy_g2s(dst + 2 * JT, a.sh.z + jstart, JT * 4u, &full[stage]);
        if (!BMASS) bulk_copy_g2s(dst + S::kOffM * JT, a.sh.m + jstart, JT * 4u, &full[stage]);
        if (!UNIF) bulk_copy_g2s(dst + S::kOffH * JT, a.sh.h + jstart, JT * 4u, &full[stage]);
    };
    // The thread's compensated running sums, component c of i body k.
    auto RH = [&](int c, int k) -> float& { return runs[(c * K + k) * NT + tid]; };
    auto RL = [&](int c, int k) -> float& { return runs[((NC + c) * K + k) * NT + tid]; };

    const float2 e2 = f2(a.h_uniform + a.h_uniform, a.h_uniform + a.h_uniform);
    unsigned consumed = 0;  // tiles this CTA has consumed, over all its items
    for (;;) {
        if (tid == 0) s_item = static_cast<int>(atomicAdd(a.queue, 1u));
        __syncthreads();
        const int it = s_item;
        if (it >= a.n_items) break;
        const PairItem w = a.items[it];
        const int ntiles = (w.j_end - w.j_begin) / JT;
        if (tid == 0) {
            fence_proxy_async();
            for (int s = 0; s < STAGES && s < ntiles; ++s) issue((consumed + s) % STAGES, w.j_begin + s * JT);
        }

        // The thread's i bodies k (index i_begin + k NT + tid), each duplicated
        // in both lanes: negated coordinates, the eps term and the mass (1 in
        // the block-mass form, whose mass is applied per partial).  Lanes past
        // the block's end add no reaction: mass 0, and in the block-mass form
        // (mass not in the pair term) a position kFar away.
        float2 nx[K], ny[K], nz[K], hi[K], mi[K];
#pragma unroll
        for (int k = 0; k < K; ++k) {
            const int i = w.i_begin + k * NT + tid;
            const bool in = i < w.i_end;
            const float far = BMASS ? -kFar : 0.f;
            const float x = in ? -a.sh.x[i] : far, y = in ? -a.sh.y[i] : far, z = in ? -a.sh.z[i] : far;
            const float h = UNIF ? 0.f : (in ? a.sh.h[i] : 1.f);
            const float m = in ? (BMASS ? 1.f : a.sh.m[i]) : 0.f;
            nx[k] = f2(x, x);
            ny[k] = f2(y, y);
            nz[k] = f2(z, z);
            hi[k] = f2(h, h);
            mi[k] = f2(m, m);
#pragma unroll
            for (int c = 0; c < NC; ++c) RH(c, k) = RL(c, k) = 0.f;
        }
        const float mI = BMASS ? a.tile_mass[w.i_begin / JT] : 1.f;

        // i-side partials since the last fold: folded every kFoldEvery-th tile
        // in the acceleration-only variants (every tile: 151.2 ms per pass at
        // 786k, every second 149.6-150.3, every eighth 148.3), every tile where
        // the potential adds to the registers live across tiles (172.3 against
        // 171.0 ms).
        constexpr bool kFoldPairs = !PHI;
        float2 ai[NC][K];
#pragma unroll
        for (int c = 0; c < NC; ++c)
#pragma unroll
            for (int k = 0; k < K; ++k) ai[c][k] = f2(0.f, 0.f);
        for (int t = 0; t < ntiles; ++t) {
            const unsigned q = consumed + static_cast<unsigned>(t);
            const int stage = static_cast<int>(q % STAGES);
            const int jt0 = w.j_begin + t * JT;
            const bool sym = jt0 >= w.diag_end;
            float* jw = jwbuf + (q & 1u) * S::kJwFloats;
            const float mt = BMASS ? a.tile_mass[jt0 / JT] : 1.f;
            const bool ok = mbar_wait_bounded(&full[stage], (q / STAGES) & 1u);

            if (ok) {
                const float* tile = ring + stage * NCOMP * JT;
                if (sym) pair_tile<F, true>(tile, jw, nx, ny, nz, hi, mi, e2, ai, lane, warp);
                else pair_tile<F, false>(tile, jw, nx, ny, nz, hi, mi, e2, ai, lane, warp);
            }
            // Fold the i-side partials (times the tile mass when it was factored
            // out) into the running sums: every tile, or every second tile, at
            // the item's end and before a tile of another mass.
            const bool fold = !kFoldPairs || (t % kFoldEvery) == kFoldEvery - 1 || t + 1 == ntiles ||
                              (BMASS && a.tile_mass[jt0 / JT + 1] != mt);
            if (fold) {
#pragma unroll
                for (int c = 0; c < NC; ++c)
#pragma unroll
                    for (int k = 0; k < K; ++k) {
                        const float v = ai[c][k].x + ai[c][k].y;
                        two_sum_into(RH(c, k), RL(c, k), BMASS ? mt * v : v);
                        ai[c][k] = f2(0.f, 0.f);
                    }
            }
            // Every thread is done with this stage and its reaction buffer
            // (and all waits ended).
            if (__syncthreads_or(!ok)) {
                if (tid == 0) {
                    atomicOr(a.err, kErrTimeout);
                    for (int u = t + 1; u < ntiles && u < t + STAGES; ++u) {
                        const unsigned qu = consumed + static_cast<unsigned>(u);
                        (void)mbar_wait_bounded(&full[qu % STAGES], (qu / STAGES) & 1u);
                    }
                }
                return;
            }
            if (tid == 0 && t + STAGES < ntiles) {
                fence_proxy_async();
                issue(stage, w.j_begin + (t + STAGES) * JT);
            }
            if (sym) {
                // The tile's reactions: one thread per j body adds the four
                // warps' sums (times -m_I when the mass was factored out).
                float r[NC];
#pragma unroll
                for (int c = 0; c < NC; ++c) {
                    float s = 0.f;
#pragma unroll
                    for (int v = 0; v < W; ++v) s += jw[(v * NC + c) * JT + tid];
                    r[c] = s;
                }
                const int j = jt0 + tid;
                if (j < w.real_end) {
                    const FxScale sc = a.scale[jt0 / JT];
                    if (ACC) {
                        fx_add(a.fx + j, to_fx(-mI * r[0], sc.acc));
                        fx_add(a.fx + a.npad + j, to_fx(-mI * r[1], sc.acc));
                        fx_add(a.fx + 2 * a.npad + j, to_fx(-mI * r[2], sc.acc));
                    }
                    if (PHI) fx_add(a.fx + 3 * a.npad + j, to_fx(mI * r[CP], sc.phi));
                }
            }
        }
        consumed += static_cast<unsigned>(ntiles);

        // The i block's sums over the chunk: high and low parts rounded to
        // the fixed point separately (the compensation survives).
#pragma unroll
        for (int k = 0; k < K; ++k) {
            const int i = w.i_begin + k * NT + tid;
            if (i < w.real_end) {
                const FxScale sc = a.scale[w.i_begin / JT + k];
                if (ACC) {
#pragma unroll
                    for (int c = 0; c < 3; ++c)
                        fx_add(a.fx + c * a.npad + i, to_fx(RH(c, k), sc.acc) + to_fx(RL(c, k), sc.acc));
                }
                if (PHI) fx_add(a.fx + 3 * a.npad + i, to_fx(RH(CP, k), sc.phi) + to_fx(RL(CP, k), sc.phi));
            }
        }
    }
}

template <unsigned F>
ForceVariant make_pair_variant() {
    using S = PairShape<F>;
    ForceVariant v{NT,
                   K,
                   JT,
                   STAGES,
                   true,
                   (F & kUnif) != 0,
                   (F & kAcc) != 0,
                   (F & kPhi) != 0,
                   (F & kBMass) != 0,
                   reinterpret_cast<const void*>(&pair_kernel<F>),
                   S::kSmem};
    v.pair = true;
    return v;
}

template <unsigned BASE>
void add_outputs(ForceVariant* v, int& n) {
    v[n++] = make_pair_variant<BASE | kAcc>();
    v[n++] = make_pair_variant<BASE | kAcc | kPhi>();
    v[n++] = make_pair_variant<BASE | kPhi>();
}

struct PairTable {
    ForceVariant v[12];
    int n = 0;
    PairTable() {
        add_outputs<0>(v, n);
        add_outputs<kUnif>(v, n);
        add_outputs<kBMass>(v, n);
        add_outputs<kUnif | kBMass>(v, n);
    }
};

const PairTable& pair_table() {
    static PairTable t;
    return t;
}

// The fixed-point scale of one 128-body tile (FxScale): E = 61 - e with
// bound < 2^e, for the acceleration bound 0.3849 M / (h_t + h_min) (0.385
// used) and the potential bound M / sqrt(h_t + h_min).  A bound of zero (no
// mass) or not finite takes E = 0.
__host__ __device__ inline double fx_pow2(double bound, bool inverse) {
    int e = 0;
    if (bound > 0.0 && bound < 1e300) (void)frexp(bound, &e);
    else e = 61;
    int E = 61 - e;
    E = E < -960 ? -960 : (E > 960 ? 960 : E);
    return ldexp(1.0, inverse ? -E : E);
}

__host__ __device__ inline FxScale fx_scale_of(double h_tile_min, double h_sys_min, double mass_sys) {
    const double H = h_tile_min + h_sys_min;
    const double ba = 0.385 * mass_sys / H, bp = mass_sys / sqrt(H);
    return FxScale{fx_pow2(ba, false), fx_pow2(bp, false), fx_pow2(ba, true), fx_pow2(bp, true)};
}

// Fixed-point sums -> out[i] (+)= sums times the tile's inverse scale, in
// FP64 (the kernel-level entry points; the state path converts them in the
// corrector).
__global__ void reduce_pair_fx_kernel(const unsigned long long* __restrict__ fx, long long npad,
                                      const FxScale* __restrict__ scale, int64_t n, double* __restrict__ acc,
                                      double* __restrict__ phi, int overwrite) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const FxScale sc = scale[i / kPad];
        if (acc) {
            const double sx = static_cast<double>(static_cast<long long>(fx[i])) * sc.inv_acc;
            const double sy = static_cast<double>(static_cast<long long>(fx[npad + i])) * sc.inv_acc;
            const double sz = static_cast<double>(static_cast<long long>(fx[2 * npad + i])) * sc.inv_acc;
            if (overwrite) {
                acc[3 * i] = sx;
                acc[3 * i + 1] = sy;
                acc[3 * i + 2] = sz;
            } else {
                acc[3 * i] += sx;
                acc[3 * i + 1] += sy;
                acc[3 * i + 2] += sz;
            }
        }
        if (phi) {
            const double sp = static_cast<double>(static_cast<long long>(fx[3 * npad + i])) * sc.inv_phi;
            phi[i] = overwrite ? -sp : phi[i] - sp;
        }
    }
}

// Classification of a caller's body arrays for the kernel-level entry points,
// one warp per 128-body tile: tile_mass[t] = the tile's first mass; bit 0 of
// *flags is cleared unless every body of the tile is real and has the mass of
// its 1024 block's first body (the block-mass form), bit 1 unless every
// softening equals eps2[0] (the uniform form), bit 2 unless every softening
// is positive (needed for the fixed-point bounds).  tile_hmin[t] and
// tile_msum[t] receive the tile's smallest eps2 / 2 and its sum of |m|.
__global__ void classify_kernel(const double* __restrict__ mass, const double* __restrict__ eps2, int64_t n,
                                float* __restrict__ tile_mass, double* __restrict__ tile_hmin,
                                double* __restrict__ tile_msum, unsigned* __restrict__ flags) {
    const int64_t warps = (static_cast<int64_t>(gridDim.x) * blockDim.x) >> 5;
    const int lane = threadIdx.x & 31;
    const int64_t ntiles = (n + kPad - 1) / kPad;
    const double e0 = eps2[0];
    for (int64_t t = (blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x) >> 5; t < ntiles; t += warps) {
        const double mt = mass[t * kPad], mb = mass[(t * kPad / kPairBlock) * kPairBlock];
        bool same_mass = true, same_eps = true, pos_eps = true;
        double hmin = 1e300, msum = 0.0;
#pragma unroll
        for (int q = 0; q < kPad / 32; ++q) {
            const int64_t i = t * kPad + q * 32 + lane;
            if (i < n) {
                const double m = mass[i], e = eps2[i];
                same_mass = same_mass && m == mt && m == mb;
                same_eps = same_eps && e == e0;
                pos_eps = pos_eps && e > 0.0;
                hmin = fmin(hmin, 0.5 * e);
                msum += fabs(m);
            } else {
                same_mass = false;
            }
        }
        same_mass = __all_sync(0xffffffffu, same_mass);
        same_eps = __all_sync(0xffffffffu, same_eps);
        pos_eps = __all_sync(0xffffffffu, pos_eps);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            hmin = fmin(hmin, __shfl_xor_sync(0xffffffffu, hmin, o));
            msum += __shfl_xor_sync(0xffffffffu, msum, o);
        }
        if (lane == 0) {
            tile_mass[t] = static_cast<float>(mt);
            tile_hmin[t] = hmin;
            tile_msum[t] = msum;
            if (!same_mass) atomicAnd(flags, ~1u);
            if (!same_eps) atomicAnd(flags, ~2u);
            if (!pos_eps) atomicAnd(flags, ~4u);
        }
    }
}

// One CTA: the system's total |m| (tile sums added in tile order, so the
// bound and hence the scales are the same on every call) and smallest h,
// then every tile's scale.
__global__ void fx_scales_kernel(const double* __restrict__ tile_hmin, const double* __restrict__ tile_msum,
                                 int64_t ntiles, FxScale* __restrict__ scale) {
    __shared__ double s_m[256], s_h[256];
    double m = 0.0, h = 1e300;
    const int64_t per = (ntiles + blockDim.x - 1) / blockDim.x;
    const int64_t t0 = threadIdx.x * per, t1 = t0 + per < ntiles ? t0 + per : ntiles;
    for (int64_t t = t0; t < t1; ++t) {
        m += tile_msum[t];
        h = fmin(h, tile_hmin[t]);
    }
    s_m[threadIdx.x] = m;
    s_h[threadIdx.x] = h;
    __syncthreads();
    if (threadIdx.x == 0) {
        double M = 0.0, Hm = 1e300;
        for (int k = 0; k < blockDim.x; ++k) {
            M += s_m[k];
            Hm = fmin(Hm, s_h[k]);
        }
        s_m[0] = M;
        s_h[0] = Hm;
    }
    __syncthreads();
    const double M = s_m[0], Hm = s_h[0];
    for (int64_t t = threadIdx.x; t < ntiles; t += blockDim.x) scale[t] = fx_scale_of(tile_hmin[t], Hm, M);
}

}  // namespace

FxScale fx_scale(double h_tile_min, double h_sys_min, double mass_sys) {
    return fx_scale_of(h_tile_min, h_sys_min, mass_sys);
}

int pair_variant_count() { return pair_table().n; }

const ForceVariant* pair_variant(int idx) {
    return (idx >= 0 && idx < pair_table().n) ? &pair_table().v[idx] : nullptr;
}

const ForceVariant* find_pair_variant(bool unif, bool acc, bool phi, bool block_mass) {
    const PairTable& t = pair_table();
    for (int i = 0; i < t.n; ++i) {
        const ForceVariant& v = t.v[i];
        if (v.uniform_eps == unif && v.acc == acc && v.phi == phi && v.tile_mass == block_mass) return &v;
    }
    return nullptr;
}

cudaError_t launch_reduce_pair_fx(const unsigned long long* fx, long long npad, const FxScale* scale, int64_t n,
                                  double* acc, double* phi, bool overwrite, cudaStream_t s) {
    int64_t g = (n + 255) / 256;
    if (g > 148 * 32) g = 148 * 32;
    if (g < 1) g = 1;
    reduce_pair_fx_kernel<<<static_cast<unsigned>(g), 256, 0, s>>>(fx, npad, scale, n, acc, phi, overwrite ? 1 : 0);
    return cudaGetLastError();
}

cudaError_t launch_classify(const double* mass, const double* eps2, int64_t n, float* tile_mass, double* tile_hmin,
                            double* tile_msum, FxScale* scale, unsigned* flags, cudaStream_t s) {
    const int64_t ntiles = (n + kPad - 1) / kPad;
    int64_t g = (ntiles * 32 + 255) / 256;
    if (g > 148 * 16) g = 148 * 16;
    if (g < 1) g = 1;
    classify_kernel<<<static_cast<unsigned>(g), 256, 0, s>>>(mass, eps2, n, tile_mass, tile_hmin, tile_msum, flags);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    fx_scales_kernel<<<1, 256, 0, s>>>(tile_hmin, tile_msum, ntiles, scale);
    return cudaGetLastError();
}

cudaError_t launch_pair(const ForceVariant* v, const PairArgs& a, int grid, cudaStream_t s) {
    PairArgs args = a;
    void* params[] = {&args};
    return cudaLaunchKernel(v->fn, dim3(grid), dim3(v->threads), params, v->smem, s);
}

}  // namespace khrr
