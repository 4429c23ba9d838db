// Symmetric direct-sum gravity on sm_100a: every unordered pair of bodies of a
// system is evaluated once and applied to both bodies (Newton's third law).
// The sums are those of ACCEL_kernel (nbody-kernel.cuh:89-142) and PHI_kernel
// (nbody-kernel.cuh:43-86); the reference's softening term
// 0.5 (eps2_i + eps2_j) is symmetric in i and j, so one r^-3 serves both.
//
// Decomposition.  A system's padded bodies form blocks of kPairBlock = 1024
// (the last block may be shorter).  Block row b is the block pairs (b, J),
// J >= b, cut into chunks of C blocks, one PairItem each.  A CTA holds the
// bodies of block b in registers (8 per thread, 128 threads) and streams the
// chunk's j bodies through a 3-stage ring of 128-body shared-memory tiles
// filled by cp.async.bulk (no multicast) completing on mbarriers.  Tiles of
// block b itself are evaluated one-sided (every ordered pair once, i side
// only).  Tiles of J > b are evaluated symmetrically: the i side accumulates
// in registers, and the reaction on each j body, summed over the CTA's i
// bodies, is written once as an FP32 partial.
//
// Partial slots (float4 {ax, ay, az, sum m/r} per [slot][body]).  A body of
// block B receives the reaction of every block I < B in slot I and one i-side
// sum per chunk u of its own row in slot B + u; the corrector adds its
// B + (chunks of row B) slots in FP64.  Every slot is written exactly once per
// pass: no atomics, and the result is bitwise reproducible.
//
// The reaction sum across a warp.  In a 32-body sub-chunk of the tile, lane l
// evaluates j = (l + s) mod 32 at step s against its 8 i bodies, adds the
// result to the running reaction it holds for that j and hands the reaction
// to lane l - 1 (one shuffle per component); after 32 steps lane l holds the
// reaction of j = l summed over the warp's 256 i bodies.  The four warps' sums
// meet in shared memory (double-buffered by tile parity) and one thread per j
// body adds them and writes the partial.
//
// Inner loop: packed f32x2 instructions over pairs of i bodies (k, k + 1)
// against one j: d (3 add), r^2 (3 fma), two MUFU.RSQ, r^-3 (2 mul), i side
// (3 fma), j side (3 fma): 14 packed instructions per two pair evaluations,
// that is 7 FP32 operations per interaction against 11 for the one-sided
// kernel.  Tile-uniform masses (every 1024 block one mass) are factored out of
// both sums; otherwise m_j and m_i enter per pair (2 more multiplies).
//
// Accuracy: i-side tile partials (128 terms) fold into compensated (hi + lo)
// running sums; a reaction partial is a sum of 1024 terms in three levels
// (8 i bodies, 32 lanes, 4 warps).
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

constexpr int kBarBytes = 128;
constexpr int NT = kPairThreads;   // threads per CTA
constexpr int K = kPairBodies;     // i bodies per thread
constexpr int KP = K / 2;          // packed i pairs per thread
constexpr int JT = kPairTile;      // j bodies per tile
constexpr int STAGES = 3;
constexpr int W = NT / 32;         // warps
static_assert(NT * K == kPairBlock, "block = threads x bodies per thread");
static_assert(JT == NT, "one thread per j body writes the reaction partials");
static_assert(JT % 32 == 0 && JT == kPad, "tiles are whole 32-body sub-chunks and padding units");

constexpr unsigned kUnif = 1;   // every body has the same softening: no h array
constexpr unsigned kAcc = 2;    // accumulate accelerations
constexpr unsigned kPhi = 4;    // accumulate potentials
constexpr unsigned kBMass = 8;  // one mass per 1024 block: masses factored out

template <unsigned F>
struct PairShape {
    static constexpr bool UNIF = F & kUnif, ACC = F & kAcc, PHI = F & kPhi, BMASS = F & kBMass;
    static constexpr int NC = (ACC ? 3 : 0) + (PHI ? 1 : 0);
    static constexpr int NCOMP = 3 + (BMASS ? 0 : 1) + (UNIF ? 0 : 1);  // x, y, z, [m], [h]
    static constexpr int kOffM = 3, kOffH = BMASS ? 3 : 4;
    static constexpr unsigned kTileBytes = NCOMP * JT * 4u;
    static constexpr int kJwFloats = W * NC * JT;  // one parity of the reaction buffer
    static constexpr size_t kSmem = kBarBytes + (size_t)STAGES * kTileBytes + 2 * (size_t)kJwFloats * 4;
};

// One tile: the lane's 8 i bodies against the tile's 128 j bodies in four
// 32-body sub-chunks, each visited in the rotated order above.  SYM adds the
// reactions (written to jw[warp][comp][j]); without it the tile is the i
// block itself and only the i side is summed.
template <unsigned F, bool SYM>
__device__ __forceinline__ void pair_tile(const float* __restrict__ tile, float* __restrict__ jw,
                                          const float2 (&nx)[KP], const float2 (&ny)[KP], const float2 (&nz)[KP],
                                          const float2 (&hi)[KP], const float2 (&mi)[KP], float2 e2,
                                          float2 (&ai)[PairShape<F>::NC][KP], int lane, int warp) {
    using S = PairShape<F>;
    constexpr bool UNIF = S::UNIF, ACC = S::ACC, PHI = S::PHI, BMASS = S::BMASS;
    constexpr int NC = S::NC, CP = NC - 1;  // CP: the potential's component
    const float* X = tile;
    const float* Y = tile + JT;
    const float* Z = tile + 2 * JT;
    const float* M = tile + S::kOffM * JT;
    const float* H = tile + S::kOffH * JT;
#pragma unroll 1
    for (int c = 0; c < JT / 32; ++c) {
        const int base = c * 32;
        float rx = 0.f, ry = 0.f, rz = 0.f, rp = 0.f;  // reaction held by this lane
#pragma unroll 2
        for (int s = 0; s < 32; ++s) {
            const int jj = base + ((lane + s) & 31);
            const float xj = X[jj], yj = Y[jj], zj = Z[jj];
            const float mj = BMASS ? 1.f : M[jj];
            const float hj = UNIF ? 0.f : H[jj];
            const float2 X2 = f2(xj, xj), Y2 = f2(yj, yj), Z2 = f2(zj, zj);
            const float2 M2 = f2(mj, mj), H2 = f2(hj, hj);
            float2 tx = f2(rx, 0.f), ty = f2(ry, 0.f), tz = f2(rz, 0.f), tp = f2(rp, 0.f);
#pragma unroll
            for (int p = 0; p < KP; ++p) {
                const float2 dx = __fadd2_rn(X2, nx[p]);
                const float2 dy = __fadd2_rn(Y2, ny[p]);
                const float2 dz = __fadd2_rn(Z2, nz[p]);
                float2 r2 = UNIF ? e2 : __fadd2_rn(H2, hi[p]);
                r2 = __ffma2_rn(dx, dx, r2);
                r2 = __ffma2_rn(dy, dy, r2);
                r2 = __ffma2_rn(dz, dz, r2);
                const float2 inv = f2(rsqrt_approx(r2.x), rsqrt_approx(r2.y));
                if (ACC) {
                    const float2 i3 = __fmul2_rn(inv, __fmul2_rn(inv, inv));
                    const float2 fi = BMASS ? i3 : __fmul2_rn(M2, i3);
                    ai[0][p] = __ffma2_rn(dx, fi, ai[0][p]);
                    ai[1][p] = __ffma2_rn(dy, fi, ai[1][p]);
                    ai[2][p] = __ffma2_rn(dz, fi, ai[2][p]);
                    if (SYM) {
                        const float2 fj = BMASS ? i3 : __fmul2_rn(mi[p], i3);
                        tx = __ffma2_rn(dx, fj, tx);
                        ty = __ffma2_rn(dy, fj, ty);
                        tz = __ffma2_rn(dz, fj, tz);
                    }
                }
                if (PHI) {
                    ai[CP][p] = BMASS ? __fadd2_rn(ai[CP][p], inv) : __ffma2_rn(M2, inv, ai[CP][p]);
                    if (SYM) tp = BMASS ? __fadd2_rn(tp, inv) : __ffma2_rn(mi[p], inv, tp);
                }
            }
            if (SYM) {
                // Hand the reaction of j to the lane that evaluates it next.
                const int src = (lane + 1) & 31;
                if (ACC) {
                    rx = __shfl_sync(0xffffffffu, tx.x + tx.y, src);
                    ry = __shfl_sync(0xffffffffu, ty.x + ty.y, src);
                    rz = __shfl_sync(0xffffffffu, tz.x + tz.y, src);
                }
                if (PHI) rp = __shfl_sync(0xffffffffu, tp.x + tp.y, src);
            }
        }
        if (SYM) {
            float* w = jw + warp * NC * JT + base + lane;  // after 32 steps: the reaction of j = base + lane
            if (ACC) {
                w[0] = rx;
                w[JT] = ry;
                w[2 * JT] = rz;
            }
            if (PHI) w[CP * JT] = rp;
        }
    }
}

template <unsigned F>
__global__ void __launch_bounds__(NT, ((F & kPhi) ? 2 : 3)) pair_kernel(const PairArgs a) {
    using S = PairShape<F>;
    constexpr bool UNIF = S::UNIF, ACC = S::ACC, PHI = S::PHI, BMASS = S::BMASS;
    constexpr int NC = S::NC, NCOMP = S::NCOMP, CP = NC - 1;
    static_assert(NC > 0, "nothing to accumulate");

    extern __shared__ __align__(128) unsigned char smem_raw[];
    uint64_t* full = reinterpret_cast<uint64_t*>(smem_raw);
    float* ring = reinterpret_cast<float*>(smem_raw + kBarBytes);  // [STAGES][NCOMP][JT]
    float* jwbuf = ring + STAGES * NCOMP * JT;                      // [2][W][NC][JT]
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

        // i bodies k = 2p, 2p + 1 of this thread: negated coordinates, the eps
        // term and the mass (0 past the block's end, so those lanes add no
        // reaction).
        float2 nx[KP], ny[KP], nz[KP], hi[KP], mi[KP];
#pragma unroll
        for (int p = 0; p < KP; ++p) {
            float v[2][5];
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int i = w.i_begin + (2 * p + h) * NT + tid;
                if (i < w.i_end) {
                    v[h][0] = -a.sh.x[i];
                    v[h][1] = -a.sh.y[i];
                    v[h][2] = -a.sh.z[i];
                    v[h][3] = UNIF ? 0.f : a.sh.h[i];
                    v[h][4] = BMASS ? 1.f : a.sh.m[i];
                } else {
                    v[h][0] = v[h][1] = v[h][2] = 0.f;
                    v[h][3] = 1.f;
                    v[h][4] = 0.f;
                }
            }
            nx[p] = f2(v[0][0], v[1][0]);
            ny[p] = f2(v[0][1], v[1][1]);
            nz[p] = f2(v[0][2], v[1][2]);
            hi[p] = f2(v[0][3], v[1][3]);
            mi[p] = f2(v[0][4], v[1][4]);
        }
        float rh[NC][K], rl[NC][K];  // compensated running i-side sums
#pragma unroll
        for (int c = 0; c < NC; ++c)
#pragma unroll
            for (int k = 0; k < K; ++k) rh[c][k] = rl[c][k] = 0.f;
        const float mI = BMASS ? a.tile_mass[w.i_begin / JT] : 1.f;

        for (int t = 0; t < ntiles; ++t) {
            const unsigned q = consumed + static_cast<unsigned>(t);
            const int stage = static_cast<int>(q % STAGES);
            const int jt0 = w.j_begin + t * JT;
            const bool sym = jt0 >= w.diag_end;
            float* jw = jwbuf + (q & 1u) * S::kJwFloats;
            const float mt = BMASS ? a.tile_mass[jt0 / JT] : 1.f;
            const bool ok = mbar_wait_bounded(&full[stage], (q / STAGES) & 1u);

            float2 ai[NC][KP];
#pragma unroll
            for (int c = 0; c < NC; ++c)
#pragma unroll
                for (int p = 0; p < KP; ++p) ai[c][p] = f2(0.f, 0.f);
            if (ok) {
                const float* tile = ring + stage * NCOMP * JT;
                if (sym) pair_tile<F, true>(tile, jw, nx, ny, nz, hi, mi, e2, ai, lane, warp);
                else pair_tile<F, false>(tile, jw, nx, ny, nz, hi, mi, e2, ai, lane, warp);
            }
            // Fold the tile's i-side partials (times the tile mass when it was
            // factored out) into the running sums.
#pragma unroll
            for (int c = 0; c < NC; ++c)
#pragma unroll
                for (int p = 0; p < KP; ++p) {
                    two_sum_into(rh[c][2 * p], rl[c][2 * p], BMASS ? mt * ai[c][p].x : ai[c][p].x);
                    two_sum_into(rh[c][2 * p + 1], rl[c][2 * p + 1], BMASS ? mt * ai[c][p].y : ai[c][p].y);
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
                float4 o = make_float4(0.f, 0.f, 0.f, 0.f);
                if (ACC) {
                    o.x = -mI * r[0];
                    o.y = -mI * r[1];
                    o.z = -mI * r[2];
                }
                if (PHI) o.w = mI * r[CP];
                a.part[static_cast<long long>(w.slot_j) * a.npad + jt0 + tid] = o;
            }
        }
        consumed += static_cast<unsigned>(ntiles);

        float4* out = a.part + static_cast<long long>(w.slot_i) * a.npad;
#pragma unroll
        for (int k = 0; k < K; ++k) {
            const int i = w.i_begin + k * NT + tid;
            if (i < w.i_end) {
                float4 o = make_float4(0.f, 0.f, 0.f, 0.f);
                if (ACC) {
                    o.x = rh[0][k] + rl[0][k];
                    o.y = rh[1][k] + rl[1][k];
                    o.z = rh[2][k] + rl[2][k];
                }
                if (PHI) o.w = rh[CP][k] + rl[CP][k];
                out[i] = o;
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

}  // namespace

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

cudaError_t launch_pair(const ForceVariant* v, const PairArgs& a, int grid, cudaStream_t s) {
    PairArgs args = a;
    void* params[] = {&args};
    return cudaLaunchKernel(v->fn, dim3(grid), dim3(v->threads), params, v->smem, s);
}

}  // namespace khrr
