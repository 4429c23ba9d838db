// khrr_accel_noalloc: the direct-sum force pass with all of its scratch in a
// file-scope device array, for callers that cannot allocate device memory on
// their call path (a host program that fixes its device-memory budget at
// start-up, or a plugin host that only hands out buffers it owns).
//
// It drives the same force kernel as khrr_accel (packed form, 128 threads x
// 4 i bodies, 128-body j tiles, non-uniform softening) over the same work
// decomposition, but takes every scratch buffer from g_noalloc_scratch:
//   counters  queue counter + error flag (cleared on every call)
//   jshadow   FP32 SoA shadow of the j bodies (x, y, z, m, eps^2 / 2)
//   ishadow   shadow of the i bodies when pos_i != pos_j
//   items     the work queue, written on the device by noalloc_items_kernel
//   part      per-chunk FP64 partial sums, reduced into acc at the end
// Host code never uses the array's name as an address: the device address is
// looked up per device with cudaGetSymbolAddress (with that device current)
// and passed to the kernels.  A set-up that failed is tried again on the next
// call; only a successful one is kept.
//
// Failure reporting: the call only enqueues work, so a bounded wait that gives
// up inside the force kernel cannot become its return status.  The final
// reduce reads the error flag the force kernel raises and then writes NaN to
// every acc entry instead of the sums, so a caller never gets partial forces
// that look valid.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <mutex>

#include "khrr.h"
#include "khrr_internal.h"

namespace khrr {
namespace {

constexpr int64_t kMaxBodies = KHRR_NOALLOC_MAX_BODIES;  // a multiple of kPad
constexpr int kThreads = 128, kIpt = 4, kJt = 128, kMaxSplit = 8;
constexpr int64_t kItile = static_cast<int64_t>(kThreads) * kIpt;
constexpr int64_t kMaxItems = (kMaxBodies + kItile - 1) / kItile * kMaxSplit;

// Byte offsets of the sections; every one is a multiple of 256.
constexpr size_t kOffCounters = 0;
constexpr size_t kOffJShadow = 256;
constexpr size_t kOffIShadow = kOffJShadow + 5 * kMaxBodies * sizeof(float);
constexpr size_t kOffItems = kOffIShadow + 5 * kMaxBodies * sizeof(float);
constexpr size_t kOffPart = kOffItems + kMaxItems * sizeof(WorkItem);
constexpr size_t kScratchBytes = kOffPart + static_cast<size_t>(kMaxSplit) * kMaxBodies * sizeof(double4);
static_assert(kMaxBodies % kPad == 0, "maximum must be a multiple of the padding");
static_assert(kOffIShadow % 256 == 0 && kOffItems % 256 == 0 && kOffPart % 256 == 0,
              "scratch sections must stay 256-byte aligned");

}  // namespace
}  // namespace khrr

// The whole scratch of khrr_accel_noalloc (about 9.3 MiB per device).
static __device__ __align__(256) unsigned char g_noalloc_scratch[khrr::kScratchBytes];

namespace khrr {
namespace {

// Work item k = (i tile k / S, j chunk k % S); the chunk bounds follow the
// same formula as the context planner (plan_force_items).
__global__ void noalloc_items_kernel(WorkItem* items, int n, int itile, int split, int tiles, int nitems) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nitems) return;
    const int it = k / split, c = k % split;
    WorkItem w{};
    w.i_begin = it * itile;
    w.i_end = n;
    w.j_begin = static_cast<int>(static_cast<int64_t>(c) * tiles / split * kJt);
    w.j_end = static_cast<int>(static_cast<int64_t>(c + 1) * tiles / split * kJt);
    w.slot = c;
    w.sys = 0;
    items[k] = w;
}

struct DeviceSetup {
    bool ok = false;
    unsigned char* base = nullptr;
    int ctas = 1;
};

constexpr int kMaxDevices = 64;
DeviceSetup g_setup[kMaxDevices];
std::mutex g_setup_mutex;

// Per device, with that device current: the scratch's device address, the
// kernel's shared-memory attribute and its resident CTA count.  Kept once it
// succeeded; after a failure (for instance a first call made inside a stream
// capture) the next call tries again.
cudaError_t setup_device(int dev, const ForceVariant* v, DeviceSetup** out) {
    if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    DeviceSetup& s = g_setup[dev];
    *out = &s;
    if (s.ok) return cudaSuccess;
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(v->fn, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(v->smem));
    if (e != cudaSuccess) return e;
    int occ = 0, sms = 0;
    if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, v->fn, v->threads, v->smem)) != cudaSuccess) return e;
    if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
    s.base = static_cast<unsigned char*>(p);
    s.ctas = std::max(1, occ) * std::max(1, sms);
    s.ok = true;
    return cudaSuccess;
}

// acc[i] (+)= sum of the body's split partials, in FP64; NaN for every body
// when the force kernel raised its error flag (a bounded wait gave up, so
// some partials were never written).
__global__ void noalloc_reduce_kernel(const double4* __restrict__ part, long long npad, int nslots, int64_t n,
                                      const unsigned* __restrict__ err, double* __restrict__ acc, int overwrite) {
    const bool failed = *err != 0u;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        if (failed) {
            acc[3 * i] = acc[3 * i + 1] = acc[3 * i + 2] = __longlong_as_double(0x7ff8000000000000LL);
            continue;
        }
        double sx = 0.0, sy = 0.0, sz = 0.0;
        for (int s = 0; s < nslots; ++s) {
            const double4 p = part[s * npad + i];
            sx += p.x;
            sy += p.y;
            sz += p.z;
        }
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
}

khrr_status as_status(cudaError_t e) { return e == cudaSuccess ? KHRR_OK : KHRR_ERR_CUDA; }

}  // namespace
}  // namespace khrr

extern "C" khrr_status khrr_accel_noalloc(double* acc, const double* pos_i, const double* pos_j,
                                          const double* mass_j, const double* eps2_j, int64_t n, int flags,
                                          void* stream) {
    using namespace khrr;
    if (!acc || !pos_i || !pos_j || !mass_j || !eps2_j || n < 1) return KHRR_ERR_INVALID_ARG;
    if (n > kMaxBodies) return KHRR_ERR_TOO_LARGE;
    const ForceVariant* v = find_force_variant(kThreads, kIpt, kJt, true, false, true, false);
    if (!v) return KHRR_ERR_UNSUPPORTED;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return as_status(e);
    DeviceSetup* s = nullptr;
    if ((e = setup_device(dev, v, &s)) != cudaSuccess) return as_status(e);

    const cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int64_t npad = (n + kPad - 1) / kPad * kPad;
    const int tiles = static_cast<int>(npad / kJt);
    const int nit = static_cast<int>((n + kItile - 1) / kItile);
    const int split = std::max(1, std::min({kMaxSplit, tiles, s->ctas / nit}));
    const int nitems = nit * split;

    unsigned* counters = reinterpret_cast<unsigned*>(s->base + kOffCounters);
    const Shadow jsh = shadow_at(reinterpret_cast<float*>(s->base + kOffJShadow), npad);
    const Shadow ish = shadow_at(reinterpret_cast<float*>(s->base + kOffIShadow), npad);
    WorkItem* items = reinterpret_cast<WorkItem*>(s->base + kOffItems);
    double4* part = reinterpret_cast<double4*>(s->base + kOffPart);

    // The array keeps the previous call's contents: the queue counter and the
    // error flag must start at zero; everything else is overwritten.
    if ((e = cudaMemsetAsync(counters, 0, 2 * sizeof(unsigned), st)) != cudaSuccess) return as_status(e);
    noalloc_items_kernel<<<(nitems + 127) / 128, 128, 0, st>>>(items, static_cast<int>(n), static_cast<int>(kItile),
                                                              split, tiles, nitems);
    if ((e = cudaGetLastError()) != cudaSuccess) return as_status(e);
    if ((e = launch_pack(pos_j, mass_j, eps2_j, n, npad, jsh, st)) != cudaSuccess) return as_status(e);
    const bool distinct = pos_i != pos_j;
    if (distinct && (e = launch_pack(pos_i, mass_j, eps2_j, n, npad, ish, st)) != cudaSuccess) return as_status(e);

    ForceArgs a{};
    a.j = jsh;
    a.i = distinct ? ish : jsh;
    a.items = items;
    a.n_items = nitems;
    a.queue = counters;
    a.part = part;
    a.npad = npad;
    a.h_uniform = 0.0f;
    a.err = counters + 1;
    if ((e = launch_force(v, a, std::min(nitems, s->ctas), st)) != cudaSuccess) return as_status(e);
    const int rgrid = static_cast<int>(std::min<int64_t>((n + 255) / 256, 148 * 8));
    noalloc_reduce_kernel<<<rgrid, 256, 0, st>>>(part, npad, split, n, counters + 1, acc,
                                                 (flags & KHRR_OVERWRITE) != 0 ? 1 : 0);
    return as_status(cudaGetLastError());
}
