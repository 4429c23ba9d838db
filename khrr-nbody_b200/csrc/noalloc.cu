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
// looked up once per device with cudaGetSymbolAddress (with that device
// current) and passed to the kernels.
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
    std::once_flag once;
    cudaError_t err = cudaSuccess;
    unsigned char* base = nullptr;
    int ctas = 1;
};

constexpr int kMaxDevices = 64;
DeviceSetup g_setup[kMaxDevices];

// Once per device, with that device current: the scratch's device address,
// the kernel's shared-memory attribute and its resident CTA count.
cudaError_t setup_device(int dev, const ForceVariant* v, DeviceSetup** out) {
    if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
    DeviceSetup& s = g_setup[dev];
    std::call_once(s.once, [&] {
        void* p = nullptr;
        s.err = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (s.err != cudaSuccess) return;
        s.base = static_cast<unsigned char*>(p);
        s.err = cudaFuncSetAttribute(v->fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     static_cast<int>(v->smem));
        if (s.err != cudaSuccess) return;
        int occ = 0, sms = 0;
        s.err = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, v->fn, v->threads, v->smem);
        if (s.err != cudaSuccess) return;
        s.err = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        s.ctas = std::max(1, occ) * std::max(1, sms);
    });
    *out = &s;
    return s.err;
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
    return as_status(launch_reduce_partials(part, npad, split, n, acc, nullptr, (flags & KHRR_OVERWRITE) != 0, st));
}
