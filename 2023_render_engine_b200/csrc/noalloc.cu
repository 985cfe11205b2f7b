// rt_trace_closest_noalloc: the closest-hit trace for callers that must not allocate.
//
// Some callers cannot call cudaMalloc while they trace: code that runs on a render
// thread with a frame-time budget (an allocation can synchronise the device), hosts that
// hand all device memory to their own pool allocator and forbid allocations from
// libraries, and applications that have already claimed nearly all device memory. For
// them this entry point takes its scratch — the queue of rays that need the
// reference-order replay and the queue/status counters — from a fixed array compiled into
// this library instead of from the scene's on-demand buffers.
//
// The array is a file-scope __device__ array, so every GPU that loads the library holds
// it (a little over 4 MiB) until the process exits. Host code cannot use the array's name
// as a device address; its address is looked up once per device with
// cudaGetSymbolAddress, with that device current, and kept for the life of the process.
// A cudaDeviceReset by the application destroys the module that holds the array, so the
// kept address is stale afterwards: do not call this entry point after resetting a device.
#include <mutex>

#include "rt_internal.h"

namespace rtb {
namespace {

constexpr uint64_t kNoAllocMaxRays = 1ull << 20;  // rays per call
constexpr uint64_t kCounterWords = 16;

static __device__ __align__(256) uint32_t g_noalloc_scratch[kCounterWords + kNoAllocMaxRays];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
uint32_t *g_scratch_ptr[kMaxDevices] = {};

// Device address of the scratch array on `device` (which must be current).
int scratch_for(int device, uint32_t **out)
{
    if (device < 0 || device >= kMaxDevices) return fail(RT_ERR_INVALID, "rt_trace_closest_noalloc: device id");
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_scratch_ptr[device]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return cuda_status(e, "cudaGetSymbolAddress(g_noalloc_scratch)");
        g_scratch_ptr[device] = static_cast<uint32_t *>(p);
    }
    *out = g_scratch_ptr[device];
    return RT_OK;
}

}  // namespace
}  // namespace rtb

using namespace rtb;

extern "C" int rt_trace_closest_noalloc(rt_scene *s, const rt_ray *rays, uint64_t n, rt_hit *hits, uint32_t flags)
{
    if (!s) return fail(RT_ERR_INVALID, "rt_trace_closest_noalloc: null scene");
    if (s->merged) return fail(RT_ERR_UNSUPPORTED, "rt_trace_closest_noalloc: not available on a merged scene");
    if (!s->committed) return fail(RT_ERR_STATE, "rt_trace_closest_noalloc: scene not committed");
    if (n && (!rays || !hits)) return fail(RT_ERR_INVALID, "rt_trace_closest_noalloc: null buffer");
    if (n > kNoAllocMaxRays)
        return fail(RT_ERR_CAPACITY, "rt_trace_closest_noalloc: at most 1048576 rays per call (split the batch or "
                                     "use rt_trace_closest)");
    if ((reinterpret_cast<uintptr_t>(rays) | reinterpret_cast<uintptr_t>(hits)) & 15u)
        return fail(RT_ERR_INVALID, "rt_trace_closest_noalloc: buffers must be 16-byte aligned");
    if (n == 0) {  // nothing to launch; the shared counters may hold another call's values
        s->last_rays = 0;
        s->last_fallback = 0;
        return RT_OK;
    }
    RTB_CUDA(cudaSetDevice(s->ctx->device));
    uint32_t *scratch = nullptr;
    RTB_CHECK(scratch_for(s->ctx->device, &scratch));
    uint32_t *counters = scratch;               // cleared by the launch before the kernels run
    uint32_t *queue = scratch + kCounterWords;  // written before it is read within the call
    cudaStream_t st = s->ctx->stream;
    RTB_CHECK(launch_trace_closest(s->view(), rays, n, hits, flags, queue, (uint32_t)n, counters, st));
    uint32_t c[4] = {0, 0, 0, 0};
    RTB_CUDA(cudaMemcpyAsync(c, counters, sizeof(c), cudaMemcpyDeviceToHost, st));
    RTB_CUDA(cudaStreamSynchronize(st));
    s->last_rays = n;
    s->last_fallback = c[0];
    switch (c[1]) {
    case DEV_OK:
        return RT_OK;
    case DEV_STACK_OVERFLOW:
        return fail(RT_ERR_CAPACITY, "traversal stack overflow: a walk that could not be replayed stopped early");
    case DEV_QUEUE_OVERFLOW:
        return fail(RT_ERR_CAPACITY, "exact-traversal queue overflow");
    default:
        return fail(RT_ERR_TIMEOUT, "traversal step cap");
    }
}
