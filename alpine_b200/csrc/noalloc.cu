// alpine_gpu_trace_noalloc: a closest-hit query on host buffers that allocates
// no memory.
//
// Some callers cannot call cudaMalloc at query time. Examples: a renderer or
// plugin whose host application owns the whole device-memory budget through
// its own pools; a per-frame callback that cannot afford the implicit device
// synchronisation and possible late out-of-memory failure of an allocation;
// an embedding whose policy forbids driver allocations after set-up. The
// ordinary alpine_gpu_trace grows its device staging buffers with cudaMalloc
// as needed. This variant stages through one fixed array in device global
// memory instead, defined below at file scope.
//
// The array holds kNoAllocMaxRays rays (32 B each), as many hits (16 B each)
// and the 4-byte device status word: 3 MiB + 256 B. Every GPU that loads this
// library holds it until the process exits. Calls with more rays are rejected
// with ALPINE_GPU_ERR_INVALID_ARGUMENT.
//
// Host code must not use the array's name as a device address (on the host it
// is only a stand-in). The device address is obtained once per device with
// cudaGetSymbolAddress, with that device current, on the first call for that
// device; under CUDA's lazy module loading that first call may also load the
// module holding the array. Every call is synchronous and copies through host
// memory, so none may be made while the context's stream (or a stream it
// depends on) is being captured.
//
// All calls in a process share the one array, which keeps the contents of the
// last call; the status word is cleared at the start of every call. Calls that
// overlap on the GPU would race on the array: this entry point serialises its
// calls within the process with a mutex and waits for its own work before
// returning. Callers that bypass it must not run two calls at once on one
// device.
#include "context.cuh"
#include "trace.cuh"

#include <mutex>

namespace {

constexpr uint64_t kNoAllocMaxRays = 65536;
constexpr size_t kRayBytes = kNoAllocMaxRays * sizeof(alpine_gpu_ray);
constexpr size_t kHitBytes = kNoAllocMaxRays * sizeof(alpine_gpu_hit);
constexpr size_t kScratchBytes = kRayBytes + kHitBytes + 256;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mutex;                      // serialises calls (shared scratch)
void* g_scratch_addr[kMaxDevices] = {};  // device address of the array, per device

}  // namespace

static_assert(sizeof(alpine_gpu_ray) == 32 && sizeof(alpine_gpu_hit) == 16, "ABI record sizes");

extern "C" int alpine_gpu_trace_noalloc(alpine_gpu_ctx* c, const alpine_gpu_ray* rays, uint64_t n,
                                        alpine_gpu_hit* hits)
{
    if (!c) return ALPINE_GPU_ERR_INVALID_ARGUMENT;
    if (n && (!rays || !hits)) return c->fail(ALPINE_GPU_ERR_INVALID_ARGUMENT, "trace_noalloc: null buffer");
    if (n > kNoAllocMaxRays)
        return c->fail(ALPINE_GPU_ERR_INVALID_ARGUMENT,
                       "trace_noalloc: at most 65536 rays per call (the fixed staging array holds 65536)");
    if (c->bvhDirty) return c->fail(ALPINE_GPU_ERR_INVALID_STATE, "geometry changed since the last alpine_gpu_build");
    if (c->device < 0 || c->device >= kMaxDevices)
        return c->fail(ALPINE_GPU_ERR_INVALID_ARGUMENT, "trace_noalloc: device ordinal out of range");
    if (n == 0) return ALPINE_GPU_OK;

    std::lock_guard<std::mutex> lock(g_mutex);
    cudaError_t e = cudaSetDevice(c->device);
    if (e == cudaSuccess && !g_scratch_addr[c->device]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e == cudaSuccess) g_scratch_addr[c->device] = p;
    }
    if (e != cudaSuccess) {
        cudaGetLastError();
        return c->fail(ALPINE_GPU_ERR_CUDA, std::string("trace_noalloc: set-up: ") + cudaGetErrorString(e));
    }
    unsigned char* base = static_cast<unsigned char*>(g_scratch_addr[c->device]);
    void* dRays = base;
    void* dHits = base + kRayBytes;
    uint32_t* dStatus = reinterpret_cast<uint32_t*>(base + kRayBytes + kHitBytes);

    const ag::BvhView v = c->bvh_view();

    uint32_t status = 0;
    e = cudaMemsetAsync(dStatus, 0, sizeof(uint32_t), c->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dRays, rays, n * sizeof(alpine_gpu_ray), cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess) {
        ag::launch_trace(v, dRays, n, dHits, dStatus, c->stream);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(hits, dHits, n * sizeof(alpine_gpu_hit), cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&status, dStatus, sizeof(uint32_t), cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return c->fail(ALPINE_GPU_ERR_CUDA, std::string("trace_noalloc: ") + cudaGetErrorString(e));
    }
    if (status) return c->fail(ALPINE_GPU_ERR_LIMIT, "trace_noalloc: " + ag::status_msg(status));
    return ALPINE_GPU_OK;
}
