// Batched closest-hit / any-hit queries over device ray buffers.
#include "trace.cuh"
#include "traverse.cuh"

namespace ag {
namespace {

template <bool kAny, bool kBinary>
__global__ void __launch_bounds__(kTraceBlock) k_trace(BvhView bvh, const float4* __restrict__ rays, uint32_t n,
                                                       void* __restrict__ out, uint32_t* __restrict__ status)
{
    __shared__ uint2 stack[kTraversalStack * kTraceBlock];
    uint32_t i = blockIdx.x * kTraceBlock + threadIdx.x;
    if (i >= n) return;
    // rays and results stream through once: evict-first hints keep the BVH in L2
    float4 a = __ldcs(rays + 2ull * i);
    float4 b = __ldcs(rays + 2ull * i + 1);
    TraceResult r;
    uint32_t err = 0, nv = 0, tv = 0;
    bool hit = trace<kAny, kBinary>(bvh, mk3(a.x, a.y, a.z), mk3(b.x, b.y, b.z), a.w, b.w, r, stack + threadIdx.x,
                                    kTraceBlock, err, nv, tv);
    if (kAny) {
        __stcs(static_cast<uint8_t*>(out) + i, (uint8_t)(hit ? 1 : 0));
    } else {
        __stcs(static_cast<uint4*>(out) + i,
               make_uint4(r.prim, __float_as_uint(r.t), __float_as_uint(r.b1), __float_as_uint(r.b2)));
    }
    if (err) atomicOr(status, err);
}

// Instrumented variant: same traversal, accumulates node / triangle visits.
template <bool kAny, bool kBinary>
__global__ void __launch_bounds__(kTraceBlock) k_trace_count(BvhView bvh, const float4* __restrict__ rays, uint32_t n,
                                                             unsigned long long* __restrict__ counts,
                                                             uint32_t* __restrict__ status)
{
    __shared__ uint2 stack[kTraversalStack * kTraceBlock];
    uint32_t i = blockIdx.x * kTraceBlock + threadIdx.x;
    uint32_t nv = 0, tv = 0, err = 0;
    if (i < n) {
        float4 a = rays[2ull * i], b = rays[2ull * i + 1];
        TraceResult r;
        trace<kAny, kBinary>(bvh, mk3(a.x, a.y, a.z), mk3(b.x, b.y, b.z), a.w, b.w, r, stack + threadIdx.x,
                             kTraceBlock, err, nv, tv);
    }
    unsigned long long snv = nv, stv = tv;
#pragma unroll
    for (int o = 16; o; o >>= 1) {
        snv += __shfl_xor_sync(0xffffffffu, snv, o);
        stv += __shfl_xor_sync(0xffffffffu, stv, o);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(counts, snv);
        atomicAdd(counts + 1, stv);
    }
    if (err) atomicOr(status, err);
}

// Variant whose ray count is read from device memory (wavefront queues),
// with the block size as a parameter (chosen by the autotuner).
template <bool kAny, int kBlock, bool kBinary>
__global__ void __launch_bounds__(kBlock) k_trace_dyn(BvhView bvh, const float4* __restrict__ rays,
                                                      const uint32_t* __restrict__ count, uint32_t cap,
                                                      void* __restrict__ out, uint32_t* __restrict__ status)
{
    static_assert(kTraversalStack * kBlock * sizeof(uint2) <= 48 * 1024, "static shared memory");
    __shared__ uint2 stack[kTraversalStack * kBlock];
    // the grid covers the queue's capacity: one ray per thread (a count above
    // the capacity would be a queue overflow upstream: reported, and no ray
    // beyond the capacity is read)
    const uint32_t n = *count;
    const uint32_t i = blockIdx.x * kBlock + threadIdx.x;
    if (i == 0 && n > cap) atomicOr(status, kErrQueueOverflow);
    if (i >= n || i >= cap) return;
    float4 a = rays[2ull * i];
    float4 b = rays[2ull * i + 1];
    TraceResult r;
    uint32_t err = 0, nv = 0, tv = 0;
    bool hit = trace<kAny, kBinary>(bvh, mk3(a.x, a.y, a.z), mk3(b.x, b.y, b.z), a.w, b.w, r, stack + threadIdx.x,
                                    kBlock, err, nv, tv);
    if (kAny) static_cast<uint8_t*>(out)[i] = hit ? 1 : 0;
    else static_cast<uint4*>(out)[i] = make_uint4(r.prim, __float_as_uint(r.t), __float_as_uint(r.b1), __float_as_uint(r.b2));
    if (err) atomicOr(status, err);
}

template <bool kAny>
void launch(const BvhView& bvh, const void* rays, uint64_t n, void* out, uint32_t* status, cudaStream_t st)
{
    const uint64_t kMaxPerLaunch = 1ull << 30;
    for (uint64_t s = 0; s < n; s += kMaxPerLaunch) {
        uint32_t m = (uint32_t)(n - s < kMaxPerLaunch ? n - s : kMaxPerLaunch);
        const float4* r = static_cast<const float4*>(rays) + 2 * s;
        void* o = kAny ? static_cast<void*>(static_cast<uint8_t*>(out) + s)
                       : static_cast<void*>(static_cast<uint4*>(out) + s);
        unsigned blocks = (m + kTraceBlock - 1) / kTraceBlock;
        if (bvh.triTest == kTriTestBinary) k_trace<kAny, true><<<blocks, kTraceBlock, 0, st>>>(bvh, r, m, o, status);
        else k_trace<kAny, false><<<blocks, kTraceBlock, 0, st>>>(bvh, r, m, o, status);
    }
}
}  // namespace

namespace {
template <int kBlock>
void launch_dyn(const BvhView& bvh, const float4* r, const uint32_t* count, uint32_t maxCount, bool any, void* out,
                uint32_t* status, cudaStream_t st)
{
    const unsigned blocks = (maxCount + kBlock - 1) / kBlock;
    const bool bin = bvh.triTest == kTriTestBinary;
    if (any && bin) k_trace_dyn<true, kBlock, true><<<blocks, kBlock, 0, st>>>(bvh, r, count, maxCount, out, status);
    else if (any) k_trace_dyn<true, kBlock, false><<<blocks, kBlock, 0, st>>>(bvh, r, count, maxCount, out, status);
    else if (bin) k_trace_dyn<false, kBlock, true><<<blocks, kBlock, 0, st>>>(bvh, r, count, maxCount, out, status);
    else k_trace_dyn<false, kBlock, false><<<blocks, kBlock, 0, st>>>(bvh, r, count, maxCount, out, status);
}
}  // namespace

void launch_trace_dyn(const BvhView& bvh, const void* rays, const uint32_t* count, uint32_t maxCount, bool any,
                      void* out, uint32_t* status, cudaStream_t st, int block)
{
    if (maxCount == 0) return;
    const float4* r = static_cast<const float4*>(rays);
    if (block == 64) launch_dyn<64>(bvh, r, count, maxCount, any, out, status, st);
    else if (block == 256) launch_dyn<256>(bvh, r, count, maxCount, any, out, status, st);
    else launch_dyn<128>(bvh, r, count, maxCount, any, out, status, st);
}

void launch_trace_count(const BvhView& bvh, const void* rays, uint64_t n, bool any, unsigned long long* counts,
                        uint32_t* status, cudaStream_t st)
{
    const uint64_t kMaxPerLaunch = 1ull << 30;
    for (uint64_t s = 0; s < n; s += kMaxPerLaunch) {
        uint32_t m = (uint32_t)(n - s < kMaxPerLaunch ? n - s : kMaxPerLaunch);
        const float4* r = static_cast<const float4*>(rays) + 2 * s;
        unsigned blocks = (m + kTraceBlock - 1) / kTraceBlock;
        const bool bin = bvh.triTest == kTriTestBinary;
        if (any && bin) k_trace_count<true, true><<<blocks, kTraceBlock, 0, st>>>(bvh, r, m, counts, status);
        else if (any) k_trace_count<true, false><<<blocks, kTraceBlock, 0, st>>>(bvh, r, m, counts, status);
        else if (bin) k_trace_count<false, true><<<blocks, kTraceBlock, 0, st>>>(bvh, r, m, counts, status);
        else k_trace_count<false, false><<<blocks, kTraceBlock, 0, st>>>(bvh, r, m, counts, status);
    }
}

void launch_trace(const BvhView& bvh, const void* rays, uint64_t n, void* hits, uint32_t* status, cudaStream_t st)
{
    launch<false>(bvh, rays, n, hits, status, st);
}

void launch_occluded(const BvhView& bvh, const void* rays, uint64_t n, uint8_t* occ, uint32_t* status,
                     cudaStream_t st)
{
    launch<true>(bvh, rays, n, occ, status, st);
}

}  // namespace ag
