// Launchers for batched ray queries (rays: 32-byte alpine_gpu_ray records).
#pragma once

#include "bvh.cuh"

namespace ag {

#ifndef AG_TRACE_BLOCK
#define AG_TRACE_BLOCK 128
#endif
constexpr int kTraceBlock = AG_TRACE_BLOCK;

// hits: 16-byte {prim, t, b1, b2} records. status: device word receiving
// DeviceError bits (ORed).
void launch_trace(const BvhView& bvh, const void* rays, uint64_t n, void* hits, uint32_t* status, cudaStream_t st);
void launch_occluded(const BvhView& bvh, const void* rays, uint64_t n, uint8_t* occ, uint32_t* status,
                     cudaStream_t st);

// Queue variant: the number of rays is *count (device memory, read by the
// kernel), at most maxCount. any selects any-hit (uint8 results) or closest.
// block: threads per block, 64, 128 or 256.
void launch_trace_dyn(const BvhView& bvh, const void* rays, const uint32_t* count, uint32_t maxCount, bool any,
                      void* out, uint32_t* status, cudaStream_t st, int block = kTraceBlock);

// Instrumented traversal: counts[0] += wide nodes fetched, counts[1] += triangles tested.
void launch_trace_count(const BvhView& bvh, const void* rays, uint64_t n, bool any, unsigned long long* counts,
                        uint32_t* status, cudaStream_t st);

}  // namespace ag
