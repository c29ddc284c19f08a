// Device-wide exclusive prefix sum of uint32 (reduce-then-scan), deterministic.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace ag {

// Scratch words needed by exclusive_scan for n elements.
size_t scan_scratch_words(size_t n);

// out[i] = sum(in[0..i)); optionally *total (device pointer) = sum(in[0..n)).
// in and out may alias. scratch: scan_scratch_words(n) uint32 words.
void exclusive_scan(const uint32_t* in, uint32_t* out, size_t n, uint32_t* total, uint32_t* scratch,
                    cudaStream_t stream);

}  // namespace ag
