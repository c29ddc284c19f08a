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

// The same for 1-3 arrays of n = *count * mult elements each (count in
// device memory, read by the kernels), at most nCap, scanned by one set of
// launches. The launches depend on nCap only, so the call can be captured
// in a CUDA graph and replayed for other counts. total may be null, or hold
// null entries. scratch: scan3_scratch_words(nCap) words. expected: the
// count the caller expects (0 = nCap); it sizes the grids, which loop over
// the tiles, so any count up to nCap is still scanned.
size_t scan3_scratch_words(size_t nCap);
void exclusive_scan_count(int arrays, const uint32_t* const* in, uint32_t* const* out, const uint32_t* count,
                          uint32_t mult, size_t nCap, uint32_t* const* total, uint32_t* scratch, cudaStream_t stream,
                          size_t expected = 0);

}  // namespace ag
