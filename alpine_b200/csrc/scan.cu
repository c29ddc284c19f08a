// Deterministic device-wide exclusive prefix sum (reduce-then-scan).
#include "scan.cuh"

namespace ag {
namespace {
constexpr int kThreads = 1024;
constexpr int kPerThread = 4;
constexpr size_t kTile = size_t(kThreads) * kPerThread;

__device__ __forceinline__ uint32_t warp_incl_scan(uint32_t v)
{
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(0xffffffffu, v, o);
        if ((threadIdx.x & 31) >= (unsigned)o) v += y;
    }
    return v;
}

// Block-wide exclusive scan of one value per thread; returns the exclusive
// prefix and writes the block total to *total.
__device__ __forceinline__ uint32_t block_excl_scan(uint32_t v, uint32_t* total)
{
    __shared__ uint32_t warpSums[32];
    uint32_t inc = warp_incl_scan(v);
    int w = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 31) warpSums[w] = inc;
    __syncthreads();
    if (w == 0) {
        uint32_t s = (threadIdx.x < blockDim.x / 32) ? warpSums[threadIdx.x] : 0u;
        uint32_t si = warp_incl_scan(s);
        warpSums[threadIdx.x] = si - s;
        if (threadIdx.x == 31) *total = si;
    }
    __syncthreads();
    uint32_t r = warpSums[w] + inc - v;
    __syncthreads();
    return r;
}

__global__ void k_tile_sums(const uint32_t* __restrict__ in, size_t n, uint32_t* __restrict__ sums)
{
    size_t base = size_t(blockIdx.x) * kTile + size_t(threadIdx.x) * kPerThread;
    uint32_t s = 0;
#pragma unroll
    for (int k = 0; k < kPerThread; ++k) {
        size_t i = base + k;
        if (i < n) s += in[i];
    }
    __shared__ uint32_t tot;
    block_excl_scan(s, &tot);
    if (threadIdx.x == 0) sums[blockIdx.x] = tot;
}

__global__ void k_tile_scan(const uint32_t* in, uint32_t* out, size_t n, const uint32_t* __restrict__ offsets,
                            uint32_t* total)
{
    size_t base = size_t(blockIdx.x) * kTile + size_t(threadIdx.x) * kPerThread;
    uint32_t v[kPerThread];
    uint32_t s = 0;
#pragma unroll
    for (int k = 0; k < kPerThread; ++k) {
        size_t i = base + k;
        v[k] = i < n ? in[i] : 0u;
        s += v[k];
    }
    __shared__ uint32_t tot;
    uint32_t p = block_excl_scan(s, &tot) + (offsets ? offsets[blockIdx.x] : 0u);
#pragma unroll
    for (int k = 0; k < kPerThread; ++k) {
        size_t i = base + k;
        if (i < n) out[i] = p;
        p += v[k];
    }
    if (total && blockIdx.x == gridDim.x - 1 && threadIdx.x == blockDim.x - 1) *total = p;
}
}  // namespace

size_t scan_scratch_words(size_t n)
{
    size_t w = 0;
    while (n > kTile) {
        n = (n + kTile - 1) / kTile;
        w += n;
    }
    return w + 1;
}

void exclusive_scan(const uint32_t* in, uint32_t* out, size_t n, uint32_t* total, uint32_t* scratch,
                    cudaStream_t stream)
{
    if (n == 0) {
        if (total) cudaMemsetAsync(total, 0, sizeof(uint32_t), stream);
        return;
    }
    size_t nb = (n + kTile - 1) / kTile;
    if (nb == 1) {
        k_tile_scan<<<1, kThreads, 0, stream>>>(in, out, n, nullptr, total);
        return;
    }
    uint32_t* sums = scratch;
    k_tile_sums<<<(unsigned)nb, kThreads, 0, stream>>>(in, n, sums);
    // Scan the tile sums in place (recursively), then the tiles with offsets.
    exclusive_scan(sums, sums, nb, nullptr, scratch + nb, stream);
    k_tile_scan<<<(unsigned)nb, kThreads, 0, stream>>>(in, out, n, sums, total);
}

}  // namespace ag
