// Deterministic device-wide exclusive prefix sum (reduce-then-scan).
#include "scan.cuh"

#include <algorithm>

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

// Element count of a scan launch: n, or (device-count scans) *count * mult
// clamped to the capacity n.
__device__ __forceinline__ size_t scan_count(size_t n, const uint32_t* count, uint32_t mult)
{
    if (!count) return n;
    const size_t c = size_t(*count) * mult;
    return c < n ? c : n;
}

// Up to three arrays scanned by the same launches: blockIdx.y selects one.
struct ScanArrays {
    const uint32_t* in[3];
    uint32_t* out[3];
    uint32_t* total[3];
};

// Tiles are processed in a loop over the grid (tile = blockIdx.x, +gridDim.x,
// ... below nb), so a grid smaller than nb tiles covers them all.
__global__ void k_tile_sums(ScanArrays a, size_t nCap, const uint32_t* __restrict__ count, uint32_t mult,
                            uint32_t* __restrict__ sums, size_t sumStride, size_t nb)
{
    const size_t n = scan_count(nCap, count, mult);
    const uint32_t* in = a.in[blockIdx.y];
    for (size_t tile = blockIdx.x; tile < nb; tile += gridDim.x) {
        if (tile * kTile >= n) {  // a tile past the count (device-count scans): its sum is 0
            if (threadIdx.x == 0) sums[blockIdx.y * sumStride + tile] = 0u;
            continue;
        }
        size_t base = tile * kTile + size_t(threadIdx.x) * kPerThread;
        uint32_t s = 0;
#pragma unroll
        for (int k = 0; k < kPerThread; ++k) {
            size_t i = base + k;
            if (i < n) s += in[i];
        }
        __shared__ uint32_t tot;
        block_excl_scan(s, &tot);
        if (threadIdx.x == 0) sums[blockIdx.y * sumStride + tile] = tot;
    }
}

__global__ void k_tile_scan(ScanArrays a, size_t nCap, const uint32_t* __restrict__ count, uint32_t mult,
                            const uint32_t* __restrict__ offsets, size_t offStride, size_t nb)
{
    const size_t n = scan_count(nCap, count, mult);
    const uint32_t* in = a.in[blockIdx.y];
    uint32_t* out = a.out[blockIdx.y];
    uint32_t* total = a.total[blockIdx.y];
    for (size_t tile = blockIdx.x; tile < nb; tile += gridDim.x) {
        const uint32_t off = offsets ? offsets[blockIdx.y * offStride + tile] : 0u;
        if (tile * kTile >= n) {  // a tile past the count: nothing to write but the total
            if (total && tile == nb - 1 && threadIdx.x == 0) *total = off;
            continue;
        }
        size_t base = tile * kTile + size_t(threadIdx.x) * kPerThread;
        uint32_t v[kPerThread];
        uint32_t s = 0;
#pragma unroll
        for (int k = 0; k < kPerThread; ++k) {
            size_t i = base + k;
            v[k] = i < n ? in[i] : 0u;
            s += v[k];
        }
        __shared__ uint32_t tot;
        uint32_t p = block_excl_scan(s, &tot) + off;
#pragma unroll
        for (int k = 0; k < kPerThread; ++k) {
            size_t i = base + k;
            if (i < n) out[i] = p;
            p += v[k];
        }
        if (total && tile == nb - 1 && threadIdx.x == blockDim.x - 1) *total = p;
    }
}

ScanArrays one_array(const uint32_t* in, uint32_t* out, uint32_t* total)
{
    return ScanArrays{{in, nullptr, nullptr}, {out, nullptr, nullptr}, {total, nullptr, nullptr}};
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
        k_tile_scan<<<1, kThreads, 0, stream>>>(one_array(in, out, total), n, nullptr, 1u, nullptr, 0, 1);
        return;
    }
    uint32_t* sums = scratch;
    k_tile_sums<<<(unsigned)nb, kThreads, 0, stream>>>(one_array(in, out, total), n, nullptr, 1u, sums, 0, nb);
    // Scan the tile sums in place (recursively), then the tiles with offsets.
    exclusive_scan(sums, sums, nb, nullptr, scratch + nb, stream);
    k_tile_scan<<<(unsigned)nb, kThreads, 0, stream>>>(one_array(in, out, total), n, nullptr, 1u, sums, 0, nb);
}

size_t scan3_scratch_words(size_t n)
{
    const size_t nb = (n + kTile - 1) / kTile;
    return 3 * nb + scan_scratch_words(nb);
}

void exclusive_scan_count(int arrays, const uint32_t* const* in, uint32_t* const* out, const uint32_t* count,
                          uint32_t mult, size_t nCap, uint32_t* const* total, uint32_t* scratch, cudaStream_t stream,
                          size_t expected)
{
    // Launch sizes follow the capacity only; tiles past the count see zeros,
    // so the tile sums, their scan and the totals are those of the count.
    ScanArrays a{};
    for (int y = 0; y < arrays; ++y) {
        a.in[y] = in[y];
        a.out[y] = out[y];
        a.total[y] = total ? total[y] : nullptr;
    }
    if (nCap == 0) {
        for (int y = 0; y < arrays; ++y)
            if (a.total[y]) cudaMemsetAsync(a.total[y], 0, sizeof(uint32_t), stream);
        return;
    }
    const size_t nb = (nCap + kTile - 1) / kTile;
    // blocks per array: the tiles of the expected count (a loop covers more)
    size_t gb = expected ? (std::min(expected, nCap) + kTile - 1) / kTile : nb;
    gb = gb < 1 ? 1 : (gb > nb ? nb : gb);
    const dim3 one(1, (unsigned)arrays), grid((unsigned)gb, (unsigned)arrays);
    if (nb == 1) {
        k_tile_scan<<<one, kThreads, 0, stream>>>(a, nCap, count, mult, nullptr, 0, 1);
        return;
    }
    uint32_t* sums = scratch;  // arrays x nb tile sums
    k_tile_sums<<<grid, kThreads, 0, stream>>>(a, nCap, count, mult, sums, nb, nb);
    if (nb <= kTile) {  // every array's tile sums in one tile: one launch scans them all
        ScanArrays t{};
        for (int y = 0; y < arrays; ++y) t.in[y] = t.out[y] = sums + y * nb;
        k_tile_scan<<<one, kThreads, 0, stream>>>(t, nb, nullptr, 1u, nullptr, 0, 1);
    } else {
        for (int y = 0; y < arrays; ++y)
            exclusive_scan(sums + y * nb, sums + y * nb, nb, nullptr, scratch + 3 * nb, stream);
    }
    k_tile_scan<<<grid, kThreads, 0, stream>>>(a, nCap, count, mult, sums, nb, nb);
}

}  // namespace ag
