// GPU BVH builder (see build.cuh).
//
// Binary phase: level-synchronous top-down binned SAH over primitive
// references. Every level processes all active tasks (node ranges) at once:
//   * big tasks (> kSmallMax references) are binned by blocks of kChunk
//     references with shared-memory bins merged into per-task global bins,
//     split by one warp per task, and partitioned stably by chunk;
//   * small tasks are binned, split and partitioned by one warp each with
//     warp-private shared-memory bins.
// Children are compacted in a deterministic order with prefix sums, so a build
// is a pure function of its input (the float min/max merges and integer counts
// are order independent).
//
// Wide phase: breadth-first collapse to 8 slots, quantised child boxes,
// octant-ordered slots, triangle records in leaf order
// (src/accelerators/wide_bvh.cpp:430-472 packs TriangleN likewise). Which
// binary nodes fill a wide node's slots is chosen either
//   * SAH-optimally (the default): a bottom-up dynamic program over the
//     binary tree gives every node its least SAH cost when it may occupy
//     1..8 slots of its parent (the method of Ylitie, Karras and Laine,
//     "Efficient Incoherent Ray Traversal on GPUs Through Compressed Wide
//     BVHs", HPG 2017, restated for leaves of at most 3 triangles), and the
//     collapse follows its choices; or
//   * greedily, as the reference does (src/accelerators/wide_bvh.cpp:200-243):
//     open the internal child of largest surface area until 8 slots are used.
#include "build.cuh"
#include "scan.cuh"

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdio>
#include <cstring>

namespace ag {
namespace {

constexpr uint32_t kSmallMax = 512;  // tasks up to this size are handled by one warp
constexpr uint32_t kChunk = 1024;    // references per block for big tasks
constexpr int kChunkThreads = 256;   // kChunk / 4
constexpr int kBinWords = 13;        // lo3 hi3 clo3 chi3 count
constexpr int kAxisBinWords = kSahBins * kBinWords;
constexpr int kTaskBinWords = 3 * kAxisBinWords;
constexpr int kSmallWarps = 4;       // warps per block in the small-task kernel
constexpr uint32_t kMaxLevels = 1024;

struct alignas(16) Task {
    float clo[3];
    uint32_t node;
    float chi[3];
    uint32_t begin;
    uint32_t count;
    uint32_t pad[3];
};

struct alignas(16) Cand {
    float lo[3];
    uint32_t begin;
    float hi[3];
    uint32_t count;
    float clo[3];
    uint32_t big;    // 1 when count > kSmallMax
    float chi[3];
    uint32_t chunks; // ceil(count / kChunk) for big candidates, else 0
};

struct BigSplit {
    int axis;
    int bin;
    int mode;  // 0 = SAH bin split, 1 = median (all centroids coincide)
    uint32_t nL;
};

enum Counter { kCntTasks = 0, kCntBig, kCntChunks, kCntInt, kCntTri, kCntSlots, kCntBounds = 8, kCntWords = 32 };

// Device-driven build (Builder::enqueue): the state the host loop keeps,
// held in counter words instead, so that no kernel needs a host value.
enum DevCounter {
    kDevTasks = 20,  // tasks of the current binary level
    kDevBig,         // big tasks of the current level
    kDevChunks,      // chunks of the big tasks
    kDevNodes,       // binary nodes so far (first id of the next level)
    kDevLevels,      // binary levels that had tasks
    kDevItems,       // wide nodes of the current collapse level
    kDevWide,        // wide nodes so far
    kDevTris,        // triangle records placed so far
    kDevDepth,       // collapse levels that had items
    kDevRootAreaInv, // float bits: 1 / half-area of the root box
    kDevFailed,      // nonzero: the binary phase met a task it could not split (the build stops)
};
static_assert((int)kDevFailed < (int)kCntWords, "counter words");

// Work-item count of a level kernel: the host's count, or, in a
// device-driven build, mult times the count a previous kernel left in
// device memory.
AG_D uint32_t level_count(const uint32_t* dn, uint32_t n, uint32_t mult = 1u) { return dn ? *dn * mult : n; }

// --------------------------------------------------------------------------
// Binning arithmetic. Every kernel must compute identical bin indices, so all
// float operations are explicitly rounded (no contraction into FMA).
AG_D float centroid(float lo, float hi) { return __fmul_rn(0.5f, __fadd_rn(lo, hi)); }
AG_D float axis_scale(float clo, float chi)
{
    float e = __fsub_rn(chi, clo);
    return e > 0.0f ? __fdiv_rn(float(kSahBins), e) : 0.0f;
}
AG_D int bin_of(float c, float clo, float scale)
{
    int b = __float2int_rz(__fmul_rn(__fsub_rn(c, clo), scale));
    return min(max(b, 0), kSahBins - 1);
}

AG_D void bin_init_word(uint32_t* w, int k)
{
    int f = k % kBinWords;
    // min words (lo, clo) start at the largest key, max words (hi, chi) at 0.
    *w = (f < 3 || (f >= 6 && f < 9)) ? 0xffffffffu : 0u;
}

AG_D float area_of(float lx, float ly, float lz, float hx, float hy, float hz)
{
    float ex = hx - lx, ey = hy - ly, ez = hz - lz;
    return ex * ey + ey * ez + ez * ex;
}

// Inclusive warp scans for union-of-boxes and counts.
template <bool kForward>
AG_D float scan_min(float v)
{
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        float y = kForward ? __shfl_up_sync(0xffffffffu, v, o) : __shfl_down_sync(0xffffffffu, v, o);
        bool ok = kForward ? (lane_id() >= (uint32_t)o) : (lane_id() + o < 32);
        if (ok) v = fminf(v, y);
    }
    return v;
}
template <bool kForward>
AG_D float scan_max(float v)
{
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        float y = kForward ? __shfl_up_sync(0xffffffffu, v, o) : __shfl_down_sync(0xffffffffu, v, o);
        bool ok = kForward ? (lane_id() >= (uint32_t)o) : (lane_id() + o < 32);
        if (ok) v = fmaxf(v, y);
    }
    return v;
}
template <bool kForward>
AG_D uint32_t scan_add(uint32_t v)
{
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = kForward ? __shfl_up_sync(0xffffffffu, v, o) : __shfl_down_sync(0xffffffffu, v, o);
        bool ok = kForward ? (lane_id() >= (uint32_t)o) : (lane_id() + o < 32);
        if (ok) v += y;
    }
    return v;
}

AG_D float warp_min(float v)
{
#pragma unroll
    for (int o = 16; o; o >>= 1) v = fminf(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}
AG_D float warp_max(float v)
{
#pragma unroll
    for (int o = 16; o; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// Result of a warp-wide split search over the bins of one task.
struct SplitChoice {
    float cost;
    int axis;
    int bin;
    uint32_t nL;
    float L[12];  // lo3 hi3 clo3 chi3 of the left child
    float R[12];
};

// Evaluate all 31 split planes of one axis from bins held one per lane
// (lane = bin). `v` holds the lane's bin: lo3 hi3 clo3 chi3 as floats (empty
// bins: lo = +FLT_MAX, hi = -FLT_MAX) and `cnt`. Updates `best` when a cheaper
// split is found (ties keep the earlier axis / lower bin).
AG_D void eval_axis(int axis, const float v[12], uint32_t cnt, bool withCentroids, SplitChoice& best)
{
    float Lv[12], Rv[12];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        Lv[k] = scan_min<true>(v[k]);
        Lv[3 + k] = scan_max<true>(v[3 + k]);
        Rv[k] = scan_min<false>(v[k]);
        Rv[3 + k] = scan_max<false>(v[3 + k]);
    }
    if (withCentroids) {
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            Lv[6 + k] = scan_min<true>(v[6 + k]);
            Lv[9 + k] = scan_max<true>(v[9 + k]);
            Rv[6 + k] = scan_min<false>(v[6 + k]);
            Rv[9 + k] = scan_max<false>(v[9 + k]);
        }
    }
    uint32_t cL = scan_add<true>(cnt);
    uint32_t cR = scan_add<false>(cnt);
    // right side of the plane after bin k is bins k+1..31
    float Rn[12];
#pragma unroll
    for (int k = 0; k < 12; ++k) Rn[k] = __shfl_down_sync(0xffffffffu, Rv[k], 1);
    uint32_t cRn = __shfl_down_sync(0xffffffffu, cR, 1);
    bool valid = lane_id() < 31 && cL > 0 && cRn > 0;
    float cost = FLT_MAX;
    if (valid) {
        cost = float(cL) * area_of(Lv[0], Lv[1], Lv[2], Lv[3], Lv[4], Lv[5]) +
               float(cRn) * area_of(Rn[0], Rn[1], Rn[2], Rn[3], Rn[4], Rn[5]);
    }
    // warp argmin (cost, then lowest lane)
    float bc = cost;
    int bl = (int)lane_id();
#pragma unroll
    for (int o = 16; o; o >>= 1) {
        float oc = __shfl_xor_sync(0xffffffffu, bc, o);
        int ol = __shfl_xor_sync(0xffffffffu, bl, o);
        if (oc < bc || (oc == bc && ol < bl)) { bc = oc; bl = ol; }
    }
    if (bc < best.cost) {
        best.cost = bc;
        best.axis = axis;
        best.bin = bl;
        best.nL = __shfl_sync(0xffffffffu, cL, bl);
#pragma unroll
        for (int k = 0; k < 12; ++k) {
            best.L[k] = __shfl_sync(0xffffffffu, Lv[k], bl);
            best.R[k] = __shfl_sync(0xffffffffu, Rn[k], bl);
        }
    }
}

AG_D void load_bin(const uint32_t* b, float v[12], uint32_t& cnt)
{
    cnt = b[12];
#pragma unroll
    for (int k = 0; k < 12; ++k) {
        bool isMin = (k < 3) || (k >= 6 && k < 9);
        v[k] = cnt ? ord2f(b[k]) : (isMin ? FLT_MAX : -FLT_MAX);
    }
}

AG_D void bin_accumulate(uint32_t* bin, float4 lo, float4 hi, float cx, float cy, float cz)
{
    atomicMin(bin + 0, f2ord(lo.x));
    atomicMin(bin + 1, f2ord(lo.y));
    atomicMin(bin + 2, f2ord(lo.z));
    atomicMax(bin + 3, f2ord(hi.x));
    atomicMax(bin + 4, f2ord(hi.y));
    atomicMax(bin + 5, f2ord(hi.z));
    atomicMin(bin + 6, f2ord(cx));
    atomicMin(bin + 7, f2ord(cy));
    atomicMin(bin + 8, f2ord(cz));
    atomicMax(bin + 9, f2ord(cx));
    atomicMax(bin + 10, f2ord(cy));
    atomicMax(bin + 11, f2ord(cz));
    atomicAdd(bin + 12, 1u);
}

AG_D void write_cand(Cand* c, const float* b, uint32_t begin, uint32_t count)
{
    Cand o;
    o.lo[0] = b[0]; o.lo[1] = b[1]; o.lo[2] = b[2];
    o.hi[0] = b[3]; o.hi[1] = b[4]; o.hi[2] = b[5];
    o.clo[0] = b[6]; o.clo[1] = b[7]; o.clo[2] = b[8];
    o.chi[0] = b[9]; o.chi[1] = b[10]; o.chi[2] = b[11];
    o.begin = begin;
    o.count = count;
    o.big = count > kSmallMax ? 1u : 0u;
    o.chunks = o.big ? (count + kChunk - 1) / kChunk : 0u;
    *c = o;
}

// --------------------------------------------------------------------------
// Preparation: primitive boxes and root bounds.
// Primitives 0 .. ntris-1 are triangles, ntris .. n-1 spheres (centre +
// radius): their box is centre -+ radius.
__global__ void k_prep_prims(const float* __restrict__ verts, const uint32_t* __restrict__ idx, uint32_t ntris,
                             const float4* __restrict__ spheres, uint32_t n, float4* __restrict__ primLo,
                             float4* __restrict__ primHi, uint32_t* __restrict__ refs, uint32_t* __restrict__ bounds)
{
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    float lo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, hi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
    float c[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, cmx[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
    if (i < n) {
        float l[3], h[3];
        if (i < ntris) {
            const uint32_t* t = idx + 3ull * i;
            float p[3][3];
#pragma unroll
            for (int v = 0; v < 3; ++v)
#pragma unroll
                for (int k = 0; k < 3; ++k) p[v][k] = verts[3ull * t[v] + k];
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                l[k] = fminf(fminf(p[0][k], p[1][k]), p[2][k]);
                h[k] = fmaxf(fmaxf(p[0][k], p[1][k]), p[2][k]);
            }
        } else {
            const float4 sp = spheres[i - ntris];
            const float r = fabsf(sp.w);
            l[0] = __fsub_rd(sp.x, r); l[1] = __fsub_rd(sp.y, r); l[2] = __fsub_rd(sp.z, r);
            h[0] = __fadd_ru(sp.x, r); h[1] = __fadd_ru(sp.y, r); h[2] = __fadd_ru(sp.z, r);
        }
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            lo[k] = l[k];
            hi[k] = h[k];
            c[k] = cmx[k] = centroid(l[k], h[k]);
        }
        primLo[i] = make_float4(l[0], l[1], l[2], 0.0f);
        primHi[i] = make_float4(h[0], h[1], h[2], 0.0f);
        refs[i] = i;
    }
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        lo[k] = warp_min(lo[k]);
        hi[k] = warp_max(hi[k]);
        c[k] = warp_min(c[k]);
        cmx[k] = warp_max(cmx[k]);
    }
    if (lane_id() == 0) {
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            atomicMin(bounds + k, f2ord(lo[k]));
            atomicMax(bounds + 3 + k, f2ord(hi[k]));
            atomicMin(bounds + 6 + k, f2ord(c[k]));
            atomicMax(bounds + 9 + k, f2ord(cmx[k]));
        }
    }
}

__global__ void k_init_bounds(uint32_t* bounds)
{
    int k = threadIdx.x;
    if (k < 12) bounds[k] = (k < 3 || (k >= 6 && k < 9)) ? 0xffffffffu : 0u;
}

__global__ void k_root(uint32_t n, const uint32_t* __restrict__ bounds, Task* tasks, BinNode* bnodes,
                       uint32_t* bigList, uint32_t* chunkOff, uint32_t* chunkTask, uint32_t nChunks)
{
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i == 0) {
        Task t;
        for (int k = 0; k < 3; ++k) {
            t.clo[k] = ord2f(bounds[6 + k]);
            t.chi[k] = ord2f(bounds[9 + k]);
        }
        t.node = 0;
        t.begin = 0;
        t.count = n;
        tasks[0] = t;
        BinNode b;
        b.lo = mk3(ord2f(bounds[0]), ord2f(bounds[1]), ord2f(bounds[2]));
        b.hi = mk3(ord2f(bounds[3]), ord2f(bounds[4]), ord2f(bounds[5]));
        b.begin = 0;
        b.count = n;
        b.left = -1;
        b.right = -1;
        bnodes[0] = b;
        bigList[0] = 0;
        chunkOff[0] = 0;
    }
    if (i < nChunks) chunkTask[i] = 0;
}

// --------------------------------------------------------------------------
// Big tasks.
__global__ void k_bins_clear(uint32_t* bins, uint32_t numBig, const uint32_t* dBig)
{
    const uint32_t nb = level_count(dBig, numBig);
    for (uint32_t bi = blockIdx.x; bi < nb; bi += gridDim.x) {
        uint32_t* b = bins + size_t(bi) * kTaskBinWords;
        for (int k = threadIdx.x; k < kTaskBinWords; k += blockDim.x) bin_init_word(b + k, k);
    }
}

struct ChunkRange {
    uint32_t bi, t, begin, end, local;
};

AG_D ChunkRange chunk_range(uint32_t c, const Task* tasks, const uint32_t* bigList, const uint32_t* chunkOff,
                            const uint32_t* chunkTask, Task& task)
{
    ChunkRange r;
    r.bi = chunkTask[c];
    r.t = bigList[r.bi];
    task = tasks[r.t];
    r.local = c - chunkOff[r.bi];
    r.begin = task.begin + r.local * kChunk;
    r.end = min(task.begin + task.count, r.begin + kChunk);
    return r;
}

__global__ void __launch_bounds__(kChunkThreads) k_bin_big(const Task* __restrict__ tasks, const uint32_t* __restrict__ refs,
                                                           const float4* __restrict__ primLo, const float4* __restrict__ primHi,
                                                           const uint32_t* __restrict__ bigList, const uint32_t* __restrict__ chunkOff,
                                                           const uint32_t* __restrict__ chunkTask, uint32_t* __restrict__ bigBins,
                                                           uint32_t numChunks, const uint32_t* __restrict__ dChunks)
{
    __shared__ uint32_t sb[kTaskBinWords];
    const uint32_t nc = level_count(dChunks, numChunks);
    for (uint32_t cb = blockIdx.x; cb < nc; cb += gridDim.x) {
        for (int k = threadIdx.x; k < kTaskBinWords; k += blockDim.x) bin_init_word(sb + k, k);
        __syncthreads();
        Task task;
        ChunkRange r = chunk_range(cb, tasks, bigList, chunkOff, chunkTask, task);
        float sc[3];
#pragma unroll
        for (int a = 0; a < 3; ++a) sc[a] = axis_scale(task.clo[a], task.chi[a]);
        for (uint32_t i = r.begin + threadIdx.x; i < r.end; i += blockDim.x) {
            uint32_t p = refs[i];
            float4 lo = primLo[p], hi = primHi[p];
            float cx = centroid(lo.x, hi.x), cy = centroid(lo.y, hi.y), cz = centroid(lo.z, hi.z);
            float cc[3] = {cx, cy, cz};
#pragma unroll
            for (int a = 0; a < 3; ++a) {
                if (sc[a] == 0.0f) continue;
                int b = bin_of(cc[a], task.clo[a], sc[a]);
                bin_accumulate(sb + a * kAxisBinWords + b * kBinWords, lo, hi, cx, cy, cz);
            }
        }
        __syncthreads();
        uint32_t* g = bigBins + size_t(r.bi) * kTaskBinWords;
        for (int k = threadIdx.x; k < kTaskBinWords; k += blockDim.x) {
            int binBase = k - k % kBinWords;
            if (sb[binBase + 12] == 0) continue;  // empty bin: nothing to merge
            int f = k % kBinWords;
            if (f == 12) atomicAdd(g + k, sb[k]);
            else if (f < 3 || (f >= 6 && f < 9)) atomicMin(g + k, sb[k]);
            else atomicMax(g + k, sb[k]);
        }
        __syncthreads();  // sb is cleared again for the next chunk
    }
}

__global__ void k_split_big(const Task* __restrict__ tasks, const uint32_t* __restrict__ bigList,
                            const uint32_t* __restrict__ bigBins, BigSplit* __restrict__ splits,
                            Cand* __restrict__ cands, uint32_t* __restrict__ candFlag, uint32_t numBig,
                            const uint32_t* __restrict__ dBig)
{
    const uint32_t nb = level_count(dBig, numBig);
    for (uint32_t bi = blockIdx.x; bi < nb; bi += gridDim.x) {
        uint32_t t = bigList[bi];
        Task task = tasks[t];
        SplitChoice best;
        best.cost = FLT_MAX;
        best.axis = -1;
        best.bin = 0;
        best.nL = 0;
        for (int a = 0; a < 3; ++a) {
            if (axis_scale(task.clo[a], task.chi[a]) == 0.0f) continue;
            float v[12];
            uint32_t cnt;
            load_bin(bigBins + size_t(bi) * kTaskBinWords + a * kAxisBinWords + lane_id() * kBinWords, v, cnt);
            eval_axis(a, v, cnt, true, best);
        }
        if (lane_id() == 0) {
            BigSplit s;
            if (best.axis >= 0) {
                s.axis = best.axis;
                s.bin = best.bin;
                s.mode = 0;
                s.nL = best.nL;
                write_cand(cands + 2 * t, best.L, task.begin, best.nL);
                write_cand(cands + 2 * t + 1, best.R, task.begin + best.nL, task.count - best.nL);
            } else {
                // All centroids coincide: split by position. The children inherit
                // the parent's node box (a NaN in lo marks this for k_compact) and
                // its point-sized centroid box.
                float pb[12];
                const float nan = __uint_as_float(0x7fc00000u);
                for (int k = 0; k < 3; ++k) {
                    pb[k] = nan;
                    pb[3 + k] = nan;
                    pb[6 + k] = task.clo[k];
                    pb[9 + k] = task.chi[k];
                }
                s.axis = 0;
                s.bin = 0;
                s.mode = 1;
                s.nL = task.count / 2;
                write_cand(cands + 2 * t, pb, task.begin, s.nL);
                write_cand(cands + 2 * t + 1, pb, task.begin + s.nL, task.count - s.nL);
            }
            splits[bi] = s;
            candFlag[2 * t] = 1;
            candFlag[2 * t + 1] = 1;
        }
    }
}

AG_D bool goes_left(const BigSplit& s, const Task& task, uint32_t i, uint32_t p, const float4* primLo,
                    const float4* primHi)
{
    if (s.mode == 1) return (i - task.begin) < s.nL;
    float lo = comp(make_float3(primLo[p].x, primLo[p].y, primLo[p].z), s.axis);
    float hi = comp(make_float3(primHi[p].x, primHi[p].y, primHi[p].z), s.axis);
    float c = centroid(lo, hi);
    return bin_of(c, task.clo[s.axis], axis_scale(task.clo[s.axis], task.chi[s.axis])) <= s.bin;
}

__global__ void __launch_bounds__(kChunkThreads) k_part_count(const Task* __restrict__ tasks, const uint32_t* __restrict__ refs,
                                                              const float4* __restrict__ primLo, const float4* __restrict__ primHi,
                                                              const uint32_t* __restrict__ bigList, const uint32_t* __restrict__ chunkOff,
                                                              const uint32_t* __restrict__ chunkTask, const BigSplit* __restrict__ splits,
                                                              uint32_t* __restrict__ chunkLeft, uint32_t numChunks,
                                                              const uint32_t* __restrict__ dChunks)
{
    __shared__ uint32_t ws[kChunkThreads / 32];
    const uint32_t nc = level_count(dChunks, numChunks);
    for (uint32_t cb = blockIdx.x; cb < nc; cb += gridDim.x) {
        Task task;
        ChunkRange r = chunk_range(cb, tasks, bigList, chunkOff, chunkTask, task);
        BigSplit s = splits[r.bi];
        uint32_t c = 0;
        for (uint32_t i = r.begin + threadIdx.x; i < r.end; i += blockDim.x) c += goes_left(s, task, i, refs[i], primLo, primHi);
#pragma unroll
        for (int o = 16; o; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
        if (lane_id() == 0) ws[threadIdx.x >> 5] = c;
        __syncthreads();
        if (threadIdx.x == 0) {
            uint32_t s2 = 0;
            for (int w = 0; w < kChunkThreads / 32; ++w) s2 += ws[w];
            chunkLeft[cb] = s2;
        }
        __syncthreads();  // ws is written again for the next chunk
    }
}

__global__ void __launch_bounds__(kChunkThreads) k_part_scatter(const Task* __restrict__ tasks, const uint32_t* __restrict__ refs,
                                                                uint32_t* __restrict__ refsNext,
                                                                const float4* __restrict__ primLo, const float4* __restrict__ primHi,
                                                                const uint32_t* __restrict__ bigList, const uint32_t* __restrict__ chunkOff,
                                                                const uint32_t* __restrict__ chunkTask, const BigSplit* __restrict__ splits,
                                                                const uint32_t* __restrict__ chunkLeftOff,
                                                                uint32_t* __restrict__ status, uint32_t numChunks,
                                                                const uint32_t* __restrict__ dChunks)
{
    __shared__ uint32_t wl[kChunkThreads / 32], wv[kChunkThreads / 32];
    const uint32_t nc = level_count(dChunks, numChunks);
    for (uint32_t cb = blockIdx.x; cb < nc; cb += gridDim.x) {
        Task task;
        ChunkRange r = chunk_range(cb, tasks, bigList, chunkOff, chunkTask, task);
        BigSplit s = splits[r.bi];
        uint32_t leftBefore = chunkLeftOff[cb] - chunkLeftOff[chunkOff[r.bi]];
        uint32_t rightBefore = r.local * kChunk - leftBefore;
        // each thread owns 4 consecutive references: stable order inside the chunk
        uint32_t base = r.begin + threadIdx.x * 4;
        uint32_t p[4];
        bool f[4];
        uint32_t nl = 0;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            uint32_t i = base + k;
            f[k] = false;
            p[k] = 0;
            if (i < r.end) {
                p[k] = refs[i];
                f[k] = goes_left(s, task, i, p[k], primLo, primHi);
                nl += f[k];
            }
        }
        uint32_t nvalid = base < r.end ? min(4u, r.end - base) : 0u;
        // block exclusive scan of (left count, valid count)
        uint32_t il = nl, iv = nvalid;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t yl = __shfl_up_sync(0xffffffffu, il, o);
            uint32_t yv = __shfl_up_sync(0xffffffffu, iv, o);
            if (lane_id() >= (uint32_t)o) { il += yl; iv += yv; }
        }
        if (lane_id() == 31) { wl[threadIdx.x >> 5] = il; wv[threadIdx.x >> 5] = iv; }
        __syncthreads();
        uint32_t pl = 0, pv = 0;
        for (uint32_t w = 0; w < (threadIdx.x >> 5); ++w) { pl += wl[w]; pv += wv[w]; }
        uint32_t leftRank = pl + il - nl;
        uint32_t rightRank = (pv + iv - nvalid) - leftRank;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            uint32_t i = base + k;
            if (i >= r.end) break;
            uint32_t dst = f[k] ? task.begin + leftBefore + leftRank++ : task.begin + s.nL + rightBefore + rightRank++;
            if (dst >= task.begin + task.count) { atomicOr(status, kErrBadIndex); continue; }
            refsNext[dst] = p[k];
        }
        __syncthreads();  // wl / wv are written again for the next chunk
    }
}

// --------------------------------------------------------------------------
// Small tasks: one warp does bin + split + partition.
// Task t by one warp; sb: the warp's bins in shared memory.
AG_D void small_task(uint32_t t, const Task* __restrict__ tasks, const uint32_t* __restrict__ refs,
                     uint32_t* __restrict__ refsNext, const float4* __restrict__ primLo,
                     const float4* __restrict__ primHi, const BinNode* __restrict__ bnodes, Cand* __restrict__ cands,
                     uint32_t* __restrict__ candFlag, uint32_t* __restrict__ order, uint32_t* __restrict__ status,
                     uint32_t* sb, uint32_t* failed)
{
    Task task = tasks[t];
    if (task.count > kSmallMax) {  // handled by the big-task kernels
        // A device-driven build runs those kernels on its first levels only
        // (failed != null below them): the task gets no children, and the
        // build is stopped and reported.
        if (failed && lane_id() == 0) {
            candFlag[2 * t] = 0;
            candFlag[2 * t + 1] = 0;
            atomicOr(failed, 1u);
            atomicOr(status, kErrBuildDepth);
        }
        return;
    }
    uint32_t lane = lane_id();
    const uint32_t b0 = task.begin, n = task.count;

    auto make_leaf = [&]() {
        for (uint32_t i = lane; i < n; i += 32) order[b0 + i] = refs[b0 + i];
        if (lane == 0) { candFlag[2 * t] = 0; candFlag[2 * t + 1] = 0; }
    };
    if (n <= 1) { make_leaf(); return; }

    // centroid bounds of this task
    float clo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, chi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
    for (uint32_t i = lane; i < n; i += 32) {
        uint32_t p = refs[b0 + i];
        float4 lo = primLo[p], hi = primHi[p];
        float c[3] = {centroid(lo.x, hi.x), centroid(lo.y, hi.y), centroid(lo.z, hi.z)};
#pragma unroll
        for (int k = 0; k < 3; ++k) { clo[k] = fminf(clo[k], c[k]); chi[k] = fmaxf(chi[k], c[k]); }
    }
    float sc[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        clo[k] = warp_min(clo[k]);
        chi[k] = warp_max(chi[k]);
        sc[k] = axis_scale(clo[k], chi[k]);
    }

    __syncwarp();  // the warp's previous task has finished reading sb
    for (int k = lane; k < kTaskBinWords; k += 32) bin_init_word(sb + k, k);
    __syncwarp();
    for (uint32_t i = lane; i < n; i += 32) {
        uint32_t p = refs[b0 + i];
        float4 lo = primLo[p], hi = primHi[p];
        float cx = centroid(lo.x, hi.x), cy = centroid(lo.y, hi.y), cz = centroid(lo.z, hi.z);
        float cc[3] = {cx, cy, cz};
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            if (sc[a] == 0.0f) continue;
            bin_accumulate(sb + a * kAxisBinWords + bin_of(cc[a], clo[a], sc[a]) * kBinWords, lo, hi, cx, cy, cz);
        }
    }
    __syncwarp();
    SplitChoice best;
    best.cost = FLT_MAX;
    best.axis = -1;
    best.bin = 0;
    best.nL = 0;
    for (int a = 0; a < 3; ++a) {
        if (sc[a] == 0.0f) continue;
        float v[12];
        uint32_t cnt;
        load_bin(sb + a * kAxisBinWords + lane * kBinWords, v, cnt);
        eval_axis(a, v, cnt, false, best);
    }
    const BinNode node = bnodes[task.node];
    float nodeArea = area_of(node.lo.x, node.lo.y, node.lo.z, node.hi.x, node.hi.y, node.hi.z);
    // SAH with unit traversal and intersection costs.
    float leafCost = float(n) * nodeArea;
    float splitCost = nodeArea + best.cost;
    if (n <= (uint32_t)kMaxLeafTris && (best.axis < 0 || leafCost <= splitCost)) { make_leaf(); return; }

    uint32_t nL;
    float Lb[12], Rb[12];
    bool median = best.axis < 0;
    if (!median) {
        nL = best.nL;
        for (int k = 0; k < 12; ++k) { Lb[k] = best.L[k]; Rb[k] = best.R[k]; }
    } else {
        nL = n / 2;
        // bounds of each half by warp reduction
        float l0[6] = {FLT_MAX, FLT_MAX, FLT_MAX, -FLT_MAX, -FLT_MAX, -FLT_MAX};
        float l1[6] = {FLT_MAX, FLT_MAX, FLT_MAX, -FLT_MAX, -FLT_MAX, -FLT_MAX};
        for (uint32_t i = lane; i < n; i += 32) {
            uint32_t p = refs[b0 + i];
            float4 lo = primLo[p], hi = primHi[p];
            float* d = i < nL ? l0 : l1;
            d[0] = fminf(d[0], lo.x); d[1] = fminf(d[1], lo.y); d[2] = fminf(d[2], lo.z);
            d[3] = fmaxf(d[3], hi.x); d[4] = fmaxf(d[4], hi.y); d[5] = fmaxf(d[5], hi.z);
        }
        for (int k = 0; k < 3; ++k) {
            Lb[k] = warp_min(l0[k]); Lb[3 + k] = warp_max(l0[3 + k]);
            Rb[k] = warp_min(l1[k]); Rb[3 + k] = warp_max(l1[3 + k]);
        }
        for (int k = 0; k < 3; ++k) { Lb[6 + k] = Rb[6 + k] = clo[k]; Lb[9 + k] = Rb[9 + k] = chi[k]; }
    }
    // stable partition into refsNext
    uint32_t leftSeen = 0, rightSeen = 0;
    for (uint32_t base = 0; base < n; base += 32) {
        uint32_t i = base + lane;
        bool valid = i < n;
        uint32_t p = valid ? refs[b0 + i] : 0;
        bool left = false;
        if (valid) {
            if (median) left = i < nL;
            else {
                float4 lo = primLo[p], hi = primHi[p];
                float c = centroid(comp(make_float3(lo.x, lo.y, lo.z), best.axis), comp(make_float3(hi.x, hi.y, hi.z), best.axis));
                left = bin_of(c, clo[best.axis], sc[best.axis]) <= best.bin;
            }
        }
        uint32_t bl = __ballot_sync(0xffffffffu, valid && left);
        uint32_t br = __ballot_sync(0xffffffffu, valid && !left);
        if (valid) {
            uint32_t dst = left ? b0 + leftSeen + __popc(bl & lanemask_lt())
                                : b0 + nL + rightSeen + __popc(br & lanemask_lt());
            if (dst < b0 + n) refsNext[dst] = p;
            else atomicOr(status, kErrBadIndex);
        }
        leftSeen += __popc(bl);
        rightSeen += __popc(br);
    }
    if (lane == 0) {
        write_cand(cands + 2 * t, Lb, b0, nL);
        write_cand(cands + 2 * t + 1, Rb, b0 + nL, n - nL);
        candFlag[2 * t] = 1;
        candFlag[2 * t + 1] = 1;
    }
}

__global__ void __launch_bounds__(32 * kSmallWarps) k_small(const Task* __restrict__ tasks, uint32_t numTasks,
                                                          const uint32_t* __restrict__ refs, uint32_t* __restrict__ refsNext,
                                                          const float4* __restrict__ primLo, const float4* __restrict__ primHi,
                                                          const BinNode* __restrict__ bnodes, Cand* __restrict__ cands,
                                                          uint32_t* __restrict__ candFlag, uint32_t* __restrict__ order,
                                                          uint32_t* __restrict__ status, const uint32_t* __restrict__ dTasks,
                                                          uint32_t* __restrict__ failed)
{
    __shared__ uint32_t sbins[kSmallWarps][kTaskBinWords];
    const uint32_t w = threadIdx.x >> 5;
    const uint32_t nt = level_count(dTasks, numTasks);
    for (uint32_t t = blockIdx.x * kSmallWarps + w; t < nt; t += gridDim.x * kSmallWarps)
        small_task(t, tasks, refs, refsNext, primLo, primHi, bnodes, cands, candFlag, order, status, sbins[w],
                   failed);
}

// --------------------------------------------------------------------------
// Compaction of the children into the next level's task list.
__global__ void k_cand_keys(const Cand* __restrict__ cands, const uint32_t* __restrict__ candFlag, uint32_t nHost,
                            uint32_t* __restrict__ bigFlag, uint32_t* __restrict__ chunkCnt,
                            const uint32_t* __restrict__ dTasks)
{
    const uint32_t n = level_count(dTasks, nHost, 2u);
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
        bool v = candFlag[j] != 0;
        bigFlag[j] = v ? cands[j].big : 0u;
        chunkCnt[j] = v ? cands[j].chunks : 0u;
    }
}

__global__ void k_compact(const Task* __restrict__ tasks, const Cand* __restrict__ cands,
                          const uint32_t* __restrict__ candFlag, const uint32_t* __restrict__ candPos,
                          const uint32_t* __restrict__ bigPos, const uint32_t* __restrict__ chunkOffSparse, uint32_t nHost,
                          uint32_t nodeBaseHost, Task* __restrict__ next, BinNode* __restrict__ bnodes,
                          uint32_t* __restrict__ bigList, uint32_t* __restrict__ chunkOff, uint32_t* __restrict__ chunkTask,
                          const uint32_t* __restrict__ dTasks, const uint32_t* __restrict__ dNodes, uint32_t capTasks,
                          uint32_t capBig, uint32_t capChunks, uint32_t* __restrict__ status)
{
    const uint32_t n = level_count(dTasks, nHost, 2u);
    const uint32_t nodeBase = level_count(dNodes, nodeBaseHost);
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
        if (!candFlag[j]) continue;
        Cand c = cands[j];
        uint32_t p = candPos[j];
        uint32_t node = nodeBase + p;
        // capacities: never exceeded by a consistent build; checked so that
        // inconsistent input cannot write past the buffers
        if (p >= capTasks || node >= 2u * capTasks ||
            (c.big && (bigPos[j] >= capBig || chunkOffSparse[j] + c.chunks > capChunks))) {
            atomicOr(status, kErrBadIndex);
            continue;
        }
        uint32_t parent = tasks[j >> 1].node;
        if (j & 1) bnodes[parent].right = (int32_t)node;
        else bnodes[parent].left = (int32_t)node;
        BinNode b;
        if (c.lo[0] != c.lo[0]) {  // median split of coincident centroids: inherit parent box
            b.lo = bnodes[parent].lo;
            b.hi = bnodes[parent].hi;
        } else {
            b.lo = mk3(c.lo[0], c.lo[1], c.lo[2]);
            b.hi = mk3(c.hi[0], c.hi[1], c.hi[2]);
        }
        b.begin = c.begin;
        b.count = c.count;
        b.left = -1;
        b.right = -1;
        bnodes[node] = b;
        Task t;
        for (int k = 0; k < 3; ++k) { t.clo[k] = c.clo[k]; t.chi[k] = c.chi[k]; }
        t.node = node;
        t.begin = c.begin;
        t.count = c.count;
        next[p] = t;
        if (c.big) {
            uint32_t bi = bigPos[j];
            bigList[bi] = p;
            uint32_t off = chunkOffSparse[j];
            chunkOff[bi] = off;
            for (uint32_t k = 0; k < c.chunks; ++k) chunkTask[off + k] = bi;
        }
    }
}

// --------------------------------------------------------------------------
// Collapse to the wide layout.
AG_D float bn_area(const BinNode& b) { return area_of(b.lo.x, b.lo.y, b.lo.z, b.hi.x, b.hi.y, b.hi.z); }

// SAH cost program of the collapse, one binary level per launch from the
// deepest up. For binary node x of area A, count n and children l, r:
//   leaf(x)    = A * triCost * n                       (n <= kMaxLeafTris)
//   D(x, j)    = min over k in 1..j-1 of C(l, k) + C(r, j - k)
//   C(x, 1)    = leaf(x) if n <= kMaxLeafTris, else A + D(x, 8)  (x in one slot:
//                a leaf, or an internal child whose own wide node tests 8 slots)
//   C(x, j)    = min(C(x, j - 1), D(x, j))             (x spread over at most j slots)
// with a wide-node visit costing 1 per unit area. cost[8x + j - 1] holds
// C(x, j) for j = 1..7 and cost[8x + 7] = A + D(x, 8); nibble j - 1 of
// choice[x] holds the k of D(x, j) when it was taken (0: x keeps j - 1
// slots; nibble 7: the split of x's own wide node). A binary leaf costs
// leaf(x) for every j.
AG_D void collapse_cost_node(const BinNode* __restrict__ bnodes, uint32_t x, float triCost, float* __restrict__ cost,
                             uint32_t* __restrict__ choice)
{
    const BinNode b = bnodes[x];
    const float A = bn_area(b);
    float* C = cost + 8ull * x;
    if (b.left < 0) {
        const float leaf = b.count <= (uint32_t)kMaxLeafTris ? A * triCost * float(b.count) : INFINITY;
        for (int j = 0; j < 8; ++j) C[j] = leaf;
        choice[x] = 0;
        return;
    }
    float L[7], R[7];
    const float* cl = cost + 8ull * (uint32_t)b.left;
    const float* cr = cost + 8ull * (uint32_t)b.right;
#pragma unroll
    for (int j = 0; j < 7; ++j) {
        L[j] = cl[j];
        R[j] = cr[j];
    }
    float D[9];
    uint32_t K[9];
#pragma unroll
    for (int j = 2; j <= 8; ++j) {
        float best = INFINITY;
        uint32_t bk = 1;
#pragma unroll
        for (int k = 1; k < j; ++k) {
            const float v = L[k - 1] + R[j - k - 1];
            if (v < best) {
                best = v;
                bk = (uint32_t)k;
            }
        }
        D[j] = best;
        K[j] = bk;
    }
    const float node = A + D[8];
    float prev = b.count <= (uint32_t)kMaxLeafTris ? A * triCost * float(b.count) : node;
    C[0] = prev;
    uint32_t ch = K[8] << 28;
#pragma unroll
    for (int j = 2; j <= 7; ++j) {
        if (D[j] < prev) {
            prev = D[j];
            ch |= K[j] << (4 * (j - 1));
        }
        C[j - 1] = prev;
    }
    C[7] = node;
    choice[x] = ch;
}

// One binary level per launch: nodes [first, first + count), or, in a
// device-driven build, [levelStart[level], levelStart[level + 1]).
__global__ void k_collapse_cost(const BinNode* __restrict__ bnodes, uint32_t firstHost, uint32_t countHost,
                                float triCost, float* __restrict__ cost, uint32_t* __restrict__ choice,
                                const uint32_t* __restrict__ levelStart, uint32_t level)
{
    const uint32_t first = levelStart ? levelStart[level] : firstHost;
    const uint32_t count = levelStart ? levelStart[level + 1] - first : countHost;
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < count; t += gridDim.x * blockDim.x)
        collapse_cost_node(bnodes, first + t, triCost, cost, choice);
}

// The slots of one wide node per thread. choice (the cost program's
// decisions) selects the SAH-optimal distribution; null selects the greedy
// rule. Slots are then assigned to octants.
AG_D void collapse_decide_item(uint32_t i, const uint2* __restrict__ items, const BinNode* __restrict__ bnodes,
                               const uint32_t* __restrict__ choice, int32_t* __restrict__ slots,
                               uint32_t* __restrict__ intCount, uint32_t* __restrict__ triCount,
                               uint32_t* __restrict__ slotTotal)
{
    uint32_t b = items[i].x;
    int32_t ent[kWidth];
    int n = 0;
    const BinNode root = bnodes[b];
    if (root.count <= (uint32_t)kMaxLeafTris || root.left < 0) {
        ent[n++] = (int32_t)b;
    } else if (choice) {
        // follow the cost program: (node, slots it may use), root split first
        int32_t stN[kWidth];
        uint32_t stJ[kWidth];
        int sp = 0;
        const uint32_t k8 = min(max(choice[b] >> 28, 1u), 7u);  // 1..7 by construction; clamped so j stays <= 8
        stN[sp] = root.right;
        stJ[sp++] = 8u - k8;
        stN[sp] = root.left;
        stJ[sp++] = k8;
        while (sp > 0) {
            const int32_t x = stN[--sp];
            uint32_t j = stJ[sp];
            const BinNode c = bnodes[x];
            uint32_t k = 0;
            if (c.left >= 0)
                while (j > 1 && (k = (choice[x] >> (4 * (j - 1))) & 0xfu) == 0u) --j;
            if (j <= 1 || c.left < 0 || k == 0u || k >= j || sp + 2 > kWidth || n + sp + 2 > kWidth) {
                ent[n++] = x;  // one slot (the last tests only guard malformed input)
                continue;
            }
            stN[sp] = c.right;
            stJ[sp++] = j - k;
            stN[sp] = c.left;
            stJ[sp++] = k;
        }
    } else {
        ent[n++] = root.left;
        ent[n++] = root.right;
        // Open children until all 8 slots are used: first those too large for
        // a leaf slot, then small internal ones (tighter leaf boxes are free
        // since every slot box is tested anyway).
        for (int phase = 0; phase < 2; ++phase) {
            while (n < kWidth) {
                int pick = -1;
                float pa = -1.0f;
                for (int k = 0; k < n; ++k) {
                    const BinNode& c = bnodes[ent[k]];
                    if (c.left < 0) continue;
                    bool large = c.count > (uint32_t)kMaxLeafTris;
                    if (phase == 0 ? !large : large) continue;
                    float a = bn_area(c);
                    if (a > pa) { pa = a; pick = k; }
                }
                if (pick < 0) break;
                const BinNode& c = bnodes[ent[pick]];
                ent[pick] = c.left;
                ent[n++] = c.right;
            }
        }
    }
    atomicAdd(slotTotal, (uint32_t)n);
    // Octant slot assignment: slot s prefers the child whose centre lies
    // toward corner s of the parent box (bit k of s set = + side of axis k).
    float3 pc = 0.5f * (root.lo + root.hi);
    float3 cen[kWidth];
    for (int k = 0; k < n; ++k) {
        const BinNode& c = bnodes[ent[k]];
        cen[k] = 0.5f * (c.lo + c.hi) - pc;
    }
    int32_t slot[kWidth];
    for (int s = 0; s < kWidth; ++s) slot[s] = -1;
    uint32_t usedChild = 0, usedSlot = 0;
    for (int it = 0; it < n; ++it) {
        float bestV = -FLT_MAX;
        int bc = -1, bs = -1;
        for (int k = 0; k < n; ++k) {
            if (usedChild & (1u << k)) continue;
            for (int s = 0; s < kWidth; ++s) {
                if (usedSlot & (1u << s)) continue;
                float v = ((s & 1) ? cen[k].x : -cen[k].x) + ((s & 2) ? cen[k].y : -cen[k].y) +
                          ((s & 4) ? cen[k].z : -cen[k].z);
                if (v > bestV) { bestV = v; bc = k; bs = s; }
            }
        }
        usedChild |= 1u << bc;
        usedSlot |= 1u << bs;
        slot[bs] = ent[bc];
    }
    uint32_t ni = 0, nt = 0;
    for (int s = 0; s < kWidth; ++s) {
        slots[size_t(i) * kWidth + s] = slot[s];
        if (slot[s] < 0) continue;
        uint32_t cnt = bnodes[slot[s]].count;
        if (cnt <= (uint32_t)kMaxLeafTris) nt += cnt;
        else ni += 1;
    }
    intCount[i] = ni;
    triCount[i] = nt;
}

__global__ void k_collapse_decide(const uint2* __restrict__ items, uint32_t numItems, const BinNode* __restrict__ bnodes,
                                  const uint32_t* __restrict__ choice, int32_t* __restrict__ slots,
                                  uint32_t* __restrict__ intCount, uint32_t* __restrict__ triCount,
                                  uint32_t* __restrict__ slotTotal, const uint32_t* __restrict__ dItems)
{
    const uint32_t n = level_count(dItems, numItems);
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        collapse_decide_item(i, items, bnodes, choice, slots, intCount, triCount, slotTotal);
}

__host__ __device__ inline uint32_t quant_exponent(float extent)
{
    // smallest power of two q with 255 * q >= extent (biased exponent byte)
    if (!(extent > 0.0f)) return 1u;
    int e;
    frexpf(extent / 255.0f, &e);
    float q = ldexpf(1.0f, e);
    if (255.0f * q < extent * 1.000001f) { e += 1; q *= 2.0f; }
    int biased = e + 127;
    biased = biased < 1 ? 1 : (biased > 253 ? 253 : biased);
    return (uint32_t)biased;
}

AG_D void collapse_emit_item(uint32_t i, const uint2* __restrict__ items, const BinNode* __restrict__ bnodes,
                             const int32_t* __restrict__ slots, const uint32_t* __restrict__ intOff,
                             const uint32_t* __restrict__ triOff, uint32_t wideBase, uint32_t triBase0,
                             const uint32_t* __restrict__ order, const float* __restrict__ verts,
                             const uint32_t* __restrict__ idx, uint32_t ntris, const float4* __restrict__ spheres,
                             WideNode* __restrict__ nodes, TriRecord* __restrict__ tris, uint2* __restrict__ itemsNext,
                             float* sahAccum, float rootAreaInv, uint32_t nodeCap, uint32_t triCap,
                             uint32_t* __restrict__ status)
{
    uint2 it = items[i];
    const BinNode nb = bnodes[it.x];
    WideNode w;
    w.px = nb.lo.x;
    w.py = nb.lo.y;
    w.pz = nb.lo.z;
    uint32_t E[3] = {quant_exponent(nb.hi.x - nb.lo.x), quant_exponent(nb.hi.y - nb.lo.y),
                     quant_exponent(nb.hi.z - nb.lo.z)};
    float q[3], invq[3];
    for (int k = 0; k < 3; ++k) {
        q[k] = __uint_as_float(E[k] << 23);
        invq[k] = __uint_as_float((254u - E[k]) << 23);  // exact 1/q
    }
    float p[3] = {w.px, w.py, w.pz};
    uint32_t imask = 0;
    uint32_t childBase = wideBase + intOff[i];
    uint32_t triBase = triBase0 + triOff[i];
    uint8_t meta[8], qlo[3][8], qhi[3][8];
    uint32_t rank = 0, toff = 0;
    float sah = bn_area(nb) * rootAreaInv;  // one node visit
    for (int s = 0; s < kWidth; ++s) {
        int32_t e = slots[size_t(i) * kWidth + s];
        if (e < 0) {
            meta[s] = 0;
            for (int k = 0; k < 3; ++k) { qlo[k][s] = 0xff; qhi[k][s] = 0; }
            continue;
        }
        const BinNode c = bnodes[e];
        float clo[3] = {c.lo.x, c.lo.y, c.lo.z}, chi[3] = {c.hi.x, c.hi.y, c.hi.z};
        for (int k = 0; k < 3; ++k) {
            float fl = floorf((clo[k] - p[k]) * invq[k]);
            float fh = ceilf((chi[k] - p[k]) * invq[k]);
            int l = (int)fmaxf(0.0f, fminf(255.0f, fl));
            int h = (int)fmaxf(0.0f, fminf(255.0f, fh));
            while (l > 0 && p[k] + float(l) * q[k] > clo[k]) --l;
            while (h < 255 && p[k] + float(h) * q[k] < chi[k]) ++h;
            qlo[k][s] = (uint8_t)l;
            qhi[k][s] = (uint8_t)h;
        }
        if (c.count <= (uint32_t)kMaxLeafTris) {
            meta[s] = (uint8_t)((((1u << c.count) - 1u) << 5) | toff);
            for (uint32_t k = 0; k < c.count; ++k) {
                uint32_t prim = order[c.begin + k];
                if (prim >= ntris) {  // a sphere record
                    const float4 sp = spheres[prim - ntris];
                    TriRecord r;
                    r.v0 = make_float4(sp.x, sp.y, sp.z, __uint_as_float(kSpherePrim | (prim - ntris)));
                    r.e0 = make_float4(fabsf(sp.w), 0.0f, 0.0f, __uint_as_float(kSphereTag));
                    r.e1 = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
                    if (triBase + toff + k < triCap) tris[triBase + toff + k] = r;
                    else atomicOr(status, kErrBadIndex);
                    continue;
                }
                const uint32_t* ti = idx + 3ull * prim;
                float v0[3], v1[3], v2[3];
                for (int a = 0; a < 3; ++a) {
                    v0[a] = verts[3ull * ti[0] + a];
                    v1[a] = verts[3ull * ti[1] + a];
                    v2[a] = verts[3ull * ti[2] + a];
                }
                TriRecord r;
                r.v0 = make_float4(v0[0], v0[1], v0[2], __uint_as_float(prim));
                r.e0 = make_float4(__fsub_rn(v1[0], v0[0]), __fsub_rn(v1[1], v0[1]), __fsub_rn(v1[2], v0[2]), 0.0f);
                r.e1 = make_float4(__fsub_rn(v2[0], v0[0]), __fsub_rn(v2[1], v0[1]), __fsub_rn(v2[2], v0[2]), 0.0f);
                if (triBase + toff + k < triCap) tris[triBase + toff + k] = r;
                else atomicOr(status, kErrBadIndex);
            }
            toff += c.count;
            sah += bn_area(c) * rootAreaInv * float(c.count);
        } else {
            meta[s] = (uint8_t)(0x20u | (24u + s));
            imask |= 1u << s;
            itemsNext[intOff[i] + rank] = make_uint2((uint32_t)e, childBase + rank);
            ++rank;
        }
    }
    w.e_imask = E[0] | (E[1] << 8) | (E[2] << 16) | (imask << 24);
    w.childBase = childBase;
    w.triBase = triBase;
    w.meta[0] = meta[0] | (meta[1] << 8) | (meta[2] << 16) | ((uint32_t)meta[3] << 24);
    w.meta[1] = meta[4] | (meta[5] << 8) | (meta[6] << 16) | ((uint32_t)meta[7] << 24);
    for (int k = 0; k < 3; ++k) {
        w.qlo[k][0] = qlo[k][0] | (qlo[k][1] << 8) | (qlo[k][2] << 16) | ((uint32_t)qlo[k][3] << 24);
        w.qlo[k][1] = qlo[k][4] | (qlo[k][5] << 8) | (qlo[k][6] << 16) | ((uint32_t)qlo[k][7] << 24);
        w.qhi[k][0] = qhi[k][0] | (qhi[k][1] << 8) | (qhi[k][2] << 16) | ((uint32_t)qhi[k][3] << 24);
        w.qhi[k][1] = qhi[k][4] | (qhi[k][5] << 8) | (qhi[k][6] << 16) | ((uint32_t)qhi[k][7] << 24);
    }
    if (it.y < nodeCap) nodes[it.y] = w;
    else atomicOr(status, kErrBadIndex);
    atomicAdd(sahAccum, sah);
}

// One collapse level: the counts and bases are the host's, or, in a
// device-driven build, counter words (dDev != null: items, wide nodes and
// triangle records so far, and the root's inverse area).
__global__ void k_collapse_emit(const uint2* __restrict__ items, uint32_t numItems, const BinNode* __restrict__ bnodes,
                                const int32_t* __restrict__ slots, const uint32_t* __restrict__ intOff,
                                const uint32_t* __restrict__ triOff, uint32_t wideBase, uint32_t triBase0,
                                const uint32_t* __restrict__ order, const float* __restrict__ verts,
                                const uint32_t* __restrict__ idx, uint32_t ntris, const float4* __restrict__ spheres,
                                WideNode* __restrict__ nodes,
                                TriRecord* __restrict__ tris, uint2* __restrict__ itemsNext, float* sahAccum,
                                float rootAreaInv, uint32_t nodeCap, uint32_t triCap, uint32_t* __restrict__ status,
                                const uint32_t* __restrict__ dDev)
{
    const uint32_t n = dDev ? dDev[kDevItems] : numItems;
    const uint32_t wb = dDev ? dDev[kDevWide] : wideBase;
    const uint32_t tb = dDev ? dDev[kDevTris] : triBase0;
    const float ria = dDev ? __uint_as_float(dDev[kDevRootAreaInv]) : rootAreaInv;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        collapse_emit_item(i, items, bnodes, slots, intOff, triOff, wb, tb, order, verts, idx, ntris, spheres, nodes,
                           tris, itemsNext, sahAccum, ria, nodeCap, triCap, status);
}

// --------------------------------------------------------------------------
// Device-driven build: the host loop's bookkeeping as single-thread kernels.
__global__ void k_dev_begin(uint32_t n, uint32_t* __restrict__ dv, uint32_t* __restrict__ levelStart)
{
    const uint32_t big = n > kSmallMax ? 1u : 0u;
    dv[kDevTasks] = 1u;
    dv[kDevBig] = big;
    dv[kDevChunks] = big ? (n + kChunk - 1) / kChunk : 0u;
    dv[kDevNodes] = 1u;
    dv[kDevLevels] = 0u;
    dv[kDevFailed] = 0u;
    levelStart[0] = 0u;
}

// After binary level L: the next level's counts (the scans' totals) become
// current, the next level's nodes start at the node count so far. Counts
// beyond the buffers' capacities (impossible for a consistent build) stop
// the build with an error instead of reaching past the buffers.
__global__ void k_dev_level_end(uint32_t* __restrict__ dv, uint32_t* __restrict__ levelStart, uint32_t L,
                                uint32_t capTasks, uint32_t capBig, uint32_t capChunks, uint32_t* __restrict__ status)
{
    if (dv[kDevTasks] > 0u) dv[kDevLevels] += 1u;
    levelStart[L + 1] = dv[kDevNodes];
    uint32_t t = dv[kCntTasks], b = dv[kCntBig], c = dv[kCntChunks];
    if (t > capTasks || b > capBig || c > capChunks || dv[kDevNodes] + t > 2u * capTasks) {
        atomicOr(status, kErrBadIndex);
        dv[kDevFailed] = 1u;
    }
    if (dv[kDevFailed]) t = b = c = 0u;  // the build stops; the collapse is skipped
    dv[kDevNodes] += t;
    dv[kDevTasks] = t;
    dv[kDevBig] = b;
    dv[kDevChunks] = c;
}

// Before the collapse: the root item, the counters, the root's inverse area
// (in the host build's order of rounded operations). Tasks left over mean
// the level cap was too small: the collapse is then skipped (the previous
// tree stays in place) and the status word says so.
__global__ void k_dev_collapse_begin(uint32_t* __restrict__ dv, const BinNode* __restrict__ bnodes,
                                     uint2* __restrict__ items, float* __restrict__ sahAccum,
                                     uint32_t* __restrict__ status)
{
    const bool failed = dv[kDevTasks] != 0u || dv[kDevFailed] != 0u;
    if (failed) atomicOr(status, kErrBuildDepth);
    items[0] = make_uint2(0u, 0u);
    dv[kDevItems] = failed ? 0u : 1u;
    dv[kDevWide] = 1u;
    dv[kDevTris] = 0u;
    dv[kDevDepth] = 0u;
    dv[kCntSlots] = 0u;
    *sahAccum = 0.0f;
    const BinNode rb = bnodes[0];
    const float ex = __fsub_rn(rb.hi.x, rb.lo.x), ey = __fsub_rn(rb.hi.y, rb.lo.y), ez = __fsub_rn(rb.hi.z, rb.lo.z);
    const float area = __fadd_rn(__fadd_rn(__fmul_rn(ex, ey), __fmul_rn(ey, ez)), __fmul_rn(ez, ex));
    dv[kDevRootAreaInv] = __float_as_uint(area > 0.0f ? __fdiv_rn(1.0f, area) : 0.0f);
}

__global__ void k_dev_wide_end(uint32_t* __restrict__ dv, uint32_t capItems, uint32_t* __restrict__ status)
{
    if (dv[kDevItems] > 0u) dv[kDevDepth] += 1u;
    uint32_t items = dv[kCntInt];
    if (items > capItems || dv[kDevWide] + items > capItems) {
        atomicOr(status, kErrBadIndex);
        items = 0u;
    }
    dv[kDevItems] = items;
    dv[kDevWide] += items;
    dv[kDevTris] += dv[kCntTri];
}

__global__ void k_dev_end(const uint32_t* __restrict__ dv, uint32_t n, uint32_t* __restrict__ status)
{
    const bool skipped = dv[kDevWide] == 1u && dv[kDevTris] == 0u && dv[kDevDepth] == 0u;
    if (dv[kDevItems] != 0u || dv[kDevDepth] > (uint32_t)kTraversalStack || (!skipped && dv[kDevTris] != n))
        atomicOr(status, kErrBuildDepth);
}

template <typename T>
T* carve(char*& p, size_t count)
{
    size_t bytes = (count * sizeof(T) + 255) & ~size_t(255);
    T* r = reinterpret_cast<T*>(p);
    p += bytes;
    return r;
}
template <typename T>
size_t carve_bytes(size_t count)
{
    return (count * sizeof(T) + 255) & ~size_t(255);
}

inline unsigned blocks_for(size_t n, int threads) { return (unsigned)((n + threads - 1) / threads); }

}  // namespace

Builder::~Builder() { release(); }

void Builder::release()
{
    if (graphExec_) cudaGraphExecDestroy(graphExec_);
    graphExec_ = nullptr;
    graphKey_.clear();
    if (mem_) cudaFree(mem_);
    if (hostCounters_) cudaFreeHost(hostCounters_);
    if (ev0_) cudaEventDestroy(ev0_);
    if (ev1_) cudaEventDestroy(ev1_);
    mem_ = nullptr;
    hostCounters_ = nullptr;
    ev0_ = ev1_ = nullptr;
    cap_ = 0;
}

int Builder::reserve(uint32_t n, char* err, size_t errLen)
{
    if (n <= cap_ && mem_) return 0;
    release();
    size_t N = n ? n : 1;
    size_t maxBig = N / kSmallMax + 2;
    size_t maxChunks = N / kChunk + maxBig + 2;
    size_t bytes = 0;
    bytes += 2 * carve_bytes<float4>(N);           // primLo, primHi
    bytes += 3 * carve_bytes<uint32_t>(N);         // refs x2, order
    bytes += carve_bytes<BinNode>(2 * N);          // bnodes
    bytes += 2 * carve_bytes<Task>(N);             // tasks x2
    bytes += carve_bytes<Cand>(2 * N);             // cands
    bytes += 4 * carve_bytes<uint32_t>(2 * N);     // candFlag, candPos, bigFlag, bigPos
    bytes += 2 * carve_bytes<uint32_t>(2 * N);     // chunk counts (sparse) + offsets
    bytes += carve_bytes<uint32_t>(maxBig);        // bigList
    bytes += carve_bytes<uint32_t>(maxBig);        // chunkOff
    bytes += 3 * carve_bytes<uint32_t>(maxChunks); // chunkTask, chunkLeft, chunkLeftOff
    bytes += carve_bytes<uint32_t>(maxBig * kTaskBinWords);
    bytes += carve_bytes<BigSplit>(maxBig);
    bytes += 2 * carve_bytes<uint2>(N + 1);        // items x2
    bytes += carve_bytes<int32_t>((N + 1) * kWidth);
    bytes += carve_bytes<float>(2 * N * 8);        // collapse costs
    bytes += carve_bytes<uint32_t>(2 * N);         // collapse choices
    bytes += 4 * carve_bytes<uint32_t>(N + 1);     // intCount, intOff, triCount, triOff
    bytes += carve_bytes<uint32_t>(kCntWords);
    const size_t scanWords = std::max(scan_scratch_words(2 * N + 2), scan3_scratch_words(2 * N + 2));
    bytes += carve_bytes<uint32_t>(scanWords);
    bytes += carve_bytes<float>(1);
    bytes += carve_bytes<uint32_t>(kMaxLevels + 2);  // level starts of a device-driven build
    if (cudaMalloc(&mem_, bytes) != cudaSuccess) {
        snprintf(err, errLen, "BVH build: cudaMalloc of %zu bytes failed", bytes);
        mem_ = nullptr;
        cudaGetLastError();
        return -5;
    }
    memBytes_ = bytes;
    char* p = static_cast<char*>(mem_);
    primLo_ = carve<float4>(p, N);
    primHi_ = carve<float4>(p, N);
    refs_[0] = carve<uint32_t>(p, N);
    refs_[1] = carve<uint32_t>(p, N);
    order_ = carve<uint32_t>(p, N);
    bnodes_ = carve<BinNode>(p, 2 * N);
    tasks_[0] = carve<Task>(p, N);
    tasks_[1] = carve<Task>(p, N);
    cands_ = carve<Cand>(p, 2 * N);
    candFlag_ = carve<uint32_t>(p, 2 * N);
    candPos_ = carve<uint32_t>(p, 2 * N);
    bigFlag_ = carve<uint32_t>(p, 2 * N);
    bigPos_ = carve<uint32_t>(p, 2 * N);
    bigChunks_ = carve<uint32_t>(p, 2 * N);
    chunkOffSparse_ = carve<uint32_t>(p, 2 * N);
    bigList_ = carve<uint32_t>(p, maxBig);
    chunkOff_ = carve<uint32_t>(p, maxBig);
    chunkTask_ = carve<uint32_t>(p, maxChunks);
    chunkLeft_ = carve<uint32_t>(p, maxChunks);
    chunkLeftOff_ = carve<uint32_t>(p, maxChunks);
    bigBins_ = carve<uint32_t>(p, maxBig * kTaskBinWords);
    bigSplit_ = carve<BigSplit>(p, maxBig);
    items_[0] = reinterpret_cast<uint32_t*>(carve<uint2>(p, N + 1));
    items_[1] = reinterpret_cast<uint32_t*>(carve<uint2>(p, N + 1));
    slots_ = reinterpret_cast<uint32_t*>(carve<int32_t>(p, (N + 1) * kWidth));
    collapseCost_ = carve<float>(p, 2 * N * 8);
    collapseChoice_ = carve<uint32_t>(p, 2 * N);
    intCount_ = carve<uint32_t>(p, N + 1);
    intOff_ = carve<uint32_t>(p, N + 1);
    triCount_ = carve<uint32_t>(p, N + 1);
    triOff_ = carve<uint32_t>(p, N + 1);
    counters_ = carve<uint32_t>(p, kCntWords);
    scanScratch_ = carve<uint32_t>(p, scanWords);
    sahAccum_ = carve<float>(p, 1);
    levelStartDev_ = carve<uint32_t>(p, kMaxLevels + 2);
    if (cudaMallocHost(&hostCounters_, kCntWords * sizeof(uint32_t)) != cudaSuccess) {
        snprintf(err, errLen, "BVH build: cudaMallocHost failed");
        cudaGetLastError();
        release();
        return -5;
    }
    cudaEventCreate(&ev0_);
    cudaEventCreate(&ev1_);
    cap_ = n;
    return 0;
}

int Builder::build(const float* verts, const uint32_t* idx, uint32_t ntris, const float4* spheres, uint32_t nspheres,
                   WideNode* nodes, TriRecord* tris, uint32_t* deviceStatus, cudaStream_t st, BuildStats* stats,
                   char* err, size_t errLen)
{
    const uint32_t n = ntris + nspheres;
    BuildStats local;
    if (n == 0) {
        if (stats) *stats = local;
        return 0;
    }
    if (int rc = reserve(n, err, errLen)) return rc;
    const size_t N = n;
    const size_t maxBig = N / kSmallMax + 2;              // as reserve() sizes the buffers
    const size_t maxChunks = N / kChunk + maxBig + 2;
    uint32_t* chunkOffSparse = chunkOffSparse_;
    Task* tasks[2] = {static_cast<Task*>(tasks_[0]), static_cast<Task*>(tasks_[1])};
    Cand* cands = static_cast<Cand*>(cands_);
    BigSplit* splits = static_cast<BigSplit*>(bigSplit_);
    uint32_t* bounds = counters_ + kCntBounds;

    cudaEventRecord(ev0_, st);
    k_init_bounds<<<1, 32, 0, st>>>(bounds);
    k_prep_prims<<<blocks_for(N, 256), 256, 0, st>>>(verts, idx, ntris, spheres, n, primLo_, primHi_, refs_[0], bounds);
    uint32_t numTasks = 1;
    uint32_t numBig = n > kSmallMax ? 1u : 0u;
    uint32_t totalChunks = numBig ? (n + kChunk - 1) / kChunk : 0u;
    k_root<<<blocks_for(totalChunks + 1, 256), 256, 0, st>>>(n, bounds, tasks[0], bnodes_, bigList_, chunkOff_,
                                                             chunkTask_, totalChunks);
    uint32_t nodeCount = 1;
    int cur = 0;
    uint32_t level = 0;
    bigLevels_ = 0;
    levelCounts_.clear();
    wideCounts_.clear();
    ++buildGeneration_;
    levelStart_.assign(1, 0u);  // binary node ids of level L: [levelStart_[L], levelStart_[L + 1])
    while (numTasks > 0) {
        if (++level > kMaxLevels) {
            snprintf(err, errLen, "BVH build: more than %u levels", kMaxLevels);
            return -4;
        }
        Task* tk = tasks[cur];
        levelCounts_.push_back({numTasks, numBig, totalChunks});
        if (numBig > 0) {
            bigLevels_ = level;
            k_bins_clear<<<numBig, 256, 0, st>>>(bigBins_, numBig, nullptr);
            k_bin_big<<<totalChunks, kChunkThreads, 0, st>>>(tk, refs_[cur], primLo_, primHi_, bigList_, chunkOff_,
                                                             chunkTask_, bigBins_, totalChunks, nullptr);
            k_split_big<<<numBig, 32, 0, st>>>(tk, bigList_, bigBins_, splits, cands, candFlag_, numBig, nullptr);
            k_part_count<<<totalChunks, kChunkThreads, 0, st>>>(tk, refs_[cur], primLo_, primHi_, bigList_, chunkOff_,
                                                                chunkTask_, splits, chunkLeft_, totalChunks, nullptr);
            exclusive_scan(chunkLeft_, chunkLeftOff_, totalChunks, nullptr, scanScratch_, st);
            k_part_scatter<<<totalChunks, kChunkThreads, 0, st>>>(tk, refs_[cur], refs_[cur ^ 1], primLo_, primHi_,
                                                                  bigList_, chunkOff_, chunkTask_, splits,
                                                                  chunkLeftOff_, deviceStatus, totalChunks, nullptr);
        }
        k_small<<<blocks_for(numTasks, kSmallWarps), 32 * kSmallWarps, 0, st>>>(
            tk, numTasks, refs_[cur], refs_[cur ^ 1], primLo_, primHi_, bnodes_, cands, candFlag_, order_,
            deviceStatus, nullptr, nullptr);
        const uint32_t nc = 2 * numTasks;
        k_cand_keys<<<blocks_for(nc, 256), 256, 0, st>>>(cands, candFlag_, nc, bigFlag_, bigChunks_, nullptr);
        exclusive_scan(candFlag_, candPos_, nc, counters_ + kCntTasks, scanScratch_, st);
        exclusive_scan(bigFlag_, bigPos_, nc, counters_ + kCntBig, scanScratch_, st);
        exclusive_scan(bigChunks_, chunkOffSparse, nc, counters_ + kCntChunks, scanScratch_, st);
        k_compact<<<blocks_for(nc, 256), 256, 0, st>>>(tk, cands, candFlag_, candPos_, bigPos_, chunkOffSparse, nc,
                                                       nodeCount, tasks[cur ^ 1], bnodes_, bigList_, chunkOff_,
                                                       chunkTask_, nullptr, nullptr, n, (uint32_t)maxBig,
                                                       (uint32_t)maxChunks, deviceStatus);
        cudaMemcpyAsync(hostCounters_, counters_, 3 * sizeof(uint32_t), cudaMemcpyDeviceToHost, st);
        if (cudaStreamSynchronize(st) != cudaSuccess) {
            snprintf(err, errLen, "BVH build: %s", cudaGetErrorString(cudaGetLastError()));
            return -2;
        }
        numTasks = hostCounters_[kCntTasks];
        numBig = hostCounters_[kCntBig];
        totalChunks = hostCounters_[kCntChunks];
        levelStart_.push_back(nodeCount);
        nodeCount += numTasks;
        cur ^= 1;
    }
    levelStart_.push_back(nodeCount);
    local.binaryNodes = nodeCount;
    local.binaryLevels = level;
    local.bigLevels = bigLevels_;

    // SAH cost program of the collapse, deepest level first
    const bool sahCollapse = collapse_ == kCollapseSah;
    if (sahCollapse)
        for (size_t L = levelStart_.size() - 1; L-- > 0;) {
            const uint32_t first = levelStart_[L], cnt = levelStart_[L + 1] - first;
            if (cnt) k_collapse_cost<<<blocks_for(cnt, 128), 128, 0, st>>>(bnodes_, first, cnt, triCost_,
                                                                          collapseCost_, collapseChoice_, nullptr, 0u);
        }

    // Wide collapse.
    BinNode rb;
    cudaMemcpyAsync(&rb, bnodes_, sizeof(BinNode), cudaMemcpyDeviceToHost, st);
    uint2 rootItem = make_uint2(0, 0);
    cudaMemcpyAsync(items_[0], &rootItem, sizeof(uint2), cudaMemcpyHostToDevice, st);
    cudaMemsetAsync(sahAccum_, 0, sizeof(float), st);
    cudaMemsetAsync(counters_ + kCntSlots, 0, sizeof(uint32_t), st);
    cudaStreamSynchronize(st);
    float rootArea = (rb.hi.x - rb.lo.x) * (rb.hi.y - rb.lo.y) + (rb.hi.y - rb.lo.y) * (rb.hi.z - rb.lo.z) +
                     (rb.hi.z - rb.lo.z) * (rb.hi.x - rb.lo.x);
    float rootAreaInv = rootArea > 0.0f ? 1.0f / rootArea : 0.0f;
    uint32_t numItems = 1, wideCount = 1, triCount = 0, depth = 0;
    int ci = 0;
    while (numItems > 0) {
        if (++depth > 64) {
            snprintf(err, errLen, "BVH collapse: more than 64 wide levels");
            return -4;
        }
        const uint2* items = reinterpret_cast<const uint2*>(items_[ci]);
        uint2* itemsNext = reinterpret_cast<uint2*>(items_[ci ^ 1]);
        int32_t* slots = reinterpret_cast<int32_t*>(slots_);
        wideCounts_.push_back(numItems);
        k_collapse_decide<<<blocks_for(numItems, 128), 128, 0, st>>>(
            items, numItems, bnodes_, sahCollapse ? collapseChoice_ : nullptr, slots, intCount_, triCount_,
            counters_ + kCntSlots, nullptr);
        exclusive_scan(intCount_, intOff_, numItems, counters_ + kCntInt, scanScratch_, st);
        exclusive_scan(triCount_, triOff_, numItems, counters_ + kCntTri, scanScratch_, st);
        k_collapse_emit<<<blocks_for(numItems, 128), 128, 0, st>>>(items, numItems, bnodes_, slots, intOff_, triOff_,
                                                                    wideCount, triCount, order_, verts, idx, ntris,
                                                                    spheres, nodes,
                                                                    tris, itemsNext, sahAccum_, rootAreaInv, n + 1, n,
                                                                    deviceStatus, nullptr);
        cudaMemcpyAsync(hostCounters_ + kCntInt, counters_ + kCntInt, 2 * sizeof(uint32_t), cudaMemcpyDeviceToHost,
                        st);
        if (cudaStreamSynchronize(st) != cudaSuccess) {
            snprintf(err, errLen, "BVH collapse: %s", cudaGetErrorString(cudaGetLastError()));
            return -2;
        }
        numItems = hostCounters_[kCntInt];
        wideCount += numItems;
        triCount += hostCounters_[kCntTri];
        ci ^= 1;
    }
    cudaEventRecord(ev1_, st);
    float sah = 0.0f;
    cudaMemcpyAsync(&sah, sahAccum_, sizeof(float), cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(hostCounters_ + kCntSlots, counters_ + kCntSlots, sizeof(uint32_t), cudaMemcpyDeviceToHost, st);
    if (cudaStreamSynchronize(st) != cudaSuccess) {
        snprintf(err, errLen, "BVH build: %s", cudaGetErrorString(cudaGetLastError()));
        return -2;
    }
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, ev0_, ev1_);
    local.wideNodes = wideCount;
    local.wideDepth = depth;
    local.triCount = triCount;
    local.sahCost = sah;
    local.buildMs = ms;
    local.childSlots = hostCounters_[kCntSlots];
    if (triCount != n) {
        snprintf(err, errLen, "BVH build: %u triangles placed, expected %u", triCount, n);
        return -3;
    }
    if (depth > (uint32_t)kTraversalStack) {
        snprintf(err, errLen, "BVH build: wide depth %u exceeds the traversal stack (%d)", depth, kTraversalStack);
        return -4;
    }
    if (stats) *stats = local;
    return 0;
}


namespace {
// Grids of the device-driven build: the counts are not known when the
// launches are made, so each kernel loops over its work items on at most
// this many blocks (a few waves of the 148 SMs).
constexpr unsigned kDevChunkBlocks = 148 * 4;
constexpr unsigned kDevThreadBlocks = 148 * 8;
inline unsigned dev_blocks(size_t n, int threads, unsigned cap)
{
    const size_t b = (n + threads - 1) / threads;
    return (unsigned)(b < 1 ? 1 : (b > cap ? cap : b));
}
}  // namespace

void Builder::enqueue_launches(const float* verts, const uint32_t* idx, uint32_t ntris, const float4* spheres,
                               uint32_t n, WideNode* nodes, TriRecord* tris, uint32_t* deviceStatus, cudaStream_t st,
                               uint32_t maxLevels, uint32_t maxWideLevels)
{
    const size_t N = n;
    const size_t maxBig = N / kSmallMax + 2;
    const size_t maxChunks = N / kChunk + maxBig + 2;
    Task* tasks[2] = {static_cast<Task*>(tasks_[0]), static_cast<Task*>(tasks_[1])};
    Cand* cands = static_cast<Cand*>(cands_);
    BigSplit* splits = static_cast<BigSplit*>(bigSplit_);
    uint32_t* bounds = counters_ + kCntBounds;
    uint32_t* dv = counters_;
    const uint32_t rootChunks = n > kSmallMax ? (n + kChunk - 1) / kChunk : 0u;

    k_init_bounds<<<1, 32, 0, st>>>(bounds);
    k_prep_prims<<<blocks_for(N, 256), 256, 0, st>>>(verts, idx, ntris, spheres, n, primLo_, primHi_, refs_[0], bounds);
    k_root<<<blocks_for(rootChunks + 1, 256), 256, 0, st>>>(n, bounds, tasks[0], bnodes_, bigList_, chunkOff_,
                                                            chunkTask_, rootChunks);
    k_dev_begin<<<1, 1, 0, st>>>(n, dv, levelStartDev_);
    // Grids: the kernels loop over their work items, so any grid is correct.
    // Each level's grid is sized for 1.5 times the count the last host-driven
    // build had there (animated geometry keeps them close), capped by the
    // buffers' capacities, instead of the capacity itself: far fewer idle
    // blocks are dispatched.
    auto expect = [](uint32_t recorded, size_t cap) {
        return std::min(cap, size_t(recorded) + recorded / 2 + 32);
    };
    auto level_expect = [&](uint32_t L) {
        return L < levelCounts_.size() ? levelCounts_[L] : (levelCounts_.empty() ? LevelCounts{1, 1, 1} : levelCounts_.back());
    };
    // tasks above kSmallMax references occur on the top levels only: the
    // big-task kernels run on the levels where the last host-driven build had
    // them, plus a margin (k_small reports a big task met past them)
    const uint32_t bigCap = std::min(maxLevels, bigLevels_ + 2u);
    int cur = 0;
    for (uint32_t L = 0; L < maxLevels; ++L) {
        Task* tk = tasks[cur];
        const bool bigLevel = L < bigCap;
        const LevelCounts e = level_expect(L);
        const unsigned gBig = dev_blocks(expect(e.big, maxBig), 1, kDevChunkBlocks);
        const unsigned gChunks = dev_blocks(expect(e.chunks, maxChunks), 1, kDevChunkBlocks);
        const unsigned gSmall = dev_blocks(expect(e.tasks, N), kSmallWarps, kDevThreadBlocks);
        const unsigned gCand = dev_blocks(2 * expect(e.tasks, N), 256, kDevThreadBlocks);
        if (bigLevel) {
            k_bins_clear<<<gBig, 256, 0, st>>>(bigBins_, 0u, dv + kDevBig);
            k_bin_big<<<gChunks, kChunkThreads, 0, st>>>(tk, refs_[cur], primLo_, primHi_, bigList_, chunkOff_,
                                                         chunkTask_, bigBins_, 0u, dv + kDevChunks);
            k_split_big<<<gBig, 32, 0, st>>>(tk, bigList_, bigBins_, splits, cands, candFlag_, 0u, dv + kDevBig);
            k_part_count<<<gChunks, kChunkThreads, 0, st>>>(tk, refs_[cur], primLo_, primHi_, bigList_, chunkOff_,
                                                            chunkTask_, splits, chunkLeft_, 0u, dv + kDevChunks);
            {
                const uint32_t* in[] = {chunkLeft_};
                uint32_t* out[] = {chunkLeftOff_};
                exclusive_scan_count(1, in, out, dv + kDevChunks, 1u, maxChunks, nullptr, scanScratch_, st,
                                     expect(e.chunks, maxChunks));
            }
            k_part_scatter<<<gChunks, kChunkThreads, 0, st>>>(tk, refs_[cur], refs_[cur ^ 1], primLo_, primHi_,
                                                              bigList_, chunkOff_, chunkTask_, splits, chunkLeftOff_,
                                                              deviceStatus, 0u, dv + kDevChunks);
        }
        k_small<<<gSmall, 32 * kSmallWarps, 0, st>>>(tk, 0u, refs_[cur], refs_[cur ^ 1], primLo_, primHi_, bnodes_,
                                                     cands, candFlag_, order_, deviceStatus, dv + kDevTasks,
                                                     bigLevel ? nullptr : dv + kDevFailed);
        k_cand_keys<<<gCand, 256, 0, st>>>(cands, candFlag_, 0u, bigFlag_, bigChunks_, dv + kDevTasks);
        {
            const uint32_t* in[] = {candFlag_, bigFlag_, bigChunks_};
            uint32_t* out[] = {candPos_, bigPos_, chunkOffSparse_};
            uint32_t* tot[] = {counters_ + kCntTasks, counters_ + kCntBig, counters_ + kCntChunks};
            exclusive_scan_count(3, in, out, dv + kDevTasks, 2u, 2 * N, tot, scanScratch_, st,
                                 2 * expect(e.tasks, N));
        }
        k_compact<<<gCand, 256, 0, st>>>(tk, cands, candFlag_, candPos_, bigPos_, chunkOffSparse_, 0u, 0u,
                                         tasks[cur ^ 1], bnodes_, bigList_, chunkOff_, chunkTask_, dv + kDevTasks,
                                         dv + kDevNodes, n, (uint32_t)maxBig, (uint32_t)maxChunks, deviceStatus);
        k_dev_level_end<<<1, 1, 0, st>>>(dv, levelStartDev_, L, n, (uint32_t)maxBig, (uint32_t)maxChunks,
                                         deviceStatus);
        cur ^= 1;
    }

    k_dev_collapse_begin<<<1, 1, 0, st>>>(dv, bnodes_, reinterpret_cast<uint2*>(items_[0]), sahAccum_, deviceStatus);
    const bool sahCollapse = collapse_ == kCollapseSah;
    if (sahCollapse) {
        for (uint32_t L = maxLevels; L-- > 0;) {
            // the nodes of binary level L are the tasks split at level L
            const unsigned gCost = dev_blocks(expect(level_expect(L).tasks, N), 128, kDevThreadBlocks);
            k_collapse_cost<<<gCost, 128, 0, st>>>(bnodes_, 0u, 0u, triCost_, collapseCost_, collapseChoice_,
                                                   levelStartDev_, L);
        }
    }
    int ci = 0;
    for (uint32_t D = 0; D < maxWideLevels; ++D) {
        const uint32_t we = D < wideCounts_.size() ? wideCounts_[D] : (wideCounts_.empty() ? 1u : wideCounts_.back());
        const unsigned gItems = dev_blocks(expect(we, N + 1), 128, kDevThreadBlocks);
        const uint2* items = reinterpret_cast<const uint2*>(items_[ci]);
        uint2* itemsNext = reinterpret_cast<uint2*>(items_[ci ^ 1]);
        int32_t* slots = reinterpret_cast<int32_t*>(slots_);
        k_collapse_decide<<<gItems, 128, 0, st>>>(items, 0u, bnodes_, sahCollapse ? collapseChoice_ : nullptr, slots,
                                                  intCount_, triCount_, counters_ + kCntSlots, dv + kDevItems);
        {
            const uint32_t* in[] = {intCount_, triCount_};
            uint32_t* out[] = {intOff_, triOff_};
            uint32_t* tot[] = {counters_ + kCntInt, counters_ + kCntTri};
            exclusive_scan_count(2, in, out, dv + kDevItems, 1u, N + 1, tot, scanScratch_, st, expect(we, N + 1));
        }
        k_collapse_emit<<<gItems, 128, 0, st>>>(items, 0u, bnodes_, slots, intOff_, triOff_, 0u, 0u, order_, verts, idx,
                                                ntris, spheres, nodes, tris, itemsNext, sahAccum_, 0.0f, n + 1, n,
                                                deviceStatus, dv);
        k_dev_wide_end<<<1, 1, 0, st>>>(dv, n + 1, deviceStatus);
        ci ^= 1;
    }
    k_dev_end<<<1, 1, 0, st>>>(dv, n, deviceStatus);
}

int Builder::enqueue(const float* verts, const uint32_t* idx, uint32_t ntris, const float4* spheres,
                     uint32_t nspheres, WideNode* nodes, TriRecord* tris, uint32_t* deviceStatus, cudaStream_t st,
                     uint32_t maxLevels, uint32_t maxWideLevels, char* err, size_t errLen)
{
    const uint32_t n = ntris + nspheres;
    if (n == 0) return 0;
    if (!mem_ || n > cap_) {
        snprintf(err, errLen, "BVH enqueue: no buffers for %u primitives (run a build of this size first)", n);
        return -6;
    }
    if (maxLevels == 0 || maxLevels > kMaxLevels || maxWideLevels == 0 || maxWideLevels > 64) {
        snprintf(err, errLen, "BVH enqueue: level caps must be 1-%u (binary) and 1-64 (wide)", kMaxLevels);
        return -6;
    }
    const uint64_t key[] = {(uint64_t)(uintptr_t)verts, (uint64_t)(uintptr_t)idx, (uint64_t)(uintptr_t)spheres,
                            (uint64_t)(uintptr_t)nodes, (uint64_t)(uintptr_t)tris, (uint64_t)(uintptr_t)deviceStatus,
                            (uint64_t)(uintptr_t)mem_, ntris, nspheres, maxLevels, maxWideLevels, bigLevels_,
                            buildGeneration_, collapse_,
                            (uint64_t)__builtin_bit_cast(uint32_t, triCost_)};
    const std::vector<uint64_t> k(key, key + sizeof key / sizeof key[0]);
    if (!graphExec_ || k != graphKey_) {
        if (graphExec_) cudaGraphExecDestroy(graphExec_);
        graphExec_ = nullptr;
        if (cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
            snprintf(err, errLen, "BVH enqueue: stream capture could not begin: %s",
                     cudaGetErrorString(cudaGetLastError()));
            return -2;
        }
        enqueue_launches(verts, idx, ntris, spheres, n, nodes, tris, deviceStatus, st, maxLevels, maxWideLevels);
        cudaGraph_t g = nullptr;
        cudaError_t e = cudaStreamEndCapture(st, &g);
        if (e == cudaSuccess) e = cudaGraphInstantiate(&graphExec_, g, 0);
        if (g) cudaGraphDestroy(g);
        if (e != cudaSuccess) {
            graphExec_ = nullptr;
            cudaGetLastError();
            snprintf(err, errLen, "BVH enqueue: graph capture: %s", cudaGetErrorString(e));
            return -2;
        }
        graphKey_ = k;
        ++graphCaptures_;
    }
    cudaEventRecord(ev0_, st);
    cudaError_t e = cudaGraphLaunch(graphExec_, st);
    cudaEventRecord(ev1_, st);
    if (e != cudaSuccess) {
        snprintf(err, errLen, "BVH enqueue: graph launch: %s", cudaGetErrorString(e));
        return -2;
    }
    ++graphLaunches_;
    return 0;
}

int Builder::enqueued_stats(cudaStream_t st, BuildStats* stats, char* err, size_t errLen)
{
    if (!mem_ || graphLaunches_ == 0) {
        snprintf(err, errLen, "BVH stats: no device-driven build yet");
        return -6;
    }
    uint32_t h[kCntWords];
    float sah = 0.0f;
    cudaMemcpyAsync(h, counters_, sizeof h, cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(&sah, sahAccum_, sizeof(float), cudaMemcpyDeviceToHost, st);
    if (cudaStreamSynchronize(st) != cudaSuccess) {
        snprintf(err, errLen, "BVH stats: %s", cudaGetErrorString(cudaGetLastError()));
        return -2;
    }
    BuildStats s;
    s.binaryNodes = h[kDevNodes];
    s.binaryLevels = h[kDevLevels];
    s.wideNodes = h[kDevWide];
    s.wideDepth = h[kDevDepth];
    s.triCount = h[kDevTris];
    s.sahCost = sah;
    s.childSlots = h[kCntSlots];
    float ms = 0.0f;
    if (graphLaunches_ && cudaEventElapsedTime(&ms, ev0_, ev1_) == cudaSuccess) s.buildMs = ms;
    cudaGetLastError();
    *stats = s;
    return 0;
}

}  // namespace ag
