// Learned path guiding: parameters, inference and training kernels (see
// guide.cuh for the model and the published methods it restates).
#include "guide_host.cuh"

#include <algorithm>
#include <type_traits>
#include <cmath>
#include <cstring>
#include <vector>

namespace ag {
namespace guide {
namespace {

constexpr int kInferWarps = 8;

// Shared-memory strides, padded so that the mma fragment loads of a warp
// (8 rows x 4 words) fall in 32 different banks: activation rows of 72 bf16
// (36 words, rows 4 banks apart), weight rows of in + 8, and rows of 40 bf16
// for the transposed [64][32] buffers (20 words).
constexpr int kLd = kHidden + 8;
constexpr int kLdT = 32 + 8;
__host__ __device__ constexpr int wld(int l) { return layer_in(l) + 8; }
__host__ __device__ constexpr int wsm_offset(int l)
{
    int o = 0;
    for (int i = 0; i < l; ++i) o += layer_out(i) * wld(i);
    return o;
}
constexpr int kWsm = wsm_offset(kLayers);  // bf16 elements of the padded weight copy

AG_D __nv_bfloat16 bf(float x) { return __float2bfloat16_rn(x); }
AG_D float fl(__nv_bfloat16 x) { return __bfloat162float(x); }
AG_D uint32_t pack_bf2(float a, float b)
{
    __nv_bfloat162 v = __floats2bfloat162_rn(a, b);
    return *reinterpret_cast<uint32_t*>(&v);
}

// Packed [out][in] weights of every layer into the padded shared copy.
AG_D void load_weights(const __nv_bfloat16* __restrict__ g, __nv_bfloat16* s)
{
    for (int l = 0; l < kLayers; ++l) {
        const uint32_t* src = reinterpret_cast<const uint32_t*>(g + layer_offset(l));
        uint32_t* dst = reinterpret_cast<uint32_t*>(s + wsm_offset(l));
        const int words = layer_in(l) / 2, rows = layer_out(l);
        for (int i = threadIdx.x; i < rows * words; i += blockDim.x) dst[(i / words) * (wld(l) / 2) + i % words] = src[i];
    }
}

// Encodes the 64 inputs of one query into a bf16 row. The corner loads of
// kEncodeLevels levels are issued together, the trilinear weights formed
// after them (2, 4 and 8 levels per round measured the same).
constexpr int kEncodeLevels = 4;
static_assert(kLevels % kEncodeLevels == 0, "levels per round");
AG_D void encode_row(const Params& g, const Query& q, __nv_bfloat16* row)
{
    const float3 p = normalise_position(g, mk3(q.pos[0], q.pos[1], q.pos[2]));
#pragma unroll
    // one corner's kFeatures fp16 values in one load
    using Corner = typename std::conditional<kFeatures == 4, uint2, uint32_t>::type;
    for (int l0 = 0; l0 < kLevels; l0 += kEncodeLevels) {
        Corner v[kEncodeLevels][8];
#pragma unroll
        for (int j = 0; j < kEncodeLevels; ++j)
#pragma unroll
            for (int c = 0; c < 8; ++c) {
                uint32_t idx;
                float w;
                grid_corner(g.res[l0 + j], p, c, idx, w);
                v[j][c] = *reinterpret_cast<const Corner*>(g.grid + ((uint64_t)(l0 + j) * kTableSize + idx) * kFeatures);
            }
#pragma unroll
        for (int j = 0; j < kEncodeLevels; ++j) {
            float f[kFeatures] = {};
#pragma unroll
            for (int c = 0; c < 8; ++c) {
                uint32_t idx;
                float w;
                grid_corner(g.res[l0 + j], p, c, idx, w);
                const __half2* h = reinterpret_cast<const __half2*>(&v[j][c]);
#pragma unroll
                for (int k = 0; k < kFeatures / 2; ++k) {  // one rounding per corner, in corner order
                    f[2 * k] = __fmaf_rn(w, __low2float(h[k]), f[2 * k]);
                    f[2 * k + 1] = __fmaf_rn(w, __high2float(h[k]), f[2 * k + 1]);
                }
            }
#pragma unroll
            for (int k = 0; k < kFeatures; k += 2)
                *reinterpret_cast<uint32_t*>(row + kFeatures * (l0 + j) + k) = pack_bf2(f[k], f[k + 1]);
        }
    }
    float ex[8];
    extra_inputs(mk3(q.wo[0], q.wo[1], q.wo[2]), mk3(q.n[0], q.n[1], q.n[2]), q.rough, ex);
#pragma unroll
    for (int k = 0; k < 8; k += 2) *reinterpret_cast<uint32_t*>(row + kGridDims + k) = pack_bf2(ex[k], ex[k + 1]);
#pragma unroll
    for (int k = kGridDims + 8; k < kIn; k += 2) *reinterpret_cast<uint32_t*>(row + k) = 0u;
}

// acc = X[32 x K] * Wl^T for one warp's 32 rows: X row-major (stride kLd),
// Wl [N][K] row-major (stride ldw), fragments as mma m16n8k16 leaves them.
template <int N, int K>
AG_D void warp_layer(const __nv_bfloat16* X, const __nv_bfloat16* Wl, int ldw, float (&acc)[2][N / 8][4])
{
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
#pragma unroll
    for (int mt = 0; mt < 2; ++mt) {
#pragma unroll
        for (int nt = 0; nt < N / 8; ++nt) {
            float c[4] = {0.0f, 0.0f, 0.0f, 0.0f};
#pragma unroll
            for (int ks = 0; ks < K / 16; ++ks) {
                const __nv_bfloat16* a = X + (mt * 16 + g) * kLd + ks * 16 + 2 * t;
                const __nv_bfloat16* b = Wl + (nt * 8 + g) * ldw + ks * 16 + 2 * t;
                mma_bf16(c, ld32(a), ld32(a + 8 * kLd), ld32(a + 8), ld32(a + 8 * kLd + 8), ld32(b), ld32(b + 8));
            }
#pragma unroll
            for (int k = 0; k < 4; ++k) acc[mt][nt][k] = c[k];
        }
    }
}

// X = bf16(relu(acc)) (call after every lane has finished reading X).
template <int N>
AG_D void store_relu(__nv_bfloat16* X, const float (&acc)[2][N / 8][4])
{
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
#pragma unroll
    for (int mt = 0; mt < 2; ++mt)
#pragma unroll
        for (int nt = 0; nt < N / 8; ++nt) {
            const int r = mt * 16 + g, col = nt * 8 + 2 * t;
            *reinterpret_cast<uint32_t*>(X + r * kLd + col) =
                pack_bf2(fmaxf(acc[mt][nt][0], 0.0f), fmaxf(acc[mt][nt][1], 0.0f));
            *reinterpret_cast<uint32_t*>(X + (r + 8) * kLd + col) =
                pack_bf2(fmaxf(acc[mt][nt][2], 0.0f), fmaxf(acc[mt][nt][3], 0.0f));
        }
}

// Hidden layers of one warp's 32 rows in place; saved (optional) receives
// the input of every layer ([kLayers][32][kLd]). Leaves the input of the
// output layer in X.
AG_D void hidden_layers(const __nv_bfloat16* W, __nv_bfloat16* X, __nv_bfloat16* saved)
{
    for (int l = 0; l < kLayers - 1; ++l) {
        float acc[2][kHidden / 8][4];
        warp_layer<kHidden, kHidden>(X, W + wsm_offset(l), wld(l), acc);
        __syncwarp();
        store_relu<kHidden>(saved ? saved + (l + 1) * 32 * kLd : X, acc);
        if (saved) X = saved + (l + 1) * 32 * kLd;
        __syncwarp();
    }
}

// The inference kernel's shared copy of the output layer has its rows (the
// output units) permuted so that each lane's mma fragments hold whole lobes:
// fragment column c = 8 nt + 2 t + e (lane t of a quad, nt < 5, e < 2) is
// raw output (2 t + s / 5) * 5 + s % 5 with s = 2 nt + e, i.e. lane t holds
// the 5 values of lobes 2t and 2t+1 of its two rows; columns 40..47 (nt = 5)
// stay the unused outputs 40..47.
__host__ __device__ constexpr int out_column_raw(int c)
{
    return c >= 40 ? c : (2 * ((c % 8) / 2) + (2 * (c / 8) + c % 2) / 5) * 5 + (2 * (c / 8) + c % 2) % 5;
}

AG_D void load_weights_infer(const __nv_bfloat16* __restrict__ g, __nv_bfloat16* s)
{
    for (int l = 0; l < kLayers; ++l) {
        const uint32_t* src = reinterpret_cast<const uint32_t*>(g + layer_offset(l));
        uint32_t* dst = reinterpret_cast<uint32_t*>(s + wsm_offset(l));
        const int words = layer_in(l) / 2, rows = layer_out(l);
        for (int i = threadIdx.x; i < rows * words; i += blockDim.x) {
            const int r = i / words, k = i % words;
            const int from = l == kLayers - 1 ? out_column_raw(r) : r;
            dst[r * (wld(l) / 2) + k] = src[from * words + k];
        }
    }
}

// Writes the output tile of one warp's 32 queries (acc: the mma fragments of
// the permuted output layer) as raw parameters (raw[query * 40 + i]) or, with
// `packed`, as decoded mixtures in field arrays `stride` long: each lane
// decodes lobes 2t and 2t+1 of its rows from registers, the softmax over a
// row's 8 lobes reduced across the quad.
AG_D void write_outputs(const float (&acc)[2][kOut / 8][4], uint32_t row0, uint32_t n, float* out, bool packed,
                        uint32_t stride)
{
    const int lane = threadIdx.x & 31, g4 = lane >> 2, t4 = lane & 3;
#pragma unroll
    for (int mt = 0; mt < 2; ++mt)
#pragma unroll
        for (int h = 0; h < 2; ++h) {  // rows g4 and g4 + 8 of the m tile
            const uint32_t gr = row0 + mt * 16 + g4 + 8 * h;
            float r[2][kRawPerLobe];
#pragma unroll
            for (int j = 0; j < 2; ++j)
#pragma unroll
                for (int v = 0; v < kRawPerLobe; ++v) {
                    const int sIdx = kRawPerLobe * j + v;
                    r[j][v] = acc[mt][sIdx / 2][2 * h + sIdx % 2];
                }
            if (!packed) {
                if (gr < n)
#pragma unroll
                    for (int j = 0; j < 2; ++j)
#pragma unroll
                        for (int v = 0; v < kRawPerLobe; ++v)
                            out[(uint64_t)gr * 40 + (2 * t4 + j) * kRawPerLobe + v] = r[j][v];
                continue;
            }
            float mx = fmaxf(r[0][4], r[1][4]);
            mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, 1));
            mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, 2));
            float sum = expf(r[0][4] - mx) + expf(r[1][4] - mx);
            sum += __shfl_xor_sync(0xffffffffu, sum, 1);
            sum += __shfl_xor_sync(0xffffffffu, sum, 2);
            const float invSum = 1.0f / sum;
            if (gr < n)
#pragma unroll
                for (int j = 0; j < 2; ++j) pack_lobe(r[j], mx, invSum, 2 * t4 + j, out + gr, stride);
        }
}

// n queries, or min(n, *nDev) when nDev is not null (a queue length written
// on the device). Writes the 40 raw outputs per query, or with `packed` the
// decoded mixtures as kPacked field arrays of n floats each, n as passed in
// (field f of query i at raw[f * n + i]).
__global__ void __launch_bounds__(32 * kInferWarps, 2) k_infer(Params g, const Query* __restrict__ q, uint32_t n,
                                                          const uint32_t* __restrict__ nDev, float* __restrict__ raw,
                                                          bool packed)
{
    const uint32_t nMax = n;
    if (nDev) n = min(n, *nDev);
    extern __shared__ __align__(16) unsigned char smem[];
    __nv_bfloat16* W = reinterpret_cast<__nv_bfloat16*>(smem);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    __nv_bfloat16* X = W + kWsm + warp * 32 * kLd;
    load_weights_infer(g.W, W);
    __syncthreads();
    const uint32_t chunks = (n + 31) / 32;
    for (uint32_t ch = blockIdx.x * kInferWarps + warp; ch < chunks; ch += gridDim.x * kInferWarps) {
        const uint32_t i = ch * 32 + lane;
        if (i < n) {
            encode_row(g, q[i], X + lane * kLd);
        } else {
            for (int k = 0; k < kIn; ++k) X[lane * kLd + k] = bf(0.0f);
        }
        __syncwarp();
        hidden_layers(W, X, nullptr);
        float acc[2][kOut / 8][4];
        warp_layer<kOut, kHidden>(X, W + wsm_offset(kLayers - 1), wld(kLayers - 1), acc);
        write_outputs(acc, ch * 32, n, raw, packed, nMax);
        __syncwarp();
    }
}

// ---------------------------------------------------------------------------
// Inference on the 5th-generation tensor cores (tcgen05, sm_100a).
//
// One CTA of 128 threads (one warpgroup) runs tiles of 128 queries: thread r
// encodes query r of the tile into row r of the activation tile A[128 x 64]
// (bf16, shared memory); per layer one elected thread issues four
// tcgen05.mma (M 128, N 64 or 48, K 16, bf16 x bf16 -> fp32) from A and the
// layer's weights W_l[N x 64] (shared memory) into a 64-column accumulator in
// tensor memory, and commits them to an mbarrier; then warp w reads rows
// 32w..32w+31 back from tensor memory (tcgen05.ld 32x32b), applies ReLU and
// writes the bf16 row into A for the next layer.
//
// Operands use the no-swizzle K-major layout of 8 x 16-byte core matrices:
// element (row, k) at (row / 8) * 1024 + (k / 8) * 128 + (row % 8) * 16 +
// (k % 8) * 2 bytes, i.e. leading-dimension (K) core-matrix stride 128 B and
// stride-dimension (M/N) core-matrix stride 1024 B. Every completion wait
// is bounded: when it runs out the CTA records kErrTensorWait, stops, and
// still frees its tensor memory.
constexpr int kTcRows = 128;                       // queries per tile (MMA M)
constexpr uint32_t kTcCols = 64;                   // tensor-memory columns (fp32 accumulator)
constexpr uint32_t kTcLbo = 128, kTcSbo = 1024;    // core-matrix strides (bytes)
constexpr int kTcATile = kTcRows * kIn * 2;        // 16 KiB
__host__ __device__ constexpr int tc_w_offset(int l)  // bytes of W_0 .. W_{l-1}
{
    int o = 0;
    for (int i = 0; i < l; ++i) o += layer_out(i) * kIn * 2;
    return o;
}
constexpr int kTcWBytes = tc_w_offset(kLayers);   // 38,912
constexpr int kTcSmem = kTcWBytes + kTcATile + 16;  // + mbarrier + tensor-memory address
constexpr uint32_t kTcWaitLimit = 1u << 24;

AG_D uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Shared-memory matrix descriptor of tcgen05 (no swizzle): start address,
// leading- and stride-dimension byte offsets (all >> 4), version 1 at bit 46.
AG_D uint64_t tc_desc(uint32_t saddr)
{
    return (uint64_t)((saddr & 0x3FFFFu) >> 4) | ((uint64_t)(kTcLbo >> 4) << 16) | ((uint64_t)(kTcSbo >> 4) << 32) |
           (1ull << 46);
}

// Instruction descriptor of tcgen05.mma kind::f16: fp32 accumulator (bits
// 4-5 = 1), bf16 A and B (bits 7-9, 10-12 = 1), both K-major, N >> 3 at bits
// 17-22, M >> 4 at bits 24-28.
__host__ __device__ constexpr uint32_t tc_idesc(int m, int n)
{
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(m >> 4) << 24);
}

AG_D void tc_mma(uint32_t d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t accumulate)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d),
        "l"(a), "l"(b), "r"(idesc), "r"(accumulate)
        : "memory");
}

AG_D void tc_commit(uint32_t mbar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar) : "memory");
}

AG_D bool mbar_try_wait(uint32_t mbar, uint32_t parity)
{
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(mbar), "r"(parity)
        : "memory");
    return done != 0;
}

AG_D void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
AG_D void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// 16 consecutive fp32 columns of this thread's tensor-memory lane, waited for.
AG_D void tc_ld16(uint32_t taddr, float (&v)[16])
{
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, "
        "[%16];\n\ttcgen05.wait::ld.sync.aligned;"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
          "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr)
        : "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// Byte offset of (row, k) in a no-swizzle K-major operand tile.
AG_HD uint32_t tc_offset(uint32_t row, uint32_t k)
{
    return (row >> 3) * kTcSbo + (k >> 3) * kTcLbo + (row & 7u) * 16u + (k & 7u) * 2u;
}

// Threads of the CTA barrier around tensor-core work (the fences order
// tcgen05 operations against the thread barrier).
AG_D void tc_sync()
{
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
}

__global__ void __launch_bounds__(kTcRows, 4) k_infer_tc(Params g, const Query* __restrict__ q, uint32_t n,
                                                      const uint32_t* __restrict__ nDev, float* __restrict__ raw,
                                                      uint32_t* __restrict__ status, bool packed)
{
    const uint32_t nMax = n;
    if (nDev) n = min(n, *nDev);
    extern __shared__ __align__(1024) unsigned char smem[];
    unsigned char* wt = smem;                                 // W_0..W_4, core-matrix layout
    unsigned char* at = smem + kTcWBytes;                     // activation tile A
    uint64_t* mbar = reinterpret_cast<uint64_t*>(at + kTcATile);
    uint32_t* tslot = reinterpret_cast<uint32_t*>(at + kTcATile + 8);
    const uint32_t tid = threadIdx.x, warp = tid >> 5;

    // weights: packed [out][in] bf16 -> core-matrix layout, 16 bytes at a time
    for (int l = 0; l < kLayers; ++l) {
        const uint4* src = reinterpret_cast<const uint4*>(g.W + layer_offset(l));
        const int chunks = layer_out(l) * (kIn / 8);
        for (int i = tid; i < chunks; i += kTcRows) {
            const uint32_t row = (uint32_t)(i / (kIn / 8)), c = (uint32_t)(i % (kIn / 8));
            *reinterpret_cast<uint4*>(wt + tc_w_offset(l) + tc_offset(row, 8 * c)) = src[i];
        }
    }
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(mbar)) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(tslot)),
                     "r"(kTcCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    tc_sync();
    const uint32_t tmem = *tslot;
    const uint32_t mb = smem_addr(mbar);
    const uint32_t aBase = smem_addr(at), wBase = smem_addr(wt);
    const uint32_t myLane = tmem + ((warp * 32u) << 16);      // this warp's 32 lanes
    uint32_t phase = 0;
    bool failed = false;
    const uint32_t tiles = (n + kTcRows - 1) / kTcRows;
    for (uint32_t tile = blockIdx.x; tile < tiles && !failed; tile += gridDim.x) {
        const uint32_t i = tile * kTcRows + tid;
        {
            __align__(16) __nv_bfloat16 row[kIn];
            if (i < n) {
                encode_row(g, q[i], row);
            } else {
#pragma unroll
                for (int k = 0; k < kIn; ++k) row[k] = bf(0.0f);
            }
#pragma unroll
            for (int c = 0; c < kIn / 8; ++c)
                *reinterpret_cast<uint4*>(at + tc_offset(tid, 8 * c)) = *reinterpret_cast<const uint4*>(row + 8 * c);
        }
        for (int l = 0; l < kLayers && !failed; ++l) {
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // A visible to the tensor cores
            tc_sync();
            const int nOut = layer_out(l);
            if (tid == 0) {
                const uint32_t idesc = tc_idesc(kTcRows, nOut);
#pragma unroll
                for (int ks = 0; ks < kIn / 16; ++ks)
                    tc_mma(tmem, tc_desc(aBase + ks * 2 * kTcLbo), tc_desc(wBase + tc_w_offset(l) + ks * 2 * kTcLbo),
                           idesc, ks > 0 ? 1u : 0u);
                tc_commit(mb);
            }
            uint32_t tries = 0;
            bool late = false;
            while (!mbar_try_wait(mb, phase))
                if (++tries >= kTcWaitLimit) {
                    late = true;
                    break;
                }
            phase ^= 1u;
            // one decision for the whole CTA: the loads below are warp-collective
            failed = __syncthreads_or(late) != 0;
            if (failed) break;
            tc_fence_after();
            if (l < kLayers - 1) {
#pragma unroll
                for (int c16 = 0; c16 < kHidden / 16; ++c16) {
                    float v[16];
                    tc_ld16(myLane + 16u * c16, v);
                    uint4 lo, hi;
                    lo.x = pack_bf2(fmaxf(v[0], 0.0f), fmaxf(v[1], 0.0f));
                    lo.y = pack_bf2(fmaxf(v[2], 0.0f), fmaxf(v[3], 0.0f));
                    lo.z = pack_bf2(fmaxf(v[4], 0.0f), fmaxf(v[5], 0.0f));
                    lo.w = pack_bf2(fmaxf(v[6], 0.0f), fmaxf(v[7], 0.0f));
                    hi.x = pack_bf2(fmaxf(v[8], 0.0f), fmaxf(v[9], 0.0f));
                    hi.y = pack_bf2(fmaxf(v[10], 0.0f), fmaxf(v[11], 0.0f));
                    hi.z = pack_bf2(fmaxf(v[12], 0.0f), fmaxf(v[13], 0.0f));
                    hi.w = pack_bf2(fmaxf(v[14], 0.0f), fmaxf(v[15], 0.0f));
                    // the MMAs reading A have completed (mbarrier), so A is rewritten in place
                    *reinterpret_cast<uint4*>(at + tc_offset(tid, 16 * c16)) = lo;
                    *reinterpret_cast<uint4*>(at + tc_offset(tid, 16 * c16 + 8)) = hi;
                }
            } else {
                float r[48];  // columns 0..47; 0..39 are the mixture
#pragma unroll
                for (int c16 = 0; c16 < 3; ++c16) {
                    float v[16];
                    tc_ld16(myLane + 16u * c16, v);
#pragma unroll
                    for (int k = 0; k < 16; ++k) r[16 * c16 + k] = v[k];
                }
                if (i < n) {
                    if (packed) {
                        pack_mixture(r, raw + i, nMax);
                    } else {
#pragma unroll
                        for (int k = 0; k < 40; k += 4)
                            *reinterpret_cast<float4*>(raw + (uint64_t)i * 40 + k) =
                                make_float4(r[k], r[k + 1], r[k + 2], r[k + 3]);
                    }
                }
            }
        }
        tc_sync();  // tensor memory read by every warp before the next tile's MMAs
    }
    if (failed && status) atomicOr(status, kErrTensorWait);
    tc_sync();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTcCols) : "memory");
}

// Training, in two kernels per slice of at most kTrainSlice samples.
//
// k_train_rows: one warp per 32 samples runs the encoding and the forward
// pass (keeping every layer's input in shared memory), the mixture's output
// gradient, and the backward data pass through the layers (dX = dY W_l,
// then ReLU'). It scatters the grid gradients with float2 atomics, and
// writes, for the weight gradients, every layer's input X_l and output
// gradient dY_l transposed: XT[l][k][s] and DT[l][m][s] (bf16, s = sample
// of the slice, rows kTrainSlice long).
//
// k_dw: dW_l = dY_l^T X_l over the slice, one warp per (layer, 16-row tile
// of dW_l, split of the samples), with the mma tiles reading XT and DT
// directly; each split writes its own partial dW, summed in fixed order by
// k_reduce_dw. Sample i of the slice is s[offset + i * stride].
constexpr uint32_t kTrainSlice = 16384;
constexpr int kTrainRowWarps = 2;
constexpr uint32_t kDwSplits = 32;
constexpr int kDwTasks = (kLayers - 1) * (kHidden / 16) + kOut / 16;  // (layer, 16-row tile) pairs: 19

// Columns 0..cols-1 of a warp's [32][kLd] bf16 tile, transposed into dst
// (dst[c * ld + r], rows of the tile are consecutive samples): two columns
// per instruction, each lane storing a pair of samples.
AG_D void store_transposed(const __nv_bfloat16* src, int cols, __nv_bfloat16* dst, uint32_t ld)
{
    const int lane = threadIdx.x & 31, pr = lane & 15, half = lane >> 4;
    for (int c0 = 0; c0 < cols; c0 += 2) {
        const int c = c0 + half;
        __nv_bfloat162 v;
        v.x = src[(2 * pr) * kLd + c];
        v.y = src[(2 * pr + 1) * kLd + c];
        *reinterpret_cast<__nv_bfloat162*>(dst + (uint64_t)c * ld + 2 * pr) = v;
    }
}

size_t train_rows_smem()
{
    // padded weights + per warp: G0 [32][kLd] followed by the inputs of the kLayers layers
    return (size_t)kWsm * 2 + (size_t)kTrainRowWarps * (kLayers + 1) * 32 * kLd * 2;
}

__global__ void __launch_bounds__(32 * kTrainRowWarps) k_train_rows(Params g, const Sample* __restrict__ s, uint32_t n,
                                                                  uint32_t offset, uint32_t stride, float invBatch,
                                                                  __nv_bfloat16* __restrict__ XT,
                                                                  __nv_bfloat16* __restrict__ DT,
                                                                  float* __restrict__ dGrid, float* __restrict__ loss)
{
    extern __shared__ __align__(16) unsigned char smem[];
    __nv_bfloat16* W = reinterpret_cast<__nv_bfloat16*>(smem);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g4 = lane >> 2, t4 = lane & 3;
    __nv_bfloat16* G0 = W + kWsm + warp * (kLayers + 1) * 32 * kLd;  // [32][kLd] gradient dY of the current layer
    __nv_bfloat16* saved = G0 + 32 * kLd;                              // [kLayers][32][kLd] layer inputs
    // outputs in fp32 over G0 and saved[0] (X_0 is in XT by then)
    float* outF = reinterpret_cast<float*>(G0);                        // [32][kOut]
    static_assert(32 * kOut * 4 <= 2 * 32 * kLd * 2, "output tile fits G0 + saved[0]");
    // grid-feature gradients over saved[1] (X_1 has served its ReLU' by then)
    float* dIn = reinterpret_cast<float*>(saved + 32 * kLd);           // [32][kGridDims]
    static_assert(32 * kGridDims * 4 <= 32 * kLd * 2, "grid-feature gradients fit saved[1]");
    load_weights(g.W, W);
    __syncthreads();
    float lossSum = 0.0f;
    const uint32_t ch = blockIdx.x * kTrainRowWarps + warp;
    if (ch * 32 < n) {
        const uint32_t row0 = ch * 32, i = row0 + lane;
        const bool valid = i < n;
        Sample smp;
        if (valid) {
            smp = s[offset + (uint64_t)i * stride];
            encode_row(g, smp.q, saved + lane * kLd);
        } else {
            for (int k = 0; k < kIn; ++k) saved[lane * kLd + k] = bf(0.0f);
        }
        __syncwarp();
        hidden_layers(W, saved, saved);
        for (int l = 0; l < kLayers; ++l)
            store_transposed(saved + l * 32 * kLd, kIn, XT + (uint64_t)l * kHidden * kTrainSlice + row0, kTrainSlice);
        {
            float acc[2][kOut / 8][4];
            warp_layer<kOut, kHidden>(saved + (kLayers - 1) * 32 * kLd, W + wsm_offset(kLayers - 1),
                                      wld(kLayers - 1), acc);
            __syncwarp();  // X_0 (under outF) has been stored by every lane
#pragma unroll
            for (int mt = 0; mt < 2; ++mt)
#pragma unroll
                for (int nt = 0; nt < kOut / 8; ++nt) {
                    const int r = mt * 16 + g4, col = nt * 8 + 2 * t4;
                    *reinterpret_cast<float2*>(outF + r * kOut + col) = make_float2(acc[mt][nt][0], acc[mt][nt][1]);
                    *reinterpret_cast<float2*>(outF + (r + 8) * kOut + col) = make_float2(acc[mt][nt][2], acc[mt][nt][3]);
                }
        }
        __syncwarp();
        // output gradient (lane = sample)
        {
            float raw[40], grad[40];
            for (int k = 0; k < 40; ++k) raw[k] = outF[lane * kOut + k];
            if (valid) {
                const float3 dir = mk3(smp.dir[0], smp.dir[1], smp.dir[2]);
                const float w = smp.weight * invBatch;
                mixture_grad(raw, dir, w, grad);
                Mixture m;
                decode_mixture(raw, m);
                lossSum += -w * logf(fmaxf(mixture_pdf(m, dir), 1e-30f));
            } else {
                for (int k = 0; k < 40; ++k) grad[k] = 0.0f;
            }
            __syncwarp();  // every lane has read its outputs
            for (int k = 0; k < kOut; ++k) G0[lane * kLd + k] = bf(k < 40 ? grad[k] : 0.0f);
        }
        __syncwarp();
        store_transposed(G0, kOut, DT + (uint64_t)(kLayers - 1) * kHidden * kTrainSlice + row0, kTrainSlice);
        // backward: G0 holds dY_l; dX_l = dY_l W_l, dY_{l-1} = dX_l * [X_l > 0]
        for (int l = kLayers - 1; l >= 1; --l) {
            const __nv_bfloat16* Xl = saved + l * 32 * kLd;
            const __nv_bfloat16* WTl = g.WT + layer_offset(l);
            float acc[2][kHidden / 8][4];
            if (l == kLayers - 1) warp_layer<kHidden, kOut>(G0, WTl, kOut, acc);
            else warp_layer<kHidden, kHidden>(G0, WTl, kHidden, acc);
            __syncwarp();
#pragma unroll
            for (int mt = 0; mt < 2; ++mt)
#pragma unroll
                for (int nt = 0; nt < kHidden / 8; ++nt) {
                    const int r = mt * 16 + g4, c = nt * 8 + 2 * t4;
                    const __nv_bfloat162 x0 = *reinterpret_cast<const __nv_bfloat162*>(Xl + r * kLd + c);
                    const __nv_bfloat162 x1 = *reinterpret_cast<const __nv_bfloat162*>(Xl + (r + 8) * kLd + c);
                    *reinterpret_cast<uint32_t*>(G0 + r * kLd + c) =
                        pack_bf2(fl(x0.x) > 0.0f ? acc[mt][nt][0] : 0.0f, fl(x0.y) > 0.0f ? acc[mt][nt][1] : 0.0f);
                    *reinterpret_cast<uint32_t*>(G0 + (r + 8) * kLd + c) =
                        pack_bf2(fl(x1.x) > 0.0f ? acc[mt][nt][2] : 0.0f, fl(x1.y) > 0.0f ? acc[mt][nt][3] : 0.0f);
                }
            __syncwarp();
            store_transposed(G0, kHidden, DT + (uint64_t)(l - 1) * kHidden * kTrainSlice + row0, kTrainSlice);
        }
        // grid-feature gradients: dX0[s][k] = sum_m dY_0[s][m] W_0[m][k], k < kGridDims
        warp_gemm<32, kGridDims, kHidden>(G0, kLd, g.WT + layer_offset(0), layer_out(0),
                                          [&](int r, int c, float v) { dIn[r * kGridDims + c] = v; });
        __syncwarp();
        if (valid) {
            const float3 p = normalise_position(g, mk3(smp.q.pos[0], smp.q.pos[1], smp.q.pos[2]));
            for (int lv = 0; lv < kLevels; ++lv) {
                float d[kFeatures];
#pragma unroll
                for (int k = 0; k < kFeatures; ++k) d[k] = dIn[lane * kGridDims + kFeatures * lv + k];
#pragma unroll
                for (int c = 0; c < 8; ++c) {
                    uint32_t idx;
                    float w;
                    grid_corner(g.res[lv], p, c, idx, w);
                    float2* dst = reinterpret_cast<float2*>(dGrid + ((uint64_t)lv * kTableSize + idx) * kFeatures);
#pragma unroll
                    for (int k = 0; k < kFeatures / 2; ++k) atomicAdd(dst + k, make_float2(w * d[2 * k], w * d[2 * k + 1]));
                }
            }
        }
    }
    for (int o = 16; o; o >>= 1) lossSum += __shfl_xor_sync(0xffffffffu, lossSum, o);
    if (lane == 0 && loss && lossSum != 0.0f) atomicAdd(loss, lossSum);
}

// One warp: rows 16 mt .. 16 mt + 15 of dW_l over the samples of its split
// (k-steps of 16 samples; the slice's last partial 32-sample chunk is zero
// padded by k_train_rows), written to partial[split].
__global__ void __launch_bounds__(32) k_dw(const __nv_bfloat16* __restrict__ XT, const __nv_bfloat16* __restrict__ DT,
                                          uint32_t n, float* __restrict__ partial)
{
    int task = blockIdx.y, l = 0;
    while (l < kLayers - 1 && task >= kHidden / 16) {
        task -= kHidden / 16;
        ++l;
    }
    const int mt = task;
    const uint32_t split = blockIdx.x, splits = gridDim.x;
    const uint32_t ksteps = (n + 15) / 16, per = (ksteps + splits - 1) / splits;
    const uint32_t k0 = split * per, k1 = min(ksteps, k0 + per);
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    const __nv_bfloat16* A = DT + ((uint64_t)l * kHidden + mt * 16) * kTrainSlice;  // dY_l^T rows
    const __nv_bfloat16* B = XT + (uint64_t)l * kHidden * kTrainSlice;              // X_l^T rows
    float c[kHidden / 8][4] = {};
    for (uint32_t ks = k0; ks < k1; ++ks) {
        const uint32_t k = ks * 16 + 2 * t;
        const __nv_bfloat16* a = A + (uint64_t)g * kTrainSlice + k;
        const uint32_t a0 = ld32(a), a1 = ld32(a + 8 * kTrainSlice), a2 = ld32(a + 8), a3 = ld32(a + 8 * kTrainSlice + 8);
#pragma unroll
        for (int nt = 0; nt < kHidden / 8; ++nt) {
            const __nv_bfloat16* b = B + (uint64_t)(nt * 8 + g) * kTrainSlice + k;
            mma_bf16(c[nt], a0, a1, a2, a3, ld32(b), ld32(b + 8));
        }
    }
    float* out = partial + (uint64_t)split * kWeightCount + layer_offset(l);
    const int inDim = layer_in(l);
#pragma unroll
    for (int nt = 0; nt < kHidden / 8; ++nt) {
        const int r = mt * 16 + g, col = nt * 8 + 2 * t;
        *reinterpret_cast<float2*>(out + r * inDim + col) = make_float2(c[nt][0], c[nt][1]);
        *reinterpret_cast<float2*>(out + (r + 8) * inDim + col) = make_float2(c[nt][2], c[nt][3]);
    }
}

// k_dw_tc: the same product on the 5th-generation tensor cores. One CTA of
// 128 threads per (split of the samples, layer) accumulates
// dW_l = dY_l^T X_l in tensor memory over chunks of 64 samples: A = dY_l^T
// (the layer's output rows, zero-padded to M = 128 so that the accumulator
// has the lane-per-row layout of k_infer_tc) and B = X_l^T (N = 64 input
// rows), both K-major over the samples in the no-swizzle core-matrix
// layout. The chunks stream through kDwTcStages shared-memory stages:
// cp.async copies (16 bytes, zero-filled past n) run kDwTcStages - 1 chunks
// ahead of the MMAs, one elected thread issues each chunk's four
// tcgen05.mma (K = 16) and commits them to the stage's mbarrier, and a
// stage is refilled only after that mbarrier says the MMAs that read it are
// done. Warps 0 and 1 then read rows 0..63 back (tcgen05.ld) into the
// split's partial dW, summed by k_reduce_dw like k_dw's. Every wait is
// bounded: a CTA that runs out records kErrTensorWait, writes nothing,
// waits for its own copies and still frees its tensor memory.
constexpr int kDwTcChunk = 64;                                   // samples per stage (K)
constexpr int kDwTcStages = 4;
constexpr int kDwTcATile = kTcRows * kDwTcChunk * 2;             // 16 KiB
constexpr int kDwTcBTile = kHidden * kDwTcChunk * 2;             // 8 KiB
constexpr int kDwTcStage = kDwTcATile + kDwTcBTile;
constexpr int kDwTcSmem = kDwTcStages * kDwTcStage + kDwTcStages * 8 + 8;  // + mbarriers + tensor-memory address
static_assert(kTrainSlice % kDwTcChunk == 0, "whole chunks per slice");
static_assert(kDwTcStage % 1024 == 0, "stages keep the operand tiles' alignment");

// 16 bytes from global to shared memory, asynchronously; bytes past `bytes`
// (0..16) are written as zeros and not read.
AG_D void cp_async16(uint32_t dst, const void* src, uint32_t bytes)
{
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src), "r"(bytes) : "memory");
}
AG_D void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N> AG_D void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

__global__ void __launch_bounds__(kTcRows) k_dw_tc(const __nv_bfloat16* __restrict__ XT,
                                                   const __nv_bfloat16* __restrict__ DT, uint32_t n,
                                                   float* __restrict__ partial, uint32_t* __restrict__ status)
{
    extern __shared__ __align__(1024) unsigned char smem[];
    uint64_t* mbar = reinterpret_cast<uint64_t*>(smem + kDwTcStages * kDwTcStage);
    uint32_t* tslot = reinterpret_cast<uint32_t*>(mbar + kDwTcStages);
    const uint32_t tid = threadIdx.x, warp = tid >> 5;
    const int l = blockIdx.y;
    const int rows = layer_out(l);
    const uint32_t split = blockIdx.x, splits = gridDim.x;
    const uint32_t chunks = (n + kDwTcChunk - 1) / kDwTcChunk, per = (chunks + splits - 1) / splits;
    const uint32_t c0 = min(chunks, split * per), cnt = min(chunks, c0 + per) - c0;
    const __nv_bfloat16* A = DT + (uint64_t)l * kHidden * kTrainSlice;  // row m: dY_l[., m] over the samples
    const __nv_bfloat16* B = XT + (uint64_t)l * kHidden * kTrainSlice;  // row k: X_l[., k]
    const uint32_t sBase = smem_addr(smem);

    // the padding rows of every stage's A (rows .. 127) stay zero for the whole kernel
    for (int i = tid; i < kDwTcStages * (kTcRows - rows) * (kDwTcChunk / 8); i += kTcRows) {
        const int st = i / ((kTcRows - rows) * (kDwTcChunk / 8)), j = i % ((kTcRows - rows) * (kDwTcChunk / 8));
        const uint32_t row = (uint32_t)(rows + j / (kDwTcChunk / 8)), c = (uint32_t)(j % (kDwTcChunk / 8));
        *reinterpret_cast<uint4*>(smem + st * kDwTcStage + tc_offset(row, 8 * c)) = make_uint4(0u, 0u, 0u, 0u);
    }
    if (tid == 0) {
        for (int st = 0; st < kDwTcStages; ++st)
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(mbar + st)) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(tslot)),
                     "r"(kTcCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    // chunk j (of this split) into stage j % kDwTcStages
    auto load = [&](uint32_t j) {
        const uint32_t sbase = (c0 + j) * kDwTcChunk;
        const uint32_t at = sBase + (j % kDwTcStages) * kDwTcStage, bt = at + kDwTcATile;
        for (int i = tid; i < (rows + kHidden) * (kDwTcChunk / 8); i += kTcRows) {
            const bool isA = i < rows * (kDwTcChunk / 8);
            const int k = isA ? i : i - rows * (kDwTcChunk / 8);
            const uint32_t row = (uint32_t)(k / (kDwTcChunk / 8)), s0 = sbase + 8 * (uint32_t)(k % (kDwTcChunk / 8));
            const uint32_t bytes = s0 >= n ? 0u : min(16u, (n - s0) * 2u);
            cp_async16((isA ? at : bt) + tc_offset(row, s0 - sbase), (isA ? A : B) + (uint64_t)row * kTrainSlice + s0,
                       bytes);
        }
    };
    // bounded wait for the MMAs of chunk j
    auto wait_mma = [&](uint32_t j) -> bool {
        const uint32_t mb = smem_addr(mbar + j % kDwTcStages), parity = (j / kDwTcStages) & 1u;
        for (uint32_t tries = 0; !mbar_try_wait(mb, parity);)
            if (++tries >= kTcWaitLimit) return false;
        return true;
    };
#pragma unroll
    for (int j = 0; j < kDwTcStages - 1; ++j) {
        if ((uint32_t)j < cnt) load(j);
        cp_async_commit();
    }
    tc_sync();
    const uint32_t tmem = *tslot;
    const uint32_t idesc = tc_idesc(kTcRows, kHidden);
    bool late = false, failed = false;
    for (uint32_t j = 0; j < cnt; ++j) {
        cp_async_wait<kDwTcStages - 2>();                             // chunk j has landed (this thread's copies)
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // visible to the tensor cores
        tc_fence_before();
        failed = __syncthreads_or(late) != 0;
        tc_fence_after();
        if (failed) break;
        if (tid == 0) {
            const uint32_t at = sBase + (j % kDwTcStages) * kDwTcStage, bt = at + kDwTcATile;
#pragma unroll
            for (int ks = 0; ks < kDwTcChunk / 16; ++ks)
                tc_mma(tmem, tc_desc(at + ks * 2 * kTcLbo), tc_desc(bt + ks * 2 * kTcLbo), idesc,
                       (j > 0 || ks > 0) ? 1u : 0u);
            tc_commit(smem_addr(mbar + j % kDwTcStages));
        }
        // refill the stage that chunk j - 1 read with chunk j + kDwTcStages - 1
        const uint32_t next = j + kDwTcStages - 1;
        if (next < cnt) {
            if (j >= 1 && !wait_mma(j - 1)) late = true;
            if (!late) load(next);
        }
        cp_async_commit();
    }
    // the MMAs of the last chunks (the earlier ones were waited for above)
    if (!failed)
        for (uint32_t j = cnt > (uint32_t)kDwTcStages ? cnt - kDwTcStages : 0u; j < cnt; ++j)
            if (!wait_mma(j)) late = true;
    cp_async_wait<0>();
    tc_fence_before();
    failed = __syncthreads_or(late || failed) != 0;
    tc_fence_after();
    if (!failed) {
        const int inDim = layer_in(l);
        float* out = partial + (uint64_t)split * kWeightCount + layer_offset(l);
        if (warp < 2) {  // rows 0..63 live in lanes 0..63 (warps 0 and 1)
            const uint32_t lane = tmem + ((warp * 32u) << 16);
            const int row = (int)(warp * 32 + (tid & 31));
#pragma unroll
            for (int c16 = 0; c16 < kHidden / 16; ++c16) {
                float v[16];
                tc_ld16(lane + 16u * c16, v);
                if (row < rows)
#pragma unroll
                    for (int k = 0; k < 16; k += 4)
                        *reinterpret_cast<float4*>(out + row * inDim + 16 * c16 + k) =
                            cnt ? make_float4(v[k], v[k + 1], v[k + 2], v[k + 3]) : make_float4(0.f, 0.f, 0.f, 0.f);
            }
        }
    } else if (status && tid == 0) {
        atomicOr(status, kErrTensorWait);
    }
    tc_sync();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTcCols) : "memory");
}

// dW[i] += sum over blocks of the blocks' partial dW (fixed order).
__global__ void k_reduce_dw(const float* __restrict__ partial, uint32_t blocks, float* __restrict__ dW)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (uint32_t)kWeightCount) return;
    float sum = 0.0f;
    for (uint32_t b = 0; b < blocks; ++b) sum += partial[(uint64_t)b * kWeightCount + i];
    dW[i] += sum;
}

// Adam (Kingma & Ba 2015) on fp32 master parameters; writes the compute copies.
__global__ void k_adam_weights(float* p, float* m, float* v, float* grad, uint32_t n, float lr, float b1, float b2,
                               float eps, float c1, float c2, __nv_bfloat16* W, __nv_bfloat16* WT)
{
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float gr = grad[i];
    float mi = b1 * m[i] + (1.0f - b1) * gr;
    float vi = b2 * v[i] + (1.0f - b2) * gr * gr;
    m[i] = mi;
    v[i] = vi;
    float pi = p[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    p[i] = pi;
    grad[i] = 0.0f;
    // locate (layer, out, in) for the transposed copy
    int l = 0;
    while (l < kLayers - 1 && (int)i >= layer_offset(l + 1)) ++l;
    int local = (int)i - layer_offset(l);
    int o = local / layer_in(l), in = local % layer_in(l);
    W[i] = __float2bfloat16_rn(pi);
    WT[layer_offset(l) + in * layer_out(l) + o] = __float2bfloat16_rn(pi);
}

// Adam on the grid, lazily: an entry is updated only in the steps in which
// its gradient is non-zero, i.e. some sample of the batch interpolated from
// it (the sparse rule of Mueller et al. 2022 for hash tables). Four entries
// per thread; groups without a gradient cost one 16-byte read. Against
// updating every entry with non-zero momentum, this measured 48 against
// 111 us per step and the same samples to a given error.
__global__ void k_adam_grid(float* p, float* m, float* v, float* grad, uint64_t n4, float lr, float b1, float b2,
                            float eps, float c1, float c2, __half* h)
{
    const uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (i >= n4) return;
    const float4 g4 = reinterpret_cast<const float4*>(grad)[i];
    if (g4.x == 0.0f && g4.y == 0.0f && g4.z == 0.0f && g4.w == 0.0f) return;
    const float gs[4] = {g4.x, g4.y, g4.z, g4.w};
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const uint64_t j = 4 * i + k;
        const float gr = gs[k];
        if (gr == 0.0f) continue;
        const float mi = b1 * m[j] + (1.0f - b1) * gr;
        const float vi = b2 * v[j] + (1.0f - b2) * gr * gr;
        m[j] = mi;
        v[j] = vi;
        const float pi = p[j] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
        p[j] = pi;
        h[j] = __float2half_rn(pi);
    }
    reinterpret_cast<float4*>(grad)[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
}

__global__ void k_publish(const float* pw, uint32_t nw, __nv_bfloat16* W, __nv_bfloat16* WT, const float* pg,
                          uint64_t ng, __half* h)
{
    uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (i < nw) {
        int l = 0;
        while (l < kLayers - 1 && (int)i >= layer_offset(l + 1)) ++l;
        int local = (int)i - layer_offset(l);
        int o = local / layer_in(l), in = local % layer_in(l);
        W[i] = __float2bfloat16_rn(pw[i]);
        WT[layer_offset(l) + in * layer_out(l) + o] = __float2bfloat16_rn(pw[i]);
    }
    if (i < ng) h[i] = __float2half_rn(pg[i]);
}

// Grid parameters uniform in [-1e-4, 1e-4], from a hash of (seed, index).
__global__ void k_init_grid(float* p, uint64_t n, uint64_t seed)
{
    const uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint64_t h = splitmix64(seed * 0x9e3779b97f4a7c15ull + i);
    p[i] = (2.0f * ((float)(h >> 40) * (1.0f / 16777216.0f)) - 1.0f) * 1e-4f;
}

size_t infer_smem() { return (size_t)kWsm * 2 + (size_t)kInferWarps * 32 * kLd * 2; }

uint64_t splitmix(uint64_t& s)
{
    uint64_t z = (s += 0x9e3779b97f4a7c15ull);
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}
float uniform(uint64_t& s) { return (float)(splitmix(s) >> 40) * (1.0f / 16777216.0f); }

}  // namespace

Guide::~Guide() { release(); }

void Guide::release()
{
    if (mem_) cudaFree(mem_);
    mem_ = nullptr;
    ready_ = false;
}

bool Guide::allocate()
{
    if (mem_) return true;
    size_t bytes = 0;
    bytes += 4 * kGridParams * sizeof(float);             // grid master, m, v, grad
    bytes += kGridParams * sizeof(__half);                // grid compute copy
    bytes += 4 * (size_t)kWeightCount * sizeof(float);    // W master, m, v, grad
    bytes += 2 * (size_t)kWeightCount * sizeof(__nv_bfloat16);
    bytes += (size_t)kDwSplits * kWeightCount * sizeof(float);        // per-split dW partials
    bytes += 2 * (size_t)kLayers * kHidden * kTrainSlice * sizeof(__nv_bfloat16);  // XT, DT
    bytes += 256 * 8;
    if (cudaMalloc(&mem_, bytes) != cudaSuccess) {
        cudaGetLastError();
        mem_ = nullptr;
        return false;
    }
    char* p = static_cast<char*>(mem_);
    auto take = [&](size_t b) {
        char* r = p;
        p += (b + 255) & ~size_t(255);
        return r;
    };
    gridP_ = (float*)take(kGridParams * 4);
    gridM_ = (float*)take(kGridParams * 4);
    gridV_ = (float*)take(kGridParams * 4);
    gridG_ = (float*)take(kGridParams * 4);
    gridH_ = (__half*)take(kGridParams * 2);
    wP_ = (float*)take(kWeightCount * 4);
    wM_ = (float*)take(kWeightCount * 4);
    wV_ = (float*)take(kWeightCount * 4);
    wG_ = (float*)take(kWeightCount * 4);
    wB_ = (__nv_bfloat16*)take(kWeightCount * 2);
    wT_ = (__nv_bfloat16*)take(kWeightCount * 2);
    partial_ = (float*)take((size_t)kDwSplits * kWeightCount * 4);
    xt_ = (__nv_bfloat16*)take((size_t)kLayers * kHidden * kTrainSlice * 2);
    dt_ = (__nv_bfloat16*)take((size_t)kLayers * kHidden * kTrainSlice * 2);
    loss_ = (float*)take(256);
    return true;
}

int Guide::reset(uint32_t seed, cudaStream_t st)
{
    if (!allocate()) return -5;
    // He-uniform weights, small uniform grid (deterministic in the seed)
    std::vector<float> w(kWeightCount);
    uint64_t s = 0x5eed0000ull + seed;
    for (int l = 0; l < kLayers; ++l) {
        float a = std::sqrt(6.0f / (float)layer_in(l));
        for (int i = 0; i < layer_out(l) * layer_in(l); ++i) w[layer_offset(l) + i] = (2.0f * uniform(s) - 1.0f) * a;
    }
    cudaError_t e = cudaMemcpyAsync(wP_, w.data(), w.size() * 4, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) {
        k_init_grid<<<(unsigned)((kGridParams + 255) / 256), 256, 0, st>>>(gridP_, kGridParams, 0x6d1d0000ull + seed);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemsetAsync(wM_, 0, kWeightCount * 4, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(wV_, 0, kWeightCount * 4, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(wG_, 0, kWeightCount * 4, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(gridM_, 0, kGridParams * 4, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(gridV_, 0, kGridParams * 4, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(gridG_, 0, kGridParams * 4, st);
    if (e != cudaSuccess) return -2;
    publish(st);
    step_ = 0;
    e = cudaStreamSynchronize(st);
    ready_ = e == cudaSuccess;
    return ready_ ? 0 : -2;
}

void Guide::publish(cudaStream_t st)
{
    uint64_t n = kGridParams > (uint64_t)kWeightCount ? kGridParams : (uint64_t)kWeightCount;
    k_publish<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(wP_, kWeightCount, wB_, wT_, gridP_, kGridParams, gridH_);
}

void Guide::set_scene_box(float3 lo, float3 hi)
{
    bmin_ = lo;
    float3 e = hi - lo;
    float m = fmaxf(e.x, fmaxf(e.y, e.z));
    m = m > 0.0f ? m * 1.0001f : 1.0f;
    invExtent_ = mk3(1.0f / m, 1.0f / m, 1.0f / m);  // isotropic: cells stay cubic
}

Params Guide::params() const
{
    Params p;
    p.grid = gridH_;
    p.W = wB_;
    p.WT = wT_;
    p.bmin = bmin_;
    p.invExtent = invExtent_;
    double b = std::exp((std::log((double)kMaxRes) - std::log((double)kMinRes)) / (kLevels - 1));
    for (int l = 0; l < kLevels; ++l) p.res[l] = (uint32_t)std::floor(kMinRes * std::pow(b, l));
    return p;
}

void Guide::infer(const Query* q, uint32_t n, float* raw, cudaStream_t st, uint32_t* status) const
{
    infer_queue(q, nullptr, n, raw, st, status);
}

void Guide::infer_queue(const Query* q, const uint32_t* count, uint32_t maxN, float* out, cudaStream_t st,
                        uint32_t* status, bool packed) const
{
    if (maxN == 0) return;
    if (kernel_ == kKernelTensorMemory) {
        cudaFuncSetAttribute(k_infer_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, kTcSmem);
        uint32_t tiles = (maxN + kTcRows - 1) / kTcRows;
        int dev = 0, sms = 148;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        // four CTAs per SM: 4 x 55 KB of shared memory, 4 x 64 of the 512 tensor-memory columns
        const uint32_t blocks = std::min<uint32_t>(tiles, 4u * (uint32_t)sms);
        k_infer_tc<<<blocks, kTcRows, kTcSmem, st>>>(params(), q, maxN, count, out, status, packed);
        return;
    }
    // per call: the attribute belongs to the current device
    cudaFuncSetAttribute(k_infer, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)infer_smem());
    uint32_t chunks = (maxN + 31) / 32;
    uint32_t blocks = (chunks + kInferWarps - 1) / kInferWarps;
    if (blocks > 148 * 2) blocks = 148 * 2;  // two resident blocks per SM; each loads the weights once
    k_infer<<<blocks, 32 * kInferWarps, infer_smem(), st>>>(params(), q, maxN, count, out, packed);
}

void Guide::accumulate_gradients(const Sample* s, uint32_t n, float invBatch, cudaStream_t st, uint32_t offset,
                                 uint32_t stride, uint32_t* status)
{
    cudaFuncSetAttribute(k_train_rows, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)train_rows_smem());
    for (uint32_t start = 0; start < n; start += kTrainSlice) {
        const uint32_t m = std::min(kTrainSlice, n - start);
        const uint32_t chunks = (m + 31) / 32;
        k_train_rows<<<(chunks + kTrainRowWarps - 1) / kTrainRowWarps, 32 * kTrainRowWarps, train_rows_smem(), st>>>(
            params(), s, m, offset + start * stride, stride, invBatch, xt_, dt_, gridG_, loss_);
        if (gradKernel_ == kKernelTensorMemory) {
            cudaFuncSetAttribute(k_dw_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, kDwTcSmem);
            const uint32_t splits = std::min(kDwSplits, (m + kDwTcChunk - 1) / kDwTcChunk);
            k_dw_tc<<<dim3(splits, kLayers), kTcRows, kDwTcSmem, st>>>(xt_, dt_, m, partial_, status);
            k_reduce_dw<<<(kWeightCount + 255) / 256, 256, 0, st>>>(partial_, splits, wG_);
        } else {
            const uint32_t splits = std::min(kDwSplits, (m + 15) / 16);
            k_dw<<<dim3(splits, kDwTasks), 32, 0, st>>>(xt_, dt_, m, partial_);
            k_reduce_dw<<<(kWeightCount + 255) / 256, 256, 0, st>>>(partial_, splits, wG_);
        }
    }
}

void Guide::apply_adam(float lr, cudaStream_t st)
{
    ++step_;
    const float b1 = 0.9f, b2 = 0.99f, eps = 1e-8f;
    float c1 = 1.0f - (float)std::pow(b1, step_), c2 = 1.0f - (float)std::pow(b2, step_);
    k_adam_weights<<<(kWeightCount + 255) / 256, 256, 0, st>>>(wP_, wM_, wV_, wG_, kWeightCount, lr, b1, b2, eps, c1,
                                                               c2, wB_, wT_);
    static_assert(kGridParams % 4 == 0, "grid Adam reads gradients four at a time");
    k_adam_grid<<<(unsigned)((kGridParams / 4 + 255) / 256), 256, 0, st>>>(gridP_, gridM_, gridV_, gridG_, kGridParams / 4, lr,
                                                                        b1, b2, eps, c1, c2, gridH_);
}

float Guide::train_step(const Sample* s, uint32_t n, float lr, cudaStream_t st)
{
    cudaMemsetAsync(loss_, 0, 4, st);
    accumulate_gradients(s, n, n ? 1.0f / (float)n : 0.0f, st);
    apply_adam(lr, st);
    float h = 0.0f;
    cudaMemcpyAsync(&h, loss_, 4, cudaMemcpyDeviceToHost, st);
    cudaStreamSynchronize(st);
    return h;
}

}  // namespace guide
}  // namespace ag
