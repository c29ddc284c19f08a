// Learned path guiding: parameters, inference and training kernels (see
// guide.cuh for the model and the published methods it restates).
#include "guide_host.cuh"

#include <cmath>
#include <cstring>
#include <vector>

namespace ag {
namespace guide {
namespace {

constexpr int kInferWarps = 4;
constexpr int kTrainWarps = 2;

AG_D __nv_bfloat16 bf(float x) { return __float2bfloat16_rn(x); }
AG_D float fl(__nv_bfloat16 x) { return __bfloat162float(x); }

// Encodes the 64 inputs of one query into a bf16 row.
AG_D void encode_row(const Params& g, const Query& q, __nv_bfloat16* row)
{
    float3 p = normalise_position(g, mk3(q.pos[0], q.pos[1], q.pos[2]));
    for (int l = 0; l < kLevels; ++l) {
        float f0 = 0.0f, f1 = 0.0f;
        for (int c = 0; c < 8; ++c) {
            uint32_t idx;
            float w;
            grid_corner(g.res[l], p, c, idx, w);
            const __half2 v = *reinterpret_cast<const __half2*>(g.grid + ((uint64_t)l * kTableSize + idx) * kFeatures);
            f0 += w * __low2float(v);
            f1 += w * __high2float(v);
        }
        row[2 * l] = bf(f0);
        row[2 * l + 1] = bf(f1);
    }
    float ex[8];
    extra_inputs(mk3(q.wo[0], q.wo[1], q.wo[2]), mk3(q.n[0], q.n[1], q.n[2]), q.rough, ex);
    for (int k = 0; k < 8; ++k) row[kGridDims + k] = bf(ex[k]);
    for (int k = kGridDims + 8; k < kIn; ++k) row[k] = bf(0.0f);
}

// Forward of one warp's 32 rows. X: [32][64] input rows; ping/pong buffers
// [32][64]; out: [32][48] fp32. saved (optional): the input of every layer.
AG_D void forward32(const __nv_bfloat16* W, __nv_bfloat16* X, __nv_bfloat16* tmp, float* out,
                    __nv_bfloat16* saved)
{
    __nv_bfloat16* cur = X;
    __nv_bfloat16* nxt = tmp;
    for (int l = 0; l < kLayers; ++l) {
        if (saved) {
            __syncwarp();
            for (int i = threadIdx.x & 31; i < 32 * kHidden / 2; i += 32)
                reinterpret_cast<uint32_t*>(saved + l * 32 * kHidden)[i] = reinterpret_cast<const uint32_t*>(cur)[i];
        }
        __syncwarp();
        const __nv_bfloat16* Wl = W + layer_offset(l);
        if (l < kLayers - 1) {
            warp_gemm<32, kHidden, kHidden>(cur, kHidden, Wl, layer_in(l),
                                            [&](int r, int c, float v) { nxt[r * kHidden + c] = bf(fmaxf(v, 0.0f)); });
            __nv_bfloat16* t = cur;
            cur = nxt;
            nxt = t;
        } else {
            warp_gemm<32, kOut, kHidden>(cur, kHidden, Wl, layer_in(l),
                                         [&](int r, int c, float v) { out[r * kOut + c] = v; });
        }
    }
    __syncwarp();
}

// n queries, or *nDev when nDev is not null (a queue length written on the device).
__global__ void __launch_bounds__(32 * kInferWarps) k_infer(Params g, const Query* __restrict__ q, uint32_t n,
                                                          const uint32_t* __restrict__ nDev, float* __restrict__ raw)
{
    if (nDev) n = min(n, *nDev);
    extern __shared__ __align__(16) unsigned char smem[];
    __nv_bfloat16* W = reinterpret_cast<__nv_bfloat16*>(smem);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    unsigned char* wbase = smem + kWeightCount * 2 + warp * (2 * 32 * kHidden * 2 + 32 * kOut * 4);
    __nv_bfloat16* X = reinterpret_cast<__nv_bfloat16*>(wbase);
    __nv_bfloat16* T = X + 32 * kHidden;
    float* out = reinterpret_cast<float*>(T + 32 * kHidden);
    for (int i = threadIdx.x; i < kWeightCount / 2; i += blockDim.x)
        reinterpret_cast<uint32_t*>(W)[i] = reinterpret_cast<const uint32_t*>(g.W)[i];
    __syncthreads();
    const uint32_t chunks = (n + 31) / 32;
    for (uint32_t ch = blockIdx.x * kInferWarps + warp; ch < chunks; ch += gridDim.x * kInferWarps) {
        const uint32_t i = ch * 32 + lane;
        if (i < n) {
            encode_row(g, q[i], X + lane * kHidden);
        } else {
            for (int k = 0; k < kIn; ++k) X[lane * kHidden + k] = bf(0.0f);
        }
        forward32(W, X, T, out, nullptr);
        if (i < n)
            for (int k = 0; k < 40; ++k) raw[(uint64_t)i * 40 + k] = out[lane * kOut + k];
        __syncwarp();
    }
}

// Training: forward with saved activations, mixture gradient, backward with
// tensor cores; dW accumulated per block in shared memory then merged into
// the global gradient with atomics; grid gradients scattered with atomics.
// Sample i of the batch is s[offset + i * stride].
__global__ void __launch_bounds__(32 * kTrainWarps) k_train(Params g, const Sample* __restrict__ s, uint32_t n,
                                                          uint32_t offset, uint32_t stride,
                                                          float invBatch, float* __restrict__ dW,
                                                          float* __restrict__ dGrid, float* __restrict__ loss)
{
    extern __shared__ __align__(16) unsigned char smem[];
    __nv_bfloat16* W = reinterpret_cast<__nv_bfloat16*>(smem);
    float* accW = reinterpret_cast<float*>(smem + kWeightCount * 2);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const size_t perWarp = (size_t)kLayers * 32 * kHidden * 2 + 2 * 32 * kHidden * 2 + 2 * kHidden * 32 * 2;
    unsigned char* wb = smem + kWeightCount * 2 + kWeightCount * 4 + warp * perWarp;
    __nv_bfloat16* saved = reinterpret_cast<__nv_bfloat16*>(wb);       // [5][32][64]
    __nv_bfloat16* G0 = saved + kLayers * 32 * kHidden;                // [32][64]
    __nv_bfloat16* G1 = G0 + 32 * kHidden;                             // [32][64]
    __nv_bfloat16* GT = G1 + 32 * kHidden;                             // [64][32] transposed gradient
    __nv_bfloat16* XT = GT + kHidden * 32;                             // [64][32] transposed input
    float* outF = reinterpret_cast<float*>(G0);                        // [32][48] fp32, aliases G0/G1
    for (int i = threadIdx.x; i < kWeightCount / 2; i += blockDim.x)
        reinterpret_cast<uint32_t*>(W)[i] = reinterpret_cast<const uint32_t*>(g.W)[i];
    for (int i = threadIdx.x; i < kWeightCount; i += blockDim.x) accW[i] = 0.0f;
    __syncthreads();
    float lossSum = 0.0f;
    const uint32_t chunks = (n + 31) / 32;
    for (uint32_t ch = blockIdx.x * kTrainWarps + warp; ch < chunks; ch += gridDim.x * kTrainWarps) {
        const uint32_t i = ch * 32 + lane;
        const bool valid = i < n;
        Sample smp;
        if (valid) smp = s[offset + (uint64_t)i * stride];
        __nv_bfloat16* X0 = saved;  // the encoded input is layer 0's saved input
        if (valid) encode_row(g, smp.q, X0 + lane * kHidden);
        else
            for (int k = 0; k < kIn; ++k) X0[lane * kHidden + k] = bf(0.0f);
        // forward; saved[l] = input of layer l (saved[0] already holds X0)
        {
            __nv_bfloat16* cur = X0;
            for (int l = 0; l < kLayers; ++l) {
                __syncwarp();
                const __nv_bfloat16* Wl = W + layer_offset(l);
                if (l < kLayers - 1) {
                    __nv_bfloat16* nxt = saved + (l + 1) * 32 * kHidden;
                    warp_gemm<32, kHidden, kHidden>(cur, kHidden, Wl, layer_in(l),
                                                    [&](int r, int c, float v) { nxt[r * kHidden + c] = bf(fmaxf(v, 0.0f)); });
                    cur = nxt;
                } else {
                    warp_gemm<32, kOut, kHidden>(cur, kHidden, Wl, layer_in(l),
                                                 [&](int r, int c, float v) { outF[r * kOut + c] = v; });
                }
            }
        }
        __syncwarp();
        // output gradient (lane = sample)
        float raw[40], grad[40];
        for (int k = 0; k < 40; ++k) raw[k] = outF[lane * kOut + k];
        if (valid) {
            float3 dir = mk3(smp.dir[0], smp.dir[1], smp.dir[2]);
            float w = smp.weight * invBatch;
            mixture_grad(raw, dir, w, grad);
            Mixture m;
            decode_mixture(raw, m);
            lossSum += -w * logf(fmaxf(mixture_pdf(m, dir), 1e-30f));
        } else {
            for (int k = 0; k < 40; ++k) grad[k] = 0.0f;
        }
        __syncwarp();
        for (int k = 0; k < kOut; ++k) {
            __nv_bfloat16 v = bf(k < 40 ? grad[k] : 0.0f);
            G0[lane * kHidden + k] = v;
            GT[k * 32 + lane] = v;
        }
        // backward through the layers
        __nv_bfloat16* dY = G0;
        __nv_bfloat16* dX = G1;
        for (int l = kLayers - 1; l >= 0; --l) {
            const int outDim = layer_out(l), inDim = layer_in(l);
            const __nv_bfloat16* Xl = saved + l * 32 * kHidden;
            __syncwarp();
            for (int e = lane; e < 32 * kHidden; e += 32) {  // XT = Xl^T
                int r = e / kHidden, c = e % kHidden;
                XT[c * 32 + r] = Xl[e];
            }
            __syncwarp();
            float* accL = accW + layer_offset(l);
            // dW_l[m][k] += sum_s dY[s][m] X_l[s][k]
            if (outDim == kOut)
                warp_gemm<kOut, kHidden, 32>(GT, 32, XT, 32, [&](int r, int c, float v) { atomicAdd(&accL[r * inDim + c], v); });
            else
                warp_gemm<kHidden, kHidden, 32>(GT, 32, XT, 32, [&](int r, int c, float v) { atomicAdd(&accL[r * inDim + c], v); });
            if (l == 0) {
                // input gradient of the grid features: dX0[s][k] = sum_m dY[s][m] W0[m][k], k < 32
                float* dIn = reinterpret_cast<float*>(dX);  // [32][32] fp32 in the spare buffer
                __syncwarp();
                const __nv_bfloat16* WT0 = g.WT + layer_offset(0);
                warp_gemm<32, kGridDims, kHidden>(dY, kHidden, WT0, layer_out(0),
                                                  [&](int r, int c, float v) { dIn[r * kGridDims + c] = v; });
                __syncwarp();
                if (valid) {
                    float3 p = normalise_position(g, mk3(smp.q.pos[0], smp.q.pos[1], smp.q.pos[2]));
                    for (int lv = 0; lv < kLevels; ++lv) {
                        float d0 = dIn[lane * kGridDims + 2 * lv], d1 = dIn[lane * kGridDims + 2 * lv + 1];
                        for (int c = 0; c < 8; ++c) {
                            uint32_t idx;
                            float w;
                            grid_corner(g.res[lv], p, c, idx, w);
                            float* dst = dGrid + ((uint64_t)lv * kTableSize + idx) * kFeatures;
                            atomicAdd(dst, w * d0);
                            atomicAdd(dst + 1, w * d1);
                        }
                    }
                }
                break;
            }
            // dX = dY W_l (through B^t = W_l^T, read from global), then ReLU'
            const __nv_bfloat16* WTl = g.WT + layer_offset(l);
            const __nv_bfloat16* Xrelu = Xl;  // input of layer l = relu output of layer l-1
            __syncwarp();
            if (outDim == kOut)
                warp_gemm<32, kHidden, kOut>(dY, kHidden, WTl, kOut, [&](int r, int c, float v) {
                    dX[r * kHidden + c] = bf(fl(Xrelu[r * kHidden + c]) > 0.0f ? v : 0.0f);
                });
            else
                warp_gemm<32, kHidden, kHidden>(dY, kHidden, WTl, kHidden, [&](int r, int c, float v) {
                    dX[r * kHidden + c] = bf(fl(Xrelu[r * kHidden + c]) > 0.0f ? v : 0.0f);
                });
            __syncwarp();
            for (int e = lane; e < 32 * kHidden; e += 32) {  // GT = dX^T
                int r = e / kHidden, c = e % kHidden;
                GT[c * 32 + r] = dX[e];
            }
            __nv_bfloat16* t = dY;
            dY = dX;
            dX = t;
        }
        __syncwarp();
    }
    __syncthreads();
    for (int i = threadIdx.x; i < kWeightCount; i += blockDim.x)
        if (accW[i] != 0.0f) atomicAdd(&dW[i], accW[i]);
    for (int o = 16; o; o >>= 1) lossSum += __shfl_xor_sync(0xffffffffu, lossSum, o);
    if (lane == 0 && loss) atomicAdd(loss, lossSum);
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

__global__ void k_adam_grid(float* p, float* m, float* v, float* grad, uint64_t n, float lr, float b1, float b2,
                            float eps, float c1, float c2, __half* h)
{
    uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    float gr = grad[i];
    if (gr == 0.0f && m[i] == 0.0f) return;  // untouched entry: nothing to do
    float mi = b1 * m[i] + (1.0f - b1) * gr;
    float vi = b2 * v[i] + (1.0f - b2) * gr * gr;
    m[i] = mi;
    v[i] = vi;
    float pi = p[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    p[i] = pi;
    grad[i] = 0.0f;
    h[i] = __float2half_rn(pi);
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

size_t infer_smem() { return (size_t)kWeightCount * 2 + kInferWarps * (2 * 32 * kHidden * 2 + 32 * kOut * 4); }
size_t train_smem()
{
    size_t perWarp = (size_t)kLayers * 32 * kHidden * 2 + 2 * 32 * kHidden * 2 + 2 * kHidden * 32 * 2;
    return (size_t)kWeightCount * 2 + (size_t)kWeightCount * 4 + kTrainWarps * perWarp;
}

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
    std::vector<float> gp(kGridParams);
    for (uint64_t i = 0; i < kGridParams; ++i) gp[i] = (2.0f * uniform(s) - 1.0f) * 1e-4f;
    cudaError_t e = cudaMemcpyAsync(wP_, w.data(), w.size() * 4, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(gridP_, gp.data(), gp.size() * 4, cudaMemcpyHostToDevice, st);
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

void Guide::infer(const Query* q, uint32_t n, float* raw, cudaStream_t st) const { infer_queue(q, nullptr, n, raw, st); }

void Guide::infer_queue(const Query* q, const uint32_t* count, uint32_t maxN, float* raw, cudaStream_t st) const
{
    if (maxN == 0) return;
    // per call: the attribute belongs to the current device
    cudaFuncSetAttribute(k_infer, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)infer_smem());
    uint32_t chunks = (maxN + 31) / 32;
    uint32_t blocks = (chunks + kInferWarps - 1) / kInferWarps;
    if (blocks > 148 * 8) blocks = 148 * 8;
    k_infer<<<blocks, 32 * kInferWarps, infer_smem(), st>>>(params(), q, maxN, count, raw);
}

void Guide::accumulate_gradients(const Sample* s, uint32_t n, float invBatch, cudaStream_t st, uint32_t offset,
                                 uint32_t stride)
{
    if (n == 0) return;
    cudaFuncSetAttribute(k_train, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)train_smem());
    uint32_t chunks = (n + 31) / 32;
    uint32_t blocks = (chunks + kTrainWarps - 1) / kTrainWarps;
    if (blocks > 148 * 4) blocks = 148 * 4;
    k_train<<<blocks, 32 * kTrainWarps, train_smem(), st>>>(params(), s, n, offset, stride, invBatch, wG_, gridG_,
                                                            loss_);
}

void Guide::apply_adam(float lr, cudaStream_t st)
{
    ++step_;
    const float b1 = 0.9f, b2 = 0.99f, eps = 1e-8f;
    float c1 = 1.0f - (float)std::pow(b1, step_), c2 = 1.0f - (float)std::pow(b2, step_);
    k_adam_weights<<<(kWeightCount + 255) / 256, 256, 0, st>>>(wP_, wM_, wV_, wG_, kWeightCount, lr, b1, b2, eps, c1,
                                                               c2, wB_, wT_);
    k_adam_grid<<<(unsigned)((kGridParams + 255) / 256), 256, 0, st>>>(gridP_, gridM_, gridV_, gridG_, kGridParams, lr,
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
