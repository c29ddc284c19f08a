// Learned path guiding: a multiresolution hash-grid encoding of the shading
// position plus (wo, shading normal, roughness) feeds an MLP with 4 hidden
// layers of width 64 (BF16 weights, FP32 accumulation on the tensor cores),
// whose 40 outputs parameterise a mixture of 8 von Mises-Fisher lobes over
// incident directions. No counterpart in the reference.
//
// Published methods restated here: the hash-grid encoding of Mueller, Evans,
// Schied, Keller (Instant Neural Graphics Primitives, SIGGRAPH 2022: spatial
// hash with primes 1, 2654435761, 805459861, trilinear interpolation,
// geometric level resolutions), vMF sampling by inverting the CDF of
// cos(theta) (Jakob, "Numerically stable sampling of the von Mises-Fisher
// distribution on S^2", 2012), and the KL-divergence gradient of Mueller et
// al. (Neural Importance Sampling, TOG 2019) for online training.
#pragma once

#include "common.cuh"
#include "shading.cuh"

#include <cuda_bf16.h>
#include <cuda_fp16.h>

namespace ag {
namespace guide {

#ifndef AG_GUIDE_FEATURES
#define AG_GUIDE_FEATURES 4
#endif
constexpr int kFeatures = AG_GUIDE_FEATURES;  // per level (2 or 4)
constexpr int kLevels = 32 / kFeatures;
static_assert(kFeatures == 2 || kFeatures == 4, "2 or 4 features per level");
constexpr uint32_t kTableLog2 = 19;
constexpr uint32_t kTableSize = 1u << kTableLog2;
constexpr int kGridDims = kLevels * kFeatures;  // 32
constexpr int kIn = 64;                      // 32 grid + 3 wo + 3 normal + 1 roughness + 1 constant + padding
constexpr int kHidden = 64;
constexpr int kOut = 48;                     // 40 used: 8 lobes x (3 direction, 1 log-kappa, 1 logit)
constexpr int kLobes = 8;
constexpr int kRawPerLobe = 5;
constexpr int kLayers = 5;                   // in->h, h->h x3, h->out
constexpr int kMinRes = 16;
constexpr int kMaxRes = 2048;
constexpr float kLogKappaMin = -2.0f;
constexpr float kLogKappaMax = 8.0f;

// Offsets (in elements) of each layer's weight matrix [out][in] in the packed buffer.
__host__ __device__ constexpr int layer_out(int l) { return l == kLayers - 1 ? kOut : kHidden; }
__host__ __device__ constexpr int layer_in(int l) { return l == 0 ? kIn : kHidden; }
__host__ __device__ constexpr int layer_offset(int l)
{
    int o = 0;
    for (int i = 0; i < l; ++i) o += layer_out(i) * layer_in(i);
    return o;
}
constexpr int kWeightCount = layer_offset(kLayers);
constexpr uint64_t kGridParams = (uint64_t)kLevels * kTableSize * kFeatures;

struct Params {
    const __half* grid;            // [level][entry][feature] (inference copy)
    const __nv_bfloat16* W;        // packed [out][in] per layer
    const __nv_bfloat16* WT;       // packed transposes [in][out] per layer
    float3 bmin;                   // scene box used to normalise positions
    float3 invExtent;
    uint32_t res[kLevels];         // grid resolution per level
};

// One inference query: the shading position, roughness, outgoing direction
// (world space, towards the previous vertex) and shading normal. 48 bytes.
struct Query {
    float pos[3];
    float rough;
    float wo[3];
    float pad0;
    float n[3];
    float pad1;
};
static_assert(sizeof(Query) == 48, "Query layout");

// One training sample: query, sampled incident direction and the weight of
// the KL gradient (incident radiance luminance / sampling pdf). 64 bytes.
struct Sample {
    Query q;
    float dir[3];
    float weight;
};
static_assert(sizeof(Sample) == 64, "Sample layout");

// ---------------------------------------------------------------------------
// Hash-grid encoding.
AG_HD uint32_t grid_index(uint32_t res, uint32_t x, uint32_t y, uint32_t z)
{
    uint64_t dense = (uint64_t)(res + 1) * (res + 1) * (res + 1);
    if (dense <= kTableSize) return x + (res + 1) * (y + (res + 1) * z);
    return (x * 1u ^ y * 2654435761u ^ z * 805459861u) & (kTableSize - 1);
}

// Corner c (0..7) of the cell of `p` (in [0,1]^3) at `level`: table index and
// trilinear weight.
AG_HD void grid_corner(uint32_t res, float3 p, int c, uint32_t& index, float& weight)
{
    float fx = p.x * (float)res, fy = p.y * (float)res, fz = p.z * (float)res;
    float ix = floorf(fx), iy = floorf(fy), iz = floorf(fz);
    float tx = fx - ix, ty = fy - iy, tz = fz - iz;
    uint32_t x = (uint32_t)ix + (c & 1), y = (uint32_t)iy + ((c >> 1) & 1), z = (uint32_t)iz + ((c >> 2) & 1);
    weight = ((c & 1) ? tx : 1.0f - tx) * ((c & 2) ? ty : 1.0f - ty) * ((c & 4) ? tz : 1.0f - tz);
    index = grid_index(res, x, y, z);
}

AG_HD float3 normalise_position(const Params& g, float3 p)
{
    float3 q = (p - g.bmin) * g.invExtent;
    q.x = fminf(fmaxf(q.x, 0.0f), 0.99999f);
    q.y = fminf(fmaxf(q.y, 0.0f), 0.99999f);
    q.z = fminf(fmaxf(q.z, 0.0f), 0.99999f);
    return q;
}

// Non-grid inputs of one vertex (written after the 32 grid features).
AG_HD void extra_inputs(float3 wo, float3 n, float rough, float out[8])
{
    float nl = sqrtf(dot(n, n));
    float3 nn = nl > 0.0f ? n / nl : mk3(0.0f, 0.0f, 1.0f);
    out[0] = wo.x; out[1] = wo.y; out[2] = wo.z;
    out[3] = nn.x; out[4] = nn.y; out[5] = nn.z;
    out[6] = rough;
    out[7] = 1.0f;  // constant input: acts as the first layer's bias
}

// ---------------------------------------------------------------------------
// von Mises-Fisher mixture.
struct Mixture {
    float3 mu[kLobes];
    float kappa[kLobes];
    float lambda[kLobes];
};

AG_HD float vmf_pdf(float3 mu, float kappa, float3 w)
{
    // kappa / (2 pi (1 - exp(-2 kappa))) * exp(kappa (mu.w - 1))
    float norm = kappa / (2.0f * kPi * (-expm1f(-2.0f * kappa)));
    return norm * expf(kappa * (dot(mu, w) - 1.0f));
}

AG_HD void decode_mixture(const float raw[40], Mixture& m)
{
    float mx = -3.4e38f;
    for (int k = 0; k < kLobes; ++k) mx = fmaxf(mx, raw[k * kRawPerLobe + 4]);
    float sum = 0.0f;
    for (int k = 0; k < kLobes; ++k) {
        const float* r = raw + k * kRawPerLobe;
        float3 d = mk3(r[0], r[1], r[2]);
        float l = sqrtf(dot(d, d));
        m.mu[k] = l > 1e-12f ? d / l : mk3(0.0f, 0.0f, 1.0f);
        float s = fminf(fmaxf(r[3], kLogKappaMin), kLogKappaMax);
        m.kappa[k] = expf(s);
        m.lambda[k] = expf(r[4] - mx);
        sum += m.lambda[k];
    }
    for (int k = 0; k < kLobes; ++k) m.lambda[k] /= sum;
}

AG_HD float mixture_pdf(const Mixture& m, float3 w)
{
    float p = 0.0f;
    for (int k = 0; k < kLobes; ++k) p += m.lambda[k] * vmf_pdf(m.mu[k], m.kappa[k], w);
    return p;
}

// The decoded mixture as the shading kernel reads it: 48 fields per vertex,
// lambda[8] (selection probabilities), c[8] (density constants lambda kappa /
// (2 pi (1 - exp(-2 kappa)))), kappa[8], mu.x[8], mu.y[8], mu.z[8] (unit
// mean directions, world space). Field f of a vertex is at L[f * stride]:
// the render keeps the fields of a wave's vertices in separate arrays
// (stride = the wave's capacity), so the loads of a warp's consecutive
// vertices coalesce. Sampling and the density read the mixture lobe by
// lobe; a thread never holds all of it. Offsets are 32-bit: a wave holds
// fewer than 2^32 / kPacked vertices.
constexpr int kPacked = 48;
constexpr int kPackLambda = 0, kPackC = 8, kPackKappa = 16, kPackMu = 24;

// Lobe k from its 5 raw outputs r, given the largest logit mx and 1 / the
// sum of exp(logit - mx) over the lobes (the softmax of decode_mixture).
AG_HD void pack_lobe(const float* r, float mx, float invSum, int k, float* out, uint32_t stride)
{
    const float3 d = mk3(r[0], r[1], r[2]);
    const float l = sqrtf(dot(d, d));
    const float3 mu = l > 1e-12f ? d / l : mk3(0.0f, 0.0f, 1.0f);
    const float kappa = expf(fminf(fmaxf(r[3], kLogKappaMin), kLogKappaMax));
    const float lambda = expf(r[4] - mx) * invSum;
    out[(kPackLambda + k) * stride] = lambda;
    out[(kPackC + k) * stride] = lambda * kappa / (2.0f * kPi * (-expm1f(-2.0f * kappa)));
    out[(kPackKappa + k) * stride] = kappa;
    out[(kPackMu + k) * stride] = mu.x;
    out[(kPackMu + 8 + k) * stride] = mu.y;
    out[(kPackMu + 16 + k) * stride] = mu.z;
}

// All 8 lobes of one vertex's 40 raw outputs.
AG_HD void pack_mixture(const float raw[40], float* out, uint32_t stride)
{
    float mx = -3.4e38f;
    for (int k = 0; k < kLobes; ++k) mx = fmaxf(mx, raw[k * kRawPerLobe + 4]);
    float sum = 0.0f;
    for (int k = 0; k < kLobes; ++k) sum += expf(raw[k * kRawPerLobe + 4] - mx);
    const float invSum = 1.0f / sum;
    for (int k = 0; k < kLobes; ++k) pack_lobe(raw + k * kRawPerLobe, mx, invSum, k, out, stride);
}

// A direction from a packed mixture: the first lobe k with u0 < lambda_0 +
// ... + lambda_k (the last one if rounding leaves u0 above the total), then
// cos(theta) about its mean by inverting the vMF CDF (Jakob 2012).
AG_HD float3 lobes_sample(const float* L, uint32_t stride, float u0, float u1, float u2)
{
    int k = kLobes - 1;
    float c = 0.0f;
    for (int j = 0; j < kLobes - 1; ++j) {
        c += L[(kPackLambda + j) * stride];
        if (u0 < c) {
            k = j;
            break;
        }
    }
    const float kappa = L[(kPackKappa + k) * stride];
    const float3 mu = mk3(L[(kPackMu + k) * stride], L[(kPackMu + 8 + k) * stride], L[(kPackMu + 16 + k) * stride]);
    float wc = 1.0f + logf(u1 + (1.0f - u1) * expf(-2.0f * kappa)) / kappa;
    wc = fminf(fmaxf(wc, -1.0f), 1.0f);
    const float st = sqrtf(fmaxf(0.0f, 1.0f - wc * wc));
    const float phi = 2.0f * kPi * u2;
    float3 t1, t2;
    get_basis(mu, t1, t2);
    return t1 * (st * cosf(phi)) + t2 * (st * sinf(phi)) + mu * wc;
}

// Density of a packed mixture at the unit direction w:
// sum_k c_k exp(kappa_k (mu_k . w - 1)).
AG_HD float lobes_pdf(const float* L, uint32_t stride, float3 w)
{
    float p = 0.0f;
#pragma unroll
    for (int k = 0; k < kLobes; ++k) {
        const float cosMu = L[(kPackMu + k) * stride] * w.x + L[(kPackMu + 8 + k) * stride] * w.y +
                            L[(kPackMu + 16 + k) * stride] * w.z;
        p += L[(kPackC + k) * stride] * expf(L[(kPackKappa + k) * stride] * (cosMu - 1.0f));
    }
    return p;
}

// d(-w log q)/d raw for one sample direction w (q = mixture pdf).
AG_HD void mixture_grad(const float raw[40], float3 w, float weight, float grad[40])
{
    Mixture m;
    decode_mixture(raw, m);
    float v[kLobes];
    float q = 0.0f;
    for (int k = 0; k < kLobes; ++k) {
        v[k] = vmf_pdf(m.mu[k], m.kappa[k], w);
        q += m.lambda[k] * v[k];
    }
    q = fmaxf(q, 1e-30f);
    for (int k = 0; k < kLobes; ++k) {
        const float* r = raw + k * kRawPerLobe;
        float* g = grad + k * kRawPerLobe;
        float resp = m.lambda[k] * v[k] / q;
        // logit: d log q / d a_k = resp_k - lambda_k
        g[4] = -weight * (resp - m.lambda[k]);
        // log-kappa: d log v / d kappa = 1/kappa - 2 / expm1(2 kappa) + (mu.w - 1)
        float kap = m.kappa[k];
        float s = r[3];
        float dk = 1.0f / kap - 2.0f / expm1f(2.0f * kap) + (dot(m.mu[k], w) - 1.0f);
        g[3] = (s > kLogKappaMin && s < kLogKappaMax) ? -weight * resp * dk * kap : 0.0f;
        // direction: mu = d / |d|, d log v / d d = kappa / |d| (w - (mu.w) mu)
        float3 d = mk3(r[0], r[1], r[2]);
        float l = sqrtf(dot(d, d));
        float3 gd = mk3(0.0f, 0.0f, 0.0f);
        if (l > 1e-12f) gd = (w - m.mu[k] * dot(m.mu[k], w)) * (kap / l);
        g[0] = -weight * resp * gd.x;
        g[1] = -weight * resp * gd.y;
        g[2] = -weight * resp * gd.z;
    }
    for (int i = kLobes * kRawPerLobe; i < 40; ++i) grad[i] = 0.0f;
}

// ---------------------------------------------------------------------------
// Warp-level BF16 tensor-core GEMM (mma.sync m16n8k16, FP32 accumulate).
AG_D void mma_bf16(float c[4], uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3, uint32_t b0, uint32_t b1)
{
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

AG_D uint32_t ld32(const __nv_bfloat16* p) { return *reinterpret_cast<const uint32_t*>(p); }

// D[M x N] (+)= A[M x K] * B, with A row-major in shared memory (lda
// elements per row) and B given as Bt[N x K] row-major (ldb), i.e.
// D[m][n] = sum_k A[m][k] * Bt[n][k]. M multiple of 16, N of 8, K of 16.
// The warp calls `emit(m, n, value)` for every output element.
template <int M, int N, int K, typename Emit>
AG_D void warp_gemm(const __nv_bfloat16* A, int lda, const __nv_bfloat16* Bt, int ldb, Emit emit)
{
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
#pragma unroll
    for (int mt = 0; mt < M / 16; ++mt) {
#pragma unroll
        for (int nt = 0; nt < N / 8; ++nt) {
            float c[4] = {0.0f, 0.0f, 0.0f, 0.0f};
#pragma unroll
            for (int ks = 0; ks < K / 16; ++ks) {
                const __nv_bfloat16* a = A + (mt * 16 + g) * lda + ks * 16 + 2 * t;
                const __nv_bfloat16* b = Bt + (nt * 8 + g) * ldb + ks * 16 + 2 * t;
                mma_bf16(c, ld32(a), ld32(a + 8 * lda), ld32(a + 8), ld32(a + 8 * lda + 8), ld32(b), ld32(b + 8));
            }
            const int r = mt * 16 + g, col = nt * 8 + 2 * t;
            emit(r, col, c[0]);
            emit(r, col + 1, c[1]);
            emit(r + 8, col, c[2]);
            emit(r + 8, col + 1, c[3]);
        }
    }
}

}  // namespace guide
}  // namespace ag
