// Host side of rendering: materials, lights and light samplers, camera, the
// wave loop over the integrator kernels, accumulation read-back and the
// post-process (alpine::render / resetAccumulation / postProcess /
// getFrameBuffer, src/alpine.cpp:259-288, 446-483).
#include "context.cuh"
#include "integrator.cuh"
#include "trace.cuh"

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstring>
#include <numeric>
#include <vector>

using ag::DeviceBuffer;

namespace {

// ---------------------------------------------------------------------------
// Host float3 helpers (reference operation order, src/math/vector.h)
float3 h3(float x, float y, float z) { return make_float3(x, y, z); }
float3 hadd(float3 a, float3 b) { return h3(a.x + b.x, a.y + b.y, a.z + b.z); }
float3 hsub(float3 a, float3 b) { return h3(a.x - b.x, a.y - b.y, a.z - b.z); }
float3 hmul(float3 a, float s) { return h3(a.x * s, a.y * s, a.z * s); }
float3 hdiv(float3 a, float s) { return h3(a.x / s, a.y / s, a.z / s); }
float hdot(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
float hlen(float3 a) { return std::sqrt(hdot(a, a)); }
float3 hnorm(float3 a) { return hdiv(a, hlen(a)); }
float3 hcross(float3 a, float3 b)
{
    return h3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
float3 hmin(float3 a, float3 b) { return h3(std::min(a.x, b.x), std::min(a.y, b.y), std::min(a.z, b.z)); }
float3 hmax(float3 a, float3 b) { return h3(std::max(a.x, b.x), std::max(a.y, b.y), std::max(a.z, b.z)); }
float hcomp(float3 v, int k) { return k == 0 ? v.x : (k == 1 ? v.y : v.z); }
float hmaxc(float3 v) { return std::max(v.x, std::max(v.y, v.z)); }

struct HBox {
    float3 lo = h3(FLT_MAX, FLT_MAX, FLT_MAX);
    float3 hi = h3(-FLT_MAX, -FLT_MAX, -FLT_MAX);
    float3 center() const { return hmul(hadd(lo, hi), 0.5f); }
    float3 diag() const { return hsub(hi, lo); }
    float area() const
    {
        float3 l = hsub(hi, lo);
        return (l.x * l.y + l.y * l.z + l.z * l.x) * 2.0f;
    }
};
HBox hmerge(const HBox& a, const HBox& b)
{
    HBox r;
    r.lo = hmin(a.lo, b.lo);
    r.hi = hmax(a.hi, b.hi);
    return r;
}

void hbasis(float3 v, float3& b1, float3& b2)  // getBasis (src/math/vector.h:214-222)
{
    b1 = std::fabs(v.x) > std::fabs(v.y) ? hnorm(h3(-v.z, 0.0f, v.x)) : hnorm(h3(0.0f, v.z, -v.y));
    b2 = hcross(v, b1);
}

HBox light_box(const ag::Light& l)
{
    HBox b;
    b.lo = l.bmin;
    b.hi = l.bmax;
    return b;
}
float light_power_len(const ag::Light& l) { return hlen(hmul(l.power, l.scale)); }

// ---------------------------------------------------------------------------
// AliasTable (src/utils/alias_table.cpp:8-69) restated.
std::vector<ag::AliasBin> build_alias(const std::vector<float>& weights)
{
    const size_t n = weights.size();
    std::vector<ag::AliasBin> bins(n);
    std::vector<float> scaled(n);
    float sum = static_cast<float>(std::accumulate(weights.begin(), weights.end(), 0.0));
    for (size_t i = 0; i < n; ++i) {
        bins[i].p = weights[i] / sum;
        scaled[i] = bins[i].p * (float)n;
    }
    std::vector<uint32_t> small, large;
    for (uint32_t i = 0; i < n; ++i) (scaled[i] < 1.0f ? small : large).push_back(i);
    while (!small.empty() && !large.empty()) {
        uint32_t s = small.back(), l = large.back();
        small.pop_back();
        large.pop_back();
        bins[s].q = scaled[s];
        bins[s].alias = l;
        scaled[l] += scaled[s] - 1.0f;
        (scaled[l] < 1.0f ? small : large).push_back(l);
    }
    for (auto* work : {&small, &large}) {
        while (!work->empty()) {
            auto& b = bins[work->back()];
            work->pop_back();
            b.q = 1.0f;
            b.alias = 0xffffffffu;
        }
    }
    return bins;
}

// ---------------------------------------------------------------------------
// Light BVH (src/light_samplers/bvh_light_sampler.cpp:54-263) restated,
// flattened depth-first for the device.
struct LightSplit {
    bool valid = false;
    int dim = 0, splitIdx = 0;
    float lo = 0.0f, hi = 0.0f;
};
constexpr int kLightSplits = 4;  // SPLITS_PER_DIM (bvh_light_sampler.cpp:13)
constexpr int kLightBins = kLightSplits + 1;

uint8_t light_bin(float c, float lo, float hi)
{
    uint8_t b = static_cast<uint8_t>(kLightBins * (c - lo) / (hi - lo));
    return std::min<uint8_t>(b, kLightBins - 1);
}

LightSplit split_light_cluster(const std::vector<ag::Light>& L, const std::vector<uint32_t>& cl, float3 diagonal)
{
    LightSplit split;
    if (cl.size() <= 2) return split;
    HBox cb;
    for (uint32_t i : cl) {
        float3 c = light_box(L[i]).center();
        HBox p;
        p.lo = c;
        p.hi = c;
        cb = hmerge(cb, p);
    }
    if (hmaxc(cb.diag()) == 0.0f) return split;
    float minCost = FLT_MAX;
    struct Bin {
        float power = 0.0f;
        HBox box;
    } bins[kLightBins];
    for (int dim = 0; dim < 3; ++dim) {
        float cmin = hcomp(cb.lo, dim), cmax = hcomp(cb.hi, dim);
        if (cmin == cmax) continue;
        float kr = hmaxc(diagonal) / std::max(hcomp(diagonal, dim), 0.001f);
        for (auto& b : bins) b = Bin();
        for (uint32_t i : cl) {
            HBox bb = light_box(L[i]);
            auto& b = bins[light_bin(hcomp(bb.center(), dim), cmin, cmax)];
            b.power += light_power_len(L[i]);
            b.box = hmerge(b.box, bb);
        }
        float costs[kLightSplits] = {0.0f};
        auto accumulate = [&](int binIdx, int splitIdx, Bin& acc) {
            acc.power += bins[binIdx].power;
            acc.box = hmerge(acc.box, bins[binIdx].box);
            float sa = acc.box.lo.x < FLT_MAX ? acc.box.area() : 0.0f;
            costs[splitIdx] += acc.power * sa;
        };
        Bin below;
        for (int s = 0; s < kLightSplits; ++s) accumulate(s, s, below);
        Bin above;
        for (int s = kLightSplits - 1; s >= 0; --s) accumulate(s + 1, s, above);
        for (int s = 0; s < kLightSplits; ++s) {
            costs[s] *= kr;
            if (costs[s] < minCost) {
                minCost = costs[s];
                split.valid = true;
                split.dim = dim;
                split.splitIdx = s;
                split.lo = cmin;
                split.hi = cmax;
            }
        }
    }
    return split;
}

int32_t create_light_node(const std::vector<ag::Light>& L, const std::vector<uint32_t>& cl,
                          std::vector<ag::LightNode>& out)
{
    int32_t id = (int32_t)out.size();
    out.emplace_back();
    float power = 0.0f;
    HBox box;
    for (uint32_t i : cl) {
        power += light_power_len(L[i]);
        box = hmerge(light_box(L[i]), box);
    }
    out[id].power = power;
    out[id].bmin = box.lo;
    out[id].bmax = box.hi;
    out[id].left = out[id].right = -1;
    out[id].light = -1;
    if (cl.size() == 1) {
        out[id].light = (int32_t)cl[0];
        return id;
    }
    LightSplit s = split_light_cluster(L, cl, box.diag());
    std::vector<uint32_t> sub[2];
    if (s.valid) {
        for (uint32_t i : cl) {
            bool below = light_bin(hcomp(light_box(L[i]).center(), s.dim), s.lo, s.hi) <= s.splitIdx;
            sub[below ? 0 : 1].push_back(i);
        }
    }
    if (!s.valid || sub[0].empty() || sub[1].empty()) {
        // median split by index (bvh_light_sampler.cpp:207-213); also taken
        // when a split leaves one side empty, where the reference asserts
        sub[0].clear();
        sub[1].clear();
        uint32_t mid = (uint32_t)(cl.size() / 2);
        for (uint32_t i = 0; i < cl.size(); ++i) sub[i < mid ? 0 : 1].push_back(cl[i]);
    }
    int32_t l = create_light_node(L, sub[0], out);
    int32_t r = create_light_node(L, sub[1], out);
    out[id].left = l;
    out[id].right = r;
    return id;
}

// ---------------------------------------------------------------------------
int add_light(alpine_gpu_ctx* c, const ag::Light& l, uint32_t* id)
{
    c->lights.push_back(l);
    c->lightsDirty = true;
    if (id) *id = (uint32_t)(c->lights.size() - 1);
    return ALPINE_GPU_OK;
}

void finish_light(ag::Light& l, const float3* corners, int ncorners)
{
    HBox b;
    for (int i = 0; i < ncorners; ++i) {
        HBox p;
        p.lo = corners[i];
        p.hi = corners[i];
        b = hmerge(b, p);
    }
    l.bmin = b.lo;
    l.bmax = b.hi;
}

template <typename T>
bool upload(DeviceBuffer& buf, const std::vector<T>& v, cudaStream_t st)
{
    if (!buf.reserve(std::max<size_t>(1, v.size()) * sizeof(T))) return false;
    if (v.empty()) return true;
    return cudaMemcpyAsync(buf.ptr, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, st) == cudaSuccess;
}

int upload_scene_data(alpine_gpu_ctx* c)
{
    cudaStream_t st = c->stream;
    if (c->materialsDirty) {
        std::vector<ag::Material> mats = c->materials;
        if (mats.empty()) {  // default: grey Lambertian (Dielectric with alpha 1)
            ag::Material m{};
            m.kind = ag::kMatDielectric;
            m.r = m.g = m.b = 0.5f;
            m.ax = m.ay = 1.0f;
            m.lobes = 1;
            mats.push_back(m);
        }
        if (!upload(c->dMaterials, mats, st)) return c->fail(ALPINE_GPU_ERR_CUDA, "material upload failed");
        c->materialCount = (uint32_t)mats.size();
        c->materialsDirty = false;
    }
    if (c->attribsDirty) {
        if (!upload(c->dTriInfo, c->triInfo, st) || !upload(c->dNormals, c->normals, st) ||
            !upload(c->dUvs, c->uvs, st) || !upload(c->dTangents, c->tangents, st))
            return c->fail(ALPINE_GPU_ERR_CUDA, "attribute upload failed");
        c->attribsDirty = false;
    }
    if (c->texturesDirty) {
        if (!upload(c->dTextures, c->textures, st) || !upload(c->dTexels, c->texels, st))
            return c->fail(ALPINE_GPU_ERR_CUDA, "texture upload failed");
        c->texturesDirty = false;
    }
    if (c->envDirty) {
        if (!upload(c->dEnv, c->env, st)) return c->fail(ALPINE_GPU_ERR_CUDA, "environment map upload failed");
        c->envDirty = false;
    }
    if (c->lightsDirty) {
        if (!upload(c->dLights, c->lights, st)) return c->fail(ALPINE_GPU_ERR_CUDA, "light upload failed");
        c->lightsDirty = false;
    }
    return ALPINE_GPU_OK;
}

size_t round256(size_t b) { return (b + 255) & ~size_t(255); }

// Wave buffers for up to `paths` paths.
bool reserve_wave(alpine_gpu_ctx* c, uint32_t paths)
{
    if (paths <= c->waveCapacity) return true;
    size_t P = paths;
    size_t bytes = 0;
    bytes += 7 * round256(P * sizeof(float4));             // thr rad albedo nrm pendL pendB pendThr
    bytes += round256(P * sizeof(uint4));                  // rng
    bytes += round256(P * sizeof(int2));                   // pendShadow
    bytes += 2 * round256(P * sizeof(alpine_gpu_ray));     // rays, raysNext
    bytes += 2 * round256(P * sizeof(uint32_t));           // queuePath x2
    bytes += round256(P * sizeof(uint4));                  // hits
    bytes += round256(2 * P * sizeof(alpine_gpu_ray));     // shadow rays
    bytes += round256(2 * P);                              // shadow occlusion
    bytes += round256(P) + round256(P * sizeof(uint32_t)); // shading-order keys and order
    bytes += 256;                                          // counters
    if (!c->dWave.reserve(bytes)) return false;
    c->waveCapacity = paths;
    return true;
}

ag::WaveView carve_wave(alpine_gpu_ctx* c)
{
    ag::WaveView w{};
    size_t P = c->waveCapacity;
    char* p = c->dWave.as<char>();
    auto take = [&](size_t b) {
        char* r = p;
        p += round256(b);
        return r;
    };
    w.thr = (float4*)take(P * sizeof(float4));
    w.rad = (float4*)take(P * sizeof(float4));
    w.albedo = (float4*)take(P * sizeof(float4));
    w.nrm = (float4*)take(P * sizeof(float4));
    w.pendL = (float4*)take(P * sizeof(float4));
    w.pendB = (float4*)take(P * sizeof(float4));
    w.pendThr = (float4*)take(P * sizeof(float4));
    w.rng = (uint4*)take(P * sizeof(uint4));
    w.pendShadow = (int2*)take(P * sizeof(int2));
    w.rays = (alpine_gpu_ray*)take(P * sizeof(alpine_gpu_ray));
    w.raysNext = (alpine_gpu_ray*)take(P * sizeof(alpine_gpu_ray));
    w.queuePath = (uint32_t*)take(P * sizeof(uint32_t));
    w.queuePathNext = (uint32_t*)take(P * sizeof(uint32_t));
    w.hits = (uint4*)take(P * sizeof(uint4));
    w.shadowRays = (alpine_gpu_ray*)take(2 * P * sizeof(alpine_gpu_ray));
    w.shadowOcc = (uint8_t*)take(2 * P);
    w.shadeKeys = (uint8_t*)take(P);
    w.shadeOrderBuf = (uint32_t*)take(P * sizeof(uint32_t));
    uint32_t* counters = (uint32_t*)take(256);
    w.queueCount = counters;
    w.queueCountNext = counters + 1;
    w.shadowCount = counters + 2;
    w.shadeBins = counters + 16;  // 16 words: bin counts, bin cursors
    return w;
}

// Guiding buffers for `paths` paths and `cap` training records.
struct GuideWave {
    ag::guide::Query* query;
    int* querySlot;      // per queue entry
    float* lobes;        // per guided vertex: the decoded mixture (kPacked floats)
    int* slot;
    ag::guide::Sample* rec;
    float4* aux;
    ag::guide::Sample* out;
    uint32_t* counters;  // [0] records, [1] kept samples, [2] guided vertices of the queue
};

bool reserve_guide_wave(alpine_gpu_ctx* c, uint32_t paths, uint32_t cap, GuideWave& g)
{
    size_t P = paths, R = cap;
    size_t bytes = round256(P * sizeof(ag::guide::Query)) + round256(P * sizeof(int)) + round256(P * ag::guide::kPacked * sizeof(float)) +
                   round256(P * sizeof(int)) + round256(R * sizeof(ag::guide::Sample)) +
                   round256(2 * R * sizeof(float4)) + round256(R * sizeof(ag::guide::Sample)) + 256;
    if (!c->dGuideWave.reserve(bytes)) return false;
    char* p = c->dGuideWave.as<char>();
    auto take = [&](size_t b) {
        char* r = p;
        p += round256(b);
        return r;
    };
    g.query = (ag::guide::Query*)take(P * sizeof(ag::guide::Query));
    g.querySlot = (int*)take(P * sizeof(int));
    g.lobes = (float*)take(P * ag::guide::kPacked * sizeof(float));
    g.slot = (int*)take(P * sizeof(int));
    g.rec = (ag::guide::Sample*)take(R * sizeof(ag::guide::Sample));
    g.aux = (float4*)take(2 * R * sizeof(float4));
    g.out = (ag::guide::Sample*)take(R * sizeof(ag::guide::Sample));
    g.counters = (uint32_t*)take(256);
    return true;
}

bool reserve_accum(alpine_gpu_ctx* c)
{
    size_t pixels = (size_t)c->cfg.width * c->cfg.height;
    size_t bytes = pixels * 9 * (c->options.accumulate_fp64 ? sizeof(double) : sizeof(float));
    if (c->accumBytes == bytes && c->dAccum.ptr) return true;
    if (!c->dAccum.reserve(bytes) || !c->dPixelRng.reserve(pixels * sizeof(uint4))) return false;
    c->accumBytes = bytes;
    return true;
}

__global__ void k_reset_accum(float* a, size_t words, uint4* rng, uint32_t pixels)
{
    size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (i < words) a[i] = 0.0f;
    if (i < pixels) {  // Sampler::reset(pixel index) (src/sampler.cpp:7-13)
        ag::XorShift128 r;
        ag::xorshift_seed(r, (uint32_t)i);
        rng[i] = make_uint4(r.s[0], r.s[1], r.s[2], r.s[3]);
    }
}

// postProcess (alpine.cpp:446-483): mean, optional ACES, clamp, sRGB, 8 bits
__global__ void k_post(const float* a32, const double* a64, uint32_t pixels, uint32_t total, int tonemap,
                       float* meanOut, uint8_t* rgbOut)
{
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= pixels) return;
    float c[3];
    for (int k = 0; k < 3; ++k)
        c[k] = a64 ? (float)a64[9ull * i + k] / (float)total : a32[9ull * i + k] / (float)total;
    if (meanOut)
        for (int k = 0; k < 3; ++k) meanOut[3ull * i + k] = c[k];
    if (!rgbOut) return;
    for (int k = 0; k < 3; ++k) {
        float x = c[k];
        if (tonemap) x = (x * (x * 2.51f + 0.03f)) / (x * (x * 2.43f + 0.59f) + 0.14f);
        x = fminf(fmaxf(x, 0.0f), 1.0f);
        x = x <= 0.0031308f ? 12.92f * x : 1.055f * powf(x, 1.0f / 2.4f) - 0.055f;
        rgbOut[3ull * i + k] = (uint8_t)(x * 255.0f + 0.5f);
    }
}

__global__ void k_set_word(uint32_t* p, uint32_t v) { *p = v; }

// Turns the wave's recorded vertices into training samples and takes up to
// `maxSteps` Adam steps; step i uses samples i, i + stride, i + 2 stride, ...
// so that every batch spans the whole image. The stride is the number of
// steps, or larger when the wave kept more than steps x batch samples: a
// step then takes `batch` samples (the surplus is not used), which keeps it
// one k_train_rows launch (a second slice would cost a whole latency-bound
// launch for a few samples).
int train_guide(alpine_gpu_ctx* c, const ag::IntegratorKernels& K, const ag::WaveView& w, const GuideWave& gw,
                uint32_t batch, uint32_t maxSteps, float lr)
{
    cudaStream_t st = c->stream;
    K.train_finalize(w, gw.out, gw.counters + 1, st);
    uint32_t kept = 0;
    cudaError_t e = cudaMemcpyAsync(c->hStatus + 1, gw.counters + 1, sizeof(uint32_t), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return c->fail(ALPINE_GPU_ERR_CUDA, std::string("guide training: ") + cudaGetErrorString(e));
    kept = std::min(c->hStatus[1], w.trainCap);
    if (kept == 0) return ALPINE_GPU_OK;
    const uint32_t steps = std::min(maxSteps, (kept + batch - 1) / batch);
    c->guide.reset_loss(st);
    // with a surplus, stride = kept / batch >= steps: the steps' residues are
    // disjoint and i + (batch - 1) stride < kept
    const bool surplus = (uint64_t)kept > (uint64_t)steps * batch;
    const uint32_t stride = surplus ? kept / batch : steps;
    for (uint32_t i = 0; i < steps; ++i) {
        const uint32_t n = surplus ? batch : (kept - i + steps - 1) / steps;
        c->guide.accumulate_gradients(gw.out, n, 1.0f / (float)n, st, i, stride, c->dStatus);
        c->guide.apply_adam(lr, st);
    }
    c->guideLastLossSteps = steps;
    c->guide.read_loss_async(reinterpret_cast<float*>(c->hStatus + 2), st);  // read after the next synchronisation
    return ALPINE_GPU_OK;
}

}  // namespace

extern "C" {

int alpine_gpu_set_materials(alpine_gpu_ctx* c, const alpine_gpu_material* m, uint32_t n)
{
    if (!c) return ALPINE_GPU_ERR_INVALID_ARGUMENT;
    if (n && !m) return c->fail(ALPINE_GPU_ERR_INVALID_ARGUMENT, "set_materials: null array");
    c->materials.clear();
    for (uint32_t i = 0; i < n; ++i) {
        ag::Material x{};
        if (!ag::make_material(m[i], x)) return c->fail(ALPINE_GPU_ERR_INVALID_ARGUMENT, "set_materials: unknown kind");
        c->materials.push_back(x);
    }
    c->materialsDirty = true;
    return ALPINE_GPU_OK;
}

int alpine_gpu_set_triangle_attributes(alpine_gpu_ctx* c, uint32_t shape, const float* normals,
                                       const uint32_t* tri_material)
{
    if (!c) return ALPINE_GPU_ERR_INVALID_ARGUMENT;
    if (shape >= c->shapeVertBase.size()) return c->fail(ALPINE_GPU_ERR_INVALID_ARGUMENT, "bad shape id");
    const uint32_t vb = c->shapeVertBase[shape], vc = c->shapeVertCount[shape];
    const uint32_t tb = c->shapeTriBase[shape], tc = c->shapeTriCount[shape];
    if (int rc = c->pull_host_geometry()) return rc;
    if (c->triInfo.size() < c->idx.size() / 3) c->triInfo.resize(c->idx.size() / 3, 0u);
    if (c->normals.size() < c->verts.size()) c->normals.resize(c->verts.size(), 0.0f);
    if (normals) std::memcpy(c->normals.data() + 3ull * vb, normals, 3ull * vc * sizeof(float));
    for (uint32_t t = 0; t < tc; ++t) {
        uint32_t mid = tri_material ? tri_material[t] : 0u;
        if (mid & ~ag::kTriMaterialMask) return c->fail(ALPINE_GPU_ERR_INVALID_ARGUMENT, "material id too large");
        // kept: the morph-target and texture-coordinate flags, set by their own calls
        const uint32_t kept = c->triInfo[tb + t] & (ag::kTriMorphedNormals | ag::kTriHasUvs | ag::kTriHasTangents);
        c->triInfo[tb + t] = mid | (normals ? ag::kTriHasNormals : 0u) | kept;
    }
    c->attribsDirty = true;
    return ALPINE_GPU_OK;
}

int alpine_gpu_set_triangle_uvs(alpine_gpu_ctx* c, uint32_t shape, const float* uvs, const float* tangents)
{
    if (!c) return ALPINE_GPU_ERR_INVALID_ARGUMENT;
    if (shape >= c->shapeVertBase.size()) return c->fail(ALPINE_GPU_ERR_INVALID_ARGUMENT, "bad shape id");
    if (tangents && !uvs)
        return c->fail(ALPINE_GPU_ERR_INVALID_ARGUMENT, "set_triangle_uvs: tangents need texture coordinates");
    const uint32_t vb = c->shapeVertBase[shape], vc = c->shapeVertCount[shape];
    const uint32_t tb = c->shapeTriBase[shape], tc = c->shapeTriCount[shape];
    if (c->triInfo.size() < c->idx.size() / 3) c->triInfo.resize(c->idx.size() / 3, 0u);
    if (tangents)
        for (uint32_t t = 0; t < tc; ++t)
            if (!(c->triInfo[tb + t] & ag::kTriHasNormals))
                return c->fail(ALPINE_GPU_ERR_INVALID_STATE,
                               "set_triangle_uvs: tangents need vertex normals (alpine_gpu_set_triangle_attributes)");
    const size_t V = c->verts.size() / 3;
    if (uvs) {
        if (c->uvs.size() < 2 * V) c->uvs.resize(2 * V, 0.0f);
        std::memcpy(c->uvs.data() + 2ull * vb, uvs, 2ull * vc * sizeof(float));
    }
    if (tangents) {
        if (c->tangents.size() < 4 * V) c->tangents.resize(4 * V, 0.0f);
        std::memcpy(c->tangents.data() + 4ull * vb, tangents, 4ull * vc * sizeof(float));
    }
    for (uint32_t t = 0; t < tc; ++t) {
        uint32_t& f = c->triInfo[tb + t];
        f = (f & ~(ag::kTriHasUvs | ag::kTriHasTangents)) | (uvs ? ag::kTriHasUvs : 0u) |
            (tangents ? ag::kTriHasTangents : 0u);
    }
    c->attribsDirty = true;
    return ALPINE_GPU_OK;
}

int alpine_gpu_add_texture(alpine_gpu_ctx* c, const float* texels, uint32_t width, uint32_t height, uint32_t* id)
{
    if (!c) return ALPINE_GPU_ERR_INVALID_ARGUMENT;
    if (!texels || width == 0 || height == 0)
        return c->fail(ALPINE_GPU_ERR_INVALID_ARGUMENT, "add_texture: empty texture");
    const uint64_t n = (uint64_t)width * height;
    if (c->texels.size() + n >= 0xffffffffull) return c->fail(ALPINE_GPU_ERR_LIMIT, "add_texture: texel pool full");
    ag::TextureInfo t{(uint32_t)c->texels.size(), width, height, 0u};
    c->texels.resize(c->texels.size() + n);
    std::memcpy(c->texels.data() + t.offset, texels, n * sizeof(float4));
    c->textures.push_back(t);
    c->texturesDirty = true;
    if (id) *id = (uint32_t)(c->textures.size() - 1);
    return ALPINE_GPU_OK;
}

int alpine_gpu_set_material_textures(alpine_gpu_ctx* c, uint32_t material, int32_t base_color_texture,
                                     int32_t normal_texture)
{
    if (!c) return ALPINE_GPU_ERR_INVALID_ARGUMENT;
    if (material >= c->materials.size())
        return c->fail(ALPINE_GPU_ERR_INVALID_ARGUMENT, "set_material_textures: bad material id");
    const int32_t nt = (int32_t)c->textures.size();
    if (base_color_texture >= nt || normal_texture >= nt || base_color_texture < -1 || normal_texture < -1)
        return c->fail(ALPINE_GPU_ERR_INVALID_ARGUMENT, "set_material_textures: bad texture id");
    c->materials[material].baseTex = (uint32_t)(base_color_texture + 1);
    c->materials[material].normalTex = (uint32_t)(normal_texture + 1);
    c->materialsDirty = true;
    return ALPINE_GPU_OK;
}

int alpine_gpu_set_environment_map(alpine_gpu_ctx* c, const float* rgb, uint32_t width, uint32_t height)
{
    if (!c) return ALPINE_GPU_ERR_INVALID_ARGUMENT;
    if (!rgb || width == 0 || height == 0) {
        c->env.clear();
        c->envW = c->envH = 0;
        return ALPINE_GPU_OK;
    }
    c->env.assign(rgb, rgb + 3ull * width * height);
    c->envW = width;
    c->envH = height;
    c->envDirty = true;
    return ALPINE_GPU_OK;
}

int alpine_gpu_add_point_light(alpine_gpu_ctx* c, float power, const float color[3], const float position[3],
                               uint32_t* id)
{
    if (!c || !color || !position) return ALPINE_GPU_ERR_INVALID_ARGUMENT;
    ag::Light l{};
    l.kind = ag::kLightPoint;
    l.scale = 1.0f;
    l.position = h3(position[0], position[1], position[2]);
    l.power = hmul(h3(color[0], color[1], color[2]), power);
    l.radiance = hdiv(l.power, 4.0f * ag::kPi);  // intensity (point_light.cpp:14-20)
    float3 corners[1] = {l.position};
    finish_light(l, corners, 1);
    return add_light(c, l, id);
}

int alpine_gpu_add_disk_light(alpine_gpu_ctx* c, float power, const float color[3], const float position[3],
                              const float target[3], float radius, uint32_t* id)
{
    if (!c || !color || !position || !target) return ALPINE_GPU_ERR_INVALID_ARGUMENT;
    ag::Light l{};
    l.kind = ag::kLightDisk;
    l.scale = 1.0f;
    l.position = h3(position[0], position[1], position[2]);
    // Alpine::addDiskLight: normal = normalize(target - position) (alpine.cpp:221-233)
    l.normal = hnorm(hsub(h3(target[0], target[1], target[2]), l.position));
    l.power = hmul(h3(color[0], color[1], color[2]), power);
    l.radius = radius;
    hbasis(l.normal, l.axisU, l.axisV);  // DiskLight (disk_light.cpp:9-28)
    l.area = radius * radius * ag::kPi;
    l.radiance = hdiv(l.power, l.area * ag::kPi);
    float3 corners[4] = {hadd(l.position, hmul(l.axisU, radius)), hsub(l.position, hmul(l.axisU, radius)),
                         hadd(l.position, hmul(l.axisV, radius)), hsub(l.position, hmul(l.axisV, radius))};
    finish_light(l, corners, 4);
    return add_light(c, l, id);
}

int alpine_gpu_add_quad_light(alpine_gpu_ctx* c, const float radiance[3], const float corner[3],
                              const float edge_u[3], const float edge_v[3], uint32_t* id)
{
    if (!c || !radiance || !corner || !edge_u || !edge_v) return ALPINE_GPU_ERR_INVALID_ARGUMENT;
    ag::Light l{};
    l.kind = ag::kLightQuad;
    l.scale = 1.0f;
    l.position = h3(corner[0], corner[1], corner[2]);
    l.axisU = h3(edge_u[0], edge_u[1], edge_u[2]);
    l.axisV = h3(edge_v[0], edge_v[1], edge_v[2]);
    float3 n = hcross(l.axisU, l.axisV);
    l.area = hlen(n);
    if (!(l.area > 0.0f)) return c->fail(ALPINE_GPU_ERR_INVALID_ARGUMENT, "add_quad_light: degenerate quad");
    l.normal = hdiv(n, l.area);  // emits on the side of cross(edge_u, edge_v)
    l.radiance = h3(radiance[0], radiance[1], radiance[2]);
    l.power = hmul(l.radiance, l.area * ag::kPi);  // Lambertian emitter: power = L * A * pi
    float3 corners[4] = {l.position, hadd(l.position, l.axisU), hadd(l.position, l.axisV),
                         hadd(hadd(l.position, l.axisU), l.axisV)};
    finish_light(l, corners, 4);
    return add_light(c, l, id);
}

int alpine_gpu_set_light_scale(alpine_gpu_ctx* c, uint32_t id, float scale)
{
    if (!c || id >= c->lights.size()) return c ? c->fail(ALPINE_GPU_ERR_INVALID_ARGUMENT, "bad light id") : -1;
    c->lights[id].scale = scale;  // LightHandle::setScale (include/alpine/light.h:6-7)
    c->lightsDirty = true;
    return ALPINE_GPU_OK;
}

int alpine_gpu_build_light_sampler(alpine_gpu_ctx* c, int type)
{
    if (!c) return ALPINE_GPU_ERR_INVALID_ARGUMENT;
    if (type < ALPINE_GPU_LIGHT_SAMPLER_UNIFORM || type > ALPINE_GPU_LIGHT_SAMPLER_BVH)
        return c->fail(ALPINE_GPU_ERR_INVALID_ARGUMENT, "build_light_sampler: unknown type");
    // Alpine::buildLightSampler (alpine.cpp:235-251)
    c->samplerKind = type == ALPINE_GPU_LIGHT_SAMPLER_POWER ? ag::kSamplerPower
                   : type == ALPINE_GPU_LIGHT_SAMPLER_BVH  ? ag::kSamplerBvh
                                                           : ag::kSamplerUniform;
    c->samplerLightCount = (uint32_t)c->lights.size();
    if (c->samplerKind == ag::kSamplerPower && !c->lights.empty()) {
        std::vector<float> w(c->lights.size());
        for (size_t i = 0; i < w.size(); ++i) w[i] = light_power_len(c->lights[i]);
        if (!upload(c->dAlias, build_alias(w), c->stream)) return c->fail(ALPINE_GPU_ERR_CUDA, "alias upload failed");
    }
    if (c->samplerKind == ag::kSamplerBvh && !c->lights.empty()) {
        std::vector<uint32_t> all(c->lights.size());
        for (uint32_t i = 0; i < all.size(); ++i) all[i] = i;
        std::vector<ag::LightNode> nodes;
        nodes.reserve(2 * all.size());
        create_light_node(c->lights, all, nodes);
        // the descent's packed records: both children of every interior node
        std::vector<ag::LightPair> pairs(nodes.size());
        auto ref = [&](int32_t i) {
            const ag::LightNode& n = nodes[i];
            const int32_t r = (n.left >= 0 && n.right >= 0) ? i : -(n.light + 1);
            float f;
            std::memcpy(&f, &r, sizeof f);
            return f;
        };
        for (size_t i = 0; i < nodes.size(); ++i) {
            const ag::LightNode& n = nodes[i];
            if (n.left < 0 || n.right < 0) continue;
            const ag::LightNode& a = nodes[n.left];
            const ag::LightNode& b = nodes[n.right];
            pairs[i].lo0 = make_float4(a.bmin.x, a.bmin.y, a.bmin.z, a.power);
            pairs[i].hi0 = make_float4(a.bmax.x, a.bmax.y, a.bmax.z, ref(n.left));
            pairs[i].lo1 = make_float4(b.bmin.x, b.bmin.y, b.bmin.z, b.power);
            pairs[i].hi1 = make_float4(b.bmax.x, b.bmax.y, b.bmax.z, ref(n.right));
        }
        if (!upload(c->dLightNodes, nodes, c->stream) || !upload(c->dLightPairs, pairs, c->stream))
            return c->fail(ALPINE_GPU_ERR_CUDA, "light BVH upload failed");
        c->lightNodeCount = (uint32_t)nodes.size();
    }
    if (cudaStreamSynchronize(c->stream) != cudaSuccess)
        return c->fail(ALPINE_GPU_ERR_CUDA, "build_light_sampler: synchronisation failed");
    return ALPINE_GPU_OK;
}

int alpine_gpu_set_background(alpine_gpu_ctx* c, float r, float g, float b)
{
    if (!c) return ALPINE_GPU_ERR_INVALID_ARGUMENT;
    c->background = h3(r, g, b);
    return ALPINE_GPU_OK;
}

int alpine_gpu_set_camera(alpine_gpu_ctx* c, const float eye[3], const float target[3], const float up[3],
                          float fovy, float aspect)
{
    if (!c || !eye || !target || !up) return ALPINE_GPU_ERR_INVALID_ARGUMENT;
    // Camera::setLookAt / updateViewMatrix (src/camera.cpp:13-29, 87-96)
    ag::Camera& cam = c->camera;
    cam.eye = h3(eye[0], eye[1], eye[2]);
    float3 tg = h3(target[0], target[1], target[2]), u = h3(up[0], up[1], up[2]);
    cam.filmH = 1.0f * std::tan(0.5f * fovy);
    cam.filmW = cam.filmH * aspect;
    cam.viewZ = hnorm(hsub(tg, cam.eye));
    cam.viewX = hnorm(hcross(cam.viewZ, u));
    cam.viewY = hcross(cam.viewX, cam.viewZ);
    c->cameraSet = true;
    return ALPINE_GPU_OK;
}

int alpine_gpu_set_render_options(alpine_gpu_ctx* c, const alpine_gpu_render_options* o)
{
    if (!c || !o) return ALPINE_GPU_ERR_INVALID_ARGUMENT;
    if (o->sampler != ALPINE_GPU_SAMPLER_REFERENCE_STREAM && o->sampler != ALPINE_GPU_SAMPLER_COUNTER)
        return c->fail(ALPINE_GPU_ERR_INVALID_ARGUMENT, "render options: unknown sampler");
    bool accumChange = o->accumulate_fp64 != c->options.accumulate_fp64 || o->sampler != c->options.sampler;
    c->options = *o;
    if (accumChange) c->accumValid = false;
    return ALPINE_GPU_OK;
}

int alpine_gpu_reset_accumulation(alpine_gpu_ctx* c)
{
    if (!c) return ALPINE_GPU_ERR_INVALID_ARGUMENT;
    if (c->cfg.width == 0 || c->cfg.height == 0) return c->fail(ALPINE_GPU_ERR_INVALID_STATE, "no framebuffer");
    cudaSetDevice(c->device);
    if (!reserve_accum(c)) return c->fail(ALPINE_GPU_ERR_OUT_OF_MEMORY, "accumulation buffers");
    uint32_t pixels = c->cfg.width * c->cfg.height;
    size_t words = c->accumBytes / sizeof(float);
    size_t n = std::max<size_t>(words, pixels);
    k_reset_accum<<<(unsigned)((n + 255) / 256), 256, 0, c->stream>>>(c->dAccum.as<float>(), words,
                                                                       c->dPixelRng.as<uint4>(), pixels);
    c->totalSamples = 0;
    c->accumValid = true;
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return c->fail(ALPINE_GPU_ERR_CUDA, cudaGetErrorString(e));
    return ALPINE_GPU_OK;
}

static int render_enqueue(alpine_gpu_ctx* c, uint32_t spp)
{
    if (!c) return ALPINE_GPU_ERR_INVALID_ARGUMENT;
    if (c->cfg.width == 0 || c->cfg.height == 0) return c->fail(ALPINE_GPU_ERR_INVALID_STATE, "no framebuffer");
    if (c->bvhDirty) return c->fail(ALPINE_GPU_ERR_INVALID_STATE, "geometry changed since the last alpine_gpu_build");
    if (!c->cameraSet) return c->fail(ALPINE_GPU_ERR_INVALID_STATE, "camera not set");
    cudaSetDevice(c->device);
    if (!c->accumValid)
        if (int rc = alpine_gpu_reset_accumulation(c)) return rc;
    if (c->triInfo.size() < c->idx.size() / 3) {
        if (int rc = c->pull_host_geometry()) return rc;
        c->triInfo.resize(c->idx.size() / 3, 0u);
        c->attribsDirty = true;
    }
    if (int rc = upload_scene_data(c)) return rc;
    if (spp == 0) return ALPINE_GPU_OK;

    const bool stream = c->options.sampler == ALPINE_GPU_SAMPLER_REFERENCE_STREAM;
    const ag::IntegratorKernels& K = stream ? ag::integrator_exact() : ag::integrator_fast();
    const uint32_t pixels = c->cfg.width * c->cfg.height;
    uint32_t maxPaths = c->options.max_paths_per_wave ? c->options.max_paths_per_wave : (1u << 21);
    if (maxPaths < 1024) maxPaths = 1024;
    // samples per wave: one in stream mode (the per-pixel RNG is sequential)
    uint32_t S = stream ? 1u : std::max(1u, std::min(spp, maxPaths / std::max(1u, pixels)));
    const alpine_gpu_render_options& o = c->options;
    const bool guiding = !stream && o.guide != 0;
    const bool trainEnabled = guiding && o.guide_train != 0;
    const uint32_t gBatch = o.guide_batch ? o.guide_batch : 16384u;
    const uint32_t gSteps = o.guide_steps_per_wave ? o.guide_steps_per_wave : 8u;
    const float gLr = o.guide_lr > 0.0f ? o.guide_lr : 1e-2f;
    const float gFrac = o.guide_fraction > 0.0f ? std::min(o.guide_fraction, 1.0f) : 0.5f;
    // waves while the guide trains hold few samples per pixel, so that
    // training happens often; afterwards they are as large as unguided ones
    const uint32_t sTrain = std::min(S, o.guide_spp_per_wave ? o.guide_spp_per_wave : 1u);
    uint32_t pixelChunk = std::min(pixels, maxPaths / S);
    if (!reserve_wave(c, S * pixelChunk)) return c->fail(ALPINE_GPU_ERR_OUT_OF_MEMORY, "wave buffers");
    GuideWave gw{};
    // Recorded vertices per wave: only those that later receive radiance
    // become samples (about 12% in a dim interior), so 8 x steps x batch
    // records keep every step of the wave at about a full batch (2 x, 4 x and
    // 8 x measured 2.45, 2.76 and 2.78 x plain's speed to a relMSE of 0.01).
    const uint32_t trainCap = trainEnabled ? std::min<uint32_t>(1u << 22, 8u * gSteps * gBatch) : 0u;
    if (guiding) {
        if (!c->guide.ready() && c->guide.reset(c->guideSeed, c->stream) != 0)
            return c->fail(ALPINE_GPU_ERR_OUT_OF_MEMORY, "guide: parameter allocation failed");
        if (!c->guideBoxSet && !c->verts.empty()) {  // the scene's bounds
            float3 lo = h3(c->verts[0], c->verts[1], c->verts[2]), hi = lo;
            for (size_t i = 0; i + 2 < c->verts.size(); i += 3) {
                float3 v = h3(c->verts[i], c->verts[i + 1], c->verts[i + 2]);
                lo = hmin(lo, v);
                hi = hmax(hi, v);
            }
            c->guide.set_scene_box(lo, hi);
            c->guideBoxSet = true;
        }
        if (!reserve_guide_wave(c, S * pixelChunk, std::max(trainCap, 1u), gw))
            return c->fail(ALPINE_GPU_ERR_OUT_OF_MEMORY, "guide wave buffers");
    }

    ag::SceneView sc{};
    sc.verts = c->dVerts.as<float>();
    sc.idx = c->dIdx.as<uint32_t>();
    sc.normals = c->dNormals.as<float>();
    sc.triInfo = c->dTriInfo.as<uint32_t>();
    sc.uvs = c->dUvs.as<float>();
    sc.tangents = c->dTangents.as<float>();
    sc.textures = c->dTextures.as<ag::TextureInfo>();
    sc.texels = c->dTexels.as<float4>();
    sc.textureCount = (uint32_t)c->textures.size();
    sc.env = c->envW ? c->dEnv.as<float>() : nullptr;
    sc.spheres = c->dSpheres.as<float4>();
    sc.sphereMaterial = c->dSphereMaterial.as<uint32_t>();
    sc.sphereCount = (uint32_t)c->spheres.size();
    sc.envW = c->envW;
    sc.envH = c->envH;
    sc.materials = c->dMaterials.as<ag::Material>();
    sc.materialCount = c->materialCount;
    sc.lights.kind = c->samplerKind;
    sc.lights.count = std::min<uint32_t>(c->samplerLightCount, (uint32_t)c->lights.size());
    sc.lights.lights = c->dLights.as<ag::Light>();
    sc.lights.alias = c->dAlias.as<ag::AliasBin>();
    sc.lights.nodes = c->dLightNodes.as<ag::LightNode>();
    sc.lights.pairs = c->dLightPairs.as<ag::LightPair>();
    sc.background = c->background;
    sc.cam = c->camera;
    sc.width = c->cfg.width;
    sc.height = c->cfg.height;
    sc.maxDepth = c->cfg.max_depth;
    ag::BvhView bvh = c->bvh_view();
    // bounds checks against the allocations, so that a rebuilt BVH of the
    // same scene replays the same captured graph
    bvh.nodeCount = (uint32_t)(c->dNodes.bytes / sizeof(ag::WideNode));
    bvh.triCount = (uint32_t)(c->dTris.bytes / sizeof(ag::TriRecord));

    const bool fp64 = c->options.accumulate_fp64 != 0;
    float* acc32 = fp64 ? nullptr : c->dAccum.as<float>();
    double* acc64 = fp64 ? c->dAccum.as<double>() : nullptr;
    cudaStream_t st = c->stream;

    // CUDA graph: the whole wave loop of an unguided render, captured once per
    // launch configuration and replayed; the first sample index is read from
    // device memory so that successive renders replay the same graph
    const bool useGraph = o.cuda_graph != 0 && !guiding;
    std::vector<unsigned char> key;
    if (useGraph) {
        auto put = [&](const void* p, size_t n) {
            const unsigned char* b = static_cast<const unsigned char*>(p);
            key.insert(key.end(), b, b + n);
        };
        const uint32_t cfgWords[] = {spp, S, pixelChunk, pixels, (uint32_t)stream, (uint32_t)fp64,
                                     (uint32_t)c->traceBlock, c->options.seed, c->options.russian_roulette_depth,
                                     c->waveCapacity, bvh.triTest, bvh.maxVisits, bvh.stackLimit,
                                     c->options.shade_order};
        const void* ptrs[] = {c->dWave.ptr, c->dAccum.ptr, c->dPixelRng.ptr, c->dStatus};
        put(cfgWords, sizeof cfgWords);
        put(ptrs, sizeof ptrs);
        put(&sc, sizeof sc);
        put(&bvh, sizeof bvh);
        if (c->graphExec && key == c->graphKey) {
            k_set_word<<<1, 1, 0, st>>>(c->dSampleBase, c->totalSamples);
            cudaError_t e = cudaGraphLaunch(c->graphExec, st);
            if (e != cudaSuccess) return c->fail(ALPINE_GPU_ERR_CUDA, std::string("graph launch: ") + cudaGetErrorString(e));
            c->totalSamples += spp;
            ++c->graphLaunches;
            return ALPINE_GPU_OK;
        }
        if (c->graphExec) {
            cudaGraphExecDestroy(c->graphExec);
            c->graphExec = nullptr;
        }
        k_set_word<<<1, 1, 0, st>>>(c->dSampleBase, c->totalSamples);
        if (cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal) != cudaSuccess)
            return c->fail(ALPINE_GPU_ERR_CUDA, "render: stream capture could not begin");
    }
    const uint32_t sampleOrigin = useGraph ? 0u : c->totalSamples;
    const bool shadeSort = o.shade_order == ALPINE_GPU_SHADE_ORDER_BY_MATERIAL;
    for (uint32_t done = 0; done < spp;) {
        const bool trainNow = trainEnabled && (o.guide_train_steps == 0 || c->guide.steps() < o.guide_train_steps);
        const uint32_t s = std::min(trainNow ? sTrain : S, spp - done);
        for (uint32_t px = 0; px < pixels; px += pixelChunk) {
            ag::WaveView w = carve_wave(c);
            w.numPixels = std::min(pixelChunk, pixels - px);
            w.numPaths = s * w.numPixels;
            w.pixelBase = px;
            w.samplesInWave = s;
            w.sampleBase = sampleOrigin + done;
            w.sampleBaseDev = useGraph ? c->dSampleBase : nullptr;
            w.seed = c->options.seed;
            w.rrStart = stream ? 0u : c->options.russian_roulette_depth;
            w.pixelRng = c->dPixelRng.as<uint4>();
            const bool sampleGuide = guiding && c->guide.steps() >= o.guide_warmup_steps;
            const bool training = trainNow && (o.guide_train_steps == 0 || c->guide.steps() < o.guide_train_steps);
            if (guiding) {
                w.guideQuery = gw.query;
                w.guideSlot = gw.querySlot;
                w.guideCount = gw.counters + 2;
                w.guideLobes = sampleGuide ? gw.lobes : nullptr;
                w.guideFraction = gFrac;
                w.guideMinRough = o.guide_min_roughness;
            }
            if (training) {
                // record about trainCap vertices: ~3 continuations per path
                const uint64_t expected = 3ull * w.numPaths;
                w.trainStride = (uint32_t)std::max<uint64_t>(1, (expected + trainCap - 1) / trainCap);
                w.trainCap = trainCap;
                w.trainRec = gw.rec;
                w.trainAux = gw.aux;
                w.trainSlot = gw.slot;
                w.trainCount = gw.counters;
                w.waveIndex = c->guideWaveIndex;
                cudaMemsetAsync(gw.counters, 0, 2 * sizeof(uint32_t), st);
            }
            K.generate(sc, w, stream, st);
            for (uint32_t depth = 0; depth < sc.maxDepth; ++depth) {
                w.depth = depth;
                ag::launch_trace_dyn(bvh, w.rays, w.queueCount, w.numPaths, false, w.hits, c->dStatus, st,
                                     c->traceBlock);
                cudaMemsetAsync(w.queueCountNext, 0, sizeof(uint32_t), st);
                cudaMemsetAsync(w.shadowCount, 0, sizeof(uint32_t), st);
                const bool guideHere = guiding && (o.guide_max_depth == 0 || depth < o.guide_max_depth);
                ag::WaveView sw = w;
                if (!guideHere) {  // unguided shading (pending training records still resolve)
                    sw.guideQuery = nullptr;
                    sw.guideLobes = nullptr;
                }
                if (guideHere) {
                    cudaMemsetAsync(w.guideCount, 0, sizeof(uint32_t), st);
                    K.guide_query(sc, w, w.numPaths, st);
                    if (sampleGuide)
                        c->guide.infer_queue(gw.query, w.guideCount, w.numPaths, gw.lobes, st, c->dStatus, true);
                }
                if (shadeSort) {  // group the queue by shade_key before shading
                    cudaMemsetAsync(w.shadeBins, 0, 2 * ag::kShadeBins * sizeof(uint32_t), st);
                    K.sort(sc, sw, w.numPaths, w.shadeBins, w.shadeKeys, w.shadeOrderBuf, st);
                    sw.shadeOrder = w.shadeOrderBuf;
                }
                K.shade(sc, sw, stream, w.numPaths, st);
                ag::launch_trace_dyn(bvh, w.shadowRays, w.shadowCount, 2 * w.numPaths, true, w.shadowOcc,
                                     c->dStatus, st, c->traceBlock);
                K.resolve(w, w.numPaths, st);
                std::swap(w.rays, w.raysNext);
                std::swap(w.queuePath, w.queuePathNext);
                std::swap(w.queueCount, w.queueCountNext);
            }
            K.accumulate(w, acc32, acc64, stream, st);
            if (guiding) ++c->guideWaveIndex;
            if (training) {
                uint32_t steps = gSteps;
                if (o.guide_train_steps) steps = std::min(steps, o.guide_train_steps - c->guide.steps());
                if (int rc = train_guide(c, K, w, gw, gBatch, steps, gLr)) return rc;
            }
        }
        done += s;
    }
    if (useGraph) {
        cudaGraph_t g = nullptr;
        cudaError_t e = cudaStreamEndCapture(st, &g);
        if (e == cudaSuccess) e = cudaGraphInstantiate(&c->graphExec, g, 0);
        if (g) cudaGraphDestroy(g);
        if (e != cudaSuccess) {
            c->graphExec = nullptr;
            return c->fail(ALPINE_GPU_ERR_CUDA, std::string("render: graph capture: ") + cudaGetErrorString(e));
        }
        c->graphKey = key;
        ++c->graphCaptures;
        e = cudaGraphLaunch(c->graphExec, st);
        if (e != cudaSuccess) return c->fail(ALPINE_GPU_ERR_CUDA, std::string("graph launch: ") + cudaGetErrorString(e));
        ++c->graphLaunches;
    }
    c->totalSamples += spp;
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return c->fail(ALPINE_GPU_ERR_CUDA, std::string("render: ") + cudaGetErrorString(e));
    return ALPINE_GPU_OK;
}

// Waits for the context's stream and reads the device status word.
static int render_wait(alpine_gpu_ctx* c)
{
    cudaError_t e = cudaStreamSynchronize(c->stream);
    if (e == cudaSuccess) e = cudaGetLastError();
    if (e != cudaSuccess) return c->fail(ALPINE_GPU_ERR_CUDA, std::string("render: ") + cudaGetErrorString(e));
    return c->check_device_status();
}

int alpine_gpu_render(alpine_gpu_ctx* c, uint32_t spp)
{
    if (!c) return ALPINE_GPU_ERR_INVALID_ARGUMENT;
    if (int rc = render_enqueue(c, spp)) {
        cudaStreamSynchronize(c->stream);
        return rc;
    }
    return render_wait(c);
}

int alpine_gpu_render_async(alpine_gpu_ctx* c, uint32_t spp)
{
    if (!c) return ALPINE_GPU_ERR_INVALID_ARGUMENT;
    return render_enqueue(c, spp);
}

int alpine_gpu_render_wait(alpine_gpu_ctx* c)
{
    if (!c) return ALPINE_GPU_ERR_INVALID_ARGUMENT;
    return render_wait(c);
}

int alpine_gpu_render_graph_stats(alpine_gpu_ctx* c, uint32_t* captures, uint32_t* launches)
{
    if (!c) return ALPINE_GPU_ERR_INVALID_ARGUMENT;
    if (captures) *captures = c->graphCaptures;
    if (launches) *launches = c->graphLaunches;
    return ALPINE_GPU_OK;
}

// Times probe renders over wave sizes and traversal block sizes and keeps the
// fastest pair (samples per second); for a guided render then also the
// guide's inference kernels (warp MMA and tensor-memory tcgen05, whose
// outputs are identical). Guided probes sample the guide from the first
// probe on and do not train it, so the model is left as it was. The probes
// add to the accumulation, which is reset afterwards.
int alpine_gpu_autotune(alpine_gpu_ctx* c, uint32_t probe_spp, alpine_gpu_tuning* out)
{
    if (!c) return ALPINE_GPU_ERR_INVALID_ARGUMENT;
    if (probe_spp == 0) probe_spp = 4;
    const uint32_t waves[] = {1u << 18, 1u << 19, 1u << 20, 1u << 21, 1u << 22};
    const int blocks[] = {64, 128, 256};
    const alpine_gpu_render_options saved = c->options;
    const int savedBlock = c->traceBlock;
    alpine_gpu_tuning best{};
    best.samples_per_second = -1.0f;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    int rc = ALPINE_GPU_OK;
    if (c->options.guide) {
        c->options.guide_train = 0;
        c->options.guide_warmup_steps = 0;
    }
    // warm-up: allocations, module loading
    c->options.max_paths_per_wave = waves[0];
    rc = alpine_gpu_render(c, 1);
    const uint32_t pixels = c->cfg.width * c->cfg.height;
    for (uint32_t wi = 0; rc == ALPINE_GPU_OK && wi < sizeof(waves) / sizeof(waves[0]); ++wi) {
        // more paths than one wave of all samples cannot help
        if (wi > 0 && waves[wi - 1] >= (uint64_t)pixels * probe_spp) break;
        for (int b : blocks) {
            c->options.max_paths_per_wave = waves[wi];
            c->traceBlock = b;
            if ((rc = alpine_gpu_render(c, 1))) break;  // buffers for this wave size
            cudaEventRecord(e0, c->stream);
            if ((rc = render_enqueue(c, probe_spp))) break;
            cudaEventRecord(e1, c->stream);
            if ((rc = render_wait(c))) break;
            float ms = 0.0f;
            cudaEventElapsedTime(&ms, e0, e1);
            const float rate = ms > 0.0f ? (float)pixels * probe_spp / (ms * 1e-3f) : 0.0f;
            if (rate > best.samples_per_second) {
                best.samples_per_second = rate;
                best.max_paths_per_wave = waves[wi];
                best.trace_block = (uint32_t)b;
            }
        }
    }
    best.guide_kernel = (uint32_t)c->guide.kernel();
    if (rc == ALPINE_GPU_OK && c->options.guide) {
        c->options.max_paths_per_wave = best.max_paths_per_wave;
        c->traceBlock = (int)best.trace_block;
        float bestRate = -1.0f;
        const int kernels[] = {ag::guide::Guide::kKernelWarpMma, ag::guide::Guide::kKernelTensorMemory};
        for (int k : kernels) {
            c->guide.set_kernel(k);
            if ((rc = alpine_gpu_render(c, 1))) break;  // warm-up of this kernel
            cudaEventRecord(e0, c->stream);
            if ((rc = render_enqueue(c, probe_spp))) break;
            cudaEventRecord(e1, c->stream);
            if ((rc = render_wait(c))) break;
            float ms = 0.0f;
            cudaEventElapsedTime(&ms, e0, e1);
            const float rate = ms > 0.0f ? (float)pixels * probe_spp / (ms * 1e-3f) : 0.0f;
            if (rate > bestRate) {
                bestRate = rate;
                best.guide_kernel = (uint32_t)k;
            }
        }
        c->guide.set_kernel((int)best.guide_kernel);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    c->options = saved;
    c->traceBlock = savedBlock;
    if (rc) return rc;
    c->options.max_paths_per_wave = best.max_paths_per_wave;
    c->traceBlock = (int)best.trace_block;
    if (out) *out = best;
    return alpine_gpu_reset_accumulation(c);
}



int alpine_gpu_read_accumulation(alpine_gpu_ctx* c, float* sums, uint32_t* total_samples)
{
    if (!c) return ALPINE_GPU_ERR_INVALID_ARGUMENT;
    if (!c->accumValid) return c->fail(ALPINE_GPU_ERR_INVALID_STATE, "nothing rendered");
    cudaStreamSynchronize(c->stream);  // a render_async may be in flight
    size_t pixels = (size_t)c->cfg.width * c->cfg.height;
    if (sums) {
        if (c->options.accumulate_fp64) {
            std::vector<double> tmp(pixels * 9);
            if (cudaMemcpy(tmp.data(), c->dAccum.ptr, tmp.size() * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess)
                return c->fail(ALPINE_GPU_ERR_CUDA, "read_accumulation");
            for (size_t i = 0; i < tmp.size(); ++i) sums[i] = (float)tmp[i];
        } else if (cudaMemcpy(sums, c->dAccum.ptr, pixels * 9 * sizeof(float), cudaMemcpyDeviceToHost) != cudaSuccess) {
            return c->fail(ALPINE_GPU_ERR_CUDA, "read_accumulation");
        }
    }
    if (total_samples) *total_samples = c->totalSamples;
    return ALPINE_GPU_OK;
}

int alpine_gpu_read_accumulation_f64(alpine_gpu_ctx* c, double* sums, uint32_t* total_samples)
{
    if (!c) return ALPINE_GPU_ERR_INVALID_ARGUMENT;
    if (!c->accumValid) return c->fail(ALPINE_GPU_ERR_INVALID_STATE, "nothing rendered");
    cudaStreamSynchronize(c->stream);  // a render_async may be in flight
    size_t pixels = (size_t)c->cfg.width * c->cfg.height;
    if (sums) {
        if (c->options.accumulate_fp64) {
            if (cudaMemcpy(sums, c->dAccum.ptr, pixels * 9 * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess)
                return c->fail(ALPINE_GPU_ERR_CUDA, "read_accumulation");
        } else {
            std::vector<float> tmp(pixels * 9);
            if (cudaMemcpy(tmp.data(), c->dAccum.ptr, tmp.size() * sizeof(float), cudaMemcpyDeviceToHost) != cudaSuccess)
                return c->fail(ALPINE_GPU_ERR_CUDA, "read_accumulation");
            for (size_t i = 0; i < tmp.size(); ++i) sums[i] = tmp[i];
        }
    }
    if (total_samples) *total_samples = c->totalSamples;
    return ALPINE_GPU_OK;
}

int alpine_gpu_read_sampler_state(alpine_gpu_ctx* c, uint32_t* state)
{
    if (!c || !state) return ALPINE_GPU_ERR_INVALID_ARGUMENT;
    if (!c->accumValid) return c->fail(ALPINE_GPU_ERR_INVALID_STATE, "nothing rendered");
    cudaStreamSynchronize(c->stream);
    size_t pixels = (size_t)c->cfg.width * c->cfg.height;
    if (cudaMemcpy(state, c->dPixelRng.ptr, pixels * sizeof(uint4), cudaMemcpyDeviceToHost) != cudaSuccess)
        return c->fail(ALPINE_GPU_ERR_CUDA, "read_sampler_state");
    return ALPINE_GPU_OK;
}

// Checkpoint restore: the accumulation (sums and sample count) and the
// per-pixel reference streams of an earlier run. The next render continues
// from them as the interrupted run would have: the counter RNG numbers
// samples from total_samples on, the reference streams continue from the
// restored states.
extern "C++" {
template <typename T>
static int write_accumulation(alpine_gpu_ctx* c, const T* sums, uint32_t total)
{
    if (!c) return ALPINE_GPU_ERR_INVALID_ARGUMENT;
    if (!sums) return c->fail(ALPINE_GPU_ERR_INVALID_ARGUMENT, "write_accumulation: null sums");
    if (c->cfg.width == 0 || c->cfg.height == 0) return c->fail(ALPINE_GPU_ERR_INVALID_STATE, "no framebuffer");
    cudaSetDevice(c->device);
    if (!c->accumValid)
        if (int rc = alpine_gpu_reset_accumulation(c)) return rc;
    cudaStreamSynchronize(c->stream);
    const size_t n = (size_t)c->cfg.width * c->cfg.height * 9;
    cudaError_t e;
    if (c->options.accumulate_fp64) {
        std::vector<double> tmp(sums, sums + n);
        e = cudaMemcpy(c->dAccum.ptr, tmp.data(), n * sizeof(double), cudaMemcpyHostToDevice);
    } else {
        std::vector<float> tmp(n);
        for (size_t i = 0; i < n; ++i) tmp[i] = (float)sums[i];
        e = cudaMemcpy(c->dAccum.ptr, tmp.data(), n * sizeof(float), cudaMemcpyHostToDevice);
    }
    if (e != cudaSuccess) return c->fail(ALPINE_GPU_ERR_CUDA, std::string("write_accumulation: ") + cudaGetErrorString(e));
    c->totalSamples = total;
    return ALPINE_GPU_OK;
}
}  // extern "C++"

int alpine_gpu_write_accumulation(alpine_gpu_ctx* c, const float* sums, uint32_t total_samples)
{
    return write_accumulation(c, sums, total_samples);
}

int alpine_gpu_write_accumulation_f64(alpine_gpu_ctx* c, const double* sums, uint32_t total_samples)
{
    return write_accumulation(c, sums, total_samples);
}

int alpine_gpu_write_sampler_state(alpine_gpu_ctx* c, const uint32_t* state)
{
    if (!c) return ALPINE_GPU_ERR_INVALID_ARGUMENT;
    if (!state) return c->fail(ALPINE_GPU_ERR_INVALID_ARGUMENT, "write_sampler_state: null state");
    if (c->cfg.width == 0 || c->cfg.height == 0) return c->fail(ALPINE_GPU_ERR_INVALID_STATE, "no framebuffer");
    cudaSetDevice(c->device);
    if (!c->accumValid)
        if (int rc = alpine_gpu_reset_accumulation(c)) return rc;
    cudaStreamSynchronize(c->stream);
    const size_t pixels = (size_t)c->cfg.width * c->cfg.height;
    if (cudaMemcpy(c->dPixelRng.ptr, state, pixels * sizeof(uint4), cudaMemcpyHostToDevice) != cudaSuccess)
        return c->fail(ALPINE_GPU_ERR_CUDA, "write_sampler_state");
    return ALPINE_GPU_OK;
}

int alpine_gpu_post_process(alpine_gpu_ctx* c, int tonemap, float* mean_rgb, uint8_t* rgb8)
{
    if (!c) return ALPINE_GPU_ERR_INVALID_ARGUMENT;
    if (!c->accumValid || c->totalSamples == 0) return c->fail(ALPINE_GPU_ERR_INVALID_STATE, "nothing rendered");
    uint32_t pixels = c->cfg.width * c->cfg.height;
    DeviceBuffer mean, ldr;
    if ((mean_rgb && !mean.reserve(pixels * 3ull * sizeof(float))) || (rgb8 && !ldr.reserve(pixels * 3ull)))
        return c->fail(ALPINE_GPU_ERR_OUT_OF_MEMORY, "post_process buffers");
    bool fp64 = c->options.accumulate_fp64 != 0;
    k_post<<<(pixels + 255) / 256, 256, 0, c->stream>>>(fp64 ? nullptr : c->dAccum.as<float>(),
                                                        fp64 ? c->dAccum.as<double>() : nullptr, pixels,
                                                        c->totalSamples, tonemap, mean_rgb ? mean.as<float>() : nullptr,
                                                        rgb8 ? ldr.as<uint8_t>() : nullptr);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess && mean_rgb)
        e = cudaMemcpyAsync(mean_rgb, mean.ptr, pixels * 3ull * sizeof(float), cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess && rgb8) e = cudaMemcpyAsync(rgb8, ldr.ptr, pixels * 3ull, cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) return c->fail(ALPINE_GPU_ERR_CUDA, std::string("post_process: ") + cudaGetErrorString(e));
    return ALPINE_GPU_OK;
}

}  // extern "C"

namespace ag {
int upload_render_scene(alpine_gpu_ctx* c) { return upload_scene_data(c); }
}  // namespace ag

namespace ag {
// PointLight(intensity, position) (src/lights/point_light.cpp:8-13): the
// radiant intensity given directly, power = intensity * 4 * pi.
int add_point_light_intensity(alpine_gpu_ctx* c, float3 intensity, float3 position, uint32_t* id)
{
    ag::Light l{};
    l.kind = ag::kLightPoint;
    l.scale = 1.0f;
    l.position = position;
    l.radiance = intensity;
    l.power = hmul(hmul(intensity, 4.0f), ag::kPi);
    float3 corners[1] = {l.position};
    finish_light(l, corners, 1);
    return add_light(c, l, id);
}
}  // namespace ag
