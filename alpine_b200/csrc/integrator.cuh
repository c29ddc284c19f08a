// Wavefront path-tracing kernels.
//
// The reference integrator (src/alpine.cpp:290-432) runs one path at a time
// per host thread. Here a wave of paths (S samples of every pixel) advances
// bounce by bounce through queue kernels:
//   generate -> [extend (closest hit) -> shade -> shadow (any hit) -> resolve]
//   x maxDepth -> accumulate.
// shade does, per path vertex, exactly the reference's steps: miss ->
// background; AOVs at depth 0; next-event estimation (light selection, light
// sample + MIS, BSDF sample + MIS; estimateDirectIllumination,
// alpine.cpp:370-432) whose shadow rays are traced in a batch; continuation
// sample, the geometric-normal reflection test and the ray offsets
// (alpine.cpp:342-361). resolve adds the unoccluded direct light in the
// reference's summation order. Queues are compacted with warp-aggregated
// atomics; every path's arithmetic is independent of its queue position, so
// results do not depend on scheduling.
//
// The header is compiled twice: integrator_fast.cu (default flags, counter
// RNG) and integrator_exact.cu (no FMA contraction; also serves the reference
// RNG stream), inside different namespaces.
#pragma once

#include "../../include/alpine_gpu.h"
#include "bvh.cuh"
#include "guide.cuh"
#include "shading.cuh"

namespace ag {

struct SceneView {
    const float* verts;
    const uint32_t* idx;
    const float* normals;      // per vertex, may be null
    const uint32_t* triInfo;   // per triangle: material id | kTri* flags
    const float* uvs;          // per vertex (2 floats), read for kTriHasUvs triangles
    const float* tangents;     // per vertex (xyz, bitangent sign), read for kTriHasTangents triangles
    const TextureInfo* textures;
    const float4* texels;
    uint32_t textureCount;
    const float* env;          // lat-long environment map (3 floats per texel), null = background colour
    uint32_t envW, envH;
    const float4* spheres;     // analytic spheres: centre, radius
    const uint32_t* sphereMaterial;
    uint32_t sphereCount;
    const Material* materials;
    uint32_t materialCount;
    LightSamplerView lights;
    float3 background;
    Camera cam;
    uint32_t width, height, maxDepth;
};

struct WaveView {
    uint32_t numPaths;     // S * numPixels
    uint32_t numPixels;
    uint32_t sampleBase;   // sample index of slice 0 (counter RNG), plus *sampleBaseDev when set
    const uint32_t* sampleBaseDev;
    uint32_t samplesInWave;
    uint32_t seed;
    uint32_t rrStart;      // Russian roulette from this depth; 0 = off (reference behaviour)
    uint32_t depth;        // bounce being shaded
    uint32_t pixelBase;    // first pixel of this wave's pixel range
    // per path
    float4* thr;
    float4* rad;
    float4* albedo;
    float4* nrm;
    uint4* rng;
    float4* pendL;         // light-sample term of the pending direct light
    float4* pendB;         // BSDF-sample term; w = light-selection pdf
    float4* pendThr;       // throughput at the vertex
    int2* pendShadow;      // shadow-queue slots of the two terms (-1 = none)
    // queues
    alpine_gpu_ray* rays;
    uint32_t* queuePath;
    uint4* hits;
    uint32_t* queueCount;
    alpine_gpu_ray* raysNext;
    uint32_t* queuePathNext;
    uint32_t* queueCountNext;
    alpine_gpu_ray* shadowRays;
    uint8_t* shadowOcc;
    uint32_t* shadowCount;
    // persistent per-pixel reference RNG state (stream mode)
    uint4* pixelRng;
    // learned guiding (counter RNG only)
    guide::Query* guideQuery;  // compacted queries of the guided vertices; null = guiding off
    int* guideSlot;            // per queue entry: index into guideQuery / guideLobes, -1 = not guided
    uint32_t* guideCount;      // number of guided vertices of the current queue
    const float* guideLobes;   // decoded mixtures of the guided vertices: guide::kPacked field arrays of numPaths
                               // floats (field f of slot s at [f * numPaths + s]); null = material sampling only
    float guideFraction;       // probability of sampling the guide at an eligible vertex
    float guideMinRough;       // eligible vertices: material alpha >= this
    guide::Sample* trainRec;   // recorded vertices: query, direction (weight filled by finalize)
    float4* trainAux;          // 2 per record: (radiance after the vertex, path bits), (throughput at it, 0)
    int* trainSlot;            // per path: record waiting for its radiance-after value, -1 = none
    uint32_t* trainCount;
    uint32_t trainCap;
    uint32_t trainStride;      // record the vertices of paths whose hash % stride == 0; 0 = none
    uint32_t waveIndex;
    // shading order: when set, shading thread i handles queue entry
    // shadeOrder[i] (queue entries grouped by shade_key); null = queue order
    const uint32_t* shadeOrder;
    // the counting sort's buffers: a key byte per queue entry, the order, and
    // 16 counters (bin counts, bin cursors)
    uint8_t* shadeKeys;
    uint32_t* shadeOrderBuf;
    uint32_t* shadeBins;
};

// Shading-queue bins (shade_key): a miss; a Dielectric with its Lambertian
// lobe only; a Dielectric with both lobes; a Conductor; plus kShadeGuided for
// a vertex the guide samples. Threads of one warp then mostly take the same
// branches of the shading kernel.
constexpr uint32_t kShadeBins = 8;
constexpr uint32_t kShadeGuided = 4;

struct IntegratorKernels {
    void (*generate)(const SceneView&, const WaveView&, bool streamRng, cudaStream_t);
    void (*shade)(const SceneView&, const WaveView&, bool streamRng, uint32_t maxQueue, cudaStream_t);
    void (*resolve)(const WaveView&, uint32_t maxQueue, cudaStream_t);
    void (*accumulate)(const WaveView&, float* accum, double* accum64, bool streamRng, cudaStream_t);
    // guiding: queries of the current queue; recorded vertices -> training samples
    void (*guide_query)(const SceneView&, const WaveView&, uint32_t maxQueue, cudaStream_t);
    void (*train_finalize)(const WaveView&, guide::Sample* out, uint32_t* outCount, cudaStream_t);
    // shading order of the current queue: bins[0..7] counts, bins[8..15]
    // cursors (both zeroed by the caller), keys: one byte per queue entry,
    // order: the queue entries grouped by bin
    void (*sort)(const SceneView&, const WaveView&, uint32_t maxQueue, uint32_t* bins, uint8_t* keys,
                 uint32_t* order, cudaStream_t);
};

const IntegratorKernels& integrator_fast();
const IntegratorKernels& integrator_exact();

}  // namespace ag

#ifdef AG_INTEGRATOR_NS
namespace ag {
namespace AG_INTEGRATOR_NS {

constexpr int kThreads = 128;

// Random numbers of one path: the reference's per-pixel xorshift stream, or
// the counter hash.
struct PathRng {
    bool stream;
    XorShift128 xs;
    CounterRng cr;
    AG_D void load(uint4 s)
    {
        if (stream) {
            xs.s[0] = s.x; xs.s[1] = s.y; xs.s[2] = s.z; xs.s[3] = s.w;
        } else {
            cr.key = ((uint64_t)s.y << 32) | s.x;
            cr.dim = s.z;
        }
    }
    AG_D uint4 save() const
    {
        if (stream) return make_uint4(xs.s[0], xs.s[1], xs.s[2], xs.s[3]);
        return make_uint4((uint32_t)cr.key, (uint32_t)(cr.key >> 32), cr.dim, 0u);
    }
    AG_D float next() { return stream ? xorshift_1d(xs) : counter_1d(cr); }
};

// Appends one entry per calling lane with pred set: one atomic per warp.
AG_D uint32_t warp_append(uint32_t* counter, bool pred)
{
    const uint32_t am = __activemask();
    const uint32_t m = __ballot_sync(am, pred);
    uint32_t base = 0;
    const int leader = m ? __ffs(m) - 1 : __ffs(am) - 1;
    if (m && (int)(threadIdx.x & 31) == leader) base = atomicAdd(counter, __popc(m));
    base = __shfl_sync(am, base, leader);
    return base + __popc(m & lanemask_lt());
}

AG_D float4 f4(float3 v, float w = 0.0f) { return make_float4(v.x, v.y, v.z, w); }
AG_D float3 f3(float4 v) { return mk3(v.x, v.y, v.z); }

// Shading-kernel code size: specialising k_shade per light-sampler kind keeps
// one sampler's code in each kernel, and an out-of-line material sample keeps
// one copy of the BSDF sampling code; both against instruction-cache misses.
#ifndef AG_SHADE_SPECIALISE
#define AG_SHADE_SPECIALISE 1
#endif
#ifndef AG_SHADE_NOINLINE_BSDF
#define AG_SHADE_NOINLINE_BSDF 1  // measured: +28% samples/s on the room (one copy of the sampling code)
#endif
#ifndef AG_SHADE_NOINLINE_EVAL
#define AG_SHADE_NOINLINE_EVAL 0
#endif
#ifndef AG_SHADE_NOINLINE_LIGHT
#define AG_SHADE_NOINLINE_LIGHT 1  // measured: +5% (room), +8% (light BVH)
#endif
#if AG_SHADE_NOINLINE_EVAL
__device__ __noinline__
#else
AG_D
#endif
float eval_material(const Material& m, float3 wo, float3 wi, float3& bsdf)
{
    const float pdf = mat_pdf(m, wo, wi);
    if (pdf > 0.0f) bsdf = mat_bsdf(m, wo, wi);
    return pdf;
}
#if AG_SHADE_NOINLINE_LIGHT
__device__ __noinline__
#else
AG_D
#endif
bool sample_light_point(const Light& l, float u0, float u1, float3 hit, LightSample& out)
{
    return light_sample(l, u0, u1, hit, out);
}
#if AG_SHADE_NOINLINE_LIGHT
__device__ __noinline__
#else
AG_D
#endif
float light_density(const Light& l, float3 hit, float3 wi, float& dist)
{
    return light_pdf(l, hit, wi, dist);
}
#if AG_SHADE_NOINLINE_BSDF
__device__ __noinline__ bool sample_material(const Material& m, float3 wo, float u0, float u1, BsdfSample& out)
{
    return mat_sample(m, wo, u0, u1, out);
}
#else
AG_D bool sample_material(const Material& m, float3 wo, float u0, float u1, BsdfSample& out)
{
    return mat_sample(m, wo, u0, u1, out);
}
#endif

__global__ void __launch_bounds__(kThreads) k_generate(SceneView sc, WaveView w, bool streamRng)
{
    uint32_t p = blockIdx.x * kThreads + threadIdx.x;
    if (p >= w.numPaths) return;
    uint32_t slice = p / w.numPixels;
    uint32_t pixel = w.pixelBase + p % w.numPixels;
    PathRng r;
    r.stream = streamRng;
    if (streamRng) r.load(w.pixelRng[pixel]);
    else counter_init(r.cr, w.seed, pixel, w.sampleBase + (w.sampleBaseDev ? *w.sampleBaseDev : 0u) + slice);
    uint32_t x = pixel % sc.width, y = pixel / sc.width;
    // Sampler::get2D draws x then y (src/sampler.cpp:24-27)
    float jx = r.next();
    float jy = r.next();
    float3 org, dir;
    camera_ray(sc.cam, ((float)x + jx) / (float)sc.width, ((float)y + jy) / (float)sc.height, org, dir);
    w.thr[p] = make_float4(1.0f, 1.0f, 1.0f, 0.0f);
    w.rad[p] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    w.albedo[p] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    w.nrm[p] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    w.pendShadow[p] = make_int2(-1, -1);
    if (w.trainSlot) w.trainSlot[p] = -1;
    w.rng[p] = r.save();
    alpine_gpu_ray ray;
    ray.org[0] = org.x; ray.org[1] = org.y; ray.org[2] = org.z;
    ray.tmin = 0.0f;
    ray.dir[0] = dir.x; ray.dir[1] = dir.y; ray.dir[2] = dir.z;
    ray.tmax = 3.402823466e38f;
    w.rays[p] = ray;
    w.queuePath[p] = p;
    if (p == 0) *w.queueCount = w.numPaths;
}

// Surface attributes at a hit (Mesh::getIntersectionAttributes, mesh.cpp:57-154).
struct Surface {
    float3 ng;      // Primitive::ng = normalize(cross(e0, e1)) (bvh_common.cpp:114-117)
    float3 ns;      // interpolated vertex normal (b0 = 1 - b1 - b2), not re-normalised; else ng
    Material mat;
};

AG_D void surface_at(const SceneView& sc, const uint4 h, float3 ro, float3 rd, Surface& s)
{
    const uint32_t prim = h.x;
    if (prim & kSpherePrim) {
        // Sphere::getIntersectionAttributes (src/shapes/sphere.cpp:23-37):
        // ns = ng, the outward normal at the hit; the sphere's material
        uint32_t k = prim & ~kSpherePrim;
        if (k >= sc.sphereCount) k = 0;
        const float4 sp = sc.spheres[k];
        const float3 hit = ro + rd * __uint_as_float(h.y);
        s.ng = normalize3(hit - mk3(sp.x, sp.y, sp.z));
        s.ns = s.ng;
        uint32_t mid = sc.sphereMaterial[k];
        if (mid >= sc.materialCount) mid = 0;
        s.mat = sc.materials[mid];
        if (s.mat.baseTex && s.mat.baseTex <= sc.textureCount) {  // uv = 0 on a sphere
            const float4 t = texture_sample(sc.textures[s.mat.baseTex - 1u], sc.texels, 0.0f, 0.0f);
            s.mat.r = t.x;
            s.mat.g = t.y;
            s.mat.b = t.z;
        }
        return;
    }
    const float b1 = __uint_as_float(h.z), b2 = __uint_as_float(h.w);
    const uint32_t* ti = sc.idx + 3ull * prim;
    const uint32_t i0 = ti[0], i1 = ti[1], i2 = ti[2];
    const float3 v0 = mk3(sc.verts[3ull * i0], sc.verts[3ull * i0 + 1], sc.verts[3ull * i0 + 2]);
    const float3 v1 = mk3(sc.verts[3ull * i1], sc.verts[3ull * i1 + 1], sc.verts[3ull * i1 + 2]);
    const float3 v2 = mk3(sc.verts[3ull * i2], sc.verts[3ull * i2 + 1], sc.verts[3ull * i2 + 2]);
    s.ng = normalize3(cross(v1 - v0, v2 - v0));
    const uint32_t info = sc.triInfo[prim];
    uint32_t mid = info & kTriMaterialMask;
    if (mid >= sc.materialCount) mid = 0;
    s.mat = sc.materials[mid];
    const float b0 = 1.0f - b1 - b2;
    float2 uv = make_float2(0.0f, 0.0f);
    if (info & kTriHasUvs) {  // mesh.cpp:66-74
        uv.x = sc.uvs[2ull * i0] * b0 + sc.uvs[2ull * i1] * b1 + sc.uvs[2ull * i2] * b2;
        uv.y = sc.uvs[2ull * i0 + 1] * b0 + sc.uvs[2ull * i1 + 1] * b1 + sc.uvs[2ull * i2 + 1] * b2;
    }
    // Material::getBaseColor(uv) (dielectric.cpp:97-101, conductor.cpp:45-49):
    // the texture replaces the constant colour everywhere the material uses it
    if (s.mat.baseTex && s.mat.baseTex <= sc.textureCount) {
        const float4 t = texture_sample(sc.textures[s.mat.baseTex - 1u], sc.texels, uv.x, uv.y);
        s.mat.r = t.x;
        s.mat.g = t.y;
        s.mat.b = t.z;
    }
    if (info & kTriHasNormals) {
        const float3 n0 = mk3(sc.normals[3ull * i0], sc.normals[3ull * i0 + 1], sc.normals[3ull * i0 + 2]);
        const float3 n1 = mk3(sc.normals[3ull * i1], sc.normals[3ull * i1 + 1], sc.normals[3ull * i1 + 2]);
        const float3 n2 = mk3(sc.normals[3ull * i2], sc.normals[3ull * i2 + 1], sc.normals[3ull * i2 + 2]);
        s.ns = n0 * b0 + n1 * b1 + n2 * b2;
        // a morphed normal is re-normalised (mesh.cpp:86-101)
        if (info & kTriMorphedNormals) s.ns = normalize3(s.ns);
        if (info & kTriHasTangents) {
            // tangent space (mesh.cpp:104-144): per corner the tangent and the
            // bitangent normalize(cross(n, t) * sign), both interpolated; the
            // normal-map value v (0, 0, 1 without a map) gives
            // ns = normalize(bitangent v.x + tangent v.y + ns v.z)
            const uint32_t ci[3] = {i0, i1, i2};
            const float3 nc[3] = {n0, n1, n2};
            const float bw[3] = {b0, b1, b2};
            float3 tan = mk3(0.0f, 0.0f, 0.0f), bit = mk3(0.0f, 0.0f, 0.0f);
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                const float* tp = sc.tangents + 4ull * ci[k];
                const float3 t = mk3(tp[0], tp[1], tp[2]);
                const float3 bt = normalize3(cross(nc[k], t) * tp[3]);
                tan = k == 0 ? t * bw[0] : tan + t * bw[k];
                bit = k == 0 ? bt * bw[0] : bit + bt * bw[k];
            }
            float3 v = mk3(0.0f, 0.0f, 1.0f);
            if (s.mat.normalTex && s.mat.normalTex <= sc.textureCount) {
                const float4 t = texture_sample(sc.textures[s.mat.normalTex - 1u], sc.texels, uv.x, uv.y);
                v = mk3(t.x, t.y, t.z);
            }
            s.ns = normalize3(bit * v.x + tan * v.y + s.ns * v.z);
        }
    } else {
        s.ns = s.ng;
    }
}

AG_D alpine_gpu_ray make_ray(float3 o, float3 d, float tmax)
{
    alpine_gpu_ray r;
    r.org[0] = o.x; r.org[1] = o.y; r.org[2] = o.z;
    r.tmin = 0.0f;
    r.dir[0] = d.x; r.dir[1] = d.y; r.dir[2] = d.z;
    r.tmax = tmax;
    return r;
}

// One-sample MIS continuation: the direction comes from the guide's mixture
// with probability alpha, else from the material's procedure; either way the
// weight is f / (alpha p_guide + (1 - alpha) p_mat) with f and p_mat the
// material procedure's effective integrand and true density (plain_eval),
// an unbiased estimate of what the material's own sampling estimates. The
// mixture (guide::kPacked fields `stride` apart, world space) is read lobe
// by lobe; its density is evaluated at the world-space direction.
AG_D bool guided_continuation(const Material& mat, float3 wo, const float* lobes, uint32_t stride, float alpha,
                              float3 ss, float3 ts, float3 ns, PathRng& rng, float3& wi, float3& est)
{
    const float us = rng.next();
    const float u0 = rng.next();
    const float u1 = rng.next();
    const float u2 = rng.next();
    if (us < alpha) {
        wi = normalize3(to_local(guide::lobes_sample(lobes, stride, u0, u1, u2), ss, ts, ns));
    } else {
        BsdfSample ms;
        if (!sample_material(mat, wo, u0, u1, ms)) return false;
        wi = ms.wi;
    }
    float pm;
    float3 fcos;
    if (!plain_eval(mat, wo, wi, pm, fcos)) return false;  // outside the procedure's support: f = 0
    float pg = guide::lobes_pdf(lobes, stride, normalize3(to_world(wi, ss, ts, ns)));
    if (!(pg >= 0.0f && pg < 3.0e38f)) pg = 0.0f;
    const float qm = alpha * pg + (1.0f - alpha) * pm;
    if (!(qm > 0.0f)) return false;
    est = fcos / qm;
    return true;
}

// Guide queries of the vertices of the current queue that will be guided
// (a hit, the view direction above the shading surface, material alpha >=
// guideMinRough), compacted: shading position, roughness, direction towards
// the previous vertex and shading normal.
__global__ void __launch_bounds__(kThreads) k_guide_query(SceneView sc, WaveView w)
{
    const uint32_t n = *w.queueCount;
    uint32_t q = blockIdx.x * kThreads + threadIdx.x;
    if (q >= n) return;
    const uint4 h = w.hits[q];
    bool guided = false;
    guide::Query gq = {};
    if (h.x != 0xffffffffu) {
        const alpine_gpu_ray ray = w.rays[q];
        Surface sf;
        const float3 rd = mk3(ray.dir[0], ray.dir[1], ray.dir[2]);
        surface_at(sc, h, mk3(ray.org[0], ray.org[1], ray.org[2]), rd, sf);
        // wo.z of the shading frame: to_local(-rd, ss, ts, ns).z
        guided = dot(sf.ns, -rd) > 0.0f && sf.mat.ax >= w.guideMinRough;
        if (guided) {
            const float t = __uint_as_float(h.y);
            const float3 ro = mk3(ray.org[0], ray.org[1], ray.org[2]);
            const float3 hit = ro + rd * t;
            const float3 wo = normalize3(-rd);
            gq.pos[0] = hit.x; gq.pos[1] = hit.y; gq.pos[2] = hit.z;
            gq.rough = sf.mat.ax;
            gq.wo[0] = wo.x; gq.wo[1] = wo.y; gq.wo[2] = wo.z;
            gq.n[0] = sf.ns.x; gq.n[1] = sf.ns.y; gq.n[2] = sf.ns.z;
        }
    }
    const uint32_t slot = warp_append(w.guideCount, guided);
    if (guided) w.guideQuery[slot] = gq;
    w.guideSlot[q] = guided ? (int)slot : -1;
}

// kSampler: the light sampler kind, or -1 to read it from the scene.
// Resident blocks per SM: the shading kernel waits on instruction fetch and
// memory, so more warps beat fewer spills (measured on B200: 14 blocks of
// 128, 32 registers with spills to L1, +28-41 % samples/s over 6 blocks for
// unguided shading; the guided kernel, with more live state, is best at 10).
#ifndef AG_SHADE_MIN_BLOCKS
#define AG_SHADE_MIN_BLOCKS 14
#endif
#ifndef AG_SHADE_MIN_BLOCKS_GUIDED
#define AG_SHADE_MIN_BLOCKS_GUIDED 10
#endif
template <bool kGuided, int kSampler>
__global__ void __launch_bounds__(kThreads, kGuided ? AG_SHADE_MIN_BLOCKS_GUIDED : AG_SHADE_MIN_BLOCKS)
    k_shade(SceneView sc, WaveView w, bool streamRng)
{
    const uint32_t n = *w.queueCount;
    const uint32_t i = blockIdx.x * kThreads + threadIdx.x;
    if (i >= n) return;
    // every arithmetic step below depends on the path only, not on i
    const uint32_t q = w.shadeOrder ? __ldg(w.shadeOrder + i) : i;
    const uint32_t p = w.queuePath[q];
    const uint4 h = w.hits[q];
    const alpine_gpu_ray ray = w.rays[q];
    const float3 ro = mk3(ray.org[0], ray.org[1], ray.org[2]);
    const float3 rd = mk3(ray.dir[0], ray.dir[1], ray.dir[2]);
    float3 thr = f3(w.thr[p]);
    PathRng rng;
    rng.stream = streamRng;
    rng.load(w.rng[p]);
    int2 shadow = make_int2(-1, -1);
    bool cont = false;

    if (h.x == 0xffffffffu) {
        // miss: the environment map, else the background colour (alpine.cpp:318-324)
        float3 rad = f3(w.rad[p]);
        rad += thr * (sc.env ? environment_sample(sc.env, sc.envW, sc.envH, rd) : sc.background);
        w.rad[p] = f4(rad);
    } else {
        const float t = __uint_as_float(h.y);
        Surface sf;
        surface_at(sc, h, ro, rd, sf);
        const float3 ng = sf.ng, ns = sf.ns;
        const Material mat = sf.mat;
        float3 ss, ts;
        get_basis(ns, ss, ts);
        const float3 hit = ro + rd * t;
        if (w.depth == 0) {
            w.albedo[p] = f4(mat_color(mat));
            w.nrm[p] = f4(ns);
        }
        const float3 wo = to_local(-rd, ss, ts, ns);

        // estimateDirectIllumination (alpine.cpp:370-432)
        // the selection number is drawn whenever a sampler exists, even with
        // no lights (LightSampler::sample(sampler.get1D(), ...))
        if ((kSampler >= 0 ? (uint32_t)kSampler : sc.lights.kind) != kSamplerNone) {
            float lssPdf = 0.0f;
            int li = sample_light<kSampler>(sc.lights, rng.next(), hit, ns, lssPdf);
            if (li >= 0) {
                const Light light = sc.lights.lights[li];
                float3 termL = mk3(0.0f, 0.0f, 0.0f), termB = mk3(0.0f, 0.0f, 0.0f);
                const float3 so = hit + ns * kRayOffset;  // shadow rays leave along ns (alpine.cpp:389-395)
                // light sampling
                LightSample ls;
                float lu0 = rng.next();
                float lu1 = rng.next();
                if (sample_light_point(light, lu0, lu1, hit, ls)) {
                    float3 wi = to_local(ls.wi, ss, ts, ns);
                    float3 bsdf;
                    float bsdfPdf = eval_material(mat, wo, wi, bsdf);
                    if (bsdfPdf > 0.0f) {
                        float cosTerm = fmaxf(0.0f, dot(ls.wi, ns));
                        float mis = !light_is_delta(light) ? power_heuristic(ls.pdf, bsdfPdf) : 1.0f;
                        termL = ls.L * mis * bsdf * cosTerm / ls.pdf;
                        uint32_t slot = warp_append(w.shadowCount, true);
                        w.shadowRays[slot] = make_ray(so, ls.wi, ls.distance);
                        shadow.x = (int)slot;
                    }
                }
                // BSDF sampling (non-delta lights only)
                if (!light_is_delta(light)) {
                    BsdfSample ms;
                    float bu0 = rng.next();
                    float bu1 = rng.next();
                    if (sample_material(mat, wo, bu0, bu1, ms)) {
                        float3 lightDir = to_world(ms.wi, ss, ts, ns);
                        float lightDist;
                        float lightPdf = light_density(light, hit, lightDir, lightDist);
                        if (lightPdf > 0.0f) {
                            float3 em = light_emitted(light);
                            float mis = power_heuristic(ms.pdf, lightPdf);
                            termB = em * mis * ms.estimator;
                            uint32_t slot = warp_append(w.shadowCount, true);
                            w.shadowRays[slot] = make_ray(so, lightDir, lightDist);
                            shadow.y = (int)slot;
                        }
                    }
                }
                if (shadow.x >= 0 || shadow.y >= 0) {
                    w.pendL[p] = f4(termL);
                    w.pendB[p] = f4(termB, lssPdf);
                    w.pendThr[p] = f4(thr);
                }
            }
        }

        // continuation (alpine.cpp:342-361); with a guide, one-sample MIS
        // between the guide and the material's procedure
        bool ok;
        float3 wiL, est;
        // guided when the query kernel selected the vertex (and wo.z > 0 here
        // as well, should contraction round the two tests differently)
        const int gslot = kGuided ? w.guideSlot[q] : -1;
        const bool guidable = gslot >= 0 && wo.z > 0.0f;
        if (guidable && w.guideLobes) {
            ok = guided_continuation(mat, wo, w.guideLobes + gslot, w.numPaths, w.guideFraction, ss, ts, ns, rng, wiL,
                                     est);
        } else {
            BsdfSample ms;
            float cu0 = rng.next();
            float cu1 = rng.next();
            ok = sample_material(mat, wo, cu0, cu1, ms);
            wiL = ms.wi;
            est = ms.estimator;
        }
        if (ok) {
            float3 wiW = to_world(wiL, ss, ts, ns);
            if (dot(wiW, ng) > 0.0f) {
                const float3 thrV = thr;
                thr = thr * est;
                cont = w.depth + 1 < sc.maxDepth;
                // Russian roulette (not in the reference; off unless rrStart > 0)
                if (cont && w.rrStart > 0 && w.depth + 1 >= w.rrStart) {
                    float qs = fminf(0.95f, maxc(thr));
                    if (rng.next() >= qs) cont = false;
                    else thr = thr / qs;
                }
                if (cont) {
                    uint32_t slot = warp_append(w.queueCountNext, true);
                    w.raysNext[slot] = make_ray(hit + ng * kRayOffset, wiW, 3.402823466e38f);
                    w.queuePathNext[slot] = p;
                }
                // training record: the radiance this direction brings is
                // (R_final - R_after) / throughput at the vertex
                const bool rec = cont && guidable && w.trainStride &&
                                 (uint32_t)(splitmix64(((uint64_t)w.waveIndex << 32) | p) % w.trainStride) == 0u;
                if (kGuided && w.trainStride) {
                    const uint32_t r = warp_append(w.trainCount, rec);
                    if (rec && r < w.trainCap) {
                        guide::Sample smp;
                        smp.q = w.guideQuery[gslot];
                        const float3 d = normalize3(wiW);
                        smp.dir[0] = d.x; smp.dir[1] = d.y; smp.dir[2] = d.z;
                        smp.weight = 0.0f;
                        w.trainRec[r] = smp;
                        w.trainAux[2ull * r] = make_float4(0.0f, 0.0f, 0.0f, __uint_as_float(p));
                        w.trainAux[2ull * r + 1] = f4(thrV);
                        w.trainSlot[p] = (int)r;
                    }
                }
                w.thr[p] = f4(thr);
            }
        }
    }
    w.pendShadow[p] = shadow;
    w.rng[p] = rng.save();
}

AG_D uint32_t shade_key(const SceneView& sc, const WaveView& w, uint32_t q)
{
    const uint32_t prim = w.hits[q].x;
    uint32_t key = 0;
    if (prim != 0xffffffffu) {
        uint32_t mid = (prim & kSpherePrim) ? sc.sphereMaterial[min(prim & ~kSpherePrim, sc.sphereCount - 1u)]
                                            : __ldg(sc.triInfo + prim) & kTriMaterialMask;
        if (mid >= sc.materialCount) mid = 0;
        const Material& m = sc.materials[mid];
        key = m.kind == kMatConductor ? 3u : (m.lobes == 2u ? 2u : 1u);
        if (w.guideSlot && w.guideLobes && w.guideSlot[q] >= 0) key |= kShadeGuided;
    }
    return key;
}

// Warp-aggregated rank of this thread among the block's threads with the
// same key, added to hist[key] (shared memory).
AG_D uint32_t bin_rank(uint32_t* hist, uint32_t key)
{
    const uint32_t am = __activemask();
    const uint32_t peers = __match_any_sync(am, key);
    const int leader = __ffs(peers) - 1;
    uint32_t base = 0;
    if ((int)(threadIdx.x & 31) == leader) base = atomicAdd(hist + key, __popc(peers));
    base = __shfl_sync(am, base, leader);
    return base + __popc(peers & lanemask_lt());
}

// Pass 1 of the shading-order counting sort: the key of every queue entry
// and the global count of each bin.
__global__ void __launch_bounds__(kThreads) k_shade_bins(SceneView sc, WaveView w, uint32_t* bins, uint8_t* keys)
{
    __shared__ uint32_t hist[kShadeBins];
    if (threadIdx.x < kShadeBins) hist[threadIdx.x] = 0;
    __syncthreads();
    const uint32_t n = *w.queueCount;
    const uint32_t q = blockIdx.x * kThreads + threadIdx.x;
    if (q < n) {
        const uint32_t key = shade_key(sc, w, q);
        keys[q] = (uint8_t)key;
        bin_rank(hist, key);
    }
    __syncthreads();
    if (threadIdx.x < kShadeBins && hist[threadIdx.x]) atomicAdd(bins + threadIdx.x, hist[threadIdx.x]);
}

// Pass 2: each block reserves a run in every bin it holds (bin start =
// counts of the lower bins, then a cursor) and writes its entries there.
// The order inside a bin depends on scheduling; shading results do not.
__global__ void __launch_bounds__(kThreads) k_shade_scatter(WaveView w, uint32_t* bins, const uint8_t* keys,
                                                            uint32_t* order)
{
    __shared__ uint32_t hist[kShadeBins], base[kShadeBins];
    if (threadIdx.x < kShadeBins) hist[threadIdx.x] = 0;
    __syncthreads();
    const uint32_t n = *w.queueCount;
    const uint32_t q = blockIdx.x * kThreads + threadIdx.x;
    uint32_t key = 0, rank = 0;
    if (q < n) {
        key = keys[q];
        rank = bin_rank(hist, key);
    }
    __syncthreads();
    if (threadIdx.x < kShadeBins && hist[threadIdx.x]) {
        uint32_t start = 0;
        for (uint32_t k = 0; k < threadIdx.x; ++k) start += bins[k];
        base[threadIdx.x] = start + atomicAdd(bins + kShadeBins + threadIdx.x, hist[threadIdx.x]);
    }
    __syncthreads();
    if (q < n) order[base[key] + rank] = q;
}

__global__ void __launch_bounds__(kThreads) k_resolve(WaveView w)
{
    const uint32_t n = *w.queueCount;
    uint32_t q = blockIdx.x * kThreads + threadIdx.x;
    if (q >= n) return;
    const uint32_t p = w.queuePath[q];
    const int2 s = w.pendShadow[p];
    if (s.x >= 0 || s.y >= 0) {
        const bool visL = s.x >= 0 && !w.shadowOcc[s.x];
        const bool visB = s.y >= 0 && !w.shadowOcc[s.y];
        if (visL || visB) {
            // radiance(local) = 0; += light term; += BSDF term; / selection pdf
            const float4 pb = w.pendB[p];
            float3 direct = mk3(0.0f, 0.0f, 0.0f);
            if (visL) direct += f3(w.pendL[p]);
            if (visB) direct += f3(pb);
            direct = direct / pb.w;
            float3 rad = f3(w.rad[p]);
            rad += f3(w.pendThr[p]) * direct;
            w.rad[p] = f4(rad);
        }
        w.pendShadow[p] = make_int2(-1, -1);
    }
    if (w.trainSlot) {
        const int r = w.trainSlot[p];
        if (r >= 0) {
            const float4 rad = w.rad[p];
            w.trainAux[2ull * r] = make_float4(rad.x, rad.y, rad.z, __uint_as_float(p));
            w.trainSlot[p] = -1;
        }
    }
}

// Training samples of the wave's recorded vertices: weight = luminance of
// (R_final - R_after) / throughput, i.e. f cos Li / q of the sampled
// direction; vertices that received no radiance are dropped.
__global__ void __launch_bounds__(kThreads) k_train_finalize(WaveView w, guide::Sample* out, uint32_t* outCount)
{
    const uint32_t n = min(*w.trainCount, w.trainCap);
    const uint32_t r = blockIdx.x * kThreads + threadIdx.x;
    float wgt = 0.0f;
    if (r < n) {
        const float4 a0 = w.trainAux[2ull * r], a1 = w.trainAux[2ull * r + 1];
        const uint32_t path = __float_as_uint(a0.w);
        const float4 R = w.rad[path];
        const float dx = R.x - a0.x, dy = R.y - a0.y, dz = R.z - a0.z;
        const float lx = a1.x > 0.0f ? dx / a1.x : 0.0f;
        const float ly = a1.y > 0.0f ? dy / a1.y : 0.0f;
        const float lz = a1.z > 0.0f ? dz / a1.z : 0.0f;
        wgt = 0.2126f * lx + 0.7152f * ly + 0.0722f * lz;
        if (!(wgt > 0.0f && wgt < 3.0e38f)) wgt = 0.0f;
    }
    if (r >= ((n + 31u) & ~31u)) return;  // whole warps from here on
    const bool keep = wgt > 0.0f;
    const uint32_t slot = warp_append(outCount, keep);
    if (keep) {
        guide::Sample smp = w.trainRec[r];
        smp.weight = wgt;
        out[slot] = smp;
    }
}

// Adds the wave's per-sample results to the per-pixel sums in sample order
// (the reference adds sample after sample, alpine.cpp:364).
__global__ void __launch_bounds__(kThreads) k_accumulate(WaveView w, float* accum, double* accum64, bool streamRng)
{
    uint32_t i = blockIdx.x * kThreads + threadIdx.x;
    if (i >= w.numPixels) return;
    const uint32_t pixel = w.pixelBase + i;
    if (accum64) {
        double* a = accum64 + 9ull * pixel;
        double s[9];
        for (int k = 0; k < 9; ++k) s[k] = a[k];
        for (uint32_t sl = 0; sl < w.samplesInWave; ++sl) {
            uint32_t p = sl * w.numPixels + i;
            float4 c = w.rad[p], al = w.albedo[p], nm = w.nrm[p];
            s[0] += c.x; s[1] += c.y; s[2] += c.z;
            s[3] += al.x; s[4] += al.y; s[5] += al.z;
            s[6] += nm.x; s[7] += nm.y; s[8] += nm.z;
        }
        for (int k = 0; k < 9; ++k) a[k] = s[k];
    } else {
        float* a = accum + 9ull * pixel;
        float s[9];
        for (int k = 0; k < 9; ++k) s[k] = a[k];
        for (uint32_t sl = 0; sl < w.samplesInWave; ++sl) {
            uint32_t p = sl * w.numPixels + i;
            float4 c = w.rad[p], al = w.albedo[p], nm = w.nrm[p];
            s[0] += c.x; s[1] += c.y; s[2] += c.z;
            s[3] += al.x; s[4] += al.y; s[5] += al.z;
            s[6] += nm.x; s[7] += nm.y; s[8] += nm.z;
        }
        for (int k = 0; k < 9; ++k) a[k] = s[k];
    }
    if (streamRng) w.pixelRng[pixel] = w.rng[i];  // one sample per pixel per wave in stream mode
}

inline unsigned grid(uint32_t n) { return (n + kThreads - 1) / kThreads; }

template <bool kGuided>
void launch_shade(const SceneView& sc, const WaveView& w, bool streamRng, uint32_t maxQueue, cudaStream_t st)
{
#if AG_SHADE_SPECIALISE
    switch (sc.lights.kind) {
    case kSamplerUniform: k_shade<kGuided, kSamplerUniform><<<grid(maxQueue), kThreads, 0, st>>>(sc, w, streamRng); break;
    case kSamplerPower: k_shade<kGuided, kSamplerPower><<<grid(maxQueue), kThreads, 0, st>>>(sc, w, streamRng); break;
    case kSamplerBvh: k_shade<kGuided, kSamplerBvh><<<grid(maxQueue), kThreads, 0, st>>>(sc, w, streamRng); break;
    default: k_shade<kGuided, kSamplerNone><<<grid(maxQueue), kThreads, 0, st>>>(sc, w, streamRng); break;
    }
#else
    k_shade<kGuided, -1><<<grid(maxQueue), kThreads, 0, st>>>(sc, w, streamRng);
#endif
}

void generate(const SceneView& sc, const WaveView& w, bool streamRng, cudaStream_t st)
{
    if (w.numPaths) k_generate<<<grid(w.numPaths), kThreads, 0, st>>>(sc, w, streamRng);
}
void shade(const SceneView& sc, const WaveView& w, bool streamRng, uint32_t maxQueue, cudaStream_t st)
{
    if (!maxQueue) return;
    if (w.guideQuery) launch_shade<true>(sc, w, streamRng, maxQueue, st);
    else launch_shade<false>(sc, w, streamRng, maxQueue, st);
}
void resolve(const WaveView& w, uint32_t maxQueue, cudaStream_t st)
{
    if (maxQueue) k_resolve<<<grid(maxQueue), kThreads, 0, st>>>(w);
}
void accumulate(const WaveView& w, float* accum, double* accum64, bool streamRng, cudaStream_t st)
{
    if (w.numPixels) k_accumulate<<<grid(w.numPixels), kThreads, 0, st>>>(w, accum, accum64, streamRng);
}
void guide_query(const SceneView& sc, const WaveView& w, uint32_t maxQueue, cudaStream_t st)
{
    if (maxQueue) k_guide_query<<<grid(maxQueue), kThreads, 0, st>>>(sc, w);
}
void train_finalize(const WaveView& w, guide::Sample* out, uint32_t* outCount, cudaStream_t st)
{
    if (w.trainCap) k_train_finalize<<<grid(w.trainCap), kThreads, 0, st>>>(w, out, outCount);
}
void sort(const SceneView& sc, const WaveView& w, uint32_t maxQueue, uint32_t* bins, uint8_t* keys, uint32_t* order,
          cudaStream_t st)
{
    if (!maxQueue) return;
    k_shade_bins<<<grid(maxQueue), kThreads, 0, st>>>(sc, w, bins, keys);
    k_shade_scatter<<<grid(maxQueue), kThreads, 0, st>>>(w, bins, keys, order);
}

}  // namespace AG_INTEGRATOR_NS
}  // namespace ag
#endif
