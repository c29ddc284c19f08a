// Test infrastructure (oracle): a C-ABI harness around the UNMODIFIED reference
// sources, compiled from the reference tree by oracle/Makefile into
// oracle/_ref/libalpine_ref.so. It is used only by the tests, by smoke() as the
// checker, and by bench.py's CPU-baseline / `--impl reference` arms.
//
// Two parts:
//  * ref_accel_*  : drive alpine::Bvh / alpine::WideBvh directly through the
//                   reference's Accelerator interface
//                   (src/accelerators/accelerator.h:13-39) with a thread pool
//                   calling intersect / intersectAny, as a microbenchmark
//                   would.
//  * ref_render_* : drive the reference integrator (class Alpine in
//                   src/alpine.cpp) through its own methods. alpine.cpp is
//                   included into this translation unit with `private`
//                   redefined so that the HDR accumulator (mAccumBuffer,
//                   mTotalSamples; src/alpine.cpp:109-112) can be read back.
//                   No reference file is modified.
//
// Built a second time with ALPINE_GPU_PLUGIN defined (oracle/_ref/
// libalpine_ref_plugin.so), the harness also installs the GPU plug-in that a
// maintainer adds to the reference (alpine_b200/plugin): accelerator kinds
// 2 / 3 (ref_accel_create) and AcceleratorType values 3 / 4
// (ref_render_reset_scene) are the GpuAccelerator with the 8-wide / binary
// triangle rule, as a new `case AcceleratorType::Gpu` in Alpine::resetScene
// would create it; ref_render_gpu_branch switches the Alpine methods to the
// GpuBackend render branch, each entry point below forwarding to it as the
// maintainer's branch in alpine.cpp would.
//
// The reference's loaders need tinyobjloader / tinygltf / stb, which are not
// vendored; this harness therefore defines loadObj and loadHdr
// (src/loaders/file_loader.h:10-12): loadObj is a minimal reader for the
// `v / vn / f / usemtl / mtllib Kd` subset, building Mesh::Data the way
// src/loaders/obj_loader.cpp:45-119 does; HDR loading reports failure. The
// reference's own GLB loader (src/loaders/gltf_loader.cpp) is compiled
// unchanged against refshim/tinygltf/tiny_gltf.h, a stand-in for tinygltf's
// model filled by the project's GLB reader.

// Standard headers first, so that the `private` redefinition below only
// reaches the reference's own headers.
#include <algorithm>
#include <array>
#include <atomic>
#include <cassert>
#include <cfloat>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <functional>
#include <future>
#include <limits>
#include <map>
#include <memory>
#include <memory_resource>
#include <mutex>
#include <numbers>
#include <optional>
#include <span>
#include <sstream>
#include <string>
#include <string_view>
#include <thread>
#include <tuple>
#include <utility>
#include <vector>

#define private public
#include "alpine.cpp"
#undef private

#include <accelerators/bvh.h>
#include <accelerators/wide_bvh.h>
#ifdef ALPINE_GPU_PLUGIN
#include <gpu_accelerator.h>
#include <gpu_backend.h>
#endif
#include <environment_map.h>
#include <texture.h>
#include <materials/conductor.h>
#include <materials/dielectric.h>
#include <shapes/mesh.h>
#include <intersection.h>
#include <ray.h>

namespace alpine {
// ---------------------------------------------------------------------------
// Loaders (see file header).
bool
loadObj(Scene* scene, std::string_view filename)
{
    std::ifstream in{std::string(filename)};
    if (!in)
    {
        printf("ERROR: cannot open %s\n", std::string(filename).c_str());
        return false;
    }
    std::string dir(filename);
    auto slash = dir.find_last_of('/');
    dir = slash == std::string::npos ? std::string() : dir.substr(0, slash + 1);

    std::map<std::string, float3> kd;
    std::vector<std::string> names;
    Mesh::Data data;
    std::vector<std::shared_ptr<Material>> mats;
    std::map<std::string, uint32_t> matIndex;
    int32_t current = -1;

    auto loadMtl = [&](const std::string& file) {
        std::ifstream m(dir + file);
        std::string line, cur;
        while (std::getline(m, line))
        {
            std::istringstream ls(line);
            std::string tok;
            ls >> tok;
            if (tok == "newmtl") { ls >> cur; kd[cur] = float3(0.0f); }
            else if (tok == "Kd") { float r, g, b; ls >> r >> g >> b; kd[cur] = float3(r, g, b); }
        }
    };

    std::string line;
    while (std::getline(in, line))
    {
        std::istringstream ls(line);
        std::string tok;
        ls >> tok;
        if (tok == "v") { float x, y, z; ls >> x >> y >> z; data.vertices.push_back(float3(x, y, z)); }
        else if (tok == "vn") { float x, y, z; ls >> x >> y >> z; data.normals.push_back(float3(x, y, z)); }
        else if (tok == "mtllib") { std::string f; ls >> f; loadMtl(f); }
        else if (tok == "usemtl")
        {
            std::string n; ls >> n;
            auto it = matIndex.find(n);
            if (it == matIndex.end())
            {
                // obj_loader.cpp:73-75: every OBJ material is Dielectric(alpha = 1).
                mats.push_back(std::make_shared<Dielectric>(float2(1.0f), kd[n], nullptr, nullptr));
                it = matIndex.emplace(n, static_cast<uint32_t>(mats.size() - 1)).first;
            }
            current = static_cast<int32_t>(it->second);
        }
        else if (tok == "f")
        {
            uint32_t v[3], n[3];
            bool hasN = true;
            for (int k = 0; k < 3; ++k)
            {
                std::string f; ls >> f;
                v[k] = static_cast<uint32_t>(std::stoul(f)) - 1;
                auto p = f.find("//");
                if (p != std::string::npos) { n[k] = static_cast<uint32_t>(std::stoul(f.substr(p + 2))) - 1; }
                else
                {
                    auto p1 = f.find('/');
                    auto p2 = p1 == std::string::npos ? p1 : f.find('/', p1 + 1);
                    if (p2 != std::string::npos) { n[k] = static_cast<uint32_t>(std::stoul(f.substr(p2 + 1))) - 1; }
                    else { hasN = false; n[k] = 0; }
                }
            }
            if (current < 0)
            {
                printf("ERROR: face without material in %s\n", std::string(filename).c_str());
                return false;
            }
            data.prims.push_back(uint3(v[0], v[1], v[2]));
            if (hasN) { data.normalPrims.push_back(uint3(n[0], n[1], n[2])); }
            data.materials.push_back(mats[current]);
        }
    }
    if (data.normalPrims.size() != data.prims.size()) { data.normalPrims.clear(); data.normals.clear(); }
    scene->shapes.push_back(std::make_shared<Mesh>(std::move(data), 0));
    return true;
}


bool
loadHdr(std::unique_ptr<EnvironmentMap>&, std::string_view)
{
    printf("ERROR: HDR loading needs stb_image, which is not vendored.\n");
    return false;
}
}

using namespace alpine;

namespace {
// Project-written oracle light (the reference has point and disk lights only):
// a one-sided parallelogram corner + u * edgeU + v * edgeV of constant
// radiance, emitting on the side of cross(edgeU, edgeV), following the
// DiskLight contract (src/lights/disk_light.cpp:30-81): area sampling with
// pdf = d^2 / (A cos), computePdf by ray/plane intersection.
class QuadLight final : public Light
{
public:
    QuadLight(const float3& radiance, const float3& corner, const float3& eu, const float3& ev)
        : mRadiance(radiance), mEu(eu), mEv(ev)
    {
        mPosition = corner;
        float3 n = cross(eu, ev);
        mArea = length(n);
        mNormal = n / mArea;
        float3 c[4] = {corner, corner + eu, corner + ev, corner + eu + ev};
        for (const auto& p : c) { mBbox = merge(mBbox, BoundingBox{p, p}); }
    }

    std::optional<Sample> sample(const float2& u, const float3& hit) const override
    {
        float3 p = mPosition + mEu * u.x + mEv * u.y;
        float3 wi = p - hit;
        float d = length(wi);
        if (d == 0.0f) { return {}; }
        wi /= d;
        float c = std::max(0.0f, dot(-wi, mNormal));
        if (c == 0.0f) { return {}; }
        return Sample{mRadiance * mScale, wi, d, (d * d) / (mArea * c)};
    }

    std::pair<float, float> computePdf(const float3& hit, const float3& wi) const override
    {
        float c = std::max(0.0f, dot(-wi, mNormal));
        if (c == 0.0f) { return {0.0f, 0.0f}; }
        float dist = dot(hit - mPosition, mNormal) / c;
        if (dist < 0.0f) { return {0.0f, 0.0f}; }
        float3 q = hit + wi * dist - mPosition;
        float su = dot(q, mEu) / dot(mEu, mEu);
        float sv = dot(q, mEv) / dot(mEv, mEv);
        bool inside = su >= 0.0f && su <= 1.0f && sv >= 0.0f && sv <= 1.0f;
        if (inside && c > 0.0f) { return {(dist * dist) / (mArea * c), dist}; }
        return {0.0f, 0.0f};
    }

    float3 getEmittedRadiance() const override { return mRadiance * mScale; }
    float3 getPower() const override { return mRadiance * (mArea * std::numbers::pi_v<float>) * mScale; }
    bool isDelta() const override { return false; }
    BoundingBox getBoundingBox() const override { return mBbox; }

private:
    float3 mRadiance, mEu, mEv, mNormal;
    float mArea = 0.0f;
    BoundingBox mBbox;
};

struct RefAccel
{
    std::vector<std::byte> arena;
    std::unique_ptr<Accelerator> acc;
    int dummyShape = 0;
};

template <typename F>
void parallelFor(uint64_t n, int nthreads, F&& body)
{
    if (nthreads <= 0)
    {
        nthreads = static_cast<int>(std::max(1u, std::thread::hardware_concurrency()));
    }
    constexpr uint64_t kChunk = 256;
    std::atomic<uint64_t> next{0};
    auto worker = [&]() {
        for (;;)
        {
            uint64_t b = next.fetch_add(kChunk);
            if (b >= n) { break; }
            uint64_t e = std::min(n, b + kChunk);
            for (uint64_t i = b; i < e; ++i) { body(i); }
        }
    };
    std::vector<std::thread> pool;
    for (int t = 1; t < nthreads; ++t) { pool.emplace_back(worker); }
    worker();
    for (auto& th : pool) { th.join(); }
}

inline Ray makeRay(const float* r)
{
    Ray ray;
    ray.org = float3(r[0], r[1], r[2]);
    ray.dir = float3(r[4], r[5], r[6]);
    return ray;
}
}

// Textures added through ref_render_add_texture (the loaders' Texture4f).
static std::vector<std::shared_ptr<Texture4f>> sTextures;

static std::shared_ptr<Texture4f>
texture_or_null(float id)
{
    int32_t i = static_cast<int32_t>(id);
    return (i >= 0 && i < static_cast<int32_t>(sTextures.size())) ? sTextures[i] : nullptr;
}

// One material record {kind, r, g, b, roughness[, base texture, normal
// texture]} as the reference class (kind 0 = Dielectric, 1 = Conductor; the
// loaders' alpha = roughness; texture ids -1 = none).
static std::shared_ptr<Material>
make_ref_material(const float* r, uint32_t stride = 5)
{
    float3 bc(r[1], r[2], r[3]);
    auto bt = stride >= 7 ? texture_or_null(r[5]) : nullptr;
    auto nt = stride >= 7 ? texture_or_null(r[6]) : nullptr;
    if (r[0] == 1.0f) { return std::make_shared<Conductor>(float2(r[4]), bc, bt, nt); }
    return std::make_shared<Dielectric>(float2(r[4]), bc, bt, nt);
}

#ifdef ALPINE_GPU_PLUGIN
// The GPU render branch (GpuBackend) when switched on, and the material
// records of the meshes forwarded to it.
static std::unique_ptr<GpuBackend> sGpu;

static alpine_gpu_material
to_gpu_material(const float* r)
{
    alpine_gpu_material m{};
    m.kind = r[0] == 1.0f ? ALPINE_GPU_MATERIAL_CONDUCTOR : ALPINE_GPU_MATERIAL_DIELECTRIC;
    m.base_color[0] = r[1];
    m.base_color[1] = r[2];
    m.base_color[2] = r[3];
    m.roughness = r[4];
    return m;
}
#endif

extern "C" {
// kind: 0 = Bvh (binary), 1 = WideBvh (8-wide, ISPC kernels restated); in the
// plug-in build 2 / 3 = GpuAccelerator with the 8-wide / binary triangle rule.
void*
ref_accel_create(int kind, uint64_t arenaBytes)
{
    auto* h = new RefAccel;
#ifdef ALPINE_GPU_PLUGIN
    if (kind == 2 || kind == 3)
    {
        h->acc = std::make_unique<GpuAccelerator>(kind == 3 ? GpuAccelerator::Rule::Binary : GpuAccelerator::Rule::Wide);
        return h;
    }
#endif
    h->arena.resize(arenaBytes);
    if (kind == 1)
    {
        h->acc = std::make_unique<WideBvh>(std::span<std::byte>(h->arena));
    }
    else
    {
        h->acc = std::make_unique<Bvh>(std::span<std::byte>(h->arena));
    }
    return h;
}

uint32_t
ref_accel_add_mesh(void* hp, const float* verts, uint32_t nverts, const uint32_t* tris, uint32_t ntris)
{
    auto* h = static_cast<RefAccel*>(hp);
    std::vector<float3> v(nverts);
    for (uint32_t i = 0; i < nverts; ++i) { v[i] = float3(verts[3 * i], verts[3 * i + 1], verts[3 * i + 2]); }
    std::vector<uint3> p(ntris);
    for (uint32_t i = 0; i < ntris; ++i) { p[i] = uint3(tris[3 * i], tris[3 * i + 1], tris[3 * i + 2]); }
    return h->acc->appendMesh(v, p, &h->dummyShape);
}

// The path Mesh::update takes (src/shapes/mesh.cpp:29-55): new positions
// written into the accelerator's vertex buffer of one shape, updateShape, then
// Accelerator::updateScene (full rebuild).
void
ref_accel_update_vertices(void* hp, uint32_t shape, const float* verts, uint32_t nverts)
{
    auto* h = static_cast<RefAccel*>(hp);
    auto* vb = static_cast<float3*>(h->acc->getVertexBuffer(shape));
    for (uint32_t i = 0; i < nverts; ++i) { vb[i] = float3(verts[3 * i], verts[3 * i + 1], verts[3 * i + 2]); }
    h->acc->updateShape(shape);
    h->acc->updateScene();
}

// Returns the wall time of Accelerator::updateScene (full build) in ms.
double
ref_accel_build(void* hp)
{
    auto* h = static_cast<RefAccel*>(hp);
    auto t0 = std::chrono::steady_clock::now();
    h->acc->updateScene();
    auto t1 = std::chrono::steady_clock::now();
    return std::chrono::duration<double, std::milli>(t1 - t0).count();
}

// rays: 8 floats per ray {ox, oy, oz, tmin, dx, dy, dz, tmax}. The reference's
// intersect() has no tmin/tmax (t >= 0, tFar = FLT_MAX); both are ignored here.
// Misses write prim = 0xffffffff, t = FLT_MAX, b1 = b2 = 0.
void
ref_accel_intersect(void* hp, const float* rays, uint64_t n, int nthreads,
    uint32_t* prim, float* t, float* b1, float* b2)
{
    auto* h = static_cast<RefAccel*>(hp);
    parallelFor(n, nthreads, [&](uint64_t i) {
        auto isect = h->acc->intersect(makeRay(rays + 8 * i));
        if (isect.has_value())
        {
            prim[i] = isect->primId;
            t[i] = isect->t;
            b1[i] = isect->barycentric.x;
            b2[i] = isect->barycentric.y;
        }
        else
        {
            prim[i] = 0xffffffffu;
            t[i] = FLT_MAX;
            b1[i] = 0.0f;
            b2[i] = 0.0f;
        }
    });
}

// ref_accel_intersect plus the shapePtr check and the geometric normal of
// every hit (Intersection::shapePtr / ng; ng = 0 on a miss). shape_ok[i] = 1
// when the hit reports the harness's dummy shape pointer.
void
ref_accel_intersect_ng(void* hp, const float* rays, uint64_t n, int nthreads,
    uint32_t* prim, float* t, float* b1, float* b2, float* ng, uint8_t* shape_ok)
{
    auto* h = static_cast<RefAccel*>(hp);
    parallelFor(n, nthreads, [&](uint64_t i) {
        auto isect = h->acc->intersect(makeRay(rays + 8 * i));
        prim[i] = isect ? isect->primId : 0xffffffffu;
        t[i] = isect ? isect->t : FLT_MAX;
        b1[i] = isect ? isect->barycentric.x : 0.0f;
        b2[i] = isect ? isect->barycentric.y : 0.0f;
        for (int k = 0; k < 3; ++k) { ng[3 * i + k] = isect ? isect->ng[k] : 0.0f; }
        shape_ok[i] = isect && isect->shapePtr == &h->dummyShape ? 1 : 0;
    });
}

// intersectAny(ray, tFar = tmax) for each ray; writes 1 when occluded.
void
ref_accel_occluded(void* hp, const float* rays, uint64_t n, int nthreads, uint8_t* occluded)
{
    auto* h = static_cast<RefAccel*>(hp);
    parallelFor(n, nthreads, [&](uint64_t i) {
        occluded[i] = h->acc->intersectAny(makeRay(rays + 8 * i), rays[8 * i + 7]) ? 1 : 0;
    });
}

void
ref_accel_destroy(void* hp)
{
    delete static_cast<RefAccel*>(hp);
}

// ---------------------------------------------------------------------------
// Integrator harness: the public alpine:: API plus direct mesh/material input.
int
ref_render_init(uint32_t width, uint32_t height, uint32_t maxDepth, uint64_t arenaBytes)
{
#ifdef ALPINE_GPU_PLUGIN
    sGpu.reset();
#endif
    sTextures.clear();
    if (sAlpine) { shutdown(); }
    return initialize(static_cast<uint32_t>(arenaBytes), width, height, maxDepth) ? 1 : 0;
}

// acc: AcceleratorType (0 = Bvh, 1 = WideBvh); in the plug-in build 3 / 4 =
// the GpuAccelerator with the 8-wide / binary triangle rule.
void
ref_render_reset_scene(int acc)
{
#ifdef ALPINE_GPU_PLUGIN
    if (acc == 3 || acc == 4)
    {
        resetScene(AcceleratorType::Bvh);
        alpine::alpine().mAccelerator =
            std::make_unique<GpuAccelerator>(acc == 4 ? GpuAccelerator::Rule::Binary : GpuAccelerator::Rule::Wide);
        if (sGpu) { sGpu->resetScene(acc == 4); }
        return;
    }
    if (sGpu) { sGpu->resetScene(acc == 0); }
#endif
    resetScene(static_cast<AcceleratorType>(acc));
}

#ifdef ALPINE_GPU_PLUGIN
// Switches the render branch on (GpuBackend with the Alpine's framebuffer size
// and path depth, counter RNG with `seed`) or off. Call right after
// ref_render_reset_scene, before the scene is added. Returns 1 on success.
int
ref_render_gpu_branch(int enable, uint32_t seed, int binaryRule)
{
    sGpu.reset();
    if (!enable) { return 1; }
    auto& a = alpine::alpine();
    sGpu = std::make_unique<GpuBackend>(a.mWidth, a.mHeight, a.mMaxDepth);
    if (!sGpu->valid() || !sGpu->resetScene(binaryRule != 0)) { sGpu.reset(); return 0; }
    alpine_gpu_render_options o{};
    o.sampler = ALPINE_GPU_SAMPLER_COUNTER;
    o.seed = seed;
    return sGpu->setRenderOptions(o) ? 1 : 0;
}
#endif

// Adds one mesh. materials: `nmat` records of 5 floats {kind, r, g, b, roughness}
// with kind 0 = Dielectric, 1 = Conductor (the two material classes the loaders
// create, gltf_loader.cpp:404-414). normals: per-vertex, may be null.
int
ref_render_add_mesh(const float* verts, uint32_t nverts, const uint32_t* tris, uint32_t ntris,
    const float* normals, const uint32_t* triMaterial, const float* materials, uint32_t nmat)
{
    Mesh::Data d;
    d.vertices.resize(nverts);
    for (uint32_t i = 0; i < nverts; ++i) { d.vertices[i] = float3(verts[3 * i], verts[3 * i + 1], verts[3 * i + 2]); }
    if (normals)
    {
        d.normals.resize(nverts);
        for (uint32_t i = 0; i < nverts; ++i) { d.normals[i] = float3(normals[3 * i], normals[3 * i + 1], normals[3 * i + 2]); }
    }
    std::vector<std::shared_ptr<Material>> mats(nmat);
    for (uint32_t m = 0; m < nmat; ++m) { mats[m] = make_ref_material(materials + 5 * m); }
    d.prims.resize(ntris);
    d.materials.resize(ntris);
    for (uint32_t i = 0; i < ntris; ++i)
    {
        d.prims[i] = uint3(tris[3 * i], tris[3 * i + 1], tris[3 * i + 2]);
        uint32_t m = triMaterial[i];
        if (m >= nmat) { return 0; }
        d.materials[i] = mats[m];
    }
#ifdef ALPINE_GPU_PLUGIN
    if (sGpu)
    {
        std::vector<alpine_gpu_material> recs(nmat);
        for (uint32_t m = 0; m < nmat; ++m) { recs[m] = to_gpu_material(materials + 5 * m); }
        uint32_t base = sGpu->addMaterials(recs);
        std::vector<uint32_t> ids(ntris);
        for (uint32_t i = 0; i < ntris; ++i) { ids[i] = base + triMaterial[i]; }
        if (sGpu->addMesh(d.vertices, d.normals, d.prims, d.normalPrims, ids) < 0) { return 0; }
    }
#endif
    auto mesh = std::make_shared<Mesh>(std::move(d), 0);
    auto& a = alpine::alpine();
    a.mScene.shapes.push_back(mesh);
    mesh->appendTo(a.mAccelerator.get());
    return 1;
}

#ifdef ALPINE_GPU_PLUGIN
#define GPU_BRANCH(call) do { if (sGpu) { sGpu->call; } } while (0)
#else
#define GPU_BRANCH(call) do { } while (0)
#endif

// Texture4f of w x h float4 texels (row-major); returns its id.
int
ref_render_add_texture(const float* rgba, uint32_t w, uint32_t h)
{
    std::vector<float4> d((size_t)w * h);
    for (size_t i = 0; i < d.size(); ++i) { d[i] = float4(rgba[4 * i], rgba[4 * i + 1], rgba[4 * i + 2], rgba[4 * i + 3]); }
#ifdef ALPINE_GPU_PLUGIN
    if (sGpu && sGpu->addTexture(d, w, h) != (int)sTextures.size()) { return -1; }
#endif
    sTextures.push_back(std::make_shared<Texture4f>(w, h, std::move(d)));
    return static_cast<int>(sTextures.size() - 1);
}

// ref_render_add_mesh with texture coordinates (2 per vertex, may be null),
// tangents (4 per vertex, may be null) and 7-float material records
// {kind, r, g, b, roughness, base texture, normal texture}.
int
ref_render_add_mesh_ex(const float* verts, uint32_t nverts, const uint32_t* tris, uint32_t ntris,
    const float* normals, const float* uvs, const float* tangents, const uint32_t* triMaterial,
    const float* materials, uint32_t nmat)
{
    Mesh::Data d;
    d.vertices.resize(nverts);
    for (uint32_t i = 0; i < nverts; ++i) { d.vertices[i] = float3(verts[3 * i], verts[3 * i + 1], verts[3 * i + 2]); }
    if (normals)
    {
        d.normals.resize(nverts);
        for (uint32_t i = 0; i < nverts; ++i) { d.normals[i] = float3(normals[3 * i], normals[3 * i + 1], normals[3 * i + 2]); }
    }
    if (uvs)
    {
        d.uvs.resize(nverts);
        for (uint32_t i = 0; i < nverts; ++i) { d.uvs[i] = float2(uvs[2 * i], uvs[2 * i + 1]); }
    }
    if (tangents)
    {
        d.tangents.resize(nverts);
        for (uint32_t i = 0; i < nverts; ++i)
        {
            d.tangents[i] = float4(tangents[4 * i], tangents[4 * i + 1], tangents[4 * i + 2], tangents[4 * i + 3]);
        }
    }
    std::vector<std::shared_ptr<Material>> mats(nmat);
    for (uint32_t m = 0; m < nmat; ++m) { mats[m] = make_ref_material(materials + 7 * m, 7); }
    d.prims.resize(ntris);
    d.materials.resize(ntris);
    for (uint32_t i = 0; i < ntris; ++i)
    {
        d.prims[i] = uint3(tris[3 * i], tris[3 * i + 1], tris[3 * i + 2]);
        uint32_t m = triMaterial[i];
        if (m >= nmat) { return 0; }
        d.materials[i] = mats[m];
    }
#ifdef ALPINE_GPU_PLUGIN
    if (sGpu)
    {
        std::vector<alpine_gpu_material> recs(nmat);
        for (uint32_t m = 0; m < nmat; ++m) { recs[m] = to_gpu_material(materials + 7 * m); }
        uint32_t base = sGpu->addMaterials(recs);
        for (uint32_t m = 0; m < nmat; ++m)
        {
            const int bt = (int)materials[7 * m + 5], nt = (int)materials[7 * m + 6];
            if (bt >= 0 || nt >= 0) { sGpu->setMaterialTextures(base + m, bt, nt); }
        }
        std::vector<uint32_t> ids(ntris);
        for (uint32_t i = 0; i < ntris; ++i) { ids[i] = base + triMaterial[i]; }
        int sid = sGpu->addMesh(d.vertices, d.normals, d.prims, d.normalPrims, ids);
        if (sid < 0 || !sGpu->setMeshUvs(sid, d.uvs, d.tangents)) { return 0; }
    }
#endif
    auto mesh = std::make_shared<Mesh>(std::move(d), 0);
    auto& a = alpine::alpine();
    a.mScene.shapes.push_back(mesh);
    mesh->appendTo(a.mAccelerator.get());
    return 1;
}

// Alpine::mEnvironmentMap (what loadEnvironmentMap installs): w x h RGB texels.
void
ref_render_set_environment(const float* rgb, uint32_t w, uint32_t h)
{
    auto& a = alpine::alpine();
    if (!rgb) {
        a.mEnvironmentMap.reset();
        GPU_BRANCH(setEnvironmentMap({}, 0, 0));
        return;
    }
    std::vector<float3> d((size_t)w * h);
    for (size_t i = 0; i < d.size(); ++i) { d[i] = float3(rgb[3 * i], rgb[3 * i + 1], rgb[3 * i + 2]); }
    GPU_BRANCH(setEnvironmentMap(d, w, h));
    a.mEnvironmentMap = std::make_unique<EnvironmentMap>(std::move(d), w, h);
}

// Morph targets (Mesh::Data::targets) and one animation channel for a mesh
// record: T targets of vertex deltas [T][V][3] and optional normal deltas,
// K keyframes: times[K], weights[K][T].
static void
add_targets(Mesh::Data& d, uint32_t nverts, const float* vdeltas, const float* ndeltas, uint32_t T)
{
    d.targets.resize(T);
    for (uint32_t j = 0; j < T; ++j)
    {
        auto& tg = d.targets[j];
        tg.vertices.resize(nverts);
        for (uint32_t i = 0; i < nverts; ++i)
        {
            const float* v = vdeltas + (3ull * nverts * j) + 3ull * i;
            tg.vertices[i] = float3(v[0], v[1], v[2]);
        }
        if (ndeltas)
        {
            tg.normals.resize(nverts);
            for (uint32_t i = 0; i < nverts; ++i)
            {
                const float* v = ndeltas + (3ull * nverts * j) + 3ull * i;
                tg.normals[i] = float3(v[0], v[1], v[2]);
            }
        }
    }
}

static std::shared_ptr<Animation>
make_channel(const std::shared_ptr<Shape>& shape, const float* times, const float* weights, uint32_t K, uint32_t T)
{
    Animation::Channel ch;
    ch.shape = shape;
    for (uint32_t k = 0; k < K; ++k)
    {
        Animation::Channel::MorphKeyframe kf;
        kf.time = times[k];
        kf.weights.assign(weights + (size_t)k * T, weights + (size_t)(k + 1) * T);
        ch.morphKeyframes.push_back(std::move(kf));
    }
    std::vector<Animation::Channel> chans;
    chans.push_back(std::move(ch));
    return std::make_shared<Animation>(std::move(chans));
}

// Animation::update + Mesh::update on the reference's own Bvh accelerator:
// writes the morphed positions of a V-vertex mesh at `time`.
void
ref_morph_vertices(const float* verts, uint32_t nverts, const uint32_t* tris, uint32_t ntris, const float* vdeltas,
    uint32_t T, const float* times, const float* weights, uint32_t K, float time, float* out)
{
    std::vector<std::byte> arena(std::max<size_t>(1 << 20, (size_t)ntris * 512 + (size_t)nverts * 64));
    Bvh acc{std::span<std::byte>(arena)};
    Mesh::Data d;
    d.vertices.resize(nverts);
    for (uint32_t i = 0; i < nverts; ++i) { d.vertices[i] = float3(verts[3 * i], verts[3 * i + 1], verts[3 * i + 2]); }
    d.prims.resize(ntris);
    for (uint32_t i = 0; i < ntris; ++i) { d.prims[i] = uint3(tris[3 * i], tris[3 * i + 1], tris[3 * i + 2]); }
    add_targets(d, nverts, vdeltas, nullptr, T);
    auto mesh = std::make_shared<Mesh>(std::move(d), T);
    mesh->appendTo(&acc);
    auto anim = make_channel(mesh, times, weights, K, T);
    anim->update(&acc, time);
    const float3* vb = static_cast<const float3*>(acc.getVertexBuffer(0));
    for (uint32_t i = 0; i < nverts; ++i)
    {
        for (int k = 0; k < 3; ++k) { out[3 * i + k] = vb[i][k]; }
    }
}

// ref_render_add_mesh with T morph targets and one animation channel, which
// Alpine::updateScene (ref_render_update_scene) then applies.
int
ref_render_add_morph_mesh(const float* verts, uint32_t nverts, const uint32_t* tris, uint32_t ntris,
    const float* normals, const uint32_t* triMaterial, const float* materials, uint32_t nmat, const float* vdeltas,
    const float* ndeltas, uint32_t T, const float* times, const float* weights, uint32_t K)
{
    Mesh::Data d;
    d.vertices.resize(nverts);
    for (uint32_t i = 0; i < nverts; ++i) { d.vertices[i] = float3(verts[3 * i], verts[3 * i + 1], verts[3 * i + 2]); }
    if (normals)
    {
        d.normals.resize(nverts);
        for (uint32_t i = 0; i < nverts; ++i) { d.normals[i] = float3(normals[3 * i], normals[3 * i + 1], normals[3 * i + 2]); }
    }
    std::vector<std::shared_ptr<Material>> mats(nmat);
    for (uint32_t m = 0; m < nmat; ++m) { mats[m] = make_ref_material(materials + 5 * m); }
    d.prims.resize(ntris);
    d.materials.resize(ntris);
    for (uint32_t i = 0; i < ntris; ++i)
    {
        d.prims[i] = uint3(tris[3 * i], tris[3 * i + 1], tris[3 * i + 2]);
        uint32_t m = triMaterial[i];
        if (m >= nmat) { return 0; }
        d.materials[i] = mats[m];
    }
#ifdef ALPINE_GPU_PLUGIN
    if (sGpu)
    {
        printf("ERROR: the GPU render branch of this harness does not forward morph targets\n");
        return 0;
    }
#endif
    add_targets(d, nverts, vdeltas, normals ? ndeltas : nullptr, T);
    auto mesh = std::make_shared<Mesh>(std::move(d), T);
    auto& a = alpine::alpine();
    a.mScene.shapes.push_back(mesh);
    mesh->appendTo(a.mAccelerator.get());
    a.mScene.animations.push_back(make_channel(mesh, times, weights, K, T));
    return 1;
}

int ref_render_load_obj(const char* path) { return loadScene(path, FileType::Obj) ? 1 : 0; }

// alpine::loadScene(path, FileType::Gltf): the reference's GltfLoader.
int
ref_render_load_glb(const char* path)
{
#ifdef ALPINE_GPU_PLUGIN
    if (sGpu && !sGpu->loadGlb(path)) { return 0; }
#endif
    return loadScene(path, FileType::Gltf) ? 1 : 0;
}

// The loaded scene as the reference holds it: shape count, and one mesh's
// Mesh::Data (positions / normals / uvs / tangents: floats, may be null;
// prims: 3 per triangle) and the current (possibly morphed) vertex buffer
// the accelerator holds. Returns the vertex count and writes the triangle count.
uint32_t ref_render_shape_count() { return (uint32_t)alpine::alpine().mScene.shapes.size(); }

uint32_t
ref_render_mesh_data(uint32_t i, uint32_t* ntris, float* pos, float* nrm, float* uv, float* tan, uint32_t* prims,
    float* current)
{
    auto& a = alpine::alpine();
    auto* mesh = dynamic_cast<Mesh*>(a.mScene.shapes[i].get());
    if (!mesh) { return 0; }
    const auto& d = mesh->mData;
    *ntris = (uint32_t)d.prims.size();
    for (size_t v = 0; v < d.vertices.size(); ++v)
    {
        for (int k = 0; k < 3; ++k)
        {
            if (pos) { pos[3 * v + k] = d.vertices[v][k]; }
            if (nrm && v < d.normals.size()) { nrm[3 * v + k] = d.normals[v][k]; }
            if (current) { current[3 * v + k] = mesh->mVertexBuffer[v][k]; }
        }
        if (uv && v < d.uvs.size()) { uv[2 * v] = d.uvs[v].x; uv[2 * v + 1] = d.uvs[v].y; }
        if (tan && v < d.tangents.size()) { for (int k = 0; k < 4; ++k) { tan[4 * v + k] = d.tangents[v][k]; } }
    }
    if (prims)
    {
        for (size_t t = 0; t < d.prims.size(); ++t) { for (int k = 0; k < 3; ++k) { prims[3 * t + k] = d.prims[t][k]; } }
    }
    return (uint32_t)d.vertices.size();
}

// Light i of the loaded scene: power (getPower, RGB) and position.
void
ref_render_light_info(uint32_t i, float* power, float* position)
{
    auto& l = alpine::alpine().mScene.lights[i];
    float3 p = l->getPower();
    float3 c = l->getBoundingBox().getCenter();  // a point light's box is its position
    for (int k = 0; k < 3; ++k) { power[k] = p[k]; position[k] = c[k]; }
}
uint32_t ref_render_light_count() { return (uint32_t)alpine::alpine().mScene.lights.size(); }


void
ref_render_add_disk_light(float power, const float* color, const float* pos, const float* target, float radius)
{
    addDiskLight(power, color, pos, target, radius);
    GPU_BRANCH(addDiskLight(power, color, pos, target, radius));
}

void
ref_render_add_point_light(float power, const float* color, const float* pos)
{
    addPointLight(power, color, pos);
    GPU_BRANCH(addPointLight(power, color, pos));
}

void
ref_render_add_quad_light(const float* radiance, const float* corner, const float* eu, const float* ev)
{
    alpine::alpine().mScene.lights.push_back(std::make_shared<QuadLight>(
        float3(radiance), float3(corner), float3(eu), float3(ev)));
    GPU_BRANCH(addQuadLight(radiance, corner, eu, ev));
}
void ref_render_update_scene(float time) { updateScene(time); }

void
ref_render_build_light_sampler(int type)
{
    buildLightSampler(static_cast<LightSamplerType>(type));
    GPU_BRANCH(buildLightSampler(type));
}

void
ref_render_set_background(float r, float g, float b)
{
    setBackgroundColor(r, g, b);
    GPU_BRANCH(setBackgroundColor(r, g, b));
}

void
ref_render_set_camera(const float* eye, const float* target, const float* up, float fovy, float aspect)
{
    getCamera()->setLookAt(eye, target, up, fovy, aspect);
    GPU_BRANCH(setCamera(eye, target, up, fovy, aspect));
}

void
ref_render_reset_accumulation()
{
    resetAccumulation();
    GPU_BRANCH(resetAccumulation());
}

// Alpine::render; with the GPU render branch on, the GPU renders and its sums
// become the Alpine's accumulation (mAccumBuffer, mTotalSamples), which the
// reference's own postProcess / getFrameBuffer then read. Returns ms, or a
// negative value when the GPU branch failed.
double
ref_render(uint32_t spp)
{
    auto t0 = std::chrono::steady_clock::now();
#ifdef ALPINE_GPU_PLUGIN
    if (sGpu)
    {
        std::vector<float> sums;
        uint32_t total = 0;
        if (!sGpu->render(spp) || !sGpu->readAccumulation(sums, total)) { return -1.0; }
        auto& a = alpine::alpine();
        for (size_t i = 0; i < a.mAccumBuffer.size(); ++i)
        {
            const float* s = sums.data() + 9 * i;
            a.mAccumBuffer[i].color = float3(s[0], s[1], s[2]);
            a.mAccumBuffer[i].albedo = float3(s[3], s[4], s[5]);
            a.mAccumBuffer[i].normal = float3(s[6], s[7], s[8]);
        }
        a.mTotalSamples = total;
        auto t1 = std::chrono::steady_clock::now();
        return std::chrono::duration<double, std::milli>(t1 - t0).count();
    }
#endif
    render(spp);
    auto t1 = std::chrono::steady_clock::now();
    return std::chrono::duration<double, std::milli>(t1 - t0).count();
}

// Copies the per-pixel radiance SUMS (color, albedo, normal; 9 floats per pixel,
// denoiser::RenderTarget layout) and returns the accumulated sample count.
uint32_t
ref_render_read_accum(float* out)
{
    auto& a = alpine::alpine();
    for (size_t i = 0; i < a.mAccumBuffer.size(); ++i)
    {
        const auto& p = a.mAccumBuffer[i];
        float* o = out + 9 * i;
        o[0] = p.color.x; o[1] = p.color.y; o[2] = p.color.z;
        o[3] = p.albedo.x; o[4] = p.albedo.y; o[5] = p.albedo.z;
        o[6] = p.normal.x; o[7] = p.normal.y; o[8] = p.normal.z;
    }
    return a.mTotalSamples;
}

void
ref_render_post_process(int tonemap, uint8_t* rgb)
{
    postProcess(false, tonemap != 0);
    auto& a = alpine::alpine();
    std::memcpy(rgb, getFrameBuffer(), a.mFrameBuffer.size() * 3);
}

// Per-pixel sampler state (Sampler::mSeed, src/sampler.h), 4 words per pixel.
void
ref_render_read_sampler_state(uint32_t* out)
{
    auto& a = alpine::alpine();
    for (size_t i = 0; i < a.mSamplers.size(); ++i)
        for (int k = 0; k < 4; ++k) out[4 * i + k] = a.mSamplers[i].mSeed[k];
}

void
ref_render_shutdown()
{
#ifdef ALPINE_GPU_PLUGIN
    sGpu.reset();
#endif
    shutdown();
}

// Material::sample for n (wo, u) pairs in the local frame.
void
ref_material_sample(const float* rec, const float* wo, const float* u, uint32_t n, float* wi, float* est,
    float* pdf, uint8_t* ok)
{
    auto m = make_ref_material(rec);
    IntersectionAttributes ia{};
    for (uint32_t i = 0; i < n; ++i)
    {
        auto s = m->sample(float3(wo[3 * i], wo[3 * i + 1], wo[3 * i + 2]), float2(u[2 * i], u[2 * i + 1]), ia);
        ok[i] = s.has_value() ? 1 : 0;
        for (int k = 0; k < 3; ++k)
        {
            wi[3 * i + k] = s ? s->wi[k] : 0.0f;
            est[3 * i + k] = s ? s->estimator[k] : 0.0f;
        }
        pdf[i] = s ? s->pdf : 0.0f;
    }
}

// Material::computeBsdf / computePdf for n (wo, wi) pairs in the local frame.
void
ref_material_eval(const float* rec, const float* wo, const float* wi, uint32_t n, float* bsdf, float* pdf)
{
    auto m = make_ref_material(rec);
    IntersectionAttributes ia{};
    for (uint32_t i = 0; i < n; ++i)
    {
        float3 a(wo[3 * i], wo[3 * i + 1], wo[3 * i + 2]), b(wi[3 * i], wi[3 * i + 1], wi[3 * i + 2]);
        float3 f = m->computeBsdf(a, b, ia);
        for (int k = 0; k < 3; ++k) { bsdf[3 * i + k] = f[k]; }
        pdf[i] = m->computePdf(a, b);
    }
}
}
