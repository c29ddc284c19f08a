// GpuAccelerator (see gpu_accelerator.h).
#include "gpu_accelerator.h"

#include <cfloat>
#include <cstdio>

namespace alpine {
namespace {
alpine_gpu_ray toGpuRay(const Ray& r, float tmax)
{
    return alpine_gpu_ray{{r.org.x, r.org.y, r.org.z}, 0.0f, {r.dir.x, r.dir.y, r.dir.z}, tmax};
}
}

GpuAccelerator::GpuAccelerator(Rule rule, int device)
{
    alpine_gpu_config cfg{device, 0, 0, 0};
    if (alpine_gpu_create(&cfg, &mCtx) != ALPINE_GPU_OK)
    {
        printf("ERROR: GpuAccelerator: no CUDA device %d\n", device);
        mCtx = nullptr;
        return;
    }
    alpine_gpu_traversal_options o{
        rule == Rule::Binary ? ALPINE_GPU_TRIANGLE_TEST_BINARY_BVH : ALPINE_GPU_TRIANGLE_TEST_WIDE_BVH, 0u, 0u};
    report(alpine_gpu_set_traversal_options(mCtx, &o), "set_traversal_options");
}

GpuAccelerator::~GpuAccelerator()
{
    if (mCtx) { alpine_gpu_destroy(mCtx); }
}

void
GpuAccelerator::report(int rc, const char* what) const
{
    if (rc != ALPINE_GPU_OK)
    {
        printf("ERROR: GpuAccelerator %s: %s\n", what, mCtx ? alpine_gpu_last_error(mCtx) : "no context");
    }
}

// Primitive::updateVertices (src/accelerators/bvh_common.cpp:105-125): the
// same float3 operations on the same vertices, so ng is bit-identical.
void
GpuAccelerator::computeNormals(Shape& s)
{
    s.ng.resize(s.prims.size());
    for (size_t i = 0; i < s.prims.size(); ++i)
    {
        const float3& v0 = s.vertices[s.prims[i][0]];
        float3 e0 = s.vertices[s.prims[i][1]] - v0;
        float3 e1 = s.vertices[s.prims[i][2]] - v0;
        s.ng[i] = normalize(cross(e0, e1));
    }
}

uint32_t
GpuAccelerator::appendMesh(const std::vector<float3>& vertices, const std::vector<uint3>& prims, const void* ptr)
{
    std::lock_guard<std::mutex> lock(mMutex);
    if (!mCtx) { return INVALID_SHAPE_ID; }
    uint32_t id = INVALID_SHAPE_ID;
    int rc = alpine_gpu_add_mesh(mCtx, vertices.empty() ? nullptr : &vertices[0][0], (uint32_t)vertices.size(),
        prims.empty() ? nullptr : &prims[0][0], (uint32_t)prims.size(), &id);
    if (rc != ALPINE_GPU_OK)
    {
        report(rc, "appendMesh");
        return INVALID_SHAPE_ID;
    }
    Shape s;
    s.ptr = ptr;
    s.triBase = mTriCount;
    s.vertices = vertices;
    s.prims = prims;
    computeNormals(s);
    mTriCount += (uint32_t)prims.size();
    mShapes.push_back(std::move(s));
    return id;
}

void
GpuAccelerator::appendSphere(const std::vector<float4>& vertices, const void* ptr)
{
    std::lock_guard<std::mutex> lock(mMutex);
    if (!mCtx || vertices.empty()) { return; }
    uint32_t first = 0;
    int rc = alpine_gpu_add_spheres(mCtx, &vertices[0][0], (uint32_t)vertices.size(), nullptr, &first);
    if (rc != ALPINE_GPU_OK)
    {
        report(rc, "appendSphere");
        return;
    }
    mSphereShapes.push_back({ptr, first, vertices});
}

void*
GpuAccelerator::getVertexBuffer(uint32_t shapeId)
{
    return shapeId < mShapes.size() ? mShapes[shapeId].vertices.data() : nullptr;
}

void
GpuAccelerator::updateShape(uint32_t shapeId)
{
    std::lock_guard<std::mutex> lock(mMutex);
    if (!mCtx || shapeId >= mShapes.size()) { return; }
    Shape& s = mShapes[shapeId];
    computeNormals(s);
    report(alpine_gpu_update_vertices(mCtx, shapeId, &s.vertices[0][0]), "updateShape");
}

void
GpuAccelerator::updateScene()
{
    std::lock_guard<std::mutex> lock(mMutex);
    if (mCtx) { report(alpine_gpu_build(mCtx, nullptr), "updateScene"); }
}

Intersection
GpuAccelerator::toIntersection(const alpine_gpu_hit& h, const Ray& ray) const
{
    if (h.prim & 0x80000000u)
    {
        const uint32_t k = h.prim & 0x7fffffffu;
        size_t s = mSphereShapes.size() - 1;
        while (s > 0 && mSphereShapes[s].first > k) { --s; }
        const SphereShape& sh = mSphereShapes[s];
        const float4& c = sh.spheres[k - sh.first];
        Intersection i;
        i.shapePtr = sh.ptr;
        i.primId = k - sh.first;
        i.ng = normalize(ray.org + ray.dir * h.t - float3(c.x, c.y, c.z));
        i.barycentric = float2(0.0f, 0.0f);
        i.t = h.t;
        return i;
    }
    // the shape holding global triangle h.prim (shapes are in triBase order)
    size_t lo = 0, hi = mShapes.size();
    while (hi - lo > 1)
    {
        size_t mid = (lo + hi) / 2;
        if (mShapes[mid].triBase <= h.prim) { lo = mid; } else { hi = mid; }
    }
    const Shape& s = mShapes[lo];
    Intersection i;
    i.shapePtr = s.ptr;
    i.primId = h.prim - s.triBase;
    i.ng = s.ng[i.primId];
    i.barycentric = float2(h.b1, h.b2);
    i.t = h.t;
    return i;
}

std::optional<Intersection>
GpuAccelerator::intersect(const Ray& ray) const
{
    std::optional<Intersection> out;
    intersectBatch(&ray, 1, &out);
    return out;
}

bool
GpuAccelerator::intersectAny(const Ray& ray, float tFar) const
{
    bool occ = false;
    intersectAnyBatch(&ray, &tFar, 1, &occ);
    return occ;
}

void
GpuAccelerator::intersectBatch(const Ray* rays, size_t n, std::optional<Intersection>* out) const
{
    std::vector<alpine_gpu_ray> q(n);
    for (size_t i = 0; i < n; ++i) { q[i] = toGpuRay(rays[i], FLT_MAX); }
    std::vector<alpine_gpu_hit> h(n);
    std::lock_guard<std::mutex> lock(mMutex);
    int rc = mCtx ? alpine_gpu_trace(mCtx, q.data(), n, h.data()) : ALPINE_GPU_ERR_INVALID_STATE;
    if (rc != ALPINE_GPU_OK)
    {
        report(rc, "intersect");
        for (size_t i = 0; i < n; ++i) { out[i].reset(); }
        return;
    }
    for (size_t i = 0; i < n; ++i)
    {
        if (h[i].prim == 0xffffffffu) { out[i].reset(); }
        else { out[i] = toIntersection(h[i], rays[i]); }
    }
}

void
GpuAccelerator::intersectAnyBatch(const Ray* rays, const float* tFar, size_t n, bool* occluded) const
{
    std::vector<alpine_gpu_ray> q(n);
    for (size_t i = 0; i < n; ++i) { q[i] = toGpuRay(rays[i], tFar[i]); }
    std::vector<uint8_t> o(n);
    std::lock_guard<std::mutex> lock(mMutex);
    int rc = mCtx ? alpine_gpu_occluded(mCtx, q.data(), n, o.data()) : ALPINE_GPU_ERR_INVALID_STATE;
    if (rc != ALPINE_GPU_OK) { report(rc, "intersectAny"); }
    for (size_t i = 0; i < n; ++i) { occluded[i] = rc == ALPINE_GPU_OK && o[i] != 0; }
}
}
