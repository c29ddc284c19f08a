// GpuAccelerator: the reference's Accelerator interface
// (src/accelerators/accelerator.h:13-39) implemented on the C ABI of the
// B200 backend (include/alpine_gpu.h). It is the class a maintainer adds next
// to Bvh / WideBvh / Embree and selects in Alpine::resetScene
// (src/alpine.cpp:158-176) with a new AcceleratorType value.
//
// Compiled against the reference's own headers (src/ on the include path).
//
// * Results: intersect() fills every Intersection field the reference's
//   accelerators fill (src/intersection.h:8-16): shapePtr and the mesh-local
//   primId, t and the barycentrics from the GPU, and ng =
//   normalize(cross(v1 - v0, v2 - v0)) of the hit triangle computed on the
//   host from the current vertex buffer exactly as Primitive::updateVertices
//   does (src/accelerators/bvh_common.cpp:105-125). The hit rule is the
//   reference's 8-wide BVH (WideRule) or its binary BVH (BinaryRule).
// * Threads: Alpine::render calls intersect / intersectAny from one
//   std::async task per 16x16 tile at once (src/alpine.cpp:276-285, 316).
//   One backend context is not re-entrant, so every query takes a mutex;
//   the per-ray path is correct but slow (one round trip per ray). Callers
//   that can batch use intersectBatch / intersectAnyBatch, and the whole
//   integrator runs on the GPU through GpuBackend (gpu_backend.h).
// * Spheres: appendSphere adds analytic spheres (Sphere::Data vertices:
//   centre + radius) to the same BVH, as the reference's Embree accelerator
//   does (src/accelerators/embree.cpp:107-122; its Bvh and WideBvh print an
//   error instead). A sphere hit reports the sphere's index in its shape as
//   primId and ng = normalize(hit - centre), as Embree's normalised Ng.
#pragma once

#include <accelerators/accelerator.h>
#include <intersection.h>
#include <ray.h>

#include <alpine_gpu.h>

#include <mutex>
#include <optional>
#include <vector>

namespace alpine {
class GpuAccelerator final : public Accelerator
{
public:
    enum class Rule { Wide, Binary };

    explicit GpuAccelerator(Rule rule = Rule::Wide, int device = 0);
    ~GpuAccelerator() override;

    GpuAccelerator(const GpuAccelerator&) = delete;
    GpuAccelerator& operator=(const GpuAccelerator&) = delete;

    bool valid() const { return mCtx != nullptr; }

    uint32_t appendMesh(
        const std::vector<float3>& vertices, const std::vector<uint3>& prims, const void* ptr) override;

    void appendSphere(const std::vector<float4>& vertices, const void* ptr) override;

    void* getVertexBuffer(uint32_t shapeId) override;

    void updateShape(uint32_t shapeId) override;

    void updateScene() override;

    std::optional<Intersection> intersect(const Ray& ray) const override;

    bool intersectAny(const Ray& ray, float tFar) const override;

    // Batched queries (one GPU round trip for n rays); thread-safe.
    void intersectBatch(const Ray* rays, size_t n, std::optional<Intersection>* out) const;
    void intersectAnyBatch(const Ray* rays, const float* tFar, size_t n, bool* occluded) const;

private:
    struct Shape
    {
        const void* ptr = nullptr;
        uint32_t triBase = 0;                 // global index of the shape's first triangle
        std::vector<float3> vertices;         // the buffer Mesh::update writes (getVertexBuffer)
        std::vector<uint3> prims;
        std::vector<float3> ng;               // per triangle, as Primitive::ng
    };

    struct SphereShape
    {
        const void* ptr = nullptr;
        uint32_t first = 0;                   // global index of the shape's first sphere
        std::vector<float4> spheres;
    };

    static void computeNormals(Shape& s);
    Intersection toIntersection(const alpine_gpu_hit& h, const Ray& ray) const;
    void report(int rc, const char* what) const;

    alpine_gpu_ctx* mCtx = nullptr;
    std::vector<Shape> mShapes;
    std::vector<SphereShape> mSphereShapes;
    uint32_t mTriCount = 0;
    mutable std::mutex mMutex;
};
}
