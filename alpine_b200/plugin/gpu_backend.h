// GpuBackend: the render branch of the reference's Alpine class
// (src/alpine.cpp:44-126) on the C ABI of the B200 backend. A maintainer
// holds one GpuBackend in Alpine and, when the GPU is selected, forwards each
// Alpine method that owns render state to it; every other choice keeps the
// reference code unchanged:
//
//   Alpine::initialize(.., w, h, maxDepth)   -> GpuBackend(w, h, maxDepth)
//   Alpine::resetScene                       -> resetScene
//   Alpine::loadScene (per Mesh::Data)       -> addMesh (positions, normals,
//                                               material ids) + materials
//   Alpine::loadScene (FileType::Gltf)       -> loadGlb (the whole file)
//   Alpine::loadEnvironmentMap               -> setEnvironmentMap
//   Alpine::addPointLight / addDiskLight     -> addPointLight / addDiskLight
//   LightHandle::setScale                    -> setLightScale
//   Alpine::buildLightSampler                -> buildLightSampler
//   Alpine::setBackgroundColor               -> setBackgroundColor
//   CameraHandle::setLookAt                  -> setCamera
//   Alpine::resetAccumulation                -> resetAccumulation
//   Alpine::render(spp)                      -> render(spp), then
//                                               readAccumulation into mAccumBuffer
//
// Alpine::postProcess and getFrameBuffer then run unchanged on the
// accumulation (or postProcess forwards to alpine_gpu_post_process).
// The whole integrator (camera rays, traversal, BSDF and light sampling, MIS,
// accumulation) runs on the GPU; see alpine_gpu.h for the options.
#pragma once

#include <math/vector.h>

#include <alpine_gpu.h>

#include <cstdint>
#include <string>
#include <vector>

namespace alpine {
class GpuBackend
{
public:
    GpuBackend(uint32_t width, uint32_t height, uint32_t maxDepth, int device = 0);
    ~GpuBackend();

    GpuBackend(const GpuBackend&) = delete;
    GpuBackend& operator=(const GpuBackend&) = delete;

    bool valid() const { return mCtx != nullptr; }
    alpine_gpu_ctx* context() { return mCtx; }
    const char* lastError() const;

    // binaryRule: the reference binary BVH's triangle rule (AcceleratorType::Bvh)
    bool resetScene(bool binaryRule);

    // One mesh of Mesh::Data (src/shapes/mesh.h:16-36): positions and prims;
    // per-vertex normals (empty: the geometric normal shades) indexed by
    // normalPrims (empty: by prims); per-triangle material ids into the
    // records given to addMaterials. Returns the shape id or -1.
    int addMesh(const std::vector<float3>& vertices, const std::vector<float3>& normals,
        const std::vector<uint3>& prims, const std::vector<uint3>& normalPrims,
        const std::vector<uint32_t>& materialIds);

    // Texture coordinates and tangents of a mesh added by addMesh, per vertex
    // (Mesh::Data uvs / tangents); either may be empty.
    bool setMeshUvs(int shape, const std::vector<float2>& uvs, const std::vector<float4>& tangents);

    // A texture (the loader's Texture4f data); returns its id or -1.
    int addTexture(const std::vector<float4>& texels, uint32_t width, uint32_t height);
    // Binds textures (-1 = none) to a material appended by addMaterials.
    bool setMaterialTextures(uint32_t material, int baseColorTexture, int normalTexture);

    // A whole binary glTF file (alpine_gpu_load_glb); false on failure.
    bool loadGlb(const char* path);

    // The lat-long environment map (width x height RGB texels); empty removes it.
    bool setEnvironmentMap(const std::vector<float3>& texels, uint32_t width, uint32_t height);

    // Appends material records (the loaders' Dielectric / Conductor with
    // alpha = roughness); returns the index of the first one.
    uint32_t addMaterials(const std::vector<alpine_gpu_material>& materials);

    int addPointLight(float power, const float color[3], const float position[3]);
    int addDiskLight(float power, const float color[3], const float position[3], const float target[3], float radius);
    int addQuadLight(const float radiance[3], const float corner[3], const float edgeU[3], const float edgeV[3]);
    bool setLightScale(uint32_t light, float scale);
    bool buildLightSampler(int type);
    bool setBackgroundColor(float r, float g, float b);
    bool setCamera(const float eye[3], const float target[3], const float up[3], float fovy, float aspect);
    bool setRenderOptions(const alpine_gpu_render_options& options);

    bool resetAccumulation();
    // Builds the BVH and uploads the scene when needed, then renders spp
    // samples per pixel (synchronous, like Alpine::render).
    bool render(uint32_t spp);
    // The per-pixel sums (9 floats per pixel: colour, albedo, normal, the
    // RenderTarget layout of src/denoisers/denoiser.h:7-12).
    bool readAccumulation(std::vector<float>& sums, uint32_t& totalSamples);
    bool postProcess(bool tonemap, std::vector<uint8_t>& rgb8);

private:
    bool ok(int rc, const char* what);
    bool flushMaterials();

    struct TextureBinding
    {
        uint32_t material;
        int base, normal;
    };
    std::vector<TextureBinding> mTextureBindings;
    uint32_t mGlbMaterials = 0;

    alpine_gpu_ctx* mCtx = nullptr;
    uint32_t mWidth = 0, mHeight = 0;
    std::vector<alpine_gpu_material> mMaterials;
    bool mMaterialsDirty = false;
    bool mGeometryDirty = true;
    std::string mError;
};
}
