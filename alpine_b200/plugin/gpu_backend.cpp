// GpuBackend (see gpu_backend.h).
#include "gpu_backend.h"

#include <cstdio>

namespace alpine {
GpuBackend::GpuBackend(uint32_t width, uint32_t height, uint32_t maxDepth, int device)
    : mWidth(width), mHeight(height)
{
    alpine_gpu_config cfg{device, width, height, maxDepth};
    if (alpine_gpu_create(&cfg, &mCtx) != ALPINE_GPU_OK)
    {
        printf("ERROR: GpuBackend: no CUDA device %d\n", device);
        mCtx = nullptr;
        mError = "no CUDA device";
    }
}

GpuBackend::~GpuBackend()
{
    if (mCtx) { alpine_gpu_destroy(mCtx); }
}

const char*
GpuBackend::lastError() const
{
    return mError.c_str();
}

bool
GpuBackend::ok(int rc, const char* what)
{
    if (rc == ALPINE_GPU_OK) { return true; }
    mError = std::string(what) + ": " + (mCtx ? alpine_gpu_last_error(mCtx) : "no context");
    printf("ERROR: GpuBackend %s\n", mError.c_str());
    return false;
}

bool
GpuBackend::resetScene(bool binaryRule)
{
    if (!mCtx) { return false; }
    mMaterials.clear();
    mTextureBindings.clear();
    mGlbMaterials = 0;
    mMaterialsDirty = true;
    mGeometryDirty = true;
    alpine_gpu_traversal_options o{
        binaryRule ? ALPINE_GPU_TRIANGLE_TEST_BINARY_BVH : ALPINE_GPU_TRIANGLE_TEST_WIDE_BVH, 0u, 0u};
    return ok(alpine_gpu_reset_scene(mCtx), "resetScene") &&
           ok(alpine_gpu_set_traversal_options(mCtx, &o), "resetScene");
}

uint32_t
GpuBackend::addMaterials(const std::vector<alpine_gpu_material>& materials)
{
    uint32_t base = (uint32_t)mMaterials.size();
    mMaterials.insert(mMaterials.end(), materials.begin(), materials.end());
    mMaterialsDirty = true;
    return base;
}

int
GpuBackend::addMesh(const std::vector<float3>& vertices, const std::vector<float3>& normals,
    const std::vector<uint3>& prims, const std::vector<uint3>& normalPrims, const std::vector<uint32_t>& materialIds)
{
    if (!mCtx) { return -1; }
    bool separateNormals = false;
    if (!normals.empty() && !normalPrims.empty())
    {
        for (size_t i = 0; i < prims.size() && !separateNormals; ++i)
        {
            for (int k = 0; k < 3; ++k) { separateNormals |= normalPrims[i][k] != prims[i][k]; }
        }
    }
    std::vector<float3> pos;
    std::vector<float3> nrm;
    std::vector<uint3> tri;
    const std::vector<float3>* P = &vertices;
    const std::vector<float3>* N = normals.empty() ? nullptr : &normals;
    const std::vector<uint3>* T = &prims;
    if (separateNormals)
    {
        // positions and normals are indexed differently: one vertex per corner
        pos.reserve(3 * prims.size());
        nrm.reserve(3 * prims.size());
        tri.reserve(prims.size());
        for (size_t i = 0; i < prims.size(); ++i)
        {
            uint32_t b = (uint32_t)pos.size();
            for (int k = 0; k < 3; ++k)
            {
                pos.push_back(vertices[prims[i][k]]);
                nrm.push_back(normals[normalPrims[i][k]]);
            }
            tri.push_back(uint3(b, b + 1, b + 2));
        }
        P = &pos;
        N = &nrm;
        T = &tri;
    }
    uint32_t id = 0;
    if (!ok(alpine_gpu_add_mesh(mCtx, P->empty() ? nullptr : &(*P)[0][0], (uint32_t)P->size(),
                T->empty() ? nullptr : &(*T)[0][0], (uint32_t)T->size(), &id),
            "addMesh"))
    {
        return -1;
    }
    if (!ok(alpine_gpu_set_triangle_attributes(mCtx, id, N ? &(*N)[0][0] : nullptr,
                materialIds.empty() ? nullptr : materialIds.data()),
            "addMesh"))
    {
        return -1;
    }
    mGeometryDirty = true;
    return (int)id;
}

bool
GpuBackend::setMeshUvs(int shape, const std::vector<float2>& uvs, const std::vector<float4>& tangents)
{
    if (!mCtx || shape < 0 || uvs.empty()) { return uvs.empty(); }
    return ok(alpine_gpu_set_triangle_uvs(mCtx, (uint32_t)shape, &uvs[0][0], tangents.empty() ? nullptr : &tangents[0][0]),
              "setMeshUvs");
}

int
GpuBackend::addTexture(const std::vector<float4>& texels, uint32_t width, uint32_t height)
{
    uint32_t id = 0;
    if (!mCtx || texels.size() != (size_t)width * height) { return -1; }
    return ok(alpine_gpu_add_texture(mCtx, &texels[0][0], width, height, &id), "addTexture") ? (int)id : -1;
}

bool
GpuBackend::setMaterialTextures(uint32_t material, int baseColorTexture, int normalTexture)
{
    // the material table reaches the context at the next render: bind then
    mTextureBindings.push_back({material, baseColorTexture, normalTexture});
    mMaterialsDirty = true;
    return true;
}

bool
GpuBackend::loadGlb(const char* path)
{
    if (!mCtx) { return false; }
    // materials added before stay in front of the file's
    if (mMaterialsDirty && !flushMaterials()) { return false; }
    alpine_gpu_glb_info info{};
    if (!ok(alpine_gpu_load_glb(mCtx, path, &info), "loadGlb")) { return false; }
    mGlbMaterials += info.materials;
    mGeometryDirty = true;
    return true;
}

bool
GpuBackend::setEnvironmentMap(const std::vector<float3>& texels, uint32_t width, uint32_t height)
{
    if (!mCtx) { return false; }
    if (texels.empty()) { return ok(alpine_gpu_set_environment_map(mCtx, nullptr, 0, 0), "setEnvironmentMap"); }
    return ok(alpine_gpu_set_environment_map(mCtx, &texels[0][0], width, height), "setEnvironmentMap");
}

bool
GpuBackend::flushMaterials()
{
    if (mGlbMaterials)
    {
        // a loaded GLB appended its own materials to the context's table; the
        // records added here come first and are set again with them
        mError = "GpuBackend: addMaterials after loadGlb is not supported";
        return false;
    }
    if (!ok(alpine_gpu_set_materials(mCtx, mMaterials.empty() ? nullptr : mMaterials.data(), (uint32_t)mMaterials.size()),
            "render"))
    {
        return false;
    }
    for (const auto& b : mTextureBindings)
    {
        if (!ok(alpine_gpu_set_material_textures(mCtx, b.material, b.base, b.normal), "setMaterialTextures"))
        {
            return false;
        }
    }
    mMaterialsDirty = false;
    return true;
}

int
GpuBackend::addPointLight(float power, const float color[3], const float position[3])
{
    uint32_t id = 0;
    return ok(alpine_gpu_add_point_light(mCtx, power, color, position, &id), "addPointLight") ? (int)id : -1;
}

int
GpuBackend::addDiskLight(float power, const float color[3], const float position[3], const float target[3], float radius)
{
    uint32_t id = 0;
    return ok(alpine_gpu_add_disk_light(mCtx, power, color, position, target, radius, &id), "addDiskLight") ? (int)id
                                                                                                             : -1;
}

int
GpuBackend::addQuadLight(const float radiance[3], const float corner[3], const float edgeU[3], const float edgeV[3])
{
    uint32_t id = 0;
    return ok(alpine_gpu_add_quad_light(mCtx, radiance, corner, edgeU, edgeV, &id), "addQuadLight") ? (int)id : -1;
}

bool GpuBackend::setLightScale(uint32_t light, float scale)
{
    return ok(alpine_gpu_set_light_scale(mCtx, light, scale), "setLightScale");
}

bool GpuBackend::buildLightSampler(int type)
{
    return ok(alpine_gpu_build_light_sampler(mCtx, type), "buildLightSampler");
}

bool GpuBackend::setBackgroundColor(float r, float g, float b)
{
    return ok(alpine_gpu_set_background(mCtx, r, g, b), "setBackgroundColor");
}

bool
GpuBackend::setCamera(const float eye[3], const float target[3], const float up[3], float fovy, float aspect)
{
    return ok(alpine_gpu_set_camera(mCtx, eye, target, up, fovy, aspect), "setCamera");
}

bool GpuBackend::setRenderOptions(const alpine_gpu_render_options& options)
{
    return ok(alpine_gpu_set_render_options(mCtx, &options), "setRenderOptions");
}

bool GpuBackend::resetAccumulation()
{
    return ok(alpine_gpu_reset_accumulation(mCtx), "resetAccumulation");
}

bool
GpuBackend::render(uint32_t spp)
{
    if (!mCtx) { return false; }
    if (mMaterialsDirty && !flushMaterials()) { return false; }
    if (mGeometryDirty)
    {
        if (!ok(alpine_gpu_build(mCtx, nullptr), "render")) { return false; }
        mGeometryDirty = false;
    }
    return ok(alpine_gpu_render(mCtx, spp), "render");
}

bool
GpuBackend::readAccumulation(std::vector<float>& sums, uint32_t& totalSamples)
{
    sums.resize((size_t)mWidth * mHeight * 9);
    return ok(alpine_gpu_read_accumulation(mCtx, sums.data(), &totalSamples), "readAccumulation");
}

bool
GpuBackend::postProcess(bool tonemap, std::vector<uint8_t>& rgb8)
{
    rgb8.resize((size_t)mWidth * mHeight * 3);
    return ok(alpine_gpu_post_process(mCtx, tonemap ? 1 : 0, nullptr, rgb8.data()), "postProcess");
}
}
