// The context behind the C ABI: device memory, streams, scene state.
#pragma once

#include "../../include/alpine_gpu.h"
#include "build.cuh"
#include "guide_host.cuh"
#include "shading.cuh"

#include <memory>
#include <string>
#include <vector>

namespace ag {

// A growable device buffer.
struct DeviceBuffer {
    void* ptr = nullptr;
    size_t bytes = 0;
    ~DeviceBuffer() { release(); }
    void release()
    {
        if (ptr) cudaFree(ptr);
        ptr = nullptr;
        bytes = 0;
    }
    // Returns false when the allocation fails. Contents are not preserved.
    bool reserve(size_t n)
    {
        if (n <= bytes && ptr) return true;
        release();
        size_t want = n < 256 ? 256 : n;
        if (cudaMalloc(&ptr, want) != cudaSuccess) {
            cudaGetLastError();
            ptr = nullptr;
            return false;
        }
        bytes = want;
        return true;
    }
    template <typename T>
    T* as() const { return static_cast<T*>(ptr); }
};

constexpr int kCopyStreams = 8;  // host-query pipeline streams: copies in, 6 traversal streams, copies out
constexpr int kPipeChunks = 32;  // host-query pipeline: at most this many chunks per call

// Human-readable description of DeviceError bits.
inline std::string status_msg(uint32_t bits)
{
    std::string m = "device-side limit:";
    if (bits & kErrStackOverflow) m += " traversal stack overflow;";
    if (bits & kErrBadIndex) m += " node/triangle index out of range;";
    if (bits & kErrIterations) m += " traversal visit cap reached;";
    if (bits & kErrBuildDepth) m += " BVH build level cap reached;";
    if (bits & kErrQueueOverflow) m += " wavefront queue overflow;";
    if (bits & kErrTensorWait) m += " tensor-core completion wait timed out;";
    return m;
}

int upload_render_scene(alpine_gpu_ctx* c);  // render.cu: materials, attributes, lights to the device
int add_point_light_intensity(alpine_gpu_ctx* c, float3 intensity, float3 position, uint32_t* id);  // render.cu
int upload_geometry(alpine_gpu_ctx* c);      // api.cu: vertices and indices to the device

// A material record of the C ABI as the device Material: Dielectric or
// Conductor with alpha = roughness (gltf_loader.cpp:404-414), alpha clamped
// to 0.001 (microfacet.h:9-12); a Dielectric adds the microfacet lobe when
// dot(alpha, alpha) < 1 (dielectric.cpp:15-27). False for an unknown kind.
inline bool make_material(const alpine_gpu_material& in, Material& x)
{
    if (in.kind != ALPINE_GPU_MATERIAL_DIELECTRIC && in.kind != ALPINE_GPU_MATERIAL_CONDUCTOR) return false;
    x = Material{};
    x.kind = in.kind == ALPINE_GPU_MATERIAL_CONDUCTOR ? kMatConductor : kMatDielectric;
    x.r = in.base_color[0];
    x.g = in.base_color[1];
    x.b = in.base_color[2];
    const float a = in.roughness;
    x.ax = a > 0.001f ? a : 0.001f;
    x.ay = x.ax;
    x.lobes = (a * a + a * a < 1.0f) ? 2u : 1u;
    x.baseTex = 0u;
    x.normalTex = 0u;
    return true;
}

}  // namespace ag

struct alpine_gpu_ctx {
    int device = 0;
    alpine_gpu_config cfg{};
    cudaStream_t stream = nullptr;
    cudaStream_t copyStreams[ag::kCopyStreams] = {};
    cudaEvent_t pipeIn[ag::kPipeChunks] = {};    // host-query pipeline: chunk k's rays have landed
    cudaEvent_t pipeDone[ag::kPipeChunks] = {};  // chunk k's traversal is done
    cudaEvent_t pipeStart = nullptr;             // the context stream's work before a query
    std::string error;

    // scene geometry (host mirror + device copy)
    std::vector<float> verts;       // 3 per vertex, all meshes
    std::vector<uint32_t> idx;      // 3 per triangle, global vertex indices
    std::vector<uint32_t> shapeVertBase, shapeVertCount, shapeTriBase, shapeTriCount;
    bool geometryDirty = true;      // device vertex/index copy out of date
    bool bvhDirty = true;           // BVH out of date w.r.t. geometry
    ag::DeviceBuffer dVerts, dIdx;
    // analytic spheres (Sphere::Data: centre + radius, material per sphere)
    std::vector<float4> spheres;
    std::vector<uint32_t> sphereMaterial;
    ag::DeviceBuffer dSpheres, dSphereMaterial;

    // acceleration structure
    ag::Builder builder;
    ag::DeviceBuffer dNodes, dTris;
    uint32_t nodeCount = 0, triCount = 0;
    alpine_gpu_bvh_stats stats{};
    uint32_t syncBuildPrims = 0;  // primitives of the last alpine_gpu_build (buffers for alpine_gpu_build_async)

    // device status word (DeviceError bits) and its pinned host mirror
    // (16 words: [0] status, [1..] small read-backs)
    uint32_t* dStatus = nullptr;
    uint32_t* hStatus = nullptr;

    // staging for host-memory queries
    ag::DeviceBuffer dRays, dOut;

    // rendering: per-triangle material/normal flags and per-vertex normals
    std::vector<uint32_t> triInfo;  // material id | kTriHasNormals | kTriMorphedNormals
    std::vector<float> normals;     // 3 per vertex (zero for meshes without normals)
    std::vector<float> uvs;         // 2 per vertex (zero for meshes without texture coordinates)
    std::vector<float> tangents;    // 4 per vertex: xyz and the bitangent sign
    bool attribsDirty = true;
    ag::DeviceBuffer dTriInfo, dNormals, dUvs, dTangents;
    // textures (the loaders' Texture4f) and the environment map
    std::vector<ag::TextureInfo> textures;
    std::vector<float4> texels;
    bool texturesDirty = false;
    ag::DeviceBuffer dTextures, dTexels;
    std::vector<float> env;         // lat-long, 3 floats per texel, row-major
    uint32_t envW = 0, envH = 0;
    bool envDirty = false;
    ag::DeviceBuffer dEnv;
    std::vector<ag::Material> materials;
    bool materialsDirty = true;
    ag::DeviceBuffer dMaterials;
    uint32_t materialCount = 0;
    // lights and the light sampler
    std::vector<ag::Light> lights;
    bool lightsDirty = true;
    ag::DeviceBuffer dLights, dAlias, dLightNodes, dLightPairs;
    uint32_t samplerKind = ag::kSamplerNone;
    uint32_t samplerLightCount = 0;
    uint32_t lightNodeCount = 0;
    // camera, background, options, accumulation
    float3 background = make_float3(0.0f, 0.0f, 0.0f);
    ag::Camera camera{};
    bool cameraSet = false;
    alpine_gpu_render_options options{ALPINE_GPU_SAMPLER_COUNTER, 0u, 0u, 0u, 0u};
    bool accumValid = false;
    ag::DeviceBuffer dAccum, dPixelRng;
    size_t accumBytes = 0;
    uint32_t totalSamples = 0;
    ag::DeviceBuffer dWave;
    uint32_t waveCapacity = 0;
    int traceBlock = 128;             // k_trace_dyn block size (autotuned)
    // CUDA-graph replay of the render loop: the captured graph and the launch
    // configuration it was captured for
    cudaGraphExec_t graphExec = nullptr;
    std::vector<unsigned char> graphKey;
    uint32_t graphLaunches = 0, graphCaptures = 0;
    uint32_t* dSampleBase = nullptr;  // first sample index of a replayed render

    // traversal options (triangle rule, device-side limits)
    alpine_gpu_traversal_options traversal{};

    // morph-target animation (Mesh::Data::targets, src/shapes/mesh.h:27-33;
    // Animation channels, src/animation.h). The morphed positions and normals
    // are written on the device; the host mirrors are refreshed on demand.
    struct Morph {
        uint32_t shape = 0, targets = 0;
        bool normals = false;
        ag::DeviceBuffer dBase, dDeltas;      // positions [V][3], deltas [T][V][3]
        ag::DeviceBuffer dBaseN, dDeltasN;    // the same for the vertex normals
        std::vector<float> weights;           // Mesh::mWeights
    };
    struct Channel {
        uint32_t morph = 0;
        std::vector<float> times;             // keyframe times
        std::vector<float> weights;           // [keyframes][targets]
    };
    std::vector<std::unique_ptr<Morph>> morphs;
    std::vector<Channel> channels;
    bool hostVertsStale = false, hostNormalsStale = false;

    // learned path guiding
    ag::guide::Guide guide;
    uint32_t guideSeed = 1;
    bool guideBoxSet = false;
    ag::DeviceBuffer dGuideWave;     // queries, mixture parameters, training records
    uint32_t guideWavePaths = 0, guideTrainCap = 0;
    uint32_t guideWaveIndex = 0;     // waves rendered with guiding (record selection hash)
    uint32_t guideLastLossSteps = 0;  // Adam steps behind the loss sum in hStatus[2]

    // Reads and clears the device status word (stream must be idle).
    int check_device_status()
    {
        cudaError_t e = cudaMemcpyAsync(hStatus, dStatus, sizeof(uint32_t), cudaMemcpyDeviceToHost, stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
        if (e != cudaSuccess) return fail(ALPINE_GPU_ERR_CUDA, std::string("status readback: ") + cudaGetErrorString(e));
        if (*hStatus) {
            uint32_t bits = *hStatus;
            cudaMemsetAsync(dStatus, 0, sizeof(uint32_t), stream);
            cudaStreamSynchronize(stream);
            return fail(ALPINE_GPU_ERR_LIMIT, ag::status_msg(bits));
        }
        return ALPINE_GPU_OK;
    }

    // The BVH as the traversal kernels see it, with this context's options.
    // nodeCount / triCount are the built counts (the render passes its
    // allocation sizes instead, see render.cu).
    ag::BvhView bvh_view() const
    {
        ag::BvhView v;
        v.nodes = dNodes.as<ag::WideNode>();
        v.tris = dTris.as<ag::TriRecord>();
        v.nodeCount = nodeCount;
        v.triCount = triCount;
        v.triTest = traversal.triangle_test;
        v.maxVisits = traversal.max_visits ? traversal.max_visits : ag::kMaxVisits;
        v.stackLimit = traversal.stack_limit ? traversal.stack_limit : (uint32_t)ag::kTraversalStack;
        return v;
    }

    // Copies device-side morph results into the host mirrors (before a host
    // edit of the geometry or attributes would otherwise upload stale data).
    int pull_host_geometry()
    {
        if (!hostVertsStale && !hostNormalsStale) return ALPINE_GPU_OK;
        cudaError_t e = cudaSuccess;
        if (hostVertsStale && !verts.empty())
            e = cudaMemcpyAsync(verts.data(), dVerts.ptr, verts.size() * sizeof(float), cudaMemcpyDeviceToHost, stream);
        if (e == cudaSuccess && hostNormalsStale && !normals.empty())
            e = cudaMemcpyAsync(normals.data(), dNormals.ptr, normals.size() * sizeof(float), cudaMemcpyDeviceToHost,
                                stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
        if (e != cudaSuccess) return fail(ALPINE_GPU_ERR_CUDA, std::string("geometry read-back: ") + cudaGetErrorString(e));
        hostVertsStale = hostNormalsStale = false;
        return ALPINE_GPU_OK;
    }

    int fail(int code, const std::string& msg)
    {
        error = msg;
        return code;
    }
};
