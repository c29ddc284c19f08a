// C ABI entry points (include/alpine_gpu.h).
#include "context.cuh"
#include "trace.cuh"

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <new>

using ag::DeviceBuffer;

namespace {

const char* kNoError = "";

std::string cuda_msg(const char* what, cudaError_t e)
{
    return std::string(what) + ": " + cudaGetErrorString(e);
}

// Reads and clears the device status word (stream must be idle).
int check_status(alpine_gpu_ctx* c)
{
    cudaError_t e = cudaMemcpyAsync(c->hStatus, c->dStatus, sizeof(uint32_t), cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) return c->fail(ALPINE_GPU_ERR_CUDA, cuda_msg("status readback", e));
    if (*c->hStatus) {
        uint32_t bits = *c->hStatus;
        cudaMemsetAsync(c->dStatus, 0, sizeof(uint32_t), c->stream);
        cudaStreamSynchronize(c->stream);
        return c->fail(ALPINE_GPU_ERR_LIMIT, ag::status_msg(bits));
    }
    return ALPINE_GPU_OK;
}

int upload_geometry_now(alpine_gpu_ctx* c)
{
    if (!c->geometryDirty) return ALPINE_GPU_OK;
    size_t vb = c->verts.size() * sizeof(float), ib = c->idx.size() * sizeof(uint32_t);
    if (!c->dVerts.reserve(vb) || !c->dIdx.reserve(ib))
        return c->fail(ALPINE_GPU_ERR_OUT_OF_MEMORY, "geometry upload: cudaMalloc failed");
    cudaError_t e = cudaSuccess;
    if (vb) e = cudaMemcpyAsync(c->dVerts.ptr, c->verts.data(), vb, cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess && ib) e = cudaMemcpyAsync(c->dIdx.ptr, c->idx.data(), ib, cudaMemcpyHostToDevice, c->stream);
    const size_t sb = c->spheres.size() * sizeof(float4), mb = c->sphereMaterial.size() * sizeof(uint32_t);
    if (!c->dSpheres.reserve(sb) || !c->dSphereMaterial.reserve(mb))
        return c->fail(ALPINE_GPU_ERR_OUT_OF_MEMORY, "sphere upload: cudaMalloc failed");
    if (e == cudaSuccess && sb) e = cudaMemcpyAsync(c->dSpheres.ptr, c->spheres.data(), sb, cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess && mb)
        e = cudaMemcpyAsync(c->dSphereMaterial.ptr, c->sphereMaterial.data(), mb, cudaMemcpyHostToDevice, c->stream);
    if (e != cudaSuccess) return c->fail(ALPINE_GPU_ERR_CUDA, cuda_msg("geometry upload", e));
    c->geometryDirty = false;
    return ALPINE_GPU_OK;
}

ag::BvhView view(const alpine_gpu_ctx* c) { return c->bvh_view(); }

int require_bvh(alpine_gpu_ctx* c)
{
    if (c->bvhDirty) return c->fail(ALPINE_GPU_ERR_INVALID_STATE, "geometry changed since the last alpine_gpu_build");
    return ALPINE_GPU_OK;
}

bool is_pinned(const void* p)
{
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeHost;
}

// Host-memory query: pinned buffers go through a chunked three-stage
// pipeline; pageable buffers are staged whole. The rays of all chunks are
// copied in back to back on one stream, so the host link never waits for a
// traversal; chunk k's traversal runs on one of six streams once its
// copy has landed (an event), so the traversals of neighbouring chunks
// overlap each other's tails; its results are copied out on the last stream
// once it is done. Everything waits for the work already enqueued on the
// context stream (an asynchronous rebuild, for instance). Up to 32 chunks of
// at least 65,536 rays, issued in bit-reversed order (0, 16, 8, 24, ... of
// 32): the cost of rays often varies along a batch (primary rays first,
// incoherent secondaries after), and spreading the chunks lets the
// expensive ones' traversals overlap the copies of the others. Measured on
// the 4M-ray workload, whose second half costs almost all the any-hit time:
// in batch order the any-hit call waited for its last copies before most of
// its work could start.
template <bool kAny>
int host_query(alpine_gpu_ctx* c, const alpine_gpu_ray* rays, uint64_t n, void* out)
{
    if (!c || (n && (!rays || !out))) return c ? c->fail(ALPINE_GPU_ERR_INVALID_ARGUMENT, "null buffer") : -1;
    if (int rc = require_bvh(c)) return rc;
    if (n == 0) return ALPINE_GPU_OK;
    const size_t outSize = kAny ? 1 : sizeof(alpine_gpu_hit);
    if (!c->dRays.reserve(n * sizeof(alpine_gpu_ray)) || !c->dOut.reserve(n * outSize))
        return c->fail(ALPINE_GPU_ERR_OUT_OF_MEMORY, "ray staging: cudaMalloc failed");
    ag::BvhView v = view(c);
    cudaError_t e = cudaSuccess;
    if (is_pinned(rays) && is_pinned(out)) {
        const uint64_t kMinChunk = 1ull << 16;
        uint64_t chunk = (n + ag::kPipeChunks - 1) / ag::kPipeChunks;
        if (chunk < kMinChunk) chunk = kMinChunk;
        cudaStream_t in = c->copyStreams[0], back = c->copyStreams[ag::kCopyStreams - 1];
        e = cudaEventRecord(c->pipeStart, c->stream);
        for (int i = 0; i < ag::kCopyStreams && e == cudaSuccess; ++i)
            e = cudaStreamWaitEvent(c->copyStreams[i], c->pipeStart, 0);
        const uint32_t chunks = (uint32_t)((n + chunk - 1) / chunk);
        uint32_t bits = 0;
        while ((1u << bits) < chunks) ++bits;
        int k = 0;  // issue position
        for (uint32_t j = 0; j < (1u << bits) && e == cudaSuccess; ++j) {
            uint32_t r = 0;  // chunk index: j with its low `bits` bits reversed
            for (uint32_t b = 0; b < bits; ++b) r |= ((j >> b) & 1u) << (bits - 1 - b);
            if (r >= chunks) continue;
            const uint64_t s = uint64_t(r) * chunk;
            const uint64_t m = n - s < chunk ? n - s : chunk;
            cudaStream_t st = c->copyStreams[1 + k % (ag::kCopyStreams - 2)];
            const char* src = reinterpret_cast<const char*>(rays) + s * sizeof(alpine_gpu_ray);
            char* dr = c->dRays.as<char>() + s * sizeof(alpine_gpu_ray);
            char* dout = c->dOut.as<char>() + s * outSize;
            e = cudaMemcpyAsync(dr, src, m * sizeof(alpine_gpu_ray), cudaMemcpyHostToDevice, in);
            if (e == cudaSuccess) e = cudaEventRecord(c->pipeIn[k], in);
            if (e == cudaSuccess) e = cudaStreamWaitEvent(st, c->pipeIn[k], 0);
            if (e != cudaSuccess) break;
            if (kAny) ag::launch_occluded(v, dr, m, reinterpret_cast<uint8_t*>(dout), c->dStatus, st);
            else ag::launch_trace(v, dr, m, dout, c->dStatus, st);
            e = cudaEventRecord(c->pipeDone[k], st);
            if (e == cudaSuccess) e = cudaStreamWaitEvent(back, c->pipeDone[k], 0);
            if (e == cudaSuccess)
                e = cudaMemcpyAsync(static_cast<char*>(out) + s * outSize, dout, m * outSize, cudaMemcpyDeviceToHost,
                                    back);
            ++k;
        }
        for (int i = 0; i < ag::kCopyStreams; ++i) {
            cudaError_t e2 = cudaStreamSynchronize(c->copyStreams[i]);
            if (e == cudaSuccess) e = e2;
        }
    } else {
        e = cudaMemcpyAsync(c->dRays.ptr, rays, n * sizeof(alpine_gpu_ray), cudaMemcpyHostToDevice, c->stream);
        if (e == cudaSuccess) {
            if (kAny) ag::launch_occluded(v, c->dRays.ptr, n, c->dOut.as<uint8_t>(), c->dStatus, c->stream);
            else ag::launch_trace(v, c->dRays.ptr, n, c->dOut.ptr, c->dStatus, c->stream);
            e = cudaGetLastError();
        }
        if (e == cudaSuccess) e = cudaMemcpyAsync(out, c->dOut.ptr, n * outSize, cudaMemcpyDeviceToHost, c->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    }
    if (e == cudaSuccess) e = cudaGetLastError();
    if (e != cudaSuccess) return c->fail(ALPINE_GPU_ERR_CUDA, cuda_msg(kAny ? "occluded" : "trace", e));
    return check_status(c);
}

template <bool kAny>
int device_query(alpine_gpu_ctx* c, const alpine_gpu_ray* rays, uint64_t n, void* out, void* stream)
{
    if (!c || (n && (!rays || !out))) return c ? c->fail(ALPINE_GPU_ERR_INVALID_ARGUMENT, "null buffer") : -1;
    if (int rc = require_bvh(c)) return rc;
    if (n == 0) return ALPINE_GPU_OK;
    cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : c->stream;
    ag::BvhView v = view(c);
    if (kAny) ag::launch_occluded(v, rays, n, static_cast<uint8_t*>(out), c->dStatus, st);
    else ag::launch_trace(v, rays, n, out, c->dStatus, st);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return c->fail(ALPINE_GPU_ERR_CUDA, cuda_msg("launch", e));
    return ALPINE_GPU_OK;
}

}  // namespace

extern "C" {

int alpine_gpu_create(const alpine_gpu_config* cfg, alpine_gpu_ctx** out)
{
    if (!cfg || !out) return ALPINE_GPU_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || cfg->device < 0 || cfg->device >= n) {
        cudaGetLastError();
        return ALPINE_GPU_ERR_CUDA;
    }
    auto* c = new (std::nothrow) alpine_gpu_ctx;
    if (!c) return ALPINE_GPU_ERR_OUT_OF_MEMORY;
    c->cfg = *cfg;
    c->device = cfg->device;
    cudaError_t e = cudaSetDevice(c->device);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
    for (int i = 0; i < ag::kCopyStreams && e == cudaSuccess; ++i)
        e = cudaStreamCreateWithFlags(&c->copyStreams[i], cudaStreamNonBlocking);
    for (int i = 0; i < ag::kPipeChunks && e == cudaSuccess; ++i) {
        e = cudaEventCreateWithFlags(&c->pipeIn[i], cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&c->pipeDone[i], cudaEventDisableTiming);
    }
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&c->pipeStart, cudaEventDisableTiming);
    // 16 device words: [0] status bits, [4] the sample base of a replayed render
    if (e == cudaSuccess) e = cudaMalloc(&c->dStatus, 16 * sizeof(uint32_t));
    if (e == cudaSuccess) e = cudaMallocHost(&c->hStatus, 16 * sizeof(uint32_t));
    if (e == cudaSuccess) e = cudaMemset(c->dStatus, 0, 16 * sizeof(uint32_t));
    if (e == cudaSuccess) c->dSampleBase = c->dStatus + 4;
    if (e != cudaSuccess) {
        cudaGetLastError();
        alpine_gpu_destroy(c);
        return ALPINE_GPU_ERR_CUDA;
    }
    *out = c;
    return ALPINE_GPU_OK;
}

void alpine_gpu_destroy(alpine_gpu_ctx* c)
{
    if (!c) return;
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    for (auto& s : c->copyStreams)
        if (s) { cudaStreamSynchronize(s); cudaStreamDestroy(s); }
    for (int i = 0; i < ag::kPipeChunks; ++i) {
        if (c->pipeIn[i]) cudaEventDestroy(c->pipeIn[i]);
        if (c->pipeDone[i]) cudaEventDestroy(c->pipeDone[i]);
    }
    if (c->pipeStart) cudaEventDestroy(c->pipeStart);
    if (c->graphExec) cudaGraphExecDestroy(c->graphExec);
    if (c->stream) cudaStreamDestroy(c->stream);
    if (c->dStatus) cudaFree(c->dStatus);
    if (c->hStatus) cudaFreeHost(c->hStatus);
    delete c;
}

const char* alpine_gpu_last_error(const alpine_gpu_ctx* c) { return c ? c->error.c_str() : kNoError; }

int alpine_gpu_reset_scene(alpine_gpu_ctx* c)
{
    if (!c) return ALPINE_GPU_ERR_INVALID_ARGUMENT;
    c->verts.clear();
    c->idx.clear();
    c->spheres.clear();
    c->sphereMaterial.clear();
    c->morphs.clear();
    c->channels.clear();
    c->hostVertsStale = c->hostNormalsStale = false;
    c->shapeVertBase.clear();
    c->shapeVertCount.clear();
    c->shapeTriBase.clear();
    c->shapeTriCount.clear();
    c->geometryDirty = true;
    c->bvhDirty = true;
    c->nodeCount = 0;
    c->triCount = 0;
    // Scene::reset also drops the lights (src/scenes/scene.h:21-26)
    c->triInfo.clear();
    c->normals.clear();
    c->uvs.clear();
    c->tangents.clear();
    c->attribsDirty = true;
    c->lights.clear();
    c->lightsDirty = true;
    c->samplerKind = ag::kSamplerNone;
    c->samplerLightCount = 0;
    return ALPINE_GPU_OK;
}

int alpine_gpu_add_mesh(alpine_gpu_ctx* c, const float* vertices, uint32_t vcount, const uint32_t* indices,
                        uint32_t tcount, uint32_t* shape_id)
{
    if (!c) return ALPINE_GPU_ERR_INVALID_ARGUMENT;
    if ((vcount && !vertices) || (tcount && !indices))
        return c->fail(ALPINE_GPU_ERR_INVALID_ARGUMENT, "add_mesh: null array");
    uint64_t totalTris = c->idx.size() / 3 + (uint64_t)tcount;
    uint64_t totalVerts = c->verts.size() / 3 + (uint64_t)vcount;
    if (totalTris >= 0x7fffffffull || totalVerts >= 0x7fffffffull)
        return c->fail(ALPINE_GPU_ERR_LIMIT, "add_mesh: more than 2^31 - 1 triangles or vertices");
    for (uint64_t i = 0; i < 3ull * tcount; ++i)
        if (indices[i] >= vcount) return c->fail(ALPINE_GPU_ERR_INVALID_ARGUMENT, "add_mesh: vertex index out of range");
    if (int rc = c->pull_host_geometry()) return rc;
    uint32_t vbase = (uint32_t)(c->verts.size() / 3);
    c->shapeVertBase.push_back(vbase);
    c->shapeVertCount.push_back(vcount);
    c->shapeTriBase.push_back((uint32_t)(c->idx.size() / 3));
    c->shapeTriCount.push_back(tcount);
    c->verts.insert(c->verts.end(), vertices, vertices + 3ull * vcount);
    c->idx.reserve(c->idx.size() + 3ull * tcount);
    for (uint64_t i = 0; i < 3ull * tcount; ++i) c->idx.push_back(indices[i] + vbase);
    c->geometryDirty = true;
    c->bvhDirty = true;
    if (shape_id) *shape_id = (uint32_t)(c->shapeVertBase.size() - 1);
    return ALPINE_GPU_OK;
}

int alpine_gpu_add_spheres(alpine_gpu_ctx* c, const float* spheres, uint32_t count, const uint32_t* material,
                           uint32_t* first_sphere)
{
    if (!c) return ALPINE_GPU_ERR_INVALID_ARGUMENT;
    if (count && !spheres) return c->fail(ALPINE_GPU_ERR_INVALID_ARGUMENT, "add_spheres: null array");
    if (c->spheres.size() + count >= (size_t)ag::kSpherePrim)
        return c->fail(ALPINE_GPU_ERR_LIMIT, "add_spheres: more than 2^31 - 1 spheres");
    if (first_sphere) *first_sphere = (uint32_t)c->spheres.size();
    for (uint32_t i = 0; i < count; ++i) {
        float4 v;
        std::memcpy(&v, spheres + 4ull * i, sizeof v);
        const uint32_t m = material ? material[i] : 0u;
        if (m & ~ag::kTriMaterialMask) return c->fail(ALPINE_GPU_ERR_INVALID_ARGUMENT, "add_spheres: material id too large");
        c->spheres.push_back(v);
        c->sphereMaterial.push_back(m);
    }
    c->geometryDirty = true;
    c->bvhDirty = true;
    return ALPINE_GPU_OK;
}

int alpine_gpu_update_vertices(alpine_gpu_ctx* c, uint32_t shape, const float* vertices)
{
    if (!c) return ALPINE_GPU_ERR_INVALID_ARGUMENT;
    if (shape >= c->shapeVertBase.size() || !vertices)
        return c->fail(ALPINE_GPU_ERR_INVALID_ARGUMENT, "update_vertices: bad shape id or null array");
    if (int rc = c->pull_host_geometry()) return rc;
    std::memcpy(c->verts.data() + 3ull * c->shapeVertBase[shape], vertices,
                3ull * c->shapeVertCount[shape] * sizeof(float));
    c->geometryDirty = true;
    c->bvhDirty = true;
    return ALPINE_GPU_OK;
}

int alpine_gpu_build(alpine_gpu_ctx* c, alpine_gpu_bvh_stats* stats)
{
    if (!c) return ALPINE_GPU_ERR_INVALID_ARGUMENT;
    cudaSetDevice(c->device);
    if (int rc = upload_geometry_now(c)) return rc;
    uint32_t n = (uint32_t)(c->idx.size() / 3);
    const uint32_t ns = (uint32_t)c->spheres.size();
    const size_t prims = size_t(n) + ns;
    if (!c->dNodes.reserve((prims + 1) * sizeof(ag::WideNode)) || !c->dTris.reserve(prims * sizeof(ag::TriRecord)))
        return c->fail(ALPINE_GPU_ERR_OUT_OF_MEMORY, "build: cudaMalloc failed");
    ag::BuildStats bs;
    char err[256] = {0};
    int rc = c->builder.build(c->dVerts.as<float>(), c->dIdx.as<uint32_t>(), n, c->dSpheres.as<float4>(), ns,
                              c->dNodes.as<ag::WideNode>(), c->dTris.as<ag::TriRecord>(), c->dStatus, c->stream, &bs,
                              err, sizeof err);
    if (rc) {
        c->nodeCount = 0;
        c->triCount = 0;
        int code = rc == -2 ? ALPINE_GPU_ERR_CUDA : (rc == -5 ? ALPINE_GPU_ERR_OUT_OF_MEMORY : ALPINE_GPU_ERR_LIMIT);
        return c->fail(code, err);
    }
    c->nodeCount = prims ? bs.wideNodes : 0;
    c->triCount = (uint32_t)prims;
    c->bvhDirty = false;
    c->stats.triangles = n;
    c->stats.spheres = ns;
    c->stats.binary_nodes = bs.binaryNodes;
    c->stats.binary_levels = bs.binaryLevels;
    c->stats.wide_nodes = bs.wideNodes;
    c->stats.wide_depth = bs.wideDepth;
    c->stats.sah_cost = bs.sahCost;
    c->stats.build_ms = bs.buildMs;
    c->stats.child_slots = bs.childSlots;
    c->stats.big_levels = bs.bigLevels;
    c->syncBuildPrims = (uint32_t)prims;
    if (stats) *stats = c->stats;
    return check_status(c);
}

int alpine_gpu_build_async(alpine_gpu_ctx* c, uint32_t max_binary_levels, uint32_t max_wide_levels)
{
    if (!c) return ALPINE_GPU_ERR_INVALID_ARGUMENT;
    cudaSetDevice(c->device);
    if (int rc = upload_geometry_now(c)) return rc;
    const uint32_t n = (uint32_t)(c->idx.size() / 3);
    const uint32_t ns = (uint32_t)c->spheres.size();
    const uint32_t prims = n + ns;
    if (prims == 0 || prims != c->syncBuildPrims)
        return c->fail(ALPINE_GPU_ERR_INVALID_STATE,
                       "build_async: run alpine_gpu_build first with this scene's primitive count");
    // default caps: the last synchronous build's depths with a margin for
    // moving geometry (a deeper tree is reported, not built)
    const uint32_t lb = c->stats.binary_levels, wd = c->stats.wide_depth;
    const uint32_t L = max_binary_levels ? max_binary_levels : std::min<uint32_t>(1024u, lb + std::max(4u, lb / 4));
    const uint32_t W = max_wide_levels ? max_wide_levels : std::min<uint32_t>(64u, wd + 2u);
    char err[256] = {0};
    int rc = c->builder.enqueue(c->dVerts.as<float>(), c->dIdx.as<uint32_t>(), n, c->dSpheres.as<float4>(), ns,
                                c->dNodes.as<ag::WideNode>(), c->dTris.as<ag::TriRecord>(), c->dStatus, c->stream, L,
                                W, err, sizeof err);
    if (rc) return c->fail(rc == -2 ? ALPINE_GPU_ERR_CUDA : ALPINE_GPU_ERR_INVALID_ARGUMENT, err);
    // the node count of the new tree stays on the device: traversals check
    // child indices against the node array's capacity
    c->nodeCount = prims + 1;
    c->triCount = prims;
    c->bvhDirty = false;
    return ALPINE_GPU_OK;
}

int alpine_gpu_read_build_stats(alpine_gpu_ctx* c, alpine_gpu_bvh_stats* stats, uint32_t* graph_captures,
                                uint32_t* graph_launches)
{
    if (!c) return ALPINE_GPU_ERR_INVALID_ARGUMENT;
    cudaSetDevice(c->device);
    if (graph_captures) *graph_captures = c->builder.graph_captures();
    if (graph_launches) *graph_launches = c->builder.graph_launches();
    if (!stats) return check_status(c);
    ag::BuildStats bs;
    char err[256] = {0};
    if (int rc = c->builder.enqueued_stats(c->stream, &bs, err, sizeof err))
        return c->fail(rc == -2 ? ALPINE_GPU_ERR_CUDA : ALPINE_GPU_ERR_INVALID_STATE, err);
    *stats = c->stats;
    stats->binary_nodes = bs.binaryNodes;
    stats->binary_levels = bs.binaryLevels;
    stats->wide_nodes = bs.wideNodes;
    stats->wide_depth = bs.wideDepth;
    stats->sah_cost = bs.sahCost;
    stats->build_ms = bs.buildMs;
    stats->child_slots = bs.childSlots;
    return check_status(c);
}

int alpine_gpu_trace(alpine_gpu_ctx* c, const alpine_gpu_ray* rays, uint64_t n, alpine_gpu_hit* hits)
{
    return host_query<false>(c, rays, n, hits);
}

int alpine_gpu_occluded(alpine_gpu_ctx* c, const alpine_gpu_ray* rays, uint64_t n, uint8_t* occ)
{
    return host_query<true>(c, rays, n, occ);
}

int alpine_gpu_trace_device(alpine_gpu_ctx* c, const alpine_gpu_ray* rays, uint64_t n, alpine_gpu_hit* hits,
                            void* stream)
{
    return device_query<false>(c, rays, n, hits, stream);
}

int alpine_gpu_occluded_device(alpine_gpu_ctx* c, const alpine_gpu_ray* rays, uint64_t n, uint8_t* occ,
                               void* stream)
{
    return device_query<true>(c, rays, n, occ, stream);
}

int alpine_gpu_traversal_stats(alpine_gpu_ctx* c, const alpine_gpu_ray* rays, uint64_t n, int any,
                               uint64_t* nodeVisits, uint64_t* triVisits)
{
    if (!c || (n && !rays) || !nodeVisits || !triVisits)
        return c ? c->fail(ALPINE_GPU_ERR_INVALID_ARGUMENT, "traversal_stats: null argument") : -1;
    if (int rc = require_bvh(c)) return rc;
    DeviceBuffer counts;
    if (!counts.reserve(2 * sizeof(unsigned long long)))
        return c->fail(ALPINE_GPU_ERR_OUT_OF_MEMORY, "traversal_stats: cudaMalloc failed");
    unsigned long long h[2] = {0, 0};
    cudaError_t e = cudaMemsetAsync(counts.ptr, 0, sizeof h, c->stream);
    if (e == cudaSuccess && n) {
        ag::launch_trace_count(view(c), rays, n, any != 0, counts.as<unsigned long long>(), c->dStatus, c->stream);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(h, counts.ptr, sizeof h, cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) return c->fail(ALPINE_GPU_ERR_CUDA, cuda_msg("traversal_stats", e));
    *nodeVisits = h[0];
    *triVisits = h[1];
    return check_status(c);
}

int alpine_gpu_set_traversal_options(alpine_gpu_ctx* c, const alpine_gpu_traversal_options* o)
{
    if (!c) return ALPINE_GPU_ERR_INVALID_ARGUMENT;
    if (!o) return c->fail(ALPINE_GPU_ERR_INVALID_ARGUMENT, "set_traversal_options: null options");
    if (o->triangle_test != ALPINE_GPU_TRIANGLE_TEST_WIDE_BVH && o->triangle_test != ALPINE_GPU_TRIANGLE_TEST_BINARY_BVH)
        return c->fail(ALPINE_GPU_ERR_INVALID_ARGUMENT, "set_traversal_options: unknown triangle_test");
    if (o->stack_limit > (uint32_t)ag::kTraversalStack)
        return c->fail(ALPINE_GPU_ERR_INVALID_ARGUMENT,
                       "set_traversal_options: stack_limit above " + std::to_string(ag::kTraversalStack));
    c->traversal = *o;
    return ALPINE_GPU_OK;
}

int alpine_gpu_set_build_options(alpine_gpu_ctx* c, const alpine_gpu_build_options* o)
{
    if (!c) return ALPINE_GPU_ERR_INVALID_ARGUMENT;
    if (!o) return c->fail(ALPINE_GPU_ERR_INVALID_ARGUMENT, "set_build_options: null options");
    if (o->collapse != ALPINE_GPU_COLLAPSE_SAH && o->collapse != ALPINE_GPU_COLLAPSE_GREEDY)
        return c->fail(ALPINE_GPU_ERR_INVALID_ARGUMENT, "set_build_options: unknown collapse");
    if (!(o->triangle_cost >= 0.0f) || !(o->triangle_cost <= 1e6f))
        return c->fail(ALPINE_GPU_ERR_INVALID_ARGUMENT, "set_build_options: triangle_cost outside [0, 1e6]");
    c->builder.set_collapse(o->collapse == ALPINE_GPU_COLLAPSE_SAH ? ag::kCollapseSah : ag::kCollapseGreedy,
                            o->triangle_cost > 0.0f ? o->triangle_cost : ag::kCollapseTriCost);
    c->bvhDirty = true;
    return ALPINE_GPU_OK;
}

int alpine_gpu_synchronize(alpine_gpu_ctx* c)
{
    if (!c) return ALPINE_GPU_ERR_INVALID_ARGUMENT;
    cudaError_t e = cudaDeviceSynchronize();
    if (e != cudaSuccess) return c->fail(ALPINE_GPU_ERR_CUDA, cuda_msg("synchronize", e));
    return check_status(c);
}

}  // extern "C"

namespace ag {
int upload_geometry(alpine_gpu_ctx* c) { return upload_geometry_now(c); }
}  // namespace ag
