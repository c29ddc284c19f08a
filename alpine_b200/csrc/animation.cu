// Morph-target animation on the device: Mesh::update (src/shapes/mesh.cpp:
// 29-55) and Animation::update (src/animation.cpp:10-39) behind
// Alpine::updateScene (src/alpine.cpp:204-212), followed by a BVH rebuild.
//
// The keyframe weights of each channel are computed on the host exactly as the
// reference does (clamp, segment search, std::lerp); the vertices (and the
// vertex normals, when the targets carry normals) are morphed on the device
// with every product and sum rounded separately, in the reference's order:
// v = base; v += target_j * w_j for j = 0, 1, ...
#include "context.cuh"

#include <algorithm>
#include <cstring>

namespace {

constexpr uint32_t kMaxTargets = 32;

struct Weights {
    float w[kMaxTargets];
};

// out[i] = base[i] + sum_j deltas[j][i] * w_j over n floats (x, y, z interleaved).
__global__ void k_morph(const float* __restrict__ base, const float* __restrict__ deltas, uint32_t n, uint32_t targets,
                        Weights w, float* __restrict__ out)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float v = base[i];
    for (uint32_t j = 0; j < targets; ++j) v = __fadd_rn(v, __fmul_rn(deltas[(uint64_t)j * n + i], w.w[j]));
    out[i] = v;
}

// std::lerp as specified by P0811R3 (C++20 [c.math.lerp]) in the form the
// GNU C++ library evaluates it: exact at t = 0 and t = 1, monotonic, and
// t * b + (1 - t) * a when a and b differ in sign.
float lerp_c20(float a, float b, float t)
{
    if ((a <= 0.0f && b >= 0.0f) || (a >= 0.0f && b <= 0.0f)) return t * b + (1.0f - t) * a;
    if (t == 1.0f) return b;
    const float x = a + t * (b - a);
    return (t > 1.0f) == (b > a) ? (b < x ? x : b) : (b > x ? x : b);
}

// Animation::update for one channel (animation.cpp:13-37): the channel's
// weights at `time`.
void channel_weights(const alpine_gpu_ctx::Channel& ch, uint32_t targets, float time, std::vector<float>& out)
{
    const size_t K = ch.times.size();
    const float ct = std::clamp(time, ch.times.front(), ch.times.back());
    uint32_t index = (uint32_t)K - 2;
    for (uint32_t i = 0; i + 1 < K; ++i)
        if (ct <= ch.times[i + 1]) {
            index = i;
            break;
        }
    const float t0 = ch.times[index], t1 = ch.times[index + 1];
    const float t = (ct - t0) / (t1 - t0);
    out.resize(targets);
    for (uint32_t j = 0; j < targets; ++j)
        out[j] = lerp_c20(ch.weights[(size_t)index * targets + j], ch.weights[(size_t)(index + 1) * targets + j], t);
}

int morph_shape(alpine_gpu_ctx* c, alpine_gpu_ctx::Morph& m)
{
    Weights w{};
    for (uint32_t j = 0; j < m.targets; ++j) w.w[j] = m.weights[j];
    const uint32_t n = 3 * c->shapeVertCount[m.shape];
    if (n == 0) return ALPINE_GPU_OK;
    const size_t off = 3ull * c->shapeVertBase[m.shape];
    k_morph<<<(n + 255) / 256, 256, 0, c->stream>>>(m.dBase.as<float>(), m.dDeltas.as<float>(), n, m.targets, w,
                                                     c->dVerts.as<float>() + off);
    if (m.normals)
        k_morph<<<(n + 255) / 256, 256, 0, c->stream>>>(m.dBaseN.as<float>(), m.dDeltasN.as<float>(), n, m.targets, w,
                                                         c->dNormals.as<float>() + off);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? ALPINE_GPU_OK : c->fail(ALPINE_GPU_ERR_CUDA, std::string("morph: ") + cudaGetErrorString(e));
}

bool upload(ag::DeviceBuffer& b, const float* src, size_t count, cudaStream_t st)
{
    if (!b.reserve(std::max<size_t>(count, 1) * sizeof(float))) return false;
    return count == 0 || cudaMemcpyAsync(b.ptr, src, count * sizeof(float), cudaMemcpyHostToDevice, st) == cudaSuccess;
}

alpine_gpu_ctx::Morph* find_morph(alpine_gpu_ctx* c, uint32_t shape, uint32_t* index = nullptr)
{
    for (uint32_t i = 0; i < c->morphs.size(); ++i)
        if (c->morphs[i]->shape == shape) {
            if (index) *index = i;
            return c->morphs[i].get();
        }
    return nullptr;
}

}  // namespace

extern "C" {

int alpine_gpu_set_morph_targets(alpine_gpu_ctx* c, uint32_t shape, const float* vertex_deltas,
                                 const float* normal_deltas, uint32_t count)
{
    if (!c) return ALPINE_GPU_ERR_INVALID_ARGUMENT;
    if (shape >= c->shapeVertBase.size()) return c->fail(ALPINE_GPU_ERR_INVALID_ARGUMENT, "set_morph_targets: bad shape id");
    if (count == 0 || count > kMaxTargets || !vertex_deltas)
        return c->fail(ALPINE_GPU_ERR_INVALID_ARGUMENT, "set_morph_targets: 1 to 32 targets with vertex deltas");
    if (int rc = c->pull_host_geometry()) return rc;
    const uint32_t vb = c->shapeVertBase[shape], vc = c->shapeVertCount[shape];
    const uint32_t tb = c->shapeTriBase[shape], tc = c->shapeTriCount[shape];
    bool hasNormals = false;
    if (normal_deltas) {
        // the mesh's own vertex normals are the base (set_triangle_attributes)
        hasNormals = c->triInfo.size() >= (size_t)tb + tc && tc && (c->triInfo[tb] & ag::kTriHasNormals);
        if (!hasNormals)
            return c->fail(ALPINE_GPU_ERR_INVALID_STATE, "set_morph_targets: normal deltas for a mesh without normals");
    }
    uint32_t idx = 0;
    alpine_gpu_ctx::Morph* m = find_morph(c, shape, &idx);
    if (!m) {
        c->morphs.push_back(std::make_unique<alpine_gpu_ctx::Morph>());
        m = c->morphs.back().get();
    }
    m->shape = shape;
    m->targets = count;
    m->normals = hasNormals;
    m->weights.assign(count, 0.0f);  // Mesh::Mesh starts from zero weights (mesh.cpp:14-20)
    cudaSetDevice(c->device);
    const size_t n = 3ull * vc;
    bool ok = upload(m->dBase, c->verts.data() + 3ull * vb, n, c->stream) &&
              upload(m->dDeltas, vertex_deltas, n * count, c->stream);
    if (ok && hasNormals)
        ok = upload(m->dBaseN, c->normals.data() + 3ull * vb, n, c->stream) &&
             upload(m->dDeltasN, normal_deltas, n * count, c->stream);
    if (ok) ok = cudaStreamSynchronize(c->stream) == cudaSuccess;
    if (!ok) return c->fail(ALPINE_GPU_ERR_OUT_OF_MEMORY, "set_morph_targets: upload failed");
    if (hasNormals) {
        for (uint32_t t = 0; t < tc; ++t) c->triInfo[tb + t] |= ag::kTriMorphedNormals;
        c->attribsDirty = true;
    }
    return ALPINE_GPU_OK;
}

int alpine_gpu_add_animation_channel(alpine_gpu_ctx* c, uint32_t shape, const float* times, const float* weights,
                                     uint32_t keyframes)
{
    if (!c) return ALPINE_GPU_ERR_INVALID_ARGUMENT;
    uint32_t idx = 0;
    alpine_gpu_ctx::Morph* m = find_morph(c, shape, &idx);
    if (!m) return c->fail(ALPINE_GPU_ERR_INVALID_STATE, "add_animation_channel: the shape has no morph targets");
    if (keyframes < 2 || !times || !weights)
        return c->fail(ALPINE_GPU_ERR_INVALID_ARGUMENT, "add_animation_channel: at least two keyframes");
    for (uint32_t k = 0; k + 1 < keyframes; ++k)
        if (!(times[k] <= times[k + 1]))
            return c->fail(ALPINE_GPU_ERR_INVALID_ARGUMENT, "add_animation_channel: keyframe times must not decrease");
    alpine_gpu_ctx::Channel ch;
    ch.morph = idx;
    ch.times.assign(times, times + keyframes);
    ch.weights.assign(weights, weights + (size_t)keyframes * m->targets);
    c->channels.push_back(std::move(ch));
    return ALPINE_GPU_OK;
}

namespace {
// Alpine::updateScene's morph (src/alpine.cpp:204-212) on the context stream,
// without waiting.
int morph_all(alpine_gpu_ctx* c, float time)
{
    cudaSetDevice(c->device);
    // device copies of the geometry and the attributes first: the morph
    // writes into them
    if (int rc = ag::upload_geometry(c)) return rc;
    bool normalsMorphed = false;
    for (const auto& m : c->morphs) normalsMorphed |= m->normals;
    if (normalsMorphed) {
        if (c->triInfo.size() < c->idx.size() / 3) {
            c->triInfo.resize(c->idx.size() / 3, 0u);
            c->attribsDirty = true;
        }
        if (int rc = ag::upload_render_scene(c)) return rc;
    }
    std::vector<float> w;
    for (const auto& ch : c->channels) {
        alpine_gpu_ctx::Morph& m = *c->morphs[ch.morph];
        channel_weights(ch, m.targets, time, w);
        m.weights = w;
        if (int rc = morph_shape(c, m)) return rc;
        c->hostVertsStale = true;
        c->hostNormalsStale |= m.normals;
    }
    c->geometryDirty = false;  // the device copy is the newest
    c->bvhDirty = true;
    return ALPINE_GPU_OK;
}
}  // namespace

int alpine_gpu_update_scene(alpine_gpu_ctx* c, float time, alpine_gpu_bvh_stats* stats)
{
    if (!c) return ALPINE_GPU_ERR_INVALID_ARGUMENT;
    if (int rc = morph_all(c, time)) return rc;
    return alpine_gpu_build(c, stats);  // Accelerator::updateScene
}

int alpine_gpu_update_scene_async(alpine_gpu_ctx* c, float time)
{
    if (!c) return ALPINE_GPU_ERR_INVALID_ARGUMENT;
    if (int rc = morph_all(c, time)) return rc;
    return alpine_gpu_build_async(c, 0u, 0u);
}

int alpine_gpu_get_vertices(alpine_gpu_ctx* c, uint32_t shape, float* vertices, float* normals)
{
    if (!c) return ALPINE_GPU_ERR_INVALID_ARGUMENT;
    if (shape >= c->shapeVertBase.size()) return c->fail(ALPINE_GPU_ERR_INVALID_ARGUMENT, "get_vertices: bad shape id");
    cudaSetDevice(c->device);
    if (int rc = c->pull_host_geometry()) return rc;
    const size_t off = 3ull * c->shapeVertBase[shape], n = 3ull * c->shapeVertCount[shape];
    if (vertices) std::memcpy(vertices, c->verts.data() + off, n * sizeof(float));
    if (normals) {
        if (c->normals.size() >= off + n) std::memcpy(normals, c->normals.data() + off, n * sizeof(float));
        else std::memset(normals, 0, n * sizeof(float));
    }
    return ALPINE_GPU_OK;
}

}  // extern "C"
