// alpine_gpu_load_glb / alpine_gpu_glb_inspect: binary glTF scenes loaded
// straight into a context, with the semantics of the reference's loader
// (src/loaders/gltf_loader.cpp, restated; the file parser is glb_parse.h):
//
// * materials (createMaterial, 384-415): base colour = baseColorFactor.rgb,
//   alpha = roughnessFactor, Conductor when metallicFactor > 0 else
//   Dielectric; textures (createTexture, 417-460) from 8-bit RGB / RGBA
//   images as float4(c / 255), base colours sRGB-decoded, normal maps
//   remapped to [-1, 1];
// * meshes (createMesh, 206-273): the primitives of a mesh concatenated
//   (indices offset by the vertices before them), POSITION / NORMAL /
//   TEXCOORD_0 / TANGENT, positions transformed by the node's matrix with
//   w = 1 and normals / tangents with w = 0 (not re-normalised), morph
//   targets (dense or sparse POSITION deltas, NORMAL deltas) left
//   untransformed; a mesh takes the transform of the last node that
//   references it, and meshes are added in mesh order, as the reference's
//   Scene::shapes[mesh index] then Alpine::loadScene do;
// * node transforms (getMatrix, 120-180; traverse, 182-204): the matrix, or
//   translation * rotation * scale from the quaternion, composed parent
//   first, column-major float4x4 arithmetic as src/math/matrix.h;
// * KHR_lights_punctual lights (createLight, 466-478): every light a point
//   light of intensity colour * intensity at the node's origin;
// * animations (createAnimation, 480-537): channels whose path is "weights",
//   whose node has a mesh and whose sampler is LINEAR, one keyframe per
//   input time with output / input weights each.
// The float arithmetic is written in the reference's order on the host, so
// positions, normals, texels and light powers are bit-identical to what the
// reference's loader builds from the same file.
#include "context.cuh"
#include "glb_parse.h"

#include <cmath>
#include <map>
#include <string>
#include <utility>
#include <vector>

namespace {

struct M4 {
    float v[16] = {1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1};  // column-major
};

struct V4 {
    float x, y, z, w;
};

// mul(Matrix4x4, Vector4) (src/math/matrix.h): columns scaled and summed in order
V4 mul(const M4& m, V4 a)
{
    const float s[4] = {a.x, a.y, a.z, a.w};
    V4 r{};
    float* o = &r.x;
    for (int k = 0; k < 4; ++k) {
        float acc = m.v[k] * s[0];
        acc = acc + m.v[4 + k] * s[1];
        acc = acc + m.v[8 + k] * s[2];
        acc = acc + m.v[12 + k] * s[3];
        o[k] = acc;
    }
    return r;
}

M4 mul(const M4& a, const M4& b)
{
    M4 m;
    for (int c = 0; c < 4; ++c) {
        V4 col{b.v[4 * c], b.v[4 * c + 1], b.v[4 * c + 2], b.v[4 * c + 3]};
        V4 r = mul(a, col);
        m.v[4 * c] = r.x;
        m.v[4 * c + 1] = r.y;
        m.v[4 * c + 2] = r.z;
        m.v[4 * c + 3] = r.w;
    }
    return m;
}

// getMatrix (gltf_loader.cpp:120-180)
M4 node_matrix(const glb::Node& n)
{
    M4 m;
    if (n.matrix.size() == 16) {
        for (int i = 0; i < 16; ++i) m.v[i] = (float)n.matrix[i];
        return m;
    }
    float qx = 0, qy = 0, qz = 0, qw = 1, sx = 1, sy = 1, sz = 1, tx = 0, ty = 0, tz = 0;
    if (n.rotation.size() == 4) {
        qx = (float)n.rotation[0]; qy = (float)n.rotation[1]; qz = (float)n.rotation[2]; qw = (float)n.rotation[3];
    }
    if (n.scale.size() == 3) { sx = (float)n.scale[0]; sy = (float)n.scale[1]; sz = (float)n.scale[2]; }
    if (n.translation.size() == 3) {
        tx = (float)n.translation[0]; ty = (float)n.translation[1]; tz = (float)n.translation[2];
    }
    m.v[0] = (1.0f - 2.0f * qy * qy - 2.0f * qz * qz) * sx;
    m.v[1] = (2.0f * qx * qy + 2.0f * qz * qw) * sx;
    m.v[2] = (2.0f * qx * qz - 2.0f * qy * qw) * sx;
    m.v[3] = 0.0f;
    m.v[4] = (2.0f * qx * qy - 2.0f * qz * qw) * sy;
    m.v[5] = (1.0f - 2.0f * qx * qx - 2.0f * qz * qz) * sy;
    m.v[6] = (2.0f * qy * qz + 2.0f * qx * qw) * sy;
    m.v[7] = 0.0f;
    m.v[8] = (2.0f * qx * qz + 2.0f * qy * qw) * sz;
    m.v[9] = (2.0f * qy * qz - 2.0f * qx * qw) * sz;
    m.v[10] = (1.0f - 2.0f * qx * qx - 2.0f * qy * qy) * sz;
    m.v[11] = 0.0f;
    m.v[12] = tx;
    m.v[13] = ty;
    m.v[14] = tz;
    m.v[15] = 1.0f;
    return m;
}

struct MeshData {
    std::vector<float> pos, nrm, uv, tan;        // 3, 3, 2, 4 floats per vertex
    std::vector<uint32_t> prims;                 // 3 per triangle
    std::vector<int> mats;                       // glTF material per triangle
    std::vector<std::vector<float>> tpos, tnrm;  // per target, 3 floats per vertex
    size_t weightCount = 0;
    bool used = false;
};

template <typename T>
const T* values(const glb::Document& d, const glb::Accessor& a)
{
    return reinterpret_cast<const T*>(d.data(a.bufferView, a.byteOffset, 0));
}

// appendVertexBuffer (gltf_loader.cpp:275-296) for a float attribute of
// `comps` components; returns the element count (0 when absent).
size_t append_attr(const glb::Document& d, const std::map<std::string, int>& attrs, const char* name, size_t comps,
                   std::vector<float>& dst, std::string& err)
{
    auto it = attrs.find(name);
    if (it == attrs.end()) return 0;
    if (it->second < 0 || it->second >= (int)d.accessors.size()) { err = "glb: bad accessor index"; return 0; }
    const glb::Accessor& a = d.accessors[it->second];
    if (a.componentType != glb::kFloat || glb::component_count(a.type) != comps) {
        err = std::string("glb: attribute ") + name + " must be float";
        return 0;
    }
    const float* v = values<float>(d, a);
    if (!v && a.count) { err = "glb: attribute outside its buffer"; return 0; }
    dst.insert(dst.end(), v, v + comps * a.count);
    return a.count;
}

bool build_mesh(const glb::Document& d, const glb::Mesh& src, const M4& matrix, MeshData& out, std::string& err)
{
    out = MeshData{};
    size_t indexOffset = 0;
    for (const glb::Primitive& p : src.primitives) {
        if (p.mode != 4) { err = "glb: only triangle primitives are read"; return false; }
        if (p.indices < 0 || p.indices >= (int)d.accessors.size()) { err = "glb: primitive without indices"; return false; }
        const glb::Accessor& ia = d.accessors[p.indices];
        const size_t primCount = ia.count / 3;
        const uint32_t off = (uint32_t)indexOffset;
        if (ia.componentType == glb::kUnsignedInt) {
            const uint32_t* v = values<uint32_t>(d, ia);
            for (size_t i = 0; i < 3 * primCount; ++i) out.prims.push_back(v[i] + off);
        } else if (ia.componentType == glb::kUnsignedShort) {
            const uint16_t* v = values<uint16_t>(d, ia);
            for (size_t i = 0; i < 3 * primCount; ++i) out.prims.push_back(v[i] + off);
        } else {
            err = "glb: indices must be unsigned short or int";
            return false;
        }
        for (size_t i = 0; i < primCount; ++i) out.mats.push_back(p.material);
        const size_t vertexCount = append_attr(d, p.attributes, "POSITION", 3, out.pos, err);
        if (!err.empty()) return false;
        indexOffset += vertexCount;
        append_attr(d, p.attributes, "NORMAL", 3, out.nrm, err);
        append_attr(d, p.attributes, "TEXCOORD_0", 2, out.uv, err);
        append_attr(d, p.attributes, "TANGENT", 4, out.tan, err);
        if (!err.empty()) return false;
        if (!p.targets.empty()) {
            if (out.tpos.empty()) { out.tpos.resize(p.targets.size()); out.tnrm.resize(p.targets.size()); }
            if (out.tpos.size() != p.targets.size()) { err = "glb: primitives differ in morph target count"; return false; }
            for (size_t t = 0; t < p.targets.size(); ++t) {
                const auto& tm = p.targets[t];
                auto pit = tm.find("POSITION");
                if (pit != tm.end()) {
                    const glb::Accessor& pa = d.accessors.at(pit->second);
                    if (!pa.sparse) {
                        append_attr(d, tm, "POSITION", 3, out.tpos[t], err);
                    } else {
                        // appendTargetVertexBuffer (gltf_loader.cpp:298-343): the
                        // target resized to this primitive's vertex count, zeroed,
                        // the sparse deltas written at their indices
                        std::vector<float>& dst = out.tpos[t];
                        dst.assign(3 * vertexCount, 0.0f);
                        const float* dv = reinterpret_cast<const float*>(
                            d.data(pa.sparseValues.bufferView, pa.sparseValues.byteOffset, 0));
                        for (size_t i = 0; i < pa.sparseCount; ++i) {
                            size_t idx;
                            if (pa.sparseIndices.componentType == glb::kUnsignedInt)
                                idx = reinterpret_cast<const uint32_t*>(
                                    d.data(pa.sparseIndices.bufferView, pa.sparseIndices.byteOffset, 0))[i];
                            else if (pa.sparseIndices.componentType == glb::kUnsignedShort)
                                idx = reinterpret_cast<const uint16_t*>(
                                    d.data(pa.sparseIndices.bufferView, pa.sparseIndices.byteOffset, 0))[i];
                            else { err = "glb: sparse indices must be unsigned short or int"; return false; }
                            if (idx >= vertexCount) { err = "glb: sparse index out of range"; return false; }
                            for (int k = 0; k < 3; ++k) dst[3 * idx + k] = dv[3 * i + k];
                        }
                    }
                }
                append_attr(d, tm, "NORMAL", 3, out.tnrm[t], err);
                if (!err.empty()) return false;
            }
        }
    }
    const size_t V = out.pos.size() / 3;
    if (out.nrm.size() != out.pos.size()) { err = "glb: every mesh needs vertex normals"; return false; }
    for (size_t i = 0; i < V; ++i) {  // createMesh's transform (gltf_loader.cpp:254-270)
        V4 p = mul(matrix, V4{out.pos[3 * i], out.pos[3 * i + 1], out.pos[3 * i + 2], 1.0f});
        out.pos[3 * i] = p.x; out.pos[3 * i + 1] = p.y; out.pos[3 * i + 2] = p.z;
        V4 n = mul(matrix, V4{out.nrm[3 * i], out.nrm[3 * i + 1], out.nrm[3 * i + 2], 0.0f});
        out.nrm[3 * i] = n.x; out.nrm[3 * i + 1] = n.y; out.nrm[3 * i + 2] = n.z;
        if (out.tan.size() == 4 * V) {
            V4 t = mul(matrix, V4{out.tan[4 * i], out.tan[4 * i + 1], out.tan[4 * i + 2], 0.0f});
            out.tan[4 * i] = t.x; out.tan[4 * i + 1] = t.y; out.tan[4 * i + 2] = t.z;
        }
    }
    out.weightCount = src.weights.size();
    return true;
}

// createTexture (gltf_loader.cpp:417-460)
bool make_texture(const glb::Image& im, bool isSigned, bool isSrgb, std::vector<float>& texels)
{
    if (im.component != 3 && im.component != 4) return false;
    const size_t n = (size_t)im.width * im.height;
    texels.resize(4 * n);
    auto srgbToLinear = [](float c) { return c <= 0.04045f ? c / 12.92f : std::pow((c + 0.055f) / 1.055f, 2.4f); };
    for (size_t i = 0; i < n; ++i) {
        const uint8_t* s = im.pixels.data() + im.component * i;
        float t[4] = {(float)s[0], (float)s[1], (float)s[2], im.component == 4 ? (float)s[3] : 255.0f};
        for (int k = 0; k < 4; ++k) {
            t[k] = t[k] / 255.0f;
            if (isSigned) t[k] = t[k] * 2.0f - 1.0f;
        }
        if (isSrgb)
            for (int k = 0; k < 3; ++k) t[k] = srgbToLinear(t[k]);
        for (int k = 0; k < 4; ++k) texels[4 * i + k] = t[k];
    }
    return true;
}

}  // namespace

extern "C" {

int alpine_gpu_glb_inspect(const char* path, alpine_gpu_glb_info* info)
{
    if (!path || !info) return ALPINE_GPU_ERR_INVALID_ARGUMENT;
    glb::Document d;
    std::string err;
    if (!glb::read_document(path, d, err)) return ALPINE_GPU_ERR_INVALID_ARGUMENT;
    *info = alpine_gpu_glb_info{};
    info->shapes = (uint32_t)d.meshes.size();
    for (const glb::Mesh& m : d.meshes)
        for (const glb::Primitive& p : m.primitives)
            if (p.indices >= 0 && p.indices < (int)d.accessors.size())
                info->triangles += (uint32_t)(d.accessors[p.indices].count / 3);
    info->materials = (uint32_t)d.materials.size();
    info->images = (uint32_t)d.images.size();
    info->lights = (uint32_t)d.lights.size();
    for (const glb::Animation& a : d.animations) info->channels += (uint32_t)a.channels.size();
    return ALPINE_GPU_OK;
}

int alpine_gpu_load_glb(alpine_gpu_ctx* c, const char* path, alpine_gpu_glb_info* info)
{
    if (!c) return ALPINE_GPU_ERR_INVALID_ARGUMENT;
    if (!path) return c->fail(ALPINE_GPU_ERR_INVALID_ARGUMENT, "load_glb: null path");
    glb::Document d;
    std::string err;
    if (!glb::read_document(path, d, err)) return c->fail(ALPINE_GPU_ERR_INVALID_ARGUMENT, err);
    alpine_gpu_glb_info out{};
    out.first_shape = (uint32_t)c->shapeVertBase.size();
    out.first_material = (uint32_t)c->materials.size();

    // materials and their textures (one texture per material use, as the reference)
    std::vector<ag::Material> mats;
    for (const glb::Material& m : d.materials) {
        alpine_gpu_material rec{};
        rec.kind = m.metallicFactor > 0.0 ? ALPINE_GPU_MATERIAL_CONDUCTOR : ALPINE_GPU_MATERIAL_DIELECTRIC;
        for (int k = 0; k < 3; ++k) rec.base_color[k] = (float)m.baseColorFactor[k];
        rec.roughness = (float)m.roughnessFactor;
        ag::Material x{};
        ag::make_material(rec, x);
        auto texture = [&](int texIdx, bool isSigned, bool isSrgb) -> uint32_t {
            if (texIdx < 0 || texIdx >= (int)d.textures.size()) return 0u;
            const int img = d.textures[texIdx];
            std::vector<float> t;
            if (img < 0 || img >= (int)d.images.size() || !make_texture(d.images[img], isSigned, isSrgb, t)) return 0u;
            uint32_t id = 0;
            if (alpine_gpu_add_texture(c, t.data(), d.images[img].width, d.images[img].height, &id) != ALPINE_GPU_OK)
                return 0u;
            ++out.textures;
            return id + 1u;
        };
        x.baseTex = texture(m.baseColorTexture, false, true);
        x.normalTex = texture(m.normalTexture, true, false);
        mats.push_back(x);
    }

    // nodes: transforms, meshes (the last node referencing a mesh wins), lights
    std::vector<MeshData> meshes(d.meshes.size());
    struct PendingLight { float3 intensity, position; };
    std::vector<PendingLight> lights;
    std::vector<int> stackNodes;
    std::vector<M4> stackMats;
    for (const auto& roots : d.scenes)
        for (int r : roots) {
            stackNodes.push_back(r);
            stackMats.push_back(M4{});
            while (!stackNodes.empty()) {  // depth-first, children in order
                const int ni = stackNodes.back();
                const M4 parent = stackMats.back();
                stackNodes.pop_back();
                stackMats.pop_back();
                if (ni < 0 || ni >= (int)d.nodes.size()) return c->fail(ALPINE_GPU_ERR_INVALID_ARGUMENT, "glb: bad node");
                const glb::Node& n = d.nodes[ni];
                const M4 m = mul(parent, node_matrix(n));
                if (n.mesh >= 0) {
                    if (n.mesh >= (int)d.meshes.size()) return c->fail(ALPINE_GPU_ERR_INVALID_ARGUMENT, "glb: bad mesh");
                    if (!build_mesh(d, d.meshes[n.mesh], m, meshes[n.mesh], err))
                        return c->fail(ALPINE_GPU_ERR_INVALID_ARGUMENT, err);
                    meshes[n.mesh].used = true;
                }
                if (n.light >= 0 && n.light < (int)d.lights.size()) {
                    const glb::Light& l = d.lights[n.light];
                    const float in = (float)l.intensity;
                    PendingLight pl;
                    pl.intensity = make_float3((float)l.color[0] * in, (float)l.color[1] * in, (float)l.color[2] * in);
                    const V4 o = mul(m, V4{0.0f, 0.0f, 0.0f, 1.0f});
                    pl.position = make_float3(o.x, o.y, o.z);
                    lights.push_back(pl);
                }
                for (auto it = n.children.rbegin(); it != n.children.rend(); ++it) {
                    stackNodes.push_back(*it);
                    stackMats.push_back(m);
                }
            }
        }

    c->materials.insert(c->materials.end(), mats.begin(), mats.end());
    c->materialsDirty = true;
    std::vector<int> shapeOf(d.meshes.size(), -1);
    for (size_t mi = 0; mi < meshes.size(); ++mi) {
        MeshData& md = meshes[mi];
        if (!md.used) continue;  // the reference would dereference an empty shape here
        const uint32_t V = (uint32_t)(md.pos.size() / 3), T = (uint32_t)(md.prims.size() / 3);
        uint32_t sid = 0;
        if (int rc = alpine_gpu_add_mesh(c, md.pos.data(), V, md.prims.data(), T, &sid)) return rc;
        std::vector<uint32_t> tm(T);
        for (uint32_t t = 0; t < T; ++t) {
            const int gm = md.mats[t];
            if (gm < 0 || gm >= (int)mats.size()) return c->fail(ALPINE_GPU_ERR_INVALID_ARGUMENT, "glb: primitive without material");
            tm[t] = out.first_material + (uint32_t)gm;
        }
        if (int rc = alpine_gpu_set_triangle_attributes(c, sid, md.nrm.data(), tm.data())) return rc;
        const bool uv = md.uv.size() == 2ull * V, tan = uv && md.tan.size() == 4ull * V;
        if (uv)
            if (int rc = alpine_gpu_set_triangle_uvs(c, sid, md.uv.data(), tan ? md.tan.data() : nullptr)) return rc;
        if (!md.tpos.empty()) {
            const uint32_t targets = (uint32_t)md.tpos.size();
            std::vector<float> dv(3ull * V * targets, 0.0f), dn;
            bool normals = true;
            for (uint32_t t = 0; t < targets; ++t) {
                if (md.tpos[t].size() != 3ull * V) return c->fail(ALPINE_GPU_ERR_INVALID_ARGUMENT, "glb: morph target size");
                std::copy(md.tpos[t].begin(), md.tpos[t].end(), dv.begin() + 3ull * V * t);
                normals &= md.tnrm[t].size() == 3ull * V;
            }
            if (normals) {
                dn.resize(dv.size());
                for (uint32_t t = 0; t < targets; ++t) std::copy(md.tnrm[t].begin(), md.tnrm[t].end(), dn.begin() + 3ull * V * t);
            }
            if (int rc = alpine_gpu_set_morph_targets(c, sid, dv.data(), normals ? dn.data() : nullptr, targets)) return rc;
        }
        shapeOf[mi] = (int)sid;
        ++out.shapes;
        out.triangles += T;
    }
    for (const PendingLight& pl : lights) {
        if (int rc = ag::add_point_light_intensity(c, pl.intensity, pl.position, nullptr)) return rc;
        ++out.lights;
    }
    // animations: weights channels of meshes, LINEAR samplers
    for (const glb::Animation& an : d.animations)
        for (const glb::AnimChannel& ch : an.channels) {
            if (ch.path != "weights" || ch.node < 0 || ch.node >= (int)d.nodes.size()) continue;
            const int mesh = d.nodes[ch.node].mesh;
            if (mesh < 0 || shapeOf[mesh] < 0) continue;
            if (ch.sampler < 0 || ch.sampler >= (int)an.samplers.size()) continue;
            const glb::AnimSampler& s = an.samplers[ch.sampler];
            if (s.interpolation != "LINEAR") continue;
            if (s.input < 0 || s.output < 0 || s.input >= (int)d.accessors.size() || s.output >= (int)d.accessors.size())
                return c->fail(ALPINE_GPU_ERR_INVALID_ARGUMENT, "glb: bad animation sampler");
            const glb::Accessor& ia = d.accessors[s.input];
            const glb::Accessor& oa = d.accessors[s.output];
            const float* times = values<float>(d, ia);
            const float* w = values<float>(d, oa);
            if (!times || !w || ia.count < 2) return c->fail(ALPINE_GPU_ERR_INVALID_ARGUMENT, "glb: bad animation data");
            const size_t morphCount = oa.count / ia.count;
            if (morphCount != meshes[mesh].tpos.size() || morphCount != meshes[mesh].weightCount)
                return c->fail(ALPINE_GPU_ERR_INVALID_ARGUMENT,
                               "glb: animation weights differ from the mesh's morph targets / default weights");
            std::vector<float> weights(w, w + morphCount * ia.count);
            if (int rc = alpine_gpu_add_animation_channel(c, (uint32_t)shapeOf[mesh], times, weights.data(),
                                                          (uint32_t)ia.count))
                return rc;
            ++out.channels;
        }
    out.images = (uint32_t)d.images.size();
    out.materials = (uint32_t)mats.size();
    if (info) *info = out;
    return ALPINE_GPU_OK;
}

}  // extern "C"
