// Test infrastructure (oracle): a stand-in for tinygltf's tiny_gltf.h, which
// the reference's loader includes (src/loaders/gltf_loader.cpp:15-18) but
// which is not vendored with it. It declares the part of tinygltf's public
// model the loader reads (tinygltf 2.x: Model, Node, Mesh, Primitive,
// Accessor with Sparse, BufferView, Buffer, Material, Texture, Image, Light,
// Animation, Scene; TinyGLTF::LoadBinaryFromFile) with tinygltf's names and
// glTF defaults, and fills it from the project's GLB reader
// (alpine_b200/csrc/glb_parse.h), so that the reference's own loader code
// runs unchanged on the same files as the GPU backend's loader.
#pragma once

#include <glb_parse.h>

#include <map>
#include <string>
#include <vector>

#define TINYGLTF_MODE_TRIANGLES 4
#define TINYGLTF_COMPONENT_TYPE_UNSIGNED_BYTE 5121
#define TINYGLTF_COMPONENT_TYPE_UNSIGNED_SHORT 5123
#define TINYGLTF_COMPONENT_TYPE_UNSIGNED_INT 5125
#define TINYGLTF_COMPONENT_TYPE_FLOAT 5126

namespace tinygltf {
struct Buffer {
    std::vector<unsigned char> data;
};
struct BufferView {
    int buffer = -1;
    size_t byteOffset = 0;
    size_t byteLength = 0;
    size_t byteStride = 0;
};
struct Accessor {
    int bufferView = -1;
    size_t byteOffset = 0;
    int componentType = -1;
    size_t count = 0;
    struct Sparse {
        int count = 0;
        bool isSparse = false;
        struct {
            int bufferView = -1;
            int byteOffset = 0;
            int componentType = -1;
        } indices;
        struct {
            int bufferView = -1;
            int byteOffset = 0;
        } values;
    } sparse;
};
struct Primitive {
    std::map<std::string, int> attributes;
    int material = -1;
    int indices = -1;
    int mode = -1;
    std::vector<std::map<std::string, int>> targets;
};
struct Mesh {
    std::vector<Primitive> primitives;
    std::vector<double> weights;
};
struct Node {
    int mesh = -1;
    int light = -1;
    std::vector<int> children;
    std::vector<double> rotation, scale, translation, matrix;
};
struct TextureInfo {
    int index = -1;
};
struct NormalTextureInfo {
    int index = -1;
};
struct PbrMetallicRoughness {
    std::vector<double> baseColorFactor{1.0, 1.0, 1.0, 1.0};
    TextureInfo baseColorTexture;
    double metallicFactor = 1.0;
    double roughnessFactor = 1.0;
};
struct Material {
    PbrMetallicRoughness pbrMetallicRoughness;
    NormalTextureInfo normalTexture;
};
struct Texture {
    int source = -1;
};
struct Image {
    std::string name;
    int width = -1, height = -1, component = -1, bits = -1;
    std::vector<unsigned char> image;
};
struct Light {
    std::string type;
    std::vector<double> color;
    double intensity = 1.0;
};
struct AnimationChannel {
    int sampler = -1;
    int target_node = -1;
    std::string target_path;
};
struct AnimationSampler {
    int input = -1;
    int output = -1;
    std::string interpolation;
};
struct Animation {
    std::vector<AnimationChannel> channels;
    std::vector<AnimationSampler> samplers;
};
struct Scene {
    std::vector<int> nodes;
};
struct Model {
    std::vector<Accessor> accessors;
    std::vector<Animation> animations;
    std::vector<Buffer> buffers;
    std::vector<BufferView> bufferViews;
    std::vector<Material> materials;
    std::vector<Mesh> meshes;
    std::vector<Node> nodes;
    std::vector<Texture> textures;
    std::vector<Image> images;
    std::vector<Scene> scenes;
    std::vector<Light> lights;
};

class TinyGLTF {
public:
    bool LoadBinaryFromFile(Model* model, std::string* err, std::string* warn, const std::string& filename)
    {
        if (warn) warn->clear();
        glb::Document d;
        std::string e;
        if (!glb::read_document(filename.c_str(), d, e)) {
            if (err) *err = e + "\n";
            return false;
        }
        Model m;
        for (auto& b : d.buffers) m.buffers.push_back(Buffer{b});
        for (auto& v : d.bufferViews) m.bufferViews.push_back(BufferView{v.buffer, v.byteOffset, v.byteLength, v.byteStride});
        for (auto& x : d.accessors) {
            Accessor a;
            a.bufferView = x.bufferView;
            a.byteOffset = x.byteOffset;
            a.componentType = x.componentType;
            a.count = x.count;
            a.sparse.isSparse = x.sparse;
            a.sparse.count = (int)x.sparseCount;
            a.sparse.indices.bufferView = x.sparseIndices.bufferView;
            a.sparse.indices.byteOffset = (int)x.sparseIndices.byteOffset;
            a.sparse.indices.componentType = x.sparseIndices.componentType;
            a.sparse.values.bufferView = x.sparseValues.bufferView;
            a.sparse.values.byteOffset = (int)x.sparseValues.byteOffset;
            m.accessors.push_back(a);
        }
        for (auto& me : d.meshes) {
            Mesh o;
            o.weights = me.weights;
            for (auto& p : me.primitives) o.primitives.push_back(Primitive{p.attributes, p.material, p.indices, p.mode, p.targets});
            m.meshes.push_back(std::move(o));
        }
        for (auto& n : d.nodes) {
            Node o;
            o.mesh = n.mesh;
            o.light = n.light;
            o.children = n.children;
            o.rotation = n.rotation;
            o.scale = n.scale;
            o.translation = n.translation;
            o.matrix = n.matrix;
            m.nodes.push_back(std::move(o));
        }
        for (auto& mt : d.materials) {
            Material o;
            o.pbrMetallicRoughness.baseColorFactor = mt.baseColorFactor;
            o.pbrMetallicRoughness.baseColorTexture.index = mt.baseColorTexture;
            o.pbrMetallicRoughness.metallicFactor = mt.metallicFactor;
            o.pbrMetallicRoughness.roughnessFactor = mt.roughnessFactor;
            o.normalTexture.index = mt.normalTexture;
            m.materials.push_back(o);
        }
        for (int s : d.textures) m.textures.push_back(Texture{s});
        for (auto& im : d.images) {
            Image o;
            o.name = im.name;
            o.width = im.width;
            o.height = im.height;
            o.component = im.component;
            o.bits = 8;
            o.image = im.pixels;
            m.images.push_back(std::move(o));
        }
        for (auto& l : d.lights) m.lights.push_back(Light{l.type, l.color, l.intensity});
        for (auto& an : d.animations) {
            Animation o;
            for (auto& c : an.channels) o.channels.push_back(AnimationChannel{c.sampler, c.node, c.path});
            for (auto& s : an.samplers) o.samplers.push_back(AnimationSampler{s.input, s.output, s.interpolation});
            m.animations.push_back(std::move(o));
        }
        for (auto& sc : d.scenes) m.scenes.push_back(Scene{sc});
        *model = std::move(m);
        if (err) err->clear();
        return true;
    }
};
}  // namespace tinygltf
