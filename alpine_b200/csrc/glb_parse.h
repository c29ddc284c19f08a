// Binary glTF 2.0 (.glb) reader: the container, the JSON document, buffers,
// accessors and PNG images, for the subset alpine's loader reads
// (src/loaders/gltf_loader.cpp): scenes, nodes (matrix or TRS, children,
// mesh, KHR_lights_punctual light), meshes (triangle primitives, POSITION /
// NORMAL / TEXCOORD_0 / TANGENT, morph targets with dense or sparse
// positions), materials (pbrMetallicRoughness factors and base-colour
// texture, normal texture), textures and images (PNG, 8-bit RGB / RGBA),
// punctual lights and animations (sampler input / output / interpolation,
// channel target node and path).
//
// The reference reads these files through tinygltf (not vendored with it);
// this is a project-written parser of the published formats: the glTF 2.0
// binary container and JSON schema (Khronos), PNG (ISO/IEC 15948) and zlib /
// DEFLATE (RFC 1950 / 1951). Host-only C++17, no dependencies. glTF defaults
// apply where a property is absent (metallicFactor = roughnessFactor = 1,
// baseColorFactor = (1, 1, 1, 1), light colour (1, 1, 1), intensity 1,
// interpolation LINEAR, primitive mode 4 = triangles).
#pragma once

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <string>
#include <vector>

namespace glb {

// ---------------------------------------------------------------------------
// JSON (RFC 8259) value and a recursive-descent parser.
struct Json {
    enum Kind { Null, Bool, Number, String, Array, Object } kind = Null;
    bool b = false;
    double num = 0.0;
    std::string str;
    std::vector<Json> arr;
    std::map<std::string, Json> obj;

    const Json* get(const char* key) const
    {
        if (kind != Object) return nullptr;
        auto it = obj.find(key);
        return it == obj.end() ? nullptr : &it->second;
    }
    double number(const char* key, double dflt) const
    {
        const Json* j = get(key);
        return j && j->kind == Number ? j->num : dflt;
    }
    int integer(const char* key, int dflt) const { return (int)number(key, dflt); }
    std::string string(const char* key, const char* dflt) const
    {
        const Json* j = get(key);
        return j && j->kind == String ? j->str : std::string(dflt);
    }
    std::vector<double> numbers(const char* key) const
    {
        std::vector<double> out;
        const Json* j = get(key);
        if (j && j->kind == Array)
            for (const Json& e : j->arr)
                if (e.kind == Number) out.push_back(e.num);
        return out;
    }
};

class JsonParser {
public:
    JsonParser(const char* p, size_t n) : p_(p), end_(p + n) {}

    bool parse(Json& out, std::string& err)
    {
        if (!value(out, 0)) {
            err = "glb: JSON syntax error near byte " + std::to_string(pos_);
            return false;
        }
        ws();
        return true;
    }

private:
    const char* p_;
    const char* end_;
    size_t pos_ = 0;

    bool eof() const { return p_ >= end_; }
    void adv() { ++p_; ++pos_; }
    void ws()
    {
        while (!eof() && (*p_ == ' ' || *p_ == '\t' || *p_ == '\n' || *p_ == '\r')) adv();
    }
    bool lit(const char* s)
    {
        size_t n = std::strlen(s);
        if ((size_t)(end_ - p_) < n || std::memcmp(p_, s, n) != 0) return false;
        for (size_t i = 0; i < n; ++i) adv();
        return true;
    }
    static void put_utf8(std::string& s, uint32_t c)
    {
        if (c < 0x80) {
            s += (char)c;
        } else if (c < 0x800) {
            s += (char)(0xc0 | (c >> 6));
            s += (char)(0x80 | (c & 0x3f));
        } else if (c < 0x10000) {
            s += (char)(0xe0 | (c >> 12));
            s += (char)(0x80 | ((c >> 6) & 0x3f));
            s += (char)(0x80 | (c & 0x3f));
        } else {
            s += (char)(0xf0 | (c >> 18));
            s += (char)(0x80 | ((c >> 12) & 0x3f));
            s += (char)(0x80 | ((c >> 6) & 0x3f));
            s += (char)(0x80 | (c & 0x3f));
        }
    }
    bool hex4(uint32_t& v)
    {
        v = 0;
        for (int i = 0; i < 4; ++i) {
            if (eof()) return false;
            char c = *p_;
            adv();
            v <<= 4;
            if (c >= '0' && c <= '9') v |= (uint32_t)(c - '0');
            else if (c >= 'a' && c <= 'f') v |= (uint32_t)(c - 'a' + 10);
            else if (c >= 'A' && c <= 'F') v |= (uint32_t)(c - 'A' + 10);
            else return false;
        }
        return true;
    }
    bool string(std::string& s)
    {
        if (eof() || *p_ != '"') return false;
        adv();
        while (!eof() && *p_ != '"') {
            char c = *p_;
            adv();
            if (c != '\\') {
                s += c;
                continue;
            }
            if (eof()) return false;
            char e = *p_;
            adv();
            switch (e) {
            case '"': s += '"'; break;
            case '\\': s += '\\'; break;
            case '/': s += '/'; break;
            case 'b': s += '\b'; break;
            case 'f': s += '\f'; break;
            case 'n': s += '\n'; break;
            case 'r': s += '\r'; break;
            case 't': s += '\t'; break;
            case 'u': {
                uint32_t c1;
                if (!hex4(c1)) return false;
                if (c1 >= 0xd800 && c1 < 0xdc00) {  // surrogate pair
                    uint32_t c2;
                    if (!lit("\\u") || !hex4(c2) || c2 < 0xdc00 || c2 >= 0xe000) return false;
                    c1 = 0x10000 + ((c1 - 0xd800) << 10) + (c2 - 0xdc00);
                }
                put_utf8(s, c1);
                break;
            }
            default: return false;
            }
        }
        if (eof()) return false;
        adv();
        return true;
    }
    bool value(Json& v, int depth)
    {
        if (depth > 256) return false;
        ws();
        if (eof()) return false;
        const char c = *p_;
        if (c == '{') {
            adv();
            v.kind = Json::Object;
            ws();
            if (!eof() && *p_ == '}') { adv(); return true; }
            for (;;) {
                ws();
                std::string key;
                if (!string(key)) return false;
                ws();
                if (eof() || *p_ != ':') return false;
                adv();
                Json child;
                if (!value(child, depth + 1)) return false;
                v.obj[key] = std::move(child);
                ws();
                if (eof()) return false;
                if (*p_ == ',') { adv(); continue; }
                if (*p_ == '}') { adv(); return true; }
                return false;
            }
        }
        if (c == '[') {
            adv();
            v.kind = Json::Array;
            ws();
            if (!eof() && *p_ == ']') { adv(); return true; }
            for (;;) {
                Json child;
                if (!value(child, depth + 1)) return false;
                v.arr.push_back(std::move(child));
                ws();
                if (eof()) return false;
                if (*p_ == ',') { adv(); continue; }
                if (*p_ == ']') { adv(); return true; }
                return false;
            }
        }
        if (c == '"') {
            v.kind = Json::String;
            return string(v.str);
        }
        if (lit("true")) { v.kind = Json::Bool; v.b = true; return true; }
        if (lit("false")) { v.kind = Json::Bool; v.b = false; return true; }
        if (lit("null")) { v.kind = Json::Null; return true; }
        // number
        const char* s = p_;
        if (*p_ == '-') adv();
        bool digits = false;
        while (!eof() && *p_ >= '0' && *p_ <= '9') { adv(); digits = true; }
        if (!eof() && *p_ == '.') {
            adv();
            while (!eof() && *p_ >= '0' && *p_ <= '9') { adv(); digits = true; }
        }
        if (!digits) return false;
        if (!eof() && (*p_ == 'e' || *p_ == 'E')) {
            adv();
            if (!eof() && (*p_ == '+' || *p_ == '-')) adv();
            bool ed = false;
            while (!eof() && *p_ >= '0' && *p_ <= '9') { adv(); ed = true; }
            if (!ed) return false;
        }
        v.kind = Json::Number;
        v.num = std::strtod(std::string(s, p_).c_str(), nullptr);
        return true;
    }
};

// ---------------------------------------------------------------------------
// DEFLATE (RFC 1951) decoder: stored, fixed-Huffman and dynamic-Huffman
// blocks, canonical Huffman codes decoded bit by bit.
class Inflate {
public:
    Inflate(const uint8_t* p, size_t n) : p_(p), n_(n) {}

    bool run(std::vector<uint8_t>& out)
    {
        for (;;) {
            int final = bits(1);
            int type = bits(2);
            if (bad_) return false;
            if (type == 0) {
                if (!stored(out)) return false;
            } else if (type == 1) {
                Huff lit, dist;
                fixed(lit, dist);
                if (!codes(out, lit, dist)) return false;
            } else if (type == 2) {
                Huff lit, dist;
                if (!dynamic(lit, dist) || !codes(out, lit, dist)) return false;
            } else {
                return false;
            }
            if (final) return !bad_;
        }
    }

private:
    struct Huff {
        uint16_t count[16] = {};
        uint16_t symbol[320] = {};
    };
    const uint8_t* p_;
    size_t n_;
    size_t pos_ = 0;
    uint32_t bitbuf_ = 0;
    int bitcnt_ = 0;
    bool bad_ = false;

    int bits(int need)
    {
        uint32_t v = bitbuf_;
        while (bitcnt_ < need) {
            if (pos_ >= n_) { bad_ = true; return 0; }
            v |= (uint32_t)p_[pos_++] << bitcnt_;
            bitcnt_ += 8;
        }
        bitbuf_ = v >> need;
        bitcnt_ -= need;
        return (int)(v & ((1u << need) - 1u));
    }
    bool stored(std::vector<uint8_t>& out)
    {
        bitbuf_ = 0;
        bitcnt_ = 0;
        if (pos_ + 4 > n_) return false;
        uint32_t len = p_[pos_] | (p_[pos_ + 1] << 8);
        uint32_t nlen = p_[pos_ + 2] | (p_[pos_ + 3] << 8);
        pos_ += 4;
        if (len != (~nlen & 0xffffu) || pos_ + len > n_) return false;
        out.insert(out.end(), p_ + pos_, p_ + pos_ + len);
        pos_ += len;
        return true;
    }
    // Builds a canonical code from code lengths; false when over-subscribed.
    static bool build(Huff& h, const uint8_t* lengths, int n)
    {
        std::memset(h.count, 0, sizeof h.count);
        for (int i = 0; i < n; ++i) h.count[lengths[i]]++;
        if (h.count[0] == n) return true;
        int left = 1;
        for (int len = 1; len < 16; ++len) {
            left <<= 1;
            left -= h.count[len];
            if (left < 0) return false;
        }
        uint16_t offs[16];
        offs[1] = 0;
        for (int len = 1; len < 15; ++len) offs[len + 1] = offs[len] + h.count[len];
        for (int i = 0; i < n; ++i)
            if (lengths[i]) h.symbol[offs[lengths[i]]++] = (uint16_t)i;
        return true;
    }
    int decode(const Huff& h)
    {
        int code = 0, first = 0, index = 0;
        for (int len = 1; len < 16; ++len) {
            code |= bits(1);
            if (bad_) return -1;
            int count = h.count[len];
            if (code - count < first) return h.symbol[index + (code - first)];
            index += count;
            first += count;
            first <<= 1;
            code <<= 1;
        }
        return -1;
    }
    static void fixed(Huff& lit, Huff& dist)
    {
        uint8_t l[288];
        int i = 0;
        for (; i < 144; ++i) l[i] = 8;
        for (; i < 256; ++i) l[i] = 9;
        for (; i < 280; ++i) l[i] = 7;
        for (; i < 288; ++i) l[i] = 8;
        build(lit, l, 288);
        uint8_t d[30];
        for (i = 0; i < 30; ++i) d[i] = 5;
        build(dist, d, 30);
    }
    bool dynamic(Huff& lit, Huff& dist)
    {
        static const uint8_t order[19] = {16, 17, 18, 0, 8, 7, 9, 6, 10, 5, 11, 4, 12, 3, 13, 2, 14, 1, 15};
        int nlen = bits(5) + 257, ndist = bits(5) + 1, ncode = bits(4) + 4;
        if (bad_ || nlen > 286 || ndist > 30) return false;
        uint8_t lengths[320] = {};
        for (int i = 0; i < ncode; ++i) lengths[order[i]] = (uint8_t)bits(3);
        Huff lencode;
        if (!build(lencode, lengths, 19)) return false;
        int index = 0;
        while (index < nlen + ndist) {
            int sym = decode(lencode);
            if (sym < 0) return false;
            if (sym < 16) {
                lengths[index++] = (uint8_t)sym;
                continue;
            }
            int len = 0, rep;
            if (sym == 16) {
                if (index == 0) return false;
                len = lengths[index - 1];
                rep = 3 + bits(2);
            } else if (sym == 17) {
                rep = 3 + bits(3);
            } else {
                rep = 11 + bits(7);
            }
            if (bad_ || index + rep > nlen + ndist) return false;
            while (rep--) lengths[index++] = (uint8_t)len;
        }
        if (lengths[256] == 0) return false;
        return build(lit, lengths, nlen) && build(dist, lengths + nlen, ndist);
    }
    bool codes(std::vector<uint8_t>& out, const Huff& lit, const Huff& dist)
    {
        static const uint16_t lbase[29] = {3, 4, 5, 6, 7, 8, 9, 10, 11, 13, 15, 17, 19, 23, 27, 31,
                                           35, 43, 51, 59, 67, 83, 99, 115, 131, 163, 195, 227, 258};
        static const uint8_t lext[29] = {0, 0, 0, 0, 0, 0, 0, 0, 1, 1, 1, 1, 2, 2, 2, 2,
                                         3, 3, 3, 3, 4, 4, 4, 4, 5, 5, 5, 5, 0};
        static const uint16_t dbase[30] = {1, 2, 3, 4, 5, 7, 9, 13, 17, 25, 33, 49, 65, 97, 129,
                                           193, 257, 385, 513, 769, 1025, 1537, 2049, 3073, 4097,
                                           6145, 8193, 12289, 16385, 24577};
        static const uint8_t dext[30] = {0, 0, 0, 0, 1, 1, 2, 2, 3, 3, 4, 4, 5, 5, 6,
                                         6, 7, 7, 8, 8, 9, 9, 10, 10, 11, 11, 12, 12, 13, 13};
        for (;;) {
            int sym = decode(lit);
            if (sym < 0) return false;
            if (sym < 256) {
                out.push_back((uint8_t)sym);
            } else if (sym == 256) {
                return true;
            } else {
                sym -= 257;
                if (sym >= 29) return false;
                int len = lbase[sym] + bits(lext[sym]);
                int ds = decode(dist);
                if (ds < 0 || ds >= 30) return false;
                size_t d = dbase[ds] + (size_t)bits(dext[ds]);
                if (bad_ || d > out.size()) return false;
                size_t from = out.size() - d;
                for (int k = 0; k < len; ++k) out.push_back(out[from + k]);
            }
        }
    }
};

// ---------------------------------------------------------------------------
// PNG: 8-bit RGB / RGBA / grey / grey-alpha, not interlaced; returns the
// pixels row-major with `channels` bytes each.
inline uint32_t be32(const uint8_t* p) { return (uint32_t)p[0] << 24 | (uint32_t)p[1] << 16 | (uint32_t)p[2] << 8 | p[3]; }

inline bool decode_png(const uint8_t* d, size_t n, std::vector<uint8_t>& pixels, int& width, int& height,
                       int& channels, std::string& err)
{
    static const uint8_t sig[8] = {137, 80, 78, 71, 13, 10, 26, 10};
    if (n < 8 || std::memcmp(d, sig, 8) != 0) {
        err = "glb: image is not a PNG";
        return false;
    }
    size_t pos = 8;
    std::vector<uint8_t> idat;
    int depth = 0, ctype = -1, interlace = 0;
    width = height = 0;
    while (pos + 12 <= n) {
        uint32_t len = be32(d + pos);
        const uint8_t* type = d + pos + 4;
        const uint8_t* body = d + pos + 8;
        if (pos + 12 + (size_t)len > n) break;
        if (!std::memcmp(type, "IHDR", 4) && len >= 13) {
            width = (int)be32(body);
            height = (int)be32(body + 4);
            depth = body[8];
            ctype = body[9];
            interlace = body[12];
        } else if (!std::memcmp(type, "IDAT", 4)) {
            idat.insert(idat.end(), body, body + len);
        } else if (!std::memcmp(type, "IEND", 4)) {
            break;
        }
        pos += 12 + len;
    }
    channels = ctype == 2 ? 3 : ctype == 6 ? 4 : ctype == 0 ? 1 : ctype == 4 ? 2 : 0;
    if (width <= 0 || height <= 0 || depth != 8 || channels == 0 || interlace != 0) {
        err = "glb: only 8-bit, non-interlaced grey / RGB / RGBA PNG images are read";
        return false;
    }
    if (idat.size() < 6 || (idat[0] & 0x0f) != 8 || ((idat[0] << 8) | idat[1]) % 31 != 0) {
        err = "glb: PNG zlib stream header invalid";
        return false;
    }
    std::vector<uint8_t> raw;
    raw.reserve((size_t)height * (1 + (size_t)width * channels));
    Inflate inf(idat.data() + 2, idat.size() - 2);
    if (!inf.run(raw)) {
        err = "glb: PNG deflate stream invalid";
        return false;
    }
    const size_t stride = (size_t)width * channels;
    if (raw.size() < (size_t)height * (stride + 1)) {
        err = "glb: PNG image data too short";
        return false;
    }
    pixels.assign((size_t)height * stride, 0);
    const int bpp = channels;
    for (int y = 0; y < height; ++y) {
        const uint8_t f = raw[(size_t)y * (stride + 1)];
        const uint8_t* src = raw.data() + (size_t)y * (stride + 1) + 1;
        uint8_t* row = pixels.data() + (size_t)y * stride;
        const uint8_t* prev = y ? row - stride : nullptr;
        for (size_t x = 0; x < stride; ++x) {
            const int a = x >= (size_t)bpp ? row[x - bpp] : 0;
            const int b = prev ? prev[x] : 0;
            const int c = (prev && x >= (size_t)bpp) ? prev[x - bpp] : 0;
            int pr;
            switch (f) {
            case 0: pr = 0; break;
            case 1: pr = a; break;
            case 2: pr = b; break;
            case 3: pr = (a + b) >> 1; break;
            case 4: {  // Paeth
                const int p = a + b - c, pa = std::abs(p - a), pb = std::abs(p - b), pc = std::abs(p - c);
                pr = (pa <= pb && pa <= pc) ? a : (pb <= pc ? b : c);
                break;
            }
            default: err = "glb: PNG filter type invalid"; return false;
            }
            row[x] = (uint8_t)(src[x] + pr);
        }
    }
    return true;
}

// ---------------------------------------------------------------------------
// The document.
constexpr int kFloat = 5126, kUnsignedInt = 5125, kUnsignedShort = 5123, kUnsignedByte = 5121;

struct AccessorRef {
    int bufferView = -1;
    size_t byteOffset = 0;
    int componentType = 0;
};

struct Accessor {
    int bufferView = -1;
    size_t byteOffset = 0;
    int componentType = 0;
    size_t count = 0;
    std::string type;
    bool sparse = false;
    size_t sparseCount = 0;
    AccessorRef sparseIndices, sparseValues;
};

struct BufferView {
    int buffer = 0;
    size_t byteOffset = 0, byteLength = 0, byteStride = 0;
};

struct Primitive {
    std::map<std::string, int> attributes;
    int indices = -1, material = -1, mode = 4;
    std::vector<std::map<std::string, int>> targets;
};

struct Mesh {
    std::vector<Primitive> primitives;
    std::vector<double> weights;
};

struct Node {
    std::vector<double> matrix, rotation, scale, translation;
    int mesh = -1, light = -1;
    std::vector<int> children;
};

struct Material {
    std::vector<double> baseColorFactor{1.0, 1.0, 1.0, 1.0};
    double metallicFactor = 1.0, roughnessFactor = 1.0;
    int baseColorTexture = -1, normalTexture = -1;
};

struct Image {
    int width = 0, height = 0, component = 0;
    std::vector<uint8_t> pixels;
    std::string name;
};

struct Light {
    std::vector<double> color{1.0, 1.0, 1.0};
    double intensity = 1.0;
    std::string type;
};

struct AnimSampler {
    int input = -1, output = -1;
    std::string interpolation = "LINEAR";
};

struct AnimChannel {
    int sampler = -1, node = -1;
    std::string path;
};

struct Animation {
    std::vector<AnimSampler> samplers;
    std::vector<AnimChannel> channels;
};

struct Document {
    std::vector<std::vector<int>> scenes;  // root nodes of each scene
    std::vector<Node> nodes;
    std::vector<Mesh> meshes;
    std::vector<Accessor> accessors;
    std::vector<BufferView> bufferViews;
    std::vector<std::vector<uint8_t>> buffers;
    std::vector<Material> materials;
    std::vector<int> textures;  // image index of each texture
    std::vector<Image> images;
    std::vector<Light> lights;
    std::vector<Animation> animations;

    // Address of an accessor's (or sparse part's) first element; nullptr
    // when the view or the range is out of the buffers.
    const uint8_t* data(int bufferView, size_t byteOffset, size_t bytes) const
    {
        if (bufferView < 0 || bufferView >= (int)bufferViews.size()) return nullptr;
        const BufferView& v = bufferViews[bufferView];
        if (v.buffer < 0 || v.buffer >= (int)buffers.size()) return nullptr;
        const std::vector<uint8_t>& b = buffers[v.buffer];
        const size_t start = v.byteOffset + byteOffset;
        if (start + bytes > b.size() || byteOffset + bytes > v.byteLength) return nullptr;
        return b.data() + start;
    }
};

inline size_t component_count(const std::string& type)
{
    if (type == "SCALAR") return 1;
    if (type == "VEC2") return 2;
    if (type == "VEC3") return 3;
    if (type == "VEC4") return 4;
    if (type == "MAT4") return 16;
    return 0;
}

inline size_t component_size(int t)
{
    return t == kFloat || t == kUnsignedInt ? 4 : t == kUnsignedShort ? 2 : t == kUnsignedByte ? 1 : 0;
}

inline std::map<std::string, int> attribute_map(const Json* j)
{
    std::map<std::string, int> m;
    if (j && j->kind == Json::Object)
        for (const auto& kv : j->obj)
            if (kv.second.kind == Json::Number) m[kv.first] = (int)kv.second.num;
    return m;
}

inline bool parse_document(const uint8_t* bytes, size_t n, Document& doc, std::string& err)
{
    if (n < 20 || std::memcmp(bytes, "glTF", 4) != 0) {
        err = "glb: not a binary glTF file";
        return false;
    }
    auto le32 = [&](size_t o) {
        return (uint32_t)bytes[o] | (uint32_t)bytes[o + 1] << 8 | (uint32_t)bytes[o + 2] << 16 |
               (uint32_t)bytes[o + 3] << 24;
    };
    if (le32(4) != 2) {
        err = "glb: only glTF 2.0 is read";
        return false;
    }
    const size_t total = std::min<size_t>(le32(8), n);
    size_t pos = 12;
    const char* json = nullptr;
    size_t jsonLen = 0;
    std::vector<uint8_t> bin;
    bool haveBin = false;
    while (pos + 8 <= total) {
        const uint32_t len = le32(pos), type = le32(pos + 4);
        if (pos + 8 + (size_t)len > total) {
            err = "glb: chunk runs past the end of the file";
            return false;
        }
        if (type == 0x4E4F534Au && !json) {
            json = reinterpret_cast<const char*>(bytes + pos + 8);
            jsonLen = len;
        } else if (type == 0x004E4942u && !haveBin) {
            bin.assign(bytes + pos + 8, bytes + pos + 8 + len);
            haveBin = true;
        }
        pos += 8 + ((len + 3u) & ~3u);
    }
    if (!json) {
        err = "glb: no JSON chunk";
        return false;
    }
    Json root;
    JsonParser jp(json, jsonLen);
    if (!jp.parse(root, err)) return false;

    auto array = [&](const char* key) -> const std::vector<Json>* {
        const Json* j = root.get(key);
        return j && j->kind == Json::Array ? &j->arr : nullptr;
    };
    // buffers: the BIN chunk is buffer 0 (no uri); external uris are not read
    if (auto a = array("buffers"))
        for (size_t i = 0; i < a->size(); ++i) {
            if ((*a)[i].get("uri")) {
                err = "glb: external buffers are not read";
                return false;
            }
            doc.buffers.push_back(i == 0 ? bin : std::vector<uint8_t>());
        }
    if (auto a = array("bufferViews"))
        for (const Json& j : *a) {
            BufferView v;
            v.buffer = j.integer("buffer", 0);
            v.byteOffset = (size_t)j.number("byteOffset", 0);
            v.byteLength = (size_t)j.number("byteLength", 0);
            v.byteStride = (size_t)j.number("byteStride", 0);
            doc.bufferViews.push_back(v);
        }
    if (auto a = array("accessors"))
        for (const Json& j : *a) {
            Accessor x;
            x.bufferView = j.integer("bufferView", -1);
            x.byteOffset = (size_t)j.number("byteOffset", 0);
            x.componentType = j.integer("componentType", 0);
            x.count = (size_t)j.number("count", 0);
            x.type = j.string("type", "");
            if (const Json* s = j.get("sparse")) {
                x.sparse = true;
                x.sparseCount = (size_t)s->number("count", 0);
                if (const Json* si = s->get("indices")) {
                    x.sparseIndices.bufferView = si->integer("bufferView", -1);
                    x.sparseIndices.byteOffset = (size_t)si->number("byteOffset", 0);
                    x.sparseIndices.componentType = si->integer("componentType", 0);
                }
                if (const Json* sv = s->get("values")) {
                    x.sparseValues.bufferView = sv->integer("bufferView", -1);
                    x.sparseValues.byteOffset = (size_t)sv->number("byteOffset", 0);
                    x.sparseValues.componentType = x.componentType;
                }
            }
            doc.accessors.push_back(x);
        }
    if (auto a = array("meshes"))
        for (const Json& j : *a) {
            Mesh m;
            m.weights = j.numbers("weights");
            if (const Json* ps = j.get("primitives"); ps && ps->kind == Json::Array)
                for (const Json& pj : ps->arr) {
                    Primitive p;
                    p.attributes = attribute_map(pj.get("attributes"));
                    p.indices = pj.integer("indices", -1);
                    p.material = pj.integer("material", -1);
                    p.mode = pj.integer("mode", 4);
                    if (const Json* ts = pj.get("targets"); ts && ts->kind == Json::Array)
                        for (const Json& tj : ts->arr) p.targets.push_back(attribute_map(&tj));
                    m.primitives.push_back(std::move(p));
                }
            doc.meshes.push_back(std::move(m));
        }
    if (auto a = array("nodes"))
        for (const Json& j : *a) {
            Node nd;
            nd.matrix = j.numbers("matrix");
            nd.rotation = j.numbers("rotation");
            nd.scale = j.numbers("scale");
            nd.translation = j.numbers("translation");
            nd.mesh = j.integer("mesh", -1);
            for (double c : j.numbers("children")) nd.children.push_back((int)c);
            if (const Json* e = j.get("extensions"))
                if (const Json* l = e->get("KHR_lights_punctual")) nd.light = l->integer("light", -1);
            doc.nodes.push_back(std::move(nd));
        }
    if (auto a = array("scenes"))
        for (const Json& j : *a) {
            std::vector<int> roots;
            for (double c : j.numbers("nodes")) roots.push_back((int)c);
            doc.scenes.push_back(std::move(roots));
        }
    if (auto a = array("materials"))
        for (const Json& j : *a) {
            Material m;
            if (const Json* pbr = j.get("pbrMetallicRoughness")) {
                std::vector<double> f = pbr->numbers("baseColorFactor");
                if (f.size() == 4) m.baseColorFactor = f;
                m.metallicFactor = pbr->number("metallicFactor", 1.0);
                m.roughnessFactor = pbr->number("roughnessFactor", 1.0);
                if (const Json* t = pbr->get("baseColorTexture")) m.baseColorTexture = t->integer("index", -1);
            }
            if (const Json* t = j.get("normalTexture")) m.normalTexture = t->integer("index", -1);
            doc.materials.push_back(std::move(m));
        }
    if (auto a = array("textures"))
        for (const Json& j : *a) doc.textures.push_back(j.integer("source", -1));
    if (auto a = array("images"))
        for (const Json& j : *a) {
            Image im;
            im.name = j.string("name", "");
            const int view = j.integer("bufferView", -1);
            if (view < 0 || view >= (int)doc.bufferViews.size()) {
                err = "glb: images must be stored in the binary chunk";
                return false;
            }
            const uint8_t* p = doc.data(view, 0, doc.bufferViews[view].byteLength);
            if (!p || !decode_png(p, doc.bufferViews[view].byteLength, im.pixels, im.width, im.height, im.component,
                                  err))
                return false;
            doc.images.push_back(std::move(im));
        }
    if (const Json* ext = root.get("extensions"))
        if (const Json* lp = ext->get("KHR_lights_punctual"))
            if (const Json* ls = lp->get("lights"); ls && ls->kind == Json::Array)
                for (const Json& j : ls->arr) {
                    Light l;
                    std::vector<double> c = j.numbers("color");
                    if (c.size() == 3) l.color = c;
                    l.intensity = j.number("intensity", 1.0);
                    l.type = j.string("type", "point");
                    doc.lights.push_back(std::move(l));
                }
    if (auto a = array("animations"))
        for (const Json& j : *a) {
            Animation an;
            if (const Json* ss = j.get("samplers"); ss && ss->kind == Json::Array)
                for (const Json& sj : ss->arr) {
                    AnimSampler s;
                    s.input = sj.integer("input", -1);
                    s.output = sj.integer("output", -1);
                    s.interpolation = sj.string("interpolation", "LINEAR");
                    an.samplers.push_back(s);
                }
            if (const Json* cs = j.get("channels"); cs && cs->kind == Json::Array)
                for (const Json& cj : cs->arr) {
                    AnimChannel c;
                    c.sampler = cj.integer("sampler", -1);
                    if (const Json* t = cj.get("target")) {
                        c.node = t->integer("node", -1);
                        c.path = t->string("path", "");
                    }
                    an.channels.push_back(c);
                }
            doc.animations.push_back(std::move(an));
        }
    // every accessor a loader may dereference must lie inside its view
    for (const Accessor& x : doc.accessors) {
        const size_t elem = component_count(x.type) * component_size(x.componentType);
        if (x.bufferView >= 0 && x.count && (!elem || !doc.data(x.bufferView, x.byteOffset, elem * x.count))) {
            err = "glb: an accessor lies outside its buffer view";
            return false;
        }
        if (x.sparse) {
            const size_t ie = component_size(x.sparseIndices.componentType);
            if (!ie || !doc.data(x.sparseIndices.bufferView, x.sparseIndices.byteOffset, ie * x.sparseCount) ||
                !doc.data(x.sparseValues.bufferView, x.sparseValues.byteOffset, elem * x.sparseCount)) {
                err = "glb: a sparse accessor lies outside its buffer views";
                return false;
            }
        }
    }
    return true;
}

inline bool read_document(const char* path, Document& doc, std::string& err)
{
    FILE* f = std::fopen(path, "rb");
    if (!f) {
        err = std::string("glb: cannot open ") + path;
        return false;
    }
    std::vector<uint8_t> bytes;
    uint8_t buf[1 << 16];
    size_t r;
    while ((r = std::fread(buf, 1, sizeof buf, f)) > 0) bytes.insert(bytes.end(), buf, buf + r);
    std::fclose(f);
    return parse_document(bytes.data(), bytes.size(), doc, err);
}

}  // namespace glb
