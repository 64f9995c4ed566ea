// glTF 2.0 compound mesh assets: a JSON reader, the .glb container, buffers / buffer views /
// accessors, meshes and primitives, the node hierarchy and constant metallic-roughness
// materials, following the glTF 2.0 specification and the reference's use of it
// (CompoundMeshAsset::load_from_gltf, mesh_asset.cpp:551-1091).
#include "gltf.h"
#include "image_io.h"

#include <algorithm>
#include <array>
#include <cctype>
#include <cmath>
#include <cstring>
#include <fstream>
#include <utility>

namespace fs = std::filesystem;

namespace ksb
{
namespace gltf
{

namespace
{

// ---- JSON --------------------------------------------------------------------------------------
struct Json
{
    enum Kind
    {
        Null,
        Bool,
        Number,
        String,
        Array,
        Object
    } kind = Null;
    bool b = false;
    double num = 0.0;
    std::string str;
    std::vector<Json> arr;
    std::vector<std::pair<std::string, Json>> obj;

    const Json *get(const std::string &key) const
    {
        if (kind != Object)
            return nullptr;
        for (const auto &kv : obj)
            if (kv.first == key)
                return &kv.second;
        return nullptr;
    }
    double number(const std::string &key, double dflt) const
    {
        const Json *v = get(key);
        if (!v)
            return dflt;
        if (v->kind != Number)
            throw Error("glTF: '" + key + "' is not a number");
        return v->num;
    }
    long integer(const std::string &key, long dflt) const
    {
        const double d = number(key, (double)dflt);
        if (d != std::floor(d))
            throw Error("glTF: '" + key + "' is not an integer");
        return (long)d;
    }
    std::string string(const std::string &key, const std::string &dflt) const
    {
        const Json *v = get(key);
        if (!v)
            return dflt;
        if (v->kind != String)
            throw Error("glTF: '" + key + "' is not a string");
        return v->str;
    }
    const std::vector<Json> &array(const std::string &key) const
    {
        static const std::vector<Json> empty;
        const Json *v = get(key);
        if (!v)
            return empty;
        if (v->kind != Array)
            throw Error("glTF: '" + key + "' is not an array");
        return v->arr;
    }
    // numbers of an array member (empty when absent)
    std::vector<double> numbers(const std::string &key) const
    {
        std::vector<double> out;
        for (const Json &e : array(key)) {
            if (e.kind != Number)
                throw Error("glTF: '" + key + "' holds a non-number");
            out.push_back(e.num);
        }
        return out;
    }
};

struct JsonParser
{
    const char *p, *end;
    int depth = 0;

    [[noreturn]] void fail(const std::string &what) { throw Error("glTF: JSON " + what); }
    void ws()
    {
        while (p < end && (*p == ' ' || *p == '\t' || *p == '\n' || *p == '\r'))
            ++p;
    }
    bool lit(const char *s)
    {
        const size_t n = std::strlen(s);
        if ((size_t)(end - p) >= n && std::memcmp(p, s, n) == 0) {
            p += n;
            return true;
        }
        return false;
    }
    static void utf8(std::string &out, uint32_t cp)
    {
        if (cp < 0x80) {
            out += (char)cp;
        } else if (cp < 0x800) {
            out += (char)(0xc0 | (cp >> 6));
            out += (char)(0x80 | (cp & 0x3f));
        } else if (cp < 0x10000) {
            out += (char)(0xe0 | (cp >> 12));
            out += (char)(0x80 | ((cp >> 6) & 0x3f));
            out += (char)(0x80 | (cp & 0x3f));
        } else {
            out += (char)(0xf0 | (cp >> 18));
            out += (char)(0x80 | ((cp >> 12) & 0x3f));
            out += (char)(0x80 | ((cp >> 6) & 0x3f));
            out += (char)(0x80 | (cp & 0x3f));
        }
    }
    uint32_t hex4()
    {
        if (end - p < 4)
            fail("truncated \\u escape");
        uint32_t v = 0;
        for (int i = 0; i < 4; ++i) {
            const char c = *p++;
            v <<= 4;
            if (c >= '0' && c <= '9')
                v |= (uint32_t)(c - '0');
            else if (c >= 'a' && c <= 'f')
                v |= (uint32_t)(c - 'a' + 10);
            else if (c >= 'A' && c <= 'F')
                v |= (uint32_t)(c - 'A' + 10);
            else
                fail("bad \\u escape");
        }
        return v;
    }
    std::string string()
    {
        if (p >= end || *p != '"')
            fail("expected a string");
        ++p;
        std::string s;
        for (;;) {
            if (p >= end)
                fail("unterminated string");
            const char c = *p++;
            if (c == '"')
                return s;
            if (c != '\\') {
                s += c;
                continue;
            }
            if (p >= end)
                fail("unterminated escape");
            const char e = *p++;
            switch (e) {
            case '"':
            case '\\':
            case '/':
                s += e;
                break;
            case 'b':
                s += '\b';
                break;
            case 'f':
                s += '\f';
                break;
            case 'n':
                s += '\n';
                break;
            case 'r':
                s += '\r';
                break;
            case 't':
                s += '\t';
                break;
            case 'u': {
                uint32_t cp = hex4();
                if (cp >= 0xd800 && cp < 0xdc00 && end - p >= 6 && p[0] == '\\' && p[1] == 'u') {
                    p += 2;
                    const uint32_t lo = hex4();
                    if (lo >= 0xdc00 && lo < 0xe000)
                        cp = 0x10000 + ((cp - 0xd800) << 10) + (lo - 0xdc00);
                }
                utf8(s, cp);
                break;
            }
            default:
                fail("bad escape");
            }
        }
    }
    Json value()
    {
        if (++depth > 256)
            fail("nested too deeply");
        ws();
        if (p >= end)
            fail("unexpected end");
        Json v;
        if (*p == '{') {
            ++p;
            v.kind = Json::Object;
            ws();
            if (p < end && *p == '}') {
                ++p;
            } else {
                for (;;) {
                    ws();
                    std::string k = string();
                    ws();
                    if (p >= end || *p != ':')
                        fail("expected ':'");
                    ++p;
                    v.obj.emplace_back(std::move(k), value());
                    ws();
                    if (p < end && *p == ',') {
                        ++p;
                        continue;
                    }
                    if (p < end && *p == '}') {
                        ++p;
                        break;
                    }
                    fail("expected ',' or '}'");
                }
            }
        } else if (*p == '[') {
            ++p;
            v.kind = Json::Array;
            ws();
            if (p < end && *p == ']') {
                ++p;
            } else {
                for (;;) {
                    v.arr.push_back(value());
                    ws();
                    if (p < end && *p == ',') {
                        ++p;
                        continue;
                    }
                    if (p < end && *p == ']') {
                        ++p;
                        break;
                    }
                    fail("expected ',' or ']'");
                }
            }
        } else if (*p == '"') {
            v.kind = Json::String;
            v.str = string();
        } else if (lit("true")) {
            v.kind = Json::Bool;
            v.b = true;
        } else if (lit("false")) {
            v.kind = Json::Bool;
        } else if (lit("null")) {
            v.kind = Json::Null;
        } else {
            const std::string tok(p, (size_t)std::min<ptrdiff_t>(end - p, 64));
            char *stop = nullptr;
            v.num = std::strtod(tok.c_str(), &stop);
            if (stop == tok.c_str())
                fail("unexpected character");
            v.kind = Json::Number;
            p += stop - tok.c_str();
        }
        --depth;
        return v;
    }
};

Json parse_json(const std::string &text)
{
    JsonParser jp{text.data(), text.data() + text.size()};
    Json v = jp.value();
    jp.ws();
    if (jp.p != jp.end)
        jp.fail("trailing characters");
    return v;
}

// ---- files and buffers -------------------------------------------------------------------------
std::string read_all(const fs::path &path)
{
    std::ifstream f(path, std::ios::binary);
    if (!f)
        throw Error("cannot open " + path.string());
    return std::string((std::istreambuf_iterator<char>(f)), std::istreambuf_iterator<char>());
}

std::string base64_decode(const std::string &s, size_t from)
{
    auto val = [](char c) -> int {
        if (c >= 'A' && c <= 'Z')
            return c - 'A';
        if (c >= 'a' && c <= 'z')
            return c - 'a' + 26;
        if (c >= '0' && c <= '9')
            return c - '0' + 52;
        if (c == '+' || c == '-')
            return 62;
        if (c == '/' || c == '_')
            return 63;
        return -1;
    };
    std::string out;
    uint32_t acc = 0;
    int bits = 0;
    for (size_t i = from; i < s.size(); ++i) {
        const char c = s[i];
        if (c == '=')
            break;
        const int v = val(c);
        if (v < 0)
            throw Error("glTF: bad base64 data URI");
        acc = (acc << 6) | (uint32_t)v;
        bits += 6;
        if (bits >= 8) {
            bits -= 8;
            out += (char)((acc >> bits) & 0xff);
        }
    }
    return out;
}

std::string uri_decode(const std::string &u)
{
    std::string out;
    for (size_t i = 0; i < u.size(); ++i) {
        if (u[i] == '%' && i + 2 < u.size() && std::isxdigit((unsigned char)u[i + 1]) &&
            std::isxdigit((unsigned char)u[i + 2])) {
            out += (char)std::stoi(u.substr(i + 1, 2), nullptr, 16);
            i += 2;
        } else {
            out += u[i];
        }
    }
    return out;
}

uint32_t le32(const std::string &s, size_t at)
{
    uint32_t v;
    std::memcpy(&v, s.data() + at, 4);
    return v;
}

struct Model
{
    Json doc;
    std::vector<std::string> buffers;
};

Model load_model(const fs::path &path)
{
    Model m;
    const std::string file = read_all(path);
    std::string glb_bin;
    bool have_bin = false;
    if (file.size() >= 12 && le32(file, 0) == 0x46546c67u) { // "glTF": binary container
        if (le32(file, 4) != 2)
            throw Error(path.string() + ": glb version " + std::to_string(le32(file, 4)) + " is not supported", true);
        const size_t length = std::min<size_t>(le32(file, 8), file.size());
        size_t at = 12;
        bool have_json = false;
        while (at + 8 <= length) {
            const uint32_t n = le32(file, at), type = le32(file, at + 4);
            if (at + 8 + (size_t)n > length)
                throw Error(path.string() + ": truncated glb chunk");
            if (type == 0x4e4f534au && !have_json) { // JSON
                m.doc = parse_json(file.substr(at + 8, n));
                have_json = true;
            } else if (type == 0x004e4942u && !have_bin) { // BIN
                glb_bin = file.substr(at + 8, n);
                have_bin = true;
            }
            at += 8 + (size_t)((n + 3) & ~3u);
        }
        if (!have_json)
            throw Error(path.string() + ": glb without a JSON chunk");
    } else {
        m.doc = parse_json(file);
    }
    if (m.doc.kind != Json::Object)
        throw Error(path.string() + ": not a glTF document");
    const Json *asset = m.doc.get("asset");
    const std::string version = asset ? asset->string("version", "") : "";
    if (version.empty() || version[0] != '2')
        throw Error(path.string() + ": glTF version '" + version + "' is not supported (2.x)", true);
    const auto &bufs = m.doc.array("buffers");
    for (size_t i = 0; i < bufs.size(); ++i) {
        const Json &b = bufs[i];
        const size_t len = (size_t)b.integer("byteLength", 0);
        std::string data;
        const Json *uri = b.get("uri");
        if (!uri) {
            if (i != 0 || !have_bin)
                throw Error(path.string() + ": buffer " + std::to_string(i) + " has no data");
            data = glb_bin;
        } else {
            const std::string u = b.string("uri", "");
            if (u.rfind("data:", 0) == 0) {
                const size_t comma = u.find(',');
                if (comma == std::string::npos || u.substr(0, comma).find(";base64") == std::string::npos)
                    throw Error(path.string() + ": only base64 data URIs are supported", true);
                data = base64_decode(u, comma + 1);
            } else {
                data = read_all(path.parent_path() / uri_decode(u));
            }
        }
        if (data.size() < len)
            throw Error(path.string() + ": buffer " + std::to_string(i) + " is shorter than its byteLength");
        m.buffers.push_back(std::move(data));
    }
    return m;
}

// ---- accessors ---------------------------------------------------------------------------------
int component_bytes(long type)
{
    switch (type) {
    case 5120:
    case 5121:
        return 1;
    case 5122:
    case 5123:
        return 2;
    case 5125:
    case 5126:
        return 4;
    default:
        throw Error("glTF: unknown accessor componentType " + std::to_string(type));
    }
}

int type_components(const std::string &t)
{
    if (t == "SCALAR")
        return 1;
    if (t == "VEC2")
        return 2;
    if (t == "VEC3")
        return 3;
    if (t == "VEC4" || t == "MAT2")
        return 4;
    if (t == "MAT3")
        return 9;
    if (t == "MAT4")
        return 16;
    throw Error("glTF: unknown accessor type '" + t + "'");
}

// copy_accessor_to_linear (mesh_asset.cpp:312-329): the accessor's elements, packed.  An
// accessor without a buffer view is all zeros (glTF 2.0, 3.6.2.3).
std::string accessor_bytes(const Model &m, long index, long want_component, const std::string &want_type,
                           size_t &count)
{
    const auto &accs = m.doc.array("accessors");
    if (index < 0 || index >= (long)accs.size())
        throw Error("glTF: accessor index out of range");
    const Json &a = accs[(size_t)index];
    if (a.get("sparse"))
        throw Error("glTF: sparse accessors are not supported", true);
    const long ct = a.integer("componentType", -1);
    const std::string type = a.string("type", "");
    if (ct != want_component || type != want_type)
        throw Error("glTF: accessor " + std::to_string(index) + " is not of component type " +
                        std::to_string(want_component) + " and type " + want_type,
                    true);
    const long cnt = a.integer("count", -1);
    if (cnt < 0)
        throw Error("glTF: accessor without a count");
    count = (size_t)cnt;
    const size_t elem = (size_t)component_bytes(ct) * (size_t)type_components(type);
    std::string out(count * elem, '\0');
    if (!a.get("bufferView"))
        return out;
    const auto &views = m.doc.array("bufferViews");
    const long vi = a.integer("bufferView", -1);
    if (vi < 0 || vi >= (long)views.size())
        throw Error("glTF: buffer view index out of range");
    const Json &v = views[(size_t)vi];
    const long bi = v.integer("buffer", -1);
    if (bi < 0 || bi >= (long)m.buffers.size())
        throw Error("glTF: buffer index out of range");
    const std::string &buf = m.buffers[(size_t)bi];
    const size_t view_off = (size_t)v.integer("byteOffset", 0), view_len = (size_t)v.integer("byteLength", 0);
    const size_t stride = v.get("byteStride") ? (size_t)v.integer("byteStride", 0) : elem;
    const size_t off = (size_t)a.integer("byteOffset", 0);
    if (view_off + view_len > buf.size() || stride < elem ||
        (count > 0 && off + stride * (count - 1) + elem > view_len))
        throw Error("glTF: accessor " + std::to_string(index) + " reaches past its buffer view");
    for (size_t i = 0; i < count; ++i)
        std::memcpy(&out[i * elem], buf.data() + view_off + off + i * stride, elem);
    return out;
}

std::vector<float> floats(const Model &m, long index, const std::string &type, size_t &count)
{
    const std::string b = accessor_bytes(m, index, 5126, type, count);
    std::vector<float> out(b.size() / 4);
    std::memcpy(out.data(), b.data(), b.size());
    return out;
}

std::vector<uint32_t> indices(const Model &m, long index)
{
    const auto &accs = m.doc.array("accessors");
    if (index < 0 || index >= (long)accs.size())
        throw Error("glTF: primitive without indices (non-indexed primitives are not supported)", true);
    const long ct = accs[(size_t)index].integer("componentType", -1);
    if (ct != 5125 && ct != 5123)
        throw Error("glTF: index component type " + std::to_string(ct) + " is not supported", true);
    size_t count = 0;
    const std::string b = accessor_bytes(m, index, ct, "SCALAR", count);
    std::vector<uint32_t> out(count);
    for (size_t i = 0; i < count; ++i) {
        if (ct == 5125) {
            std::memcpy(&out[i], &b[4 * i], 4);
        } else {
            uint16_t s;
            std::memcpy(&s, &b[2 * i], 2);
            out[i] = s;
        }
    }
    if (count % 3)
        throw Error("glTF: index count is not a multiple of 3");
    return out;
}

// ---- materials ---------------------------------------------------------------------------------
// Textures of the document's images, decoded once each when a material first binds them
// (create_texture_from_gltf, mesh_asset.cpp:370-388): tinygltf's default loading forces four
// channels, keeps 16-bit PNGs at 16 bits (u16) and gives 8-bit images as u8; an image is sRGB when
// any material of the document uses it as a base colour or emissive texture
// (mesh_asset.cpp:566-582).
struct TextureSet
{
    const Model &m;
    const fs::path &path;
    std::vector<Texture> &out;
    std::vector<long> slot;   // glTF image -> index into `out`, -1 before its first use
    std::vector<int> srgb;    // per glTF image
};

long texture_image(TextureSet &ts, long tex_index, const std::string &where)
{
    const auto &texs = ts.m.doc.array("textures");
    if (tex_index < 0 || tex_index >= (long)texs.size())
        throw Error(where + ": texture index out of range");
    const long img = texs[(size_t)tex_index].integer("source", -1);
    const auto &imgs = ts.m.doc.array("images");
    if (img < 0 || img >= (long)imgs.size())
        throw Error(where + ": texture without a valid image source", true);
    if (ts.slot[(size_t)img] >= 0)
        return ts.slot[(size_t)img];
    const Json &im = imgs[(size_t)img];
    std::string bytes;
    if (const Json *bv = im.get("bufferView")) {
        if (bv->kind != Json::Number)
            throw Error(where + ": bad image bufferView");
        const auto &views = ts.m.doc.array("bufferViews");
        const long vi = (long)bv->num;
        if (vi < 0 || vi >= (long)views.size())
            throw Error(where + ": image bufferView out of range");
        const Json &v = views[(size_t)vi];
        const long bi = v.integer("buffer", -1);
        const size_t off = (size_t)v.integer("byteOffset", 0), len = (size_t)v.integer("byteLength", 0);
        if (bi < 0 || bi >= (long)ts.m.buffers.size() || off + len > ts.m.buffers[(size_t)bi].size())
            throw Error(where + ": image bufferView outside its buffer");
        bytes = ts.m.buffers[(size_t)bi].substr(off, len);
    } else {
        const std::string u = im.string("uri", "");
        if (u.empty())
            throw Error(where + ": image without a uri or bufferView");
        if (u.rfind("data:", 0) == 0) {
            const size_t comma = u.find(',');
            if (comma == std::string::npos || u.substr(0, comma).find(";base64") == std::string::npos)
                throw Error(where + ": only base64 data URIs are supported", true);
            bytes = base64_decode(u, comma + 1);
        } else {
            bytes = read_all(ts.path.parent_path() / uri_decode(u));
        }
    }
    static const uint8_t png_sig[4] = {137, 'P', 'N', 'G'};
    if (bytes.size() < 8 || std::memcmp(bytes.data(), png_sig, 4) != 0)
        throw Error(where + ": image " + std::to_string(img) + " is not a PNG (JPEG and other image formats are "
                                                                "not supported)",
                    true);
    image::Png png;
    try {
        png = image::read_png((const uint8_t *)bytes.data(), bytes.size(), where + ": image " + std::to_string(img));
    } catch (const image::Error &e) {
        throw Error(e.what(), e.unsupported);
    }
    Texture t;
    t.width = png.width;
    t.height = png.height;
    t.channels = 4;
    t.srgb = ts.srgb[(size_t)img] != 0;
    const std::vector<uint16_t> s = image::convert_channels(png, 4, png.depth);
    if (png.depth == 16) {
        t.format = 1;
        t.bytes.resize(s.size() * 2);
        std::memcpy(t.bytes.data(), s.data(), t.bytes.size());
    } else {
        t.format = 0;
        t.bytes.resize(s.size());
        for (size_t k = 0; k < s.size(); ++k)
            t.bytes[k] = (uint8_t)s[k];
    }
    ts.slot[(size_t)img] = (long)ts.out.size();
    ts.out.push_back(std::move(t));
    return ts.slot[(size_t)img];
}

// A texture-info object bound to `field` (create_texture_shader_field, mesh_asset.cpp:446-464):
// the glTF sampler's minification filter picks EWA for the mipmap filters and nearest otherwise; no
// v flip; KHR_texture_transform's scale and offset (get_texture_transform, :390-444); the glTF
// sampler's wrap modes are not read (repeat).  EWA filtering reads the camera ray's differentials
// on mipmapped textures, which this build does not have: such bindings are unsupported.  A texture
// without a sampler is read with the nearest filter.
ks_texture_binding texture_binding(TextureSet &ts, const Json &info, uint32_t material, int32_t field,
                                   const float scale[4], const int32_t swizzle[4], const std::string &where)
{
    ks_texture_binding b{};
    b.material = material;
    b.field = field;
    const long ti = info.integer("index", -1);
    b.texture = (uint32_t)texture_image(ts, ti, where);
    const long si = ts.m.doc.array("textures")[(size_t)ti].integer("sampler", -1);
    if (si >= 0) {
        const auto &samplers = ts.m.doc.array("samplers");
        if (si >= (long)samplers.size())
            throw Error(where + ": sampler index out of range");
        const long mf = samplers[(size_t)si].integer("minFilter", -1);
        if (mf >= 9984 && mf <= 9987)
            throw Error(where + ": textures with a mipmap minification filter (EWA filtering of mipmapped textures) "
                                "are not supported",
                        true);
    }
    b.filter = 0;
    b.flip_v = 0;
    for (int c = 0; c < 4; ++c) {
        b.swizzle[c] = swizzle[c];
        b.scale[c] = scale[c];
    }
    b.uv_scale[0] = b.uv_scale[1] = 1.0f;
    if (const Json *ext = info.get("extensions"))
        if (const Json *tt = ext->get("KHR_texture_transform")) {
            const std::vector<double> sc = tt->numbers("scale"), of = tt->numbers("offset");
            for (size_t k = 0; k < 2 && k < sc.size(); ++k)
                b.uv_scale[k] = (float)sc[k];
            for (size_t k = 0; k < 2 && k < of.size(); ++k)
                b.uv_offset[k] = (float)of[k];
        }
    b.normal_space = 0;
    b.range01 = 1;
    b.strength = 1.0f;
    for (int k = 0; k < 4; ++k)
        b.to_world[5 * k] = 1.0f;
    return b;
}

// The metallic-roughness material as a principled BSDF (mesh_asset.cpp:672-940): basecolor,
// roughness, metallic; emissive = KHR_materials_emissive_strength x emissiveFactor, an emitter when
// both are positive; ior (KHR_materials_ior, 1.5); specular_r0_mul (KHR_materials_specular:
// specularFactor x mean(specularColorFactor), 0.5 without it); specular_trans
// (KHR_materials_transmission, which also makes the mesh one-sided); no diffuse transmission; GGX.
// Textures (with TextureSet): baseColorTexture x baseColorFactor, metallicRoughnessTexture's G x
// roughnessFactor and B x metallicFactor, specularTexture x the specular factor,
// transmissionTexture x transmissionFactor, normalTexture as a tangent-space normal map of strength
// normalTexture.scale, for alpha modes other than OPAQUE an opacity map of the base colour
// texture's alpha x baseColorFactor[3] (the constant factor without a texture), and an emitter's
// emissiveTexture x strength x emissiveFactor as its emission.
ks_material_desc material(const Json &src, const std::string &where, bool &twosided, TextureSet *ts,
                          uint32_t index, std::vector<ks_texture_binding> &binds)
{
    ks_material_desc d{};
    const Json *pbr = src.get("pbrMetallicRoughness");
    const Json *ext = src.get("extensions");
    auto extension = [&](const char *name) { return ext ? ext->get(name) : nullptr; };
    const Json *bct = pbr ? pbr->get("baseColorTexture") : nullptr;
    const Json *mrt = pbr ? pbr->get("metallicRoughnessTexture") : nullptr;
    std::vector<double> bc = pbr ? pbr->numbers("baseColorFactor") : std::vector<double>{};
    if (bc.empty())
        bc = {1.0, 1.0, 1.0, 1.0};
    if (bc.size() != 4)
        throw Error(where + ": baseColorFactor needs 4 numbers");
    for (int c = 0; c < 3; ++c)
        d.basecolor[c] = (float)bc[c];
    d.roughness = pbr ? (float)pbr->number("roughnessFactor", 1.0) : 1.0f;
    d.metallic = pbr ? (float)pbr->number("metallicFactor", 1.0) : 1.0f;
    float strength = 1.0f;
    if (const Json *e = extension("KHR_materials_emissive_strength"))
        strength = (float)e->number("emissiveStrength", 1.0);
    std::vector<double> ef = src.numbers("emissiveFactor");
    if (ef.empty())
        ef = {0.0, 0.0, 0.0};
    if (ef.size() != 3)
        throw Error(where + ": emissiveFactor needs 3 numbers");
    for (int c = 0; c < 3; ++c)
        d.emissive[c] = strength * (float)ef[c];
    if (strength > 0.0f && (ef[0] > 0.0 || ef[1] > 0.0 || ef[2] > 0.0)) {
        d.has_emission = 1;
        for (int c = 0; c < 3; ++c)
            d.emission[c] = d.emissive[c];
    }
    d.ior = 1.5f;
    if (const Json *e = extension("KHR_materials_ior"))
        d.ior = (float)e->number("ior", 1.5);
    d.specular_r0_mul = 0.5f;
    const Json *spec_tex = nullptr, *trans_tex = nullptr;
    if (const Json *e = extension("KHR_materials_specular")) {
        const std::vector<double> scf = e->numbers("specularColorFactor");
        float sf = 0.5f;
        if (e->get("specularFactor") || !scf.empty()) {
            sf = (float)e->number("specularFactor", 1.0);
            if (scf.size() == 3)
                sf *= (float)((scf[0] + scf[1] + scf[2]) / 3.0);
        }
        d.specular_r0_mul = sf;
        spec_tex = e->get("specularTexture");
    }
    float trans = 0.0f;
    if (const Json *e = extension("KHR_materials_transmission")) {
        twosided = false;
        trans = (float)e->number("transmissionFactor", 0.0);
        d.specular_trans = trans;
        trans_tex = e->get("transmissionTexture");
    }
    d.diffuse_trans = 0.0f;
    d.diffuse_trans_fwd = 0.0f;
    d.microfacet = 0;
    const bool alpha = src.string("alphaMode", "OPAQUE") != "OPAQUE";
    const Json *nt = src.get("normalTexture");
    if (!ts) {
        if (bct || mrt || nt || spec_tex || trans_tex || (d.has_emission && src.get("emissiveTexture")))
            throw Error(where + ": textured materials are not supported (constant fields only)", true);
        if (alpha)
            throw Error(where + ": alpha modes other than OPAQUE (opacity maps) are not supported", true);
        return d;
    }
    const int32_t id4[4] = {0, 1, 2, 3};
    const float one4[4] = {1, 1, 1, 1};
    if (bct) {
        const float sc[4] = {(float)bc[0], (float)bc[1], (float)bc[2], 1.0f};
        binds.push_back(texture_binding(*ts, *bct, index, KS_FIELD_BASECOLOR, sc, id4, where));
        if (alpha) {
            const float sa[4] = {(float)bc[3], 1, 1, 1};
            const int32_t sw[4] = {3, -1, -1, -1};
            binds.push_back(texture_binding(*ts, *bct, index, KS_FIELD_OPACITY_MAP, sa, sw, where));
        }
    } else if (alpha) {
        // the constant opacity baseColorFactor[3]: a one-texel texture of 1 scaled by it
        Texture t;
        t.width = t.height = t.channels = 1;
        t.format = 2;
        t.srgb = false;
        const float v = 1.0f;
        t.bytes.resize(4);
        std::memcpy(t.bytes.data(), &v, 4);
        ks_texture_binding b{};
        b.material = index;
        b.field = KS_FIELD_OPACITY_MAP;
        b.texture = (uint32_t)ts->out.size();
        ts->out.push_back(std::move(t));
        b.swizzle[0] = 0;
        b.swizzle[1] = b.swizzle[2] = b.swizzle[3] = -1;
        b.scale[0] = (float)bc[3];
        b.scale[1] = b.scale[2] = b.scale[3] = 1.0f;
        b.uv_scale[0] = b.uv_scale[1] = 1.0f;
        b.range01 = 1;
        b.strength = 1.0f;
        for (int k = 0; k < 4; ++k)
            b.to_world[5 * k] = 1.0f;
        binds.push_back(b);
    }
    if (mrt) {
        const float sr[4] = {d.roughness, 1, 1, 1}, sm[4] = {d.metallic, 1, 1, 1};
        const int32_t g[4] = {1, -1, -1, -1}, bl[4] = {2, -1, -1, -1};
        binds.push_back(texture_binding(*ts, *mrt, index, KS_FIELD_ROUGHNESS, sr, g, where));
        binds.push_back(texture_binding(*ts, *mrt, index, KS_FIELD_METALLIC, sm, bl, where));
    }
    if (spec_tex) {
        const float ss[4] = {d.specular_r0_mul, 1, 1, 1};
        binds.push_back(texture_binding(*ts, *spec_tex, index, KS_FIELD_SPECULAR_R0_MUL, ss, id4, where));
    }
    if (trans_tex) {
        const float st[4] = {trans, 1, 1, 1};
        binds.push_back(texture_binding(*ts, *trans_tex, index, KS_FIELD_SPECULAR_TRANS, st, id4, where));
    }
    if (nt) {
        ks_texture_binding b = texture_binding(*ts, *nt, index, KS_FIELD_NORMAL_MAP, one4, id4, where);
        b.strength = (float)nt->number("scale", 1.0);
        binds.push_back(b);
    }
    // an emitter's emissive texture x (emissive strength x emissiveFactor), sRGB
    if (const Json *et = src.get("emissiveTexture"); et && d.has_emission) {
        const float se[4] = {d.emissive[0], d.emissive[1], d.emissive[2], 1.0f};
        binds.push_back(texture_binding(*ts, *et, index, KS_FIELD_EMISSION, se, id4, where));
    }
    return d;
}

// ---- node transforms ---------------------------------------------------------------------------
using Mat4 = std::array<double, 16>; // row-major

Mat4 mul(const Mat4 &a, const Mat4 &b)
{
    Mat4 c{};
    for (int r = 0; r < 4; ++r)
        for (int k = 0; k < 4; ++k)
            for (int j = 0; j < 4; ++j)
                c[4 * r + j] += a[4 * r + k] * b[4 * k + j];
    return c;
}

// A node's local transform: its column-major `matrix`, else T * R * S of its translation,
// rotation (x, y, z, w) and scale (traverse_gltf_scene_graph, mesh_asset.cpp:466-498).
Mat4 local_transform(const Json &node)
{
    const std::vector<double> mat = node.numbers("matrix");
    Mat4 m{};
    if (!mat.empty()) {
        if (mat.size() != 16)
            throw Error("glTF: node matrix needs 16 numbers");
        for (int r = 0; r < 4; ++r)
            for (int c = 0; c < 4; ++c)
                m[4 * r + c] = mat[4 * c + r];
        return m;
    }
    std::vector<double> s = node.numbers("scale"), q = node.numbers("rotation"), t = node.numbers("translation");
    if (s.empty())
        s = {1, 1, 1};
    if (q.empty())
        q = {0, 0, 0, 1};
    if (t.empty())
        t = {0, 0, 0};
    if (s.size() != 3 || q.size() != 4 || t.size() != 3)
        throw Error("glTF: bad node scale / rotation / translation");
    // rotation matrix of the quaternion (taken as given, like Eigen's toRotationMatrix)
    const double x = q[0], y = q[1], z = q[2], w = q[3];
    const double R[9] = {1 - 2 * (y * y + z * z), 2 * (x * y - w * z),     2 * (x * z + w * y),
                         2 * (x * y + w * z),     1 - 2 * (x * x + z * z), 2 * (y * z - w * x),
                         2 * (x * z - w * y),     2 * (y * z + w * x),     1 - 2 * (x * x + y * y)};
    for (int r = 0; r < 3; ++r) {
        for (int c = 0; c < 3; ++c)
            m[4 * r + c] = R[3 * r + c] * s[c];
        m[4 * r + 3] = t[r];
    }
    m[15] = 1.0;
    return m;
}

} // namespace

Compound load(const fs::path &path, bool load_materials, bool load_textures)
{
    Model m = load_model(path);
    Compound out;
    const auto &meshes = m.doc.array("meshes");
    const auto &mats = m.doc.array("materials");
    TextureSet ts{m, path, out.textures, std::vector<long>(m.doc.array("images").size(), -1),
                  std::vector<int>(m.doc.array("images").size(), 0)};
    for (const Json &mat : mats) {
        auto mark = [&](const Json *info) {
            if (!info)
                return;
            const long ti = info->integer("index", -1);
            const auto &texs = m.doc.array("textures");
            if (ti >= 0 && ti < (long)texs.size()) {
                const long img = texs[(size_t)ti].integer("source", -1);
                if (img >= 0 && img < (long)ts.srgb.size())
                    ts.srgb[(size_t)img] = 1;
            }
        };
        const Json *pbr = mat.get("pbrMetallicRoughness");
        mark(pbr ? pbr->get("baseColorTexture") : nullptr);
        mark(mat.get("emissiveTexture"));
    }
    for (size_t i = 0; i < meshes.size(); ++i) {
        Prototype proto;
        const auto &prims = meshes[i].array("primitives");
        for (size_t j = 0; j < prims.size(); ++j) {
            const Json &pr = prims[j];
            const std::string where = path.string() + ": mesh " + std::to_string(i) + " primitive " + std::to_string(j);
            if (pr.integer("mode", 4) != 4)
                throw Error(where + ": only triangle primitives are supported", true);
            const Json *attrs = pr.get("attributes");
            if (!attrs || !attrs->get("POSITION"))
                throw Error(where + ": primitive without positions");
            mesh::MeshData md;
            size_t nv = 0, n = 0;
            md.vertices = floats(m, attrs->integer("POSITION", -1), "VEC3", nv);
            md.indices = indices(m, pr.integer("indices", -1));
            for (uint32_t k : md.indices)
                if (k >= nv)
                    throw Error(where + ": vertex index out of range");
            if (attrs->get("NORMAL")) {
                md.normals = floats(m, attrs->integer("NORMAL", -1), "VEC3", n);
                if (n != nv)
                    throw Error(where + ": NORMAL count differs from POSITION count");
            }
            if (attrs->get("TEXCOORD_0")) {
                md.texcoords = floats(m, attrs->integer("TEXCOORD_0", -1), "VEC2", n);
                if (n != nv)
                    throw Error(where + ": TEXCOORD_0 count differs from POSITION count");
            }
            md.twosided = true;
            md.use_smooth_normal = true;
            md.name = meshes[i].string("name", "");
            if (load_materials) {
                const long mi = pr.integer("material", -1);
                if (mi < 0 || mi >= (long)mats.size())
                    throw Error(where + ": primitive without a material", true);
                proto.materials.push_back(material(mats[(size_t)mi], where, md.twosided,
                                                   load_textures ? &ts : nullptr, (uint32_t)j, proto.bindings));
            }
            proto.meshes.push_back(std::move(md));
        }
        if (proto.meshes.empty())
            throw Error(path.string() + ": mesh " + std::to_string(i) + " has no primitives");
        out.prototypes.push_back(std::move(proto));
    }
    // the default scene's node trees, depth first, world = parent x local
    const auto &nodes = m.doc.array("nodes");
    const auto &scenes = m.doc.array("scenes");
    if (scenes.empty())
        return out;
    const long si = m.doc.integer("scene", 0);
    if (si < 0 || si >= (long)scenes.size())
        throw Error(path.string() + ": scene index out of range");
    std::vector<int> on_path(nodes.size(), 0);
    auto dfs = [&](long ni, const Mat4 &parent, auto &self) -> void {
        if (ni < 0 || ni >= (long)nodes.size())
            throw Error(path.string() + ": node index out of range");
        if (on_path[(size_t)ni])
            throw Error(path.string() + ": the node graph has a cycle");
        on_path[(size_t)ni] = 1;
        const Json &node = nodes[(size_t)ni];
        const Mat4 world = mul(parent, local_transform(node));
        if (node.get("mesh")) {
            const long mi = node.integer("mesh", -1);
            if (mi < 0 || mi >= (long)out.prototypes.size())
                throw Error(path.string() + ": node mesh index out of range");
            Instance inst;
            inst.prototype = (uint32_t)mi;
            for (int r = 0; r < 3; ++r)
                for (int c = 0; c < 4; ++c)
                    inst.to_world[4 * r + c] = (float)world[4 * r + c];
            out.instances.push_back(inst);
        }
        for (const Json &c : node.array("children")) {
            if (c.kind != Json::Number)
                throw Error(path.string() + ": bad child index");
            self((long)c.num, world, self);
        }
        on_path[(size_t)ni] = 0;
    };
    Mat4 id{};
    id[0] = id[5] = id[10] = id[15] = 1.0;
    for (const Json &root : scenes[(size_t)si].array("nodes")) {
        if (root.kind != Json::Number)
            throw Error(path.string() + ": bad scene node index");
        dfs((long)root.num, id, dfs);
    }
    return out;
}

} // namespace gltf
} // namespace ksb

namespace ksb
{
namespace gltf
{

namespace
{

// Shortest-arc spherical interpolation of unit quaternions (x, y, z, w) (Shoemake), with the
// linear blend near parallel quaternions, as Eigen's QuaternionBase::slerp does it.
void slerp(const float *a, const float *b, float t, float *out)
{
    const float d = a[0] * b[0] + a[1] * b[1] + a[2] * b[2] + a[3] * b[3];
    const float ad = std::fabs(d);
    float s0, s1;
    if (ad >= 1.0f - 1e-5f) {
        s0 = 1.0f - t;
        s1 = t;
    } else {
        const float theta = std::acos(ad), st = std::sin(theta);
        s0 = std::sin((1.0f - t) * theta) / st;
        s1 = std::sin(t * theta) / st;
    }
    if (d < 0.0f)
        s1 = -s1;
    for (int k = 0; k < 4; ++k)
        out[k] = s0 * a[k] + s1 * b[k];
}

// The interpolation interval of `time` among ascending keys (CameraAnimation::eval): the first
// key above time and the one before it, or the last two; delta clamped to [0, 1] (0 when both
// keys coincide, where the reference divides zero by zero).
void interval(const std::vector<float> &keys, float time, int &left, int &right, float &delta)
{
    const auto it = std::upper_bound(keys.begin(), keys.end(), time);
    if (it != keys.end()) {
        right = (int)(it - keys.begin());
        left = std::max(right - 1, 0);
    } else {
        right = (int)keys.size() - 1;
        left = std::max(right - 1, 0);
    }
    const float t0 = keys[(size_t)left], t1 = keys[(size_t)right];
    delta = t1 == t0 ? 0.0f : std::clamp((time - t0) / (t1 - t0), 0.0f, 1.0f);
}

} // namespace

void CameraAnimation::eval(float time, float m[16]) const
{
    int l, r;
    float dt;
    float t[3] = {0, 0, 0}, q[4] = {0, 0, 0, 1};
    if (!translation_keys.empty()) {
        interval(translation_keys, time, l, r, dt);
        for (int k = 0; k < 3; ++k)
            t[k] = (1.0f - dt) * translation_values[3 * (size_t)l + k] + dt * translation_values[3 * (size_t)r + k];
    }
    if (!rotation_keys.empty()) {
        interval(rotation_keys, time, l, r, dt);
        slerp(&rotation_values[4 * (size_t)l], &rotation_values[4 * (size_t)r], dt, q);
    }
    const float x = q[0], y = q[1], z = q[2], w = q[3];
    const float R[9] = {1 - 2 * (y * y + z * z), 2 * (x * y - w * z),     2 * (x * z + w * y),
                        2 * (x * y + w * z),     1 - 2 * (x * x + z * z), 2 * (y * z - w * x),
                        2 * (x * z - w * y),     2 * (y * z + w * x),     1 - 2 * (x * x + y * y)};
    for (int row = 0; row < 3; ++row) {
        for (int c = 0; c < 3; ++c)
            m[4 * row + c] = R[3 * row + c];
        m[4 * row + 3] = t[row];
    }
    m[12] = m[13] = m[14] = 0.0f;
    m[15] = 1.0f;
}

CameraAnimation load_camera_animation(const fs::path &path, const std::string &name, bool y_up_to_z_up)
{
    Model m = load_model(path);
    const auto &nodes = m.doc.array("nodes");
    const auto &cameras = m.doc.array("cameras");
    const auto &scenes = m.doc.array("scenes");
    const long si = m.doc.integer("scene", 0);
    if (si < 0 || si >= (long)scenes.size())
        throw Error(path.string() + ": no default scene");
    std::vector<int> seen(nodes.size(), 0);
    auto find = [&](long ni, auto &self) -> long {
        if (ni < 0 || ni >= (long)nodes.size() || seen[(size_t)ni]++)
            throw Error(path.string() + ": bad node graph");
        const Json &node = nodes[(size_t)ni];
        const long ci = node.integer("camera", -1);
        if (ci >= 0 && ci < (long)cameras.size() && cameras[(size_t)ci].string("name", "") == name)
            return ni;
        for (const Json &c : node.array("children")) {
            const long r = self(c.kind == Json::Number ? (long)c.num : -1, self);
            if (r >= 0)
                return r;
        }
        return -1;
    };
    long cam_node = -1;
    for (const Json &root : scenes[(size_t)si].array("nodes")) {
        cam_node = find(root.kind == Json::Number ? (long)root.num : -1, find);
        if (cam_node >= 0)
            break;
    }
    if (cam_node < 0)
        throw Error(path.string() + ": no camera node named [" + name + "]");
    const Json &cam = cameras[(size_t)nodes[(size_t)cam_node].integer("camera", -1)];
    CameraAnimation a;
    if (cam.string("type", "") != "perspective")
        throw Error(path.string() + ": camera [" + name + "] is not a perspective camera", true);
    const Json *persp = cam.get("perspective");
    if (!persp)
        throw Error(path.string() + ": camera [" + name + "] without perspective parameters");
    a.vfov = (float)persp->number("yfov", 0.0);
    a.aspect = (float)persp->number("aspectRatio", 0.0);
    long t_in = -1, t_out = -1, r_in = -1, r_out = -1;
    for (const Json &anim : m.doc.array("animations")) {
        long ts = -1, rs = -1;
        for (const Json &ch : anim.array("channels")) {
            const Json *target = ch.get("target");
            if (!target || target->integer("node", -1) != cam_node)
                continue;
            const std::string what = target->string("path", "");
            if (what == "translation")
                ts = ch.integer("sampler", -1);
            else if (what == "rotation")
                rs = ch.integer("sampler", -1);
        }
        const auto &samplers = anim.array("samplers");
        auto io = [&](long s, long &in, long &out) {
            if (s < 0 || s >= (long)samplers.size())
                throw Error(path.string() + ": animation sampler index out of range");
            in = samplers[(size_t)s].integer("input", -1);
            out = samplers[(size_t)s].integer("output", -1);
        };
        if (ts >= 0)
            io(ts, t_in, t_out);
        if (rs >= 0)
            io(rs, r_in, r_out);
        if (ts >= 0 && rs >= 0)
            break;
    }
    if (t_in < 0)
        throw Error(path.string() + ": no translation animation for the camera [" + name + "]", r_in >= 0);
    size_t n = 0, n2 = 0;
    a.translation_keys = floats(m, t_in, "SCALAR", n);
    a.translation_values = floats(m, t_out, "VEC3", n2);
    if (n == 0 || n2 != n)
        throw Error(path.string() + ": translation keys and values differ in count");
    if (r_in >= 0) {
        a.rotation_keys = floats(m, r_in, "SCALAR", n);
        a.rotation_values = floats(m, r_out, "VEC4", n2);
        if (n == 0 || n2 != n)
            throw Error(path.string() + ": rotation keys and values differ in count");
    }
    if (!std::is_sorted(a.translation_keys.begin(), a.translation_keys.end()) ||
        !std::is_sorted(a.rotation_keys.begin(), a.rotation_keys.end()))
        throw Error(path.string() + ": animation keys are not in ascending order");
    if (y_up_to_z_up) {
        for (size_t i = 0; i + 2 < a.translation_values.size(); i += 3) {
            const float y = a.translation_values[i + 1], z = a.translation_values[i + 2];
            a.translation_values[i + 1] = -z;
            a.translation_values[i + 2] = y;
        }
        // r * q with r the quarter turn about x of convert_yup_to_zup: (sin 45, 0, 0, cos 45)
        const float s = std::sqrt(0.5f);
        for (size_t i = 0; i + 3 < a.rotation_values.size(); i += 4) {
            const float qx = a.rotation_values[i], qy = a.rotation_values[i + 1], qz = a.rotation_values[i + 2],
                        qw = a.rotation_values[i + 3];
            a.rotation_values[i] = s * qw + s * qx;
            a.rotation_values[i + 1] = s * qy - s * qz;
            a.rotation_values[i + 2] = s * qz + s * qy;
            a.rotation_values[i + 3] = s * qw - s * qx;
        }
    }
    return a;
}

} // namespace gltf
} // namespace ksb
