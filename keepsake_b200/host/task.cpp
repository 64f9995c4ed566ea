// The TOML task boundary (include/ks_b200_task.hpp): keepsake's configuration service for the
// small_pt path, running the GPU small_pt through the C ABI.
//
//   ConfigService / run_all_tasks      config.cpp:262-312 (task_dir, override, config.toml copy)
//   asset tables                       ConfigurableTable::load, config.cpp:315-329 ("field.key")
//   small_pt task                      small_pt.cpp:180-300
//   create_scene / material lists      scene.cpp:345-365, mesh_asset.cpp:286-299
//   create_principled_bsdf             principled_bsdf.cpp:707-733 (constant shader fields,
//                                      shader_field.h:89-156)
//   create_sky_light                   light.cpp:257-275
//   create_camera / look_at            camera.cpp:12-31,172-205
//   load_transform_field               config.cpp:204-260
//   create_mesh_asset                  mesh_asset.cpp:243-266 (obj / bin formats, to_world)
//   create_compound_mesh_asset         mesh_asset.cpp:1114-1132 (glTF: prototypes + instances)
//   convert_mesh_asset task            mesh_asset.cpp:301-311
//   composite_and_save_to_exr          render_target.cpp:181-208 (interval images)
#include "../../include/ks_b200.h"
#include "../../include/ks_b200_task.hpp"
#include "gltf.h"
#include "image_io.h"
#include "mesh_io.h"
#include "procedural.h"
#include "toml.h"

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <algorithm>
#include <cstring>
#include <fstream>
#include <map>
#include <sstream>
#include <stdexcept>
#include <vector>

namespace fs = std::filesystem;
using ksb::toml::Value;

namespace ks_b200
{

namespace
{

struct StatusError : std::runtime_error
{
    ks_status status;
    StatusError(ks_status s, const std::string &what) : std::runtime_error(what), status(s) {}
};

struct ParseError : std::runtime_error
{
    using std::runtime_error::runtime_error;
};

struct IoError : std::runtime_error
{
    using std::runtime_error::runtime_error;
};

// One geometry of a mesh asset (one MeshGeometry of a subscene).
struct Geometry
{
    std::vector<float> vertices;
    std::vector<uint32_t> indices;
    std::vector<float> normals;   // 3 per vertex or empty
    std::vector<float> texcoords; // 2 per vertex or empty
    bool twosided = true;
    bool use_smooth_normal = true;
    int own_material = -1; // index into MeshAsset::materials (procedural assets)
};

struct MeshAsset
{
    std::vector<Geometry> geometries;
    std::vector<ks_material_desc> materials; // procedural assets bring their own
    // textured fields of `materials` (glTF assets): `material` indexes `materials`, `texture` the
    // service's texture store
    std::vector<ks_texture_binding> bindings;
    std::vector<float> sky_map;              // procedural assets: their sky
    ks_sky_desc sky{};
    // compound (glTF) assets: prototypes as runs of geometries, and their instances
    std::vector<ks_prototype_desc> prototypes;
    std::vector<ks_instance_desc> instances;
};

} // namespace

struct ConfigServiceImpl
{
    ksb::toml::Table root;
    fs::path asset_root = fs::current_path();
    fs::path output_dir = fs::current_path();
    std::map<std::string, ConfigTask> tasks;
    std::map<std::string, std::shared_ptr<MeshAsset>> meshes;
    // a material and the bindings of its textured fields (`material` unset, `texture` an index
    // into `textures`)
    struct TaskMaterial
    {
        ks_material_desc d{};
        std::vector<ks_texture_binding> binds;
    };
    std::map<std::string, TaskMaterial> materials;
    // every texture the configuration loaded: texture assets, glTF images, one-texel constants
    std::vector<ksb::gltf::Texture> textures;
    std::vector<int> texture_mips; // per texture: created with build_mipmaps
    std::map<std::string, uint32_t> texture_assets;

    const Value *find_asset(const std::string &path) const;
    std::shared_ptr<MeshAsset> mesh_asset(const std::string &path);
    std::shared_ptr<MeshAsset> compound_asset(const std::string &path);
    std::shared_ptr<ksb::gltf::CameraAnimation> camera_animation(const std::string &path);
    std::map<std::string, std::shared_ptr<ksb::gltf::CameraAnimation>> animations;
    const TaskMaterial &material(const std::string &path);
    uint32_t texture(const std::string &path);
    uint32_t constant_texture(const float *value, int channels);
    ks_texture_binding texture_field(const ConfigArgs &f, int n, int32_t field, const std::string &where);
};

struct ConfigArgsInternal
{
    ConfigServiceImpl *service = nullptr;
    const Value *node = nullptr;
    std::shared_ptr<Value> owner; // keeps merged task tables alive
    std::string where;
};

namespace
{

const Value &child(const ConfigArgsInternal &a, std::string_view key)
{
    if (!a.node || a.node->kind != Value::Kind::Table)
        throw ParseError("config: '" + a.where + "' is not a table");
    auto it = a.node->table->find(std::string(key));
    if (it == a.node->table->end())
        throw ParseError("config: missing key '" + std::string(key) + "' in '" + a.where + "'");
    return it->second;
}

bool has(const ConfigArgsInternal &a, std::string_view key)
{
    return a.node && a.node->kind == Value::Kind::Table && a.node->table->count(std::string(key));
}

double as_number(const Value &v, const std::string &what)
{
    if (!v.is_number())
        throw ParseError("config: '" + what + "' must be a number");
    return v.number();
}

void vec_n(const Value &v, int n, float *out, const std::string &what)
{
    if (v.kind != Value::Kind::Array || (int)v.array->size() != n)
        throw ParseError("config: '" + what + "' must be an array of " + std::to_string(n) + " numbers");
    for (int i = 0; i < n; ++i)
        out[i] = (float)as_number((*v.array)[i], what);
}

} // namespace

// ---- ConfigArgs -----------------------------------------------------------------------------
ConfigArgs::ConfigArgs(std::shared_ptr<ConfigArgsInternal> in) : internal(std::move(in)) {}

ConfigArgs ConfigArgs::operator[](std::string_view key) const
{
    auto a = std::make_shared<ConfigArgsInternal>(*internal);
    a->node = &child(*internal, key);
    a->where = internal->where + "." + std::string(key);
    return ConfigArgs(a);
}

ConfigArgs ConfigArgs::operator[](int index) const
{
    const Value *n = internal->node;
    if (!n || n->kind != Value::Kind::Array || index < 0 || index >= (int)n->array->size())
        throw ParseError("config: index " + std::to_string(index) + " out of range in '" + internal->where + "'");
    auto a = std::make_shared<ConfigArgsInternal>(*internal);
    a->node = &(*n->array)[index];
    a->where = internal->where + "[" + std::to_string(index) + "]";
    return ConfigArgs(a);
}

bool ConfigArgs::contains(std::string_view key) const { return has(*internal, key); }

int ConfigArgs::array_size() const
{
    const Value *n = internal->node;
    if (!n || n->kind != Value::Kind::Array)
        throw ParseError("config: '" + internal->where + "' is not an array");
    return (int)n->array->size();
}

int ConfigArgs::load_integer(std::string_view key) const
{
    const Value &v = child(*internal, key);
    if (v.kind != Value::Kind::Integer)
        throw ParseError("config: '" + std::string(key) + "' must be an integer");
    return (int)v.integer;
}
int ConfigArgs::load_integer(std::string_view key, int d) const { return contains(key) ? load_integer(key) : d; }
float ConfigArgs::load_float(std::string_view key) const
{
    return (float)as_number(child(*internal, key), std::string(key));
}
float ConfigArgs::load_float(std::string_view key, float d) const { return contains(key) ? load_float(key) : d; }
bool ConfigArgs::load_bool(std::string_view key) const
{
    const Value &v = child(*internal, key);
    if (v.kind != Value::Kind::Boolean)
        throw ParseError("config: '" + std::string(key) + "' must be a boolean");
    return v.boolean;
}
bool ConfigArgs::load_bool(std::string_view key, bool d) const { return contains(key) ? load_bool(key) : d; }
std::string ConfigArgs::load_string(std::string_view key) const
{
    const Value &v = child(*internal, key);
    if (v.kind != Value::Kind::String)
        throw ParseError("config: '" + std::string(key) + "' must be a string");
    return v.str;
}
std::string ConfigArgs::load_string(std::string_view key, std::string_view d) const
{
    return contains(key) ? load_string(key) : std::string(d);
}
std::string ConfigArgs::load_string(int index) const
{
    const Value &v = *(*this)[index].internal->node;
    if (v.kind != Value::Kind::String)
        throw ParseError("config: element " + std::to_string(index) + " of '" + internal->where + "' must be a string");
    return v.str;
}
void ConfigArgs::load_vec3(std::string_view key, float out[3]) const
{
    vec_n(child(*internal, key), 3, out, std::string(key));
}

fs::path ConfigArgs::load_path(std::string_view key) const
{
    fs::path p = load_string(key);
    return p.is_absolute() ? p : internal->service->asset_root / p;
}

namespace
{

void mat_mul(const double a[16], const double b[16], double out[16])
{
    for (int r = 0; r < 4; ++r)
        for (int c = 0; c < 4; ++c) {
            double s = 0.0;
            for (int k = 0; k < 4; ++k)
                s += a[4 * r + k] * b[4 * k + c];
            out[4 * r + c] = s;
        }
}

} // namespace

void ConfigArgs::load_transform(std::string_view key, float out[16]) const
{
    ConfigArgs t = (*this)[key];
    if (t.contains("matrix_rm") || t.contains("matrix_cm")) {
        bool rm = t.contains("matrix_rm");
        float m[16];
        vec_n(child(*t.internal, rm ? "matrix_rm" : "matrix_cm"), 16, m, rm ? "matrix_rm" : "matrix_cm");
        for (int r = 0; r < 4; ++r)
            for (int c = 0; c < 4; ++c)
                out[4 * r + c] = rm ? m[4 * r + c] : m[4 * c + r];
        return;
    }
    float s[3] = {1, 1, 1}, tr[3] = {0, 0, 0};
    if (t.contains("scale"))
        t.load_vec3("scale", s);
    if (t.contains("translation"))
        t.load_vec3("translation", tr);
    double R[16] = {1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1};
    if (t.contains("rotation")) {
        ConfigArgs r = t["rotation"];
        if (r.contains("euler")) {
            // XYZ Euler angles in degrees: R = Rx(a0) Ry(a1) Rz(a2)
            float e[3];
            r.load_vec3("euler", e);
            double a[3];
            for (int i = 0; i < 3; ++i)
                a[i] = (double)(e[i] / 180.0f * 3.14159265358979323846f);
            double Rx[16] = {1, 0, 0, 0, 0, std::cos(a[0]), -std::sin(a[0]), 0, 0, std::sin(a[0]), std::cos(a[0]), 0,
                             0, 0, 0, 1};
            double Ry[16] = {std::cos(a[1]), 0, std::sin(a[1]), 0, 0, 1, 0, 0, -std::sin(a[1]), 0, std::cos(a[1]), 0,
                             0, 0, 0, 1};
            double Rz[16] = {std::cos(a[2]), -std::sin(a[2]), 0, 0, std::sin(a[2]), std::cos(a[2]), 0, 0, 0, 0, 1, 0,
                             0, 0, 0, 1};
            double t1[16];
            mat_mul(Rx, Ry, t1);
            mat_mul(t1, Rz, R);
        } else if (r.contains("quat")) {
            float q[4];
            vec_n(child(*r.internal, "quat"), 4, q, "quat");
            double w = q[0], x = q[1], y = q[2], z = q[3];
            double n = std::sqrt(w * w + x * x + y * y + z * z);
            w /= n, x /= n, y /= n, z /= n;
            double M[16] = {1 - 2 * (y * y + z * z), 2 * (x * y - w * z),     2 * (x * z + w * y),     0,
                            2 * (x * y + w * z),     1 - 2 * (x * x + z * z), 2 * (y * z - w * x),     0,
                            2 * (x * z - w * y),     2 * (y * z + w * x),     1 - 2 * (x * x + y * y), 0,
                            0,                       0,                       0,                       1};
            std::memcpy(R, M, sizeof(M));
        } else {
            throw ParseError("config: rotation must be given as (XYZ) euler angles or a quaternion");
        }
    }
    // scale_rotate_translate (maths.h:863-879): T * R * S
    for (int r = 0; r < 4; ++r)
        for (int c = 0; c < 4; ++c) {
            double v = R[4 * r + c] * (c < 3 ? s[c] : 1.0);
            if (r < 3 && c == 3)
                v = tr[r];
            out[4 * r + c] = (float)v;
        }
}

// ---- assets ---------------------------------------------------------------------------------
const Value *ConfigServiceImpl::find_asset(const std::string &path) const
{
    size_t dot = path.find('.');
    if (dot == std::string::npos)
        return nullptr;
    auto f = root.find(path.substr(0, dot));
    if (f == root.end() || f->second.kind != Value::Kind::Table)
        return nullptr;
    auto k = f->second.table->find(path.substr(dot + 1));
    return k == f->second.table->end() ? nullptr : &k->second;
}

namespace
{

ConfigArgs args_of(ConfigServiceImpl *svc, const Value *node, const std::string &where)
{
    auto a = std::make_shared<ConfigArgsInternal>();
    a->service = svc;
    a->node = node;
    a->where = where;
    return ConfigArgs(a);
}

// MeshData (mesh files) to the task's geometries.
void add_meshes(std::vector<ksb::mesh::MeshData> &&meshes, MeshAsset &out)
{
    for (auto &md : meshes) {
        Geometry g;
        g.vertices = std::move(md.vertices);
        g.indices = std::move(md.indices);
        g.normals = std::move(md.normals);
        g.texcoords = std::move(md.texcoords);
        g.twosided = md.twosided;
        g.use_smooth_normal = md.use_smooth_normal;
        out.geometries.push_back(std::move(g));
    }
}

void flat_numbers(const Value &v, std::vector<double> &out, const std::string &what)
{
    if (v.kind == Value::Kind::Array) {
        for (const Value &e : *v.array)
            flat_numbers(e, out, what);
    } else {
        out.push_back(as_number(v, what));
    }
}

} // namespace

std::shared_ptr<MeshAsset> ConfigServiceImpl::mesh_asset(const std::string &path)
{
    auto it = meshes.find(path);
    if (it != meshes.end())
        return it->second;
    const Value *node = find_asset(path);
    if (!node || path.rfind("mesh_asset.", 0) != 0)
        throw ParseError("config: unknown mesh asset '" + path + "'");
    ConfigArgs a = args_of(this, node, path);
    auto m = std::make_shared<MeshAsset>();
    // a mesh file (create_mesh_asset: "format" obj | bin), or an extension "type" of this build
    std::string type = a.contains("type") ? a.load_string("type") : a.contains("path") ? "file" : "inline";
    if (type == "obj" || type == "bin") // the file types spelled as "type"
        type = "file";
    if (type == "file") {
        const std::string fmt = a.contains("format") ? a.load_string("format")
                                : a.contains("type") ? a.load_string("type")
                                                     : "obj";
        const fs::path file = a.load_path("path");
        try {
            if (fmt == "obj") {
                if (a.load_bool("load_materials", false))
                    throw StatusError(KS_ERR_UNSUPPORTED, "config: load_materials (MTL Lambertian materials) is not "
                                                          "supported; give the task a material list");
                add_meshes(ksb::mesh::load_obj(file, a.load_bool("twosided", false),
                                               a.load_bool("use_smooth_normal", true)),
                           *m);
            } else if (fmt == "bin") {
                add_meshes(ksb::mesh::load_binary(file), *m);
            } else {
                throw StatusError(KS_ERR_UNSUPPORTED, "config: unsupported mesh asset format '" + fmt + "'");
            }
        } catch (const ksb::mesh::Error &e) {
            throw IoError(e.what());
        }
        if (a.contains("to_world")) {
            // MeshData::transform (geometry.cpp:15-32) of every mesh of the asset
            float xf[16];
            a.load_transform("to_world", xf);
            std::vector<ksb::mesh::MeshData> tmp(m->geometries.size());
            for (size_t k = 0; k < tmp.size(); ++k) {
                tmp[k].vertices = std::move(m->geometries[k].vertices);
                tmp[k].normals = std::move(m->geometries[k].normals);
            }
            try {
                ksb::mesh::transform(tmp, xf);
            } catch (const ksb::mesh::Error &e) {
                throw ParseError(std::string("config: ") + e.what());
            }
            for (size_t k = 0; k < tmp.size(); ++k) {
                m->geometries[k].vertices = std::move(tmp[k].vertices);
                m->geometries[k].normals = std::move(tmp[k].normals);
            }
        }
    } else if (type == "procedural") {
        // seeded synthetic scene (extension): kind "box_room" | "icosphere"
        ksb::ProceduralOptions o;
        o.level = a.load_integer("level", o.level);
        if (a.contains("roughness")) {
            float r[2];
            vec_n(child(*a.internal, "roughness"), 2, r, "roughness");
            o.roughness_min = r[0];
            o.roughness_max = r[1];
        }
        o.occluder = a.load_bool("occluder", false) ? 1 : 0;
        if (a.contains("sky_resolution")) {
            float r[2];
            vec_n(child(*a.internal, "sky_resolution"), 2, r, "sky_resolution");
            o.sky_width = (uint32_t)r[0];
            o.sky_height = (uint32_t)r[1];
        }
        ksb::GeneratedScene g;
        if (!ksb::generate_scene(a.load_string("kind"), (uint64_t)a.load_integer("seed", 0), o, g))
            throw ParseError("config: unknown procedural kind in '" + path + "'");
        for (auto &gm : g.meshes) {
            Geometry geo;
            geo.vertices = std::move(gm.vertices);
            geo.indices = std::move(gm.indices);
            geo.own_material = (int)gm.material;
            m->geometries.push_back(std::move(geo));
        }
        m->materials = g.materials;
        m->sky_map = std::move(g.sky_map);
        m->sky = g.sky;
        m->sky.map_rgb = nullptr;
    } else if (type == "inline") {
        // extension for small scenes written in the file: geometry = [{vertices = [...], indices = [...]}]
        // (optional texcoords = [...], 2 numbers per vertex)
        ConfigArgs list = a["geometry"];
        for (int i = 0; i < list.array_size(); ++i) {
            ConfigArgs gi = list[i];
            std::vector<double> v, idx;
            flat_numbers(child(*gi.internal, "vertices"), v, "vertices");
            flat_numbers(child(*gi.internal, "indices"), idx, "indices");
            if (v.size() % 3 || idx.size() % 3 || idx.empty())
                throw ParseError("config: inline geometry needs 3 numbers per vertex and per triangle");
            Geometry geo;
            for (double x : v)
                geo.vertices.push_back((float)x);
            for (double x : idx) {
                if (x < 0 || x >= (double)(v.size() / 3))
                    throw ParseError("config: inline geometry index out of range");
                geo.indices.push_back((uint32_t)x);
            }
            if (gi.contains("texcoords")) {
                std::vector<double> tc;
                flat_numbers(child(*gi.internal, "texcoords"), tc, "texcoords");
                if (tc.size() != 2 * (v.size() / 3))
                    throw ParseError("config: inline geometry needs 2 texcoords per vertex");
                for (double x : tc)
                    geo.texcoords.push_back((float)x);
            }
            m->geometries.push_back(std::move(geo));
        }
    } else {
        throw StatusError(KS_ERR_UNSUPPORTED, "config: mesh asset type '" + type + "' is not supported");
    }
    meshes[path] = m;
    return m;
}

// create_compound_mesh_asset (mesh_asset.cpp:1114-1132): a glTF file ("format" glb | gltf) as
// prototypes (its meshes) and instances (its nodes), with its materials when load_materials.
std::shared_ptr<MeshAsset> ConfigServiceImpl::compound_asset(const std::string &path)
{
    auto it = meshes.find(path);
    if (it != meshes.end())
        return it->second;
    const Value *node = find_asset(path);
    if (!node || path.rfind("compound_mesh_asset.", 0) != 0)
        throw ParseError("config: unknown compound mesh asset '" + path + "'");
    ConfigArgs a = args_of(this, node, path);
    const std::string fmt = a.load_string("format", "glb");
    if (fmt != "glb" && fmt != "gltf")
        throw StatusError(KS_ERR_UNSUPPORTED, "config: unsupported compound mesh asset format '" + fmt + "'");
    if (a.load_string("bsdf_type", "principled_bsdf") != "principled_bsdf")
        throw StatusError(KS_ERR_UNSUPPORTED, "config: only principled_bsdf materials are supported");
    const bool load_materials = a.load_bool("load_materials", false);
    ksb::gltf::Compound c;
    try {
        c = ksb::gltf::load(a.load_path("path"), load_materials);
    } catch (const ksb::gltf::Error &e) {
        if (e.unsupported)
            throw StatusError(KS_ERR_UNSUPPORTED, std::string("config: ") + e.what());
        throw IoError(e.what());
    }
    if (c.instances.empty())
        throw ParseError("config: compound mesh asset '" + path + "' instances no mesh");
    auto m = std::make_shared<MeshAsset>();
    const uint32_t tex_base = (uint32_t)textures.size();
    for (auto &t : c.textures) {
        textures.push_back(std::move(t));
        texture_mips.push_back(0);
    }
    for (auto &p : c.prototypes) {
        for (ks_texture_binding b : p.bindings) {
            b.material += (uint32_t)m->materials.size(); // primitive index -> asset material
            b.texture += tex_base;
            m->bindings.push_back(b);
        }
        m->prototypes.push_back({(uint32_t)m->geometries.size(), (uint32_t)p.meshes.size()});
        for (size_t k = 0; k < p.meshes.size(); ++k) {
            std::vector<ksb::mesh::MeshData> one(1);
            one[0] = std::move(p.meshes[k]);
            add_meshes(std::move(one), *m);
            if (load_materials) {
                m->geometries.back().own_material = (int)m->materials.size();
                m->materials.push_back(p.materials[k]);
            }
        }
    }
    for (const auto &i : c.instances) {
        ks_instance_desc d{};
        d.prototype = i.prototype;
        std::memcpy(d.to_world, i.to_world, sizeof(d.to_world));
        m->instances.push_back(d);
    }
    meshes[path] = m;
    return m;
}

// create_camera_animation (camera.cpp:276-465): keys path, camera_name, convert_y_up_to_z_up.
std::shared_ptr<ksb::gltf::CameraAnimation> ConfigServiceImpl::camera_animation(const std::string &path)
{
    auto it = animations.find(path);
    if (it != animations.end())
        return it->second;
    const Value *node = find_asset(path);
    if (!node || path.rfind("camera_animation.", 0) != 0)
        throw ParseError("config: unknown camera animation '" + path + "'");
    ConfigArgs a = args_of(this, node, path);
    std::shared_ptr<ksb::gltf::CameraAnimation> anim;
    try {
        anim = std::make_shared<ksb::gltf::CameraAnimation>(ksb::gltf::load_camera_animation(
            a.load_path("path"), a.load_string("camera_name"), a.load_bool("convert_y_up_to_z_up", false)));
    } catch (const ksb::gltf::Error &e) {
        if (e.unsupported)
            throw StatusError(KS_ERR_UNSUPPORTED, std::string("config: ") + e.what());
        throw IoError(e.what());
    }
    animations[path] = anim;
    return anim;
}

// create_texture_from_image (texture.cpp:922-944): .exr / .hdr (and .pfm) as float texels, PNG as
// 8-bit texels through stb_image's 8-bit loader with the requested channel count (16-bit PNGs kept
// at 16 bits with keep_16bit, as tinygltf keeps glTF images).  Throws image::Error.
ksb::gltf::Texture load_texture_file(const fs::path &file, int ch, bool srgb, bool keep_16bit)
{
    const std::string ext = file.extension().string();
    ksb::gltf::Texture t;
    t.channels = ch;
    t.srgb = srgb;
    if (ext == ".exr" || ext == ".hdr" || ext == ".pfm") {
        const std::vector<float> v = ksb::image::read_float_texture(file, ch, t.width, t.height);
        t.format = 2;
        t.bytes.resize(v.size() * 4);
        std::memcpy(t.bytes.data(), v.data(), t.bytes.size());
    } else if (ext == ".png") {
        const ksb::image::Png png = ksb::image::read_png(file);
        const int depth = keep_16bit ? png.depth : 8;
        const std::vector<uint16_t> v = ksb::image::convert_channels(png, ch, depth);
        t.width = png.width;
        t.height = png.height;
        if (depth == 16) {
            t.format = 1;
            t.bytes.resize(v.size() * 2);
            std::memcpy(t.bytes.data(), v.data(), t.bytes.size());
        } else {
            t.format = 0;
            t.bytes.assign(v.begin(), v.end());
        }
    } else {
        throw ksb::image::Error(file.string() + ": texture images are read from .png, .exr, .hdr or .pfm files",
                                true);
    }
    return t;
}

// create_texture (texture.cpp:1068-1084) with create_texture_from_image (:922-944): `path`,
// `channels`, `build_mipmaps`, `colorspace` ("Linear" or "sRGB"); .exr / .hdr (and .pfm) as float
// texels, PNG as 8-bit texels (stb_image's 8-bit loader with the requested channel count).
// Serialized (lz4) textures and other image formats are unsupported.
uint32_t ConfigServiceImpl::texture(const std::string &path)
{
    auto it = texture_assets.find(path);
    if (it != texture_assets.end())
        return it->second;
    const Value *node = find_asset(path);
    if (!node || path.rfind("texture.", 0) != 0)
        throw ParseError("config: unknown texture '" + path + "'");
    ConfigArgs a = args_of(this, node, path);
    if (a.load_bool("serialized", false))
        throw StatusError(KS_ERR_UNSUPPORTED, "config: serialized textures are not supported");
    const int ch = a.load_integer("channels");
    const bool mips = a.load_bool("build_mipmaps");
    const bool srgb = a.load_string("colorspace", "Linear") == "sRGB";
    if (ch < 1 || ch > 4)
        throw ParseError("config: texture '" + path + "' needs 1 to 4 channels");
    ksb::gltf::Texture t;
    try {
        t = load_texture_file(a.load_path("path"), ch, srgb, false);
    } catch (const ksb::image::Error &e) {
        if (e.unsupported)
            throw StatusError(KS_ERR_UNSUPPORTED, std::string("config: ") + e.what());
        throw IoError(e.what());
    }
    textures.push_back(std::move(t));
    texture_mips.push_back(mips ? 1 : 0);
    texture_assets[path] = (uint32_t)textures.size() - 1;
    return (uint32_t)textures.size() - 1;
}

// A constant field as a one-texel float texture (read with the nearest filter, scale 1).
uint32_t ConfigServiceImpl::constant_texture(const float *value, int channels)
{
    ksb::gltf::Texture t;
    t.width = t.height = 1;
    t.channels = channels;
    t.format = 2;
    t.bytes.resize(4 * (size_t)channels);
    std::memcpy(t.bytes.data(), value, t.bytes.size());
    textures.push_back(std::move(t));
    texture_mips.push_back(0);
    return (uint32_t)textures.size() - 1;
}

// create_texture_shader_field_color<N> (shader_field.h:107-142): map (a texture asset), sampler
// (create_texture_sampler, texture.cpp:1086-1121: nearest | linear | cubic with kernel mitchell |
// bspline | catmull_rom; wrap_mode_u / wrap_mode_v repeat | clamp), flip_v (true), swizzle,
// uv_scale, uv_offset, scale.  Linear and cubic lookups of a mipmapped texture choose their level
// from the camera ray's differentials, and EWA filters with them: those are unsupported (the
// nearest filter always reads level 0, and a texture without mipmaps has only level 0).
ks_texture_binding ConfigServiceImpl::texture_field(const ConfigArgs &f, int n, int32_t field,
                                                    const std::string &where)
{
    ks_texture_binding b{};
    b.field = field;
    b.texture = texture(f.load_string("map"));
    ConfigArgs sm = f["sampler"];
    const std::string st = sm.load_string("type");
    if (st == "nearest") {
        b.filter = 0;
    } else if (st == "linear") {
        b.filter = 1;
    } else if (st == "cubic") {
        b.filter = 2;
        const std::string k = sm.load_string("kernel", "mitchell");
        b.cubic_kernel = k == "bspline" ? 1 : (k == "catmull_rom" ? 2 : 0);
    } else if (st == "ewa") {
        throw StatusError(KS_ERR_UNSUPPORTED, "config: '" + where + "': EWA texture filtering is not supported");
    } else {
        throw ParseError("config: '" + where + "': unknown texture sampler type '" + st + "'");
    }
    if (b.filter != 0 && texture_mips[b.texture])
        throw StatusError(KS_ERR_UNSUPPORTED, "config: '" + where + "': linear and cubic filtering of a texture "
                                                                     "with mipmaps are not supported");
    b.wrap_u = sm.load_string("wrap_mode_u", "repeat") == "clamp" ? 1 : 0;
    b.wrap_v = sm.load_string("wrap_mode_v", "repeat") == "clamp" ? 1 : 0;
    b.flip_v = f.load_bool("flip_v", true) ? 1 : 0;
    for (int c = 0; c < 4; ++c) {
        b.swizzle[c] = c < n ? c : -1;
        b.scale[c] = 1.0f;
    }
    if (f.contains("swizzle")) {
        if (n == 1) {
            b.swizzle[0] = f.load_integer("swizzle");
        } else {
            float sw[4];
            vec_n(child(*f.internal, "swizzle"), n, sw, "swizzle");
            for (int c = 0; c < n; ++c)
                b.swizzle[c] = (int32_t)sw[c];
        }
    }
    b.uv_scale[0] = b.uv_scale[1] = 1.0f;
    if (f.contains("uv_scale"))
        vec_n(child(*f.internal, "uv_scale"), 2, b.uv_scale, "uv_scale");
    if (f.contains("uv_offset"))
        vec_n(child(*f.internal, "uv_offset"), 2, b.uv_offset, "uv_offset");
    if (f.contains("scale")) {
        if (n == 1)
            b.scale[0] = f.load_float("scale");
        else
            vec_n(child(*f.internal, "scale"), n, b.scale, "scale");
    }
    b.range01 = 1;
    b.strength = 1.0f;
    for (int k = 0; k < 4; ++k)
        b.to_world[5 * k] = 1.0f;
    return b;
}

// create_material (material.cpp:169-178) over create_bsdf (bsdf.cpp:50-62): the BSDF's shader
// fields, constant or textured, and the material's normal map (create_normal_map,
// normal_map.cpp:40-55: map, space tangent | world, range01, strength, to_world).
const ConfigServiceImpl::TaskMaterial &ConfigServiceImpl::material(const std::string &path)
{
    auto it = materials.find(path);
    if (it != materials.end())
        return it->second;
    const Value *node = find_asset(path);
    if (!node || path.rfind("material.", 0) != 0)
        throw ParseError("config: unknown material '" + path + "'");
    ConfigArgs a = args_of(this, node, path);
    std::string bsdf_path = a.load_string("bsdf");
    const Value *bnode = find_asset(bsdf_path);
    if (!bnode)
        throw ParseError("config: unknown bsdf '" + bsdf_path + "'");
    ConfigArgs b = args_of(this, bnode, bsdf_path);
    std::string type = b.load_string("type");
    // create_bsdf (bsdf.cpp:50-62)
    if (type != "principled_bsdf" && type != "principled_brdf" && type != "lambertian")
        throw StatusError(KS_ERR_UNSUPPORTED, "config: bsdf type '" + type +
                                                  "' is not supported (principled_bsdf, principled_brdf, lambertian)");
    TaskMaterial tm;
    ks_material_desc &d = tm.d;
    // create_bssrdf (subsurface.cpp:536-545): albedo and radius (constant shader fields), anisotropy,
    // ior, rfr_entry_prob
    const std::string ss_path = a.load_string("subsurface", "");
    if (!ss_path.empty()) {
        const Value *snode = find_asset(ss_path);
        if (!snode || ss_path.rfind("bssrdf.", 0) != 0)
            throw ParseError("config: unknown bssrdf '" + ss_path + "'");
        ConfigArgs ss = args_of(this, snode, ss_path);
        auto constant3 = [&](const char *key, float out[3]) {
            const Value &v = child(*ss.internal, key);
            if (v.kind == Value::Kind::Table) {
                ConfigArgs f = ss[key];
                if (f.load_string("type") != "constant")
                    throw StatusError(KS_ERR_UNSUPPORTED, "config: '" + ss_path + "': textured " + key +
                                                              " is not supported");
                f.load_vec3("value", out);
            } else {
                vec_n(v, 3, out, key);
            }
        };
        d.has_subsurface = 1;
        constant3("albedo", d.ss_albedo);
        constant3("radius", d.ss_radius);
        d.ss_anisotropy = ss.load_float("anisotropy");
        d.ss_ior = ss.load_float("ior");
        d.ss_rfr_entry_prob = ss.load_float("rfr_entry_prob");
    }
    // a shader field: { type = "constant", value = ... } (or, as an extension, the bare value), or
    // { type = "texture", ... }
    auto field = [&](const char *key, int n, float *out, const float *dflt, int32_t field_id) {
        std::memcpy(out, dflt, sizeof(float) * n);
        if (!b.contains(key))
            return;
        const Value &v = child(*b.internal, key);
        const Value *val = &v;
        if (v.kind == Value::Kind::Table) {
            ConfigArgs f = b[key];
            std::string ft = f.load_string("type");
            if (ft == "texture") {
                if (field_id < 0)
                    throw StatusError(KS_ERR_UNSUPPORTED, std::string("config: textured '") + key +
                                                              "' is not supported");
                tm.binds.push_back(texture_field(f, n, field_id, bsdf_path + "." + key));
                return;
            }
            if (ft != "constant")
                throw StatusError(KS_ERR_UNSUPPORTED, std::string("config: shader field type '") + ft + "' of '" +
                                                          key + "' is not supported");
            val = &child(*f.internal, "value");
        }
        if (n == 1)
            out[0] = (float)as_number(*val, key);
        else
            vec_n(*val, n, out, key);
    };
    const float c08[3] = {0.8f, 0.8f, 0.8f}, one = 1.0f, zero = 0.0f, ior = 1.5f, half = 0.5f, z3[3] = {0, 0, 0};
    // the PrincipledBSDF defaults of the fields a BSDF type does not read
    d.roughness = one;
    d.ior = ior;
    d.specular_r0_mul = half;
    d.diffuse_trans_fwd = half;
    if (type == "lambertian") {
        // create_lambertian (bsdf.cpp:43-48): albedo
        d.bsdf = 2;
        field("albedo", 3, d.basecolor, c08, KS_FIELD_BASECOLOR);
    } else if (type == "principled_brdf") {
        // create_principled_brdf (principled_bsdf.cpp:227-244)
        d.bsdf = 1;
        field("basecolor", 3, d.basecolor, c08, KS_FIELD_BASECOLOR);
        field("roughness", 1, &d.roughness, &one, KS_FIELD_ROUGHNESS);
        field("metallic", 1, &d.metallic, &zero, KS_FIELD_METALLIC);
        field("specular", 1, &d.specular, &half, KS_FIELD_SPECULAR);
    } else {
        field("basecolor", 3, d.basecolor, c08, KS_FIELD_BASECOLOR);
        field("roughness", 1, &d.roughness, &one, KS_FIELD_ROUGHNESS);
        field("metallic", 1, &d.metallic, &zero, KS_FIELD_METALLIC);
        field("ior", 1, &d.ior, &ior, KS_FIELD_IOR);
        field("specular_r0_mul", 1, &d.specular_r0_mul, &half, KS_FIELD_SPECULAR_R0_MUL);
        field("specular_trans", 1, &d.specular_trans, &zero, KS_FIELD_SPECULAR_TRANS);
        field("diffuse_trans", 1, &d.diffuse_trans, &zero, KS_FIELD_DIFFUSE_TRANS);
        field("diffuse_trans_fwd", 1, &d.diffuse_trans_fwd, &half, KS_FIELD_DIFFUSE_TRANS_FWD);
        // a textured emissive field would make a textured emitter, which needs its texture's importance
        field("emissive", 3, d.emissive, z3, -1);
    }
    if (type != "lambertian") {
        std::string mf = b.load_string("microfacet", "ggx");
        if (mf == "ggx")
            d.microfacet = 0;
        else if (mf == "beckmann")
            d.microfacet = 1;
        else
            throw StatusError(KS_ERR_UNSUPPORTED, "config: microfacet '" + mf + "' is not supported (ggx, beckmann)");
    }
    if (a.contains("emission")) {
        a.load_vec3("emission", d.emission);
        d.has_emission = 1;
    }
    const std::string nm_path = a.load_string("normal_map", "");
    if (!nm_path.empty()) {
        const Value *nnode = find_asset(nm_path);
        if (!nnode || nm_path.rfind("normal_map.", 0) != 0)
            throw ParseError("config: unknown normal map '" + nm_path + "'");
        ConfigArgs nm = args_of(this, nnode, nm_path);
        ConfigArgs mf = nm["map"];
        ks_texture_binding nb{};
        if (mf.load_string("type") == "texture") {
            nb = texture_field(mf, 3, KS_FIELD_NORMAL_MAP, nm_path + ".map");
        } else {
            if (mf.load_string("type") != "constant")
                throw StatusError(KS_ERR_UNSUPPORTED, "config: '" + nm_path + "': shader field type '" +
                                                          mf.load_string("type") + "' is not supported");
            float v[3];
            mf.load_vec3("value", v);
            nb.field = KS_FIELD_NORMAL_MAP;
            nb.texture = constant_texture(v, 3);
            for (int c = 0; c < 4; ++c) {
                nb.swizzle[c] = c < 3 ? c : -1;
                nb.scale[c] = 1.0f;
            }
            nb.uv_scale[0] = nb.uv_scale[1] = 1.0f;
        }
        const std::string space = nm.load_string("space", "tangent");
        if (space != "tangent" && space != "world")
            throw ParseError("config: '" + nm_path + "': normal map space is tangent or world");
        nb.normal_space = space == "world" ? 1 : 0;
        nb.range01 = nm.load_bool("range01", true) ? 1 : 0;
        nb.strength = nm.load_float("strength", 1.0f);
        float id[16] = {1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1};
        if (nm.contains("to_world"))
            nm.load_transform("to_world", id);
        std::memcpy(nb.to_world, id, sizeof(id));
        tm.binds.push_back(nb);
    }
    return materials[path] = std::move(tm);
}

// ---- small_pt task ---------------------------------------------------------------------------
namespace
{

void check(ks_status s, ks_context *ctx, const char *what)
{
    if (s != KS_OK)
        throw StatusError(s, std::string(what) + ": " + ks_status_string(s) + (ctx ? std::string(" (") +
                                                                                     ks_last_error(ctx) + ")"
                                                                               : std::string()));
}

// look_at (camera.cpp:12-31), float arithmetic
void look_at(const float pos[3], const float target[3], float up[3], float m[16])
{
    float back[3] = {pos[0] - target[0], pos[1] - target[1], pos[2] - target[2]};
    float bn = std::sqrt(back[0] * back[0] + back[1] * back[1] + back[2] * back[2]);
    for (float &x : back)
        x /= bn;
    float right[3] = {up[1] * back[2] - up[2] * back[1], up[2] * back[0] - up[0] * back[2],
                      up[0] * back[1] - up[1] * back[0]};
    float rn2 = right[0] * right[0] + right[1] * right[1] + right[2] * right[2];
    if (rn2 < 1e-8f) {
        // orthonormal_basis (maths.h:814-821)
        float sign = std::copysign(1.0f, back[2]);
        const float a = -1.0f / (sign + back[2]);
        const float b = back[0] * back[1] * a;
        right[0] = 1.0f + sign * back[0] * back[0] * a;
        right[1] = sign * b;
        right[2] = -sign * back[0];
        up[0] = b;
        up[1] = sign + back[1] * back[1] * a;
        up[2] = -back[1];
    } else {
        float rn = std::sqrt(rn2);
        for (float &x : right)
            x /= rn;
        up[0] = back[1] * right[2] - back[2] * right[1];
        up[1] = back[2] * right[0] - back[0] * right[2];
        up[2] = back[0] * right[1] - back[1] * right[0];
    }
    const float mm[16] = {right[0], up[0], back[0], pos[0], right[1], up[1], back[1], pos[1],
                          right[2], up[2], back[2], pos[2], 0.0f,     0.0f,  0.0f,    1.0f};
    std::memcpy(m, mm, sizeof(mm));
}

struct TaskOutput
{
    fs::path dir;
    int w, h;
    float backdrop[3];
    std::string error;   // the first failed image write (reported after the render returns)
    std::string postfix; // "_<frame>" of animated renders (composite_and_save_to_exr's path_postfix)
};

// RenderTarget2::composite_and_save_to_exr (render_target.cpp:181-208): the composite of each
// progressive interval as small_pt_spp<N>.exr (FP32 RGB)
void save_interval(int spp, const double *accum, const double *weights, void *user)
{
    auto *o = static_cast<TaskOutput *>(user);
    std::vector<float> rgb((size_t)o->w * o->h * 3);
    for (size_t i = 0; i < (size_t)o->w * o->h; ++i) {
        double w0 = weights[2 * i], w_sum = (double)(uint32_t)(weights[2 * i] + weights[2 * i + 1]);
        double a = w_sum == 0.0 ? 0.0 : w0 / std::max(w_sum, 1.0);
        for (int c = 0; c < 3; ++c) {
            double fg = w0 == 0.0 ? 0.0 : accum[3 * i + c] / w0;
            rgb[3 * i + c] = (float)((1.0 - a) * o->backdrop[c] + a * fg);
        }
    }
    char name[96];
    std::snprintf(name, sizeof(name), "small_pt_spp%d%s.exr", spp, o->postfix.c_str());
    try {
        ksb::image::write_exr(o->dir / name, rgb.data(), o->w, o->h, 3, false);
    } catch (const ksb::image::Error &e) {
        if (o->error.empty())
            o->error = e.what();
    }
}

struct ContextGuard
{
    ks_context *ctx = nullptr;
    ks_scene *scene = nullptr;
    ~ContextGuard()
    {
        if (scene)
            ks_scene_destroy(scene);
        if (ctx)
            ks_context_destroy(ctx);
    }
};

} // namespace

void small_pt_b200(const ConfigArgs &args, const fs::path &task_dir, int task_id)
{
    (void)task_id;
    ConfigServiceImpl *svc = args.internal->service;
    // ---- scene (create_scene, scene.cpp:345-365) ----
    const bool compound = !args.contains("object") && args.contains("compound_object");
    std::shared_ptr<MeshAsset> asset = compound ? svc->compound_asset(args.load_string("compound_object"))
                                                : svc->mesh_asset(args.load_string("object"));
    // subscenes: one per mesh asset, one per prototype of a compound asset
    std::vector<ks_prototype_desc> subscenes = asset->prototypes;
    if (!compound)
        subscenes = {ks_prototype_desc{0, (uint32_t)asset->geometries.size()}};
    std::vector<ks_material_desc> mats;
    std::vector<ks_texture_binding> binds; // `texture` indexes svc->textures until remapped below
    std::vector<uint32_t> geom_mat(asset->geometries.size());
    if (args.contains("material")) {
        // assign_material_list (mesh_asset.cpp:286-299): one list per subscene, one material per
        // geometry
        ConfigArgs lists = args["material"];
        if (lists.array_size() != (int)subscenes.size())
            throw ParseError("config: material list mismatch dimension");
        std::map<std::string, uint32_t> index;
        for (int sub = 0; sub < (int)subscenes.size(); ++sub) {
            if (lists[sub].array_size() != (int)subscenes[sub].n_meshes)
                throw ParseError("config: material list mismatch dimension");
            for (int k = 0; k < (int)subscenes[sub].n_meshes; ++k) {
                std::string name = lists[sub].load_string(k);
                auto it = index.find(name);
                if (it == index.end()) {
                    it = index.emplace(name, (uint32_t)mats.size()).first;
                    const auto &tm = svc->material(name);
                    for (ks_texture_binding b : tm.binds) {
                        b.material = (uint32_t)mats.size();
                        binds.push_back(b);
                    }
                    mats.push_back(tm.d);
                }
                geom_mat[subscenes[sub].first_mesh + k] = it->second;
            }
        }
    } else {
        for (size_t g = 0; g < asset->geometries.size(); ++g) {
            if (asset->geometries[g].own_material < 0)
                throw ParseError("config: no materials; either load materials from file(s) or provide a material list");
            geom_mat[g] = (uint32_t)asset->geometries[g].own_material;
        }
        mats = asset->materials;
        binds = asset->bindings;
    }
    // the textures the bindings use, in order of first use
    std::vector<ks_texture_desc> tex_descs;
    {
        std::map<uint32_t, uint32_t> used;
        for (ks_texture_binding &b : binds) {
            auto u = used.find(b.texture);
            if (u == used.end()) {
                const ksb::gltf::Texture &t = svc->textures[b.texture];
                ks_texture_desc td{};
                td.texels = t.bytes.data();
                td.width = (uint32_t)t.width;
                td.height = (uint32_t)t.height;
                td.channels = (uint32_t)t.channels;
                td.format = t.format;
                td.srgb = t.srgb ? 1 : 0;
                u = used.emplace(b.texture, (uint32_t)tex_descs.size()).first;
                tex_descs.push_back(td);
            }
            b.texture = u->second;
        }
    }
    std::vector<ks_mesh_desc> meshes(asset->geometries.size());
    for (size_t g = 0; g < meshes.size(); ++g) {
        const Geometry &geo = asset->geometries[g];
        meshes[g] = ks_mesh_desc{geo.vertices.data(),
                                 (uint32_t)(geo.vertices.size() / 3),
                                 geo.indices.data(),
                                 (uint32_t)(geo.indices.size() / 3),
                                 geo.normals.empty() ? nullptr : geo.normals.data(),
                                 geom_mat[g],
                                 geo.twosided ? 1 : 0,
                                 geo.use_smooth_normal ? 1 : 0,
                                 geo.texcoords.empty() ? nullptr : geo.texcoords.data()};
    }
    ks_scene_desc desc{};
    desc.meshes = meshes.data();
    desc.n_meshes = (uint32_t)meshes.size();
    desc.materials = mats.data();
    desc.n_materials = (uint32_t)mats.size();
    desc.textures = tex_descs.empty() ? nullptr : tex_descs.data();
    desc.n_textures = (uint32_t)tex_descs.size();
    desc.bindings = binds.empty() ? nullptr : binds.data();
    desc.n_bindings = (uint32_t)binds.size();
    if (compound) {
        desc.prototypes = asset->prototypes.data();
        desc.n_prototypes = (uint32_t)asset->prototypes.size();
        desc.instances = asset->instances.data();
        desc.n_instances = (uint32_t)asset->instances.size();
    }
    // ---- sky (create_sky_light, light.cpp:257-275) ----
    std::vector<float> sky_map;
    if (args.contains("sky")) {
        ConfigArgs s = args["sky"];
        float id[16] = {1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1};
        if (s.contains("ambient")) {
            desc.sky.kind = 1;
            s.load_vec3("ambient", desc.sky.ambient);
            std::memcpy(desc.sky.to_world, id, sizeof(id));
            desc.sky.transform_y_up = 1;
            desc.sky.strength = 1.0f;
        } else {
            if (s.contains("procedural")) {
                // extension: the sky generated with a procedural mesh asset
                std::shared_ptr<MeshAsset> src = svc->mesh_asset(s.load_string("procedural"));
                if (src->sky.kind != 2)
                    throw ParseError("config: that procedural asset has no sky");
                sky_map = src->sky_map;
                desc.sky = src->sky;
            } else {
                // SkyLight reads .hdr and .exr maps (light.cpp:19-31); .pfm is an extension
                fs::path p = s.load_path("map");
                int w = 0, h = 0;
                try {
                    sky_map = ksb::image::read_rgb(p, w, h);
                } catch (const ksb::image::Error &e) {
                    if (e.unsupported)
                        throw StatusError(KS_ERR_UNSUPPORTED, std::string("config: sky map: ") + e.what());
                    throw IoError(e.what());
                }
                desc.sky.width = (uint32_t)w;
                desc.sky.height = (uint32_t)h;
                desc.sky.kind = 2;
                std::memcpy(desc.sky.to_world, id, sizeof(id));
            }
            desc.sky.map_rgb = sky_map.data();
            if (s.contains("to_world"))
                s.load_transform("to_world", desc.sky.to_world);
            desc.sky.transform_y_up = s.load_bool("transform_y_up", true) ? 1 : 0;
            desc.sky.strength = s.load_float("strength", 1.0f);
        }
    }
    // ---- lights (create_light, light.cpp:243-305): point and directional ----
    std::vector<ks_light_desc> lights;
    if (args.contains("light")) {
        ConfigArgs list = args["light"];
        for (int i = 0; i < list.array_size(); ++i) {
            ConfigArgs l = list[i];
            const std::string type = l.load_string("type");
            ks_light_desc d{};
            if (type == "point") {
                d.type = 0;
                if (l.contains("I")) {
                    l.load_vec3("I", d.color);
                } else {
                    float c[3];
                    l.load_vec3("color", c);
                    const float power = l.load_float("power");
                    for (int k = 0; k < 3; ++k)
                        d.color[k] = c[k] * power / (4.0f * 3.14159265359f);
                }
                l.load_vec3("pos", d.vec);
            } else if (type == "directional") {
                d.type = 1;
                l.load_vec3("L", d.color);
                l.load_vec3("dir", d.vec);
                const float n = std::sqrt(d.vec[0] * d.vec[0] + d.vec[1] * d.vec[1] + d.vec[2] * d.vec[2]);
                for (int k = 0; k < 3; ++k)
                    d.vec[k] /= n;
            } else if (type == "equal_area_sky") {
                // create_equal_area_sky_light (light.cpp:274-283): an .exr / .hdr map of a square
                // equal-area parameterisation, a quaternion to_world (x, y, z, w) and a strength.
                // The scene's one sky slot takes it (first in the light list).
                if (desc.sky.kind != 0)
                    throw StatusError(KS_ERR_UNSUPPORTED, "config: an equal_area_sky light with a sky: the "
                                                          "library renders one sky light");
                fs::path path = l.load_path("map");
                int w = 0, h = 0;
                try {
                    sky_map = ksb::image::read_rgb(path, w, h);
                } catch (const ksb::image::Error &e) {
                    if (e.unsupported)
                        throw StatusError(KS_ERR_UNSUPPORTED, std::string("config: sky map: ") + e.what());
                    throw IoError(e.what());
                }
                if (w != h)
                    throw ParseError("config: the equal-area map must be square (light.cpp:178)");
                float q[4] = {0, 0, 0, 1};
                if (l.contains("to_world"))
                    vec_n(child(*l.internal, "to_world"), 4, q, "to_world");
                // Eigen's quaternion from its coefficients (x, y, z, w), as a rotation matrix
                const double n2 = (double)q[0] * q[0] + (double)q[1] * q[1] + (double)q[2] * q[2] + (double)q[3] * q[3];
                const double x = q[0] / std::sqrt(n2), y = q[1] / std::sqrt(n2), z = q[2] / std::sqrt(n2),
                             qw = q[3] / std::sqrt(n2);
                const double r[9] = {1 - 2 * (y * y + z * z), 2 * (x * y - z * qw),     2 * (x * z + y * qw),
                                     2 * (x * y + z * qw),     1 - 2 * (x * x + z * z), 2 * (y * z - x * qw),
                                     2 * (x * z - y * qw),     2 * (y * z + x * qw),     1 - 2 * (x * x + y * y)};
                float m[16] = {0};
                for (int a = 0; a < 3; ++a)
                    for (int b = 0; b < 3; ++b)
                        m[4 * a + b] = (float)r[3 * a + b];
                m[15] = 1.0f;
                desc.sky.kind = 3;
                desc.sky.map_rgb = sky_map.data();
                desc.sky.width = (uint32_t)w;
                desc.sky.height = (uint32_t)h;
                std::memcpy(desc.sky.to_world, m, sizeof(m));
                desc.sky.transform_y_up = 0;
                desc.sky.strength = l.load_float("strength", 1.0f);
                continue;
            } else {
                throw StatusError(KS_ERR_UNSUPPORTED, "config: light type '" + type + "' is not supported");
            }
            lights.push_back(d);
        }
    }
    desc.lights = lights.empty() ? nullptr : lights.data();
    desc.n_lights = (uint32_t)lights.size();
    // ---- parameters (small_pt.cpp:224-241) ----
    ks_small_pt_params p;
    ks_small_pt_params_default(&p);
    if (args.contains("backdrop")) {
        args.load_vec3("backdrop", p.backdrop);
        p.include_background = 0;
    } else {
        p.include_background = 1;
    }
    p.bounces = args.load_integer("bounces");
    p.clamp_direct = args.load_float("clamp_direct", 0.0f);
    p.clamp_indirect = args.load_float("clamp_indirect", 10.0f);
    p.render_width = args.load_integer("render_width");
    p.render_height = args.load_integer("render_height");
    p.crop_start_x = args.load_integer("crop_start_x", 0);
    p.crop_start_y = args.load_integer("crop_start_y", 0);
    p.crop_width = args.load_integer("crop_width", 0);
    p.crop_height = args.load_integer("crop_height", 0);
    p.spp = args.load_integer("spp");
    p.scale_ray_diff = args.load_bool("scale_ray_diff", true) ? 1 : 0;
    p.rng_seed = args.load_integer("rng_seed", 0);
    p.spp_prog_interval = args.load_integer("spp_prog_interval", 32);
    if (args.contains("pixel_filter")) {
        // create_pixel_filter (render_target.cpp:28-44)
        ConfigArgs f = args["pixel_filter"];
        const std::string type = f.load_string("type");
        if (type == "box") {
            p.pixel_filter = 0;
            p.pixel_filter_width = f.load_float("width", 1.0f);
        } else if (type == "gaussian") {
            p.pixel_filter = 1;
            p.pixel_filter_width = f.load_float("width", 3.0f);
            p.pixel_filter_sigma = f.load_float("sigma", 0.5f);
        } else if (type == "blackman_harris") {
            p.pixel_filter = 2;
            p.pixel_filter_width = f.load_float("width", 3.0f);
        } else {
            throw ParseError("config: invalid pixel filter type [" + type + "]");
        }
    }
    // ---- camera (create_camera, camera.cpp:172-205), or the frames of a camera_animation
    // (small_pt.cpp:243-296: frame i at duration x (i + 0.5) / frames) ----
    ks_camera_desc cam{};
    std::shared_ptr<ksb::gltf::CameraAnimation> anim;
    uint32_t n_frames = 1, frame_start = 0, frame_end = 1;
    if (args.contains("camera_animation")) {
        anim = svc->camera_animation(args.load_string("camera_animation"));
        n_frames = anim->n_frames();
        frame_start = (uint32_t)args.load_integer("camera_animation_offset", 0);
        const uint32_t count = (uint32_t)args.load_integer("camera_animation_count", 0);
        frame_end = count == 0 ? n_frames : frame_start + count;
    } else {
        ConfigArgs c = args["camera"];
        float c2w[16];
        if (c.contains("to_world")) {
            c.load_transform("to_world", c2w);
        } else {
            float pos[3], target[3], up[3];
            c.load_vec3("pos", pos);
            c.load_vec3("target", target);
            c.load_vec3("up", up);
            look_at(pos, target, up, c2w);
        }
        const std::string ctype = c.load_string("type");
        if (ctype == "orthographic") {
            check(ks_camera_orthographic(c2w, c.load_float("left"), c.load_float("right"), c.load_float("bottom"),
                                         c.load_float("top"), c.load_float("near_clip"), c.load_float("far_clip"),
                                         &cam),
                  nullptr, "camera");
        } else if (ctype != "perspective") {
            throw StatusError(KS_ERR_UNSUPPORTED, "config: camera type '" + ctype + "' is not supported");
        } else {
        float aspect = c.load_float("aspect");
        float vfov;
        if (c.contains("vfov"))
            vfov = c.load_float("vfov") / 180.0f * 3.14159265358979323846f;
        else
            vfov = 2.0f * std::atan((1.0f / aspect) * std::tan(0.5f * (c.load_float("hfov") / 180.0f *
                                                                        3.14159265358979323846f)));
        check(ks_camera_perspective(c2w, vfov, aspect, &cam), nullptr, "camera");
        }
    }
    // ---- render ----
    int device = 0;
    if (const char *e = std::getenv("KS_B200_DEVICE"))
        device = std::atoi(e);
    ContextGuard g;
    check(ks_context_create(device, &g.ctx), nullptr, "ks_context_create");
    check(ks_scene_create(g.ctx, &desc, &g.scene), g.ctx, "ks_scene_create");
    check(ks_scene_build_bvh(g.scene, nullptr, nullptr), g.ctx, "ks_scene_build_bvh");
    TaskOutput out{task_dir, p.render_width, p.render_height, {p.backdrop[0], p.backdrop[1], p.backdrop[2]}};
    if (p.include_background)
        out.backdrop[0] = out.backdrop[1] = out.backdrop[2] = 0.0f;
    for (uint32_t frame = frame_start; frame < frame_end; ++frame) {
        if (anim) {
            float m[16];
            anim->eval(anim->duration() * ((float)frame + 0.5f) / (float)n_frames, m);
            check(ks_camera_perspective(m, anim->vfov, anim->aspect, &cam), nullptr, "camera animation");
        }
        char postfix[16] = "";
        if (n_frames > 1)
            std::snprintf(postfix, sizeof(postfix), "_%06u", frame);
        out.postfix = postfix;
        // a fresh render target per frame (SmallPT::run)
        std::vector<double> accum((size_t)p.render_width * p.render_height * 3, 0.0);
        std::vector<double> weights((size_t)p.render_width * p.render_height * 2, 0.0);
        check(ks_small_pt_render(g.scene, &cam, &p, save_interval, &out, accum.data(), weights.data()), g.ctx,
              "ks_small_pt_render");
        if (!out.error.empty())
            throw IoError(out.error);
    }
}

// convert_mesh_asset (mesh_asset.cpp:301-311): each listed mesh asset written as a binary mesh
// asset named after the last component of its asset path, <name>.bin, in the task directory.
void convert_mesh_asset(const ConfigArgs &args, const fs::path &task_dir, int task_id)
{
    (void)task_id;
    ConfigServiceImpl *svc = args.internal->service;
    ConfigArgs list = args["assets"];
    for (int i = 0; i < list.array_size(); ++i) {
        const std::string asset_path = list.load_string(i);
        std::shared_ptr<MeshAsset> asset = svc->mesh_asset(asset_path);
        std::vector<ksb::mesh::MeshData> meshes(asset->geometries.size());
        for (size_t k = 0; k < meshes.size(); ++k) {
            const Geometry &g = asset->geometries[k];
            meshes[k].vertices = g.vertices;
            meshes[k].indices = g.indices;
            meshes[k].normals = g.normals;
            meshes[k].texcoords = g.texcoords;
            meshes[k].twosided = g.twosided;
            meshes[k].use_smooth_normal = g.use_smooth_normal;
        }
        const std::string name = asset_path.substr(asset_path.rfind('.') + 1);
        try {
            ksb::mesh::write_binary(task_dir / (name + ".bin"), meshes);
        } catch (const ksb::mesh::Error &e) {
            throw IoError(e.what());
        }
    }
}

// ---- ConfigService ----------------------------------------------------------------------------
ConfigService::ConfigService() : impl(std::make_unique<ConfigServiceImpl>())
{
    register_task("small_pt", small_pt_b200);
    register_task("small_pt_b200", small_pt_b200);
    register_task("convert_mesh_asset", convert_mesh_asset);
}
ConfigService::~ConfigService() = default;

void ConfigService::parse_file(const fs::path &file_path)
{
    std::ifstream f(file_path);
    if (!f)
        throw IoError("cannot open " + file_path.string());
    std::stringstream ss;
    ss << f.rdbuf();
    parse(ss.str());
}

void ConfigService::parse(std::string_view text) { impl->root = ksb::toml::parse(std::string(text)); }
void ConfigService::set_asset_root_dir(const fs::path &root) { impl->asset_root = fs::absolute(root); }
void ConfigService::set_output_directory(const fs::path &dir) { impl->output_dir = dir; }
void ConfigService::register_task(std::string_view name, const ConfigTask &task) { impl->tasks[std::string(name)] = task; }
fs::path ConfigService::output_directory() const { return impl->output_dir; }

void ConfigService::run_all_tasks() const
{
    auto it = impl->root.find("task");
    if (it == impl->root.end())
        return;
    if (it->second.kind != Value::Kind::Array)
        throw ParseError("config: 'task' must be an array of tables");
    const ksb::toml::Array &tasks = *it->second.array;
    fs::create_directories(impl->output_dir);
    for (int task_id = 0; task_id < (int)tasks.size(); ++task_id) {
        if (tasks[task_id].kind != Value::Kind::Table)
            throw ParseError("config: task " + std::to_string(task_id) + " is not a table");
        auto merged = std::make_shared<Value>(ksb::toml::clone(tasks[task_id]));
        ksb::toml::Table &tt = *merged->table;
        if (tt.count("override")) {
            const Value &o = tt.at("override");
            if (o.kind != Value::Kind::Integer || o.integer < 0 || o.integer >= task_id)
                throw ParseError("config: override must name an earlier task");
            const Value &base = tasks[o.integer];
            if (base.table->count("override"))
                throw ParseError("config: an overridden task may not override another");
            Value m = ksb::toml::clone(base);
            for (const auto &[k, v] : tt)
                if (k != "override")
                    (*m.table)[k] = v;
            merged = std::make_shared<Value>(m);
        }
        const ksb::toml::Table &task = *merged->table;
        fs::path task_dir = task.count("task_dir") && task.at("task_dir").kind == Value::Kind::String
                                ? fs::path(task.at("task_dir").str)
                                : fs::path("task_" + std::to_string(task_id));
        task_dir = impl->output_dir / task_dir;
        fs::create_directories(task_dir);
        {
            std::ofstream w(task_dir / "config.toml");
            w << ksb::toml::write(task) << std::endl;
        }
        if (!task.count("type") || task.at("type").kind != Value::Kind::String)
            throw ParseError("config: task " + std::to_string(task_id) + " has no type");
        auto f = impl->tasks.find(task.at("type").str);
        if (f == impl->tasks.end())
            throw StatusError(KS_ERR_UNSUPPORTED, "config: unknown task type '" + task.at("type").str + "'");
        auto a = std::make_shared<ConfigArgsInternal>();
        a->service = impl.get();
        a->node = merged.get();
        a->owner = merged;
        a->where = "task[" + std::to_string(task_id) + "]";
        f->second(ConfigArgs(a), task_dir, task_id);
    }
}

} // namespace ks_b200

// ---- C entry point --------------------------------------------------------------------------
namespace
{
thread_local std::string g_config_error;
}

namespace ksb
{
// The message ks_config_last_error() returns, for the other host-side entry points.
void set_host_error(const std::string &msg) { g_config_error = msg; }
} // namespace ksb

extern "C" {

ks_status ks_config_run(const char *config_text, const char *asset_root_dir, const char *output_dir)
{
    g_config_error.clear();
    if (!config_text || !output_dir) {
        g_config_error = "ks_config_run: null argument";
        return KS_ERR_INVALID_ARGUMENT;
    }
    try {
        ks_b200::ConfigService svc;
        svc.parse(config_text);
        if (asset_root_dir)
            svc.set_asset_root_dir(asset_root_dir);
        svc.set_output_directory(output_dir);
        svc.run_all_tasks();
        return KS_OK;
    } catch (const ks_b200::StatusError &e) {
        g_config_error = e.what();
        return e.status;
    } catch (const ks_b200::IoError &e) {
        g_config_error = e.what();
        return KS_ERR_IO;
    } catch (const std::filesystem::filesystem_error &e) {
        g_config_error = e.what();
        return KS_ERR_IO;
    } catch (const std::exception &e) {
        g_config_error = e.what();
        return KS_ERR_PARSE;
    }
}

const char *ks_config_last_error(void) { return g_config_error.c_str(); }

ks_status ks_config_parse(const char *config_text, char *normalised, size_t capacity, size_t *length)
{
    g_config_error.clear();
    if (!config_text) {
        g_config_error = "ks_config_parse: null argument";
        return KS_ERR_INVALID_ARGUMENT;
    }
    try {
        std::string w = ksb::toml::write(ksb::toml::parse(config_text));
        if (length)
            *length = w.size();
        if (normalised && capacity) {
            size_t n = std::min(capacity - 1, w.size());
            std::memcpy(normalised, w.data(), n);
            normalised[n] = '\0';
        }
        return KS_OK;
    } catch (const std::exception &e) {
        g_config_error = e.what();
        return KS_ERR_PARSE;
    }
}

ks_status ks_image_save_exr(const char *path, const float *pixels, int32_t width, int32_t height, int32_t channels,
                            int32_t half)
{
    g_config_error.clear();
    if (!path || !pixels || width <= 0 || height <= 0 || channels < 1 || channels > 4) {
        g_config_error = "ks_image_save_exr: bad argument";
        return KS_ERR_INVALID_ARGUMENT;
    }
    try {
        ksb::image::write_exr(path, pixels, width, height, channels, half != 0);
        return KS_OK;
    } catch (const std::exception &e) {
        g_config_error = e.what();
        return KS_ERR_IO;
    }
}

ks_status ks_texture_load(const char *path, int32_t channels, int32_t srgb, int32_t keep_16bit,
                          ks_texture_desc *out)
{
    g_config_error.clear();
    if (!path || !out || channels < 1 || channels > 4) {
        g_config_error = "ks_texture_load: null argument or channels outside 1-4";
        return KS_ERR_INVALID_ARGUMENT;
    }
    *out = ks_texture_desc{};
    try {
        ksb::gltf::Texture t = ks_b200::load_texture_file(path, channels, srgb != 0, keep_16bit != 0);
        void *texels = std::malloc(t.bytes.size());
        if (!texels)
            return KS_ERR_OUT_OF_MEMORY;
        std::memcpy(texels, t.bytes.data(), t.bytes.size());
        out->texels = texels;
        out->width = (uint32_t)t.width;
        out->height = (uint32_t)t.height;
        out->channels = (uint32_t)t.channels;
        out->format = t.format;
        out->srgb = t.srgb ? 1 : 0;
        return KS_OK;
    } catch (const ksb::image::Error &e) {
        g_config_error = e.what();
        return e.unsupported ? KS_ERR_UNSUPPORTED : KS_ERR_IO;
    } catch (const std::exception &e) {
        g_config_error = e.what();
        return KS_ERR_IO;
    }
}

void ks_texture_free(ks_texture_desc *t)
{
    if (!t)
        return;
    std::free(const_cast<void *>(t->texels));
    t->texels = nullptr;
}

ks_status ks_image_load_rgb(const char *path, float **pixels, int32_t *width, int32_t *height)
{
    g_config_error.clear();
    if (!path || !pixels || !width || !height) {
        g_config_error = "ks_image_load_rgb: null argument";
        return KS_ERR_INVALID_ARGUMENT;
    }
    *pixels = nullptr;
    try {
        int w = 0, h = 0;
        std::vector<float> rgb = ksb::image::read_rgb(path, w, h);
        float *out = static_cast<float *>(std::malloc(sizeof(float) * rgb.size()));
        if (!out)
            return KS_ERR_OUT_OF_MEMORY;
        std::memcpy(out, rgb.data(), sizeof(float) * rgb.size());
        *pixels = out;
        *width = w;
        *height = h;
        return KS_OK;
    } catch (const ksb::image::Error &e) {
        g_config_error = e.what();
        return e.unsupported ? KS_ERR_UNSUPPORTED : KS_ERR_IO;
    } catch (const std::exception &e) {
        g_config_error = e.what();
        return KS_ERR_IO;
    }
}

void ks_image_free(float *pixels) { std::free(pixels); }

} // extern "C"
