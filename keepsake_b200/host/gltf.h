// glTF 2.0 compound mesh assets (CompoundMeshAsset::load_from_gltf, mesh_asset.cpp:551-1091;
// create_compound_mesh_asset, mesh_asset.cpp:1114-1132): each glTF mesh a prototype whose
// primitives are its meshes, each node with a mesh an instance under the node's world transform
// (traverse_gltf_scene_graph, mesh_asset.cpp:466-520), and, with load_materials, the
// primitives' metallic-roughness materials as principled BSDFs with constant fields.
//
// .gltf (JSON, buffers in files next to it or in base64 data URIs) and .glb (binary container).
// Textures: PNG images (8- and 16-bit) bound to the base colour, metallic-roughness, specular,
// transmission, normal and (for emitters) emissive slots with the nearest filter, and alpha modes
// other than OPAQUE as opacity maps.  Not handled, each an error marked unsupported: JPEG and other
// image formats, samplers with a mipmap minification filter (EWA filtering), sparse accessors,
// non-triangle primitives, index types other than unsigned short / unsigned int (the reference
// asserts on those too).  Animations are not
// read (camera and transform animation are outside the small_pt path).
#pragma once
#include "../../include/ks_b200.h"
#include "mesh_io.h"

#include <filesystem>
#include <stdexcept>
#include <string>
#include <vector>

namespace ksb
{
namespace gltf
{

struct Error : std::runtime_error
{
    bool unsupported;
    Error(const std::string &what, bool unsupported = false) : std::runtime_error(what), unsupported(unsupported) {}
};

// A decoded texture image: width x height x channels samples of `format` (0 u8, 1 u16, 2 f32).
struct Texture
{
    int width = 0, height = 0, channels = 0, format = 0;
    bool srgb = false;
    std::vector<uint8_t> bytes;
};

struct Prototype
{
    std::vector<mesh::MeshData> meshes;        // one per primitive
    std::vector<ks_material_desc> materials;   // one per primitive (load_materials), else empty
    // textured fields of the materials (load_textures): `material` is the primitive's index in
    // this prototype, `texture` an index into Compound::textures
    std::vector<ks_texture_binding> bindings;
};

struct Instance
{
    uint32_t prototype;
    float to_world[12]; // row-major 3x4
};

struct Compound
{
    std::vector<Prototype> prototypes;
    std::vector<Instance> instances;
    std::vector<Texture> textures;
};

// load_textures: textured materials read their PNG images (see material() in gltf.cpp); without
// it a textured material is an unsupported-status error.
Compound load(const std::filesystem::path &path, bool load_materials, bool load_textures = true);

// CameraAnimation (camera.h:44-61, camera.cpp:207-465): the translation and rotation keys of a
// named perspective camera's node in a .glb file, evaluated with linear interpolation of the
// translation and spherical interpolation of the rotation (CameraAnimation::eval).
struct CameraAnimation
{
    float vfov = 0.0f, aspect = 1.0f;
    std::vector<float> translation_keys, translation_values; // 3 values per key
    std::vector<float> rotation_keys, rotation_values;       // x, y, z, w per key
    uint32_t n_frames() const { return (uint32_t)translation_keys.size(); }
    float duration() const { return translation_keys.empty() ? 0.0f : translation_keys.back(); }
    // camera-to-world (row-major 4x4) at `time`
    void eval(float time, float camera_to_world[16]) const;
};

// create_camera_animation (camera.cpp:276-465): camera `name` found depth first in the default
// scene; the first animation that drives its node's translation or rotation (the search stops at
// one that drives both); convert_y_up_to_z_up turns the keys by convert_yup_to_zup (maths.h:916-927).
CameraAnimation load_camera_animation(const std::filesystem::path &path, const std::string &name,
                                      bool convert_y_up_to_z_up);

} // namespace gltf
} // namespace ksb
