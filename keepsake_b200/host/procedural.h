// Seeded procedural scenes used as synthetic inputs (host side).
#pragma once
#include "../../include/ks_b200.h"

#include <cstdint>
#include <string>
#include <vector>

namespace ksb
{

struct ProceduralOptions
{
    int level = 8;               // icosphere subdivision level
    float roughness_min = 0.05f; // per-patch roughness range
    float roughness_max = 1.0f;
    int occluder = 0;            // slab between sphere and sun
    uint32_t sky_width = 2048;
    uint32_t sky_height = 1024;
    uint32_t width = 1024; // render resolution (sets the camera aspect)
    uint32_t height = 1024;
    // "instanced": prototypes, instances, geodesic frequency (20 f^2 triangles per prototype),
    // emissive triangles
    uint32_t prototypes = 8;
    uint32_t instances = 400;
    uint32_t frequency = 50;
    uint32_t emitters = 64;
    bool geodesic_sphere = false; // "icosphere": a geodesic sphere of `frequency` instead of `level`
};

struct GeneratedMesh
{
    std::vector<float> vertices;
    std::vector<uint32_t> indices;
    uint32_t material = 0;
    std::vector<float> normals;   // 3 per vertex or empty (loaded assets)
    std::vector<float> texcoords; // 2 per vertex or empty
    int twosided = 1;
    int use_smooth_normal = 1;
};

struct GeneratedScene
{
    std::vector<GeneratedMesh> meshes;
    std::vector<ks_material_desc> materials;
    std::vector<float> sky_map;
    ks_sky_desc sky{};
    std::vector<ks_mesh_desc> mesh_descs;
    std::vector<ks_prototype_desc> prototypes; // empty: flat scene
    std::vector<ks_instance_desc> instances;
    // textures (loaded assets): texels per texture, described by `textures` (texels set by
    // finalize), and the bindings of textured material fields
    std::vector<std::vector<uint8_t>> texture_bytes;
    std::vector<ks_texture_desc> textures;
    std::vector<ks_texture_binding> bindings;
    ks_scene_desc desc{};
    float camera_to_world[16]{};
    float vfov = 0.7f;
    float aspect = 1.0f;
    uint32_t width = 256, height = 256;
    void finalize();
};

bool generate_scene(const std::string &kind, uint64_t seed, const ProceduralOptions &opts, GeneratedScene &out);

} // namespace ksb
