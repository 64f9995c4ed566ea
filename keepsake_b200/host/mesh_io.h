// Mesh files of keepsake's mesh assets (mesh_asset.cpp): Wavefront OBJ (load_from_obj,
// mesh_asset.cpp:70-178) and the binary mesh asset (load_from_binary / write_to_binary,
// mesh_asset.cpp:180-240), plus the `to_world` transform create_mesh_asset applies
// (MeshData::transform, geometry.cpp:15-32).
#pragma once
#include <cstdint>
#include <filesystem>
#include <stdexcept>
#include <string>
#include <vector>

namespace ksb
{
namespace mesh
{

struct Error : std::runtime_error
{
    using std::runtime_error::runtime_error;
};

// One MeshData: positions, triangles and the optional per-vertex attributes (empty when absent).
struct MeshData
{
    std::vector<float> vertices;  // 3 per vertex
    std::vector<uint32_t> indices; // 3 per triangle
    std::vector<float> texcoords; // 2 per vertex or empty
    std::vector<float> normals;   // 3 per vertex or empty
    bool twosided = false;
    bool use_smooth_normal = true;
    std::string name;
    uint32_t vertex_count() const { return (uint32_t)(vertices.size() / 3); }
    uint32_t tri_count() const { return (uint32_t)(indices.size() / 3); }
};

// Every `o` / `g` statement starts a mesh (a tinyobj shape); faces (v, v/t, v//n, v/t/n, negative
// indices) are fanned into triangles; vertices are the distinct (position, texcoord, normal)
// index triples of a mesh in the order they first appear; a mesh's faces carry texcoords (and
// normals) at all of their corners or at none.
std::vector<MeshData> load_obj(const std::filesystem::path &path, bool twosided, bool use_smooth_normal);

// "i_am_a_binary_mesh_asset", int32 mesh count, then per mesh: bool twosided, bool
// use_smooth_normal, int32 vertex count V, int32 triangle count T, bool has_texcoord, bool
// has_vertex_normal, float[3V + 1] positions, uint32[3T] indices, [float[2V + 2] texcoords],
// [float[3V + 1] normals] (the trailing floats are the padding the reference keeps for Embree).
std::vector<MeshData> load_binary(const std::filesystem::path &path);
void write_binary(const std::filesystem::path &path, const std::vector<MeshData> &meshes);

// Points through the transform m (row-major 4x4, affine), normals through the inverse transpose
// of its 3x3 block, normalised (Transform::point / Transform::normal, maths.h:979-987).
void transform(std::vector<MeshData> &meshes, const float m[16]);

} // namespace mesh
} // namespace ksb
