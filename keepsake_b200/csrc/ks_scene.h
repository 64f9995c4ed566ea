// Device-resident scene: geometry, SBVH (reference layout + traversal layout), materials, lights.
#pragma once
#include "ks_internal.h"
#include "ks_math.cuh"
#include "ks_texture.cuh"

#include <vector>

namespace ksb
{

// SBVH node in the reference's flattened layout (cuda/sbvh.cuh:18-28), kept for export/parity.
struct RefNode
{
    float bmin[3];
    float bmax[3];
    uint32_t axis;
    uint32_t right; // 0 = leaf
    uint32_t prim_offset;
};

// Traversal node: an interior node of the flattened SBVH with both children's boxes (64 bytes).
//   a = (L.min.x, L.min.y, L.min.z, L.max.x)   b = (L.max.y, L.max.z, R.min.x, R.min.y)
//   c = (R.min.z, R.max.x, R.max.y, R.max.z)   d = (L.ref, R.ref, L.count | axis << 30, R.count)
// A child ref with the top bit set is a leaf: (ref & 0x7fffffff) is its first primitive slot.
struct TravNode
{
    float4 a, b, c;
    uint4 d;
};
constexpr uint32_t kLeafBit = 0x80000000u;

// 4-wide view of the same SBVH, read by the renderer's traversal kernels: wide node i holds the
// children of interior node i, each interior child replaced by its own two children (2 to 4 slots).
// Slot boxes are the SBVH's boxes of those nodes; unused slots hold an empty box (lo +inf, hi -inf),
// which the slab test always rejects.  Indexed like the TravNode array (entries of nodes at odd
// depth are written but never read), so child refs need no renumbering.
struct WideNode
{
    float4 lo[3]; // per axis: the 4 slots' lower bounds
    float4 hi[3]; // per axis: the 4 slots' upper bounds
    uint4 ref;    // child refs (kLeafBit: leaf, first primitive slot)
    uint4 cnt;    // primitive counts of leaf children
};
static_assert(sizeof(WideNode) == 128, "one 128-byte line per wide node");

// Per-mesh shading flags (MeshData::twosided; use_smooth_normal with vertex normals given;
// texcoords given).
enum : int
{
    kMeshTwosided = 1,
    kMeshSmooth = 2,
    kMeshTexcoords = 4
};

// Device copy of one material (constant principled fields + emission).
struct MaterialGPU
{
    float basecolor[3];
    float roughness, metallic, ior, specular_r0_mul, specular_trans, diffuse_trans, diffuse_trans_fwd;
    int microfacet; // 0 GGX, 1 Beckmann
    int has_emission;
    float emission[3];
    int mesh_light; // index of the MeshLightShared for emissive meshes, -1 otherwise
    int bsdf;       // 0 PrincipledBSDF, 1 PrincipledBRDF, 2 Lambertian (albedo = basecolor)
    float specular; // PrincipledBRDF's specular field
    int bind_begin, bind_count; // the material's texture bindings (SceneView::bindings)
    int tex_flags;              // kMatNormalMap | kMatOpacityMap | kMatEmissionMap
    int has_ss;                 // a BSSRDF (ks_material_desc.has_subsurface)
    float ss_albedo[3], ss_radius[3], ss_g, ss_ior, ss_rfr;
};
enum : int
{
    kMatNormalMap = 1,
    kMatOpacityMap = 2,
    kMatEmissionMap = 4
};

struct SceneHost
{
    std::vector<uint32_t> mesh_tri_offset; // first global triangle of each mesh (+ total at the end)
    std::vector<uint32_t> mesh_material;
    std::vector<int> mesh_flags; // kMeshTwosided | kMeshSmooth | kMeshTexcoords (ks_wavefront.cuh)
    std::vector<ks_material_desc> materials;
    // instancing (empty: flat scene)
    std::vector<uint32_t> proto_tri_begin, proto_tri_end; // global triangle range of each prototype
    std::vector<uint32_t> inst_proto;
    std::vector<float> inst_xf, inst_inv; // 12 floats (row-major 3x4) per instance
};


} // namespace ksb

struct ks_scene
{
    ks_context *ctx = nullptr;
    uint32_t n_tris = 0;
    uint32_t n_verts = 0;
    ksb::SceneHost host;
    // geometry, concatenated over meshes: vertices (float3), indices (uint3, global vertex ids),
    // per-triangle mesh id
    ksb::DevBuf<float> verts;
    ksb::DevBuf<uint32_t> indices;
    ksb::DevBuf<uint32_t> tri_mesh;
    // SBVH in the reference layout + ordered primitive list
    ksb::DevBuf<ksb::RefNode> ref_nodes;
    ksb::DevBuf<uint32_t> prims;
    uint32_t n_nodes = 0, n_prims = 0;
    // traversal layout
    ksb::DevBuf<ksb::TravNode> trav_nodes;
    ksb::DevBuf<ksb::WideNode> wide_nodes; // the 4-wide view of trav_nodes
    ksb::DevBuf<float4> prim_tris; // 3 float4 per primitive slot: v0 (+tri index bits in w), v1, v2
    uint32_t n_trav = 0;
    uint32_t root_ref = 0;   // ref of the root (leaf bit when the whole tree is one leaf)
    uint32_t root_count = 0; // prim count of the root
    bool bvh_built = false;
    float scene_bound[6] = {0, 0, 0, 0, 0, 0};
    // materials (device copies of the per-mesh tables)
    ksb::DevBuf<ksb::MaterialGPU> materials;
    ksb::DevBuf<uint32_t> mesh_material;
    ksb::DevBuf<int> mesh_flags;
    bool ext_materials = false; // some material is not a GGX PrincipledBSDF
    // textures (linear float texels, 4 per texel), their sizes, the bindings grouped by material
    ksb::DevBuf<float4> tex_texels;
    ksb::DevBuf<ksb::TexInfo> tex_info;
    ksb::DevBuf<ksb::BindingGPU> bindings;
    bool any_bindings = false, any_opacity = false;
    // host copies for the light build of textured emitters (filled only when some emitter has an
    // emission texture): converted texels, texture sizes, bindings, materials, texcoords
    struct EmissionTextures
    {
        std::vector<float4> texels;
        std::vector<ksb::TexInfo> info;
        std::vector<ksb::BindingGPU> binds;
        std::vector<ksb::MaterialGPU> mats;
        std::vector<float> texcoords; // 2 per global vertex (zeros for meshes without)
    } emit_tex;
    bool any_emission_map = false;
    bool any_subsurface = false; // some material has a BSSRDF
    // per-vertex shading attributes, indexed like verts (allocated only when some mesh has them)
    ksb::DevBuf<float> normals;   // 3 per vertex: MeshData::vertex_normals of smooth-shaded meshes
    ksb::DevBuf<float> texcoords; // 2 per vertex: MeshData::texcoords
    // lights (PowerLightSampler over [sky] + mesh-light triangles)
    bool lights_built = false;
    uint32_t light_count = 0, n_nonmesh = 0;
    std::vector<float> h_powers, h_power_cdf;
    ksb::DevBuf<float> power_cdf;
    ksb::DevBuf<int32_t> tri_light;
    ksb::DevBuf<uint32_t> ml_tri;
    ksb::DevBuf<float> ml_area;
    ksb::DevBuf<float4> ml_emission;
    // sky
    ks_sky_desc sky_desc{};
    std::vector<ks_light_desc> lights; // point / directional lights, after the sky in the light list
    ksb::DevBuf<float4> punctual;      // per light: (vec, type), (color, 0)
    ksb::DevBuf<float> sky_rgb;   // kinds 2, 3: the map as given (3 floats per texel), for the light build
    std::vector<float> sky_host;  // kind 3: the equal-area map on the host, for its alias table
    ksb::DevBuf<float4> sky_alias; // kind 3: alias-table bins (q, p, alias bits, 0) over the texels
    float sky_l2w[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1}, sky_w2l[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
    ksb::DevBuf<float4> sky_map;
    ksb::DevBuf<float> sky_cond, sky_margin;
    ksb::DevBuf<uint32_t> sky_cond_guide, sky_margin_guide;
    int sky_w = 0, sky_h = 0;
    ks_render_stats last_stats{};
    // instancing: per-prototype BLAS roots inside trav_nodes / prim_tris, a TLAS over instances
    uint32_t n_instances = 0, n_protos = 0;
    ksb::DevBuf<float> inst_xf, inst_inv;   // 12 floats per instance
    ksb::DevBuf<uint32_t> inst_proto;
    ksb::DevBuf<uint4> proto_root;          // (root ref, root count) per prototype
    ksb::DevBuf<float> proto_bound;         // 6 floats per prototype
    ksb::DevBuf<ksb::TravNode> tlas_nodes;
    ksb::DevBuf<uint32_t> tlas_items;       // instance ids in TLAS leaf order
    uint32_t tlas_root_ref = 0, tlas_root_count = 0;
    ksb::DevBuf<int32_t> inst_light_base;   // per instance: flat index of its first mesh light
    ksb::DevBuf<float4> ml_verts;           // 3 per mesh light: world-space vertices
};

namespace ksb
{
bool material_to_gpu(const ks_material_desc &m, MaterialGPU &g);
ks_status build_sbvh(ks_scene *scene, const ks_sbvh_options &opts, float *build_ms);
ks_status build_lights(ks_scene *scene);
}
