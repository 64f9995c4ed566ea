/* keepsake-b200: C ABI of the B200-native small_pt path tracer.
 *
 * The entry points replace the parts of keepsake's CPU `small_pt` path that a C/C++ host calls
 * (reference interfaces cited per function).  Plain C types only; every call returns a
 * ks_status and never aborts; host pointers unless a name says `device`.
 *
 * Threading: a context owns one CUDA stream.  Calls on one context must not overlap; distinct
 * contexts may be used from distinct threads.
 */
#ifndef KS_B200_H
#define KS_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum ks_status {
    KS_OK = 0,
    KS_ERR_INVALID_ARGUMENT = 1,
    KS_ERR_OUT_OF_MEMORY = 2,
    KS_ERR_CUDA = 3,
    KS_ERR_QUEUE_OVERFLOW = 4,
    KS_ERR_WATCHDOG = 5,
    KS_ERR_NOT_BUILT = 6,
    KS_ERR_UNSUPPORTED = 7,
    KS_ERR_PARSE = 8,
    KS_ERR_IO = 9,
} ks_status;

typedef struct ks_context ks_context;

/* Context: one CUDA device + one stream.  (Replaces the reference's implicit global state:
 * EmbreeDevice in small_pt.cpp:182 and the TBB arena of parallel.h:93-113.)  The context keeps the
 * scratch of its SBVH builds and the buffers of its renders (wavefront state, about 300 bytes per
 * path slot up to 32 M slots, the accumulators and a pinned staging copy of them) from one call to
 * the next, and frees them in ks_context_destroy.  One thread at a time per context.
 * Device memory comes from a pool per GPU that keeps freed blocks for reuse (a scene destroyed
 * and a new one created reuse the same memory without the driver's allocator); ks_context_destroy
 * returns the pool's free blocks to the driver. */
ks_status ks_context_create(int device, ks_context **out);
void ks_context_destroy(ks_context *ctx);
const char *ks_status_string(ks_status s);
/* Detail message of the last failing call on this context ("" if none). */
const char *ks_last_error(const ks_context *ctx);

/* Failure-detection limits of a context, for tests of the error paths (the reference aborts on its
 * failures instead: ASSERT, cuda_check, the Embree error handler).  Each limit ends a loop that
 * would otherwise run longer with a status code, and the context stays usable afterwards.  0
 * keeps the library's own bound.
 *   sbvh_max_levels:          SBVH build levels (own bound 4096) -> KS_ERR_WATCHDOG from
 *                             ks_scene_build_bvh, the scene stays unbuilt;
 *   wavefront_max_iterations: wavefront iterations per spp interval of a render, and per batch
 *                             (own bound: (paths / path slots + 2) x (bounces + 2) + 64) ->
 *                             KS_ERR_WATCHDOG from the render.
 * ks_context_set_limits(ctx, NULL) restores the defaults. */
typedef struct ks_context_limits {
    uint32_t sbvh_max_levels;
    uint32_t wavefront_max_iterations;
} ks_context_limits;
ks_status ks_context_set_limits(ks_context *ctx, const ks_context_limits *limits);

/* The bounded mbarrier wait of the tensor-core kernels (the guide network's MMA completion wait)
 * run on its own: one CTA initialises an mbarrier for one arrival, arrives on it when `arrive` is
 * nonzero, and waits for its phase with at most max_polls try_wait polls.  KS_OK when the phase
 * completed, KS_ERR_WATCHDOG when the polls ran out (nothing arrives when arrive = 0; no
 * asynchronous operation is in flight, so the kernel returns cleanly).  No reference counterpart:
 * it tests the timeout path that keeps a lost completion from hanging the GPU. */
ks_status ks_mbarrier_wait_probe(ks_context *ctx, uint32_t max_polls, int arrive);

/* Sobol parity hook.  For every pixel (x0..x0+nx-1, y0..y0+ny-1), sample index s0..s0+ns-1 and
 * dimension d in 0..nd-1 it starts a PTRenderSampler(full_res, pixel, spp, s, seed) at dimension d
 * (sobol.h:235-241 + start_pixel :140) and writes three floats:
 *   out[0] = sobol.next()   (sobol.h:148-156)
 *   out[1..2] = sobol.next2d() (sobol.h:158-167), each from a fresh sampler at dimension d.
 * Layout: out[(((py * nx + px) * ns + s) * nd + d) * 3 + c], host memory. */
ks_status ks_sobol_points(ks_context *ctx, uint32_t full_width, uint32_t full_height, uint32_t spp, uint32_t seed,
                          uint32_t x0, uint32_t y0, uint32_t nx, uint32_t ny, uint32_t s0, uint32_t ns, uint32_t nd,
                          float *out);

/* Sobol parity hook for the renderer's per-bounce draw.  For every pixel and sample index of the
 * window above it starts the sampler at dimension dim and writes the seven values one path vertex
 * draws, in the order next(), next2d(), next(), next2d(), next() (light selection, light uv, BSDF
 * lobe, BSDF direction, roulette: nee.cpp:28-34, material.cpp:157-158, small_pt.cpp:168-174),
 * through the same code as the sampling kernel.  Layout: out[((py * nx + px) * ns + s) * 7 + c]. */
ks_status ks_sobol_bounce(ks_context *ctx, uint32_t full_width, uint32_t full_height, uint32_t spp, uint32_t seed,
                          uint32_t x0, uint32_t y0, uint32_t nx, uint32_t ny, uint32_t s0, uint32_t ns, uint32_t dim,
                          float *out);

/* ---------------------------------------------------------------------------------------------
 * Scene description (host arrays; ks_scene_create copies everything it needs to the device).
 * One mesh = one reference `MeshGeometry` with one `Material` (scene.cpp:315-336 pairs
 * subscene.geometries[geom_id] with subscene.materials[geom_id]).
 * ------------------------------------------------------------------------------------------- */
typedef struct ks_mesh_desc {
    const float *vertices;       /* 3 floats per vertex */
    uint32_t n_vertices;
    const uint32_t *indices;     /* 3 per triangle */
    uint32_t n_triangles;
    const float *vertex_normals; /* optional, 3 per vertex (object space); the shading frame
                                    follows the interpolated normal when use_smooth_normal != 0
                                    (geometry.cpp:139-156); NULL = flat shading */
    uint32_t material;           /* index into ks_scene_desc.materials */
    int32_t twosided;            /* MeshData::twosided (geometry.h:84); reference default 1 */
    int32_t use_smooth_normal;   /* MeshData::use_smooth_normal (geometry.h:85) */
    const float *texcoords;      /* optional, 2 per vertex (MeshData::texcoords); when given, the
                                    frame's tangent is dP/du of this parameterisation
                                    (geometry.cpp:94-116); NULL = dP/du of the barycentrics */
} ks_mesh_desc;

/* A material's BSDF with constant shader fields plus the Material::emission field
 * (material.h:45), which the TOML task reads from an `emission` key.  bsdf selects the reference
 * type (create_bsdf, bsdf.cpp:50-62):
 *   0 PrincipledBSDF (principled_bsdf.cpp:707-733): every field below but `specular`;
 *   1 PrincipledBRDF (principled_bsdf.cpp:227-244): basecolor, roughness, metallic, specular,
 *     microfacet;
 *   2 Lambertian (bsdf.cpp:43-48): albedo = basecolor.
 * Zero-initialise the descriptor before filling it: the fields after `emission` were added later
 * and zero selects PrincipledBSDF; out-of-range enums are KS_ERR_INVALID_ARGUMENT. */
typedef struct ks_material_desc {
    float basecolor[3];
    float roughness;
    float metallic;
    float ior;
    float specular_r0_mul;
    float specular_trans;
    float diffuse_trans;
    float diffuse_trans_fwd;
    float emissive[3];
    int32_t microfacet;   /* 0 GGX, 1 Beckmann (microfacet.h:20-257) */
    int32_t has_emission; /* Material::emission != nullptr */
    float emission[3];
    int32_t bsdf;         /* 0 principled_bsdf, 1 principled_brdf, 2 lambertian */
    float specular;       /* principled_brdf: specular, clamped to [0, 1] and scaled by 0.08 */
    /* Material::subsurface (a BSSRDF, subsurface.h:35-43; create_bssrdf, subsurface.cpp:536-545):
     * at each hit the material picks its BSDF or, with probability 1/2, a random walk inside its
     * mesh (subsurface_random_walk, subsurface.cpp:222-500) whose exit point shades with a
     * Lambertian exit lobe (material.cpp:101-160).  Flat scenes, materials without emission. */
    int32_t has_subsurface;
    float ss_albedo[3];      /* BSSRDF::albedo, clamped to [0, 1] */
    float ss_radius[3];      /* BSSRDF::radius: mean free path per channel (scene units) */
    float ss_anisotropy;     /* Henyey-Greenstein g of the walk, in (-1, 1) */
    float ss_ior;            /* BSSRDF::ior (> 0) */
    float ss_rfr_entry_prob; /* probability of the refractive entry (else a cosine entry) */
} ks_material_desc;

/* The sky light: SkyLight (light.h:34-58), an ambient colour or a lat-long RGB map, or
 * EqualAreaSkyLight (light.h:60-86, light.cpp:161-206), a square map in the equal-area octahedral
 * parameterisation of the sphere sampled through an alias table over its texels' luminance (its
 * sample / pdf / eval as the reference's GPU path defines them, gpu/shaders/light.slang:92-186;
 * the reference's CPU path leaves them unimplemented). */
typedef struct ks_sky_desc {
    int32_t kind;         /* 0 none, 1 ambient, 2 lat-long map, 3 equal-area map */
    float ambient[3];
    const float *map_rgb; /* width*height*3 floats; lat-long: row 0 = theta 0 (light.cpp:33-40);
                             equal-area: width = height, a power of two, at most 16384 */
    uint32_t width;
    uint32_t height;
    float to_world[16];   /* row-major 4x4 light-to-world (equal-area: its 3x3 part, a rotation) */
    int32_t transform_y_up; /* lat-long maps only */
    float strength;
} ks_sky_desc;

/* Instancing (Scene::subscenes / SubSceneInstance, scene.h:27-49): a prototype is a run of
 * consecutive meshes (one SubScene); an instance places a prototype with an affine object-to-
 * world transform (row-major 3x4; the inverse is computed in double).  Mesh lights of instanced
 * prototypes are one light per (instance, emissive triangle), like Scene::build_mesh_lights
 * (scene.cpp:315-336).  Meshes that belong to no prototype are not rendered. */
typedef struct ks_prototype_desc {
    uint32_t first_mesh;
    uint32_t n_meshes;
} ks_prototype_desc;

typedef struct ks_instance_desc {
    uint32_t prototype;
    float to_world[12];
} ks_instance_desc;

/* Point and directional lights (PointLight / DirectionalLight, light.h:91-123, light.cpp:208-240;
 * create_point_light / create_directional_light, light.cpp:285-305): delta lights, sampled by
 * next-event estimation only (MIS weight 1, nee.cpp:45-48), ordered after the sky in the light
 * list of PowerLightSampler with powers 4 pi I and L pi r^2 (r: half the scene box diagonal). */
typedef struct ks_light_desc {
    int32_t type;    /* 0 point, 1 directional */
    float color[3];  /* I (point intensity) or L (directional radiance) */
    float vec[3];    /* point: position; directional: unit direction toward the light */
} ks_light_desc;

/* ---------------------------------------------------------------------------------------------
 * Textures and textured shader fields (Texture, texture.h:43-65; TextureField, shader_field.h:38-86;
 * NormalMap, normal_map.cpp:9-40; OpacityMap, opacity_map.cpp:6-30).
 * ------------------------------------------------------------------------------------------- */
/* A texture without mipmaps (create_texture with build_mipmaps = false, texture.cpp:1068-1084):
 * width x height texels of `channels` values, rows first, in `format`; sRGB-encoded texels are read
 * as linear (Texture::fetch_as_float, texture.cpp:403-460). */
typedef struct ks_texture_desc {
    const void *texels;
    uint32_t width;
    uint32_t height;
    uint32_t channels; /* 1..4 */
    int32_t format;    /* 0 u8, 1 u16, 2 f32 (TextureDataType) */
    int32_t srgb;      /* 1: ColorSpace::sRGB */
} ks_texture_desc;

/* What a texture binding drives: a shader field of the material's BSDF (the constant value in
 * ks_material_desc is then ignored), the material's normal map, its opacity map or its emission. */
enum {
    KS_FIELD_BASECOLOR = 0, /* 3 channels; Lambertian: albedo */
    KS_FIELD_ROUGHNESS = 1,
    KS_FIELD_METALLIC = 2,
    KS_FIELD_IOR = 3,
    KS_FIELD_SPECULAR_R0_MUL = 4,
    KS_FIELD_SPECULAR_TRANS = 5,
    KS_FIELD_DIFFUSE_TRANS = 6,
    KS_FIELD_DIFFUSE_TRANS_FWD = 7,
    KS_FIELD_SPECULAR = 8,   /* PrincipledBRDF's specular */
    KS_FIELD_NORMAL_MAP = 9, /* Material::normal_map (material.h:41) */
    KS_FIELD_OPACITY_MAP = 10, /* Material::opacity_map (material.h:42): stochastic any-hit test */
    KS_FIELD_EMISSION = 11     /* Material::emission of an emitter (has_emission = 1; 3 channels, in place
                                  of ks_material_desc.emission): its triangles' light-selection power
                                  comes from a summed-area table of the texture's luminance
                                  (compute_mesh_light_importance, light.cpp:307-522) */
};

/* A texture bound to a material: the TextureField's lookup (flip_v, uv_scale, uv_offset, the
 * sampler, swizzle, scale) and, for normal maps, NormalMap's parameters.  Zero-initialise, then set
 * every field: the reference's defaults (create_texture_shader_field_color, create_texture_sampler,
 * create_normal_map) are flip_v 1, uv_scale (1, 1), uv_offset (0, 0), swizzle (0, 1, 2, 3),
 * scale (1, 1, 1, 1), repeat wrapping, tangent space, range01 1, strength 1, to_world identity. */
typedef struct ks_texture_binding {
    uint32_t material;   /* index into ks_scene_desc.materials */
    int32_t field;       /* KS_FIELD_* */
    uint32_t texture;    /* index into ks_scene_desc.textures */
    int32_t filter;      /* 0 nearest (NearestSampler), 1 linear (LinearSampler), 2 cubic (CubicSampler);
                            textures have one level, so linear is bilinear and cubic bicubic at level 0 */
    int32_t cubic_kernel; /* 0 Mitchell-Netravali, 1 B-spline, 2 Catmull-Rom (texture.h:91-121) */
    int32_t wrap_u;      /* 0 repeat, 1 clamp (TextureWrapMode) */
    int32_t wrap_v;
    int32_t flip_v;      /* TextureField::flip_v (reference default true) */
    int32_t swizzle[4];  /* output channel c reads texel channel swizzle[c]; -1: 0 */
    float uv_scale[2];
    float uv_offset[2];
    float scale[4];      /* TextureField::scale */
    /* normal maps (create_normal_map, normal_map.cpp:42-56) */
    int32_t normal_space; /* 0 tangent, 1 world */
    int32_t range01;      /* 1: texel values in [0, 1] are remapped to [-1, 1] */
    float strength;       /* tangent space: lerp from (0, 0, 1) toward the mapped normal */
    float to_world[16];   /* world space: the map's to_world (row-major 4x4; normals by its inverse transpose) */
} ks_texture_binding;

typedef struct ks_scene_desc {
    const ks_mesh_desc *meshes;
    uint32_t n_meshes;
    const ks_material_desc *materials;
    uint32_t n_materials;
    ks_sky_desc sky;
    /* n_instances = 0: every mesh, untransformed (one implicit identity instance) */
    const ks_prototype_desc *prototypes;
    uint32_t n_prototypes;
    const ks_instance_desc *instances;
    uint32_t n_instances;
    const ks_light_desc *lights; /* the task's `light` list (small_pt.cpp:186-199); may be NULL */
    uint32_t n_lights;
    /* textures and their bindings to materials (may be NULL / 0).  Textured emission and the
     * instanced scenes' textured materials are KS_ERR_UNSUPPORTED. */
    const ks_texture_desc *textures;
    uint32_t n_textures;
    const ks_texture_binding *bindings;
    uint32_t n_bindings;
} ks_scene_desc;

/* SBVHBuildOption (cuda/sbvh.cuh:9-16); clamped like SBVH::build (cuda/sbvh.cu:411-414). */
typedef struct ks_sbvh_options {
    uint32_t max_prims_in_node; /* default 4, clamped to <= 8 */
    uint32_t bucket_count;      /* default 12, clamped to <= 16 */
    float trav_weight;          /* default 1, clamped to [0, 10] */
    float alpha;                /* default 1e-5, clamped to [0, 1] */
} ks_sbvh_options;

typedef struct ks_scene ks_scene;

/* Copies the scene to the device and builds the light tables (Scene::build_mesh_lights,
 * scene.cpp:315; PowerLightSampler::build, light.cpp:636; SkyLight, light.cpp:19-49). */
ks_status ks_scene_create(ks_context *ctx, const ks_scene_desc *desc, ks_scene **out);
void ks_scene_destroy(ks_scene *scene);

/* Parallel SBVH build on the GPU over all triangles of the scene, concatenated in mesh order.
 * Replaces ksc::SBVH::build (cuda/sbvh.cu:404-440) and Embree's rtcCommitScene (scene.cpp:60).
 * opts may be NULL (defaults).  build_ms (optional) receives the device time of the build. */
ks_status ks_scene_build_bvh(ks_scene *scene, const ks_sbvh_options *opts, float *build_ms);

/* Counts of the flattened SBVH (cuda/sbvh.cuh:90-93): nodes and ordered primitive references. */
ks_status ks_sbvh_counts(const ks_scene *scene, uint32_t *n_nodes, uint32_t *n_prims);

/* Copies the flattened SBVH to host arrays in the reference's layout (SBVHNode, sbvh.cuh:18-28):
 * bounds 6 floats/node (min xyz, max xyz), split axis, rightChildOffset (0 = leaf), primOffset,
 * and the ordered primitive list (global triangle index per reference). */
ks_status ks_sbvh_export(const ks_scene *scene, float *node_bounds, uint32_t *node_axis, uint32_t *node_right,
                         uint32_t *node_prim_offset, uint32_t *prims);

/* Ray-query parity hook: SBVH::intersect / intersectBool (cuda/sbvh.cu:512-603) over a batch of
 * host rays, 8 floats each (ox oy oz tmin dx dy dz tmax).  any_hit = 0: tri_idx = global triangle
 * index or 0xFFFFFFFF, t and bary (3 per ray) filled; any_hit = 1: tri_idx = 1 occluded / 0 not.
 * culling: 0 back faces, 1 front faces, 2 none (SBVHCulling, sbvh.cuh:30-35). */
ks_status ks_trace_rays(ks_scene *scene, const float *rays, uint32_t n, int any_hit, int culling, uint32_t *tri_idx,
                        float *t, float *bary);

/* The same queries through the renderer's traversal kernels.  Flat scenes: a 4-wide view of the
 * same SBVH (each node with its interior children replaced by theirs, boxes tested with the same
 * slab test), nearest slot first; it reaches the same leaves, so the result equals
 * ks_trace_rays' except where two triangles are hit at exactly the same distance (the visiting
 * order then picks one of them).  Instanced scenes: the persistent two-level traversal over the
 * TLAS and the 4-wide view of the BLAS nodes, the same except at exact ties.  Replaces the same
 * reference calls as
 * ks_trace_rays (cuda/sbvh.cu:512-603); exists to test the rendering traversal. */
ks_status ks_trace_rays_wide(ks_scene *scene, const float *rays, uint32_t n, int any_hit, int culling,
                             uint32_t *tri_idx, float *t, float *bary);

/* ks_trace_rays without any device allocation.  No counterpart in the reference: it exists for
 * callers that may not allocate device memory (a host application that owns the device-memory
 * budget through its own allocator, or a frame loop that forbids cudaMalloc/cudaFree).  Rays and
 * results are staged in one static device array of the library (KS_TRACE_NOALLOC_MAX_RAYS rays,
 * 3.4 MB, resident on every GPU that loads the library until the process exits); larger n is
 * rejected with KS_ERR_INVALID_ARGUMENT.  Each call returns once the results are in the caller's
 * host arrays.  The first call on a device looks up that array's device address
 * (cudaGetSymbolAddress) and keeps it for the life of the process; do not reset the device
 * (cudaDeviceReset) between calls, which would leave the kept address stale.  All calls share the
 * array, so calls that overlap on the GPU (two contexts on one device, two threads) race;
 * serialise them. */
#define KS_TRACE_NOALLOC_MAX_RAYS 65536
ks_status ks_trace_rays_noalloc(ks_scene *scene, const float *rays, uint32_t n, int any_hit, int culling,
                                uint32_t *tri_idx, float *t, float *bary);

/* BSDF parity hooks: the renderer's own device BSDF code (the shading unit's arithmetic) over
 * host batches of directions in the local shading frame (z = shading normal).
 * ks_bsdf_eval: per pair (wo, wi) the cosine-weighted value f cos(theta_i) (3 floats) and the
 * pdf of sampling wi (BSDF::eval_and_pdf, bsdf.h:14-22; PrincipledBSDF::eval_and_pdf,
 * principled_bsdf.cpp:297-307).  ks_bsdf_sample: per (wo, u) with u = (u_lobe, u_wi.x, u_wi.y) the
 * sampled wi, the throughput weight f cos / pdf (3 floats) and the pdf (BSDF::sample, bsdf.h:18-21;
 * PrincipledBSDF::sample, principled_bsdf.cpp:326-393); wi = 0, weight 0 and pdf 0 where the
 * reference returns no sample.  Arrays hold 3 floats per entry (pdf: 1), host memory, n <= 2^26. */
ks_status ks_bsdf_eval(ks_context *ctx, const ks_material_desc *material, const float *wo, const float *wi,
                       uint32_t n, float *f, float *pdf);
ks_status ks_bsdf_sample(ks_context *ctx, const ks_material_desc *material, const float *wo, const float *u,
                         uint32_t n, float *wi, float *weight, float *pdf);

/* ---------------------------------------------------------------------------------------------
 * Camera.  The render consumes the matrices of a reference `Camera` (camera.cpp:85-94):
 * camera_to_world, proj_to_camera = inverse(rev_inf_projection(vfov, aspect, 0.1)) and
 * proj_to_world = inverse(rev_inf_projection * inverse(camera_to_world)); row-major 4x4.
 * ------------------------------------------------------------------------------------------- */
typedef struct ks_camera_desc {
    float camera_to_world[16];
    float proj_to_camera[16];
    float proj_to_world[16];
    int32_t orthographic; /* 1: rays start on the film plane and share the view direction; 0:
                             perspective.  Fill descriptors with ks_camera_perspective /
                             ks_camera_orthographic (or zero-initialise them): any other value is
                             KS_ERR_INVALID_ARGUMENT at render time. */
} ks_camera_desc;

/* Orthographic camera (Camera's orthographic constructor with rev_orthographic, camera.cpp:72-
 * 114): film window [left, right] x [bottom, top] and the clip range in camera space; rays start
 * at the film point and run along -z of camera_to_world (Camera::spawn_ray, camera.cpp:155-160). */
ks_status ks_camera_orthographic(const float camera_to_world[16], float left, float right, float bottom, float top,
                                 float near_clip, float far_clip, ks_camera_desc *out);

/* Perspective camera from a camera-to-world matrix (row-major 4x4), vertical field of view in
 * radians and aspect ratio: Camera::Camera(to_world, vfov, aspect) (camera.cpp:85-92). */
ks_status ks_camera_perspective(const float camera_to_world[16], float vfov, float aspect, ks_camera_desc *out);

/* ---------------------------------------------------------------------------------------------
 * small_pt render parameters: the scalar fields of SmallPTInput (small_pt.h:17-39) with the
 * TOML defaults of the small_pt task (small_pt.cpp:224-241).
 * ------------------------------------------------------------------------------------------- */
typedef struct ks_small_pt_params {
    int32_t include_background; /* 1 unless the task has a `backdrop` (small_pt.cpp:224-229) */
    float backdrop[3];
    int32_t bounces;
    int32_t render_width;
    int32_t render_height;
    int32_t crop_start_x;
    int32_t crop_start_y;
    int32_t crop_width;  /* 0 = full frame */
    int32_t crop_height;
    int32_t spp;
    int32_t rng_seed;
    int32_t scale_ray_diff;
    float clamp_direct;   /* default 0 (off) */
    float clamp_indirect; /* default 10 */
    int32_t spp_prog_interval; /* default 32 */
    float pixel_filter_width;  /* filter width; default 1 (box).  The task's defaults for the
                                  Gaussian and Blackman-Harris filters are 3 (render_target.cpp:28-44) */
    int32_t pixel_filter;      /* 0 box (BoxPixelFilter), 1 Gaussian, 2 Blackman-Harris
                                  (render_target.h:108-180): camera samples are drawn from the
                                  filter's tabulated distribution (PixelFilterSampleTable,
                                  render_target.h:79-106) with weight 1; default 0 */
    float pixel_filter_sigma;  /* Gaussian sigma; default 0.5 */
} ks_small_pt_params;

/* Fills the defaults of SmallPTInput (small_pt.h:17-39) and the task (small_pt.cpp:224-241). */
void ks_small_pt_params_default(ks_small_pt_params *p);

/* Progress callback, called on the caller's thread after every spp interval with the running
 * FP64 accumulation (prog_interval_callback, small_pt.h:38 and small_pt.cpp:64-66). */
typedef void (*ks_progress_fn)(int spp_finished, const double *accum_rgb, const double *weights, void *user);

/* SmallPT::run (small_pt.cpp:15-70) on the GPU: wavefront path tracing of the crop window.
 * accum_rgb (W*H*3) and weights (W*H*2: hit, miss) are caller-owned HOST buffers in the layout
 * of RenderTarget2 (render_target.h:286-287); the render ADDS into them (FP64), like
 * RenderTarget2::add / add_miss.  cb may be NULL.  Requires ks_scene_build_bvh. */
ks_status ks_small_pt_render(ks_scene *scene, const ks_camera_desc *camera, const ks_small_pt_params *params,
                             ks_progress_fn cb, void *user, double *accum_rgb, double *weights);

/* Same render with DEVICE buffers (W*H*3 and W*H*2 doubles on the context's device), no host
 * copies and no callback: for callers that keep the image resident in HBM. */
ks_status ks_small_pt_render_device(ks_scene *scene, const ks_camera_desc *camera, const ks_small_pt_params *params,
                                    double *accum_rgb_device, double *weights_device);

/* Work and device time of the last render on this scene. */
typedef struct ks_render_stats {
    uint64_t paths;          /* camera samples traced */
    uint64_t extension_rays; /* closest-hit queries (camera + bounce rays) */
    uint64_t shadow_rays;    /* any-hit queries (next-event estimation) */
    uint32_t iterations;     /* wavefront iterations */
    uint32_t kernel_launches;
    float ms_total;          /* device time of the whole render */
    float ms_extend;         /* closest-hit kernel time, summed */
    float ms_shade;          /* shading kernel time (incl. ray generation), summed */
    float ms_shadow;         /* any-hit kernel time, summed */
    uint64_t ext_nodes;      /* interior SBVH nodes fetched by closest-hit queries (64 B each) */
    uint64_t ext_tris;       /* triangles tested by closest-hit queries (48 B each) */
    uint64_t shadow_nodes;   /* interior nodes fetched by any-hit queries */
    uint64_t shadow_tris;    /* triangles tested by any-hit queries */
    float ms_guide_infer;    /* guided renders: guide inference over the hit queues, summed */
    float ms_guide_train;    /* guided renders: training (forward, backward, Adam), summed */
    uint64_t guide_records;  /* guided renders: training samples captured */
    uint32_t guide_train_steps; /* guided renders: Adam steps taken */
    uint64_t guide_rows;     /* guided renders: path vertices the guide network was evaluated for */
} ks_render_stats;

ks_status ks_render_stats_last(const ks_scene *scene, ks_render_stats *out);

/* ---------------------------------------------------------------------------------------------
 * Learned guiding network.  The reference's guiding runs as Slang compute shaders
 * (gpu/shaders/adam.slang, the vMF mixture of vmf.h / vmf.cpp); this is its CUDA counterpart:
 *   input   16-level hash grid (2^19 entries x 2 features per level) of the position + degree-3
 *           real spherical harmonics (16 values each) of the outgoing direction and of the
 *           geometric normal on its side = 64 values
 *   MLP     64 -> 64 -> 64 -> 64 -> 64 -> 41, ReLU, no biases, BF16 weights and activations,
 *           FP32 accumulation (tcgen05 tensor cores, accumulators in TMEM)
 *   output  8 vMF lobes x (mean direction xyz, log concentration, mixture logit), then the logit
 *           z of the selection probability alpha = alpha_max * sigmoid(z) of the mixture against
 *           the BSDF in one-sample MIS
 * Training sample (x, wo, normal, wi, t, p_bsdf), t = f cos L / p: the mixture minimises
 * -t/n log q(wi), the selection logit -t/n log(alpha q(wi) + (1 - alpha) p_bsdf) with q held
 * fixed (n = rows of the batch); the reported loss is the latter.
 * Parameters are kept in FP32; Adam follows adam.slang:25-51 (beta 0.9 / 0.999, eps 1e-8).
 * ------------------------------------------------------------------------------------------- */
typedef struct ks_guide ks_guide;

typedef struct ks_guide_params {
    float bound[6];      /* scene bound (min xyz, max xyz) that normalises positions */
    float base_res;      /* cells per axis of the coarsest level (0 -> 16) */
    float max_res;       /* cells per axis of the finest level (0 -> 2048) */
    float learning_rate; /* Adam step size (0 -> 1e-2) */
    float alpha_max;     /* largest selection probability of the mixture (0 -> 0.8) */
    uint64_t seed;       /* initialisation of weights and grid */
} ks_guide_params;

#define KS_GUIDE_LEVELS 16
#define KS_GUIDE_TABLE_SIZE (1u << 19)
#define KS_GUIDE_WEIGHTS 19456 /* 4*64*64 + 48*64 (output layer padded to 48 rows) */
#define KS_GUIDE_OUTPUTS 41

ks_status ks_guide_create(ks_context *ctx, const ks_guide_params *params, ks_guide **out);
void ks_guide_destroy(ks_guide *g);
/* Cells per axis of each level (KS_GUIDE_LEVELS values). */
ks_status ks_guide_level_res(const ks_guide *g, uint32_t res[KS_GUIDE_LEVELS]);
/* Loss of the most recent training batch (ks_guide_gradients or a guided render's training). */
ks_status ks_guide_last_loss(ks_guide *g, double *loss);
/* FP32 master parameters: mlp_weights[KS_GUIDE_WEIGHTS] (layer by layer, W[out][in] row-major),
 * grid[KS_GUIDE_LEVELS * KS_GUIDE_TABLE_SIZE * 2].  Either pointer may be NULL. */
ks_status ks_guide_get_weights(ks_guide *g, float *mlp_weights, float *grid);
ks_status ks_guide_set_weights(ks_guide *g, const float *mlp_weights, const float *grid);
/* Raw network outputs (n x KS_GUIDE_OUTPUTS) for host positions, outgoing directions and normals
 * (n x 3 each). */
ks_status ks_guide_infer(ks_guide *g, const float *pos, const float *wo, const float *normal, uint32_t n,
                         float *raw_out);
/* One training batch: loss (sum over rows of -t/n log m) and gradients of the parameters; with
 * apply_adam the gradients then drive one Adam step, else they are discarded.  bsdf_pdf (n
 * values) may be NULL (p_bsdf = 0); loss, mlp_grad and grid_grad may be NULL. */
ks_status ks_guide_gradients(ks_guide *g, const float *pos, const float *wo, const float *normal, const float *wi,
                             const float *target, const float *bsdf_pdf, uint32_t n, int apply_adam, double *loss,
                             float *mlp_grad, float *grid_grad);

/* ---------------------------------------------------------------------------------------------
 * Guided rendering: small_pt with the guide network as a second proposal.  At every surface
 * vertex the direction is drawn from the guide's mixture with the probability alpha the guide
 * outputs for that vertex, else from the BSDF, and the throughput is divided by the combined
 * density alpha q + (1 - alpha) p_bsdf (one-sample MIS).  The MIS weights between NEE and emitter
 * hits stay functions of the BSDF pdf exactly as in small_pt (nee.cpp:40-48, small_pt.cpp:95,126),
 * so every pass has the expectation of the unguided render whatever the guide has learned.  The render proceeds in passes of params->spp_prog_interval samples per pixel.  During
 * the first train_passes passes, paths record one vertex each (position, wo, sampled wi, and the
 * radiance later gathered along wi); after each such pass the records train the guide (one Adam
 * step per train_batch records).  Passes before guide_from_pass sample the BSDF only.
 * No reference counterpart: the reference's small_pt samples the BSDF only.
 * ------------------------------------------------------------------------------------------- */
typedef struct ks_guide_render_options {
    int32_t guide_from_pass; /* first pass that samples the guide */
    int32_t train_passes;    /* passes that capture records and train afterwards */
    uint32_t max_records;    /* records captured per pass (0 -> 2^19) */
    uint32_t train_batch;    /* records per Adam step (0 -> 2^18) */
    int32_t record_bounces;  /* the recorded vertex is drawn from bounces [0, record_bounces) (0 -> 6);
                                the guide samples directions at those bounces only */
    float min_roughness;     /* vertices whose material roughness is below this sample the BSDF only:
                                no network inference there and no training records (default 0.3; 0
                                guides every vertex).  A narrow BSDF lobe is already sampled well by
                                the BSDF, and the inference costs as much there as anywhere. */
} ks_guide_render_options;

void ks_guide_render_options_default(ks_guide_render_options *out);

/* Progressive device render: after every pass of params->spp_prog_interval samples per pixel the
 * stream is synchronised and progress(spp_done, user) is called with accum / weights up to date
 * on the device; a nonzero return ends the render there.  guide may be NULL (plain small_pt) or a
 * guide with its options (guided render).  No reference counterpart: it exists to time a render
 * to a target error without copying images to the host. */
typedef int (*ks_device_progress_fn)(int spp_done, void *user);
ks_status ks_small_pt_render_device_progress(ks_scene *scene, const ks_camera_desc *camera,
                                             const ks_small_pt_params *params, ks_guide *guide,
                                             const ks_guide_render_options *options, ks_device_progress_fn progress,
                                             void *user, double *accum_rgb_device, double *weights_device);

/* Relative MSE of a device image against a device reference (n_pixels x 3 doubles): the image is
 * composited like RenderTarget2::composite_and_save_to_exr (render_target.cpp:181-205, backdrop
 * may be NULL = black), then mean over pixels and channels of (x - r)^2 / (r^2 + eps), reduced in
 * FP64 on the GPU. */
ks_status ks_image_rel_mse_device(ks_context *ctx, const double *accum_rgb_device, const double *weights_device,
                                  const double *reference_rgb_device, uint32_t n_pixels, double eps,
                                  const float backdrop[3], double *rel_mse);
ks_status ks_small_pt_render_guided(ks_scene *scene, const ks_camera_desc *camera, const ks_small_pt_params *params,
                                    ks_guide *guide, const ks_guide_render_options *options, ks_progress_fn progress,
                                    void *user, double *accum_rgb, double *weights);
ks_status ks_small_pt_render_guided_device(ks_scene *scene, const ks_camera_desc *camera,
                                           const ks_small_pt_params *params, ks_guide *guide,
                                           const ks_guide_render_options *options, double *accum_rgb_device,
                                           double *weights_device);

/* ---------------------------------------------------------------------------------------------
 * TOML tasks: the configuration service of keepsake's test driver (ConfigService::parse +
 * run_all_tasks, config.cpp:262-312; test/main.cpp:60-86) with the small_pt task registered as
 * "small_pt" and "small_pt_b200" (same keys as small_pt.cpp:180-241, plus `emission` on a
 * material).  Runs every [[task]] of config_text in order; asset paths are relative to
 * asset_root_dir (NULL = current directory); outputs go to output_dir/<task_dir or task_N>/
 * (config.toml and small_pt_spp<N>.exr per spp interval).  Also registered: "convert_mesh_asset"
 * (mesh_asset.cpp:301-311: the listed mesh assets as <name>.bin binary mesh assets).  Supported
 * assets: [bsdf.X] of type principled_bsdf with constant fields, [material.X] {bsdf, emission},
 * [mesh_asset.X] with a `path` and `format` "obj" (positions, texcoords, normals; twosided,
 * use_smooth_normal) or "bin" (keepsake's binary mesh asset), optional `to_world`
 * (create_mesh_asset, mesh_asset.cpp:243-266), or of `type` "inline" (geometry list) or
 * "procedural" (kind box_room | icosphere); [compound_mesh_asset.X] glTF files for the task's
 * `compound_object` (see ks_compound_asset_load); sky maps from .exr, .hdr or .pfm files.  Returns
 * KS_ERR_PARSE, KS_ERR_IO or KS_ERR_UNSUPPORTED with a message in ks_config_last_error().
 * C++ hosts can use the ConfigTask-shaped API of ks_b200_task.hpp instead.
 * ------------------------------------------------------------------------------------------- */
ks_status ks_config_run(const char *config_text, const char *asset_root_dir, const char *output_dir);
/* Message of the last failing host-side call on this thread (ks_config_run, ks_config_parse, the
 * image and asset loaders; "" if none). */
const char *ks_config_last_error(void);
/* Parses config_text without running anything: KS_OK or KS_ERR_PARSE (message with the line).
 * The document, normalised (keys sorted, nested tables inline), is written to normalised
 * (NUL-terminated, truncated to capacity; may be NULL) and its length to *length (may be NULL). */
ks_status ks_config_parse(const char *config_text, char *normalised, size_t capacity, size_t *length);

/* ---------------------------------------------------------------------------------------------
 * Image files of the small_pt task (save_to_exr / load_from_exr, image_util.cpp:71-190; the
 * Radiance .hdr maps SkyLight reads through stb_image, light.cpp:19-31).
 * ------------------------------------------------------------------------------------------- */
/* Writes width x height pixels of `channels` (1-4) interleaved floats, rows top first, as an
 * OpenEXR scanline file with save_to_exr's channel names (R, G, B, A), FP32 (half = 0) or FP16
 * (half = 1, rounded to nearest even), ZIP-compressed.  KS_ERR_INVALID_ARGUMENT, KS_ERR_IO. */
ks_status ks_image_save_exr(const char *path, const float *pixels, int32_t width, int32_t height,
                            int32_t channels, int32_t half);
/* Reads the RGB pixels of an .exr (NONE, RLE, ZIPS or ZIP compression; R, G, B channels or a
 * single one), .hdr (RGBE) or .pfm file, by extension, into a buffer the library allocates
 * (width * height * 3 floats, rows top first; release it with ks_image_free).  KS_ERR_IO, or
 * KS_ERR_UNSUPPORTED for a variant of the format this reader does not handle; the message is in
 * ks_config_last_error(). */
ks_status ks_image_load_rgb(const char *path, float **pixels, int32_t *width, int32_t *height);
void ks_image_free(float *pixels);
/* create_texture_from_image (texture.cpp:922-944) without mipmaps: a texture file read into *out,
 * texels in a buffer the library allocates (release it with ks_texture_free).  `channels` 1-4.
 * .png: 8-bit texels (format 0) as stb_image's 8-bit loader converts to the requested channel
 * count (grey replicated, RGB to grey by (77 R + 150 G + 29 B) >> 8, missing alpha opaque, 16-bit
 * samples reduced to their high byte); keep_16bit = 1 keeps 16-bit PNGs as format 1, as glTF
 * images are kept.  .exr: the first `channels` of R, G, B, A (A = 1 when absent; a one-channel file
 * in all four), format 2.  .hdr / .pfm: RGB, or for 1-2 channels their mean (then alpha 1), format 2.
 * `srgb` is copied to out->srgb.  KS_ERR_IO, KS_ERR_UNSUPPORTED (message in ks_config_last_error). */
ks_status ks_texture_load(const char *path, int32_t channels, int32_t srgb, int32_t keep_16bit,
                          ks_texture_desc *out);
void ks_texture_free(ks_texture_desc *texture);

/* ---------------------------------------------------------------------------------------------
 * Batched rendering: many (scene, camera, parameters) jobs in one wavefront.  The paths of all
 * jobs share one pool of path slots, so scenes of uneven size and frames of uneven resolution
 * keep the GPU full; refill, the bounce loop and its termination run on the device, and the
 * whole batch is one CUDA graph launch (a while node around two wavefront iterations) unless
 * use_graph is 0 (then the host re-launches the iterations).  Jobs: flat (non-instanced) scenes
 * of one context, built; frames of at most 2^21 pixels; at most 1024 jobs; accumulators on the
 * device, added into as in ks_small_pt_render_device.  Each job's image equals its own
 * ks_small_pt_render_device (same Sobol samples and estimator).  No reference counterpart.
 * ------------------------------------------------------------------------------------------- */
typedef struct ks_batch_job {
    ks_scene *scene;
    ks_camera_desc camera;
    ks_small_pt_params params; /* spp_prog_interval is ignored: the whole job in one pass */
    double *accum_rgb_device;  /* W * H * 3 */
    double *weights_device;    /* W * H * 2 */
} ks_batch_job;

typedef struct ks_batch_options {
    uint32_t capacity;       /* path slots (0 -> 2^22) */
    uint32_t grid_per_sm;    /* blocks per SM of the traversal and shading kernels (0 -> 16) */
    int32_t use_graph;       /* 1: one CUDA graph launch for the batch */
} ks_batch_options;

typedef struct ks_batch_stats {
    uint64_t paths;
    uint64_t extension_rays;
    uint64_t shadow_rays;
    uint32_t iterations;     /* wavefront iterations run on the device */
    uint32_t graph_launches; /* 1 in graph mode */
    float ms_total;          /* device time of the batch */
} ks_batch_stats;

ks_status ks_batch_render_device(ks_context *ctx, const ks_batch_job *jobs, uint32_t n_jobs,
                                 const ks_batch_options *options, ks_batch_stats *stats);
/* Autotuner: times short renders of a sample of the jobs (up to 8 jobs, at most 4 spp each, into
 * scratch images) for path capacities 2^20 .. 2^23 and 4 .. 32 blocks per SM, and writes the
 * fastest into *best (use_graph kept as given); best_ms (may be NULL) receives its time. */
ks_status ks_batch_autotune(ks_context *ctx, const ks_batch_job *jobs, uint32_t n_jobs, ks_batch_options *best,
                            float *best_ms);

/* ---------------------------------------------------------------------------------------------
 * Procedural scenes: seeded synthetic inputs standing in for mesh-asset loading
 * (mesh_asset.cpp).  kind: "box_room", "icosphere" or "instanced" (prototypes + instances; the
 * scene description then carries prototypes and instances).
 * ------------------------------------------------------------------------------------------- */
typedef struct ks_procedural_options {
    int32_t level;        /* icosphere subdivision level (8 -> 1,310,720 triangles) */
    float roughness_min;  /* per-patch roughness U[min, max] */
    float roughness_max;
    int32_t occluder;     /* 1: slab between the sphere and the sun lobe */
    uint32_t sky_width;   /* lat-long sky resolution */
    uint32_t sky_height;
    uint32_t width;       /* render resolution (sets the camera aspect) */
    uint32_t height;
    /* "instanced": sphere prototypes, instances, geodesic frequency (20 f^2 triangles per
     * prototype), emissive triangles; 0 = defaults 8, 400, 50, 64 */
    uint32_t prototypes;
    uint32_t instances;
    uint32_t frequency;
    uint32_t emitters;
} ks_procedural_options;

typedef struct ks_generated ks_generated;

ks_status ks_procedural_scene(const char *kind, uint64_t seed, const ks_procedural_options *opts,
                              ks_generated **out);
/* The generated scene description; valid until ks_generated_destroy. */
const ks_scene_desc *ks_generated_scene_desc(const ks_generated *g);
/* Camera-to-world (row-major 4x4), vertical fov (radians) and aspect of the generated view. */
ks_status ks_generated_camera(const ks_generated *g, float camera_to_world[16], float *vfov, float *aspect);
void ks_generated_destroy(ks_generated *g);
/* A glTF 2.0 compound mesh asset (.gltf or .glb; CompoundMeshAsset::load_from_gltf,
 * mesh_asset.cpp:551-1091) as a scene description: each glTF mesh a prototype (its primitives
 * the meshes, with normals and texcoords; twosided), each node with a mesh of the default scene
 * an instance under the node's world transform.  load_materials: each primitive's
 * metallic-roughness material as a principled material with constant fields (emission from
 * emissiveFactor x KHR_materials_emissive_strength, ior, specular, transmission extensions);
 * otherwise every mesh has material 0 and the description no materials (the caller supplies
 * them).  No camera (ks_generated_camera returns the default view).  KS_ERR_IO, or
 * KS_ERR_UNSUPPORTED for textures, non-opaque alpha, sparse accessors, non-triangle primitives;
 * the message is in ks_config_last_error(). */
ks_status ks_compound_asset_load(const char *path, int32_t load_materials, ks_generated **out);

/* Camera animation (CameraAnimation, camera.h:44-61; create_camera_animation, camera.cpp:276-465):
 * the translation and rotation keys of the perspective camera `camera_name` in a .glb file
 * (found depth first in the default scene), optionally turned from y-up to z-up.  Frames: one per
 * translation key; eval: translation interpolated linearly, rotation spherically
 * (CameraAnimation::eval, camera.cpp:207-255), as a camera-to-world matrix (row-major) plus the
 * camera's vfov (radians) and aspect, ready for ks_camera_perspective.  The small_pt task renders
 * frame i at duration * (i + 0.5) / frames (small_pt.cpp:243-296). */
typedef struct ks_camera_animation ks_camera_animation;
ks_status ks_camera_animation_load(const char *path, const char *camera_name, int32_t convert_y_up_to_z_up,
                                   ks_camera_animation **out);
uint32_t ks_camera_animation_frames(const ks_camera_animation *a);
float ks_camera_animation_duration(const ks_camera_animation *a);
ks_status ks_camera_animation_eval(const ks_camera_animation *a, float time, float camera_to_world[16], float *vfov,
                                   float *aspect);
void ks_camera_animation_destroy(ks_camera_animation *a);

#ifdef __cplusplus
}
#endif

#endif /* KS_B200_H */
