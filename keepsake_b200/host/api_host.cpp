// Host-only C-ABI entry points: camera matrices, procedural scenes and loaded compound assets.
#include "../../include/ks_b200.h"
#include "gltf.h"
#include "procedural.h"

#include <cmath>
#include <cstring>
#include <memory>
#include <new>
#include <string>

namespace ksb
{
void set_host_error(const std::string &msg); // task.cpp
}

namespace
{

using M4 = double[4][4];

// Inverse of a 4x4 matrix by Gauss-Jordan elimination with partial pivoting, in double precision.
bool invert4(const double in[4][4], double out[4][4])
{
    double a[4][8];
    for (int r = 0; r < 4; ++r)
        for (int c = 0; c < 8; ++c)
            a[r][c] = c < 4 ? in[r][c] : (c - 4 == r ? 1.0 : 0.0);
    for (int col = 0; col < 4; ++col) {
        int piv = col;
        for (int r = col + 1; r < 4; ++r)
            if (std::fabs(a[r][col]) > std::fabs(a[piv][col]))
                piv = r;
        if (a[piv][col] == 0.0)
            return false;
        if (piv != col)
            for (int c = 0; c < 8; ++c)
                std::swap(a[piv][c], a[col][c]);
        double inv = 1.0 / a[col][col];
        for (int c = 0; c < 8; ++c)
            a[col][c] *= inv;
        for (int r = 0; r < 4; ++r) {
            if (r == col)
                continue;
            double f = a[r][col];
            if (f != 0.0)
                for (int c = 0; c < 8; ++c)
                    a[r][c] -= f * a[col][c];
        }
    }
    for (int r = 0; r < 4; ++r)
        for (int c = 0; c < 4; ++c)
            out[r][c] = a[r][c + 4];
    return true;
}

void mul4(const double a[4][4], const double b[4][4], double out[4][4])
{
    for (int r = 0; r < 4; ++r)
        for (int c = 0; c < 4; ++c) {
            double s = 0;
            for (int k = 0; k < 4; ++k)
                s += a[r][k] * b[k][c];
            out[r][c] = s;
        }
}

void store(const double m[4][4], float *out)
{
    for (int r = 0; r < 4; ++r)
        for (int c = 0; c < 4; ++c)
            out[4 * r + c] = (float)m[r][c];
}

} // namespace

struct ks_generated
{
    ksb::GeneratedScene scene;
};

struct ks_camera_animation
{
    ksb::gltf::CameraAnimation anim;
};

extern "C" {

ks_status ks_camera_perspective(const float camera_to_world[16], float vfov, float aspect, ks_camera_desc *out)
{
    if (!camera_to_world || !out || !(vfov > 0.0f) || !(aspect > 0.0f))
        return KS_ERR_INVALID_ARGUMENT;
    double c2w[4][4], w2c[4][4], proj[4][4] = {}, p2c[4][4], p2w[4][4], w2p[4][4];
    for (int r = 0; r < 4; ++r)
        for (int c = 0; c < 4; ++c)
            c2w[r][c] = camera_to_world[4 * r + c];
    if (!invert4(c2w, w2c))
        return KS_ERR_INVALID_ARGUMENT;
    // rev_inf_projection(vfov, aspect, near_clip = 0.1) (camera.cpp:56-70), built in float like
    // the reference, then promoted.
    float cot_half_vfov = 1.0f / std::tan(vfov * 0.5f);
    proj[0][0] = cot_half_vfov / aspect;
    proj[1][1] = -cot_half_vfov;
    proj[2][3] = 0.1f;
    proj[3][2] = -1.0f;
    mul4(proj, w2c, w2p);
    if (!invert4(proj, p2c) || !invert4(w2p, p2w))
        return KS_ERR_INVALID_ARGUMENT;
    std::memcpy(out->camera_to_world, camera_to_world, sizeof(float) * 16);
    store(p2c, out->proj_to_camera);
    store(p2w, out->proj_to_world);
    out->orthographic = 0;
    return KS_OK;
}

ks_status ks_camera_orthographic(const float camera_to_world[16], float left, float right, float bottom, float top,
                                 float near_clip, float far_clip, ks_camera_desc *out)
{
    if (!camera_to_world || !out || !(right != left) || !(top != bottom) || !(far_clip != near_clip))
        return KS_ERR_INVALID_ARGUMENT;
    double c2w[4][4], w2c[4][4], proj[4][4] = {}, p2c[4][4], p2w[4][4], w2p[4][4];
    for (int r = 0; r < 4; ++r)
        for (int c = 0; c < 4; ++c)
            c2w[r][c] = camera_to_world[4 * r + c];
    if (!invert4(c2w, w2c))
        return KS_ERR_INVALID_ARGUMENT;
    // rev_orthographic (camera.cpp:72-83), built in float like the reference, then promoted
    proj[0][0] = 2.0f / (right - left);
    proj[0][3] = -(right + left) / (right - left);
    proj[1][1] = 2.0f / (bottom - top);
    proj[1][3] = -(top + bottom) / (bottom - top);
    proj[2][2] = 1.0f / (far_clip - near_clip);
    proj[2][3] = far_clip / (far_clip - near_clip);
    proj[3][3] = 1.0f;
    mul4(proj, w2c, w2p);
    if (!invert4(proj, p2c) || !invert4(w2p, p2w))
        return KS_ERR_INVALID_ARGUMENT;
    std::memcpy(out->camera_to_world, camera_to_world, sizeof(float) * 16);
    store(p2c, out->proj_to_camera);
    store(p2w, out->proj_to_world);
    out->orthographic = 1;
    return KS_OK;
}

ks_status ks_procedural_scene(const char *kind, uint64_t seed, const ks_procedural_options *opts, ks_generated **out)
{
    if (!kind || !out)
        return KS_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    ksb::ProceduralOptions o;
    if (opts) {
        if (opts->level > 0)
            o.level = opts->level;
        if (opts->roughness_max > 0.0f) {
            o.roughness_min = opts->roughness_min;
            o.roughness_max = opts->roughness_max;
        }
        o.occluder = opts->occluder;
        if (opts->sky_width)
            o.sky_width = opts->sky_width;
        if (opts->sky_height)
            o.sky_height = opts->sky_height;
        if (opts->width)
            o.width = opts->width;
        if (opts->height)
            o.height = opts->height;
        if (opts->prototypes)
            o.prototypes = opts->prototypes;
        if (opts->instances)
            o.instances = opts->instances;
        if (opts->frequency) {
            o.frequency = opts->frequency;
            o.geodesic_sphere = true;
        }
        if (opts->emitters)
            o.emitters = opts->emitters;
    }
    if (o.level > 10 || o.frequency > 2000 || o.prototypes > 4096 || o.instances > (1u << 24))
        return KS_ERR_INVALID_ARGUMENT;
    auto *g = new (std::nothrow) ks_generated();
    if (!g)
        return KS_ERR_OUT_OF_MEMORY;
    if (!ksb::generate_scene(kind, seed, o, g->scene)) {
        delete g;
        return KS_ERR_INVALID_ARGUMENT;
    }
    *out = g;
    return KS_OK;
}

const ks_scene_desc *ks_generated_scene_desc(const ks_generated *g) { return g ? &g->scene.desc : nullptr; }

ks_status ks_generated_camera(const ks_generated *g, float camera_to_world[16], float *vfov, float *aspect)
{
    if (!g || !camera_to_world || !vfov || !aspect)
        return KS_ERR_INVALID_ARGUMENT;
    std::memcpy(camera_to_world, g->scene.camera_to_world, sizeof(float) * 16);
    *vfov = g->scene.vfov;
    *aspect = g->scene.aspect;
    return KS_OK;
}

void ks_generated_destroy(ks_generated *g) { delete g; }

ks_status ks_camera_animation_load(const char *path, const char *camera_name, int32_t convert_y_up_to_z_up,
                                   ks_camera_animation **out)
{
    if (!path || !camera_name || !out)
        return KS_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    try {
        auto a = std::make_unique<ks_camera_animation>();
        a->anim = ksb::gltf::load_camera_animation(path, camera_name, convert_y_up_to_z_up != 0);
        *out = a.release();
        return KS_OK;
    } catch (const ksb::gltf::Error &e) {
        ksb::set_host_error(e.what());
        return e.unsupported ? KS_ERR_UNSUPPORTED : KS_ERR_IO;
    } catch (const std::exception &e) {
        ksb::set_host_error(e.what());
        return KS_ERR_IO;
    }
}

uint32_t ks_camera_animation_frames(const ks_camera_animation *a) { return a ? a->anim.n_frames() : 0; }

float ks_camera_animation_duration(const ks_camera_animation *a) { return a ? a->anim.duration() : 0.0f; }

ks_status ks_camera_animation_eval(const ks_camera_animation *a, float time, float camera_to_world[16], float *vfov,
                                   float *aspect)
{
    if (!a || !camera_to_world || !vfov || !aspect)
        return KS_ERR_INVALID_ARGUMENT;
    a->anim.eval(time, camera_to_world);
    *vfov = a->anim.vfov;
    *aspect = a->anim.aspect;
    return KS_OK;
}

void ks_camera_animation_destroy(ks_camera_animation *a) { delete a; }

ks_status ks_compound_asset_load(const char *path, int32_t load_materials, ks_generated **out)
{
    if (!path || !out)
        return KS_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    auto g = std::make_unique<ks_generated>();
    ksb::GeneratedScene &sc = g->scene;
    try {
        ksb::gltf::Compound c = ksb::gltf::load(path, load_materials != 0);
        if (c.instances.empty())
            throw ksb::gltf::Error(std::string(path) + ": the default scene instances no mesh");
        for (auto &t : c.textures) {
            ks_texture_desc d{};
            d.width = (uint32_t)t.width;
            d.height = (uint32_t)t.height;
            d.channels = (uint32_t)t.channels;
            d.format = t.format;
            d.srgb = t.srgb ? 1 : 0;
            sc.textures.push_back(d);
            sc.texture_bytes.push_back(std::move(t.bytes));
        }
        for (const auto &p : c.prototypes) {
            for (ks_texture_binding b : p.bindings) {
                b.material += (uint32_t)sc.materials.size(); // primitive index -> scene material
                sc.bindings.push_back(b);
            }
            sc.prototypes.push_back({(uint32_t)sc.meshes.size(), (uint32_t)p.meshes.size()});
            for (size_t k = 0; k < p.meshes.size(); ++k) {
                const ksb::mesh::MeshData &md = p.meshes[k];
                ksb::GeneratedMesh gm;
                gm.vertices = md.vertices;
                gm.indices = md.indices;
                gm.normals = md.normals;
                gm.texcoords = md.texcoords;
                gm.twosided = md.twosided ? 1 : 0;
                gm.use_smooth_normal = md.use_smooth_normal ? 1 : 0;
                if (load_materials) {
                    gm.material = (uint32_t)sc.materials.size();
                    sc.materials.push_back(p.materials[k]);
                }
                sc.meshes.push_back(std::move(gm));
            }
        }
        for (const auto &i : c.instances) {
            ks_instance_desc d{};
            d.prototype = i.prototype;
            std::memcpy(d.to_world, i.to_world, sizeof(d.to_world));
            sc.instances.push_back(d);
        }
    } catch (const ksb::gltf::Error &e) {
        ksb::set_host_error(e.what());
        return e.unsupported ? KS_ERR_UNSUPPORTED : KS_ERR_IO;
    } catch (const std::exception &e) {
        ksb::set_host_error(e.what());
        return KS_ERR_IO;
    }
    sc.finalize();
    *out = g.release();
    return KS_OK;
}

void ks_small_pt_params_default(ks_small_pt_params *p)
{
    if (!p)
        return;
    *p = ks_small_pt_params{};
    p->include_background = 1;
    p->bounces = 1;
    p->render_width = 256;
    p->render_height = 256;
    p->spp = 1;
    p->rng_seed = 0;
    p->scale_ray_diff = 1;
    p->clamp_direct = 0.0f;
    p->clamp_indirect = 10.0f;
    p->spp_prog_interval = 32;
    p->pixel_filter_width = 1.0f;
    p->pixel_filter = 0;
    p->pixel_filter_sigma = 0.5f;
}

} // extern "C"
