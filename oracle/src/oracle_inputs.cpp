// ORACLE (test infrastructure only).  The CPU side of the benchmark's inputs, so that the CPU
// baseline builds its scene, camera and render parameters without loading the CUDA library:
//   * the seeded synthetic scenes, made by the library's own host generator
//     (keepsake_b200/host/procedural.cpp, compiled into this library from the same source file:
//     input generation, not the path under test);
//   * Camera::Camera(to_world, vfov, aspect) (camera.cpp:85-92): the reverse-infinite projection of
//     rev_inf_projection (camera.cpp:56-70, near clip 0.1) built in float, the transforms inverted;
//   * the small_pt task's parameter defaults (small_pt.cpp:224-241).
#include "../../include/ks_b200.h"
#include "../../keepsake_b200/host/procedural.h"

#include <cmath>
#include <cstring>
#include <new>

namespace
{

// Gauss-Jordan inverse with partial pivoting in double; false when singular.
bool inverse4(const double m[4][4], double out[4][4])
{
    double a[4][8];
    for (int r = 0; r < 4; ++r)
        for (int c = 0; c < 8; ++c)
            a[r][c] = c < 4 ? m[r][c] : (c - 4 == r ? 1.0 : 0.0);
    for (int c = 0; c < 4; ++c) {
        int p = c;
        for (int r = c + 1; r < 4; ++r)
            if (std::fabs(a[r][c]) > std::fabs(a[p][c]))
                p = r;
        if (a[p][c] == 0.0)
            return false;
        for (int k = 0; k < 8; ++k)
            std::swap(a[c][k], a[p][k]);
        const double inv = 1.0 / a[c][c];
        for (int k = 0; k < 8; ++k)
            a[c][k] *= inv;
        for (int r = 0; r < 4; ++r)
            if (r != c) {
                const double f = a[r][c];
                for (int k = 0; k < 8; ++k)
                    a[r][k] -= f * a[c][k];
            }
    }
    for (int r = 0; r < 4; ++r)
        for (int c = 0; c < 4; ++c)
            out[r][c] = a[r][c + 4];
    return true;
}

} // namespace

extern "C" {

void *oracle_generate(const char *kind, uint64_t seed, int level, float roughness_min, float roughness_max,
                      int occluder, uint32_t sky_w, uint32_t sky_h, uint32_t width, uint32_t height)
{
    auto *g = new (std::nothrow) ksb::GeneratedScene();
    if (!g || !kind)
        return nullptr;
    ksb::ProceduralOptions o;
    if (level > 0)
        o.level = level;
    if (roughness_max > 0.0f) {
        o.roughness_min = roughness_min;
        o.roughness_max = roughness_max;
    }
    o.occluder = occluder;
    if (sky_w)
        o.sky_width = sky_w;
    if (sky_h)
        o.sky_height = sky_h;
    if (width)
        o.width = width;
    if (height)
        o.height = height;
    if (!ksb::generate_scene(kind, seed, o, *g)) {
        delete g;
        return nullptr;
    }
    return g;
}

const ks_scene_desc *oracle_generated_desc(void *g) { return g ? &((ksb::GeneratedScene *)g)->desc : nullptr; }

void oracle_generated_camera(void *gp, float camera_to_world[16], float *vfov, float *aspect)
{
    auto *g = (ksb::GeneratedScene *)gp;
    std::memcpy(camera_to_world, g->camera_to_world, sizeof(float) * 16);
    *vfov = g->vfov;
    *aspect = g->aspect;
}

void oracle_generated_destroy(void *g) { delete (ksb::GeneratedScene *)g; }

int oracle_camera_perspective(const float camera_to_world[16], float vfov, float aspect, ks_camera_desc *out)
{
    double c2w[4][4], w2c[4][4], proj[4][4] = {}, w2p[4][4], p2w[4][4], p2c[4][4];
    for (int r = 0; r < 4; ++r)
        for (int c = 0; c < 4; ++c)
            c2w[r][c] = camera_to_world[4 * r + c];
    if (!inverse4(c2w, w2c))
        return 1;
    const float cot_half_vfov = 1.0f / std::tan(vfov * 0.5f);
    proj[0][0] = cot_half_vfov / aspect;
    proj[1][1] = -cot_half_vfov;
    proj[2][3] = 0.1f;
    proj[3][2] = -1.0f;
    for (int r = 0; r < 4; ++r)
        for (int c = 0; c < 4; ++c) {
            double s = 0.0;
            for (int k = 0; k < 4; ++k)
                s += proj[r][k] * w2c[k][c];
            w2p[r][c] = s;
        }
    if (!inverse4(w2p, p2w) || !inverse4(proj, p2c))
        return 1;
    std::memcpy(out->camera_to_world, camera_to_world, sizeof(float) * 16);
    for (int r = 0; r < 4; ++r)
        for (int c = 0; c < 4; ++c) {
            out->proj_to_world[4 * r + c] = (float)p2w[r][c];
            out->proj_to_camera[4 * r + c] = (float)p2c[r][c];
        }
    out->orthographic = 0;
    return 0;
}

void oracle_params_default(ks_small_pt_params *p)
{
    *p = ks_small_pt_params{};
    p->include_background = 1;
    p->bounces = 1;
    p->render_width = 256;
    p->render_height = 256;
    p->spp = 1;
    p->scale_ray_diff = 1;
    p->clamp_indirect = 10.0f;
    p->spp_prog_interval = 32;
    p->pixel_filter_width = 1.0f;
    p->pixel_filter_sigma = 0.5f;
}

} // extern "C"
