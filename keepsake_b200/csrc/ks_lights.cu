// Light tables: sky distribution (GPU), sky power (GPU), mesh-light importance (host, a handful of
// emissive triangles), and the PowerLightSampler CDF.
//
//   SkyLight::SkyLight (light.cpp:19-49): lum = sin(theta) * luminance, threshold at the mean,
//     DistribTable2D of the thresholded values.  The conditional CDFs are float prefix sums in
//     index order, exactly as DistribTable (distrib.cpp:9-29): one GPU thread per row runs the
//     row's sum in the reference's order over tiles staged in shared memory, so the table is
//     bit-identical to a sequential host build.
//     The mean is a double sum (rows in order) - the reference uses an unordered float atomic.
//   SkyLight::power (light.cpp:136-159): float row sums in column order (one thread per row),
//     rows added in order in double.
//   compute_mesh_light_importance (light.cpp:307-522): the uniform branch for constant emission,
//     the summed-area-table branch for emission / opacity textures (mesh_uv_importance), and the
//     zero-importance compaction of MeshLightShared (light.cpp:524-560).
//   PowerLightSampler::build (light.cpp:636-672).
#include "ks_lights.cuh"
#include "ks_scene.h"

#include <algorithm>
#include <cmath>
#include <cstring>

namespace ksb
{
namespace
{

// The per-row sums below keep the reference's summation order (one running sum per row, columns in
// order); the rows' texels are staged through shared memory in tiles of kTileRows x kTileCols so
// that the loads are coalesced and many rows progress at once.
constexpr int kTileRows = 32, kTileCols = 64, kTileThreads = 256;

// RGB (3 floats per texel) -> float4 texels.
__global__ void k_sky_unpack(const float *rgb, size_t n, float4 *map)
{
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        map[i] = make_float4(rgb[3 * i], rgb[3 * i + 1], rgb[3 * i + 2], 0.0f);
}

// lum = sin(theta) * luminance per texel, and its double row sums in column order.
__global__ void __launch_bounds__(kTileThreads) k_sky_rows(const float4 *map, int w, int h, const float *row_sin,
                                                           float *lum, double *row_sum)
{
    __shared__ float tile[kTileRows][kTileCols + 1];
    const int y0 = blockIdx.x * kTileRows, r0 = threadIdx.x;
    double s = 0.0;
    for (int x0 = 0; x0 < w; x0 += kTileCols) {
        for (int k = threadIdx.x; k < kTileRows * kTileCols; k += kTileThreads) {
            const int r = k / kTileCols, c = k % kTileCols, y = y0 + r, x = x0 + c;
            float l = 0.0f;
            if (y < h && x < w) {
                float4 t = map[(size_t)y * w + x];
                l = row_sin[y] * luminance(mk(t.x, t.y, t.z));
                lum[(size_t)y * w + x] = l;
            }
            tile[r][c] = l;
        }
        __syncthreads();
        if (r0 < kTileRows && y0 + r0 < h)
            for (int c = 0; c < kTileCols && x0 + c < w; ++c)
                s += tile[r0][c];
        __syncthreads();
    }
    if (r0 < kTileRows && y0 + r0 < h)
        row_sum[y0 + r0] = s;
}

// DistribTable(f, n) per row with f = max(lum - average, 0) (distrib.cpp:9-29): the float prefix
// sums in column order, then the normalisation.
__global__ void __launch_bounds__(kTileThreads) k_sky_cond(const float *lum, int w, int h, float average,
                                                           float *cond, float *acc, int threshold)
{
    __shared__ float tile[kTileRows][kTileCols + 1];
    __shared__ float total[kTileRows];
    const int y0 = blockIdx.x * kTileRows, r0 = threadIdx.x;
    const float invn = 1.0f / (float)w;
    float prev = 0.0f;
    for (int x0 = 0; x0 < w; x0 += kTileCols) {
        for (int k = threadIdx.x; k < kTileRows * kTileCols; k += kTileThreads) {
            const int r = k / kTileCols, c = k % kTileCols, y = y0 + r, x = x0 + c;
            tile[r][c] = (y < h && x < w) ? lum[(size_t)y * w + x] : 0.0f;
        }
        __syncthreads();
        if (r0 < kTileRows && y0 + r0 < h)
            for (int c = 0; c < kTileCols && x0 + c < w; ++c) {
                float v = tile[r0][c];
                if (threshold) {
                    v = v - average;
                    v = v < 0.0f ? 0.0f : v; // std::max(lum - average, 0.0f)
                }
                prev = prev + v * invn;
                tile[r0][c] = prev; // cdf[x0 + c + 1]
            }
        __syncthreads();
        for (int k = threadIdx.x; k < kTileRows * kTileCols; k += kTileThreads) {
            const int r = k / kTileCols, c = k % kTileCols, y = y0 + r, x = x0 + c;
            if (y < h && x < w)
                cond[(size_t)y * (w + 1) + x + 1] = tile[r][c];
        }
        __syncthreads();
    }
    if (r0 < kTileRows && y0 + r0 < h) {
        cond[(size_t)(y0 + r0) * (w + 1)] = 0.0f;
        acc[y0 + r0] = prev;
        total[r0] = prev;
    }
    __syncthreads();
    // normalisation, every entry independently
    for (int r = 0; r < kTileRows && y0 + r < h; ++r) {
        float *cdf = cond + (size_t)(y0 + r) * (w + 1);
        const float a = total[r];
        const float inva = a == 0.0f ? 0.0f : 1.0f / a;
        for (int i = threadIdx.x; i < w + 1; i += kTileThreads) {
            if (i == w)
                cdf[i] = 1.0f;
            else if (a == 0.0f)
                cdf[i] = (float)i / (float)w;
            else
                cdf[i] *= inva;
        }
    }
}

// Row sums of SkyLight::power (light.cpp:140-153); eval() through the same device code as shading.
// Each texel's term is computed by its own thread; the float row sums run in column order.
__global__ void __launch_bounds__(kTileThreads) k_sky_power_rows(SceneView s, double *row_sums)
{
    __shared__ float tile[3][kTileRows][kTileCols + 1];
    const int y0 = blockIdx.x * kTileRows, r0 = threadIdx.x;
    f3 rs = mk(0, 0, 0);
    for (int x0 = 0; x0 < s.sky_w; x0 += kTileCols) {
        for (int k = threadIdx.x; k < kTileRows * kTileCols; k += kTileThreads) {
            const int r = k / kTileCols, c = k % kTileCols, row = y0 + r, col = x0 + c;
            f3 v = mk(0, 0, 0);
            if (row < s.sky_h && col < s.sky_w) {
                float theta = (row + 0.5f) / (float)s.sky_h * kPi;
                float sin_theta = sinf(theta);
                float phi = (col + 0.5f) / (float)s.sky_w * kTwoPi;
                float ct = cosf(theta), st = sinf(theta), cp = cosf(phi), sp = sinf(phi);
                f3 dir = mk(cp * st, sp * st, ct); // to_cartesian (z up), as the reference does here
                v = sky_eval(s, dir) * sin_theta;
            }
            tile[0][r][c] = v.x;
            tile[1][r][c] = v.y;
            tile[2][r][c] = v.z;
        }
        __syncthreads();
        if (r0 < kTileRows && y0 + r0 < s.sky_h)
            for (int c = 0; c < kTileCols && x0 + c < s.sky_w; ++c)
                rs += mk(tile[0][r0][c], tile[1][r0][c], tile[2][r0][c]);
        __syncthreads();
    }
    if (r0 < kTileRows && y0 + r0 < s.sky_h) {
        const int row = y0 + r0;
        row_sums[3 * row + 0] = rs.x;
        row_sums[3 * row + 1] = rs.y;
        row_sums[3 * row + 2] = rs.z;
    }
}

// Guide tables (see cdf_find_guided): one thread per (row, entry).
__global__ void k_guide(const float *cdf, uint32_t n, uint32_t rows, uint32_t *guide)
{
    const size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (t >= (size_t)rows * kGuide)
        return;
    const uint32_t r = (uint32_t)(t / kGuide), k = (uint32_t)(t % kGuide);
    const float *c = cdf + (size_t)r * (n + 1);
    guide[t] = cdf_find(c, n, (float)k / (float)kGuide);
}

// DistribTable on the host, identical to distrib.cpp:9-29.
std::vector<float> host_cdf(const float *f, uint32_t n, float *acc_out = nullptr)
{
    std::vector<float> cdf(n + 1);
    cdf[0] = 0;
    float invn = 1.0f / (float)n;
    for (uint32_t i = 1; i < n + 1; ++i)
        cdf[i] = cdf[i - 1] + f[i - 1] * invn;
    float acc = cdf[n];
    if (acc == 0.0f) {
        for (uint32_t i = 0; i < n + 1; ++i)
            cdf[i] = (float)i / (float)n;
    } else {
        float invacc = 1.0f / acc;
        for (uint32_t i = 0; i < n + 1; ++i)
            cdf[i] *= invacc;
    }
    cdf[n] = 1.0f;
    if (acc_out)
        *acc_out = acc;
    return cdf;
}

bool invert4(const float *m, float *out)
{
    double a[4][8];
    for (int r = 0; r < 4; ++r)
        for (int c = 0; c < 8; ++c)
            a[r][c] = c < 4 ? m[4 * r + c] : (c - 4 == r ? 1.0 : 0.0);
    for (int col = 0; col < 4; ++col) {
        int piv = col;
        for (int r = col + 1; r < 4; ++r)
            if (std::fabs(a[r][col]) > std::fabs(a[piv][col]))
                piv = r;
        if (a[piv][col] == 0.0)
            return false;
        for (int c = 0; c < 8; ++c)
            std::swap(a[piv][c], a[col][c]);
        double inv = 1.0 / a[col][col];
        for (int c = 0; c < 8; ++c)
            a[col][c] *= inv;
        for (int r = 0; r < 4; ++r)
            if (r != col) {
                double f = a[r][col];
                for (int c = 0; c < 8; ++c)
                    a[r][c] -= f * a[col][c];
            }
    }
    for (int r = 0; r < 4; ++r)
        for (int c = 0; c < 4; ++c)
            out[4 * r + c] = (float)a[r][c + 4];
    return true;
}

// SummedAreaTable (sat.h): double prefix sums of float values, looked up bilinearly over the
// (nx + 1) x (ny + 1) grid of corners with clamping and boundary ticks (lerp_helper,
// maths.h:760-788); a box's sum from its four corners, never below zero.
struct SatTable
{
    int nx = 0, ny = 0;
    std::vector<double> table;
    SatTable(const std::vector<float> &v, int nx_, int ny_) : nx(nx_), ny(ny_), table(v.size())
    {
        table[0] = v[0];
        for (int x = 1; x < nx; ++x)
            table[x] = v[x] + table[x - 1];
        for (int y = 1; y < ny; ++y)
            table[(size_t)y * nx] = v[(size_t)y * nx] + table[(size_t)(y - 1) * nx];
        for (int y = 1; y < ny; ++y)
            for (int x = 1; x < nx; ++x)
                table[(size_t)y * nx + x] = (v[(size_t)y * nx + x] + table[(size_t)y * nx + (x - 1)] +
                                             table[(size_t)(y - 1) * nx + x] - table[(size_t)(y - 1) * nx + (x - 1)]);
    }
    double fetch(int x, int y) const
    {
        if (x == 0 || y == 0)
            return 0;
        x = std::min(x - 1, nx - 1);
        y = std::min(y - 1, ny - 1);
        return table[(size_t)y * nx + x];
    }
    static void lerp(float u, int res, int &u0, int &u1, float &t)
    {
        const float us = u * (float)(res - 1);
        u0 = (int)std::floor(us);
        u1 = u0 + 1;
        t = us - (float)u0;
        u0 = std::clamp(u0, 0, res - 1);
        u1 = std::clamp(u1, 0, res - 1);
    }
    double lookup(float px, float py) const
    {
        int x0, x1, y0, y1;
        float wx, wy;
        lerp(px, nx + 1, x0, x1, wx);
        lerp(py, ny + 1, y0, y1, wy);
        return fetch(x0, y0) * (1.0 - wx) * (1.0 - wy) + fetch(x1, y0) * (wx) * (1.0 - wy) +
               fetch(x0, y1) * (1.0 - wx) * (wy) + fetch(x1, y1) * (wx) * (wy);
    }
    float sum(float x0, float y0, float x1, float y1) const
    {
        const double v = (lookup(x1, y1) - lookup(x0, y1)) + (lookup(x0, y0) - lookup(x1, y0));
        return std::max((float)v, 0.0f);
    }
};

// mod (maths.h:133-138) for floats
float fmod_pos(float a, float b)
{
    const float r = a - std::floor(a / b) * b;
    return r < 0 ? r + b : r;
}

float luminance3(float r, float g, float b) { return 0.212671f * r + 0.715160f * g + 0.072169f * b; }

// compute_mesh_light_importance (light.cpp:307-522), per triangle of one emissive mesh: the factor
// that multiplies 2 pi x the triangle's area.  A constant emission (and no opacity texture) is the
// uniform branch: the luminance of the emission.  With an emission or opacity texture, the
// luminance of the emission (times the opacity) at the texel centres of the larger texture goes
// into a summed-area table, and each triangle takes the table's mean over the bounding box of its
// texture coordinates (after flip_v, uv_scale, uv_offset), tile by tile with the texture's
// wrapping; textures whose lookups disagree in those settings fall back to the mean over the grid.
void mesh_uv_importance(const ks_scene *s, const MaterialGPU &mat, uint32_t first, uint32_t n,
                        const std::vector<float> &h_verts, const std::vector<uint32_t> &h_idx, std::vector<float> &out)
{
    out.assign(n, 0.0f);
    const ks_scene::EmissionTextures &et = s->emit_tex;
    const BindingGPU *em = nullptr, *op = nullptr;
    if (s->any_emission_map || s->any_opacity)
        for (int k = 0; k < mat.bind_count && !et.binds.empty(); ++k) {
            const BindingGPU &b = et.binds[mat.bind_begin + k];
            if (b.field == KS_FIELD_EMISSION)
                em = &b;
            else if (b.field == KS_FIELD_OPACITY_MAP)
                op = &b;
        }
    if (!em && !op) {
        const float avg = luminance3(mat.emission[0], mat.emission[1], mat.emission[2]);
        for (uint32_t k = 0; k < n; ++k)
            out[k] = avg;
        return;
    }
    bool fallback = false;
    int rx = 1, ry = 1;
    const BindingGPU *first_b = em ? em : op;
    if (em) {
        rx = et.info[em->tex].w;
        ry = et.info[em->tex].h;
    }
    if (op) {
        rx = std::max(rx, et.info[op->tex].w);
        ry = std::max(ry, et.info[op->tex].h);
        if (em && (em->wrap_u != op->wrap_u || em->wrap_v != op->wrap_v || em->flip_v != op->flip_v ||
                   em->uv_scale[0] != op->uv_scale[0] || em->uv_scale[1] != op->uv_scale[1] ||
                   em->uv_offset[0] != op->uv_offset[0] || em->uv_offset[1] != op->uv_offset[1]))
            fallback = true;
    }
    std::vector<float> imp((size_t)rx * ry);
    double sum = 0.0;
    for (int y = 0; y < ry; ++y)
        for (int x = 0; x < rx; ++x) {
            const float u = (x + 0.5f) / (float)rx, v = (y + 0.5f) / (float)ry;
            float e;
            if (em) {
                const float4 c = field_eval(et.texels.data(), et.info.data(), *em, u, v);
                e = luminance3(c.x, c.y, c.z);
            } else {
                e = luminance3(mat.emission[0], mat.emission[1], mat.emission[2]);
            }
            if (op)
                e *= field_eval(et.texels.data(), et.info.data(), *op, u, v).x;
            imp[(size_t)y * rx + x] = e;
            sum += e;
        }
    if (fallback) {
        // the mean over the grid (the reference sums it with an unordered float atomic)
        const float avg = (float)(sum / (double)imp.size());
        for (uint32_t k = 0; k < n; ++k)
            out[k] = avg;
        return;
    }
    const SatTable sat(imp, rx, ry);
    constexpr float kBeforeOne = 0x1.fffffep-1f; // fp32_before_one
    for (uint32_t k = 0; k < n; ++k) {
        float tc[3][2];
        for (int c = 0; c < 3; ++c) {
            const uint32_t vi = h_idx[3 * (size_t)(first + k) + c];
            tc[c][0] = et.texcoords.empty() ? 0.0f : et.texcoords[2 * (size_t)vi];
            tc[c][1] = et.texcoords.empty() ? 0.0f : et.texcoords[2 * (size_t)vi + 1];
            if (first_b->flip_v)
                tc[c][1] = 1.0f - tc[c][1];
            tc[c][0] = tc[c][0] * first_b->uv_scale[0] + first_b->uv_offset[0];
            tc[c][1] = tc[c][1] * first_b->uv_scale[1] + first_b->uv_offset[1];
        }
        float bmin[2] = {INFINITY, INFINITY}, bmax[2] = {-INFINITY, -INFINITY};
        for (int c = 0; c < 3; ++c)
            for (int a = 0; a < 2; ++a) {
                bmin[a] = std::min(bmin[a], tc[c][a]);
                bmax[a] = std::max(bmax[a], tc[c][a]);
            }
        const int txmin = (int)std::floor(bmin[0]), txmax = (int)std::ceil(bmax[0]);
        const int tymin = (int)std::floor(bmin[1]), tymax = (int)std::ceil(bmax[1]);
        float acc = 0.0f, sum_area = 0.0f;
        for (int ty = tymin; ty < tymax; ++ty)
            for (int tx = txmin; tx < txmax; ++tx) {
                // the box within this tile (an empty intersection has zero extents)
                float lo[2] = {std::max(bmin[0], (float)tx), std::max(bmin[1], (float)ty)};
                float hi[2] = {std::min(bmax[0], tx + kBeforeOne), std::min(bmax[1], ty + kBeforeOne)};
                if (lo[0] > hi[0] || lo[1] > hi[1])
                    continue;
                const float b_area = (hi[0] - lo[0]) * (hi[1] - lo[1]);
                if (b_area == 0.0f)
                    continue;
                const int wrap[2] = {first_b->wrap_u, first_b->wrap_v};
                for (int a = 0; a < 2; ++a) {
                    if (wrap[a] == 0) {
                        lo[a] = fmod_pos(lo[a], 1.0f);
                        hi[a] = fmod_pos(hi[a], 1.0f);
                    } else {
                        lo[a] = std::clamp(lo[a], 0.0f, 1.0f);
                        hi[a] = std::clamp(hi[a], 0.0f, 1.0f);
                    }
                }
                const int res[2] = {rx, ry};
                for (int a = 0; a < 2; ++a) {
                    if (lo[a] == 0.0f && hi[a] == 0.0f)
                        hi[a] = 1.0f / (res[a] + 1);
                    if (lo[a] == 1.0f && hi[a] == 1.0f)
                        lo[a] = 1.0f - 1.0f / (res[a] + 1);
                }
                const float ex = lo[0] > hi[0] || lo[1] > hi[1] ? 0.0f : hi[0] - lo[0];
                const float ey = lo[0] > hi[0] || lo[1] > hi[1] ? 0.0f : hi[1] - lo[1];
                // (the reference asserts a non-empty wrapped box: tx + fp32_before_one rounds up to
                // tx + 1 for tiles at |tx| >= 1, which wraps to an empty box; such a tile is skipped)
                if (ex * ey == 0.0f)
                    continue;
                const float mean = sat.sum(lo[0], lo[1], hi[0], hi[1]) / ((ex * (float)rx) * (ey * (float)ry));
                acc += mean * b_area;
                sum_area += b_area;
            }
        if (sum_area > 0.0f)
            acc /= sum_area;
        out[k] = acc;
    }
}

} // namespace

SceneView make_view(const ks_scene *s)
{
    SceneView v{};
    v.inst.n = s->n_instances;
    if (s->n_instances) {
        v.inst.tlas = s->tlas_nodes.ptr;
        v.inst.items = s->tlas_items.ptr;
        v.inst.root_ref = s->tlas_root_ref;
        v.inst.root_count = s->tlas_root_count;
        v.inst.xf = s->inst_xf.ptr;
        v.inst.inv = s->inst_inv.ptr;
        v.inst.proto = s->inst_proto.ptr;
        v.inst.proto_root = s->proto_root.ptr;
        v.inst.proto_bound = s->proto_bound.ptr;
        for (int k = 0; k < 3; ++k) {
            v.inst.bmin[k] = s->scene_bound[k];
            v.inst.bmax[k] = s->scene_bound[3 + k];
        }
    }
    v.ml_verts = s->ml_verts.ptr;
    v.inst_light_base = s->inst_light_base.ptr;
    v.nodes = s->trav_nodes.ptr;
    v.wide = s->wide_nodes.ptr;
    v.prim_tris = s->prim_tris.ptr;
    v.verts = s->verts.ptr;
    v.indices = s->indices.ptr;
    v.root_ref = s->root_ref;
    v.root_count = s->root_count;
    for (int k = 0; k < 3; ++k) {
        v.bmin[k] = s->scene_bound[k];
        v.bmax[k] = s->scene_bound[3 + k];
    }
    v.tri_mesh = s->tri_mesh.ptr;
    v.mesh_material = s->mesh_material.ptr;
    v.mesh_flags = s->mesh_flags.ptr;
    v.normals = s->normals.ptr;
    v.texcoords = s->texcoords.ptr;
    v.materials = s->materials.ptr;
    v.tex_texels = s->tex_texels.ptr;
    v.tex_info = s->tex_info.ptr;
    v.bindings = s->bindings.ptr;
    v.shade_variant = (s->ext_materials || s->any_bindings) ? kShadeGeneral
                      : (s->normals.ptr != nullptr || s->texcoords.ptr != nullptr) ? kShadeAttribs
                                                                                     : kShadePlain;
    v.light_count = s->light_count;
    v.n_nonmesh = s->n_nonmesh;
    v.n_sky = (s->sky_desc.kind >= 1 && s->sky_desc.kind <= 3) ? 1u : 0u;
    v.punctual = s->punctual.ptr;
    v.power_cdf = s->power_cdf.ptr;
    v.tri_light = s->tri_light.ptr;
    v.ml_tri = s->ml_tri.ptr;
    v.ml_area = s->ml_area.ptr;
    v.ml_emission = s->ml_emission.ptr;
    v.sky_kind = s->sky_desc.kind;
    v.sky_w = s->sky_w;
    v.sky_h = s->sky_h;
    std::memcpy(v.sky_l2w, s->sky_l2w, sizeof(v.sky_l2w));
    std::memcpy(v.sky_w2l, s->sky_w2l, sizeof(v.sky_w2l));
    v.sky_y_up = s->sky_desc.kind == 2 ? s->sky_desc.transform_y_up : 1;
    v.sky_strength = s->sky_desc.kind >= 2 ? s->sky_desc.strength : 1.0f;
    v.sky_alias = s->sky_alias.ptr;
    v.sky_map = s->sky_map.ptr;
    v.sky_cond = s->sky_cond.ptr;
    v.sky_margin = s->sky_margin.ptr;
    v.sky_cond_guide = s->sky_cond_guide.ptr;
    v.sky_margin_guide = s->sky_margin_guide.ptr;
    return v;
}

// AliasTable::AliasTable (distrib.cpp:109-165): the weights normalised by their double sum, then
// Vose's pairing of under- and over-full bins from two work lists used as stacks.  Bins hold
// (q, p, alias as bits, 0).  False when no weight is positive.
bool alias_table(const std::vector<float> &weights, std::vector<float4> &bins)
{
    const size_t n = weights.size();
    double sum = 0.0;
    for (float w : weights)
        sum += w;
    if (!(sum > 0.0))
        return false;
    std::vector<float> q(n, 0.0f), p(n);
    std::vector<uint32_t> alias(n, 0);
    for (size_t i = 0; i < n; ++i)
        p[i] = (float)(weights[i] / sum);
    struct Outcome
    {
        float p_hat;
        size_t index;
    };
    std::vector<Outcome> under, over;
    for (size_t i = 0; i < n; ++i) {
        const float p_hat = p[i] * n;
        (p_hat < 1 ? under : over).push_back(Outcome{p_hat, i});
    }
    while (!under.empty() && !over.empty()) {
        const Outcome un = under.back(), ov = over.back();
        under.pop_back();
        over.pop_back();
        q[un.index] = un.p_hat;
        alias[un.index] = (uint32_t)ov.index;
        const float excess = un.p_hat + ov.p_hat - 1;
        (excess < 1 ? under : over).push_back(Outcome{excess, ov.index});
    }
    while (!over.empty()) {
        const Outcome ov = over.back();
        over.pop_back();
        q[ov.index] = 1;
        alias[ov.index] = 0xffffffffu;
    }
    while (!under.empty()) {
        const Outcome un = under.back();
        under.pop_back();
        q[un.index] = 1;
        alias[un.index] = 0xffffffffu;
    }
    bins.resize(n);
    for (size_t i = 0; i < n; ++i) {
        const uint32_t a = alias[i] == 0xffffffffu ? (uint32_t)i : alias[i]; // q = 1: never taken
        float a_bits;
        std::memcpy(&a_bits, &a, sizeof(a_bits));
        bins[i] = make_float4(q[i], p[i], a_bits, 0.0f);
    }
    return true;
}

ks_status build_lights(ks_scene *s)
{
    ks_context *ctx = s->ctx;
    cudaStream_t st = ctx->stream;
    const ks_sky_desc &sd = s->sky_desc;
    // ---- sky distribution ----
    s->n_nonmesh = 0;
    float sky_power_mean = 0.0f;
    if (sd.kind == 1 || sd.kind == 2) {
        s->n_nonmesh = 1;
        int w, h;
        if (sd.kind == 1) {
            w = h = 1;
        } else {
            w = (int)sd.width;
            h = (int)sd.height;
            float m4[16], inv4[16];
            std::memcpy(m4, sd.to_world, sizeof(m4));
            if (!invert4(m4, inv4))
                return fail(ctx, KS_ERR_INVALID_ARGUMENT, "sky to_world is singular");
            for (int r = 0; r < 3; ++r)
                for (int c = 0; c < 3; ++c) {
                    s->sky_l2w[3 * r + c] = m4[4 * r + c];
                    s->sky_w2l[3 * r + c] = inv4[4 * r + c];
                }
        }
        s->sky_w = w;
        s->sky_h = h;
        KS_CUDA_TRY(ctx, s->sky_map.alloc((size_t)w * h));
        if (sd.kind == 1) {
            const float4 amb = make_float4(sd.ambient[0], sd.ambient[1], sd.ambient[2], 0.0f);
            KS_CUDA_TRY(ctx, cudaMemcpyAsync(s->sky_map.ptr, &amb, sizeof(amb), cudaMemcpyHostToDevice, st));
            KS_CUDA_TRY(ctx, cudaStreamSynchronize(st)); // amb lives on this stack frame
        } else {
            // the map was uploaded as RGB at ks_scene_create
            k_sky_unpack<<<(unsigned)std::min<size_t>(((size_t)w * h + 255) / 256, 4096), 256, 0, st>>>(
                s->sky_rgb.ptr, (size_t)w * h, s->sky_map.ptr);
        }
        KS_CUDA_TRY(ctx, s->sky_cond.alloc((size_t)h * (w + 1)));
        DevBuf<float> lum, acc, row_sin;
        DevBuf<double> row_sum;
        KS_CUDA_TRY(ctx, lum.alloc((size_t)w * h));
        KS_CUDA_TRY(ctx, acc.alloc(h));
        KS_CUDA_TRY(ctx, row_sin.alloc(h));
        KS_CUDA_TRY(ctx, row_sum.alloc((size_t)3 * h));
        std::vector<float> h_sin(h);
        const float pi = 3.14159265359f;
        for (int y = 0; y < h; ++y)
            h_sin[y] = std::sin((y + 0.5f) / (float)h * pi); // host libm, like the reference
        if (sd.kind == 1)
            h_sin[0] = 1.0f; // the ambient constructor uses plain luminance (light.cpp:52-57)
        KS_CUDA_TRY(ctx, cudaMemcpyAsync(row_sin.ptr, h_sin.data(), sizeof(float) * h, cudaMemcpyHostToDevice, st));
        const unsigned row_tiles = (unsigned)((h + kTileRows - 1) / kTileRows);
        k_sky_rows<<<row_tiles, kTileThreads, 0, st>>>(s->sky_map.ptr, w, h, row_sin.ptr, lum.ptr, row_sum.ptr);
        std::vector<double> h_rows(h);
        KS_CUDA_TRY(ctx, cudaMemcpyAsync(h_rows.data(), row_sum.ptr, sizeof(double) * h, cudaMemcpyDeviceToHost, st));
        KS_CUDA_TRY(ctx, cudaStreamSynchronize(st));
        double lum_sum = 0.0;
        for (int y = 0; y < h; ++y)
            lum_sum += h_rows[y];
        float average = (float)lum_sum / (size_t)((size_t)w * h);
        k_sky_cond<<<row_tiles, kTileThreads, 0, st>>>(lum.ptr, w, h, average, s->sky_cond.ptr, acc.ptr,
                                                    sd.kind == 2 ? 1 : 0);
        std::vector<float> h_acc(h);
        KS_CUDA_TRY(ctx, cudaMemcpyAsync(h_acc.data(), acc.ptr, sizeof(float) * h, cudaMemcpyDeviceToHost, st));
        KS_CUDA_TRY(ctx, cudaStreamSynchronize(st));
        std::vector<float> margin = host_cdf(h_acc.data(), (uint32_t)h);
        KS_CUDA_TRY(ctx, s->sky_margin.alloc(margin.size()));
        KS_CUDA_TRY(ctx, cudaMemcpyAsync(s->sky_margin.ptr, margin.data(), sizeof(float) * margin.size(),
                                         cudaMemcpyHostToDevice, st));
        KS_CUDA_TRY(ctx, s->sky_cond_guide.alloc((size_t)h * kGuide));
        KS_CUDA_TRY(ctx, s->sky_margin_guide.alloc(kGuide));
        k_guide<<<(unsigned)(((size_t)h * kGuide + 255) / 256), 256, 0, st>>>(s->sky_cond.ptr, (uint32_t)w,
                                                                               (uint32_t)h, s->sky_cond_guide.ptr);
        k_guide<<<(kGuide + 255) / 256, 256, 0, st>>>(s->sky_margin.ptr, (uint32_t)h, 1u, s->sky_margin_guide.ptr);
        // power (light.cpp:136-159)
        SceneView v = make_view(s);
        k_sky_power_rows<<<row_tiles, kTileThreads, 0, st>>>(v, row_sum.ptr);
        std::vector<double> h_pr(3 * h);
        KS_CUDA_TRY(ctx, cudaMemcpyAsync(h_pr.data(), row_sum.ptr, sizeof(double) * 3 * h, cudaMemcpyDeviceToHost, st));
        KS_CUDA_TRY(ctx, cudaStreamSynchronize(st));
        double sum[3] = {0, 0, 0};
        for (int y = 0; y < h; ++y)
            for (int c = 0; c < 3; ++c)
                sum[c] += (double)(float)h_pr[3 * y + c];
        float Phi[3] = {(float)sum[0], (float)sum[1], (float)sum[2]};
        float scale = (pi / h) * (6.28318530718f / w);
        float ex = s->scene_bound[3] - s->scene_bound[0], ey = s->scene_bound[4] - s->scene_bound[1],
              ez = s->scene_bound[5] - s->scene_bound[2];
        float radius = 0.5f * std::sqrt(ex * ex + ey * ey + ez * ez);
        for (int c = 0; c < 3; ++c) {
            Phi[c] *= scale;
            Phi[c] *= pi * (radius * radius);
        }
        sky_power_mean = (Phi[0] + Phi[1] + Phi[2]) / 3.0f;
    }
    if (sd.kind == 3) {
        // EqualAreaSkyLight (light.cpp:161-206): the map, an alias table over its texels'
        // luminance, and unit_power * pi r^2 as its power
        s->n_nonmesh = 1;
        const int res = (int)sd.width;
        const size_t n = (size_t)res * res;
        s->sky_w = s->sky_h = res;
        // a rotation: the light-to-world 3x3 of to_world and its transpose (light.slang:104, 153)
        for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 3; ++c) {
                s->sky_l2w[3 * r + c] = sd.to_world[4 * r + c];
                s->sky_w2l[3 * c + r] = sd.to_world[4 * r + c];
            }
        KS_CUDA_TRY(ctx, s->sky_map.alloc(n));
        k_sky_unpack<<<(unsigned)std::min<size_t>((n + 255) / 256, 4096), 256, 0, st>>>(s->sky_rgb.ptr, n,
                                                                                          s->sky_map.ptr);
        const std::vector<float> &t = s->sky_host;
        std::vector<float> lum(n);
        for (size_t i = 0; i < n; ++i)
            lum[i] = 0.212671f * t[3 * i] + 0.715160f * t[3 * i + 1] + 0.072169f * t[3 * i + 2];
        std::vector<float4> bins;
        if (!alias_table(lum, bins))
            return fail(ctx, KS_ERR_INVALID_ARGUMENT, "equal-area sky: the map has no positive luminance");
        KS_CUDA_TRY(ctx, s->sky_alias.alloc(n));
        KS_CUDA_TRY(ctx, cudaMemcpyAsync(s->sky_alias.ptr, bins.data(), sizeof(float4) * n, cudaMemcpyHostToDevice,
                                         st));
        KS_CUDA_TRY(ctx, cudaStreamSynchronize(st)); // bins lives on this stack frame
        // unit_power (light.cpp:182-198): row sums in float, rows summed in a fixed order
        double sum[3] = {0, 0, 0};
        for (int row = 0; row < res; ++row) {
            float rs[3] = {0, 0, 0};
            for (int col = 0; col < res; ++col)
                for (int c = 0; c < 3; ++c)
                    rs[c] += t[3 * ((size_t)row * res + col) + c];
            for (int c = 0; c < 3; ++c)
                sum[c] += rs[c];
        }
        const float pi = 3.14159265359f;
        float Phi[3] = {(float)sum[0], (float)sum[1], (float)sum[2]};
        const float scale = (4 * pi) / (float)(res * res);
        float ex = s->scene_bound[3] - s->scene_bound[0], ey = s->scene_bound[4] - s->scene_bound[1],
              ez = s->scene_bound[5] - s->scene_bound[2];
        float radius = 0.5f * std::sqrt(ex * ex + ey * ey + ez * ez);
        for (int c = 0; c < 3; ++c) {
            Phi[c] *= scale;
            Phi[c] *= pi * (radius * radius);
        }
        sky_power_mean = (Phi[0] + Phi[1] + Phi[2]) / 3.0f;
    }
    // ---- mesh lights (host: constant emission, a few triangles) ----
    std::vector<float> h_verts;
    std::vector<uint32_t> h_idx;
    std::vector<uint32_t> ml_tri;
    std::vector<float> ml_area, ml_importance;
    std::vector<float4> ml_em, ml_verts;
    std::vector<int32_t> inst_light_base;
    // ---- point and directional lights: after the sky, before the mesh lights ----
    s->n_nonmesh += (uint32_t)s->lights.size();
    if (!s->lights.empty()) {
        std::vector<float4> pl;
        for (const ks_light_desc &l : s->lights) {
            pl.push_back(make_float4(l.vec[0], l.vec[1], l.vec[2], (float)l.type));
            pl.push_back(make_float4(l.color[0], l.color[1], l.color[2], 0.0f));
        }
        KS_CUDA_TRY(ctx, s->punctual.alloc(pl.size()));
        KS_CUDA_TRY(ctx, cudaMemcpyAsync(s->punctual.ptr, pl.data(), sizeof(float4) * pl.size(),
                                         cudaMemcpyHostToDevice, st));
    }
    bool any_emission = false;
    for (size_t m = 0; m + 1 < s->host.mesh_tri_offset.size(); ++m)
        if (s->host.materials[s->host.mesh_material[m]].has_emission)
            any_emission = true;
    std::vector<int32_t> tri_light;
    if (any_emission) {
        h_idx.resize(3 * (size_t)s->n_tris);
        h_verts.resize(3 * (size_t)s->n_verts);
        KS_CUDA_TRY(ctx, cudaMemcpy(h_verts.data(), s->verts.ptr, s->verts.bytes(), cudaMemcpyDeviceToHost));
        KS_CUDA_TRY(ctx, cudaMemcpy(h_idx.data(), s->indices.ptr, s->indices.bytes(), cudaMemcpyDeviceToHost));
        tri_light.assign(s->n_tris, -1);
        auto vert = [&](uint32_t v, float out[3]) {
            out[0] = h_verts[3 * v];
            out[1] = h_verts[3 * v + 1];
            out[2] = h_verts[3 * v + 2];
        };
        // instanced scenes: the emissive triangles of each prototype, in light order, then one light
        // per (instance, triangle) with world-space vertices (Scene::build_mesh_lights, scene.cpp:315)
        const bool instanced = s->n_instances > 0;
        std::vector<std::vector<uint32_t>> proto_tris(s->n_protos);
        std::vector<std::vector<float4>> proto_em(s->n_protos);
        std::vector<std::vector<float>> proto_uvw(s->n_protos);
        std::vector<int> mesh_proto(s->host.mesh_material.size(), -1);
        if (instanced)
            for (uint32_t q = 0; q < s->n_protos; ++q)
                for (size_t m = 0; m + 1 < s->host.mesh_tri_offset.size(); ++m)
                    if (s->host.mesh_tri_offset[m] >= s->host.proto_tri_begin[q] &&
                        s->host.mesh_tri_offset[m + 1] <= s->host.proto_tri_end[q] &&
                        s->host.mesh_tri_offset[m + 1] > s->host.mesh_tri_offset[m])
                        mesh_proto[m] = (int)q;
        for (size_t m = 0; m + 1 < s->host.mesh_tri_offset.size(); ++m) {
            const ks_material_desc &mat = s->host.materials[s->host.mesh_material[m]];
            if (!mat.has_emission)
                continue;
            if (instanced && mesh_proto[m] < 0)
                continue;
            uint32_t first = s->host.mesh_tri_offset[m], n = s->host.mesh_tri_offset[m + 1] - first;
            // the per-triangle factor of 2 pi x area: the emission's luminance, or its texture's mean
            const MaterialGPU &mg = s->any_emission_map ? s->emit_tex.mats[s->host.mesh_material[m]] : MaterialGPU{};
            std::vector<float> uvw;
            if (s->any_emission_map) {
                mesh_uv_importance(s, mg, first, n, h_verts, h_idx, uvw);
            } else {
                uvw.assign(n, 0.212671f * mat.emission[0] + 0.715160f * mat.emission[1] + 0.072169f * mat.emission[2]);
            }
            // the emission binding of a textured emitter (index into the scene's bindings), else -1
            int em_bind = -1;
            if (s->any_emission_map)
                for (int b = 0; b < mg.bind_count; ++b)
                    if (s->emit_tex.binds[mg.bind_begin + b].field == KS_FIELD_EMISSION)
                        em_bind = mg.bind_begin + b;
            float em_bits;
            std::memcpy(&em_bits, &em_bind, 4);
            const float4 em4 = make_float4(mat.emission[0], mat.emission[1], mat.emission[2], em_bits);
            std::vector<float> importance(n), areas(n);
            std::vector<uint32_t> prim_ids(n);
            for (uint32_t k = 0; k < n; ++k) {
                float v0[3], v1[3], v2[3];
                vert(h_idx[3 * (first + k)], v0);
                vert(h_idx[3 * (first + k) + 1], v1);
                vert(h_idx[3 * (first + k) + 2], v2);
                float e01[3] = {v1[0] - v0[0], v1[1] - v0[1], v1[2] - v0[2]};
                float e12[3] = {v2[0] - v1[0], v2[1] - v1[1], v2[2] - v1[2]};
                float c[3] = {e01[1] * e12[2] - e01[2] * e12[1], e01[2] * e12[0] - e01[0] * e12[2],
                              e01[0] * e12[1] - e01[1] * e12[0]};
                float area = 0.5f * std::sqrt(c[0] * c[0] + c[1] * c[1] + c[2] * c[2]);
                importance[k] = 6.28318530718f * area * uvw[k];
                areas[k] = area;
                prim_ids[k] = k;
            }
            uint32_t N = n;
            for (uint32_t i = 0; i < N;) {
                if (importance[i] == 0.0f) {
                    std::swap(prim_ids[N - 1], prim_ids[i]);
                    std::swap(importance[N - 1], importance[i]);
                    std::swap(areas[N - 1], areas[i]);
                    --N;
                } else {
                    ++i;
                }
            }
            for (uint32_t k = 0; k < N; ++k) {
                if (instanced) {
                    int q = mesh_proto[m];
                    tri_light[first + prim_ids[k]] = (int32_t)proto_tris[q].size(); // rank in the prototype
                    proto_tris[q].push_back(first + prim_ids[k]);
                    proto_em[q].push_back(em4);
                    proto_uvw[q].push_back(uvw[prim_ids[k]]);
                    continue;
                }
                ml_tri.push_back(first + prim_ids[k]);
                ml_area.push_back(areas[k]);
                ml_importance.push_back(importance[k]);
                ml_em.push_back(em4);
                float v0[3], v1[3], v2[3];
                vert(h_idx[3 * (first + prim_ids[k])], v0);
                vert(h_idx[3 * (first + prim_ids[k]) + 1], v1);
                vert(h_idx[3 * (first + prim_ids[k]) + 2], v2);
                ml_verts.push_back(make_float4(v0[0], v0[1], v0[2], 0.0f));
                ml_verts.push_back(make_float4(v1[0], v1[1], v1[2], 0.0f));
                ml_verts.push_back(make_float4(v2[0], v2[1], v2[2], 0.0f));
            }
        }
        if (instanced) {
            for (uint32_t i = 0; i < s->n_instances; ++i) {
                inst_light_base.push_back((int32_t)(s->n_nonmesh + ml_tri.size()));
                const uint32_t q = s->host.inst_proto[i];
                const float *xf = &s->host.inst_xf[12 * (size_t)i];
                for (size_t r = 0; r < proto_tris[q].size(); ++r) {
                    uint32_t t = proto_tris[q][r];
                    f3 w[3];
                    for (int c = 0; c < 3; ++c) {
                        float v[3];
                        vert(h_idx[3 * (size_t)t + c], v);
                        w[c] = xf_point(xf, mk(v[0], v[1], v[2]));
                    }
                    f3 e01 = w[1] - w[0], e12 = w[2] - w[1];
                    f3 c = cross(e01, e12);
                    float area = 0.5f * std::sqrt(c.x * c.x + c.y * c.y + c.z * c.z);
                    float4 em = proto_em[q][r];
                    ml_tri.push_back(t);
                    ml_area.push_back(area);
                    ml_importance.push_back(6.28318530718f * area * proto_uvw[q][r]);
                    ml_em.push_back(em);
                    for (int c2 = 0; c2 < 3; ++c2)
                        ml_verts.push_back(make_float4(w[c2].x, w[c2].y, w[c2].z, 0.0f));
                }
            }
        }
    }
    // ---- PowerLightSampler::build ----
    uint32_t count = s->n_nonmesh + (uint32_t)ml_tri.size();
    s->light_count = count;
    s->h_powers.assign(count, 0.0f);
    uint32_t flat = 0;
    if (s->n_nonmesh > s->lights.size())
        s->h_powers[flat++] = sky_power_mean;
    for (const ks_light_desc &l : s->lights) {
        // PointLight::power = 4 pi I; DirectionalLight::power = L pi r^2 (light.cpp:218-240); mean
        float p[3];
        if (l.type == 0) {
            for (int c = 0; c < 3; ++c)
                p[c] = 4.0f * 3.14159265359f * l.color[c];
        } else {
            const float ex = s->scene_bound[3] - s->scene_bound[0], ey = s->scene_bound[4] - s->scene_bound[1],
                        ez = s->scene_bound[5] - s->scene_bound[2];
            const float r = 0.5f * std::sqrt(ex * ex + ey * ey + ez * ez);
            for (int c = 0; c < 3; ++c)
                p[c] = l.color[c] * 3.14159265359f * (r * r);
        }
        s->h_powers[flat++] = (p[0] + p[1] + p[2]) / 3.0f;
    }
    for (size_t k = 0; k < ml_tri.size(); ++k) {
        float pw = ml_importance[k];
        s->h_powers[flat] = (pw + pw + pw) / 3.0f;
        if (any_emission && s->n_instances == 0)
            tri_light[ml_tri[k]] = (int32_t)flat;
        ++flat;
    }
    if (count == 0) {
        // nothing to sample; ks_small_pt_render refuses such a scene
        s->lights_built = true;
        return KS_OK;
    }
    s->h_power_cdf = host_cdf(s->h_powers.data(), count);
    KS_CUDA_TRY(ctx, s->power_cdf.alloc(s->h_power_cdf.size()));
    KS_CUDA_TRY(ctx, cudaMemcpyAsync(s->power_cdf.ptr, s->h_power_cdf.data(), sizeof(float) * s->h_power_cdf.size(),
                                     cudaMemcpyHostToDevice, st));
    if (any_emission) {
        KS_CUDA_TRY(ctx, s->tri_light.alloc(tri_light.size()));
        KS_CUDA_TRY(ctx, s->ml_tri.alloc(ml_tri.size()));
        KS_CUDA_TRY(ctx, s->ml_area.alloc(ml_area.size()));
        KS_CUDA_TRY(ctx, s->ml_emission.alloc(ml_em.size()));
        KS_CUDA_TRY(ctx, cudaMemcpyAsync(s->tri_light.ptr, tri_light.data(), s->tri_light.bytes(),
                                         cudaMemcpyHostToDevice, st));
        KS_CUDA_TRY(ctx, cudaMemcpyAsync(s->ml_tri.ptr, ml_tri.data(), s->ml_tri.bytes(), cudaMemcpyHostToDevice, st));
        KS_CUDA_TRY(ctx,
                    cudaMemcpyAsync(s->ml_area.ptr, ml_area.data(), s->ml_area.bytes(), cudaMemcpyHostToDevice, st));
        KS_CUDA_TRY(ctx, cudaMemcpyAsync(s->ml_emission.ptr, ml_em.data(), s->ml_emission.bytes(),
                                         cudaMemcpyHostToDevice, st));
        KS_CUDA_TRY(ctx, s->ml_verts.alloc(std::max<size_t>(ml_verts.size(), 3)));
        if (!ml_verts.empty())
            KS_CUDA_TRY(ctx, cudaMemcpyAsync(s->ml_verts.ptr, ml_verts.data(), sizeof(float4) * ml_verts.size(),
                                             cudaMemcpyHostToDevice, st));
        if (!inst_light_base.empty()) {
            KS_CUDA_TRY(ctx, s->inst_light_base.alloc(inst_light_base.size()));
            KS_CUDA_TRY(ctx, cudaMemcpyAsync(s->inst_light_base.ptr, inst_light_base.data(),
                                             s->inst_light_base.bytes(), cudaMemcpyHostToDevice, st));
        }
    }
    KS_CUDA_TRY(ctx, cudaStreamSynchronize(st));
    s->lights_built = true;
    return KS_OK;
}

} // namespace ksb
