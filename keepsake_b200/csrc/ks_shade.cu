// Sampling and shading kernels of the small_pt wavefront (the k_sample and k_shade stages of
// ks_integrator.cu's loop).
//
// This translation unit is compiled with -use_fast_math (approximate division and square root,
// flush-to-zero, FMA contraction, fast sin/cos/exp/log); the rest of the library keeps IEEE
// arithmetic without contraction.  The bit-exact parts of the path (Sobol points, camera rays,
// SBVH traversal, the watertight triangle test) live in the other units; the arithmetic here
// (BSDF, light sampling, MIS, path throughput) is checked statistically against the FP64 oracle.
// Correctly rounded division and square root cost the shading kernel about 40 % of its time
// (their slow-path calls stall instruction fetch); the rest of fast math takes another 5 % off
// the frame.
#include "ks_bsdf.cuh"
#include "ks_sampler.cuh"
#include "ks_wavefront.cuh"
#include "ks_subsurface.cuh"

#include <type_traits>

namespace ksb
{
namespace
{
using namespace wave;

// Minimum resident CTAs per SM asked of the compiler (a register cap) for the shading kernel: it is
// latency bound, and at 8 CTAs of 128 (64 registers, a few dozen bytes of spills) it runs about
// 1.25x faster than at its natural register count (about 110: 4 CTAs).
#ifndef KS_SHADE_MIN_BLOCKS
#define KS_SHADE_MIN_BLOCKS 8
#endif

// NormalMap::apply (normal_map.cpp:24-40): the shading frame around the mapped normal, its tangent
// the old one tilted by the normal's slope (the frame's n is respected, t and b re-orthogonalised).
KS_D void apply_normal_map(const SceneView &sv, const BindingGPU &b, float u, float v, ShadeFrame &it)
{
    const float4 c = field_eval(sv.tex_texels, sv.tex_info, b, u, v);
    f3 s = mk(c.x, c.y, c.z);
    if (b.range01)
        s = mk(s.x * 2.0f - 1.0f, s.y * 2.0f - 1.0f, s.z * 2.0f - 1.0f);
    f3 normal = normalize(s);
    if (b.space == 0 && b.strength < 1.0f)
        normal = normalize((1.0f - b.strength) * mk(0.0f, 0.0f, 1.0f) + b.strength * normal);
    f3 np;
    if (b.space == 0)
        np = it.st * normal.x + it.sb * normal.y + it.sn * normal.z;
    else
        np = normalize(mk(b.nrm[0] * normal.x + b.nrm[1] * normal.y + b.nrm[2] * normal.z,
                          b.nrm[3] * normal.x + b.nrm[4] * normal.y + b.nrm[5] * normal.z,
                          b.nrm[6] * normal.x + b.nrm[7] * normal.y + b.nrm[8] * normal.z));
    const float bump_x = -normal.x / normal.z;
    f3 tp = normalize(it.st + bump_x * it.sn);
    const f3 bp = normalize(cross(np, tp));
    tp = normalize(cross(bp, np));
    it.st = tp;
    it.sb = bp;
    it.sn = np;
}

// The material's textured shader fields at the hit (TextureField, shader_field.h:61-80) over its
// constant ones, and its normal map applied to the shading frame.
KS_BIG MaterialGPU textured_material(const SceneView &sv, const MaterialGPU &mat, uint32_t tri, int flags, float u,
                                   float v, ShadeFrame &it)
{
    MaterialGPU m = mat;
    float tu, tv;
    hit_uv(sv, tri, flags, u, v, tu, tv);
    for (int k = 0; k < mat.bind_count; ++k) {
        const BindingGPU &b = sv.bindings[mat.bind_begin + k];
        if (b.field == KS_FIELD_OPACITY_MAP || b.field == KS_FIELD_EMISSION)
            continue; // applied by the traversal / the emitter's light (mesh_light_Le)
        if (b.field == KS_FIELD_NORMAL_MAP) {
            apply_normal_map(sv, b, tu, tv, it);
            continue;
        }
        const float4 c = field_eval(sv.tex_texels, sv.tex_info, b, tu, tv);
        switch (b.field) {
        case KS_FIELD_BASECOLOR:
            m.basecolor[0] = c.x;
            m.basecolor[1] = c.y;
            m.basecolor[2] = c.z;
            break;
        case KS_FIELD_ROUGHNESS: m.roughness = c.x; break;
        case KS_FIELD_METALLIC: m.metallic = c.x; break;
        case KS_FIELD_IOR: m.ior = c.x; break;
        case KS_FIELD_SPECULAR_R0_MUL: m.specular_r0_mul = c.x; break;
        case KS_FIELD_SPECULAR_TRANS: m.specular_trans = c.x; break;
        case KS_FIELD_DIFFUSE_TRANS: m.diffuse_trans = c.x; break;
        case KS_FIELD_DIFFUSE_TRANS_FWD: m.diffuse_trans_fwd = c.x; break;
        default: m.specular = c.x; break;
        }
    }
    return m;
}

// Sobol samples and the NEE light sample of one bounce for every path in the hit queue (whose
// bounce is below the limit).  Sobol dimensions: light selection (d), light uv (d+1, d+2), BSDF
// lobe (d+3), BSDF direction (d+4, d+5) and Russian roulette (d+6), exactly as sample_with_nee +
// trace() draw them (nee.cpp:28-34, material.cpp:157-158, small_pt.cpp:168-174).  The light is
// selected and sampled here too (next_event_estimate, nee.cpp:28-40), so the shading kernel keeps
// only the BSDF work: this kernel runs at full occupancy and SIMT efficiency, and the sky's
// binary searches no longer sit in the large shading kernel.
// samples[4 i + 0] = (lobe, wi u, wi v, roulette)
// samples[4 i + 1] = (light direction, light distance)
// samples[4 i + 2] = (Le / pdf of the light sample (Le_beta), pdf of the direction)
// samples[4 i + 3] = (light selection probability, 1 for a delta light, -, -)
template <bool kBatch = false>
__global__ void __launch_bounds__(128) k_sample(const __grid_constant__ SceneView sv_in,
                                                const __grid_constant__ RenderParams rp_in, PathBuf cur,
                                                const float4 *hits, const uint32_t *hit_inst, const uint32_t *queue,
                                                const uint32_t *queue_count, float4 *samples, BatchView bv)
{
    const uint32_t count = *queue_count;
    for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < count; q += gridDim.x * blockDim.x) {
        uint32_t i = queue[q];
        uint32_t pix = bits(cur.beta_pix[i].w), smp = bits(cur.L_smp[i].w);
        const uint32_t job = kBatch ? (pix >> kJobShift) : 0u;
        const RenderParams &rp = job_of<kBatch>(rp_in, bv.params, job);
        if constexpr (kBatch)
            pix &= kPixMask;
        uint32_t info = bits(cur.d_info[i].w);
        int bounce = (int)(info & 0xffffu);
        if (bounce == rp.bounces)
            continue;
        int dim = (int)(info >> 16);
        SobolSampler smp_s = SobolSampler::start(pix % (uint32_t)rp.W, pix / (uint32_t)rp.W, smp, rp.log2_spp,
                                                 rp.n_digits, (uint32_t)rp.seed, dim);
        float uv[7];
        smp_s.bounce_values(uv);
        const float ul = uv[0], u0 = uv[1], u1 = uv[2], u_lobe = uv[3], b0 = uv[4], b1 = uv[5], u_rr = uv[6];
        // next_event_estimate: light selection and the light's sample (nee.cpp:28-40)
        const SceneView &sv = job_of<kBatch>(sv_in, bv.views, job);
        uint32_t light = cdf_find(sv.power_cdf, sv.light_count, clamp_u(ul));
        float pr_light = sv.power_cdf[light + 1] - sv.power_cdf[light];
        f3 wi = mk(0, 0, 0);
        float wi_dist = 0.0f, pdf_wi_light = 0.0f;
        f3 Le_beta;
        float delta_light = 0.0f;
        if (light < sv.n_sky) {
            Le_beta = sky_sample(sv, u0, u1, wi, wi_dist, pdf_wi_light);
        } else if (light < sv.n_nonmesh) {
            // PointLight / DirectionalLight::sample (light.cpp:208-236): a delta light, weight 1
            delta_light = 1.0f;
            const float4 a = __ldg(&sv.punctual[2 * (size_t)(light - sv.n_sky)]);
            const float4 c = __ldg(&sv.punctual[2 * (size_t)(light - sv.n_sky) + 1]);
            pdf_wi_light = 1.0f;
            if (a.w == 0.0f) {
                const float4 h = hits[i];
                const float4 *pt = sv.prim_tris + 3 * (size_t)bits(h.w);
                float4 v0 = __ldg(pt), v1 = __ldg(pt + 1), v2 = __ldg(pt + 2);
                f3 p0 = mk(v0.x, v0.y, v0.z), p1 = mk(v1.x, v1.y, v1.z), p2 = mk(v2.x, v2.y, v2.z);
                if (sv.inst.n) {
                    const uint32_t inst = hit_inst[i];
                    float m[12];
#pragma unroll
                    for (int e = 0; e < 12; ++e)
                        m[e] = __ldg(&sv.inst.xf[12 * (size_t)inst + e]);
                    p0 = xf_point(m, p0);
                    p1 = xf_point(m, p1);
                    p2 = xf_point(m, p2);
                }
                wi = mk(a.x, a.y, a.z) - hit_point(p0, p1, p2, h.y, h.z);
                const float l2 = dot(wi, wi);
                if (l2 == 0.0f) {
                    Le_beta = mk(0, 0, 0);
                    pdf_wi_light = 0.0f;
                } else {
                    const float l = sqrtf(l2);
                    wi = mk(wi.x / l, wi.y / l, wi.z / l);
                    wi_dist = l;
                    Le_beta = mk(c.x / l2, c.y / l2, c.z / l2);
                }
            } else {
                wi = mk(a.x, a.y, a.z);
                wi_dist = kInf;
                Le_beta = mk(c.x, c.y, c.z);
            }
        } else {
            // the shading point as the hit record computes it (make_frame)
            const float4 h = hits[i];
            const float4 *pt = sv.prim_tris + 3 * (size_t)bits(h.w);
            float4 v0 = __ldg(pt), v1 = __ldg(pt + 1), v2 = __ldg(pt + 2);
            f3 p0 = mk(v0.x, v0.y, v0.z), p1 = mk(v1.x, v1.y, v1.z), p2 = mk(v2.x, v2.y, v2.z);
            if (sv.inst.n) {
                const uint32_t inst = hit_inst[i];
                float m[12];
#pragma unroll
                for (int e = 0; e < 12; ++e)
                    m[e] = __ldg(&sv.inst.xf[12 * (size_t)inst + e]);
                p0 = xf_point(m, p0);
                p1 = xf_point(m, p1);
                p2 = xf_point(m, p2);
            }
            const f3 p = hit_point(p0, p1, p2, h.y, h.z);
            uint32_t k = light - sv.n_nonmesh;
            const float4 *mv = sv.ml_verts + 3 * (size_t)k;
            float4 a0 = __ldg(mv), a1 = __ldg(mv + 1), a2 = __ldg(mv + 2);
            TriVerts tv{mk(a0.x, a0.y, a0.z), mk(a1.x, a1.y, a1.z), mk(a2.x, a2.y, a2.z)};
            Le_beta = mesh_light_sample(sv, k, tv, p, u0, u1, wi, wi_dist, pdf_wi_light);
        }
        samples[4 * (size_t)i] = make_float4(u_lobe, b0, b1, u_rr);
        samples[4 * (size_t)i + 1] = make_float4(wi.x, wi.y, wi.z, wi_dist);
        samples[4 * (size_t)i + 2] = make_float4(Le_beta.x, Le_beta.y, Le_beta.z, pdf_wi_light);
        samples[4 * (size_t)i + 3] = make_float4(pr_light, delta_light, 0.0f, 0.0f);
    }
}

// Shading of the paths listed in `queue` (indices into the current path buffer).  kMiss = true
// handles the rays that left the scene, kMiss = false the rays that hit a triangle; the extension
// kernel sorts the two kinds into separate queues so that a warp runs one of the two code paths.
// kGuided: directions are drawn from the guide's mixture or the BSDF (one-sample MIS: the
// throughput divides by the combined density) and paths capture training records (layout in
// ks_guide_view.cuh).  The light MIS weights keep the BSDF pdf, so the estimator has the
// expectation of the unguided one: the reference's NEE weight omits the light-selection
// probability that its emitter-hit weight includes, and the two only stay the same functions of
// the direction if both keep seeing the BSDF pdf.
// kBatch: paths of many jobs; the view, parameters and accumulators of a path's job come from bv.
// kVariant (kShadePlain, kShadeAttribs, kShadeGeneral): kShadeAttribs lets meshes carry vertex
// normals (smooth shading frames) and texcoords (tangents); kShadeGeneral also takes materials of
// any BSDF kind (AnyBsdf).  The plain variant's materials are all GGX PrincipledBSDFs, whose code
// alone keeps the kernel's register budget; each variant keeps the spills of its own features.
template <bool kMiss, bool kGuided, bool kBatch = false, int kVariant = kShadePlain>
__global__ void __launch_bounds__(128, KS_SHADE_MIN_BLOCKS) k_shade(const __grid_constant__ SceneView sv_in,
                                               const __grid_constant__ RenderParams rp_in, PathBuf cur, PathBuf nxt,
                                               const float4 *hits, const uint32_t *hit_inst,
                                               const float4 *samples, const uint32_t *queue,
                                               const uint32_t *queue_count, uint32_t *next_count, ShadowBuf sb,
                                               uint32_t *shadow_count, double *accum_in, double *weights_in,
                                               GuideView gv, BatchView bv)
{
    const uint32_t stride = gridDim.x * blockDim.x;
    const uint32_t count = *queue_count;
    for (uint32_t base = blockIdx.x * blockDim.x; base < count; base += stride) {
        bool valid = base + threadIdx.x < count;
        uint32_t i = valid ? queue[base + threadIdx.x] : 0u;
        bool cont = false, shadow = false;
        // outputs
        f3 n_o = mk(0, 0, 0), n_d = n_o, n_beta = n_o, L = n_o, sh_o = n_o, sh_d = n_o, sh_c = n_o;
        float n_pdf = 0.0f, sh_tmax = 0.0f;
        uint32_t n_info = 0, pix = 0, smp = 0;
        bool finish = false, miss_only = false;
        // guided renders: the path's record, and a record to create at this vertex
        uint32_t rec = kNoRecord;
        bool want_rec = false;
        f3 rc_p = mk(0, 0, 0), rc_wo = mk(0, 0, 0), rc_wi = mk(0, 0, 0), rc_beta = mk(0, 0, 0), rc_n = mk(0, 0, 0);
        float rc_pb = 0.0f;
        int rc_bounce = 0;
        if (valid) {
            float4 a = cur.o_pdf[i], b = cur.d_info[i], c = cur.beta_pix[i], d = cur.L_smp[i];
            f3 ro = mk(a.x, a.y, a.z), rd = mk(b.x, b.y, b.z);
            float pdf_wi_bsdf = a.w;
            uint32_t info = bits(b.w);
            int bounce = (int)(info & 0xffffu);
            int dim = (int)(info >> 16);
            f3 beta = mk(c.x, c.y, c.z);
            pix = bits(c.w);
            L = mk(d.x, d.y, d.z);
            smp = bits(d.w);
            const uint32_t job = kBatch ? (pix >> kJobShift) : 0u;
            const SceneView &sv = job_of<kBatch>(sv_in, bv.views, job);
            const RenderParams &rp = job_of<kBatch>(rp_in, bv.params, job);
            float4 h = hits[i];
            uint32_t slot = bits(h.w);
            if constexpr (kGuided)
                rec = cur.rec[i];
            if constexpr (kMiss) {
                (void)slot;
                // miss: unidirectional sky strategy (small_pt.cpp:83-110)
                if (sv.sky_kind != 0) {
                    f3 wi = normalize(rd);
                    f3 Le = sky_eval(sv, wi);
                    if (bounce == 0) {
                        if (rp.include_background)
                            L += beta * Le;
                    } else {
                        float pr_light = light_probability(sv, 0);
                        float pdf_wi_light = sky_pdf(sv, wi);
                        float mis = power_heur(pdf_wi_bsdf, pdf_wi_light * pr_light);
                        f3 beta_uni = clamp_contrib(Le * mis, bounce, rp, false);
                        L += beta * beta_uni;
                        if constexpr (kGuided)
                            if (rec != kNoRecord)
                                record_add(gv, rec, beta * beta_uni);
                    }
                }
                finish = true;
                if (bounce == 0 && !rp.include_background)
                    miss_only = true;
            } else {
                const float4 *pt = sv.prim_tris + 3 * (size_t)slot;
                float4 v0 = __ldg(pt), v1 = __ldg(pt + 1), v2 = __ldg(pt + 2);
                uint32_t tri = bits(v0.w);
                f3 p0 = mk(v0.x, v0.y, v0.z), p1 = mk(v1.x, v1.y, v1.z), p2 = mk(v2.x, v2.y, v2.z);
                uint32_t inst = 0;
                float m[12];
                if (sv.inst.n) {
                    // instanced: the hit triangle in world space (transform_it, ray.h:166-183)
                    inst = hit_inst[i];
#pragma unroll
                    for (int e = 0; e < 12; ++e)
                        m[e] = __ldg(&sv.inst.xf[12 * (size_t)inst + e]);
                    p0 = xf_point(m, p0);
                    p1 = xf_point(m, p1);
                    p2 = xf_point(m, p2);
                }
                uint32_t mesh = __ldg(&sv.tri_mesh[tri]);
                const MaterialGPU &mat_c = sv.materials[__ldg(&sv.mesh_material[mesh])];
                const int mesh_flags = __ldg(&sv.mesh_flags[mesh]);
                ShadeFrame it = hit_frame<(kVariant >= kShadeAttribs)>(sv, tri, mesh_flags, p0, p1, p2, h.y, h.z, rd,
                                          sv.inst.n ? m : nullptr);
                // textured fields and normal maps (general variant; Scene::intersect1 applies the
                // normal map right after the hit record, scene.cpp:229-233)
                MaterialGPU mat_t;
                if constexpr (kVariant == kShadeGeneral)
                    if (mat_c.bind_count)
                        mat_t = textured_material(sv, mat_c, tri, mesh_flags, h.y, h.z, it);
                const MaterialGPU &mat = (kVariant == kShadeGeneral && mat_c.bind_count) ? mat_t : mat_c;
                // emitter hit (small_pt.cpp:112-138)
                if (mat.has_emission && sv.tri_light) {
                    int32_t light = __ldg(&sv.tri_light[tri]);
                    if (light >= 0 && sv.inst.n)
                        light += __ldg(&sv.inst_light_base[inst]); // rank within the prototype
                    if (light >= 0) {
                        uint32_t k = (uint32_t)light - sv.n_nonmesh;
                        // textured emitters have bindings, so only the general variant meets them
                        f3 Le;
                        if constexpr (kVariant == kShadeGeneral) {
                            Le = mesh_light_Le(sv, k, h.y, h.z, true);
                        } else {
                            const float4 e = __ldg(&sv.ml_emission[k]);
                            Le = mk(e.x, e.y, e.z);
                        }
                        if (bounce == 0) {
                            L += beta * Le;
                        } else {
                            float pr_light = light_probability(sv, (uint32_t)light);
                            if (pr_light > 0.0f) {
                                f3 wi = normalize(rd);
                                TriVerts tv{p0, p1, p2};
                                float pdf_wi_light = mesh_light_pdf(sv, k, tv, wi, h.x);
                                float mis = power_heur(pdf_wi_bsdf, pdf_wi_light * pr_light);
                                f3 beta_uni = clamp_contrib(Le * mis, bounce, rp, false);
                                L += beta * beta_uni;
                                if constexpr (kGuided)
                                    if (rec != kNoRecord)
                                        record_add(gv, rec, beta * beta_uni);
                            }
                        }
                    }
                }
                if (bounce == rp.bounces) {
                    finish = true;
                } else {
                    f3 wo = -normalize(rd);
                    // a random walk's exit (k_subsurface marks its hit distance negative) shades with the
                    // Lambertian exit lobe
                    const std::conditional_t<kVariant == kShadeGeneral, AnyBsdf, Principled> bsdf{
                        kVariant == kShadeGeneral && h.x < 0.0f ? subsurface_exit_closure(mat.ss_ior) : make_closure(mat)};
                    // this bounce's Sobol values and light sample, drawn by k_sample
                    const float4 sa = samples[4 * (size_t)i], sl = samples[4 * (size_t)i + 1];
                    const float4 se = samples[4 * (size_t)i + 2];
                    const float4 s3 = samples[4 * (size_t)i + 3];
                    const float pr_light = s3.x;
                    // next_event_estimate (nee.cpp:11-57): the light sample's BSDF term and MIS
                    const f3 wi = mk(sl.x, sl.y, sl.z);
                    const float wi_dist = sl.w, pdf_wi_light = se.w;
                    const f3 Le_beta = mk(se.x, se.y, se.z);
                    if (!is_zero(Le_beta) && pdf_wi_light > 0.0f) {
                        f3 wo_l = sh_to_local(it, wo), wi_l = sh_to_local(it, wi);
                        f3 f;
                        float pdf_b;
                        bsdf.eval_and_pdf(wo_l, wi_l, f, pdf_b);
                        if (!is_zero(f) && pdf_b > 0.0f) {
                            // delta lights: weight 1 (nee.cpp:45-48)
                            float mis = s3.y != 0.0f ? 1.0f : power_heur(pdf_wi_light, pdf_b);
                            f3 Ld = Le_beta * f * mis / pr_light;
                            Ld = clamp_contrib(Ld, bounce, rp, true);
                            shadow = true;
                            sh_o = spawn_origin(it.p, wi, it.n);
                            sh_d = wi;
                            sh_tmax = wi_dist;
                            sh_c = beta * Ld;
                        }
                    }
                    // BSDF sampling (material.cpp:155-166)
                    f3 wo_local = sh_to_local(it, wo);
                    float u_lobe = sa.x;
                    float b0 = sa.y, b1 = sa.z;
                    int next_dim = dim + 6;
                    f3 wi_local;
                    float pdf_wi = 0.0f;
                    f3 sbeta, wnext;
                    bool guided = false;
                    float p_bsdf = 0.0f; // BSDF pdf of the sampled direction
                    if constexpr (kGuided)
                        guided = gv.active != 0;
                    if (guided) {
                        // one-sample MIS of the guide (probability alpha of this vertex) and the BSDF
                        const float al = guide_alpha(gv, i);
                        f3 fcos;
                        float p_b = 0.0f;
                        if (u_lobe < al) {
                            wnext = guide_sample(gv, i, b0, b1);
                            wi_local = sh_to_local(it, wnext);
                            bsdf.eval_and_pdf(wo_local, wi_local, fcos, p_b);
                        } else {
                            float ub = fminf((u_lobe - al) / (1.0f - al), 0x1.fffffep-1f);
                            f3 fs = bsdf.sample(wo_local, wi_local, ub, b0, b1, p_b);
                            fcos = fs * p_b;
                            wnext = sh_to_world(it, wi_local);
                        }
                        // throughput over the density the direction was drawn from; the MIS weights
                        // with the lights keep the BSDF pdf (pdf_wi), as in the unguided estimator
                        // (alpha 0: a vertex the guide skipped; its mixture slots hold nothing)
                        const float q_al = al > 0.0f ? guide_pdf(gv, i, wnext) : 0.0f;
                        const float pdf_mix = is_zero(fcos) ? 0.0f : q_al + (1.0f - al) * p_b;
                        sbeta = pdf_mix > 0.0f ? fcos / pdf_mix : mk(0, 0, 0);
                        pdf_wi = p_b;
                        p_bsdf = p_b;
                    } else {
                        sbeta = bsdf.sample(wo_local, wi_local, u_lobe, b0, b1, pdf_wi);
                        p_bsdf = pdf_wi;
                    }
                    f3 nbeta = beta * sbeta;
                    if (max3(nbeta) == 0.0f) {
                        finish = true;
                    } else {
                        if (!guided)
                            wnext = sh_to_world(it, wi_local);
                        n_o = spawn_origin(it.p, wnext, it.n);
                        n_d = wnext;
                        n_pdf = pdf_wi;
                        // Russian roulette (small_pt.cpp:168-175)
                        if (max3(nbeta) < 1.0f && bounce >= 1) {
                            float q = 1.0f - max3(nbeta);
                            q = q < 0.0f ? 0.0f : q;
                            next_dim = dim + 7;
                            if (sa.w < q)
                                finish = true;
                            else
                                nbeta /= 1.0f - q;
                        }
                        if (!finish) {
                            cont = true;
                            n_beta = nbeta;
                            n_info = ((uint32_t)next_dim << 16) | (uint32_t)(bounce + 1);
                            if constexpr (kGuided) {
                                if (gv.rec_cap && rec == kNoRecord && mat.roughness >= gv.min_roughness) {
                                    uint32_t hh = path_hash(pix, smp);
                                    if ((hh & 0xffffu) < gv.rec_threshold && (uint32_t)bounce == (hh >> 16) % gv.rec_bounces) {
                                        want_rec = true;
                                        rc_p = it.p;
                                        rc_wo = wo;
                                        rc_wi = wnext;
                                        rc_beta = beta;
                                        rc_pb = p_bsdf;
                                        rc_n = guide::facing_normal(p0, p1, p2, wo);
                                        rc_bounce = bounce;
                                    }
                                }
                            }
                        }
                    }
                }
            }
        }
        uint32_t jc, js;
        block_append2(next_count, cont, shadow_count, shadow, jc, js);
        const uint32_t sh_rec = rec; // the shadow ray of this vertex feeds the path's earlier record
        if constexpr (kGuided) {
            uint32_t jr = warp_append(gv.rec_count, want_rec);
            if (want_rec && jr < gv.rec_cap) {
                gv.rec_pos[jr] = make_float4(rc_p.x, rc_p.y, rc_p.z, fbits((uint32_t)rc_bounce));
                gv.rec_wo[jr] = make_float4(rc_wo.x, rc_wo.y, rc_wo.z, rc_pb);
                gv.rec_wi[jr] = make_float4(rc_wi.x, rc_wi.y, rc_wi.z, 0.0f);
                gv.rec_n[jr] = make_float4(rc_n.x, rc_n.y, rc_n.z, 0.0f);
                gv.rec_ibeta[jr] = make_float4(rc_beta.x > 0.0f ? 1.0f / rc_beta.x : 0.0f,
                                               rc_beta.y > 0.0f ? 1.0f / rc_beta.y : 0.0f,
                                               rc_beta.z > 0.0f ? 1.0f / rc_beta.z : 0.0f, 0.0f);
                gv.rec_t[jr] = 0.0f;
                rec = jr;
            }
            if (cont)
                nxt.rec[jc] = rec;
        }
        if (cont) {
            nxt.o_pdf[jc] = make_float4(n_o.x, n_o.y, n_o.z, n_pdf);
            nxt.d_info[jc] = make_float4(n_d.x, n_d.y, n_d.z, fbits(n_info));
            nxt.beta_pix[jc] = make_float4(n_beta.x, n_beta.y, n_beta.z, fbits(pix));
            nxt.L_smp[jc] = make_float4(L.x, L.y, L.z, fbits(smp));
        }
        if (shadow) {
            sb.o_tmax[js] = make_float4(sh_o.x, sh_o.y, sh_o.z, sh_tmax);
            sb.d_target[js] = make_float4(sh_d.x, sh_d.y, sh_d.z, fbits(cont ? jc : (kTermBit | pix)));
            // the w component: the path's earlier record (guided), or its job (batched)
            sb.contrib[js] = make_float4(sh_c.x, sh_c.y, sh_c.z, fbits(kBatch ? (pix >> kJobShift) : sh_rec));
            if (!cont)
                sb.L_term[js] = make_float4(L.x, L.y, L.z, 0.0f);
        }
        if (valid && !cont && !shadow) {
            double *accum = accum_in, *weights = weights_in;
            uint32_t px = pix;
            if constexpr (kBatch) {
                accum = bv.accum[pix >> kJobShift];
                weights = bv.weights[pix >> kJobShift];
                px = pix & kPixMask;
            }
            if (miss_only)
                atomicAdd(&weights[2 * (size_t)px + 1], 1.0);
            else
                accumulate(accum, weights, px, L);
        }
    }
}

// BSDF parity hooks: the shading kernels' BSDF code (AnyBsdf, compiled in this fast-math unit)
// on batches of local directions.
__global__ void k_bsdf_eval(const MaterialGPU m, const float *wo, const float *wi, uint32_t n, float *f, float *pdf)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    const AnyBsdf b{make_closure(m)};
    f3 fv;
    float p;
    b.eval_and_pdf(mk(wo[3 * i], wo[3 * i + 1], wo[3 * i + 2]), mk(wi[3 * i], wi[3 * i + 1], wi[3 * i + 2]), fv, p);
    f[3 * i] = fv.x;
    f[3 * i + 1] = fv.y;
    f[3 * i + 2] = fv.z;
    pdf[i] = p;
}

__global__ void k_bsdf_sample(const MaterialGPU m, const float *wo, const float *u, uint32_t n, float *wi,
                              float *beta, float *pdf)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    const AnyBsdf b{make_closure(m)};
    f3 w = mk(0, 0, 0);
    float p = 0.0f;
    const f3 bt = b.sample(mk(wo[3 * i], wo[3 * i + 1], wo[3 * i + 2]), w, u[3 * i], u[3 * i + 1], u[3 * i + 2], p);
    wi[3 * i] = w.x;
    wi[3 * i + 1] = w.y;
    wi[3 * i + 2] = w.z;
    beta[3 * i] = bt.x;
    beta[3 * i + 1] = bt.y;
    beta[3 * i + 2] = bt.z;
    pdf[i] = p;
}

// Runs one of the hooks over host arrays of n entries: two inputs of 3 floats each, outputs of 3
// floats (out3a, and out3b when sampling) and of one float, copied back.
template <class Launch>
ks_status bsdf_hook(ks_context *ctx, const ks_material_desc *mat, uint32_t n, const float *in0, const float *in1,
                    float *out3a, float *out3b, bool sampling, float *out1, Launch launch, const char *what)
{
    if (!ctx || !mat || (n && (!in0 || !in1 || !out3a || !out1 || (sampling && !out3b))))
        return fail(ctx, KS_ERR_INVALID_ARGUMENT, std::string(what) + ": null argument");
    if (n > (1u << 26))
        return fail(ctx, KS_ERR_INVALID_ARGUMENT, std::string(what) + ": at most 2^26 entries per call");
    if (n == 0)
        return KS_OK;
    MaterialGPU g;
    if (!material_to_gpu(*mat, g))
        return fail(ctx, KS_ERR_INVALID_ARGUMENT, std::string(what) + ": invalid material");
    KS_CUDA_TRY(ctx, enter_device(ctx));
    const size_t v3 = 3 * (size_t)n * sizeof(float);
    DevBuf<float> buf;
    KS_CUDA_TRY(ctx, buf.alloc(3 * 3 * (size_t)n + 3 * (size_t)n + n));
    float *d_in0 = buf.ptr, *d_in1 = d_in0 + 3 * (size_t)n, *d_a = d_in1 + 3 * (size_t)n, *d_b = d_a + 3 * (size_t)n,
          *d_p = d_b + 3 * (size_t)n;
    cudaStream_t st = ctx->stream;
    KS_CUDA_TRY(ctx, cudaMemcpyAsync(d_in0, in0, v3, cudaMemcpyHostToDevice, st));
    KS_CUDA_TRY(ctx, cudaMemcpyAsync(d_in1, in1, v3, cudaMemcpyHostToDevice, st));
    launch((n + 127) / 128, st, g, d_in0, d_in1, d_a, d_b, d_p);
    KS_CUDA_TRY(ctx, cudaGetLastError());
    KS_CUDA_TRY(ctx, cudaMemcpyAsync(out3a, d_a, v3, cudaMemcpyDeviceToHost, st));
    if (sampling)
        KS_CUDA_TRY(ctx, cudaMemcpyAsync(out3b, d_b, v3, cudaMemcpyDeviceToHost, st));
    KS_CUDA_TRY(ctx, cudaMemcpyAsync(out1, d_p, n * sizeof(float), cudaMemcpyDeviceToHost, st));
    KS_CUDA_TRY(ctx, cudaStreamSynchronize(st));
    return KS_OK;
}

} // namespace

namespace wave
{

// Subsurface entries (Material::sample_with_nee, material.cpp:101-140), before the light samples of
// a bounce: every hit on a material with a BSSRDF draws one Sobol value (the path's dimension moves
// on by one): below 1/2 the path keeps its BSDF (beta x 2); else beta x 2 / ior^2 and a random walk
// from the hit (subsurface_walk).  A successful walk replaces the hit record by its exit (a negative
// distance marks it: the shading there uses the Lambertian exit lobe) and the ray direction by its
// last direction (the exit's wo), and multiplies beta by its throughput; a failed walk zeroes beta,
// which ends the path.
struct MeshOnly
{
    const uint32_t *tri_mesh;
    uint32_t mesh;
    KS_D bool operator()(uint32_t tri, float, float, const RayQuery &) const { return __ldg(&tri_mesh[tri]) == mesh; }
};

__global__ void __launch_bounds__(128) k_subsurface(const __grid_constant__ SceneView sv, const __grid_constant__ RenderParams rp,
                                                    PathBuf cur, float4 *hits, const uint32_t *queue,
                                                    const uint32_t *queue_count, int *overflow)
{
    const uint32_t count = *queue_count;
    for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < count; q += gridDim.x * blockDim.x) {
        const uint32_t i = queue[q];
        const float4 h = hits[i];
        const float4 *pt = sv.prim_tris + 3 * (size_t)bits(h.w);
        const float4 v0 = __ldg(pt), v1 = __ldg(pt + 1), v2 = __ldg(pt + 2);
        const uint32_t tri = bits(v0.w);
        const uint32_t mesh = __ldg(&sv.tri_mesh[tri]);
        const MaterialGPU &mat = sv.materials[__ldg(&sv.mesh_material[mesh])];
        if (!mat.has_ss)
            continue;
        float4 d4 = cur.d_info[i];
        const uint32_t info = bits(d4.w);
        const uint32_t bounce = info & 0xffffu;
        if ((int)bounce == rp.bounces)
            continue; // the path ends at this hit (small_pt.cpp:140-142): nothing is sampled
        const int dim = (int)(info >> 16);
        const float4 bp = cur.beta_pix[i];
        const uint32_t pix = bits(bp.w), smp = bits(cur.L_smp[i].w);
        SobolSampler sob = SobolSampler::start(pix % (uint32_t)rp.W, pix / (uint32_t)rp.W, smp, rp.log2_spp,
                                               rp.n_digits, (uint32_t)rp.seed, dim);
        const float u_sel = sob.next();
        d4.w = fbits(((uint32_t)(dim + 1) << 16) | bounce);
        f3 beta = mk(bp.x, bp.y, bp.z);
        if (u_sel < 0.5f) {
            beta *= 2.0f;
        } else {
            f3 tp = mk(2.0f, 2.0f, 2.0f);
            tp /= sqr(mat.ss_ior);
            const f3 p0 = mk(v0.x, v0.y, v0.z), p1 = mk(v1.x, v1.y, v1.z), p2 = mk(v2.x, v2.y, v2.z);
            const int flags = __ldg(&sv.mesh_flags[mesh]);
            ShadeFrame it = hit_frame<true>(sv, tri, flags, p0, p1, p2, h.y, h.z, mk(d4.x, d4.y, d4.z), nullptr);
            if (mat.tex_flags & kMatNormalMap)
                (void)textured_material(sv, mat, tri, flags, h.y, h.z, it);
            SsProfile prof;
            prof.albedo = mk(mat.ss_albedo[0], mat.ss_albedo[1], mat.ss_albedo[2]);
            prof.radius = mk(mat.ss_radius[0], mat.ss_radius[1], mat.ss_radius[2]);
            prof.g = mat.ss_g;
            prof.ior = mat.ss_ior;
            prof.rfr_entry_prob = mat.ss_rfr;
            Pcg32 rng = subsurface_stream(pix % (uint32_t)rp.W, pix / (uint32_t)rp.W, (uint32_t)rp.seed, smp, bounce);
            int of = 0;
            auto cast = [&](const RayQuery &ray, WalkExit &e) {
                Hit hh;
                traverse<false>(sv.nodes, sv.prim_tris, sv.root_ref, sv.root_count, sv.bmin, sv.bmax, ray, 2, hh, of,
                                nullptr, MeshOnly{sv.tri_mesh, mesh});
                if (hh.tri == ~0u)
                    return false;
                e = WalkExit{hh.slot, hh.t, hh.b1, hh.b2};
                return true;
            };
            WalkExit ex;
            f3 wi;
            if (subsurface_walk(prof, it.p, it.sn, it.n, rng, cast, tp, ex, wi)) {
                beta = beta * tp;
                hits[i] = make_float4(-1.0f, ex.b1, ex.b2, fbits(ex.slot));
                d4.x = wi.x;
                d4.y = wi.y;
                d4.z = wi.z;
            } else {
                beta = mk(0, 0, 0);
            }
            if (of)
                atomicOr(overflow, 1);
        }
        cur.d_info[i] = d4;
        cur.beta_pix[i] = make_float4(beta.x, beta.y, beta.z, bp.w);
    }
}

void launch_subsurface(unsigned grid, cudaStream_t st, const SceneView &sv, const RenderParams &rp, PathBuf cur,
                       float4 *hits, const uint32_t *queue, const uint32_t *queue_count, int *overflow)
{
    k_subsurface<<<grid, 128, 0, st>>>(sv, rp, cur, hits, queue, queue_count, overflow);
}

void launch_sample(bool batch, unsigned grid, cudaStream_t st, const SceneView &sv, const RenderParams &rp,
                   PathBuf cur, const float4 *hits, const uint32_t *hit_inst, const uint32_t *queue,
                   const uint32_t *queue_count, float4 *samples, const BatchView &bv)
{
    if (batch)
        k_sample<true><<<grid, 128, 0, st>>>(sv, rp, cur, hits, hit_inst, queue, queue_count, samples, bv);
    else
        k_sample<false><<<grid, 128, 0, st>>>(sv, rp, cur, hits, hit_inst, queue, queue_count, samples, bv);
}

void launch_shade(bool miss, bool guided, bool batch, int variant, unsigned grid, cudaStream_t st,
                  const SceneView &sv, const RenderParams &rp, PathBuf cur, PathBuf nxt, const float4 *hits,
                  const uint32_t *hit_inst, const float4 *samples, const uint32_t *queue, const uint32_t *queue_count,
                  uint32_t *next_count, ShadowBuf sb, uint32_t *shadow_count, double *accum, double *weights,
                  const GuideView &gv, const BatchView &bv)
{
#define KS_SHADE_ARGS                                                                                              \
    sv, rp, cur, nxt, hits, hit_inst, samples, queue, queue_count, next_count, sb, shadow_count, accum, weights, gv, bv
#define KS_SHADE_HIT(G, B)                                                                                         \
    do {                                                                                                           \
        if (variant == kShadeGeneral)                                                                             \
            k_shade<false, G, B, kShadeGeneral><<<grid, 128, 0, st>>>(KS_SHADE_ARGS);                              \
        else if (variant == kShadeAttribs)                                                                        \
            k_shade<false, G, B, kShadeAttribs><<<grid, 128, 0, st>>>(KS_SHADE_ARGS);                              \
        else                                                                                                       \
            k_shade<false, G, B, kShadePlain><<<grid, 128, 0, st>>>(KS_SHADE_ARGS);                                \
    } while (0)
    if (batch) {
        if (miss)
            k_shade<true, false, true><<<grid, 128, 0, st>>>(KS_SHADE_ARGS);
        else
            KS_SHADE_HIT(false, true);
    } else if (guided) {
        if (miss)
            k_shade<true, true><<<grid, 128, 0, st>>>(KS_SHADE_ARGS);
        else
            KS_SHADE_HIT(true, false);
    } else {
        if (miss)
            k_shade<true, false><<<grid, 128, 0, st>>>(KS_SHADE_ARGS);
        else
            KS_SHADE_HIT(false, false);
    }
#undef KS_SHADE_HIT
#undef KS_SHADE_ARGS
}

} // namespace wave
} // namespace ksb

extern "C" {

ks_status ks_bsdf_eval(ks_context *ctx, const ks_material_desc *mat, const float *wo, const float *wi, uint32_t n,
                       float *f, float *pdf)
{
    using namespace ksb;
    return bsdf_hook(ctx, mat, n, wo, wi, f, nullptr, false, pdf,
                     [n](unsigned grid, cudaStream_t st, const MaterialGPU &g, const float *a, const float *b,
                         float *oa, float *, float *op) { k_bsdf_eval<<<grid, 128, 0, st>>>(g, a, b, n, oa, op); },
                     "ks_bsdf_eval");
}

ks_status ks_bsdf_sample(ks_context *ctx, const ks_material_desc *mat, const float *wo, const float *u, uint32_t n,
                         float *wi, float *beta, float *pdf)
{
    using namespace ksb;
    return bsdf_hook(ctx, mat, n, wo, u, wi, beta, true, pdf,
                     [n](unsigned grid, cudaStream_t st, const MaterialGPU &g, const float *a, const float *b,
                         float *oa, float *ob, float *op) {
                         k_bsdf_sample<<<grid, 128, 0, st>>>(g, a, b, n, oa, ob, op);
                     },
                     "ks_bsdf_sample");
}

} // extern "C"
