"""Textured shader fields and normal maps (TextureField, shader_field.h:38-86; Texture, texture.cpp;
NormalMap, normal_map.cpp:9-40): the CUDA renderer against the oracle's restatement on the same
samples, with the tolerances of tests/test_render.py.

The scene is the box room with its floor, back wall and boxes textured: 8-bit sRGB, 16-bit and
float textures of 1, 3 and 4 channels; nearest, bilinear and bicubic (Catmull-Rom, B-spline)
lookups with repeat and clamp wrapping, flip_v, uv_scale / uv_offset, swizzle and scale; base colour,
roughness and metallic fields; a tangent-space normal map with strength 0.7 and a world-space one
under a rotation.  The back wall carries texture coordinates that run past [0, 1] (wrapping); the
other meshes use their barycentrics, as the reference does without texcoords (geometry.cpp:78-80)."""
import ctypes

import numpy as np
import pytest

from imaging import composite, rel_mse


def textures():
    rng = np.random.default_rng(5)
    ys, xs = np.mgrid[0:64, 0:64]
    checker = (((xs // 8) + (ys // 8)) % 2).astype(np.float32)
    t0 = np.stack([40 + 200 * checker, 60 + 150 * checker, 200 - 150 * checker], -1).astype(np.uint8)
    gy, gx = np.mgrid[0:32, 0:32] / 31.0
    t1 = np.stack([gx, gy, 0.5 * (gx + gy)], -1).astype(np.float32)
    t2 = (rng.random((16, 16, 1)) * 65535).astype(np.uint16)
    # a bumpy tangent-space normal map (range01 encoding, alpha channel unused)
    a = np.sin(gx * 9.0) * 0.35
    b = np.cos(gy * 7.0) * 0.35
    n = np.stack([a, b, np.ones_like(a)], -1)
    n /= np.linalg.norm(n, axis=-1, keepdims=True)
    t3 = np.concatenate([n * 0.5 + 0.5, np.ones_like(a)[..., None]], -1).astype(np.float32)
    return [(t0, True), (t1, False), (t2, False), (t3, False)]


def rot_z(deg):
    c, s = np.cos(np.radians(deg)), np.sin(np.radians(deg))
    return np.array([[c, -s, 0, 0], [s, c, 0, 0], [0, 0, 1, 0], [0, 0, 0, 1]], np.float32)


def bindings(ks):
    B = ks.TextureBinding.make
    return [
        B(0, "basecolor", 0, filter=0, uv_scale=(3.0, 3.0)),                        # floor: checker, nearest
        B(0, "normal_map", 3, filter=1, strength=0.7),                              # floor: tangent space
        B(2, "basecolor", 1, filter=1, wrap_u=1, wrap_v=1, uv_offset=(-0.2, 0.1)),  # back wall, clamp
        B(5, "roughness", 2, filter=2, cubic_kernel=2, scale=(0.9, 1, 1, 1)),       # box: Catmull-Rom
        B(5, "basecolor", 0, filter=2, cubic_kernel=1, flip_v=0),                   # box: B-spline
        B(6, "metallic", 1, filter=1, swizzle=(1, -1, -1, -1)),                     # box: metallic from G
        B(6, "normal_map", 3, filter=0, normal_space=1, to_world=rot_z(30)),         # box: world space
    ]


def case(ks, W=48, H=48, spp=16, bounces=6):
    g = ks.Generated("box_room", 0)
    d = g.desc.contents
    tc = np.array([[0.0, 0.0], [2.0, 0.0], [2.0, 2.0], [0.0, 2.0]], np.float32)  # the back wall's 4 vertices
    d.meshes[2].texcoords = tc.ctypes.data
    for k in (5, 6):
        d.materials[k].roughness = 0.4
    keep = ks.attach_textures(g.desc, textures(), bindings(ks))
    g._tex = (tc, keep)
    cam = ks.camera_perspective(g.camera_to_world, g.vfov, g.aspect)
    p = ks.SmallPTParams.make(render_width=W, render_height=H, spp=spp, bounces=bounces, clamp_indirect=0.0)
    return g, cam, p


def test_oracle_textured_render(oracle):
    import keepsake_b200 as ks
    g, cam, p = case(ks, W=24, H=24, spp=4)
    a, w, _ = oracle.scene(g.desc).render(cam, p, threads=4)
    plain = ks.Generated("box_room", 0)
    a0, w0, _ = oracle.scene(plain.desc).render(cam, p, threads=4)
    img, img0 = composite(a, w), composite(a0, w0)
    assert np.isfinite(img).all() and (img >= 0).all()
    assert np.array_equal(w, w0)
    assert rel_mse(img, img0) > 1e-2


def test_binding_helpers():
    import keepsake_b200 as ks
    b = ks.TextureBinding.make(3, "normal_map", 1, strength=0.5)
    assert b.field == 9 and b.flip_v == 1 and list(b.swizzle) == [0, 1, 2, 3] and b.strength == 0.5
    assert ctypes.sizeof(ks.TextureBinding) == 156


@pytest.mark.gpu
def test_textured_render_matches_oracle(ctx, oracle):
    import keepsake_b200 as ks
    g, cam, p = case(ks)
    s = ks.Scene(ctx, g.desc)
    s.build_bvh()
    acc, w = s.render(cam, p)
    oacc, ow, ocnt = oracle.scene(g.desc).render(cam, p)
    assert np.array_equal(w, ow)
    img, ref = composite(acc, w), composite(oacc, ow)
    err = rel_mse(img, ref)
    assert err < 2e-3, err
    rel = np.abs(img - ref) / (np.abs(ref) + 1e-3)
    assert np.median(rel) < 1e-4
    st = s.stats()
    assert abs(st.extension_rays - int(ocnt[0])) <= 0.01 * ocnt[0] + 16
    s.close()


@pytest.mark.gpu
def test_texture_bindings_are_validated(ctx):
    import keepsake_b200 as ks
    for bad in (dict(filter=3), dict(field=11), dict(texture=9), dict(wrap_u=2), dict(swizzle=(4, 0, 0, 0))):
        g = ks.Generated("box_room", 0)
        kw = dict(bad)
        tex = kw.pop("texture", 0)
        field = kw.pop("field", "basecolor")
        keep = ks.attach_textures(g.desc, textures(), [ks.TextureBinding.make(0, field, tex, **kw)])
        h = ctypes.c_void_p()
        assert ks.lib.ks_scene_create(ctx.handle, g.desc, ctypes.byref(h)) == 1, bad
        del keep


def opacity_case(ks, W=48, H=48, spp=16):
    """The box room with an opacity map on both boxes (OpacityMap, opacity_map.cpp): an 8-bit mask of
    fully opaque, fully clear and half-transparent stripes, and a float ramp on the back wall.  The
    opacity test reads the mesh's texcoords (compute_hit_texcoord, geometry.cpp:165-173: (0, 0)
    without them), so the boxes get texcoords from their vertex positions and the back wall its
    corners'."""
    g = ks.Generated("box_room", 0)
    d = g.desc.contents
    tcs = []
    for k in (5, 6):
        v = g.meshes[k]["vertices"]
        tc = np.ascontiguousarray(np.stack([(v[:, 0] + v[:, 2]) * 1.7, v[:, 1] * 1.3], -1), np.float32)
        d.meshes[k].texcoords = tc.ctypes.data
        tcs.append(tc)
    tc = np.array([[0.0, 0.0], [1.0, 0.0], [1.0, 1.0], [0.0, 1.0]], np.float32)
    d.meshes[2].texcoords = tc.ctypes.data
    tcs.append(tc)
    ys, xs = np.mgrid[0:32, 0:32]
    stripes = np.where((xs // 4) % 3 == 0, 255, np.where((xs // 4) % 3 == 1, 0, 128)).astype(np.uint8)
    ramp = np.clip(xs / 31.0, 0.0, 1.0).astype(np.float32)
    B = ks.TextureBinding.make
    binds = [B(5, "opacity_map", 0, filter=0), B(6, "opacity_map", 0, filter=0, uv_scale=(2.0, 2.0)),
             B(2, "opacity_map", 1, filter=1)]
    keep = ks.attach_textures(g.desc, [(stripes, False), (ramp, False)], binds)
    g._tex = (keep, tcs)
    cam = ks.camera_perspective(g.camera_to_world, g.vfov, g.aspect)
    # a backdrop instead of the background: camera rays that leave the scene count as misses
    p = ks.SmallPTParams.make(render_width=W, render_height=H, spp=spp, bounces=6, clamp_indirect=0.0,
                              include_background=0, backdrop=(0.0, 0.0, 0.0))
    return g, cam, p


def test_oracle_opacity_render(oracle):
    """Opacity maps let light through: the back wall's clear part and the boxes' stripes change the
    image, and the weights stay those of the same camera samples."""
    import keepsake_b200 as ks
    g, cam, p = opacity_case(ks, W=24, H=24, spp=4)
    a, w, cnt = oracle.scene(g.desc).render(cam, p, threads=4)
    plain = ks.Generated("box_room", 0)
    a0, w0, cnt0 = oracle.scene(plain.desc).render(cam, p, threads=4)
    assert np.isfinite(a).all()
    assert rel_mse(composite(a, w), composite(a0, w0)) > 1e-2
    # rays leave through the transparent back wall: fewer hits than the closed room
    assert w[..., 1].sum() > w0[..., 1].sum()


@pytest.mark.gpu
def test_opacity_render_matches_oracle(ctx, oracle):
    """Camera rays: the opacity test hashes the ray's origin and direction, which the camera
    kernel computes bit for bit like the oracle, so every camera ray is decided the same way (equal
    hit / miss weights; at depth 0 equal images).  Later rays start from directions the fast-math
    shading unit computes to within a few ulps of the oracle's, so their hashes (and stochastic
    decisions) differ: the full-depth image is compared by convergence to a 16x spp oracle image."""
    import keepsake_b200 as ks
    g, cam, p = opacity_case(ks)
    s = ks.Scene(ctx, g.desc)
    s.build_bvh()
    osc = oracle.scene(g.desc)
    p0 = ks.SmallPTParams.make(render_width=p.render_width, render_height=p.render_height, spp=p.spp, bounces=0,
                               clamp_indirect=0.0, include_background=0, backdrop=(0.0, 0.0, 0.0))
    acc, w = s.render(cam, p0)
    oacc, ow, _ = osc.render(cam, p0)
    assert np.array_equal(w, ow), "hit / miss weights differ: the opacity test decided a camera ray differently"
    assert rel_mse(composite(acc, w), composite(oacc, ow)) < 1e-6
    acc, w = s.render(cam, p)
    oacc, ow, ocnt = osc.render(cam, p)
    assert np.array_equal(w, ow)
    st = s.stats()
    assert abs(st.extension_rays - int(ocnt[0])) <= 0.03 * ocnt[0] + 16
    spp = p.spp
    p.spp = 16 * spp
    p.rng_seed = 3  # a reference that shares no samples with the compared renders
    hi = composite(*osc.render(cam, p)[:2])
    gpu = rel_mse(composite(acc, w), hi)
    cpu = rel_mse(composite(oacc, ow), hi)
    assert gpu <= 1.25 * cpu + 1e-6, (gpu, cpu)
    s.close()


def emitter_case(ks, W=48, H=48, spp=16, uv_scale=(1.0, 1.0), wrap=0):
    """The box room's lamp with an emission texture (MeshTriLight with a TextureField emission,
    light.cpp:307-565): a float texture of bright and dim cells and a zero corner, on the lamp's
    texcoords; its two triangles' selection powers come from the texture's summed-area table."""
    g = ks.Generated("box_room", 0)
    d = g.desc.contents
    ys, xs = np.mgrid[0:16, 0:16]
    cells = ((xs // 4 + ys // 4) % 2).astype(np.float32)
    tex = np.stack([20 + 40 * cells, 15 + 25 * cells, 4 + 10 * cells * (xs / 15.0)], -1).astype(np.float32)
    tex[:4, :4] = 0.0
    tc = np.array([[0.0, 0.0], [1.0, 0.0], [1.0, 1.0], [0.0, 1.0]], np.float32)
    d.meshes[7].texcoords = tc.ctypes.data
    b = ks.TextureBinding.make(7, "emission", 0, filter=1, uv_scale=uv_scale, wrap_u=wrap, wrap_v=wrap,
                               scale=(0.8, 0.8, 0.8, 1.0))
    g._tex = (ks.attach_textures(g.desc, [(tex, False)], [b]), tc)
    cam = ks.camera_perspective(g.camera_to_world, g.vfov, g.aspect)
    p = ks.SmallPTParams.make(render_width=W, render_height=H, spp=spp, bounces=6, clamp_indirect=0.0)
    return g, cam, p


def test_oracle_textured_emitter(oracle):
    """A textured lamp changes the image and keeps its light weights (same camera samples)."""
    import keepsake_b200 as ks
    g, cam, p = emitter_case(ks, W=24, H=24, spp=4)
    a, w, _ = oracle.scene(g.desc).render(cam, p, threads=4)
    plain = ks.Generated("box_room", 0)
    a0, w0, _ = oracle.scene(plain.desc).render(cam, p, threads=4)
    assert np.isfinite(a).all() and (a >= 0).all()
    assert np.array_equal(w, w0)
    assert rel_mse(composite(a, w), composite(a0, w0)) > 1e-2


@pytest.mark.gpu
@pytest.mark.parametrize("uv_scale,wrap", [((1.0, 1.0), 0), ((2.5, 1.5), 0), ((1.7, 1.0), 1)])
def test_textured_emitter_matches_oracle(ctx, oracle, uv_scale, wrap):
    """Same samples: the light-selection powers (summed-area-table importance, built by the library's
    light build and by the oracle's restatement), the emission at light samples and at lamp hits."""
    import keepsake_b200 as ks
    g, cam, p = emitter_case(ks, uv_scale=uv_scale, wrap=wrap)
    s = ks.Scene(ctx, g.desc)
    s.build_bvh()
    acc, w = s.render(cam, p)
    oacc, ow, ocnt = oracle.scene(g.desc).render(cam, p)
    assert np.array_equal(w, ow)
    img, ref = composite(acc, w), composite(oacc, ow)
    assert rel_mse(img, ref) < 2e-3
    assert np.median(np.abs(img - ref) / (np.abs(ref) + 1e-3)) < 1e-4
    st = s.stats()
    assert abs(st.shadow_rays - int(ocnt[1])) <= 0.01 * ocnt[1] + 16
    s.close()


@pytest.mark.gpu
def test_emission_binding_needs_an_emitter(ctx):
    import ctypes
    import keepsake_b200 as ks
    g = ks.Generated("box_room", 0)
    keep = ks.attach_textures(g.desc, [(np.ones((2, 2, 3), np.float32), False)],
                              [ks.TextureBinding.make(0, "emission", 0)])  # material 0 emits nothing
    h = ctypes.c_void_p()
    assert ks.lib.ks_scene_create(ctx.handle, g.desc, ctypes.byref(h)) == 1
    del keep
