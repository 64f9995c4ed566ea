"""The equal-area sky light (EqualAreaSkyLight, light.cpp:161-206): a square map in the equal-area
octahedral parameterisation, sampled through an alias table over its texels' luminance.  The
reference's CPU path leaves its sample / pdf / eval unimplemented (light.h:63-79 assert) and
defines them in its GPU path (gpu/shaders/light.slang:92-186), which the oracle restates.

CPU: the oracle's sampler reports the density its pdf() gives back for the sampled direction
(except where Clarberg's approximate inverse mapping puts the direction into a neighbouring
texel), and its mean weight equals the radiance integrated over the sphere.  GPU: renders under an
equal-area sky equal the oracle's on the same samples (the tolerances of tests/test_render.py), and
converge like them."""
import ctypes

import numpy as np
import pytest

from imaging import composite, rel_mse


def ea_square_to_sphere(px, py):
    """equal_area_square_to_sphere (gpu/shaders/common.slang:245-265) in float64."""
    u, v = 2 * px - 1, 2 * py - 1
    up, vp = np.abs(u), np.abs(v)
    sd = 1 - (up + vp)
    r = 1 - np.abs(sd)
    phi = np.where(r == 0, 1.0, (vp - up) / np.where(r == 0, 1.0, r) + 1) * np.pi / 4
    z = np.copysign(1 - r * r, sd)
    s = r * np.sqrt(np.maximum(2 - r * r, 0.0))
    return np.stack([np.copysign(np.cos(phi), u) * s, np.copysign(np.sin(phi), v) * s, z], -1)


def radiance(d):
    """A sky: a vertical gradient and a bright lobe around a sun direction."""
    sun = np.array([0.4, 0.3, 0.866])
    sun /= np.linalg.norm(sun)
    lobe = np.exp(200.0 * (d @ sun - 1.0))[..., None] * np.array([400.0, 350.0, 300.0])
    grad = (0.3 + 0.7 * np.clip(d[..., 2:3], 0, 1)) * np.array([0.3, 0.5, 0.9])
    return (grad + lobe).astype(np.float32)


def equal_area_map(res=128):
    ys, xs = np.mgrid[0:res, 0:res]
    d = ea_square_to_sphere((xs + 0.5) / res, (ys + 0.5) / res)
    return np.ascontiguousarray(radiance(d))


def sky_desc(ks, m, to_world=None, strength=1.5):
    sd = ks.SkyDesc()
    sd.kind = 3
    sd.map_rgb = m.ctypes.data
    sd.width = sd.height = m.shape[0]
    t = np.eye(4, dtype=np.float32) if to_world is None else np.asarray(to_world, np.float32)
    sd.to_world[:] = [float(x) for x in t.reshape(16)]
    sd.transform_y_up = 0
    sd.strength = strength
    return sd


def rot_x(deg):
    a = np.radians(deg)
    m = np.eye(4, dtype=np.float32)
    m[1, 1], m[1, 2], m[2, 1], m[2, 2] = np.cos(a), -np.sin(a), np.sin(a), np.cos(a)
    return m


def case(ks, level=4, W=48, H=48, spp=8, bounces=8, to_world=None):
    g = ks.Generated("icosphere", 0, level=level, sky=(64, 32), resolution=(W, H))
    m = equal_area_map()
    d = g.desc.contents
    d.sky = sky_desc(ks, m, to_world)
    g._ea_map = m  # keeps the map alive with the description
    cam = ks.camera_perspective(g.camera_to_world, g.vfov, g.aspect)
    return g, cam, ks.SmallPTParams.make(render_width=W, render_height=H, spp=spp, bounces=bounces)


def test_oracle_equal_area_sampling(oracle):
    import keepsake_b200 as ks
    g, cam, p = case(ks, to_world=rot_x(30))
    sc = oracle.scene(g.desc)
    n = 200_000
    u = np.random.default_rng(0).random((n, 2), dtype=np.float32)
    wi, pdf, lb = sc.sky_sample(u)
    assert (pdf > 0).all() and np.isfinite(lb).all()
    assert np.allclose(np.linalg.norm(wi, axis=1), 1.0, atol=1e-5)
    p2, le = sc.sky_eval(wi)
    same = np.isclose(p2, pdf, rtol=1e-5)
    assert same.mean() > 0.99, same.mean()
    # weight = Le / pdf: the sampler evaluates the map at the exact square point, eval() at the
    # approximate inverse of its direction, a few 1e-6 of the square away
    close = np.isclose(lb[same] * pdf[same, None], le[same], rtol=2e-3, atol=1e-5).all(1)
    assert close.mean() > 0.999, close.mean()
    # E[Le / pdf] = integral of Le over the sphere (uniform-sphere estimate of the same eval)
    d = np.random.default_rng(1).normal(size=(n, 3))
    d = (d / np.linalg.norm(d, axis=1, keepdims=True)).astype(np.float32)
    _, le_u = sc.sky_eval(d)
    est_u = le_u.mean(0) * 4 * np.pi
    se = le_u.std(0) * 4 * np.pi / np.sqrt(n) + lb.std(0) / np.sqrt(n)
    assert (np.abs(lb.mean(0) - est_u) <= 5 * se).all(), (lb.mean(0), est_u)
    # the light-to-world rotation turns the sun lobe: the brightest sample direction follows it
    sun = np.array([0.4, 0.3, 0.866]) / np.linalg.norm([0.4, 0.3, 0.866])
    k = np.argmax(lb.sum(1) * pdf)
    assert np.dot(wi[k], rot_x(30)[:3, :3] @ sun) > 0.98


def test_oracle_equal_area_sky_renders(oracle):
    import keepsake_b200 as ks
    g, cam, p = case(ks, W=24, H=24, spp=4)
    a, w, cnt = oracle.scene(g.desc).render(cam, p, threads=4)
    assert np.isfinite(a).all() and (a >= 0).all() and a.sum() > 0
    assert cnt[1] > 0


@pytest.mark.gpu
def test_equal_area_sky_rejects_bad_maps(ctx):
    """A map that is not a square of a power-of-two side is an invalid argument."""
    import keepsake_b200 as ks
    for shape in ((16, 32), (24, 24)):
        g = ks.Generated("box_room", 0)
        m = np.ones(shape + (3,), np.float32)
        sd = sky_desc(ks, m)
        sd.height, sd.width = shape
        g.desc.contents.sky = sd
        h = ctypes.c_void_p()
        assert ks.lib.ks_scene_create(ctx.handle, g.desc, ctypes.byref(h)) == 1, shape


@pytest.mark.gpu
def test_equal_area_sky_matches_oracle(ctx, oracle):
    import keepsake_b200 as ks
    g, cam, p = case(ks, to_world=rot_x(30))
    s = ks.Scene(ctx, g.desc)
    s.build_bvh()
    acc, w = s.render(cam, p)
    oacc, ow, ocnt = oracle.scene(g.desc).render(cam, p)
    assert np.array_equal(w, ow)
    img, ref = composite(acc, w), composite(oacc, ow)
    assert rel_mse(img, ref) < 2e-3
    rel = np.abs(img - ref) / (np.abs(ref) + 1e-3)
    assert np.median(rel) < 1e-4
    st = s.stats()
    assert abs(st.shadow_rays - int(ocnt[1])) <= 0.01 * ocnt[1] + 16
    # convergence against a 16x spp oracle image
    p16 = ks.SmallPTParams.make(render_width=p.render_width, render_height=p.render_height, spp=16 * p.spp,
                                bounces=p.bounces, rng_seed=3)  # shares no samples with the compared renders
    osc = oracle.scene(g.desc)
    hi = composite(*osc.render(cam, p16)[:2])
    assert rel_mse(img, hi) <= 1.25 * rel_mse(ref, hi) + 1e-6
    s.close()


def quat_matrix(q):
    """Rotation matrix (4x4, float32) of the quaternion (x, y, z, w), as the task builds it: the
    components read as float32, normalised and expanded in float64."""
    q = np.asarray(q, np.float32).astype(np.float64)
    n2 = q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3]
    x, y, z, w = (c / np.sqrt(n2) for c in q)
    r = np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
                  [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
                  [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)]])
    m = np.eye(4, dtype=np.float32)
    m[:3, :3] = r
    return m


@pytest.mark.gpu
def test_task_equal_area_sky_equals_c_abi(ctx, tmp_path):
    """The small_pt task's `light = [{ type = "equal_area_sky", ... }]` (create_equal_area_sky_light,
    light.cpp:274-283) renders what the C ABI renders with the same map, rotation and strength."""
    import keepsake_b200 as ks
    m = equal_area_map(64)
    ks.save_exr(tmp_path / "sky_ea.exr", m)
    q = [0.2, -0.1, 0.3, 0.9]
    g = ks.Generated("box_room", 0)
    c2w = [float(x) for x in g.camera_to_world]
    deg = float(np.float32(np.degrees(g.vfov)))
    doc = f"""
[mesh_asset.room]
type = "procedural"
kind = "box_room"
seed = 0

[[task]]
type = "small_pt"
object = "mesh_asset.room"
light = [{{ type = "equal_area_sky", map = "sky_ea.exr", to_world = {q}, strength = 0.7 }}]
bounces = 6
clamp_indirect = 0.0
render_width = 40
render_height = 32
spp = 8
spp_prog_interval = 8
camera = {{ type = "perspective", to_world = {{ matrix_rm = {c2w} }}, vfov = {deg!r}, aspect = 1.25 }}
"""
    ks.config_run(doc, str(tmp_path / "out"), str(tmp_path))
    img = ks.load_image(tmp_path / "out" / "task_0" / "small_pt_spp8.exr")
    back = ks.load_image(tmp_path / "sky_ea.exr")
    d = g.desc.contents
    d.sky = sky_desc(ks, np.ascontiguousarray(back), quat_matrix(q), strength=0.7)
    g._ea = back
    vfov = np.float32(deg) / np.float32(180.0) * np.float32(np.pi)
    cam = ks.camera_perspective(np.array(c2w, np.float32), float(vfov), 1.25)
    s = ks.Scene(ctx, g.desc)
    s.build_bvh()
    p = ks.SmallPTParams.make(render_width=40, render_height=32, spp=8, bounces=6, clamp_indirect=0.0,
                              spp_prog_interval=8)
    ref = composite(*s.render(cam, p)).astype(np.float32)
    s.close()
    assert ref.mean() > 0.0
    assert np.array_equal(img, ref)
