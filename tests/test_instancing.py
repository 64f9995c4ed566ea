"""Instancing (two-level BVH): an instanced scene renders like the same scene flattened to world
space (every instance's triangles transformed), which the flat path and the oracle render."""
import numpy as np
import pytest

from imaging import composite, rel_mse

OPTS = dict(sky=(256, 128), resolution=(96, 54), prototypes=4, instances=24, frequency=6, emitters=8)


def _generated():
    import keepsake_b200 as ks
    return ks.Generated("instanced", 5, **OPTS)


def _params(spp, seed=1, bounces=8):
    import keepsake_b200 as ks
    return ks.SmallPTParams.make(render_width=96, render_height=54, spp=spp, bounces=bounces, rng_seed=seed,
                                 clamp_indirect=0.0)


def test_generator_counts():
    g = _generated()
    assert len(g.prototypes) == 4 + 2 and len(g.instances) == 24 + 2
    assert g.n_triangles == 4 * 20 * 36 + 8 + 2
    flat = g.flattened()
    assert sum(len(t) for _, t, _ in flat) == 24 * 720 + 8 + 2
    # affine transforms are non-singular
    for _, xf in g.instances:
        assert abs(np.linalg.det(xf[:, :3].astype(np.float64))) > 1e-6


@pytest.fixture(scope="module")
def scenes(ctx):
    import keepsake_b200 as ks
    g = _generated()
    inst = ks.Scene(ctx, g.desc, keepalive=g)
    inst.build_bvh()
    d, keep = ks.scene_desc(g.flattened(), g.materials, g.desc.contents.sky)
    flat = ks.Scene(ctx, d, keepalive=(keep, g))
    flat.build_bvh()
    cam = ks.camera_perspective(g.camera_to_world, g.vfov, g.aspect)
    yield g, inst, flat, cam, d, keep
    inst.close()
    flat.close()


@pytest.mark.gpu
def test_instanced_trace_matches_flattened(scenes):
    g, inst, flat, cam, _, _ = scenes
    rng = np.random.default_rng(3)
    n = 20000
    lo, hi = g.bound
    o = lo + (hi - lo) * rng.random((n, 3))
    o[:, 1] = np.abs(o[:, 1]) + 0.5
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    rays = np.zeros((n, 8), np.float32)
    rays[:, :3] = o
    rays[:, 4:7] = d
    rays[:, 7] = np.inf
    ti, t_i, _ = inst.trace(rays)
    tf, t_f, _ = flat.trace(rays)
    hit_i, hit_f = ti != 0xFFFFFFFF, tf != 0xFFFFFFFF
    assert hit_i.mean() > 0.3
    # hit / miss agree except for grazing rays at silhouettes (object- vs world-space rounding)
    assert np.mean(hit_i != hit_f) < 1e-3
    both = hit_i & hit_f
    rel = np.abs(t_i[both] - t_f[both]) / np.maximum(t_f[both], 1e-6)
    assert np.mean(rel < 1e-4) > 0.999
    occ_i, _, _ = inst.trace(rays, any_hit=True)
    assert np.mean(occ_i != hit_f) < 1e-3


@pytest.mark.gpu
def test_instanced_render_matches_flattened(scenes):
    g, inst, flat, cam, _, _ = scenes
    a = composite(*inst.render(cam, _params(64)))
    b = composite(*flat.render(cam, _params(64)))
    assert a.mean() > 0.0
    # same estimator on the same samples; a few paths part at silhouettes
    assert rel_mse(a, b) < 2e-3, rel_mse(a, b)
    st = inst.stats()
    assert st.paths == 96 * 54 * 64


@pytest.mark.gpu
def test_instanced_render_converges_like_oracle(scenes, oracle):
    g, inst, flat, cam, d, keep = scenes
    sc = oracle.scene(d, keepalive=keep)
    ref = composite(*sc.render(cam, _params(512, seed=9), threads=None)[:2])
    orc = composite(*sc.render(cam, _params(32, seed=2), threads=None)[:2])
    gpu = composite(*inst.render(cam, _params(32, seed=2)))
    e_o, e_g = rel_mse(orc, ref), rel_mse(gpu, ref)
    assert e_g <= 1.25 * e_o, (e_g, e_o)


@pytest.mark.gpu
def test_instanced_guided_render_runs(scenes, ctx):
    import keepsake_b200 as ks
    g, inst, flat, cam, _, _ = scenes
    lo, hi = g.bound
    guide = ks.Guide(ctx, list(lo - 0.05) + list(hi + 0.05), seed=2)
    o = ks.GuideRenderOptions.make(train_passes=1 << 20, train_batch=4096, max_records=1 << 14)
    a = composite(*inst.render_guided(cam, _params(64, seed=4), guide, o))
    b = composite(*inst.render(cam, _params(256, seed=5)))
    guide.close()
    assert abs(a.mean() / b.mean() - 1.0) < 0.03


@pytest.mark.gpu
def test_instance_validation(ctx):
    import keepsake_b200 as ks
    g = _generated()
    d = g.desc.contents
    saved = d.instances[0].prototype
    d.instances[0].prototype = 99
    with pytest.raises(ks.KsError) as e:
        ks.Scene(ctx, g.desc)
    assert e.value.status == 1
    d.instances[0].prototype = saved
    xf = list(d.instances[0].to_world)
    for k in range(12):
        d.instances[0].to_world[k] = 0.0
    with pytest.raises(ks.KsError):
        ks.Scene(ctx, g.desc)
    for k in range(12):
        d.instances[0].to_world[k] = xf[k]
    s = ks.Scene(ctx, g.desc)
    s.build_bvh()
    with pytest.raises(ks.KsError) as e:
        s.export_sbvh()
    assert e.value.status == 7
    s.close()
