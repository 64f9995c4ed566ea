"""Failure detection: each bounded loop of the library runs out on a small input and ends in a
status code, and the context stays usable for the next call.

The reference aborts on its failures (ASSERT, cuda_check, the Embree error handler); the library
reports them instead:
  * traversal stack overflow (a tree deeper than the 64-entry stack) -> KS_ERR_QUEUE_OVERFLOW from
    ks_trace_rays, ks_trace_rays_wide, ks_trace_rays_noalloc and the render;
  * the SBVH builder's level limit -> KS_ERR_WATCHDOG, the scene stays unbuilt;
  * the wavefront iteration limit of a render and of a batch -> KS_ERR_WATCHDOG;
  * the tensor-core kernels' bounded mbarrier wait -> KS_ERR_WATCHDOG when nothing arrives.
Every failure is made on the host (a geometry, a limit, a barrier nothing arrives on); nothing
faults, traps or hangs the GPU: every push is bounds-checked and every wait has a poll limit."""
import numpy as np
import pytest

import scenes
from imaging import composite

KS_ERR_QUEUE_OVERFLOW = 4
KS_ERR_WATCHDOG = 5
KS_ERR_NOT_BUILT = 6


def chain_scene(ks):
    v, idx = scenes.deep_chain()
    m = ks.MaterialDesc()
    m.basecolor[:] = (0.5, 0.5, 0.5)
    m.roughness, m.ior, m.specular_r0_mul, m.diffuse_trans_fwd = 1.0, 1.5, 0.5, 0.5
    desc, keep = ks.scene_desc([(v, idx, 0)], [m])
    light = (ks.LightDesc * 1)()
    light[0].type = 0
    light[0].color[:] = (1.0, 1.0, 1.0)
    light[0].vec[:] = (-1.0, 0.5, 0.0)
    desc.lights = light
    desc.n_lights = 1
    return desc, keep + [light, v, idx]


def chain_rays(n=256):
    rng = np.random.default_rng(0)
    r = np.zeros((n, 8), np.float32)
    r[:, 0] = -1.0
    r[:, 1:3] = rng.uniform(-0.2, 0.2, (n, 2))
    r[:, 4] = 1.0
    r[:, 7] = np.inf
    return r


def chain_camera(ks):
    # orthographic, from x = -1 toward +x (up +y; columns right (0, 0, 1), up, back (-1, 0, 0), pos):
    # every camera ray runs parallel to the chain's axis and meets both children at every level
    c2w = np.array([[0, 0, -1, -1.0], [0, 1, 0, 0.0], [1, 0, 0, 0.0], [0, 0, 0, 1]], np.float32)
    return ks.camera_orthographic(c2w, -0.2, 0.2, -0.2, 0.2, 0.1, 10.0)


def test_deep_chain_outgrows_the_stack(oracle):
    """The reference builder makes the chain about 130 levels deep (2 buckets): more pushes along
    a ray through all triangles than the 64 stack entries (cuda/sbvh.cu:512-603 keeps 64 too)."""
    import oracle_lib
    v, idx = scenes.deep_chain()
    t = oracle_lib.ref_sbvh().build(v, idx, buckets=2)
    assert scenes.sbvh_depth(t.right) > 2 * 64


def test_limits_and_probe_need_a_context():
    import ctypes

    import keepsake_b200 as ks
    assert ks.lib.ks_context_set_limits(None, None) == 1
    assert ks.lib.ks_mbarrier_wait_probe(None, 10, 1) == 1
    lim = ks.ContextLimits(3, 7)
    assert ctypes.sizeof(lim) == 8 and lim.sbvh_max_levels == 3


@pytest.mark.gpu
def test_traversal_stack_overflow_is_reported(ctx, oracle):
    import keepsake_b200 as ks
    desc, keep = chain_scene(ks)
    s = ks.Scene(ctx, desc, keep)
    s.build_bvh(buckets=2)
    exp = s.export_sbvh()
    assert scenes.sbvh_depth(exp["right"]) > 2 * 64
    rays = chain_rays()
    for wide in (False, True):
        for any_hit in (False, True):
            with pytest.raises(ks.KsError) as e:
                s.trace(rays, any_hit=any_hit, wide=wide)
            assert e.value.status == KS_ERR_QUEUE_OVERFLOW, (wide, any_hit)
    p = ks.SmallPTParams.make(render_width=16, render_height=16, spp=1, bounces=2)
    with pytest.raises(ks.KsError) as e:
        s.render(chain_camera(ks), p)
    assert e.value.status == KS_ERR_QUEUE_OVERFLOW
    # rays that miss the chain's upper levels need no deep stack: a ray at x beyond the chain
    far = chain_rays(8)
    far[:, 0] = 3e37
    tri, _, _ = s.trace(far)
    assert (tri == 0xFFFFFFFF).all()
    s.close()
    # the context still renders
    g = ks.Generated("box_room", 0)
    cam = ks.camera_perspective(g.camera_to_world, g.vfov, g.aspect)
    p = ks.SmallPTParams.make(render_width=24, render_height=24, spp=2, bounces=4)
    s2 = ks.Scene(ctx, g.desc)
    s2.build_bvh()
    a, w = s2.render(cam, p)
    assert (w.sum(-1) == 2).all() and a.sum() > 0
    s2.close()


@pytest.mark.gpu
def test_sbvh_level_limit(ctx):
    import keepsake_b200 as ks
    g = ks.Generated("icosphere", 0, level=3, sky=(32, 16), resolution=(16, 16))
    cam = ks.camera_perspective(g.camera_to_world, g.vfov, g.aspect)
    p = ks.SmallPTParams.make(render_width=16, render_height=16, spp=2, bounces=3)
    s = ks.Scene(ctx, g.desc)
    try:
        ctx.set_limits(sbvh_max_levels=3)
        with pytest.raises(ks.KsError) as e:
            s.build_bvh()
        assert e.value.status == KS_ERR_WATCHDOG
        with pytest.raises(ks.KsError) as e:
            s.render(cam, p)
        assert e.value.status == KS_ERR_NOT_BUILT
    finally:
        ctx.set_limits()
    s.build_bvh()
    a, w = s.render(cam, p)
    assert (w.sum(-1) == 2).all() and np.isfinite(a).all()
    s.close()


@pytest.mark.gpu
def test_wavefront_iteration_limit(ctx):
    import keepsake_b200 as ks
    g = ks.Generated("box_room", 0)
    cam = ks.camera_perspective(g.camera_to_world, g.vfov, g.aspect)
    p = ks.SmallPTParams.make(render_width=32, render_height=32, spp=4, bounces=8, clamp_indirect=0.0)
    s = ks.Scene(ctx, g.desc)
    s.build_bvh()
    want = composite(*s.render(cam, p))
    try:
        ctx.set_limits(wavefront_max_iterations=2)
        with pytest.raises(ks.KsError) as e:
            s.render(cam, p)
        assert e.value.status == KS_ERR_WATCHDOG
        import torch
        acc = torch.zeros((32, 32, 3), dtype=torch.float64, device="cuda")
        wts = torch.zeros((32, 32, 2), dtype=torch.float64, device="cuda")
        for use_graph in (True, False):
            with pytest.raises(ks.KsError) as e:
                ks.batch_render(ctx, [(s, cam, p, acc.data_ptr(), wts.data_ptr())], use_graph=use_graph)
            assert e.value.status == KS_ERR_WATCHDOG, use_graph
    finally:
        ctx.set_limits()
    # the same render after the limits are lifted equals the one before
    got = composite(*s.render(cam, p))
    assert np.array_equal(got, want)
    s.close()


@pytest.mark.gpu
def test_mbarrier_wait_times_out_and_recovers(ctx):
    assert ctx.mbarrier_probe(1000, arrive=True) == 0
    assert ctx.mbarrier_probe(1000, arrive=False) == KS_ERR_WATCHDOG
    assert ctx.mbarrier_probe(1 << 16, arrive=False) == KS_ERR_WATCHDOG
    assert ctx.mbarrier_probe(1000, arrive=True) == 0
