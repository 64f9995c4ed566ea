"""Guided small_pt: the guide network as a second proposal (one-sample MIS with the BSDF),
trained online on the render's own paths.

  * unbiased: whatever the guide has learned, the guided image converges to the plain image;
  * useful: on the glossy scene whose sun is hidden behind a slab (indirect light from the
    sun-lit ground dominates), once trained the guide lowers the error of a pass: the late passes
    of a guided render have a lower relative MSE against a high-spp reference than the passes of
    the plain render on the same Sobol samples.
"""
import numpy as np
import pytest

from imaging import composite, rel_mse

SCENE = dict(level=5, sky=(256, 128), W=64, H=48, roughness=(0.02, 0.2), occluder=True, bounces=12)


def _scene(ctx):
    import keepsake_b200 as ks
    g = ks.Generated("icosphere", 0, level=SCENE["level"], sky=SCENE["sky"], resolution=(SCENE["W"], SCENE["H"]),
                     roughness=SCENE["roughness"], occluder=SCENE["occluder"])
    sc = ks.Scene(ctx, g.desc, keepalive=g)
    sc.build_bvh()
    cam = ks.camera_perspective(g.camera_to_world, g.vfov, g.aspect)
    lo, hi = g.bound
    lo, hi = lo - 0.05, hi + 0.05
    return g, sc, cam, np.concatenate([lo, hi])


def _params(spp, seed, interval=8):
    import keepsake_b200 as ks
    return ks.SmallPTParams.make(render_width=SCENE["W"], render_height=SCENE["H"], spp=spp,
                                 bounces=SCENE["bounces"], rng_seed=seed, spp_prog_interval=interval)


@pytest.fixture(scope="module")
def setup(ctx):
    g, sc, cam, bound = _scene(ctx)
    ref = composite(*sc.render(cam, _params(4096, 7, interval=256)))
    yield g, sc, cam, bound, ref
    sc.close()


def _guided(ctx, sc, cam, bound, spp, seed, **opt):
    import keepsake_b200 as ks
    guide = ks.Guide(ctx, bound, seed=seed)
    o = ks.GuideRenderOptions.make(train_passes=1 << 20, train_batch=4096, max_records=1 << 15, **opt)
    img = composite(*sc.render_guided(cam, _params(spp, seed), guide, o))
    st = sc.stats()
    guide.close()
    return img, st


@pytest.mark.gpu
def test_guided_render_is_unbiased(ctx, setup):
    g, sc, cam, bound, ref = setup
    img, st = _guided(ctx, sc, cam, bound, 1024, 3)
    assert st.guide_train_steps > 100 and st.guide_records > 0
    assert st.ms_guide_infer > 0.0
    # total flux: within 1% of the 4096-spp plain reference
    assert abs(img.mean() / ref.mean() - 1.0) < 1e-2, (img.mean(), ref.mean())
    plain = composite(*sc.render(cam, _params(1024, 3)))
    e_g, e_p = rel_mse(img, ref), rel_mse(plain, ref)
    print(f"relMSE guided {e_g:.4g} plain {e_p:.4g}")
    assert e_g < 2.0 * e_p


@pytest.mark.gpu
def test_guided_render_bsdf_only_passes_match_plain(ctx, setup):
    """With guide_from_pass beyond the last pass the guided kernels sample the BSDF only: the
    image equals the plain one (same Sobol samples, same estimator)."""
    g, sc, cam, bound, ref = setup
    img, _ = _guided(ctx, sc, cam, bound, 64, 5, guide_from_pass=1 << 20)
    plain = composite(*sc.render(cam, _params(64, 5)))
    assert rel_mse(img, plain) < 1e-10


@pytest.mark.gpu
def test_guided_render_roughness_filter(ctx, setup):
    """min_roughness above every material: the guide is evaluated for no vertex (alpha 0
    everywhere), the render samples the BSDF only and comes out as the plain one up to the
    rounding of dividing by the one-sample MIS density; min_roughness 0 evaluates the guide at
    every vertex that samples a direction, 0.3 (the default) only at the rough ground and slab."""
    g, sc, cam, bound, ref = setup
    img, st = _guided(ctx, sc, cam, bound, 64, 5, min_roughness=2.0)
    assert st.guide_rows == 0 and st.guide_records == 0
    plain = composite(*sc.render(cam, _params(64, 5)))
    assert rel_mse(img, plain) < 1e-6
    _, st_all = _guided(ctx, sc, cam, bound, 16, 6, min_roughness=0.0)
    _, st_def = _guided(ctx, sc, cam, bound, 16, 6)
    assert 0 < st_def.guide_rows < st_all.guide_rows
    # every vertex that samples a direction (bounce below the limit) on a hit, after the first pass
    assert st_all.guide_rows <= st_all.extension_rays


def _pass_images(render):
    """Per-pass images (differences of the progress callback's running totals)."""
    imgs, prev = [], [None, None]

    def cb(spp, a, w):
        da, dw = (a, w) if prev[0] is None else (a - prev[0], w - prev[1])
        prev[0], prev[1] = a, w
        imgs.append(composite(da, dw))
    render(cb)
    return imgs


@pytest.mark.gpu
def test_trained_guide_lowers_error_per_pass(ctx, setup):
    import keepsake_b200 as ks
    g, sc, cam, bound, ref = setup
    ratios = []
    for seed in (11, 12):
        guide = ks.Guide(ctx, bound, seed=seed)
        o = ks.GuideRenderOptions.make(train_passes=1 << 20, train_batch=4096, max_records=1 << 15)
        gi = _pass_images(lambda cb: sc.render_guided(cam, _params(1024, seed), guide, o, callback=cb))
        guide.close()
        pi = _pass_images(lambda cb: sc.render(cam, _params(1024, seed), callback=cb))
        late = slice(len(gi) // 2, None)
        ratios.append(np.mean([rel_mse(x, ref) for x in gi[late]]) / np.mean([rel_mse(x, ref) for x in pi[late]]))
    print("late-pass relMSE guided / plain:", ratios)
    assert np.mean(ratios) < 0.95, ratios


@pytest.mark.gpu
def test_guided_render_rejects_bad_options(ctx, setup):
    import keepsake_b200 as ks
    g, sc, cam, bound, ref = setup
    guide = ks.Guide(ctx, bound)
    with pytest.raises(ks.KsError):
        sc.render_guided(cam, _params(8, 1), guide, ks.GuideRenderOptions.make(train_passes=-1))
    with pytest.raises(ks.KsError):
        sc.render_guided(cam, _params(8, 1), guide, ks.GuideRenderOptions.make(min_roughness=-1.0))
    guide.close()
