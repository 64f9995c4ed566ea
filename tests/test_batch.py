"""Batched rendering: many (scene, camera, parameters) jobs in one wavefront (one CUDA graph
launch); every job's image equals its own single render (same Sobol samples and estimator; only
the order of the FP64 accumulation differs)."""
import numpy as np
import pytest


def _jobs(ctx):
    import torch
    import keepsake_b200 as ks
    specs = [
        (ks.Generated("box_room", 0), 64, 48, 16, 8, 0),
        (ks.Generated("icosphere", 1, level=4, sky=(256, 128), resolution=(96, 64)), 96, 64, 8, 12, 3),
        (ks.Generated("icosphere", 2, frequency=9, sky=(128, 64), resolution=(40, 30), roughness=(0.02, 0.2),
                      occluder=True), 40, 30, 32, 6, 7),
        (ks.Generated("box_room", 0), 33, 17, 4, 3, 11),
    ]
    jobs, keep = [], []
    for g, W, H, spp, bounces, seed in specs:
        s = ks.Scene(ctx, g.desc, keepalive=g)
        s.build_bvh()
        cam = ks.camera_perspective(g.camera_to_world, g.vfov, g.aspect)
        p = ks.SmallPTParams.make(render_width=W, render_height=H, spp=spp, bounces=bounces, rng_seed=seed)
        acc = torch.zeros((H, W, 3), dtype=torch.float64, device="cuda")
        wts = torch.zeros((H, W, 2), dtype=torch.float64, device="cuda")
        jobs.append((s, cam, p, acc, wts))
        keep.append(g)
    return jobs, keep


def _single(job):
    import torch
    s, cam, p, _, _ = job
    acc = torch.zeros((p.render_height, p.render_width, 3), dtype=torch.float64, device="cuda")
    wts = torch.zeros((p.render_height, p.render_width, 2), dtype=torch.float64, device="cuda")
    s.render_device(cam, p, acc.data_ptr(), wts.data_ptr())
    return acc.cpu().numpy(), wts.cpu().numpy()


@pytest.mark.gpu
@pytest.mark.parametrize("use_graph,capacity", [(True, 0), (False, 0), (True, 1000)])
def test_batch_equals_single_renders(ctx, use_graph, capacity):
    import torch
    import keepsake_b200 as ks
    jobs, keep = _jobs(ctx)
    st = ks.batch_render(ctx, [(s, c, p, a.data_ptr(), w.data_ptr()) for s, c, p, a, w in jobs],
                         capacity=capacity, use_graph=use_graph)
    torch.cuda.synchronize()
    assert st.paths == sum(p.render_width * p.render_height * p.spp for _, _, p, _, _ in jobs)
    assert st.graph_launches == (1 if use_graph else 0)
    assert st.extension_rays >= st.paths and st.iterations > 0
    for job in jobs:
        ref_a, ref_w = _single(job)
        a, w = job[3].cpu().numpy(), job[4].cpu().numpy()
        assert np.array_equal(w, ref_w)
        np.testing.assert_allclose(a, ref_a, rtol=1e-12, atol=1e-12)
    for s, *_ in jobs:
        s.close()


@pytest.mark.gpu
def test_batch_autotune_and_errors(ctx):
    import keepsake_b200 as ks
    jobs, keep = _jobs(ctx)
    desc = [(s, c, p, a.data_ptr(), w.data_ptr()) for s, c, p, a, w in jobs]
    o, ms = ks.batch_autotune(ctx, desc)
    assert o.capacity in (1 << 21, 1 << 22, 1 << 23, 1 << 24, 1 << 25) and o.grid_per_sm in (4, 8, 16, 32) and ms > 0
    st = ks.batch_render(ctx, desc, capacity=o.capacity, grid_per_sm=o.grid_per_sm)
    assert st.paths > 0
    big = ks.SmallPTParams.make(render_width=2048, render_height=1025, spp=1, bounces=1)
    with pytest.raises(ks.KsError) as e:
        ks.batch_render(ctx, [(jobs[0][0], jobs[0][1], big, desc[0][3], desc[0][4])])
    assert e.value.status == 1
    with pytest.raises(ks.KsError):
        ks.batch_render(ctx, [])
    for s, *_ in jobs:
        s.close()
