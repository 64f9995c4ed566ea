"""ks_trace_rays_noalloc: ray queries for callers that may not allocate device memory (a host
application that owns the device-memory budget, or a frame loop that forbids cudaMalloc).  The
entry point stages rays and results in a static device array instead of allocating; its results
must equal ks_trace_rays's bit for bit, call after call, since the array keeps the previous
call's contents.  This file is collected last so that a failure here never hides another test."""
import ctypes

import numpy as np
import pytest

import scenes

KS_ERR_QUEUE_OVERFLOW = 4


def _noalloc(ks, scene, rays, any_hit=0, culling=2):
    lib = ks.lib
    lib.ks_trace_rays_noalloc.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint32, ctypes.c_int,
                                          ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    lib.ks_trace_rays_noalloc.restype = ctypes.c_int
    rays = np.ascontiguousarray(rays, dtype=np.float32).reshape(-1, 8)
    n = len(rays)
    tri = np.full(n, 0xDEADBEEF, np.uint32)
    t = np.full(n, np.nan, np.float32)
    bary = np.full((n, 3), np.nan, np.float32)
    st = lib.ks_trace_rays_noalloc(scene.handle, ks.ptr(rays), n, any_hit, culling, ks.ptr(tri), ks.ptr(t),
                                   ks.ptr(bary))
    return st, tri, t, bary


@pytest.mark.gpu
def test_noalloc_matches_trace_rays_twice(ctx):
    import keepsake_b200 as ks
    g = ks.Generated("icosphere", 0, level=5, sky=(64, 32), resolution=(64, 64))
    s = ks.Scene(ctx, g.desc)
    s.build_bvh()
    v, i = g.flat_geometry()
    batches = [scenes.rays_at_triangles(v, i, 50000, seed=21), scenes.random_rays(v, 30000, seed=22, inside=False)]
    for rays in batches:  # two calls in a row: the second must not see the first call's data
        st, tri, t, bary = _noalloc(ks, s, rays)
        assert st == 0, ks.lib.ks_last_error(ctx.handle)
        rtri, rt, rbary = s.trace(rays)
        assert np.array_equal(tri, rtri)
        hit = rtri != 0xFFFFFFFF
        assert hit.any()
        assert np.array_equal(t[hit].view(np.uint32), rt[hit].view(np.uint32))
        assert np.array_equal(bary[hit].view(np.uint32), rbary[hit].view(np.uint32))
        st, occ, _, _ = _noalloc(ks, s, rays, any_hit=1)
        assert st == 0
        rocc, _, _ = s.trace(rays, any_hit=True)
        assert np.array_equal(occ.astype(bool), rocc)


@pytest.mark.gpu
def test_noalloc_rejects_oversized_batch(ctx):
    import keepsake_b200 as ks
    g = ks.Generated("box_room", 0)
    s = ks.Scene(ctx, g.desc)
    s.build_bvh()
    rays = np.zeros((65537, 8), np.float32)
    rays[:, 6] = 1.0
    rays[:, 7] = np.inf
    st, _, _, _ = _noalloc(ks, s, rays)
    assert st == 1  # KS_ERR_INVALID_ARGUMENT
    assert b"65536" in ks.lib.ks_last_error(ctx.handle)


@pytest.mark.gpu
def test_noalloc_matches_reference_sbvh_and_culling(ctx):
    """Against the reference's own SBVH queries (cuda/sbvh.cu:512-603, compiled from the reference
    tree): identical hit ids, distances and barycentrics except proven ties, for every culling mode;
    an empty batch is a no-op."""
    import keepsake_b200 as ks
    import oracle_lib
    from test_sbvh import check_ties
    v, i = scenes.soup(3000, seed=31)
    desc, keep = ks.triangle_soup_desc(v, i)
    s = ks.Scene(ctx, desc, keep)
    s.build_bvh()
    ref = oracle_lib.ref_sbvh().build(v, i)
    rays = scenes.rays_at_triangles(v, i, 20000, seed=32)
    for culling in (0, 1, 2):
        st, tri, t, bary = _noalloc(ks, s, rays, culling=culling)
        assert st == 0
        rtri, rt, rbary = ref.intersect(rays, culling=culling)
        hit = rtri != 0xFFFFFFFF
        assert np.array_equal(tri != 0xFFFFFFFF, hit)
        tie = tri != rtri
        assert tie.mean() <= 1e-3
        same = hit & ~tie
        assert np.array_equal(t[same].view(np.uint32), rt[same].view(np.uint32))
        assert np.array_equal(bary[same].view(np.uint32), rbary[same].view(np.uint32))
        if tie.any():
            check_ties(ref, rays[tie], tri[tie], t[tie], rtri[tie], rt[tie], np.nonzero(tie)[0])
        st, occ, _, _ = _noalloc(ks, s, rays, any_hit=1, culling=culling)
        assert st == 0
        rocc, _, _ = ref.intersect(rays, any_hit=True, culling=culling)
        assert np.array_equal(occ.astype(bool), rocc)
    st, tri, _, _ = _noalloc(ks, s, rays[:0])
    assert st == 0 and len(tri) == 0
    s.close()


@pytest.mark.gpu
def test_noalloc_overflow_then_next_call_succeeds(ctx):
    """A tree deeper than the traversal stack makes a call fail with KS_ERR_QUEUE_OVERFLOW (the
    overflow flag lives in the shared array); the next call on an ordinary scene clears the flag
    and returns ks_trace_rays's results."""
    import keepsake_b200 as ks
    from test_failures import chain_rays, chain_scene
    desc, keep = chain_scene(ks)
    deep = ks.Scene(ctx, desc, keep)
    deep.build_bvh(buckets=2)
    st, _, _, _ = _noalloc(ks, deep, chain_rays())
    assert st == KS_ERR_QUEUE_OVERFLOW
    deep.close()
    g = ks.Generated("box_room", 0)
    s = ks.Scene(ctx, g.desc)
    s.build_bvh()
    v, i = g.flat_geometry()
    rays = scenes.random_rays(v, 4000, seed=33)
    st, tri, t, _ = _noalloc(ks, s, rays)
    assert st == 0, ks.lib.ks_last_error(ctx.handle)
    rtri, rt, _ = s.trace(rays)
    assert np.array_equal(tri, rtri)
    hit = rtri != 0xFFFFFFFF
    assert np.array_equal(t[hit].view(np.uint32), rt[hit].view(np.uint32))
    s.close()
