"""SBVH parity: the GPU builder's tree against the reference builder (cuda/sbvh.cu, compiled
host-side in oracle/_ref), and GPU ray queries against SBVH::intersect / intersectBool.

Topology = node count, DFS node order, node bounds, split axes, rightChildOffset, primOffset,
and the multiset of primitives in every leaf (their order inside a leaf comes from
std::partition's swap order in the reference and is not part of the contract)."""
import numpy as np
import pytest

import scenes


def leaf_multisets(right, prim_offset, prims):
    n = len(right)
    ends = np.append(prim_offset[1:], len(prims))
    out = {}
    for i in np.nonzero(right == 0)[0]:
        out[int(i)] = np.sort(prims[prim_offset[i]:ends[i]])
    return out


def assert_same_tree(got, ref):
    assert len(got["axis"]) == len(ref.axis), "node count differs"
    assert len(got["prims"]) == len(ref.prims), "primitive reference count differs"
    assert np.array_equal(got["right"], ref.right), "rightChildOffset differs"
    assert np.array_equal(got["prim_offset"], ref.prim_offset), "primOffset differs"
    interior = ref.right != 0
    assert np.array_equal(got["axis"][interior], ref.axis[interior]), "split axis differs"
    # float compare (== treats -0 and +0 alike)
    assert np.array_equal(got["bounds"], ref.bounds), "node bounds differ"
    a = leaf_multisets(ref.right, ref.prim_offset, ref.prims)
    b = leaf_multisets(got["right"], got["prim_offset"], got["prims"])
    for k in a:
        assert np.array_equal(a[k], b[k]), f"leaf {k} primitives differ"


def test_reference_builder_runs_on_cpu():
    import oracle_lib
    v, i = scenes.soup(500, seed=3)
    tree = oracle_lib.ref_sbvh().build(v, i)
    assert len(tree.prims) >= 500 and tree.right[0] != 0


def _check_build(ctx, v, i, **opts):
    import keepsake_b200 as ks
    import oracle_lib
    d, keep = ks.triangle_soup_desc(v, i)
    s = ks.Scene(ctx, d, keep)
    s.build_bvh(**opts)
    got = s.export_sbvh()
    ref = oracle_lib.ref_sbvh().build(v, i, **{
        "max_prims": opts.get("max_prims", 4), "buckets": opts.get("buckets", 12),
        "trav_weight": opts.get("trav_weight", 1.0), "alpha": opts.get("alpha", 1e-5)})
    assert_same_tree(got, ref)
    return s, ref


@pytest.mark.gpu
@pytest.mark.parametrize("n,seed", [(1, 0), (2, 1), (7, 2), (100, 3), (2000, 4), (30000, 5)])
def test_builder_topology_soup(ctx, n, seed):
    v, i = scenes.soup(n, seed=seed)
    _check_build(ctx, v, i)


@pytest.mark.gpu
def test_builder_topology_degenerate(ctx):
    v, i = scenes.degenerate_soup(0)
    _check_build(ctx, v, i)


@pytest.mark.gpu
@pytest.mark.parametrize("opts", [dict(max_prims=1), dict(max_prims=8, buckets=16), dict(buckets=2),
                                  dict(alpha=0.0), dict(alpha=1.0), dict(trav_weight=0.0), dict(trav_weight=10.0)])
def test_builder_topology_options(ctx, opts):
    v, i = scenes.soup(3000, seed=11, spread=4.0, size=1.5)  # overlapping: spatial splits happen
    _check_build(ctx, v, i, **opts)


@pytest.mark.gpu
def test_builder_topology_box_room(ctx):
    import keepsake_b200 as ks
    g = ks.Generated("box_room", 0)
    v, i = g.flat_geometry()
    _check_build(ctx, v, i)


@pytest.mark.gpu
@pytest.mark.parametrize("level", [4, 6, 8])
def test_builder_topology_icosphere(ctx, level):
    import keepsake_b200 as ks
    g = ks.Generated("icosphere", 0, level=level)
    v, i = g.flat_geometry()
    _check_build(ctx, v, i)


# A differing hit id is a tie when the reference's own watertight test of the triangle the GPU
# reported hits the ray at a distance within MAX_TIE_ULP of the reference's closest hit: the
# reference then holds two candidates that close, and the strict "t < tmax" acceptance of its leaf
# loop (cuda/sbvh.cu:531), with the scaled comparison of T against tmax * det in the triangle test
# (cuda/ray_tri.cuh:83-87), leaves the pick to the visiting order.
MAX_TIE_ULP = 8


def check_ties(ref, rays, tri, t, rtri, rt, index):
    """Proves every differing hit id a tie (see MAX_TIE_ULP) and prints the list of those rays:
    ray index, reference triangle and distance, GPU triangle, its distance under the reference's
    test, and the gap in ulp."""
    rays = np.array(rays, np.float32)
    rays[:, 7] = np.inf
    ghit, gt = ref.tri_test(rays, tri)
    assert ghit.all(), "a differing hit id is not a candidate of the reference's own triangle test"
    assert np.array_equal(gt.view(np.uint32), t.view(np.uint32)), "the GPU distance differs from the reference test"
    ulps = np.abs(gt.view(np.int32).astype(np.int64) - rt.view(np.int32).astype(np.int64))
    print(f"\n{len(index)} tie rays (index, ref tri, ref t, gpu tri, gpu t, ulp); ulp histogram "
          f"{np.bincount(ulps.clip(0, 9)).tolist()}")
    for k in range(len(index)):
        print(f"  {index[k]} {rtri[k]} {rt[k]!r} {tri[k]} {gt[k]!r} {ulps[k]}")
    assert ulps.max() <= MAX_TIE_ULP, f"tie distances differ by {ulps.max()} ulp"


def _check_trace(scene, ref, rays, max_tie_frac=0.0, wide=False):
    """Hit ids, distances and barycentrics must match bit for bit.  The one documented exception
    is a near tie: triangles hit at the same or a few-ulp-apart t (duplicate or coplanar
    overlapping triangles, a shared edge or vertex).  The order of the triangles inside a leaf
    follows the reference's std::partition swap order, which the parallel builder does not
    reproduce (leaf contents are identical as multisets); with a near tie that order decides
    which triangle is accepted first, and because the triangle test compares T against
    tmax * det in scaled form, it can also decide whether a triangle of a later leaf passes.
    For such rays the distances must agree within 8 ulp.  wide: the renderer's 4-wide traversal
    (ks_trace_rays_wide), whose visiting order differs from the reference's, so exact ties may
    resolve to the other triangle as well."""
    tri, t, bary = scene.trace(rays, wide=wide)
    rtri, rt, rbary = ref.intersect(rays)
    hit = rtri != 0xFFFFFFFF
    assert np.array_equal(tri != 0xFFFFFFFF, hit), "hit/miss differs"
    tie = tri != rtri
    assert tie.mean() <= max_tie_frac, f"{tie.sum()} of {len(rays)} hit ids differ (ties allowed: {max_tie_frac})"
    same = hit & ~tie
    assert np.array_equal(t[same].view(np.uint32), rt[same].view(np.uint32)), "hit distances differ"
    assert np.array_equal(bary[same].view(np.uint32), rbary[same].view(np.uint32)), "barycentrics differ"
    if tie.any():
        check_ties(ref, rays[tie], tri[tie], t[tie], rtri[tie], rt[tie], np.nonzero(tie)[0])
    occ, _, _ = scene.trace(rays, any_hit=True, wide=wide)
    rocc, _, _ = ref.intersect(rays, any_hit=True)
    assert np.array_equal(occ, rocc), "occlusion results differ"
    return hit.mean()


@pytest.mark.gpu
def test_trace_soup_bit_exact(ctx):
    v, i = scenes.soup(5000, seed=7)
    s, ref = _check_build(ctx, v, i)
    _check_trace(s, ref, scenes.random_rays(v, 20000, seed=1))
    _check_trace(s, ref, scenes.random_rays(v, 20000, seed=2, inside=False))
    _check_trace(s, ref, scenes.rays_at_triangles(v, i, 20000, seed=3))
    short = scenes.random_rays(v, 20000, seed=4, tmax=0.7)
    _check_trace(s, ref, short)


@pytest.mark.gpu
def test_trace_degenerate_bit_exact(ctx):
    v, i = scenes.degenerate_soup(1)
    s, ref = _check_build(ctx, v, i)
    # 12 identical triangles: every ray that hits them is an exact tie
    _check_trace(s, ref, scenes.rays_at_triangles(v, i, 20000, seed=5), max_tie_frac=0.1)
    _check_trace(s, ref, scenes.random_rays(v, 20000, seed=6), max_tie_frac=0.1)


@pytest.mark.gpu
@pytest.mark.parametrize("culling", [0, 1])
def test_trace_culling(ctx, culling):
    import oracle_lib
    v, i = scenes.soup(2000, seed=9)
    s, ref = _check_build(ctx, v, i)
    rays = scenes.rays_at_triangles(v, i, 10000, seed=6)
    tri, _, _ = s.trace(rays, culling=culling)
    rtri, _, _ = ref.intersect(rays, culling=culling)
    assert np.array_equal(tri, rtri)


@pytest.mark.gpu
def test_trace_icosphere_bit_exact(ctx):
    import keepsake_b200 as ks
    g = ks.Generated("icosphere", 0, level=8)
    v, i = g.flat_geometry()
    s, ref = _check_build(ctx, v, i)
    # 10% of these rays aim exactly at a vertex or an edge midpoint shared by several triangles
    frac = _check_trace(s, ref, scenes.rays_at_triangles(v, i, 200000, seed=8), max_tie_frac=0.02)
    assert frac > 0.5
    _check_trace(s, ref, scenes.random_rays(v, 200000, seed=9, inside=False), max_tie_frac=1e-4)


@pytest.mark.gpu
def test_trace_wide_matches_reference(ctx):
    """The renderer's 4-wide traversal against the reference SBVH queries: same hits and occlusion,
    identical ids, distances and barycentrics except at exact ties."""
    v, i = scenes.soup(5000, seed=7)
    s, ref = _check_build(ctx, v, i)
    _check_trace(s, ref, scenes.random_rays(v, 20000, seed=1), wide=True)
    _check_trace(s, ref, scenes.random_rays(v, 20000, seed=2, inside=False), wide=True)
    _check_trace(s, ref, scenes.rays_at_triangles(v, i, 20000, seed=3), max_tie_frac=1e-3, wide=True)
    _check_trace(s, ref, scenes.random_rays(v, 20000, seed=4, tmax=0.7), wide=True)
    # 12 identical triangles: every ray that hits them is an exact tie, which either traversal
    # order may resolve to any of the 12 (distances still within 8 ulp)
    v, i = scenes.degenerate_soup(1)
    s, ref = _check_build(ctx, v, i)
    _check_trace(s, ref, scenes.rays_at_triangles(v, i, 20000, seed=5), max_tie_frac=1.0, wide=True)


@pytest.mark.gpu
def test_trace_wide_icosphere(ctx):
    import keepsake_b200 as ks
    g = ks.Generated("icosphere", 0, level=8)
    v, i = g.flat_geometry()
    s, ref = _check_build(ctx, v, i)
    frac = _check_trace(s, ref, scenes.rays_at_triangles(v, i, 200000, seed=8), max_tie_frac=0.02, wide=True)
    assert frac > 0.5
    _check_trace(s, ref, scenes.random_rays(v, 200000, seed=9, inside=False), max_tie_frac=1e-4, wide=True)
    for culling in (0, 1):
        rays = scenes.rays_at_triangles(v, i, 20000, seed=6)
        a, _, _ = s.trace(rays, culling=culling, wide=True)
        b, _, _ = s.trace(rays, culling=culling)
        assert (a != b).mean() <= 0.02


@pytest.mark.gpu
def test_trace_wide_instanced(ctx):
    """Instanced scenes: the renderer's persistent two-level traversal (TLAS, then the 4-wide view of
    the BLAS) against the one-thread-per-ray kernel of ks_trace_rays: same hits and occlusion, ids,
    distances and barycentrics identical except at exact ties (distances within 8 ulp there)."""
    import keepsake_b200 as ks
    g = ks.Generated("instanced", 5, sky=(64, 32), resolution=(32, 32), prototypes=4, instances=24, frequency=6,
                     emitters=8)
    s = ks.Scene(ctx, g.desc)
    s.build_bvh()
    base, vs, ids = 0, [], []
    for mv, mi, _ in g.flattened():
        vs.append(np.asarray(mv, np.float32))
        ids.append(np.asarray(mi, np.int64) + base)
        base += len(mv)
    v, i = np.concatenate(vs), np.concatenate(ids)
    for rays, ties in ((scenes.random_rays(v, 50000, seed=21), 1e-3),
                       (scenes.random_rays(v, 50000, seed=22, inside=False), 1e-3),
                       (scenes.rays_at_triangles(v, i, 50000, seed=23), 0.02)):
        a, ta, ba = s.trace(rays, wide=True)
        b, tb, bb = s.trace(rays)
        hit = b != 0xFFFFFFFF
        assert np.array_equal(a != 0xFFFFFFFF, hit), "hit/miss differs"
        assert hit.mean() > 0.05
        tie = a != b
        assert tie.mean() <= ties, f"{tie.sum()} ids differ"
        same = hit & ~tie
        assert np.array_equal(ta[same].view(np.uint32), tb[same].view(np.uint32))
        assert np.array_equal(ba[same].view(np.uint32), bb[same].view(np.uint32))
        if tie.any():
            ulps = np.abs(ta[tie].view(np.int32).astype(np.int64) - tb[tie].view(np.int32).astype(np.int64))
            assert ulps.max() <= 8
        oa, _, _ = s.trace(rays, any_hit=True, wide=True)
        ob, _, _ = s.trace(rays, any_hit=True)
        assert np.array_equal(oa, ob)
    s.close()
