"""Sobol sampler parity: oracle pinned to the reference's generator table, CUDA kernel bit-exact
against the oracle (PTRenderSampler / OwenScrambledSobol02Morton, sobol.h:131-248)."""
import json
import os

import numpy as np
import pytest

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def test_oracle_matrices_match_reference_table(oracle):
    g = json.load(open(os.path.join(GOLDEN, "sobol_matrices.json")))
    m = oracle.sobol_matrices01()
    assert list(m[:52]) == g["dim0"]
    assert list(m[52:]) == g["dim1"]


def test_oracle_points_in_unit_interval(oracle):
    pts = oracle.sobol_points(256, 256, 64, 0, 100, 37, 4, 4, 0, 64, 12)
    assert pts.dtype == np.float32
    assert (pts >= 0).all() and (pts < 1).all()


@pytest.mark.parametrize("spp", [16, 64])
def test_oracle_first_dims_are_02_net(oracle, spp):
    # Dimensions (0,1) of next2d() over the spp samples of one pixel are a scrambled (0,2)-net in
    # base 2: every elementary interval of area 1/spp holds exactly one point.
    pts = oracle.sobol_points(256, 256, spp, 7, 31, 9, 1, 1, 0, spp, 1)[0, 0, :, 0, 1:3]
    k = int(np.log2(spp))
    for a in range(k + 1):
        nx, ny = 2 ** a, 2 ** (k - a)
        cells = np.floor(pts[:, 0] * nx).astype(int) * ny + np.floor(pts[:, 1] * ny).astype(int)
        assert len(np.unique(cells)) == spp


def test_oracle_non_pow4_spp(oracle):
    # odd log2(spp): the extra binary digit path (sobol.h:216-219)
    pts = oracle.sobol_points(64, 64, 32, 3, 5, 5, 2, 2, 0, 32, 4)
    assert (pts >= 0).all() and (pts < 1).all()
    assert len(np.unique(pts[0, 0, :, 0, 1])) == 32


CASES = [
    # name, full_w, full_h, spp, seed, x0, y0, nx, ny, s0, ns, nd
    ("box_room_256_64spp", 256, 256, 64, 0, 0, 0, 32, 32, 0, 64, 62),
    ("box_room_corner", 256, 256, 64, 0, 224, 224, 32, 32, 0, 64, 20),
    ("icosphere_1024_256spp", 1024, 1024, 256, 0, 511, 700, 8, 8, 0, 256, 16),
    ("guided_1080p_odd_log2", 1920, 1080, 128, 5, 1900, 1060, 20, 20, 0, 128, 8),
    # 4096^2 padded Morton x 1024 spp: sample indices reach 2^34 (Morton shift overflows 32 bits)
    ("instanced_4k_1024spp", 3840, 2160, 1024, 0, 3800, 2140, 16, 16, 1000, 24, 8),
    ("spp1", 640, 480, 1, 9, 0, 0, 64, 64, 0, 1, 40),
    ("spp_non_pow2", 128, 128, 24, 1, 10, 10, 8, 8, 0, 24, 8),
]


@pytest.mark.gpu
@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
def test_sobol_kernel_bit_exact(ctx, oracle, case):
    _, *args = case
    got = ctx.sobol_points(*args)
    want = oracle.sobol_points(*args)
    assert got.shape == want.shape
    diff = got.view(np.uint32) != want.view(np.uint32)
    assert not diff.any(), f"{diff.sum()} of {diff.size} Sobol values differ"


@pytest.mark.gpu
@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
def test_sobol_bounce_bit_exact(ctx, oracle, case):
    """The sampling kernel's per-vertex draw (five permuted indices from one digit pass) equals the
    reference's next(), next2d(), next(), next2d(), next() in turn, at the first dimension of a
    bounce (2 + 7 b in the renderer, camera dimensions first) and at a late one."""
    _, fw, fh, spp, seed, x0, y0, nx, ny, s0, ns, _nd = case
    for dim in (2, 9, 2 + 7 * 11):
        got = ctx.sobol_bounce(fw, fh, spp, seed, x0, y0, nx, ny, s0, ns, dim)
        pts = oracle.sobol_points(fw, fh, spp, seed, x0, y0, nx, ny, s0, ns, dim + 7)
        want = np.stack([pts[..., dim, 0], pts[..., dim + 1, 1], pts[..., dim + 1, 2], pts[..., dim + 3, 0],
                         pts[..., dim + 4, 1], pts[..., dim + 4, 2], pts[..., dim + 6, 0]], axis=-1)
        diff = got.view(np.uint32) != want.view(np.uint32)
        assert not diff.any(), f"dim {dim}: {diff.sum()} of {diff.size} values differ"
