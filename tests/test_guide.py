"""Learned guiding network: CUDA kernels (tcgen05 BF16 MLP, hash grid, vMF head, Adam) against
the FP64 oracle (oracle/guide_oracle.py), and the oracle's hand-derived gradients against torch
float64 autograd."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import guide_oracle as go  # noqa: E402

BOUND = [-1.0, -0.5, -2.0, 1.0, 1.5, 0.0]


def rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def random_dirs(rng, n):
    v = rng.normal(size=(n, 3))
    return v / np.linalg.norm(v, axis=1, keepdims=True)


def random_inputs(rng, n, edge_rows=True):
    lo, hi = np.array(BOUND[:3]), np.array(BOUND[3:])
    pos = lo + (hi - lo) * rng.random((n, 3))
    if edge_rows and n >= 8:
        # positions on and beyond the faces of the bound (clamped to the outermost cells)
        pos[0] = lo
        pos[1] = hi
        pos[2] = hi + 0.3
        pos[3] = lo - 0.3
    return pos.astype(np.float32), random_dirs(rng, n).astype(np.float32), random_dirs(rng, n).astype(np.float32)


def random_params(rng, table_size=1 << 19):
    w = []
    for l, (n, k) in enumerate(go.LAYERS):
        m = rng.uniform(-1, 1, (n, k)) * np.sqrt(6.0 / k)
        if l == len(go.LAYERS) - 1:
            m[go.N_OUT:] = 0.0
        w.append(m.ravel())
    w = np.concatenate(w).astype(np.float32)
    grid = rng.uniform(-1, 1, (go.LEVELS, table_size, 2)).astype(np.float32)
    return w, grid


# ---------------------------------------------------------------------------------------------
# CPU: the oracle's analytic derivatives against autograd
# ---------------------------------------------------------------------------------------------
def _torch_loss(o, wi, t, pb, alpha_max=0.8):
    """(reported loss -t log m, training objective): the mixture follows -t log q, the selection
    logit -t log m with q held fixed."""
    import torch
    alpha = alpha_max * torch.sigmoid(o[:, go.SEL])
    o = o[:, :go.SEL].reshape(-1, go.LOBES, 5)
    raw = o[:, :, :3]
    mu = raw / raw.norm(dim=2, keepdim=True)
    z = o[:, :, 3]
    lk = go.MIN_LOG_KAPPA + torch.nn.functional.softplus(z - go.MIN_LOG_KAPPA) \
        - torch.nn.functional.softplus(z - float(go.LOG_KAPPA_HI))
    kappa = torch.exp(lk)
    w = torch.softmax(o[:, :, 4], dim=1)
    scale = kappa / (2 * np.pi * (1 - torch.exp(-2 * kappa)))
    c = (mu * wi[:, None, :]).sum(2) - 1
    v = scale * torch.exp(kappa * torch.clamp(c, max=0.0))
    q = (w * v).sum(1)
    reported = -(t * torch.log(alpha * q + (1 - alpha) * pb))
    objective = -(t * torch.log(q)) - t * torch.log(alpha * q.detach() + (1 - alpha) * pb)
    return reported, objective


def test_oracle_loss_gradient_matches_autograd():
    import torch
    rng = np.random.default_rng(5)
    n = 64
    o = rng.normal(size=(n, go.N_OUT))
    o[:, 3::5] = rng.uniform(-3, 5, (n, go.LOBES))
    o[0, 3] = -9.0  # below the soft lower bound of log kappa
    o[1, 8] = 12.0  # above the soft upper bound
    wi = random_dirs(rng, n)
    t = rng.uniform(0.1, 2.0, n)
    t[1] = 0.0
    pb = rng.exponential(0.5, n)
    pb[2:6] = 0.0
    loss, g = go.loss_and_grad(o, wi, t, pb)
    ot = torch.tensor(o, dtype=torch.float64, requires_grad=True)
    lt, obj = _torch_loss(ot, torch.tensor(wi), torch.tensor(t), torch.tensor(pb))
    obj.sum().backward()
    np.testing.assert_allclose(loss, lt.detach().numpy(), rtol=1e-12, atol=1e-12)
    np.testing.assert_allclose(g, ot.grad.numpy(), rtol=1e-9, atol=1e-11)


def test_oracle_network_backward_matches_autograd():
    import torch
    rng = np.random.default_rng(6)
    T = 1 << 10
    w, grid = random_params(rng, T)
    res = [2, 3, 4, 5, 6, 7, 8, 9, 10, 12, 14, 16, 20, 24, 28, 32]  # coarse levels dense, fine hashed
    net = go.Network(w, grid, res, BOUND, table_size=T)
    pos, wo, nrm = random_inputs(rng, 96)
    wi = random_dirs(rng, 96)
    t = rng.uniform(0.0, 1.0, 96)
    pb = rng.exponential(0.5, 96)
    o, xs, cs = net.forward(pos, wo, nrm)
    loss, d_o = go.loss_and_grad(o, wi, t, pb)
    gW, gG = net.backward(xs, cs, d_o)

    Wt = [torch.tensor(m, requires_grad=True) for m in net.W]
    Gt = torch.tensor(net.grid, requires_grad=True)
    feats = []
    for lev, (idx, cw) in enumerate(cs):
        feats.append((torch.tensor(cw)[:, :, None] * Gt[lev][torch.tensor(idx)]).sum(1))
    x = torch.cat(feats + [torch.tensor(go.sh16(go.unit(wo))), torch.tensor(go.sh16(go.unit(nrm)))], dim=1)
    for l, W in enumerate(Wt):
        x = x @ W.T
        if l < len(Wt) - 1:
            x = torch.relu(x)
    lt, obj = _torch_loss(x[:, :go.N_OUT], torch.tensor(go.unit(wi)), torch.tensor(t), torch.tensor(pb))
    obj.sum().backward()
    np.testing.assert_allclose(loss.sum(), lt.sum().item(), rtol=1e-12)
    np.testing.assert_allclose(gW, np.concatenate([W.grad.numpy().ravel() for W in Wt]), rtol=1e-9, atol=1e-12)
    np.testing.assert_allclose(gG, Gt.grad.numpy(), rtol=1e-9, atol=1e-12)


def test_oracle_hash_indices_stay_in_table():
    rng = np.random.default_rng(7)
    pos, _, _ = random_inputs(rng, 512)
    res = [16, 2048]
    for T in (1 << 10, 1 << 19):
        for idx, w in go.corners(pos, BOUND[:3], BOUND[3:], res, T):
            assert idx.min() >= 0 and idx.max() < T
            np.testing.assert_allclose(w.sum(1), 1.0, rtol=1e-5)


def test_oracle_mixture_sample_density():
    """Directions drawn by sample_vmm follow the mixture density (an expectation against quadrature)."""
    rng = np.random.default_rng(8)
    o = np.zeros((1, go.N_OUT))
    o[0, 0:5] = [0, 0, 1, np.log(4.0), 0.0]
    o[0, 5:10] = [1, 0, 0, np.log(20.0), 0.5]
    o[0, 14::5] = -50.0
    n = 200000
    oo = np.repeat(o, n, axis=0)
    d = go.mixture_sample(oo, rng.random(n), rng.random(n))
    np.testing.assert_allclose(np.linalg.norm(d, axis=1), 1.0, atol=1e-9)
    # E[f] under the samples vs the density integrated on a fine sphere grid
    f = lambda v: v[:, 2] ** 2 + 0.5 * v[:, 0]  # noqa: E731
    th = (np.arange(400) + 0.5) / 400 * np.pi
    ph = (np.arange(800) + 0.5) / 800 * 2 * np.pi
    T, P = np.meshgrid(th, ph, indexing="ij")
    v = np.stack([np.sin(T) * np.cos(P), np.sin(T) * np.sin(P), np.cos(T)], -1).reshape(-1, 3)
    dA = (np.sin(T) * (np.pi / 400) * (2 * np.pi / 800)).ravel()
    pdf = go.mixture_pdf(np.repeat(o, len(v), axis=0), v)
    assert abs((pdf * dA).sum() - 1.0) < 1e-3
    expect = (f(v) * pdf * dA).sum()
    assert abs(f(d).mean() - expect) < 5e-3


# ---------------------------------------------------------------------------------------------
# GPU parity
# ---------------------------------------------------------------------------------------------
@pytest.fixture(scope="module")
def guide(ctx):
    import keepsake_b200 as ks
    g = ks.Guide(ctx, BOUND, seed=11)
    yield g
    g.close()


@pytest.mark.gpu
def test_guide_init_and_level_res(guide):
    res = guide.level_res()
    assert res[0] == 16 and res[-1] == 2048 and np.all(np.diff(res.astype(np.int64)) > 0)
    w, grid = guide.get_weights()
    assert np.all(np.isfinite(w)) and np.abs(grid).max() <= 1e-4
    assert np.all(go.split_weights(w)[-1][go.N_OUT:] == 0)


@pytest.mark.gpu
@pytest.mark.parametrize("n", [1, 127, 1000, 148 * 128 * 2 + 5])
def test_guide_infer_matches_fp64(guide, n):
    rng = np.random.default_rng(100 + n)
    w, grid = random_params(rng)
    guide.set_weights(w, grid)
    pos, wo, nrm = random_inputs(rng, n)
    out = guide.infer(pos, wo, nrm)
    net = go.Network(w, grid, guide.level_res(), BOUND)
    ref_bf, _, _ = net.forward(pos, wo, nrm, bf=True, half_grid=True)
    ref64, _, _ = net.forward(pos, wo, nrm, bf=False)
    # same FP16 table entries and BF16 operands: only FP32 summation order differs
    assert rel(out, ref_bf) < 2e-3, rel(out, ref_bf)
    # against exact FP64 of the same FP32 weights: BF16 operand precision
    assert rel(out, ref64) < 3e-2, rel(out, ref64)


@pytest.mark.gpu
def test_guide_infer_empty(guide):
    assert guide.infer(np.zeros((0, 3)), np.zeros((0, 3)), np.zeros((0, 3))).shape == (0, go.N_OUT)


@pytest.mark.gpu
@pytest.mark.parametrize("n", [200, 148 * 128 * 2 + 77])
def test_guide_gradients_match_fp64(guide, n):
    rng = np.random.default_rng(200 + n)
    w, grid = random_params(rng)
    w *= 0.5
    guide.set_weights(w, grid)
    pos, wo, nrm = random_inputs(rng, n)
    wi = random_dirs(rng, n).astype(np.float32)
    t = rng.exponential(1.0, n).astype(np.float32)
    t[::7] = 0.0
    pb = rng.exponential(0.3, n).astype(np.float32)
    pb[::5] = 0.0
    loss, gw, gg = guide.gradients(pos, wo, nrm, wi, t, pb)
    net = go.Network(w, grid, guide.level_res(), BOUND)
    # (1) the same BF16 operands in FP64: only FP32 summation order differs
    o, xs, cs = net.forward(pos, wo, nrm, bf=True)
    l_ref, d_o = go.loss_and_grad(o, wi, t.astype(np.float64) / n, pb)
    gw_ref, gg_ref = net.backward(xs, cs, d_o, bf=True)
    assert abs(loss - l_ref.sum()) <= 5e-3 * abs(l_ref.sum()), (loss, l_ref.sum())
    assert rel(gw, gw_ref) < 5e-3, rel(gw, gw_ref)
    assert rel(gg, gg_ref) < 5e-3, rel(gg, gg_ref)
    # (2) exact FP64 of the same FP32 parameters.  The batch gradient is a small residual of
    # per-row terms of both signs, so its error is bounded against the absolute-value backward
    # pass: within BF16's unit roundoff (2^-8) of that scale.
    o, xs, cs = net.forward(pos, wo, nrm, bf=False)
    l_ref, d_o = go.loss_and_grad(o, wi, t.astype(np.float64) / n, pb)
    gw_ref, gg_ref = net.backward(xs, cs, d_o)
    gw_abs, gg_abs = net.backward_abs(xs, cs, d_o)
    assert abs(loss - l_ref.sum()) <= 2e-2 * abs(l_ref.sum()), (loss, l_ref.sum())
    assert np.linalg.norm(gw - gw_ref) <= 2.0 ** -8 * np.linalg.norm(gw_abs)
    assert np.linalg.norm(gg - gg_ref) <= 2.0 ** -8 * np.linalg.norm(gg_abs)
    # gradients were discarded: a second call returns the same values
    loss2, gw2, _ = guide.gradients(pos, wo, nrm, wi, t, pb)
    assert abs(loss2 - loss) <= 1e-6 * abs(loss)
    assert rel(gw2, gw) < 1e-5


@pytest.mark.gpu
def test_guide_adam_step_matches_oracle(ctx):
    import keepsake_b200 as ks
    g = ks.Guide(ctx, BOUND, seed=3, learning_rate=1e-2)
    rng = np.random.default_rng(9)
    pos, wo, nrm = random_inputs(rng, 3000)
    wi = random_dirs(rng, 3000)
    t = rng.exponential(1.0, 3000)
    w0, grid0 = g.get_weights()
    m = np.zeros_like(w0)
    v = np.zeros_like(w0)
    mg = np.zeros_like(grid0)
    vg = np.zeros_like(grid0)
    for it in (1, 2):
        _, gw, gg = g.gradients(pos, wo, nrm, wi, t, apply_adam=True)
        w0, m, v = go.adam(w0, gw, m, v, it, 1e-2)
        grid0, mg, vg = go.adam(grid0, gg, mg, vg, it, 1e-2)
        w1, grid1 = g.get_weights()
        np.testing.assert_allclose(w1, w0, rtol=2e-6, atol=1e-9)
        np.testing.assert_allclose(grid1, grid0, rtol=2e-6, atol=1e-9)
    g.close()


@pytest.mark.gpu
def test_guide_training_learns_directional_field(ctx):
    """Online training on samples of a position-dependent vMF: the learned mixture's
    cross-entropy approaches the target's own."""
    import keepsake_b200 as ks
    g = ks.Guide(ctx, BOUND, seed=4, learning_rate=1e-2)
    rng = np.random.default_rng(10)
    kappa = 30.0

    def batch(n):
        pos, wo, nrm = random_inputs(rng, n, edge_rows=False)
        c = np.array([0.0, 0.5, -1.0])
        d = go.unit(np.asarray(pos, np.float64) - c + np.array([0.0, 0.0, 0.3]))
        o = np.full((n, go.N_OUT), -50.0)
        o[:, 0:3] = d
        o[:, 3] = np.log(kappa)
        o[:, 4] = 0.0
        wi = go.mixture_sample(o, rng.random(n), rng.random(n))
        return pos, wo, nrm, wi.astype(np.float32), np.ones(n, np.float32)

    vpos, vwo, vnrm, vwi, vt = batch(4096)

    def xent():
        return float(-np.mean(np.log(go.mixture_pdf(g.infer(vpos, vwo, vnrm), vwi))))

    start = xent()
    for _ in range(400):
        g.train_step(*batch(1 << 14))
    end = xent()
    # cross-entropy of the target vMF with itself (its differential entropy)
    mean_cos = 1.0 / np.tanh(kappa) - 1.0 / kappa
    h = -np.log(kappa / (2 * np.pi * (1 - np.exp(-2 * kappa)))) + kappa * (1.0 - mean_cos)
    assert start > 2.0
    assert end < start - 2.0, (start, end, h)
    assert end < h + 0.5, (start, end, h)
    g.close()
