"""ORACLE (test infrastructure only): FP64 evaluation of the learned guiding network.

Tests and ``__graft_entry__.smoke()`` use this module to check the CUDA guide kernels
(keepsake_b200/csrc/ks_guide.cu); the product never imports it.

The network (position hash grid + direction spherical harmonics -> 4 x 64 ReLU MLP -> 8-lobe vMF
mixture) has no CPU counterpart in the reference; what it shares with the reference is followed
here line by line:

  vMF density            VMF::eval                   vmf.h:32-39 (max_kappa 1e4, vmf.h:110)
  mixture sampling       sample_vmm                  vmf.h:123-127, sample_small_distrib rng.h:399-432
  vMF sampling           VMF::sample                 vmf.h:41-56, orthonormal_basis maths.h:814-821
  Adam                   adam_optimizer_step         gpu/shaders/adam.slang:25-51

Everything is float64 except where the CUDA path's own float32 arithmetic decides a discrete
outcome (grid cell of a position, trilinear corner weights): those steps are repeated in float32
so that both sides pick the same table entries.  ``bf16=True`` additionally rounds the operands
the tensor cores read (weights, activations, back-propagated gradients) to bfloat16 at the same
points as the CUDA kernels, which isolates layout errors from the expected precision loss.
"""
from __future__ import annotations

import numpy as np

LEVELS = 16
FEATS = 2
N_SH = 16
N_IN = LEVELS * FEATS + 2 * N_SH
HIDDEN = 64
LOBES = 8
SEL = LOBES * 5  # selection logit
N_OUT = LOBES * 5 + 1
LAYERS = [(64, 64), (64, 64), (64, 64), (64, 64), (48, 64)]  # (out, in); the last padded 41 -> 48
MAX_KAPPA = 1e4
MIN_LOG_KAPPA = -6.0
PRIMES = (1, 2654435761, 805459861)


def bf16(x):
    """Rounds to bfloat16 (round to nearest even) via float32, returned as float64."""
    f = np.asarray(x, np.float64).astype(np.float32)
    b = f.view(np.uint32).astype(np.uint64)
    b = (b + 0x7FFF + ((b >> 16) & 1)) & 0xFFFF0000
    return b.astype(np.uint32).view(np.float32).astype(np.float64)


def split_weights(flat):
    out, o = [], 0
    for n, k in LAYERS:
        out.append(np.asarray(flat[o:o + n * k], np.float64).reshape(n, k))
        o += n * k
    return out


def corners(pos, bmin, bmax, res, table_size):
    """Per level: table indices (n, 8) and trilinear weights (n, 8) of the enclosing cell."""
    pos = np.asarray(pos, np.float32)
    bmin = np.asarray(bmin, np.float32)
    inv = (np.float32(1.0) / (np.asarray(bmax, np.float32) - bmin)).astype(np.float32)
    pn = ((pos - bmin) * inv).astype(np.float32)
    pn = np.clip(pn, np.float32(0), np.float32(1))
    out = []
    for r in res:
        r = int(r)
        p = (pn * np.float32(r)).astype(np.float32)
        f0 = np.minimum(np.floor(p), np.float32(r - 1)).astype(np.float32)
        t = (p - f0).astype(np.float32)
        i0 = f0.astype(np.uint64)
        # while the level fits: corners in 2 x 2 x 2 blocks of 8 consecutive entries, blocks indexed
        # densely; finer levels: each corner hashed
        side = (r + 2) >> 1
        dense = side ** 3 * 8 <= table_size
        idx = np.empty((len(pos), 8), np.int64)
        w = np.empty((len(pos), 8), np.float64)
        for k in range(8):
            d = np.array([k & 1, (k >> 1) & 1, (k >> 2) & 1], np.uint64)
            c = i0 + d
            if dense:
                inner = (c[:, 0] & 1) | ((c[:, 1] & 1) << 1) | ((c[:, 2] & 1) << 2)
                b = c >> np.uint64(1)
                blk = b[:, 0] + np.uint64(side) * (b[:, 1] + np.uint64(side) * b[:, 2])
                idx[:, k] = (blk * np.uint64(8) + inner).astype(np.int64)
            else:
                h = (c[:, 0] * np.uint64(PRIMES[0])) ^ (c[:, 1] * np.uint64(PRIMES[1])) ^ \
                    (c[:, 2] * np.uint64(PRIMES[2]))
                idx[:, k] = (h & np.uint64(table_size - 1)).astype(np.int64)
            wk = np.ones(len(pos), np.float32)
            for a in range(3):
                wk = (wk * np.where(d[a] == 1, t[:, a], np.float32(1) - t[:, a])).astype(np.float32)
            w[:, k] = wk
        out.append((idx, w))
    return out


def sh16(d):
    """Real spherical harmonics up to degree 3 of unit directions (n, 3)."""
    x, y, z = d[:, 0], d[:, 1], d[:, 2]
    xx, yy, zz = x * x, y * y, z * z
    c = np.empty((len(d), 16))
    c[:, 0] = 0.28209479177387814
    c[:, 1] = -0.48860251190291987 * y
    c[:, 2] = 0.48860251190291987 * z
    c[:, 3] = -0.48860251190291987 * x
    c[:, 4] = 1.0925484305920792 * x * y
    c[:, 5] = -1.0925484305920792 * y * z
    c[:, 6] = 0.94617469575755997 * zz - 0.31539156525251999
    c[:, 7] = -1.0925484305920792 * x * z
    c[:, 8] = 0.54627421529603959 * (xx - yy)
    c[:, 9] = 0.59004358992664352 * y * (-3.0 * xx + yy)
    c[:, 10] = 2.8906114426405538 * x * y * z
    c[:, 11] = 0.45704579946446572 * y * (1.0 - 5.0 * zz)
    c[:, 12] = 0.3731763325901154 * z * (5.0 * zz - 3.0)
    c[:, 13] = 0.45704579946446572 * x * (1.0 - 5.0 * zz)
    c[:, 14] = 1.4453057213202769 * z * (xx - yy)
    c[:, 15] = 0.59004358992664352 * x * (-xx + 3.0 * yy)
    return c


def unit(v):
    v = np.asarray(v, np.float64)
    return v / np.linalg.norm(v, axis=1, keepdims=True)


class Network:
    """FP64 guide network with the same parameters as a ks_guide."""

    def __init__(self, weights_flat, grid, res, bound, table_size=None):
        self.W = split_weights(weights_flat)
        self.grid = np.asarray(grid, np.float64).reshape(LEVELS, -1, FEATS)
        self.table_size = table_size or self.grid.shape[1]
        self.res = [int(r) for r in res]
        self.bmin = np.asarray(bound[:3], np.float32)
        self.bmax = np.asarray(bound[3:], np.float32)

    def encode(self, pos, wo, nrm, half_grid=False):
        cs = corners(pos, self.bmin, self.bmax, self.res, self.table_size)
        grid = self.grid
        if half_grid:
            # the inference kernels read an FP16 copy of the table (round to nearest even)
            grid = np.clip(grid, -65504.0, 65504.0).astype(np.float32).astype(np.float16).astype(np.float64)
        feats = [np.einsum("nk,nkf->nf", w, grid[l][idx]) for l, (idx, w) in enumerate(cs)]
        x0 = np.concatenate(feats + [sh16(unit(wo)), sh16(unit(nrm))], axis=1)
        return x0, cs

    def forward(self, pos, wo, nrm, bf=False, half_grid=False):
        """Raw outputs (n, 41) and the per-layer inputs X_l kept for the backward pass.
        half_grid: the hash-grid features as the inference kernels read them (FP16)."""
        x, cs = self.encode(pos, wo, nrm, half_grid)
        rnd = bf16 if bf else (lambda a: a)
        xs = []
        for l, W in enumerate(self.W):
            x = rnd(x)
            xs.append(x)
            z = x @ rnd(W).T
            x = np.maximum(z, 0.0) if l < len(self.W) - 1 else z
        return x[:, :N_OUT], xs, cs

    def backward(self, xs, cs, d_out, bf=False):
        """Gradients (flat weights, grid) of sum(d_out * outputs)."""
        rnd = bf16 if bf else (lambda a: a)
        dy = np.zeros((len(d_out), LAYERS[-1][0]))
        dy[:, :N_OUT] = d_out
        gW = [None] * len(self.W)
        for l in range(len(self.W) - 1, -1, -1):
            dy = rnd(dy)
            gW[l] = dy.T @ xs[l]
            dx = dy @ rnd(self.W[l])
            if l > 0:
                dy = np.where(xs[l] > 0.0, dx, 0.0)
        g_grid = np.zeros_like(self.grid)
        for lev, (idx, w) in enumerate(cs):
            for f in range(FEATS):
                contrib = w * dx[:, 2 * lev + f][:, None]
                np.add.at(g_grid[lev][:, f], idx.ravel(), contrib.ravel())
        return np.concatenate([g.ravel() for g in gW]), g_grid

    def backward_abs(self, xs, cs, d_out):
        """The backward pass on absolute values (|d_out|, |W|, |X|, corner weights, same ReLU
        masks): the scale against which the rounding error of a gradient sum is bounded.  A batch
        gradient can be orders of magnitude smaller than this scale (per-row terms of both signs
        cancel), so its relative error says little about the arithmetic; its error over this
        scale does."""
        W = self.W
        try:
            self.W = [np.abs(m) for m in W]
            # hidden inputs are ReLU outputs (>= 0): their masks are unchanged by abs
            return self.backward([np.abs(x) for x in xs], [(i, np.abs(w)) for i, w in cs], np.abs(d_out))
        finally:
            self.W = W


def softplus(x):
    return np.where(x > 20.0, x, np.log1p(np.exp(np.minimum(x, 20.0))))


def sigmoid(x):
    return 1.0 / (1.0 + np.exp(-x))


LOG_KAPPA_HI = np.log(MAX_KAPPA)


def log_kappa(z):
    """Smooth clamp of the raw concentration output into (MIN_LOG_KAPPA, log MAX_KAPPA)."""
    return MIN_LOG_KAPPA + softplus(z - MIN_LOG_KAPPA) - softplus(z - LOG_KAPPA_HI)


def log_kappa_grad(z):
    return sigmoid(z - MIN_LOG_KAPPA) - sigmoid(z - LOG_KAPPA_HI)


def decode(o):
    """Raw outputs (n, 41) -> mean directions (n, 8, 3), concentrations (n, 8), weights (n, 8)."""
    o = np.asarray(o, np.float64).reshape(-1, N_OUT)[:, :SEL].reshape(-1, LOBES, 5)
    raw = o[:, :, :3]
    nrm = np.linalg.norm(raw, axis=2, keepdims=True)
    mu = np.where(nrm > 1e-20, raw / np.maximum(nrm, 1e-300), np.array([0.0, 0.0, 1.0]))
    kappa = np.minimum(np.exp(log_kappa(o[:, :, 3])), MAX_KAPPA)
    lg = o[:, :, 4] - o[:, :, 4].max(axis=1, keepdims=True)
    w = np.exp(lg)
    w /= w.sum(axis=1, keepdims=True)
    return mu, kappa, w


def vmf_eval(mu, kappa, wi):
    """VMF::eval (vmf.h:32-39), broadcast over lobes; wi (n, 3)."""
    scale = kappa / (2.0 * np.pi * (1.0 - np.exp(-2.0 * kappa)))
    c = np.einsum("nlk,nk->nl", mu, wi) - 1.0
    return scale * np.exp(kappa * np.minimum(0.0, c))


def mixture_pdf(o, wi):
    mu, kappa, w = decode(o)
    return (w * vmf_eval(mu, kappa, unit(wi))).sum(axis=1)


def selection(o, alpha_max):
    """Selection probability alpha = alpha_max * sigmoid(z) of the mixture against the BSDF."""
    z = np.asarray(o, np.float64).reshape(-1, N_OUT)[:, SEL]
    return alpha_max / (1.0 + np.exp(-z))


def loss_and_grad(o, wi, t, p_bsdf=None, alpha_max=0.8):
    """Per-row loss -t log m(wi), m = alpha q + (1 - alpha) p_bsdf (the combined proposal of
    one-sample MIS), and the training gradient w.r.t. the 41 raw outputs: the mixture outputs
    follow -t log q(wi), the selection logit follows -t log m with q held fixed."""
    full = np.asarray(o, np.float64).reshape(-1, N_OUT)
    n = len(full)
    o = full[:, :SEL].reshape(-1, LOBES, 5)
    wi = unit(wi)
    t = np.asarray(t, np.float64)
    pb = np.zeros(n) if p_bsdf is None else np.asarray(p_bsdf, np.float64)
    mu, kappa, w = decode(full)
    v = vmf_eval(mu, kappa, wi)
    q = (w * v).sum(axis=1)
    sg = 1.0 / (1.0 + np.exp(-full[:, SEL]))
    alpha = alpha_max * sg
    m = alpha * q + (1.0 - alpha) * pb
    ok = (t > 0) & (q > 1e-30) & (m > 1e-30)
    ms = np.where(ok, m, 1.0)
    qs = np.where(ok, q, 1.0)
    loss = np.where(ok, -t * np.log(ms), 0.0)
    g_sel = np.where(ok, -t * (q - pb) / ms * alpha_max * sg * (1.0 - sg), 0.0)
    r = np.where(ok[:, None], w * v / qs[:, None], 0.0)
    g = np.zeros_like(o)
    tt = np.where(ok, t, 0.0)[:, None]
    g[:, :, 4] = -tt * (r - np.where(ok[:, None], w, 0.0))
    cosd = np.einsum("nlk,nk->nl", mu, wi)
    with np.errstate(over="ignore"):
        dlog = 1.0 / kappa - 2.0 / np.expm1(2.0 * kappa) + (cosd - 1.0)
    g[:, :, 3] = -tt * r * dlog * kappa * log_kappa_grad(o[:, :, 3])
    raw = o[:, :, :3]
    nrm = np.linalg.norm(raw, axis=2, keepdims=True)
    gm = kappa[:, :, None] * wi[:, None, :]
    proj = (gm - (gm * mu).sum(axis=2, keepdims=True) * mu) / np.maximum(nrm, 1e-300)
    g[:, :, :3] = np.where(nrm > 1e-20, -(tt * r)[:, :, None] * proj, 0.0)
    return loss, np.concatenate([g.reshape(n, SEL), g_sel[:, None]], axis=1)


def adam(p, g, m, v, it, lr, b1=0.9, b2=0.999, eps=1e-8):
    """adam_optimizer_step (adam.slang:39-50) in float32; returns (p, m, v)."""
    f = np.float32
    p, g, m, v = (np.asarray(a, np.float32) for a in (p, g, m, v))
    mt = (g + f(b1) * (m - g)).astype(f)
    vt = (g * g + f(b2) * (v - g * g)).astype(f)
    c1 = f(1.0) - f(b1) ** f(it)
    c2 = f(1.0) - f(b2) ** f(it)
    p = (p - f(lr) * (mt / c1) / (np.sqrt(vt / c2) + f(eps))).astype(f)
    return p, mt, vt


def orthonormal_basis(n):
    """orthonormal_basis (maths.h:814-821) for unit vectors (n, 3)."""
    sign = np.copysign(1.0, n[:, 2])
    a = -1.0 / (sign + n[:, 2])
    b = n[:, 0] * n[:, 1] * a
    X = np.stack([1.0 + sign * n[:, 0] ** 2 * a, sign * b, -sign * n[:, 0]], axis=1)
    Y = np.stack([b, sign + n[:, 1] ** 2 * a, -n[:, 1]], axis=1)
    return X, Y


def mixture_sample(o, u0, u1):
    """sample_vmm (vmf.h:123-127): lobe by sample_small_distrib, then VMF::sample."""
    mu, kappa, w = decode(o)
    n = len(w)
    sel = np.full(n, -1)
    u = np.asarray(u0, np.float64).copy()
    cdf = np.zeros(n)
    inv = 1.0 / w.sum(axis=1)
    for j in range(LOBES):
        nx = cdf + w[:, j] * inv
        hit = (sel < 0) & (u < nx)
        u = np.where(hit, (u - cdf) / np.where(hit, nx - cdf, 1.0), u)
        sel = np.where(hit, j, sel)
        cdf = nx
    last = np.array([max([j for j in range(LOBES) if w[i, j] > 0]) for i in range(n)])
    sel = np.where(sel < 0, last, sel)
    m = mu[np.arange(n), sel]
    k = kappa[np.arange(n), sel]
    ct = 1.0 + np.log(u + np.exp(-2.0 * k) * (1.0 - u)) / k
    st = np.sqrt(np.maximum(0.0, 1.0 - ct * ct))
    phi = 2.0 * np.pi * np.asarray(u1, np.float64)
    X, Y = orthonormal_basis(m)
    return (np.cos(phi) * st)[:, None] * X + (np.sin(phi) * st)[:, None] * Y + ct[:, None] * m
