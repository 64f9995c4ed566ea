"""Seeded test inputs: triangle soups, ray batches."""
import numpy as np


def soup(n, seed=0, spread=10.0, size=0.5):
    rng = np.random.default_rng(seed)
    c = rng.random((n, 3), dtype=np.float32) * spread
    v = (rng.random((n, 3, 3), dtype=np.float32) - 0.5) * size + c[:, None, :]
    return v.reshape(-1, 3).astype(np.float32), np.arange(3 * n, dtype=np.uint32).reshape(-1, 3)


def degenerate_soup(seed=0):
    """Duplicates, axis-aligned flat triangles, zero-area slivers and shared centroids."""
    rng = np.random.default_rng(seed)
    tris = []
    base = rng.random((3, 3), dtype=np.float32)
    for _ in range(12):  # identical triangles: identical centroids -> degenerate leaf
        tris.append(base.copy())
    for k in range(40):  # flat in z
        t = rng.random((3, 3), dtype=np.float32) * 4
        t[:, 2] = 1.0
        tris.append(t)
    for k in range(20):  # slivers
        a = rng.random(3, dtype=np.float32) * 4
        b = rng.random(3, dtype=np.float32) * 4
        tris.append(np.stack([a, b, (a + b) * 0.5]).astype(np.float32))
    for k in range(60):
        tris.append((rng.random((3, 3), dtype=np.float32) - 0.5) * 0.3 + rng.random(3, dtype=np.float32) * 4)
    v = np.concatenate(tris).astype(np.float32)
    return v, np.arange(len(v), dtype=np.uint32).reshape(-1, 3)


def random_rays(verts, n, seed=0, tmax=np.inf, inside=True):
    rng = np.random.default_rng(seed)
    lo, hi = verts.min(0), verts.max(0)
    ext = hi - lo
    if inside:
        o = lo + rng.random((n, 3)) * ext
    else:
        o = lo - ext + rng.random((n, 3)) * 3 * ext
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    r = np.zeros((n, 8), np.float32)
    r[:, 0:3] = o
    r[:, 3] = 0.0
    r[:, 4:7] = d
    r[:, 7] = tmax
    return r


def rays_at_triangles(verts, idx, n, seed=0):
    """Rays aimed at random points of random triangles (dense hits, many near edges)."""
    rng = np.random.default_rng(seed)
    lo, hi = verts.min(0), verts.max(0)
    ext = hi - lo
    t = rng.integers(0, len(idx), n)
    u = rng.random((n, 2))
    flip = u.sum(1) > 1
    u[flip] = 1 - u[flip]
    # a few exact vertices / edge midpoints
    u[: n // 20] = 0.0
    u[n // 20: n // 10, 0] = 0.5
    u[n // 20: n // 10, 1] = 0.5
    p = verts[idx[t, 0]] * (1 - u[:, :1] - u[:, 1:]) + verts[idx[t, 1]] * u[:, :1] + verts[idx[t, 2]] * u[:, 1:]
    o = lo - 0.5 * ext + rng.random((n, 3)) * 2 * ext
    d = p - o
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    r = np.zeros((n, 8), np.float32)
    r[:, 0:3] = o
    r[:, 4:7] = d
    r[:, 7] = np.inf
    return r


def deep_chain(n=250, k0=-125):
    """Triangles across the x axis at x = 2^k, k = k0 .. k0 + n - 1 (each spanning y, z in [-1, 1]).
    Built with 2 SAH buckets, every split peels the farthest triangle off the rest, so the SBVH is
    about n / 2 levels deep and a ray along +x through all of them meets both children at every
    level: deeper than a 64-entry traversal stack."""
    v = []
    for k in range(k0, k0 + n):
        x = np.float32(2.0) ** k
        v += [[x, -1, -1], [x, 1, -1], [x, 0, 1]]
    v = np.array(v, np.float32)
    return v, np.arange(len(v), dtype=np.uint32).reshape(-1, 3)


def sbvh_depth(right):
    """Levels of a flattened SBVH (DFS order: left child i + 1, right child right[i], 0 = leaf)."""
    best, stack = 0, [(0, 1)]
    while stack:
        i, d = stack.pop()
        best = max(best, d)
        if right[i] != 0:
            stack.append((i + 1, d + 1))
            stack.append((int(right[i]), d + 1))
    return best
