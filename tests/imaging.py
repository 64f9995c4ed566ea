"""Image helpers shared by the render tests and bench.py (no oracle imports here)."""
import numpy as np


def composite(accum, weights, backdrop=(0.0, 0.0, 0.0)):
    """RenderTarget2::composite_and_save_to_exr (render_target.cpp:181-205) in FP64."""
    w_sum = (weights[..., 0] + weights[..., 1]).astype(np.uint32).astype(np.float64)
    w = np.where(w_sum == 0, 0.0, weights[..., 0] / np.maximum(w_sum, 1))
    fg = np.where(weights[..., :1] == 0, 0.0, accum / np.maximum(weights[..., :1], 1e-300))
    b = np.asarray(backdrop, np.float64)
    return (1.0 - w)[..., None] * b + w[..., None] * fg


def rel_mse(x, ref, eps=1e-2):
    """mean over pixels and channels of (x - r)^2 / (r^2 + eps)."""
    x = np.asarray(x, np.float64)
    ref = np.asarray(ref, np.float64)
    return float(np.mean((x - ref) ** 2 / (ref ** 2 + eps)))
