"""Crafted "Color" frames for the accumulation tests (CPU and GPU).

AccumulationPass clamps fireflies in place in row-major order
(passes/accumulation_pass.cpp:22-60); the GPU accumulation shader clamps
against the unclamped input (accumulation.slang:55-81). The two agree for
finite colours. They differ when a pixel with infinite luminance is clamped
(its scale is 0, inf * 0 is NaN, and a NaN luminance drops out of its later
neighbours' maximum), so later neighbours with large luminance get clamped in
place but not by the shader. These frames hold such chains, negative and NaN
luminance, fireflies on every border and corner, and plain noise.
"""
import numpy as np


def crafted_frames(width: int, height: int, n_frames: int, seed: int, chains: bool = True):
    rng = np.random.default_rng(seed)
    n = width * height
    out = []
    for _ in range(n_frames):
        c = (rng.random((n, 4), dtype=np.float32) * np.float32(0.8)).astype(np.float32)
        img = c.reshape(height, width, 4)
        # fireflies, including every corner and border pixel of small frames
        k = max(1, n // 40)
        idx = rng.choice(n, size=k, replace=False)
        c[idx, :3] *= np.float32(300.0)
        for (y, x) in ((0, 0), (0, width - 1), (height - 1, 0), (height - 1, width - 1)):
            img[y, x, :3] = np.float32(500.0) * rng.random(3, dtype=np.float32)
        # negative luminance (never clamped, never raises a neighbour's threshold)
        neg = rng.choice(n, size=max(1, n // 60), replace=False)
        c[neg, :3] = -rng.random((len(neg), 3), dtype=np.float32) * np.float32(50.0)
        # NaN luminance (never clamped, skipped by the neighbourhood maximum)
        nan = rng.choice(n, size=max(1, n // 200), replace=False)
        c[nan, 0] = np.float32(np.nan)
        if chains and width >= 4 and height >= 2:
            # an isolated infinite pixel followed by one bright pixel in a dim
            # neighbourhood: the in-place order clamps the bright pixel (the
            # infinite one became NaN), the shader does not (it still sees inf)
            for _ in range(max(1, n // 300)):
                y = int(rng.integers(0, height))
                x = int(rng.integers(1, width - 2))
                img[max(0, y - 1):y + 2, x - 1:x + 3, :3] = np.float32(0.05)
                img[y, x, :3] = (np.float32(np.inf), np.float32(1.0), np.float32(1.0))
                img[y, x + 1, :3] = np.float32(40.0)
        out.append(np.ascontiguousarray(c))
    return out


SIZES = [(1, 1), (1, 7), (9, 1), (2, 2), (3, 5), (16, 16), (37, 23), (64, 48)]


def same_or_both_nan(a: np.ndarray, b: np.ndarray) -> bool:
    """Bit equality, except that NaNs compare by position only: x86 and the GPU
    make NaNs with different payloads (and propagate them differently)."""
    na, nb = np.isnan(a), np.isnan(b)
    if not np.array_equal(na, nb):
        return False
    return np.array_equal(a[~na].view(np.uint32), b[~nb].view(np.uint32))
