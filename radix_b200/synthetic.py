"""Seeded synthetic splat tables and cameras of the benchmark workloads.

Random numbers are mulberry32 (the generator of the reference's checks,
scripts/check-core.ts:43-48) with normals by Box-Muller. mulberry32's state
advances by a constant, so output k of a stream is a pure function of
seed + (k + 1) * 0x6D2B79F5: streams are generated vectorised, in numpy or in
torch, one field after another from a single seeded stream.
"""
import math

import numpy as np

from .camera import Camera

_INC = 0x6D2B79F5
_MASK = 0xFFFFFFFF


class Mulberry32:
    """A mulberry32 stream; uniform(n) returns its next n outputs in [0, 1)."""

    def __init__(self, seed, device=None):
        self.state = seed & _MASK
        self.device = device  # None: numpy; else a torch device

    def _bits(self, n):
        if self.device is None:
            k = np.arange(1, n + 1, dtype=np.uint64)
            s = (np.uint64(self.state) + k * np.uint64(_INC)) & np.uint64(_MASK)
            t = ((s ^ (s >> np.uint64(15))) * (s | np.uint64(1))) & np.uint64(_MASK)
            t = ((t + (((t ^ (t >> np.uint64(7))) * (t | np.uint64(61))) & np.uint64(_MASK))) & np.uint64(_MASK)) ^ t
            out = (t ^ (t >> np.uint64(14))) & np.uint64(_MASK)
        else:
            import torch
            k = torch.arange(1, n + 1, dtype=torch.int64, device=self.device)
            s = (self.state + k * _INC) & _MASK
            t = ((s ^ (s >> 15)) * (s | 1)) & _MASK
            t = ((t + (((t ^ (t >> 7)) * (t | 61)) & _MASK)) & _MASK) ^ t
            out = (t ^ (t >> 14)) & _MASK
        self.state = (self.state + n * _INC) & _MASK
        return out

    def uniform(self, n):
        b = self._bits(n)
        return b.astype(np.float64) / 4294967296.0 if self.device is None else b.double() / 4294967296.0

    def normal(self, n, mean=0.0, std=1.0):
        u1 = self.uniform(n)
        u2 = self.uniform(n)
        if self.device is None:
            z = np.sqrt(-2.0 * np.log(1.0 - u1)) * np.cos(2.0 * math.pi * u2)
        else:
            import torch
            z = torch.sqrt(-2.0 * torch.log(1.0 - u1)) * torch.cos(2.0 * math.pi * u2)
        return mean + std * z


def _np(x):
    return x if isinstance(x, np.ndarray) else x.cpu().numpy()


def _sigmoid(x):
    return 1.0 / (1.0 + np.exp(-x))


def _unit_quats(rng, n):
    q = _np(rng.normal(4 * n)).reshape(n, 4)
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    return q


def plain_table(n, seed=0, device=None):
    """Uniform centres in [-1, 1]^3, log-scales N(-4, 0.5), unit quaternions,
    opacity sigmoid(N(0, 1)), SH degree 0 with rgb U[0, 1]."""
    rng = Mulberry32(seed, device)
    centers = _np(rng.uniform(3 * n)).reshape(n, 3) * 2.0 - 1.0
    log_scales = _np(rng.normal(3 * n, -4.0, 0.5)).reshape(n, 3)
    quats = _unit_quats(rng, n)
    opacities = _sigmoid(_np(rng.normal(n)))
    colors = _np(rng.uniform(3 * n)).reshape(n, 1, 3)
    return dict(centers=centers.astype(np.float32), log_scales=log_scales.astype(np.float32),
                quats=quats.astype(np.float32), opacities=opacities.astype(np.float32),
                colors=colors.astype(np.float32), sh_degree=0)


def mixture_table(n, seed=0, sh_degree=3, color_dtype=np.float32, components=32, device=None):
    """Centres from a mixture of `components` Gaussians (sigma 0.2, means
    U[-5, 5]^3, equal weights, clamped to the box), log-scales N(-4.5, 0.7),
    unit quaternions, opacity sigmoid(N(0, 1.5)), base rgb U[0, 1] and the
    higher SH bands N(0, 0.1)."""
    rng = Mulberry32(seed, device)
    means = _np(rng.uniform(3 * components)).reshape(components, 3) * 10.0 - 5.0
    comp = np.minimum((_np(rng.uniform(n)) * components).astype(np.int64), components - 1)
    centers = means[comp] + _np(rng.normal(3 * n, 0.0, 0.2)).reshape(n, 3)
    centers = np.clip(centers, -5.0, 5.0)
    log_scales = _np(rng.normal(3 * n, -4.5, 0.7)).reshape(n, 3)
    quats = _unit_quats(rng, n)
    opacities = _sigmoid(_np(rng.normal(n, 0.0, 1.5)))
    k = (sh_degree + 1) ** 2 - 1
    colors = np.empty((n, 1 + k, 3), dtype=color_dtype)
    colors[:, 0, :] = _np(rng.uniform(3 * n)).reshape(n, 3)
    if k:
        chunk = max(1, (1 << 24) // (3 * k))
        for start in range(0, n, chunk):
            m = min(chunk, n - start)
            colors[start:start + m, 1:, :] = _np(rng.normal(3 * k * m, 0.0, 0.1)).reshape(m, k, 3)
    return dict(centers=centers.astype(np.float32), log_scales=log_scales.astype(np.float32),
                quats=quats.astype(np.float32), opacities=opacities.astype(np.float32),
                colors=colors, sh_degree=sh_degree)


def plain_camera():
    """1280x720, vertical fov 60, at (0, 0.5, 3) looking at the origin, near 0.01, far 1000."""
    return Camera.mono((0.0, 0.5, 3.0), (0.0, 0.0, 0.0), 60.0, 1280, 720)


def scale_camera():
    """1920x1080, vertical fov 50, the same pose."""
    return Camera.mono((0.0, 0.5, 3.0), (0.0, 0.0, 0.0), 50.0, 1920, 1080)


def all_visible_camera():
    """1920x1080, vertical fov 50, at (0, 0.5, 30) looking at the origin: the
    whole [-5, 5]^3 box of the mixture tables lies inside the view's culls."""
    return Camera.mono((0.0, 0.5, 30.0), (0.0, 0.0, 0.0), 50.0, 1920, 1080)


def stereo_camera():
    """Two eyes 64 mm apart, 2064x2208 each, vertical fov 100, the head at (0, 0.5, 3)."""
    return Camera.stereo((0.0, 0.5, 3.0), (0.0, 0.0, 0.0), 100.0, 2064, 2208, baseline=0.064)


def sphere_cameras(views, seed=1, radius=4.0):
    """Cameras uniform on a sphere of `radius` looking at the origin, 1920x1080, fov 50."""
    rng = Mulberry32(seed)
    d = rng.normal(3 * views).reshape(views, 3)
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    return [Camera.mono(tuple(radius * d[v]), (0.0, 0.0, 0.0), 50.0, 1920, 1080) for v in range(views)]


def batched_counts(scenes=16, seed=2, lo=50_000, hi=2_000_000):
    """Scene sizes log-uniform in [lo, hi]."""
    rng = Mulberry32(seed)
    u = rng.uniform(scenes)
    return [int(round(math.exp(math.log(lo) + float(x) * (math.log(hi) - math.log(lo))))) for x in u]
