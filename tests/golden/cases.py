"""Scan/volume geometry recipes shared by the golden-vector generators and
the tests. Plain data only: each case names a base projection geometry,
per-angle (roll, pitch, yaw) rotations applied with ``rotate`` and the
keyword arguments of the volume geometry, so the reference's code and this
repository's code can each build the same scan from it."""
from __future__ import annotations

import math

import numpy as np


def _circle(n, extra=(0.0, 0.0)):
    """n yaw angles uniform over [0, 2 pi), optional fixed roll/pitch."""
    return [(extra[0], extra[1], 2 * math.pi * k / n) for k in range(n)]


CASES = {
    # small, non-square detector so row/column mix-ups show
    "small": dict(
        source=(-60.0, 0.0, 0.0), detector=(60.0, 0.0, 0.0),
        rows=40, cols=48, pixel_height=1.5, pixel_width=1.5,
        rotations=_circle(24),
        volume=dict(resolve=dict(shape=32, voxel_size=1.0)),
    ),
    # tilted detector plane, shifted volume with 0.5 voxels
    "tilted": dict(
        source=(-50.0, 3.0, -2.0), detector=(45.0, -1.0, 1.5),
        rows=30, cols=36, pixel_height=1.1, pixel_width=0.9,
        u=(0.0, math.cos(0.2), math.sin(0.2)),
        v=(0.0, -math.sin(0.2), math.cos(0.2)),
        rotations=[(0.05 * k, 0.1, 2 * math.pi * k / 16) for k in range(16)],
        volume=dict(resolve=dict(shape=(24, 28, 20), voxel_size=0.5,
                                 extent_min=(-5.0, -7.0, -4.5),
                                 extent_max=(7.0, 7.0, 5.5))),
    ),
    # pitch sweep: x-, y- and z-dominant rays (all three ray directions)
    "alldirs": dict(
        source=(-40.0, 0.0, 0.0), detector=(40.0, 0.0, 0.0),
        rows=26, cols=30, pixel_height=1.2, pixel_width=1.2,
        rotations=[(0.0, -1.3 + 2.6 * k / 17, 0.9 * k) for k in range(18)],
        volume=dict(resolve=dict(shape=(20, 24, 28), voxel_size=1.0)),
    ),
    # rotated volume (VolumeGeometry.rotation), isotropic
    "volrot": dict(
        source=(-45.0, 0.0, 0.0), detector=(35.0, 0.0, 0.0),
        rows=22, cols=26, pixel_height=1.0, pixel_width=1.0,
        rotations=_circle(12),
        volume=dict(explicit=dict(shape=(18, 20, 16), voxel_size=(1.0,) * 3,
                                  extent_min=(-9.0, -10.0, -8.0),
                                  extent_max=(9.0, 10.0, 8.0),
                                  rotation=(0.1, -0.2, 0.3))),
    ),
    # anisotropic voxels (forward projector only; the reference
    # backprojector refuses them)
    "aniso": dict(
        source=(-40.0, 0.0, 0.0), detector=(40.0, 0.0, 0.0),
        rows=24, cols=32, pixel_height=1.0, pixel_width=1.0,
        rotations=_circle(10),
        volume=dict(explicit=dict(shape=(16, 16, 16),
                                  voxel_size=(1.0, 0.5, 1.5),
                                  extent_min=(-8.0, -4.0, -12.0),
                                  extent_max=(8.0, 4.0, 12.0))),
        bp=False,
    ),
    # 64^3, 96 angles, 96^2 detector, SOD 200, SDD 400, pitch 1.5
    "config1": dict(
        source=(-200.0, 0.0, 0.0), detector=(200.0, 0.0, 0.0),
        rows=96, cols=96, pixel_height=1.5, pixel_width=1.5,
        rotations=_circle(96),
        volume=dict(resolve=dict(shape=64, voxel_size=1.0)),
    ),
    # 256^3, 360 angles, 384^2, SOD 800, SDD 1600, pitch 1.3
    "config2": dict(
        source=(-800.0, 0.0, 0.0), detector=(800.0, 0.0, 0.0),
        rows=384, cols=384, pixel_height=1.3, pixel_width=1.3,
        rotations=_circle(360),
        volume=dict(resolve=dict(shape=256, voxel_size=1.0)),
    ),
    # headline: 512^3, 720 angles, 768^2, SOD 1600, SDD 3200, pitch 1.3
    "headline": dict(
        source=(-1600.0, 0.0, 0.0), detector=(1600.0, 0.0, 0.0),
        rows=768, cols=768, pixel_height=1.3, pixel_width=1.3,
        rotations=_circle(720),
        volume=dict(resolve=dict(shape=512, voxel_size=1.0)),
    ),
    # 1024^3, 1440 angles, 1536^2, SOD 3000, SDD 6000, pitch 1.0
    "config5": dict(
        source=(-3000.0, 0.0, 0.0), detector=(3000.0, 0.0, 0.0),
        rows=1536, cols=1536, pixel_height=1.0, pixel_width=1.0,
        rotations=_circle(1440),
        volume=dict(resolve=dict(shape=1024, voxel_size=1.0)),
    ),
}

#: cases whose kernels are run on the GPU for golden outputs
GPU_CASES = ("small", "tilted", "alldirs", "volrot", "aniso", "config1")

#: resolve_volume_geometry argument sets (reference: geom/__init__.py:8-254)
RESOLVE_CASES = [
    dict(shape=64, voxel_size=1.0),
    dict(shape=(100, 110, 120), extent_min=(-0.2, None, None),
         extent_max=(0.2, None, None)),
    dict(shape=(2, 2, 2), extent_min=(-0.5, None, None),
         extent_max=(0.5, None, None)),
    dict(shape=(9, 9, 9), extent_min=(-0.5,) * 3, extent_max=(0.5,) * 3),
    dict(shape=(100, 100, 1), voxel_size=0.05),
    dict(shape=(10, 10, 10), voxel_size=0.02),
    dict(shape=(16, 16, 16), voxel_size=(1.0, 0.5, 1.5)),
    dict(extent_min=(-3.0, -3.0, -2.0), extent_max=(3.0, 3.0, 2.0),
         voxel_size=0.25),
    dict(shape=(60, 60, 60), voxel_size=0.5),
    dict(shape=(None, None, 40), extent_min=(-10.0, -10.0, -5.0),
         extent_max=(10.0, 10.0, 5.0)),
]


def phantom_for(case: str, shape):
    """Seeded ellipsoid parameters for a golden case (semi-axes scale with
    the volume)."""
    n = float(max(shape))
    seed = 1000 + sorted(CASES).index(case)
    k = 10
    return dict(k=k, center_range=0.35 * n, axes_range=(0.06 * n, 0.3 * n),
                seed=seed)


def sinogram_seed(case: str) -> int:
    return 2000 + sorted(CASES).index(case)


def random_sinogram(case: str, n, rows, cols):
    rng = np.random.default_rng(sinogram_seed(case))
    return rng.uniform(0.0, 1.0, size=(n, rows, cols)).astype(np.float32)


def probe_coordinates():
    """Texture coordinates for the filtering probe: a 1/2048 grid over
    eight texels (contains every 1/256 step and every half step), the
    float32 neighbours of the half steps, and a sweep across both borders.
    Returns float32 arrays (grid_and_ties, border_sweep)."""
    grid = 8.0 + np.arange(8 * 2048) / 2048.0
    half = 8.0 + (np.arange(8 * 256) + 0.5) / 256.0
    h32 = half.astype(np.float32)
    ties = np.concatenate([np.nextafter(h32, np.float32(-np.inf)),
                           np.nextafter(h32, np.float32(np.inf))])
    fine = np.concatenate([grid.astype(np.float32), ties])
    border = (-3.0 + np.arange(70 * 64) / 64.0).astype(np.float32)
    return fine, border


def probe_random(seed=5):
    """Random texel values and coordinates for the value-level probe."""
    rng = np.random.default_rng(seed)
    tex = rng.uniform(-10, 10, size=(1, 64, 64)).astype(np.float32)
    xs = rng.uniform(-1, 65, 20000).astype(np.float32)
    ys = rng.uniform(-1, 65, 20000).astype(np.float32)
    return tex, xs, ys


def probe_random3d(seed=6):
    """Random 16^3 texels and, per pair of texture axes, random coordinates
    with the third axis at a texel centre (as the forward projector samples
    a 3D array): keys 'uv', 'uw', 'vw' -> (xs, ys, zs)."""
    rng = np.random.default_rng(seed)
    tex = rng.uniform(-10, 10, size=(16, 16, 16)).astype(np.float32)
    out = {}
    for pair in ("uv", "uw", "vw"):
        c = [rng.uniform(-1, 17, 20000).astype(np.float32) for _ in range(3)]
        fixed = "uvw".index(next(a for a in "uvw" if a not in pair))
        c[fixed] = (rng.integers(0, 16, 20000) + 0.5).astype(np.float32)
        out[pair] = tuple(c)
    return tex, out
