"""Seeded ellipsoid phantoms and their exact line integrals.

Synthetic workload generator for the cone-beam path (no public dataset is
involved): ellipsoids with uniform random centres, semi-axes, Euler
rotations and additive densities, voxelised at voxel centres, plus the
exact FP64 line integral of every ray through them (chord length times
density), optionally with Poisson noise and log transform.

Voxelisation runs in NumPy; the line integrals run in PyTorch float64 on
whatever device the caller chooses (GPU for large scans).
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from .geom.proj import angles2mat


@dataclass
class Ellipsoids:
    """Arrays describing ``k`` ellipsoids in world coordinates."""

    centers: np.ndarray     # (k, 3)
    semi_axes: np.ndarray   # (k, 3)
    rotations: np.ndarray   # (k, 3, 3), columns are the ellipsoid axes
    densities: np.ndarray   # (k,)

    def __len__(self):
        return len(self.densities)


def random_ellipsoids(k, center_range, axes_range, seed,
                      density_range=(0.1, 1.0)) -> Ellipsoids:
    """``k`` ellipsoids: centres U[-c, c]^3, semi-axes U(lo, hi), random
    roll/pitch/yaw in [0, 2 pi), densities U(density_range)."""
    rng = np.random.default_rng(seed)
    c = float(center_range)
    centers = rng.uniform(-c, c, size=(k, 3))
    semi = rng.uniform(axes_range[0], axes_range[1], size=(k, 3))
    angles = rng.uniform(0.0, 2 * np.pi, size=(k, 3))
    rots = np.stack([angles2mat(*a) for a in angles])
    dens = rng.uniform(density_range[0], density_range[1], size=k)
    return Ellipsoids(centers, semi, rots, dens)


def voxelize(ell: Ellipsoids, shape, extent_min, voxel_size,
             dtype=np.float32) -> np.ndarray:
    """Sum of densities of the ellipsoids containing each voxel centre.

    Returns ``vol[x, y, z]`` (world axis order, z fastest)."""
    shape = tuple(int(s) for s in shape)
    vs = np.asarray(voxel_size, np.float64).reshape(3)
    lo = np.asarray(extent_min, np.float64).reshape(3)
    axes = [lo[i] + (np.arange(shape[i]) + 0.5) * vs[i] for i in range(3)]
    vol = np.zeros(shape, np.float64)
    for c, a, R, d in zip(ell.centers, ell.semi_axes, ell.rotations,
                          ell.densities):
        # bounding box of the ellipsoid (radius along each world axis)
        ext = np.sqrt(((R * a[None, :]) ** 2).sum(axis=1))
        sl = []
        for i in range(3):
            i0 = max(0, int(np.floor((c[i] - ext[i] - lo[i]) / vs[i])) - 1)
            i1 = min(shape[i], int(np.ceil((c[i] + ext[i] - lo[i]) / vs[i]))
                     + 1)
            sl.append((i0, i1))
        if any(i0 >= i1 for i0, i1 in sl):
            continue
        X = axes[0][sl[0][0]:sl[0][1]][:, None, None] - c[0]
        Y = axes[1][sl[1][0]:sl[1][1]][None, :, None] - c[1]
        Z = axes[2][sl[2][0]:sl[2][1]][None, None, :] - c[2]
        # coordinates in the ellipsoid frame: q = R^T p / a
        q = 0.0
        for j in range(3):
            qj = (R[0, j] * X + R[1, j] * Y + R[2, j] * Z) / a[j]
            q = q + qj * qj
        vol[sl[0][0]:sl[0][1], sl[1][0]:sl[1][1], sl[2][0]:sl[2][1]] += (
            d * (q <= 1.0))
    return vol.astype(dtype)


def voxelize_torch(ell: Ellipsoids, shape, extent_min, voxel_size,
                   device="cuda", dtype=None):
    """``voxelize`` evaluated with PyTorch on ``device`` (float64 geometry,
    same inclusion rule), for large volumes. Returns a float32 tensor
    ``vol[x, y, z]``."""
    import torch

    dtype = dtype or torch.float32
    shape = tuple(int(s) for s in shape)
    vs = np.asarray(voxel_size, np.float64).reshape(3)
    lo = np.asarray(extent_min, np.float64).reshape(3)
    vol = torch.zeros(shape, dtype=torch.float32, device=device)
    for c, a, R, d in zip(ell.centers, ell.semi_axes, ell.rotations,
                          ell.densities):
        ext = np.sqrt(((R * a[None, :]) ** 2).sum(axis=1))
        sl = []
        for i in range(3):
            i0 = max(0, int(np.floor((c[i] - ext[i] - lo[i]) / vs[i])) - 1)
            i1 = min(shape[i], int(np.ceil((c[i] + ext[i] - lo[i]) / vs[i]))
                     + 1)
            sl.append((i0, i1))
        if any(i0 >= i1 for i0, i1 in sl):
            continue
        ax = [torch.arange(i0, i1, dtype=torch.float64, device=device)
              for (i0, i1) in sl]
        X = (lo[0] + (ax[0] + 0.5) * vs[0] - c[0])[:, None, None]
        Y = (lo[1] + (ax[1] + 0.5) * vs[1] - c[1])[None, :, None]
        Z = (lo[2] + (ax[2] + 0.5) * vs[2] - c[2])[None, None, :]
        q = 0.0
        for j in range(3):
            qj = (R[0, j] * X + R[1, j] * Y + R[2, j] * Z) / a[j]
            q = q + qj * qj
        vol[sl[0][0]:sl[0][1], sl[1][0]:sl[1][1], sl[2][0]:sl[2][1]] += (
            float(d) * (q <= 1.0)).float()
    return vol.to(dtype)


def line_integrals(ell: Ellipsoids, sources, pixels, device="cpu",
                   chunk=1 << 22):
    """Exact FP64 line integrals through the ellipsoids.

    ``sources`` (n, 3) and ``pixels`` (n, rows, cols, 3) in world
    coordinates; each ray runs from its source through the pixel and
    beyond (the whole line). Returns a float64 torch tensor (n, rows, cols)
    on ``device``.
    """
    import torch

    dev = torch.device(device)
    src = torch.as_tensor(np.asarray(sources, np.float64), device=dev)
    pix = torch.as_tensor(np.asarray(pixels, np.float64), device=dev)
    n, rows, cols, _ = pix.shape
    out = torch.zeros((n, rows, cols), dtype=torch.float64, device=dev)
    dirs = pix - src[:, None, None, :]
    dirs = dirs / torch.linalg.norm(dirs, dim=-1, keepdim=True)
    flat_dir = dirs.reshape(-1, 3)
    flat_src = src[:, None, None, :].expand(n, rows, cols, 3).reshape(-1, 3)
    flat_out = out.reshape(-1)
    for e in range(len(ell)):
        c = torch.as_tensor(ell.centers[e], device=dev)
        a = torch.as_tensor(ell.semi_axes[e], device=dev)
        Rt = torch.as_tensor(ell.rotations[e].T.copy(), device=dev)
        for s in range(0, flat_dir.shape[0], chunk):
            q0 = ((flat_src[s:s + chunk] - c) @ Rt.T) / a
            w = (flat_dir[s:s + chunk] @ Rt.T) / a
            ww = (w * w).sum(-1)
            qw = (q0 * w).sum(-1)
            qq = (q0 * q0).sum(-1) - 1.0
            disc = qw * qw - ww * qq
            chord = 2.0 * torch.sqrt(torch.clamp(disc, min=0.0)) / ww
            flat_out[s:s + chunk] += float(ell.densities[e]) * chord
    return out


def pixel_centres(geometries):
    """World positions of every detector pixel centre, (n, rows, cols, 3),
    and the sources (n, 3), from a list of ``ProjectionGeometry``."""
    srcs, pixs = [], []
    for g in geometries:
        det = g.detector
        u = np.asarray(g.u, np.float64) * det.pixel_width
        v = np.asarray(g.v, np.float64) * det.pixel_height
        corner = (np.asarray(g.detector_position, np.float64)
                  - np.asarray(g.v, np.float64) * det.height / 2
                  - np.asarray(g.u, np.float64) * det.width / 2)
        r = np.arange(det.rows)[:, None, None] + 0.5
        c = np.arange(det.cols)[None, :, None] + 0.5
        pixs.append(corner + c * u + r * v)
        srcs.append(np.asarray(g.source_position, np.float64))
    return np.stack(srcs), np.stack(pixs)


def noisy_projections(clean, photons=1e4, mu_max=3.0, seed=0):
    """Poisson noise at ``photons`` per pixel on ``exp(-k p)`` and the
    log transform back, with ``k = mu_max / max(p)`` so the most
    attenuating ray keeps ``exp(-mu_max)`` of the beam. Returns the noisy
    line integrals in the units of ``clean`` (float32 NumPy)."""
    import torch

    p = torch.as_tensor(clean, dtype=torch.float64)
    k = mu_max / max(float(p.max()), 1e-12)
    gen = torch.Generator(device=p.device).manual_seed(int(seed))
    counts = torch.poisson(photons * torch.exp(-k * p), generator=gen)
    counts = torch.clamp(counts, min=1.0)
    return (-torch.log(counts / photons) / k).float().cpu().numpy()


__all__ = ["Ellipsoids", "random_ellipsoids", "voxelize", "line_integrals",
           "pixel_centres", "noisy_projections"]
