"""Geometry helpers: volume auto-resolution and normalisation of scan
geometries into the unit-voxel frame the kernels work in.

Reference: ``kernelkit/geom/__init__.py``.
"""
from __future__ import annotations

import copy
import warnings
from typing import Sequence

import numpy as np

from .proj import *  # noqa: F401,F403
from .proj import ProjectionGeometry, rotate_, scale_, shift_
from .vol import VolumeGeometry


def _as_triple(arg):
    if arg is None or np.isscalar(arg):
        return [arg] * 3
    return list(arg)


def resolve_volume_geometry(shape=None, extent_min=None, extent_max=None,
                            voxel_size=None, projection_geometry=None,
                            verbose=False) -> VolumeGeometry:
    """Complete a ``VolumeGeometry`` from partial information.

    Each axis obeys ``n * voxel_size == extent_max - extent_min``; any two
    of the three determine the third. Unresolved axes borrow the smallest
    known voxel size (isotropic voxels), x/y share a voxel count, and as a
    last resort the extent suggested by ``projection_geometry`` is used.
    Same procedure and error messages as ``geom/__init__.py:8-254``.
    """
    shape = _as_triple(shape)
    lo = _as_triple(extent_min)
    hi = _as_triple(extent_max)
    size = _as_triple(voxel_size)
    done = [False] * 3

    def solve(n, xmin, xmax, sz, dim):
        ok = False
        if n is not None:
            if xmin is not None and xmax is not None:
                ext = xmax - xmin
                if sz is not None:
                    if not np.allclose(n * sz, ext):
                        raise ValueError(
                            f"The {dim}-th dimension contains conflicting "
                            f"parameter values: nr_voxels={n}, voxel_size="
                            f"{sz}, extent_min={xmin}, extent_max={xmax}. It "
                            "must hold that nr_voxels * voxel_size = "
                            "extent_max - extent_min.")
                else:
                    sz = ext / n
                ok = True
            elif xmin is None and xmax is None:
                if sz is not None:
                    xmin, xmax = -n * sz / 2, n * sz / 2
                    ok = True
            else:
                raise ValueError(
                    f"Volume extent in dim {dim} must be given with both max"
                    " and min value, or inferred automatically.")
        else:
            if xmin is not None and xmax is not None:
                if sz is not None:
                    cnt = (xmax - xmin) / sz
                    if not np.allclose(cnt, np.round(cnt)):
                        raise ValueError(
                            f"Number of voxels in dim {dim} was inferred to "
                            f"be {cnt}, which is not a rounded number. To "
                            "have isotropic voxels, please give in larger "
                            "volume size, or leave the volume extent out in "
                            f"dim {dim} to have it inferred automatically.")
                    n = int(np.round(cnt))
                    ok = True
            elif not (xmin is None and xmax is None):
                raise ValueError(
                    f"Volume extent in dim {dim} must be given with both max"
                    " and min value, or inferred automatically.")
        if ok:
            if verbose:
                print(f"Solved:\n - shape: \t\t {n}\n - extent min: \t {xmin}"
                      f"\n - extent max: \t {xmax}\n - voxel size: \t {sz}")
            return n, xmin, xmax, sz
        return None

    def resolve(dims, ext_lo, ext_hi):
        for d in dims:
            if done[d]:
                continue
            if verbose:
                print(f"Attempting dimension {d}...")
            res = solve(shape[d], ext_lo[d], ext_hi[d], size[d], d)
            if res is not None:
                shape[d], lo[d], hi[d], size[d] = res
                done[d] = True

    # 1. any directly solvable axis fixes a voxel size
    resolve(range(3), lo, hi)

    # 2. otherwise fall back to the scan geometry's suggested extent
    if not any(done):
        if projection_geometry is None:
            raise ValueError(
                "Not enough information is provided to infer a voxel size, "
                "number of voxels and volume extent of at least a single "
                "dimension. Consider passing a geometry for automatic "
                "inference.")
        s_lo, s_hi = suggest_volume_extent(projection_geometry[0],
                                           (0.0, 0.0, 0))
        for d in range(3):
            if done[d]:
                continue
            try_lo, try_hi = np.copy(lo), np.copy(hi)
            try_lo[d], try_hi[d] = s_lo[d], s_hi[d]
            resolve([d], try_lo, try_hi)
            if done[d]:
                break

    # 3. propagate the smallest known voxel size (isotropy) and retry
    size = np.array(size)
    size[size == None] = np.min(size[np.where(size != None)])  # noqa: E711
    resolve(range(3), lo, hi)

    if done[0] and not done[1]:
        shape[1] = shape[0]
    if done[1] and not done[0]:
        shape[0] = shape[1]
    resolve(range(2), lo, hi)

    # 4. axes with only a voxel size: take the suggested extent, rounded up
    #    to whole voxels
    if not all(done) and projection_geometry is not None:
        s_lo, s_hi = suggest_volume_extent(projection_geometry[0],
                                           (0.0, 0.0, 0))
        for d in range(3):
            if done[d]:
                continue
            try_lo, try_hi = np.copy(lo), np.copy(hi)
            need = (s_hi[d] - s_lo[d]) / size[d]
            if np.allclose(np.round(need), need):
                need = np.round(need)
            else:
                need = np.ceil(need)
            try_lo[d] = -need / 2 * size[d]
            try_hi[d] = need / 2 * size[d]
            resolve([d], try_lo, try_hi)

    if verbose:
        print(f"The final deduced volume parameters are: \n - shape: \t\t "
              f"{shape}\n - extent min: \t {lo}\n - extent max: \t {hi}\n"
              f" - voxel size: \t {size}")
    if not all(done):
        raise RuntimeError(
            "Could not resolve the volume geometry. The following dimensions "
            f"cannot be inferred: {np.where(np.logical_not(done))[0]}. "
            "Provide two of the three unknowns and/or one of the projection "
            "geometries to deduce the dimensions.")
    return VolumeGeometry(shape=shape, voxel_size=size, extent_min=lo,
                          extent_max=hi)


def suggest_volume_extent(geometry: ProjectionGeometry,
                          object_position: Sequence = (0.0, 0.0, 0.0)):
    """Extent of the field of view seen by one projection, scaled back from
    the detector by the magnification SOD/SDD (``geom/__init__.py:257-302``).
    """
    g = copy.deepcopy(geometry)
    shift_(g, -np.array(object_position))
    src = g.source_position
    ray = g.detector_position - g.source_position
    if not np.linalg.matrix_rank([src, ray]) == 1:
        warnings.warn("Volume extents may not be suggested correctly when "
                      " the geometry does not project through the origin.")
    sod = np.linalg.norm(src)
    sdd = np.linalg.norm(ray)
    w = sod * g.detector.width / sdd
    h = sod * g.detector.height / sdd
    return (np.array([-w / 2, -w / 2, -h / 2]),
            np.array([w / 2, w / 2, h / 2]))


def normalize_(geometries, volume_geometry: VolumeGeometry) -> None:
    """Move a geometry sequence into the kernel frame, in place: the volume
    centre becomes the origin, a voxel becomes a unit cube and the volume
    rotation is undone (``geom/__init__.py:305-330``; same float32 order)."""
    center = -(np.asarray(volume_geometry.extent_min)
               + np.asarray(volume_geometry.extent_max)) / 2
    shift_(geometries, center)
    scale_(geometries, np.asarray(volume_geometry.voxel_size))
    rotate_(geometries, *volume_geometry.rotation)


__all__ = ["resolve_volume_geometry", "suggest_volume_extent", "normalize_",
           "VolumeGeometry"]
