"""Reconstruction-volume geometry (``kernelkit/geom/vol.py`` of the
reference). Shapes and extents are given in world (x, y, z) order."""
from __future__ import annotations

import numpy as np


def _voxel_size(shape, extent_min, extent_max):
    """Per-axis voxel size from extents (``geom/vol.py:4-22``)."""
    return tuple((extent_max[i] - extent_min[i]) / shape[i] for i in range(3))


class VolumeGeometry:
    """Shape, voxel size, extents and rotation of one volume.

    Values are stored as tuples of NumPy scalars (int32 shape, float32
    lengths), exactly as the reference does (``geom/vol.py:25-62``); the
    kernels receive these float32 values.
    """

    def __init__(self, shape, voxel_size, extent_min, extent_max,
                 rotation=(0.0, 0.0, 0.0)):
        self.shape = tuple(np.array(shape, dtype=np.int32))
        self.voxel_size = tuple(np.array(voxel_size, dtype=np.float32))
        self.extent_min = tuple(np.array(extent_min, dtype=np.float32))
        self.extent_max = tuple(np.array(extent_max, dtype=np.float32))
        self.rotation = tuple(np.array(rotation, dtype=np.float32))

    def has_isotropic_voxels(self, atol: float = 1e-8) -> bool:
        return bool(np.allclose(self.voxel_size, self.voxel_size[0],
                                atol=atol))

    def voxel_volume(self) -> float:
        """Volume of one voxel, from the extents (``geom/vol.py:79-89``)."""
        s = _voxel_size(self.shape, self.extent_min, self.extent_max)
        return float(s[0] * s[1] * s[2])

    def check_consistency(self) -> bool:
        """Raise ``ValueError`` unless shape, voxel size and extents agree
        (``geom/vol.py:91-147``)."""
        n = len(self.shape)
        if n not in (2, 3):
            raise ValueError(f"Shape must have 2 or 3 dimensions, got {n}.")
        for name, val in (("Voxel size", self.voxel_size),
                          ("Extent min", self.extent_min),
                          ("Extent max", self.extent_max)):
            if len(val) != n:
                raise ValueError(f"{name} must match the shape dimensions, "
                                 f"got {len(val)} dimensions.")
        if len(self.rotation) != 3:
            raise ValueError("Rotation must have 3 dimensions, "
                             f"got {len(self.rotation)} dimensions.")
        for lo, hi in zip(self.extent_min, self.extent_max):
            if lo >= hi:
                raise ValueError(f"Extent min {lo} must be less than "
                                 f"extent max {hi}.")
        for n_vox, size in zip(self.shape, self.voxel_size):
            if n_vox <= 0:
                raise ValueError(f"Shape dimension {n_vox} must be positive.")
            if size <= 0:
                raise ValueError(f"Voxel size {size} must be positive.")
        for n_vox, size, lo, hi in zip(self.shape, self.voxel_size,
                                       self.extent_min, self.extent_max):
            if not np.isclose(n_vox * size, hi - lo):
                raise ValueError(f"Expected extent {n_vox * size} does not "
                                 f"match actual extent {hi - lo} "
                                 "for dimension.")
        return True

    def __repr__(self):
        return (f"VolumeGeometry(shape={tuple(int(s) for s in self.shape)}, "
                f"voxel_size={tuple(float(s) for s in self.voxel_size)}, "
                f"extent_min={tuple(float(s) for s in self.extent_min)}, "
                f"extent_max={tuple(float(s) for s in self.extent_max)}, "
                f"rotation={tuple(float(s) for s in self.rotation)})")


__all__ = ["VolumeGeometry"]
