"""Projectors: geometry and memory state around one kernel.

Mirrors ``kernelkit/projector.py`` of the reference: the same classes,
properties, setter ordering (kernel parameters are pushed as soon as both
geometries are known), ``__call__(additive)`` semantics and exceptions.
Differences: the forward projector reads the volume in place (no texture
copy); the backprojector copies projections into a layered texture only
for the CUDA-array texture types, as the reference does; non-additive
calls overwrite instead of zero-filling first; the caller's geometry
objects are never normalised in place.
"""
from __future__ import annotations

from abc import ABC, abstractmethod
from typing import Any

import numpy as np

from . import _arrays
from .geom.proj import ProjectionGeometry, ProjectionGeometrySequence
from .geom.vol import VolumeGeometry
from .kernel import BaseKernel
from .kernels.cone_bp import VoxelDrivenConeBP
from .kernels.cone_fp import RayDrivenConeFP


class ProjectionGeometryNotSetError(AttributeError):
    """Raised when the projection geometry is not set in the projector."""


class VolumeGeometryNotSetError(AttributeError):
    """Raised when the volume geometry is not set in the projector."""


class VolumeNotSetError(AttributeError):
    """Raised when the volume is not set in the projector."""


class ProjectionsNotSetError(AttributeError):
    """Raised when the projections are not set in the projector."""


class BaseProjector(ABC):
    """Interface of projectors (``projector.py:41-123``)."""

    @property
    @abstractmethod
    def projection_axes(self) -> tuple: ...

    @property
    @abstractmethod
    def volume_axes(self) -> tuple: ...

    @property
    @abstractmethod
    def projection_geometry(self): ...

    @property
    @abstractmethod
    def volume_geometry(self): ...

    @property
    @abstractmethod
    def volume(self): ...

    @property
    @abstractmethod
    def projections(self): ...

    @abstractmethod
    def __call__(self, additive: bool = False): ...


class Projector(BaseProjector, ABC):
    """Holds the geometries and pushes kernel parameters when both are set
    (``projector.py:126-215``)."""

    def __init__(self, kernel: BaseKernel):
        self._K = kernel

    @property
    def kernel(self) -> BaseKernel:
        return self._K

    @property
    def projection_axes(self):
        return self._K.projection_axes

    @property
    def volume_axes(self):
        return self._K.volume_axes

    def _push_params(self):
        if hasattr(self, "_proj_geom_seq") and hasattr(self, "_vol_geom"):
            self._params = self._K.geoms2params(self._proj_geom_seq,
                                                self._vol_geom)
            self._K.set_params(self._params)

    @property
    def projection_geometry(self):
        try:
            return self._proj_geom
        except AttributeError:
            raise ProjectionGeometryNotSetError(
                f"Projection geometry not set in "
                f"'{self.__class__.__name__}'. Please set the projection "
                "geometry using `projection_geometry`.")

    @projection_geometry.setter
    def projection_geometry(self, value):
        if isinstance(value, ProjectionGeometrySequence):
            seq = value
        else:
            for p in value:
                if p.beam != value[0].beam:
                    raise NotImplementedError(
                        "All geometries in the list must have the same beam "
                        "type.")
            seq = ProjectionGeometrySequence.fromList(value)
        if len(set(seq.detector.rows.tolist())) != 1 or len(
                set(seq.detector.cols.tolist())) != 1:
            raise NotImplementedError(
                "All projections must share one detector shape.")
        self._proj_geom = value
        self._proj_geom_seq = seq
        self._push_params()

    @projection_geometry.deleter
    def projection_geometry(self):
        del self._proj_geom
        del self._proj_geom_seq

    @property
    def volume_geometry(self) -> VolumeGeometry:
        try:
            return self._vol_geom
        except AttributeError:
            raise VolumeGeometryNotSetError(
                f"Volume geometry not set in '{self.__class__.__name__}'. "
                "Please set the volume geometry using `volume_geometry`.")

    @volume_geometry.setter
    def volume_geometry(self, value: VolumeGeometry):
        self._vol_geom = value
        self._push_params()

    @volume_geometry.deleter
    def volume_geometry(self):
        del self._vol_geom

    @property
    def _detector_shape(self):
        seq = self._proj_geom_seq
        return len(seq), int(seq.detector.rows[0]), int(seq.detector.cols[0])

    def _expected_projection_shape(self):
        shp = self._detector_shape
        return tuple(shp[i] for i in self.projection_axes)

    def _expected_volume_shape(self):
        return tuple(int(self._vol_geom.shape[i]) for i in self.volume_axes)


class ForwardProjector(Projector):
    """Cone-beam forward projector (``projector.py:218-346``)."""

    def __init__(self, kernel: RayDrivenConeFP = None, volume_axes=(0, 1, 2),
                 projection_axes=(0, 1, 2), **kernel_kwargs):
        if kernel is not None and kernel_kwargs:
            raise ValueError(
                "If `kernel` is given, other keyword arguments cannot be "
                f"passed to the kernel constructor. You passed "
                f"`{kernel_kwargs}`.")
        K = kernel or RayDrivenConeFP(volume_axes=volume_axes,
                                      projection_axes=projection_axes,
                                      **kernel_kwargs)
        super().__init__(K)
        if not self._K.is_compiled:
            self._K.compile()

    @property
    def volume(self):
        try:
            return self._vol_ref
        except AttributeError:
            raise VolumeNotSetError(
                "Volume not set. Use the `volume` setter before calling the "
                "projector.")

    @volume.setter
    def volume(self, value):
        """Set the volume to project (a device array laid out by
        ``volume_axes``; NumPy input is copied to the device)."""
        if not (_arrays.is_device_array(value)
                or isinstance(value, np.ndarray)):
            raise TypeError("Volume must be a device array.")
        self._vol_ref = _arrays.as_tensor(value)

    @volume.deleter
    def volume(self):
        del self._vol_ref

    @property
    def projections(self):
        try:
            return self._projs
        except AttributeError:
            raise ProjectionsNotSetError(
                "Projections not set. Use the `projections` setter before "
                "calling the projector.")

    @projections.setter
    def projections(self, value):
        """Set the output projections: a device array laid out by
        ``projection_axes`` or a list of 2D device arrays (one per angle,
        each in its own memory)."""
        if isinstance(value, list):
            ptrs = [_arrays.as_tensor(p).data_ptr() for p in value]
            if len(ptrs) != len(set(ptrs)):
                raise ValueError(
                    "All projection files need to reside in own memory.")
            self._projs = value
            self._proj_list = [_arrays.as_tensor(p) for p in value]
        elif _arrays.is_device_array(value):
            self._projs = value
            self._proj_list = None
        else:
            raise TypeError("Projections must be a device array or `list`.")

    @projections.deleter
    def projections(self):
        del self._projs

    def __call__(self, additive: bool = False):
        """Project the volume into the projections (overwriting them unless
        ``additive``)."""
        target = self._proj_list if self._proj_list is not None else \
            _arrays.as_tensor(self.projections)
        self._K(self.volume, self._proj_geom_seq, self.volume_geometry,
                target, additive=additive)


class BackProjector(Projector):
    """Cone-beam backprojector (``projector.py:349-588``)."""

    TEXTURE_TYPES = "array", "layered", "array2d", "pitch2d"

    def __init__(self, kernel: VoxelDrivenConeBP = None,
                 texture_type: str = "layered", **kernel_kwargs):
        if kernel is not None and kernel_kwargs:
            raise ValueError(
                "If `kernel` is given, other keyword arguments cannot be "
                f"passed to the kernel constructor. You passed "
                f"`{kernel_kwargs}`.")
        kernel_kwargs.pop("beam", None)
        K = kernel or VoxelDrivenConeBP(**kernel_kwargs)
        super().__init__(K)
        self._texture_type = texture_type.lower()
        if self._texture_type not in self.TEXTURE_TYPES:
            raise ValueError("`TEXTURE_TYPE` not supported. Please choose "
                             f"one of the following: {self.TEXTURE_TYPES}.")
        kinds = {"pitch2d": K.InterpolationMethod.Tex2D,
                 "array2d": K.InterpolationMethod.Tex2D,
                 "array": K.InterpolationMethod.Tex3D,
                 "layered": K.InterpolationMethod.Tex2DLayered}
        if not self._K.is_compiled:
            self._K.compile(texture=kinds[self._texture_type])

    @property
    def volume(self):
        try:
            return self._vol
        except AttributeError:
            raise VolumeNotSetError(
                "No volume set. Please set the volume before calling the "
                "backprojector.")

    @volume.setter
    def volume(self, value):
        if hasattr(self, "_vol_geom"):
            expected = self._expected_volume_shape()
            if tuple(value.shape) != expected:
                raise ValueError(
                    f"Volume shape {tuple(value.shape)} does not match volume"
                    f" geometry {tuple(int(s) for s in self._vol_geom.shape)}"
                    f" with axes {self._K.volume_axes}.")
        self._vol = value

    @volume.deleter
    def volume(self):
        del self._vol

    @property
    def projections(self):
        try:
            return self._projs
        except AttributeError:
            raise ProjectionsNotSetError("No projections set in the "
                                         "projector.")

    @projections.setter
    def projections(self, value: Any):
        """Set the projections to backproject: a device array laid out by
        ``projection_axes`` (NumPy input is copied to the device) or a list
        of 2D arrays."""
        if not (isinstance(value, (list, np.ndarray))
                or _arrays.is_device_array(value)):
            raise TypeError("Projections must be a `ndarray` or `list`.")
        if hasattr(self, "_proj_geom_seq"):
            expected = self._expected_projection_shape()
            if isinstance(value, list):
                if len(value) != expected[0]:
                    raise ValueError(
                        f"Projections shape {len(value)} does not match "
                        f"projection geometry {self._detector_shape} with "
                        f"axes {self._K.projection_axes}.")
                if tuple(value[0].shape) != expected[1:]:
                    raise ValueError(
                        f"Projections shape {tuple(value[0].shape)} does not"
                        f" match projection geometry {self._detector_shape} "
                        f"with axes {self._K.projection_axes}.")
            elif tuple(value.shape) != expected:
                raise ValueError(
                    f"Projections shape {tuple(value.shape)} does not match "
                    f"projection geometry {self._detector_shape} with axes "
                    f"{self._K.projection_axes}.")
        if isinstance(value, list):
            if self._K.projection_axes[0] != 0:
                raise ValueError("Can only use a list of projections when "
                                 "projection axis is 0.")
            self._projs = [_arrays.as_tensor(p) for p in value]
            self._layered = None
        else:
            if (self._texture_type == "layered"
                    and self._K.projection_axes[0] != 0):
                raise ValueError("Can only use layered texture when the "
                                 "first projection axis is 0.")
            self._projs = _arrays.as_tensor(value)
            self._layered = self._fill_texture(self._projs)

    def _fill_texture(self, projs):
        """For the texture types backed by a CUDA array ('layered',
        'array'), copy the projections into the projector's layered
        texture (made once per shape), as the reference copies them into
        its CUDA array (projector.py:529-542)."""
        t = _arrays.torch()
        K = self._K
        if (self._texture_type not in ("layered", "array")
                or K.projection_axes[0] != 0
                or K.interpolation.lower() not in ("texture", "tex8")
                or projs.dim() != 3
                or projs.dtype != t.float32
                or projs.shape[0] > 2048):
            return None
        from . import _native

        lay = getattr(self, "_layered_tex", None)
        code = _native.dtype_code(projs)
        if lay is None or lay.shape != tuple(projs.shape) or lay.dtype != code:
            lay = _native.Layered(*projs.shape, code)
            self._layered_tex = lay
        lay.copy_from(projs.contiguous())
        return lay

    @projections.deleter
    def projections(self):
        try:
            del self._projs
        except AttributeError:
            pass

    def __call__(self, additive: bool = False):
        """Backproject into the volume (overwriting it unless
        ``additive``)."""
        src = getattr(self, "_layered", None) or self.projections
        self._K(src, self.volume, self.volume_geometry, additive=additive)


__all__ = ["ProjectionGeometryNotSetError", "VolumeGeometryNotSetError",
           "VolumeNotSetError", "ProjectionsNotSetError", "BaseProjector",
           "Projector", "ForwardProjector", "BackProjector"]
