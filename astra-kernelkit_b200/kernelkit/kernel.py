"""Kernel base class, exceptions and compatibility helpers.

Reference: ``kernelkit/kernel.py``. The reference compiles Jinja2-templated
CUDA with NVRTC at run time and samples CUDA texture objects. Here every
kernel is compiled ahead of time for sm_100a (``libkk.so``) and reads plain
device memory, so ``compile()`` only validates options and loads the
library, and a "texture" is a device array.
"""
from __future__ import annotations

from abc import ABC, abstractmethod
from dataclasses import dataclass

import numpy as np

from . import _arrays
from . import _native


class KernelNotCompiledException(Exception):
    """Raised when a kernel is called before ``compile()``
    (``kernel.py:35-38``)."""


class KernelMemoryUnpreparedException(Exception):
    """Raised when a kernel is called before its parameters are set
    (``kernel.py:41-44``)."""


@dataclass
class Texture:
    """Device-array stand-in for the reference's texture objects.

    ``array`` is a CUDA tensor holding the data in the layout it was given;
    ``layered`` records whether the reference would have made a layered
    texture. The kernels interpolate from it exactly as the texture unit
    would (see ``KK_INTERP_TEX8`` in ``include/kk.h``)."""

    array: object
    texture_type: str = "array"
    layered: bool = False
    _layered: object = None

    @property
    def shape(self):
        return tuple(self.array.shape)

    def layered_texture(self):
        """The 2D-layered texture (one layer per entry of the first axis)
        of a 3D float32/float16 array, made on first use."""
        if self._layered is None:
            self._layered = _native.Layered(*self.array.shape,
                                            _native.dtype_code(self.array))
            self._layered.copy_from(self.array)
        return self._layered


def copy_to_texture(array, texture_type: str = "array",
                    layered: bool = False) -> Texture:
    """Copy ``array`` into a device "texture" (``kernel.py:47-119``).

    The data is copied, as the reference copies into a CUDA array, so later
    changes to ``array`` do not reach the texture."""
    t = _arrays.torch()
    if not (isinstance(array, (np.ndarray, t.Tensor))
            or hasattr(array, "__cuda_array_interface__")):
        raise TypeError(
            f"Expected a NumPy or device array, got {type(array)} instead.")
    dev = _arrays.as_tensor(array)
    if dev.dtype != t.float32:
        raise ValueError(
            f"Array must be of type float32, got {dev.dtype} instead.")
    kind = texture_type.lower()
    if kind in ("array", "array2d"):
        if not dev.is_contiguous():
            raise ValueError("Array must be C-contiguous.")
        if not ((dev.dim() == 2 and kind == "array2d")
                or (dev.dim() == 3 and kind == "array")):
            raise ValueError(f"Type '{texture_type}' is not compatible with "
                             f"array of ndim {dev.dim()}.")
        if layered and dev.dim() != 3:
            raise ValueError("Only 3D arrays can be layered.")
    elif kind == "pitch2d":
        if dev.dim() != 2:
            raise ValueError("pitch2d textures are 2D.")
    else:
        raise ValueError(f"Type `{texture_type}` not understood.")
    return Texture(dev.clone(), kind, layered)


def copy_to_symbol(*args, **kwargs):
    """Not needed: kernel parameters live in device memory owned by the
    kernel objects (see ``set_params``)."""
    raise NotImplementedError(
        "There is no constant memory to copy to; use Kernel.set_params().")


@dataclass(frozen=True, order=True)
class cuda_float4:
    """Four-component vector in CUDA's (x, y, z, w) order
    (``kernel.py:150-163``)."""

    x: object
    y: object
    z: object
    w: object

    def to_list(self):
        return [self.x, self.y, self.z, self.w]

    def __str__(self):
        return str(self.to_list())


class BaseKernel(ABC):
    """Base class of the projection kernels (``kernel.py:166-239``).

    Contract kept from the reference (``docs/user_guide/kernels.rst``):
    ``__call__`` launches work and returns None, performs no device
    allocation and no device-to-host transfer, so it can be captured in a
    CUDA graph; ``compile()`` must precede the first call."""

    def __init__(self):
        self._compiled_options = None

    @abstractmethod
    def __call__(self, *args, **kwargs) -> None:
        pass

    def _compile(self, options: dict):
        _native.load()
        self._compiled_options = dict(options)
        return self

    @property
    def _compiled_template_kwargs(self) -> dict:
        if self._compiled_options is None:
            raise KernelNotCompiledException(
                f"Cannot query the compiled options of kernel "
                f"{self.__class__.__name__} before compilation.")
        return self._compiled_options

    @property
    def is_compiled(self) -> bool:
        return self._compiled_options is not None


__all__ = ["KernelNotCompiledException", "KernelMemoryUnpreparedException",
           "Texture", "copy_to_texture", "copy_to_symbol", "cuda_float4",
           "BaseKernel"]
