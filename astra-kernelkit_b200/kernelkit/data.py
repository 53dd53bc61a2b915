"""Pitched-array helpers (``kernelkit/data.py`` of the reference).

Rows are padded to a multiple of 32 bytes and a view of the original width
is returned; the projectors accept such views (and lists of them) directly
through their strides. Works on NumPy arrays and torch tensors.
"""
from __future__ import annotations

import numpy as np

from . import _arrays

_CUDA_PITCH = 32  # bytes


def _itemsize(array) -> int:
    t = _arrays.torch()
    if isinstance(array, t.Tensor):
        return array.element_size()
    return array.dtype.itemsize


def _base(array):
    t = _arrays.torch()
    if isinstance(array, t.Tensor):
        return array._base if array._base is not None else array
    return array.base if array.base is not None else array


def pitched_shape(array) -> tuple:
    """Shape with the last axis padded to a whole number of 32-byte rows."""
    nbytes = int(np.ceil(array.shape[-1] * _itemsize(array) / _CUDA_PITCH)
                 ) * _CUDA_PITCH
    return (*tuple(array.shape[:-1]), nbytes // _itemsize(array))


def ispitched(array) -> bool:
    """Whether ``array`` (or the array it views) has a pitched shape."""
    b = _base(array)
    return tuple(pitched_shape(b)) == tuple(b.shape)


def aspitched(array, xp=None):
    """Copy into a pitched array (on the device when ``xp`` is torch or
    ``"cuda"``) and return a view of the original width."""
    t = _arrays.torch()
    to_device = xp is not None and xp is not np
    if isinstance(array, t.Tensor):
        to_device = to_device or array.is_cuda
    if ispitched(array) and (to_device == (isinstance(array, t.Tensor)
                                           and array.is_cuda)):
        return array
    if to_device:
        src = _arrays.as_tensor(array)
        base = t.zeros(pitched_shape(src), dtype=src.dtype, device="cuda")
        base[..., :src.shape[-1]] = src
        return base[..., :src.shape[-1]]
    src = np.asarray(array)
    base = np.zeros(pitched_shape(src), dtype=src.dtype)
    base[..., :src.shape[-1]] = src
    return base[..., :src.shape[-1]]


def pitched_like(array, xp=None, fill=None):
    """New pitched array with the shape of ``array`` (a pitched view)."""
    if not ispitched(array):
        raise ValueError("Input array needs to be pitched.")
    t = _arrays.torch()
    shape = pitched_shape(array)
    if isinstance(array, t.Tensor):
        base = t.empty(shape, dtype=array.dtype, device=array.device)
    else:
        base = np.empty(shape, dtype=array.dtype)
    view = base[..., :array.shape[-1]]
    if fill is not None:
        view[...] = fill
    return view


__all__ = ["pitched_shape", "ispitched", "aspitched", "pitched_like"]
