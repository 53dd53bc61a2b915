"""ctypes binding of ``libkk.so`` (C ABI declared in ``include/kk.h``).

The library is built in-tree by ``astra-kernelkit_b200/csrc/build.py``.
There is no fallback: if the library or a CUDA device is missing, every
projection call raises.
"""
from __future__ import annotations

import ctypes
import os
from typing import Sequence

import numpy as np

LIB_PATH = os.environ.get(
    "KERNELKIT_LIBKK",
    os.path.join(os.path.dirname(os.path.abspath(__file__)), "libkk.so"))

KK_OK = 0
KK_ERR_INVALID_ARGUMENT = 1
KK_ERR_UNSUPPORTED = 2
KK_ERR_CUDA = 3
KK_ERR_TIMEOUT = 4

KK_F32, KK_BF16, KK_F16 = 0, 1, 2
KK_INTERP_TEX8, KK_INTERP_EXACT = 0, 1

c_i64_3 = ctypes.c_int64 * 3


class kk_volume(ctypes.Structure):
    _fields_ = [("data", ctypes.c_void_p), ("shape", c_i64_3),
                ("stride", c_i64_3), ("dtype", ctypes.c_int32)]


class kk_projections(ctypes.Structure):
    _fields_ = [("data", ctypes.c_void_p), ("table", ctypes.c_void_p),
                ("table_axis", ctypes.c_int32), ("n_angles", ctypes.c_int64),
                ("rows", ctypes.c_int64), ("cols", ctypes.c_int64),
                ("stride", c_i64_3), ("dtype", ctypes.c_int32)]


class kk_fp_residual(ctypes.Structure):
    _fields_ = [("y", ctypes.c_void_p), ("weight", ctypes.c_void_p)]


class kk_fp_options(ctypes.Structure):
    _fields_ = [("interp", ctypes.c_int32), ("slab", ctypes.c_int32),
                ("additive", ctypes.c_int32), ("span", ctypes.c_int32),
                ("flags", ctypes.c_int32), ("vtex", ctypes.c_void_p),
                ("residual", ctypes.c_void_p), ("sums", ctypes.c_void_p),
                ("sums_elems", ctypes.c_int64), ("padded", ctypes.c_void_p),
                ("padded_elems", ctypes.c_int64)]


#: kk_fp_options.flags: shared-memory tiles staged by the tensor-copy
#: unit instead of direct loads for CUDA-core rays
KK_FP_OPT_TILES = 1


class kk_bp_update(ctypes.Structure):
    _fields_ = [("scale", ctypes.c_void_p), ("mask", ctypes.c_void_p),
                ("min_value", ctypes.c_float), ("max_value", ctypes.c_float),
                ("has_min", ctypes.c_int32), ("has_max", ctypes.c_int32)]


#: most problems one batched call takes (KK_MAX_BATCH of include/kk.h)
KK_MAX_BATCH = 64


class kk_fp_problem(ctypes.Structure):
    _fields_ = [("vol", kk_volume), ("proj", kk_projections),
                ("angles", ctypes.c_void_p),
                ("out_scale", ctypes.c_float * 9), ("vtex", ctypes.c_void_p),
                ("residual", kk_fp_residual), ("additive", ctypes.c_int32),
                ("span", ctypes.c_int32)]


class kk_bp_problem(ctypes.Structure):
    _fields_ = [("tex", ctypes.c_void_p), ("vol", kk_volume),
                ("angles", ctypes.c_void_p), ("out_scale", ctypes.c_float),
                ("update", kk_bp_update), ("work", ctypes.c_void_p),
                ("additive", ctypes.c_int32), ("tile_z", ctypes.c_int32),
                ("tile_y", ctypes.c_int32)]


class kk_bp_batch_options(ctypes.Structure):
    _fields_ = [("persistent", ctypes.c_int32), ("sync", ctypes.c_void_p),
                ("sync_elems", ctypes.c_int64),
                ("wait_budget_cycles", ctypes.c_int64),
                ("test_skip_item", ctypes.c_int32)]


#: kk_fp_angle as a NumPy record (64 bytes)
FP_ANGLE_DTYPE = np.dtype([("src", "<f4", 3), ("corner", "<f4", 3),
                           ("u", "<f4", 3), ("v", "<f4", 3),
                           ("axis", "<i4"), ("index", "<i4"),
                           ("flags", "<i4"), ("pad", "<i4")])
#: kk_fp_angle.flags bit: trace on the CUDA cores even with a texture
KK_FP_NO_TEXTURE = 1
#: kk_bp_angle as a NumPy record (48 bytes)
BP_ANGLE_DTYPE = np.dtype([("num_u", "<f4", 4), ("num_v", "<f4", 4),
                           ("den", "<f4", 4)])

#: every symbol include/kk.h declares
EXPORTS = ("kk_cone_fp_ex", "kk_fp_launches_ex", "kk_wait_timeouts",
           "kk_bp_launches",
           "kk_fdk_filter", "kk_fdk_plan", "kk_fdk_plan_size",
           "kk_cone_bp_layered_batched_ex", "kk_bp_batch_sync_elems",
           "kk_cone_fp", "kk_cone_fp_residual", "kk_cone_fp_layered",
           "kk_cone_fp_adjoint", "kk_cone_fp_batched",
           "kk_cone_bp_layered_batched",
           "kk_cone_bp", "kk_cone_bp_static",
           "kk_cone_bp_update", "kk_layered_create", "kk_layered_copy",
           "kk_layered_destroy", "kk_cone_bp_layered",
           "kk_cone_bp_layered_update", "kk_preweight", "kk_filter_rows",
           "kk_reciprocal", "kk_sirt_update", "kk_fp_set_span",
           "kk_fp_launches", "kk_last_error",
           "kk_abi_version")

_lib = None


class KernelKitError(RuntimeError):
    """A native call failed (CUDA error or rejected launch)."""


def load():
    """Load ``libkk.so`` once and declare its prototypes."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"{LIB_PATH} is missing: build it with "
            "`python astra-kernelkit_b200/csrc/build.py`")
    L = ctypes.CDLL(LIB_PATH)
    vp = ctypes.c_void_p
    P = ctypes.POINTER
    i32, i64, f32 = ctypes.c_int32, ctypes.c_int64, ctypes.c_float
    L.kk_cone_fp_ex.argtypes = [P(kk_volume), P(kk_projections), vp, vp,
                                P(kk_fp_options), vp]
    L.kk_fp_launches_ex.argtypes = [i32, i32, i32, i32]
    L.kk_bp_launches.argtypes = [i64]
    L.kk_bp_launches.restype = i32
    L.kk_wait_timeouts.argtypes = [P(i32)]
    L.kk_cone_fp.argtypes = [P(kk_volume), P(kk_projections), vp, vp, i32,
                             i32, i32, vp]
    L.kk_cone_fp_residual.argtypes = [P(kk_volume), P(kk_projections), vp, vp,
                                      P(kk_fp_residual), i32, i32, vp]
    L.kk_cone_fp_layered.argtypes = [vp, P(kk_volume), P(kk_projections), vp,
                                     vp, P(kk_fp_residual), i32, i32, vp]
    L.kk_cone_fp_adjoint.argtypes = [P(kk_projections), P(kk_volume), vp,
                                     vp, i32, i32, i32, vp, i64, vp]
    L.kk_cone_fp_batched.argtypes = [P(kk_fp_problem), i32, i32, i32, vp]
    L.kk_cone_bp_layered_batched.argtypes = [P(kk_bp_problem), i32, vp]
    L.kk_cone_bp_layered_batched_ex.argtypes = [P(kk_bp_problem), i32,
                                                P(kk_bp_batch_options), vp]
    L.kk_bp_batch_sync_elems.argtypes = [P(kk_bp_problem), i32]
    L.kk_cone_bp.argtypes = [P(kk_projections), P(kk_volume), vp, f32, i32,
                             i32, vp, vp]
    L.kk_cone_bp_update.argtypes = [P(kk_projections), P(kk_volume), vp, f32,
                                    P(kk_bp_update), i32, vp, vp]
    L.kk_cone_bp_static.argtypes = [P(kk_projections), P(kk_volume), vp, f32,
                                    i32, i32, vp]
    L.kk_layered_create.argtypes = [i64, i64, i64, i32, P(vp)]
    L.kk_layered_copy.argtypes = [vp, P(kk_projections), vp]
    L.kk_layered_destroy.argtypes = [vp]
    L.kk_cone_bp_layered.argtypes = [vp, P(kk_volume), vp, f32, i32, vp, vp]
    L.kk_cone_bp_layered_update.argtypes = [vp, P(kk_volume), vp, f32,
                                            P(kk_bp_update), vp, vp]
    L.kk_preweight.argtypes = [P(kk_projections), vp, vp]
    L.kk_filter_rows.argtypes = [P(kk_projections), vp, i64, vp]
    L.kk_fdk_filter.argtypes = [P(kk_projections), vp, vp, i64,
                                P(kk_projections), vp, i64, vp]
    L.kk_fdk_plan.argtypes = [vp, vp, i64, vp]
    L.kk_fdk_plan_size.argtypes = [i64]
    L.kk_reciprocal.argtypes = [vp, i64, vp]
    L.kk_sirt_update.argtypes = [vp, vp, vp, vp, f32, f32, i32, i32, i64, vp]
    L.kk_fp_set_span.argtypes = [i32]
    L.kk_fp_launches.argtypes = [i32, i32, i32]
    for name in EXPORTS[:-2]:
        getattr(L, name).restype = ctypes.c_int
    L.kk_fdk_plan_size.restype = ctypes.c_int64
    L.kk_bp_batch_sync_elems.restype = ctypes.c_int64
    L.kk_last_error.restype = ctypes.c_char_p
    L.kk_last_error.argtypes = []
    L.kk_abi_version.restype = ctypes.c_int
    L.kk_abi_version.argtypes = []
    _lib = L
    return L


def wait_timeouts() -> int:
    """Waits inside the library's kernels on the current device that gave
    up since the previous call (0 in normal operation). Synchronous."""
    n = ctypes.c_int32(0)
    check(load().kk_wait_timeouts(ctypes.byref(n)))
    return int(n.value)


def check(rc: int) -> None:
    """Map a kk_status to an exception."""
    if rc == KK_OK:
        return
    msg = load().kk_last_error().decode(errors="replace")
    if rc == KK_ERR_INVALID_ARGUMENT:
        raise ValueError(msg)
    if rc == KK_ERR_UNSUPPORTED:
        raise NotImplementedError(msg)
    raise KernelKitError(msg)


# ---------------------------------------------------------------------------
# descriptors from torch tensors
# ---------------------------------------------------------------------------
def _torch():
    import torch

    return torch


def dtype_code(t) -> int:
    torch = _torch()
    codes = {torch.float32: KK_F32, torch.bfloat16: KK_BF16,
             torch.float16: KK_F16}
    if t.dtype not in codes:
        raise NotImplementedError(
            f"Only float32, bfloat16 and float16 storage is supported, got "
            f"{t.dtype}.")
    return codes[t.dtype]


def current_stream() -> ctypes.c_void_p:
    return ctypes.c_void_p(_torch().cuda.current_stream().cuda_stream)


def volume_desc(t, volume_axes: Sequence[int] = (0, 1, 2)) -> kk_volume:
    """Descriptor of a CUDA tensor whose array axis k holds world axis
    ``volume_axes[k]``."""
    if not t.is_cuda:
        raise TypeError("Volume must be a CUDA array.")
    if t.dim() != 3:
        raise ValueError(f"Volume must be 3D, got shape {tuple(t.shape)}.")
    d = kk_volume()
    d.data = t.data_ptr()
    for k in range(3):
        d.shape[volume_axes[k]] = t.shape[k]
        d.stride[volume_axes[k]] = t.stride(k)
    d.dtype = dtype_code(t)
    return d


def projections_desc(t, projection_axes: Sequence[int] = (0, 1, 2)
                     ) -> kk_projections:
    """Descriptor of a CUDA tensor whose array axis k holds logical axis
    ``projection_axes[k]`` (0 angle, 1 row, 2 column)."""
    if not t.is_cuda:
        raise TypeError("Projections must be a CUDA array.")
    if t.dim() != 3:
        raise ValueError(
            f"Projections must be 3D, got shape {tuple(t.shape)}.")
    d = kk_projections()
    d.data = t.data_ptr()
    d.table = None
    d.table_axis = 0
    shape = [0, 0, 0]
    for k in range(3):
        shape[projection_axes[k]] = t.shape[k]
        d.stride[projection_axes[k]] = t.stride(k)
    d.n_angles, d.rows, d.cols = shape
    d.dtype = dtype_code(t)
    return d


def table_desc(table, n_angles, rows, cols, row_stride, col_stride,
               dtype) -> kk_projections:
    """Descriptor of per-angle 2D arrays given by a device table of base
    addresses (int64 CUDA tensor of length ``n_angles``)."""
    d = kk_projections()
    d.data = None
    d.table = table.data_ptr()
    d.table_axis = 0
    d.n_angles, d.rows, d.cols = int(n_angles), int(rows), int(cols)
    d.stride[0] = 0
    d.stride[1] = int(row_stride)
    d.stride[2] = int(col_stride)
    d.dtype = dtype
    return d


def ptr(t) -> int:
    return 0 if t is None else t.data_ptr()


class Layered:
    """Owner of a ``kk_layered`` texture (destroyed with the object)."""

    def __init__(self, layers, height, width, dtype):
        self.shape = (int(layers), int(height), int(width))
        self.dtype = int(dtype)
        h = ctypes.c_void_p()
        check(load().kk_layered_create(self.shape[0], self.shape[1],
                                       self.shape[2], self.dtype,
                                       ctypes.byref(h)))
        self.handle = h

    def copy_from(self, t):
        """Copy a (layers, height, width) CUDA tensor on the current
        stream."""
        d = projections_desc(t)
        if (d.n_angles, d.rows, d.cols) != self.shape:
            raise ValueError(f"Shape {tuple(t.shape)} does not match the "
                             f"texture {self.shape}.")
        check(load().kk_layered_copy(self.handle, d, current_stream()))

    def __del__(self):
        h = getattr(self, "handle", None)
        if h is not None and h.value and _lib is not None:
            _lib.kk_layered_destroy(h)
            self.handle = None
