"""Array plumbing: device memory is PyTorch CUDA memory.

Accepted inputs are torch tensors, any object exposing
``__cuda_array_interface__`` (e.g. CuPy arrays, wrapped without a copy)
and NumPy arrays (copied to the device).
"""
from __future__ import annotations

import numpy as np


def torch():
    import torch as _t

    return _t


def require_cuda():
    t = torch()
    if not t.cuda.is_available():
        raise RuntimeError(
            "A CUDA device is required: the cone-beam projectors run only "
            "as CUDA kernels.")


def is_device_array(x) -> bool:
    t = torch()
    if isinstance(x, t.Tensor):
        return x.is_cuda
    return hasattr(x, "__cuda_array_interface__")


def as_tensor(x, dtype=None, copy=False):
    """CUDA tensor view of ``x`` (zero-copy for device arrays of the right
    dtype; NumPy input is copied to the device)."""
    t = torch()
    require_cuda()
    if isinstance(x, t.Tensor):
        out = x if x.is_cuda else x.cuda()
    elif hasattr(x, "__cuda_array_interface__"):
        out = t.as_tensor(x, device="cuda")
    else:
        arr = np.asarray(x)
        out = t.from_numpy(np.ascontiguousarray(arr)).cuda()
    if dtype is not None and out.dtype != dtype:
        out = out.to(dtype)
    elif copy:
        out = out.clone()
    return out


def to_numpy(x) -> np.ndarray:
    t = torch()
    if isinstance(x, t.Tensor):
        return x.detach().cpu().numpy()
    if hasattr(x, "get"):
        return x.get()
    return np.asarray(x)


def dtype_of(name):
    """torch dtype from a name or dtype ('float32', np.float32, ...)."""
    t = torch()
    if isinstance(name, t.dtype):
        return name
    key = np.dtype(name).name if not isinstance(name, str) else name
    table = {"float32": t.float32, "bfloat16": t.bfloat16,
             "float16": t.float16, "half": t.float16}
    if key not in table:
        raise NotImplementedError(f"Unsupported storage dtype {name!r}.")
    return table[key]
