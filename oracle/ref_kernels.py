"""ctypes wrapper around ``oracle/_ref/libkkref.so``: the reference's own
cone-beam kernels (built from its sources by ``oracle/build_ref.py``) and
the texture-filter probe. Test infrastructure only; needs a CUDA GPU.

Device buffers are torch CUDA tensors; every call runs on the current
torch stream.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_ref", "libkkref.so")

_lib = None


def available() -> bool:
    return os.path.exists(LIB_PATH)


def lib():
    global _lib
    if _lib is None:
        if not available():
            raise RuntimeError(
                f"{LIB_PATH} missing; build it with oracle/build_ref.py")
        L = ctypes.CDLL(LIB_PATH)
        vp, i, f = ctypes.c_void_p, ctypes.c_int, ctypes.c_float
        L.kkref_cone_fp.argtypes = [vp, i, i, i, vp, vp, i, i, i, vp, vp, vp,
                                    vp]
        L.kkref_cone_fp.restype = i
        L.kkref_cone_bp.argtypes = [vp, i, i, i, vp, vp, i, i, i, f, vp, vp]
        L.kkref_cone_bp.restype = i
        L.kkp_probe.argtypes = [vp, i, i, i, i, i, vp, vp, vp, vp, i]
        L.kkp_probe.restype = i
        _lib = L
    return _lib


def _stream():
    import torch

    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def ref_cone_fp(volume, params, axes, rows, cols, out_scale):
    """Reference forward projection. ``volume`` float32 CUDA tensor
    (nx, ny, nz); ``params`` (n, 12) float32 host; ``axes`` (n,) ints;
    ``out_scale`` (3, 3). Returns (projections tensor, kernel ms)."""
    import torch

    assert volume.is_cuda and volume.dtype == torch.float32
    volume = volume.contiguous()
    nx, ny, nz = volume.shape
    params = np.ascontiguousarray(params, np.float32).reshape(-1, 12)
    n = len(params)
    axes = np.ascontiguousarray(axes, np.int32)
    osc = np.ascontiguousarray(out_scale, np.float32).reshape(9)
    proj = torch.empty((n, rows, cols), dtype=torch.float32,
                       device=volume.device)
    ms = ctypes.c_float(0)
    rc = lib().kkref_cone_fp(
        volume.data_ptr(), nx, ny, nz, params.ctypes.data, axes.ctypes.data,
        n, rows, cols, osc.ctypes.data, proj.data_ptr(), ctypes.byref(ms),
        _stream())
    if rc != 0:
        raise RuntimeError(f"kkref_cone_fp failed with CUDA error {rc}")
    return proj, ms.value


def ref_cone_bp(projections, params, vol_shape, voxel_volume):
    """Reference backprojection of float32 CUDA ``projections`` (n, rows,
    cols) with (n, 12) ``params``. Returns (volume tensor, kernel ms)."""
    import torch

    assert projections.is_cuda and projections.dtype == torch.float32
    projections = projections.contiguous()
    n, rows, cols = projections.shape
    params = np.ascontiguousarray(params, np.float32).reshape(-1, 12)
    assert len(params) == n
    nx, ny, nz = (int(s) for s in vol_shape)
    vol = torch.empty((nx, ny, nz), dtype=torch.float32,
                      device=projections.device)
    ms = ctypes.c_float(0)
    rc = lib().kkref_cone_bp(
        projections.data_ptr(), n, rows, cols, params.ctypes.data,
        vol.data_ptr(), nx, ny, nz, float(voxel_volume), ctypes.byref(ms),
        _stream())
    if rc != 0:
        raise RuntimeError(f"kkref_cone_bp failed with CUDA error {rc}")
    return vol, ms.value


def tex_probe(data, xs, ys, zs=None, layered=True, layer=0):
    """Linear-filtered texture fetches of ``data`` (depth, h, w) float32 at
    float32 coordinates; returns a NumPy float32 array."""
    import torch

    dev = torch.device("cuda")
    d = torch.as_tensor(np.ascontiguousarray(data, np.float32), device=dev)
    depth, h, w = d.shape
    x = torch.as_tensor(np.ascontiguousarray(xs, np.float32), device=dev)
    y = torch.as_tensor(np.ascontiguousarray(ys, np.float32), device=dev)
    z = torch.as_tensor(np.ascontiguousarray(
        zs if zs is not None else np.zeros_like(xs), np.float32), device=dev)
    n = x.numel()
    assert y.numel() == n and z.numel() == n
    out = torch.empty(n, dtype=torch.float32, device=dev)
    torch.cuda.synchronize()
    rc = lib().kkp_probe(d.data_ptr(), w, h, depth, int(layered), int(layer),
                         x.data_ptr(), y.data_ptr(), z.data_ptr(),
                         out.data_ptr(), n)
    if rc != 0:
        raise RuntimeError(f"kkp_probe failed with CUDA error {rc}")
    return out.cpu().numpy()
