"""Import the reference's Python package from its checkout for golden-vector
generation (run only where the checkout exists, never on the GPU machine).

The reference imports CuPy and transforms3d at module level. Neither is
installed here, and the code paths used for golden vectors (geometry,
``geoms2params``, ``processing.preweight``/``filter``) only need NumPy
semantics, so both are replaced by small stand-ins before import:
``cupy`` by NumPy plus inert texture/runtime placeholders, and
``transforms3d.euler.euler2mat`` (static ``sxyz`` frame) by the published
Euler-angle closed form (Shoemake, Graphics Gems IV).
"""
from __future__ import annotations

import math
import os
import sys
import types

import numpy as np

#: checkout of the reference (KK_REFERENCE overrides the default location)
REFERENCE = os.environ.get("KK_REFERENCE", "/root/reference")


def _cupy_stand_in():
    cp = types.ModuleType("cupy")
    for name in dir(np):
        if not name.startswith("__"):
            setattr(cp, name, getattr(np, name))
    cp.get_array_module = lambda *a, **k: np

    class _Inert:
        def __init__(self, *a, **k):
            pass

    cuda = types.ModuleType("cupy.cuda")
    tex = types.ModuleType("cupy.cuda.texture")
    for n in ("TextureObject", "TextureDescriptor", "ChannelFormatDescriptor",
              "CUDAarray", "ResourceDescriptor"):
        setattr(tex, n, _Inert)
    rt = types.ModuleType("cupy.cuda.runtime")
    for n in ("cudaAddressModeBorder", "cudaChannelFormatKindFloat",
              "cudaFilterModeLinear", "cudaReadModeElementType",
              "cudaResourceTypeArray", "cudaResourceTypePitch2D"):
        setattr(rt, n, 0)
    cuda.texture, cuda.runtime = tex, rt
    cp.cuda = cuda
    cp.RawModule = _Inert
    cpx = types.ModuleType("cupyx")
    return {"cupy": cp, "cupy.cuda": cuda, "cupy.cuda.texture": tex,
            "cupy.cuda.runtime": rt, "cupyx": cpx}


def _euler2mat(ai, aj, ak, axes="sxyz"):
    if axes != "sxyz":
        raise NotImplementedError(axes)
    si, sj, sk = math.sin(ai), math.sin(aj), math.sin(ak)
    ci, cj, ck = math.cos(ai), math.cos(aj), math.cos(ak)
    cc, cs = ci * ck, ci * sk
    sc, ss = si * ck, si * sk
    M = np.eye(3)
    M[0, 0] = cj * ck
    M[0, 1] = sj * sc - cs
    M[0, 2] = sj * cc + ss
    M[1, 0] = cj * sk
    M[1, 1] = sj * ss + cc
    M[1, 2] = sj * cs - sc
    M[2, 0] = -sj
    M[2, 1] = cj * si
    M[2, 2] = cj * ci
    return M


def import_reference(path: str = REFERENCE):
    """Return the reference's ``kernelkit`` module (with stand-ins)."""
    stand_ins = _cupy_stand_in()
    t3 = types.ModuleType("transforms3d")
    eu = types.ModuleType("transforms3d.euler")
    eu.euler2mat = _euler2mat
    t3.euler = eu
    stand_ins.update({"transforms3d": t3, "transforms3d.euler": eu})
    sys.modules.update(stand_ins)
    if path not in sys.path:
        sys.path.insert(0, path)
    for name in list(sys.modules):
        if name == "kernelkit" or name.startswith("kernelkit."):
            del sys.modules[name]
    import kernelkit  # noqa: E402

    return kernelkit
