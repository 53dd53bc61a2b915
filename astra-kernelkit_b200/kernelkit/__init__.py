"""B200-native cone-beam projection path with the API of ASTRA KernelKit.

Drop-in for ``kernelkit``'s cone-beam hot path: geometry
(``ProjectionGeometry``, ``resolve_volume_geometry``, ...), the kernels
``RayDrivenConeFP``/``VoxelDrivenConeBP`` (also as ``ConeProjector``/
``ConeBackprojector``), ``ForwardProjector``/``BackProjector``,
``ProjectorOperator``/``XrayTransform``, ``fp``/``bp``/``fdk``/``sirt`` and
``torch_support``. The kernels are hand-written CUDA for sm_100a in
``libkk.so`` (C ABI ``include/kk.h``); device arrays are torch tensors (or
any ``__cuda_array_interface__`` array).
"""
__version__ = "1.0.0-alpha.2+b200"

KERNELKIT_VERSION = __version__

from .operator import *  # noqa: E402,F401,F403
from .algo import fp, bp, fdk, sirt, SIRT  # noqa: E402,F401
from .data import *  # noqa: E402,F401,F403
from .geom import resolve_volume_geometry, suggest_volume_extent, normalize_  # noqa: E402,F401
from .geom.proj import *  # noqa: E402,F401,F403
from .geom.vol import *  # noqa: E402,F401,F403
from . import kernel  # noqa: E402,F401
from . import kernels  # noqa: E402,F401
from . import experimental  # noqa: E402,F401
from . import processing  # noqa: E402,F401
from . import batch  # noqa: E402,F401
from . import distributed  # noqa: E402,F401
from .kernels import RayDrivenConeFP, VoxelDrivenConeBP  # noqa: E402,F401
from .projector import (ProjectionGeometryNotSetError,  # noqa: E402,F401
                        VolumeGeometryNotSetError, VolumeNotSetError,
                        ProjectionsNotSetError)

# names used by the reference's older API
ConeProjector = RayDrivenConeFP
ConeBackprojector = VoxelDrivenConeBP
