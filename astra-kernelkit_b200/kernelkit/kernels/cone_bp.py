"""Voxel-driven cone-beam backprojection kernel.

Python face of ``kk_cone_bp`` (``include/kk.h``), mirroring
``kernelkit/kernels/cone_bp.py`` of the reference (class name, options,
``InterpolationMethod``, ``compile``/``geoms2params``/``set_params``/
``__call__`` and exceptions). Projections are read from device memory;
the texture kinds of the reference are accepted as layout hints.
"""
from __future__ import annotations

import copy
from enum import Enum

import numpy as np

from .. import _arrays, _native
from ..geom import normalize_
from ..geom.proj import ProjectionGeometrySequence
from ..geom.vol import VolumeGeometry
from ..kernel import (BaseKernel, KernelMemoryUnpreparedException,
                      KernelNotCompiledException, Texture, cuda_float4)
from .cone_fp import interp_code, list_desc


class VoxelDrivenConeBP(BaseKernel):
    """Voxel-driven cone-beam backprojection.

    Each voxel centre is projected onto every detector with three affine
    forms (numerators of u and v and a common denominator); the voxel gains
    ``r^2 * proj(V, U)`` with ``r = 1/den``, which with the parameter
    scaling of ``geoms2params`` makes the result the reference's (scaled)
    adjoint of the forward projector."""

    FLOAT_DTYPE = np.float32
    SUPPORTED_DTYPES = ("float32", "bfloat16", "float16")

    class InterpolationMethod(Enum):
        """Texture kinds of the reference (``kernels/cone_bp.py:29-41``).
        Here they only describe how the projections are laid out."""

        Tex3D = "tex3D"
        Tex2DLayered = "tex2DLayered"
        Surf2DLayered = "surf2DLayered"
        Tex2D = "tex2D"

    voxels_per_block = (6, 32, 16)
    projs_per_block = 32

    def __init__(self, voxels_per_block: tuple = None,
                 projs_per_block: int = None,
                 volume_axes: tuple = (0, 1, 2),
                 projection_axes: tuple = (0, 1, 2),
                 interpolation: str = "texture"):
        super().__init__()
        if voxels_per_block is not None and len(voxels_per_block) != 3:
            raise ValueError("`voxels_per_block` must have 3 elements.")
        if voxels_per_block is not None and voxels_per_block[0] != 6:
            raise NotImplementedError(
                "Backprojection groups voxels by 6 along the first memory "
                "axis (the reference default).")
        if projs_per_block is not None and projs_per_block != 32:
            raise NotImplementedError(
                "Backprojection accumulates angles in chunks of 32 (the "
                "reference default).")
        self._vox_block = tuple(voxels_per_block or self.voxels_per_block)
        self._projs_block = projs_per_block or self.projs_per_block
        for name, axes in (("volume_axes", volume_axes),
                           ("projection_axes", projection_axes)):
            if sorted(axes) != [0, 1, 2]:
                raise ValueError(f"`{name}` must be a permutation of "
                                 f"(0, 1, 2), got {axes}.")
        self._vol_axs = tuple(volume_axes)
        self._proj_axs = tuple(projection_axes)
        self._interp = interp_code(interpolation)
        self.interpolation = interpolation
        self._params_dev = None
        self._n_params = 0

    @property
    def volume_axes(self):
        return self._vol_axs

    @property
    def projection_axes(self):
        return self._proj_axs

    @property
    def _params_are_set(self) -> bool:
        return self._params_dev is not None

    def compile(self, max_projs: int = 1024,
                texture: "VoxelDrivenConeBP.InterpolationMethod | str | None"
                = InterpolationMethod.Tex3D):
        """Validate options (as ``kernels/cone_bp.py:114-166``) and load the
        native library. ``max_projs`` is accepted for compatibility."""
        if texture is not None:
            if isinstance(texture, str):
                texture = self.InterpolationMethod(texture)
            if texture not in self.InterpolationMethod:
                raise ValueError(f"`texture` must be one of "
                                 f"{list(self.InterpolationMethod)} or None.")
            if texture in (self.InterpolationMethod.Tex2D,
                           self.InterpolationMethod.Tex2DLayered):
                if self._proj_axs[0] != 0:
                    raise ValueError(
                        "If an array of textures or a layered texture is "
                        "given, the first `projection_axes` axis must be "
                        "angles, i.e., must be 0.")
        return self._compile(dict(
            voxels_per_block=self._vox_block,
            nr_projs_block=self._projs_block, nr_projs_global=int(max_projs),
            texture=texture.value if texture is not None else None,
            volume_axes=self._vol_axs, projection_axes=self._proj_axs,
            interpolation=self.interpolation))

    def set_params(self, params):
        """Upload the flat (12 n,) float32 parameters of ``geoms2params``."""
        if not self.is_compiled:
            raise KernelNotCompiledException(
                f"Kernel {self.__class__.__name__} must be compiled before "
                "uploading parameters to the GPU.")
        arr = np.ascontiguousarray(_arrays.to_numpy(params), np.float32)
        if arr.size % 12 != 0:
            raise ValueError("Parameters must hold 12 floats per angle.")
        t = _arrays.torch()
        self._params_dev = t.from_numpy(arr.reshape(-1)).cuda()
        self._n_params = arr.size // 12

    def _work_for(self, vol, update: bool):
        """float32 running-sum buffer for chunked launches (one element per
        voxel), made on first use; 0 when the volume itself can hold the
        running sum."""
        t = _arrays.torch()
        if self._n_params <= 32 or (vol.dtype == t.float32 and not update):
            return 0
        w = getattr(self, "_work", None)
        if w is None or w.numel() != vol.numel() or w.device != vol.device:
            w = t.empty(vol.numel(), dtype=t.float32, device=vol.device)
            self._work = w
        return w.data_ptr()

    def _layered_source(self, textures):
        """The layered texture to sample, or None for the device-memory
        path: texture interpolation is only the reference's own filter,
        for angle-first projections."""
        t = _arrays.torch()
        if self._interp != _native.KK_INTERP_TEX8 or self._proj_axs[0] != 0:
            return None
        if isinstance(textures, _native.Layered):
            return textures
        if (isinstance(textures, Texture) and textures.array.dim() == 3
                and textures.array.dtype == t.float32):
            return textures.layered_texture()
        return None

    def _input(self, textures):
        t = _arrays.torch()
        if isinstance(textures, Texture):
            textures = textures.array
        if isinstance(textures, (list, tuple)):
            return list_desc(textures, self._proj_axs)
        arr = _arrays.as_tensor(textures)
        if arr.dtype == t.int64:
            raise TypeError(
                "Arrays of texture-object pointers do not exist here; pass "
                "the projections (a 3D device array or a list of 2D device "
                "arrays).")
        return _native.projections_desc(arr, self._proj_axs), (arr,)

    def __call__(self, textures, volume, volume_geometry: VolumeGeometry,
                 additive: bool = True):
        """Backproject ``textures`` into ``volume``.

        As in the reference the result is added to ``volume``; pass
        ``additive=False`` to overwrite instead. ``textures`` is a
        ``Texture`` (sampled through its layered texture, i.e. the
        reference's own filter), a layered texture, a device array laid out
        by ``projection_axes`` or a list of 2D device arrays; ``volume`` a
        C-contiguous device array laid out by ``volume_axes``."""
        t = _arrays.torch()
        if not _arrays.is_device_array(volume):
            raise TypeError("`volume` must be a device array.")
        vol = _arrays.as_tensor(volume)
        if vol.dtype not in (t.float32, t.bfloat16, t.float16):
            raise NotImplementedError(
                f"Volume has a dtype '{vol.dtype}'. However, currently there "
                f"is only support for dtype={self.SUPPORTED_DTYPES}.")
        if not vol.is_contiguous():
            raise ValueError(
                f"`{self.__class__.__name__}` needs a C-contiguous volume.")
        if not volume_geometry.has_isotropic_voxels():
            raise NotImplementedError(
                f"`{self.__class__.__name__}` is not tested with anisotropic "
                "voxels yet.")
        if not self.is_compiled:
            raise KernelNotCompiledException(
                "Please compile the kernel with `compile()`.")
        vdesc = _native.volume_desc(vol, self._vol_axs)
        vox_vol = np.float32(volume_geometry.voxel_volume())
        lay = self._layered_source(textures)
        if not self._params_are_set:
            raise KernelMemoryUnpreparedException(
                "Please set the parameters with `set_params()`.")
        if lay is not None:
            if lay.shape[0] != self._n_params:
                raise ValueError(f"{lay.shape[0]} projections given, but "
                                 f"parameters for {self._n_params} angles.")
            _native.check(_native.load().kk_cone_bp_layered(
                lay.handle, vdesc, self._params_dev.data_ptr(),
                float(vox_vol), int(bool(additive)),
                self._work_for(vol, False), _native.current_stream()))
            return
        pdesc, keep = self._input(textures)
        if pdesc.n_angles != self._n_params:
            raise ValueError(f"{pdesc.n_angles} projections given, but "
                             f"parameters for {self._n_params} angles.")
        _native.check(_native.load().kk_cone_bp(
            pdesc, vdesc, self._params_dev.data_ptr(), float(vox_vol),
            self._interp, int(bool(additive)), self._work_for(vol, False),
            _native.current_stream()))
        del keep

    def update(self, projections, volume, volume_geometry: VolumeGeometry,
               scale, mask=None, min_value=None, max_value=None):
        """Fused SIRT update (one kernel; reference ``algo.py:356-362``):
        ``volume = clip(mask * (volume - scale * A^T projections))``. All
        arrays float32 device arrays; ``scale``/``mask`` in the layout of
        ``volume``."""
        if not self._params_are_set:
            raise KernelMemoryUnpreparedException(
                "Please set the parameters with `set_params()`.")
        vdesc = _native.volume_desc(volume, self._vol_axs)
        for name, a in (("scale", scale), ("mask", mask)):
            if a is not None and (a.shape != volume.shape
                                  or a.stride() != volume.stride()):
                raise ValueError(f"`{name}` must have the layout of `volume`.")
        upd = _native.kk_bp_update(
            scale.data_ptr(), _native.ptr(mask),
            float(min_value) if min_value is not None else 0.0,
            float(max_value) if max_value is not None else 0.0,
            int(min_value is not None), int(max_value is not None))
        vox_vol = np.float32(volume_geometry.voxel_volume())
        lay = self._layered_source(projections)
        if lay is not None:
            _native.check(_native.load().kk_cone_bp_layered_update(
                lay.handle, vdesc, self._params_dev.data_ptr(),
                float(vox_vol), upd, self._work_for(volume, True),
                _native.current_stream()))
            return
        pdesc, keep = self._input(projections)
        _native.check(_native.load().kk_cone_bp_update(
            pdesc, vdesc, self._params_dev.data_ptr(), float(vox_vol), upd,
            self._interp, self._work_for(volume, True),
            _native.current_stream()))
        del keep

    @staticmethod
    def geoms2params(projection_geometry, volume_geometry: VolumeGeometry,
                     with_adjoint_scaling: bool = True) -> np.ndarray:
        """Per-angle affine forms of the voxel-to-detector projection.

        With ``u = u_hat * pixel_width``, ``v = v_hat * pixel_height``,
        ``s`` the source and ``d`` the detector corner (unit-voxel frame):
        ``U = det[(x-s) v (s-d)] / det[u v (s-x)]`` and ``V = -det[u (x-s)
        (s-d)] / det[u v (s-x)]``, written as affine numerators over an
        affine denominator in the voxel position x. All three are scaled by
        ``sqrt(|u x v|') / det[u v (d-s)]`` (``|u x v|'`` with the
        voxel-size factors) so that ``1/den^2`` is the ray-density weight
        of the adjoint. Same float32 evaluation as the reference
        (``kernels/cone_bp.py:304-421``). Returns (12 n,) float32 laid out
        per angle as numU.xyzw, numV.xyzw, den.xyzw."""
        if isinstance(projection_geometry, ProjectionGeometrySequence):
            g = copy.deepcopy(projection_geometry)
        else:
            g = ProjectionGeometrySequence.fromList(projection_geometry)
        normalize_(g, volume_geometry)
        vs = volume_geometry.voxel_size
        u = g.u * g.detector.pixel_width[..., np.newaxis]
        v = g.v * g.detector.pixel_height[..., np.newaxis]
        s = g.source_position
        d = g.detector_extent_min

        cr = np.cross(u, v)
        cr *= np.array([vs[1] * vs[2], vs[0] * vs[2], vs[0] * vs[1]])
        scale = np.sqrt(np.linalg.norm(cr, axis=1))
        if with_adjoint_scaling:
            scale /= np.linalg.det(np.asarray((u, v, d - s)).swapaxes(0, 1))
        else:
            scale = 1.0

        def det3x(b, c):
            return b[:, 1] * c[:, 2] - b[:, 2] * c[:, 1]

        def det3y(b, c):
            return b[:, 0] * c[:, 2] - b[:, 2] * c[:, 0]

        def det3z(b, c):
            return b[:, 0] * c[:, 1] - b[:, 1] * c[:, 0]

        def det3(a, b, c):
            return np.linalg.det(np.asarray((a, b, c)).swapaxes(0, 1))

        smd = s - d
        num_u = cuda_float4(x=scale * det3x(v, smd), y=-scale * det3y(v, smd),
                            z=scale * det3z(v, smd), w=scale * det3(s, v, d))
        num_v = cuda_float4(x=-scale * det3x(u, smd), y=scale * det3y(u, smd),
                            z=-scale * det3z(u, smd),
                            w=-scale * det3(s, u, d))
        den = cuda_float4(x=-scale * det3x(u, v), y=scale * det3y(u, v),
                          z=-scale * det3z(u, v), w=scale * det3(u, v, s))
        rows = np.asarray(num_u.to_list() + num_v.to_list() + den.to_list())
        return np.ascontiguousarray(rows.T.astype(np.float32)).reshape(-1)


__all__ = ["VoxelDrivenConeBP"]
