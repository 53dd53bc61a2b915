"""Ray-driven cone-beam forward projection kernel.

Python face of ``kk_cone_fp`` (``include/kk.h``), mirroring
``kernelkit/kernels/cone_fp.py`` of the reference: same class name,
constructor options, ``compile``/``geoms2params``/``set_params``/
``__call__`` protocol and exceptions. Per-angle parameters live in device
memory owned by the kernel object (the reference uses ``__constant__``
memory capped at ``max_projs`` angles; here there is no cap).
"""
from __future__ import annotations

import copy
import ctypes
from typing import Sequence

import numpy as np

from .. import _arrays, _native
from ..geom import normalize_
from ..geom.proj import ProjectionGeometrySequence
from ..geom.vol import VolumeGeometry
from ..kernel import (BaseKernel, KernelMemoryUnpreparedException,
                      KernelNotCompiledException, Texture)

_INTERP = {"texture": _native.KK_INTERP_TEX8, "tex8": _native.KK_INTERP_TEX8,
           "exact": _native.KK_INTERP_EXACT, "linear": _native.KK_INTERP_EXACT}


def interp_code(name: str) -> int:
    try:
        return _INTERP[name.lower()]
    except KeyError:
        raise ValueError(
            f"`interpolation` must be one of {sorted(_INTERP)}, got {name!r}.")


class ConeFPParams(tuple):
    """The 12 float32 parameter arrays of ``geoms2params`` (source xyz,
    detector corner xyz, u*pixel_width xyz, v*pixel_height xyz; reference
    ``kernels/cone_fp.py:330-339``) plus ``axes``, the dominant ray axis
    per angle (``kernels/cone_fp.py:264-285``)."""

    axes: np.ndarray | None

    def __new__(cls, arrays, axes=None):
        obj = super().__new__(cls, arrays)
        obj.axes = axes
        return obj


#: device pointer tables of recently used projection lists, so repeated
#: calls on the same list upload nothing (and can be graph-captured)
_TABLES: dict = {}


def list_desc(projections, projection_axes):
    """Descriptor (and keep-alive objects) of a list of 2D per-angle device
    arrays, e.g. pitched views from ``kernelkit.aspitched``; entry axes are
    the logical axes ``projection_axes[1:]``. All entries must share one
    layout."""
    t = _arrays.torch()
    if projection_axes[0] != 0:
        raise ValueError(
            "A list of projections requires projection_axes[0] == 0.")
    arrs = [_arrays.as_tensor(p) for p in projections]
    if len(arrs) == 0:
        raise ValueError("Empty list of projections.")
    first = arrs[0]
    for a in arrs:
        if a.dim() != 2:
            raise ValueError("Projection list entries must be 2D.")
        if (a.shape != first.shape or a.stride() != first.stride()
                or a.dtype != first.dtype):
            raise ValueError("Projection list entries must share shape, "
                             "strides and dtype.")
    r_ax = projection_axes.index(1) - 1
    c_ax = projection_axes.index(2) - 1
    key = tuple(a.data_ptr() for a in arrs)
    table = _TABLES.pop(key, None)
    if table is None:
        table = t.tensor(key, dtype=t.int64, device="cuda")
    _TABLES[key] = table  # most recent last
    while len(_TABLES) > 8:
        _TABLES.pop(next(iter(_TABLES)))
    d = _native.table_desc(table, len(arrs), first.shape[r_ax],
                           first.shape[c_ax], first.stride(r_ax),
                           first.stride(c_ax), _native.dtype_code(first))
    return d, (arrs, table)


def _sequence(projection_geometry) -> ProjectionGeometrySequence:
    if isinstance(projection_geometry, ProjectionGeometrySequence):
        return copy.deepcopy(projection_geometry)
    return ProjectionGeometrySequence.fromList(projection_geometry)


class RayDrivenConeFP(BaseKernel):
    """Ray-driven (Joseph) cone-beam forward projection.

    Every ray steps one slice at a time along its dominant world axis and
    sums bilinear samples of the volume at the slice centres, times the
    distance correction; ``interpolation='texture'`` (default) samples with
    the texture unit's 1/256 weights as the reference does,
    ``'exact'`` with exact weights.
    """

    FLOAT_DTYPE = np.float32
    SUPPORTED_DTYPES = ("float32", "bfloat16", "float16")

    pixels_per_block = (1, 32, 32)
    slices_per_block = 16
    #: share of the texture-path angles traced on the CUDA cores instead,
    #: so that the texture unit and the arithmetic pipes finish together
    cuda_core_fraction = 0.0
    #: records of one ray axis launched back to back before the next axis
    axis_group = 4
    #: let 16-bit volumes use a float16 layered texture (reduced-precision
    #: filtering: for 16-bit storage runs, whose tolerance is the storage's)
    half_texture = False
    #: slices of every ray's own axis traced per launch (None: the module
    #: default of ``set_slices_per_launch``; -1: one launch)
    slices_per_launch = None
    #: rays traced on the CUDA cores sample shared-memory tiles of the
    #: volume staged by the tensor-copy unit instead of loading it
    #: directly (same results bit for bit; slower at the measured shapes,
    #: so off by default)
    use_tiles = False
    #: bytes of the float32 buffer that carries the running sums between
    #: slice-span launches when the projections are 16-bit (angles are
    #: traced in chunks that fit it); 0 traces 16-bit projections in one
    #: launch
    sums_bytes = 1 << 30
    #: texture-compatible weights: trace from a copy of the volume with two
    #: zero texels around every axis, made at the start of every call
    #: (same results; the CUDA-core rays of circular scans then sample the
    #: slabs that cross the volume's boundary without per-texel tests)
    padded_copy = True

    def __init__(self, pixels_per_block: tuple = None,
                 slices_per_block: int = None,
                 volume_axes: tuple = (0, 1, 2),
                 projection_axes: tuple = (0, 1, 2),
                 interpolation: str = "texture",
                 use_texture_unit: bool = True,
                 cuda_core_fraction: float = None):
        super().__init__()
        if cuda_core_fraction is not None:
            if not 0.0 <= float(cuda_core_fraction) <= 1.0:
                raise ValueError("`cuda_core_fraction` must be in [0, 1].")
            self.cuda_core_fraction = float(cuda_core_fraction)
        # rays along the volume's slowest axis may sample a layered copy of
        # the volume through the texture unit (same filter as the
        # reference); the others run on the CUDA cores
        self.use_texture_unit = bool(use_texture_unit)
        self._vtex = None
        if pixels_per_block is not None:
            self.pixels_per_block = tuple(pixels_per_block)
        if slices_per_block is not None:
            if int(slices_per_block) <= 0:
                raise ValueError("`slices_per_block` must be positive.")
            self.slices_per_block = int(slices_per_block)
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
        self._axes_known = False

    @property
    def volume_axes(self) -> tuple:
        return self._vol_axs

    @property
    def projection_axes(self) -> tuple:
        return self._proj_axs

    @property
    def _params_are_set(self) -> bool:
        return self._params_dev is not None

    def compile(self, max_projs: int = 1024):
        """Validate options and load the native library. ``max_projs`` is
        accepted for compatibility; there is no per-kernel angle cap."""
        return self._compile(dict(
            slices_per_block=self.slices_per_block,
            rows_per_block=self.pixels_per_block[1],
            cols_per_block=self.pixels_per_block[2],
            nr_projs_global=int(max_projs),
            volume_axes=self._vol_axs, projection_axes=self._proj_axs,
            interpolation=self.interpolation))

    # -- parameters ---------------------------------------------------------
    @staticmethod
    def _geom_axes(projection_geometry) -> np.ndarray:
        """Dominant world axis of each ray (argmax |source - detector|)."""
        pg = projection_geometry
        return np.argmax(np.abs(pg.source_position - pg.detector_position),
                         axis=1)

    @staticmethod
    def _output_scale(voxel_size) -> list:
        """(scale1, scale2, outputScale) per dominant axis
        (``kernels/cone_fp.py:287-300``)."""
        eps = 1e-4
        v = voxel_size
        if abs(v[0] / v[1] - 1) > eps or abs(v[0] / v[2] - 1) > eps:
            x = [(v[1] / v[0]) ** 2, (v[2] / v[0]) ** 2, v[0] ** 2]
            y = [(v[0] / v[1]) ** 2, (v[2] / v[1]) ** 2, v[0] * v[1]]
            z = [(v[0] / v[2]) ** 2, (v[1] / v[2]) ** 2, v[0] * v[2]]
            return [x, y, z]
        return [[1.0, 1.0, v[0]]] * 3

    @staticmethod
    def geoms2params(projection_geometry, volume_geometry: VolumeGeometry
                     ) -> ConeFPParams:
        """Kernel parameters in the volume's unit-voxel frame.

        Same float32 values as the reference (``kernels/cone_fp.py:
        302-339``) but computed on a copy: the caller's geometry is not
        normalised in place."""
        pg = _sequence(projection_geometry)
        normalize_(pg, volume_geometry)
        src = np.ascontiguousarray(pg.source_position.T)
        corner = np.ascontiguousarray(pg.detector_extent_min.T)
        u = np.ascontiguousarray(pg.u.T * pg.detector.pixel_width)
        v = np.ascontiguousarray(pg.v.T * pg.detector.pixel_height)
        arrays = (src[0], src[1], src[2], corner[0], corner[1], corner[2],
                  u[0], u[1], u[2], v[0], v[1], v[2])
        return ConeFPParams(arrays, RayDrivenConeFP._geom_axes(pg))

    def set_params(self, params):
        """Upload the per-angle parameters to the device."""
        if not self.is_compiled:
            raise KernelNotCompiledException(
                f"Compile {self.__class__.__name__} before setting its "
                "parameters.")
        if len(params) != 12 or any(len(p) != len(params[0]) for p in params):
            raise ValueError("Expected 12 equally long parameter arrays.")
        n = len(params[0])
        rec = np.zeros(n, _native.FP_ANGLE_DTYPE)
        stack = np.stack([np.asarray(p, np.float32) for p in params], axis=1)
        rec["src"] = stack[:, 0:3]
        rec["corner"] = stack[:, 3:6]
        rec["u"] = stack[:, 6:9]
        rec["v"] = stack[:, 9:12]
        axes = getattr(params, "axes", None)
        self._axes_known = axes is not None
        rec["axis"] = axes if axes is not None else 0
        rec["index"] = np.arange(n)
        self._host_params = rec
        self._upload()
        self._n_params = n

    def _upload(self):
        """Upload the records interleaved by ray axis, so that every part
        of the launch mixes texture-unit and CUDA-core work."""
        rec = self._host_params.copy()
        key = np.empty(len(rec))
        f = float(self.cuda_core_fraction)
        g = max(int(self.axis_group), 1)
        for ax in range(3):
            sel = np.flatnonzero(rec["axis"] == ax)
            pos = np.arange(len(sel))
            # groups of g consecutive records of one axis alternate
            # between the axes
            key[sel] = ((pos // g + 0.5) / max((len(sel) + g - 1) // g, 1)
                        + 1e-6 * ax + 1e-12 * pos)
            # an evenly spread share of the texture-path records is traced
            # on the CUDA cores instead (the kernel ignores the flag for
            # records without a texture path)
            core = np.floor((pos + 1) * f) > np.floor(pos * f)
            rec["flags"][sel] = np.where(core, _native.KK_FP_NO_TEXTURE, 0)
        order = np.argsort(key, kind="stable")
        t = _arrays.torch()
        self._params_dev = t.from_numpy(
            np.ascontiguousarray(rec[order]).view(np.uint8)).cuda()

    def _ensure_axes(self, projection_geometry, volume_geometry):
        if self._axes_known:
            return
        pg = _sequence(projection_geometry)
        normalize_(pg, volume_geometry)
        self._host_params["axis"] = self._geom_axes(pg)
        self._upload()
        self._axes_known = True

    def _volume_texture(self, vol, vdesc):
        """Layered texture of ``vol`` (one layer per slice of its slowest
        axis), refilled from ``vol``; None when the texture unit is not
        used for this call."""
        t = _arrays.torch()
        # The texture unit filters 16-bit texels in reduced precision while
        # the reference's arithmetic is float32, so 16-bit volumes use a
        # (float16) texture only when half_texture allows it, for 16-bit
        # storage runs whose tolerance is that of the storage anyway.
        half = vol.dtype in (t.float16, t.bfloat16)
        if (not self.use_texture_unit or self._interp != _native.KK_INTERP_TEX8
                or (half and not self.half_texture)
                or vol.dtype not in (t.float32, t.float16, t.bfloat16)
                or not vol.is_contiguous() or vol.shape[0] > 2048):
            return None
        slowest = self._vol_axs[0]
        if not np.any(self._host_params["axis"] == slowest):
            return None
        code = _native.KK_F16 if half else _native.KK_F32
        lay = self._vtex
        if lay is None or lay.shape != tuple(vol.shape) or lay.dtype != code:
            lay = _native.Layered(*vol.shape, code)
            self._vtex = lay
        src = vol
        if vol.dtype == t.bfloat16:  # texels are float16: convert first
            stage = getattr(self, "_half_stage", None)
            if stage is None or stage.shape != vol.shape:
                stage = t.empty(vol.shape, dtype=t.float16, device=vol.device)
                self._half_stage = stage
            stage.copy_(vol)
            src = stage
        lay.copy_from(src)
        return lay

    # -- launch -------------------------------------------------------------
    def _output(self, projections, projection_geometry, projections_pitch):
        """(descriptor, keep-alive objects) for the projections argument."""
        t = _arrays.torch()
        if isinstance(projections, (list, tuple)):
            if self._proj_axs[0] != 0:
                raise ValueError(
                    "A list of projections requires projection_axes[0] == 0.")
            return list_desc(projections, self._proj_axs)
        arr = _arrays.as_tensor(projections)
        if arr.dtype == t.int64 and arr.dim() == 1:
            # the reference's low-level form: device table of per-angle
            # pointers, optionally into pitched rows
            if self._proj_axs[0] != 0:
                raise NotImplementedError(
                    "Pointer tables are supported along the angle axis only.")
            rows = int(projection_geometry.detector.rows[0])
            cols = int(projection_geometry.detector.cols[0])
            pitch = projections_pitch or (len(arr), rows, cols)
            if self._proj_axs == (0, 1, 2):
                rs, cs = pitch[2], 1
            else:
                rs, cs = 1, pitch[1]
            d = _native.table_desc(arr, len(arr), rows, cols, rs, cs,
                                   _native.KK_F32)
            return d, (arr,)
        return _native.projections_desc(arr, self._proj_axs), (arr,)

    def __call__(self, volume_texture, projection_geometry,
                 volume_geometry: VolumeGeometry, projections,
                 projections_pitch: tuple | None = None,
                 additive: bool = True):
        """Project ``volume_texture`` into ``projections``.

        As in the reference the result is added to ``projections``; pass
        ``additive=False`` to overwrite instead (saves zero-filling).
        ``volume_texture`` is a ``Texture`` from ``copy_to_texture`` or a
        device array laid out by ``volume_axes``; ``projections`` a device
        array laid out by ``projection_axes``, a list of 2D device arrays,
        or an int64 device array of per-angle pointers."""
        if volume_texture is None:
            raise ValueError("`volume_texture` is None.")
        if not self.is_compiled:
            raise KernelNotCompiledException(
                "Please compile the kernel with `compile()`.")
        if not self._params_are_set:
            raise KernelMemoryUnpreparedException(
                "Please set the projection geometry with `set_params()`.")
        if not isinstance(projection_geometry, ProjectionGeometrySequence):
            projection_geometry = ProjectionGeometrySequence.fromList(
                projection_geometry)
        if len(projection_geometry) != self._n_params:
            raise ValueError(
                f"Parameters were set for {self._n_params} angles, but the "
                f"geometry has {len(projection_geometry)}.")
        self._ensure_axes(projection_geometry, volume_geometry)
        vol = (volume_texture.array if isinstance(volume_texture, Texture)
               else _arrays.as_tensor(volume_texture))
        vdesc = _native.volume_desc(vol, self._vol_axs)
        expect = tuple(int(s) for s in volume_geometry.shape)
        if tuple(vdesc.shape) != expect:
            raise ValueError(
                f"Volume of world shape {tuple(vdesc.shape)} does not match "
                f"the volume geometry {expect}.")
        pdesc, keep = self._output(projections, projection_geometry,
                                   projections_pitch)
        if pdesc.n_angles != self._n_params:
            raise ValueError(
                f"{pdesc.n_angles} projections given for {self._n_params} "
                "angles.")
        det = projection_geometry.detector
        if (pdesc.rows, pdesc.cols) != (int(det.rows[0]), int(det.cols[0])):
            raise ValueError(
                f"Projections of {pdesc.rows}x{pdesc.cols} pixels do not "
                f"match the detector {int(det.rows[0])}x{int(det.cols[0])}.")
        osc = np.asarray(self._output_scale(volume_geometry.voxel_size),
                         np.float32).reshape(9)
        lay = self._volume_texture(vol, vdesc)
        self._launch(vdesc, pdesc, osc, lay, None, additive)
        del keep

    def _sums(self, pdesc):
        """(pointer, elements) of the running-sum buffer for 16-bit
        projections, allocated once per projector and device."""
        if pdesc.dtype == _native.KK_F32 or self.sums_bytes <= 0:
            return None, 0
        per = int(pdesc.rows) * int(pdesc.cols)
        n = min(int(pdesc.n_angles), max(1, int(self.sums_bytes) // (4 * per)))
        t = _arrays.torch()
        buf = getattr(self, "_sums_buf", None)
        dev = t.cuda.current_device()
        if buf is None or buf.numel() < n * per or buf.device.index != dev:
            buf = t.empty(n * per, dtype=t.float32, device="cuda")
            self._sums_buf = buf
        return buf.data_ptr(), buf.numel()

    def _padded(self, vdesc):
        """(pointer, elements) of the zero-padded volume copy's buffer,
        allocated once per projector, device, volume shape and type."""
        if not self.padded_copy or self._interp != _native.KK_INTERP_TEX8:
            return None, 0
        t = _arrays.torch()
        dt = {_native.KK_F32: t.float32, _native.KK_BF16: t.bfloat16,
              _native.KK_F16: t.float16}[int(vdesc.dtype)]
        n = int(np.prod([int(x) + 4 for x in vdesc.shape]))
        buf = getattr(self, "_pad_buf", None)
        dev = t.cuda.current_device()
        if (buf is None or buf.numel() != n or buf.dtype != dt
                or buf.device.index != dev):
            self._pad_buf = None
            buf = t.empty(n, dtype=dt, device="cuda")
            self._pad_buf = buf
        return buf.data_ptr(), buf.numel()

    def _options(self, lay, residual, additive, pdesc=None, vdesc=None
                 ) -> "_native.kk_fp_options":
        o = _native.kk_fp_options()
        if pdesc is not None:
            o.sums, o.sums_elems = self._sums(pdesc)
        if vdesc is not None:
            o.padded, o.padded_elems = self._padded(vdesc)
        o.interp = self._interp if lay is None else _native.KK_INTERP_TEX8
        o.slab = self.slices_per_block
        o.additive = int(bool(additive))
        o.span = int(_DEFAULT_SPAN if self.slices_per_launch is None
                     else self.slices_per_launch)
        o.flags = _native.KK_FP_OPT_TILES if self.use_tiles else 0
        o.vtex = None if lay is None else lay.handle
        o.residual = (None if residual is None
                      else ctypes.cast(ctypes.pointer(residual),
                                       ctypes.c_void_p))
        return o

    def _launch(self, vdesc, pdesc, osc, lay, residual, additive):
        o = self._options(lay, residual, additive, pdesc, vdesc)
        _native.check(_native.load().kk_cone_fp_ex(
            vdesc, pdesc, self._params_dev.data_ptr(), osc.ctypes.data, o,
            _native.current_stream()))
        del residual

    #: bytes of ray set-ups the exact adjoint keeps at once (angles are
    #: processed in chunks that fit, recomputing set-ups per chunk)
    adjoint_work_bytes = 1 << 29

    def transpose(self, projections, projection_geometry,
                  volume_geometry: VolumeGeometry, volume,
                  additive: bool = False):
        """Exact adjoint of ``__call__``: ``volume = A^T projections``
        (``+=`` with ``additive``), with exactly the weights the forward
        projection applies, so ``<A x, y> = <x, A^T y>`` up to float32
        rounding. ``projections`` is a float32 device array in the
        ``projection_axes`` layout (or a list of 2D arrays), ``volume`` a
        float32 device array in the ``volume_axes`` layout. The reference
        has no such operator; its autograd backward is the backprojector."""
        if not self._params_are_set:
            raise KernelMemoryUnpreparedException(
                "Please set the projection geometry with `set_params()`.")
        if not isinstance(projection_geometry, ProjectionGeometrySequence):
            projection_geometry = ProjectionGeometrySequence.fromList(
                projection_geometry)
        self._ensure_axes(projection_geometry, volume_geometry)
        t = _arrays.torch()
        vol = _arrays.as_tensor(volume)
        vdesc = _native.volume_desc(vol, self._vol_axs)
        expect = tuple(int(s) for s in volume_geometry.shape)
        if tuple(vdesc.shape) != expect:
            raise ValueError(
                f"Volume of world shape {tuple(vdesc.shape)} does not match "
                f"the volume geometry {expect}.")
        pdesc, keep = self._output(projections, projection_geometry, None)
        if pdesc.n_angles != self._n_params:
            raise ValueError(
                f"{pdesc.n_angles} projections given for {self._n_params} "
                "angles.")
        per = int(pdesc.rows) * int(pdesc.cols)
        chunk = max(1, min(self._n_params,
                           int(self.adjoint_work_bytes) // (20 * per)))
        need = 5 * chunk * per
        work = getattr(self, "_adj_work", None)
        if work is None or work.numel() < need or work.device != vol.device:
            work = t.empty(need, dtype=t.float32, device=vol.device)
            self._adj_work = work
        osc = np.asarray(self._output_scale(volume_geometry.voxel_size),
                         np.float32).reshape(9)
        _native.check(_native.load().kk_cone_fp_adjoint(
            pdesc, vdesc, self._params_dev.data_ptr(), osc.ctypes.data,
            self._interp, self.slices_per_block, int(bool(additive)),
            work.data_ptr(), work.numel(), _native.current_stream()))
        del keep

    def residual(self, volume, projection_geometry,
                 volume_geometry: VolumeGeometry, out, measured, weight):
        """Fused SIRT residual step: ``out = (A volume - measured) * weight``
        (one kernel; reference ``algo.py:339-344``). All arrays are float32
        device arrays in the ``projection_axes`` layout."""
        if not self._params_are_set:
            raise KernelMemoryUnpreparedException(
                "Please set the projection geometry with `set_params()`.")
        self._ensure_axes(projection_geometry, volume_geometry)
        vdesc = _native.volume_desc(volume, self._vol_axs)
        pdesc = _native.projections_desc(out, self._proj_axs)
        for name, a in (("measured", measured), ("weight", weight)):
            if a.shape != out.shape or a.stride() != out.stride():
                raise ValueError(f"`{name}` must have the layout of `out`.")
        res = _native.kk_fp_residual(measured.data_ptr(), weight.data_ptr())
        osc = np.asarray(self._output_scale(volume_geometry.voxel_size),
                         np.float32).reshape(9)
        lay = self._volume_texture(volume, vdesc)
        self._launch(vdesc, pdesc, osc, lay, res, False)


#: span of projectors whose ``slices_per_launch`` is None
_DEFAULT_SPAN = 0


def set_slices_per_launch(slices: int = 0) -> None:
    """How many slices of every ray's own slice axis one forward-projection
    launch traces (float32 projections) for projectors that do not set
    ``slices_per_launch`` themselves: 0 = the library's automatic span
    (one launch up to 256 slices, 192 slices up to 640, 128 beyond), -1 =
    the whole ray in one launch. Results are the same bit for bit;
    shorter spans keep the volume band each launch reads in L2."""
    global _DEFAULT_SPAN
    if int(slices) < -1:
        raise ValueError(f"slices must be >= -1, got {slices}")
    _DEFAULT_SPAN = int(slices)


def launches_per_projection(max_slices: int, slab: int = 16,
                            float32: bool = True, span: int = None,
                            sums: bool = False) -> int:
    """Kernel launches of one forward projection of a volume whose longest
    axis has ``max_slices`` voxels (16-bit projections: per chunk of
    angles when a running-sum buffer is used, else one)."""
    if not float32 and not sums:
        return 1
    return int(_native.load().kk_fp_launches_ex(
        int(max_slices), int(slab),
        _native.KK_F32 if float32 else _native.KK_F16,
        int(_DEFAULT_SPAN if span is None else span)))


__all__ = ["RayDrivenConeFP", "ConeFPParams", "set_slices_per_launch",
           "launches_per_projection"]
