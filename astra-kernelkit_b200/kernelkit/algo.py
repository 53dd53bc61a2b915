"""Reconstruction algorithms: forward/back projection helpers, FDK and SIRT.

Mirrors ``kernelkit/algo.py`` of the reference (signatures, defaults and
return conventions: host NumPy arrays unless device output is requested).
SIRT runs two fused kernels per iteration, ``(A x - y) R`` in the forward
projection's epilogue and ``x = clip(mask (x - C A^T r))`` in the
backprojection's, and replays them from a CUDA graph when no per-iteration
host work is requested.
"""
from __future__ import annotations

from typing import Any, Callable, Sequence

import numpy as np

from . import _arrays, _native
from .geom.proj import Beam, ProjectionGeometrySequence
from .geom.vol import VolumeGeometry
from .kernel import BaseKernel
from .kernels.cone_bp import VoxelDrivenConeBP
from .kernels.cone_fp import RayDrivenConeFP
from .operator import XrayTransform
from .processing import filter as filt
from .processing import preweight
from .projector import BackProjector


def _host_copy(dev):
    """A host copy of a device tensor in pinned memory, as the reference
    returns its results (``algo.py:46-48, 122-126``): the copy runs at
    full bus speed and torch's host allocator reuses the pinned block."""
    t = _arrays.torch()
    host = t.empty(dev.shape, dtype=dev.dtype, pin_memory=True)
    host.copy_(dev)
    return host.numpy()


def _to_host(dev, out=None):
    host = _host_copy(dev) if out is None else None
    if out is None:
        return host
    if isinstance(out, np.ndarray):
        out[...] = dev.cpu().numpy()
        return out
    return out


def fp(volume: Any, projection_geometry, volume_geometry: VolumeGeometry,
       out=None):
    """X-ray forward projection (``algo.py:18-49``). Returns a host array
    unless ``out`` is a device array, which is then filled and returned."""
    t = _arrays.torch()
    op = XrayTransform(projection_geometry, volume_geometry)
    vol = _arrays.as_tensor(volume, dtype=t.float32)
    dev_out = out if (out is not None and _arrays.is_device_array(out)) \
        else None
    result = op(vol, out=_arrays.as_tensor(dev_out) if dev_out is not None
                else None)
    if dev_out is not None:
        return out
    return _to_host(result, out)


#: angles per streamed chunk: the backprojector's own summation chunk, so
#: chunked and whole-scan backprojections add in the same order
_CHUNK = 32
_STREAM: dict = {}


def _stream_buffers(rows: int, cols: int) -> dict:
    """Two-slot ring of pinned staging blocks, device blocks and 32-layer
    textures for streaming host projections, kept for the most recent
    detector shape (about 6 x 75 MB at 768^2)."""
    t = _arrays.torch()
    key = (rows, cols)
    st = _STREAM.get(key)
    if st is None:
        _STREAM.clear()
        shape = (_CHUNK, rows, cols)
        st = {"host": [t.empty(shape, dtype=t.float32, pin_memory=True)
                       for _ in range(2)],
              "dev": [t.empty(shape, dtype=t.float32, device="cuda")
                      for _ in range(2)],
              "tex": {},  # layers -> two textures
              "copy": t.cuda.Stream()}
        _STREAM[key] = st
    return st


def release_stream_buffers() -> None:
    """Free the staging, device and texture ring that ``bp``/``fdk`` keep
    between calls for the last detector shape (waits for its last use)."""
    st = _STREAM.pop(next(iter(_STREAM)), None) if _STREAM else None
    if st is not None and st.get("last") is not None:
        st["last"].synchronize()


def _can_stream(projections, projection_geometry, volume_geometry, preproc_fn,
                kernel, out, projection_axes, kwargs) -> bool:
    """The chunked path takes host (NumPy) projections, or a C-contiguous
    float32 device array, in the default layout with the default
    backprojector; anything else goes through the general path."""
    if isinstance(projections, np.ndarray):
        if (projections.ndim != 3 or not projections.dtype.isnative
                or not np.issubdtype(projections.dtype, np.floating)
                or any(s < 0 for s in projections.strides)):
            return False
    elif _arrays.is_device_array(projections):
        t = _arrays.torch()
        d = _arrays.as_tensor(projections)
        if d.dim() != 3 or d.dtype != t.float32 or not d.is_contiguous():
            return False
    else:
        return False
    if preproc_fn is not None or kwargs:
        return False
    if kernel is not None and not (
            type(kernel) is VoxelDrivenConeBP
            and kernel._interp == _native.KK_INTERP_TEX8
            and tuple(kernel._vol_axs) == (0, 1, 2)
            and tuple(kernel._proj_axs) == (0, 1, 2)):
        return False
    if tuple(projection_axes) != (0, 1, 2):
        return False
    if out is not None and not isinstance(out, np.ndarray):
        return False
    if not volume_geometry.has_isotropic_voxels():
        return False
    if len(projections) == 0 or len(projection_geometry) != len(projections):
        return False
    det = (projection_geometry.detector
           if isinstance(projection_geometry, ProjectionGeometrySequence)
           else projection_geometry[0].detector)
    return (int(np.asarray(det.rows).flat[0]), int(np.asarray(det.cols).flat[0])) \
        == projections.shape[1:]


def _streamed_bp(projections: np.ndarray, projection_geometry,
                 volume_geometry: VolumeGeometry, filter: Any,
                 kernel: VoxelDrivenConeBP = None):
    """Backprojection (with FDK pre-weighting and filtering when ``filter``
    is given) in stages of 32 angles (host input) or 128 angles (device
    input) through a two-slot ring of textures, so no whole-scan texture
    is allocated. Host projections are
    streamed: while the host stages chunk c+1 into pinned memory and a
    copy stream uploads it, the GPU pre-weights and filters chunk c,
    copies it into a texture and backprojects it onto the volume; the
    caller's array is left untouched (the reference also processes a
    device copy). Device projections are pre-weighted and filtered in
    place, as in the reference, then backprojected chunk by chunk. Every
    kernel is the one of the whole-scan path, on the same angles and in the
    same summation order, so the volume is bit for bit the same."""
    from . import processing

    t = _arrays.torch()
    L = _native.load()
    n, rows, cols = projections.shape
    st = _stream_buffers(rows, cols)
    cs = t.cuda.current_stream()
    stream = _native.current_stream()
    K = kernel if kernel is not None else VoxelDrivenConeBP()
    K.compile()
    K.set_params(K.geoms2params(projection_geometry, volume_geometry))
    vol = t.empty(tuple(int(s) for s in volume_geometry.shape),
                  dtype=t.float32, device="cuda")
    vdesc = _native.volume_desc(vol, K._vol_axs)
    vox_vol = float(np.float32(volume_geometry.voxel_volume()))
    params = K._params_dev.data_ptr()
    if filter is not None:
        pw = t.from_numpy(processing.preweight_params(
            projection_geometry)).cuda()
        P = processing.padded_length(cols)
        if P <= processing.FFT_MAX_P:
            plan = processing.device_plan(P, filter)
        else:
            h = processing._device_filter(P, filter)
    if st.get("last") is not None:
        # the ring's previous user may run on another stream
        cs.wait_event(st["last"])
        st["copy"].wait_event(st["last"])
    on_host = isinstance(projections, np.ndarray)
    if on_host:
        src = t.from_numpy(projections)
    else:
        src = _arrays.as_tensor(projections)

    def fill(tex, chunk, a, in_place):
        """Pre-weight, filter and store one chunk into its texture in one
        pass (device input is also rewritten in place, as the reference
        pre-processes it), or copy it when there is no filter."""
        if filter is None:
            tex.copy_from(chunk)
            return
        d = _native.projections_desc(chunk)
        if P > processing.FFT_MAX_P:  # rows beyond the FFT's reach
            _native.check(L.kk_preweight(d, pw.data_ptr() + a * 13 * 8,
                                         stream))
            _native.check(L.kk_filter_rows(d, h.data_ptr(), P, stream))
            tex.copy_from(chunk)
            return
        _native.check(L.kk_fdk_filter(
            d, pw.data_ptr() + a * 13 * 8, plan.data_ptr(), P,
            d if in_place else None, tex.handle, 0, stream))
    staged, used = [None, None], [None, None]
    # device input: four chunks per stage, so that each BP launch covers
    # four 32-angle chunks (added one by one, as in the whole-scan path);
    # host input: one chunk per stage, for a finer overlap with the copies
    step = _CHUNK if on_host else 4 * _CHUNK
    for c, a in enumerate(range(0, n, step)):
        m, b = min(step, n - a), c & 1
        texs = st["tex"].get(m)
        if texs is None:
            texs = [_native.Layered(m, rows, cols, _native.KK_F32)
                    for _ in range(2)]
            st["tex"][m] = texs
        if not on_host:
            fill(texs[b], src[a:a + m], a, True)
            _native.check(L.kk_cone_bp_layered(
                texs[b].handle, vdesc, params + a * 12 * 4, vox_vol,
                int(c > 0), 0, stream))
            continue
        if staged[b] is not None:
            staged[b].synchronize()  # the upload from this block is done
        host = st["host"][b][:m]
        host.copy_(src[a:a + m])
        dev = st["dev"][b][:m]
        with t.cuda.stream(st["copy"]):
            if used[b] is not None:
                st["copy"].wait_event(used[b])
            dev.copy_(host, non_blocking=True)
            staged[b] = t.cuda.Event()
            staged[b].record(st["copy"])
        cs.wait_event(staged[b])
        fill(texs[b], dev, a, False)
        used[b] = t.cuda.Event()
        used[b].record(cs)
        _native.check(L.kk_cone_bp_layered(
            texs[b].handle, vdesc, params + a * 12 * 4, vox_vol,
            int(c > 0), 0, stream))
    st["last"] = t.cuda.Event()
    st["last"].record(cs)
    return vol


def bp(projections: Any, projection_geometry, volume_geometry: VolumeGeometry,
       filter: Any = None, preproc_fn: Callable = None,
       kernel: BaseKernel = None, out=None,
       projection_axes: Sequence[int] = (0, 1, 2), **kwargs):
    """X-ray backprojection, optionally with FDK pre-weighting and
    filtering (``algo.py:52-126``). Device float32 projections are
    pre-processed in place, as in the reference. Host (NumPy) projections
    are streamed to the GPU in 32-angle chunks that overlap the upload
    with the pre-processing and backprojection of the previous chunk.
    Returns a host array (or fills a host ``out``)."""
    t = _arrays.torch()
    if _can_stream(projections, projection_geometry, volume_geometry,
                   preproc_fn, kernel, out, projection_axes, kwargs):
        vol = _streamed_bp(projections, projection_geometry, volume_geometry,
                           filter, kernel)
        if isinstance(out, np.ndarray):
            out[...] = vol.cpu().numpy()
            return out
        return _host_copy(vol)
    if out is not None and _arrays.is_device_array(out):
        out_gpu = _arrays.as_tensor(out, dtype=t.float32)
    else:
        out_gpu = t.zeros(tuple(int(s) for s in volume_geometry.shape),
                          dtype=t.float32, device="cuda")
    projections = _arrays.as_tensor(projections, dtype=t.float32)
    if preproc_fn is not None:
        preproc_fn(projections, projection_geometry)
    if filter is not None:
        if tuple(projection_axes) != (0, 1, 2):
            raise NotImplementedError()
        preweight(projections, projection_geometry)
        filt(projections, filter=filter)
    kwargs.pop("beam", None)
    kwargs.update(projection_axes=projection_axes)
    ptor = BackProjector(VoxelDrivenConeBP(**kwargs) if kernel is None
                         else kernel, texture_type="layered")
    ptor.projection_geometry = projection_geometry
    ptor.volume_geometry = volume_geometry
    ptor.projections = projections
    ptor.volume = out_gpu
    ptor()
    if isinstance(out, np.ndarray):
        out[...] = out_gpu.cpu().numpy()
        return out
    return _host_copy(out_gpu)


def fbp(projections: Any, projection_geometry, volume_geometry,
        filter: Any = "ramlak", **bp_kwargs):
    """Parallel-beam FBP is not implemented (as in the reference,
    ``algo.py:129-166``)."""
    raise NotImplementedError(
        "FBP is not implemented yet. Use a conebeam geometry with the `bp` "
        "function, or file an issue.")


def fdk(projections: Any, projection_geometry: Any,
        volume_geometry: VolumeGeometry, filter: Any = "ramlak", **bp_kwargs):
    """Feldkamp-Davis-Kress reconstruction (``algo.py:169-223``):
    pre-weighting, row filtering, then backprojection with the adjoint
    scaling of ``VoxelDrivenConeBP``. No extra angular normalisation is
    applied, exactly as in the reference."""
    beams = ([projection_geometry.beam]
             if isinstance(projection_geometry, ProjectionGeometrySequence)
             else [p.beam for p in projection_geometry])
    if any(b != Beam.CONE for b in beams):
        raise NotImplementedError(
            "Only cone beam geometry is supported at the moment.")
    if "kernel" not in bp_kwargs:
        bp_kwargs.update(kernel=VoxelDrivenConeBP())
    return bp(projections, projection_geometry, volume_geometry,
              filter=filter, **bp_kwargs)


class SIRT:
    """Reusable SIRT solver state (device buffers, kernel parameters and an
    optional captured CUDA graph of one iteration).

    ``x <- clip(mask * (x - C * A^T (R * (A x - y))))`` with
    ``C = 1 / A^T 1`` and ``R = 1 / A 1`` (``+inf -> 0``), ``x_0 = 0``
    (``algo.py:226-368``)."""

    def __init__(self, projections, projection_geometry,
                 volume_geometry: VolumeGeometry, mask=None,
                 min_constraint: float = None, max_constraint: float = None,
                 interpolation: str = "texture", volume_dtype=None,
                 projection_dtype=None):
        """``volume_dtype`` / ``projection_dtype`` (torch dtypes, default
        float32) choose the storage of the iterate, ``C`` and the mask, and
        of the measured data, ``R`` and the residual: 16-bit storage
        (``torch.bfloat16`` / ``torch.float16`` volumes, ``torch.float16``
        projections) keeps FP32 accumulation inside every projection and
        samples float16 textures."""
        t = _arrays.torch()
        if len(projections) != len(projection_geometry):
            raise ValueError(
                "Number of projections does not match number of geometries.")
        vdt = volume_dtype or t.float32
        pdt = projection_dtype or t.float32
        if vdt not in (t.float32, t.bfloat16, t.float16) or pdt not in (
                t.float32, t.float16) or ((vdt == t.float32) != (pdt == t.float32)):
            raise NotImplementedError(
                "SIRT storage: float32 throughout, or a bfloat16/float16 "
                "volume with float16 projections.")
        half = vdt != t.float32
        self.vg = volume_geometry
        self.pg = projection_geometry
        self.y = _arrays.as_tensor(projections).to(pdt).contiguous()
        if self.y.dim() != 3:
            raise ValueError("Projections must be (angles, rows, cols).")
        shape = tuple(int(s) for s in volume_geometry.shape)
        self.fp = RayDrivenConeFP(interpolation=interpolation)
        self.fp.half_texture = half
        self.fp.compile()
        self.fp.set_params(self.fp.geoms2params(projection_geometry,
                                                volume_geometry))
        self.bp = VoxelDrivenConeBP(interpolation=interpolation)
        self.bp.compile()
        self.bp.set_params(self.bp.geoms2params(projection_geometry,
                                                volume_geometry))
        self.x = t.zeros(shape, dtype=vdt, device="cuda")
        self.mask = (None if mask is None
                     else _arrays.as_tensor(mask).to(vdt).contiguous())
        self.min_c, self.max_c = min_constraint, max_constraint
        L = _native.load()
        stream = _native.current_stream()
        # C = 1 / A^T 1 and R = 1 / A 1, formed in float32
        C = t.empty(shape, dtype=t.float32, device="cuda")
        ones = t.ones(self.y.shape, dtype=t.float32, device="cuda")
        self.bp(ones, C, volume_geometry, additive=False)
        _native.check(L.kk_reciprocal(C.data_ptr(), C.numel(), stream))
        del ones
        self.C = C if not half else C.to(vdt)
        del C
        R = t.empty(self.y.shape, dtype=t.float32, device="cuda")
        ones = t.ones(shape, dtype=t.float32, device="cuda")
        self.fp(ones, self.pg, volume_geometry, R, additive=False)
        _native.check(L.kk_reciprocal(R.data_ptr(), R.numel(), stream))
        del ones
        self.R = R if not half else R.to(pdt)
        del R
        # make the forward projector's volume texture for the iterate's
        # storage type now, and its padded volume copy: they cannot be
        # created during graph capture
        self.fp._volume_texture(self.x, _native.volume_desc(self.x))
        self.fp._padded(_native.volume_desc(self.x))
        self.y_tmp = t.empty_like(self.y)
        # the backprojection samples the residual through a layered
        # texture (the reference's filter), refilled every iteration
        self.tex = (_native.Layered(*self.y.shape, _native.KK_F16 if half
                                    else _native.KK_F32)
                    if interpolation == "texture" and len(self.y) <= 2048
                    else None)
        self.bp._work_for(self.x, True)  # allocate before any graph capture
        self._graph = None

    def step(self):
        """One iteration: forward projection with the residual epilogue,
        (texture refill) and backprojection with the update epilogue."""
        self.fp.residual(self.x, self.pg, self.vg, self.y_tmp, self.y, self.R)
        src = self.y_tmp
        if self.tex is not None:
            self.tex.copy_from(self.y_tmp)
            src = self.tex
        self.bp.update(src, self.x, self.vg, self.C, self.mask,
                       self.min_c, self.max_c)

    def capture(self):
        """Capture one iteration into a CUDA graph (no work runs)."""
        t = _arrays.torch()
        g = t.cuda.CUDAGraph()
        s = t.cuda.Stream()
        s.wait_stream(t.cuda.current_stream())
        with t.cuda.stream(s):
            with t.cuda.graph(g, stream=s):
                self.step()
        t.cuda.current_stream().wait_stream(s)
        self._graph = g
        return g

    def run(self, iters: int, use_graph: bool = True, callback=None,
            progress=None):
        for i in range(iters):
            if use_graph:
                if self._graph is None:
                    self.capture()
                self._graph.replay()
            else:
                self.step()
            if progress is not None:
                progress(i)
            if callback is not None:
                callback(i, self.x, self.y_tmp)
        return self.x


def sirt(projections: np.ndarray, projection_geometry: Any,
         volume_geometry: VolumeGeometry, iters: int = 100,
         verbose: bool = True, mask: Any = None,
         min_constraint: float = None, max_constraint: float = None,
         return_gpu: bool = False, callback: callable = None,
         residual_every: int = 10, use_graph: bool | None = None):
    """Simultaneous Iterative Reconstruction Technique (``algo.py:226-368``).

    Projections are (angles, rows, cols). Returns the volume as a host
    array, or as a device tensor with ``return_gpu``. ``callback(i, x,
    residual)`` runs after each iteration. The iteration is replayed from a
    CUDA graph unless a callback or the verbose residual display needs the
    host between iterations (``use_graph`` overrides)."""
    solver = SIRT(projections, projection_geometry, volume_geometry,
                  mask=mask, min_constraint=min_constraint,
                  max_constraint=max_constraint)
    show = verbose and residual_every is not None
    if use_graph is None:
        use_graph = callback is None and not show
    progress = None
    bar = None
    if verbose:
        from tqdm import tqdm

        bar = tqdm(total=iters, desc="SIRT")
        state = {"norm": ""}

        def progress(i):
            if show:
                E = residual_every
                if i % E == 0:
                    state["norm"] = str(float(solver.y_tmp.norm()))
                desc = "SIRT [" + "*" * (i % E) + "." * (E - i % E) + "]"
                bar.set_description(f"{desc}: {state['norm']})")
            bar.update(1)
    x = solver.run(iters, use_graph=use_graph, callback=callback,
                   progress=progress)
    if bar is not None:
        bar.close()
    if return_gpu:
        return x
    return _host_copy(x)


__all__ = ["fp", "bp", "fbp", "fdk", "sirt", "SIRT", "release_stream_buffers"]
