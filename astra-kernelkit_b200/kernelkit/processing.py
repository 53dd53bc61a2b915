"""FDK pre-processing: cone-beam pre-weighting and detector-row filtering.

Mirrors ``kernelkit/processing.py`` of the reference. Both steps run as
CUDA kernels in float64 (``kk_preweight``; ``kk_fdk_filter``, a float64
FFT filter as the reference's, or ``kk_filter_rows``, a direct circular
convolution, for padded rows beyond 8192) and update the projections in
place, as the reference does. NumPy input is processed on the device and
written back. FDK fuses both with the texture store (``kk_fdk_filter``).
"""
from __future__ import annotations

from functools import lru_cache

import numpy as np

from . import _arrays, _native


@lru_cache
def _filter(num: int, filter_name: str = "ramlak", use_cupy: bool = False):
    """Frequency response (float64, length ``num``) of the row filter.

    Ram-Lak is built from its spatial-domain samples (Kak & Slaney, ch. 3):
    h[0] = 1/4, h[n] = -1/(pi n)^2 for odd n, 0 for even n != 0, placed
    circularly on ``num`` points and transformed, H = 4 Re(FFT(h)); this
    avoids the cupping of a sampled |f| ramp. 'cosine' multiplies H by
    sin(pi k / num) rotated by half a period. Same construction as the
    reference (``processing.py:44-93``)."""
    if num % 2:
        raise ValueError("Filter must be even.")
    n = np.concatenate((np.arange(0, num // 2 + 1),
                        np.arange(num // 2 - 1, 0, -1)))
    h = np.zeros(len(n))
    h[0] = 0.25
    h[1::2] = -1.0 / (np.pi * n[1::2]) ** 2
    H = 4 * np.real(np.fft.fft(h))
    name = filter_name.lower()
    if name in ("ramp", "ramlak"):
        pass
    elif name == "cosine":
        H = H * np.fft.fftshift(np.sin(np.linspace(0, np.pi, num,
                                                   endpoint=False)))
    else:
        raise ValueError(f"Filter with `filter_name` {filter_name} not known "
                         "or not yet implemented.")
    return H


def padded_length(cols: int) -> int:
    """Zero-padded row length: the next power of two >= 2 cols, at least
    64 (``processing.py:111-113``)."""
    return max(64, int(2 ** int(np.ceil(np.log2(2 * cols)))))


@lru_cache
def impulse_response(num: int, filter_name: str = "ramlak") -> np.ndarray:
    """Circular impulse response of the row filter: filtering a zero-padded
    row by ``H`` equals circular convolution with ``Re(IFFT(H))``."""
    return np.ascontiguousarray(np.real(np.fft.ifft(_filter(num,
                                                            filter_name))))


_DEVICE_FILTERS: dict = {}

#: largest padded length the one-pass FFT filter (kk_fdk_filter) handles
FFT_MAX_P = 8192


def _device_filter(num, name):
    key = (num, name.lower())
    if key not in _DEVICE_FILTERS:
        t = _arrays.torch()
        _DEVICE_FILTERS[key] = t.from_numpy(impulse_response(num, name)).cuda()
    return _DEVICE_FILTERS[key]


def device_plan(num, name):
    """The ``kk_fdk_filter`` plan (device float64) of the filter's
    frequency response for padded length ``num``."""
    key = ("plan", num, name.lower())
    if key not in _DEVICE_FILTERS:
        t = _arrays.torch()
        L = _native.load()
        H = t.from_numpy(np.ascontiguousarray(_filter(num, name),
                                              np.float64)).cuda()
        plan = t.empty(int(L.kk_fdk_plan_size(num)), dtype=t.float64,
                       device="cuda")
        _native.check(L.kk_fdk_plan(plan.data_ptr(), H.data_ptr(), num,
                                    _native.current_stream()))
        _DEVICE_FILTERS[key] = plan
    return _DEVICE_FILTERS[key]


def _as_stack(projections):
    """Device descriptor and writeback closure for 3D arrays, lists of 2D
    arrays (device or NumPy)."""
    t = _arrays.torch()
    if isinstance(projections, (list, tuple)):
        dev = [_arrays.as_tensor(p) for p in projections]
        for p in dev:
            if p.dtype != t.float32:
                raise NotImplementedError("float32 projections only.")
        from .kernels.cone_fp import list_desc

        desc, keep = list_desc(dev, (0, 1, 2))

        def writeback():
            for src, d in zip(projections, dev):
                if isinstance(src, np.ndarray):
                    src[...] = d.cpu().numpy()
        return desc, keep, writeback
    dev = _arrays.as_tensor(projections)
    if dev.dtype != t.float32:
        raise NotImplementedError("float32 projections only.")
    if dev.dim() != 3:
        raise ValueError("Projections must be (angles, rows, cols).")
    desc = _native.projections_desc(dev)

    def writeback():
        if isinstance(projections, np.ndarray):
            projections[...] = dev.cpu().numpy()
    return desc, (dev,), writeback


def filter(projections, verbose: bool = False, filter: str = "ramlak"):
    """Filter every detector row in place with the Ram-Lak ('ramp',
    'ramlak') or 'cosine' filter (``processing.py:96-126``): rows are
    zero-padded to ``padded_length(cols)`` and circularly convolved with
    the filter's impulse response, in float64."""
    desc, keep, writeback = _as_stack(projections)
    P = padded_length(int(desc.cols))
    if P <= FFT_MAX_P:
        # float64 FFT filtering in one pass, as the reference (cuFFT)
        plan = device_plan(P, filter)
        _native.check(_native.load().kk_fdk_filter(
            desc, None, plan.data_ptr(), P, desc, None, 0,
            _native.current_stream()))
    else:  # direct circular convolution with the impulse response
        h = _device_filter(P, filter)
        _native.check(_native.load().kk_filter_rows(
            desc, h.data_ptr(), P, _native.current_stream()))
    writeback()
    del keep


def preweight_params(geoms, detector_piercings=None) -> np.ndarray:
    """Per-angle float64 parameters of ``kk_preweight``: detector corner,
    u*pixel_width, v*pixel_height, source and the central-ray length
    |piercing - source| (piercing point defaults to the detector centre).
    Evaluated with each geometry's own dtypes, as ``processing.py:176-186``
    does."""
    out = np.empty((len(geoms), 13), np.float64)
    for i, g in enumerate(geoms):
        pierce = (g.detector_position if detector_piercings is None
                  else detector_piercings[i])
        out[i, 12] = np.linalg.norm(pierce - g.source_position)
        out[i, 0:3] = np.array(g.detector_extent_min)
        out[i, 3:6] = np.array(g.u * g.detector.pixel_width)
        out[i, 6:9] = np.array(g.v * g.detector.pixel_height)
        out[i, 9:12] = np.array(g.source_position)
    return out


def preweight(projections, geoms, detector_piercings: list = None,
              verbose: bool = False):
    """Multiply every pixel by |d - s| / |pixel - s| in place, the
    cone-beam ray-length weighting of FDK (``processing.py:149-188``).
    ``pixel`` is the pixel's corner position, as in the reference."""
    if len(geoms) != len(projections):
        raise ValueError("One geometry per projection is required.")
    desc, keep, writeback = _as_stack(projections)
    t = _arrays.torch()
    g = t.from_numpy(preweight_params(geoms, detector_piercings)).cuda()
    _native.check(_native.load().kk_preweight(desc, g.data_ptr(),
                                              _native.current_stream()))
    writeback()
    del keep, g


__all__ = ["filter", "preweight", "padded_length", "impulse_response"]
