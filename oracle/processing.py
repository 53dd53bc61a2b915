"""FP64 NumPy restatement of KernelKit's FDK pre-processing and of the FDK
and SIRT algorithms (test infrastructure only; see the package docstring).

* ``preweight`` follows ``processing.py:149-188``: every pixel is scaled by
  |d - s| / |pixel - s| in float64, the pixel taken at its corner.
* ``filter_rows`` follows ``processing.py:96-126``: each row is zero-padded
  to P = max(64, 2^ceil(log2(2 cols))) samples and multiplied in the
  Fourier domain by the filter of ``ramlak_fourier``.
* ``fdk`` chains them with a backprojector (``algo.py:169-223``).
* ``sirt`` is the update of ``algo.py:226-368`` around caller-given
  forward/backprojection functions.
"""
from __future__ import annotations

import numpy as np


def ramlak_fourier(num: int, name: str = "ramlak") -> np.ndarray:
    """Frequency response of the row filter (``processing.py:44-93``):
    the Ram-Lak kernel sampled in the spatial domain (1/4 at 0,
    -1/(pi n)^2 at odd n, 0 at even n), circularly placed and transformed;
    'cosine' additionally multiplies by a half-period-shifted sine."""
    assert num % 2 == 0
    n = np.concatenate((np.arange(0, num // 2 + 1), np.arange(num // 2 - 1, 0,
                                                               -1)))
    g = np.zeros(num)
    g[0] = 0.25
    g[1::2] = -1.0 / (np.pi * n[1::2]) ** 2
    H = 4 * np.real(np.fft.fft(g))
    if name.lower() == "cosine":
        H = H * np.fft.fftshift(np.sin(np.linspace(0, np.pi, num,
                                                   endpoint=False)))
    elif name.lower() not in ("ramp", "ramlak"):
        raise ValueError(name)
    return H


def filter_rows(projections, name: str = "ramlak") -> np.ndarray:
    """Filtered copy (float32) of (n, rows, cols) projections."""
    p = np.asarray(projections, np.float64)
    cols = p.shape[-1]
    P = max(64, int(2 ** int(np.ceil(np.log2(2 * cols)))))
    H = ramlak_fourier(P, name)
    pad = np.zeros(p.shape[:-1] + (P,))
    pad[..., :cols] = p
    out = np.real(np.fft.ifft(np.fft.fft(pad, axis=-1) * H, axis=-1))
    return out[..., :cols].astype(np.float32)


def preweight(projections, geoms) -> np.ndarray:
    """Pre-weighted copy (float32) of (n, rows, cols) projections for a
    list of geometries (any objects with source_position,
    detector_position, detector_extent_min, u, v, detector)."""
    p = np.asarray(projections, np.float32)
    out = np.empty_like(p)
    rows, cols = p.shape[1], p.shape[2]
    r = np.arange(rows)[:, None, None]
    c = np.arange(cols)[None, :, None]
    for i, g in enumerate(geoms):
        central = np.linalg.norm(g.detector_position - g.source_position)
        pix = (np.array(g.detector_extent_min, np.float64)
               + c * np.array(g.u * g.detector.pixel_width, np.float64)
               + r * np.array(g.v * g.detector.pixel_height, np.float64))
        d = pix - np.array(g.source_position, np.float64)
        dist = np.sqrt((d[..., 0] * d[..., 0] + d[..., 1] * d[..., 1])
                       + d[..., 2] * d[..., 2])
        out[i] = (p[i].astype(np.float64) * (np.float64(central) / dist)
                  ).astype(np.float32)
    return out


def fdk(projections, geoms, backproject, name: str = "ramlak"):
    """FDK: pre-weight, filter, then ``backproject`` (a function of the
    filtered (n, rows, cols) projections)."""
    return backproject(filter_rows(preweight(projections, geoms), name))


def sirt(y, forward, backward, vol_shape, iters, mask=None, vmin=None,
         vmax=None):
    """SIRT in float64: x <- clip(mask (x - C A^T (R (A x - y)))) with
    C = 1 / A^T 1, R = 1 / A 1 (infinities -> 0), x_0 = 0."""
    with np.errstate(divide="ignore"):
        C = 1.0 / backward(np.ones_like(y, np.float64))
        R = 1.0 / forward(np.ones(vol_shape, np.float64))
    C[np.isinf(C)] = 0.0
    R[np.isinf(R)] = 0.0
    x = np.zeros(vol_shape, np.float64)
    for _ in range(iters):
        x = x - C * backward(R * (forward(x) - y))
        if mask is not None:
            x = x * mask
        if vmin is not None or vmax is not None:
            x = np.clip(x, vmin, vmax)
    return x
