"""Backprojection and FDK in 32-angle chunks through a ring of 32-layer
textures (``kernelkit.algo._streamed_bp``), for host (NumPy) projections
streamed to the GPU and for device arrays: the volume must be bit for bit
the one of the whole-scan path (one texture of all angles), for angle
counts that are and are not multiples of the chunk; a host array stays
untouched and a device array is pre-processed in place, as in the
reference."""
from __future__ import annotations

import numpy as np
import pytest
import torch

import kernelkit as kk
from kernelkit import algo

pytestmark = pytest.mark.gpu


def _scan(n_angles, rows=20, cols=24, n=24):
    det = kk.Detector(rows=rows, cols=cols, pixel_height=1.6, pixel_width=1.5)
    g0 = kk.ProjectionGeometry([-60.0, 0.0, 0.0], [40.0, 0.0, 0.0], det)
    pgs = [kk.rotate(g0, yaw=2 * np.pi * k / n_angles) for k in range(n_angles)]
    vg = kk.resolve_volume_geometry(shape=(n,) * 3, voxel_size=1.0)
    return pgs, vg


def _whole_scan(y, pgs, vg, **kw):
    """The general path: a pre-processing callback (here a no-op) routes
    the call through one whole-scan texture."""
    return kk.bp(y, pgs, vg, preproc_fn=lambda p, g: None, **kw)


def _projections(pgs, seed=0):
    det = pgs[0].detector
    rng = np.random.default_rng(seed)
    return rng.random((len(pgs), det.rows, det.cols), dtype=np.float32)


@pytest.mark.parametrize("n_angles", [70, 64, 5])
@pytest.mark.parametrize("filt", [None, "ramlak", "cosine"])
def test_streamed_equals_whole_scan(n_angles, filt):
    pgs, vg = _scan(n_angles)
    y = _projections(pgs)
    keep = y.copy()
    assert algo._can_stream(y, pgs, vg, None, None, None, (0, 1, 2), {})
    got = kk.bp(y, pgs, vg, filter=filt)
    np.testing.assert_array_equal(y, keep)  # input untouched
    d_ref = torch.from_numpy(y.copy()).cuda()
    ref = _whole_scan(d_ref, pgs, vg, filter=filt)
    assert np.array_equal(got, ref)
    assert np.abs(ref).max() > 0
    d = torch.from_numpy(y.copy()).cuda()
    assert algo._can_stream(d, pgs, vg, None, None, None, (0, 1, 2), {})
    assert np.array_equal(kk.bp(d, pgs, vg, filter=filt), ref)
    assert torch.equal(d, d_ref)  # pre-processed in place alike


def test_streamed_fdk_out_argument_and_reuse():
    pgs, vg = _scan(70)
    y = _projections(pgs, 1)
    ref = _whole_scan(torch.from_numpy(y.copy()).cuda(), pgs, vg,
                      filter="ramlak")
    out = np.zeros(vg.shape, np.float32)
    assert kk.fdk(y, pgs, vg, out=out) is out
    assert np.array_equal(out, ref)
    # another detector shape (the ring is rebuilt), then the first again
    pgs2, vg2 = _scan(40, rows=12, cols=30)
    y2 = _projections(pgs2, 2)
    ref2 = _whole_scan(torch.from_numpy(y2.copy()).cuda(), pgs2, vg2,
                       filter="ramlak")
    assert np.array_equal(kk.fdk(y2, pgs2, vg2), ref2)
    assert np.array_equal(kk.fdk(y, pgs, vg), ref)


def test_release_and_rebuild_the_ring():
    pgs, vg = _scan(40)
    y = _projections(pgs, 4)
    ref = kk.fdk(y, pgs, vg)
    algo.release_stream_buffers()
    assert not algo._STREAM
    assert np.array_equal(kk.fdk(y, pgs, vg), ref)


def test_streamed_on_a_side_stream():
    pgs, vg = _scan(70)
    y = _projections(pgs, 3)
    ref = kk.fdk(y, pgs, vg)
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        got = kk.fdk(y, pgs, vg)
    assert np.array_equal(got, ref)
