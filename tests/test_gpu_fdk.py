"""The one-pass FDK pre-processing kernel, kk_fdk_filter: float64 FFT
filtering (the reference's method, processing.py:111-126) against the
direct circular convolution of kk_filter_rows, the fused pre-weighting
against kk_preweight followed by the filter, and the store into a layered
texture against a plain copy of the filtered rows."""
from __future__ import annotations

import numpy as np
import pytest
import torch

import kernelkit as kk
from kernelkit import _native, processing

pytestmark = pytest.mark.gpu


def _rows(n, rows, cols, seed):
    g = torch.Generator(device="cuda").manual_seed(seed)
    return torch.rand((n, rows, cols), generator=g, device="cuda") - 0.3


def _fft_filter(p, name, geom=None, dst=True, tex=None, layer0=0):
    P = processing.padded_length(p.shape[2])
    plan = processing.device_plan(P, name)
    d = _native.projections_desc(p)
    _native.check(_native.load().kk_fdk_filter(
        d, None if geom is None else geom.data_ptr(), plan.data_ptr(),
        P, d if dst else None,
        None if tex is None else tex.handle, layer0,
        _native.current_stream()))


@pytest.mark.parametrize("cols", [1, 20, 37, 96, 384, 768, 1536, 4096])
@pytest.mark.parametrize("name", ["ramlak", "cosine"])
def test_fft_filter_matches_direct_convolution(cols, name):
    """Both evaluate the same float64 filter; the float32 results agree to
    float32 rounding of float64 values that differ in the last bits."""
    p = _rows(3, 5, cols, cols)
    ref = p.clone()
    P = processing.padded_length(cols)
    h = processing._device_filter(P, name)
    _native.check(_native.load().kk_filter_rows(
        _native.projections_desc(ref), h.data_ptr(), P,
        _native.current_stream()))
    _fft_filter(p, name)
    torch.cuda.synchronize()
    scale = float(ref.abs().max())
    assert float((p - ref).abs().max()) <= 2e-7 * scale
    assert scale > 0


def test_fused_preweight_equals_two_passes():
    """Pre-weighting inside the row load stores what kk_preweight stores,
    so the filtered rows are bit for bit those of the two passes."""
    det = kk.Detector(rows=7, cols=50, pixel_height=1.3, pixel_width=1.1)
    g0 = kk.ProjectionGeometry([-80.0, 2.0, 1.0], [70.0, 0.0, -1.0], det)
    pgs = [kk.rotate(g0, yaw=0.3 * k, pitch=0.05 * k) for k in range(5)]
    p = _rows(5, 7, 50, 4)
    two = p.clone()
    kk.processing.preweight(two, pgs)
    _fft_filter(two, "ramlak")
    geom = torch.from_numpy(processing.preweight_params(pgs)).cuda()
    _fft_filter(p, "ramlak", geom=geom)
    torch.cuda.synchronize()
    assert torch.equal(p, two)


@pytest.mark.parametrize("n", [5, 32])
def test_texture_store_equals_copy(n):
    """Rows written into layers [2, 2 + n) of a layered texture by the
    filter equal the filtered rows copied in; backprojecting either gives
    the same volume."""
    rows, cols = 9, 33
    p = _rows(n, rows, cols, 7)
    filt = p.clone()
    _fft_filter(filt, "ramlak")
    stage = torch.zeros((n + 4, rows, cols), device="cuda")
    direct = _native.Layered(n + 4, rows, cols, _native.KK_F32)
    direct.copy_from(stage)  # the layers the filter does not write
    _fft_filter(p.clone(), "ramlak", dst=False, tex=direct, layer0=2)
    stage[2:2 + n] = filt
    copied = _native.Layered(n + 4, rows, cols, _native.KK_F32)
    copied.copy_from(stage)
    det = kk.Detector(rows=rows, cols=cols, pixel_height=1.0, pixel_width=1.0)
    g0 = kk.ProjectionGeometry([-40.0, 0.0, 0.0], [30.0, 0.0, 0.0], det)
    pgs = [kk.rotate(g0, yaw=2 * np.pi * k / (n + 4)) for k in range(n + 4)]
    vg = kk.resolve_volume_geometry(shape=12, voxel_size=1.0)
    from kernelkit.kernels import VoxelDrivenConeBP

    B = VoxelDrivenConeBP()
    B.compile()
    B.set_params(B.geoms2params(pgs, vg))
    outs = []
    for tex in (direct, copied):
        v = torch.zeros((12, 12, 12), device="cuda")
        B(tex, v, vg, additive=False)
        outs.append(v)
    torch.cuda.synchronize()
    assert torch.equal(outs[0], outs[1])
    assert float(outs[0].abs().max()) > 0


def test_fdk_filter_rejects_bad_lengths():
    p = _rows(1, 2, 40, 1)
    d = _native.projections_desc(p)
    plan = processing.device_plan(128, "ramlak")
    L = _native.load()
    for P in (64, 96, 16384):  # shorter than 2 cols, not a power of two, too long
        rc = L.kk_fdk_filter(d, None, plan.data_ptr(), P, d, None, 0,
                             _native.current_stream())
        assert rc != _native.KK_OK


@pytest.mark.parametrize("P", [64, 128, 2048, 8192])
def test_plan_layout(P):
    """H in bit-reversed order, then per radix-4 stage the twiddles
    exp(-2 pi i j / len), j < len / 4."""
    plan = processing.device_plan(P, "cosine").cpu().numpy()
    H = processing._filter(P, "cosine")
    L = P.bit_length() - 1
    rev = [int(format(i, f"0{L}b")[::-1], 2) for i in range(P)]
    assert np.array_equal(plan[:P], H[rev])
    off, ln = P, P
    while ln >= 4:
        j = np.arange(ln // 4)
        rec = plan[off:off + 2 * len(j)].reshape(-1, 2)
        w = np.exp(-2j * np.pi * j / ln)
        np.testing.assert_allclose(rec[:, 0], w.real, atol=1e-15)
        np.testing.assert_allclose(rec[:, 1], w.imag, atol=1e-15)
        off += 2 * len(j)
        ln //= 4
    assert off <= 3 * P
