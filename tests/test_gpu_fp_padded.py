"""The zero-padded volume copy (kk_fp_options.padded,
RayDrivenConeFP.padded_copy): rays are traced from a copy of the volume
with two zero texels before and after every axis, and the CUDA-core rays
of circular scans sample the slabs that cross the volume's boundary with
clamped coordinates and test-free paired loads (the padding's zeros are
the texture's border). Same results bit for bit as the volume itself,
with every epilogue, slice spans, with or without the texture path, for
permuted, strided and 16-bit volumes."""
from __future__ import annotations

import numpy as np
import pytest
import torch

from helpers import build_case, case_volume
from kernelkit import _native
from kernelkit.kernels import RayDrivenConeFP

pytestmark = pytest.mark.gpu


def _projector(pgs, vg, padded, tex=True, span=None, axes=None):
    kw = {} if axes is None else {"volume_axes": axes}
    K = RayDrivenConeFP(use_texture_unit=tex, **kw)
    K.padded_copy = padded
    K.slices_per_launch = span
    K.compile()
    K.set_params(K.geoms2params(pgs, vg))
    return K


def _project(K, pgs, vg, vol, residual=None):
    det = pgs[0].detector
    out = torch.full((len(pgs), det.rows, det.cols), 0.25, device="cuda")
    if residual is None:
        K(vol, pgs, vg, out, additive=True)
    else:
        K.residual(vol, pgs, vg, out, *residual)
    torch.cuda.synchronize()
    return out


@pytest.mark.parametrize("case", ["small", "tilted", "alldirs", "volrot",
                                  "aniso", "config1"])
@pytest.mark.parametrize("tex", [True, False])
def test_padded_equals_volume(case, tex):
    pgs, vg = build_case(case)
    vol = torch.from_numpy(case_volume(case, vg)).float().cuda()
    ref = _project(_projector(pgs, vg, False, tex), pgs, vg, vol)
    K = _projector(pgs, vg, True, tex)
    got = _project(K, pgs, vg, vol)
    n = tuple(vol.shape)
    assert K._pad_buf.numel() == (n[0] + 4) * (n[1] + 4) * (n[2] + 4)
    assert torch.equal(got, ref)


@pytest.mark.parametrize("span", [16, -1])
def test_padded_with_spans_and_residual(span):
    pgs, vg = build_case("config1")
    vol = torch.from_numpy(case_volume("config1", vg)).float().cuda()
    det = pgs[0].detector
    g = torch.Generator(device="cuda").manual_seed(31)
    y = torch.rand((len(pgs), det.rows, det.cols), generator=g, device="cuda")
    w = torch.rand(y.shape, generator=g, device="cuda")
    for residual in (None, (y, w)):
        ref = _project(_projector(pgs, vg, False, span=span), pgs, vg, vol,
                       residual)
        got = _project(_projector(pgs, vg, True, span=span), pgs, vg, vol,
                       residual)
        assert torch.equal(got, ref)


def test_padded_permuted_strided_and_16bit_volumes():
    pgs, vg = build_case("config1")
    vol = torch.from_numpy(case_volume("config1", vg)).float().cuda()
    # a dense volume in another memory order (world axes permuted)
    perm = vol.permute(2, 1, 0).contiguous()
    ref = _project(_projector(pgs, vg, False, axes=(2, 1, 0)), pgs, vg, perm)
    got = _project(_projector(pgs, vg, True, axes=(2, 1, 0)), pgs, vg, perm)
    assert torch.equal(got, ref)
    # a strided view (rows with a gap; no texture for it either)
    n = tuple(vol.shape)
    wide = torch.zeros((n[0], n[1], n[2] + 3), device="cuda")
    wide[:, :, :n[2]] = vol
    view = wide[:, :, :n[2]]
    ref = _project(_projector(pgs, vg, False), pgs, vg, view)
    got = _project(_projector(pgs, vg, True), pgs, vg, view)
    assert torch.equal(got, ref)
    # 16-bit storage: the copy keeps the volume's type
    half = vol.to(torch.bfloat16)
    ref = _project(_projector(pgs, vg, False), pgs, vg, half)
    K = _projector(pgs, vg, True)
    got = _project(K, pgs, vg, half)
    assert K._pad_buf.dtype == torch.bfloat16
    assert torch.equal(got, ref)


def test_padded_buffer_size_checked():
    pgs, vg = build_case("small")
    vol = torch.from_numpy(case_volume("small", vg)).float().cuda()
    K = _projector(pgs, vg, False)
    vdesc = _native.volume_desc(vol, K._vol_axs)
    det = pgs[0].detector
    out = torch.zeros((len(pgs), det.rows, det.cols), device="cuda")
    pdesc = _native.projections_desc(out)
    n = tuple(vol.shape)
    small = torch.empty((n[0] + 4) * (n[1] + 4) * (n[2] + 4) - 1,
                        device="cuda")
    o = _native.kk_fp_options()
    o.interp = _native.KK_INTERP_TEX8
    o.padded, o.padded_elems = small.data_ptr(), small.numel()
    osc = np.asarray(K._output_scale(vg.voxel_size), np.float32).reshape(9)
    lib = _native.load()
    rc = lib.kk_cone_fp_ex(vdesc, pdesc, K._params_dev.data_ptr(),
                           osc.ctypes.data, o, _native.current_stream())
    assert rc == _native.KK_ERR_INVALID_ARGUMENT
    assert b"padded copy" in lib.kk_last_error()
