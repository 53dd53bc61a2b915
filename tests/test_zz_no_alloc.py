"""The allocation-free backprojection entry point, kk_cone_bp_static.

It exists for callers that cannot allocate device memory themselves (for
example an application whose device memory belongs to its own pooled
allocator, or a program that links only this library's C entry points):
instead of a caller-provided float32 work buffer it uses a buffer built
into the library. These tests call it through the C ABI and compare it
with kk_cone_bp given an ordinary work buffer, twice in a row, since every
call reuses the same built-in buffer. They live in their own file, named
to be collected last.
"""
from __future__ import annotations


import numpy as np
import pytest
import torch

import kernelkit as kk
from helpers import build_case
from kernelkit import _native
from kernelkit.kernels import VoxelDrivenConeBP

pytestmark = pytest.mark.gpu


def _inputs():
    pgs, vg = build_case("config1")          # 96 angles: three 32-angle chunks
    det = pgs[0].detector
    rng = np.random.default_rng(11)
    sino = torch.as_tensor(rng.uniform(0, 1, (len(pgs), det.rows, det.cols))
                           .astype(np.float32), device="cuda")
    params = torch.as_tensor(VoxelDrivenConeBP.geoms2params(pgs, vg),
                             device="cuda")
    return vg, sino, params


def _bp(fn, vg, sino, params, out, work=None, additive=0):
    L = _native.load()
    pdesc = _native.projections_desc(sino)
    vdesc = _native.volume_desc(out)
    scale = float(np.float32(vg.voxel_volume()))
    stream = _native.current_stream()
    if fn == "static":
        rc = L.kk_cone_bp_static(pdesc, vdesc, params.data_ptr(), scale,
                                 _native.KK_INTERP_TEX8, additive, stream)
    else:
        rc = L.kk_cone_bp(pdesc, vdesc, params.data_ptr(), scale,
                          _native.KK_INTERP_TEX8, additive,
                          None if work is None else work.data_ptr(), stream)
    _native.check(rc)
    torch.cuda.synchronize()
    return out


@pytest.mark.parametrize("additive", [0, 1])
@pytest.mark.parametrize("dtype", [torch.bfloat16, torch.float16])
def test_static_entry_point_matches_work_buffer_entry_point(dtype, additive):
    """Same kernels, same chunks, same running sums: the built-in buffer
    gives the caller-buffer result bit for bit, on two calls in a row
    (the second finds the first call's sums in the buffer). With additive
    the first chunk starts from the 16-bit volume and later chunks read the
    buffer."""
    vg, sino, params = _inputs()
    shape = tuple(int(s) for s in vg.shape)
    g = torch.Generator(device="cuda").manual_seed(3)
    start = torch.rand(shape, generator=g, device="cuda").to(dtype)
    work = torch.empty(int(np.prod(shape)), dtype=torch.float32,
                       device="cuda")
    ref = _bp("work", vg, sino, params, start.clone(), work, additive)
    assert float(ref.float().abs().max()) > 0
    for _ in range(2):  # the built-in buffer keeps the previous call's data
        got = _bp("static", vg, sino, params, start.clone(), None, additive)
        assert torch.equal(got, ref)


def test_static_entry_point_float32_volume_of_any_size():
    """A float32 volume carries its own running sums, so the buffer's size
    does not limit it: a 256^3 float32 volume (more voxels than the
    buffer) gives kk_cone_bp's result."""
    _, sino, _ = _inputs()
    pgs, _ = build_case("config1")
    vg = kk.resolve_volume_geometry(shape=256, voxel_size=0.25)
    params = torch.as_tensor(VoxelDrivenConeBP.geoms2params(pgs, vg),
                             device="cuda")
    ref = _bp("work", vg, sino, params,
              torch.empty((256, 256, 256), device="cuda"))
    got = _bp("static", vg, sino, params,
              torch.full((256, 256, 256), 7.0, device="cuda"))
    assert torch.equal(got, ref)
    assert float(ref.abs().max()) > 0


def test_static_entry_point_rejects_large_16bit_volumes():
    L = _native.load()
    _, sino, params = _inputs()
    big = torch.empty((256, 256, 256), dtype=torch.bfloat16, device="cuda")
    rc = L.kk_cone_bp_static(_native.projections_desc(sino),
                             _native.volume_desc(big), params.data_ptr(), 1.0,
                             _native.KK_INTERP_TEX8, 0,
                             _native.current_stream())
    assert rc == _native.KK_ERR_INVALID_ARGUMENT
    assert b"exceed" in L.kk_last_error()
