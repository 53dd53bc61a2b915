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

from conftest import rel_l2
from helpers import build_case
from kernelkit import _native
from kernelkit.kernels import VoxelDrivenConeBP

pytestmark = pytest.mark.gpu

#: the tolerance of the backprojection parity tests
TOL = 1e-5


def _inputs():
    pgs, vg = build_case("config1")          # 96 angles: three 32-angle chunks
    det = pgs[0].detector
    rng = np.random.default_rng(11)
    sino = torch.as_tensor(rng.uniform(0, 1, (len(pgs), det.rows, det.cols))
                           .astype(np.float32), device="cuda")
    params = torch.as_tensor(VoxelDrivenConeBP.geoms2params(pgs, vg),
                             device="cuda")
    return vg, sino, params


def _bp(fn, vg, sino, params, out, work=None):
    L = _native.load()
    pdesc = _native.projections_desc(sino)
    vdesc = _native.volume_desc(out)
    scale = float(np.float32(vg.voxel_volume()))
    stream = _native.current_stream()
    if fn == "static":
        rc = L.kk_cone_bp_static(pdesc, vdesc, params.data_ptr(), scale,
                                 _native.KK_INTERP_TEX8, 0, stream)
    else:
        rc = L.kk_cone_bp(pdesc, vdesc, params.data_ptr(), scale,
                          _native.KK_INTERP_TEX8, 0, work.data_ptr(), stream)
    _native.check(rc)
    torch.cuda.synchronize()
    return out.float().cpu().numpy()


@pytest.mark.parametrize("dtype", [torch.bfloat16, torch.float16])
def test_static_entry_point_matches_work_buffer_entry_point(dtype):
    vg, sino, params = _inputs()
    shape = tuple(int(s) for s in vg.shape)
    work = torch.empty(int(np.prod(shape)), dtype=torch.float32,
                       device="cuda")
    ref = _bp("work", vg, sino, params, torch.empty(shape, dtype=dtype,
                                                    device="cuda"), work)
    for _ in range(2):  # the built-in buffer keeps the previous call's data
        out = torch.full(shape, 7.0, dtype=dtype, device="cuda")
        got = _bp("static", vg, sino, params, out)
        assert rel_l2(got, ref) <= TOL


def test_static_entry_point_rejects_large_volumes():
    L = _native.load()
    _, sino, params = _inputs()
    big = torch.empty((256, 256, 256), dtype=torch.bfloat16, device="cuda")
    rc = L.kk_cone_bp_static(_native.projections_desc(sino),
                             _native.volume_desc(big), params.data_ptr(), 1.0,
                             _native.KK_INTERP_TEX8, 0,
                             _native.current_stream())
    assert rc == _native.KK_ERR_INVALID_ARGUMENT
    assert b"exceed" in L.kk_last_error()
