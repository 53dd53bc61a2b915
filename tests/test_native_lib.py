"""The C ABI library: it loads without a GPU, exports every symbol that
include/kk.h declares, and rejects bad arguments with status codes before
touching the device."""
from __future__ import annotations

import ctypes
import os
import re

import pytest

from kernelkit import _native

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    src = open(os.path.join(ROOT, "include", "kk.h")).read()
    return sorted(set(re.findall(r"KK_API\s+[\w\s\*]+?\b(kk_\w+)\s*\(", src)))


def test_header_and_binding_agree():
    assert declared_symbols() == sorted(_native.EXPORTS)


def test_library_exports_every_declared_symbol():
    L = _native.load()
    for name in declared_symbols():
        assert hasattr(L, name), name
    assert L.kk_abi_version() == 1


def test_null_arguments_are_rejected():
    L = _native.load()
    vol = _native.kk_volume()
    proj = _native.kk_projections()
    osc = (ctypes.c_float * 9)()
    rc = L.kk_cone_fp(vol, proj, None, osc, 0, 16, 0, None)
    assert rc == _native.KK_ERR_INVALID_ARGUMENT
    assert b"volume" in L.kk_last_error()
    with pytest.raises(ValueError):
        _native.check(rc)


def test_bad_shapes_are_rejected():
    L = _native.load()
    vol = _native.kk_volume()
    vol.data = 0x1000
    vol.shape[:] = (4, 4, 40000)
    vol.stride[:] = (16, 4, 1)
    proj = _native.kk_projections()
    proj.data = 0x2000
    proj.n_angles, proj.rows, proj.cols = 1, 4, 4
    proj.stride[:] = (16, 4, 1)
    osc = (ctypes.c_float * 9)()
    rc = L.kk_cone_fp(vol, proj, ctypes.c_void_p(0x3000), osc, 0, 16, 0,
                      None)
    assert rc == _native.KK_ERR_INVALID_ARGUMENT
    vol.shape[:] = (4, 4, 4)
    proj.table = 0x4000
    proj.table_axis = 1
    rc = L.kk_cone_bp(proj, vol, ctypes.c_void_p(0x3000), 1.0, 0, 0, None,
                      None)
    assert rc == _native.KK_ERR_UNSUPPORTED
    vol.dtype = 7
    proj.table = None
    proj.table_axis = 0
    rc = L.kk_cone_bp(proj, vol, ctypes.c_void_p(0x3000), 1.0, 0, 0, None,
                      None)
    assert rc == _native.KK_ERR_INVALID_ARGUMENT


def test_interpolation_mode_checked():
    L = _native.load()
    vol = _native.kk_volume()
    vol.data = 0x1000
    vol.shape[:] = (4, 4, 4)
    vol.stride[:] = (16, 4, 1)
    proj = _native.kk_projections()
    proj.data = 0x2000
    proj.n_angles, proj.rows, proj.cols = 1, 4, 4
    proj.stride[:] = (16, 4, 1)
    osc = (ctypes.c_float * 9)()
    rc = L.kk_cone_fp(vol, proj, ctypes.c_void_p(0x3000), osc, 9, 16, 0, None)
    assert rc == _native.KK_ERR_INVALID_ARGUMENT
    assert b"interpolation" in L.kk_last_error()


def test_bp_launch_count_is_host_logic():
    """kk_bp_launches (no GPU needed): one launch per four 32-angle
    chunks."""
    L = _native.load()
    assert [L.kk_bp_launches(n) for n in (0, 1, 32, 128, 129, 720, 1440)] \
        == [0, 1, 1, 1, 2, 6, 12]


def test_fp_launch_split_is_host_logic():
    """kk_fp_launches / kk_fp_set_span (no GPU needed): float32 projections
    are traced in one launch up to 256 slices, in 192-slice launches up to
    640 and in 128-slice launches beyond by default; 16-bit projections in
    one launch, unless a float32 running-sum buffer carries the sums (then
    per chunk of angles)."""
    from kernelkit.kernels.cone_fp import (launches_per_projection,
                                           set_slices_per_launch)

    assert launches_per_projection(256) == 1
    assert launches_per_projection(384) == 2
    assert launches_per_projection(512) == 3
    assert launches_per_projection(1024) == 8
    assert launches_per_projection(1024, float32=False) == 1
    assert launches_per_projection(1024, float32=False, sums=True) == 8
    L = _native.load()
    assert L.kk_fp_launches(1024, 16, _native.KK_F16) == 1
    try:
        set_slices_per_launch(-1)
        assert launches_per_projection(1024) == 1
        set_slices_per_launch(100)  # rounded up to 112 = 7 slabs of 16
        assert launches_per_projection(512) == 5
        with pytest.raises(Exception):
            set_slices_per_launch(-2)
    finally:
        set_slices_per_launch(0)
