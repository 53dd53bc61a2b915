"""Pinning of the CPU oracle (oracle/) against the reference: golden
outputs of the reference's CUDA kernels run on a B200, golden outputs of
the reference's Python processing, and the known-answer tests of the
reference's own test suite restated on the oracle."""
from __future__ import annotations

import itertools

import numpy as np
import pytest

import kernelkit as kk
from cases import CASES, GPU_CASES, random_sinogram
from conftest import rel_l2
from helpers import build_case, case_volume
from kernelkit.kernels import RayDrivenConeFP, VoxelDrivenConeBP
from oracle import cone
from oracle import processing as oproc


@pytest.mark.parametrize("name", GPU_CASES)
def test_oracle_fp_matches_reference_kernel(name, host_golden, gpu_golden):
    """Sample-level model of cuda/cone_fp.cu: float32 coordinates and the
    texture weights reproduce the reference to FP64-vs-FP32 accumulation."""
    spec = CASES[name]
    _, vg = build_case(name)
    stride = int(gpu_golden[f"{name}/ref_fp_stride"])
    out = cone.cone_fp(case_volume(name, vg),
                       host_golden[f"{name}/fp_params"][::stride],
                       host_golden[f"{name}/fp_axes"][::stride],
                       spec["rows"], spec["cols"],
                       host_golden[f"{name}/fp_out_scale"])
    assert rel_l2(out, gpu_golden[f"{name}/ref_fp"]) < 5e-7


@pytest.mark.parametrize("name", [n for n in GPU_CASES
                                  if CASES[n].get("bp", True)])
def test_oracle_bp_matches_reference_kernel(name, host_golden, gpu_golden):
    """Model of cuda/cone_bp.cu. The reference divides with the hardware's
    approximate reciprocal (__fdividef); the oracle divides exactly, so a
    few samples land on a neighbouring 1/256 weight step."""
    spec = CASES[name]
    pgs, vg = build_case(name)
    sino = random_sinogram(name, len(pgs), spec["rows"], spec["cols"])
    out = cone.cone_bp(sino, host_golden[f"{name}/bp_params"], vg.shape,
                       host_golden[f"{name}/vol_voxel_volume"])
    assert rel_l2(out, gpu_golden[f"{name}/ref_bp"]) < 2e-5


@pytest.mark.parametrize("name", ["small", "tilted"])
def test_oracle_preweight_and_filter(name, host_golden):
    pgs, _ = build_case(name)
    pgs = pgs[:5]
    p = host_golden[f"proc/{name}/input"]
    pw = oproc.preweight(p, pgs)
    np.testing.assert_array_equal(pw, host_golden[f"proc/{name}/preweight"])
    for filt in ("ramlak", "cosine"):
        q = oproc.filter_rows(pw, filt)
        ref = host_golden[f"proc/{name}/filter_{filt}"]
        np.testing.assert_allclose(q, ref, rtol=0, atol=1e-6 * np.abs(ref).max())


@pytest.mark.parametrize("cols", [37, 100, 1])
def test_oracle_filter_widths(cols, host_golden):
    p = host_golden[f"proc/filter_w{cols}/input"]
    for filt in ("ramlak", "cosine"):
        ref = host_golden[f"proc/filter_w{cols}/{filt}"]
        np.testing.assert_allclose(oproc.filter_rows(p, filt), ref, rtol=0,
                                   atol=1e-6 * max(np.abs(ref).max(), 1e-30))


# ---- known-answer tests of the reference suite, on the oracle -------------

def fp_oracle(vol, pgs, vg, interp="tex8", memory_order=(0, 1, 2)):
    params = RayDrivenConeFP.geoms2params(pgs, vg)
    rows = np.stack([np.asarray(p, np.float32) for p in params], axis=1)
    det = pgs[0].detector
    return cone.cone_fp(vol, rows, params.axes, det.rows, det.cols,
                        RayDrivenConeFP._output_scale(vg.voxel_size),
                        interp=interp, memory_order=memory_order)


@pytest.mark.parametrize("n", [1, 7, 100])
def test_kat_unit_cube_integral(n):
    """tests/kernels/test_cone_fp.py:172-221: the ray through the centre of
    a unit cube integrates to 1 whatever the discretisation."""
    det = kk.Detector(rows=1, cols=1, pixel_height=1 / 1024,
                      pixel_width=1 / 1024)
    g = kk.ProjectionGeometry([-4.0, 0, 0], [4.4 - 4.0, 0, 0], det)
    vg = kk.resolve_volume_geometry(shape=(n,) * 3, extent_min=[-.5] * 3,
                                    extent_max=[.5] * 3)
    out = fp_oracle(np.ones((n,) * 3, np.float32), [g], vg)
    np.testing.assert_almost_equal(out[0, 0, 0], 1.0)


@pytest.mark.parametrize("axes,direction",
                         list(itertools.product(
                             itertools.permutations((0, 1, 2)), (0, 1, 2))))
def test_kat_line_integral_any_axes(axes, direction):
    """tests/kernels/test_cone_fp.py:224-302: a line of ones along the ray
    integrates to 1 for every volume axis order and ray direction."""
    det = kk.Detector(rows=9, cols=9, pixel_height=1 / 128,
                      pixel_width=1 / 128)
    g = kk.ProjectionGeometry([-4.0, 0, 0], [0.4, 0, 0], det)
    gt = np.zeros([9] * 3, np.float32)
    if direction == 0:
        gt[:, 4, 4] = 1.0
    elif direction == 1:
        g = kk.rotate(g, yaw=np.pi / 2)
        gt[4, :, 4] = 1.0
    else:
        g = kk.rotate(g, pitch=np.pi / 2)
        gt[4, 4] = 1.0
    vg = kk.resolve_volume_geometry(shape=gt.shape, extent_min=[-.5] * 3,
                                    extent_max=[.5] * 3)
    params = RayDrivenConeFP.geoms2params([g], vg)
    assert params.axes[0] == direction
    out = fp_oracle(gt, [g], vg, memory_order=axes)
    np.testing.assert_almost_equal(out[0, 4, 4], 1.0)


@pytest.mark.parametrize("axis", [0, 1, 2])
def test_kat_footprint(axis):
    """tests/kernels/test_cone_fp.py:74-169: a 20x10 slab lights exactly
    128 pixels of the upper detector half, in the expected direction."""
    det = kk.Detector(rows=128, cols=128, pixel_height=8. / 128,
                      pixel_width=8. / 128)
    sod = 1e6
    if axis == 0:
        gt = np.zeros((1, 100, 100), np.float32)
        gt[..., 80:100, 90:100] = 1.0
        g = kk.ProjectionGeometry([-sod, 0, 0], [0, 0, 0], det,
                                  u=[0, 1, 0], v=[0, 0, 1])
    elif axis == 1:
        gt = np.zeros((100, 1, 100), np.float32)
        gt[80:100, ..., 90:100] = 1.0
        g = kk.ProjectionGeometry([0, -sod, 0], [0, 0, 0], det,
                                  u=[1, 0, 0], v=[0, 0, 1])
    else:
        gt = np.zeros((100, 100, 1), np.float32)
        gt[80:100, 90:100] = 1.0
        g = kk.ProjectionGeometry([0, 0, -sod], [0, 0, 0], det,
                                  u=[1, 0, 0], v=[0, 1, 0])
    vg = kk.resolve_volume_geometry(shape=gt.shape, voxel_size=[0.05] * 3)
    out = fp_oracle(gt, [g], vg)
    lit = (out[0] > 1e-8).astype(np.int64)
    lit[:64, :] = 0
    assert lit.sum() == 128


@pytest.mark.parametrize("axis", [0, 1, 2])
def test_kat_backprojected_line(axis):
    """tests/kernels/test_cone_bp.py:84-142: one near-parallel ray of value
    1 backprojects to a line of ones (decimal 4)."""
    det = kk.Detector(rows=1, cols=1, pixel_height=1., pixel_width=1.)
    g = kk.ProjectionGeometry([-1e5, 0, 0], [0, 0, 0], det)
    expected = np.zeros((3, 3, 3), np.float32)
    if axis == 0:
        g = kk.rotate(g, yaw=0.0)
        expected[:, 1, 1] = 1
    elif axis == 1:
        g = kk.rotate(g, yaw=np.pi / 2)
        expected[1, :, 1] = 1
    else:
        g = kk.rotate(g, pitch=np.pi / 2)
        expected[1, 1, :] = 1
    vg = kk.resolve_volume_geometry(shape=(3, 3, 3), voxel_size=(1., 1., 1.))
    params = VoxelDrivenConeBP.geoms2params([g], vg)
    out = cone.cone_bp(np.ones((1, 1, 1), np.float32), params, vg.shape,
                       vg.voxel_volume())
    np.testing.assert_array_almost_equal(out, expected, decimal=4)


def test_oracle_sirt_reduces_residual():
    """SIRT on a tiny scan: the projection residual falls monotonically."""
    pgs, vg = build_case("small")
    pgs = pgs[::3]
    vol = case_volume("small", vg)
    fpar = RayDrivenConeFP.geoms2params(pgs, vg)
    rows = np.stack([np.asarray(p, np.float32) for p in fpar], axis=1)
    bpar = VoxelDrivenConeBP.geoms2params(pgs, vg)
    det = pgs[0].detector
    osc = RayDrivenConeFP._output_scale(vg.voxel_size)

    def A(x):
        return cone.cone_fp(x, rows, fpar.axes, det.rows, det.cols, osc)

    def AT(y):
        return cone.cone_bp(y, bpar, vg.shape, vg.voxel_volume())

    y = A(vol)
    res = []
    for it in (1, 3, 6):
        x = oproc.sirt(y, A, AT, vol.shape, it)
        res.append(np.linalg.norm(A(x) - y))
    assert res[0] > res[1] > res[2]
