"""Edge cases of the CUDA path: degenerate sizes (one voxel, one pixel,
one angle, flat volumes), volumes whose element offsets exceed 2^31 (the
64-bit addressing path), and empty or inconsistent inputs, which must
fail with an exception rather than launch anything."""
from __future__ import annotations

import numpy as np
import pytest
import torch

import kernelkit as kk
from conftest import rel_l2
from helpers import fp_params_rows
from kernelkit.kernels import RayDrivenConeFP, VoxelDrivenConeBP
from oracle import cone

pytestmark = pytest.mark.gpu

ORACLE_TOL = 1e-5


def _scan(vol_shape, rows, cols, rotations, voxel=1.0):
    det = kk.Detector(rows=rows, cols=cols, pixel_height=1.3,
                      pixel_width=1.1)
    g0 = kk.ProjectionGeometry([-12.0, 0.2, -0.1], [10.0, 0.0, 0.1], det)
    pgs = [kk.rotate(g0, roll=r, pitch=p, yaw=y) for (r, p, y) in rotations]
    vg = kk.resolve_volume_geometry(shape=vol_shape, voxel_size=voxel)
    return pgs, vg


TINY = [
    ((1, 1, 1), 1, 1, [(0.0, 0.0, 0.3)]),
    ((2, 3, 1), 2, 3, [(0.0, 0.0, 0.0), (0.0, 1.2, 0.7), (0.3, -0.4, 2.5)]),
    ((5, 1, 4), 3, 7, [(0.0, 0.0, 1.6), (0.0, -1.3, 0.2)]),
    ((3, 4, 5), 7, 1, [(0.0, 0.0, k * 0.9) for k in range(5)]),
]


def _fp(pgs, vg, vol, interp):
    K = RayDrivenConeFP(interpolation=interp)
    K.compile()
    K.set_params(K.geoms2params(pgs, vg))
    det = pgs[0].detector
    out = torch.full((len(pgs), det.rows, det.cols), 3.0, device="cuda")
    K(torch.as_tensor(vol, device="cuda"), pgs, vg, out, additive=False)
    return out.cpu().numpy()


@pytest.mark.parametrize("case", range(len(TINY)))
def test_tiny_shapes_forward_projection(case):
    shape, rows, cols, rots = TINY[case]
    pgs, vg = _scan(shape, rows, cols, rots)
    vol = np.random.default_rng(case).uniform(0.5, 1.5, shape).astype(
        np.float32)
    p = RayDrivenConeFP.geoms2params(pgs, vg)
    osc = RayDrivenConeFP._output_scale(vg.voxel_size)
    for interp, coords, oi, tol in (("exact", "fp64", "exact", ORACLE_TOL),
                                    ("texture", "fp32", "tex8", 1e-6)):
        out = _fp(pgs, vg, vol, interp)
        ref = cone.cone_fp(vol, fp_params_rows(p), p.axes, rows, cols, osc,
                           coords=coords, interp=oi)
        assert np.abs(ref).sum() > 0
        assert rel_l2(out, ref) <= tol


@pytest.mark.parametrize("case", range(len(TINY)))
def test_tiny_shapes_backprojection(case):
    shape, rows, cols, rots = TINY[case]
    pgs, vg = _scan(shape, rows, cols, rots)
    sino = np.random.default_rng(10 + case).uniform(
        0.5, 1.5, (len(pgs), rows, cols)).astype(np.float32)
    K = VoxelDrivenConeBP(interpolation="exact")
    K.compile()
    params = VoxelDrivenConeBP.geoms2params(pgs, vg)
    K.set_params(params)
    out = torch.full(shape, 3.0, device="cuda")
    K(torch.as_tensor(sino, device="cuda"), out, vg, additive=False)
    ref = cone.cone_bp(sino, params, vg.shape, vg.voxel_volume(),
                       coords="fp64", interp="exact")
    assert np.abs(ref).sum() > 0
    assert rel_l2(out.cpu().numpy(), ref) <= ORACLE_TOL


def test_element_offsets_beyond_31_bits():
    """A volume viewed with a stride that puts its last element beyond
    2^31 elements takes the 64-bit addressing path; it must project
    exactly as the same volume stored densely."""
    pgs, vg = _scan((6, 7, 8), 9, 11, [(0.0, 0.0, k * 0.7) for k in range(6)])
    vol = torch.rand((6, 7, 8), generator=torch.Generator().manual_seed(3))
    s0 = (1 << 29) + 64
    buf = torch.zeros(5 * s0 + 7 * 8 + 8, device="cuda")
    view = torch.as_strided(buf, (6, 7, 8), (s0, 8, 1))
    view.copy_(vol.cuda())
    assert (5 * s0 + 6 * 8 + 7) > (1 << 31)
    det = pgs[0].detector
    outs = []
    for v in (vol.cuda(), view):
        K = RayDrivenConeFP(use_texture_unit=False)
        K.compile()
        K.set_params(K.geoms2params(pgs, vg))
        out = torch.empty((len(pgs), det.rows, det.cols), device="cuda")
        K(v, pgs, vg, out, additive=False)
        outs.append(out.cpu().numpy())
    assert np.abs(outs[0]).sum() > 0
    assert np.array_equal(outs[0], outs[1])
    del buf, view


def test_empty_and_inconsistent_inputs_raise():
    pgs, vg = _scan((4, 4, 4), 5, 5, [(0.0, 0.0, 0.0), (0.0, 0.0, 1.0)])
    with pytest.raises(Exception):
        kk.XrayTransform([], vg)
    op = kk.XrayTransform(pgs, vg)
    with pytest.raises(ValueError):  # wrong volume shape
        op(torch.zeros((4, 4, 5), device="cuda"))
    K = RayDrivenConeFP()
    K.compile()
    K.set_params(K.geoms2params(pgs, vg))
    with pytest.raises(ValueError):  # projections for the wrong angle count
        K(torch.zeros((4, 4, 4), device="cuda"), pgs, vg,
          torch.zeros((3, 5, 5), device="cuda"))
