"""Live comparison with the reference's own CUDA kernels, compiled from
its sources into oracle/_ref/libkkref.so (oracle/build_ref.py), on inputs
larger than the committed golden vectors: config 1 (64^3, 96 angles, 96^2)
and config 2 (256^3, 360 angles, 384^2), at the north-star tolerance of
rel. L2 <= 1e-5 for float32 storage."""
from __future__ import annotations

import numpy as np
import pytest
import torch

from conftest import rel_l2
from helpers import build_case
from kernelkit import phantom
from kernelkit.kernels import RayDrivenConeFP, VoxelDrivenConeBP
from oracle import ref_kernels
from cases import phantom_for

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not ref_kernels.available(),
                                 reason="oracle/_ref/libkkref.so not built")]


def _volume(name, vg):
    ph = phantom_for(name, vg.shape)
    ell = phantom.random_ellipsoids(ph["k"], ph["center_range"],
                                    ph["axes_range"], seed=ph["seed"])
    return phantom.voxelize_torch(ell, vg.shape, vg.extent_min,
                                  vg.voxel_size, device="cuda")


@pytest.mark.parametrize("name", ["config1", "config2"])
def test_fp_bp_full_config(name):
    pgs, vg = build_case(name)
    det = pgs[0].detector
    vol = _volume(name, vg)
    fpar = RayDrivenConeFP.geoms2params(pgs, vg)
    rows12 = np.stack([np.asarray(p, np.float32) for p in fpar], axis=1)
    ref_fp, _ = ref_kernels.ref_cone_fp(
        vol, rows12, fpar.axes, det.rows, det.cols,
        RayDrivenConeFP._output_scale(vg.voxel_size))
    K = RayDrivenConeFP()
    K.compile()
    K.set_params(fpar)
    out = torch.zeros_like(ref_fp)
    K(vol, pgs, vg, out)
    assert rel_l2(out.cpu().numpy(), ref_fp.cpu().numpy()) <= 1e-5
    # the CUDA-core path alone (no texture unit) as well
    K2 = RayDrivenConeFP(use_texture_unit=False)
    K2.compile()
    K2.set_params(fpar)
    out2 = torch.zeros_like(ref_fp)
    K2(vol, pgs, vg, out2)
    assert rel_l2(out2.cpu().numpy(), ref_fp.cpu().numpy()) <= 1e-5

    B = VoxelDrivenConeBP()
    B.compile()
    bpar = B.geoms2params(pgs, vg)
    B.set_params(bpar)
    ref_bp, _ = ref_kernels.ref_cone_bp(ref_fp, np.asarray(bpar).reshape(-1, 12),
                                        vg.shape, vg.voxel_volume())
    v2 = torch.zeros_like(vol)
    B(ref_fp, v2, vg)
    assert rel_l2(v2.cpu().numpy(), ref_bp.cpu().numpy()) <= 1e-5
