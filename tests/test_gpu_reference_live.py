"""Live comparison with the reference's own CUDA kernels, compiled from
its sources into oracle/_ref/libkkref.so (oracle/build_ref.py), on inputs
larger than the committed golden vectors."""
from __future__ import annotations

import numpy as np
import pytest
import torch

from cases import CASES
from conftest import rel_l2
from helpers import build_case, case_volume
from kernelkit.kernels import RayDrivenConeFP, VoxelDrivenConeBP
from oracle import ref_kernels

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not ref_kernels.available(),
                                 reason="oracle/_ref/libkkref.so not built")]


@pytest.mark.parametrize("name", ["config1"])
def test_fp_bp_full_config(name, host_golden):
    pgs, vg = build_case(name)
    det = pgs[0].detector
    vol = torch.as_tensor(case_volume(name, vg), device="cuda")
    ref_fp, _ = ref_kernels.ref_cone_fp(
        vol, host_golden[f"{name}/fp_params"], host_golden[f"{name}/fp_axes"],
        det.rows, det.cols, host_golden[f"{name}/fp_out_scale"])
    K = RayDrivenConeFP()
    K.compile()
    K.set_params(K.geoms2params(pgs, vg))
    out = torch.zeros_like(ref_fp)
    K(vol, pgs, vg, out)
    assert rel_l2(out.cpu().numpy(), ref_fp.cpu().numpy()) <= 1e-5

    B = VoxelDrivenConeBP()
    B.compile()
    B.set_params(B.geoms2params(pgs, vg))
    ref_bp, _ = ref_kernels.ref_cone_bp(ref_fp, host_golden[f"{name}/bp_params"],
                                        vg.shape,
                                        host_golden[f"{name}/vol_voxel_volume"])
    v2 = torch.zeros_like(vol)
    B(ref_fp, v2, vg)
    assert rel_l2(v2.cpu().numpy(), ref_bp.cpu().numpy()) <= 1e-5
