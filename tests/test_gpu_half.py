"""16-bit storage with float16 textures (north-star precision form):
volumes in bfloat16/float16 and projections in float16, FP32 accumulation
in every projection, the texture unit sampling float16 texels. The
tolerance is that of 16-bit storage (rel. L2 <= 5e-3 against the float32
path), not the float32 parity bar."""
from __future__ import annotations

import pytest
import torch

from conftest import rel_l2
from helpers import build_case, case_volume
from kernelkit.algo import SIRT
from kernelkit.kernels import RayDrivenConeFP

pytestmark = pytest.mark.gpu

#: 16-bit storage tolerance
HALF_TOL = 5e-3


@pytest.mark.parametrize("vdt", [torch.bfloat16, torch.float16])
def test_forward_projection_with_half_texture(vdt):
    pgs, vg = build_case("config1")
    vol = torch.as_tensor(case_volume("config1", vg), device="cuda")
    det = pgs[0].detector
    ref = torch.empty((len(pgs), det.rows, det.cols), device="cuda")
    fp = RayDrivenConeFP()
    fp.compile()
    fp.set_params(fp.geoms2params(pgs, vg))
    fp(vol.to(vdt).float(), pgs, vg, ref, additive=False)
    out = torch.empty(ref.shape, dtype=torch.float16, device="cuda")
    fp.half_texture = True
    fp(vol.to(vdt), pgs, vg, out, additive=False)
    assert fp._vtex is not None and fp._vtex.dtype == 2  # float16 texels
    assert rel_l2(out.float().cpu().numpy(), ref.cpu().numpy()) <= HALF_TOL


def test_sirt_16bit_storage_matches_float32():
    pgs, vg = build_case("config1")
    vol = torch.as_tensor(case_volume("config1", vg), device="cuda")
    det = pgs[0].detector
    y = torch.empty((len(pgs), det.rows, det.cols), device="cuda")
    fp = RayDrivenConeFP()
    fp.compile()
    fp.set_params(fp.geoms2params(pgs, vg))
    fp(vol, pgs, vg, y, additive=False)
    ref = SIRT(y, pgs, vg, min_constraint=0.0).run(12, use_graph=True)
    s = SIRT(y, pgs, vg, min_constraint=0.0, volume_dtype=torch.bfloat16,
             projection_dtype=torch.float16)
    assert s.x.dtype == torch.bfloat16 and s.y.dtype == torch.float16
    x = s.run(12, use_graph=True)
    assert rel_l2(x.float().cpu().numpy(), ref.cpu().numpy()) <= HALF_TOL
    e32 = rel_l2(ref.cpu().numpy(), vol.cpu().numpy())
    e16 = rel_l2(x.float().cpu().numpy(), vol.cpu().numpy())
    assert abs(e16 - e32) <= HALF_TOL
