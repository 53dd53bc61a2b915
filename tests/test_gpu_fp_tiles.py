"""Forward projection with shared-memory volume tiles staged by the
tensor-copy unit (kk_fp_options KK_FP_OPT_TILES): the rays that use them
get the direct-load result bit for bit (same samples, same operations),
with and without the texture path, with slice spans and the residual
epilogue; and no wait of the tile pipeline runs out."""
from __future__ import annotations

import pytest
import torch

from helpers import build_case, case_volume
from kernelkit import _native
from kernelkit.kernels import RayDrivenConeFP

pytestmark = pytest.mark.gpu


def _project(pgs, vg, vol, tiles, tex, span=None, residual=None):
    K = RayDrivenConeFP(use_texture_unit=tex)
    K.use_tiles = tiles
    K.slices_per_launch = span
    K.compile()
    K.set_params(K.geoms2params(pgs, vg))
    det = pgs[0].detector
    out = torch.full((len(pgs), det.rows, det.cols), 0.5, device="cuda")
    if residual is None:
        K(vol, pgs, vg, out, additive=True)
    else:
        K.residual(vol, pgs, vg, out, *residual)
    torch.cuda.synchronize()
    return out


@pytest.mark.parametrize("case", ["small", "tilted", "alldirs", "volrot",
                                  "aniso", "config1"])
@pytest.mark.parametrize("tex", [True, False])
def test_tiles_equal_direct_loads(case, tex):
    pgs, vg = build_case(case)
    vol = torch.from_numpy(case_volume(case, vg)).float().cuda()
    ref = _project(pgs, vg, vol, False, tex)
    got = _project(pgs, vg, vol, True, tex)
    assert torch.equal(got, ref)
    assert _native.wait_timeouts() == 0


@pytest.mark.parametrize("span", [16, -1])
def test_tiles_with_spans_and_residual(span):
    pgs, vg = build_case("config1")
    vol = torch.from_numpy(case_volume("config1", vg)).float().cuda()
    det = pgs[0].detector
    g = torch.Generator(device="cuda").manual_seed(12)
    y = torch.rand((len(pgs), det.rows, det.cols), generator=g, device="cuda")
    w = torch.rand(y.shape, generator=g, device="cuda")
    for residual in (None, (y, w)):
        ref = _project(pgs, vg, vol, False, False, span, residual)
        got = _project(pgs, vg, vol, True, False, span, residual)
        assert torch.equal(got, ref)
    assert _native.wait_timeouts() == 0
