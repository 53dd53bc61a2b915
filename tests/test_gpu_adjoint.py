"""Exact adjoint of the ray-driven forward projector (kk_cone_fp_adjoint).

The reference's autograd backward is its backprojector, which is not the
transpose of its forward projector. These tests check that
``RayDrivenConeFP.transpose`` is: against the explicit matrix of the
forward projector (built column by column from unit volumes), by the
FP64 dot-product identity <A x, y> = <x, A^T y> on seeded Gaussian data
(mismatch <= 1e-6 relative to |A x| |y|), through angle chunking, and by
central finite differences of a least-squares loss through the autograd
module.
"""
from __future__ import annotations

import numpy as np
import pytest
import torch

import kernelkit as kk
from conftest import rel_l2
from helpers import build_case
from kernelkit.kernels import RayDrivenConeFP

pytestmark = pytest.mark.gpu

#: relative dot-test mismatch bound (north-star adjoint target)
DOT_TOL = 1e-6


def _kernel(pgs, vg, interp, volume_axes=(0, 1, 2), **kw):
    K = RayDrivenConeFP(interpolation=interp, volume_axes=volume_axes, **kw)
    K.compile()
    K.set_params(K.geoms2params(pgs, vg))
    return K


def _shapes(pgs, vg, volume_axes=(0, 1, 2)):
    shape = tuple(int(vg.shape[i]) for i in volume_axes)
    det = pgs[0].detector
    return shape, (len(pgs), det.rows, det.cols)


def _tiny():
    """6 x 5 x 7 volume, 9 x 8 detector, five angles including steep
    pitches (rays along every axis)."""
    det = kk.Detector(rows=9, cols=8, pixel_height=1.3, pixel_width=1.1)
    g0 = kk.ProjectionGeometry([-20.0, 0.4, -0.3], [16.0, 0.0, 0.2], det)
    rots = [(0.0, 0.0, 0.0), (0.0, 0.0, 1.1), (0.2, 0.4, 2.0),
            (0.0, -1.2, 0.5), (0.1, 1.3, 4.0)]
    pgs = [kk.rotate(g0, roll=r, pitch=p, yaw=y) for (r, p, y) in rots]
    vg = kk.resolve_volume_geometry(shape=(6, 5, 7), voxel_size=1.0)
    return pgs, vg


@pytest.mark.parametrize("interp", ["texture", "exact"])
def test_adjoint_equals_explicit_transpose(interp):
    pgs, vg = _tiny()
    K = _kernel(pgs, vg, interp)
    shape, pshape = _shapes(pgs, vg)
    n = int(np.prod(shape))
    cols = []
    e = torch.zeros(n, device="cuda")
    out = torch.empty(pshape, device="cuda")
    for i in range(n):
        e.zero_()
        e[i] = 1.0
        K(e.view(shape), pgs, vg, out, additive=False)
        cols.append(out.flatten().double().cpu())
    A = torch.stack(cols, dim=1)  # (pixels, voxels)
    assert float(A.abs().sum()) > 0
    g = torch.Generator().manual_seed(7)
    y = torch.randn(pshape, generator=g)
    ref = (A.T @ y.flatten().double()).view(shape).numpy()
    got = torch.empty(shape, device="cuda")
    K.transpose(y.cuda(), pgs, vg, got)
    assert rel_l2(got.cpu().numpy(), ref) <= 1e-6


def _dot_mismatch(K, pgs, vg, shape, pshape, seed=3):
    g = torch.Generator(device="cuda").manual_seed(seed)
    x = torch.randn(shape, generator=g, device="cuda")
    y = torch.randn(pshape, generator=g, device="cuda")
    Ax = torch.empty(pshape, device="cuda")
    K(x, pgs, vg, Ax, additive=False)
    ATy = torch.empty(shape, device="cuda")
    K.transpose(y, pgs, vg, ATy)
    lhs = float((Ax.double() * y.double()).sum())
    rhs = float((x.double() * ATy.double()).sum())
    scale = float(Ax.double().norm() * y.double().norm())
    return abs(lhs - rhs) / scale, ATy


@pytest.mark.parametrize("case", ["small", "tilted", "alldirs", "volrot",
                                  "aniso", "config1"])
@pytest.mark.parametrize("interp", ["texture", "exact"])
def test_dot_product_identity(case, interp):
    pgs, vg = build_case(case)
    K = _kernel(pgs, vg, interp)
    shape, pshape = _shapes(pgs, vg)
    mismatch, _ = _dot_mismatch(K, pgs, vg, shape, pshape)
    assert mismatch <= DOT_TOL


@pytest.mark.parametrize("volume_axes", [(2, 1, 0), (1, 0, 2)])
def test_dot_product_identity_permuted_volume(volume_axes):
    pgs, vg = build_case("alldirs")
    K = _kernel(pgs, vg, "texture", volume_axes=volume_axes)
    shape, pshape = _shapes(pgs, vg, volume_axes)
    mismatch, _ = _dot_mismatch(K, pgs, vg, shape, pshape)
    assert mismatch <= DOT_TOL


def test_angle_chunks_give_the_same_adjoint():
    pgs, vg = build_case("small")
    shape, pshape = _shapes(pgs, vg)
    y = torch.randn(pshape, generator=torch.Generator(device="cuda")
                    .manual_seed(5), device="cuda")
    outs = []
    for work in (1 << 29, 20 * 40 * 48 * 5):  # all angles; 5 per chunk
        K = _kernel(pgs, vg, "texture")
        K.adjoint_work_bytes = work
        out = torch.full(shape, 3.0, device="cuda")
        K.transpose(y, pgs, vg, out)
        outs.append(out.cpu().numpy())
    assert rel_l2(outs[1], outs[0]) <= 1e-6
    # additive accumulates onto the volume
    K = _kernel(pgs, vg, "texture")
    out = torch.full(shape, 3.0, device="cuda")
    K.transpose(y, pgs, vg, out, additive=True)
    assert rel_l2(out.cpu().numpy(), outs[0] + 3.0) <= 1e-6


def test_exact_operator_and_autograd_gradient_by_finite_differences():
    pgs, vg = build_case("small")
    shape, pshape = _shapes(pgs, vg)
    g = torch.Generator(device="cuda").manual_seed(11)
    x0 = torch.rand(shape, generator=g, device="cuda")
    y = torch.rand(pshape, generator=g, device="cuda") * 10.0
    op = kk.ExactXrayTransform(pgs, vg)
    # the operator's .T is the kernel's transpose
    mismatch, _ = _dot_mismatch(op.projector.kernel, pgs, vg, shape, pshape)
    assert mismatch <= DOT_TOL
    from kernelkit.torch_support import ExactXrayForwardProjection

    module = ExactXrayForwardProjection(pgs, vg)
    x = x0[None, None].clone().requires_grad_(True)
    loss = ((module(x) - y[None, None]).double() ** 2).sum()
    loss.backward()
    grad = x.grad[0, 0].double()
    # the gradient is 2 A^T (A x - y)
    Ax = op(x0)
    ref = 2.0 * op.T((Ax - y).contiguous())
    assert rel_l2(grad.cpu().numpy(), ref.double().cpu().numpy()) <= 1e-6

    def L(v):
        return float(((op(v) - y).double() ** 2).sum())

    eps = 1e-3
    for k in range(8):
        d = torch.randn(shape, generator=g, device="cuda")
        fd = (L(x0 + eps * d) - L(x0 - eps * d)) / (2 * eps)
        an = float((grad * d.double()).sum())
        assert abs(fd - an) <= 1e-3 * abs(an) + 1e-6
