"""Public API on the GPU: the reference's own known-answer tests restated
on the CUDA kernels, projector/operator semantics, list and pitched
inputs, FDK, SIRT and the autograd bridge."""
from __future__ import annotations

import itertools

import numpy as np
import pytest
import torch

import kernelkit as kk
from cases import CASES
from conftest import rel_l2
from helpers import build_case, case_volume
from kernelkit.kernel import (KernelMemoryUnpreparedException,
                              KernelNotCompiledException, copy_to_texture)
from kernelkit.kernels import RayDrivenConeFP, VoxelDrivenConeBP
from oracle import cone
from oracle import processing as oproc

pytestmark = pytest.mark.gpu


def cuda(x):
    return torch.as_tensor(np.ascontiguousarray(x), device="cuda")


def fp_kernel(pgs, vg, **kw):
    K = RayDrivenConeFP(**kw)
    K.compile()
    K.set_params(K.geoms2params(pgs, vg))
    return K


def bp_kernel(pgs, vg, **kw):
    K = VoxelDrivenConeBP(**kw)
    K.compile()
    K.set_params(K.geoms2params(pgs, vg))
    return K


# ---- tests/kernels/test_cone_fp.py of the reference ----------------------

def test_fp_exceptions():
    g = kk.ProjectionGeometry([-5., 0, 0], [5., 0, 0], kk.Detector(9, 9, 1, 1))
    vg = kk.resolve_volume_geometry(shape=(2, 2, 2), extent_min=[-.5, None,
                                    None], extent_max=[.5, None, None])
    pg = kk.ProjectionGeometrySequence.fromList([g])
    tex = copy_to_texture(torch.ones((2, 2, 2), device="cuda"))
    projs = torch.zeros((1, 9, 9), device="cuda")
    K = RayDrivenConeFP()
    with pytest.raises(KernelNotCompiledException):
        K(tex, pg, vg, projs)
    K.compile()
    with pytest.raises(KernelMemoryUnpreparedException):
        K(tex, pg, vg, projs)


@pytest.mark.parametrize("n", [1, 7, 100])
def test_fp_unit_cube_integral(n):
    det = kk.Detector(rows=1, cols=1, pixel_height=1 / 1024,
                      pixel_width=1 / 1024)
    g = kk.ProjectionGeometry([-4.0, 0, 0], [0.4, 0, 0], det)
    vg = kk.resolve_volume_geometry(shape=(n,) * 3, extent_min=[-.5] * 3,
                                    extent_max=[.5] * 3)
    K = fp_kernel([g], vg)
    projs = torch.zeros((1, 1, 1), device="cuda")
    K(copy_to_texture(torch.ones((n,) * 3, device="cuda")), [g], vg, projs)
    np.testing.assert_almost_equal(projs[0, 0, 0].item(), 1.0)


@pytest.mark.parametrize("axes,direction", list(itertools.product(
    itertools.permutations((0, 1, 2)), (0, 1, 2))))
def test_fp_line_integral_any_axes(axes, direction):
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
    K = fp_kernel([g], vg, volume_axes=axes)
    projs = torch.zeros((1, 9, 9), device="cuda")
    K(cuda(np.transpose(gt, axes)), [g], vg, projs)
    np.testing.assert_almost_equal(projs[0, 4, 4].item(), 1.0)


@pytest.mark.parametrize("axis", [0, 1, 2])
def test_fp_footprint(axis):
    det = kk.Detector(rows=128, cols=128, pixel_height=8. / 128,
                      pixel_width=8. / 128)
    sod = 1e6
    if axis == 0:
        gt = np.zeros((1, 100, 100), np.float32)
        gt[..., 80:100, 90:100] = 1.0
        g = kk.ProjectionGeometry([-sod, 0, 0], [0, 0, 0], det)
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
    K = fp_kernel([g], vg)
    projs = torch.zeros((1, 128, 128), device="cuda")
    K(cuda(gt), [g], vg, projs)
    lit = (projs[0].cpu().numpy() > 1e-8).astype(np.int64)
    lit[:64, :] = 0
    assert lit.sum() == 128


def test_fp_projection_axes_invariance():
    """tests/kernels/test_cone_fp.py:308-374: every projection layout gives
    the same projections."""
    det = kk.Detector(rows=11, cols=13, pixel_height=4. / 121,
                      pixel_width=4. / 121)
    g = kk.ProjectionGeometry([-4.0, 0, 0], [0.0, 0, 0], det)
    pgs = [kk.rotate(g, yaw=i * 2 * np.pi / 7) for i in range(7)]
    gt = np.zeros((10, 10, 10), np.float32)
    gt[2:3] = 1.
    gt[:, 2:3] = 2.
    gt[:, :, 2:3] = 3.
    vg = kk.resolve_volume_geometry(shape=gt.shape, voxel_size=0.02)
    results = []
    for axes in itertools.permutations((0, 1, 2)):
        K = fp_kernel(pgs, vg, projection_axes=axes)
        shape = tuple((7, 11, 13)[a] for a in axes)
        out = torch.zeros(shape, device="cuda")
        K(cuda(gt), pgs, vg, out)
        results.append(out.permute(*np.argsort(axes)).cpu().numpy())
    for r in results[1:]:
        np.testing.assert_array_equal(r, results[0])


# ---- tests/kernels/test_cone_bp.py of the reference -----------------------

def test_bp_exceptions():
    vg = kk.resolve_volume_geometry((2, 2, 2), [-.2, None, None],
                                    [.2, None, None])
    projs = torch.zeros((3, 9, 9), device="cuda")
    vol = torch.ones((2, 2, 2), device="cuda")
    K = VoxelDrivenConeBP()
    with pytest.raises(KernelNotCompiledException):
        K(copy_to_texture(projs), vol, vg)
    K.compile()
    with pytest.raises(KernelMemoryUnpreparedException):
        K(copy_to_texture(projs), vol, vg)


@pytest.mark.parametrize("axis", [0, 1, 2])
def test_bp_line_of_ones(axis):
    det = kk.Detector(rows=1, cols=1, pixel_height=1., pixel_width=1.)
    g = kk.ProjectionGeometry([-1e5, 0, 0], [0, 0, 0], det)
    expected = np.zeros((3, 3, 3), np.float32)
    if axis == 0:
        expected[:, 1, 1] = 1
    elif axis == 1:
        g = kk.rotate(g, yaw=np.pi / 2)
        expected[1, :, 1] = 1
    else:
        g = kk.rotate(g, pitch=np.pi / 2)
        expected[1, 1, :] = 1
    vg = kk.resolve_volume_geometry(shape=(3, 3, 3), voxel_size=(1., 1., 1.))
    K = bp_kernel([g], vg)
    vol = torch.zeros((3, 3, 3), device="cuda")
    K(copy_to_texture(torch.ones((1, 1, 1), device="cuda"), layered=True),
      vol, vg)
    np.testing.assert_array_almost_equal(vol.cpu().numpy(), expected,
                                         decimal=4)


def test_bp_volume_axes_invariance():
    """tests/kernels/test_cone_bp.py:147-224 (decimal 3)."""
    det = kk.Detector(rows=20, cols=20, pixel_height=1., pixel_width=1.)
    g = kk.ProjectionGeometry([-1000., 0, 0], [0, 0, 0], det)
    vg = kk.resolve_volume_geometry(shape=(60, 60, 60), voxel_size=0.5)
    outcome = None
    for axes in itertools.permutations((0, 1, 2)):
        K = bp_kernel([g], vg, volume_axes=axes)
        vol_t = torch.zeros(tuple(60 for _ in axes), device="cuda")
        K(torch.ones((1, 20, 20), device="cuda"), vol_t, vg)
        vol = vol_t.permute(*np.argsort(axes)).cpu().numpy()
        sl = vol[..., 30]
        if outcome is None:
            outcome = sl
        else:
            np.testing.assert_almost_equal(outcome, sl, decimal=3)


def test_bp_volume_axes_match_reference_model():
    """Permuted volume layouts group voxels along their own slowest axis,
    as the reference does; the oracle with the same step axis agrees."""
    pgs, vg = build_case("small")
    pgs = pgs[:6]
    det = pgs[0].detector
    rng = np.random.default_rng(1)
    sino = rng.uniform(0, 1, (6, det.rows, det.cols)).astype(np.float32)
    params = VoxelDrivenConeBP.geoms2params(pgs, vg)
    for axes in [(2, 1, 0), (1, 0, 2)]:
        K = bp_kernel(pgs, vg, volume_axes=axes)
        shape = tuple(int(vg.shape[a]) for a in axes)
        v = torch.zeros(shape, device="cuda")
        K(cuda(sino), v, vg)
        got = v.permute(*np.argsort(axes)).cpu().numpy()
        ref = cone.cone_bp(sino, params, vg.shape, vg.voxel_volume(),
                           step_axis=axes[0])
        assert rel_l2(got, ref) < 2e-5


# ---- projectors and operators -----------------------------------------

def test_xray_transform_matches_kernels():
    pgs, vg = build_case("config1")
    vol = cuda(case_volume("config1", vg))
    A = kk.XrayTransform(pgs, vg)
    assert A.domain_shape == (64, 64, 64) and A.range_shape == (96, 96, 96)
    y = A(vol)
    K = fp_kernel(pgs, vg)
    y2 = torch.zeros_like(y)
    K(vol, pgs, vg, y2)
    assert torch.equal(y, y2)
    x = A.T(y)  # through the projector's layered texture
    B = bp_kernel(pgs, vg)
    x2 = torch.zeros_like(x)
    B(y, x2, vg)  # device-memory path emulating the same filter
    assert rel_l2(x.cpu().numpy(), x2.cpu().numpy()) < 1e-6
    # additive calls accumulate
    A(vol, out=y2, additive=True)
    torch.testing.assert_close(y2, 2 * y, rtol=1e-6, atol=1e-6)
    assert A.T.T is A


def test_xray_transform_layouts():
    pgs, vg = build_case("small")
    pgs = pgs[:5]
    vol = case_volume("small", vg)
    A = kk.XrayTransform(pgs, vg)
    # a layered BP texture needs angles first, as in the reference
    with pytest.raises(ValueError):
        kk.XrayTransform(pgs, vg, projection_axes=(1, 0, 2))
    B = kk.XrayTransform(pgs, vg, volume_axes=(2, 1, 0),
                         projection_axes=(1, 0, 2),
                         bp_kwargs={"texture_type": "array"})
    assert B.range_shape == (40, 5, 48)
    y = A(cuda(vol)).cpu().numpy()
    yB = np.transpose(B(cuda(np.transpose(vol, (2, 1, 0)))).cpu().numpy(),
                      (1, 0, 2))
    # the memory order of the volume picks the texture weight rule, so the
    # two layouts agree to the 1/256 weight steps and each matches the
    # oracle for its own layout
    assert rel_l2(yB, y) < 1e-3
    fpar = RayDrivenConeFP.geoms2params(pgs, vg)
    rows = np.stack([np.asarray(p, np.float32) for p in fpar], axis=1)
    osc = RayDrivenConeFP._output_scale(vg.voxel_size)
    for out, order in ((y, (0, 1, 2)), (yB, (2, 1, 0))):
        ref = cone.cone_fp(vol, rows, fpar.axes, 40, 48, osc,
                           memory_order=order)
        assert rel_l2(out, ref) < 1e-6


def test_projection_lists_and_pitched_views():
    pgs, vg = build_case("small")
    pgs = pgs[:4]
    vol = cuda(case_volume("small", vg))
    fp = kk.ForwardProjector()
    fp.volume_geometry = vg
    fp.projection_geometry = pgs
    fp.volume = vol
    ref = torch.zeros((4, 40, 48), device="cuda")
    fp.projections = ref
    fp()
    views = [kk.aspitched(torch.zeros((40, 48), device="cuda"))
             for _ in range(4)]
    assert kk.ispitched(views[0])
    fp.projections = views
    fp()
    for v, r in zip(views, ref):
        assert torch.equal(v, r)
    bp = kk.BackProjector(texture_type="pitch2d")
    bp.projection_geometry = pgs
    bp.volume_geometry = vg
    out1 = torch.zeros(tuple(int(s) for s in vg.shape), device="cuda")
    bp.projections = views
    bp.volume = out1
    bp()
    out2 = torch.zeros_like(out1)
    bp.projections = ref
    bp.volume = out2
    bp()
    assert torch.equal(out1, out2)
    with pytest.raises(ValueError):
        bp.projections = torch.zeros((3, 40, 48), device="cuda")


def test_fp_bp_algorithms_return_host_arrays():
    pgs, vg = build_case("small")
    pgs = pgs[:3]
    vol = case_volume("small", vg)
    y = kk.fp(vol, pgs, vg)
    assert isinstance(y, np.ndarray) and y.shape == (3, 40, 48)
    x = kk.bp(y, pgs, vg)
    assert isinstance(x, np.ndarray) and x.shape == (32, 32, 32)
    out = np.zeros_like(x)
    assert kk.bp(y, pgs, vg, out=out) is out


# ---- FDK processing -----------------------------------------------------

@pytest.mark.parametrize("name", ["small", "tilted"])
def test_preweight_and_filter_match_reference_python(name, host_golden):
    pgs, _ = build_case(name)
    pgs = pgs[:5]
    p = cuda(host_golden[f"proc/{name}/input"])
    kk.processing.preweight(p, pgs)
    np.testing.assert_array_equal(p.cpu().numpy(),
                                  host_golden[f"proc/{name}/preweight"])
    for filt in ("ramlak", "cosine"):
        q = p.clone()
        kk.processing.filter(q, filter=filt)
        ref = host_golden[f"proc/{name}/filter_{filt}"]
        np.testing.assert_allclose(q.cpu().numpy(), ref, rtol=0,
                                   atol=1e-6 * np.abs(ref).max())


@pytest.mark.parametrize("cols", [37, 100, 1])
def test_filter_widths(cols, host_golden):
    for filt in ("ramlak", "cosine"):
        p = cuda(host_golden[f"proc/filter_w{cols}/input"])
        kk.processing.filter(p, filter=filt)
        ref = host_golden[f"proc/filter_w{cols}/{filt}"]
        np.testing.assert_allclose(p.cpu().numpy(), ref, rtol=0,
                                   atol=1e-6 * max(np.abs(ref).max(), 1e-30))


def test_fdk_matches_oracle():
    pgs, vg = build_case("config1")
    vol = case_volume("config1", vg)
    y = kk.fp(vol, pgs, vg)
    rec = kk.fdk(y.copy(), pgs, vg)
    params = VoxelDrivenConeBP.geoms2params(pgs, vg)
    ref = oproc.fdk(y, pgs, lambda q: cone.cone_bp(
        q, params, vg.shape, vg.voxel_volume()))
    assert rel_l2(rec, ref) < 5e-5


# ---- SIRT ---------------------------------------------------------------

def test_sirt_graph_equals_eager_and_oracle():
    pgs, vg = build_case("small")
    pgs = pgs[::2]
    vol = case_volume("small", vg)
    y = kk.fp(vol, pgs, vg)
    x_graph = kk.sirt(y, pgs, vg, iters=8, verbose=False, use_graph=True)
    x_eager = kk.sirt(y, pgs, vg, iters=8, verbose=False, use_graph=False)
    np.testing.assert_array_equal(x_graph, x_eager)
    fpar = RayDrivenConeFP.geoms2params(pgs, vg)
    rows = np.stack([np.asarray(p, np.float32) for p in fpar], axis=1)
    bpar = VoxelDrivenConeBP.geoms2params(pgs, vg)
    det = pgs[0].detector
    osc = RayDrivenConeFP._output_scale(vg.voxel_size)
    ref = oproc.sirt(y, lambda x: cone.cone_fp(x, rows, fpar.axes, det.rows,
                                               det.cols, osc),
                     lambda p: cone.cone_bp(p, bpar, vg.shape,
                                            vg.voxel_volume()),
                     vol.shape, 8)
    assert rel_l2(x_graph, ref) < 1e-4


def test_sirt_constraints_mask_and_callback():
    pgs, vg = build_case("small")
    pgs = pgs[::3]
    vol = case_volume("small", vg)
    y = kk.fp(vol, pgs, vg)
    mask = np.ones(vol.shape, np.float32)
    mask[:4] = 0
    seen = []
    x = kk.sirt(y, pgs, vg, iters=3, verbose=False, mask=mask,
                min_constraint=0.0, max_constraint=0.5,
                callback=lambda i, xx, r: seen.append(i), return_gpu=True)
    assert seen == [0, 1, 2]
    x = x.cpu().numpy()
    assert x.min() >= 0.0 and x.max() <= 0.5 and np.all(x[:4] == 0)


# ---- torch_support --------------------------------------------------------

def test_autograd_operator():
    from kernelkit.torch_support import (XrayBackprojection,
                                         XrayForwardProjection)

    pgs, vg = build_case("small")
    pgs = pgs[:3]
    m = XrayForwardProjection(pgs, vg)
    x = torch.rand((2, 1, 32, 32, 32), device="cuda", requires_grad=True)
    y = m(x)
    assert y.shape == (2, 1, 3, 40, 48)
    g = torch.rand_like(y)
    y.backward(g)
    ref = m.op.T(g[1, 0].contiguous())
    torch.testing.assert_close(x.grad[1, 0], ref)
    mb = XrayBackprojection(pgs, vg)
    z = mb(g)
    assert z.shape == (2, 1, 32, 32, 32)


# ---- reduced-precision storage ----------------------------------------

@pytest.mark.parametrize("dtype", [torch.bfloat16, torch.float16])
def test_half_storage_fp_accumulates_in_fp32(dtype):
    pgs, vg = build_case("config1")
    vol = cuda(case_volume("config1", vg)).to(dtype)
    K = fp_kernel(pgs, vg)
    out_h = torch.zeros((96, 96, 96), device="cuda")
    K(vol, pgs, vg, out_h)
    out_f = torch.zeros_like(out_h)
    K(vol.float(), pgs, vg, out_f)
    assert rel_l2(out_h.cpu().numpy(), out_f.cpu().numpy()) < 1e-6
    B = bp_kernel(pgs, vg)
    v_h = torch.zeros((64, 64, 64), device="cuda")
    B(out_f.to(dtype), v_h, vg)
    v_f = torch.zeros_like(v_h)
    B(out_f.to(dtype).float(), v_f, vg)
    assert rel_l2(v_h.cpu().numpy(), v_f.cpu().numpy()) < 1e-6
