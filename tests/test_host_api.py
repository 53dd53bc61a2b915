"""Host-side behaviour of the public API that needs no GPU: exceptions of
the kernel/projector state machines (reference kernels/*.py, projector.py),
filter construction, pitched-array helpers and the phantom generator."""
from __future__ import annotations

import numpy as np
import pytest

import kernelkit as kk
from kernelkit import data, phantom, processing
from kernelkit.kernel import (KernelMemoryUnpreparedException,
                              KernelNotCompiledException)
from kernelkit.kernels import RayDrivenConeFP, VoxelDrivenConeBP
from oracle import processing as oproc


@pytest.fixture
def geom():
    return kk.ProjectionGeometry([-5.0, 0, 0], [5.0, 0, 0],
                                 kk.Detector(9, 9, 1.0, 1.0))


@pytest.fixture
def vg():
    return kk.resolve_volume_geometry(shape=(2, 2, 2),
                                      extent_min=[-.5, None, None],
                                      extent_max=[.5, None, None])


def test_fp_not_compiled(geom, vg):
    K = RayDrivenConeFP()
    assert not K.is_compiled
    seq = kk.ProjectionGeometrySequence.fromList([geom])
    with pytest.raises(KernelNotCompiledException):
        K(np.ones((2, 2, 2), np.float32), seq, vg, None)
    with pytest.raises(KernelNotCompiledException):
        K.set_params(K.geoms2params(seq, vg))
    K.compile()
    assert K.is_compiled


def test_fp_params_not_set(geom, vg):
    K = RayDrivenConeFP()
    K.compile()
    seq = kk.ProjectionGeometrySequence.fromList([geom])
    with pytest.raises(KernelMemoryUnpreparedException):
        K(np.ones((2, 2, 2), np.float32), seq, vg, None)


def test_bp_compile_options():
    K = VoxelDrivenConeBP(projection_axes=(1, 0, 2))
    with pytest.raises(ValueError):
        K.compile(texture=K.InterpolationMethod.Tex2DLayered)
    K.compile(texture=K.InterpolationMethod.Tex3D)
    assert K._compiled_template_kwargs["texture"] == "tex3D"
    with pytest.raises(ValueError):
        VoxelDrivenConeBP(voxels_per_block=(6, 32))
    with pytest.raises(ValueError):
        RayDrivenConeFP(volume_axes=(0, 0, 1))
    with pytest.raises(ValueError):
        RayDrivenConeFP(interpolation="cubic")


def test_projector_state_errors(geom, vg):
    fp = kk.ForwardProjector()
    with pytest.raises(kk.ProjectionGeometryNotSetError):
        fp.projection_geometry
    with pytest.raises(kk.VolumeGeometryNotSetError):
        fp.volume_geometry
    with pytest.raises(kk.VolumeNotSetError):
        fp.volume
    with pytest.raises(kk.ProjectionsNotSetError):
        fp.projections
    bp = kk.BackProjector()
    with pytest.raises(kk.ProjectionsNotSetError):
        bp.projections
    with pytest.raises(ValueError):
        kk.BackProjector(texture_type="surface")
    with pytest.raises(TypeError):
        fp.volume = [1, 2, 3]


def test_projector_requires_one_beam(geom):
    other = kk.ProjectionGeometry([-5.0, 0, 0], [5.0, 0, 0],
                                  kk.Detector(9, 9, 1.0, 1.0),
                                  beam=kk.Beam.PARALLEL)
    fp = kk.ForwardProjector()
    with pytest.raises(NotImplementedError):
        fp.projection_geometry = [geom, other]


def test_fdk_rejects_parallel_beam(vg):
    g = kk.ProjectionGeometry([-5.0, 0, 0], [5.0, 0, 0],
                              kk.Detector(9, 9, 1.0, 1.0),
                              beam=kk.Beam.PARALLEL)
    with pytest.raises(NotImplementedError):
        kk.fdk(np.zeros((1, 9, 9), np.float32), [g], vg)
    with pytest.raises(NotImplementedError):
        kk.algo.fbp(np.zeros((1, 9, 9), np.float32), [g], vg)


@pytest.mark.parametrize("num", [64, 128, 1024])
@pytest.mark.parametrize("name", ["ramlak", "cosine"])
def test_filter_response_matches_oracle(num, name):
    np.testing.assert_array_equal(processing._filter(num, name),
                                  oproc.ramlak_fourier(num, name))
    h = processing.impulse_response(num, name)
    np.testing.assert_allclose(np.fft.fft(h).real,
                               processing._filter(num, name), atol=1e-12)
    if name == "ramlak":
        # the spatial Ram-Lak kernel, times 4
        assert np.isclose(h[0], 1.0)
        assert np.isclose(h[1], -4 / np.pi ** 2)
        assert np.isclose(h[2], 0.0, atol=1e-12)


def test_padded_length():
    assert processing.padded_length(1) == 64
    assert processing.padded_length(96) == 256
    assert processing.padded_length(384) == 1024
    assert processing.padded_length(768) == 2048


def test_pitched_helpers_numpy():
    a = np.arange(3 * 5, dtype=np.float32).reshape(3, 5)
    assert data.pitched_shape(a) == (3, 8)
    assert not data.ispitched(a)
    p = data.aspitched(a)
    assert data.ispitched(p)
    np.testing.assert_array_equal(p, a)
    q = data.pitched_like(p, fill=2.0)
    assert q.shape == a.shape and np.all(q == 2.0)
    with pytest.raises(ValueError):
        data.pitched_like(a)


def test_phantom_sphere_line_integral():
    ell = phantom.Ellipsoids(np.zeros((1, 3)), np.full((1, 3), 5.0),
                             np.eye(3)[None], np.array([0.5]))
    src = np.array([[-50.0, 0, 0]])
    pix = np.array([[[[50.0, 0.0, 0.0], [50.0, 3.0, 0.0]]]])
    li = phantom.line_integrals(ell, src, pix).numpy()
    assert np.isclose(li[0, 0, 0], 5.0)
    # chord at distance d from the centre along a slanted line
    d = 50 * 3.0 / np.hypot(100, 3.0)
    assert np.isclose(li[0, 0, 1], 0.5 * 2 * np.sqrt(25 - d * d))
    vol = phantom.voxelize(ell, (20, 20, 20), (-10, -10, -10), (1, 1, 1))
    assert np.isclose(vol.sum() * 1.0, 0.5 * 4 / 3 * np.pi * 125, rtol=0.1)


def test_autotuner_reuses_its_json_cache(tmp_path):
    """A cached choice is returned without timing anything (the timing
    itself needs a GPU and is covered by the GPU batch tests)."""
    import json

    from kernelkit.batch import Autotuner

    path = tmp_path / "tune.json"
    path.write_text(json.dumps({"fp_axis_group:[[8,8,8],6,[9,9]]": 2}))
    tuner = Autotuner(str(path))
    calls = []
    assert tuner.pick("fp_axis_group:[[8,8,8],6,[9,9]]", (1, 2, 4),
                      calls.append) == 2
    assert calls == []


def test_streamed_bp_is_taken_only_for_host_projections_in_default_layout():
    """``kernelkit.algo._can_stream``: NumPy projections in the default
    layout with the default backprojector take the chunked path; other
    layouts, pre-processing callbacks and other kernels take the general
    one (device arrays are checked on the GPU)."""
    import torch

    from kernelkit import algo
    from kernelkit.kernels import VoxelDrivenConeBP

    det = kk.Detector(rows=4, cols=6, pixel_height=1.0, pixel_width=1.0)
    g0 = kk.ProjectionGeometry([-10.0, 0, 0], [10.0, 0, 0], det)
    pgs = [kk.rotate(g0, yaw=0.1 * k) for k in range(3)]
    vg = kk.resolve_volume_geometry(shape=(4, 4, 4), voxel_size=1.0)
    y = np.zeros((3, 4, 6), np.float32)
    ok = dict(preproc_fn=None, kernel=None, out=None,
              projection_axes=(0, 1, 2), kwargs={})
    assert algo._can_stream(y, pgs, vg, **ok)
    assert algo._can_stream(y, pgs, vg, **{**ok, "kernel": VoxelDrivenConeBP()})
    assert algo._can_stream(y, pgs, vg, **{**ok, "out": np.zeros((4, 4, 4))})
    assert not algo._can_stream(torch.from_numpy(y), pgs, vg, **ok)  # host tensor
    assert not algo._can_stream(y.tolist(), pgs, vg, **ok)
    assert not algo._can_stream(y[::-1], pgs, vg, **ok)      # negative stride
    assert not algo._can_stream(y.astype(">f4"), pgs, vg, **ok)
    assert not algo._can_stream(y.astype(np.int16), pgs, vg, **ok)
    assert algo._can_stream(y.astype(np.float64), pgs, vg, **ok)
    assert not algo._can_stream(y, pgs, vg, **{**ok, "preproc_fn": print})
    assert not algo._can_stream(y, pgs, vg,
                                **{**ok, "projection_axes": (1, 0, 2)})
    assert not algo._can_stream(
        y, pgs, vg, **{**ok, "kernel": VoxelDrivenConeBP(interpolation="exact")})
    assert not algo._can_stream(y[:2], pgs, vg, **ok)        # count mismatch
    assert not algo._can_stream(y[:0], pgs[:0], vg, **ok)    # no angles
    assert not algo._can_stream(y[:, :3], pgs, vg, **ok)     # detector mismatch
    assert not algo._can_stream(y, pgs, vg, **{**ok, "kwargs": {"x": 1}})
