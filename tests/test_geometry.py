"""Host-side geometry: this repository's geometry code must reproduce, bit
for bit, the kernel parameters the reference's own Python computes for the
same scans (golden vectors from tests/golden/make_host_golden.py)."""
from __future__ import annotations

import math

import numpy as np
import pytest

import kernelkit as kk
from cases import CASES, RESOLVE_CASES
from helpers import build_case, fp_params_rows
from kernelkit.kernels import RayDrivenConeFP, VoxelDrivenConeBP


@pytest.mark.parametrize("name", sorted(CASES))
def test_fp_params_bit_exact(name, host_golden):
    pgs, vg = build_case(name)
    params = RayDrivenConeFP.geoms2params(pgs, vg)
    np.testing.assert_array_equal(fp_params_rows(params),
                                  host_golden[f"{name}/fp_params"])
    np.testing.assert_array_equal(params.axes, host_golden[f"{name}/fp_axes"])
    np.testing.assert_array_equal(
        np.asarray(RayDrivenConeFP._output_scale(vg.voxel_size), np.float32),
        host_golden[f"{name}/fp_out_scale"])


@pytest.mark.parametrize("name", sorted(n for n in CASES
                                        if CASES[n].get("bp", True)))
def test_bp_params_bit_exact(name, host_golden):
    pgs, vg = build_case(name)
    params = VoxelDrivenConeBP.geoms2params(pgs, vg)
    np.testing.assert_array_equal(params.reshape(-1, 12),
                                  host_golden[f"{name}/bp_params"])


@pytest.mark.parametrize("name", sorted(CASES))
def test_volume_geometry(name, host_golden):
    _, vg = build_case(name)
    np.testing.assert_array_equal(np.asarray(vg.shape),
                                  host_golden[f"{name}/vol_shape"])
    np.testing.assert_array_equal(np.asarray(vg.voxel_size, np.float32),
                                  host_golden[f"{name}/vol_voxel_size"])
    np.testing.assert_array_equal(np.asarray(vg.extent_min, np.float32),
                                  host_golden[f"{name}/vol_extent_min"])
    assert vg.voxel_volume() == host_golden[f"{name}/vol_voxel_volume"]


@pytest.mark.parametrize("i", range(len(RESOLVE_CASES)))
def test_resolve_volume_geometry(i, host_golden):
    vg = kk.resolve_volume_geometry(**RESOLVE_CASES[i])
    np.testing.assert_array_equal(np.asarray(vg.shape),
                                  host_golden[f"resolve/{i}/shape"])
    for key in ("voxel_size", "extent_min", "extent_max"):
        np.testing.assert_array_equal(np.asarray(getattr(vg, key), np.float32),
                                      host_golden[f"resolve/{i}/{key}"])


def test_resolve_errors():
    with pytest.raises(ValueError):
        kk.resolve_volume_geometry()
    with pytest.raises(ValueError):
        kk.resolve_volume_geometry(shape=10, extent_min=-1.0, extent_max=1.0,
                                   voxel_size=0.3)
    with pytest.raises(ValueError):
        kk.resolve_volume_geometry(shape=10, extent_min=(-1.0, None, None))


def test_resolve_from_projection_geometry():
    g = kk.ProjectionGeometry([-100, 0, 0], [100, 0, 0],
                              kk.Detector(50, 60, 1.0, 1.0))
    vg = kk.resolve_volume_geometry(voxel_size=0.5, projection_geometry=[g])
    assert vg.shape == (60, 60, 50)
    vg.check_consistency()


def test_angles2mat_is_rotation():
    rng = np.random.default_rng(3)
    for r, p, y in rng.uniform(-math.pi, math.pi, (20, 3)):
        R = kk.angles2mat(r, p, y)
        np.testing.assert_allclose(R @ R.T, np.eye(3), atol=1e-12)
        assert np.isclose(np.linalg.det(R), 1.0)
        Rz = np.array([[math.cos(y), -math.sin(y), 0],
                       [math.sin(y), math.cos(y), 0], [0, 0, 1]])
        Ry = np.array([[math.cos(p), 0, math.sin(p)], [0, 1, 0],
                       [-math.sin(p), 0, math.cos(p)]])
        Rx = np.array([[1, 0, 0], [0, math.cos(r), -math.sin(r)],
                       [0, math.sin(r), math.cos(r)]])
        np.testing.assert_allclose(R, Rz @ Ry @ Rx, atol=1e-14)


def test_rotate_yaw_quarter_turn():
    g = kk.ProjectionGeometry([-5.0, 0, 0], [5.0, 0, 0],
                              kk.Detector(3, 3, 1.0, 1.0))
    r = kk.rotate(g, yaw=np.pi / 2)
    np.testing.assert_allclose(r.source_position, [0, -5, 0], atol=1e-12)
    np.testing.assert_allclose(r.u, [-1, 0, 0], atol=1e-12)
    np.testing.assert_allclose(g.source_position, [-5, 0, 0])  # copy


def test_unit_vector_validation():
    det = kk.Detector(3, 3, 1.0, 1.0)
    with pytest.raises(ValueError):
        kk.ProjectionGeometry([0, 0, 0], [1, 0, 0], det, u=(0, 2, 0))
    with pytest.raises(ValueError):
        kk.ProjectionGeometry([0, 0, 0], [1, 0, 0], det, v=(0, 0, 0))


def test_geoms2params_leaves_caller_geometry_alone():
    pgs, vg = build_case("tilted")
    seq = kk.ProjectionGeometrySequence.fromList(pgs)
    before = seq.source_position.copy()
    RayDrivenConeFP.geoms2params(seq, vg)
    VoxelDrivenConeBP.geoms2params(seq, vg)
    np.testing.assert_array_equal(seq.source_position, before)


def test_sequence_take_and_detector():
    pgs, _ = build_case("small")
    seq = kk.ProjectionGeometrySequence.fromList(pgs)
    assert len(seq) == 24
    sub = seq[2:5]
    assert len(sub) == 3
    np.testing.assert_array_equal(sub.u, seq.u[2:5])
    assert seq.detector.width[0] == np.float32(48 * 1.5)
    corner = seq.detector_extent_min[0]
    np.testing.assert_allclose(corner, [60.0, -36.0, -30.0], atol=1e-5)


def test_beam_parsing():
    assert kk.Beam.from_string("Cone") is kk.Beam.CONE
    with pytest.raises(ValueError):
        kk.Beam.from_string("fan")
    with pytest.raises(TypeError):
        kk.process_beam_type(3)
