"""Parity of the CUDA kernels (through the public kernel classes and the C
ABI) with the reference's own kernels and with the FP64 oracle.

Tolerances (relative L2): 1e-5 against the reference kernels for float32
storage, as the north-star parity bar; 1e-5 against the FP64 oracle with
exact interpolation weights."""
from __future__ import annotations

import numpy as np
import pytest
import torch

import kernelkit as kk
from cases import CASES, GPU_CASES, random_sinogram
from conftest import rel_l2
from helpers import build_case, case_volume
from kernelkit.kernels import RayDrivenConeFP, VoxelDrivenConeBP
from oracle import cone

pytestmark = pytest.mark.gpu

REF_TOL = 1e-5
ORACLE_TOL = 1e-5


def run_fp(pgs, vg, vol, interpolation="texture", texture_unit=True):
    K = RayDrivenConeFP(interpolation=interpolation,
                        use_texture_unit=texture_unit)
    K.compile()
    K.set_params(K.geoms2params(pgs, vg))
    det = pgs[0].detector
    out = torch.zeros((len(pgs), det.rows, det.cols), device="cuda")
    K(torch.as_tensor(vol, device="cuda"), pgs, vg, out)
    return out.cpu().numpy()


def run_bp(pgs, vg, sino, interpolation="texture", fetch="global"):
    K = VoxelDrivenConeBP(interpolation=interpolation)
    K.compile()
    K.set_params(K.geoms2params(pgs, vg))
    vol = torch.zeros(tuple(int(s) for s in vg.shape), device="cuda")
    src = torch.as_tensor(sino, device="cuda")
    if fetch == "texture":  # through the layered texture (hardware filter)
        src = kk.kernel.copy_to_texture(src, layered=True)
    K(src, vol, vg)
    return vol.cpu().numpy()


@pytest.mark.parametrize("texture_unit", [True, False])
@pytest.mark.parametrize("name", GPU_CASES)
def test_fp_matches_reference_kernel(name, texture_unit, gpu_golden):
    pgs, vg = build_case(name)
    out = run_fp(pgs, vg, case_volume(name, vg), texture_unit=texture_unit)
    stride = int(gpu_golden[f"{name}/ref_fp_stride"])
    assert rel_l2(out[::stride], gpu_golden[f"{name}/ref_fp"]) <= REF_TOL


@pytest.mark.parametrize("fetch", ["global", "texture"])
@pytest.mark.parametrize("name", [n for n in GPU_CASES
                                  if CASES[n].get("bp", True)])
def test_bp_matches_reference_kernel(name, fetch, gpu_golden):
    pgs, vg = build_case(name)
    det = pgs[0].detector
    sino = random_sinogram(name, len(pgs), det.rows, det.cols)
    out = run_bp(pgs, vg, sino, fetch=fetch)
    assert rel_l2(out, gpu_golden[f"{name}/ref_bp"]) <= REF_TOL


@pytest.mark.parametrize("name", ["small", "tilted", "alldirs", "aniso"])
def test_fp_exact_matches_fp64_oracle(name, host_golden):
    pgs, vg = build_case(name)
    vol = case_volume(name, vg)
    out = run_fp(pgs, vg, vol, interpolation="exact")
    det = pgs[0].detector
    ref = cone.cone_fp(vol, host_golden[f"{name}/fp_params"],
                       host_golden[f"{name}/fp_axes"], det.rows, det.cols,
                       host_golden[f"{name}/fp_out_scale"], coords="fp64",
                       interp="exact")
    assert rel_l2(out, ref) <= ORACLE_TOL


@pytest.mark.parametrize("name", ["small", "tilted", "alldirs", "volrot"])
def test_bp_exact_matches_fp64_oracle(name, host_golden):
    pgs, vg = build_case(name)
    det = pgs[0].detector
    sino = random_sinogram(name, len(pgs), det.rows, det.cols)
    out = run_bp(pgs, vg, sino, interpolation="exact")
    ref = cone.cone_bp(sino, host_golden[f"{name}/bp_params"], vg.shape,
                       host_golden[f"{name}/vol_voxel_volume"],
                       coords="fp64", interp="exact")
    assert rel_l2(out, ref) <= ORACLE_TOL


@pytest.mark.parametrize("name", ["small", "alldirs"])
def test_texture_mode_matches_tex8_oracle(name, host_golden):
    """Sample-level model: the oracle with float32 coordinates and the
    texture weights tracks the kernels up to float32 accumulation."""
    pgs, vg = build_case(name)
    vol = case_volume(name, vg)
    out = run_fp(pgs, vg, vol)
    det = pgs[0].detector
    ref = cone.cone_fp(vol, host_golden[f"{name}/fp_params"],
                       host_golden[f"{name}/fp_axes"], det.rows, det.cols,
                       host_golden[f"{name}/fp_out_scale"])
    assert rel_l2(out, ref) <= 1e-6
