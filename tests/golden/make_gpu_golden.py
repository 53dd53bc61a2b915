"""Generate ``gpu_golden.npz``: outputs of the reference's own CUDA kernels
(``oracle/_ref/libkkref.so``, built from the reference sources by
``oracle/build_ref.py``) and of the texture-filter probe, on a GPU.

Inputs are the reference-computed kernel parameters of ``host_golden.npz``
(``make_host_golden.py``), seeded ellipsoid phantoms
(``kernelkit.phantom``) for the forward projections and seeded uniform
sinograms for the backprojections (``cases.py``).

Usage (on a machine with a CUDA GPU, from the repository root):
``python tests/golden/make_gpu_golden.py OUT.npz``
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, HERE)
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "astra-kernelkit_b200"))

import torch  # noqa: E402

from cases import (CASES, GPU_CASES, phantom_for, probe_coordinates,  # noqa: E402
                   probe_random, probe_random3d, random_sinogram)
from oracle import ref_kernels  # noqa: E402
from kernelkit import phantom  # noqa: E402

#: config1 is stored on a subset of angles to keep the fixture small
FP_ANGLE_STRIDE = {"config1": 8}


def case_volume(name, host):
    shape = tuple(int(s) for s in host[f"{name}/vol_shape"])
    ph = phantom_for(name, shape)
    vs = host[f"{name}/vol_voxel_size"].astype(np.float64)
    lo = host[f"{name}/vol_extent_min"].astype(np.float64)
    hi = host[f"{name}/vol_extent_max"].astype(np.float64)
    centre = (lo + hi) / 2
    ell = phantom.random_ellipsoids(ph["k"], ph["center_range"] * vs.min(),
                                    np.asarray(ph["axes_range"]) * vs.min(),
                                    ph["seed"])
    ell.centers += centre
    return phantom.voxelize(ell, shape, lo, vs)


def main(out_path):
    host = dict(np.load(os.path.join(HERE, "host_golden.npz")))
    out = {}
    for name in GPU_CASES:
        spec = CASES[name]
        rows, cols = spec["rows"], spec["cols"]
        vol = case_volume(name, host)
        out[f"{name}/volume_sum"] = np.float64(vol.astype(np.float64).sum())
        v = torch.as_tensor(vol, device="cuda")
        proj, ms_fp = ref_kernels.ref_cone_fp(
            v, host[f"{name}/fp_params"], host[f"{name}/fp_axes"], rows, cols,
            host[f"{name}/fp_out_scale"])
        stride = FP_ANGLE_STRIDE.get(name, 1)
        out[f"{name}/ref_fp"] = proj.cpu().numpy()[::stride]
        out[f"{name}/ref_fp_stride"] = np.int64(stride)
        out[f"{name}/ref_fp_ms"] = np.float64(ms_fp)
        if f"{name}/bp_params" in host:
            n = len(host[f"{name}/bp_params"])
            sino = torch.as_tensor(random_sinogram(name, n, rows, cols),
                                   device="cuda")
            vbp, ms_bp = ref_kernels.ref_cone_bp(
                sino, host[f"{name}/bp_params"], host[f"{name}/vol_shape"],
                host[f"{name}/vol_voxel_volume"])
            out[f"{name}/ref_bp"] = vbp.cpu().numpy()
            out[f"{name}/ref_bp_ms"] = np.float64(ms_bp)
        print(name, "fp ms", ms_fp, flush=True)

    fine, border = probe_coordinates()
    ramp_x = np.broadcast_to(np.arange(64, dtype=np.float32)[None, None, :],
                             (2, 64, 64)).copy()
    ramp_x[1] = np.arange(64, dtype=np.float32)[:, None]  # layer 1: ramp in y
    c = np.full_like(fine, 20.5)
    out["probe/layered_x"] = ref_kernels.tex_probe(ramp_x, fine, c, layer=0)
    out["probe/layered_y"] = ref_kernels.tex_probe(ramp_x, c, fine, layer=1)
    cb = np.full_like(border, 20.5)
    out["probe/border_x"] = ref_kernels.tex_probe(ramp_x, border, cb, layer=0)
    # 3D array, ramp along depth (w axis fixed at texel centres)
    ramp_z = np.broadcast_to(np.arange(16, dtype=np.float32)[:, None, None],
                             (16, 16, 16)).copy()
    c3 = np.full_like(fine, 5.5)
    fine3 = fine - np.float32(4.0)  # keep inside 16 texels
    out["probe/tex3d_z"] = ref_kernels.tex_probe(ramp_z, c3, c3, fine3,
                                                 layered=False)
    ramp_w = np.broadcast_to(np.arange(16, dtype=np.float32)[None, None, :],
                             (16, 16, 16)).copy()
    out["probe/tex3d_x"] = ref_kernels.tex_probe(ramp_w, fine3, c3, c3,
                                                 layered=False)
    tex, xs, ys = probe_random()
    out["probe/random"] = ref_kernels.tex_probe(tex, xs, ys, layer=0)
    tex3, pairs = probe_random3d()
    for pair, (xs, ys, zs) in pairs.items():
        out[f"probe/random3d_{pair}"] = ref_kernels.tex_probe(
            tex3, xs, ys, zs, layered=False)
    out["device"] = np.array(torch.cuda.get_device_name())
    np.savez_compressed(out_path, **out)
    print("wrote", out_path, os.path.getsize(out_path), "bytes")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "gpu_golden.npz")
