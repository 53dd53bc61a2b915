"""FDK and SIRT pinned to the reference's own chain at config 1 (64^3, 96
angles, 96^2) and config 2 (256^3, 360 angles, 384^2).

* FDK: the oracle's pre-weighting and Ram-Lak filter (the reference's
  ``processing.py:96-188`` restated in float64 and pinned to the
  reference's own Python output by ``tests/test_oracle.py``) feed the
  reference's own backprojection kernel (``cuda/cone_bp.cu``, built from
  its sources into ``oracle/_ref``); ``kk.fdk`` from host and from device
  input must agree with it to rel. L2 <= 1e-5, the float32 bar.
* SIRT: the oracle's SIRT update (``algo.py:226-368``, float64) iterated
  with the reference's own forward and backprojection kernels as A and
  A^T; ``kk.sirt`` and ``ShardedSIRT`` (one NCCL rank) must agree with it.
  Tolerance 1e-5: our iteration keeps the update in float32 (as the
  reference does) where the oracle keeps it in float64, and the
  difference stays at float32 rounding over the iterations (measured
  ~1e-7).
"""
from __future__ import annotations

import socket

import numpy as np
import pytest
import torch

import kernelkit as kk
from cases import phantom_for
from conftest import rel_l2
from helpers import build_case
from kernelkit import phantom
from kernelkit.kernels import RayDrivenConeFP, VoxelDrivenConeBP
from oracle import processing as oproc
from oracle import ref_kernels

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not ref_kernels.available(),
                                 reason="oracle/_ref/libkkref.so not built")]

TOL = 1e-5


def _problem(name):
    pgs, vg = build_case(name)
    ph = phantom_for(name, vg.shape)
    ell = phantom.random_ellipsoids(ph["k"], ph["center_range"],
                                    ph["axes_range"], seed=ph["seed"])
    vol = phantom.voxelize_torch(ell, vg.shape, vg.extent_min,
                                 vg.voxel_size, device="cuda")
    return pgs, vg, vol


class RefOps:
    """The reference's own kernels as float64-in/float64-out operators."""

    def __init__(self, pgs, vg):
        det = pgs[0].detector
        self.rows, self.cols = det.rows, det.cols
        fpar = RayDrivenConeFP.geoms2params(pgs, vg)
        self.rows12 = np.stack([np.asarray(p, np.float32) for p in fpar], 1)
        self.axes = fpar.axes
        self.osc = RayDrivenConeFP._output_scale(vg.voxel_size)
        self.bpar = np.asarray(VoxelDrivenConeBP.geoms2params(pgs, vg)
                               ).reshape(-1, 12)
        self.shape = tuple(int(s) for s in vg.shape)
        self.vox = vg.voxel_volume()

    def A(self, x):
        v = torch.as_tensor(np.asarray(x, np.float32), device="cuda")
        p, _ = ref_kernels.ref_cone_fp(v, self.rows12, self.axes, self.rows,
                                       self.cols, self.osc)
        return p.double().cpu().numpy()

    def AT(self, y):
        p = torch.as_tensor(np.asarray(y, np.float32), device="cuda")
        v, _ = ref_kernels.ref_cone_bp(p, self.bpar, self.shape, self.vox)
        return v.double().cpu().numpy()


@pytest.mark.parametrize("name", ["config1", "config2"])
def test_fdk_matches_reference_chain(name):
    pgs, vg, vol = _problem(name)
    y = kk.XrayTransform(pgs, vg)(vol).cpu().numpy()
    ops = RefOps(pgs, vg)
    ref = ops.AT(oproc.filter_rows(oproc.preweight(y, pgs)))
    got_host = kk.fdk(y.copy(), pgs, vg)
    assert rel_l2(got_host, ref) <= TOL
    dev = torch.as_tensor(y, device="cuda")
    got_dev = kk.fdk(dev, pgs, vg)
    assert rel_l2(got_dev, ref) <= TOL
    assert np.abs(ref).max() > 0


@pytest.mark.parametrize("name", ["config1", "config2"])
def test_sirt_matches_reference_chain(name):
    iters = 10
    pgs, vg, vol = _problem(name)
    y = kk.XrayTransform(pgs, vg)(vol).cpu().numpy()
    ops = RefOps(pgs, vg)
    ref = oproc.sirt(y, ops.A, ops.AT, ops.shape, iters, vmin=0.0)
    got = kk.sirt(y, pgs, vg, iters=iters, verbose=False, min_constraint=0.0)
    assert rel_l2(got, ref) <= TOL
    assert np.abs(ref).max() > 0


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_sharded_sirt_one_rank_matches_reference_chain():
    import torch.distributed as dist

    from kernelkit.distributed import ShardedSIRT

    pgs, vg, vol = _problem("config1")
    y = kk.XrayTransform(pgs, vg)(vol).contiguous()
    ops = RefOps(pgs, vg)
    ref = oproc.sirt(y.cpu().numpy(), ops.A, ops.AT, ops.shape, 5, vmin=0.0)
    dist.init_process_group("nccl", rank=0, world_size=1,
                            init_method=f"tcp://127.0.0.1:{_free_port()}")
    try:
        x = ShardedSIRT(y, pgs, vg, min_constraint=0.0).run(5)
        torch.cuda.synchronize()
    finally:
        dist.destroy_process_group()
    assert rel_l2(x.cpu().numpy(), ref) <= TOL
