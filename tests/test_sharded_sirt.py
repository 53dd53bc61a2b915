"""SIRT sharded by angle (kernelkit.distributed).

Host part (no GPU): two gloo ranks, each with the oracle's projectors on
its own share of the angles, run ``ShardedSIRT``; the result must equal the
oracle's unsharded SIRT over all angles (float64, so to rounding). The
GPU part checks the update kernel ``kk_sirt_update`` against a float32
torch reference and ``ShardedSIRT`` on one rank (NCCL, world size 1)
against the single-GPU solver, plus that summing the per-shard
backprojections gives the whole-scan backprojection.
"""
from __future__ import annotations

import os
import socket

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

from kernelkit.distributed import angle_shard


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("n,world", [(10, 3), (7, 7), (3, 4), (720, 8)])
def test_angle_shards_cover_the_scan_once(n, world):
    spans = [angle_shard(n, world, r) for r in range(world)]
    assert spans[0][0] == 0 and spans[-1][1] == n
    for (a, b), (c, d) in zip(spans, spans[1:]):
        assert b == c
    sizes = [b - a for a, b in spans]
    assert max(sizes) - min(sizes) <= 1 and min(sizes) >= 0
    with pytest.raises(ValueError):
        angle_shard(n, world, world)


def _oracle_problem():
    """Tiny scan of the 'small' golden case (every third angle), its
    phantom and the oracle's projector functions for a subset of angles."""
    from helpers import build_case, case_volume, fp_params_rows
    from kernelkit.kernels import RayDrivenConeFP, VoxelDrivenConeBP
    from oracle import cone

    pgs, vg = build_case("small")
    pgs = pgs[::3]
    vol = case_volume("small", vg)
    det = pgs[0].detector
    osc = RayDrivenConeFP._output_scale(vg.voxel_size)

    def ops_for(sub):
        fpar = RayDrivenConeFP.geoms2params(sub, vg)
        rows = fp_params_rows(fpar)
        bpar = VoxelDrivenConeBP.geoms2params(sub, vg)

        def A(x):
            return cone.cone_fp(x, rows, fpar.axes, det.rows, det.cols, osc)

        def AT(y):
            return cone.cone_bp(y, bpar, vg.shape, vg.voxel_volume())
        return A, AT
    return pgs, vg, vol, ops_for


class OracleShardOps:
    """Rank-local operators of ``ShardedSIRT`` computed by the oracle in
    float64 on host tensors (the checker's stand-in for the GPU kernels)."""

    def __init__(self, A, AT, vol_shape, proj_shape):
        self.A, self.AT = A, AT
        self.vol_shape, self.proj_shape = tuple(vol_shape), tuple(proj_shape)

    def projections(self, y):
        return torch.as_tensor(np.asarray(y, np.float64))

    def empty_volume(self):
        return torch.zeros(self.vol_shape, dtype=torch.float64)

    def empty_projections(self):
        return torch.zeros(self.proj_shape, dtype=torch.float64)

    def volume_array(self, a):
        return torch.as_tensor(np.asarray(a, np.float64))

    def project(self, x, out):
        out.copy_(torch.from_numpy(self.A(x.numpy())))

    def residual(self, x, y, weight, out):
        out.copy_((torch.from_numpy(self.A(x.numpy())) - y) * weight)

    def backproject(self, r, out):
        out.copy_(torch.from_numpy(self.AT(r.numpy())))

    def reciprocal(self, a):
        with np.errstate(divide="ignore"):
            a.copy_(1.0 / a)
        a[torch.isinf(a)] = 0.0

    def update(self, x, g, scale, mask, lo, hi):
        v = x - scale * g
        if mask is not None:
            v = v * mask
        if lo is not None or hi is not None:
            v = v.clamp(lo, hi)
        x.copy_(v)


def _mask(shape):
    """A seeded 0/1 mask (about 80 % ones)."""
    return (np.random.default_rng(9).random(shape) < 0.8).astype(np.float64)


def _rank_main(rank, world, port, iters, lo, masked, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port),
                      CUDA_VISIBLE_DEVICES="")
    import sys

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    for p in (root, os.path.join(root, "astra-kernelkit_b200"),
              os.path.join(root, "tests")):
        sys.path.insert(0, p)
    import torch.distributed as dist
    from kernelkit.distributed import ShardedSIRT, angle_shard

    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        pgs, vg, vol, ops_for = _oracle_problem()
        a, b = angle_shard(len(pgs), world, rank)
        A, AT = ops_for(pgs[a:b])
        y = A(vol)
        det = pgs[0].detector
        ops = OracleShardOps(A, AT, vol.shape, (b - a, det.rows, det.cols))
        mask = torch.from_numpy(_mask(vol.shape)) if masked else None
        solver = ShardedSIRT(y, pgs[a:b], vg, ops=ops, min_constraint=lo,
                             mask=mask)
        x = solver.run(iters).numpy().copy()
        out.put((rank, a, b, x))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,lo,masked", [(2, None, False),
                                             (3, 0.0, False), (2, 0.0, True)])
def test_sharded_sirt_equals_the_unsharded_oracle(world, lo, masked):
    """ShardedSIRT over gloo ranks, each with a share of the angles, gives
    the oracle's SIRT over the whole scan."""
    iters = 3
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main,
                         args=(r, world, port, iters, lo, masked, q))
             for r in range(world)]
    for p in procs:
        p.start()
    res = sorted((q.get(timeout=300) for _ in range(world)),
                 key=lambda r: r[0])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    from oracle import processing as oproc

    pgs, vg, vol, ops_for = _oracle_problem()
    # the shares tile the scan
    assert [r[1] for r in res][0] == 0 and res[-1][2] == len(pgs)
    A, AT = ops_for(pgs)
    ref = oproc.sirt(A(vol), A, AT, vol.shape, iters, vmin=lo,
                     mask=_mask(vol.shape) if masked else None)
    for _, _, _, x in res:
        np.testing.assert_allclose(x, ref, rtol=1e-9, atol=1e-12)
    assert np.linalg.norm(ref) > 0


def _rank_empty_share(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port),
                      CUDA_VISIBLE_DEVICES="")
    import sys

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    for p in (root, os.path.join(root, "astra-kernelkit_b200"),
              os.path.join(root, "tests")):
        sys.path.insert(0, p)
    import torch.distributed as dist
    from kernelkit.distributed import ShardedSIRT, angle_shard

    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        pgs, vg, vol, ops_for = _oracle_problem()
        pgs = pgs[:world - 1]             # one angle short of a full share
        a, b = angle_shard(len(pgs), world, rank)
        try:
            ShardedSIRT(None, pgs[a:b], vg, ops=object())
            out.put((rank, "constructed"))
        except ValueError as e:
            out.put((rank, "ValueError" if "every rank" in str(e) else str(e)))
    finally:
        dist.destroy_process_group()


def test_sharded_sirt_with_an_empty_share_fails_on_every_rank():
    """Fewer angles than ranks: every rank raises the same ValueError
    before any rank builds its operators, so none waits alone in a
    collective."""
    world = 3
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_empty_share, args=(r, world, port, q))
             for r in range(world)]
    for p in procs:
        p.start()
    res = sorted((q.get(timeout=300) for _ in range(world)))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r[1] for r in res] == ["ValueError"] * world


# ---- GPU ---------------------------------------------------------------

@pytest.mark.gpu
@pytest.mark.parametrize("masked,lo,hi", [(False, None, None),
                                          (True, 0.0, None),
                                          (True, -0.2, 0.3)])
def test_sirt_update_kernel(masked, lo, hi):
    from kernelkit import _native

    g = torch.Generator(device="cuda").manual_seed(2)
    n = 1_000_003
    x = torch.randn(n, generator=g, device="cuda")
    grad = torch.randn(n, generator=g, device="cuda")
    scale = torch.rand(n, generator=g, device="cuda")
    mask = (torch.rand(n, generator=g, device="cuda") > 0.3).float() \
        if masked else None
    ref = x - scale * grad
    if mask is not None:
        ref = ref * mask
    if lo is not None or hi is not None:
        ref = ref.clamp(lo, hi)
    _native.check(_native.load().kk_sirt_update(
        x.data_ptr(), grad.data_ptr(), scale.data_ptr(), _native.ptr(mask),
        float(lo or 0.0), float(hi or 0.0), int(lo is not None),
        int(hi is not None), n, _native.current_stream()))
    torch.cuda.synchronize()
    assert torch.equal(x, ref)


@pytest.mark.gpu
def test_shard_backprojections_sum_to_the_whole_scan():
    from helpers import build_case
    from kernelkit.distributed import CudaShardOps

    pgs, vg = build_case("small")
    det = pgs[0].detector
    y = torch.rand((len(pgs), det.rows, det.cols), device="cuda",
                   generator=torch.Generator(device="cuda").manual_seed(4))
    whole = CudaShardOps(pgs, vg)
    ref = whole.empty_volume()
    whole.backproject(y, ref)
    acc = whole.empty_volume()
    for r in range(3):
        a, b = angle_shard(len(pgs), 3, r)
        part = CudaShardOps(pgs[a:b], vg)
        g = part.empty_volume()
        part.backproject(y[a:b].contiguous(), g)
        acc += g
    rel = float((acc - ref).norm() / ref.norm())
    assert rel <= 1e-6


@pytest.mark.gpu
def test_sharded_sirt_on_one_rank_matches_the_single_gpu_solver():
    import torch.distributed as dist

    import kernelkit as kk
    from helpers import build_case, case_volume
    from kernelkit.distributed import ShardedSIRT

    pgs, vg = build_case("small")
    vol = torch.from_numpy(case_volume("small", vg)).float().cuda()
    y = kk.XrayTransform(pgs, vg)(vol).contiguous()
    dist.init_process_group("nccl", rank=0, world_size=1,
                            init_method=f"tcp://127.0.0.1:{_free_port()}")
    try:
        x = ShardedSIRT(y, pgs, vg, min_constraint=0.0).run(5)
        torch.cuda.synchronize()
    finally:
        dist.destroy_process_group()
    ref = kk.SIRT(y, pgs, vg, min_constraint=0.0).run(5, use_graph=False)
    rel = float((x - ref).norm() / ref.norm())
    assert rel <= 1e-5
