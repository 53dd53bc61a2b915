"""SIRT sharded by angle over several GPUs (one process per GPU).

Each rank holds the whole volume and a contiguous share of the angles
(``angle_shard``). An iteration projects the volume over the rank's own
angles with the residual epilogue ``r = (A_k x - y_k) R_k``, backprojects
``r`` into a gradient volume ``g_k = A_k^T r``, sums ``g = sum_k g_k`` with
one all-reduce over the process group (NCCL over NVLink between GPUs),
and applies ``x = clip(mask (x - C g))`` with ``C = 1 / sum_k A_k^T 1``.
That is the single-GPU ``kernelkit.sirt`` (``algo.py:226-368`` of the
reference) except for the order in which the per-angle contributions are
summed, so results agree to float32 rounding.

The per-rank work goes through an operator object (``CudaShardOps`` by
default: this package's kernels on the rank's GPU); any object with the
same methods works, which is how the partition and reduction logic is
tested on host ranks.
"""
from __future__ import annotations

from typing import Sequence

from . import _arrays, _native
from .geom.vol import VolumeGeometry


def angle_shard(n_angles: int, world: int, rank: int) -> tuple:
    """The contiguous angle range ``[start, stop)`` of ``rank``: shares
    differ by at most one angle."""
    if not 0 <= rank < world:
        raise ValueError(f"rank {rank} outside a world of {world}")
    base, extra = divmod(int(n_angles), int(world))
    start = rank * base + min(rank, extra)
    return start, start + base + (1 if rank < extra else 0)


class CudaShardOps:
    """The rank-local operators on this GPU for the angles
    ``projection_geometry`` (the rank's share): forward projection with the
    residual epilogue and backprojection through the layered texture."""

    def __init__(self, projection_geometry: Sequence, volume_geometry:
                 VolumeGeometry):
        from .kernels import RayDrivenConeFP, VoxelDrivenConeBP

        self.pg = list(projection_geometry)
        self.vg = volume_geometry
        self.fp = RayDrivenConeFP()
        self.fp.compile()
        self.fp.set_params(self.fp.geoms2params(self.pg, volume_geometry))
        self.bp = VoxelDrivenConeBP()
        self.bp.compile()
        self.bp.set_params(self.bp.geoms2params(self.pg, volume_geometry))
        det = self.pg[0].detector
        self.shape = (len(self.pg), det.rows, det.cols)
        # the backprojection samples through a layered texture (the
        # reference's filter) while the share fits one
        self.tex = (_native.Layered(*self.shape, _native.KK_F32)
                    if len(self.pg) <= 2048 else None)

    def projections(self, y):
        """The rank's measured projections as a float32 device array."""
        t = _arrays.torch()
        y = _arrays.as_tensor(y).to(t.float32).contiguous()
        if tuple(y.shape) != self.shape:
            raise ValueError(f"projections {tuple(y.shape)} do not match "
                             f"the rank's geometry {self.shape}")
        return y

    def empty_volume(self):
        t = _arrays.torch()
        return t.zeros(tuple(int(s) for s in self.vg.shape),
                       dtype=t.float32, device="cuda")

    def volume_array(self, a):
        """``a`` (NumPy, torch, boolean or float) as a contiguous float32
        device array of the volume's shape, as the reference converts the
        SIRT mask (``algo.py:316-317``)."""
        t = _arrays.torch()
        v = _arrays.as_tensor(a, dtype=t.float32)
        shape = tuple(int(s) for s in self.vg.shape)
        if tuple(v.shape) != shape:
            raise ValueError(f"array of shape {tuple(v.shape)} does not "
                             f"match the volume {shape}")
        return v.contiguous()

    def empty_projections(self):
        t = _arrays.torch()
        return t.zeros(self.shape, dtype=t.float32, device="cuda")

    def project(self, x, out):
        """out = A_k x."""
        self.fp(x, self.pg, self.vg, out, additive=False)

    def residual(self, x, y, weight, out):
        """out = (A_k x - y) * weight."""
        self.fp.residual(x, self.pg, self.vg, out, y, weight)

    def backproject(self, r, out):
        """out = A_k^T r."""
        src = r
        if self.tex is not None:
            self.tex.copy_from(r)
            src = self.tex
        self.bp(src, out, self.vg, additive=False)

    def reciprocal(self, a):
        """a = 1 / a with +inf mapped to 0."""
        _native.check(_native.load().kk_reciprocal(a.data_ptr(), a.numel(),
                                                   _native.current_stream()))

    def update(self, x, g, scale, mask, lo, hi):
        """x = clip(mask * (x - scale * g))."""
        t = _arrays.torch()
        for a in (x, g, scale) + (() if mask is None else (mask,)):
            if (a.dtype != t.float32 or not a.is_cuda
                    or not a.is_contiguous() or a.numel() != x.numel()):
                raise ValueError("the update takes contiguous float32 "
                                 "device arrays of the volume's size")
        _native.check(_native.load().kk_sirt_update(
            x.data_ptr(), g.data_ptr(), scale.data_ptr(), _native.ptr(mask),
            float(lo or 0.0), float(hi or 0.0), int(lo is not None),
            int(hi is not None), x.numel(), _native.current_stream()))


class ShardedSIRT:
    """SIRT over the ranks of ``group`` (the default process group when
    None), each holding the measured projections ``projections`` of its
    own angles ``projection_geometry`` (the share ``angle_shard`` gives it
    of the full scan) and the full volume geometry. ``run`` returns the
    volume, the same on every rank."""

    def __init__(self, projections, projection_geometry: Sequence,
                 volume_geometry: VolumeGeometry, group=None, mask=None,
                 min_constraint: float = None, max_constraint: float = None,
                 ops=None):
        import torch.distributed as dist

        self.dist = dist
        self.group = group
        # every rank needs a share of the angles; agree on that before any
        # rank builds its operators, so that no rank fails alone while the
        # others wait in a collective
        t = _arrays.torch()
        dev = "cuda" if dist.get_backend(group) == "nccl" else "cpu"
        have = t.tensor([1 if len(projection_geometry) > 0 else 0],
                        dtype=t.int32, device=dev)
        dist.all_reduce(have, op=dist.ReduceOp.MIN, group=group)
        if int(have.item()) == 0:
            raise ValueError(
                "ShardedSIRT needs at least one angle on every rank: the "
                "scan has fewer angles than the process group has ranks")
        self.ops = ops or CudaShardOps(projection_geometry, volume_geometry)
        o = self.ops
        self.y = o.projections(projections)
        self.mask = None if mask is None else o.volume_array(mask)
        self.lo, self.hi = min_constraint, max_constraint
        self.x = o.empty_volume()
        # R = 1 / A_k 1 (this rank's angles only)
        self.R = o.empty_projections()
        ones = o.empty_volume() + 1
        o.project(ones, self.R)
        o.reciprocal(self.R)
        # C = 1 / sum_k A_k^T 1 (all angles: summed over the ranks)
        self.C = o.empty_volume()
        o.backproject(o.empty_projections() + 1, self.C)
        dist.all_reduce(self.C, group=group)
        o.reciprocal(self.C)
        self.r = o.empty_projections()
        self.g = o.empty_volume()

    def step(self):
        """One iteration: local residual and backprojection, the gradient
        summed over the ranks, then the update."""
        o = self.ops
        o.residual(self.x, self.y, self.R, self.r)
        o.backproject(self.r, self.g)
        self.dist.all_reduce(self.g, group=self.group)
        o.update(self.x, self.g, self.C, self.mask, self.lo, self.hi)

    def run(self, iters: int):
        for _ in range(int(iters)):
            self.step()
        return self.x


__all__ = ["angle_shard", "CudaShardOps", "ShardedSIRT"]
