"""Many independent reconstruction problems at once.

Volumes and scans of different sizes (e.g. a stack of small samples) are
solved together: every SIRT iteration of every problem is one batched
forward-projection launch (``kk_cone_fp_batched``: up to 64 problems per
launch, each thread block picking its own problem), the texture refills,
and one batched backprojection launch per 32-angle chunk index
(``kk_cone_bp_layered_batched``). The whole iteration sequence can be
captured in one CUDA graph. Launch-shape choices are made per problem
shape by ``Autotuner`` (timed on the problems themselves, cached).

This has no counterpart in the reference, which solves one problem per
call (``algo.py:226-368``); each problem's arithmetic is the same as
``kernelkit.sirt``'s.
"""
from __future__ import annotations

import json
import os
from typing import Callable, Sequence

import numpy as np

from . import _arrays, _native
from .algo import SIRT


class Autotuner:
    """Picks, per problem signature, the fastest of a few candidate
    settings by timing them with CUDA events (median of ``reps`` runs after
    one warm-up). Results are kept in memory and, when ``path`` is given,
    in a JSON file so later processes reuse them."""

    def __init__(self, path: str | None = None, reps: int = 3):
        self.path = path
        self.reps = int(reps)
        self.cache: dict = {}
        if path and os.path.exists(path):
            with open(path) as f:
                self.cache = json.load(f)

    def pick(self, key: str, candidates: Sequence, run: Callable) -> object:
        """The candidate with the smallest median time of ``run(c)``."""
        if key in self.cache:
            return self.cache[key]
        t = _arrays.torch()
        best, best_ms = None, float("inf")
        for c in candidates:
            run(c)  # warm-up (and first-use allocations)
            times = []
            for _ in range(self.reps):
                a = t.cuda.Event(enable_timing=True)
                b = t.cuda.Event(enable_timing=True)
                a.record()
                run(c)
                b.record()
                b.synchronize()
                times.append(a.elapsed_time(b))
            ms = float(np.median(times))
            if ms < best_ms:
                best, best_ms = c, ms
        self.cache[key] = best
        if self.path:
            os.makedirs(os.path.dirname(os.path.abspath(self.path)),
                        exist_ok=True)
            with open(self.path, "w") as f:
                json.dump(self.cache, f)
        return best


#: record-group sizes tried for the forward projection (how many records
#: of one ray axis are launched back to back)
AXIS_GROUPS = (1, 2, 4, 8)


class BatchedSIRT:
    """SIRT on many problems at once.

    ``problems`` is a sequence of ``(projections, projection_geometry,
    volume_geometry)``; projections are (angles, rows, cols) arrays. Each
    problem's state is that of ``kernelkit.algo.SIRT`` (``x`` starts at 0,
    ``C = 1 / A^T 1``, ``R = 1 / A 1``); constraints apply to every
    problem. ``autotuner`` (optional) picks the forward projector's record
    grouping per problem shape."""

    def __init__(self, problems, mask=None, min_constraint: float = None,
                 max_constraint: float = None,
                 autotuner: Autotuner | None = None):
        t = _arrays.torch()
        self.solvers = []
        self._vtex = []
        for i, (y, pg, vg) in enumerate(problems):
            s = SIRT(y, pg, vg, mask=None if mask is None else mask[i],
                     min_constraint=min_constraint,
                     max_constraint=max_constraint)
            if s.tex is None:
                raise NotImplementedError(
                    "Batched SIRT needs at most 2048 angles per problem.")
            if autotuner is not None:
                self._tune(s, autotuner)
            self.solvers.append(s)
            x = s.x
            self._vtex.append(_native.Layered(*x.shape, _native.KK_F32)
                              if x.shape[0] <= 2048 else None)
        self._fp = []
        self._bp = []
        for s, lay in zip(self.solvers, self._vtex):
            osc = np.asarray(s.fp._output_scale(s.vg.voxel_size),
                             np.float32).reshape(9)
            self._fp.append(_native.kk_fp_problem(
                _native.volume_desc(s.x), _native.projections_desc(s.y_tmp),
                s.fp._params_dev.data_ptr(),
                (ctypes_float9(osc)), lay.handle if lay is not None else None,
                _native.kk_fp_residual(s.y.data_ptr(), s.R.data_ptr()), 0))
            upd = _native.kk_bp_update(
                s.C.data_ptr(), _native.ptr(s.mask),
                float(s.min_c) if s.min_c is not None else 0.0,
                float(s.max_c) if s.max_c is not None else 0.0,
                int(s.min_c is not None), int(s.max_c is not None))
            self._bp.append(_native.kk_bp_problem(
                s.tex.handle, _native.volume_desc(s.x),
                s.bp._params_dev.data_ptr(),
                float(np.float32(s.vg.voxel_volume())), upd,
                s.bp._work_for(s.x, True) or None, 0))
        n = len(self.solvers)
        self._fp_groups = []
        self._bp_groups = []
        for g in range(0, n, _native.KK_MAX_BATCH):
            m = min(_native.KK_MAX_BATCH, n - g)
            fa = (_native.kk_fp_problem * m)(*self._fp[g:g + m])
            ba = (_native.kk_bp_problem * m)(*self._bp[g:g + m])
            self._fp_groups.append((fa, m))
            self._bp_groups.append((ba, m))
        self._graph = None
        self._t = t

    @staticmethod
    def _tune(s: SIRT, tuner: Autotuner):
        key = "fp_axis_group:" + json.dumps(
            [list(s.x.shape), int(s.y.shape[0]), list(s.y.shape[1:])])

        def run(g):
            s.fp.axis_group = int(g)
            s.fp._upload()
            s.fp.residual(s.x, s.pg, s.vg, s.y_tmp, s.y, s.R)

        best = tuner.pick(key, AXIS_GROUPS, run)
        s.fp.axis_group = int(best)
        s.fp._upload()

    @property
    def volumes(self):
        """The current reconstructions (one device tensor per problem)."""
        return [s.x for s in self.solvers]

    def step(self):
        """One iteration of every problem: volume-texture refills, one
        batched residual projection, projection-texture refills and the
        batched update backprojection."""
        L = _native.load()
        stream = _native.current_stream()
        for s, lay in zip(self.solvers, self._vtex):
            if lay is not None:
                lay.copy_from(s.x)
        for fa, m in self._fp_groups:
            _native.check(L.kk_cone_fp_batched(
                fa, m, _native.KK_INTERP_TEX8, 16, stream))
        for s in self.solvers:
            s.tex.copy_from(s.y_tmp)
        for ba, m in self._bp_groups:
            _native.check(L.kk_cone_bp_layered_batched(ba, m, stream))

    def capture(self, iters: int = 1):
        """Capture ``iters`` iterations into one CUDA graph."""
        t = self._t
        g = t.cuda.CUDAGraph()
        st = t.cuda.Stream()
        st.wait_stream(t.cuda.current_stream())
        with t.cuda.stream(st):
            with t.cuda.graph(g, stream=st):
                for _ in range(iters):
                    self.step()
        t.cuda.current_stream().wait_stream(st)
        self._graph = (g, iters)
        return g

    def run(self, iters: int, use_graph: bool = True):
        """Run ``iters`` iterations (in one captured graph when
        ``use_graph``); returns the volumes."""
        if not use_graph:
            for _ in range(iters):
                self.step()
            return self.volumes
        if self._graph is None or self._graph[1] != iters:
            self.capture(iters)
        self._graph[0].replay()
        return self.volumes


def ctypes_float9(a) -> object:
    import ctypes

    return (ctypes.c_float * 9)(*[float(v) for v in np.asarray(a).reshape(9)])


__all__ = ["Autotuner", "BatchedSIRT", "AXIS_GROUPS"]
