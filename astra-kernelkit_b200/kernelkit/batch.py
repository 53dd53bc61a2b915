"""Many independent reconstruction problems at once.

Volumes and scans of different sizes (e.g. a stack of small samples) are
solved together: every SIRT iteration of every problem is one batched
forward-projection launch (``kk_cone_fp_batched``: up to 64 problems per
launch, each thread block picking its own problem), the texture refills,
and one persistent backprojection launch (``kk_cone_bp_layered_batched_ex``:
resident thread blocks claim (chunk group, problem, tile) items in group
order, a group being four 32-angle chunks, each waiting with a bounded
spin for its tile's previous group) or, with ``persistent=False``, one
launch per 32-angle chunk index. The whole
iteration sequence can be captured in one CUDA graph. Launch-shape
choices (the forward projector's record grouping, the backprojection's
super-column shape, the slice span per launch) are made per problem
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

#: backprojection super-column shapes tried (thread blocks along the
#: fastest x middle volume axes swept together along the slowest)
BP_TILES = ((8, 64), (4, 32), (8, 16), (2, 8))

#: forward-projection slice spans tried (slices per launch; 0 = the
#: library's automatic span)
FP_SPANS = (0, 96, 64)


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
                 autotuner: Autotuner | None = None, persistent: bool = True):
        t = _arrays.torch()
        self.solvers = []
        self._vtex = []
        self.persistent = bool(persistent)
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
                _native.kk_fp_residual(s.y.data_ptr(), s.R.data_ptr()), 0,
                int(getattr(s, "_fp_span", 0))))
            upd = _native.kk_bp_update(
                s.C.data_ptr(), _native.ptr(s.mask),
                float(s.min_c) if s.min_c is not None else 0.0,
                float(s.max_c) if s.max_c is not None else 0.0,
                int(s.min_c is not None), int(s.max_c is not None))
            tz, ty = getattr(s, "_bp_tile", (0, 0))
            self._bp.append(_native.kk_bp_problem(
                s.tex.handle, _native.volume_desc(s.x),
                s.bp._params_dev.data_ptr(),
                float(np.float32(s.vg.voxel_volume())), upd,
                s.bp._work_for(s.x, True) or None, 0, tz, ty))
        n = len(self.solvers)
        self._fp_groups = []
        self._bp_groups = []
        L = _native.load()
        for g in range(0, n, _native.KK_MAX_BATCH):
            m = min(_native.KK_MAX_BATCH, n - g)
            fa = (_native.kk_fp_problem * m)(*self._fp[g:g + m])
            ba = (_native.kk_bp_problem * m)(*self._bp[g:g + m])
            opts = None
            if self.persistent:
                elems = int(L.kk_bp_batch_sync_elems(ba, m))
                if elems < 0:
                    _native.check(_native.KK_ERR_INVALID_ARGUMENT)
                sync = t.zeros(elems, dtype=t.int32, device="cuda")
                opts = _native.kk_bp_batch_options(1, sync.data_ptr(), elems,
                                                   0, -1)
                opts._sync = sync  # keep the buffer alive with the options
            self._fp_groups.append((fa, m))
            self._bp_groups.append((ba, m, opts))
        self._graph = None
        self._t = t

    @staticmethod
    def _tune(s: SIRT, tuner: Autotuner):
        sig = json.dumps([list(s.x.shape), int(s.y.shape[0]),
                          list(s.y.shape[1:])])

        def run(g):
            s.fp.axis_group = int(g)
            s.fp._upload()
            s.fp.residual(s.x, s.pg, s.vg, s.y_tmp, s.y, s.R)

        best = tuner.pick("fp_axis_group:" + sig, AXIS_GROUPS, run)
        s.fp.axis_group = int(best)
        s.fp._upload()

        def run_span(span):
            s.fp.slices_per_launch = int(span)
            s.fp.residual(s.x, s.pg, s.vg, s.y_tmp, s.y, s.R)

        s._fp_span = int(tuner.pick("fp_span:" + sig, FP_SPANS, run_span))
        s.fp.slices_per_launch = s._fp_span
        # backprojection block order: a plain backprojection of the
        # problem's texture into a scratch volume per candidate shape
        scratch = _arrays.torch().empty_like(s.x)
        L = _native.load()
        zero = _native.kk_bp_update(None, None, 0.0, 0.0, 0, 0)

        def run_bp(shape):
            one = (_native.kk_bp_problem * 1)(_native.kk_bp_problem(
                s.tex.handle, _native.volume_desc(scratch),
                s.bp._params_dev.data_ptr(),
                float(np.float32(s.vg.voxel_volume())), zero, None, 0,
                int(shape[0]), int(shape[1])))
            _native.check(L.kk_cone_bp_layered_batched(
                one, 1, _native.current_stream()))

        s._bp_tile = tuple(tuner.pick("bp_tile:" + sig, BP_TILES, run_bp))
        del scratch

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
        for ba, m, opts in self._bp_groups:
            if opts is None:
                _native.check(L.kk_cone_bp_layered_batched(ba, m, stream))
            else:
                _native.check(L.kk_cone_bp_layered_batched_ex(ba, m, opts,
                                                              stream))

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


__all__ = ["Autotuner", "BatchedSIRT", "AXIS_GROUPS", "BP_TILES", "FP_SPANS"]
