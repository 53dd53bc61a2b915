"""Batched problems (kk_cone_fp_batched, kk_cone_bp_layered_batched,
kernelkit.batch.BatchedSIRT): several volumes and scans of different sizes
in one launch must give what the one-problem calls give."""
from __future__ import annotations

import ctypes

import numpy as np
import pytest
import torch

import kernelkit as kk
from conftest import rel_l2
from helpers import build_case, case_volume
from kernelkit import _native
from kernelkit.batch import BP_TILES, FP_SPANS, Autotuner, BatchedSIRT
from kernelkit.kernels import RayDrivenConeFP, VoxelDrivenConeBP

pytestmark = pytest.mark.gpu

CASES = ("small", "config1", "alldirs", "volrot")


def _problem(case):
    pgs, vg = build_case(case)
    vol = torch.as_tensor(case_volume(case, vg), device="cuda")
    fp = RayDrivenConeFP()
    fp.compile()
    fp.set_params(fp.geoms2params(pgs, vg))
    det = pgs[0].detector
    proj = torch.empty((len(pgs), det.rows, det.cols), device="cuda")
    return pgs, vg, vol, fp, proj


def test_batched_forward_projection_equals_single_calls():
    probs = [_problem(c) for c in CASES]
    refs = []
    for pgs, vg, vol, fp, proj in probs:
        fp(vol, pgs, vg, proj, additive=False)
        refs.append(proj.clone())
    arr = (_native.kk_fp_problem * len(probs))()
    keep = []
    for i, (pgs, vg, vol, fp, proj) in enumerate(probs):
        proj.fill_(5.0)
        vdesc = _native.volume_desc(vol)
        lay = fp._volume_texture(vol, vdesc)
        keep.append(lay)
        osc = np.asarray(fp._output_scale(vg.voxel_size), np.float32)
        arr[i] = _native.kk_fp_problem(
            vdesc, _native.projections_desc(proj), fp._params_dev.data_ptr(),
            (ctypes.c_float * 9)(*osc.reshape(9).tolist()),
            lay.handle if lay is not None else None,
            _native.kk_fp_residual(None, None), 0)
    _native.check(_native.load().kk_cone_fp_batched(
        arr, len(probs), _native.KK_INTERP_TEX8, 16,
        _native.current_stream()))
    torch.cuda.synchronize()
    for (_, _, _, _, proj), ref in zip(probs, refs):
        assert rel_l2(proj.cpu().numpy(), ref.cpu().numpy()) <= 1e-7


def test_batched_backprojection_equals_single_calls():
    arr = (_native.kk_bp_problem * len(CASES))()
    outs, refs, keep = [], [], []
    for i, case in enumerate(CASES):
        pgs, vg = build_case(case)
        det = pgs[0].detector
        g = torch.Generator(device="cuda").manual_seed(i)
        y = torch.rand((len(pgs), det.rows, det.cols), generator=g,
                       device="cuda")
        bp = VoxelDrivenConeBP()
        bp.compile()
        bp.set_params(bp.geoms2params(pgs, vg))
        lay = _native.Layered(*y.shape, _native.KK_F32)
        lay.copy_from(y)
        shape = tuple(int(s) for s in vg.shape)
        ref = torch.empty(shape, device="cuda")
        bp(lay, ref, vg, additive=False)
        out = torch.full(shape, 9.0, device="cuda")
        arr[i] = _native.kk_bp_problem(
            lay.handle, _native.volume_desc(out), bp._params_dev.data_ptr(),
            float(np.float32(vg.voxel_volume())),
            _native.kk_bp_update(None, None, 0.0, 0.0, 0, 0), None, 0)
        keep += [lay, bp, y]
        outs.append(out)
        refs.append(ref)
    _native.check(_native.load().kk_cone_bp_layered_batched(
        arr, len(CASES), _native.current_stream()))
    torch.cuda.synchronize()
    for out, ref in zip(outs, refs):
        assert rel_l2(out.cpu().numpy(), ref.cpu().numpy()) <= 1e-7


def _sirt_problems():
    probs = []
    for case in CASES:
        pgs, vg, vol, fp, proj = _problem(case)
        fp(vol, pgs, vg, proj, additive=False)
        probs.append((proj.cpu().numpy(), pgs, vg))
    return probs


def test_batched_sirt_equals_single_sirt_eager_and_graph():
    probs = _sirt_problems()
    iters = 4
    refs = [kk.sirt(y, pgs, vg, iters=iters, verbose=False, use_graph=False,
                    min_constraint=0.0) for (y, pgs, vg) in probs]
    eager = BatchedSIRT(probs, min_constraint=0.0)
    xs = [x.cpu().numpy() for x in eager.run(iters, use_graph=False)]
    graph = BatchedSIRT(probs, min_constraint=0.0)
    xg = [x.cpu().numpy() for x in graph.run(iters, use_graph=True)]
    for r, a, b in zip(refs, xs, xg):
        assert rel_l2(a, r) <= 1e-6
        assert rel_l2(b, a) <= 1e-7


def test_more_problems_than_one_launch_takes():
    pgs, vg = build_case("small")
    pgs = pgs[:6]
    vg = kk.resolve_volume_geometry(shape=8, voxel_size=2.0)
    det = pgs[0].detector
    g = torch.Generator().manual_seed(3)
    probs = [(torch.rand((len(pgs), det.rows, det.cols), generator=g).numpy(),
              pgs, vg) for _ in range(_native.KK_MAX_BATCH + 3)]
    b = BatchedSIRT(probs)
    xs = b.run(2, use_graph=False)
    for i in (0, _native.KK_MAX_BATCH + 2):
        ref = kk.sirt(probs[i][0], pgs, vg, iters=2, verbose=False,
                      use_graph=False)
        assert rel_l2(xs[i].cpu().numpy(), ref) <= 1e-6


def test_autotuner_picks_and_caches(tmp_path):
    probs = _sirt_problems()[:2]
    path = tmp_path / "tune.json"
    tuner = Autotuner(str(path), reps=1)
    b = BatchedSIRT(probs, autotuner=tuner)
    fp_keys = [k for k in tuner.cache if k.startswith("fp_axis_group:")]
    bp_keys = [k for k in tuner.cache if k.startswith("bp_tile:")]
    span_keys = [k for k in tuner.cache if k.startswith("fp_span:")]
    assert len(fp_keys) == 2 and len(bp_keys) == 2 and len(span_keys) == 2
    assert all(tuner.cache[k] in FP_SPANS for k in span_keys)
    assert all(tuner.cache[k] in (1, 2, 4, 8) for k in fp_keys)
    assert all(tuple(tuner.cache[k]) in BP_TILES for k in bp_keys)
    assert [s.fp.axis_group for s in b.solvers] == [tuner.cache[k]
                                                    for k in fp_keys]
    assert [s._bp_tile for s in b.solvers] == [tuple(tuner.cache[k])
                                               for k in bp_keys]
    # a second tuner reads the file and times nothing
    again = Autotuner(str(path))
    calls = []
    assert again.pick(fp_keys[0], (1, 2),
                      lambda c: calls.append(c)) in (1, 2, 4, 8)
    assert calls == []


def _bp_batch(cases, update=False):
    """kk_bp_problem array over random sinograms of the golden cases (with
    the SIRT update epilogue when ``update``), fresh volumes, keep-alive."""
    arr = (_native.kk_bp_problem * len(cases))()
    outs, keep = [], []
    for i, case in enumerate(cases):
        pgs, vg = build_case(case)
        det = pgs[0].detector
        g = torch.Generator(device="cuda").manual_seed(20 + i)
        y = torch.rand((len(pgs), det.rows, det.cols), generator=g,
                       device="cuda")
        bp = VoxelDrivenConeBP()
        bp.compile()
        bp.set_params(bp.geoms2params(pgs, vg))
        lay = _native.Layered(*y.shape, _native.KK_F32)
        lay.copy_from(y)
        shape = tuple(int(s) for s in vg.shape)
        out = torch.rand(shape, generator=g, device="cuda")
        scale = torch.rand(shape, generator=g, device="cuda")
        work = torch.empty(out.numel(), device="cuda")
        upd = (_native.kk_bp_update(scale.data_ptr(), None, 0.0, 0.0, 1, 0)
               if update else _native.kk_bp_update(None, None, 0.0, 0.0, 0, 0))
        arr[i] = _native.kk_bp_problem(
            lay.handle, _native.volume_desc(out), bp._params_dev.data_ptr(),
            float(np.float32(vg.voxel_volume())), upd,
            work.data_ptr() if update else None, 0, 2 * (i % 2), 0)
        keep += [lay, bp, y, scale, work]
        outs.append(out)
    return arr, outs, keep


@pytest.mark.parametrize("update", [False, True])
def test_persistent_backprojection_equals_per_chunk_launches(update):
    """One persistent launch walking (chunk group, problem, tile) items
    gives the per-chunk-index launches' volumes bit for bit (360-, 96-,
    24-, 18- and 12-angle scans: 12, 3, 1, 1 and 1 chunks, i.e. 3, 1, 1, 1
    and 1 groups of four, so items of later groups wait on earlier ones)."""
    cases = ("config2", "config1", "small", "alldirs", "volrot")
    arr, ref, keep = _bp_batch(cases, update)
    start = [o.clone() for o in ref]
    _native.check(_native.load().kk_cone_bp_layered_batched(
        arr, len(cases), _native.current_stream()))
    arr2, got, keep2 = _bp_batch(cases, update)
    for g, s0 in zip(got, start):
        g.copy_(s0)
    L = _native.load()
    elems = int(L.kk_bp_batch_sync_elems(arr2, len(cases)))
    sync = torch.zeros(elems, dtype=torch.int32, device="cuda")
    opts = _native.kk_bp_batch_options(1, sync.data_ptr(), elems, 0, -1)
    for _ in range(2):  # the counters are re-zeroed by every call
        for g, s0 in zip(got, start):
            g.copy_(s0)
        _native.check(L.kk_cone_bp_layered_batched_ex(
            arr2, len(cases), opts, _native.current_stream()))
        torch.cuda.synchronize()
        for a, b in zip(got, ref):
            assert torch.equal(a, b)
    assert _native.wait_timeouts() == 0


def test_persistent_backprojection_wait_runs_out():
    """An item that never completes (a flag nothing sets): the item of the
    tile's next chunk group waits out a short budget, the launch aborts
    instead of hanging and the host reads the timeout; the library keeps
    working. The first problem has more than one group of four 32-angle
    chunks (config 2: 360 angles), so a later item waits on item 0."""
    cases = ("config2", "small")
    arr, outs, keep = _bp_batch(cases)
    L = _native.load()
    elems = int(L.kk_bp_batch_sync_elems(arr, len(cases)))
    sync = torch.zeros(elems, dtype=torch.int32, device="cuda")
    assert _native.wait_timeouts() == 0
    opts = _native.kk_bp_batch_options(1, sync.data_ptr(), elems, 1 << 20, 0)
    _native.check(L.kk_cone_bp_layered_batched_ex(
        arr, len(cases), opts, _native.current_stream()))
    torch.cuda.synchronize()
    assert _native.wait_timeouts() >= 1
    assert int(sync[1]) == 1  # the abort flag
    # a normal call afterwards completes without timeouts
    opts.test_skip_item = -1
    _native.check(L.kk_cone_bp_layered_batched_ex(
        arr, len(cases), opts, _native.current_stream()))
    torch.cuda.synchronize()
    assert _native.wait_timeouts() == 0
    assert int(sync[0]) >= 1


def test_batched_forward_projection_spans_per_problem():
    """Problems traced in slice spans of their own (16, 48, one launch)
    within the batched launches give their one-launch results bit for
    bit."""
    probs = [_problem(c) for c in CASES]
    arr = (_native.kk_fp_problem * len(probs))()
    refs, keep = [], []
    for i, (pgs, vg, vol, fp, proj) in enumerate(probs):
        vdesc = _native.volume_desc(vol)
        osc = np.asarray(fp._output_scale(vg.voxel_size), np.float32)
        arr[i] = _native.kk_fp_problem(
            vdesc, _native.projections_desc(proj), fp._params_dev.data_ptr(),
            (ctypes.c_float * 9)(*osc.reshape(9).tolist()), None,
            _native.kk_fp_residual(None, None), 1, -1)
    L = _native.load()
    for _, _, _, _, proj in probs:
        proj.fill_(0.5)
    _native.check(L.kk_cone_fp_batched(arr, len(probs),
                                       _native.KK_INTERP_TEX8, 16,
                                       _native.current_stream()))
    refs = [p[4].clone() for p in probs]
    for i, span in enumerate((16, 48, -1, 16)):
        arr[i].span = span
    for _, _, _, _, proj in probs:
        proj.fill_(0.5)
    _native.check(L.kk_cone_fp_batched(arr, len(probs),
                                       _native.KK_INTERP_TEX8, 16,
                                       _native.current_stream()))
    torch.cuda.synchronize()
    for (_, _, _, _, proj), ref in zip(probs, refs):
        assert torch.equal(proj, ref)


def test_batched_sirt_persistent_equals_per_chunk():
    probs = _sirt_problems()
    a = BatchedSIRT(probs, min_constraint=0.0, persistent=True)
    b = BatchedSIRT(probs, min_constraint=0.0, persistent=False)
    xa = [x.clone() for x in a.run(3, use_graph=True)]
    xb = b.run(3, use_graph=True)
    for u, v in zip(xa, xb):
        assert torch.equal(u, v)
