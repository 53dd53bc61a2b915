#!/usr/bin/env python
"""Benchmark of the cone-beam hot path: forward projection + backprojection
GUPS (giga voxel-angle updates per second) at 512^3 voxels / 720 angles /
768^2 detector, the headline workload.

One step = one forward projection of the volume over all angles plus one
backprojection of a full sinogram, with the data resident in HBM (inputs
larger than L2, so no flush is needed). GUPS(FP+BP) = 2 N / (t_FP + t_BP)
with N = voxels x angles. Also reported: the same metric end to end
through ``XrayTransform`` with the volume coming from and going back to
pinned host memory (x -> A^T A x), a roofline entry for the dominant
kernel, and a CPU baseline (the FP64 NumPy oracle on a bounded sample on
the host cores). ``--impl reference`` times the reference arm, the
oracle's restatement of the reference algorithm on all host cores.

Usage: python bench.py [--gpus N] [--steps K] [--warmup W]
       [--impl ours|reference] [--workload headline|config2|profile]
Multi-GPU runs (torchrun) are independent replicas, one per GPU.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
for _p in (ROOT, os.path.join(ROOT, "astra-kernelkit_b200")):
    if _p not in sys.path:
        sys.path.insert(0, _p)

import numpy as np  # noqa: E402

METRIC = "cone FP+BP GUPS @512^3/720 ang"
#: float32 2D-layered bilinear fetches per clock per SM of the B200's
#: texture unit, measured (profiles/texture_unit_rate.md)
TMU_FETCH_PER_CLK_SM = 3.83
UNIT = "GUPS"

WORKLOADS = {
    # 512^3, 720 angles over 2 pi, 768^2 detector, SOD 1600, SDD 3200,
    # pitch 1.3, voxel 1.0, 200 ellipsoids (config-2 ranges scaled x2)
    "headline": dict(n=512, angles=720, det=768, sod=1600.0, sdd=3200.0,
                     pitch=1.3, ellipsoids=200, center=192.0,
                     axes=(16.0, 160.0), seed=1234),
    # 256^3, 360 angles, 384^2, SOD 800, SDD 1600, pitch 1.3, 40 ellipsoids
    "config2": dict(n=256, angles=360, det=384, sod=800.0, sdd=1600.0,
                    pitch=1.3, ellipsoids=40, center=96.0, axes=(8.0, 80.0),
                    seed=1236),
    # small case for profiler captures: inputs still larger than L2
    "profile": dict(n=384, angles=128, det=576, sod=1200.0, sdd=2400.0,
                    pitch=1.3, ellipsoids=60, center=144.0,
                    axes=(12.0, 120.0), seed=1240),
}


def make_scan(w):
    import kernelkit as kk

    det = kk.Detector(rows=w["det"], cols=w["det"], pixel_height=w["pitch"],
                      pixel_width=w["pitch"])
    g0 = kk.ProjectionGeometry([-w["sod"], 0.0, 0.0],
                               [w["sdd"] - w["sod"], 0.0, 0.0], det)
    pgs = [kk.rotate(g0, yaw=2 * np.pi * k / w["angles"])
           for k in range(w["angles"])]
    vg = kk.resolve_volume_geometry(shape=w["n"], voxel_size=1.0)
    return pgs, vg


def make_volume(w, vg, device="cuda"):
    from kernelkit import phantom

    ell = phantom.random_ellipsoids(w["ellipsoids"], w["center"], w["axes"],
                                    seed=w["seed"])
    return phantom.voxelize_torch(ell, vg.shape, vg.extent_min,
                                  vg.voxel_size, device=device)


# ---------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    """Samples nvidia-smi clocks and throttle reasons every 200 ms."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,"
             "clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index=0):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(prefix="kk_clocks_", suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}",
                 f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=open(self.path, "w"),
                stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [],
                    "samples": 0}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown",
                 "sw_power_cap"]
        with open(self.path) as f:
            for line in f:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) < 9:
                    continue
                try:
                    sm.append(float(parts[1]))
                    smax.append(float(parts[2]))
                except ValueError:
                    continue
                for name, val in zip(names, parts[5:9]):
                    if val.lower() == "active":
                        reasons.add(name)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------
# CPU baseline: the oracle on a bounded sample, on all host cores
# ---------------------------------------------------------------------------
_SHARED = {}


def _cpu_init(shm_name, shape):
    from multiprocessing import shared_memory

    os.environ["OMP_NUM_THREADS"] = "1"
    shm = shared_memory.SharedMemory(name=shm_name)
    _SHARED["shm"] = shm
    _SHARED["vol"] = np.ndarray(shape, np.float32, buffer=shm.buf)


def _cpu_fp_task(args):
    from oracle import cone

    p, axis, rows, cols, osc = args
    t = time.perf_counter()
    cone.cone_fp_angle(_SHARED["vol"], p, axis, rows, cols, osc)
    return time.perf_counter() - t


def _cpu_bp_task(args):
    from oracle import cone

    sino, p, shape, scale = args
    t = time.perf_counter()
    cone.cone_bp(sino, p, shape, scale)
    return time.perf_counter() - t


def cpu_sample(w, pgs, vg, vol_host, cores, fp_rows=16, bp_slab=8,
               tasks_per_core=1):
    """Oracle FP and BP on a bounded sample: ``fp_rows`` detector rows of
    one angle per FP task and one angle over a ``bp_slab``-voxel slab per
    BP task, ``cores`` tasks at a time. Returns (GUPS FP+BP, description)."""
    import multiprocessing as mp
    from multiprocessing import shared_memory

    from kernelkit.kernels import RayDrivenConeFP, VoxelDrivenConeBP

    fpar = RayDrivenConeFP.geoms2params(pgs, vg)
    rows12 = np.stack([np.asarray(p, np.float32) for p in fpar], axis=1)
    bpar = VoxelDrivenConeBP.geoms2params(pgs, vg).reshape(-1, 12)
    osc = RayDrivenConeFP._output_scale(vg.voxel_size)
    n = int(vg.shape[0])
    det = w["det"]
    ntasks = cores * tasks_per_core
    idx = np.linspace(0, len(pgs) - 1, ntasks).astype(int)
    fp_args = []
    for k, j in enumerate(idx):
        p = rows12[j].copy()
        r0 = (det // 2 - fp_rows // 2)
        p[3:6] = p[3:6] + np.float32(r0) * p[9:12]   # start at row r0
        fp_args.append((p, int(fpar.axes[j]), fp_rows, det, osc))
    rng = np.random.default_rng(0)
    sino = rng.uniform(0, 1, (1, det, det)).astype(np.float32)
    bp_args = [(sino, bpar[j:j + 1], (bp_slab, n, n), vg.voxel_volume())
               for j in idx]
    shm = shared_memory.SharedMemory(create=True, size=vol_host.nbytes)
    try:
        np.ndarray(vol_host.shape, np.float32, buffer=shm.buf)[...] = vol_host
        ctx = mp.get_context("spawn")
        with ctx.Pool(cores, initializer=_cpu_init,
                      initargs=(shm.name, vol_host.shape)) as pool:
            t0 = time.perf_counter()
            pool.map(_cpu_fp_task, fp_args, chunksize=1)
            t_fp = time.perf_counter() - t0
            t0 = time.perf_counter()
            pool.map(_cpu_bp_task, bp_args, chunksize=1)
            t_bp = time.perf_counter() - t0
    finally:
        shm.close()
        shm.unlink()
    # updates covered: FP sample = fp_rows/det of one angle's N voxels
    nvox = float(n) ** 3
    fp_upd = ntasks * nvox * fp_rows / det
    bp_upd = ntasks * bp_slab * float(n) * n
    fp_rate = fp_upd / t_fp
    bp_rate = bp_upd / t_bp
    gups = 2.0 / (1.0 / fp_rate + 1.0 / bp_rate) / 1e9
    desc = (f"oracle FP {ntasks} x ({fp_rows} rows x {det} cols of one angle)"
            f" in {t_fp:.1f}s + BP {ntasks} x ({bp_slab}x{n}x{n} voxels, one "
            f"angle) in {t_bp:.1f}s; per-update rates extrapolated to the "
            "full workload")
    return gups, desc, t_fp + t_bp


# ---------------------------------------------------------------------------
def dist_setup():
    import torch

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch.distributed as dist

        timeout = datetime.timedelta(seconds=120)
        if torch.cuda.is_available():
            torch.cuda.set_device(local)
            dist.init_process_group("nccl", timeout=timeout,
                                    device_id=torch.device("cuda", local))
        else:  # host-only runs of the replica logic
            dist.init_process_group("gloo", timeout=timeout)
    elif torch.cuda.is_available():
        torch.cuda.set_device(0)
    return rank, world, local


def _reduce_device():
    import torch.distributed as dist

    return "cuda" if dist.get_backend() == "nccl" else "cpu"


def max_over_ranks(x, world):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist

    t = torch.tensor([x], dtype=torch.float64, device=_reduce_device())
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world):
    import torch

    if world > 1:
        import torch.distributed as dist

        dist.barrier()
    if torch.cuda.is_available():
        torch.cuda.synchronize()


def load_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def load_traffic(workload, kernel):
    """DRAM bytes of ``kernel`` from the committed ncu summary
    (profiles/traffic.json: per forward projection, i.e. summed over its
    slice-span launches, for the FP; per 32-angle launch for the BP) at
    ``workload``; None if absent."""
    try:
        with open(os.path.join(ROOT, "profiles", "traffic.json")) as f:
            t = json.load(f)
        return t[workload][kernel]
    except (OSError, KeyError, ValueError):
        return None


def run_fdk(pgs, vg, sino, t_bp, reps=3):
    """FDK (pre-weighting, Ram-Lak filtering, backprojection) of the
    workload's own sinogram: device-resident input (pre-processed in place
    as the reference does, so every repetition starts from a fresh copy,
    outside the timed region), CUDA events around the chunked pipeline;
    and end to end through ``kk.fdk`` from a host array to a host result
    (wall clock, synchronised)."""
    import torch

    import kernelkit as kk
    from kernelkit import algo

    work = torch.empty_like(sino)
    ms = []
    for k in range(reps + 1):
        work.copy_(sino)
        torch.cuda.synchronize()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record()
        vol = algo._streamed_bp(work, pgs, vg, "ramlak")
        b.record()
        torch.cuda.synchronize()
        if k:
            ms.append(a.elapsed_time(b))
        del vol
    del work
    host = sino.cpu().numpy()
    kk.fdk(host, pgs, vg)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    rec = kk.fdk(host, pgs, vg)
    torch.cuda.synchronize()
    e2e = (time.perf_counter() - t0) * 1e3
    del rec, host
    torch.cuda.empty_cache()
    dev = statistics.median(ms)
    return {"ms": dev, "bp_ms": t_bp, "over_bp_ms": dev - t_bp,
            "e2e_host_ms": e2e,
            "pipeline": "per 32-angle chunk: one kernel pre-weights, "
                        "filters (float64 FFT) and writes the chunk into "
                        "its layered texture, then the BP launch",
            "timing": f"device input: CUDA events, median of {reps} after "
                      "one warm-up; e2e: host array in, pinned host "
                      "volume out, wall clock"}


def run_sirt(workload="config2", iters=50):
    """SIRT it/s on a noisy scan (config 2: 256^3, 360 angles, 384^2,
    40 ellipsoids, exact FP64 line integrals with Poisson noise at 1e4
    photons, log transformed), device-timed over CUDA-graph replays, with
    the reconstruction's rel. L2 to the phantom; FDK's rel. L2 too (raw,
    and after the least-squares scale, since FDK keeps the reference's
    unnormalised amplitude)."""
    import torch

    import kernelkit as kk
    from kernelkit import phantom
    from kernelkit.algo import SIRT

    w = WORKLOADS[workload]
    pgs, vg = make_scan(w)
    ell = phantom.random_ellipsoids(w["ellipsoids"], w["center"], w["axes"],
                                    seed=w["seed"])
    truth = phantom.voxelize_torch(ell, vg.shape, vg.extent_min,
                                   vg.voxel_size, device="cuda")
    srcs, pixs = phantom.pixel_centres(pgs)
    clean = phantom.line_integrals(ell, srcs, pixs, device="cuda")
    y = phantom.noisy_projections(clean, photons=1e4, seed=w["seed"])
    del clean

    def rel(x):
        return float((x - truth).norm() / truth.norm())

    rec = torch.as_tensor(kk.fdk(y.copy(), pgs, vg), device="cuda")
    fdk_raw = rel(rec)
    scale = float((rec * truth).sum() / (rec * rec).sum())
    fdk_fit = rel(scale * rec)
    del rec
    # the reconstructions' projections against exact FP64 line integrals
    # of the phantom on 16 evenly spaced angles
    from kernelkit.kernels import RayDrivenConeFP

    sel = list(range(0, len(pgs), len(pgs) // 16))[:16]
    ssrc, spix = phantom.pixel_centres([pgs[i] for i in sel])
    exact = phantom.line_integrals(ell, ssrc, spix, device="cuda")
    fsub = RayDrivenConeFP()
    fsub.compile()
    fsub.set_params(fsub.geoms2params([pgs[i] for i in sel], vg))

    def proj_err(x):
        sub = torch.empty(exact.shape, device="cuda")
        fsub(x.float(), [pgs[i] for i in sel], vg, sub, additive=False)
        return float((sub.double() - exact).norm() / exact.norm())

    out = {"workload": workload, "iters": iters,
           "noise": "Poisson, 1e4 photons, log transformed",
           "fdk_rel_l2_phantom": fdk_raw,
           "fdk_rel_l2_phantom_scaled": fdk_fit,
           "timing": "CUDA events around the graph replays (FP with "
                     "residual epilogue, texture refill, BP with update "
                     "epilogue per iteration)"}
    xs = {}
    for name, vdt, pdt in (("f32", None, None),
                           ("bf16_volume_f16_projections", torch.bfloat16,
                            torch.float16)):
        solver = SIRT(y, pgs, vg, volume_dtype=vdt, projection_dtype=pdt)
        solver.capture()
        torch.cuda.synchronize()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record()
        solver.run(iters, use_graph=True)
        b.record()
        torch.cuda.synchronize()
        ms = a.elapsed_time(b)
        xs[name] = solver.x.float().clone()
        out[name] = {"it_per_s": iters / (ms * 1e-3), "ms_per_iter": ms / iters,
                     "rel_l2_phantom": rel(xs[name]),
                     "rel_l2_projections_vs_fp64_16_angles":
                         proj_err(xs[name])}
        del solver
        torch.cuda.empty_cache()
    h = out["bf16_volume_f16_projections"]
    h["rel_l2_to_f32_reconstruction"] = float(
        (xs["bf16_volume_f16_projections"] - xs["f32"]).norm()
        / xs["f32"].norm())
    out["speedup_16bit_over_f32"] = h["it_per_s"] / out["f32"]["it_per_s"]
    # the f32 figures at the top level as before
    out.update(it_per_s=out["f32"]["it_per_s"],
               ms_per_iter=out["f32"]["ms_per_iter"], dtype="f32",
               rel_l2_phantom=out["f32"]["rel_l2_phantom"])
    del xs, exact
    torch.cuda.empty_cache()
    return out


def run_batched(n_problems=32, iters=30, seed=1237):
    """Config 4: independent problems of uneven size solved together
    (BatchedSIRT: batched launches, all iterations in one CUDA graph,
    autotuned record grouping). Edges N in {64, 96, 128, 160, 192}, angles
    U[60, 360], detector 1.5 N at pitch 1, SOD U(150, 1000), SDD 2 SOD,
    10 seeded ellipsoids per problem, noise-free exact line integrals.
    Aggregate GUPS = sum over problems of 2 N^3 angles iters / time."""
    import torch

    import kernelkit as kk
    from kernelkit import phantom
    from kernelkit.batch import Autotuner, BatchedSIRT

    rng = np.random.default_rng(seed)
    problems, truths, updates = [], [], 0
    for p in range(n_problems):
        n = int(rng.choice([64, 96, 128, 160, 192]))
        na = int(rng.integers(60, 361))
        sod = float(rng.uniform(150.0, 1000.0))
        det_n = int(round(1.5 * n))
        det = kk.Detector(rows=det_n, cols=det_n, pixel_height=1.0,
                          pixel_width=1.0)
        g0 = kk.ProjectionGeometry([-sod, 0.0, 0.0], [sod, 0.0, 0.0], det)
        pgs = [kk.rotate(g0, yaw=2 * np.pi * k / na) for k in range(na)]
        vg = kk.resolve_volume_geometry(shape=n, voxel_size=1.0)
        ell = phantom.random_ellipsoids(10, 3 * n / 8, (n / 32, 5 * n / 16),
                                        seed=seed + p)
        truths.append(phantom.voxelize_torch(ell, vg.shape, vg.extent_min,
                                             vg.voxel_size, device="cuda"))
        srcs, pixs = phantom.pixel_centres(pgs)
        y = phantom.line_integrals(ell, srcs, pixs, device="cuda")
        problems.append((y.float(), pgs, vg))
        updates += 2 * n ** 3 * na * iters
    tuner = Autotuner()
    b = BatchedSIRT(problems, autotuner=tuner)
    b.capture(iters)
    torch.cuda.synchronize()
    a = torch.cuda.Event(enable_timing=True)
    e = torch.cuda.Event(enable_timing=True)
    a.record()
    xs = b.run(iters)
    e.record()
    torch.cuda.synchronize()
    ms = a.elapsed_time(e)
    rels = [float((x - t).norm() / t.norm()) for x, t in zip(xs, truths)]
    return {"workload": "config4", "problems": n_problems, "iters": iters,
            "gups": updates / (ms * 1e-3) / 1e9, "ms": ms,
            "rel_l2_phantom": {"min": min(rels),
                               "median": float(np.median(rels)),
                               "max": max(rels)},
            "launches_per_iter": "1 FP launch per slice span + 1 persistent "
                                 "BP launch (+ texture refills); all "
                                 "iterations in one CUDA graph",
            "autotuned": {kind: sorted({json.dumps(v) for k, v in
                                        tuner.cache.items()
                                        if k.startswith(kind + ":")})
                          for kind in ("fp_axis_group", "fp_span",
                                       "bp_tile")}}


def run_sirt_config5(iters=20, seed=1239):
    """Config 5: 20 SIRT iterations at 1024^3 voxels / 1440 angles /
    1536^2 detector (SOD 3000, SDD 6000, pitch 1), plain float32 storage
    against a bfloat16 volume with float16 projections (FP32 accumulation,
    float16 textures). Data: the float32 forward projection of a voxelised
    200-ellipsoid phantom. Reported per storage: it/s (CUDA events around
    graph replays), one FP and one BP time, the reconstruction's rel. L2 to
    the phantom on the central 128^3 voxels, and the rel. L2 of A x_rec
    against the exact FP64 line integrals of the phantom on 16 angles."""
    import torch

    import kernelkit as kk
    from kernelkit import phantom
    from kernelkit.algo import SIRT
    from kernelkit.kernels import RayDrivenConeFP, VoxelDrivenConeBP

    n, na, det_n = 1024, 1440, 1536
    det = kk.Detector(rows=det_n, cols=det_n, pixel_height=1.0,
                      pixel_width=1.0)
    g0 = kk.ProjectionGeometry([-3000.0, 0.0, 0.0], [3000.0, 0.0, 0.0], det)
    pgs = [kk.rotate(g0, yaw=2 * np.pi * k / na) for k in range(na)]
    vg = kk.resolve_volume_geometry(shape=n, voxel_size=1.0)
    ell = phantom.random_ellipsoids(200, 384.0, (32.0, 320.0), seed=seed)
    truth = phantom.voxelize_torch(ell, vg.shape, vg.extent_min,
                                   vg.voxel_size, device="cuda")
    fp = RayDrivenConeFP()
    fp.compile()
    fp.set_params(fp.geoms2params(pgs, vg))
    y = torch.empty((na, det_n, det_n), device="cuda")
    fp(truth, pgs, vg, y, additive=False)
    sel = list(range(0, na, na // 16))[:16]
    srcs, pixs = phantom.pixel_centres([pgs[i] for i in sel])
    exact = phantom.line_integrals(ell, srcs, pixs, device="cuda")
    c = slice(n // 2 - 64, n // 2 + 64)
    tc = truth[c, c, c].double()
    fsub = RayDrivenConeFP()
    fsub.compile()
    fsub.set_params(fsub.geoms2params([pgs[i] for i in sel], vg))

    def timed(fn):
        torch.cuda.synchronize()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record()
        fn()
        b.record()
        torch.cuda.synchronize()
        return a.elapsed_time(b)

    out = {}
    for name, vdt, pdt in (("fp32", None, None),
                           ("bf16_volume_f16_projections", torch.bfloat16,
                            torch.float16)):
        s = SIRT(y, pgs, vg, volume_dtype=vdt, projection_dtype=pdt)
        s.capture()
        ms = timed(lambda: s.run(iters, use_graph=True))
        x = s.x
        # one forward projection and one backprojection in this storage
        f = RayDrivenConeFP()
        f.half_texture = vdt is not None
        f.compile()
        f.set_params(f.geoms2params(pgs, vg))
        t_fp = timed(lambda: f(x, pgs, vg, s.y_tmp, additive=False))
        bp = VoxelDrivenConeBP()
        bp.compile()
        bp.set_params(bp.geoms2params(pgs, vg))
        s.tex.copy_from(s.y_tmp)
        tmpv = torch.empty_like(x)
        t_bp = timed(lambda: bp(s.tex, tmpv, vg, additive=False))
        del tmpv, f, bp
        xs = x.float()
        sub = torch.empty((16, det_n, det_n), device="cuda")
        fsub(xs, [pgs[i] for i in sel], vg, sub, additive=False)
        out[name] = {
            "it_per_s": iters / (ms * 1e-3), "ms_per_iter": ms / iters,
            "fp_ms": t_fp, "bp_ms": t_bp,
            "rel_l2_phantom_center128": float(
                (xs[c, c, c].double() - tc).norm() / tc.norm()),
            "rel_l2_projections_vs_fp64_16_angles": float(
                (sub.double() - exact).norm() / exact.norm()),
            "storage": {"volume": str(x.dtype).replace("torch.", ""),
                        "projections": str(s.y.dtype).replace("torch.", "")}}
        if name == "fp32":
            x32 = xs.clone()
        else:
            out[name]["rel_l2_to_fp32_reconstruction"] = float(
                (xs - x32).norm() / x32.norm())
        del s, x, xs, sub
        torch.cuda.empty_cache()
    out["speedup_16bit_over_fp32"] = (
        out["bf16_volume_f16_projections"]["it_per_s"] / out["fp32"]["it_per_s"])
    return {"metric": "SIRT it/s @1024^3/1440 ang, 16-bit storage vs fp32",
            "workload": "config5", "iters": iters, **out}


def run_autograd_config3(steps=100, seed=1238):
    """Config 3: differentiable reconstruction at 256^3 on the config-2
    scan: loss = ||A x - y||^2 + 1e-3 TV(x), x_0 = 0, Adam (lr 1e-2) for
    100 steps, with backward = the exact adjoint of the forward projector
    (ExactXrayForwardProjection). Checks: FP64 dot test on seeded Gaussian
    x, y; central finite differences (eps 1e-3) along 64 seeded random
    directions; and the cosine between this gradient and the one the
    reference's autograd would give (backprojector as backward)."""
    import torch

    import kernelkit as kk
    from kernelkit import phantom
    from kernelkit.torch_support import ExactXrayForwardProjection

    w = WORKLOADS["config2"]
    pgs, vg = make_scan(w)
    ell = phantom.random_ellipsoids(w["ellipsoids"], w["center"], w["axes"],
                                    seed=w["seed"])
    truth = phantom.voxelize_torch(ell, vg.shape, vg.extent_min,
                                   vg.voxel_size, device="cuda")
    srcs, pixs = phantom.pixel_centres(pgs)
    y = torch.as_tensor(phantom.noisy_projections(
        phantom.line_integrals(ell, srcs, pixs, device="cuda"),
        photons=1e4, seed=w["seed"]), device="cuda")
    shape = tuple(truth.shape)
    module = ExactXrayForwardProjection(pgs, vg)
    op = module.op
    g = torch.Generator(device="cuda").manual_seed(seed)
    # FP64 dot test
    xr = torch.randn(shape, generator=g, device="cuda")
    yr = torch.randn(y.shape, generator=g, device="cuda")
    Ax = op(xr)
    ATy = op.T(yr)
    dot = abs(float((Ax.double() * yr.double()).sum())
              - float((xr.double() * ATy.double()).sum())) / float(
        Ax.double().norm() * yr.double().norm())
    del xr, yr, Ax, ATy

    def tv(x):
        dx = x[1:, :-1, :-1] - x[:-1, :-1, :-1]
        dy = x[:-1, 1:, :-1] - x[:-1, :-1, :-1]
        dz = x[:-1, :-1, 1:] - x[:-1, :-1, :-1]
        return torch.sqrt(dx * dx + dy * dy + dz * dz + 1e-8).sum()

    def loss_fn(x):
        r = module(x[None, None])[0, 0] - y
        return (r.double() ** 2).sum() + 1e-3 * tv(x).double()

    x = torch.zeros(shape, device="cuda", requires_grad=True)
    opt = torch.optim.Adam([x], lr=1e-2)
    torch.cuda.synchronize()
    a = torch.cuda.Event(enable_timing=True)
    b = torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(steps):
        opt.zero_grad(set_to_none=True)
        loss = loss_fn(x)
        loss.backward()
        opt.step()
    b.record()
    torch.cuda.synchronize()
    ms = a.elapsed_time(b)
    final = float(loss.detach())
    rel = float((x.detach() - truth).norm() / truth.norm())
    # gradient checks at the final iterate (data term)
    x0 = x.detach().clone().requires_grad_(True)
    data = ((module(x0[None, None])[0, 0] - y).double() ** 2).sum()
    data.backward()
    grad = x0.grad.double()

    def L(v):
        return float(((op(v) - y).double() ** 2).sum())

    errs = []
    gnorm = float(grad.norm())
    for _ in range(64):
        d = torch.randn(shape, generator=g, device="cuda")
        fd = (L(x0.detach() + 1e-3 * d) - L(x0.detach() - 1e-3 * d)) / 2e-3
        an = float((grad * d.double()).sum())
        # error relative to |grad| |d| (directional derivatives of random
        # directions can be near zero)
        errs.append(abs(fd - an) / (gnorm * float(d.double().norm())))
    # the reference's autograd backward: 2 * BP(A x - y) with its
    # (scaled, unmatched) backprojector
    ref_op = kk.XrayTransform(pgs, vg)
    r = (op(x0.detach()) - y).contiguous()
    g_ref = 2.0 * ref_op.T(r).double()
    cos = float((g_ref * grad).sum() / (g_ref.norm() * grad.norm()))
    return {"metric": "differentiable reconstruction, exact adjoint",
            "workload": "config3 (config-2 scan, 256^3)", "steps": steps,
            "ms_per_step": ms / steps, "final_loss": final,
            "rel_l2_phantom": rel, "dot_test_mismatch_fp64": dot,
            "fd_error_rel_to_grad_norm": {"max": max(errs),
                             "median": float(np.median(errs)),
                             "directions": 64, "eps": 1e-3},
            "cosine_to_backprojector_gradient": cos}


def run_reference_kernels(w, pgs, vg, vol, proj, bp, reps=3):
    """The reference's own CUDA kernels (its cone_fp.cu / cone_bp.cu
    templates rendered with its default arguments and compiled for sm_100a
    by oracle/build_ref.py) on this workload, after the timed region:
    kernel-only time (CUDA events around its launch loops, inputs already
    in its textures; median of ``reps`` after one warm-up), and, as the
    checker, the rel. L2 between its outputs and ours on the same inputs:
    FP of the same volume; BP of the reference's own sinogram by both."""
    import torch

    from kernelkit import _native
    from kernelkit.kernels import RayDrivenConeFP, VoxelDrivenConeBP
    from oracle import ref_kernels

    if not ref_kernels.available():
        return {"error": "oracle/_ref/libkkref.so not built"}
    fpar = RayDrivenConeFP.geoms2params(pgs, vg)
    rows12 = np.stack([np.asarray(p, np.float32) for p in fpar], axis=1)
    osc = np.asarray(RayDrivenConeFP._output_scale(vg.voxel_size), np.float32)
    bpar = VoxelDrivenConeBP.geoms2params(pgs, vg).reshape(-1, 12)
    det = w["det"]
    fp_ms, bp_ms = [], []
    ref_fp = None
    for k in range(reps + 1):
        ref_fp, ms = ref_kernels.ref_cone_fp(vol, rows12, fpar.axes, det, det,
                                             osc)
        if k:
            fp_ms.append(ms)
    rel_fp = float((proj.double() - ref_fp.double()).norm()
                   / ref_fp.double().norm())
    ref_bp = None
    for k in range(reps + 1):
        ref_bp, ms = ref_kernels.ref_cone_bp(ref_fp, bpar, vg.shape,
                                             float(vg.voxel_volume()))
        if k:
            bp_ms.append(ms)
    tex = _native.Layered(len(pgs), det, det, _native.KK_F32)
    tex.copy_from(ref_fp)
    ours_bp = torch.empty_like(vol)
    bp(tex, ours_bp, vg, additive=False)
    torch.cuda.synchronize()
    rel_bp = float((ours_bp.double() - ref_bp.double()).norm()
                   / ref_bp.double().norm())
    del tex, ref_fp, ref_bp, ours_bp
    torch.cuda.empty_cache()
    nupd = float(np.prod([int(s) for s in vg.shape])) * len(pgs)
    t_fp, t_bp = statistics.median(fp_ms), statistics.median(bp_ms)
    return {"fp_ms": t_fp, "bp_ms": t_bp,
            "fp_gups": nupd / (t_fp * 1e-3) / 1e9,
            "bp_gups": nupd / (t_bp * 1e-3) / 1e9,
            "gups": 2 * nupd / ((t_fp + t_bp) * 1e-3) / 1e9,
            "rel_l2_fp": rel_fp, "rel_l2_bp": rel_bp,
            "source": "reference cone_fp.cu/cone_bp.cu templates rendered "
                      "with the reference's defaults, built for sm_100a "
                      "(oracle/build_ref.py); kernel-only CUDA events "
                      f"around its launch loops, median of {reps} after one "
                      "warm-up; rel_l2 = ours vs the reference on the same "
                      "inputs (FP of the volume, BP of the reference's "
                      "sinogram)"}


def run_ours(args):
    import torch

    from kernelkit import XrayTransform
    from kernelkit.kernels import RayDrivenConeFP, VoxelDrivenConeBP

    rank, world, local = dist_setup()
    w = WORKLOADS[args.workload]
    pgs, vg = make_scan(w)
    shape = tuple(int(s) for s in vg.shape)
    nupd = float(np.prod(shape)) * len(pgs)
    vol = make_volume(w, vg)
    fp = RayDrivenConeFP()
    fp.compile()
    fp.set_params(fp.geoms2params(pgs, vg))
    bp = VoxelDrivenConeBP()
    bp.compile()
    bp.set_params(bp.geoms2params(pgs, vg))
    proj = torch.empty((len(pgs), w["det"], w["det"]), device="cuda")
    back = torch.empty(shape, device="cuda")
    stream = torch.cuda.current_stream()
    from kernelkit import _native

    # the backprojector samples a layered texture of the sinogram (the
    # reference's filter); the copy into it is part of the step
    ptex = _native.Layered(len(pgs), w["det"], w["det"], _native.KK_F32)

    def step(ev):
        ev[0].record(stream)
        fp(vol, pgs, vg, proj, additive=False)
        ev[1].record(stream)
        ptex.copy_from(proj)
        bp(ptex, back, vg, additive=False)
        ev[2].record(stream)

    for _ in range(args.warmup):
        step([torch.cuda.Event(enable_timing=True) for _ in range(3)])
    barrier(world)
    sampler = ClockSampler(local)
    sampler.start()
    events = [[torch.cuda.Event(enable_timing=True) for _ in range(3)]
              for _ in range(args.steps)]
    t_start = torch.cuda.Event(enable_timing=True)
    t_end = torch.cuda.Event(enable_timing=True)
    t_start.record(stream)
    for k in range(args.steps):
        step(events[k])
    t_end.record(stream)
    barrier(world)
    clocks = sampler.stop()
    fp_ms = [e[0].elapsed_time(e[1]) for e in events]
    bp_ms = [e[1].elapsed_time(e[2]) for e in events]
    total_ms = t_start.elapsed_time(t_end)
    ms_step = max_over_ranks(total_ms / args.steps, world)
    t_fp = statistics.mean(fp_ms)
    t_bp = statistics.mean(bp_ms)
    value = world * 2 * nupd / (ms_step * 1e-3) / 1e9

    e2e = None
    if not args.no_e2e:
        op = XrayTransform(pgs, vg)
        # Double-buffered: step k's input copy and step k-1's result copy
        # run on copy streams while step k-1 / k computes. Every step still
        # moves its whole input in and its whole result out; the copies
        # only leave the critical path.
        host_in = torch.empty(shape, dtype=torch.float32, pin_memory=True)
        host_in.copy_(vol.cpu())
        host_out = [torch.empty(shape, dtype=torch.float32, pin_memory=True)
                    for _ in range(2)]
        dev_in = [torch.empty(shape, device="cuda") for _ in range(2)]
        dev_y = torch.empty((len(pgs), w["det"], w["det"]), device="cuda")
        dev_out = [torch.empty(shape, device="cuda") for _ in range(2)]
        s_in, s_out = torch.cuda.Stream(), torch.cuda.Stream()

        def ev():
            return torch.cuda.Event()

        def e2e_run(n):
            """n steps; returns after queueing them (all streams joined
            into the current stream)."""
            read_done = [None, None]   # compute finished reading dev_in[b]
            out_free = [None, None]    # D2H finished reading dev_out[b]
            s_in.wait_stream(stream)
            s_out.wait_stream(stream)
            for k in range(n):
                b = k & 1
                with torch.cuda.stream(s_in):
                    if read_done[b] is not None:
                        s_in.wait_event(read_done[b])
                    dev_in[b].copy_(host_in, non_blocking=True)
                    landed = ev()
                    landed.record(s_in)
                stream.wait_event(landed)
                if out_free[b] is not None:
                    stream.wait_event(out_free[b])
                op(dev_in[b], out=dev_y)
                read_done[b] = ev()
                read_done[b].record(stream)
                op.T(dev_y, out=dev_out[b])
                done = ev()
                done.record(stream)
                with torch.cuda.stream(s_out):
                    s_out.wait_event(done)
                    host_out[b].copy_(dev_out[b], non_blocking=True)
                    out_free[b] = ev()
                    out_free[b].record(s_out)
            stream.wait_stream(s_in)
            stream.wait_stream(s_out)

        e2e_run(max(1, args.warmup))
        barrier(world)
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        e2e_run(args.steps)
        b.record(stream)
        barrier(world)
        torch.cuda.synchronize()
        e2e_ms = max_over_ranks(a.elapsed_time(b) / args.steps, world)
        got = host_out[(args.steps - 1) & 1]
        e2e = {"value": world * 2 * nupd / (e2e_ms * 1e-3) / 1e9,
               "unit": UNIT, "ms_per_step": e2e_ms,
               "h2d_bytes_per_step": host_in.numel() * 4,
               "d2h_bytes_per_step": got.numel() * 4,
               "result_checksum": float(got.double().sum()),
               "path": "XrayTransform: pinned host x -> A x -> A^T (A x) -> "
                       "pinned host; input and result copies on two copy "
                       "streams, double-buffered, overlapping the "
                       "neighbouring steps' compute"}
        del dev_in, dev_y, dev_out

    peak, peak_kind = load_peaks()
    from kernelkit.kernels.cone_fp import launches_per_projection
    fp_launches = launches_per_projection(max(shape))
    # the projector traces a zero-padded copy of the volume (one
    # fp_pad_kernel launch per projection, inside the FP's time) with
    # cone_fp_pad_kernel, or the volume itself with cone_fp_kernel
    fp_name = "cone_fp_pad_kernel" if fp.padded_copy else "cone_fp_kernel"
    pad_launches = 1 if fp.padded_copy else 0
    # one BP launch per four 32-angle chunks
    bp_launches = int(_native.load().kk_bp_launches(len(pgs)))
    fp_bytes = 4.0 * nupd  # algorithmic: one float32 voxel operand / update
    roofline = {"kernel": fp_name, "bound": "hbm",
                "achieved": fp_bytes / (t_fp * 1e-3) / 1e9, "peak": peak,
                "unit": "GB/s",
                "frac": fp_bytes / (t_fp * 1e-3) / 1e9 / peak,
                "peak_kind": peak_kind,
                "traffic": load_traffic(args.workload, fp_name),
                "algorithmic_bytes_per_launch": fp_bytes,
                # one forward projection is fp_launches launches of slice
                # spans: bytes, time and traffic are per projection
                "per": f"forward projection ({fp_launches} launches)"}
    # The backprojector samples one bilinear texel quad per update; its
    # ceiling is the texture unit's fetch rate, measured on this GPU model
    # (3.83 float32 bilinear fetches per clock per SM,
    # profiles/texture_unit_rate.md), at the SM clock seen during the timed
    # region.
    sm_hz = 1e6 * float(clocks.get("sm_mhz") or clocks.get("sm_max_mhz")
                        or 1965.0)
    sms = torch.cuda.get_device_properties(0).multi_processor_count
    tmu_peak = TMU_FETCH_PER_CLK_SM * sms * sm_hz
    texture_roofline = {
        "kernel": "cone_bp_kernel", "bound": "texture unit",
        "achieved": nupd / (t_bp * 1e-3), "peak": tmu_peak,
        "unit": "bilinear fetches/s",
        "frac": nupd / (t_bp * 1e-3) / tmu_peak,
        "peak_source": f"{TMU_FETCH_PER_CLK_SM} fetches/clk/SM measured "
                       "(profiles/texture_unit_rate.md) x SMs x SM clock"}
    kernels = {
        # "traffic": ncu DRAM bytes per launch (profiles/), "ms": all
        # launches of one operator application
        fp_name: {"ms": t_fp, "launches": fp_launches,
                  "pad_copy_launches": pad_launches,
                  "gups": nupd / (t_fp * 1e-3) / 1e9,
                  "achieved_gbs": fp_bytes / (t_fp * 1e-3) / 1e9,
                  "traffic": load_traffic(args.workload, fp_name)},
        "cone_bp_kernel": {"ms": t_bp, "launches": bp_launches,
                           "gups": nupd / (t_bp * 1e-3) / 1e9,
                           "achieved_gbs": fp_bytes / (t_bp * 1e-3) / 1e9,
                           "traffic": load_traffic(args.workload,
                                                   "cone_bp_kernel")},
    }
    refk = None
    if rank == 0 and world == 1 and not args.no_reference_kernels:
        try:
            refk = run_reference_kernels(w, pgs, vg, vol, proj, bp)
            if "gups" in refk:
                refk["speedup"] = (2 * nupd / ((t_fp + t_bp) * 1e-3) / 1e9
                                   / refk["gups"])
        except Exception as e:  # noqa: BLE001
            refk = {"error": f"{type(e).__name__}: {e}"[:300]}
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cores = len(os.sched_getaffinity(0))
        try:
            gups, desc, secs = cpu_sample(w, pgs, vg, vol.cpu().numpy(),
                                          cores, fp_rows=48, bp_slab=24)
            cpu = {"value": gups, "unit": UNIT, "cores": cores,
                   "kind": "port", "sample": desc, "seconds": secs}
        except Exception as e:  # noqa: BLE001
            cpu = {"value": None, "unit": UNIT, "cores": cores,
                   "kind": "port", "error": f"{type(e).__name__}: {e}"[:300]}
    fdk = None
    if rank == 0 and world == 1 and not args.no_fdk:
        try:
            fdk = run_fdk(pgs, vg, proj, t_bp)
        except Exception as e:  # noqa: BLE001
            fdk = {"error": f"{type(e).__name__}: {e}"[:300]}
    sirt = batched = None
    if rank == 0 and world == 1 and not args.no_sirt:
        # secondary measurements: a failure here is reported in the line
        # instead of costing the headline number
        for name, fn in (("sirt", lambda: run_sirt("config2", 50)),
                         ("batched", run_batched)):
            try:
                res = fn()
            except Exception as e:  # noqa: BLE001
                res = {"error": f"{type(e).__name__}: {e}"[:300]}
            if name == "sirt":
                sirt = res
            else:
                batched = res
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic",
            "config": {"workload": args.workload, "volume": list(shape),
                       "angles": len(pgs), "detector": [w["det"], w["det"]],
                       "sod": w["sod"], "sdd": w["sdd"], "pitch": w["pitch"],
                       "phantom": f"{w['ellipsoids']} seeded ellipsoids",
                       "interpolation": "texture-compatible (1/256 weights)",
                       "l2": "inputs larger than L2 (volume 537 MB, "
                             "sinogram 1.7 GB), no flush",
                       "parallelism": f"replicas x{world}"},
            "e2e": e2e, "roofline": roofline,
            "texture_roofline": texture_roofline, "cpu_baseline": cpu,
            "kernels": kernels, "reference_kernels": refk,
            # per step: the FP's padded copy and slice-span launches, the
            # BP's launches (four 32-angle chunks each)
            "gpu_launches": args.steps * (pad_launches + fp_launches
                                          + bp_launches),
            "clocks": clocks, "fdk": fdk, "sirt": sirt, "batched": batched,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()


def run_profile_op(args):
    """One operator, twice (the second is the one a profiler captures),
    on the chosen workload: ``fp`` (``--fp-tiles`` / ``--fp-no-texture``
    select its paths), ``bp``, ``fdk`` (pre-processing fused with the
    texture store, then the chunked BP) or ``adjoint`` (the exact
    transpose of the FP). Prints the second run's CUDA-event time."""
    import torch

    from kernelkit import _native, algo
    from kernelkit.kernels import RayDrivenConeFP, VoxelDrivenConeBP

    w = WORKLOADS[args.workload]
    pgs, vg = make_scan(w)
    vol = make_volume(w, vg)
    det = w["det"]
    proj = torch.empty((len(pgs), det, det), device="cuda")
    fp = RayDrivenConeFP(use_texture_unit=not args.fp_no_texture)
    fp.use_tiles = bool(args.fp_tiles)
    fp.compile()
    fp.set_params(fp.geoms2params(pgs, vg))
    fp(vol, pgs, vg, proj, additive=False)
    if args.profile_op == "fp":
        def op():
            fp(vol, pgs, vg, proj, additive=False)
    elif args.profile_op == "bp":
        bp = VoxelDrivenConeBP()
        bp.compile()
        bp.set_params(bp.geoms2params(pgs, vg))
        tex = _native.Layered(len(pgs), det, det, _native.KK_F32)
        tex.copy_from(proj)
        out = torch.empty_like(vol)

        def op():
            bp(tex, out, vg, additive=False)
    elif args.profile_op == "fdk":
        work = torch.empty_like(proj)

        def op():
            work.copy_(proj)
            algo._streamed_bp(work, pgs, vg, "ramlak")
    else:
        out = torch.empty_like(vol)

        def op():
            fp.transpose(proj, pgs, vg, out)
    op()
    torch.cuda.synchronize()
    a = torch.cuda.Event(enable_timing=True)
    b = torch.cuda.Event(enable_timing=True)
    a.record()
    op()
    b.record()
    torch.cuda.synchronize()
    print(json.dumps({"profile_op": args.profile_op, "workload": args.workload,
                      "ms": a.elapsed_time(b),
                      "wait_timeouts": _native.wait_timeouts()}), flush=True)


def run_reference(args):
    """Reference arm: the oracle's restatement of the reference algorithm
    (the reference itself has no CPU path; its GPU kernels are exercised by
    the test suite through oracle/_ref) on all host cores."""
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if rank != 0:
        return
    import torch

    w = WORKLOADS[args.workload]
    pgs, vg = make_scan(w)
    if torch.cuda.is_available():
        vol = make_volume(w, vg).cpu().numpy()
    else:
        vol = make_volume(w, vg, device="cpu").numpy()
    cores = len(os.sched_getaffinity(0))
    vals, descs, secs = [], None, []
    for k in range(args.warmup + args.steps):
        gups, descs, s = cpu_sample(w, pgs, vg, vol, cores, fp_rows=8,
                                    bp_slab=4)
        if k >= args.warmup:
            vals.append(gups)
            secs.append(s)
    value = statistics.mean(vals)
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": statistics.mean(secs) * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic", "impl": "reference",
        "config": {"workload": args.workload, "volume": [w["n"]] * 3,
                   "angles": w["angles"], "detector": [w["det"], w["det"]]},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores,
                         "kind": "port", "sample": descs},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--workload", choices=sorted(WORKLOADS),
                    default="headline")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-fdk", action="store_true",
                    help="skip the FDK timing")
    ap.add_argument("--no-reference-kernels", action="store_true",
                    help="skip timing the reference's own CUDA kernels")
    ap.add_argument("--sirt-config5", action="store_true",
                    help="only run the 1024^3 SIRT storage comparison "
                         "(several minutes; prints its own JSON line)")
    ap.add_argument("--autograd-config3", action="store_true",
                    help="only run the 256^3 differentiable reconstruction "
                         "with the exact adjoint (prints its own JSON line)")
    ap.add_argument("--no-sirt", action="store_true",
                    help="skip the SIRT measurements (config 2 and the "
                         "batched config 4)")
    ap.add_argument("--profile-op", choices=("fp", "bp", "fdk", "adjoint"),
                    help="only run one operator twice on the workload (for "
                         "profiler captures; prints its own JSON line)")
    ap.add_argument("--fp-tiles", action="store_true",
                    help="--profile-op fp: shared-memory tiles for the "
                         "CUDA-core rays")
    ap.add_argument("--fp-no-texture", action="store_true",
                    help="--profile-op fp: every ray on the CUDA cores")
    args = ap.parse_args(argv)
    if args.profile_op:
        run_profile_op(args)
        return
    if args.sirt_config5:
        print(json.dumps(run_sirt_config5()), flush=True)
        return
    if args.autograd_config3:
        print(json.dumps(run_autograd_config3()), flush=True)
        return
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
