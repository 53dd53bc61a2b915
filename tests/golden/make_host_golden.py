"""Generate ``host_golden.npz`` from the reference's own Python code.

Runs the reference (imported from its checkout with the stand-ins of
``reference_import.py``) on every case of ``cases.py`` and stores:

* ``<case>/fp_params`` (n, 12) float32: ``RayDrivenConeFP.geoms2params``
  (``kernels/cone_fp.py:302-339``), SoA arrays transposed to rows;
* ``<case>/fp_axes`` (n,): ``RayDrivenConeFP._geom_axes`` on the
  normalised sequence (``kernels/cone_fp.py:264-285``);
* ``<case>/fp_out_scale`` (3, 3): ``RayDrivenConeFP._output_scale``;
* ``<case>/bp_params`` (n, 12) float32: ``VoxelDrivenConeBP.geoms2params``
  (``kernels/cone_bp.py:304-421``);
* ``<case>/vol_*``: the resolved ``VolumeGeometry`` and its voxel volume;
* ``resolve/<i>/*``: ``resolve_volume_geometry`` results;
* ``proc/*``: ``processing.preweight`` and ``processing.filter``
  (ramlak, cosine) on seeded random projections (``processing.py``).

Usage (where the reference checkout exists):
``python tests/golden/make_host_golden.py``
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

from cases import CASES, RESOLVE_CASES  # noqa: E402
from reference_import import import_reference  # noqa: E402


def build_case(kk, spec):
    det = kk.Detector(rows=spec["rows"], cols=spec["cols"],
                      pixel_height=spec["pixel_height"],
                      pixel_width=spec["pixel_width"])
    kw = {}
    if "u" in spec:
        kw["u"] = spec["u"]
    if "v" in spec:
        kw["v"] = spec["v"]
    g0 = kk.ProjectionGeometry(source_position=spec["source"],
                               detector_position=spec["detector"],
                               detector=det, **kw)
    pgs = [kk.rotate(g0, roll=r, pitch=p, yaw=y)
           for (r, p, y) in spec["rotations"]]
    vol = spec["volume"]
    if "resolve" in vol:
        vg = kk.resolve_volume_geometry(**vol["resolve"])
    else:
        vg = kk.VolumeGeometry(**vol["explicit"])
    return pgs, vg


def main():
    kk = import_reference()
    from kernelkit.kernels.cone_bp import VoxelDrivenConeBP
    from kernelkit.kernels.cone_fp import RayDrivenConeFP
    import kernelkit.processing as proc

    out = {}
    for name, spec in CASES.items():
        pgs, vg = build_case(kk, spec)
        seq = kk.ProjectionGeometrySequence.fromList(pgs)
        fp = RayDrivenConeFP.geoms2params(seq, vg)  # normalises seq in place
        out[f"{name}/fp_params"] = np.stack(fp, axis=1).astype(np.float32)
        out[f"{name}/fp_axes"] = np.asarray(
            RayDrivenConeFP._geom_axes(seq), np.int32)
        out[f"{name}/fp_out_scale"] = np.asarray(
            RayDrivenConeFP._output_scale(vg.voxel_size), np.float32)
        if spec.get("bp", True):
            bp = VoxelDrivenConeBP.geoms2params(pgs, vg)
            out[f"{name}/bp_params"] = np.asarray(bp, np.float32).reshape(
                -1, 12)
        out[f"{name}/vol_shape"] = np.asarray(vg.shape, np.int64)
        out[f"{name}/vol_voxel_size"] = np.asarray(vg.voxel_size, np.float32)
        out[f"{name}/vol_extent_min"] = np.asarray(vg.extent_min, np.float32)
        out[f"{name}/vol_extent_max"] = np.asarray(vg.extent_max, np.float32)
        out[f"{name}/vol_voxel_volume"] = np.float64(vg.voxel_volume())
        print(name, len(pgs), "angles", out[f"{name}/fp_params"].shape)

    for i, kw in enumerate(RESOLVE_CASES):
        vg = kk.resolve_volume_geometry(**kw)
        out[f"resolve/{i}/shape"] = np.asarray(vg.shape, np.int64)
        out[f"resolve/{i}/voxel_size"] = np.asarray(vg.voxel_size, np.float32)
        out[f"resolve/{i}/extent_min"] = np.asarray(vg.extent_min, np.float32)
        out[f"resolve/{i}/extent_max"] = np.asarray(vg.extent_max, np.float32)

    # processing: preweight + filter on seeded projections of two cases
    for name, cols_override in (("small", None), ("tilted", None)):
        pgs, _ = build_case(kk, CASES[name])
        pgs = pgs[:5]
        det = pgs[0].detector
        rng = np.random.default_rng(77)
        p = rng.uniform(0, 2, (len(pgs), det.rows, det.cols)).astype(
            np.float32)
        out[f"proc/{name}/input"] = p.copy()
        pw = p.copy()
        proc.preweight(pw, pgs)
        out[f"proc/{name}/preweight"] = pw.copy()
        for filt in ("ramlak", "cosine"):
            q = pw.copy()
            proc.filter(q, filter=filt)
            out[f"proc/{name}/filter_{filt}"] = q
    # filter on a width that is not a power of two and a single row
    rng = np.random.default_rng(78)
    for cols in (37, 100, 1):
        p = rng.standard_normal((3, 4, cols)).astype(np.float32)
        out[f"proc/filter_w{cols}/input"] = p.copy()
        for filt in ("ramlak", "cosine"):
            q = p.copy()
            proc.filter(q, filter=filt)
            out[f"proc/filter_w{cols}/{filt}"] = q
    path = os.path.join(HERE, "host_golden.npz")
    np.savez_compressed(path, **out)
    print("wrote", path, os.path.getsize(path), "bytes")


if __name__ == "__main__":
    main()
