"""Shared helpers of the test suite: build the golden scans with this
repository's geometry code, and phantoms."""
from __future__ import annotations

import numpy as np

import kernelkit as kk
from cases import CASES, phantom_for
from kernelkit import phantom


def build_case(name):
    """(list of ProjectionGeometry, VolumeGeometry) of a golden case."""
    spec = CASES[name]
    det = kk.Detector(rows=spec["rows"], cols=spec["cols"],
                      pixel_height=spec["pixel_height"],
                      pixel_width=spec["pixel_width"])
    kw = {k: spec[k] for k in ("u", "v") if k in spec}
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


def case_volume(name, vg):
    """Seeded ellipsoid phantom of a golden case (as make_gpu_golden.py)."""
    shape = tuple(int(s) for s in vg.shape)
    ph = phantom_for(name, shape)
    vs = np.asarray(vg.voxel_size, np.float64)
    lo = np.asarray(vg.extent_min, np.float64)
    hi = np.asarray(vg.extent_max, np.float64)
    ell = phantom.random_ellipsoids(ph["k"], ph["center_range"] * vs.min(),
                                    np.asarray(ph["axes_range"]) * vs.min(),
                                    ph["seed"])
    ell.centers += (lo + hi) / 2
    return phantom.voxelize(ell, shape, lo, vs)


def fp_params_rows(params):
    """(n, 12) rows of a geoms2params result (12 SoA arrays)."""
    return np.stack([np.asarray(p, np.float32) for p in params], axis=1)
