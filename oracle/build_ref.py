"""Build recipe for the reference-kernel checker ``oracle/_ref/libkkref.so``.

Renders the reference's own CUDA templates (``kernelkit/cuda/cone_fp.cu``
and ``cone_bp.cu`` under the reference checkout) with Jinja2, using the
template arguments the reference's kernel classes pass by default
(``kernels/cone_fp.py:88-100``, ``kernels/cone_bp.py:114-166`` with the
'layered' texture of ``BackProjector``), and compiles each together with a
host shim of this repository (``oracle/ref_shim_*.cu``) for sm_100a. The
texture-filter probe (``oracle/tex_probe.cu``) is linked into the same
library.

Rendered sources go to a temporary directory that is deleted afterwards;
only the shared library lands in ``oracle/_ref/`` (git-ignored, shipped to
the GPU machine with the rest of the tree). Without the reference checkout
the recipe does nothing and a previously built library is used.

Usage: ``python oracle/build_ref.py [--reference PATH]`` (default: the
``KK_REFERENCE`` environment variable, else the checkout's usual place).
"""
from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
OUT_DIR = os.path.join(HERE, "_ref")
OUT_LIB = os.path.join(OUT_DIR, "libkkref.so")
#: checkout of the reference (KK_REFERENCE overrides the default location)
DEFAULT_REFERENCE = os.environ.get("KK_REFERENCE", "/root/reference")

FP_KWARGS = dict(slices_per_block=16, rows_per_block=32, cols_per_block=32,
                 nr_projs_global=1024, volume_axes=(0, 1, 2),
                 projection_axes=(0, 1, 2))
BP_KWARGS = dict(voxels_per_block=(6, 32, 16), nr_projs_block=32,
                 nr_projs_global=1024, texture="tex2DLayered",
                 volume_axes=(0, 1, 2), projection_axes=(0, 1, 2))

NVCC_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-O3",
              "-std=c++17", "-Xcompiler", "-fPIC", "-lineinfo"]


def _nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc",
                 shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def render(template_path, kwargs):
    import jinja2

    with open(template_path) as f:
        src = f.read()
    return jinja2.Template(src, undefined=jinja2.StrictUndefined).render(
        **kwargs)


def build(reference=DEFAULT_REFERENCE, verbose=False) -> str | None:
    """Build the checker library; returns its path, or None when neither
    the reference checkout nor a prebuilt library exists."""
    cuda_dir = os.path.join(reference, "kernelkit", "cuda")
    if not os.path.isdir(cuda_dir):
        return OUT_LIB if os.path.exists(OUT_LIB) else None
    os.makedirs(OUT_DIR, exist_ok=True)
    nvcc = _nvcc()
    tmp = tempfile.mkdtemp(prefix="kkref_")
    try:
        fp_src = os.path.join(tmp, "cone_fp_rendered.cu")
        bp_src = os.path.join(tmp, "cone_bp_rendered.cu")
        with open(fp_src, "w") as f:
            f.write(render(os.path.join(cuda_dir, "cone_fp.cu"), FP_KWARGS))
        with open(bp_src, "w") as f:
            f.write(render(os.path.join(cuda_dir, "cone_bp.cu"), BP_KWARGS))
        objs = []
        for shim, inc in (("ref_shim_fp.cu", fp_src), ("ref_shim_bp.cu", bp_src),
                          ("tex_probe.cu", None)):
            obj = os.path.join(tmp, shim.replace(".cu", ".o"))
            cmd = [nvcc, *NVCC_FLAGS, "-c"]
            if inc:
                cmd += ["-include", inc]
            cmd += [os.path.join(HERE, shim), "-o", obj]
            if verbose:
                print(" ".join(cmd))
            subprocess.run(cmd, check=True)
            objs.append(obj)
        tmp_lib = os.path.join(tmp, "libkkref.so")
        subprocess.run([nvcc, "-shared", *NVCC_FLAGS[:2], *objs, "-o", tmp_lib,
                        "-lcudart"], check=True)
        shutil.move(tmp_lib, OUT_LIB)
    finally:
        shutil.rmtree(tmp, ignore_errors=True)
    return OUT_LIB


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--reference", default=DEFAULT_REFERENCE)
    ap.add_argument("-v", "--verbose", action="store_true")
    args = ap.parse_args(argv)
    out = build(args.reference, verbose=args.verbose)
    print(out if out else "reference checkout absent; nothing built")
    return 0


if __name__ == "__main__":
    sys.exit(main())
