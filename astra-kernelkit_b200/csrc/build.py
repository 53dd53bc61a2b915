"""Build ``libkk.so`` (the C ABI of include/kk.h) for sm_100a with nvcc.

The library is written next to the Python package
(``astra-kernelkit_b200/kernelkit/_native/libkk.so``) so it ships with the
source tree; nothing is installed into site-packages.

Usage: ``python astra-kernelkit_b200/csrc/build.py [-v]``
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(os.path.dirname(HERE), "kernelkit")
INCLUDE = os.path.join(os.path.dirname(os.path.dirname(HERE)), "include")
OUT = os.path.join(PKG, "_native", "libkk.so")
SOURCES = ["kk_capi.cu", "kk_fp.cu", "kk_fpt.cu", "kk_bp.cu", "kk_fdk.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ARCH + ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC",
                "-Xcompiler", "-fvisibility=hidden", f"-I{INCLUDE}", f"-I{HERE}"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc",
                 shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def stale() -> bool:
    if not os.path.exists(OUT):
        return True
    t = os.path.getmtime(OUT)
    deps = [os.path.join(HERE, f) for f in os.listdir(HERE)
            if f.endswith((".cu", ".cuh"))]
    deps.append(os.path.join(INCLUDE, "kk.h"))
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose: bool = False, force: bool = False, extra=(),
          out: str = OUT) -> str:
    if not force and not stale():
        return out
    os.makedirs(os.path.dirname(out), exist_ok=True)
    tmp = tempfile.mkdtemp(prefix="kk_build_")
    try:
        objs, procs = [], []
        for src in SOURCES:  # translation units compile in parallel
            obj = os.path.join(tmp, src.replace(".cu", ".o"))
            cmd = [nvcc(), *FLAGS, *extra, "-c", os.path.join(HERE, src),
                   "-o", obj]
            if verbose:
                print(" ".join(cmd), flush=True)
            procs.append((cmd, subprocess.Popen(cmd)))
            objs.append(obj)
        for cmd, p in procs:
            if p.wait() != 0:
                raise subprocess.CalledProcessError(p.returncode, cmd)
        lib = os.path.join(tmp, "libkk.so")
        subprocess.run([nvcc(), *ARCH, "-shared", *objs, "-o", lib,
                        "-lcudart"], check=True)
        shutil.move(lib, out)
    finally:
        shutil.rmtree(tmp, ignore_errors=True)
    return out


if __name__ == "__main__":
    v = "-v" in sys.argv
    extra = ["-Xptxas", "-v"] if "--ptxas" in sys.argv else []
    print(build(verbose=v, force=True, extra=extra))
