"""CPU oracle for the cone-beam projection path (test infrastructure only).

This package restates, in FP64 NumPy, the arithmetic of ASTRA KernelKit's
cone-beam kernels and host-side processing so that the CUDA kernels of this
repository can be checked against it. It is a checker, never a fallback:
only the test suite, ``__graft_entry__.smoke()`` and the CPU-baseline /
reference legs of ``bench.py`` may import it.

Pinning: the oracle is checked against golden vectors produced by the
reference's own code (``tests/golden/``): kernel parameters and processing
outputs from the reference's Python, and forward/back-projections from the
reference's CUDA kernels compiled from their sources (``oracle/build_ref.py``)
and run on a B200.
"""
