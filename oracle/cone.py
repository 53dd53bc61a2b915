"""FP64 NumPy restatement of KernelKit's cone-beam forward projector and
backprojector (test infrastructure only; see the package docstring).

Two arithmetic modes let the same code serve two purposes:

* ``coords="fp32"`` replays, operation by operation, the float32 coordinate
  arithmetic of the reference kernels (``cuda/cone_fp.cu:141-193``,
  ``cuda/cone_bp.cu:84-118``) including the fused multiply-adds the CUDA
  compiler forms from ``a + b * c``; ``interp="tex8"`` reproduces the
  interpolation weights of the hardware texture filter (coordinates on a
  1/256 grid, bilinear product weights on the same grid), as measured on
  the B200. Together they model the reference kernel sample
  for sample; only accumulation (FP64 here) differs.
* ``coords="fp64", interp="exact"`` is the ideal continuous model: FP64
  ray/voxel coordinates and exact linear interpolation weights.

Texture semantics follow CUDA's unnormalised linear filtering with border
addressing: texel ``i`` is centred at ``i + 0.5`` and texels outside the
array read as zero.
"""
from __future__ import annotations

import numpy as np

F32 = np.float32
F64 = np.float64

#: (dominant axis, first in-slice axis, second in-slice axis) for rays
#: stepping along world x, y, z (``cuda/cone_fp.cu:59-61``).
RAY_AXES = ((0, 1, 2), (1, 0, 2), (2, 1, 0))

INTERP_MODES = ("exact", "tex8")


def fma32(a, b, c):
    """float32 fused multiply-add, evaluated in float64 and rounded once
    (the float64 product of two float32 values is exact)."""
    return (np.asarray(a, F64) * np.asarray(b, F64)
            + np.asarray(c, F64)).astype(F32)


def tex_weights(x, interp: str):
    """Split texture coordinates into (left texel index, weight of the
    right texel) for 1D linear filtering.

    ``exact``: ``xb = x - 0.5``, ``i = floor(xb)``, ``w = xb - i``.
    ``tex8`` (= ``tex8-halfup``): the coordinate is rounded half-up onto a
    1/256 grid first, so ``w`` is a multiple of 1/256 and a weight that
    rounds up to 1 moves the index instead. This is the rule of the B200
    texture unit (tests/test_texture_model.py); ``tex8-floor`` and
    ``tex8-nearest`` are the alternatives that measurement rejected, kept
    for that test.
    """
    x = np.asarray(x, F64)
    bad = ~np.isfinite(x)
    x = np.where(bad, -1.0e6, np.clip(x, -1.0e6, 1.0e6))
    if interp == "exact":
        xb = x - 0.5
        i0 = np.floor(xb)
        w = xb - i0
    else:
        s = x * 256.0
        if interp in ("tex8", "tex8-halfup"):
            q = np.floor(s + 0.5)
        elif interp == "tex8-floor":
            q = np.floor(s)
        elif interp == "tex8-nearest":
            q = np.rint(s)
        else:
            raise ValueError(f"unknown interpolation mode {interp!r}")
        q = q - 128.0
        i0 = np.floor(q / 256.0)
        w = (q - i0 * 256.0) / 256.0
    return i0.astype(np.int64), w


def bilinear_weights(wa, wb, interp: str, rule: int = 0, a_fast=True):
    """The four weights (w00, w01, w10, w11) of a bilinear footprint from
    the per-axis weights (index 0/1 = left/right texel along a, then b).

    ``exact``: plain products. ``tex8``: the texture unit's weights on the
    1/256 grid, measured on the B200 (tests/test_texture_model.py), with
    A, B the per-axis weights in units of 1/256:

    * ``rule=0`` -- 2D textures, and the plane of the two fastest axes of a
      3D texture: ``w11 = round_half_up(A B / 256)``, the others derived so
      the marginals stay A and B (weights sum to one);
    * ``rule=1`` -- fastest and slowest axis of a 3D texture: each slice of
      the slow axis (weights 256 - S, S) is split along the fast axis with
      ``round_half_up(F * slice / 256)`` for the right fast texel;
    * ``rule=2`` -- middle and slowest axis: the same split anchored on the
      left fast texel, ``round_half_up((256 - F) * slice / 256)``.

    ``a_fast`` says whether axis a is the faster one of the pair (rules 1
    and 2)."""
    if interp == "exact":
        return ((1 - wa) * (1 - wb), (1 - wa) * wb, wa * (1 - wb), wa * wb)
    A = np.round(np.asarray(wa) * 256.0)
    B = np.round(np.asarray(wb) * 256.0)
    if rule == 0:
        w11 = np.floor(A * B / 256.0 + 0.5)
        return ((256.0 - A - B + w11) / 256.0, (B - w11) / 256.0,
                (A - w11) / 256.0, w11 / 256.0)
    F, S = (A, B) if a_fast else (B, A)
    G = F if rule == 1 else 256.0 - F
    x1 = np.floor(G * S / 256.0 + 0.5)            # anchor side, slow 1
    x0 = np.floor(G * (256.0 - S) / 256.0 + 0.5)  # anchor side, slow 0
    y1, y0 = S - x1, (256.0 - S) - x0             # other side
    if rule == 1:   # anchor = fast 1
        f1s0, f1s1, f0s0, f0s1 = x0, x1, y0, y1
    else:           # anchor = fast 0
        f0s0, f0s1, f1s0, f1s1 = x0, x1, y0, y1
    if a_fast:      # (a, b) = (fast, slow)
        return f0s0 / 256, f0s1 / 256, f1s0 / 256, f1s1 / 256
    return f0s0 / 256, f1s0 / 256, f0s1 / 256, f1s1 / 256


def _gather2(plane, i0, j0):
    """Return the four texels around (i0, j0) of a 2D plane with border
    zeros; indices far outside are clamped onto the zero border."""
    n1, n2 = plane.shape
    padded = np.zeros((n1 + 4, n2 + 4), F64)
    padded[2:-2, 2:-2] = plane
    i = np.clip(i0, -2, n1) + 2
    j = np.clip(j0, -2, n2) + 2
    return (padded[i, j], padded[i, j + 1], padded[i + 1, j],
            padded[i + 1, j + 1])


def bilinear(plane, c1, c2, interp: str, rule: int = 0, a_fast=True):
    """Linear-filtered fetch of ``plane[axis0, axis1]`` at texture
    coordinates (c1 along axis 0, c2 along axis 1); ``rule``/``a_fast`` as
    in ``bilinear_weights``."""
    i0, a = tex_weights(c1, interp)
    j0, b = tex_weights(c2, interp)
    t00, t01, t10, t11 = _gather2(plane, i0, j0)
    w00, w01, w10, w11 = bilinear_weights(a, b, interp, rule, a_fast)
    return w00 * t00 + w01 * t01 + w10 * t10 + w11 * t11


def fp_weight_rule(axis, memory_order=(0, 1, 2)):
    """(rule, a_fast) of the forward projector's samples for rays along
    world ``axis`` in a 3D texture whose memory order (slowest to fastest)
    is ``memory_order``: the slice axis' memory rank picks the rule, and
    ``a_fast`` says whether the first in-slice axis (D1) is the faster."""
    rank = {ax: 2 - i for i, ax in enumerate(memory_order)}  # 0 = fastest
    A, D1, D2 = RAY_AXES[axis]
    rule = {2: 0, 1: 1, 0: 2}[rank[A]]
    return rule, rank[D1] < rank[D2]


def fp_ray_setup(p, axis, rows, cols, coords="fp32"):
    """Per-ray slopes/offsets of one angle (``cuda/cone_fp.cu:141-170``).

    ``p`` holds the 12 float32 kernel parameters of the angle: source,
    detector corner, ``u * pixel_width`` and ``v * pixel_height`` (all in
    the normalised unit-voxel frame, ``kernels/cone_fp.py:302-339``).
    Returns (a1, a2, b1, b2) arrays of shape (rows, cols).
    """
    A, D1, D2 = RAY_AXES[axis]
    s, c, u, v = p[0:3], p[3:6], p[6:9], p[9:12]
    r = np.arange(rows)[:, None]
    k = np.arange(cols)[None, :]
    if coords == "fp32":
        s, c, u, v = (np.asarray(t, F32) for t in (s, c, u, v))
        half = F32(0.5)
        ds = (c + half * u) + half * v          # pixel (0, 0) centre
        det = [fma32(r.astype(F32), v[i], fma32(k.astype(F32), u[i], ds[i]))
               for i in range(3)]
        sdd = s[A] - det[A]
        a1 = (s[D1] - det[D1]) / sdd
        a2 = (s[D2] - det[D2]) / sdd
        b1 = fma32(-a1, s[A], s[D1])
        b2 = fma32(-a2, s[A], s[D2])
    else:
        s, c, u, v = (np.asarray(t, F64) for t in (s, c, u, v))
        ds = c + 0.5 * u + 0.5 * v
        det = [ds[i] + k * u[i] + r * v[i] for i in range(3)]
        sdd = s[A] - det[A]
        a1 = (s[D1] - det[D1]) / sdd
        a2 = (s[D2] - det[D2]) / sdd
        b1 = s[D1] - a1 * s[A]
        b2 = s[D2] - a2 * s[A]
    return a1, a2, b1, b2


def _slice_plane(volume, axis, index):
    """(D1, D2) plane of the world-ordered volume at ``index`` along the
    ray axis."""
    if axis == 0:
        return volume[index, :, :]
    if axis == 1:
        return volume[:, index, :]
    return volume[:, :, index].T


def cone_fp_angle(volume, p, axis, rows, cols, out_scale,
                  coords="fp32", interp="tex8", slab=16,
                  memory_order=(0, 1, 2)):
    """Ray-driven projection of one angle; returns (rows, cols) float64.

    Restates ``cuda/cone_fp.cu:141-204`` with the launch structure of
    ``kernels/cone_fp.py:206-262``: the ray is traced in slabs of ``slab``
    slices, each slab restarting its coordinates from the slab's first
    slice and stepping by ``a1``/``a2`` per slice; each slab's sum is
    multiplied by the distance correction ``sqrt(a1^2 s1 + a2^2 s2 + 1)``
    and ``outputScale`` and added to the pixel. Samples are taken at every
    slice centre, including samples outside the volume (they read zero).
    ``memory_order`` lists the world axes of the reference's volume array
    from slowest to fastest (its ``volume_axes``); it decides the texture
    weight rule (``fp_weight_rule``).
    """
    rule, a_fast = fp_weight_rule(axis, memory_order)
    A, D1, D2 = RAY_AXES[axis]
    n_s, n_1, n_2 = (volume.shape[A], volume.shape[D1], volume.shape[D2])
    s1, s2, oscale = (float(t) for t in out_scale[axis])
    a1, a2, b1, b2 = fp_ray_setup(p, axis, rows, cols, coords)
    vol64 = np.asarray(volume, F64)
    if coords == "fp32":
        corr = np.sqrt(((a1 * a1) * F32(s1) + (a2 * a2) * F32(s2)) + F32(1)
                       ).astype(F64)
    else:
        corr = np.sqrt(a1 * a1 * s1 + a2 * a2 * s2 + 1.0)
    out = np.zeros((rows, cols), F64)
    for off in range(0, n_s, slab):
        t1 = off - 0.5 * n_s + 0.5
        if coords == "fp32":
            y = fma32(a1, F32(t1), b1) + F32(0.5 * n_1)
            z = fma32(a2, F32(t1), b2) + F32(0.5 * n_2)
        else:
            y = a1 * t1 + b1 + 0.5 * n_1
            z = a2 * t1 + b2 + 0.5 * n_2
        val = np.zeros((rows, cols), F64)
        for sl in range(off, min(off + slab, n_s)):
            val += bilinear(_slice_plane(vol64, axis, sl), y, z, interp,
                            rule, a_fast)
            if coords == "fp32":
                y = (y + a1).astype(F32)
                z = (z + a2).astype(F32)
            else:
                y = a1 * (sl + 1 - 0.5 * n_s + 0.5) + b1 + 0.5 * n_1
                z = a2 * (sl + 1 - 0.5 * n_s + 0.5) + b2 + 0.5 * n_2
        out += val * corr * oscale
    return out


def cone_fp(volume, params, axes, rows, cols, out_scale, **kw):
    """Forward projection of a world-ordered ``volume[x, y, z]`` for all
    angles: ``params`` (n, 12) float32, ``axes`` (n,) dominant ray axes,
    ``out_scale`` (3, 3). Returns (n, rows, cols) float64."""
    params = np.asarray(params, F32).reshape(-1, 12)
    out = np.empty((len(params), rows, cols), F64)
    for j in range(len(params)):
        out[j] = cone_fp_angle(volume, params[j], int(axes[j]), rows, cols,
                               out_scale, **kw)
    return out


def cone_bp(projections, params, vol_shape, out_scale, coords="fp32",
            interp="tex8", group=6, step_axis=0, angles=None):
    """Voxel-driven backprojection (``cuda/cone_bp.cu:76-158``).

    ``projections`` (n, rows, cols); ``params`` (n, 12) float32 laid out as
    [numU.xyzw, numV.xyzw, den.xyzw] per angle (``kernels/cone_bp.py:
    391-421``); ``vol_shape`` world (nx, ny, nz); ``out_scale`` the voxel
    volume. Voxel centres are ``c - N/2 + 1/2``. Along ``step_axis`` voxels
    are handled in groups of ``group``: the affine numerators/denominator
    are evaluated at the group's first voxel and stepped by one voxel per
    member, as the reference thread does. For every angle
    ``r = 1/den``, ``U = numU r``, ``V = numV r`` and the voxel gains
    ``r^2 * proj(V, U)``. Returns the world-ordered volume (float64).
    """
    params = np.asarray(params, F32).reshape(-1, 12)
    nx, ny, nz = (int(t) for t in vol_shape)
    shape = (nx, ny, nz)
    grids = []
    for ax in range(3):
        idx = np.arange(shape[ax])
        if ax == step_axis:
            idx = (idx // group) * group
        grids.append(idx)
    steps = np.zeros(shape, np.int64)
    step_idx = np.arange(shape[step_axis]) % group
    bshape = [1, 1, 1]
    bshape[step_axis] = -1
    steps += step_idx.reshape(bshape)
    coords_w = []
    for ax in range(3):
        g = grids[ax] - 0.5 * shape[ax] + 0.5
        bs = [1, 1, 1]
        bs[ax] = -1
        coords_w.append(np.broadcast_to(g.reshape(bs), shape))
    acc = np.zeros(shape, F64)
    sel = range(len(params)) if angles is None else angles
    for j in sel:
        nu, nv, de = params[j, 0:4], params[j, 4:8], params[j, 8:12]
        if coords == "fp32":
            X, Y, Z = (np.asarray(t, F32) for t in coords_w)

            def affine(q):
                return fma32(Z, q[2], fma32(Y, q[1], fma32(X, q[0], q[3])))

            num_u, num_v, den = affine(nu), affine(nv), affine(de)
            # sequential single-voxel steps inside each group
            for k in range(1, group):
                m = steps >= k
                num_u = np.where(m, (num_u + nu[step_axis]).astype(F32),
                                 num_u)
                num_v = np.where(m, (num_v + nv[step_axis]).astype(F32),
                                 num_v)
                den = np.where(m, (den + de[step_axis]).astype(F32), den)
            r = (F32(1.0) / den).astype(F32)
            U = (num_u * r).astype(F32)
            V = (num_v * r).astype(F32)
            r = r.astype(F64)
        else:
            X, Y, Z = (np.asarray(t, F64) for t in coords_w)
            off = steps.astype(F64)
            Xs = [X, Y, Z]
            Xs[step_axis] = Xs[step_axis] + off
            X, Y, Z = Xs
            nu64, nv64, de64 = (np.asarray(q, F64) for q in (nu, nv, de))
            num_u = nu64[3] + X * nu64[0] + Y * nu64[1] + Z * nu64[2]
            num_v = nv64[3] + X * nv64[0] + Y * nv64[1] + Z * nv64[2]
            den = de64[3] + X * de64[0] + Y * de64[1] + Z * de64[2]
            r = 1.0 / den
            U = num_u * r
            V = num_v * r
        val = bilinear(np.asarray(projections[j], F64), V, U, interp)
        acc += r * r * val
    return acc * float(out_scale)
