"""Scan (projection) geometry: detectors, single-angle geometries and their
structure-of-arrays sequence form.

Mirrors ``kernelkit/geom/proj.py`` of ASTRA KernelKit (same class names,
arguments and conventions). All geometry lives on the host as NumPy arrays;
only the per-angle kernel parameters derived from it travel to the GPU.

Bit-compatibility note: every float32 operation that feeds the kernel
parameters (``detector_extent_min``, ``shift_``, ``scale_``, ``rotate_``,
``ProjectionGeometrySequence.fromList``) is evaluated with the same NumPy
operations, dtypes and order as the reference (``geom/proj.py:152-164,
317-364,432-556``). The kernels sample with 1/256-quantised interpolation
weights, so a one-ulp change in a parameter would move some samples by a
whole weight step.
"""
from __future__ import annotations

import copy
import math
from dataclasses import dataclass
from enum import Enum
from typing import Sequence

import numpy as np

#: Euler convention of the reference (``geom/proj.py:9``): static frame,
#: rotations applied about x, then y, then z.
ANGLES_CONVENTION = "sxyz"


def angles2mat(r, p, y) -> np.ndarray:
    """Rotation matrix for extrinsic roll-pitch-yaw angles (radians).

    ``R = Rz(yaw) @ Ry(pitch) @ Rx(roll)``: the static-frame ``sxyz``
    convention the reference obtains from ``transforms3d.euler.euler2mat``
    (``geom/proj.py:12-29``; convention described in
    ``docs/user_guide/geometries.rst:55-59``). The closed form is the
    published Euler-angle expansion (Shoemake, Graphics Gems IV), grouped
    as in that publication's reference code so the float64 matrix — and
    hence the float32 geometry derived from it — comes out bit-identical.
    """
    si, sj, sk = math.sin(r), math.sin(p), math.sin(y)
    ci, cj, ck = math.cos(r), math.cos(p), math.cos(y)
    cc, cs = ci * ck, ci * sk
    sc, ss = si * ck, si * sk
    return np.array(
        [
            [cj * ck, sj * sc - cs, sj * cc + ss],
            [cj * sk, sj * ss + cc, sj * cs - sc],
            [-sj, cj * si, cj * ci],
        ],
        dtype=np.float64,
    )


@dataclass
class Detector:
    """Flat-panel detector: ``rows`` x ``cols`` pixels of the given size.

    Reference: ``geom/proj.py:32-74``.
    """

    __slots__ = "rows", "cols", "pixel_height", "pixel_width"

    rows: int
    cols: int
    pixel_height: float
    pixel_width: float

    @property
    def shape(self):
        return self.rows, self.cols

    @property
    def width(self):
        """Physical width (``pixel_width * cols``)."""
        return self.pixel_width * self.cols

    @property
    def height(self):
        """Physical height (``pixel_height * rows``)."""
        return self.pixel_height * self.rows

    @property
    def pixel_volume(self):
        return self.pixel_width * self.pixel_height


class Beam(Enum):
    """Beam type (``geom/proj.py:77-90``)."""

    CONE = "cone"
    PARALLEL = "parallel"

    @classmethod
    def from_string(cls, value: str):
        key = value.lower()
        for member in cls:
            if member.value == key:
                return member
        raise ValueError(f"Invalid beam type: '{key}'")


def process_beam_type(arg) -> Beam:
    if isinstance(arg, Beam):
        return arg
    if isinstance(arg, str):
        return Beam.from_string(arg)
    raise TypeError("Argument must be of type `str` or `Beam`.")


def _check_unit(name, value):
    if not np.allclose(np.linalg.norm(value), 1.0):
        raise ValueError(
            f"`{name}` must be a unit vector. Consider normalizing "
            f"`{name}` using `{name} /= np.linalg.norm({name})`."
        )
    if np.allclose(value, 0.0):
        raise ValueError(f"`{name}` must not be zero.")


class ProjectionGeometry:
    """One cone-beam projection: a point source and a flat detector.

    Positions are world (x, y, z) coordinates; the detector is centred on
    ``detector_position`` and spanned by unit vectors ``u`` (horizontal,
    column direction) and ``v`` (vertical, row direction).
    Reference: ``geom/proj.py:102-240``.
    """

    xp = np

    def __init__(
        self,
        source_position,
        detector_position,
        detector: Detector,
        u: Sequence = (0.0, 1.0, 0.0),
        v: Sequence = (0.0, 0.0, 1.0),
        beam: Beam | str = Beam.CONE,
        array_module=None,
    ):
        if array_module is not None and array_module is not np:
            raise NotImplementedError(
                "Geometries are host-side objects; only NumPy is supported.")
        self.source_position = np.array(source_position, dtype=np.float32)
        self.detector_position = np.array(detector_position, dtype=np.float32)
        self.detector = detector
        self.u = np.array(u, dtype=np.float32)
        self.v = np.array(v, dtype=np.float32)
        self.beam = process_beam_type(beam)

    @property
    def detector_extent_min(self):
        """Corner of the detector at pixel (row 0, col 0), outer edge."""
        return (self.detector_position
                - self.v * self.detector.height / 2
                - self.u * self.detector.width / 2)

    @property
    def u(self):
        return self._u

    @u.setter
    def u(self, value):
        _check_unit("u", value)
        self._u = value

    @property
    def v(self):
        return self._v

    @v.setter
    def v(self, value):
        _check_unit("v", value)
        self._v = value

    def __deepcopy__(self, memodict={}):
        return self.__class__(
            source_position=np.copy(self.source_position),
            detector_position=np.copy(self.detector_position),
            u=np.copy(self.u),
            v=np.copy(self.v),
            detector=Detector(rows=self.detector.rows,
                              cols=self.detector.cols,
                              pixel_height=self.detector.pixel_height,
                              pixel_width=self.detector.pixel_width),
            beam=self.beam,
        )

    def __str__(self):
        return (f"Source {self.source_position} "
                f"Detector {self.detector_position} "
                f"Horizontal vector: {self.u} "
                f"Vertical vector: {self.v} ")


@dataclass
class ProjectionGeometrySequence:
    """Structure-of-arrays form of a list of ``ProjectionGeometry``.

    Arrays have shape (N, 3) for vectors and (N,) for detector data.
    Reference: ``geom/proj.py:243-410``.
    """

    xp = np

    @dataclass
    class DetectorSequence:
        xp = np
        rows: np.ndarray
        cols: np.ndarray
        pixel_width: np.ndarray
        pixel_height: np.ndarray

        @property
        def height(self):
            out = np.empty_like(self.pixel_height)
            np.multiply(self.pixel_height, self.rows, out=out)
            return out

        @property
        def width(self):
            out = np.empty_like(self.pixel_width)
            np.multiply(self.pixel_width, self.cols, out=out)
            return out

        @property
        def pixel_volume(self):
            return self.pixel_width * self.pixel_height

    source_position: np.ndarray
    detector_position: np.ndarray
    u: np.ndarray
    v: np.ndarray
    detector: DetectorSequence
    beam: Beam

    def __len__(self):
        return len(self.source_position)

    @property
    def detector_extent_min(self):
        """Per-angle detector corner (pixel (0, 0) outer edge), (N, 3)."""
        return (self.detector_position
                - self.v * self.detector.height[..., np.newaxis] / 2
                - self.u * self.detector.width[..., np.newaxis] / 2)

    @classmethod
    def fromList(cls, geometries, xp=None):
        """Pack a list of geometries into float32/int32 arrays."""
        if xp is not None and xp is not np:
            raise NotImplementedError("Only NumPy geometry sequences.")
        if isinstance(geometries, ProjectionGeometrySequence):
            return copy.deepcopy(geometries)
        geometries = list(geometries)
        if len(geometries) == 0:
            raise ValueError("Empty list of projection geometries.")
        beam = geometries[0].beam
        if not all(g.beam == beam for g in geometries):
            raise ValueError("All geometries must share one beam type.")

        def pack(values, dtype):
            return np.ascontiguousarray(np.array(values, dtype=dtype))

        det = cls.DetectorSequence(
            rows=pack([g.detector.rows for g in geometries], np.int32),
            cols=pack([g.detector.cols for g in geometries], np.int32),
            pixel_width=pack([g.detector.pixel_width for g in geometries],
                             np.float32),
            pixel_height=pack([g.detector.pixel_height for g in geometries],
                              np.float32),
        )
        return cls(
            source_position=pack([g.source_position for g in geometries],
                                 np.float32),
            detector_position=pack([g.detector_position for g in geometries],
                                   np.float32),
            u=pack([g.u for g in geometries], np.float32),
            v=pack([g.v for g in geometries], np.float32),
            detector=det,
            beam=beam,
        )

    def take(self, indices):
        d = self.detector
        return ProjectionGeometrySequence(
            source_position=self.source_position[indices],
            detector_position=self.detector_position[indices],
            u=self.u[indices],
            v=self.v[indices],
            detector=self.DetectorSequence(
                rows=d.rows[indices], cols=d.cols[indices],
                pixel_width=d.pixel_width[indices],
                pixel_height=d.pixel_height[indices]),
            beam=self.beam,
        )

    def __getitem__(self, item):
        return self.take(item)

    def __deepcopy__(self, memodict={}):
        d = self.detector
        return self.__class__(
            source_position=np.copy(self.source_position),
            detector_position=np.copy(self.detector_position),
            u=np.copy(self.u),
            v=np.copy(self.v),
            beam=self.beam,
            detector=ProjectionGeometrySequence.DetectorSequence(
                rows=np.copy(d.rows), cols=np.copy(d.cols),
                pixel_width=np.copy(d.pixel_width),
                pixel_height=np.copy(d.pixel_height)),
        )


def shift(geom, vector):
    """Copy of ``geom`` translated by ``vector`` (``geom/proj.py:413-429``)."""
    geom = copy.deepcopy(geom)
    shift_(geom, vector)
    return geom


def shift_(geom, vector) -> None:
    """Translate source and detector in place (``geom/proj.py:432-442``)."""
    geom.source_position += vector
    geom.detector_position += vector


def scale(geom, factor):
    """Copy of a single geometry with all lengths divided by ``factor``
    (``geom/proj.py:445-477``)."""
    geom = copy.deepcopy(geom)
    horiz = (geom.u * geom.detector.pixel_width) / factor
    width = np.linalg.norm(horiz)
    geom.detector.pixel_width = width
    geom.u = horiz / width
    vert = (geom.v * geom.detector.pixel_height) / factor
    height = np.linalg.norm(vert)
    geom.detector.pixel_height = height
    geom.v = vert / height
    geom.source_position[:] = geom.source_position[:] / factor
    geom.detector_position[:] = geom.detector_position[:] / factor
    return geom


def scale_(geom, factor) -> None:
    """Divide all lengths of a geometry (sequence) by ``factor`` in place.

    ``factor`` may be a per-axis (3,) array (anisotropic voxels); pixel
    vectors are rescaled first and re-split into length and direction.
    Operation order follows ``geom/proj.py:480-504``.
    """
    pix = geom.u * geom.detector.pixel_width[..., np.newaxis]
    pix /= factor
    geom.detector.pixel_width = np.linalg.norm(pix, axis=-1)
    np.divide(pix, geom.detector.pixel_width[..., np.newaxis], out=geom.u)
    np.multiply(geom.v, geom.detector.pixel_height[..., np.newaxis], out=pix)
    pix /= factor
    geom.detector.pixel_height = np.linalg.norm(pix, axis=-1)
    np.divide(pix, geom.detector.pixel_height[..., np.newaxis], out=geom.v)
    np.divide(geom.source_position, factor, out=geom.source_position)
    np.divide(geom.detector_position, factor, out=geom.detector_position)


def rotate(geom, roll: float = 0.0, pitch: float = 0.0, yaw: float = 0.0):
    """Copy of ``geom`` rotated by ``R = angles2mat(roll, pitch, yaw)``,
    applied as ``R @ vector`` in float64 (``geom/proj.py:507-534``)."""
    out = copy.deepcopy(geom)
    R = angles2mat(roll, pitch, yaw)
    out.source_position = R @ geom.source_position
    out.detector_position = R @ geom.detector_position
    out.u = R @ geom.u
    out.v = R @ geom.v
    out.beam = geom.beam
    return out


def rotate_(geom, roll: float = 0.0, pitch: float = 0.0,
            yaw: float = 0.0) -> None:
    """In-place rotation applied as ``vector @ R`` with R cast to the
    geometry's dtype, i.e. by R transposed (``geom/proj.py:537-556``)."""
    R = np.asarray(angles2mat(roll, pitch, yaw),
                   dtype=geom.source_position.dtype)
    geom.source_position[...] = geom.source_position @ R
    geom.detector_position[...] = geom.detector_position @ R
    geom.u[...] = geom.u @ R
    geom.v[...] = geom.v @ R


__all__ = [
    "ANGLES_CONVENTION", "angles2mat", "Detector", "Beam", "process_beam_type",
    "ProjectionGeometry", "ProjectionGeometrySequence", "shift", "shift_",
    "scale", "scale_", "rotate", "rotate_",
]
