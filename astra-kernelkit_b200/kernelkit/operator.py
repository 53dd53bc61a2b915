"""Linear operators over a forward and a backprojector.

Mirrors ``kernelkit/operator.py`` of the reference (``BaseOperator``,
``ProjectorOperator`` with its cached ``.T``, ``XrayTransform``).
Outputs allocated by the operators are float32 torch CUDA tensors.
"""
from __future__ import annotations

from abc import ABC, abstractmethod
from typing import Any

from . import _arrays
from .projector import BackProjector, BaseProjector, ForwardProjector


class BaseOperator(ABC):
    """A mathematical operator (``operator.py:10-33``)."""

    @property
    @abstractmethod
    def domain_shape(self) -> tuple:
        raise NotImplementedError

    @property
    @abstractmethod
    def range_shape(self) -> tuple:
        raise NotImplementedError

    @abstractmethod
    def __call__(self, input, out=None):
        raise NotImplementedError

    @property
    def T(self):
        raise NotImplementedError


def _zeros(shape):
    t = _arrays.torch()
    return t.zeros(shape, dtype=t.float32, device="cuda")


class ProjectorOperator(BaseOperator):
    """``A : X -> Y`` from a forward projector, with ``A.T`` from the
    backprojector (``operator.py:36-146``). The pair is not checked to be
    matched; the reference's backprojector is a scaled, unmatched adjoint
    (use ``kernelkit.torch_support`` for an exact one)."""

    def __init__(self, projector: BaseProjector, backprojector: BaseProjector):
        self.projector = projector
        self.backprojector = backprojector

    @property
    def domain_shape(self) -> tuple:
        vg = self.projector.volume_geometry
        return tuple(int(vg.shape[i]) for i in self.projector.volume_axes)

    @property
    def range_shape(self) -> tuple:
        pg = self.projector.projection_geometry
        n = len(pg)
        det = pg[0].detector if not hasattr(pg, "source_position") else None
        if det is not None:
            rows, cols = det.rows, det.cols
        else:
            rows, cols = int(pg.detector.rows[0]), int(pg.detector.cols[0])
        return tuple((n, rows, cols)[i] for i in self.projector.projection_axes)

    def __call__(self, input, out=None, additive=False):
        """``out = A input`` (``out += A input`` if ``additive``)."""
        if tuple(input.shape) != self.domain_shape:
            raise ValueError(
                f"Input shape {tuple(input.shape)} does not match domain "
                f"shape {self.domain_shape} of operator.")
        if out is None:
            out = _zeros(self.range_shape)
        self.projector.volume = input
        self.projector.projections = out
        self.projector(additive=additive)
        return out

    @property
    def T(self):
        if not hasattr(self, "_T"):
            self._T = _Adjoint(self)
        return self._T


class _Adjoint(BaseOperator):
    """``A^* : Y -> X`` through the backprojector (``operator.py:106-146``)."""

    def __init__(self, op: ProjectorOperator):
        self._op = op
        self.projector = op.backprojector
        self.backprojector = op.projector

    @property
    def domain_shape(self) -> tuple:
        return self._op.range_shape

    @property
    def range_shape(self) -> tuple:
        return self._op.domain_shape

    def __call__(self, input, out=None, additive=False):
        if tuple(input.shape) != self.domain_shape:
            raise ValueError(
                f"Input shape {tuple(input.shape)} does not match domain "
                f"shape {self.domain_shape} of operator.")
        if out is None:
            out = _zeros(self.range_shape)
        self.projector.projections = input
        self.projector.volume = out
        self.projector(additive)
        return out

    @property
    def T(self):
        return self._op


class XrayTransform(ProjectorOperator):
    """The cone-beam X-ray transform on a volume/scan geometry pair
    (``operator.py:149-233``). ``fp_kwargs``/``bp_kwargs`` go to the kernel
    constructors (e.g. ``interpolation='exact'``)."""

    def __init__(self, projection_geometry: Any, volume_geometry: Any,
                 volume_axes: tuple = (0, 1, 2),
                 projection_axes: tuple = (0, 1, 2),
                 use_toolbox: bool = False, fp_kwargs=None, bp_kwargs=None):
        if use_toolbox:
            raise NotImplementedError(
                "ASTRA Toolbox projectors are not part of this package.")
        fp_kwargs = dict(fp_kwargs or {})
        bp_kwargs = dict(bp_kwargs or {})
        projector = ForwardProjector(volume_axes=volume_axes,
                                     projection_axes=projection_axes,
                                     **fp_kwargs)
        backprojector = BackProjector(volume_axes=volume_axes,
                                      projection_axes=projection_axes,
                                      **bp_kwargs)
        projector.volume_geometry = volume_geometry
        projector.projection_geometry = projection_geometry
        backprojector.volume_geometry = volume_geometry
        backprojector.projection_geometry = projection_geometry
        super().__init__(projector, backprojector)


class _ExactAdjoint(BaseOperator):
    """``A^T : Y -> X``, the exact transpose of the forward projector."""

    def __init__(self, op: "ExactXrayTransform"):
        self._op = op

    @property
    def domain_shape(self) -> tuple:
        return self._op.range_shape

    @property
    def range_shape(self) -> tuple:
        return self._op.domain_shape

    def __call__(self, input, out=None, additive=False):
        if tuple(input.shape) != self.domain_shape:
            raise ValueError(
                f"Input shape {tuple(input.shape)} does not match domain "
                f"shape {self.domain_shape} of operator.")
        if out is None:
            out = _zeros(self.range_shape)
        fp = self._op.projector
        fp.kernel.transpose(input, fp._proj_geom_seq, fp.volume_geometry,
                            out, additive=additive)
        return out

    @property
    def T(self):
        return self._op


class ExactXrayTransform(ProjectorOperator):
    """The cone-beam forward projection ``A`` with ``.T`` its exact
    transpose (``RayDrivenConeFP.transpose``) instead of the reference's
    scaled backprojector, so that ``<A x, y> = <x, A.T y>``: the operator
    to differentiate through. Same arguments as ``XrayTransform`` (there
    are no backprojector options)."""

    def __init__(self, projection_geometry: Any, volume_geometry: Any,
                 volume_axes: tuple = (0, 1, 2),
                 projection_axes: tuple = (0, 1, 2), fp_kwargs=None):
        projector = ForwardProjector(volume_axes=volume_axes,
                                     projection_axes=projection_axes,
                                     **dict(fp_kwargs or {}))
        projector.volume_geometry = volume_geometry
        projector.projection_geometry = projection_geometry
        super().__init__(projector, None)

    @property
    def T(self):
        if not hasattr(self, "_T"):
            self._T = _ExactAdjoint(self)
        return self._T


__all__ = ["BaseOperator", "ProjectorOperator", "XrayTransform",
           "ExactXrayTransform",
           "ForwardProjector", "BackProjector", "BaseProjector"]
