"""Grids for states and actions.

Same names and constructor arguments as the reference's grids
(``src/_lcm/grids/continuous.py:111-325``, ``src/_lcm/grids/discrete.py:11-70``,
``src/_lcm/grids/categorical.py:17``).  Grid points are materialised on the
host in float64 once; the device kernels read these tables and compute
interpolation coordinates with the same formulas as
``src/_lcm/grids/coordinates.py:30-167``.
"""

from __future__ import annotations

import dataclasses
from typing import Any

import numpy as np

from pylcm_b200.exceptions import GridInitializationError


def categorical(*, ordered: bool):
    """Class decorator giving each annotated field a consecutive int code.

    Mirrors ``src/_lcm/grids/categorical.py:17-80``: ``LaborSupply.work == 0``,
    ``LaborSupply.retire == 1``.
    """

    def decorator(cls):
        names = list(getattr(cls, "__annotations__", {}))
        if not names:
            raise GridInitializationError(f"categorical class {cls.__name__} has no fields")
        for code, name in enumerate(names):
            setattr(cls, name, code)
        cls._ordered = ordered
        cls._lcm_categories = tuple(names)
        return cls

    return decorator


def _field_names_and_values(category_class: type) -> dict[str, int]:
    if hasattr(category_class, "_lcm_categories"):
        return {n: int(getattr(category_class, n)) for n in category_class._lcm_categories}
    if dataclasses.is_dataclass(category_class):
        return {f.name: int(getattr(category_class, f.name)) for f in dataclasses.fields(category_class)}
    names = list(getattr(category_class, "__annotations__", {}))
    return {n: int(getattr(category_class, n)) for n in names}


class Grid:
    """Base class of all grids."""

    batch_size: int = 0
    distributed: bool = False

    def to_numpy(self) -> np.ndarray:  # pragma: no cover - abstract
        raise NotImplementedError

    def __len__(self) -> int:
        return int(self.to_numpy().shape[0])


class DiscreteGrid(Grid):
    """Outcome space of a categorical variable (codes 0..n-1)."""

    def __init__(self, category_class: type, batch_size: int = 0, *, distributed: bool = False) -> None:
        nv = _field_names_and_values(category_class)
        codes = tuple(nv.values())
        if sorted(codes) != list(range(len(codes))):
            raise GridInitializationError(
                "category codes must be consecutive integers starting at 0, got " f"{codes}"
            )
        self.category_class = category_class
        self.categories = tuple(nv)
        self.codes = codes
        self.ordered = bool(getattr(category_class, "_ordered", False))
        self.batch_size = batch_size
        self.distributed = distributed

    def to_numpy(self) -> np.ndarray:
        return np.asarray(self.codes, dtype=np.int32)

    def __len__(self) -> int:
        return len(self.codes)

    def __repr__(self) -> str:
        return f"DiscreteGrid({self.category_class.__name__})"


class ContinuousGrid(Grid):
    """Base class of continuous grids."""

    kind: str = ""

    def coordinate_spec(self) -> tuple:
        """(kind, a, b, n) describing how a value maps to a fractional index."""
        raise NotImplementedError


@dataclasses.dataclass(frozen=True)
class LinSpacedGrid(ContinuousGrid):
    """Linearly spaced grid, endpoints included (``continuous.py:111``)."""

    start: float
    stop: float
    n_points: int
    batch_size: int = 0
    distributed: bool = False
    kind = "lin"

    def __post_init__(self) -> None:
        if self.n_points < 1:
            raise GridInitializationError("n_points must be >= 1")
        if not self.start < self.stop and self.n_points > 1:
            raise GridInitializationError("start must be smaller than stop")

    def to_numpy(self) -> np.ndarray:
        return np.linspace(float(self.start), float(self.stop), int(self.n_points))

    def __len__(self) -> int:
        return int(self.n_points)

    def coordinate_spec(self) -> tuple:
        n_steps = self.n_points - 1
        step = (float(self.stop) - float(self.start)) / (n_steps if n_steps > 0 else 1)
        return ("lin", float(self.start), step, int(self.n_points))


UniformContinuousGrid = LinSpacedGrid


@dataclasses.dataclass(frozen=True)
class LogSpacedGrid(ContinuousGrid):
    """Logarithmically spaced grid with exact endpoints (``coordinates.py:47-71``)."""

    start: float
    stop: float
    n_points: int
    batch_size: int = 0
    distributed: bool = False
    kind = "log"

    def __post_init__(self) -> None:
        if self.start <= 0:
            raise GridInitializationError("LogSpacedGrid needs start > 0")

    def to_numpy(self) -> np.ndarray:
        a, b = np.log(float(self.start)), np.log(float(self.stop))
        g = np.logspace(a, b, int(self.n_points), base=np.e)
        g[0] = float(self.start)
        g[-1] = float(self.stop)
        return g

    def __len__(self) -> int:
        return int(self.n_points)

    def coordinate_spec(self) -> tuple:
        a, b = np.log(float(self.start)), np.log(float(self.stop))
        return ("log", float(a), float((b - a) / (self.n_points - 1)), int(self.n_points))


@dataclasses.dataclass(frozen=True)
class IrregSpacedGrid(ContinuousGrid):
    """Grid given by explicit ascending points (``coordinates.py:117-167``)."""

    points: Any
    batch_size: int = 0
    distributed: bool = False
    kind = "irreg"

    def __post_init__(self) -> None:
        pts = np.asarray(self.points, dtype=np.float64)
        if pts.ndim != 1 or pts.size < 1:
            raise GridInitializationError("points must be a non-empty 1-D sequence")
        if np.any(np.diff(pts) <= 0):
            raise GridInitializationError("points must be strictly increasing")
        object.__setattr__(self, "points", tuple(float(p) for p in pts))

    def to_numpy(self) -> np.ndarray:
        return np.asarray(self.points, dtype=np.float64)

    def __len__(self) -> int:
        return len(self.points)

    @property
    def n_points(self) -> int:
        return len(self.points)

    def coordinate_spec(self) -> tuple:
        return ("irreg", 0.0, 0.0, len(self.points))


@dataclasses.dataclass(frozen=True)
class PiecewiseGridSegment:
    """One segment of a piecewise grid: an interval written as a string such
    as ``"[1, 4)"`` (square bracket: the bound is a grid point; round
    bracket: the grid stops one representable number inside it) and its
    number of points (``piecewise.py:24-50``)."""

    interval: str
    n_points: int

    def bounds(self) -> tuple[float, float, bool, bool]:
        """(lower, upper, lower closed, upper closed)."""
        txt = str(self.interval).strip()
        if len(txt) < 5 or txt[0] not in "[(" or txt[-1] not in "])" or "," not in txt:
            raise GridInitializationError(f"segment interval {self.interval!r} is not of the form '[a, b)'")
        lo_s, hi_s = txt[1:-1].split(",", 1)
        try:
            lo, hi = float(lo_s), float(hi_s)
        except ValueError as exc:
            raise GridInitializationError(f"segment interval {self.interval!r}: bounds must be numbers") from exc
        return lo, hi, txt[0] == "[", txt[-1] == "]"

    def effective_bounds(self) -> tuple[float, float]:
        """Grid start and stop: an open bound moved one representable number
        inward (``piecewise.py:197-217``)."""
        lo, hi, lc, hc = self.bounds()
        return (lo if lc else float(np.nextafter(lo, np.inf)), hi if hc else float(np.nextafter(hi, -np.inf)))


class _PiecewiseGrid(ContinuousGrid):
    """Segments of equally (or log-) spaced points laid end to end
    (``piecewise.py:53-188``).  A value's coordinate is the offset of its
    segment -- the last segment whose effective start is at or below it -- plus
    its coordinate inside that segment, so values between or beyond segments
    extrapolate with the spacing of the segment they fall in."""

    kind = "piece"
    log = False

    def _validate(self) -> None:
        segs = self.segments
        if not isinstance(segs, tuple) or len(segs) < 1:
            raise GridInitializationError("segments must be a non-empty tuple of PiecewiseGridSegment")
        for seg in segs:
            if not isinstance(seg, PiecewiseGridSegment):
                raise GridInitializationError("segments must be PiecewiseGridSegment objects")
            if int(seg.n_points) < 2:
                raise GridInitializationError(f"segment {seg.interval!r} needs at least 2 points")
            lo, hi, _, _ = seg.bounds()
            if not lo < hi:
                raise GridInitializationError(f"segment {seg.interval!r}: lower bound must be below upper bound")
            if self.log and lo <= 0:
                raise GridInitializationError(f"segment {seg.interval!r}: log-spaced bounds must be positive")
        for a, b in zip(segs[:-1], segs[1:]):
            _, ahi, _, ahc = a.bounds()
            blo, _, blc, _ = b.bounds()
            if ahi != blo:
                raise GridInitializationError(
                    f"segments {a.interval!r} and {b.interval!r} are not adjacent (a gap or an overlap)"
                )
            if ahc == blc:
                raise GridInitializationError(
                    f"segments {a.interval!r} and {b.interval!r} must share their bound with exactly one side closed"
                )

    def _segment_points(self, start: float, stop: float, n: int) -> np.ndarray:
        if not self.log:
            return np.linspace(start, stop, n)
        g = np.logspace(np.log(start), np.log(stop), n, base=np.e)
        g[0], g[-1] = start, stop
        return g

    def to_numpy(self) -> np.ndarray:
        return np.concatenate([self._segment_points(*seg.effective_bounds(), int(seg.n_points))
                               for seg in self.segments])

    def __len__(self) -> int:
        return int(sum(int(seg.n_points) for seg in self.segments))

    @property
    def n_points(self) -> int:
        return len(self)

    def coordinate_table(self) -> np.ndarray:
        """[breakpoints (k-1) | segment start (k) | segment scale (k) |
        segment offset (k)]: start and scale are (start, (n-1)/(stop-start))
        for linear segments and (log start, log-step) for log segments."""
        bnds = [seg.effective_bounds() for seg in self.segments]
        ns = [int(seg.n_points) for seg in self.segments]
        starts, scales = [], []
        for (a, b), n in zip(bnds, ns):
            if self.log:
                la, lb = np.log(a), np.log(b)
                starts.append(la)
                scales.append((lb - la) / (n - 1))
            else:
                starts.append(a)
                scales.append(1.0 / ((b - a) / (n - 1)))
        offsets = np.concatenate([[0], np.cumsum(ns[:-1])]).astype(np.float64)
        bps = [a for a, _ in bnds[1:]]
        return np.concatenate([bps, starts, scales, offsets]).astype(np.float64)

    def coordinate_spec(self) -> tuple:
        return ("piece", float(self.log), float(len(self.segments)), len(self))


@dataclasses.dataclass(frozen=True)
class PiecewiseLinSpacedGrid(_PiecewiseGrid):
    """Piecewise linearly spaced grid (``piecewise.py:53-118``), e.g. a
    breakpoint at an eligibility threshold."""

    segments: tuple
    batch_size: int = 0
    distributed: bool = False

    def __post_init__(self) -> None:
        self._validate()


@dataclasses.dataclass(frozen=True)
class PiecewiseLogSpacedGrid(_PiecewiseGrid):
    """Piecewise logarithmically spaced grid (``piecewise.py:121-188``)."""

    segments: tuple
    batch_size: int = 0
    distributed: bool = False
    log = True

    def __post_init__(self) -> None:
        self._validate()


def grid_values(grid: Grid) -> np.ndarray:
    return np.asarray(grid.to_numpy())
