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


def grid_values(grid: Grid) -> np.ndarray:
    return np.asarray(grid.to_numpy())
